"""Host side of tensoradd!/tensortrace! (no GPU): TO's index tuples are
validated and turned into labels before any device work, and CPU tensors
are refused (there is no CPU fallback)."""
import pytest
import torch


def test_index_tuples_validated_and_no_cpu_fallback(qs):
    A = qs.StridedView(torch.zeros(6 * 5, dtype=torch.float64), (6, 5), (1, 6))
    C = qs.StridedView(torch.zeros(30, dtype=torch.float64), (5, 6), (1, 5))
    with pytest.raises(qs.ArgumentError, match="permutation"):
        qs.tensoradd(C, A, ((1, 1), ()), False, 1.0, 0.0)
    with pytest.raises(qs.ArgumentError, match="partition"):
        qs.tensortrace(C, A, ((1,), ()), ((2,), ()), False, 1.0, 0.0)
    with pytest.raises(qs.ArgumentError, match="CUDA device memory"):
        qs.tensoradd(C, A, ((2, 1), ()), False, 1.0, 0.0)
