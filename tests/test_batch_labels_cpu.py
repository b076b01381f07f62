"""Batch labels in the planner (host-only plans, no GPU): rejected with the
reference's message unless QS_PLAN_BATCH_LABELS is set; with it, labels in
A, B and C become batch labels, the M/N/K composites exclude them, and their
extents and bounds are checked."""
import numpy as np
import pytest
import torch


def view(qs, shape, parent_len=None, offset=0):
    n = int(np.prod(shape)) if len(shape) else 1
    st, acc = [], 1
    for s in shape:
        st.append(acc)
        acc *= s
    return qs.StridedView(torch.zeros(parent_len or max(n, 1), dtype=torch.float64), tuple(shape),
                          tuple(st), offset)


def test_batch_labels_rejected_by_default_and_planned_with_the_flag(qs):
    A, B, C = view(qs, (4, 5, 3)), view(qs, (5, 6, 3)), view(qs, (4, 6, 3))
    with pytest.raises(qs.ArgumentError, match="appears in indA, indB, and indC"):
        qs.plan_contract(C, A, (1, 2, 9), B, (2, 3, 9), (1, 3, 9), host_only=True)
    p = qs.plan_contract(C, A, (1, 2, 9), B, (2, 3, 9), (1, 3, 9), host_only=True, batch_labels=True)
    assert p.batch_labels == (9,) and p.batch_length == 3
    assert set(p.m_labels + p.n_labels) == {1, 3} and p.k_labels == (2,)
    assert p.path == "NestPath"
    # two batch labels, one of them first in every operand
    A2, B2, C2 = view(qs, (2, 4, 5, 3)), view(qs, (2, 5, 6, 3)), view(qs, (3, 6, 4, 2))
    p2 = qs.plan_contract(C2, A2, (8, 1, 2, 9), B2, (8, 2, 3, 9), (9, 3, 1, 8), host_only=True,
                          batch_labels=True)
    assert sorted(p2.batch_labels) == [8, 9] and p2.batch_length == 6
    # a zero-length batch label: nothing to do
    Z = qs.plan_contract(view(qs, (4, 6, 0)), view(qs, (4, 5, 0)), (1, 2, 9), view(qs, (5, 6, 0)),
                         (2, 3, 9), (1, 3, 9), host_only=True, batch_labels=True)
    assert Z.path == "EmptyPath"


def test_batch_label_extent_and_bounds_errors(qs):
    with pytest.raises(qs.DimensionMismatch):
        qs.plan_contract(view(qs, (4, 6, 3)), view(qs, (4, 5, 3)), (1, 2, 9), view(qs, (5, 6, 2)), (2, 3, 9),
                         (1, 3, 9), host_only=True, batch_labels=True)
    with pytest.raises(qs.DimensionMismatch):
        qs.plan_contract(view(qs, (4, 6, 2)), view(qs, (4, 5, 3)), (1, 2, 9), view(qs, (5, 6, 3)), (2, 3, 9),
                         (1, 3, 9), host_only=True, batch_labels=True)
    # C's parent too short for its last batch entry
    p = qs.plan_contract(view(qs, (4, 6, 3), parent_len=4 * 6 * 3 - 1), view(qs, (4, 5, 3)), (1, 2, 9),
                         view(qs, (5, 6, 3)), (2, 3, 9), (1, 3, 9), host_only=True, batch_labels=True)
    assert not p.bounds_ok


def test_batch_bounds_with_negative_stride_and_swap(qs):
    # C's batch axis runs backwards from an offset: in bounds only when the
    # offset covers the negative span.
    par = torch.zeros(4 * 6 * 3, dtype=torch.float64)
    A, B = view(qs, (4, 5, 3)), view(qs, (5, 6, 3))
    ok = qs.StridedView(par, (4, 6, 3), (1, 4, -24), 48)
    p = qs.plan_contract(ok, A, (1, 2, 9), B, (2, 3, 9), (1, 3, 9), host_only=True, batch_labels=True)
    assert p.bounds_ok and p.batch_length == 3
    bad = qs.StridedView(par, (4, 6, 3), (1, 4, -24), 24)
    p = qs.plan_contract(bad, A, (1, 2, 9), B, (2, 3, 9), (1, 3, 9), host_only=True, batch_labels=True)
    assert not p.bounds_ok
    # C row-major in (i, j): the N side has C's unit stride, so A and B swap roles;
    # the batch label stays a batch label.
    Ct = qs.StridedView(torch.zeros(4 * 64 * 3, dtype=torch.float64), (4, 64, 3), (64, 1, 256))
    Bw = view(qs, (5, 64, 3))
    p = qs.plan_contract(Ct, A, (1, 2, 9), Bw, (2, 3, 9), (1, 3, 9), host_only=True, batch_labels=True)
    assert p.swapped and p.batch_labels == (9,) and p.bounds_ok
