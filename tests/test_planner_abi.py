"""Host logic through the C ABI, on CPU: the library loads and exports every
symbol include/qsgpu.h declares, and the planner (host-only plans, no device
work) reproduces the reference's planning rules and error behaviour.
"""
import ctypes
import json
import os
import re

import numpy as np
import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def header_symbols():
    with open(os.path.join(ROOT, "include", "qsgpu.h")) as f:
        src = f.read()
    return sorted(set(re.findall(r"\b(qs_[a-z_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(qs):
    lib = qs._abi.lib()
    syms = header_symbols()
    assert "qs_plan_contract" in syms and "qs_execute" in syms
    for s in syms:
        assert hasattr(lib, s), f"libqsgpu.so does not export {s}"
    assert set(syms) <= set(qs._abi.SIGNATURES), "ctypes binding misses a declared symbol"
    assert qs._abi.lib().qs_version().startswith(b"qsgpu")


def cpu_view(qs, shape, dtype=torch.float64, strides=None, offset=0, op="identity", parent=None):
    n = int(np.prod(shape)) if len(shape) else 1
    if parent is None:
        parent = torch.zeros(max(n, 1), dtype=dtype)
    if strides is None:
        strides, acc = [], 1
        for s in shape:
            strides.append(acc)
            acc *= s
    return qs.StridedView(parent, tuple(shape), tuple(strides), offset, op)


def host_plan(qs, C, A, indA, B, indB, indC, **kw):
    return qs.plan_contract(C, A, indA, B, indB, indC, host_only=True, **kw)


@pytest.mark.parametrize("case", load("classify_labels.json")["ok"])
def test_classify_labels_known_answers(qs, case):
    ext = {}
    for l in case["indA"] + case["indB"] + case["indC"]:
        ext.setdefault(l, 2 + (abs(l) % 3))
    A = cpu_view(qs, [ext[l] for l in case["indA"]])
    B = cpu_view(qs, [ext[l] for l in case["indB"]])
    C = cpu_view(qs, [ext[l] for l in case["indC"]])
    p = host_plan(qs, C, A, case["indA"], B, case["indB"], case["indC"])
    m, n, k = case["want"]
    got_m, got_n = (p.n_labels, p.m_labels) if p.swapped else (p.m_labels, p.n_labels)
    assert sorted(got_m) == sorted(m)
    assert sorted(got_n) == sorted(n)
    assert sorted(p.k_labels) == sorted(k)


@pytest.mark.parametrize("case", load("classify_labels.json")["bad"])
def test_classify_labels_rejections(qs, case):
    ext = {l: 3 for l in case["indA"] + case["indB"] + case["indC"]}
    A = cpu_view(qs, [ext[l] for l in case["indA"]])
    B = cpu_view(qs, [ext[l] for l in case["indB"]])
    C = cpu_view(qs, [ext[l] for l in case["indC"]])
    with pytest.raises(qs.ArgumentError):
        host_plan(qs, C, A, case["indA"], B, case["indB"], case["indC"])


@pytest.mark.parametrize("case", load("label_errors.json"))
def test_label_validation_errors(qs, case):
    A, B, C = cpu_view(qs, case["A"]), cpu_view(qs, case["B"]), cpu_view(qs, case["C"])
    err = {"ArgumentError": qs.ArgumentError, "DimensionMismatch": qs.DimensionMismatch}[case["error"]]
    with pytest.raises(err):
        host_plan(qs, C, A, case["indA"], B, case["indB"], case["indC"])


@pytest.mark.parametrize("case", load("order_free_labels.json"))
def test_order_free_labels_known_answers(qs, case):
    # M = case labels (A carries them plus one K label 99); N = empty, so no swap.
    C = cpu_view(qs, case["size"], strides=case["strides"],
                 parent=torch.zeros(10000, dtype=torch.float64), offset=5000)
    lab = case["labels"]
    ext = dict(zip(case["indC"], case["size"]))
    others = [l for l in case["indC"] if l not in lab]
    A = cpu_view(qs, [ext[l] for l in lab] + [3])
    B = cpu_view(qs, [3] + [ext[l] for l in others])
    p = host_plan(qs, C, A, lab + [99], B, [99] + others, case["indC"])
    got = p.n_labels if p.swapped else p.m_labels
    assert list(got) == case["want"]


def test_axis_group_offsets_via_plan(qs):
    # Worked A/B/C example: M = (3,2) with A strides (1,15), C strides (1,12).
    g = load("axis_group.json")
    assert g[0]["offsets"][0] == [0, 1, 2, 15, 16, 17]
    # The C++ fill_offsets is exercised end to end by the GPU parity tests;
    # here: the group lengths and labels a plan reports.
    A = cpu_view(qs, (3, 5, 2), strides=(1, 3, 15))
    B = cpu_view(qs, (5, 4), strides=(1, 5))
    C = cpu_view(qs, (3, 4, 2), strides=(1, 3, 12))
    p = host_plan(qs, C, A, (1, 2, 3), B, (2, 4), (1, 4, 3))
    assert (p.m_length, p.n_length, p.k_length) == (6, 4, 5)
    assert p.m_labels == (1, 3) and p.n_labels == (4,) and p.k_labels == (2,)
    assert p.path == "NestPath" and not p.swapped


def test_contraction_labels_worked_example(qs):
    for c in load("contraction_labels.json"):
        a, b, ci = qs.contraction_labels(c["pA"], c["pB"], c["pAB"])
        assert list(a) == c["indA"] and list(b) == c["indB"] and list(ci) == c["indC"]


def test_eltype_and_conjugated_output_rejections(qs):
    A = cpu_view(qs, (3, 4), dtype=torch.complex128)
    B = cpu_view(qs, (4, 5), dtype=torch.float64)
    C = cpu_view(qs, (3, 5), dtype=torch.float64)
    with pytest.raises(qs.ArgumentError, match="complex"):
        host_plan(qs, C, A, (1, 2), B, (2, 3), (1, 3))
    with pytest.raises(qs.ArgumentError):
        cpu_view(qs, (3, 4), dtype=torch.float16)._c([])
    Cc = cpu_view(qs, (3, 5), dtype=torch.complex128, op="conj")
    with pytest.raises(qs.ArgumentError, match="conjugated"):
        host_plan(qs, Cc, A, (1, 2), cpu_view(qs, (4, 5), dtype=torch.complex128), (2, 3), (1, 3))
    # a real "conjugated" output is fine (op is a no-op on real data)
    Cr = cpu_view(qs, (3, 5), dtype=torch.float64, op="adjoint")
    host_plan(qs, Cr, cpu_view(qs, (3, 4)), (1, 2), cpu_view(qs, (4, 5)), (2, 3), (1, 3))
    with pytest.raises(qs.ArgumentError):
        qs.QuasiStridedBackend(accumulator="Float16")


def test_alias_rejection(qs):
    M = torch.zeros(32, dtype=torch.float64)
    C = qs.StridedView(M, (4, 4), (1, 8), 0)
    A = qs.StridedView(M, (4, 4), (1, 8), 4)
    B = cpu_view(qs, (4, 4))
    with pytest.raises(qs.ArgumentError, match="share memory"):
        host_plan(qs, C, A, (1, 2), B, (2, 3), (1, 3))
    with pytest.raises(qs.ArgumentError, match="share memory"):
        host_plan(qs, C, B, (1, 2), A, (2, 3), (1, 3))


def test_conjugation_folding(qs):
    T = torch.complex128
    for (conjA, opA, opB), (ca, cb) in (((True, "conj", "identity"), (False, False)),
                                        ((False, "adjoint", "identity"), (True, False)),
                                        ((False, "identity", "transpose"), (False, False))):
        A = cpu_view(qs, (40, 9), dtype=T, op=opA)
        B = cpu_view(qs, (9, 37), dtype=T, op=opB)
        C = cpu_view(qs, (40, 37), dtype=T)
        p = host_plan(qs, C, A, (1, 2), B, (2, 3), (1, 3), conjA=conjA)
        assert not p.swapped
        assert (p.conjA, p.conjB) == (ca, cb)
    # real operands never conjugate
    p = host_plan(qs, cpu_view(qs, (5, 5)), cpu_view(qs, (5, 5), op="conj"), (1, 2),
                  cpu_view(qs, (5, 5)), (2, 3), (1, 3), conjA=True)
    assert (p.conjA, p.conjB) == (False, False)


def test_bounds_detected_before_execution(qs):
    M, K, N = 8, 6, 5
    for sa, sb, sc in ((M * K - 1, K * N, M * N), (M * K, K * N - 1, M * N), (M * K, K * N, M * N - 1)):
        A = qs.StridedView(torch.zeros(sa, dtype=torch.float64), (M, K), (1, M), 0)
        B = qs.StridedView(torch.zeros(sb, dtype=torch.float64), (K, N), (1, K), 0)
        C = qs.StridedView(torch.zeros(sc, dtype=torch.float64), (M, N), (1, M), 0)
        p = host_plan(qs, C, A, (1, 2), B, (2, 3), (1, 3))
        assert not p.bounds_ok
    A = qs.StridedView(torch.zeros(M * K, dtype=torch.float64), (M, K), (1, M), 0)
    B = qs.StridedView(torch.zeros(K * N, dtype=torch.float64), (K, N), (1, K), 0)
    C = qs.StridedView(torch.zeros(M * N, dtype=torch.float64), (M, N), (1, M), 0)
    assert host_plan(qs, C, A, (1, 2), B, (2, 3), (1, 3)).bounds_ok


def test_path_selection(qs):
    v = lambda *s: cpu_view(qs, s)  # noqa: E731
    assert host_plan(qs, v(3, 0), v(3, 4), (1, 2), v(4, 0), (2, 3), (1, 3)).path == "EmptyPath"
    assert host_plan(qs, v(0, 3), v(0, 4), (1, 2), v(4, 3), (2, 3), (1, 3)).path == "EmptyPath"
    assert host_plan(qs, v(5, 4), v(5, 0), (1, 2), v(0, 4), (2, 3), (1, 3)).path == "ScalePath"
    assert host_plan(qs, v(1, 40), v(1, 70), (1, 2), v(70, 40), (2, 3), (1, 3)).path == "DotPath"
    assert host_plan(qs, v(50, 4), v(50, 1), (1, 2), v(1, 4), (2, 3), (1, 3)).path == "OuterPath"
    assert host_plan(qs, v(50, 4), v(50, 1), (1, 2), v(1, 4), (2, 3), (1, 3),
                     path_modes=qs.PathModes(outer="never")).path == "NestPath"
    assert host_plan(qs, v(1, 40), v(1, 70), (1, 2), v(70, 40), (2, 3), (1, 3),
                     path_modes=qs.PathModes(dot="never")).path == "NestPath"
    # full contraction to a scalar: M = N = 1 -> dot
    assert host_plan(qs, v(), v(3, 40), (-1, -2), v(40, 3), (-2, -1), ()).path == "DotPath"
    # outer product of a matrix and a vector: no K label, K = 1
    assert host_plan(qs, v(5, 3, 40), v(3, 40), (1, 2), v(5,), (3,), (3, 1, 2)).path == "OuterPath"


def test_swap_rule_on_transposed_output(qs):
    # C stored [n, m]: M has no unit-stride run in C, N does -> B takes M.
    Ma, Ka, Na = 90, 4, 120
    A = cpu_view(qs, (Ma, Ka))
    B = cpu_view(qs, (Ka, Na))
    C = cpu_view(qs, (Ma, Na), strides=(Na, 1))
    p = host_plan(qs, C, A, (1, 2), B, (2, 3), (1, 3))
    assert p.swapped and p.m_labels == (3,) and p.n_labels == (1,)
    p = host_plan(qs, cpu_view(qs, (Ma, Na)), A, (1, 2), B, (2, 3), (1, 3))
    assert not p.swapped


def test_blocking_keywords_validated(qs):
    A, B, C = cpu_view(qs, (9, 10)), cpu_view(qs, (10, 8)), cpu_view(qs, (9, 8))
    for kw in ({"m_block": 0}, {"k_block": 0}, {"n_block": -3}):
        with pytest.raises(qs.ArgumentError):
            host_plan(qs, C, A, (1, 2), B, (2, 3), (1, 3), **kw)
    host_plan(qs, C, A, (1, 2), B, (2, 3), (1, 3), m_block=5, k_block=100, n_block=100)


def test_accumulator_compute_type(qs):
    f32 = lambda *s: cpu_view(qs, s, dtype=torch.float32)  # noqa: E731
    f64 = lambda *s: cpu_view(qs, s, dtype=torch.float64)  # noqa: E731
    c64 = lambda *s: cpu_view(qs, s, dtype=torch.complex128)  # noqa: E731
    assert host_plan(qs, f32(4, 4), f32(4, 4), (1, 2), f64(4, 4), (2, 3), (1, 3)).compute_type == "Float64"
    assert host_plan(qs, f32(4, 4), f32(4, 4), (1, 2), f32(4, 4), (2, 3), (1, 3),
                     accumulator="Float64").compute_type == "Float64"
    assert host_plan(qs, c64(4, 4), f64(4, 4), (1, 2), f64(4, 4), (2, 3), (1, 3),
                     accumulator="Float32").compute_type == "ComplexF32"


def test_host_only_plan_cannot_execute(qs):
    A, B, C = cpu_view(qs, (4, 4)), cpu_view(qs, (4, 4)), cpu_view(qs, (4, 4))
    p = host_plan(qs, C, A, (1, 2), B, (2, 3), (1, 3))
    with pytest.raises(qs.ArgumentError, match="host-only"):
        qs.execute(p, 1.0, 0.0)
    with pytest.raises(qs.ArgumentError):
        # CPU operands are refused for a device plan: there is no CPU fallback
        qs.plan_contract(C, A, (1, 2), B, (2, 3), (1, 3))


def test_wait_limit_validation_on_host(qs):
    # qs_plan_set_wait_limit: 0 restores the default, limits above 60 s are
    # not bounds (ArgumentError); a host-only plan accepts the setting.
    C = qs.StridedView(torch.zeros(6, dtype=torch.float64), (2, 3), (1, 2))
    A = qs.StridedView(torch.zeros(8, dtype=torch.float64), (2, 4), (1, 2))
    B = qs.StridedView(torch.zeros(12, dtype=torch.float64), (4, 3), (1, 4))
    plan = qs.plan_contract(C, A, (1, 2), B, (2, 3), (1, 3), host_only=True)
    qs.set_wait_limit(plan, 1_000_000, hold_loads=True)
    qs.set_wait_limit(plan, 0)
    with pytest.raises(qs.ArgumentError, match="60 s"):
        qs.set_wait_limit(plan, 61_000_000_000)
