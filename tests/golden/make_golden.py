"""Generate the golden fixtures in tests/golden/*.json.

Each fixture restates a known-answer test of QuasiStrided.jl's own test
suite; the expected values are computed here from the formulas those tests
state (exact integer arithmetic, or the closed form the test asserts), never
by this engine or by the oracle:

  worked_fixture.json     test/helpers.jl:47-61, test/execution/test_execute.jl:3-23
  one_rounding.json       test/execution/test_c_panel.jl:5-41
  conj_xor.json           test/execution/test_nest.jl:127-143
  classify_labels.json    test/planning/test_labels.jl:3-24
  order_free_labels.json  test/planning/test_labels.jl:26-50
  leading_unit_run.json   test/planning/test_labels.jl:52-75
  axis_group.json         test/layout/test_axis_group.jl:14-26
  contraction_labels.json src/integrations/tensoroperations.jl:34-38 (worked example)
  label_errors.json       test/planning/test_plan.jl:3-35, test/planning/test_labels.jl:19-23

Julia is not available where this runs, so the reference's tests cannot be
executed; these fixtures carry their stated answers.  Run:
``python tests/golden/make_golden.py`` (rewrites the JSON files).
"""
from __future__ import annotations

import itertools
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def colmajor_index(idx, shape):
    off, acc = 0, 1
    for i, n in zip(idx, shape):
        off += i * acc
        acc *= n
    return off


def worked_fixture():
    # A = reshape(1.0:30.0, 3, 5, 2), B = reshape(1.0:20.0, 5, 4);
    # Cref[a, n, b] = sum_k A[a, k, b] * B[k, n]   (exact in Float64)
    A = [float(i + 1) for i in range(30)]
    B = [float(i + 1) for i in range(20)]
    C = [0.0] * 24
    for a, n, b in itertools.product(range(3), range(4), range(2)):
        s = 0
        for k in range(5):
            s += A[colmajor_index((a, k, b), (3, 5, 2))] * B[colmajor_index((k, n), (5, 4))]
        C[colmajor_index((a, n, b), (3, 4, 2))] = s
    # Offset views: A4 = reshape(1.0:40.0, 4, 5, 2); Av = view(A4, 2:4, :, :);
    # expected [sum(A4[a,k,b]*B[k,n] for k) for a in 2:4, n in 1:4, b in 1:2].
    A4 = [float(i + 1) for i in range(40)]
    Coff = [0.0] * 24
    for a, n, b in itertools.product(range(3), range(4), range(2)):
        s = 0
        for k in range(5):
            s += A4[colmajor_index((a + 1, k, b), (4, 5, 2))] * B[colmajor_index((k, n), (5, 4))]
        Coff[colmajor_index((a, n, b), (3, 4, 2))] = s
    return {
        "A": A, "A_shape": [3, 5, 2], "B": B, "B_shape": [5, 4], "C_shape": [3, 4, 2],
        "indA": [1, 2, 3], "indB": [2, 4], "indC": [1, 4, 3], "Cref": C,
        "permuted": {"A_perm": [1, 2, 0], "indA": [2, 3, 1], "B_perm": [1, 0], "indB": [4, 2]},
        "offset": {"A4": A4, "A4_shape": [4, 5, 2], "A_offset": 1, "C_parent_shape": [4, 4, 2],
                   "C_offset": 1, "Cref": Coff},
    }


def one_rounding():
    # Along K, A[:, 1] = 1, A[:, K/2+1] = 2^-30, A[:, K] = -1, B = fill(b),
    # C = fill(beta == 0 ? NaN : 2^-28); every C element must equal
    # TC(2^-30 * b + beta * 2^-28) (computed in the compute type, rounded once).
    cases = [
        ("Float64", "Float64", "Float32", None, 13, 40, 20, "manual_n_block_16", 0.5),
        ("Float32", "Float32", "Float32", "Float64", 13, 9, 20, "packed_b", 1),
        ("Float64", "ComplexF64", "ComplexF32", None, 13, 9, 20, "strided_c", 0.5),
        ("Float32", "Float32", "Float32", "Float64", 7, 5, 3000, "backend", 0),
        ("Float64", "Float64", "Float32", None, 1, 9, 20, "strided_c", 1),
        ("Float64", "Float64", "Float32", None, 13, 9, 20, "strided_c", 0),
    ]
    out = []
    for TA, TB, TC, acc, M, N, K, case, beta in cases:
        b = [1.0, 1.0] if TB.startswith("Complex") else [1.0, 0.0]
        want = [2.0 ** -30 * b[0] + beta * 2.0 ** -28, 2.0 ** -30 * b[1]]
        out.append({"TA": TA, "TB": TB, "TC": TC, "accumulator": acc, "M": M, "N": N, "K": K,
                    "case": case, "beta": beta, "b": b, "expected_re_im_before_rounding": want})
    return out


def conj_xor():
    # (conjA, opA, opB) => (A conjugated, B conjugated)
    return [
        {"conjA": True, "opA": "conj", "opB": "identity", "ca": False, "cb": False},
        {"conjA": False, "opA": "adjoint", "opB": "identity", "ca": True, "cb": False},
        {"conjA": False, "opA": "identity", "opB": "transpose", "ca": False, "cb": False},
    ]


def classify_labels():
    ok = [
        ([1, 2], [2, 3], [1, 3], [[1], [3], [2]]),
        ([1, 2], [2, 3], [3, 1], [[1], [3], [2]]),
        ([1, 2, 3, 4], [3, 5, 6, 7], [4, 6, 7, 1, 2, 5], [[1, 2, 4], [5, 6, 7], [3]]),
        ([1, 2], [3, 1, 4, 5], [3, 2, 4, 5], [[2], [3, 4, 5], [1]]),
        ([1, 2, 3, 4], [3, 4, 5, 6], [1, 2, 5, 6], [[1, 2], [5, 6], [3, 4]]),
        ([1], [1, 2], [2], [[], [2], [1]]),
        ([1, 2], [3, 4], [1, 2, 3, 4], [[1, 2], [3, 4], []]),
    ]
    bad = [
        ([1, 1], [1, 2], [1, 2]),
        ([1, 2], [2, 3], [1, 2, 3]),
        ([1, 2], [3, 4], [1, 3]),
        ([1, 2], [3, 4], [1, 2, 3, 9]),
    ]
    return {"ok": [{"indA": a, "indB": b, "indC": c, "want": w} for a, b, c, w in ok],
            "bad": [{"indA": a, "indB": b, "indC": c} for a, b, c in bad]}


def order_free_labels():
    # _lo_view(size, strides) with labels (10,20,30,40) etc.
    return [
        {"size": [5, 3, 2, 4], "strides": [12, 1, 60, 3], "indC": [10, 20, 30, 40],
         "labels": [10, 20, 30, 40], "want": [20, 40, 10, 30]},
        {"size": [5, 3, 2, 4], "strides": [12, 1, 60, 3], "indC": [10, 20, 30, 40],
         "labels": [40, 10], "want": [40, 10]},
        {"size": [5, 3, 2, 4], "strides": [12, 1, 60, 3], "indC": [10, 20, 30, 40],
         "labels": [30, 20], "want": [20, 30]},
        {"size": [2, 3, 4], "strides": [1, 1, 1], "indC": [7, 8, 9], "labels": [7, 8, 9], "want": [7, 8, 9]},
        {"size": [2, 3, 4], "strides": [1, 1, 1], "indC": [7, 8, 9], "labels": [9, 7, 8], "want": [9, 7, 8]},
        {"size": [3, 4], "strides": [-1, 4], "indC": [10, 20], "labels": [20, 10], "want": [10, 20]},
        {"size": [3, 4], "strides": [4, -1], "indC": [10, 20], "labels": [10, 20], "want": [20, 10]},
    ]


def leading_unit_run():
    d = 4
    st6 = [1, d, d ** 2, d ** 3, d ** 4, d ** 5]
    six = {"size": [d] * 6, "strides": st6, "indC": [1, 2, 3, 4, 5, 6]}
    a, b, c, i, j, k = 1, 2, 3, 4, 5, 6
    cases = [
        dict(six, labels=[a, i, j], want=d),
        dict(six, labels=[a, b, k], want=d ** 2),
        dict(six, labels=[a, b, c, i, j, k], want=d ** 6),
        dict(six, labels=[b, i, j], want=1),
        dict(six, labels=[a, c, b], want=d),
        dict(six, labels=[], want=1),
        {"size": [3, 4], "strides": [-1, 3], "indC": [10, 20], "labels": [10, 20], "want": 1},
        {"size": [1, 6], "strides": [5, 1], "indC": [10, 20], "labels": [10, 20], "want": 6},
        {"size": [6, 1], "strides": [1, 17], "indC": [10, 20], "labels": [10, 20], "want": 6},
        {"size": [0, 6], "strides": [1, 1], "indC": [10, 20], "labels": [10, 20], "want": 0},
    ]
    return cases


def axis_group():
    return [
        {"lengths": [3, 2], "strides": [[1, 15], [1, 12]],
         "offsets": [[0, 1, 2, 15, 16, 17], [0, 1, 2, 12, 13, 14]]},
        {"lengths": [4], "strides": [[5], [3]], "offsets": [[0, 5, 10, 15], [0, 3, 6, 9]]},
        {"lengths": [5], "strides": [[3], [1]], "offsets": [[0, 3, 6, 9, 12], [0, 1, 2, 3, 4]]},
    ]


def contraction_labels():
    return [{"pA": [[3, 1, 4], [2, 5]], "pB": [[3, 1], [2, 4]], "pAB": [[4, 2], [5, 1, 3]],
             "indA": [2, -1, 1, 3, -2], "indB": [-2, 4, -1, 5], "indC": [4, 2, 5, 1, 3]}]


def label_errors():
    # A (3,4), B (4,5), C (3,5) column-major; each entry must raise the named error.
    return [
        {"A": [3, 4], "B": [6, 5], "C": [3, 5], "indA": [1, 2], "indB": [2, 3], "indC": [1, 3], "error": "DimensionMismatch"},
        {"A": [4, 4], "B": [4, 5], "C": [3, 5], "indA": [1, 1], "indB": [2, 3], "indC": [1, 3], "error": "ArgumentError"},
        {"A": [3, 4], "B": [4, 5], "C": [3, 5], "indA": [1, 2], "indB": [2, 3], "indC": [1, 9], "error": "ArgumentError"},
        {"A": [3, 4], "B": [4, 5], "C": [3, 5], "indA": [1, 2], "indB": [5, 3], "indC": [1, 3], "error": "ArgumentError"},
        {"A": [3, 4], "B": [4, 5], "C": [3, 5], "indA": [1, 2], "indB": [2, 9], "indC": [1, 3], "error": "ArgumentError"},
        {"A": [3, 4], "B": [4, 5], "C": [4, 5], "indA": [1, 2], "indB": [2, 3], "indC": [2, 3], "error": "ArgumentError"},
    ]


def main():
    fixtures = {
        "worked_fixture.json": worked_fixture(),
        "one_rounding.json": one_rounding(),
        "conj_xor.json": conj_xor(),
        "classify_labels.json": classify_labels(),
        "order_free_labels.json": order_free_labels(),
        "leading_unit_run.json": leading_unit_run(),
        "axis_group.json": axis_group(),
        "contraction_labels.json": contraction_labels(),
        "label_errors.json": label_errors(),
    }
    for name, data in fixtures.items():
        with open(os.path.join(HERE, name), "w") as f:
            json.dump(data, f, indent=1)
            f.write("\n")


if __name__ == "__main__":
    main()
