"""GPU tests of the autotuner: it measures every candidate on scratch data
of the problem's layout, picks one that meets the accuracy target, caches it
on disk, and the tuned plan matches the oracle; every SIMT gather-GEMM
tile shape it can pick is bitwise equal to the oracle, every DMMA tile
within the reference's 50*K*eps."""
import importlib
import json

import numpy as np
import pytest

from _util import colmajor_pair, rel_fro, run_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("et,MKN,tol", [("Float64", (300, 200, 260), 1e-13), ("Float32", (256, 130, 20), 1e-5),
                                        ("ComplexF64", (130, 64, 140), 1e-13)])
def test_tuned_plan_matches_oracle_and_is_cached(qs, orc, tmp_path, et, MKN, tol):
    at = importlib.import_module(qs.__name__ + ".autotune")
    path = str(tmp_path / "tune.json")
    tuner = at.Autotuner(qs, path=path, reps=2)
    M, K, N = MKN
    rng = np.random.default_rng(M + N)
    A = colmajor_pair(qs, rng, (M, K), et)
    B = colmajor_pair(qs, rng, (K, N), et)
    C = colmajor_pair(qs, rng, (M, N), et)
    A_before = A.device_parent().copy()
    opts = tuner.options(C.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3))
    assert opts["method"] in ("native", "ozaki", "bf16x3")
    assert np.array_equal(A.device_parent(), A_before)  # the caller's data was not touched
    entry = next(iter(json.load(open(path))["entries"].values()))
    assert entry["options"] == opts and all(c["ms"] > 0 for c in entry["candidates"])
    assert any(c["ok"] for c in entry["candidates"])
    got, ref, plan = run_pair(qs, orc, C, 1.1, A, (1, 2), B, (2, 3), 0.3, (1, 3), precision=1, **opts)
    assert rel_fro(got, ref) <= tol, (opts, rel_fro(got, ref))
    t2 = at.Autotuner(qs, path=path)
    assert t2.options(C.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3)) == opts and t2.hits == 1


@pytest.mark.parametrize("tile", [1, 2, 3, 4])
def test_native_tile_override_bitwise(qs, orc, tile):
    rng = np.random.default_rng(tile)
    M, K, N = 333, 97, 45
    A = colmajor_pair(qs, rng, (M, K), "Float64")
    B = colmajor_pair(qs, rng, (K, N), "Float64")
    C = colmajor_pair(qs, rng, (M, N), "Float64")
    got, ref, plan = run_pair(qs, orc, C, 1.3, A, (1, 2), B, (2, 3), 0.7, (1, 3), method="native",
                              native_tile=tile)
    assert plan.native_tile == tile
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("tile", [5, 6, 7, 8, 9])
def test_native_tile_override_dmma(qs, orc, tile):
    # The DMMA kernel's tiles (native_tile 5..9), the autotuner's other knob.
    rng = np.random.default_rng(tile)
    M, K, N = 333, 97, 45
    A = colmajor_pair(qs, rng, (M, K), "Float64")
    B = colmajor_pair(qs, rng, (K, N), "Float64")
    C = colmajor_pair(qs, rng, (M, N), "Float64")
    got, ref, plan = run_pair(qs, orc, C, 1.3, A, (1, 2), B, (2, 3), 0.7, (1, 3), method="native",
                              native_tile=tile)
    assert plan.native_tile == tile
    assert rel_fro(got, ref) <= 50 * K * np.finfo(np.float64).eps
