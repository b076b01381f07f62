"""The autotuner's selection and on-disk cache on CPU: host-only plans give
the problem class; a fake measurement replaces the GPU timing."""
import importlib
import json

import pytest
import torch


@pytest.fixture(scope="module")
def at(qs):
    return importlib.import_module(qs.__name__ + ".autotune")


def views(qs, M, K, N, dtype=torch.float64, bt=False):
    A = qs.StridedView(torch.zeros(M * K, dtype=dtype), (M, K), (1, M))
    if bt:
        B = qs.StridedView(torch.zeros(K * N, dtype=dtype), (N, K), (1, N))
        indB = (3, 2)
    else:
        B = qs.StridedView(torch.zeros(K * N, dtype=dtype), (K, N), (1, K))
        indB = (2, 3)
    C = qs.StridedView(torch.zeros(M * N, dtype=dtype), (M, N), (1, M))
    return C, A, (1, 2), B, indB, (1, 3)


def fake(times, errs=None, calls=None):
    def measure(opts):
        if calls is not None:
            calls.append(dict(opts))
        key = (opts["method"], opts.get("native_tile", 0), bool(opts.get("per_product_gemm")))
        e = errs(opts) if errs else 0.0
        return times[key], e
    return measure


T64 = {("native", 1, False): 5.0, ("native", 2, False): 4.0, ("native", 3, False): 6.0,
       ("native", 4, False): 7.0, ("native", 5, False): 2.0, ("native", 6, False): 2.5,
       ("native", 7, False): 3.0, ("native", 8, False): 3.5, ("native", 9, False): 3.8,
       ("native", 10, False): 2.2,
       ("ozaki", 0, False): 1.0, ("ozaki", 0, True): 1.5}


def test_picks_fastest_and_caches_on_disk(qs, at, tmp_path):
    path = str(tmp_path / "tune.json")
    calls = []
    t = at.Autotuner(qs, path=path, measure=fake(T64, calls=calls), device_name="B200")
    C, A, ia, B, ib, ic = views(qs, 300, 200, 260)
    opts = t.options(C, A, ia, B, ib, ic)
    assert opts == {"method": "ozaki"}
    # SIMT tiles 1-4, DMMA tiles 5-10 (real Float64 operands), two Ozaki variants
    assert len(calls) == 12 and t.misses == 1
    assert sorted(c["native_tile"] for c in calls if c["method"] == "native") == list(range(1, 11))
    # same class (sizes in the same log2 buckets): a hit, no measurement
    C2, A2, _, B2, _, _ = views(qs, 400, 250, 300)
    assert t.options(C2, A2, ia, B2, ib, ic) == {"method": "ozaki"}
    assert t.hits == 1 and len(calls) == 12
    # a new process reads the file
    t2 = at.Autotuner(qs, path=path, measure=fake(T64, calls=calls), device_name="B200")
    assert t2.options(C, A, ia, B, ib, ic) == {"method": "ozaki"} and t2.hits == 1
    d = json.load(open(path))
    assert d["version"] == at.CACHE_VERSION and len(d["entries"]) == 1


def test_key_separates_classes(qs, at, tmp_path):
    t = at.Autotuner(qs, path=str(tmp_path / "k.json"), measure=fake(T64), device_name="B200")
    keys = set()
    for args in [(300, 200, 260, torch.float64, False), (300, 200, 260, torch.float64, True),
                 (300, 200, 260, torch.float32, False), (3000, 200, 260, torch.float64, False)]:
        C, A, ia, B, ib, ic = views(qs, *args[:3], dtype=args[3], bt=args[4])
        hp = qs.plan_contract(C, A, ia, B, ib, ic, host_only=True)
        keys.add(t.key(hp, C, A, B, None, False, False))
    assert len(keys) == 4


def test_slices_raised_until_accurate(qs, at, tmp_path):
    # the probe misses 1e-13 at 6 and 7 slices, meets it at 8
    def errs(o):
        if o["method"] != "ozaki":
            return 0.0
        return {6: 3e-13, 7: 2e-13, 8: 5e-15}[o.get("ozaki_slices", 6)]
    t = at.Autotuner(qs, path=str(tmp_path / "s.json"), measure=fake(T64, errs), device_name="B200")
    C, A, ia, B, ib, ic = views(qs, 300, 200, 260)
    assert t.options(C, A, ia, B, ib, ic) == {"method": "ozaki", "ozaki_slices": 8}


def test_float32_candidates_and_non_nest(qs, at, tmp_path):
    T32 = {("native", 1, False): 3.0, ("native", 2, False): 2.0, ("native", 3, False): 2.5,
           ("native", 4, False): 2.6,
           ("bf16x3", 0, False): 2.2, ("ozaki", 0, False): 2.4}
    t = at.Autotuner(qs, path=str(tmp_path / "f.json"), measure=fake(T32), device_name="B200")
    C, A, ia, B, ib, ic = views(qs, 300, 200, 20, dtype=torch.float32)
    assert t.options(C, A, ia, B, ib, ic) == {"method": "native", "native_tile": 2}
    # N == 1: the dot path, nothing to tune
    C1, A1, _, B1, _, _ = views(qs, 300, 200, 1)
    assert t.options(C1, A1, ia, B1, ib, ic) == {}
