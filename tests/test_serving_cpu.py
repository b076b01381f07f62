"""Host logic of the serving loop on CPU (no GPU): admission in arrival
order against the HBM budget, many ticks in flight, oversized requests
rejected, the latency statistics, and the request-stream generator.  The
device is replaced by a fake backend whose ticks complete after a few polls
and compute with numpy."""
import importlib

import collections
import threading
import time

import numpy as np
import pytest


@pytest.fixture(scope="module")
def sv(qs):
    return importlib.import_module(qs.__name__ + ".serving")


@pytest.fixture(scope="module")
def wl(qs):
    return importlib.import_module(qs.__name__ + ".workloads")


def einsum_labels(A, indA, B, indB, indC):
    letters = {}
    for l in list(indA) + list(indB):
        letters.setdefault(l, "abcdefghijklmnopqrstuvwxyz"[len(letters)])
    sub = "".join(letters[l] for l in indA) + "," + "".join(letters[l] for l in indB) + "->" + \
        "".join(letters[l] for l in indC)
    return np.einsum(sub, A, B)


class FakeBackend:
    def __init__(self, polls=3):
        self.polls = polls
        self.resident = {}
        self.launched = []
        self.max_concurrent = 0
        self.live = 0

    def shape_of(self, x):
        return self.resident[x].shape if isinstance(x, str) else x.shape

    def put_resident(self, key, array):
        self.resident[key] = np.asarray(array)
        return self.resident[key].nbytes

    def drop_resident(self, key):
        del self.resident[key]

    def request_bytes(self, r):
        n = 0
        for x in (r.A, r.B):
            if not isinstance(x, str):
                n += x.nbytes
        n += int(np.prod(r.c_shape(self.shape_of))) * np.dtype(r.dtype).itemsize
        return n

    def launch_tick(self, batch, grouped=True):
        self.launched.append([id(r) for r in batch])
        self.live += 1
        self.max_concurrent = max(self.max_concurrent, self.live)
        return {"left": self.polls, "batch": batch}

    def tick_done(self, h):
        h["left"] -= 1
        return h["left"] <= 0

    def finish_tick(self, h, batch):
        self.live -= 1
        for r in batch:
            A = self.resident[r.A] if isinstance(r.A, str) else r.A
            C = einsum_labels(A, r.indA, r.B, r.indB, r.indC)
            r.result = r.alpha * C + (r.beta * r.C0 if r.C0 is not None else 0)

    def cached_bytes(self):
        return 0

    def evict(self, nbytes):
        pass


def mk(sv, rng, n, size=8):
    reqs = []
    for i in range(n):
        A = rng.standard_normal((size, size))
        B = rng.standard_normal((size, size))
        reqs.append(sv.ContractRequest(A, (1, 2), B, (2, 3), (1, 3), alpha=1.0 + i, tag=i))
    return reqs


def test_fifo_budget_and_results(sv):
    rng = np.random.default_rng(0)
    be = FakeBackend()
    per = 3 * 8 * 8 * 8
    srv = sv.ContractionServer(be, hbm_budget_bytes=5 * per, max_ticks=3, max_tick_requests=2)
    reqs = mk(sv, rng, 40)
    for r in reqs:
        srv.submit(r)
    srv.drain(timeout=30)
    assert srv.peak_used <= 5 * per
    assert be.max_concurrent >= 2           # ticks overlapped
    order = [i for tick in be.launched for i in tick]
    assert order == [id(r) for r in reqs]   # admitted in arrival order
    for r in reqs:
        ref = einsum_labels(r.A, r.indA, r.B, r.indB, r.indC) * r.alpha
        assert np.allclose(r.result, ref)
    assert srv.used == 0


def test_resident_operands_count_and_oversize_rejected(sv):
    rng = np.random.default_rng(1)
    be = FakeBackend()
    srv = sv.ContractionServer(be, hbm_budget_bytes=4096)
    env = rng.standard_normal((8, 8))
    srv.put_resident("env", env)
    assert srv.used == env.nbytes
    big = sv.ContractRequest(rng.standard_normal((64, 64)), (1, 2), rng.standard_normal((64, 8)), (2, 3),
                             (1, 3))
    ok = sv.ContractRequest("env", (1, 2), rng.standard_normal((8, 4)), (2, 3), (1, 3))
    srv.submit(big)
    srv.submit(ok)
    srv.drain(timeout=30)
    assert big.error is not None and big.result is None
    assert ok.error is None and np.allclose(ok.result, env @ ok.B)
    srv.drop_resident("env")
    assert srv.used == 0


def test_replay_and_percentiles(sv):
    rng = np.random.default_rng(2)
    be = FakeBackend(polls=1)
    srv = sv.ContractionServer(be)
    reqs = mk(sv, rng, 30)
    offsets = np.cumsum(rng.exponential(1e-3, 30))
    srv.replay(reqs, offsets, timeout=30)
    st = srv.stats(reqs)
    assert st["requests"] == 30 and st["errors"] == 0
    assert 0 <= st["p50_ms"] <= st["p99_ms"]
    assert all(r.done >= r.arrival for r in reqs)
    assert sv.percentile([5, 1, 3, 2, 4], 50) == 3
    assert sv.percentile(list(range(1, 101)), 99) == 99


def test_serving_stream_mix(wl):
    specs, offsets, residents = wl.serving_stream(400, rate=1000.0, seed=9)
    assert np.all(np.diff(offsets) >= 0) and offsets[0] == 0
    fams = {s["family"] for s in specs}
    assert {"matmul", "permuted4", "block", "random"} <= fams and fams & {"mps1", "mps2", "mps3"}
    dts = [np.dtype(s["dtype"]).name for s in specs]
    for name, p in (("float32", 0.4), ("float64", 0.4), ("complex128", 0.2)):
        assert abs(dts.count(name) / len(dts) - p) < 0.08
    reuse = sum(1 for s in specs if s["resident"]) / len(specs)
    assert abs(reuse - 0.3) < 0.07
    for s in specs:
        if s["family"] == "random":
            ra, rb = len(s["shapeA"]), len(s["shapeB"])
            assert 2 <= ra <= 6 and 2 <= rb <= 6
            assert 1 <= len(set(s["indA"]) & set(s["indB"])) <= 3
            assert sorted(s["indC"]) == sorted(set(s["indA"]) ^ set(s["indB"]))
            total = np.prod(s["shapeA"]) + np.prod(s["shapeB"]) + \
                np.prod([dict(zip(s["indA"] + s["indB"], s["shapeA"] + s["shapeB"]))[l] for l in s["indC"]])
            assert total <= 1e8
        if s["resident"]:
            assert residents[s["resident"]][0] == s["shapeA"]


def test_arena_first_fit_and_merge(sv):
    a = sv.Arena(4096, align=256)
    x = a.alloc(100)
    y = a.alloc(1000)
    z = a.alloc(300)
    assert (x, y, z) == (0, 256, 1280)
    assert a.alloc(4096) is None
    a.free(y)
    assert a.alloc(700) == 256          # first fit into the hole
    a.free(x)
    a.free(z)
    a.free(256)
    assert a.free_list == [(0, 4096)] and a.used() == 0
    blocks = [a.alloc(256) for _ in range(16)]
    assert a.alloc(1) is None
    for b in blocks[::2]:
        a.free(b)
    for b in blocks[1::2]:
        a.free(b)
    assert a.free_list == [(0, 4096)]


def test_tick_work_cap(sv):
    rng = np.random.default_rng(4)
    be = FakeBackend(polls=2)
    reqs = mk(sv, rng, 12)                      # each 2*8*8*8 = 1024 flops
    srv = sv.ContractionServer(be, max_ticks=8, max_tick_flops=3000)
    for r in reqs:
        srv.submit(r)
    srv.drain(timeout=30)
    assert all(len(t) <= 2 for t in be.launched)  # two 1024-flop requests per tick
    assert sum(len(t) for t in be.launched) == 12


class PreparingBackend(FakeBackend):
    """A backend with `prepare`: the server stages requests on its
    preparation thread (or in the loop when the thread has not started one)
    before admitting them; a slow prepare makes both paths run."""

    def __init__(self, polls=2, delay=2e-4):
        super().__init__(polls)
        self.delay = delay
        self.prepared = collections.Counter()
        self.threads = set()
        self.lock = threading.Lock()

    def prepare(self, r):
        time.sleep(self.delay)
        with self.lock:
            self.prepared[id(r)] += 1
            self.threads.add(threading.current_thread().name)
        r._prep = True

    def launch_tick(self, batch, grouped=True):
        assert all(r._prep for r in batch)  # admitted only once prepared
        return super().launch_tick(batch, grouped)


def test_preparation_thread_budget_fifo_and_results(sv):
    rng = np.random.default_rng(4)
    be = PreparingBackend()
    per = 3 * 8 * 8 * 8
    srv = sv.ContractionServer(be, hbm_budget_bytes=5 * per, max_ticks=3, max_tick_requests=2)
    reqs = mk(sv, rng, 60)
    offsets = np.cumsum(rng.exponential(3e-4, 60))
    srv.replay(reqs, offsets, timeout=60)
    srv.close()
    assert all(be.prepared[id(r)] == 1 for r in reqs)   # each prepared exactly once
    assert srv.peak_used <= 5 * per                      # preparation is charged to the budget
    order = [i for tick in be.launched for i in tick]
    assert order == [id(r) for r in reqs]                # admitted in arrival order
    for r in reqs:
        assert r.error is None
        assert np.allclose(r.result, einsum_labels(r.A, r.indA, r.B, r.indB, r.indC) * r.alpha)
    assert srv.used == 0
