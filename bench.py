"""Benchmark of the contraction engine on one B200 (or N replicas under torchrun).

Workload: the permuted 4-index Float64 contraction
    C[a,b,c,d] = 1.3 * sum_{e,f} A[a,e,b,f] * B[f,c,e,d] + 0.7 * C[a,b,c,d]
with a=b=c=d=64, e=f=48 (M = N = 4096, K = 2304), A and B iid uniform[-1,1]
from a seeded generator, C seeded N(0,1), column-major (Julia layout).  One
step = one ``execute`` of a reused plan (pack + tensor-core GEMM + epilogue).
Inputs (A 75 MB, B 75 MB, C 268 MB) are larger than the 126 MB L2, so no
explicit flush runs between steps.

Prints one JSON line (rank 0).  ``--impl reference`` times the CPU arm: the
oracle's restatement of the reference's five-loop nest (QuasiStrided.jl is
Julia and cannot run here) on the host cores.

Other workloads (``--workload``): ``matmul`` (the permuted matmul, latency),
``mps`` (ComplexF64 MPS environment update), ``blocks`` (2000 uneven U(1)
blocks: grouped vs graph vs plain launches), ``serving`` (a Poisson stream of
mixed requests: continuous batching vs one request at a time), ``u1net`` (a
U(1)-symmetric contraction through the block-sparse front end: grouped waves
vs sequential plans vs the dense contraction).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SIZES = dict(a=64, b=64, c=64, d=64, e=48, f=48)
LABELS = dict(indA=(1, 5, 2, 6), indB=(6, 3, 5, 4), indC=(1, 2, 3, 4))
ALPHA, BETA = 1.3, 0.7
M = N = 64 * 64
K = 48 * 48
FLOPS = 2.0 * M * N * K
WORKLOAD = "permuted4_f64_M4096_N4096_K2304"


def load_engine():
    pkg = os.path.join(ROOT, "quasistrided.jl_b200")
    if "quasistrided_b200" in sys.modules:
        return sys.modules["quasistrided_b200"]
    spec = importlib.util.spec_from_file_location("quasistrided_b200", os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["quasistrided_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def shapes():
    s = SIZES
    return ((s["a"], s["e"], s["b"], s["f"]), (s["f"], s["c"], s["e"], s["d"]),
            (s["a"], s["b"], s["c"], s["d"]))


def host_inputs(seed=20261203, wide=False):
    """Seeded column-major inputs (flat float64 arrays)."""
    rng = np.random.default_rng(seed)
    sa, sb, sc = shapes()
    A = rng.uniform(-1.0, 1.0, int(np.prod(sa)))
    B = rng.uniform(-1.0, 1.0, int(np.prod(sb)))
    C = rng.standard_normal(int(np.prod(sc)))
    if wide:
        ua = rng.integers(-20, 21, sa[0]).astype(np.float64)
        ud = rng.integers(-20, 21, sb[3]).astype(np.float64)
        A = (A.reshape(sa, order="F") * np.exp2(ua)[:, None, None, None]).ravel(order="F")
        B = (B.reshape(sb, order="F") * np.exp2(ud)[None, None, None, :]).ravel(order="F")
    return A, B, C


def c1_accuracy(orc, got, A_h, B_h, C_h):
    """Relative Frobenius error of one execute's C (`got`, flat, from the
    seeded C) over every element against the oracle's FP64 nest, and over a
    sample of 8^4 elements spread over all four indices of C (every 8th
    a, b, c, d) against the oracle in binary128."""
    sa, sb, sc = shapes()
    f64 = lambda x: np.ascontiguousarray(x, dtype=np.float64)  # noqa: E731
    Ah = orc.HostView(f64(A_h), sa, colmajor_strides(sa))
    Bh = orc.HostView(f64(B_h), sb, colmajor_strides(sb))
    Cref = orc.HostView(f64(C_h).copy(), sc, colmajor_strides(sc))
    orc.nest_f64(Cref, ALPHA, Ah, LABELS["indA"], Bh, LABELS["indB"], BETA, LABELS["indC"])
    full = orc.rel_fro(got.astype(np.float64), Cref.parent)
    picks = {1: (1, 8, 8), 2: (3, 8, 8), 3: (5, 8, 8), 4: (7, 8, 8)}
    sub = lambda v, lab: orc.label_subview(v, lab, picks)  # noqa: E731
    Cq = orc.HostView(f64(C_h).copy(), sc, colmajor_strides(sc))
    Cs = sub(Cq, LABELS["indC"])
    orc.brute(Cs, ALPHA, sub(Ah, LABELS["indA"]), LABELS["indA"], sub(Bh, LABELS["indB"]), LABELS["indB"], BETA,
              LABELS["indC"], precision=1, threads=orc.max_threads())
    gs = orc.HostView(got.astype(np.float64), Cs.size, Cs.strides, Cs.offset).to_array()
    exact = orc.rel_fro(gs, Cs.to_array())
    return {"rel_err": full, "elements": int(got.size), "rel_err_binary128": exact,
            "sample": "every 8th index along each of a, b, c, d (4096 elements)"}


def colmajor_strides(shape):
    st, acc = [], 1
    for s in shape:
        st.append(acc)
        acc *= s
    return tuple(st)


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index=0):
        self.idx = device_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) > 8:
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


STAGE_NAMES = {"ozaki": ["pack_a", "pack_b", "gemm_i8", "fixup"],
               "bf16x3": ["pack", "pack_none", "gemm_bf16"],
               "native": ["gemm_native"]}


def library_peaks():
    """cuBLAS INT8 and FP64 GEMM throughput measured on this pool by
    `bench.py --peaks` (profiles/library_peaks_b200.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "library_peaks_b200.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def load_ncu_traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(kernel)
    except (OSError, ValueError):
        return None


def roofline(plan, stage_ms, nexec):
    """Roofline of the dominant kernel from the per-stage CUDA-event times of
    the timed region.  Ozaki GEMM: algorithmic work = the slice products,
    s(s+1)/2 * 2MNK int8 ops; peak = the measured cuBLAS int8 GEMM of
    profiles/library_peaks_b200.json (else 2x the dense bf16 figure).  Native
    GEMM: 2MNK fp64 flops against the measured cuBLAS DGEMM (else the
    nominal 40 TFLOP/s)."""
    peaks, kind = measured_peaks()
    lib = library_peaks()
    names = STAGE_NAMES.get(plan.method, [f"stage{i}" for i in range(len(stage_ms))])
    per = {names[i] if i < len(names) else f"stage{i}": stage_ms[i] / max(nexec, 1)
           for i in range(len(stage_ms))}
    if plan.method == "ozaki":
        s = plan.ozaki_slices
        work = s * (s + 1) / 2 * FLOPS
        ms = per.get("gemm_i8")
        if lib:
            peak = lib["int8_int_mm_tops"]
            note = "measured cuBLAS int8 GEMM (torch._int_mm 8192^3) on this pool"
        else:
            peak = 2.0 * peaks["bf16_tflops"]
            note = f"int8 dense peak = 2 x {kind} bf16 dense ({peaks['bf16_tflops']} TFLOP/s)"
        if s in (4, 6, 7) and not plan.per_product_gemm:
            kernel = f"oz_gemm_fixed_kernel<{s}, false>" if plan.oz_single_sm else f"oz_gemm_pair_kernel<{s}>"
        else:
            kernel = "tc_gemm_kernel<KIND_I8>"
    elif plan.method == "bf16x3":
        work = 3 * FLOPS
        ms = per.get("gemm_bf16")
        peak = peaks["bf16_tflops"]
        note = f"{kind} bf16 dense"
        kernel = "tc_gemm_kernel<KIND_BF16>"
    else:
        work = FLOPS
        ms = per.get("gemm_native")
        if lib:
            peak = lib["fp64_cublas_tflops"]
            note = "measured cuBLAS DGEMM (8192^3) on this pool"
        else:
            peak = 40.0
            note = "nominal B200 FP64"
        kernel = "dmma_gemm_kernel" if getattr(plan, "native_tile", 0) >= 5 else "direct_gemm_kernel"
    achieved = work / (ms * 1e-3) / 1e12 if ms else None
    roof = {"bound": "tensor", "kernel": kernel, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak if achieved else None, "traffic": load_ncu_traffic(kernel),
            "ms_per_launch": ms, "peak_note": note}
    return roof, per


def measure_library_peaks():
    """cuBLAS int8 (torch._int_mm) and fp64 (torch.matmul) GEMM throughput on
    this GPU, for context beside the roofline denominators."""
    import torch
    out = {}
    n = 8192
    a = torch.randint(-127, 128, (n, n), dtype=torch.int8, device="cuda")
    b = torch.randint(-127, 128, (n, n), dtype=torch.int8, device="cuda")
    for name, fn, flops in (("int8_int_mm_tops", lambda: torch._int_mm(a, b), 2.0 * n ** 3),):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        best = 1e30
        for _ in range(10):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        out[name] = flops / (best * 1e-3) / 1e12
    x = torch.randn(n, n, dtype=torch.float64, device="cuda")
    y = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(x, y)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(x, y)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    out["fp64_cublas_tflops"] = 2.0 * n ** 3 / (best * 1e-3) / 1e12
    out["gpu"] = torch.cuda.get_device_name()
    print(json.dumps(out), flush=True)


def run_profile_target(args):
    """A short, self-contained run for ncu: the c1 plan, one warm-up execute,
    then --steps executes."""
    import torch
    qs = load_engine()
    A_h, B_h, C_h = host_inputs()
    sa, sb, sc = shapes()
    Av = qs.StridedView(torch.from_numpy(A_h).cuda(), sa, colmajor_strides(sa), 0)
    Bv = qs.StridedView(torch.from_numpy(B_h).cuda(), sb, colmajor_strides(sb), 0)
    Cv = qs.StridedView(torch.from_numpy(C_h).cuda(), sc, colmajor_strides(sc), 0)
    plan = qs.plan_contract(Cv, Av, LABELS["indA"], Bv, LABELS["indB"], LABELS["indC"], method=args.method,
                            per_product_gemm=args.per_product, oz_single_sm=args.oz_single_sm)
    qs.execute(plan, ALPHA, BETA)
    for _ in range(args.steps):
        qs.execute(plan, ALPHA, BETA)
    torch.cuda.synchronize()
    qs.check_status(plan)
    print(json.dumps({"profile_target": WORKLOAD, "method": plan.method, "steps": args.steps}))
    plan.release()


def cpu_sample(orc, A, B, C, rows, threads):
    """Time the oracle's nest restatement on `rows` rows of M (c1 layout)."""
    sa, sb, sc = shapes()
    Av = orc.HostView(A, sa, colmajor_strides(sa))
    Bv = orc.HostView(B, sb, colmajor_strides(sb))
    Cv = orc.HostView(C.copy(), sc, colmajor_strides(sc))
    t0 = time.perf_counter()
    orc.nest_f64(Cv, ALPHA, Av, LABELS["indA"], Bv, LABELS["indB"], BETA, LABELS["indC"],
                 m_range=(0, rows), threads=threads)
    dt = time.perf_counter() - t0
    return 2.0 * rows * N * K / dt / 1e12, dt


def host_cpu():
    """The host's CPU model and logical core count (for the CPU baseline)."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": model, "logical_cores": os.cpu_count()}


def run_reference(args, rank, world):
    """CPU arm: the oracle's nest restatement on all host threads (or
    --cpu-threads), rank 0 only."""
    if rank != 0:
        return
    from oracle import oracle as orc
    threads = args.cpu_threads or orc.max_threads()
    A, B, C = host_inputs()
    rows = args.cpu_rows
    for _ in range(args.warmup):
        cpu_sample(orc, A, B, C, max(64, rows // 8), threads)
    vals, times = [], []
    for _ in range(args.steps):
        v, dt = cpu_sample(orc, A, B, C, rows, threads)
        vals.append(v)
        times.append(dt)
    value = statistics.median(vals)
    sample = f"{rows} of {M} rows of M (all N, all K) per step, oracle nest restatement, {threads} threads"
    print(json.dumps({
        "impl": "reference", "metric": "contraction TFLOP/s (Float64, rel.err<=1e-13 vs FP64)",
        "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * statistics.median(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded uniform[-1,1] A/B, N(0,1) C)",
        "config": {"workload": WORKLOAD, "M": M, "N": N, "K": K, "alpha": ALPHA, "beta": BETA,
                   "l2": "inputs larger than L2"},
        "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": threads, "kind": "port",
                         "sample": sample, "host": host_cpu()},
        "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_blocks(args):
    """Uneven blocks of a U(1)-symmetric step: 2000 independent contractions
    C[x,y,z] = sum A[x,k1,k2,y] * B[k2,z,k1] (alpha = 1, beta = 0), Float64
    and Float32, as (1) one execute per block from C (the plain launches),
    (2) a CUDA graph of those launches, (3) grouped persistent launches,
    (4) a CUDA graph of the grouped launches.  Prints one JSON line."""
    import torch
    qs = load_engine()
    from oracle import oracle as orc
    wl = __import__(qs.__name__ + ".workloads", fromlist=["u1_blocks"])
    blocks = wl.u1_blocks(n=args.blocks, seed=20261203, cap=args.block_cap)
    hist = wl.histogram(blocks)
    flops = hist["flops"]
    modes = (("plain", "sequential", False), ("plain_graph", "sequential", True),
             ("grouped", "persistent", False), ("grouped_graph", "persistent", True))
    out = {"metric": "aggregate contraction TFLOP/s over uneven blocks (grouped persistent launches)",
           "unit": "TFLOP/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "data": "synthetic (seeded N(0,1) operands)",
           "config": {"workload": f"u1_blocks_{len(blocks)}", "cap_elements": args.block_cap,
                      "alpha": 1.0, "beta": 0.0, "l2": "operands larger than L2, no flush"},
           "histogram": hist, "by_dtype": {}}
    gen = torch.Generator(device="cuda")
    for dt_name, tdt, et in (("f64", torch.float64, "Float64"), ("f32", torch.float32, "Float32")):
        if dt_name not in args.dtypes.split(","):
            continue
        gen.manual_seed(7)
        views, plans = [], []
        for b in blocks:
            sa, la = b.a_shape_labels()
            sb, lb = b.b_shape_labels()
            sc, lc = b.c_shape_labels()
            Ad = torch.randn(int(np.prod(sa)), dtype=tdt, device="cuda", generator=gen)
            Bd = torch.randn(int(np.prod(sb)), dtype=tdt, device="cuda", generator=gen)
            Cd = torch.zeros(int(np.prod(sc)), dtype=tdt, device="cuda")
            Av = qs.StridedView(Ad, sa, colmajor_strides(sa), 0)
            Bv = qs.StridedView(Bd, sb, colmajor_strides(sb), 0)
            Cv = qs.StridedView(Cd, sc, colmajor_strides(sc), 0)
            views.append((Av, Bv, Cv, la, lb, lc))
            plans.append(qs.plan_contract(Cv, Av, la, Bv, lb, lc))
        torch.cuda.synchronize()
        n = len(plans)
        ones, zeros = [1.0] * n, [0.0] * n
        res = {"methods": {}}
        for p in plans:
            res["methods"][p.method] = res["methods"].get(p.method, 0) + 1
        # Accuracy on a few blocks against the FP64 oracle (grouped result).
        g = qs.ContractGroup(plans, mode="persistent")
        g.execute(ones, zeros)
        torch.cuda.synchronize()
        errs = []
        idx = sorted(range(n), key=lambda i: blocks[i].flops)
        for i in (idx[0], idx[n // 2], idx[-1]):
            Av, Bv, Cv, la, lb, lc = views[i]
            Ah = orc.HostView(Av.parent.cpu().numpy().astype(np.float64), Av.size, Av.strides)
            Bh = orc.HostView(Bv.parent.cpu().numpy().astype(np.float64), Bv.size, Bv.strides)
            Ch = orc.HostView(np.zeros(Cv.parent.numel()), Cv.size, Cv.strides)
            orc.brute(Ch, 1.0, Ah, la, Bh, lb, 0.0, lc)
            got = Cv.parent.cpu().numpy().astype(np.float64)
            errs.append(float(np.linalg.norm(got - Ch.parent) / max(np.linalg.norm(Ch.parent), 1e-300)))
        g.release()
        res["rel_err_max_sampled"] = max(errs)
        subsets = {}
        if args.breakdown:
            for meth in res["methods"]:
                subsets["grouped_only_" + meth] = [p for p in plans if p.method == meth]
        run_modes = [m for m in modes if args.modes == "all" or m[0] in args.modes.split(",")]
        run_modes += [(k, "persistent", False) for k in subsets]
        for name, mode, graph in run_modes:
            members = subsets.get(name, plans)
            ones, zeros = [1.0] * len(members), [0.0] * len(members)
            g = qs.ContractGroup(members, mode=mode, graph=graph)
            for _ in range(args.warmup):
                g.execute(ones, zeros)
            torch.cuda.synchronize()
            l0 = qs._abi.lib().qs_launch_count()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record()
            for _ in range(args.steps):
                g.execute(ones, zeros)
            e1.record()
            torch.cuda.synchronize()
            wall = (time.perf_counter() - t0) * 1e3 / args.steps
            ms = e0.elapsed_time(e1) / args.steps
            launches = (qs._abi.lib().qs_launch_count() - l0) / args.steps
            info = g.info()
            res[name] = {"ms_per_step": ms, "host_ms_per_step": wall, "tflops": flops / (ms * 1e-3) / 1e12,
                         "kernels_per_step": launches if not graph else info["launches"],
                         "classes": info["classes"], "tc_plans": info["tc_plans"],
                         "native_plans": info["native_plans"]}
            g.release()
        out["by_dtype"][dt_name] = res
        for p in plans:
            p.release()
        del views, plans
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    f64 = out["by_dtype"].get("f64", {})
    out["value"] = f64.get("grouped", {}).get("tflops")
    out["ms_per_step"] = f64.get("grouped", {}).get("ms_per_step")
    out["dtype"] = "f64"
    print(json.dumps(out), flush=True)


def run_serving(args):
    """Mixed request stream served with continuous batching vs one request at
    a time, at several Poisson arrival rates.  Prints one JSON line."""
    import torch
    qs = load_engine()
    wl = __import__(qs.__name__ + ".workloads", fromlist=["serving_stream"])
    sv = __import__(qs.__name__ + ".serving", fromlist=["ContractionServer"])
    tdt = {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
           np.dtype(np.complex128): torch.complex128}
    pool_elems = 1 << 26
    pool = wl.pool_arrays(pool_elems, seed=11,
                          allocate=lambda n, dt: torch.empty(n, dtype=tdt[np.dtype(dt)], pin_memory=True).numpy())

    def requests(specs):
        out = []
        for sp in specs:
            buf = pool[np.dtype(sp["dtype"])]
            A = sp["resident"] or wl.colmajor_view(buf, sp["shapeA"], 0)
            nB = int(np.prod(sp["shapeB"]))
            B = wl.colmajor_view(buf, sp["shapeB"], pool_elems - nB)
            r = sv.ContractRequest(A, sp["indA"], B, sp["indB"], sp["indC"], alpha=sp["alpha"],
                                   beta=sp["beta"], dtype=sp["dtype"], tag=sp["family"])
            if sp["beta"] != 0:
                sa = sp["shapeA"]
                dims = dict(zip(sp["indA"], sa))
                dims.update(zip(sp["indB"], sp["shapeB"]))
                sc = tuple(dims[l] for l in sp["indC"])
                r.C0 = wl.colmajor_view(buf, sc, 0)
            out.append(r)
        return out

    rates = [float(x) for x in args.rates.split(",")]
    result = {"metric": "served p50/p99 latency (ms) and aggregate TFLOP/s, mixed contraction stream",
              "unit": "ms", "n_gpus": 1, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
              "dtype": "mixed f32/f64/c64", "data": "synthetic (seeded N(0,1) pools)",
              "config": {"workload": f"serving_{args.requests}_requests", "hbm_budget_gb": args.budget_gb,
                         "families": "matmul, permuted4, mps steps, u1 block, random rank-2..6 pairs",
                         "reuse": 0.3, "eltypes": "f32/f64/c64 40/40/20"},
              "rates": []}
    # One backend (its device and pinned arenas are allocated once); its plan
    # cache is cleared before every run so no run inherits another's plans.
    be = sv.DeviceBackend(qs, grouped=True, device_arena_bytes=int(args.arena_gb * (1 << 30)),
                          host_arena_bytes=int(args.host_arena_gb * (1 << 30)))
    for rate in rates:
        specs, offsets, residents = wl.serving_stream(args.requests, rate, seed=int(rate) + 7,
                                                      pool_elems=pool_elems)
        row = {"rate_per_s": rate}
        for mode in ("batched", "sequential"):
            be.clear_plan_cache()
            be.timing.clear()
            be.tick_gpu_ms.clear()
            be.fallbacks.clear()
            # the client takes each result as it completes and hands the
            # pinned buffer back
            consume = sv.ContractRequest.release_result
            srv = sv.ContractionServer(be, hbm_budget_bytes=int(args.budget_gb * (1 << 30)),
                                       max_tick_flops=args.tick_flops, on_done=consume)
            for key, (shape, dt) in residents.items():
                srv.put_resident(key, wl.colmajor_view(pool[np.dtype(dt)], shape, 0))
            # warm-up: the first requests of the stream, untimed
            warm = requests(specs[:min(10, len(specs))])
            for r in warm:
                srv.submit(r)
            srv.drain()
            reqs = requests(specs)
            torch.cuda.synchronize()
            if mode == "batched":
                makespan = srv.replay(reqs, offsets)
            else:
                makespan = sv.serve_sequential(be, reqs, offsets, on_done=consume)
            flops = sum(r.flops(be.shape_of) for r in reqs)
            st = srv.stats(reqs)
            row[mode] = {"p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"],
                         "makespan_s": makespan, "tflops": flops / makespan / 1e12,
                         "ticks": srv.ticks_launched if mode == "batched" else len(reqs),
                         "peak_budget_gb": srv.peak_used / (1 << 30), "errors": st["errors"],
                         "tick_flops": args.tick_flops if mode == "batched" else None,
                         "host_s": {k: round(v, 4) for k, v in be.timing.items()},
                         "tick_gpu_ms_sum": round(sum(be.tick_gpu_ms), 2),
                         "tick_gpu_ms_max": round(max(be.tick_gpu_ms), 2) if be.tick_gpu_ms else None,
                         "arena_fallbacks": dict(be.fallbacks)}
            for key in residents:
                srv.drop_resident(key)
            srv.close()
            del srv
            torch.cuda.synchronize()
        result["rates"].append(row)
    top = result["rates"][-1]["batched"]
    result["value"] = top["p99_ms"]
    print(json.dumps(result), flush=True)


def run_mps(args):
    """ComplexF64 MPS environment update as three pairwise contractions
    (chi = 1024, D_W = 5, d = 2):
        T1[w,al',s,be]   = L[al,w,al'] * A[al,s,be]                (5120 x 2048 x 1024)
        T2[al',be,w',t]  = T1[w,al',s,be] * W[w,s,w',t]            (1048576 x 10 x 10)
        out[be,w',be']   = T2[al',be,w',t] * conj(A)[al',t,be']    (5120 x 1024 x 2048)
    One step = the three executes on reused plans.  Prints one JSON line."""
    import torch
    qs = load_engine()
    from oracle import oracle as orc
    chi, D, d = 1024, 5, 2
    g = torch.Generator(device="cuda")
    g.manual_seed(20261203)

    def crandn(*shape):
        n = int(np.prod(shape))
        return torch.randn(n, dtype=torch.complex128, device="cuda", generator=g)

    L = crandn(chi, D, chi)
    A = crandn(chi, d, chi)
    W = crandn(D, d, D, d)
    T1 = torch.zeros(D * chi * d * chi, dtype=torch.complex128, device="cuda")
    T2 = torch.zeros(chi * chi * D * d, dtype=torch.complex128, device="cuda")
    out = torch.zeros(chi * D * chi, dtype=torch.complex128, device="cuda")
    V = lambda t, shape: qs.StridedView(t, shape, colmajor_strides(shape), 0)  # noqa: E731
    Lv, Av, Wv = V(L, (chi, D, chi)), V(A, (chi, d, chi)), V(W, (D, d, D, d))
    T1v, T2v, Ov = V(T1, (D, chi, d, chi)), V(T2, (chi, chi, D, d)), V(out, (chi, D, chi))
    steps = [
        ("T1=L*A", qs.plan_contract(T1v, Lv, (1, 2, 3), Av, (1, 4, 5), (2, 3, 4, 5)), 8.0 * 5120 * 2048 * 1024),
        ("T2=T1*W", qs.plan_contract(T2v, T1v, (2, 3, 4, 5), Wv, (2, 4, 6, 7), (3, 5, 6, 7)), 8.0 * chi * chi * 10 * 10),
        ("out=T2*conj(A)", qs.plan_contract(Ov, T2v, (3, 5, 6, 7), Av, (3, 7, 8), (5, 6, 8), conjB=True),
         8.0 * 5120 * 1024 * 2048),
    ]
    total_flops = sum(f for _, _, f in steps)
    for _ in range(args.warmup):
        for _, p, _ in steps:
            qs.execute(p, 1.0, 0.0)
    torch.cuda.synchronize()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    per = [0.0, 0.0, 0.0]
    e_all0, e_all1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_all0.record()
    for _ in range(args.steps):
        evs[0].record()
        for i, (_, p, _) in enumerate(steps):
            qs.execute(p, 1.0, 0.0)
            evs[i + 1].record()
        torch.cuda.synchronize()
        for i in range(3):
            per[i] += evs[i].elapsed_time(evs[i + 1])
    e_all1.record()
    torch.cuda.synchronize()
    per = [x / args.steps for x in per]
    ms = sum(per)
    # Accuracy per step on sampled outputs, each from the device's own inputs.
    errs = []
    host = lambda t: t.cpu().numpy()  # noqa: E731
    samples = [
        (host(T1), (D, chi, d, chi), host(L), (chi, D, chi), (1, 2, 3), host(A), (chi, d, chi), (1, 4, 5),
         (2, 3, 4, 5), False),
        (host(T2), (chi, chi, D, d), host(T1), (D, chi, d, chi), (2, 3, 4, 5), host(W), (D, d, D, d),
         (2, 4, 6, 7), (3, 5, 6, 7), False),
        (host(out), (chi, D, chi), host(T2), (chi, chi, D, d), (3, 5, 6, 7), host(A), (chi, d, chi), (3, 7, 8),
         (5, 6, 8), True),
    ]
    nsamp = 4096
    for got, sc, a, sa, ia, b, sb, ib, ic, cj in samples:
        Ch = orc.HostView(np.zeros_like(got), sc, colmajor_strides(sc))
        orc.brute(Ch, 1.0, orc.HostView(a, sa, colmajor_strides(sa)), ia, orc.HostView(b, sb, colmajor_strides(sb)),
                  ib, 0.0, ic, conjB=cj, c_range=(0, nsamp))
        ref = Ch.parent[:nsamp]
        errs.append(float(np.linalg.norm(got[:nsamp] - ref) / np.linalg.norm(ref)))
    bytes2 = (T1.numel() + W.numel() + T2.numel()) * 16
    res = {
        "metric": "contraction TFLOP/s (ComplexF64 MPS environment update, rel.err<=1e-13 vs FP64)",
        "value": total_flops / (ms * 1e-3) / 1e12, "unit": "TFLOP/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64 (ComplexF64)", "data": "synthetic (seeded complex N(0,1)/sqrt2)",
        "config": {"workload": "mps_env_update_chi1024_DW5_d2", "flops": total_flops},
        "stages": [{"step": name, "method": p.method, "complex_mode": p.complex_mode, "ms": t,
                    "tflops": f / (t * 1e-3) / 1e12, "rel_err_sampled": e}
                   for (name, p, f), t, e in zip(steps, per, errs)],
        "step2_hbm_gbs": bytes2 / (per[1] * 1e-3) / 1e9,
    }
    print(json.dumps(res), flush=True)
    for _, p, _ in steps:
        p.release()


def run_u1net(args):
    """A U(1)-symmetric two-site contraction C[a,s,t,b] = sum_{k,l}
    A[a,s,k,l] * B[l,k,t,b] in Float64 (fluxes 0; bond legs a, b: charges
    -6..6 with Gaussian sector sizes, 958 in total; k: charges -3..3, 196;
    l: charges -1..1 of 4/8/4; physical s, t: charges -1..1 of 2/4/2): 189
    block products in 3 waves, 9.5 GFLOP against 368 GFLOP dense.  Runs
    through the block-sparse front end (block products paired by charge,
    emitted as grouped problem tables in waves) and times the grouped waves,
    the same products as sequential per-plan groups, and the engine's dense
    contraction of the densified tensors; checks the block result against
    the dense one.  Prints one JSON line."""
    import importlib
    import torch
    qs = load_engine()
    bs = importlib.import_module(qs.__name__ + ".blocksparse")

    def gauss(qmax, peak, w):
        q = np.arange(-qmax, qmax + 1)
        return bs.U1Space(tuple((int(c), int(max(1, round(peak * np.exp(-c * c / w))))) for c in q))

    bond, kleg = gauss(6, 192, 8.0), gauss(3, 64, 3.0)
    lleg = bs.U1Space(((-1, 4), (0, 8), (1, 4)))
    phys = bs.U1Space(((-1, 2), (0, 4), (1, 2)))
    A = bs.BlockSparseTensor.random([bond, phys, kleg, lleg], 0, torch.float64, seed=11)
    B = bs.BlockSparseTensor.random([lleg.flip(), kleg.flip(), phys, bond.flip()], 0, torch.float64, seed=12)
    labels = ((1, 2, 3, 4), (4, 3, 5, 6), (1, 2, 5, 6))
    C = bs.BlockSparseTensor([bond, phys, phys, bond.flip()], 0, torch.float64)
    bc = bs.BlockContraction(C, A, labels[0], B, labels[1], labels[2], mode="persistent")
    C2 = bs.BlockSparseTensor([bond, phys, phys, bond.flip()], 0, torch.float64)
    bseq = bs.BlockContraction(C2, A, labels[0], B, labels[1], labels[2], mode="sequential")
    # the dense equivalent on the engine
    na, ns, nk, nl = bond.total, phys.total, kleg.total, lleg.total
    Ad = torch.from_numpy(A.to_dense().ravel(order="F")).cuda()
    Bd = torch.from_numpy(B.to_dense().ravel(order="F")).cuda()
    Cd = torch.zeros(na * ns * ns * na, dtype=torch.float64, device="cuda")
    sa, sb, sc = (na, ns, nk, nl), (nl, nk, ns, na), (na, ns, ns, na)
    dplan = qs.plan_contract(qs.StridedView(Cd, sc, colmajor_strides(sc), 0),
                             qs.StridedView(Ad, sa, colmajor_strides(sa), 0), labels[0],
                             qs.StridedView(Bd, sb, colmajor_strides(sb), 0), labels[1], labels[2])

    def timed(fn, steps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    steps = max(args.steps, 10)
    l0 = qs._abi.lib().qs_launch_count()
    ms_grouped = timed(lambda: bc.execute(1.0, 0.0), steps)
    launches = (qs._abi.lib().qs_launch_count() - l0) / (steps + args.warmup)
    ms_seq = timed(lambda: bseq.execute(1.0, 0.0), steps)
    ms_dense = timed(lambda: qs.execute(dplan, 1.0, 0.0), steps)
    torch.cuda.synchronize()
    dense_c = Cd.cpu().numpy().reshape(sc, order="F")
    got = C.to_dense()
    rel = float(np.linalg.norm(got - dense_c) / np.linalg.norm(dense_c))
    dense_flops = 2.0 * na * ns * ns * na * nk * nl
    print(json.dumps({
        "metric": "U(1) block-sparse contraction throughput (block-product TFLOP/s, Float64)",
        "value": bc.flops / (ms_grouped * 1e-3) / 1e12, "unit": "TFLOP/s", "n_gpus": 1, "steps": steps,
        "warmup": args.warmup, "ms_per_step": ms_grouped, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded N(0,1) blocks)",
        "config": {"workload": "u1net_two_site_Castb_Aaskl_Blktb", "bond": na, "phys": ns, "k": nk, "l": nl,
                   "products": bc.products, "waves": len(bc.waves), "block_flops": bc.flops,
                   "dense_flops": dense_flops},
        "modes_ms": {"grouped_waves": ms_grouped, "sequential_plans": ms_seq, "dense_engine": ms_dense},
        "gpu_launches_per_step": launches,
        "rel_err_vs_dense": rel,
    }), flush=True)
    bc.release()
    bseq.release()
    dplan.release()


def run_matmul(args):
    """The permuted matmul C[a,n,b] = sum_k A[a,k,b] * B[k,n] (a=96, k=128,
    b=32, n=80; alpha = 1, beta = 0; M = (a,b) is not contiguous in C), in
    Float64: microseconds per call for execute on a reused plan, the same
    replayed as a CUDA graph, and one-shot contract (plan, execute, release)
    with the workspace from the library's pool and from a device arena.
    Launch-latency bound (63 MFLOP).  Prints one JSON line."""
    import torch
    qs = load_engine()
    from oracle import oracle as orc
    a, k, b, n = 96, 128, 32, 80
    rng = np.random.default_rng(20261203)
    A_h = rng.standard_normal(a * k * b)
    B_h = rng.standard_normal(k * n)
    sa, sb, sc = (a, k, b), (k, n), (a, n, b)
    Ad, Bd = torch.from_numpy(A_h).cuda(), torch.from_numpy(B_h).cuda()
    Cd = torch.zeros(a * n * b, dtype=torch.float64, device="cuda")
    Av = qs.StridedView(Ad, sa, colmajor_strides(sa), 0)
    Bv = qs.StridedView(Bd, sb, colmajor_strides(sb), 0)
    Cv = qs.StridedView(Cd, sc, colmajor_strides(sc), 0)
    labels = ((1, 2, 3), (2, 4), (1, 4, 3))
    flops = 2.0 * a * b * n * k

    def timed(fn, steps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return 1e3 * e0.elapsed_time(e1) / steps, 1e6 * (time.perf_counter() - t0) / steps

    plan = qs.plan_contract(Cv, Av, labels[0], Bv, labels[1], labels[2])
    gplan = qs.plan_contract(Cv, Av, labels[0], Bv, labels[1], labels[2], cuda_graph=True)
    steps = max(args.steps, 200)
    res = {}
    res["execute_us"], res["execute_host_us"] = timed(lambda: qs.execute(plan, 1.0, 0.0), steps)
    res["graph_us"], res["graph_host_us"] = timed(lambda: qs.execute(gplan, 1.0, 0.0), steps)
    res["contract_us"], res["contract_host_us"] = timed(
        lambda: qs.contract(Cv, 1.0, Av, labels[0], Bv, labels[1], 0.0, labels[2]), max(args.steps, 50))
    # One-shot contract with the workspace from a device arena (no cudaMalloc,
    # no wait for the stream; checkpoint/reset around each call).
    arena = qs.DeviceArena(64 << 20)
    res["contract_arena_us"], res["contract_arena_host_us"] = timed(
        lambda: qs.contract(Cv, 1.0, Av, labels[0], Bv, labels[1], 0.0, labels[2], allocator=arena),
        max(args.steps, 50))
    res["arena_waits"] = arena.info()["waits"]
    qs.execute(plan, 1.0, 0.0)
    torch.cuda.synchronize()
    got = Cd.cpu().numpy()
    Ch = orc.HostView(np.zeros(a * n * b), sc, colmajor_strides(sc))
    orc.brute(Ch, 1.0, orc.HostView(A_h, sa, colmajor_strides(sa)), labels[0],
              orc.HostView(B_h, sb, colmajor_strides(sb)), labels[1], 0.0, labels[2],
              korder=list(plan.k_labels))
    t0 = time.perf_counter()
    reps = 0
    while time.perf_counter() - t0 < 2.0:
        Cn = orc.HostView(np.zeros(a * n * b), sc, colmajor_strides(sc))
        orc.nest_f64(Cn, 1.0, orc.HostView(A_h, sa, colmajor_strides(sa)), labels[0],
                     orc.HostView(B_h, sb, colmajor_strides(sb)), labels[1], 0.0, labels[2], threads=1)
        reps += 1
    cpu_us = 1e6 * (time.perf_counter() - t0) / reps
    print(json.dumps({
        "metric": "permuted matmul latency (Float64, us per execute on a reused plan)",
        "value": res["execute_us"], "unit": "us", "n_gpus": 1, "steps": steps, "warmup": args.warmup,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded N(0,1))",
        "config": {"workload": "matmul_a96_k128_b32_n80", "method": plan.method, "flops": flops},
        "tflops": flops / (res["execute_us"] * 1e-6) / 1e12, "modes_us": res,
        "bitwise_equal_to_oracle": bool(np.array_equal(got, Ch.parent)),
        "cpu_baseline": {"value": cpu_us, "unit": "us", "cores": 1, "kind": "port",
                         "sample": f"{reps} full runs of the oracle's nest restatement, 1 thread"},
    }), flush=True)
    plan.release()
    gplan.release()


def init_ranks(world: int, backend: str = "nccl", timeout_s: int = 120) -> None:
    """One process per GPU (torchrun sets RANK/WORLD_SIZE/MASTER_*); a short
    process-group timeout so ranks that wait for each other fail instead of
    hanging."""
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))


def max_over_ranks(x: float, world: int, device) -> float:
    """The slowest rank's value (the bench's whole-job time)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--method", default="auto", choices=["auto", "native", "ozaki", "bf16x3"])
    ap.add_argument("--dist", default="uniform", choices=["uniform", "wide"],
                    help="c1 inputs: uniform[-1,1], or that times 2^U (U in [-20,20]) per a-slice of A and "
                         "per d-slice of B")
    ap.add_argument("--c1-dtype", default="f64", choices=["f64", "f32"],
                    help="c1 element type (f32 runs the split-BF16x3 tensor-core method by default)")
    ap.add_argument("--per-product", action="store_true",
                    help="Ozaki: the one-product-per-stage GEMM kernel instead of grouped diagonals")
    ap.add_argument("--oz-single-sm", action="store_true",
                    help="Ozaki: the one-SM GEMM kernel instead of the CTA-pair (cta_group::2) kernel")
    ap.add_argument("--cpu-rows", type=int, default=M)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--cpu-threads", type=int, default=0, help="CPU arm threads (0: every host thread)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--profile", action="store_true",
                    help="profiling target: plan, one warm-up execute, --steps executes, exit")
    ap.add_argument("--workload", default="permuted4",
                    choices=["permuted4", "blocks", "serving", "mps", "matmul", "u1net"],
                    help="blocks: 2000 uneven U(1) blocks, grouped vs graph vs plain launches")
    ap.add_argument("--blocks", type=int, default=2000)
    ap.add_argument("--modes", default="all",
                    help="blocks: comma list of plain,plain_graph,grouped,grouped_graph (or all)")
    ap.add_argument("--breakdown", action="store_true",
                    help="blocks: also time each method's plans as their own grouped launch")
    ap.add_argument("--dtypes", default="f64,f32")
    ap.add_argument("--rates", default="100,1000,10000,100000", help="serving: Poisson arrival rates (1/s)")
    ap.add_argument("--requests", type=int, default=300, help="serving: requests per rate")
    ap.add_argument("--budget-gb", type=float, default=120.0, help="serving: HBM admission budget")
    ap.add_argument("--arena-gb", type=float, default=64.0, help="serving: device arena for request buffers")
    ap.add_argument("--host-arena-gb", type=float, default=24.0, help="serving: pinned host arena")
    ap.add_argument("--tick-flops", type=float, default=2e11, help="serving: work per tick (flops)")
    ap.add_argument("--block-cap", type=int, default=1 << 21,
                    help="max |A|+|B|+|C| elements per block")
    ap.add_argument("--peaks", action="store_true",
                    help="measure cuBLAS int8 (torch._int_mm) and fp64 GEMM throughput, print JSON")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.peaks:
        measure_library_peaks()
        return
    if args.profile:
        run_profile_target(args)
        return
    if args.workload == "blocks":
        run_blocks(args)
        return
    if args.workload == "serving":
        run_serving(args)
        return
    if args.workload == "mps":
        run_mps(args)
        return
    if args.workload == "matmul":
        run_matmul(args)
        return
    if args.workload == "u1net":
        run_u1net(args)
        return

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    init_ranks(world, "nccl")
    qs = load_engine()
    dev = torch.device("cuda", local)

    A_h, B_h, C_h = host_inputs(seed=20261203 + rank, wide=args.dist == "wide")
    f32 = args.c1_dtype == "f32"
    if f32:
        # Float32 operands; the accuracy reference is FP64 on the same values.
        A_h, B_h, C_h = (x.astype(np.float32) for x in (A_h, B_h, C_h))
    esize = A_h.itemsize
    sa, sb, sc = shapes()
    Ad = torch.from_numpy(A_h).to(dev)
    Bd = torch.from_numpy(B_h).to(dev)
    C0d = torch.from_numpy(C_h).to(dev)
    Cd = C0d.clone()
    Av = qs.StridedView(Ad, sa, colmajor_strides(sa), 0)
    Bv = qs.StridedView(Bd, sb, colmajor_strides(sb), 0)
    Cv = qs.StridedView(Cd, sc, colmajor_strides(sc), 0)
    plan = qs.plan_contract(Cv, Av, LABELS["indA"], Bv, LABELS["indB"], LABELS["indC"], method=args.method,
                            per_product_gemm=args.per_product, oz_single_sm=args.oz_single_sm)

    # Accuracy of the measured path: one execution from the seeded C, every
    # element against the FP64 oracle, and a binary128 sample spread over
    # all of C (outside the timed region).
    from oracle import oracle as orc
    qs.execute(plan, ALPHA, BETA)
    torch.cuda.synchronize()
    acc = c1_accuracy(orc, Cd.cpu().numpy(), A_h, B_h, C_h)

    stream = torch.cuda.current_stream()
    # warm-up (untimed)
    for _ in range(args.warmup):
        qs.execute(plan, ALPHA, BETA)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = qs._abi.lib().qs_launch_count()
    qs.profile(plan, True)  # CUDA events between the plan's launches
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        t_start = time.perf_counter()
        ev0.record(stream)
        for _ in range(args.steps):
            qs.execute(plan, ALPHA, BETA)
        ev1.record(stream)
        torch.cuda.synchronize()
        launches = qs._abi.lib().qs_launch_count() - launches0
        # The sampler polls every 100 ms: keep the same load on the GPU (untimed)
        # until at least 1.5 s of samples exist.
        while time.perf_counter() - t_start < 1.5:
            for _ in range(10):
                qs.execute(plan, ALPHA, BETA)
            torch.cuda.synchronize()
    stage_ms, nexec = qs.stage_times(plan)
    qs.profile(plan, False)
    ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, world, dev)
    if world > 1:
        dist.barrier()
    value = world * FLOPS / (ms * 1e-3) / 1e12

    # Dominant kernel's own duration: the plan's GEMM stage, timed alone.
    roof, stages = roofline(plan, stage_ms, nexec)

    # End to end through the public API with host buffers: every step copies
    # its A, B and C from pinned host memory and its C back.  Steps are
    # pipelined the way a caller streaming contractions would run them: two
    # device buffer sets (a plan on each), uploads on one stream, executes on
    # a second, downloads on a third, so step i+1's upload overlaps step i's
    # execute and download.
    A_p = torch.from_numpy(A_h).pin_memory()
    B_p = torch.from_numpy(B_h).pin_memory()
    C_p = torch.from_numpy(C_h).pin_memory()
    outs = [torch.empty_like(C_p).pin_memory() for _ in range(2)]
    h2d = (A_p.numel() + B_p.numel() + C_p.numel()) * esize
    d2h = outs[0].numel() * esize
    A1d, B1d, C1d = torch.empty_like(Ad), torch.empty_like(Bd), torch.empty_like(Cd)
    plan1 = qs.plan_contract(qs.StridedView(C1d, sc, colmajor_strides(sc), 0), qs.StridedView(A1d, sa, colmajor_strides(sa), 0),
                             LABELS["indA"], qs.StridedView(B1d, sb, colmajor_strides(sb), 0), LABELS["indB"],
                             LABELS["indC"], method=args.method, per_product_gemm=args.per_product,
                             oz_single_sm=args.oz_single_sm)
    bufs = [(Ad, Bd, Cd, plan), (A1d, B1d, C1d, plan1)]
    s_in, s_run, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_run = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]

    def e2e_step(i):
        a_d, b_d, c_d, p = bufs[i % 2]
        if i >= 2:
            s_in.wait_event(ev_out[i % 2])   # buffer set free: step i-2 fully done
        with torch.cuda.stream(s_in):
            a_d.copy_(A_p, non_blocking=True)
            b_d.copy_(B_p, non_blocking=True)
            c_d.copy_(C_p, non_blocking=True)
            ev_in[i % 2].record(s_in)
        s_run.wait_event(ev_in[i % 2])
        qs.execute(p, ALPHA, BETA, stream=s_run)
        ev_run[i % 2].record(s_run)
        s_out.wait_event(ev_run[i % 2])
        with torch.cuda.stream(s_out):
            outs[i % 2].copy_(c_d, non_blocking=True)
            ev_out[i % 2].record(s_out)

    for i in range(2):
        e2e_step(i)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s_in)
    s_run.wait_event(e0)
    s_out.wait_event(e0)
    for i in range(args.e2e_steps):
        e2e_step(i)
    e1.record(s_out)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.e2e_steps, world, dev)
    e2e_value = world * FLOPS / (e2e_ms * 1e-3) / 1e12
    plan1.release()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and not f32:
        # Passes over args.cpu_rows rows of M until at least args.cpu_seconds
        # of CPU work (at most 16 passes); the median rate is reported.
        rates, total = [], 0.0
        threads = args.cpu_threads or orc.max_threads()
        while total < args.cpu_seconds and len(rates) < 16:
            v, dt = cpu_sample(orc, A_h, B_h, C_h, args.cpu_rows, threads)
            rates.append(v)
            total += dt
        cpu = {"value": statistics.median(rates), "unit": "TFLOP/s", "cores": threads, "kind": "port",
               "sample": f"{len(rates)} passes of {args.cpu_rows} of {M} rows of M (all N, all K) through the "
                         f"oracle's nest restatement, {total:.1f} s in total, median pass rate",
               "host": host_cpu()}

    if rank == 0:
        print(json.dumps({
            "metric": ("contraction TFLOP/s (Float32, rel.err<=1e-5 vs FP64)" if f32 else
                       "contraction TFLOP/s (Float64, rel.err<=1e-13 vs FP64)"),
            "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": args.c1_dtype,
            "data": ("synthetic (seeded uniform[-1,1] A/B" +
                     (" x 2^U per a-slice of A and d-slice of B, U in [-20,20]" if args.dist == "wide" else "") +
                     ", N(0,1) C)"),
            "config": {"workload": WORKLOAD, "M": M, "N": N, "K": K, "alpha": ALPHA, "beta": BETA,
                       "method": plan.method, "ozaki_slices": plan.ozaki_slices,
                       "dist": args.dist,
                       "l2": f"inputs larger than L2 ({419 if not f32 else 210} MB), no flush",
                       "parallelism": f"replicas{world}"},
            "rel_err": acc["rel_err"], "rel_err_elements": acc["elements"],
            "rel_err_binary128_sample": acc["rel_err_binary128"], "binary128_sample": acc["sample"],
            "roofline": roof, "stages_ms": stages,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "TFLOP/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms, "steps": args.e2e_steps,
                    "pipelined": "uploads, executes and downloads on three streams, two buffer sets"},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }), flush=True)
    plan.release()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
