"""Benchmark: FP64 strided-batch tridiagonal solves on a 256^3 cube.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = three solves of the 256^3 FP64 cube (65,536 systems of n=256),
along solvedim 0, 1 and 2 in turn (tridDmtsvStridedBatch through the C ABI),
on inputs resident in HBM.  Inputs: a_i, c_i ~ U(-1,1), b_i = |a_i|+|c_i|+U(1,2),
d ~ N(0,1), seeded (synthetic stand-in for the workload's distribution).

Metric: solve GB/s = algorithmic bytes (read a,b,c,d + write x = 40 B per
unknown) / time, whole job (all ranks).  Each array is 134 MB, so every launch
streams 671 MB (> 126 MB L2): no L2 flush is needed between steps.

Extra keys: roofline (dominant kernel vs the measured HBM copy bandwidth),
cpu_baseline (the reference CPU solver compiled from the reference sources,
all host threads, on the same cube), e2e (the same solves through the C ABI
from pinned host buffers, host<->device copies inside the timed region),
clocks (nvidia-smi samples during the timed region), gpu_launches,
differentiation (16,384 x 1024 FP64: forward, forward + adjoint in one call
and autograd forward + backward, times and their ratio to the forward solve,
gradient error against central finite differences; rank 0 at N=1).

--suite: one JSON line per other workload (FP32 cube, complex and
FP32-storage / FP64-arithmetic cubes, long systems,
variable-length batch, block systems, ADI steps and the ADI gradient);
--scale f runs the batched workloads with a fraction f of their systems.

--impl reference: times the reference's own CPU implementation of the path
(scalar/src/cpu/trid_cpu.cpp built into oracle/_ref) on the same workload
with every host thread; with N>1 only rank 0 runs it.
"""

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

N = 256
DIMS = [N, N, N]
BYTES_PER_UNKNOWN = 5 * 8          # read a,b,c,d + write x (FP64)
UNKNOWNS = N * N * N
BYTES_PER_SOLVE = BYTES_PER_UNKNOWN * UNKNOWNS
METRIC = "Solve GB/s (% of B200 HBM peak); fwd+adjoint vs fwd-only time at <=1e-8 grad err"
WORKLOAD = "FP64 256^3 strided-batch solves along solvedim 0,1,2 (65,536 systems of n=256 each)"
FALLBACK_HBM = 6650.0


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM, "fallback"


def make_inputs(seed=1234):
    rng = np.random.default_rng(seed)
    a = rng.uniform(-1, 1, UNKNOWNS)
    c = rng.uniform(-1, 1, UNKNOWNS)
    b = np.abs(a) + np.abs(c) + rng.uniform(1, 2, UNKNOWNS)
    d = rng.standard_normal(UNKNOWNS)
    return a, b, c, d


class ClockSampler:
    """nvidia-smi samples (200 ms) while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


def read_traffic():
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu
    summary (profiles/dram_traffic_256cube_fp64.txt: 'solvedim <k> <bytes>')."""
    path = os.path.join(ROOT, "profiles", "dram_traffic_256cube_fp64.txt")
    out = {}
    try:
        with open(path) as f:
            for line in f:
                p = line.split()
                if len(p) == 3 and p[0] == "solvedim":
                    out[int(p[1])] = float(p[2])
    except OSError:
        pass
    return out


def cpu_baseline_ref(a, b, c, d, reps=2):
    """The reference CPU solver (oracle/_ref) on the full cube, all threads."""
    import ctypes

    from oracle import oracle

    lib = oracle.ref_lib()
    f = lib.tridDmtsvStridedBatch
    f.restype = ctypes.c_int
    dims = (ctypes.c_int * 3)(*DIMS)
    best = None
    placed = {}
    for aligned in (False, True):
        placed[aligned] = [oracle._placed(x, aligned) for x in (a, b, c, d)]
    for _ in range(reps + 1):
        t0 = time.perf_counter()
        for sd in range(3):
            arrs = placed[sd > 0]
            st = f(*[x.ctypes.data_as(ctypes.c_void_p) for x in arrs], None, 3, sd, dims, dims)
            assert st == 0
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    return best


def run_ours(args):
    import torch

    import tridsolver_b200 as tb
    from tridsolver_b200.shard import max_over_ranks

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    a, b, c, d0 = make_inputs(1234 + rank)
    ta, tb_, tc, td = (torch.from_numpy(x).cuda() for x in (a, b, c, d0))
    stream = torch.cuda.current_stream()

    def step():
        for sd in range(3):
            st = tb.tridDmtsvStridedBatch(ta, tb_, tc, td, None, 3, sd, DIMS, DIMS)
            if st != 0:
                raise tb.TridError(st, "tridDmtsvStridedBatch")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # per-launch timing of each axis on the launching stream: K launches of
    # one axis back to back between two events (671 MB per launch > L2)
    per_axis = [0.0, 0.0, 0.0]
    for sd in range(3):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            st = tb.tridDmtsvStridedBatch(ta, tb_, tc, td, None, 3, sd, DIMS, DIMS)
            if st != 0:
                raise tb.TridError(st, "tridDmtsvStridedBatch")
        e1.record(stream)
        torch.cuda.synchronize()
        per_axis[sd] = e0.elapsed_time(e1) / args.steps
    # whole-step timing (the reported value)
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    cvd = [x for x in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if x.strip()]
    gpu_index = cvd[local] if local < len(cvd) else str(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(gpu_index) as clk:
        t_wall = time.time()
        start.record(stream)
        for _ in range(args.steps):
            step()
        stop.record(stream)
        torch.cuda.synchronize()
        # short timed regions get the same load continued (untimed) so that the
        # 200 ms clock samples see it
        while time.time() < t_wall + 1.2:
            step()
            torch.cuda.synchronize()
    ms_total = max_over_ranks(start.elapsed_time(stop))
    if dist:
        dist.barrier()
    ms_step = ms_total / args.steps
    value = world * 3 * BYTES_PER_SOLVE / (ms_step * 1e-3) / 1e9

    # end to end through the C ABI from pinned host buffers
    e2e_steps = max(1, min(args.steps, 5))
    ha, hb, hc, hd = (torch.from_numpy(x).pin_memory() for x in (a, b, c, d0))
    hout = torch.empty_like(hd).pin_memory()
    for _ in range(2):
        for h, t in ((ha, ta), (hb, tb_), (hc, tc), (hd, td)):
            t.copy_(h, non_blocking=True)
        step()
        hout.copy_(td, non_blocking=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        for h, t in ((ha, ta), (hb, tb_), (hc, tc), (hd, td)):
            t.copy_(h, non_blocking=True)
        step()
        hout.copy_(td, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1)) / e2e_steps
    e2e_value = world * 3 * BYTES_PER_SOLVE / (e2e_ms * 1e-3) / 1e9

    peak, peak_kind = measured_peak()
    dom = int(np.argmax(per_axis))
    achieved = BYTES_PER_SOLVE / (per_axis[dom] * 1e-3) / 1e9
    traffic = read_traffic().get(dom)
    result = {
        "metric": METRIC,
        "value": round(value, 2),
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_step, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded U/N distributions of the workload)",
        "config": {"workload": WORKLOAD, "dims": DIMS, "solves_per_step": 3,
                   "bytes_per_solve": BYTES_PER_SOLVE, "l2": "inputs 671 MB/launch > 126 MB L2, no flush",
                   "parallelism": f"replicas{world}", "hbm_fraction_of_" + peak_kind: round(value / world / peak, 4),
                   "per_axis_ms": [round(x, 5) for x in per_axis],
                   "per_axis_gbs": [round(BYTES_PER_SOLVE / (x * 1e-3) / 1e9, 1) for x in per_axis]},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                     "kernel": f"solvedim {dom}",
                     "traffic": traffic, "algorithmic_bytes": BYTES_PER_SOLVE},
        "e2e": {"value": round(e2e_value, 2), "unit": "GB/s",
                "h2d_bytes_per_step": 4 * UNKNOWNS * 8, "d2h_bytes_per_step": UNKNOWNS * 8},
        "gpu_launches": 3 * args.steps,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1:
        result["differentiation"] = measure_differentiation(torch, tb, max(3, min(args.steps, 20)))
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline_entry(a, b, c, d0)
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result))


def measure_differentiation(torch, tb, steps, seed=99):
    """The differentiation workload: 16,384 FP64 systems of n=1024 along the
    unit-stride axis, loss = sum(w * x) with w ~ N(0,1).  Times the plain
    forward solve, the forward + adjoint in one call
    (tridDmtsvStridedBatchFwdAdj: x and the gradients w.r.t. a, b, c, d) and
    the autograd path (trid_solve forward + backward), and checks the
    gradients against central finite differences (h = 1e-6) on 64 sampled
    entries (16 of each of a, b, c, d).  Every array is 134 MB (> L2), so no flush between launches."""
    S, n = 16384, 1024
    gen = torch.Generator(device="cuda").manual_seed(seed)
    a = torch.rand(S, n, dtype=torch.float64, device="cuda", generator=gen) * 2 - 1
    c = torch.rand(S, n, dtype=torch.float64, device="cuda", generator=gen) * 2 - 1
    b = a.abs() + c.abs() + 1 + torch.rand(S, n, dtype=torch.float64, device="cuda", generator=gen)
    d = torch.randn(S, n, dtype=torch.float64, device="cuda", generator=gen)
    w = torch.randn(S, n, dtype=torch.float64, device="cuda", generator=gen)
    dims = [n, S]
    xs = d.clone()
    x = torch.empty_like(d)
    grads = [torch.empty_like(d) for _ in range(4)]
    leaves = [t.clone().requires_grad_(True) for t in (a, b, c, d)]

    def fwd():
        st = tb.tridDmtsvStridedBatch(a, b, c, xs, None, 2, 0, dims, dims)
        if st != 0:
            raise tb.TridError(st, "tridDmtsvStridedBatch")

    def fused():
        st = tb.tridDmtsvStridedBatchFwdAdj(a, b, c, d, w, x, *grads, 2, 0, dims, dims)
        if st != 0:
            raise tb.TridError(st, "tridDmtsvStridedBatchFwdAdj")

    def autograd():
        for t in leaves:
            t.grad = None
        u = tb.trid_solve(*leaves)
        u.backward(w)

    stream = torch.cuda.current_stream()
    times = {}
    for name, fn in (("fwd", fwd), ("fused", fused), ("autograd", autograd)):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        times[name] = e0.elapsed_time(e1) / steps
    fused()
    torch.cuda.synchronize()
    # central finite differences on one system per sample (h = 1e-6)
    rng = np.random.default_rng(seed)
    h = 1e-6
    errs, gmax = [], 0.0
    coefs = (a, b, c, d)
    for k in range(64):
        which, s_, i = k % 4, int(rng.integers(S)), int(rng.integers(1, n - 1))
        rows = [t[s_:s_ + 1].clone() for t in coefs]
        vals = []
        for sign in (1, -1):
            r = [t.clone() for t in rows]
            r[which][0, i] += sign * h
            tb.tridDmtsvStridedBatch(r[0], r[1], r[2], r[3], None, 2, 0, [n, 1], [n, 1])
            vals.append(float((r[3][0] * w[s_]).sum()))
        fd = (vals[0] - vals[1]) / (2 * h)
        g = float(grads[which][s_, i])
        errs.append(abs(fd - g))
        gmax = max(gmax, abs(g))
    unknowns = S * n
    return {
        "workload": "16,384 FP64 systems of n=1024 (unit stride), loss = sum(w*x), w ~ N(0,1)",
        "fwd_ms": round(times["fwd"], 5),
        "fwd_adj_ms": round(times["fused"], 5),
        "autograd_fwd_bwd_ms": round(times["autograd"], 5),
        "fwd_gbs": round(40 * unknowns / (times["fwd"] * 1e-3) / 1e9, 1),
        "fwd_adj_gbs": round(80 * unknowns / (times["fused"] * 1e-3) / 1e9, 1),
        "ratio_fwd_adj_over_fwd": round(times["fused"] / times["fwd"], 3),
        "ratio_autograd_over_fwd": round(times["autograd"] / times["fwd"], 3),
        "target_ratio": 2.2,
        "grad_err_vs_fd": float(f"{max(errs) / max(1.0, gmax):.3e}"),
        "fd": "central, h=1e-6, 64 sampled entries of a, b, c, d; error relative to max(1, max|g|)",
        "bytes_per_unknown": {"fwd": 40, "fwd_adj": 80, "autograd": "40 + 16 (copy of d) + 72"},
    }


def cpu_baseline_entry(a, b, c, d):
    from oracle import oracle

    threads = os.cpu_count()
    if oracle.ref_available():
        sec = cpu_baseline_ref(a, b, c, d)
        kind = "reference"
        sample = "full 256^3 cube, solvedim 0,1,2 once each, best of 2 after one warm-up"
    else:
        sec = None
        kind = "port"
        sample = "reference CPU build missing"
    return {"value": round(3 * BYTES_PER_SOLVE / sec / 1e9, 3) if sec else None, "unit": "GB/s",
            "cores": threads, "kind": kind, "sample": sample,
            "ms_per_step": round(sec * 1e3, 2) if sec else None}


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return
    from oracle import oracle

    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built"}))
        return
    import ctypes

    a, b, c, d = make_inputs(1234)
    lib = oracle.ref_lib()
    f = lib.tridDmtsvStridedBatch
    f.restype = ctypes.c_int
    dims = (ctypes.c_int * 3)(*DIMS)
    placed = {al: [oracle._placed(x, al) for x in (a, b, c, d)] for al in (False, True)}

    def step():
        for sd in range(3):
            arrs = placed[sd > 0]
            f(*[x.ctypes.data_as(ctypes.c_void_p) for x in arrs], None, 3, sd, dims, dims)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    sec = (time.perf_counter() - t0) / args.steps
    value = 3 * BYTES_PER_SOLVE / sec / 1e9
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count()))
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "GB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(sec * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD, "dims": DIMS, "solves_per_step": 3,
                   "implementation": "reference scalar/src/cpu/trid_cpu.cpp (OpenMP), "
                                     "solvedim 0 via its scalar path"},
        "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": threads,
                         "kind": "reference", "sample": "full 256^3 cube per step"},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }))


def run_suite(args):
    """The other workloads of the path, one JSON line each (GPU, N=1):
    FP32 cube per axis, long systems, variable-length batch, block systems
    (forward and adjoint), ADI steps (eager and CUDA graph) and the
    checkpointed ADI gradient.  Algorithmic bytes per workload are stated in
    each line; inputs are seeded synthetic data of the workload's shapes and
    distributions; every timing is CUDA events around K launches after 2
    warm-up launches, inputs larger than L2 unless stated."""
    import torch

    import tridsolver_b200 as tb
    from tridsolver_b200.adi import ADI
    from tridsolver_b200.block import btsv, btsv_adjoint
    from tridsolver_b200.varlen import solve_varlen

    peak, peak_kind = measured_peak()
    K = max(3, min(args.steps, 10))
    dev = torch.device("cuda")
    gen = torch.Generator(device="cuda").manual_seed(2024)

    def timed(fn, reps=K):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def emit(d):
        d["peak_gbs_" + peak_kind] = peak
        if "gbs" in d:
            d["frac_of_" + peak_kind] = round(d["gbs"] / peak, 4)
        print(json.dumps(d), flush=True)

    def coeffs(shape, dtype):
        a = torch.rand(shape, dtype=dtype, device=dev, generator=gen) * 2 - 1
        c = torch.rand(shape, dtype=dtype, device=dev, generator=gen) * 2 - 1
        b = a.abs() + c.abs() + 1 + torch.rand(shape, dtype=dtype, device=dev, generator=gen)
        d = torch.randn(shape, dtype=dtype, device=dev, generator=gen)
        return a, b, c, d

    def want(name):
        return args.only is None or args.only in name

    # FP32 256^3, each axis (20 B per unknown)
    if want("FP32 256^3"):
        a, b, c, d = coeffs((UNKNOWNS,), torch.float32)
        for sd in range(3):
            ms = timed(lambda: tb.tridSmtsvStridedBatch(a, b, c, d, None, 3, sd, DIMS, DIMS))
            emit({"workload": f"FP32 256^3 solvedim {sd}", "ms": round(ms, 5),
                  "gbs": round(20 * UNKNOWNS / (ms * 1e-3) / 1e9, 1)})
        del a, b, c, d

    # complex128 / complex64 256^3 (5 elements of 16 / 8 B per unknown) and
    # FP32 storage with FP64 arithmetic (20 B per unknown), each axis
    def ccoeffs(shape, dtype):
        rdt = torch.float64 if dtype == torch.complex128 else torch.float32
        r = lambda: torch.rand(shape, dtype=rdt, device=dev, generator=gen) * 2 - 1
        a, c = torch.complex(r(), r()), torch.complex(r(), r())
        mod = a.abs() + c.abs() + 1.5 + 0.5 * r()
        b = torch.polar(mod, torch.pi * r())
        d = torch.complex(torch.randn(shape, dtype=rdt, device=dev, generator=gen),
                          torch.randn(shape, dtype=rdt, device=dev, generator=gen))
        return a, b, c, d

    for name, dtype, fn, bpu in (("complex128", torch.complex128, tb.tridZmtsvStridedBatch, 80),
                                 ("complex64", torch.complex64, tb.tridCmtsvStridedBatch, 40),
                                 ("FP32 storage / FP64 arithmetic", torch.float32,
                                  tb.tridSmtsvStridedBatchMixed, 20)):
        if not want(name):
            continue
        a, b, c, d = (ccoeffs((UNKNOWNS,), dtype) if dtype.is_complex
                      else coeffs((UNKNOWNS,), dtype))
        for sd in range(3):
            ms = timed(lambda: fn(a, b, c, d, None, 3, sd, DIMS, DIMS))
            emit({"workload": f"{name} 256^3 solvedim {sd}", "ms": round(ms, 5),
                  "gbs": round(bpu * UNKNOWNS / (ms * 1e-3) / 1e9, 1)})
        del a, b, c, d
    if args.only is not None:  # the remaining workloads are not selectable
        return

    sc = args.scale  # fraction of each workload's systems (1 = the configured sizes)
    assert 0 < sc <= 1, "--scale in (0, 1]"

    # long systems: 2048 x n=65,536 FP64 along axis 0
    n, S = 65536, max(1, int(2048 * sc))
    a, b, c, d = coeffs((S * n,), torch.float64)
    ms = timed(lambda: tb.tridDmtsvStridedBatch(a, b, c, d, None, 2, 0, [n, S], [n, S]))
    emit({"workload": f"FP64 {S} systems of n=65,536 (axis 0, blocked partition)",
          "ms": round(ms, 4), "gbs": round(40 * n * S / (ms * 1e-3) / 1e9, 1),
          "bytes_per_unknown": {"algorithmic": 40, "moved": "72 + block systems (a, b, c, d read "
                                "twice: block reduction, then block finish)"}})
    del a, b, c, d

    # variable-length batch: 200,000 systems, lengths floor(exp(U(ln 8, ln 8192)))
    rng = np.random.default_rng(7)
    nvar = max(1, int(200000 * sc))
    lens = np.floor(np.exp(rng.uniform(np.log(8), np.log(8192), nvar))).astype(np.int64)
    off = torch.from_numpy(np.concatenate([[0], np.cumsum(lens)])).to(dev)
    total = int(lens.sum())
    a, b, c, d = coeffs((total,), torch.float64)
    ms = timed(lambda: solve_varlen(a, b, c, d, off, total))
    emit({"workload": f"FP64 variable-length batch, {nvar} systems, n ~ logU[8, 8192]",
          "unknowns": total, "ms": round(ms, 4),
          "gbs": round((40 * total + 8 * (len(lens) + 1)) / (ms * 1e-3) / 1e9, 1)})
    del a, b, c, d, off

    # systems split along the solve dimension: 256^3 FP64 along z cut into P
    # slabs, every "rank" run in turn on this one GPU (reduce of every slab,
    # the stacked numbers standing in for the all-gather, finish of every
    # slab); per-rank time on P GPUs ~ total / P plus the exchange
    import ctypes as _ct

    from tridsolver_b200 import _lib as _tl

    a, b, c, d = coeffs((UNKNOWNS,), torch.float64)
    Ls = tb.lib()
    plane = DIMS[0] * DIMS[1]
    nsys_z = plane

    def split_step(P):
        m = DIMS[2] // P
        loc, pads = _tl.int_array([DIMS[0], DIMS[1], m]), _tl.int_array(DIMS)
        bn = torch.empty((P, 6, nsys_z), dtype=torch.float64, device=dev)
        v = lambda t: _ct.c_void_p(t.data_ptr())
        for r in range(P):
            o = r * m * plane
            st = Ls.tridDmtsvStridedBatchSplitReduce(v(a[o:]), v(b[o:]), v(c[o:]), v(d[o:]), 3, 2,
                                                     loc, pads, v(bn[r]))
            assert st == 0
        for r in range(P):
            o = r * m * plane
            st = Ls.tridDmtsvStridedBatchSplitFinish(v(a[o:]), v(b[o:]), v(c[o:]), v(d[o:]), None,
                                                     3, 2, loc, pads, v(bn), P, r, 0)
            assert st == 0

    tb.scalar._bind_stream(Ls)
    ms1 = timed(lambda: tb.tridDmtsvStridedBatch(a, b, c, d, None, 3, 2, DIMS, DIMS))
    for P in (2, 4):
        ms = timed(lambda: split_step(P))
        emit({"workload": f"FP64 256^3 along z split into {P} slabs (ranks emulated on one GPU)",
              "ms_all_slabs": round(ms, 4), "ms_unsplit": round(ms1, 4),
              "ms_per_rank_estimate": round(ms / P, 4),
              "gbs_all_slabs": round(40 * UNKNOWNS / (ms * 1e-3) / 1e9, 1),
              "bytes_per_unknown": "72 (slab reduce 32 + patched local solve 40), plus 48 B per "
                                   "system and rank exchanged"})
    del a, b, c, d

    # block tridiagonal: M in {2, 4, 8}, N=256, P=32,768 (interleaved layout)
    for M in (2, 4, 8):
        N, P = 256, max(1, int(32768 * sc))
        A = (torch.rand((N, P, M, M), dtype=torch.float64, device=dev, generator=gen) * 2 - 1) / M
        C = (torch.rand((N, P, M, M), dtype=torch.float64, device=dev, generator=gen) * 2 - 1) / M
        B = (torch.rand((N, P, M, M), dtype=torch.float64, device=dev, generator=gen) * 2 - 1) / M
        B += (2 + torch.rand((N, P, 1, 1), dtype=torch.float64, device=dev, generator=gen)) * \
            torch.eye(M, dtype=torch.float64, device=dev)
        dv = torch.randn((N, P, M), dtype=torch.float64, device=dev, generator=gen)
        x = torch.empty_like(dv)
        ms = timed(lambda: btsv(A, B, C, dv, x))
        rows = N * P
        fwd_b = (3 * M * M + 2 * M) * 8 * rows
        emit({"workload": f"FP64 block tridiagonal M={M}, N=256, P={P}: forward",
              "ms": round(ms, 4), "gbs": round(fwd_b / (ms * 1e-3) / 1e9, 1),
              "bytes_per_block_row": (3 * M * M + 2 * M) * 8})
        w = torch.randn_like(dv)
        msa = timed(lambda: btsv_adjoint(A, B, C, x, w))
        adj_b = (6 * M * M + 3 * M) * 8 * rows
        emit({"workload": f"FP64 block tridiagonal M={M}, N=256, P={P}: adjoint",
              "ms": round(msa, 4), "gbs": round(adj_b / (msa * 1e-3) / 1e9, 1),
              "bytes_per_block_row": (6 * M * M + 3 * M) * 8})
        del A, B, C, dv, x, w
        torch.cuda.empty_cache()

    # ADI heat diffusion: 128^3 x 100 steps, eager and CUDA graph; 64^3 x 10
    for shape, steps in (((128, 128, 128), 100), ((64, 64, 64), 10)):
        u = torch.rand(shape, dtype=torch.float64, device=dev, generator=gen)
        adi = ADI(shape, 1.0)
        ms_e = timed(lambda: adi.step(u, steps), reps=2)
        adi.run(u, 2, graph=True)
        ms_g = timed(lambda: adi.run(u, steps, graph=True), reps=2)
        elems = int(np.prod(shape))
        emit({"workload": f"FP64 ADI {shape[0]}^3 x {steps} steps (lambda=1)",
              "ms_eager": round(ms_e, 3), "ms_graph": round(ms_g, 3),
              "us_per_step_graph": round(1e3 * ms_g / steps, 2),
              "gbs": round(56 * elems * steps / (ms_g * 1e-3) / 1e9, 1),
              "bytes_per_element_step": "56: x solve with the stencil fused (read u, write "
                                        "du1), y solve (du1 -> du2), z solve adding into u"})
        del u, adi

    # checkpointed adjoint of ||u_200|| at 128^3 w.r.t. u0 and lambda
    shape = (128, 128, 128)
    u0 = torch.rand(shape, dtype=torch.float64, device=dev, generator=gen)
    adi = ADI(shape, 1.0)
    # warm-up at full size: the caching allocator then holds the run's
    # temporaries (after the multi-GB block workloads its pool is otherwise
    # shaped by them, and the timed run spends its time in cudaMalloc)
    torch.cuda.empty_cache()
    adi.grad_final_norm(u0, 200, 20)
    torch.cuda.synchronize()
    torch.cuda.reset_peak_memory_stats()
    base = torch.cuda.memory_allocated()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    loss, du0, dlam = adi.grad_final_norm(u0, 200, 20)
    e1.record()
    torch.cuda.synchronize()
    emit({"workload": "FP64 ADI 128^3 x 200 steps: d||u_200|| / d(u0, lambda), checkpoints "
                      "every 20 steps", "ms": round(e0.elapsed_time(e1), 2),
          "peak_extra_mib": round((torch.cuda.max_memory_allocated() - base) / 2**20, 1),
          "loss": float(loss), "dloss_dlambda": float(dlam)})


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--suite", action="store_true",
                    help="instead: one JSON line per other workload of the path (1 GPU)")
    ap.add_argument("--only", default=None,
                    help="--suite: run only the cube workloads whose name contains this "
                         "(e.g. 'complex128', 'FP32 storage')")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="--suite: fraction of each workload's systems (profiling runs)")
    args = ap.parse_args()
    if args.suite:
        run_suite(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        os.environ.setdefault("OMP_STACKSIZE", "64M")
        os.environ.setdefault("OMP_PROC_BIND", "close")
        run_reference(args)
    else:
        os.environ.setdefault("OMP_STACKSIZE", "64M")
        run_ours(args)


if __name__ == "__main__":
    main()
