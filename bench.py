"""Benchmark of the batched tridiagonal solve on B200.

Workload (one step): the 512^3 FP64 grid solved along x, then y, then z with
tridDmtsvStridedBatch, d overwritten by each solve (the order of the ADI
heat solver, apps/adi/src/adi_cuda.cu:294-323); 3 * 512^3 elements per step.
Inputs are seeded synthetic data with the distribution the configs name
(a, c ~ U(-0.5, 0.5), b = 1 + |a| + |c| + U(0, 1), d ~ N(0, 1)); every array
(1 GiB) is larger than L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

`value` is device throughput with inputs resident in HBM; `e2e` is the same
metric through the C ABI with host arrays (pinned host -> device copies of
a, b, c, d and the device -> host copy of the result inside the timed
region). `cpu_baseline` times the reference's own CPU library (oracle/_ref)
on the host cores on the same full grid, and `reference_gpu` the reference's
own CUDA library (oracle/_ref, built for sm_100a) on the same B200: the two
baseline legs, the only code here that runs anything under oracle/. With
--impl reference only the CPU timing runs, as the reference arm.

Multi-GPU: one process per GPU (torchrun); the solve shards by systems with
no exchange, so every rank solves its own grid (weak scaling) and value is
the sum over ranks / the max over ranks of the timed region.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

# The reference CPU library keeps 2*N_MAX SIMD vectors on each OpenMP
# worker's stack; set before any OpenMP runtime starts.
os.environ.setdefault("OMP_STACKSIZE", "32M")

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "elements/s & HBM GB/s (x/y/z, 512^3 FP64); FP32+refine vs FP64 at 1e-12"
UNIT = "elements/s"
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=512, help="grid edge (512 = the benchmark)")
    ap.add_argument("--dtype", default="f64", choices=["f64", "f32"])
    ap.add_argument("--only-config", default=None,
                    choices=["sweep", "adi", "adi_f32", "precision", "ragged", "adjoint", "dist",
                             "long", "autotune", "adi_backprop"],
                    help="run just one of the other configurations and print its JSON (profiling)")
    ap.add_argument("--ragged-systems", type=int, default=200000,
                    help="systems in the ragged configuration (200000 = the benchmark)")
    ap.add_argument("--grid", default=None,
                    help="X,Y,Z grid instead of n^3 (smaller cases for profiling; x fastest)")
    ap.add_argument("--e2e-steps", type=int, default=8)
    ap.add_argument("--cpu-steps", type=int, default=0, help="0 = as many as fit in ~8 s")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="skip the reference CUDA library's same-box timing")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other configurations (sweep, ADI, precision, ragged, adjoint)")
    return ap.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, STREAM-style copy)"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback (6.65 TB/s pool measurement)"


def ncu_traffic():
    """Per-launch DRAM bytes from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "traffic_solve_kernels_512cubed_f64.txt")
    out = {}
    try:
        with open(path) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 2 and not line.startswith("#"):
                    out[parts[0]] = float(parts[1])
    except OSError:
        pass
    return out


# ---- clocks -----------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu_index = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.gpu_index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.25)
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]
        return False

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": smax, "reasons": [], "samples": 0}
        # samples under load: the upper half of the clock distribution is not a
        # selection here; report the median of all samples taken in the region
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---- CPU reference timing ---------------------------------------------------------

def cpu_reference_rate(n, steps, dtype, warmup=1, time_budget=8.0):
    """elements/s of the reference CPU library (oracle/_ref) on the benchmark's
    own workload: x, y and z solves of the full n^3 grid (d overwritten each
    time), all host threads. steps <= 0: as many steps as fit in about
    time_budget seconds. Returns (rate, info dict)."""
    import numpy as np

    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    os.environ["OMP_NUM_THREADS"] = str(threads)
    os.environ.setdefault("OMP_PROC_BIND", "close")
    sys.path.insert(0, ROOT)
    from oracle.pyoracle import Reference

    ref = Reference()
    npdt = np.float64 if dtype == "f64" else np.float32
    m = n * n * n
    rng = np.random.default_rng(1)
    a = (rng.random(m) - 0.5).astype(npdt)
    c = (rng.random(m) - 0.5).astype(npdt)
    b = (1 + np.abs(a) + np.abs(c) + rng.random(m)).astype(npdt)
    d = rng.standard_normal(m).astype(npdt)
    dims = [n, n, n]

    def step():
        for sd in range(3):
            ref.strided_batch(a, b, c, d, dims, sd)

    for _ in range(max(1, warmup)):
        step()  # page faults, thread start
    if steps <= 0:
        t0 = time.perf_counter()
        step()
        one = time.perf_counter() - t0
        steps = max(2, min(2000, int(time_budget / max(one, 1e-6))))
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    el = time.perf_counter() - t0
    rate = 3 * m * steps / el
    info = {"cores": threads, "kind": "reference",
            "sample": f"{steps} steps of x, y, z solves on the full {n}^3 grid ({dtype}, reference "
                      f"scalar/src/cpu/trid_cpu.cpp built -O3 -fopenmp, {ref.isa}), {el:.2f} s",
            "lib": os.path.basename(ref.path), "same_config": True}
    return rate, info


def gpu_reference_rate(n, steps=10, warmup=3):
    """The reference's own CUDA library (scalar/src/cuda/trid_cuda.cu, built
    for sm_100a into oracle/_ref by oracle/Makefile) on the benchmark's
    workload on the same B200: default opts (cuBLAS-transpose x path,
    trid_strided_multidim y and z), blocking calls as its API makes them,
    timed with CUDA events; a same-box comparator, never the measured
    product. Per axis and per x, y, z step."""
    import torch

    sys.path.insert(0, ROOT)
    from oracle.pyoracle import ReferenceGPU

    ref = ReferenceGPU()
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev).manual_seed(1234)
    shape = (n, n, n)
    a = torch.rand(shape, generator=g, device=dev, dtype=torch.float64) - 0.5
    c = torch.rand(shape, generator=g, device=dev, dtype=torch.float64) - 0.5
    b = 1 + a.abs() + c.abs() + torch.rand(shape, generator=g, device=dev, dtype=torch.float64)
    d = torch.randn(shape, generator=g, device=dev, dtype=torch.float64)
    dims = [n, n, n]
    stream = torch.cuda.current_stream()
    per_axis = {}
    for axis in range(3):
        def call():
            ref.strided_batch(a.data_ptr(), b.data_ptr(), c.data_ptr(), d.data_ptr(), dims, axis, 8)
        for _ in range(warmup):
            call()
        torch.cuda.synchronize()
        ts = []
        for _ in range(steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            call()
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        per_axis["xyz"[axis]] = statistics.median(ts)
    step_ms = sum(per_axis.values())
    del a, b, c, d
    torch.cuda.empty_cache()
    return {"impl": "reference CUDA library scalar/src/cuda/trid_cuda.cu, default opts, sm_100a",
            "lib": os.path.basename(ref.path), "grid": dims, "dtype": "f64",
            "ms_per_axis": {k: round(v, 4) for k, v in per_axis.items()},
            "ms_per_step": round(step_ms, 4), "value": 3 * n ** 3 / step_ms * 1e3,
            "unit": UNIT, "steps": steps, "warmup": warmup}


# ---- the GPU arm ------------------------------------------------------------------

def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch

    import tridsolver_b200 as tb

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    n = args.n
    dims = [int(v) for v in args.grid.split(",")] if args.grid else [n, n, n]
    if len(dims) != 3:
        raise SystemExit("--grid takes X,Y,Z")
    shape = tuple(reversed(dims))
    tdt = torch.float64 if args.dtype == "f64" else torch.float32
    es = 8 if args.dtype == "f64" else 4
    g = torch.Generator(device=dev).manual_seed(1234 + rank)
    a = torch.rand(shape, generator=g, device=dev, dtype=tdt) - 0.5
    c = torch.rand(shape, generator=g, device=dev, dtype=tdt) - 0.5
    b = 1 + a.abs() + c.abs() + torch.rand(shape, generator=g, device=dev, dtype=tdt)
    d = torch.randn(shape, generator=g, device=dev, dtype=tdt)
    solve = tb.tridDmtsvStridedBatch if args.dtype == "f64" else tb.tridSmtsvStridedBatch
    elems = dims[0] * dims[1] * dims[2]

    stream = torch.cuda.current_stream()
    tb.set_stream(stream)
    tb.set_blocking(False)

    def step(evs=None):
        for axis in range(3):
            if evs is not None:
                evs[axis][0].record(stream)
            st = solve(None, a, b, c, d, 3, axis, dims, dims)
            if st != 0:
                raise RuntimeError(f"solve status {st}")
            if evs is not None:
                evs[axis][1].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    K = args.steps
    evs = [[[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(3)]
           for _ in range(K)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    gpu_index = vis.split(",")[local_rank] if vis else str(local_rank)
    launches0 = tb.launch_count()
    with ClockSampler(gpu_index) as clk:
        torch.cuda.synchronize()
        t_start.record(stream)
        for k in range(K):
            step(evs[k])
        t_end.record(stream)
        torch.cuda.synchronize()
    launches = tb.launch_count() - launches0
    if world > 1:
        torch.distributed.barrier()
    total_ms = t_start.elapsed_time(t_end)
    axis_ms = [statistics.mean(evs[k][ax][0].elapsed_time(evs[k][ax][1]) for k in range(K))
               for ax in range(3)]
    vals = torch.tensor([total_ms] + axis_ms, dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(vals, op=torch.distributed.ReduceOp.MAX)
    total_ms, axis_ms = vals[0].item(), [v.item() for v in vals[1:]]
    ms_per_step = total_ms / K
    value = world * 3 * elems * K / (total_ms / 1e3)

    # ---- end to end through the C ABI with host arrays. Each step copies its
    # inputs in from pinned host memory, solves x, y, z, and reads the result
    # back; consecutive steps overlap on three streams (copy in | solve | copy
    # out, two device buffer sets), as an application streaming problems
    # through one GPU would, so PCIe runs both directions at once.
    e2e = None
    if not args.no_e2e:
        host = [t.cpu().pin_memory() for t in (a, b, c, d)]
        outs = [torch.empty_like(host[3]).pin_memory() for _ in range(2)]
        bufs = [(a, b, c, d), tuple(torch.empty_like(t) for t in (a, b, c, d))]
        s_in, s_out = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
        tb.set_stream(stream)
        tb.set_blocking(False)

        def e2e_run(nsteps):
            free = [None, None]  # buffer set k's result has been read back
            last = None
            for k in range(nsteps):
                buf, out = bufs[k % 2], outs[k % 2]
                with torch.cuda.stream(s_in):
                    if free[k % 2] is not None:
                        s_in.wait_event(free[k % 2])
                    for t, h in zip(buf, host):
                        t.copy_(h, non_blocking=True)
                    ready = torch.cuda.Event()
                    ready.record(s_in)
                stream.wait_event(ready)
                for axis in range(3):
                    st = solve(None, buf[0], buf[1], buf[2], buf[3], 3, axis, dims, dims)
                    if st != 0:
                        raise RuntimeError(f"solve status {st}")
                solved = torch.cuda.Event()
                solved.record(stream)
                with torch.cuda.stream(s_out):
                    s_out.wait_event(solved)
                    out.copy_(buf[3], non_blocking=True)
                    last = torch.cuda.Event(enable_timing=True)
                    last.record(s_out)
                    free[k % 2] = last
            return last

        e2e_run(2)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e0.record(s_in)
        e1 = e2e_run(args.e2e_steps)
        torch.cuda.synchronize()
        ok = bool(torch.equal(outs[(args.e2e_steps - 1) % 2], bufs[(args.e2e_steps - 1) % 2][3].cpu()))
        ems = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
        if world > 1:
            torch.distributed.all_reduce(ems, op=torch.distributed.ReduceOp.MAX)
        e2e = {"value": world * 3 * elems * args.e2e_steps / (ems.item() / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": 4 * elems * es, "d2h_bytes_per_step": elems * es,
               "ms_per_step": ems.item() / args.e2e_steps, "steps": args.e2e_steps,
               "result_read_back": ok,
               "path": "per step: pinned host -> device copies of a,b,c,d, three "
                       "tridDmtsvStridedBatch calls, device -> host copy of d; steps "
                       "overlap on three streams with two device buffer sets"}
        del bufs
        torch.cuda.empty_cache()

    hbm, hbm_src = peaks()
    traffic = ncu_traffic()
    names = ["x", "y", "z"]
    alg_bytes = 5 * es * elems  # read a, b, c, d; write d
    per_axis = {}
    for ax in range(3):
        gbs = alg_bytes / (axis_ms[ax] / 1e3) / 1e9
        per_axis[names[ax]] = {
            "ms": round(axis_ms[ax], 4),
            "elements_per_s": elems / (axis_ms[ax] / 1e3),
            "hbm_gbs": round(gbs, 1),
            "frac_of_measured_peak": round(gbs / hbm, 4),
            "plan": tb.describe_plan(es, dims, ax),
        }
    dom = max(range(3), key=lambda i: axis_ms[i])
    dom_gbs = alg_bytes / (axis_ms[dom] / 1e3) / 1e9
    key = f"{args.dtype}_n{n}_{names[dom]}" if not args.grid else None
    roofline = {"bound": "hbm", "achieved": round(dom_gbs, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(dom_gbs / hbm, 4),
                "traffic": traffic.get(key),
                "kernel": f"solve along {names[dom]} ({per_axis[names[dom]]['plan']})",
                "algorithmic_bytes_per_launch": alg_bytes, "peak_source": hbm_src}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": args.dtype, "data": "synthetic",
            "config": {"workload": (f"{n}^3 {args.dtype.upper()} tridDmtsvStridedBatch along x, y, z "
                                    f"(one step = 3 solves of {n * n} systems of length {n}, d "
                                    "overwritten, ADI order)") if not args.grid else
                       (f"{'x'.join(map(str, dims))} {args.dtype.upper()} solves along x, y, z "
                        "(profiling case, not the benchmark)"),
                       "grid": dims, "parallelism": f"replicas x{world} (systems sharded by rank)",
                       "l2": "inputs larger than L2 (each array "
                             f"{elems * es / 2**30:.2f} GiB); no flush"},
            "per_axis": per_axis, "roofline": roofline, "e2e": e2e,
            "gpu_launches": launches, "clocks": clk.summary()}
    return line


# ---- the other configurations (reported beside the headline, not in `value`) ----

def _timed(fn, reps, stream):
    import torch
    fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _system(shape, dt, dev, seed, margin_lo=None):
    import torch
    g = torch.Generator(device=dev).manual_seed(seed)
    a = torch.rand(shape, generator=g, device=dev, dtype=dt) - 0.5
    c = torch.rand(shape, generator=g, device=dev, dtype=dt) - 0.5
    if margin_lo is None:
        b = 1 + a.abs() + c.abs() + torch.rand(shape, generator=g, device=dev, dtype=dt)
    else:
        u = torch.rand(shape, generator=g, device=dev, dtype=torch.float64)
        b = (a.abs() + c.abs() + 10.0 ** (margin_lo * (1 - u))).to(dt)
    d = torch.randn(shape, generator=g, device=dev, dtype=dt)
    return a, b, c, d


def config_sweep(dev, hbm):
    """Drop-in sweep: FP32/FP64, 256^3/512^3, x/y/z, overwrite and Inc."""
    import torch
    import tridsolver_b200 as tb
    out = []
    stream = torch.cuda.current_stream()
    for n in (256, 512):
        for dt, es, name in ((torch.float64, 8, "f64"), (torch.float32, 4, "f32")):
            a, b, c, d = _system((n, n, n), dt, dev, n)
            u = torch.randn_like(d)
            dims = [n] * 3
            for axis in range(3):
                for inc in (False, True):
                    if inc:
                        fn = tb.tridDmtsvStridedBatchInc if es == 8 else tb.tridSmtsvStridedBatchInc
                        call = lambda: fn(None, a, b, c, d, u, 3, axis, dims, dims)  # noqa: E731
                    else:
                        fn = tb.tridDmtsvStridedBatch if es == 8 else tb.tridSmtsvStridedBatch
                        call = lambda: fn(None, a, b, c, d, 3, axis, dims, dims)  # noqa: E731
                    ms = _timed(call, 10, stream)
                    words = 6 if inc else 5
                    gbs = words * es * n ** 3 / ms / 1e6
                    out.append({"grid": n, "dtype": name, "axis": "xyz"[axis], "inc": inc,
                                "ms": round(ms, 4), "elements_per_s": n ** 3 / ms * 1e3,
                                "hbm_gbs": round(gbs, 1), "frac": round(gbs / hbm, 4),
                                "plan": tb.describe_plan(es, dims, axis, inc=inc)})
            del a, b, c, d, u
            torch.cuda.empty_cache()
    return out


def config_adi(dev, hbm, n=(256, 256, 256), steps=100, dtype="f64", alpha=1.0):
    """ADI heat steps replayed from a CUDA graph of one timestep, in the fused
    form (coefficients as scalars, stencil inside the x solve: 7 words per
    point and step) and in the reference application's form (coefficient
    arrays: 21 words)."""
    import numpy as np
    import torch
    from tridsolver_b200.adi import ADIHeat
    dt = torch.float64 if dtype == "f64" else torch.float32
    es = 8 if dtype == "f64" else 4
    nz, ny, nx = n
    elems = nx * ny * nz
    out = {"grid": [nx, ny, nz], "dtype": dtype, "steps": steps,
           "graph": "one timestep captured, replayed per step; lambda[step] read on the device"}
    for form, arrays, words in (("fused", False, 7), ("arrays", True, 5 + 5 + 5 + 6)):
        g = torch.Generator(device=dev).manual_seed(3)
        u = torch.randn((nz, ny, nx), generator=g, device=dev, dtype=dt)
        u[0], u[-1], u[:, 0], u[:, -1], u[:, :, 0], u[:, :, -1] = 0, 0, 0, 0, 0, 0
        lams = np.random.default_rng(4).uniform(0.1, 1.0, steps + 2)
        sim = ADIHeat(u, lams, alpha=alpha, coefficient_arrays=arrays)
        sim.capture()
        sim.reset_counter(0)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        sim.run(steps)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        gbs = words * es * elems / ms / 1e6
        out[form] = {"ms_per_step": round(ms, 4), "elements_per_s": elems / ms * 1e3,
                     "hbm_gbs": round(gbs, 1), "frac": round(gbs / hbm, 4),
                     "words_per_element_step": words,
                     "finite": bool(torch.isfinite(sim.u).all().item())}
        if form == "fused":
            u_fused = sim.u.clone()
        else:
            out["fused_vs_arrays_max_abs"] = float((u_fused - sim.u).abs().max().item())
        del sim, u
        torch.cuda.empty_cache()
    return out


def config_precision(dev, n=512, dims=None):
    """FP64-specified systems (margins b - |a| - |c| log-uniform in [10^lo, 1])
    solved along x and z three ways, each timed and its error measured
    against the direct FP64 solve of the FP64 system (tridDmtsvStridedBatch,
    which the GPU tests pin to the reference CPU solver at 1e-12):
      * refine_fp64_system: tridDmtsvStridedBatchRefine, the FP32
        factorisation of the rounded coefficients refined with the FP64
        residual of the FP64 system (40 bytes per element, one pass);
      * fp32_values: tridDmtsvStridedBatchMixed on the coefficients rounded
        to FP32, which solves that rounded system exactly (28 bytes per
        element); its error against the FP64 system is the rounding's;
      * fp64_ms: the direct FP64 solve itself."""
    import torch
    import tridsolver_b200 as tb
    stream = torch.cuda.current_stream()
    dims = list(dims) if dims else [n] * 3
    shape = tuple(reversed(dims))
    out = []

    def rel(x, ref):
        return ((x - ref).abs().max() / ref.abs().max()).item()

    for lo in (-3, -2, -1, 0):
        a, b, c, d = _system(shape, torch.float64, dev, 7 - lo, margin_lo=lo if lo < 0 else None)
        a32, b32, c32 = a.float(), b.float(), c.float()
        for axis in (0, 2):
            tb.set_blocking(True)
            x64 = d.clone()
            tb.tridDmtsvStridedBatch(None, a, b, c, x64, 3, axis, dims, dims)
            xr = d.clone()
            st_r, it_r, est_r = tb.tridDmtsvStridedBatchRefine(None, a, b, c, xr, 3, axis, dims, dims,
                                                               12, 1e-12)
            err_r = rel(xr, x64)
            xp = d.clone()
            tb.tridDmtsvStridedBatch(None, a32.double(), b32.double(), c32.double(), xp, 3, axis,
                                     dims, dims)
            xm = d.clone()
            st_m, it_m, _ = tb.tridDmtsvStridedBatchMixed(None, a32, b32, c32, xm, 3, axis, dims,
                                                          dims, 12, 1e-12)
            err_m_own, err_m_64 = rel(xm, xp), rel(xm, x64)
            tb.set_blocking(False)
            w = d.clone()
            t64 = _timed(lambda: tb.tridDmtsvStridedBatch(None, a, b, c, w, 3, axis, dims, dims), 5,
                         stream)
            tr = _timed(lambda: tb.tridDmtsvStridedBatchRefine(None, a, b, c, w, 3, axis, dims, dims,
                                                               12, 1e-12), 5, stream)
            tm = _timed(lambda: tb.tridDmtsvStridedBatchMixed(None, a32, b32, c32, w, 3, axis, dims,
                                                              dims, 12, 1e-12), 5, stream)
            # the FP32-values form with its refinement forced (mode 1)
            tb.set_mixed_mode(1)
            tmr = _timed(lambda: tb.tridDmtsvStridedBatchMixed(None, a32, b32, c32, w, 3, axis, dims,
                                                               dims, 12, 1e-12), 5, stream)
            tb.set_blocking(True)
            xmr = d.clone()
            _, it_mr, _ = tb.tridDmtsvStridedBatchMixed(None, a32, b32, c32, xmr, 3, axis, dims, dims,
                                                        12, 1e-12)
            err_mr = rel(xmr, xp)
            tb.set_mixed_mode(0)
            out.append({
                "margin_min": 10.0 ** lo, "axis": "xyz"[axis], "fp64_ms": round(t64, 4),
                "refine_fp64_system": {
                    "status": st_r, "iterations": it_r, "estimated_rel_error": est_r,
                    "max_rel_error_vs_fp64_system": err_r, "ms": round(tr, 4),
                    "time_over_fp64": round(tr / t64, 3), "bytes_per_element": 40,
                    "reaches_1e-12": err_r <= 1e-12},
                "fp32_values": {
                    "status": st_m, "iterations": it_m,
                    "strategy": "refinement" if it_m else "direct FP64 solve of the FP32 values",
                    "max_rel_error_vs_fp64_of_fp32_values": err_m_own,
                    "max_rel_error_vs_fp64_system": err_m_64, "ms": round(tm, 4),
                    "time_over_fp64": round(tm / t64, 3), "bytes_per_element": 28,
                    "refinement_forced": {"ms": round(tmr, 4), "time_over_fp64": round(tmr / t64, 3),
                                          "iterations": it_mr,
                                          "max_rel_error_vs_fp64_of_fp32_values": err_mr}},
            })
            del x64, xr, xp, xm, xmr, w
        del a32, b32, c32, a, b, c, d
        torch.cuda.empty_cache()
    return out


def config_ragged(dev, hbm, nsys=200000):
    """200,000 systems, lengths floor(exp(U(ln 8, ln 16384))), one persistent launch."""
    import numpy as np
    import torch
    import tridsolver_b200 as tb
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(0)
    lengths = np.floor(np.exp(rng.uniform(np.log(8), np.log(16384), nsys))).astype(np.int64)
    offs = torch.from_numpy(np.concatenate([[0], np.cumsum(lengths)]).astype(np.int64)).to(dev)
    n = int(lengths.sum())
    out = {"systems": nsys, "elements": n, "lengths": "floor(exp(U(ln 8, ln 16384))), seed 0"}
    for dt, es, name in ((torch.float64, 8, "f64"), (torch.float32, 4, "f32")):
        a, b, c, d = _system((n,), dt, dev, 11)
        fn = tb.tridDmtsvRaggedBatch if es == 8 else tb.tridSmtsvRaggedBatch
        ms = _timed(lambda: fn(None, a, b, c, d, offs, nsys), 5, stream)
        gbs = (5 * es * n + 8 * (nsys + 1)) / ms / 1e6
        out[name] = {"ms": round(ms, 4), "elements_per_s": n / ms * 1e3, "hbm_gbs": round(gbs, 1),
                     "frac": round(gbs / hbm, 4), "rows_per_lane_by_class": tb.ragged_table(es)}
        del a, b, c, d
        torch.cuda.empty_cache()
    return out


def config_dist(dev, hbm, n=512):
    """Per-rank device cost of the distributed solve (partition method across
    ranks): one rank's block of n^3 FP64 with a 1-rank exchange (a device
    copy), so the reduction, the reduced solve and the local solve are timed
    without the network; 9 words per element (4 for the reduction, 5 for the
    local solve) against the plain solve's 5."""
    import torch
    import tridsolver_b200 as tb
    from tridsolver_b200.distributed import DistContext, device_bytes
    stream = torch.cuda.current_stream()
    a, b, c, d = _system((n, n, n), torch.float64, dev, 21)
    dims = [n] * 3

    def local_copy(send, recv, nbytes, nranks):
        device_bytes(recv, nbytes, dev).copy_(device_bytes(send, nbytes, dev))

    out = []
    for axis in range(3):
        with DistContext(axis, rank=0, nranks=1, allgather=local_copy) as dc:
            ms_dist = _timed(lambda: dc.strided_batch(a, b, c, d, dims), 5, stream)
        ms_plain = _timed(lambda: tb.strided_batch(a, b, c, d, axis, dims), 5, stream)
        elems = n ** 3
        out.append({"axis": "xyz"[axis], "ms_dist": round(ms_dist, 4), "ms_plain": round(ms_plain, 4),
                    "dist_frac": round(9 * 8 * elems / ms_dist / 1e6 / hbm, 4),
                    "plain_frac": round(5 * 8 * elems / ms_plain / 1e6 / hbm, 4)})
    return {"grid": dims, "dtype": "f64", "words_per_element": {"dist": 9, "plain": 5},
            "exchange": "1 rank, device copy (per-rank device cost without the network)",
            "results": out}


def config_long(dev, hbm):
    """Few, long FP64 systems (the long path: chunk reduction to scratch,
    recursive solve of the reduced batch, substitution), along x (contiguous)
    and z (rows a plane apart). Its byte floor is 9 words per element: a, b,
    c, d read in the reduction and again in the substitution, x written."""
    import torch
    import tridsolver_b200 as tb
    stream = torch.cuda.current_stream()
    out = []
    for dims, axis, label in (([1 << 20, 64], 0, "64 x 2^20 rows, x"),
                              ([65536, 1024], 0, "1024 x 65536 rows, x"),
                              ([8, 8, 1 << 20], 2, "64 x 2^20 rows, z"),
                              ([32, 32, 65536], 2, "1024 x 65536 rows, z")):
        shape = tuple(reversed(dims))
        a, b, c, d = _system(shape, torch.float64, dev, 31)
        nd = len(dims)
        x = d.clone()
        ms = _timed(lambda: tb.tridDmtsvStridedBatch(None, a, b, c, x, nd, axis, dims, dims), 5,
                    stream)
        n = a.numel()
        gbs9 = 9 * 8 * n / ms / 1e6
        out.append({"case": label, "dims": dims, "solvedim": axis, "ms": round(ms, 4),
                    "elements_per_s": n / ms * 1e3, "plan": tb.describe_plan(8, dims, axis),
                    "bytes_per_element": 72, "hbm_gbs_at_9_words": round(gbs9, 1),
                    "frac_of_9_word_floor": round(gbs9 / hbm, 4)})
        del a, b, c, d, x
        torch.cuda.empty_cache()
    return out


def config_autotune(dev, hbm):
    """tridAutotune on the drop-in grids: for each shape the built-in plan and
    the tuned plan (the fastest of every applicable plan on this device),
    both timed as the solve then runs."""
    import torch
    import tridsolver_b200 as tb
    stream = torch.cuda.current_stream()
    out = []
    for n, dt, es in ((512, torch.float64, 8), (256, torch.float32, 4), (256, torch.float64, 8)):
        shape = (n, n, n)
        a, b, c, d = _system(shape, dt, dev, 41)
        dims = [n] * 3
        solve = tb.tridDmtsvStridedBatch if es == 8 else tb.tridSmtsvStridedBatch
        for axis in range(3):
            tb.autotune_reset()
            plan0 = tb.describe_plan(es, dims, axis)
            t0 = _timed(lambda: solve(None, a, b, c, d, 3, axis, dims, dims), 10, stream)
            tb.set_blocking(True)
            _, plan1 = tb.autotune(es, dims, axis)
            tb.set_blocking(False)
            t1 = _timed(lambda: solve(None, a, b, c, d, 3, axis, dims, dims), 10, stream)
            gbs = 5 * es * n ** 3 / t1 / 1e6
            out.append({"grid": dims, "dtype": "f64" if es == 8 else "f32", "axis": "xyz"[axis],
                        "builtin_plan": plan0, "builtin_ms": round(t0, 4), "tuned_plan": plan1,
                        "tuned_ms": round(t1, 4), "tuned_frac": round(gbs / hbm, 4)})
        tb.autotune_reset()
        del a, b, c, d
        torch.cuda.empty_cache()
    return out


def config_adjoint(dev, n=256, probes=1000):
    """Adjoint along y on 256^3 FP64: time against the forward solve; gradient
    entries against central finite differences (h = 1e-6) of L = sum(w x)."""
    import torch
    import tridsolver_b200 as tb
    stream = torch.cuda.current_stream()
    dims = [n] * 3
    a, b, c, d = _system((n, n, n), torch.float64, dev, 21)
    w = torch.randn_like(d)
    x = d.clone()
    tb.set_blocking(True)
    tb.tridDmtsvStridedBatch(None, a, b, c, x, 3, 1, dims, dims)
    grads = [torch.empty_like(d) for _ in range(4)]
    tb.tridDmtsvStridedBatchAdjoint(None, a, b, c, x, w, grads[3], grads[0], grads[1], grads[2], 3, 1,
                                    dims, dims)
    tb.set_blocking(False)
    xx = d.clone()
    tf = _timed(lambda: tb.tridDmtsvStridedBatch(None, a, b, c, xx, 3, 1, dims, dims), 10, stream)
    ta = _timed(lambda: tb.tridDmtsvStridedBatchAdjoint(None, a, b, c, x, w, grads[3], grads[0],
                                                        grads[1], grads[2], 3, 1, dims, dims),
                10, stream)
    td_only = _timed(lambda: tb.tridDmtsvStridedBatchAdjoint(None, a, b, c, x, w, grads[3], None, None,
                                                             None, 3, 1, dims, dims), 10, stream)
    # finite differences: perturb one entry, solve twice; only the y-line of
    # the perturbed entry changes, so the difference of L = sum(w x) is taken
    # over that line (a global sum would bury it in summation roundoff)
    tb.set_blocking(True)
    g = torch.Generator(device="cpu").manual_seed(5)
    arrays = [a, b, c, d]
    worst = 0.0
    h = 1e-6
    xp = torch.empty_like(d)
    xm = torch.empty_like(d)
    w3 = w.view(n, n, n)
    for k in range(probes):
        which = int(torch.randint(0, 4, (1,), generator=g))
        idx = int(torch.randint(0, n ** 3, (1,), generator=g))
        kz, rem = divmod(idx, n * n)
        jy, ix = divmod(rem, n)
        arr = arrays[which].view(-1)
        old = arr[idx].item()
        for sign, out in ((1.0, xp), (-1.0, xm)):
            arr[idx] = old + sign * h
            out.copy_(d)
            tb.tridDmtsvStridedBatch(None, a, b, c, out, 3, 1, dims, dims)
        arr[idx] = old
        line = (xp.view(n, n, n)[kz, :, ix] - xm.view(n, n, n)[kz, :, ix])
        fd = torch.dot(w3[kz, :, ix], line).item() / (2 * h)
        gv = grads[which].view(-1)[idx].item()
        worst = max(worst, abs(fd - gv) / max(1.0, abs(fd)))
    return {"grid": dims, "axis": "y", "forward_ms": round(tf, 4), "adjoint_ms": round(ta, 4),
            "adjoint_over_forward": round(ta / tf, 3), "adjoint_dbar_only_ms": round(td_only, 4),
            "fd_probes": probes, "fd_worst_rel_error": worst,
            "bytes_floor_ratio": "9 words (a,b,c,w,x in; 4 gradients out) vs 5 for the forward solve"}


def config_adi_backprop(dev, hbm, n=256, steps=50, every=10):
    """50-step FP64 ADI run on n^3 backpropagated to the initial field and to
    each step's lambda, checkpointing every 10 steps (the forward pass keeps
    every 10th field; the backward recomputes each segment, then runs the
    native step adjoints). Timed with CUDA events against the forward run
    alone. Words per point and step: forward 7 (fused step), segment
    recompute 7, adjoint 28 (forward intermediates 10, copy of the gradient
    2, three transposed solves 6, lambda reductions 6, stencil transpose 4)."""
    import torch
    from tridsolver_b200.adi import adi_run
    stream = torch.cuda.current_stream()
    g = torch.Generator(device=dev).manual_seed(8)
    u0 = torch.randn((n, n, n), generator=g, device=dev, dtype=torch.float64)
    lams = 0.1 + 0.9 * torch.rand(steps, generator=g, device=dev, dtype=torch.float64)
    w = torch.randn((n, n, n), generator=g, device=dev, dtype=torch.float64)

    def fwd_only():
        with torch.no_grad():
            return adi_run(u0, lams, checkpoint_every=every)

    def fwd_bwd():
        u = u0.clone().requires_grad_(True)
        lv = lams.clone().requires_grad_(True)
        (w * adi_run(u, lv, checkpoint_every=every)).sum().backward()
        return u, lv

    fwd_only()
    fwd_bwd()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fwd_only()
    e1.record(stream)
    torch.cuda.synchronize()
    t_fwd = e0.elapsed_time(e1)
    e0.record(stream)
    u, lv = fwd_bwd()
    e1.record(stream)
    torch.cuda.synchronize()
    t_all = e0.elapsed_time(e1)
    words = 7 + 7 + 28
    gbs = words * 8 * n ** 3 * steps / t_all / 1e6
    # central finite differences of the loss: 3 lambdas (h = 1e-5) and 3
    # entries of the initial field (the run is linear in u0, so h = 1 is
    # exact up to rounding)
    fd = []
    with torch.no_grad():
        def loss(uu, lvv):
            return (w * adi_run(uu, lvv, checkpoint_every=0)).sum().item()
        for k in (0, steps // 2, steps - 1):
            h = 1e-5
            lp, lm = lams.clone(), lams.clone()
            lp[k] += h
            lm[k] -= h
            est = (loss(u0, lp) - loss(u0, lm)) / (2 * h)
            fd.append(abs(est - lv.grad[k].item()) / max(1.0, abs(est)))
        for idx in ((1, 1, 1), (n // 2, n // 3, n // 4), (n - 2, 7, n // 2)):
            up, um = u0.clone(), u0.clone()
            up[idx] += 1.0
            um[idx] -= 1.0
            est = (loss(up, lams) - loss(um, lams)) / 2.0
            fd.append(abs(est - u.grad[idx].item()) / max(1.0, abs(est)))
    return {"grid": [n] * 3, "dtype": "f64", "steps": steps, "checkpoint_every": every,
            "fd_probes": len(fd), "fd_worst_rel_error": max(fd),
            "forward_ms_per_step": round(t_fwd / steps, 4),
            "forward_backward_ms_per_step": round(t_all / steps, 4),
            "backward_over_forward": round((t_all - t_fwd) / t_fwd, 2),
            "words_per_point_step": words, "hbm_gbs": round(gbs, 1), "frac": round(gbs / hbm, 4),
            "grad_u0_finite": bool(torch.isfinite(u.grad).all().item()),
            "grad_lambda": [round(v, 6) for v in lv.grad[:5].tolist()]}


def run_configs(dev, hbm):
    import torch
    import tridsolver_b200 as tb
    tb.set_stream(torch.cuda.current_stream())
    tb.set_blocking(False)
    res = {}
    for name, fn in (("sweep", lambda: config_sweep(dev, hbm)),
                     ("adi_256_f64_100", lambda: config_adi(dev, hbm)),
                     ("precision", lambda: config_precision(dev)),
                     ("ragged", lambda: config_ragged(dev, hbm)),
                     ("adi_512x512x128_f32_1000", lambda: config_adi(dev, hbm, (128, 512, 512), 1000,
                                                                      "f32")),
                     ("adjoint", lambda: config_adjoint(dev)),
                     ("long_systems", lambda: config_long(dev, hbm)),
                     ("autotune", lambda: config_autotune(dev, hbm)),
                     ("dist_512_f64", lambda: config_dist(dev, hbm)),
                     ("adi_backprop", lambda: config_adi_backprop(dev, hbm))):
        try:
            res[name] = fn()
        except Exception as e:  # keep the headline line whatever happens here
            res[name] = {"error": f"{type(e).__name__}: {e}"}
        torch.cuda.empty_cache()
    tb.set_blocking(True)
    return res


def main():
    args = parse_args()
    if args.only_config:
        import torch
        import tridsolver_b200 as tb
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        tb.set_stream(torch.cuda.current_stream())
        tb.set_blocking(False)
        hbm = peaks()[0]
        grid = [int(v) for v in args.grid.split(",")] if args.grid else None
        fn = {"sweep": lambda: config_sweep(dev, hbm), "adi": lambda: config_adi(dev, hbm),
              "adi_f32": lambda: config_adi(dev, hbm, (128, 512, 512), 1000, "f32"),
              "precision": lambda: config_precision(dev, args.n, grid),
              "ragged": lambda: config_ragged(dev, hbm, args.ragged_systems),
              "adjoint": lambda: config_adjoint(dev),
              "dist": lambda: config_dist(dev, hbm),
              "long": lambda: config_long(dev, hbm),
              "autotune": lambda: config_autotune(dev, hbm),
              "adi_backprop": lambda: config_adi_backprop(dev, hbm)}[args.only_config]
        print(json.dumps({"config": args.only_config, "result": fn()}))
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        rate, info = cpu_reference_rate(args.n, args.steps, args.dtype, warmup=args.warmup)
        line = {"metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": args.dtype, "data": "synthetic",
                "impl": "reference",
                "config": {"workload": f"{args.n}^3 {args.dtype.upper()} solves along x, y, z "
                                       "(d overwritten), the full grid each step",
                           "grid": [args.n] * 3},
                "cpu_baseline": dict(info, value=rate, unit=UNIT),
                "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    if world > 1:
        import datetime

        import torch

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    line = run_ours(args, rank, world, local_rank)
    if rank == 0 and world == 1 and not args.no_configs:
        import torch

        line["configs"] = run_configs(torch.device("cuda", local_rank), peaks()[0])
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, info = cpu_reference_rate(args.n, args.cpu_steps, args.dtype)
        line["cpu_baseline"] = dict(info, value=rate, unit=UNIT)
    if rank == 0 and world == 1 and not args.no_ref_gpu and args.dtype == "f64" and args.n <= 512:
        try:
            line["reference_gpu"] = gpu_reference_rate(args.n)
            line["reference_gpu"]["ours_over_reference_gpu"] = round(
                line["value"] / line["reference_gpu"]["value"], 3)
        except Exception as e:  # the comparator is optional
            line["reference_gpu"] = {"unavailable": f"{type(e).__name__}: {e}"}
    if world > 1:
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
