"""Benchmark of the Seldon sparse Krylov path on B200.

One step = one FP64 CSR SpMV y = A*x (Seldon's Mlt on Matrix<double,
General, RowSparse>) on the 3D 7-point upwind convection-diffusion matrix of
a 128^3 grid (n = 2,097,152, nnz = 14,581,760).  `value` is whole-job HBM
throughput in algorithmic GB/s (nnz*(8+4) + 4*(n+1) + 8*n + 8*n bytes per
SpMV); the inputs (217 MB) exceed the 126 MB L2.

The same JSON line carries the time-to-solution figures of the path (CG on
the 100^2 Laplacian; FP64 CG and FP32/FP64 iterative refinement on the 192^3
Poisson problem; GMRES(30)+Jacobi on the 128^3 convection-diffusion problem;
the Zipf SpMV; 4096 batched shifted Laplacians against a loop of FP64 CG
calls; the adjoint solve on the 512^2 anisotropic graph Laplacian with its
gradient checks; COO->CSR assembly of the 128^3 operator's triplets; ILU(0)
factor, apply and preconditioned BiCGSTAB on the same operator) and the
roofline, e2e, cpu_baseline and clock records.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: replicas only (the path does not shard, one system per GPU); under
torchrun every rank runs the same step and `value` is the sum over ranks.
"""
import argparse
import ctypes
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

METRIC = ("ms to 1e-10 rel. residual: mixed/batched vs plain FP64 GPU CG; SpMV HBM GB/s")
WORKLOAD = "fp64 CSR SpMV, 3D 7-pt upwind convection-diffusion 128^3 (n=2097152, nnz=14581760)"
GRID = 128


def spmv_bytes(n, m, nnz, vbytes=8, wbytes=8):
    return nnz * (vbytes + 4) + 4 * (m + 1) + n * wbytes + m * wbytes


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--no-extras", action="store_true", help="skip the solver/Zipf extras")
    p.add_argument("--extras", default="all",
                   help="comma list of extras to run: c1, c3, gmres, krylov, zipf, batch, adjoint, assemble, "
                        "ilu0 "
                        "(default all)")
    p.add_argument("--cpu-seconds", type=float, default=8.0,
                   help="bounded CPU-baseline sample (seconds of work)")
    p.add_argument("--gmres-grid", type=int, default=GRID,
                   help="grid side of the GMRES extras' convection-diffusion problem (profiling "
                        "captures take a smaller one)")
    p.add_argument("--batch-systems", type=int, default=4096,
                   help="systems of the batch extra (profiling captures take fewer)")
    p.add_argument("--batch-plan", default=None,
                   help="threads,warp_max[,cluster,cluster_min]: a fixed batch plan instead of "
                        "the autotuner's")
    p.add_argument("--no-cpu-solves", action="store_true",
                   help="skip the reference's host solves beside the solver extras")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ reference CPU arm

def cpu_reference_spmv(ptr, ind, val, seconds, threads):
    """The reference's own MltAdd (oracle/_ref, Seldon's templates compiled
    from its headers) on the host cores: `threads` independent products of
    the same matrix (one output vector each), repeated until ~`seconds`.
    Returns (GB/s aggregate, spmv count, threads, wall seconds)."""
    from oracle.pyoracle import REF_FAST_SO, Reference, Oracle
    if Reference.available(REF_FAST_SO):
        lib, kind = Reference(REF_FAST_SO), "reference"
    else:
        lib, kind = Oracle(), "port"
    m = ptr.size - 1
    x = np.random.default_rng(0).standard_normal(m)
    one = time.perf_counter()
    lib.mltadd(m, m, ptr, ind, val, 1.0, x, 0.0, np.zeros(m))
    one = time.perf_counter() - one
    reps = max(1, int(seconds / max(one, 1e-6) / 1.0))
    counts = [0] * threads

    p_ = np.ascontiguousarray(ptr, dtype=np.int32)
    i_ = np.ascontiguousarray(ind, dtype=np.int32)
    v_ = np.ascontiguousarray(val, dtype=np.float64)

    def work(t):
        y = np.zeros(m)
        fn = lib.lib.ref_mltadd if kind == "reference" else None
        for _ in range(reps):
            if fn is not None:
                fn(m, m, i_.size, p_.ctypes.data, i_.ctypes.data, v_.ctypes.data, 0, 0,
                   ctypes.c_double(1.0), x.ctypes.data, ctypes.c_double(0.0), y.ctypes.data)
            else:
                lib.lib.orc_mltadd(m, m, p_.ctypes.data, i_.ctypes.data, v_.ctypes.data, 0, 0,
                                   ctypes.c_double(1.0), x.ctypes.data, ctypes.c_double(0.0),
                                   y.ctypes.data)
            counts[t] += 1

    ths = [threading.Thread(target=work, args=(t,)) for t in range(threads)]
    t0 = time.perf_counter()
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    wall = time.perf_counter() - t0
    total = sum(counts)
    gbs = total * spmv_bytes(m, m, ind.size) / wall / 1e9
    return gbs, total, threads, wall, kind


def host_threads():
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference(args, rank, world):
    if rank != 0:
        return
    from seldon_b200 import matgen
    ptr, ind, val = matgen.convdiff3d(GRID)
    n = ptr.size - 1
    threads = min(host_threads(), 64)
    # each step: a bounded sample (threads concurrent products)
    per_step = []
    kind = "reference"
    for s in range(args.warmup + args.steps):
        gbs, cnt, th, wall, kind = cpu_reference_spmv(ptr, ind, val, 0.0, threads)
        if s >= args.warmup:
            per_step.append((gbs, cnt, wall))
    tot_bytes = sum(c for _, c, _ in per_step) * spmv_bytes(n, n, ind.size)
    tot_wall = sum(w for _, _, w in per_step)
    value = tot_bytes / tot_wall / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "GB/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(tot_wall / len(per_step) * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "parallelism": "host threads, one product each"},
        "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": threads,
                         "kind": kind,
                         "sample": f"{threads} concurrent Seldon MltAdd products per step"},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ our arm

def read_traffic():
    """dram bytes per SpMV launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "spmv_csr_fp64_convdiff128.md")
    try:
        for ln in open(path):
            if ln.startswith("dram_bytes_per_launch:"):
                return float(ln.split(":")[1])
    except OSError:
        pass
    return None


def measured_peak():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def job_throughput(ms_local, bytes_per_step, world, device=None):
    """Whole-job throughput of `world` replicas, one per GPU: the per-step
    time is the maximum over ranks (the slowest replica sets the job's pace)
    and the bytes of all ranks add up.  Every rank calls this (it runs an
    all-reduce when world > 1).  Returns (GB/s, max ms per step)."""
    ms_max = float(ms_local)
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor([ms_max], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    return world * bytes_per_step / (ms_max * 1e-3) / 1e9, ms_max


def run_ours(args, rank, world, local):
    import torch
    import torch.distributed as dist

    from seldon_b200 import api, matgen
    from seldon_b200 import _lib

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    L = _lib.load()

    ptr, ind, val = matgen.convdiff3d(GRID)
    n = ptr.size - 1
    nnz = ind.size
    A = api.RowSparse(n, n, ptr, ind, val)
    B = spmv_bytes(n, n, nnz)
    # rows of at most 32 entries go to the SELL slice kernel, longer ones to
    # the long-row kernel (a second launch)
    launches_per_spmv = 1 + int(np.diff(ptr).max() > 32)
    x = torch.rand(n, dtype=torch.float64, device=dev)
    y = torch.zeros(n, dtype=torch.float64, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    # The K timed products are captured once in a CUDA graph and replayed, so
    # the timed region measures the device, not Python's launch overhead.
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for _ in range(args.warmup):
            api.Mlt(A, x, y)
    torch.cuda.current_stream().wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        for _ in range(args.steps):
            api.Mlt(A, x, y)
    graph.replay()  # one untimed replay after capture
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        # the same workload before and after the timed region, so the sampler
        # (100 ms period) sees the clocks the timed region ran at; nvidia-smi
        # takes a while to start, so the load runs until it reports (3 s at
        # most) and 0.4 s beyond
        first_until = time.time() + 3.0
        while time.time() < first_until and len(clk.lines) < 2:
            graph.replay()
            torch.cuda.synchronize()
        soak_until = time.time() + 0.4
        while time.time() < soak_until:
            graph.replay()
            torch.cuda.synchronize()
        ev0.record(stream)
        graph.replay()
        ev1.record(stream)
        torch.cuda.synchronize()
        soak_until = time.time() + 0.4
        while time.time() < soak_until:
            graph.replay()
            torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1) / args.steps
    value, ms_max = job_throughput(ms, B, world, dev)
    kernel_gbs = B / (ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak()

    # e2e: host (pinned) x in, y out, every step, through the C ABI's
    # pipelined host-buffer batch (the copy of x_{i+1} in, product i and the
    # copy of y_{i-1} out overlap); G host vectors per call.  Each call fills
    # and drains the pipeline once (one copy direction alone at each end),
    # so the K steps go in as few calls as 64-vector buffers allow.
    G = max(1, min(args.steps, 64))
    xh = torch.empty((G, n), dtype=torch.float64).pin_memory()
    yh = torch.empty((G, n), dtype=torch.float64).pin_memory()
    xh.copy_(x.cpu().expand(G, n))
    sp = ctypes.c_void_p(stream.cuda_stream)

    def host_batch(count):
        _lib.check(L.sb2_mlt_host_batch(A.handle, 0, 1.0, count, ctypes.c_void_p(xh.data_ptr()),
                                        ctypes.c_void_p(yh.data_ptr()), sp), "sb2_mlt_host_batch")
    for _ in range(max(2, args.warmup)):
        host_batch(G)
    barrier()
    torch.cuda.synchronize()
    ev0.record(stream)
    left = args.steps
    while left > 0:
        host_batch(min(G, left))
        left -= G
    ev1.record(stream)
    torch.cuda.synchronize()
    e2e, e2e_ms = job_throughput(ev0.elapsed_time(ev1) / args.steps, B, world, dev)
    ok = bool(np.array_equal(yh.numpy(), np.broadcast_to(y.cpu().numpy(), (G, n))))

    extras = {}
    if rank == 0 and not args.no_extras:
        extras = run_extras(api, matgen, torch, dev, args.extras,
                            cpu=(world == 1 and not args.no_cpu_solves), gmres_grid=args.gmres_grid,
                            batch_systems=args.batch_systems, batch_plan=args.batch_plan)

    cpu = None
    if rank == 0 and world == 1:
        gbs, cnt, th, wall, kind = cpu_reference_spmv(ptr, ind, val, args.cpu_seconds,
                                                      min(host_threads(), 64))
        cpu = {"value": round(gbs, 3), "unit": "GB/s", "cores": th, "kind": kind,
               "sample": f"{cnt} Seldon MltAdd products of the same 128^3 matrix on {th} "
                         f"threads in {wall:.1f} s"}

    if rank == 0:
        traffic = read_traffic()
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max, 5),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, seldon_b200/matgen.py)",
            "config": {"workload": WORKLOAD, "nnz": int(nnz), "n": int(n),
                       "bytes_per_step": int(B), "l2": "inputs 217 MB > 126 MB L2",
                       "parallelism": f"replicas x{world}"},
            # 2 flops (one multiply, one add) per stored entry and product
            "gflops": round(world * 2 * nnz / (ms_max * 1e-3) / 1e9, 2),
            "roofline": {"bound": "hbm", "achieved": round(kernel_gbs, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(kernel_gbs / peak, 4),
                         "traffic": traffic, "peak_source": peak_kind,
                         "kernel": "sb2::sell_slices_kernel<256, true>"},
            "e2e": {"value": round(e2e, 2), "unit": "GB/s", "h2d_bytes_per_step": 8 * n,
                    "d2h_bytes_per_step": 8 * n, "ms_per_step": round(e2e_ms, 4),
                    "gflops": round(world * 2 * nnz / (e2e_ms * 1e-3) / 1e9, 2),
                    "api": f"sb2_mlt_host_batch, {G} pinned host vectors per call",
                    "matches_device_result": ok},
            "gpu_launches": args.steps * launches_per_spmv,
            "timing": "K products captured in one CUDA graph, CUDA events around one replay",
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        line.update(extras)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_extras(api, matgen, torch, dev, which="all", cpu=True, gmres_grid=128, batch_systems=4096,
               batch_plan=None):
    """Time-to-solution figures on the other configurations (device-timed).
    `which`: comma list of c1, c3, gmres, krylov, zipf, batch, adjoint,
    assemble, ilu0, or all.  With `cpu`, the reference's own solvers then run on the
    host cores on the same systems (after every device measurement, so they
    do not disturb it) and each record gains a `cpu_reference` entry."""
    out = {}
    names = {"c1", "c3", "gmres", "krylov", "zipf", "batch", "adjoint", "assemble", "ilu0"}
    want = names if which == "all" else set(w.strip() for w in which.split(","))
    unknown = want - names
    if unknown:
        raise SystemExit(f"unknown extras: {sorted(unknown)}")

    def timed(fn, reps=1):
        best, r = None, None
        for _ in range(reps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            r = fn()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        return best, r

    jobs = []  # (record key, function run on the host afterwards)
    # records whose CPU comparison matters most go last: the line's tail is
    # what a truncated log keeps
    if "zipf" in want:
        out.update(extra_zipf(api, matgen, torch, dev, timed))
    if "assemble" in want:
        out.update(extra_assemble(api, matgen, torch, dev, timed))
    if "ilu0" in want:
        out.update(extra_ilu0(api, matgen, torch, dev, timed))
    if "adjoint" in want:
        out["adjoint_aniso512"] = run_adjoint(matgen, torch, dev, timed)
    if "batch" in want:
        key = "batch_lap2d_4096" if batch_systems == 4096 else f"batch_lap2d_{batch_systems}"
        out[key] = run_batch(api, matgen, torch, dev, timed, jobs, nsys=batch_systems,
                             plan=batch_plan)
    if "krylov" in want:
        out.update(extra_krylov(api, matgen, torch, dev, timed, jobs, gmres_grid))
    if "c1" in want:
        out.update(extra_c1(api, matgen, torch, dev, timed, jobs))
    if "gmres" in want:
        out.update(extra_gmres(api, matgen, torch, dev, timed, jobs, gmres_grid))
    if "c3" in want:
        out.update(extra_c3(api, matgen, torch, dev, timed, jobs))
    if cpu and jobs:
        run_cpu_jobs(out, jobs)
    return out


def _reference_fast():
    """The reference compiled at -O3 from its headers (oracle/_ref); the
    parity build (for residual checks) beside it."""
    from oracle.pyoracle import REF_FAST_SO, REF_SO, Reference
    if not (Reference.available(REF_FAST_SO) and Reference.available(REF_SO)):
        return None, None
    return Reference(REF_FAST_SO), Reference(REF_SO)


def cpu_model():
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_cpu_jobs(out, jobs):
    """Run the reference's host solves, one thread each (Seldon is
    single-threaded; ctypes releases the interpreter lock during the call),
    all at once, and attach each result to its record.  Jobs that use several
    threads themselves (the batch) run afterwards, alone."""
    single = [(k, f) for k, f, multi in jobs if not multi]
    multi = [(k, f) for k, f, multi in jobs if multi]
    results = {}

    def run(key, fn):
        try:
            results[key] = fn()
        except Exception as e:  # the checker is optional here
            results[key] = {"unavailable": str(e)[:160]}
    ths = [threading.Thread(target=run, args=kf) for kf in single]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    for k, f in multi:
        run(k, f)
    for k, r in results.items():
        out[k]["cpu_reference"] = r


def _cpu_solve(which, ptr, ind, val, b, x_gpu, sym=False, precond=0, restart=10, tol=1e-10,
               max_iter=20000):
    """The reference's solver on the host (one core), timed; its x compared
    with the device's, both residuals recomputed by the reference's MltAdd."""
    fast, parity = _reference_fast()
    if fast is None:
        return {"unavailable": "oracle/_ref is not built"}
    n = ptr.size - 1
    # a solve under 0.2 s is repeated (best of up to 5): the host is shared and
    # the other records' solves run beside it, so one short run varies by 2x
    dt, reps = None, 0
    while reps < 5 and (dt is None or dt < 0.2):
        t0 = time.perf_counter()
        xr, code, it = fast.solve(which, ptr, ind, val, b, sym=sym, precond=precond, tol=tol,
                                  max_iter=max_iter, restart=restart)
        d = time.perf_counter() - t0
        dt = d if dt is None else min(dt, d)
        reps += 1

    def relres(x):
        r = parity.mltadd(n, n, ptr, ind, val, -1.0, x, 1.0, b, sym=sym)
        return float(np.linalg.norm(r) / np.linalg.norm(b))
    return {"ms": round(dt * 1e3, 1), "runs": reps, "iterations": it, "error_code": code,
            "true_rel_residual": relres(xr), "gpu_true_rel_residual": relres(x_gpu),
            "forward_diff_gpu_vs_reference": float(np.linalg.norm(x_gpu - xr) /
                                                  np.linalg.norm(xr)),
            "cores": 1, "host_threads": host_threads(), "cpu": cpu_model(),
            "build": "Seldon's templates from the reference's headers, g++ -O3"}


def extra_c1(api, matgen, torch, dev, timed, jobs):
    """CG, identity, 100^2 Laplacian stored RowSymSparse."""
    ptr, ind, val = matgen.lap2d(100)
    n = ptr.size - 1
    xs = np.random.default_rng(100).uniform(-1, 1, n)
    bh = matgen.matvec(ptr, ind, val, xs)
    b = torch.as_tensor(bh, device=dev)
    up, ui, uv = matgen.upper(ptr, ind, val)
    S = api.RowSymSparse(n, up, ui, uv)

    def cg_c1():
        X = torch.zeros(n, dtype=torch.float64, device=dev)
        it = api.Iteration(10000, 1e-10)
        it.HideMessages()
        api.Cg(S, X, b, api.Preconditioner_Base(), it)
        return it, X
    cg_c1()
    ms, (it, X) = timed(cg_c1, reps=5)
    x = X.cpu().numpy()
    jobs.append(("cg_lap2d_100", lambda: _cpu_solve("cg", up, ui, uv, bh, x, sym=True), False))
    return {"cg_lap2d_100": {"ms": round(ms, 3), "iterations": it.GetNumberIteration(),
                             "rel_residual": it.history[-1][1], "timing": "best of 5"}}


def extra_c3(api, matgen, torch, dev, timed, jobs):
    """FP64 CG and FP32/FP64 iterative refinement on the 192^3 Poisson problem."""
    out = {}
    ptr, ind, val = matgen.poisson3d(192)
    n = ptr.size - 1
    xs = np.random.default_rng(192).uniform(-1, 1, n)
    bh = matgen.matvec(ptr, ind, val, xs)
    b = torch.as_tensor(bh, device=dev)
    A = api.RowSparse(n, n, ptr, ind, val)

    def cg_c3():
        X = torch.zeros(n, dtype=torch.float64, device=dev)
        it = api.Iteration(20000, 1e-10)
        it.HideMessages()
        api.Cg(A, X, b, api.Preconditioner_Base(), it)
        return it, X
    cg_c3()  # warm: first call sets up the chained solver's state
    ms, (it, X) = timed(cg_c3, reps=3)
    X64 = X.cpu().numpy()
    fe = float(np.linalg.norm(X64 - xs) / np.linalg.norm(xs))
    per_it = (spmv_bytes(n, n, ind.size) + 10 * 8 * n)
    out["cg_fp64_poisson192"] = {"ms": round(ms, 2), "iterations": it.GetNumberIteration(),
                                 "rel_residual": it.history[-1][1], "forward_error": fe,
                                 "gbs_per_iteration_model": round(
                                     per_it * it.GetNumberIteration() / (ms * 1e-3) / 1e9, 1),
                                 "timing": "best of 3"}
    jobs.append(("cg_fp64_poisson192",
                 lambda: _cpu_solve("cg", ptr, ind, val, bh, X64), False))
    # mixed precision: FP32 inner CG, FP64 outer residual/update to 1e-10
    for key, restarted, inner in (("ir_reliable_poisson192", False, 1e-2),
                                  ("ir_restarted_poisson192", True, 1e-5)):
        def ir():
            Xi = torch.zeros(n, dtype=torch.float64, device=dev)
            code, info = api.IterativeRefinement(A, Xi, b, tol=1e-10, inner_tol=inner,
                                                 restarted=restarted)
            return code, info, Xi
        ir()
        ms_ir, (code, info, Xi) = timed(ir, reps=3)
        Xi = Xi.cpu().numpy()
        # the true FP64 residual, recomputed here on the host
        true_rel = float(np.linalg.norm(matgen.matvec(ptr, ind, val, Xi) - b.cpu().numpy()) /
                         np.linalg.norm(b.cpu().numpy()))
        out[key] = {"ms": round(ms_ir, 2), "inner_tol": inner, "error_code": code,
                    "outer_iter": info["outer_iter"], "inner_iter": info["inner_iter"],
                    "rel_residual_fp64": info["rel_residual"],
                    "rel_residual_host_check": true_rel,
                    "forward_error_vs_fp64_cg": float(np.linalg.norm(Xi - X64) / np.linalg.norm(X64)),
                    "forward_error_vs_xstar": float(np.linalg.norm(Xi - xs) / np.linalg.norm(xs)),
                    "speedup_vs_fp64_cg": round(ms / ms_ir, 3), "timing": "best of 3"}
    out["ir_reliable_poisson192"]["config_deviation"] = (
        "reliable updates, correction each time the FP32 residual drops by 1e-2 "
        "(the configuration's inner tolerance 1e-5 is ir_restarted_poisson192)")
    return out


def gmres_bytes(n, nnz, iterations, m, vw, mw, variant):
    """Bytes that the passes of a GMRES(m) solve read and write, for a solve
    that took `iterations` Arnoldi steps and restarts every m steps (L2 can
    serve part of them: w between the MGS passes, and part of the basis when
    it is not much larger than L2): per step i of a cycle the product
    (nnz*(mw+4) + 4(n+1) + 2*n*vw) plus the orthogonalization's vector
    passes, and per restart the FP64 residual product and the update
    x += V y.  vw: basis element bytes; mw: matrix value bytes.
      mgs   Seldon's modified Gram-Schmidt (Gmres.cxx:127-132): pass k reads
            w, V_k and V_{k+1} and writes w (4 vectors), i+1 passes, then
            V_{i+1} = w / h (2 vectors)
      cgs2  CGS2 with the second projection delayed a step: step i's dots
            read V_0..V_{i-1}, u and w, its update pass reads V_0..V_{i-1},
            u and w and writes V_i and u (2i + 6 vectors); the step that
            ends a cycle reads V and u once more (a full cycle: dots only;
            a converged one: with the product, which then goes unused)"""
    spmv = nnz * (mw + 4) + 4 * (n + 1) + 2 * n * vw
    spmv64 = nnz * 12 + 4 * (n + 1) + 3 * n * 8  # residual: x in, b in, r out
    total, done = 0, 0
    while done < iterations:
        steps = min(m, iterations - done)
        for i in range(steps):
            vec = 4 * (i + 1) + 2 if variant == "mgs" else 2 * i + 6
            total += spmv + vec * n * vw
        if variant == "cgs2":
            total += (steps + 1) * n * vw if steps == m else spmv + (steps + 2) * n * vw
        total += spmv64 + steps * n * vw + 2 * n * 8
        done += steps
    return total


def extra_gmres(api, matgen, torch, dev, timed, jobs, g=GRID):
    """GMRES(30) + Jacobi on the 128^3 convection-diffusion problem: Seldon's
    modified Gram-Schmidt order, the CGS2 variant, and the iterative
    refinement whose inner solve is GMRES(30) with an FP32 basis."""
    ptr, ind, val = matgen.convdiff3d(g)
    n = ptr.size - 1
    xs = np.random.default_rng(g).uniform(-1, 1, n)
    bh = matgen.matvec(ptr, ind, val, xs)
    b = torch.as_tensor(bh, device=dev)
    A = api.RowSparse(n, n, ptr, ind, val)
    J = api.JacobiPreconditioner()
    peak, _ = measured_peak()

    def gm(orth):
        def run():
            X = torch.zeros(n, dtype=torch.float64, device=dev)
            it = api.Iteration(20000, 1e-10)
            it.HideMessages()
            it.SetRestart(30)
            api.Gmres(A, X, b, J, it, orthogonalization=orth)
            return it, X
        return run

    def host_relres(x):
        return float(np.linalg.norm(matgen.matvec(ptr, ind, val, x) - bh) / np.linalg.norm(bh))
    out = {}
    xs_gpu = {}
    sfx = f"convdiff{g}"
    k_mgs, k_cgs2, k_ir = (f"gmres30_jacobi_{sfx}", f"gmres30_cgs2_jacobi_{sfx}",
                           f"ir_gmres30_jacobi_{sfx}")
    for key, orth in ((k_mgs, "mgs"), (k_cgs2, "cgs2")):
        gm(orth)()  # warm-up: the Krylov basis (0.5 GB) is mapped into the pool once
        ms, (it, X) = timed(gm(orth), reps=2)
        x = X.cpu().numpy()
        xs_gpu[orth] = x
        nbytes = gmres_bytes(n, ind.size, it.GetNumberIteration(), 30, 8, 8, orth)
        out[key] = {"ms": round(ms, 2), "iterations": it.GetNumberIteration(),
                    "rel_residual": it.history[-1][1], "ms_per_iteration":
                    round(ms / it.GetNumberIteration(), 4),
                    "gbs_model": round(nbytes / (ms * 1e-3) / 1e9, 1),
                    "frac_of_measured_peak": round(nbytes / (ms * 1e-3) / 1e9 / peak, 3),
                    "timing": "best of 2"}
    out[k_cgs2]["forward_diff_vs_mgs"] = float(
        np.linalg.norm(xs_gpu["cgs2"] - xs_gpu["mgs"]) / np.linalg.norm(xs_gpu["mgs"]))
    out[k_cgs2]["speedup_vs_mgs"] = round(
        out[k_mgs]["ms"] / out[k_cgs2]["ms"], 3)

    def ir():
        X = torch.zeros(n, dtype=torch.float64, device=dev)
        code, info = api.IterativeRefinement(A, X, b, M=J, tol=1e-10, solver="gmres", restart=30)
        return code, info, X
    ir()
    ms, (code, info, X) = timed(ir, reps=2)
    x = X.cpu().numpy()
    best64 = min(out[k_mgs]["ms"], out[k_cgs2]["ms"])
    nbytes = gmres_bytes(n, ind.size, info["inner_iter"], 30, 4, 4, "cgs2")
    out[k_ir] = {
        "ms": round(ms, 2), "error_code": code, "outer_iter": info["outer_iter"],
        "inner_iter": info["inner_iter"], "rel_residual_fp64": info["rel_residual"],
        "rel_residual_host_check": host_relres(x),
        "forward_error_vs_fp64_gmres": float(np.linalg.norm(x - xs_gpu["mgs"]) /
                                             np.linalg.norm(xs_gpu["mgs"])),
        "forward_error_vs_xstar": float(np.linalg.norm(x - xs) / np.linalg.norm(xs)),
        "speedup_vs_fp64_gmres_mgs": round(out[k_mgs]["ms"] / ms, 3),
        "speedup_vs_best_fp64_gmres": round(best64 / ms, 3),
        "gbs_model": round(nbytes / (ms * 1e-3) / 1e9, 1),
        "frac_of_measured_peak": round(nbytes / (ms * 1e-3) / 1e9 / peak, 3),
        "timing": "best of 2"}
    x = xs_gpu["mgs"]
    jobs.append((k_mgs,
                 lambda: _cpu_solve("gmres", ptr, ind, val, bh, x, precond=1, restart=30), False))
    return out


def krylov_bytes(which, n, nnz, jacobi, iterations, restart=10):
    """Bytes a persistent BiCg, BiCgStab, Cgs, TfQmr, QCgs, Cgne, Lsqr, BiCgcr,
    QmrSym, Symmlq, MinRes, Gcr or BiCgStabl solve of
    `iterations` (Seldon's count) reads and writes: its products
    (nnz*12 + 4(n+1) each) plus the vector streams of its passes and product
    epilogues, the gathered operand counted once per product.
      bicgstab  per loop (two counted iterations): two products, 21 vectors
                (+4 with Jacobi: two diagonal reads, phat, shat)
      cgs       per loop: two products, 18 vectors (+4 with Jacobi)
      tfqmr     per loop: two products, 30 vectors (+2 with Jacobi)
      qcgs      per loop: two products, 29 vectors (+4 with Jacobi)
      bicg      per loop: a product by A and one by A^T, 19 vectors (+4 with
                Jacobi)
      cgne      per loop: a product by A and one by A^T, 12 vectors (+2 with
                Jacobi)
      lsqr      per loop: a product by A and one by A^T, 12 vectors (no
                preconditioner)
      minres    per iteration: one product, 20 vectors (+1 with Jacobi)
      bicgcr    per iteration: one product, 19 vectors (+1 with Jacobi)
      qmrsym    per iteration: one product, 23 vectors (+1 with Jacobi)
      symmlq    per iteration: one product, 18 vectors (+1 with Jacobi)
      gcr       per inner step j of a cycle (two counted iterations): two
                products, 2j + 14 vectors (the j + 1 projections and the
                j + 1 terms of the new direction; +2 with Jacobi); per cycle
                2 more (p_0 = r / ||r||)
      bicgstabl per BiCG step j of a cycle (two counted iterations): two
                products and 6j + 15 vectors (the j + 1 u and r updates of
                both passes; +4 with Jacobi); per cycle of l steps the MR
                part's Gram-Schmidt, 3 l(l + 1) / 2, and the update pass,
                2l + 7
    L2 serves part of the re-reads, so the figure bounds DRAM traffic from
    above."""
    prod = nnz * 12 + 4 * (n + 1)
    if which == "minres":
        return iterations * (prod + (20 + jacobi) * n * 8)
    if which == "bicgcr":
        return iterations * (prod + (19 + jacobi) * n * 8)
    if which == "qmrsym":
        return iterations * (prod + (23 + jacobi) * n * 8)
    if which == "symmlq":
        return iterations * (prod + (18 + jacobi) * n * 8)
    if which == "gcr":
        steps, cycle, total = int(iterations // 2), max((restart + 1) // 2, 1), 0
        for k in range(steps):
            j = k % cycle
            total += 2 * prod + (2 * j + 14 + 2 * jacobi + (2 if j == 0 else 0)) * n * 8
        return total
    if which == "bicgstabl":
        l, steps, total = max(restart, 1), int(iterations // 2), 0
        for k in range(steps):
            j = k % l
            total += 2 * prod + (6 * j + 15 + 4 * jacobi) * n * 8
            if j == l - 1:
                total += (3 * l * (l + 1) // 2 + 2 * l + 7) * n * 8
        return total
    vec = {"bicgstab": 21 + 4 * jacobi, "cgs": 18 + 4 * jacobi, "tfqmr": 30 + 2 * jacobi,
           "qcgs": 29 + 4 * jacobi, "bicg": 19 + 4 * jacobi, "cgne": 12 + 2 * jacobi,
           "lsqr": 12}[which]
    return iterations / 2 * (2 * prod + vec * n * 8)


def extra_krylov(api, matgen, torch, dev, timed, jobs, g=GRID):
    """Seldon's other drivers, each one persistent kernel per solve, against
    the reference's own drivers on one host core, all with Jacobi:
    BiCg, BiCgStab, Cgs, QCgs, TfQmr and BiCgStabl(4) on the 128^3
    convection-diffusion operator, MinRes, QmrSym and Symmlq on the 128^3
    Poisson operator,
    Gcr(10), Cgne, Lsqr and BiCgcr on the 64^3 convection-diffusion operator
    (their iteration counts grow with the grid: Gcr's 768 at 32^3, 1494 at
    48^3; Cgne's 6080 at 48^3, 10072 at 64^3, the normal equations squaring
    the condition number, Lsqr's 7020 at 48^3; BiCgcr's 180 at 40^3, 1113 at
    64^3).  Lsqr uses no preconditioner.  BiCg.cxx:46-134, BiCgStab.cxx:43-145,
    Cgs.cxx:45-132, QCgs.cxx:46-165, TfQmr.cxx:44-243, BiCgStabl.cxx:43-180,
    MinRes.cxx:46-153, Gcr.cxx:45-141, Cgne.cxx:40-127, BiCgcr.cxx:44-118,
    Lsqr.cxx:40-135, QmrSym.cxx:41-165, Symmlq.cxx:45-161.

    BiCg's, Cgne's and Lsqr's products by A^T are, in the reference,
    MltAdd(alpha, SeldonTrans, M, X, beta, Y)'s generic loop over every
    (j, i) pair with the element access M(j, i) (Functions_MatVect.cxx:
    1274-1317): n^2 row searches a product, so their host solves are not
    run at these sizes."""
    peak, _ = measured_peak()
    out = {}
    fns = {"bicg": api.BiCg, "bicgstab": api.BiCgStab, "cgs": api.Cgs, "qcgs": api.QCgs,
           "tfqmr": api.TfQmr, "bicgstabl": api.BiCgStabl, "gcr": api.Gcr,
           "cgne": api.Cgne, "lsqr": api.Lsqr, "bicgcr": api.BiCgcr, "minres": api.MinRes,
           "qmrsym": api.QmrSym, "symmlq": api.Symmlq}
    restarts = {"bicgstabl": 4, "gcr": 10}
    systems = {}
    for which, fn in fns.items():
        op = "poisson" if which in ("minres", "qmrsym", "symmlq") else "convdiff"
        gg = g // 2 if which in ("gcr", "cgne", "lsqr", "bicgcr") else g
        if (op, gg) not in systems:
            ptr, ind, val = matgen.poisson3d(gg) if op == "poisson" else matgen.convdiff3d(gg)
            n = ptr.size - 1
            xs = np.random.default_rng(gg + 1).uniform(-1, 1, n)
            bh = matgen.matvec(ptr, ind, val, xs)
            systems[(op, gg)] = (ptr, ind, val, n, bh, torch.as_tensor(bh, device=dev),
                                 api.RowSparse(n, n, ptr, ind, val), api.JacobiPreconditioner())
        ptr, ind, val, n, bh, b, A, J = systems[(op, gg)]
        rs = restarts.get(which, 10)

        def run():
            X = torch.zeros(n, dtype=torch.float64, device=dev)
            it = api.Iteration(40000, 1e-10)
            it.SetRestart(rs)
            it.HideMessages()
            code = fn(A, X, b, J, it)
            return code, it, X
        run()
        ms, (code, it, X) = timed(run, reps=3)
        x = X.cpu().numpy()
        nit = it.GetNumberIteration()
        nbytes = krylov_bytes(which, n, ind.size, which != "lsqr", nit, rs)
        key = f"{which}{rs if which in restarts else ''}_jacobi_{op}{gg}"
        out[key] = {"ms": round(ms, 2), "error_code": code, "iterations": nit,
                    "us_per_iteration": round(ms * 1e3 / max(nit, 1), 1),
                    "rel_residual_host_check": float(
                        np.linalg.norm(matgen.matvec(ptr, ind, val, x) - bh) / np.linalg.norm(bh)),
                    "gbs_model": round(nbytes / (ms * 1e-3) / 1e9, 1),
                    "frac_of_measured_peak": round(nbytes / (ms * 1e-3) / 1e9 / peak, 3),
                    "timing": "best of 3"}
        if which in ("bicg", "cgne", "lsqr"):
            out[key]["cpu_reference"] = {
                "unavailable": f"the reference's product by A^T is its generic M(j, i) loop "
                               f"(Functions_MatVect.cxx:1274-1317): {n}^2 row searches a product"}
            continue
        jobs.append((key, (lambda w, xg, p, i, v, bb, m: lambda: _cpu_solve(
            w, p, i, v, bb, xg, precond=1, restart=m))(which, x, ptr, ind, val, bh, rs), False))
    return out


def extra_zipf(api, matgen, torch, dev, timed):
    """SpMV on the Zipf(1.5) random matrix, n = 10^6; beside it the gather
    bound: the same index and value streams and x gathers with no rows
    (sb2_probe_gather), the least time any row binning can take."""
    from seldon_b200 import _lib
    L = _lib.load()
    ptr, ind, val = matgen.zipf_csr(1_000_000, seed=1)
    n = ptr.size - 1
    A = api.RowSparse(n, n, ptr, ind, val)
    x = torch.rand(n, dtype=torch.float64, device=dev)
    y = torch.zeros(n, dtype=torch.float64, device=dev)
    for _ in range(3):
        api.Mlt(A, x, y)
    ms, _ = timed(lambda: [api.Mlt(A, x, y) for _ in range(20)], reps=3)
    Bz = spmv_bytes(n, n, ind.size)
    us = ms / 20 * 1e3
    out = {"gbs": round(Bz / (us * 1e-6) / 1e9, 1), "gflops": round(2 * ind.size / (us * 1e-6) / 1e9, 1),
           "nnz": int(ind.size), "us": round(us, 1)}
    di = torch.as_tensor(ind, device=dev)
    dv = torch.as_tensor(val, device=dev)
    part = torch.empty(4096, dtype=torch.float64, device=dev)
    nb = ctypes.c_int(0)
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def probe(with_val):
        def run():
            for _ in range(20):
                _lib.check(L.sb2_probe_gather(int(ind.size), ctypes.c_void_p(di.data_ptr()),
                                              ctypes.c_void_p(dv.data_ptr()) if with_val else None,
                                              ctypes.c_void_p(x.data_ptr()),
                                              ctypes.c_void_p(part.data_ptr()), 4096,
                                              ctypes.byref(nb), sp), "sb2_probe_gather")
        run()
        t, _ = timed(run, reps=3)
        return t / 20 * 1e3
    pv, pi = probe(True), probe(False)
    out["gather_bound"] = {
        "us": round(pv, 1), "index_and_gather_only_us": round(pi, 1),
        "gbs_algorithmic": round(Bz / (pv * 1e-6) / 1e9, 1),
        "gather_sectors_per_s": round(ind.size / (pi * 1e-6), 1),
        "spmv_frac_of_bound": round(pv / us, 3),
        "what": "sum of val[k]*x[ind[k]] over all 68.8M entries in one stream, no rows "
                "(sb2_probe_gather): the same index, value and x traffic as the product"}
    return {"spmv_zipf_1e6": out}


def _shuffled_triplets(matgen, torch, dev, g, seed=3):
    ptr, ind, val = matgen.convdiff3d(g)
    m = ptr.size - 1
    rows = np.repeat(np.arange(m, dtype=np.int32), np.diff(ptr))
    gen = torch.Generator(device=dev).manual_seed(seed)
    perm = torch.randperm(ind.size, device=dev, generator=gen)
    return m, [torch.as_tensor(a, device=dev)[perm].contiguous() for a in (rows, ind, val)]


def extra_assemble(api, matgen, torch, dev, timed):
    """COO -> CSR assembly (ConvertMatrix_from_Coordinates) of the 128^3
    convection-diffusion operator's 14.6M triplets in random order, through
    the public call (output allocation included); Seldon's own conversion
    timed beside it on the 64^3 operator's triplets."""
    m, (r, c, v) = _shuffled_triplets(matgen, torch, dev, 128)
    nnz = r.numel()
    for _ in range(3):
        api.ConvertMatrix_from_Coordinates(r, c, v, 0, m, m)
    ms, _ = timed(lambda: api.ConvertMatrix_from_Coordinates(r, c, v, 0, m, m), reps=5)
    # least traffic any assembly needs: triplets in, ind/val/ptr out
    min_bytes = nnz * 16 + nnz * 12 + 4 * (m + 1)
    out = {"nnz": nnz, "ms": round(ms, 3), "entries_per_s": round(nnz / ms * 1e3, 1),
           "min_bytes_gbs": round(min_bytes / (ms * 1e-3) / 1e9, 1)}
    try:
        from oracle.pyoracle import REF_FAST_SO, Reference
        if Reference.available(REF_FAST_SO):
            R = Reference(REF_FAST_SO)
            ms_, (rs, cs, vs) = _shuffled_triplets(matgen, torch, dev, 64)
            rs, cs, vs = (t.cpu().numpy() for t in (rs, cs, vs))
            t0 = time.perf_counter()
            R.coo_to_csr(rs, cs, vs, 0, ms_, ms_)
            dt = time.perf_counter() - t0
            out["cpu_reference"] = {"nnz": int(rs.size), "s": round(dt, 3),
                                    "entries_per_s": round(rs.size / dt, 1), "cores": 1}
    except Exception as e:  # the checker is optional here
        out["cpu_reference"] = {"unavailable": str(e)[:120]}
    return {"coo_to_csr_conv128": out}


def extra_ilu0(api, matgen, torch, dev, timed):
    """ILU(0) of the 128^3 convection-diffusion operator: factored on the
    device (GetIlu0's order), applied (SolveLU sweeps, level-scheduled), and
    BiCGSTAB with it against BiCGSTAB without.  Seldon's own apply of the
    same factor is timed on one host core beside it."""
    ptr, ind, val = matgen.convdiff3d(128)
    n = ptr.size - 1
    A = api.RowSparse(n, n, ptr, ind, val)
    M = api.IlutPreconditioning()
    M.SetFactorisationType(M.ILU_0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    M.FactorizeMatrix(A)
    torch.cuda.synchronize()
    out = {"n": n, "nnz": int(ind.size), "factor_s": round(time.perf_counter() - t0, 3)}
    r = torch.rand(n, dtype=torch.float64, device=dev)
    z = torch.empty_like(r)
    for _ in range(3):
        M.Solve(A, r, z)
    ms, _ = timed(lambda: [M.Solve(A, r, z) for _ in range(10)])
    out["apply_ms"] = round(ms / 10, 3)
    # factor entries and the vector traffic one apply needs at least
    out["apply_min_gbs"] = round((ind.size * 12 + n * 8 * 6) / (ms / 10 * 1e-3) / 1e9, 1)
    b = torch.as_tensor(matgen.matvec(ptr, ind, val, np.random.default_rng(1).uniform(-1, 1, n)),
                        device=dev)
    for key, P in (("bicgstab_plain", api.Preconditioner_Base()), ("bicgstab_ilu0", M)):
        X = torch.zeros(n, dtype=torch.float64, device=dev)

        def solve():
            X.zero_()
            it = api.Iteration(2000, 1e-8)
            it.HideMessages()
            api.BiCgStab(A, X, b, P, it)
            return it
        solve()
        ms, it = timed(solve)
        out[key] = {"ms": round(ms, 2), "iterations": it.GetNumberIteration()}
    try:
        from oracle.pyoracle import REF_FAST_SO, Reference
        if Reference.available(REF_FAST_SO):
            R = Reference(REF_FAST_SO)
            R.ilut_factor(ptr, ind, val, type_ilu=R.ILU_0)
            rh = r.cpu().numpy()
            t0 = time.perf_counter()
            R.ilut_solve(rh)
            out["cpu_reference_apply_ms"] = round((time.perf_counter() - t0) * 1e3, 2)
    except Exception as e:  # the checker is optional here
        out["cpu_reference_apply_ms"] = f"unavailable: {str(e)[:100]}"
    return {"ilu0_conv128": out}


def run_batch(api, matgen, torch, dev, timed, jobs=None, nsys=4096, sample_every=8, plan=None):
    """4096 shifted 2D Laplacians (side uniform in [8,140]) in one persistent
    launch, against a loop of plain FP64 CG calls over every 8th system; on
    the host, the reference's Cg on the same sample, K systems at a time on K
    threads."""
    from seldon_b200 import _lib
    rng = np.random.default_rng(7)
    gs = rng.integers(8, 141, nsys)
    cache, systems, rhs = {}, [], []
    for g in gs:
        g = int(g)
        if g not in cache:
            cache[g] = matgen.lap2d(g, shift=0.01)
        p, i, v = cache[g]
        systems.append(cache[g])
        rhs.append(matgen.matvec(p, i, v, rng.uniform(-1, 1, g * g)))
    Bt = api.Batch(systems)
    b = torch.as_tensor(np.concatenate(rhs), device=dev)
    X = torch.zeros(Bt.m, dtype=torch.float64, device=dev)
    its = torch.zeros(Bt.nsys, dtype=torch.int32, device=dev)
    rr = torch.zeros(Bt.nsys, dtype=torch.float64, device=dev)
    t0 = time.perf_counter()
    if plan:  # threads,warp_max[,cluster,cluster_min]
        Bt.set_plan(*(int(v) for v in plan.split(",")))
    else:
        Bt.autotune(X, b, tol=1e-9)
    tune_s = time.perf_counter() - t0
    threads, warp_max = Bt.plan()
    cluster, cluster_min = Bt.cluster_plan()
    out = {"systems": nsys, "rows": Bt.m, "nnz": int(sum(s[1].size for s in systems)),
           "tol": 1e-9, "plan": {"threads": threads, "warp_max_rows": warp_max,
                                 "cluster_ctas": cluster, "cluster_min_rows": cluster_min,
                                 "autotune_s": round(tune_s, 2)}}
    rows = np.array([s[0].size - 1 for s in systems], dtype=np.float64)
    nnzs = np.array([s[1].size for s in systems], dtype=np.float64)
    peak, _ = measured_peak()
    for key, mixed in (("mixed", True), ("fp64", False)):
        Bt.solve(X, b, its, rr, tol=1e-9, mixed=mixed)
        ms, res = timed(lambda: Bt.solve(X, b, its, rr, tol=1e-9, mixed=mixed), reps=2)
        it_s = its.cpu().numpy().astype(np.float64)
        # least traffic per iteration of one system: its matrix (values and
        # 2-byte columns), row pointers, and the vector passes (the product
        # gathers r and p and writes p and q; the update reads d or x, p, r, q
        # and writes d or x, r)
        vb, mb = (4, 6) if mixed else (8, 10)
        nbytes = float(np.sum(it_s * (nnzs * mb + rows * (4 + 10 * vb))))
        out[key] = {"ms": round(ms, 2), "systems_per_s": round(nsys / ms * 1e3, 1),
                    "converged": res.converged, "max_iter": res.max_iter,
                    "total_iter": res.total_iter, "max_rel_residual": res.max_rel_residual,
                    "gbs_model": round(nbytes / (ms * 1e-3) / 1e9, 1),
                    "frac_of_measured_hbm_peak": round(nbytes / (ms * 1e-3) / 1e9 / peak, 3)}
    # graph-captured launch (no host synchronisation inside)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        Bt.solve(X, b, its, rr, summary=False, tol=1e-9, mixed=True)
    g.replay()
    ms, _ = timed(g.replay)
    out["mixed_graph_ms"] = round(ms, 2)
    tot, n_loop = 0.0, 0
    for s in range(0, nsys, sample_every):
        p, i, v = systems[s]
        n = p.size - 1
        A = api.RowSparse(n, n, p, i, v)
        bs = torch.as_tensor(rhs[s], device=dev)
        Xs = torch.zeros(n, dtype=torch.float64, device=dev)

        def cg():
            Xs.zero_()
            itr = api.Iteration(10000, 1e-9)
            itr.HideMessages()
            api.Cg(A, Xs, bs, api.Preconditioner_Base(), itr)
        cg()
        ms, _ = timed(cg)
        tot += ms
        n_loop += 1
    per = tot / n_loop
    out["loop_fp64_cg"] = {"ms_per_system": round(per, 4), "systems_per_s": round(1e3 / per, 1),
                           "sample": f"every {sample_every}th system ({n_loop} calls)",
                           "est_ms_all": round(per * nsys, 1)}
    out["speedup_mixed_vs_loop"] = round(out["loop_fp64_cg"]["est_ms_all"] / out["mixed"]["ms"], 1)
    Bt.close()
    out["few_large_systems"] = run_batch_few_large(api, matgen, torch, dev, timed)
    if jobs is not None:
        sample = list(range(0, nsys, sample_every))
        jobs.append(("batch_lap2d_4096",
                     lambda: _cpu_batch(systems, rhs, sample, nsys, X.cpu().numpy(),
                                        np.concatenate([[0], np.cumsum([s[0].size - 1 for s in systems])])),
                     True))
    return out


def run_batch_few_large(api, matgen, torch, dev, timed, nsys=12, lo=150, hi=180):
    """Fewer large systems than the GPU's CTA slots (12 shifted 2D Laplacians,
    side U{150..180}): the autotuned plan, which may give each system a whole
    thread-block cluster, against one CTA per system."""
    rng = np.random.default_rng(9)
    systems, rhs = [], []
    for _ in range(nsys):
        g = int(rng.integers(lo, hi + 1))
        p, i, v = matgen.lap2d(g, shift=0.01)
        systems.append((p, i, v))
        rhs.append(matgen.matvec(p, i, v, rng.uniform(-1, 1, g * g)))
    Bt = api.Batch(systems)
    b = torch.as_tensor(np.concatenate(rhs), device=dev)
    X = torch.zeros(Bt.m, dtype=torch.float64, device=dev)
    its = torch.zeros(Bt.nsys, dtype=torch.int32, device=dev)
    rr = torch.zeros(Bt.nsys, dtype=torch.float64, device=dev)
    Bt.autotune(X, b, tol=1e-9)
    plan = Bt.plan() + Bt.cluster_plan()
    Bt.solve(X, b, its, rr, tol=1e-9)
    ms, res = timed(lambda: Bt.solve(X, b, its, rr, tol=1e-9), reps=3)
    Bt.set_plan(512, 0)
    Bt.solve(X, b, its, rr, tol=1e-9)
    ms_cta, _ = timed(lambda: Bt.solve(X, b, its, rr, tol=1e-9), reps=3)
    Bt.close()
    return {"systems": nsys, "rows": int(sum(s[0].size - 1 for s in systems)),
            "plan": {"threads": plan[0], "warp_max_rows": plan[1], "cluster_ctas": plan[2],
                     "cluster_min_rows": plan[3]},
            "ms": round(ms, 3), "converged": res.converged,
            "max_rel_residual": res.max_rel_residual,
            "ms_one_cta_per_system": round(ms_cta, 3),
            "speedup_vs_one_cta_per_system": round(ms_cta / ms, 2)}


def _cpu_batch(systems, rhs, sample, nsys, x_gpu, offs, tol=1e-9):
    """The reference's FP64 Cg on the sampled systems, K independent solves at
    a time on K host threads (one system per thread), timed as a whole."""
    fast, parity = _reference_fast()
    if fast is None:
        return {"unavailable": "oracle/_ref is not built"}
    K = max(1, min(host_threads(), 64))
    todo = list(sample)
    lock = threading.Lock()
    res = {}

    def worker():
        while True:
            with lock:
                if not todo:
                    return
                s = todo.pop()
            p, i, v = systems[s]
            xr, code, it = fast.solve("cg", p, i, v, rhs[s], tol=tol, max_iter=10000)
            res[s] = (xr, code, it)
    ths = [threading.Thread(target=worker) for _ in range(K)]
    t0 = time.perf_counter()
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    wall = time.perf_counter() - t0
    worst_rel, worst_fd, conv = 0.0, 0.0, 0
    for s, (xr, code, it) in res.items():
        p, i, v = systems[s]
        n = p.size - 1
        r = parity.mltadd(n, n, p, i, v, -1.0, xr, 1.0, rhs[s])
        worst_rel = max(worst_rel, float(np.linalg.norm(r) / np.linalg.norm(rhs[s])))
        xg = x_gpu[offs[s]:offs[s + 1]]
        worst_fd = max(worst_fd, float(np.linalg.norm(xg - xr) / np.linalg.norm(xr)))
        conv += int(code == 0)
    per_s = len(sample) / wall
    return {"systems": len(sample), "threads": K, "wall_ms": round(wall * 1e3, 1),
            "systems_per_s": round(per_s, 1), "est_ms_all": round(nsys / per_s * 1e3, 1),
            "converged": conv, "max_true_rel_residual": worst_rel,
            "max_forward_diff_gpu_mixed_vs_reference": worst_fd, "cpu": cpu_model(),
            "sample": f"every {nsys // len(sample)}th system, FP64 Cg to {tol}, "
                      f"{K} concurrent single-threaded solves"}


def run_adjoint(matgen, torch, dev, timed, g=512, n_fd=64, h=1e-6):
    """Adjoint CG on the 512^2 anisotropic graph Laplacian + 1e-3 I with
    theta ~ LogNormal(0,1): forward and backward times, and the gradient
    against an FP64 direct-solve gradient (all edges) and central differences
    (h = 1e-6) on 64 random edges."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as sl
    from seldon_b200 import autograd as ag
    rng = np.random.default_rng(11)
    n = g * g
    edges = matgen.grid_edges(g)
    E = edges.shape[0]
    theta0 = rng.lognormal(0.0, 1.0, E)
    bh = rng.normal(size=n)
    xt = rng.normal(size=n)
    lap = ag.GraphLaplacian(n, edges, 1e-3)
    XT = torch.as_tensor(xt, device=dev)
    b = torch.as_tensor(bh, device=dev)
    tol = 1e-12

    def fwd_bwd():
        th = torch.tensor(theta0, device=dev, requires_grad=True)
        bb = b.clone().requires_grad_(True)
        x = ag.graph_laplacian_solve(th, bb, lap, tol)
        loss = 0.5 * ((x - XT) ** 2).sum()
        return th, bb, x, loss
    th, bb, x, loss = fwd_bwd()
    loss.backward()
    ms_f, (th, bb, x, loss) = timed(fwd_bwd)
    ms_b, _ = timed(loss.backward)
    gt = th.grad.cpu().numpy()
    gb = bb.grad.cpu().numpy()
    xg = x.detach()
    # FP64 reference: sparse direct factorisation
    p, i, v, _ = matgen.aniso2d(g, theta0, 1e-3)
    lu = sl.splu(sp.csr_matrix((v, i, p), shape=(n, n)).tocsc())
    xr = lu.solve(bh)
    lr = lu.solve(xr - xt)
    gr = -(lr[edges[:, 0]] - lr[edges[:, 1]]) * (xr[edges[:, 0]] - xr[edges[:, 1]])
    out = {"n": n, "edges": E, "tol": tol, "ms_forward": round(ms_f, 2),
           "ms_backward": round(ms_b, 2),
           "grad_theta_err_vs_fp64_direct": float(np.abs(gt - gr).max() / np.abs(gr).max()),
           "grad_b_err_vs_fp64_direct": float(np.abs(gb - lr).max() / np.abs(lr).max()),
           "x_err_vs_fp64_direct": float(np.abs(xg.cpu().numpy() - xr).max() / np.abs(xr).max())}
    # central differences: L(theta +- h e) - L(theta) from the perturbation
    # dx, which solves (A +- h E_e) dx = -+ h E_e x (no cancellation in L)
    res = xg - XT
    worst = 0.0
    for e in rng.choice(E, n_fd, replace=False):
        a, c = (int(t) for t in edges[e])
        d = float(xg[a] - xg[c])
        dl = []
        for sgn in (1.0, -1.0):
            tp = torch.tensor(theta0, device=dev)
            tp[e] += sgn * h
            rhs = torch.zeros(n, dtype=torch.float64, device=dev)
            rhs[a], rhs[c] = -sgn * h * d, sgn * h * d
            with torch.no_grad():
                dx = ag.graph_laplacian_solve(tp, rhs, lap, 1e-13)
            dl.append(float(dx @ res) + 0.5 * float(dx @ dx))
        fd = (dl[0] - dl[1]) / (2 * h)
        worst = max(worst, abs(fd - gt[e]) / max(abs(gt[e]), 1e-300))
    out["fd_edges"] = n_fd
    out["fd_h"] = h
    out["grad_theta_max_rel_err_vs_fd"] = worst
    return out


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
