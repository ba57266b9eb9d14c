#!/usr/bin/env python3
"""Benchmark: SA-AMG-preconditioned CG to a 1e-8 relative residual on the 3D
7-point Poisson operator on a 128^3 grid (2,097,152 rows, 14,581,760 nonzeros),
FP64, one GPU per process.

A step is one complete time-to-solution: SA-AMG setup from the level-0 matrix
(strength, PMIS aggregation, smoothed prolongation, transpose, two SpGEMMs per
level), then PCG with one V-cycle (1+1 Jacobi sweeps, omega 1, the reference
smoother) per iteration until ||b - A x||_inf / ||b||_inf <= 1e-8.

  value  -- solves per second with A and b resident in HBM (whole job: all ranks)
  e2e    -- the same through the C ABI with HOST buffers: each step uploads A and
            b from pinned memory (lab_csr_create + lab_pcg_solve_host) and reads
            x back, copies inside the timed region
  roofline -- the dominant kernel of the step (see profiles/), timed with CUDA
            events on the launching stream
  cpu_baseline -- the reference LinAlgLib host path compiled from its sources
            (oracle/_ref) on this machine's cores, one full solve of the same system

Multi-GPU: the single system does not shard (one GPU per system); N ranks solve N
independent replicas ("replicas only"), value = N / (max over ranks of the time).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import os

if "OMP_NUM_THREADS" not in os.environ:  # the CPU reference uses every host core
    os.environ["OMP_NUM_THREADS"] = str(os.cpu_count() or 1)

import argparse
import ctypes
import json
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "AMG-PCG time-to-1e-8 (mixed vs FP64 on B200); SpMV GB/s vs ~8 TB/s HBM"
UNIT = "solves/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", "--grid", dest="n", type=int, default=None,
                    help="grid side (default: 128 for the Poisson step, 160 for mixed, "
                         "96 for adjoint, 64 for the multi-RHS batch)")
    ap.add_argument("--rtol", type=float, default=1e-8)
    ap.add_argument("--matrix", default=None, choices=["poisson", "diffusion27"],
                    help="operator of --mode spmv (default 3D 7-point Poisson) and --mode "
                         "mixed (default the 27-point diffusion operator)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the one-off SpGEMM table-sizing tuning before the timed steps")
    ap.add_argument("--level", type=int, default=0,
                    help="--mode spmv: time the SpMV of hierarchy level L's operator A_L "
                         "(0: the input matrix)")
    ap.add_argument("--no-workloads", action="store_true",
                    help="full mode: skip the batched, multi-RHS, differentiation, "
                         "27-point mixed-precision and ILU(0) summaries added to the line "
                         "after the headline's timed regions")
    ap.add_argument("--precision", default=None, choices=["fp64", "fp32", "fp32+bf16"],
                    help="--mode mixed: with --profile-range, the cycle precision whose timed "
                         "solves at rtol 1e-8 are bracketed")
    ap.add_argument("--profile-range", action="store_true",
                    help="--mode mixed: bracket the --precision solves with cudaProfilerStart/"
                         "Stop (for ncu --profile-from-start off)")
    ap.add_argument("--spmv-alg", default=None, choices=["rowseq", "vector", "stream", "halo"],
                    help="--mode spmv: force a schedule (default: the analysed plan)")
    ap.add_argument("--mode", default="full",
                    choices=["full", "profile", "spmv", "mixed", "batched", "batched_split",
                             "adjoint", "tri"],
                    help="profile: only the warm-up and timed device-resident steps (the "
                         "command the ncu launch lists in profiles/ are taken from); "
                         "spmv: only the standalone level-0 SpMV timing (5 warm-up launches, "
                         "then 3 x 20 timed back-to-back launches); mixed / batched / "
                         "adjoint / tri: the mixed-precision, batched, adjoint and "
                         "ILU(0)-PCG workloads (one JSON line each, not the driver's "
                         "bench line)")
    return ap.parse_args()


def problem(n):
    from linalglib_b200 import problems as P
    A = P.poisson3d(n)
    b, xt = P.rhs_from_solution(*A, seed=0)
    return A, b, xt


def spmv_bytes(m, n, nnz, vb=8, ib=4):
    # the reference's effective-bandwidth formula (test_functions_multiply_by_vector.cpp:122-124)
    # with the stored width of the column array (ib = 2 where the library reads its
    # 16-bit column offsets: every |col - row| <= 32767)
    return vb * (nnz + m + n) + ib * nnz + 4 * (m + 1)


def index_bytes(rp, ci):
    """Bytes per stored column index the row kernels read: 2 when every column
    offset col - row fits in 16 bits (the library then reads its offset copy)."""
    if ci.size == 0:
        return 4
    rows = np.repeat(np.arange(rp.size - 1, dtype=np.int64), np.diff(rp))
    d = ci.astype(np.int64) - rows
    return 2 if d.min() >= -32768 and d.max() <= 32767 else 4


# ------------------------------------------------------------------ distributed
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None

    def init(self, need_gpu=True):
        import torch
        self.dev = "cuda" if need_gpu else "cpu"
        if need_gpu:
            torch.cuda.set_device(self.local)
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group("nccl" if need_gpu else "gloo",
                                    timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v):
        if not self.pg:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64, device=getattr(self, "dev", "cuda"))
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ------------------------------------------------------------------ clocks
class Clocks:
    """nvidia-smi samples of this rank's GPU during the timed region.

    The sampler is started before the warm-up (nvidia-smi's own start-up takes
    about a second and must not overlap the timed steps); begin()/stop() bracket
    the timed region and only samples taken inside it are kept (the nearest
    ones if the region is shorter than the sampling period)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []
        self.t0 = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def begin(self):
        self.t0 = time.monotonic()

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        t1 = time.monotonic()
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        t0 = self.t0 if self.t0 is not None else t1
        inside = [ln for t, ln in self.lines if t0 <= t <= t1 + 0.25]
        if not inside and self.lines:
            inside = [min(self.lines, key=lambda tl: abs(tl[0] - t1))[1]]
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in inside:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ CPU baseline
def cpu_reference_solve(A, b, rtol, want_x=False):
    """One full solve on the compiled reference: (setup_s, solve_s, iters[, x])."""
    from oracle.oracle import load_reference
    ref = load_reference()
    if ref is None:
        return None
    t0 = time.perf_counter()
    h = ref.amg_setup(A, kind=0, max_level=20)
    t1 = time.perf_counter()
    x, it = h.pcg(b, rel_tol=rtol, abs_tol=1e-300, max_iter=1000)
    t2 = time.perf_counter()
    del h
    return (t1 - t0, t2 - t1, it, x) if want_x else (t1 - t0, t2 - t1, it)


def cpu_port_solve(A, b, rtol):
    from oracle.oracle import Oracle
    O = Oracle()
    t0 = time.perf_counter()
    h = O.amg_setup(A, kind=0)
    t1 = time.perf_counter()
    x, it, _ = h.pcg(b, rel_tol=rtol, abs_tol=0.0, coarse=0)
    t2 = time.perf_counter()
    return t1 - t0, t2 - t1, it, x


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_baseline(A, b, rtol, n):
    """The reference on this machine's cores; returns (line entry, its FP64 x)."""
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    r = cpu_reference_solve(A, b, rtol, want_x=True)
    kind = "reference"
    if r is None:
        r = cpu_port_solve(A, b, rtol)
        kind, cores = "port", 1
    ts, tv, it, x = r
    return {"value": 1.0 / (ts + tv), "unit": UNIT, "cores": cores, "kind": kind,
            "cpu_model": cpu_model(),
            "sample": f"one full solve of the {n}^3 system: setup {ts:.2f} s + PCG {tv:.2f} s "
                      f"({it} iterations, AMG adapter adds 2 residual SpMVs per V-cycle)"}, x


# ------------------------------------------------------------------ reference arm
def run_reference(args, d):
    if d.rank != 0:
        return 0
    A, b, _ = problem(args.n)
    warm, steps = min(args.warmup, 1), max(1, min(args.steps, 3))
    for _ in range(warm):
        if cpu_reference_solve(A, b, args.rtol) is None:
            print(json.dumps({"impl": "reference", "unavailable":
                              "oracle/_ref/liblinalg_ref.so not built (reference sources absent)"}))
            return 0
    times, parts = [], []
    for _ in range(steps):
        ts, tv, it = cpu_reference_solve(A, b, args.rtol)
        times.append(ts + tv)
        parts.append((ts, tv, it))
    total = sum(times)
    value = steps / total
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": warm, "ms_per_step": 1e3 * total / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (3D 7-point Poisson, x_true ~ U[-1,1] seed 0, b = A x_true)",
        "config": {"workload": f"SA-AMG-PCG, 3D 7-point Poisson {args.n}^3, rtol {args.rtol:g}",
                   "rows": int(A[0].size - 1), "nnz": int(A[2].size),
                   "parallelism": "host OpenMP, rank 0 only"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "cpu_model": cpu_model(),
                         "sample": f"{steps} full solves (setup + PCG) of the {args.n}^3 system"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "setup_s": [p[0] for p in parts], "solve_s": [p[1] for p in parts],
        "iterations": parts[-1][2],
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ our arm
def dominant_kernel_roofline(core, dA, m, nnz, torch, profiled=True,
                             label="A_0 (level-0 CSR pass)"):
    """CUDA-event timing of the dominant kernel class (level-0 CSR pass: SpMV on
    the 128^3 operator, the same row engine as the smoother kernels): 20 launches
    back to back between two events on the launching stream, three times; A_0
    (217 MB) is larger than L2, so every launch streams it from HBM."""
    x = torch.empty(m, dtype=torch.float64, device="cuda").uniform_(-1, 1)
    y = torch.zeros(m, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    for _ in range(5):
        dA.spmv(x, y)
    times = []
    reps = 20
    for _ in range(3):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            dA.spmv(x, y)
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) * 1e-3 / reps)
    t = statistics.median(times)
    rp, ci = dA.to_numpy()[:2]
    ib = index_bytes(rp, ci)
    algo = spmv_bytes(m, m, nnz, ib=ib)
    achieved = algo / t / 1e9
    peak, which = 6650.0, "fallback"
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak, which = float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        peak, which = 6650.0, "fallback"
    traffic = None
    prof = os.path.join(ROOT, "profiles", "spmv_poisson3d_128.md")
    if profiled and os.path.exists(prof):
        mt = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(prof).read())
        if mt:
            traffic = float(mt.group(1))
    alg, lanes = dA.algorithm()
    kname = {1: "k_pipe<op_spmv> (one thread per row, staged tiles)",
             4: f"k_vstream<op_spmv> ({lanes} lanes per row, bulk-copy stage ring)",
             5: f"k_vhalo<op_spmv> ({lanes} lanes per row, x staged per chunk of rows)"}.get(
        alg, f"k_vector<op_spmv> ({lanes} lanes per row)")
    return {"bound": "hbm", "kernel": kname + " on " + label,
            "achieved": achieved, "peak": peak, "peak_source": which, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic, "algorithmic_bytes": algo,
            "index_bytes_per_entry": ib,
            "algorithmic_bytes_int32_layout": spmv_bytes(m, m, nnz),
            "launch_us": t * 1e6}


def pcg_iteration_roofline(core, dA, solve_ms, iters, peak):
    """Whole PCG iteration against HBM: algorithmic bytes of one iteration on the
    built hierarchy, B_spmv(A_0) + B_vcycle + 8 m_0 k (k = 10 vector passes), with
    B_vcycle = sum over levels l < L of 2 B_jac(l) + B_spmv(A_l) + |R_l| + |P_l|
    + 8 (4 m_l + 2 m_l+1), B_jac(l) = |A_l| + 24 m_l, |X| = 8 nnz + ib nnz + 4 (m + 1)
    (ib = 2 or 4: the stored width of the column index the kernels read),
    plus the coarsest dense solve (8 m_L^2); time = median PCG time / iterations."""
    H = core.Hierarchy(dA)

    def size(X):
        mm, nn, zz = X.info()
        rp, ci = X.to_numpy()[:2]
        ib = index_bytes(rp, ci)
        return mm, nn, zz, 8 * zz + ib * zz + 4 * (mm + 1), ib

    L = H.levels
    b_cycle = 0
    for l in range(L):
        ml, nl, zl, al, ib = size(H.A(l))
        mc = H.A(l + 1).info()[0]
        b_cycle += (2 * (al + 24 * ml) + spmv_bytes(ml, nl, zl, ib=ib) + size(H.R(l))[3]
                    + size(H.P(l))[3] + 8 * (4 * ml + 2 * mc))
    mL = H.A(L).info()[0]
    b_cycle += 8 * mL * mL
    m0, n0, z0, _, ib0 = size(H.A(0))
    b_iter = spmv_bytes(m0, n0, z0, ib=ib0) + b_cycle + 8 * m0 * 10
    t_iter = statistics.median(solve_ms) * 1e-3 / max(1, iters[-1])
    achieved = b_iter / t_iter / 1e9
    del H
    return {"bound": "hbm", "bytes_per_iteration": int(b_iter), "us_per_iteration": t_iter * 1e6,
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak}


def run_ours(args, d):
    import torch

    d.init(need_gpu=True)
    import linalglib_b200.core as core
    from linalglib_b200 import _lib as L
    core.init()
    if args.mode == "spmv" and args.matrix == "diffusion27":
        from linalglib_b200 import problems as P
        A = P.diffusion27(args.n, seed=0)
        b, xt = P.rhs_from_solution(*A, seed=0)
    else:
        A, b, xt = problem(args.n)
    m, nnz = A[0].size - 1, A[2].size
    stream = torch.cuda.current_stream()
    dA = core.CsrMatrix.from_arrays(*A)
    dA.analyse()
    if args.mode == "spmv":
        target, H = dA, None
        if args.level > 0:
            H = core.Hierarchy(dA)
            target = H.A(min(args.level, H.levels))
            m, _, nnz = target.info()
        if args.spmv_alg:
            lanes = target.algorithm()[1]
            alg = {"rowseq": L.SPMV_ROWSEQ, "vector": L.SPMV_VECTOR,
                   "stream": L.SPMV_VECTOR_STREAM, "halo": L.SPMV_VECTOR_HALO}[args.spmv_alg]
            target.set_algorithm(alg, lanes if lanes > 1 else 0)
        roof = dominant_kernel_roofline(core, target, m, nnz, torch,
                                        profiled=(args.matrix or "poisson") == "poisson"
                                        and args.n == 128 and args.level == 0
                                        and not args.spmv_alg,
                                        label=f"A_{args.level}")
        if d.rank == 0:
            print(json.dumps({"mode": "spmv", "matrix": f"{args.matrix or 'poisson'} {args.n}^3",
                              "level": args.level, "schedule": list(target.algorithm()),
                              "rows": int(m), "nnz": int(nnz), "roofline": roof}), flush=True)
        d.close()
        return 0
    bd = core.vec(b)
    opts = core.amg_options(n1=1, n2=1, omega=1.0)
    ctl = core.iter_control(rel_tol=args.rtol, abs_tol=0.0, max_iter=1000)
    if not args.no_tune:
        # one-off plan tuning before any timed step: the Galerkin products' hash-table
        # sizing per operator shape (lab_hierarchy_tune_products; results do not
        # depend on it), kept in the process's plan cache as a saved cache file would
        # provide it.  Every timed step still runs the complete setup.
        H = core.Hierarchy(dA, kind=L.AMG_SA, max_level=20)
        L.call("lab_hierarchy_tune_products", H.h, core.stream_handle())
        del H
    def step(x):
        # setup, solve, release: the hierarchy's memory returns to the stream-ordered
        # pool, so every step reuses it (no pool growth inside the timed region)
        H = core.Hierarchy(dA, kind=L.AMG_SA, max_level=20)
        M = core.Preconditioner.amg(H, opts)
        x.zero_()
        x, info = core.pcg(dA, bd, x=x, M=M, control=ctl)
        setup_ms = H.setup_ms()
        del M, H
        return setup_ms, info

    xs = [torch.zeros(m, dtype=torch.float64, device="cuda") for _ in range(2)]
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    for i in range(args.warmup):
        step(xs[i % 2])
    torch.cuda.synchronize()

    clocks.begin()
    d.barrier()
    torch.cuda.synchronize()
    l0 = core.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    setups, solves, iters, conv = [], [], [], []
    for i in range(args.steps):
        setup_ms, info = step(xs[i % 2])
        setups.append(setup_ms)
        solves.append(info.solve_ms)
        iters.append(info.iterations)
        conv.append(info.converged)
    e1.record(stream)
    torch.cuda.synchronize()
    d.barrier()
    launches = core.launch_count() - l0
    elapsed = e0.elapsed_time(e1) * 1e-3
    clk = clocks.stop()
    t_max = d.max(elapsed)
    x_last = xs[(args.steps - 1) % 2].cpu().numpy()
    err = float(np.max(np.abs(x_last - xt)))
    if args.mode == "profile":
        if d.rank == 0:
            print(json.dumps({"mode": "profile", "ms_per_step": 1e3 * t_max / args.steps,
                              "setup_ms": setups, "solve_ms": solves, "iterations": iters[-1],
                              "gpu_launches": int(launches)}), flush=True)
        d.close()
        return 0

    # ---------------- e2e: host buffers through the C ABI
    import ctypes as C
    pin = {k: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
           for k, a in (("rp", A[0]), ("ci", A[1]), ("v", A[2]), ("b", b))}
    xh = torch.zeros(m, dtype=torch.float64).pin_memory()
    lib = L.lib()
    sh = core.stream_handle()

    def e2e_step():
        hA = C.c_void_p()
        L.check(lib.lab_csr_create(C.byref(hA), m, m, nnz, C.c_void_p(pin["rp"].data_ptr()),
                                   C.c_void_p(pin["ci"].data_ptr()),
                                   C.c_void_p(pin["v"].data_ptr()), L.MEM_HOST, sh))
        hH = C.c_void_p()
        L.check(lib.lab_amg_setup(L.AMG_SA, hA, 20, C.byref(hH), sh))
        hM = C.c_void_p()
        L.check(lib.lab_precond_create_amg(hH, C.byref(opts), C.byref(hM), sh))
        xh.zero_()
        info = L.SolveInfo()
        L.check(lib.lab_pcg_solve_host(hA, hM, C.c_void_p(pin["b"].data_ptr()),
                                       C.c_void_p(xh.data_ptr()), C.byref(ctl), C.byref(info), sh))
        return hA, hH, hM

    def e2e_free(hs):
        hA, hH, hM = hs
        lib.lab_precond_destroy(hM)
        lib.lab_hierarchy_destroy(hH)
        lib.lab_csr_destroy(hA)

    e2e_free(e2e_step())
    torch.cuda.synchronize()
    d.barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        e2e_free(e2e_step())
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_t = d.max(f0.elapsed_time(f1) * 1e-3)
    h2d = 4 * (m + 1) + 4 * nnz + 8 * nnz + 8 * m + 8 * m  # A, b, x0
    d2h = 8 * m
    e2e_parts = e2e_breakdown(lib, L, C, torch, pin, xh, m, nnz, opts, ctl, sh,
                              max(3, min(args.steps, 5)))

    roof = dominant_kernel_roofline(core, dA, m, nnz, torch, profiled=args.n == 128)
    pcg_roof = pcg_iteration_roofline(core, dA, solves, iters, roof["peak"])
    mixed, mixed_x = mixed_half(core, L, torch, dA, bd, ctl, setups, max(3, args.steps))
    setup_roof = setup_roofline(core, torch, dA, roof["peak"], setups)
    # the other workloads (batched, multi-RHS, differentiation, the 160^3 27-point
    # mixed-precision system, ILU(0)-PCG), one GPU only, after every timed region of
    # the headline
    workloads = None
    if d.world == 1 and not args.no_workloads:
        from linalglib_b200 import problems as P
        workloads = {}
        for key, fn in (("batched", lambda: batched_workloads(core, P, torch, 3,
                                                               one_by_one_reps=1)),
                        ("adjoint", lambda: adjoint_workload(core, P, torch, 3)),
                        ("mixed_config3", lambda: mixed_workload(
                            core, L, P, torch, 3, matrix="diffusion27", n=160,
                            rtols=(1e-10,))),
                        ("ilu0_pcg", lambda: dict(
                            ilu0_workload(core, torch, dA, bd, args.rtol, 3),
                            workload=f"ILU(0)-PCG, the same {args.n}^3 system, "
                                     f"rtol {args.rtol:g}"))):
            try:
                workloads.update(fn() if key == "batched" else {key: fn()})
            except Exception as e:  # reported in the line, never hides the headline
                workloads[key] = {"error": f"{type(e).__name__}: {e}"}

    if d.rank == 0:
        cpu, x_ref = None, None
        if args.gpus == 1 and d.world == 1 and not args.no_cpu_baseline:
            cpu, x_ref = cpu_baseline(A, b, args.rtol, args.n)
        scale = np.max(np.abs(x_ref)) if x_ref is not None else None
        for name, xv in mixed_x.items():
            if x_ref is not None:
                mixed[name]["err_vs_fp64_reference_solve"] = float(np.max(np.abs(xv - x_ref)) / scale)
            else:
                mixed[name]["err_vs_fp64_reference_solve"] = None
        value = d.world * args.steps / t_max
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": d.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (3D 7-point Poisson, x_true ~ U[-1,1] seed 0, b = A x_true)",
            "config": {"workload": f"SA-AMG-PCG, 3D 7-point Poisson {args.n}^3, rtol {args.rtol:g}",
                       "rows": int(m), "nnz": int(nnz),
                       "parallelism": f"replicas x{d.world} (one independent system per GPU)",
                       "l2": "inputs larger than L2 (A_0 alone is 217 MB)",
                       "smoother": "1+1 Jacobi, omega 1 (reference)", "coarse": "dense direct",
                       "tuning": ("none" if args.no_tune else
                                  "SpGEMM hash-table sizing tuned once per operator shape before "
                                  "the timed steps (plan cache; results identical); every step "
                                  "runs the complete setup")},
            "e2e": {"value": d.world * args.steps / e2e_t, "unit": UNIT,
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "e2e_parts": e2e_parts,
            "roofline": roof,
            "pcg_iteration_roofline": pcg_roof,
            "setup_roofline": setup_roof,
            "mixed_precision": mixed,
            "workloads": workloads,
            "cpu_baseline": cpu,
            "clocks": clk,
            "gpu_launches": int(launches),
            "setup_ms": setups, "solve_ms": solves, "iterations": iters[-1],
            "converged": all(conv), "max_abs_err_vs_x_true": err,
        }
        print(json.dumps(line), flush=True)
    d.close()
    return 0


def setup_roofline(core, torch, dA, peak, setups):
    """The setup's Galerkin products against HBM: for every level l, AP = A_l P_l and
    A_l+1 = R_l (AP) rerun on the built hierarchy's operators, each timed with CUDA
    events (median of 3 after one warm-up), with the reference's SpGEMM bytes
    |A| + |B| + |C|, |X| = 8 nnz + 4 (nnz + m + 1)
    (test_functions_multiply_by_matrix.cpp:198-205)."""
    H = core.Hierarchy(dA)

    def size(X):
        mm, nn, zz = X.info()
        return 8 * zz + 4 * (zz + mm + 1)

    levels, tot_b, tot_t = [], 0, 0.0
    for l in range(H.levels):
        A, P, R = H.A(l), H.P(l), H.R(l)
        AP = A.spgemm(P)
        RAP = R.spgemm(AP)
        t_ap, _ = _events_ms(torch, lambda: A.spgemm(P), 3)
        t_rap, _ = _events_ms(torch, lambda: R.spgemm(AP), 3)
        b_ap = size(A) + size(P) + size(AP)
        b_rap = size(R) + size(AP) + size(RAP)
        levels.append({"level": l, "rows": A.m, "AP_bytes": b_ap, "AP_us": 1e3 * t_ap,
                       "AP_gbs": b_ap / (t_ap * 1e-3) / 1e9, "RAP_bytes": b_rap,
                       "RAP_us": 1e3 * t_rap, "RAP_gbs": b_rap / (t_rap * 1e-3) / 1e9})
        tot_b += b_ap + b_rap
        tot_t += (t_ap + t_rap) * 1e-3
    achieved = tot_b / tot_t / 1e9
    del H
    return {"bound": "hbm", "kernel": "Galerkin SpGEMM (k_hash_gemm / k_esc_* classes), all levels",
            "algorithmic_bytes": int(tot_b), "ms": 1e3 * tot_t, "achieved": achieved,
            "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "share_of_setup": 1e3 * tot_t / statistics.median(setups), "levels": levels}


def mixed_half(core, L, torch, dA, bd, ctl, setups, reps):
    """The metric's mixed-precision half on the same system: one FP64 hierarchy,
    PCG with the FP64, FP32 and FP32 + BF16 (two finest levels) V-cycles to the
    same FP64 relative residual; solve-only and setup + solve speed-ups against
    FP64 (the setup is FP64 in every form; each form adds its one-off preparation
    of the cycle -- value conversion, work vectors, coarse inverse -- timed alone
    as prepare_ms).  The error against the FP64
    reference solve is filled in by the caller."""
    H = core.Hierarchy(dA)
    setup_ms = statistics.median(setups)
    out, xs = {}, {}
    for name, prec in (("fp64", L.PREC_FP64), ("fp32", L.PREC_FP32),
                       ("fp32+bf16", L.PREC_FP32_BF16)):
        opts = core.amg_options(n1=1, n2=1, omega=1.0, precision=prec)
        prep = []
        for _ in range(3):
            # the one-off preparation on a fresh hierarchy: value conversion to FP32
            # (or BF16) and the cycle's work vectors, timed alone
            Hp = core.Hierarchy(dA)
            torch.cuda.synchronize()
            keep = []
            t, _ = _events_ms(torch, lambda: keep.append(core.Preconditioner.amg(Hp, opts)), 1)
            prep.append(t)
            del keep, Hp
        M = core.Preconditioner.amg(H, opts)
        x = torch.zeros_like(bd)
        info = []

        def solve():
            x.zero_()
            info.append(core.pcg(dA, bd, x=x, M=M, control=ctl)[1])
        solve()
        t, ts = _events_ms(torch, solve, reps)
        out[name] = {"solve_ms": t, "iterations": info[-1].iterations,
                     "converged": bool(info[-1].converged),
                     "true_rel_residual": _rel_res(torch, dA, x, bd)}
        out[name]["prepare_ms"] = statistics.median(prep)
        xs[name] = x.cpu().numpy()
        del M
    base = out["fp64"]["solve_ms"]
    for name in ("fp32", "fp32+bf16"):
        r = out[name]
        r["speedup_solve_vs_fp64"] = base / r["solve_ms"]
        r["speedup_setup_plus_solve_vs_fp64"] = (
            (setup_ms + out["fp64"]["prepare_ms"] + base) /
            (setup_ms + r["prepare_ms"] + r["solve_ms"]))
    out["setup_ms_fp64"] = setup_ms
    out["target"] = ">= 1.6x FP64 at the same 1e-8 accuracy"
    return out, xs


def e2e_breakdown(lib, L, C, torch, pin, xh, m, nnz, opts, ctl, sh, reps):
    """Where an end-to-end step's time goes: the same C-ABI calls as the e2e step,
    in a separate pass with a device synchronisation after each phase, host wall
    time per phase (median over reps, ms).  solve_host includes the b upload, the
    SpMV plan of the new matrix, the capture of the iteration graph for the new
    preconditioner, the solve and the x download."""
    parts = {k: [] for k in ("upload_and_create", "setup", "precond_build", "spmv_plan",
                             "solve_host", "release")}

    def timed(key, fn):
        t0 = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        parts[key].append(1e3 * (time.perf_counter() - t0))
        return r

    for _ in range(reps):
        hA, hH, hM = C.c_void_p(), C.c_void_p(), C.c_void_p()
        torch.cuda.synchronize()
        timed("upload_and_create", lambda: L.check(lib.lab_csr_create(
            C.byref(hA), m, m, nnz, C.c_void_p(pin["rp"].data_ptr()),
            C.c_void_p(pin["ci"].data_ptr()), C.c_void_p(pin["v"].data_ptr()), L.MEM_HOST, sh)))
        timed("setup", lambda: L.check(lib.lab_amg_setup(L.AMG_SA, hA, 20, C.byref(hH), sh)))
        timed("precond_build", lambda: L.check(lib.lab_precond_create_amg(hH, C.byref(opts),
                                                                          C.byref(hM), sh)))
        timed("spmv_plan", lambda: L.check(lib.lab_spmv_analysis(hA, sh)))
        xh.zero_()
        info = L.SolveInfo()
        timed("solve_host", lambda: L.check(lib.lab_pcg_solve_host(
            hA, hM, C.c_void_p(pin["b"].data_ptr()), C.c_void_p(xh.data_ptr()), C.byref(ctl),
            C.byref(info), sh)))
        parts.setdefault("solve_device", []).append(info.solve_ms)

        def release():
            lib.lab_precond_destroy(hM)
            lib.lab_hierarchy_destroy(hH)
            lib.lab_csr_destroy(hA)
        timed("release", release)
    out = {k: statistics.median(v) for k, v in parts.items()}
    out["total"] = sum(v for k, v in out.items() if k != "solve_device")
    out["note"] = ("host wall ms per phase, a device synchronisation after each; "
                   "solve_device = CUDA-event time of the PCG iterations inside solve_host")
    return out


# ------------------------------------------------------------------ extra workloads
def _events_ms(torch, fn, reps):
    """Median CUDA-event time (ms) of fn() over reps runs (after the caller's warm-up)."""
    stream = torch.cuda.current_stream()
    out = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return statistics.median(out), out


def _rel_res(torch, dA, x, b):
    r = dA.residual(x, b)
    return float(torch.max(torch.abs(r)) / torch.max(torch.abs(b)))


def mixed_workload(core, L, P, torch, steps, matrix=None, n=None, rtols=(1e-8, 1e-10),
                   bracket=None):
    """27-point variable-coefficient diffusion (lognormal sigma 1.5, z x100) on an
    n^3 grid (default; matrix "poisson": the 3D 7-point Poisson problem, omega 1):
    one FP64 SA hierarchy, PCG with the FP64, FP32 and FP32+BF16 cycles to each rtol;
    error of each against the FP64 solve.  bracket: the precision whose timed solves
    at rtol 1e-8 run between cudaProfilerStart and cudaProfilerStop."""
    if matrix == "poisson":
        # the 7-point Poisson problem with the reference's smoother weight
        n = n or 128
        A = P.poisson3d(n)
        omega, wl = 1.0, f"SA-AMG-PCG, 3D 7-point Poisson {n}^3, omega 1"
    else:
        n = n or 160
        A = P.diffusion27(n, sigma=1.5, zscale=100.0, seed=0)
        omega, wl = 2.0 / 3.0, (f"SA-AMG-PCG, 27-point diffusion {n}^3 (lognormal sigma 1.5, "
                                "z x100), omega 2/3")
    b, xt = P.rhs_from_solution(*A, seed=0)
    dA = core.CsrMatrix.from_arrays(*A)
    dA.analyse()
    bd = core.vec(b)
    xtd = core.vec(xt)
    H = core.Hierarchy(dA)  # warm-up (module loading, pool growth)
    t_setup, _ = _events_ms(torch, lambda: core.Hierarchy(dA), 3)
    res = {"config": {"workload": wl, "rows": int(A[0].size - 1), "nnz": int(A[2].size),
                      "levels": H.levels},
           "setup_ms": t_setup, "runs": []}
    names = {L.PREC_FP64: "fp64", L.PREC_FP32: "fp32", L.PREC_FP32_BF16: "fp32+bf16"}
    for rtol in rtols:
        ctl = core.iter_control(rel_tol=rtol, abs_tol=0.0, max_iter=1000)
        x64 = None
        for prec in (L.PREC_FP64, L.PREC_FP32, L.PREC_FP32_BF16):
            M = core.Preconditioner.amg(H, core.amg_options(omega=omega, precision=prec))
            x = torch.zeros_like(bd)
            core.pcg(dA, bd, x=x, M=M, control=ctl)  # warm-up: value copies, graph capture
            info = []

            def solve():
                x.zero_()
                info.append(core.pcg(dA, bd, x=x, M=M, control=ctl)[1])
            brk = bracket is not None and rtol == 1e-8 and names[prec] == bracket
            if brk:
                torch.cuda.profiler.start()
            t, ts = _events_ms(torch, solve, max(3, steps))
            if brk:
                torch.cuda.profiler.stop()
            if prec == L.PREC_FP64:
                x64 = x.clone()
            err64 = float(torch.max(torch.abs(x - x64)) / torch.max(torch.abs(x64)))
            res["runs"].append({
                "rtol": rtol, "precision": names[prec], "solve_ms": t, "solve_ms_all": ts,
                "iterations": info[-1].iterations, "converged": bool(info[-1].converged),
                "true_rel_residual": _rel_res(torch, dA, x, bd),
                "err_vs_fp64_solve": err64,
                "err_vs_x_true": float(torch.max(torch.abs(x - xtd)))})
        base = [r for r in res["runs"] if r["rtol"] == rtol and r["precision"] == "fp64"][0]
        for r in res["runs"]:
            if r["rtol"] == rtol:
                r["speedup_vs_fp64"] = base["solve_ms"] / r["solve_ms"]
    return res


def run_mixed(args, d):
    """The mixed-precision workload (mixed_workload)."""
    import torch
    d.init(need_gpu=True)
    import linalglib_b200.core as core
    from linalglib_b200 import _lib as L
    from linalglib_b200 import problems as P
    core.init()
    res = mixed_workload(core, L, P, torch, args.steps, matrix=args.matrix, n=args.n,
                         bracket=(args.precision or "fp32") if args.profile_range else None)
    if d.rank == 0:
        print(json.dumps({"mode": "mixed", **res}), flush=True)
    d.close()
    return 0


def run_batched_split(args, d):
    """The 256-system batch over N GPUs (torchrun, one rank per GPU): the systems
    are split by the size-balanced partition (lab_batch_partition), every rank
    sets up and solves its share as one batched solve (no collective on the data
    path), and rank 0 gathers all solutions on the host.  Timed: setup + solve of
    each rank's share with CUDA events after a warm-up, max over ranks."""
    import torch
    d.init(need_gpu=True)
    import linalglib_b200.core as core
    from linalglib_b200 import batch
    from linalglib_b200 import problems as P
    core.init()
    rng = np.random.default_rng(0)
    sides = rng.integers(32, 257, size=256)
    mats = [P.poisson2d(int(s)) for s in sides]
    rhs = [P.rhs_from_solution(*A, seed=k)[0] for k, A in enumerate(mats)]
    costs = [int(A[0][-1]) + A[0].size - 1 for A in mats]
    part = batch.partition(costs, d.world)
    mine = [k for k in range(len(mats)) if part[k] == d.rank]
    blocks = [core.CsrMatrix.from_arrays(*mats[k]) for k in mine]
    S, offs = core.block_diag(blocks)
    S.analyse()
    bd = core.vec(np.concatenate([rhs[k] for k in mine]))
    ctl = core.iter_control(rel_tol=1e-8, abs_tol=0.0, max_iter=1000)
    out = {}

    def step():
        M = core.Preconditioner.amg(core.Hierarchy(S), core.amg_options(omega=2.0 / 3.0))
        out["r"] = core.batched_pcg(S, offs, bd, M, control=ctl)

    for _ in range(max(1, args.warmup)):
        step()
    d.barrier()
    torch.cuda.synchronize()
    t, _ = _events_ms(torch, step, max(3, args.steps))
    t_max = d.max(t)
    x, iters, conv, _ = out["r"]
    x = x.cpu().numpy()
    local = [(x[offs[i]:offs[i + 1]].copy(), int(iters[i]), bool(conv[i])) for i in range(len(mine))]
    res = batch.solve_partitioned(mats, rhs, lambda ms, bs: local, rank=d.rank, world=d.world,
                                  dist=d.pg)
    if d.rank == 0:
        worst = max(float(np.max(np.abs(P.csr_matvec(*A[:3], r[0]) - b)) / np.max(np.abs(b)))
                    for A, b, r in zip(mats, rhs, res))
        loads = np.bincount(part, weights=costs, minlength=d.world)
        print(json.dumps({
            "mode": "batched_split", "n_gpus": d.world,
            "workload": "256 2D 5-point Poisson systems, sides U{32..256} seed 0, rtol 1e-8",
            "ms_setup_plus_solve": t_max, "systems_per_s": 256 / (t_max * 1e-3),
            "scaling": "strong (the 256 systems split over the GPUs)",
            "load_balance": float(loads.max() / loads.mean()),
            "iterations_max": max(r[1] for r in res), "all_converged": all(r[2] for r in res),
            "worst_rel_residual": worst}), flush=True)
    d.close()
    return 0


def batched_workloads(core, P, torch, steps, n=64, one_by_one_reps=3):
    """(a) 256 2D 5-point Poisson systems, sides ~U{32..256} (seed 0), stacked block
    diagonally, one hierarchy, one segmented PCG (per-system convergence mask) to
    rtol 1e-8; against solving the systems one after another.  (b) 32 right-hand
    sides ~U[-1,1] on the 3D 7-point n^3 operator by block PCG; against 32 solves."""
    rng = np.random.default_rng(0)
    sides = rng.integers(32, 257, size=256)
    mats = [P.poisson2d(int(s)) for s in sides]
    blocks = [core.CsrMatrix.from_arrays(*A) for A in mats]
    S, offs = core.block_diag(blocks)
    S.analyse()
    bs = np.concatenate([P.rhs_from_solution(*A, seed=k)[0] for k, A in enumerate(mats)])
    bd = core.vec(bs)
    ctl = core.iter_control(rel_tol=1e-8, abs_tol=0.0, max_iter=1000)
    H = core.Hierarchy(S)  # warm-up
    t_setup, _ = _events_ms(torch, lambda: core.Hierarchy(S), 3)
    M = core.Preconditioner.amg(H, core.amg_options(omega=2.0 / 3.0))
    x = torch.zeros_like(bd)
    out = {}

    def batched():
        x.zero_()
        out["r"] = core.batched_pcg(S, offs, bd, M, x=x, control=ctl)
    batched()
    t_b, _ = _events_ms(torch, batched, max(3, steps))
    _, iters, conv, _ = out["r"]
    # one system at a time, each with its own hierarchy (setup excluded from the time)
    singles = []
    for k, Ak in enumerate(blocks):
        Hk = core.Hierarchy(Ak)
        singles.append((Ak, Hk, core.Preconditioner.amg(Hk, core.amg_options(omega=2.0 / 3.0)),
                        bd[int(offs[k]):int(offs[k + 1])].contiguous()))

    def one_by_one():
        for Ak, Hk, Mk, bk in singles:
            core.pcg(Ak, bk, M=Mk, control=ctl)
    one_by_one()
    t_s, _ = _events_ms(torch, one_by_one, one_by_one_reps)
    # per-system relative residual of the batched solution (inf norms)
    rr = S.residual(x, bd).cpu().numpy()
    worst = max(float(np.max(np.abs(rr[int(offs[k]):int(offs[k + 1])])))
                / max(float(np.max(np.abs(bs[int(offs[k]):int(offs[k + 1])]))), 1e-300)
                for k in range(len(mats)))
    res = {"systems": {
        "workload": "256 2D 5-point Poisson systems, sides U{32..256} seed 0, rtol 1e-8",
        "rows": int(offs[-1]), "setup_ms": t_setup, "solve_ms": t_b,
        "one_by_one_ms": t_s, "speedup": t_s / t_b, "iterations_max": int(iters.max()),
        "iterations_min": int(iters.min()), "all_converged": bool(conv.all()),
        "worst_rel_residual": worst}}
    del singles
    # (b) multi-RHS
    A = P.poisson3d(n)
    dA = core.CsrMatrix.from_arrays(*A)
    dA.analyse()
    H2 = core.Hierarchy(dA)
    M2 = core.Preconditioner.amg(H2, core.amg_options(omega=2.0 / 3.0))
    B = torch.from_numpy(np.random.default_rng(1).uniform(-1, 1, size=(32, A[0].size - 1))).cuda()
    X = torch.zeros_like(B)

    def multi():
        X.zero_()
        out["m"] = core.multi_rhs_pcg(dA, B, M2, X=X, control=ctl)
    multi()
    t_m, _ = _events_ms(torch, multi, max(3, steps))
    _, it2, conv2, _ = out["m"]
    cols = [B[k].contiguous() for k in range(32)]

    def per_rhs():
        for bk in cols:
            core.pcg(dA, bk, M=M2, control=ctl)
    per_rhs()
    t_p, _ = _events_ms(torch, per_rhs, 3)
    res["multi_rhs"] = {"workload": f"32 RHS U[-1,1] on 3D 7-point {n}^3, rtol 1e-8",
                        "solve_ms": t_m, "one_by_one_ms": t_p, "speedup": t_p / t_m,
                        "iterations_max": int(it2.max()), "all_converged": bool(conv2.all())}
    return res


def run_batched(args, d):
    """The batched workloads (batched_workloads).  Under torchrun (N > 1) the batch
    is split over the GPUs instead (run_batched_split)."""
    import torch
    if d.world > 1:
        return run_batched_split(args, d)
    d.init(need_gpu=True)
    import linalglib_b200.core as core
    from linalglib_b200 import problems as P
    core.init()
    res = batched_workloads(core, P, torch, args.steps, n=args.n or 64)
    if d.rank == 0:
        print(json.dumps({"mode": "batched", **res}), flush=True)
    d.close()
    return 0


def adjoint_workload(core, P, torch, steps, n=96):
    """Weighted 7-point graph Laplacian (lognormal sigma 1, shift 1e-3) on n^3:
    forward SA-AMG-PCG to 1e-10, adjoint solve lambda = A^-T (x - x_target), and
    dL/dA on the pattern; a central finite difference along b checks dL/db."""
    A = P.graph_laplacian3d(n, sigma=1.0, shift=1e-3, seed=0)
    b, _ = P.rhs_from_solution(*A, seed=0)
    xt = core.vec(np.random.default_rng(1).standard_normal(A[0].size - 1))
    dA = core.CsrMatrix.from_arrays(*A)
    dA.analyse()
    bd = core.vec(b)
    ctl = core.iter_control(rel_tol=1e-10, abs_tol=0.0, max_iter=2000)
    H = core.Hierarchy(dA)  # warm-up
    t_setup, _ = _events_ms(torch, lambda: core.Hierarchy(dA), 3)
    M = core.Preconditioner.amg(H, core.amg_options(omega=2.0 / 3.0))
    st = {}

    def forward():
        st["x"], st["fi"] = core.pcg(dA, bd, M=M, control=ctl)

    def backward():
        g = st["x"] - xt
        st["lam"], st["ai"] = core.adjoint_solve(dA, g, M=M, symmetric=True, control=ctl)
        st["gA"] = core.adjoint_grad_A(dA, st["lam"], st["x"])
    forward()
    backward()
    t_f, _ = _events_ms(torch, forward, max(3, steps))
    t_b, _ = _events_ms(torch, backward, max(3, steps))
    # directional check of dL/db = lambda along a random direction
    v = torch.from_numpy(np.random.default_rng(2).standard_normal(A[0].size - 1)).cuda()
    h = 1e-4

    def loss(bb):
        xx, _ = core.pcg(dA, bb.contiguous(), M=M, control=ctl)
        return 0.5 * float(torch.sum((xx - xt) ** 2))
    fd = (loss(bd + h * v) - loss(bd - h * v)) / (2 * h)
    an = float(torch.dot(st["lam"], v))
    res = {"config": {"workload": f"graph Laplacian {n}^3 (lognormal sigma 1, "
                                  "shift 1e-3), rtol 1e-10",
                      "rows": int(A[0].size - 1), "nnz": int(A[2].size)},
           "setup_ms": t_setup, "forward_ms": t_f, "adjoint_ms": t_b,
           "forward_iterations": st["fi"].iterations, "adjoint_iterations": st["ai"].iterations,
           "dLdb_directional": {"adjoint": an, "finite_difference": fd,
                                "rel_diff": abs(an - fd) / max(abs(fd), 1e-300)}}
    return res


def run_adjoint(args, d):
    """The differentiation workload (adjoint_workload)."""
    import torch
    d.init(need_gpu=True)
    import linalglib_b200.core as core
    from linalglib_b200 import problems as P
    core.init()
    res = adjoint_workload(core, P, torch, args.steps, n=args.n or 96)
    if d.rank == 0:
        print(json.dumps({"mode": "adjoint", **res}), flush=True)
    d.close()
    return 0


def _hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def tri_bytes(rp, ci, lower):
    """Algorithmic bytes of one triangular solve: the triangle's entries (value and
    column, diagonal included), row pointers, b read and x written once."""
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    nnz_t = int(np.count_nonzero(ci <= rows) if lower else np.count_nonzero(ci >= rows))
    m = rp.size - 1
    return 12 * nnz_t + 4 * (m + 1) + 16 * m, nnz_t


def ilu0_workload(core, torch, dA, bd, rtol, steps):
    """ILU(0)-PCG (the reference's ilu_precond with cg_solver) on an already built
    system: a step is the preconditioner build plus the solve, device-resident."""
    ctl = core.iter_control(rel_tol=rtol, abs_tol=0.0, max_iter=5000)
    x = torch.zeros_like(bd)
    st = {}

    def step():
        M = core.Preconditioner.ilu0(dA)
        x.zero_()
        _, st["info"] = core.pcg(dA, bd, x=x, M=M, control=ctl)
        del M
    step()
    t_step, _ = _events_ms(torch, step, max(3, steps))
    rr = dA.residual(x, bd)
    return {"step_ms": t_step, "solves_per_s": 1e3 / t_step,
            "iterations": st["info"].iterations, "converged": bool(st["info"].converged),
            "true_rel_residual": float(torch.max(torch.abs(rr)) / torch.max(torch.abs(bd)))}


def run_tri(args, d):
    """ILU(0)-preconditioned CG on the 3D 7-point Poisson n^3 system (the reference's
    ilu_precond with cg_solver).  A step is the preconditioner build (copy of A,
    level analysis, in-place ILU(0)) plus the PCG solve to rtol, device-resident.
    Also times one preconditioner application (unit-lower then upper solve of the
    factor) and each triangular solve alone (CUDA events), and the oracle's CPU
    ILU(0)-PCG (the C restatement, one core) on the same system."""
    import torch
    d.init(need_gpu=True)
    import linalglib_b200.core as core
    core.init()
    n = args.n or 128
    A, b, xt = problem(n)
    m, nnz = A[0].size - 1, A[2].size
    dA = core.CsrMatrix.from_arrays(*A)
    dA.analyse()
    bd = core.vec(b)
    ctl = core.iter_control(rel_tol=args.rtol, abs_tol=0.0, max_iter=5000)
    x = torch.zeros(m, dtype=torch.float64, device="cuda")
    st = {}

    def step():
        M = core.Preconditioner.ilu0(dA)
        x.zero_()
        _, st["info"] = core.pcg(dA, bd, x=x, M=M, control=ctl)
        del M

    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    for _ in range(max(args.warmup, 1)):
        step()
    torch.cuda.synchronize()
    clocks.begin()
    l0 = core.launch_count()
    t_step, all_steps = _events_ms(torch, step, args.steps)
    launches = (core.launch_count() - l0) / args.steps
    clk = clocks.stop()
    info = st["info"]
    err = float(torch.max(torch.abs(x - core.vec(xt))))

    M = core.Preconditioner.ilu0(dA)
    r = core.vec(np.random.default_rng(3).uniform(-1, 1, m))
    z = torch.empty_like(r)
    for _ in range(3):
        M.apply(r, z)
    t_apply, _ = _events_ms(torch, lambda: M.apply(r, z), 20)
    t_build, _ = _events_ms(torch, lambda: core.Preconditioner.ilu0(dA), 5)
    # the build's parts on a fresh copy of A: level analysis (first solve minus a
    # solve), then the in-place factorization alone
    X = core.CsrMatrix.from_arrays(*A)
    t_first, _ = _events_ms(torch, lambda: X.trsv(r, lower=True, unit_diag=True, x=z), 1)
    t_fact, _ = _events_ms(torch, lambda: X.factor("ilu0"), 1)
    del X
    t_lo, _ = _events_ms(torch, lambda: dA.trsv(r, lower=True, unit_diag=False, x=z), 20)
    t_up, _ = _events_ms(torch, lambda: dA.trsv(r, lower=False, unit_diag=False, x=z), 20)
    b_lo, nnz_lo = tri_bytes(A[0], A[1], True)
    b_up, nnz_up = tri_bytes(A[0], A[1], False)
    peak, which = _hbm_peak()
    levels = 3 * (n - 1) + 1  # dependency levels of either triangle of the 7-point stencil

    cpu = None
    if d.rank == 0 and not args.no_cpu_baseline:
        from oracle.oracle import Oracle
        t0 = time.perf_counter()
        _, it_cpu = Oracle().precond_cg(0, A, b, rel_tol=args.rtol, abs_tol=0.0, max_iter=5000)
        t_cpu = time.perf_counter() - t0
        cpu = {"value": 1.0 / t_cpu, "unit": "solves/s", "cores": 1, "kind": "port",
               "sample": f"one full ILU(0)-PCG solve of the {n}^3 system ({it_cpu} iterations, "
                         f"{t_cpu:.1f} s; the reference's own host ILU(0) allocates an n-sized "
                         "column map per row, O(m^2) at this size)"}
    line = {
        "mode": "tri", "metric": "ILU(0)-PCG time-to-rtol", "value": 1e3 / t_step,
        "unit": "solves/s", "ms_per_step": t_step, "steps_ms": all_steps, "dtype": "f64",
        "config": {"workload": f"ILU(0)-PCG, 3D 7-point Poisson {n}^3, rtol {args.rtol:g}",
                   "rows": int(m), "nnz": int(nnz), "levels_per_triangle": levels,
                   "l2": "inputs larger than L2"},
        "iterations": info.iterations, "converged": bool(info.converged),
        "max_abs_err_vs_x_true": err, "build_ms": t_build, "apply_ms": t_apply,
        "build_parts_ms": {"level_analysis": t_first - t_lo, "factorization": t_fact},
        "trsv": {"lower_us": 1e3 * t_lo, "upper_us": 1e3 * t_up,
                 "lower_bytes": b_lo, "upper_bytes": b_up,
                 "lower_GBs": b_lo / (t_lo * 1e-3) / 1e9, "upper_GBs": b_up / (t_up * 1e-3) / 1e9,
                 "frac_lower": b_lo / (t_lo * 1e-3) / 1e9 / peak,
                 "frac_upper": b_up / (t_up * 1e-3) / 1e9 / peak,
                 "peak": peak, "peak_source": which,
                 "us_per_level": 1e3 * (t_lo + t_up) / (2 * levels)},
        "gpu_launches_per_step": launches, "clocks": clk, "cpu_baseline": cpu,
    }
    if d.rank == 0:
        print(json.dumps(line), flush=True)
    d.close()
    return 0


def main():
    args = parse()
    d = Dist()
    if args.impl == "reference":
        args.n = args.n or 128
        return run_reference(args, d)
    if args.mode == "mixed":
        return run_mixed(args, d)
    if args.mode == "batched_split":
        return run_batched_split(args, d)
    if args.mode == "batched":
        return run_batched(args, d)
    if args.mode == "adjoint":
        return run_adjoint(args, d)
    if args.mode == "tri":
        return run_tri(args, d)
    args.n = args.n or 128
    return run_ours(args, d)


if __name__ == "__main__":
    sys.exit(main())
