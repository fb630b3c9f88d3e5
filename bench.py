"""Benchmark of the HODLR hot path on B200.

One step = one full pass over the workload to the metric's accuracy: ACA
compression of every off-diagonal block (storeLRinTree), recLU factorization,
the solve of all right-hand sides (together the reference's recLU_TotalTime,
src/HODLR_Matrix.cpp:775), then GMRES preconditioned by the HODLR factor with
the full FP64 kernel product (the kernel-matrix form of iterative_Solve,
src/HODLR_Matrix.cpp:1138-1213) until every column has
||b - K x|| / ||b|| <= 1e-10.

Workload (the FP64-at-scale configuration): N = 262144 points uniform in
[0,1]^2, k-d median ordered, Matern-3/2 kernel with l = 0.2 plus 1e-2 on the
diagonal, leaf 128, partial-pivot ACA tol 1e-8, 8 right-hand sides ~ N(0,1),
all FP64.  Seeded synthetic data.  The W/V panels and Y (gigabytes) are far
larger than L2, so no L2 flush is needed between steps.

Prints one JSON line.  --impl reference times the reference algorithm on the
host cores instead (the CPU oracle port; the reference itself needs Eigen and
cannot be built here): a bounded sample of the same workload per step,
extrapolated to the full factor+solve.
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

METRIC = "factor+solve s and solves/s, mixed vs FP64 GPU path, at rel residual ≤1e-10"
UNIT = "factor+solve/s"
N_PTS, DIM, LSCALE, SHIFT, LEAF, TOL, NRHS, SEED = 262144, 2, 0.2, 1e-2, 128, 1e-8, 8, 2024
RES_TOL, MAX_IR = 1e-10, 200
# GMRES iterations to 1e-10 with this workload's FP64 HODLR preconditioner
# (the reference's factors: same pivots and ranks) -- measured by the GPU path
GMRES_ITERS_FP64 = 6
WORKLOAD = ("FP64 at scale: N=262144 2D uniform [0,1]^2 k-d ordered, Matern-3/2 l=0.2 "
            "+1e-2*delta, leaf 128, partial-pivot ACA tol 1e-8, 8 RHS N(0,1), FP64")


def workload_inputs():
    from dense_hodlr_b200.points import uniform_cube
    pts = uniform_cube(N_PTS, DIM, SEED)
    b = np.asfortranarray(np.random.default_rng(SEED + 1).standard_normal((N_PTS, NRHS)))
    return pts, b


def workload_config(world):
    return {"workload": WORKLOAD, "n": N_PTS, "dim": DIM, "kernel": "matern32",
            "length_scale": LSCALE, "diag_shift": SHIFT, "leaf": LEAF, "aca_tol": TOL,
            "nrhs": NRHS, "precision": "fp64", "parallelism": f"replicas{world}",
            "l2": "no flush: W/V/Y panels (GBs) exceed the 126 MB L2"}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def profiled_figure(name, key):
    """A figure from a committed ncu summary under profiles/ (a 'key: value' line)."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith(key + ":"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except (ValueError, IndexError):
                return None
    return None


# FP64 FLOPs of the symmetric full-kernel product (kmatvec.cu / kfast.cuh),
# FMA counted as 2, as the kernel executes them: one Matern-3/2 entry in 2D is
# the distance (2 sub + 2 fma from the floor), the square root from the
# hardware seed (2 mul + 3 fma), Tang's exp (1 clamp, 1 fma + 1 sub for the
# index, 2 fma for the reduction, 3 fma + 1 mul for the polynomial, 1 fma for
# the table scale) and (1+s)e^-s (1 fma): 13 FMAs + 7 other = 33 FLOPs,
# evaluated once per entry pair, plus 2 * nrhs FMAs (row and column products,
# inside mma.m8n8k4.f64 for 8 right-hand sides) per evaluated entry.
KMV_EVAL_FLOPS = 33


def sym_slices(n):
    """Workspace slices of the symmetric product (kmatvec.cu: 256-point tiles,
    about 96 splits)."""
    nt = -(-n // 256)
    tps = 1 if nt <= 96 else -(-nt // 96)
    return -(-nt // tps)
FP64_LANES_PER_SM = 64


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([c.strip() for c in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            for k, name in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


# --------------------------------------------------------------- CPU leg
def cpu_reference_step(pts, b, threads, kmv_rows=1024):
    """The reference algorithm's recLU path on the host cores, measured in
    full on the workload: storeLRinTree (partial-pivot ACA of every block and
    the leaf blocks), recLU_Factorize and recLU_Solve of every right-hand side
    -- the reference's recLU_TotalTime (src/HODLR_Matrix.cpp:757-775).  It
    runs the CPU oracle, the restatement of the reference (the reference needs
    Eigen, absent here), on `threads` threads: blocks, leaves and sibling
    subtrees in parallel, the largest blocks with threads inside.

    The direct solution does not reach the 1e-10 residual (the reference's
    recLU_Solve stops there).  Reaching it takes HODLR-preconditioned GMRES
    with the full-kernel product, O(N^2) entry evaluations per product on the
    CPU; one product is timed on the first kmv_rows rows (every row costs the
    same) and scaled by N / kmv_rows.  That estimate is reported beside the
    measurement, never inside it."""
    from oracle import oracle as orc
    orc.build()
    n = pts.shape[1]
    o = orc.OracleHODLR.from_kernel(pts, 1, LSCALE, shift=SHIFT, leaf=LEAF)
    o.set_lr(TOL)
    t0 = time.perf_counter()
    o.compress(threads)
    t1 = time.perf_counter()
    o.factorize(threads)
    t2 = time.perf_counter()
    x = o.solve(b, threads)
    t3 = time.perf_counter()
    y = o.kernel_matvec_rows(x, 0, kmv_rows, threads)
    t4 = time.perf_counter()
    r = b[:kmv_rows] - y[:kmv_rows]
    kmv_s = (t4 - t3) * n / kmv_rows
    return {"compress_s": t1 - t0, "factor_s": t2 - t1, "solve_s": t3 - t2,
            "total_s": t3 - t0, "threads": threads,
            "direct_rel_residual_rows": float(np.linalg.norm(r) / np.linalg.norm(b[:kmv_rows])),
            "kmatvec_s_estimate": kmv_s, "kmatvec_rows_timed": kmv_rows,
            "to_1e-10_s_estimate": (t3 - t0) + (GMRES_ITERS_FP64 + 1) * kmv_s
                                   + GMRES_ITERS_FP64 * (t3 - t2)}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


# ---------------------------------------------------------------- GPU leg
def slowest_rank(x, world, device):
    """Max of x over the ranks of the process group (the slowest replica sets
    the job's pace); x itself with one rank."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(ms_max, world):
    """Whole-job steps per second of `world` replicas, each doing one step in
    at most ms_max milliseconds (weak scaling: work per replica fixed)."""
    return world * 1000.0 / ms_max


def gather_blocks(g):
    return [g.block_info(b) for b in range(g.num_blocks())]


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    from dense_hodlr_b200 import HODLR_Matrix, KernelSpec
    from dense_hodlr_b200 import _lib

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    pts, b = workload_inputs()
    spec = KernelSpec("matern32", LSCALE, SHIFT)
    g = HODLR_Matrix(N_PTS, N_PTS, spec, pts, LEAF)
    g.set_LRTolerance(TOL)
    stream = torch.cuda.current_stream(dev)
    lib = _lib.lib()
    assert lib.hodlr_set_stream(g._h, ctypes.c_void_p(stream.cuda_stream)) == 0
    b_d = torch.from_numpy(np.ascontiguousarray(b.T)).to(dev)  # column-major N x NRHS
    x_d = torch.empty_like(b_d)

    def step(max_iter=MAX_IR):
        assert lib.hodlr_reset(g._h) == 0
        g.storeLRinTree()
        g.recLU_Compute()
        return g.iterative_solve_device(b_d.data_ptr(), x_d.data_ptr(), NRHS, tol=RES_TOL,
                                        max_iter=max_iter, restart=32)

    def launches():
        c = ctypes.c_longlong()
        lib.hodlr_get_launch_count(g._h, ctypes.byref(c))
        return c.value

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    phase = {"lr": [], "fact": [], "solve": [], "aca_s": [], "aca_bytes": [], "aca_launches": [],
             "ir": [], "relres": []}
    l0 = launches()
    with ClockSampler(local_rank) as clk:
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            it, rel = step()
            phase["ir"].append(it)
            phase["relres"].append(float(rel.max()))
            st = g.aca_stats()
            phase["lr"].append(g.get_LR_ComputationTime())
            phase["fact"].append(g.get_recLU_FactorizationTime())
            phase["solve"].append(g.get_recLU_SolveTime())
            phase["aca_s"].append(st["seconds"])
            phase["aca_bytes"].append(st["bytes"])
            phase["aca_launches"].append(st["launches"])
        e1.record(stream)
        torch.cuda.synchronize()
    n_launch = launches() - l0
    x_dev = x_d.cpu().numpy().T.copy()  # the last timed step's solution (device path)
    ms = e0.elapsed_time(e1) / args.steps
    ms_max = slowest_rank(ms, world, dev)
    clocks = clk.summary()

    # end to end through the C ABI with host buffers: create (points H2D),
    # compress, factor, solve + refine (b H2D, x D2H), destroy
    x_host = np.zeros_like(b, order="F")
    e2e_times = []
    for it in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g2 = HODLR_Matrix(N_PTS, N_PTS, spec, pts, LEAF)
        g2.set_LRTolerance(TOL)
        x_host = g2.iterative_Solve(b, MAX_IR, RES_TOL)
        del g2
        torch.cuda.synchronize()
        if it >= args.warmup:
            e2e_times.append(time.perf_counter() - t0)
    e2e_s = slowest_rank(float(np.mean(e2e_times)), world, dev)

    # mixed precision (3xTF32 tensor-core Woodbury products, FP64 leaf and
    # capacitance LUs and residual) to the same accuracy.  TF32 and BF16
    # factors stop being preconditioners at this shift (cond(K) * u > 1).
    mixed = None
    if not args.no_mixed:
        g.set_precision("tf32x3")
        for _ in range(1):
            step(MIXED_C2_MAX_ITER)
        torch.cuda.synchronize()
        m0 = torch.cuda.Event(enable_timing=True)
        m1 = torch.cuda.Event(enable_timing=True)
        m_it, m_rel = [], []
        m_steps = 5
        m0.record(stream)
        for _ in range(m_steps):
            it, rel = step(MIXED_C2_MAX_ITER)
            m_it.append(it)
            m_rel.append(float(rel.max()))
        m1.record(stream)
        torch.cuda.synchronize()
        m_ms = m0.elapsed_time(m1) / m_steps
        mixed = {"precision": "tf32x3", "ms_per_step": m_ms, "steps": m_steps,
                 "gmres_iterations": int(max(m_it)), "rel_residual": max(m_rel),
                 "converged": bool(max(m_rel) <= RES_TOL),
                 "factor_s": g.get_recLU_FactorizationTime(),
                 "speedup_vs_fp64": ms_max / m_ms,
                 "note": ("TF32 and BF16 Woodbury products diverge on this system "
                          "(Matern shift 1e-2: cond(K) * u_tf32 > 1); 3xTF32 converges")}
        g.set_precision("fp64")
        g.recLU_Compute()

    scale_pairs = {}
    if not args.no_scale and world == 1:  # extra keys of the one-GPU line
        for key, cfg_name, n_cfg in SCALE_PAIRS:
            try:
                scale_pairs[key] = run_scale_pair(stream, cfg_name, n_cfg)
            except Exception as e:  # reported in the line; the headline workload stands alone
                scale_pairs[key] = {"error": f"{type(e).__name__}: {e}"}
            torch.cuda.synchronize()

    # direct solve only (no refinement), for the phase breakdown
    g.solve_device(b_d.data_ptr(), x_d.data_ptr(), NRHS)
    t_direct_solve = g.get_recLU_SolveTime()
    x_direct = x_d.cpu().numpy().T.copy()
    # one full-kernel product K X (8 columns), CUDA events on the same stream
    y_d = torch.empty_like(x_d)
    k0 = torch.cuda.Event(enable_timing=True)
    k1 = torch.cuda.Event(enable_timing=True)
    g.kernel_matvec_device(x_d.data_ptr(), y_d.data_ptr(), NRHS)
    torch.cuda.synchronize()
    k0.record(stream)
    g.kernel_matvec_device(x_d.data_ptr(), y_d.data_ptr(), NRHS)
    k1.record(stream)
    torch.cuda.synchronize()
    t_kmatvec = k0.elapsed_time(k1) / 1000.0

    # accuracy (outside the timed region): full-kernel FP64 residual
    relres = g.residual(x_host, b)
    relres_direct = g.residual(x_direct, b)
    # the same solve through the host-buffer C ABI path against the device path
    diff_dev_host = float(np.linalg.norm(x_host - x_dev) / np.linalg.norm(x_dev))

    blocks = gather_blocks(g)
    aca_bytes = float(np.mean(phase["aca_bytes"]))
    aca_s = float(np.mean(phase["aca_s"]))
    aca_launch = float(np.mean(phase["aca_launches"]))
    hbm, peak_kind = peaks()
    achieved = aca_bytes / aca_s / 1e9
    ratio = profiled_figure("aca_kernel_matern2d_n131072.md", "traffic_to_algorithmic")
    aca_per_launch = aca_bytes / max(aca_launch, 1.0)
    traffic = ratio * aca_per_launch if ratio else None
    # full-kernel product: FP64 FLOPs per launch over its event-timed duration
    sm_mhz = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("sm_max_mhz", 1965.0) \
        if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else 1965.0
    n_sms = torch.cuda.get_device_properties(dev).multi_processor_count
    fp64_peak = n_sms * FP64_LANES_PER_SM * 2 * sm_mhz * 1e6 / 1e12
    evaluated = N_PTS * (N_PTS + 256) / 2.0
    kmv_flops = evaluated * (KMV_EVAL_FLOPS + 4 * NRHS)
    kmv_tf = kmv_flops / t_kmatvec / 1e12
    kmv_dram_ref = profiled_figure("kmatvec_sym_mma_matern2d_n65536.md", "dram_bytes_per_launch")
    out = {
        "metric": METRIC,
        "value": job_rate(ms_max, world),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded uniform 2D cloud, k-d ordered; N(0,1) right-hand sides)",
        "config": workload_config(world),
        "factor_solve_s": ms_max / 1000.0,
        "phases_s": {"lr": float(np.mean(phase["lr"])), "factor": float(np.mean(phase["fact"])),
                     "solve_refine": float(np.mean(phase["solve"])),
                     "direct_solve": t_direct_solve},
        "solves_per_s": world * NRHS / float(np.mean(phase["solve"])),
        "direct_solves_per_s": world * NRHS / t_direct_solve,
        "rel_residual": float(max(relres.max(), max(phase["relres"]))),
        "rel_residual_direct": float(relres_direct.max()),
        "gmres_iterations": int(max(phase["ir"])),
        "kmatvec_s": t_kmatvec,
        "kmatvec_entries_per_s": float(N_PTS) * N_PTS / t_kmatvec,
        "ranks": {"max": int(max(bk["rank"] for bk in blocks)),
                  "levels": int(max(bk["level"] for bk in blocks)) + 1},
        "e2e": {"value": job_rate(e2e_s * 1000.0, world), "unit": UNIT,
                "h2d_bytes_per_step": int(pts.nbytes + b.nbytes),
                "d2h_bytes_per_step": int(b.nbytes),
                "dev_vs_host_solution_rel_diff": diff_dev_host},
        "roofline": {"kernel": "kmatvec_sym_mma_kernel (full-kernel FP64 product, 8 RHS, "
                               "products on mma.m8n8k4.f64; the largest share of the step)",
                     "bound": "fp64", "achieved": kmv_tf, "peak": fp64_peak,
                     "peak_kind": (f"nominal FP64 peak ({n_sms} SMs x 64 FMA/clk x 2 x "
                                   f"{sm_mhz:.0f} MHz), shared by FP64 FMAs and FP64 MMAs; "
                                   "no measured FP64 figure exists"),
                     "unit": "TFLOP/s", "frac": kmv_tf / fp64_peak,
                     "traffic": (kmv_dram_ref * (N_PTS * sym_slices(N_PTS))
                                 / (65536.0 * sym_slices(65536)) if kmv_dram_ref else None),
                     "traffic_note": ("DRAM bytes of the n=65536 capture scaled by slices x n "
                                      "(the workspace writes); the kernel is compute-bound"),
                     "algorithmic_flops_per_launch": kmv_flops,
                     "avg_launch_s": t_kmatvec},
        "roofline_aca": {"kernel": "aca_kernel (batched partial-pivot ACA, one launch per level "
                                   "group)",
                         "bound": "hbm", "achieved": achieved, "peak": hbm,
                         "peak_kind": f"{peak_kind} hbm_gbs (burst)", "unit": "GB/s",
                         "frac": achieved / hbm,
                         "traffic": traffic,
                         "traffic_note": ("DRAM/algorithmic ratio of the N=131072 capture "
                                          "applied to this launch's algorithmic bytes"),
                         "algorithmic_bytes_per_launch": aca_per_launch,
                         "avg_launch_s": aca_s / max(aca_launch, 1.0),
                         "launches_per_step": aca_launch},
        "mixed": mixed,
        "scale_pairs": scale_pairs,
        "clocks": clocks,
        "gpu_launches": int(n_launch),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        c = cpu_reference_step(pts, b, threads)
        out["cpu_baseline"] = {
            "value": 1.0 / c["total_s"], "unit": UNIT, "cores": threads, "kind": "port",
            "sample": (f"the whole workload's recLU path (compression, factorization and the "
                       f"8-RHS direct solve: the reference's recLU_TotalTime) by the CPU oracle "
                       f"(restatement; the reference needs Eigen) on {threads} threads of "
                       f"{cpu_model()}, measured once: {c['total_s']:.1f} s (compress "
                       f"{c['compress_s']:.1f}, factor {c['factor_s']:.1f}, solve "
                       f"{c['solve_s']:.2f}); direct residual {c['direct_rel_residual_rows']:.1e} "
                       f"on the first {c['kmatvec_rows_timed']} rows, not 1e-10"),
            "measured": c,
        }
    return out


# Extra keys of the bench line: the two configurations measured at their
# full size or the largest that fits, FP64 against the mixed form, one timed
# step each (compress + factor + GMRES until ||b - K x|| / ||b|| <= 1e-10).
#  * the end-to-end target's shape (unit sphere, Matern-3/2 l = 0.1 + 1e-2
#    delta, leaf 128, ACA tol 1e-10, 1 RHS) at N = 262144, the largest whose
#    FP64 factors fit one B200 (its top rank, 4117 here, grows like sqrt(N));
#  * the mixed-precision configuration (3D cube, Gaussian l = 0.3 + 0.1 delta,
#    leaf 128, tol 1e-8, 16 RHS) at its full N = 2^20.
# The mixed form keeps the configuration's tolerance (a looser preconditioner
# stalled GMRES on the sphere shape at every tolerance from 1e-8 to 1e-5)
# and runs the Woodbury products in 3xTF32 on tcgen05; its GMRES is capped at
# MIXED_MAX_ITER iterations, beyond which it is reported as not converged.
SCALE_PAIRS = (("sphere_matern", "c5", 262144), ("cube_gaussian", "c3", 1 << 20))
MIXED_PREC, MIXED_MAX_ITER = "tf32x3", 8
MIXED_C2_MAX_ITER = 30  # 3xTF32 on the headline workload converges in a few iterations


def run_scale_pair(stream, cfg_name, n):
    import torch
    from dense_hodlr_b200 import HODLR_Matrix, KernelSpec
    c = SCALE_CONFIGS[cfg_name]
    pts = scale_points(c["cloud"], n)
    b = np.random.default_rng(SEED + 1).standard_normal((n, c["nrhs"]))
    b_d = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
    x_d = torch.empty_like(b_d)
    g = HODLR_Matrix(n, n, KernelSpec(c["kernel"], c["l"], c["shift"]), pts, c["leaf"])
    g.set_LRTolerance(c["tol"])
    out = {"n": n, "aca_tol": c["tol"], "nrhs": c["nrhs"], "steps": 1,
           "note": "one step per leg, no warm-up of its own (the headline steps ran first)"}
    for name, prec, max_iter in (("fp64", "fp64", MAX_IR), ("mixed", MIXED_PREC, MIXED_MAX_ITER)):
        g.set_precision(prec)
        g.reset()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.storeLRinTree()
        g.recLU_Compute()
        n_it, rel = g.iterative_solve_device(b_d.data_ptr(), x_d.data_ptr(), c["nrhs"],
                                             tol=RES_TOL, max_iter=max_iter, restart=40)
        e1.record(stream)
        torch.cuda.synchronize()
        out[name] = {"precision": prec, "ms_per_step": e0.elapsed_time(e1),
                     "lr_s": g.get_LR_ComputationTime(),
                     "factor_s": g.get_recLU_FactorizationTime(),
                     "gmres_s": g.get_recLU_SolveTime(), "gmres_iterations": int(n_it),
                     "rel_residual": float(rel.max()), "converged": bool(rel.max() <= RES_TOL),
                     "max_rank": int(g.ranks().max())}
        out[name]["x"] = x_d.cpu().numpy().T.copy()
    xf, xm = out["fp64"].pop("x"), out["mixed"].pop("x")
    out["mixed"]["solution_rel_diff_vs_fp64"] = float(np.linalg.norm(xm - xf) /
                                                      np.linalg.norm(xf))
    out["mixed_speedup_vs_fp64"] = (out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
                                    if out["mixed"]["converged"] else None)
    del g
    return out


def run_reference(args):
    """The reference arm: the reference algorithm's recLU path on the host
    cores (cpu_reference_step), one measured step over the whole workload --
    its compression, factorization and direct solve (recLU_TotalTime).  The
    line's steps / ms_per_step are those of the step that ran; --steps and
    --warmup do not apply (one pass over the workload takes about a minute on
    16 cores).  The reference's path stops at the direct solve, whose residual
    (printed) is far above 1e-10, so this value is a conservative stand-in for
    the metric: its time to 1e-10 (refinement products estimated from a timed
    row sample) is printed beside it."""
    threads = os.cpu_count() or 1
    pts, b = workload_inputs()
    t0 = time.perf_counter()
    c = cpu_reference_step(pts, b, threads)
    wall = time.perf_counter() - t0
    T = c["total_s"]
    return {
        "metric": METRIC, "impl": "reference", "value": 1.0 / T, "unit": UNIT, "n_gpus": 1,
        "steps": 1, "warmup": 0, "ms_per_step": T * 1000.0,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded uniform 2D cloud, k-d ordered; N(0,1) right-hand sides)",
        "config": workload_config(1),
        "cpu_baseline": {"value": 1.0 / T, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": (f"the whole workload, once: compression + factorization + "
                                    f"8-RHS direct solve (recLU_TotalTime) by the CPU oracle "
                                    f"(restatement of the reference, which needs Eigen) on "
                                    f"{threads} threads of {cpu_model()}")},
        "e2e": {"value": 1.0 / T, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "measured": c,
        "note": (f"steps/warmup requested {args.steps}/{args.warmup}; one measured pass ran "
                 f"({wall:.1f} s with the residual sample).  The direct solve reaches "
                 f"{c['direct_rel_residual_rows']:.1e}, not 1e-10; reaching 1e-10 would take "
                 f"about {c['to_1e-10_s_estimate']:.0f} s ({GMRES_ITERS_FP64} GMRES iterations "
                 f"with O(N^2) kernel products, estimated from a timed "
                 f"{c['kmatvec_rows_timed']}-row sample)"),
    }


def run_profile_case(case):
    """Small cases for ncu captures (a few GB on the device).

    aca-profile: N=131072 2D uniform k-d ordered, Matern-3/2 l=0.2 + 1e-2
    delta, tol 1e-8, capacity hints large enough that every level is one
    launch; the pooled deep levels launch first and the top level (2 blocks of
    65536^2, 74 CTAs each) last, its W/V panels (~0.9 GB) far above L2.
    """
    from dense_hodlr_b200 import HODLR_Matrix, KernelSpec
    from dense_hodlr_b200.points import uniform_cube
    if case == "aca-profile":
        n = 131072
        pts = uniform_cube(n, 2, SEED)
        g = HODLR_Matrix(n, n, KernelSpec("matern32", LSCALE, SHIFT), pts, LEAF)
        g.set_LRTolerance(TOL)
        g.set_capacity_hint([512, 384, 320, 256, 192, 128, 128, 96, 96, 64])
        g.storeLRinTree()
        print(json.dumps({"case": case, "aca": g.aca_stats(), "lr_s": g.get_LR_ComputationTime(),
                          "max_rank": int(g.ranks().max())}))
    elif case == "kmatvec-profile":
        # N=65536 2D Matern-3/2, 8 right-hand sides: one full-kernel product
        import torch
        n = 65536
        pts = uniform_cube(n, 2, SEED)
        g = HODLR_Matrix(n, n, KernelSpec("matern32", LSCALE, SHIFT), pts, LEAF)
        x = torch.randn(NRHS, n, dtype=torch.float64, device="cuda")
        y = torch.empty_like(x)
        for _ in range(3):
            g.kernel_matvec_device(x.data_ptr(), y.data_ptr(), NRHS)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        g.kernel_matvec_device(x.data_ptr(), y.data_ptr(), NRHS)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        print(json.dumps({"case": case, "ms": ms, "entries_per_s": n * n / (ms / 1e3)}))
    elif case.startswith("factor-profile"):
        # the FP64-at-scale workload (or its first N points' cloud at a smaller
        # N, 'factor-profile:N'): one compression, then one factorization (the
        # launches after the aca_kernel ones) and one 8-RHS direct solve
        import torch
        from dense_hodlr_b200.points import uniform_cube
        parts = case.split(":")
        n = int(parts[1]) if len(parts) > 1 else N_PTS
        if len(parts) > 2:  # another configuration's shape, e.g. 'factor-profile:65536:c5'
            c = SCALE_CONFIGS[parts[2]]
            pts = scale_points(c["cloud"], n)
            g = HODLR_Matrix(n, n, KernelSpec(c["kernel"], c["l"], c["shift"]), pts, c["leaf"])
            g.set_LRTolerance(c["tol"])
        else:
            pts = uniform_cube(n, DIM, SEED) if n != N_PTS else workload_inputs()[0]
            g = HODLR_Matrix(n, n, KernelSpec("matern32", LSCALE, SHIFT), pts, LEAF)
            g.set_LRTolerance(TOL)
        b = np.random.default_rng(SEED + 1).standard_normal((n, NRHS))
        g.storeLRinTree()
        g.recLU_Compute()
        b_d = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
        x_d = torch.empty_like(b_d)
        g.solve_device(b_d.data_ptr(), x_d.data_ptr(), NRHS)
        print(json.dumps({"case": case, "factor_s": g.get_recLU_FactorizationTime(),
                          "solve_s": g.get_recLU_SolveTime()}))
    elif case.startswith("tune"):
        run_tune(case)
    elif case.startswith("aca-ab"):
        print(json.dumps(run_aca_ab(case)))
    elif case.split(":")[0] in SCALE_CONFIGS:
        print(json.dumps(run_scale(case)))
    elif case.startswith("batched"):
        print(json.dumps(run_batched(case)))
    else:
        raise SystemExit(f"unknown case {case}")


def run_tune(case):
    """Sweep of the preconditioner's compression tolerance and Woodbury
    precision on one configuration, case 'tune:<c3|c5|c2>:N[:tols[:precs]]'
    (comma-separated lists): per tolerance one compression, then per precision
    the factorization and GMRES on the FP64 full-kernel residual to 1e-10.
    One JSON line per combination, flushed."""
    import torch
    from dense_hodlr_b200 import HODLR_Matrix, KernelSpec
    parts = case.split(":")
    cfg = parts[1]
    n = int(parts[2])
    tols = [float(t) for t in parts[3].split(",")] if len(parts) > 3 else [1e-10, 1e-8, 1e-6, 1e-4]
    precs = parts[4].split(",") if len(parts) > 4 else ["fp64", "tf32x3", "tf32", "bf16"]
    if cfg == "c2":
        from dense_hodlr_b200.points import uniform_cube
        pts = uniform_cube(n, DIM, SEED)
        spec, leaf, nrhs = KernelSpec("matern32", LSCALE, SHIFT), LEAF, NRHS
    else:
        c = SCALE_CONFIGS[cfg]
        pts = scale_points(c["cloud"], n)
        spec, leaf, nrhs = KernelSpec(c["kernel"], c["l"], c["shift"]), c["leaf"], c["nrhs"]
    b = np.random.default_rng(SEED + 1).standard_normal((n, nrhs))
    b_d = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
    x_d = torch.empty_like(b_d)
    g = HODLR_Matrix(n, n, spec, pts, leaf)
    for tol in tols:
        g.set_precision("fp64")
        g.set_LRTolerance(tol)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g.storeLRinTree()
        t_lr = time.perf_counter() - t0
        kmax = int(g.ranks().max())
        st = g.aca_stats()
        for prec in precs:
            g.set_precision(prec)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            g.recLU_Compute()
            t_f = time.perf_counter() - t0
            t0 = time.perf_counter()
            try:
                it, rel = g.iterative_solve_device(b_d.data_ptr(), x_d.data_ptr(), nrhs,
                                                   tol=1e-10, max_iter=80, restart=40)
                err = None
            except Exception as e:  # a factor too poor to precondition
                it, rel, err = -1, np.array([np.inf]), str(e)
            torch.cuda.synchronize()
            t_g = time.perf_counter() - t0
            print(json.dumps({"case": "tune", "cfg": cfg, "n": n, "aca_tol": tol,
                              "precision": prec, "compress_s": t_lr,
                              "aca_gbs": st["bytes"] / max(st["seconds"], 1e-12) / 1e9,
                              "kmax": kmax,
                              "factor_s": t_f, "gmres_s": t_g, "gmres_iterations": int(it),
                              "rel_residual": float(rel.max()),
                              "total_s": t_lr + t_f + t_g, "error": err}), flush=True)


def run_aca_ab(case):
    """ACA with the top levels' panels streamed through the bulk-copy ring
    (mode 1: one copy per column; mode 2: one 2D tensor copy per tile)
    against per-thread loads (mode 0), case 'aca-ab[:N[:cfg]]' (default: the
    FP64 workload's cloud at N = 262144; cfg 'c5' for the sphere / Matern tol
    1e-10 shape): one compression each way (after a warm-up), the ACA time
    and algorithmic GB/s of each, and whether ranks and pivots agree."""
    from dense_hodlr_b200 import HODLR_Matrix, KernelSpec
    parts = case.split(":")
    n = int(parts[1]) if len(parts) > 1 and parts[1] else N_PTS
    cfg = parts[2] if len(parts) > 2 else "c2"
    if cfg == "c5":
        c = SCALE_CONFIGS["c5"]
        pts = scale_points(c["cloud"], n)
        spec, leaf, tol = KernelSpec(c["kernel"], c["l"], c["shift"]), c["leaf"], c["tol"]
    else:
        from dense_hodlr_b200.points import uniform_cube
        pts = uniform_cube(n, DIM, SEED)
        spec, leaf, tol = KernelSpec("matern32", LSCALE, SHIFT), LEAF, TOL
    out = {"case": "aca-ab", "n": n, "cfg": cfg}
    res = {}
    for on in (1, 2, 0, 1, 2):
        g = HODLR_Matrix(n, n, spec, pts, leaf)
        g.set_LRTolerance(tol)
        g.set_aca_streaming(on)
        g.storeLRinTree()
        st = g.aca_stats()
        res[on] = (g.ranks(), [g.pivots(b) for b in range(min(g.num_blocks(), 64))])
        out[f"stream{on}"] = {"aca_s": st["seconds"], "launches": st["launches"],
                              "gbs": st["bytes"] / st["seconds"] / 1e9,
                              "lr_s": g.get_LR_ComputationTime(),
                              "max_rank": int(g.ranks().max())}
        del g
    r0, p0 = res[0]
    out["ranks_equal"] = all(bool(np.array_equal(res[m][0], r0)) for m in (1, 2))
    out["pivots_equal"] = all(np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
                              for m in (1, 2) for a, b in zip(res[m][1], p0))
    return out


# The two 2^20-point configurations: (points, kernel, length scale, shift,
# leaf, ACA tolerance, right-hand sides).
SCALE_CONFIGS = {
    # mixed precision with refinement: 3D uniform cube, Gaussian
    "c3": dict(cloud="cube", kernel="gaussian", l=0.3, shift=0.1, leaf=128, tol=1e-8, nrhs=16),
    # the end-to-end target: unit sphere, Matern-3/2, ACA tol 1e-10
    "c5": dict(cloud="sphere", kernel="matern32", l=0.1, shift=1e-2, leaf=128, tol=1e-10,
               nrhs=1),
}


def scale_points(cloud, n, seed=SEED):
    from dense_hodlr_b200.points import uniform_cube, unit_sphere
    return uniform_cube(n, 3, seed) if cloud == "cube" else unit_sphere(n, seed)


def run_scale(case):
    """One of the 2^20-point configurations, case '<c3|c5>[:N[:prec,prec,...]]'
    (default N = 2^20, precisions fp64 then tf32x3,tf32,bf16): compression
    once (FP64 ACA), then per precision of the Woodbury products the
    factorization, a direct solve and HODLR-preconditioned GMRES on the FP64
    full-kernel residual to 1e-10.  One JSON line per phase (flushed), so a
    run cut short still reports what it finished."""
    import torch
    from dense_hodlr_b200 import HODLR_Matrix, KernelSpec
    parts = case.split(":")
    cfg = SCALE_CONFIGS[parts[0]]
    n = int(parts[1]) if len(parts) > 1 and parts[1] else 1 << 20
    precs = parts[2].split(",") if len(parts) > 2 else ["fp64", "tf32x3", "tf32", "bf16"]
    nrhs = cfg["nrhs"]

    def emit(d):
        free, total = torch.cuda.mem_get_info()
        d["device_used_gb"] = round((total - free) / 1e9, 2)
        print(json.dumps(d), flush=True)

    pts = scale_points(cfg["cloud"], n)
    b = np.random.default_rng(SEED + 1).standard_normal((n, nrhs))
    b_d = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
    x_d = torch.empty_like(b_d)
    g = HODLR_Matrix(n, n, KernelSpec(cfg["kernel"], cfg["l"], cfg["shift"]), pts, cfg["leaf"])
    g.set_LRTolerance(cfg["tol"])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g.storeLRinTree()
    lr_wall = time.perf_counter() - t0
    blocks = gather_blocks(g)
    nlev = max(bk["level"] for bk in blocks) + 1
    st = g.aca_stats()
    emit({"case": parts[0], "n": n, "nrhs": nrhs, "phase": "compress",
          "lr_s": g.get_LR_ComputationTime(), "lr_wall_s": lr_wall, "aca": st,
          "aca_gbs": st["bytes"] / max(st["seconds"], 1e-12) / 1e9,
          "kmax_per_level": [max(bk["rank"] for bk in blocks if bk["level"] == lv)
                             for lv in range(nlev)],
          "iters_max_per_level": [max(bk["iters"] for bk in blocks if bk["level"] == lv)
                                  for lv in range(nlev)]})
    x64 = None
    for prec in precs:
        g.set_precision(prec)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g.recLU_Compute()
        tf = g.get_recLU_FactorizationTime()
        g.solve_device(b_d.data_ptr(), x_d.data_ptr(), nrhs)
        ts = g.get_recLU_SolveTime()
        xd = x_d.cpu().numpy().T.copy()
        if prec == "fp64" and x64 is None:
            x64 = xd
        emit({"case": parts[0], "n": n, "precision": prec, "phase": "factor",
              "factor_s": tf, "direct_solve_s": ts})
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        it, rel = g.iterative_solve_device(b_d.data_ptr(), x_d.data_ptr(), nrhs, tol=1e-10,
                                           max_iter=60, restart=32)
        torch.cuda.synchronize()
        t_gm = time.perf_counter() - t1
        emit({"case": parts[0], "n": n, "precision": prec, "phase": "gmres",
              "gmres_s": t_gm, "gmres_iterations": int(it), "rel_residual": float(rel.max()),
              "factor_plus_gmres_s": time.perf_counter() - t0,
              "direct_solve_rel_diff_vs_fp64": (float(np.linalg.norm(xd - x64) /
                                                      np.linalg.norm(x64))
                                                if x64 is not None else None)})
    return {"case": parts[0], "n": n, "done": True}


def batched_systems(nsys, seed=SEED):
    """The uneven-systems workload: N log-uniform in [1024, 32768], 1D or 2D
    uniform points (alternating), Gaussian or Matern-3/2 (50/50), l
    log-uniform in [0.05, 0.5], diagonal shift log-uniform in [1e-2, 1]."""
    from dense_hodlr_b200 import KernelSpec
    from dense_hodlr_b200.points import uniform_1d_sorted, uniform_cube
    rng = np.random.default_rng(seed)
    out = []
    for q in range(nsys):
        n = int(np.exp(rng.uniform(np.log(1024), np.log(32768))))
        p = uniform_1d_sorted(n, 0.0, 1.0, seed + 7 * q) if q % 2 else uniform_cube(n, 2, seed + 7 * q)
        kind = "gaussian" if rng.random() < 0.5 else "matern32"
        l = float(np.exp(rng.uniform(np.log(0.05), np.log(0.5))))
        sh = float(np.exp(rng.uniform(np.log(1e-2), np.log(1.0))))
        out.append((p, KernelSpec(kind, l, sh)))
    return out


def run_batched(case):
    """Uneven batch, case
    'batched[:nsys[:max_points_per_forest[:precision[:in_place[:solver]]]]]' (in_place 1:
    K^-1 U over the U panels, which lets a forest hold more points; solver 'refine' or
    'gmres': per-system refinement or per-system HODLR-preconditioned GMRES).  The
    default forest size, 450000 points, was the fastest of 0.3M, 0.45M, 0.6M, 0.8M and
    1.2M on this batch (6.9, 6.8, 7.6, 8.5, 9.1 s with refinement): a forest's
    panels span its points at each level's largest capacity, so smaller forests of
    similar-sized systems move fewer bytes.
    Systems are sorted by size and packed into forests (waves) of at most
    max_points points, each forest one handle whose level launches span its
    systems; per wave: compress, factor, direct solve and refinement until
    every system's residual is <= 1e-10.  The same systems one handle each
    (every 8th, scaled by 8) give the unbatched time."""
    import torch
    from dense_hodlr_b200 import HODLR_Matrix, _lib
    parts = case.split(":")
    nsys = int(parts[1]) if len(parts) > 1 else 512
    cap = int(parts[2]) if len(parts) > 2 and parts[2] else 450_000
    prec = parts[3] if len(parts) > 3 and parts[3] else "fp64"
    in_place = int(parts[4]) if len(parts) > 4 and parts[4] else -1
    solver = parts[5] if len(parts) > 5 and parts[5] else "refine"
    systems = batched_systems(nsys)
    order = sorted(range(nsys), key=lambda q: -systems[q][0].shape[1])
    waves, cur, npts = [], [], 0
    for q in order:
        n = systems[q][0].shape[1]
        if cur and npts + n > cap:
            waves.append(cur)
            cur, npts = [], 0
        cur.append(q)
        npts += n
    if cur:
        waves.append(cur)
    rng = np.random.default_rng(SEED + 3)
    total_pts = sum(p.shape[1] for p, _ in systems)
    res = {"case": "batched", "systems": nsys, "points": int(total_pts), "waves": len(waves),
           "max_points_per_forest": cap, "precision": prec, "solver": solver}

    peak_gb = []

    def run_waves(timed):
        worst, its, t_total = 0.0, [], 0.0
        for w in waves:
            F = HODLR_Matrix.forest([systems[q] for q in w], leaf=64)
            F.set_LRTolerance(1e-8)
            F.set_factor_in_place(in_place)
            if prec != "fp64":
                F.set_precision(prec)
            b = torch.from_numpy(rng.standard_normal(F.n)).cuda()
            x = torch.empty_like(b)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            F.storeLRinTree()
            F.recLU_Compute()
            if solver == "gmres":
                it, rel = F.iterative_solve_device(b.data_ptr(), x.data_ptr(), 1, tol=1e-10,
                                                   max_iter=100, restart=32)
            else:
                it, rel = F.forest_refine_device(b.data_ptr(), x.data_ptr(), 1, tol=1e-10,
                                                 max_iter=100)
            torch.cuda.synchronize()
            t_total += time.perf_counter() - t0
            worst = max(worst, float(rel.max()))
            its.append(it)
            free, total = torch.cuda.mem_get_info()
            peak_gb.append(round((total - free) / 1e9, 1))
            del F
        return t_total, worst, its

    run_waves(False)  # warm-up: device pool, modules
    t, worst, its = run_waves(True)
    res.update({"seconds": t, "systems_per_s": nsys / t, "max_rel_residual": worst,
                "iterations_per_wave": its, "device_used_gb_per_wave": peak_gb,
                "in_place": in_place})
    # one handle per system, every 8th system, scaled by 8
    t1 = 0.0
    sample = list(range(0, nsys, 8))
    for q in sample:
        p, k = systems[q]
        n = p.shape[1]
        b = torch.from_numpy(rng.standard_normal(n)).cuda()
        x = torch.empty_like(b)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g = HODLR_Matrix(n, n, k, p, 64)
        g.set_LRTolerance(1e-8)
        if prec != "fp64":
            g.set_precision(prec)
        g.storeLRinTree()
        g.recLU_Compute()
        if solver == "gmres":
            g.iterative_solve_device(b.data_ptr(), x.data_ptr(), 1, tol=1e-10, max_iter=100,
                                     restart=32)
        else:
            g.solve_refined_device(b.data_ptr(), x.data_ptr(), 1, tol=1e-10, max_iter=100)
        torch.cuda.synchronize()
        t1 += time.perf_counter() - t0
        del g
    res["one_handle_per_system_seconds"] = t1 * nsys / len(sample)
    res["speedup_vs_one_handle_per_system"] = res["one_handle_per_system_seconds"] / t
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default=None, help="small profiling case (see run_profile_case)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision leg")
    ap.add_argument("--no-scale", action="store_true",
                    help="skip the FP64-vs-mixed pairs of the sphere and 2^20-point cube shapes")
    args = ap.parse_args()
    if args.case:
        run_profile_case(args.case)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return
        print(json.dumps(run_reference(args)), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    out = run_ours(args, rank, world, local_rank)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
