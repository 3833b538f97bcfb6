"""Benchmark: numeric factor + refined solve of the 64^3 variable-coefficient
3D Laplacian on B200.

One step = the hot path over one system: numeric FP32 factorization (Schur
updates of large fronts on the tensor cores) + solve of one right-hand side
with FP64 iterative refinement to backward error <= 1e-14.  The plain FP64
factor + solve of the same system is timed beside it (``fp64`` block).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--side 64] [--impl reference]

value   = reference flop count (sum over L columns of count^2, the count the
          reference prints, mdgpu.cu:1354-1359) / device time per step, inputs
          resident in HBM; GFLOP/s, whole job (N replicas for --gpus N).
e2e     = the same metric through the public C ABI with host buffers
          (mdgpu_factor + mdgpu_refine: values and right-hand side copied in,
          solution copied out, every step).
Multi-GPU: a single system does not shard -- N independent replicas, one per
GPU (weak scaling), barrier + max over ranks of the device time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "factor+solve time & GFLOP/s, FP32+IR vs FP64 on B200 at backward error <=1e-14"
UNIT = "GFLOP/s"
REF_SIDE = 28  # CPU sample of the reference arm (the full 64^3 takes ~12 min on one core)
CPU_BASELINE_SIDE = 42  # about 15 s of single-core reference work
# DRAM traffic per algorithmic byte of each kernel class:
# dram__bytes_read.sum + dram__bytes_write.sum of every launch of the class
# over three FP32 steps of the 48^3 grid (one ncu pass, three metrics,
# --clock-control none; cold caches per launch), per step, divided by the
# class's algorithmic bytes of one profiled 48^3 step.  The roofline line
# scales the class's algorithmic bytes per launch at the bench size by it
# (traffic grows with the units processed).
TRAFFIC_PER_ALGO_BYTE = {"panel": 0.79, "schur_update": 0.78, "solve_large": 1.06,
                         "solve_small": 1.06, "small_front": 1.01, "assemble": 0.53}
# the kernels behind each profiler class (one class launch = one timed group)
CLASS_KERNELS = {
    "small_front": ["k_tiny_fronts", "k_small_front"],
    "assemble": ["k_big_assemble_warp"],
    "potrf": ["k_tile_potrf"],
    "panel": ["k_panel"],
    "schur_update": ["k_schur_tc"],
    "solve_small": ["k_fwd_solve", "k_bwd_solve"],
    "solve_large": ["k_fwd_solve", "k_bwd_solve"],
}
CLASS_KERNELS_FP64 = dict(CLASS_KERNELS, schur_update=["k_schur_f64"])


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--side", type=int, default=64)
    ap.add_argument("--impl", default="mdgpu_b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # profiling helper: only one arm of the step, timed and printed alone --
    # with a small case (--side 48) for ncu captures of a few launches
    ap.add_argument("--only", choices=["fp32", "fp64"], default=None,
                    help="run only this arm's step (use --side 48 or less under ncu)")
    ap.add_argument("--only-nrhs", type=int, default=1,
                    help="right-hand sides of the --only step (uniform random columns)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-rhs64", action="store_true",
                    help="skip the 64-right-hand-side measurement")
    ap.add_argument("--no-gmres", action="store_true",
                    help="skip the FP32 factor + GMRES-IR measurement")
    ap.add_argument("--elastic-side", type=int, default=40,
                    help="nodes per side of the elasticity workload (40: the full size)")
    ap.add_argument("--workload", choices=["grid3d", "batch", "adjoint", "elasticity"],
                    default="grid3d",
                    help="batch: 1024 independent systems (512 2D, 512 3D) under one handle; "
                         "adjoint: gradient of log det A + b'A^-1 b on the 48^3 grid; "
                         "elasticity: 3 unknowns per node on a 40^3 27-point node grid, "
                         "BF16-update factor + GMRES-IR vs FP32 + GMRES-IR vs FP32 + plain "
                         "refinement vs FP64")
    ap.add_argument("--no-workloads", action="store_true",
                    help="default run: skip the adjoint and elasticity workloads that a "
                         "single-GPU run carries in its line under 'workloads'")
    return ap.parse_args()


# The adjoint (48^3) and 3-unknowns-per-node (40^3 nodes) workloads: a
# default single-GPU run also runs them, each as a child process of its own
# mode, and carries their lines under "workloads"; a child that fails or runs
# past its time limit leaves an "error" entry instead and never stops the
# bench.
SUB_WORKLOADS = (("adjoint", ["--workload", "adjoint", "--steps", "3", "--warmup", "3"]),
                 ("elasticity", ["--workload", "elasticity", "--steps", "3", "--warmup", "3"]))


def run_sub_workloads(workloads=SUB_WORKLOADS, timeout_s=300.0, script=None):
    script = script or os.path.abspath(__file__)
    out = {}
    for name, extra in workloads:
        t0 = time.perf_counter()
        try:
            p = subprocess.run([sys.executable, script] + list(extra), capture_output=True,
                               text=True, timeout=timeout_s, cwd=ROOT)
            lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
            if p.returncode == 0 and lines:
                res = json.loads(lines[-1])
            else:
                res = {"error": "exit %d: %s" % (p.returncode, (p.stderr or p.stdout)[-300:])}
        except Exception as e:  # noqa: BLE001 - a timeout or a bad line is recorded
            res = {"error": str(e)[:300]}
        res["wall_s"] = time.perf_counter() - t0
        out[name] = res
    return out


def workload(side):
    from mdgpu_b200 import matgen as mg

    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(side, seed=0, sigma=1.0, shift=1e-3)
    b = mg.rhs_uniform(n, seed=0)
    return n, Ap, Ai, Ax, b


def config(side, extra=None):
    c = {"workload": "3D 7-point Laplacian %d^3 (n=%d), lognormal(0,1) edge conductances, "
                     "shift 1e-3, AMD + supernodes (-amd -sn), 1 RHS U(-1,1)" % (side, side ** 3),
         "matrix": "laplacian_3d_varcoef(side=%d, seed=0)" % side,
         "factor": "FP32 (TF32 tensor-core Schur on large fronts) + FP64 iterative refinement",
         "tolerance": 1e-14,
         "l2": "flushed between steps (256 MiB write); working set (L + update matrices) >> L2"}
    if extra:
        c.update(extra)
    return c


# ---------------------------------------------------------------------------
# reference CPU path (oracle/_ref, compiled from the reference sources)
# ---------------------------------------------------------------------------

def reference_cpu_sample(side, timeout=600):
    """Run the reference's own CPU Factor + cs_lsolve/cs_ltsolve on one core."""
    from mdgpu_b200 import matgen as mg
    from oracle import oracle as O

    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(side, seed=0)
    b = mg.rhs_uniform(n, seed=0)
    with tempfile.TemporaryDirectory() as d:
        mf = os.path.join(d, "A.txt")
        bf = os.path.join(d, "b.f64")
        mg.write_triplets(mf, n, Ap, Ai, Ax)
        b.tofile(bf)
        if os.path.exists(O.REF_HARNESS):
            cmd = ["taskset", "-c", "0", O.REF_HARNESS, "-amd", "-sn", "-bfile", bf, mf,
                   os.path.join(d, "out")]
            os.makedirs(os.path.join(d, "out"))
            try:
                subprocess.run(cmd, check=True, capture_output=True, timeout=timeout)
            except FileNotFoundError:
                subprocess.run(cmd[3:], check=True, capture_output=True, timeout=timeout)
            meta = O.load_dir(os.path.join(d, "out"))["meta"]
            t = meta["t_factor"] + meta["t_solve"]
            return {"value": meta["flops"] / t / 1e9, "unit": UNIT, "cores": 1,
                    "kind": "reference", "seconds": t, "resid": meta["resid_rel"],
                    "sample": "reference Factor + cs_lsolve + cs_ltsolve (oracle/_ref, FP64, "
                              "-amd -sn, 1 core) on the %d^3 grid of the same generator "
                              "(n=%d, %.3g flop)" % (side, n, meta["flops"])}
        # restated port (same arithmetic, bit-identical results)
        P = O.Plan(n, Ap, Ai, Ax, amd=True, mode="sn")
        t0 = time.perf_counter()
        F = P.factor()
        P.solve(F["Li"], F["Lx"], b)
        t = time.perf_counter() - t0
        return {"value": F["flops"] / t / 1e9, "unit": UNIT, "cores": 1, "kind": "port",
                "seconds": t,
                "sample": "oracle port of the reference CPU path on the %d^3 grid" % side}


def reference_cpu_system(n, Ap, Ai, Ax, b, timeout=600, core=0):
    """The reference's own CPU Factor + cs_lsolve/cs_ltsolve (-amd -sn, on
    host core `core`) on one system: (flops, seconds of factor + solve, kind)."""
    from mdgpu_b200 import matgen as mg
    from oracle import oracle as O

    with tempfile.TemporaryDirectory() as d:
        mf = os.path.join(d, "A.txt")
        bf = os.path.join(d, "b.f64")
        mg.write_triplets(mf, n, Ap, Ai, Ax)
        np.asarray(b, np.float64).tofile(bf)
        if os.path.exists(O.REF_HARNESS):
            out = os.path.join(d, "out")
            os.makedirs(out)
            cmd = ["taskset", "-c", str(core), O.REF_HARNESS, "-amd", "-sn", "-bfile", bf, mf,
                   out]
            try:
                subprocess.run(cmd, check=True, capture_output=True, timeout=timeout)
            except FileNotFoundError:
                subprocess.run(cmd[3:], check=True, capture_output=True, timeout=timeout)
            meta = O.load_dir(out)["meta"]
            return meta["flops"], meta["t_factor"] + meta["t_solve"], "reference"
        P = O.Plan(n, Ap, Ai, Ax, amd=True, mode="sn")
        t0 = time.perf_counter()
        F = P.factor()
        P.solve(F["Li"], F["Lx"], b)
        return F["flops"], time.perf_counter() - t0, "port"


def run_reference_workload_arm(args):
    """The reference's CPU path on a bounded sample of the batch or
    elasticity workload (the reference factors one system per run, on one
    core): batch -- every 64th of the 1024 systems (8 2D + 8 3D), one after
    another; elasticity -- the same generator at 12^3 nodes, cs_amd on the
    scalar matrix (the reference's -amd)."""
    from mdgpu_b200 import matgen as mg

    if int(os.environ.get("RANK", "0")) != 0:
        return
    if args.workload == "batch":
        syss = batch_systems()[::64]
        sample = ("every 64th of the 1024 systems (%d systems, n = %d), one per core"
                  % (len(syss), sum(s[0] for s in syss)))
        work = [(n, Ap, Ai, Ax, mg.rhs_uniform(n, seed=3)) for (n, Ap, Ai, Ax) in syss]
    else:
        n, Ap, Ai, Ax = mg.elasticity_3dof(12, seed=0, sigma=1.0, shift=1e-2)
        sample = "3 unknowns per node, 12^3 nodes (n = %d), -amd on the scalar matrix" % n
        work = [(n, Ap, Ai, Ax, mg.rhs_uniform(n, seed=1))]
    # the reference factors one system per process on one core; independent
    # systems run side by side, one per host core
    cores = max(1, min(len(work), os.cpu_count() or 1))
    for _ in range(args.warmup):
        reference_cpu_system(*work[0])
    rates, secs = [], []
    kind = "reference"
    from concurrent.futures import ThreadPoolExecutor

    for _ in range(args.steps):
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=cores) as ex:
            res = list(ex.map(lambda kw: reference_cpu_system(*kw[1], core=kw[0] % cores),
                              enumerate(work)))
        # each system's own factor + solve seconds, measured while the others
        # ran: the cores' throughput on a batch large enough to keep them all
        # busy is cores x flops / the summed seconds (the 1024 systems take
        # ~60x the largest one, so the packing is not the limit there)
        tsys = np.array([r[1] for r in res])
        fl = sum(r[0] for r in res)
        t = tsys.sum() / cores
        kind = res[0][2]
        rates.append(fl / t / 1e9)
        secs.append(t)
    v = statistics.median(rates)
    base = {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample,
            "seconds": statistics.median(secs),
            "timing": "cores x flops / summed per-system factor + solve seconds, the "
                      "systems run side by side one per core"}
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * statistics.median(secs), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "sample": sample, "cpu": cpu_info(),
                       "nproc": os.cpu_count(),
                       "note": "reference Factor + cs_lsolve + cs_ltsolve, one process per "
                               "system, %d at a time on separate cores" % cores},
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_info():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    for _ in range(args.warmup):
        reference_cpu_sample(12)
    vals, secs = [], []
    base = None
    for _ in range(args.steps):
        base = reference_cpu_sample(REF_SIDE)
        vals.append(base["value"])
        secs.append(base["seconds"])
    v = statistics.median(vals)
    base["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * statistics.median(secs), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config(REF_SIDE, {"cpu": cpu_info(), "nproc": os.cpu_count(),
                                        "note": "single-threaded reference (no threading in "
                                                "its CPU path); 64^3 would take ~12 min/step"}),
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def start(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

        def loop():
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.index),
                                          "--query-gpu=" + q, "--format=csv,noheader,nounits"],
                                         capture_output=True, text=True, timeout=5).stdout
                    self.rows.append([x.strip() for x in out.strip().split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)

        self._t = threading.Thread(target=loop, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        sm = [float(r[0]) for r in self.rows if len(r) >= 6 and r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if len(r) >= 6 and r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) >= 6:
                for k, nm in enumerate(names):
                    if r[2 + k].lower().startswith("active"):
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def measure_fp64_gemm_tflops():
    """Dense FP64 throughput of this GPU, measured: a cuBLAS DGEMM (torch,
    8192^3) timed with CUDA events after warm-up (the denominator of the FP64
    Schur update's roofline; the measured-peaks file holds HBM and bf16
    figures only)."""
    import torch

    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    bm = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, bm)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    reps = 5
    e0.record()
    for _ in range(reps):
        torch.matmul(a, bm)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    del a, bm
    return 2.0 * 8192 ** 3 / (ms * 1e-3) / 1e12


def roofline(prof, cls, peaks, peak_src, fp64_peak, class_kernels):
    """Roofline figures of one kernel class from a profiled step: achieved =
    algorithmic flops (tensor- or FP64-bound classes) or bytes per launch /
    the class's mean launch time (CUDA events on the launching stream).
    Peaks: 3xTF32 = sustained dense bf16 / 2 (TF32 rate) / 3 (three products
    per FP32 product); FP64 = the measured DGEMM rate; HBM = measured copy
    bandwidth."""
    if cls is None or cls not in prof["classes"]:
        return None
    c = prof["classes"][cls]
    per_launch_s = c["ms"] / c["launches"] * 1e-3
    if fp64_peak is not None and cls == "schur_update":
        peak, unit, bound = fp64_peak, "TFLOP/s", "fp64"
        achieved = c["flops"] / c["launches"] / per_launch_s / 1e12
        note = "measured cuBLAS DGEMM (8192^3) on this GPU; algorithmic FP64 flops"
    elif c["bound"] == "tensor":
        bf16 = peaks.get("bf16_tflops_sustained", peaks["bf16_tflops"])
        peak, unit, bound = bf16 / 2.0 / 3.0, "TFLOP/s", "tensor"
        achieved = c["flops"] / c["launches"] / per_launch_s / 1e12
        note = ("3xTF32 ceiling = %s sustained dense bf16 / 2 / 3; algorithmic FP32 flops"
                % peak_src)
    else:
        peak, unit, bound = peaks["hbm_gbs"], "GB/s", "hbm"
        achieved = c["bytes"] / c["launches"] / per_launch_s / 1e9
        note = "%s HBM copy bandwidth; algorithmic bytes" % peak_src
    ratio = TRAFFIC_PER_ALGO_BYTE.get(cls)
    traffic = ratio * c["bytes"] / c["launches"] if ratio is not None else None
    return {"kernel": cls, "kernels": class_kernels.get(cls, []), "bound": bound,
            "achieved": achieved, "peak": peak, "unit": unit, "frac": achieved / peak,
            "traffic": traffic,
            "algorithmic_bytes_per_launch": c["bytes"] / c["launches"],
            "flops_per_launch": c["flops"] / c["launches"],
            "traffic_source": ("ncu DRAM bytes per algorithmic byte of the class over three "
                               "48^3 steps, times this launch's algorithmic bytes"
                               if ratio is not None else None),
            "peak_source": note, "launches": c["launches"], "ms_total": c["ms"]}


def run_gpu_arm(args):
    import torch

    import mdgpu_b200 as M
    from mdgpu_b200 import matgen as mg

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def allmax(v):
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    side = args.side
    n, Ap, Ai, Ax, b = workload(side)
    # device memory the handle holds: driver-level free memory before and
    # after each stage (the library allocates with cudaMalloc, outside torch)
    free_a, _ = torch.cuda.mem_get_info()
    t0 = time.perf_counter()
    S = M.Solver(n, Ap, Ai)
    t_analyze = time.perf_counter() - t0
    free_b, _ = torch.cuda.mem_get_info()
    flops = float(S.info("flops"))
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    dAx = torch.from_numpy(Ax).cuda()
    db = torch.from_numpy(b).cuda()
    dx = torch.empty_like(db)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step_fp32():
        S.factor(dAx, M.FP32, stream=sptr)
        return S.refine_device(db, dx, tol=1e-14, maxit=30, stream=sptr)

    def step_fp64():
        S.factor(dAx, M.FP64, stream=sptr)
        return S.refine_device(db, dx, tol=1e-14, maxit=0, stream=sptr)

    def timed(fn, steps, warmup, profile=False):
        for _ in range(warmup):
            fn()
        barrier()
        times, extra = [], None
        for _ in range(steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            extra = fn()
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        barrier()
        return times, extra

    if args.only:
        fn = step_fp32 if args.only == "fp32" else step_fp64
        if args.only_nrhs > 1:
            Bq = mg.rhs_uniform(n, seed=1, nrhs=args.only_nrhs)
            db = torch.from_numpy(np.asfortranarray(Bq)).cuda().t().contiguous().t()
            dx = torch.empty((args.only_nrhs, n), dtype=torch.float64, device="cuda").t()
        t, _ = timed(fn, args.steps, args.warmup)
        if rank == 0:
            print(json.dumps({"only": args.only, "ms_per_step": statistics.mean(t)}), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return

    free_c, _ = torch.cuda.mem_get_info()
    sampler = ClockSampler(local)
    sampler.start()
    t32, (berr32, it32) = timed(step_fp32, args.steps, args.warmup)
    clocks = sampler.stop()
    x32 = dx.cpu().numpy()
    free_d, _ = torch.cuda.mem_get_info()
    # the plain FP64 factor + solve: the same steps, warm-up and clock record
    sampler64 = ClockSampler(local)
    sampler64.start()
    t64, (berr64, _) = timed(step_fp64, args.steps, args.warmup)
    clocks64 = sampler64.stop()
    x64 = dx.cpu().numpy()
    free_e, _ = torch.cuda.mem_get_info()
    hbm = {"plan": int(free_a - free_b), "fp32_factor_and_solve": int(free_c - free_d),
           "fp64_factor_added": int(free_d - free_e),
           "handle_total": int((free_a - free_b) + (free_c - free_e)),
           "lstore_bytes_fp64": int(S.info("lstore_bytes")),
           "ustore_bytes_fp64": int(S.info("ustore_bytes")),
           "ustore_bytes_fp64_without_reuse": int(S.info("ustore_total_bytes")),
           "note": "cudaMemGetInfo deltas (2 MiB granularity); the update-matrix store "
                   "is reused over the matrices' lifetimes in the level schedule"}
    ms32 = allmax(statistics.mean(t32))
    ms64 = allmax(statistics.mean(t64))

    # kernel-level evidence for the roofline: every kernel class, timed with
    # CUDA events around each of its launches during one extra step of each
    # precision
    prof = S.profile_step(lambda: step_fp32())
    prof64 = S.profile_step(lambda: step_fp64())

    # accuracy on the host, independent of the library's residual kernel:
    # backward error ||b - A x||inf / (||A||inf ||x||inf + ||b||inf) by a
    # scipy product with the caller's values, forward error against the
    # plain FP64 GPU solution
    A_full = mg.lower_to_full_scipy(n, Ap, Ai, Ax)
    a_inf = float(abs(A_full).sum(axis=1).max())

    def host_berr(x):
        return float(np.abs(b - A_full @ x).max() / (a_inf * np.abs(x).max() + np.abs(b).max()))

    def fwd_err(x):
        return float(np.abs(x - x64).max() / np.abs(x64).max())

    # end to end through the public API with host buffers
    Axh = np.ascontiguousarray(Ax)
    e2e_t = []
    for k in range(0 if args.no_e2e else args.warmup + args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        S.factor(Axh, M.FP32)
        x, be, _ = S.refine(b, tol=1e-14, maxit=30)
        torch.cuda.synchronize()
        if k >= args.warmup:
            e2e_t.append(time.perf_counter() - t0)
    e2e_ms = allmax(1e3 * statistics.mean(e2e_t)) if e2e_t else float("nan")

    # the same step with 64 right-hand sides (FP32 factor + FP64 refinement of
    # all 64 columns; device-resident, column-major)
    rhs64 = None
    if not args.no_rhs64:
        B64 = mg.rhs_uniform(n, seed=1, nrhs=64)
        dB64 = torch.from_numpy(np.asfortranarray(B64)).cuda().t().contiguous().t()
        dX64 = torch.empty((64, n), dtype=torch.float64, device="cuda").t()

        def step_fp32_64():
            S.factor(dAx, M.FP32, stream=sptr)
            return S.refine_device(dB64, dX64, tol=1e-14, maxit=30, stream=sptr)

        t64r, (be64, it64) = timed(step_fp32_64, max(1, min(args.steps, 3)), 1)
        ms64r = allmax(statistics.mean(t64r))
        X64 = dX64.cpu().numpy()
        R = B64 - A_full @ X64
        be_host = (np.abs(R).max(axis=0) /
                   (a_inf * np.abs(X64).max(axis=0) + np.abs(B64).max(axis=0)))
        prof64r = S.profile_step(lambda: step_fp32_64())
        # forward error of every column against the plain FP64 factor's
        # solution of the same 64 columns (after the timed steps)
        try:
            S.factor(dAx, M.FP64, stream=sptr)
            X64ref = S.solve(dB64, stream=sptr).cpu().numpy()
            fwd64 = float((np.abs(X64 - X64ref).max(axis=0) / np.abs(X64ref).max(axis=0)).max())
        except Exception as e:  # noqa: BLE001 - reported in the line
            fwd64 = "error: " + str(e)[:200]
        rhs64 = {"nrhs": 64, "ms_per_step": ms64r, "kernels": prof64r["classes"],
                 "max_backward_error": float(np.max(be64)),
                 "max_backward_error_host": float(be_host.max()), "max_forward_error": fwd64,
                 "ir_iterations": int(it64),
                 "solve_flops_per_rhs_sweep_pair": 4.0 * S.info("lnz"),
                 "note": "FP32 factor + FP64 refinement of 64 columns at once"}

    # the same step with GMRES-based refinement in place of plain refinement
    # (same FP32 factor, mdgpu_gmres_ir_device); an error here is reported in
    # the line rather than ending the run
    gmres = None
    if not args.no_gmres:
        def step_fp32_gmres():
            S.factor(dAx, M.FP32, stream=sptr)
            return S.gmres_ir_device(db, dx, tol=1e-14, maxit=10, stream=sptr)

        try:
            tg, (beg, itg, ing) = timed(step_fp32_gmres, max(1, min(args.steps, 3)), 1)
            xg = dx.cpu().numpy()
            gmres = {"ms_per_step": allmax(statistics.mean(tg)),
                     "backward_error": float(np.max(beg)),
                     "backward_error_host": host_berr(xg), "forward_error": fwd_err(xg),
                     "corrections": int(np.max(itg)), "gmres_steps": int(np.sum(ing)),
                     "note": "FP32 factor + GMRES-IR (restart 30, inner tolerance 1e-8)"}
        except Exception as e:  # noqa: BLE001
            gmres = {"error": str(e)[:300]}

    # the one-product TF32 Schur update (MDGPU_TF32) + GMRES-IR: a cheaper
    # factor against more preconditioned solves
    tf32 = None
    if not args.no_gmres:
        def step_tf32_gmres():
            S.factor(dAx, M.TF32, stream=sptr)
            return S.gmres_ir_device(db, dx, tol=1e-14, maxit=10, stream=sptr)

        try:
            tt, (bet, itt, intt) = timed(step_tf32_gmres, max(1, min(args.steps, 3)), 1)
            xt = dx.cpu().numpy()
            tf32 = {"ms_per_step": allmax(statistics.mean(tt)),
                    "backward_error": float(np.max(bet)),
                    "backward_error_host": host_berr(xt), "forward_error": fwd_err(xt),
                    "corrections": int(np.max(itt)), "gmres_steps": int(np.sum(intt)),
                    "precision_used": int(S.info("precision_used")),
                    "kernels": S.profile_step(step_tf32_gmres)["classes"],
                    "note": "FP32 factor with one-product TF32 Schur updates + GMRES-IR"}
        except Exception as e:  # noqa: BLE001
            tf32 = {"error": str(e)[:300]}

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    peaks, peak_src = measured_peaks()
    fp64_peak = measure_fp64_gemm_tflops()
    value = world * flops / (ms32 * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms32, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 factor (tf32 tensor-core Schur) + f64 refinement",
        "data": "synthetic",
        "config": config(side, {"n": n, "nnz_lower": int(Ap[-1]), "nsuper": S.info("nsuper"),
                                "lnz": S.info("lnz"), "flops_per_step": flops,
                                "parallelism": "replicas x%d (a single system does not shard)"
                                               % world,
                                "analyze_s": t_analyze}),
        "backward_error": float(berr32[0]), "backward_error_host": host_berr(x32),
        "forward_error": fwd_err(x32), "ir_iterations": int(it32),
        "fp64": {"ms_per_step": ms64, "value": world * flops / (ms64 * 1e-3) / 1e9,
                 "steps": args.steps, "warmup": args.warmup,
                 "backward_error": float(berr64[0]), "backward_error_host": host_berr(x64),
                 "speedup_fp32_ir_over_fp64": ms64 / ms32, "clocks": clocks64,
                 "kernels": prof64["classes"],
                 "roofline": roofline(prof64, "schur_update", peaks, peak_src, fp64_peak,
                                      CLASS_KERNELS_FP64)},
        "e2e": {"value": world * flops / (e2e_ms * 1e-3) / 1e9, "unit": UNIT,
                "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": int(Ax.nbytes + b.nbytes),
                "d2h_bytes_per_step": int(b.nbytes)},
        "rhs64": rhs64,
        "gmres_ir": gmres,
        "tf32_gmres_ir": tf32,
        "hbm_bytes": hbm,
        "gpu_launches": prof["launches_per_step"],
        "clocks": clocks,
        "roofline": roofline(prof, prof["dominant"], peaks, peak_src, None, CLASS_KERNELS),
        "kernels": prof["classes"],
    }
    if not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = reference_cpu_sample(CPU_BASELINE_SIDE)
    if not args.no_workloads and world == 1 and args.side == 64:
        try:
            line["workloads"] = run_sub_workloads()
        except Exception as e:  # noqa: BLE001 - never lose the line
            line["workloads"] = {"error": str(e)[:300]}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def batch_systems():
    """The many-systems workload: 512 2D 5-point grids (side U[16, 96]) and
    512 3D 7-point grids (side U[8, 32]), lognormal(0, 0.5) conductances,
    shift 1e-2, seeded."""
    from mdgpu_b200 import matgen as mg

    rng = np.random.default_rng(0)
    out = []
    for q in range(1024):
        if q < 512:
            dims = (int(rng.integers(16, 97)),) * 2
        else:
            dims = (int(rng.integers(8, 33)),) * 3
        out.append(mg.laplacian_grid(dims, seed=q, sigma=0.5, shift=1e-2))
    return out


def run_batch_arm(args):
    """Factor + solve of all 1024 systems (level-scheduled launches captured
    in CUDA graphs): FP32 factor + FP64 refinement of 4 right-hand sides per
    system vs the plain FP64 factor + solve.  One GPU: one handle over all
    systems.  N GPUs (one process each): the systems are split by estimated
    flops (longest processing time first, mdgpu_b200/shard.py), each rank
    factors and solves its share under one handle; no data-path exchange;
    the step time is the slowest rank's (strong scaling: the total work is
    fixed)."""
    import torch

    from mdgpu_b200 import FP32, FP64
    from mdgpu_b200 import matgen as mg
    from mdgpu_b200.shard import ShardedBatch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def allmax(v):
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    syss = batch_systems()
    t0 = time.perf_counter()
    SB = ShardedBatch(syss, rank, world)
    S = SB.solver
    t_an = time.perf_counter() - t0
    tuned = None
    if S is not None:
        # launch shapes of the small-front kernels for these fronts (config 3:
        # autotuned), chosen on the FP32 factor before anything is timed
        tuned = S.autotune(SB.local_values([s[3] for s in syss]), FP32)
    n = SB.n
    flops = float(SB.costs.sum())  # every system's, all ranks together
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    if S is not None:
        Ax = SB.local_values([s[3] for s in syss])
        B4 = mg.rhs_uniform(n, seed=3 + rank, nrhs=4)
        dAx = torch.from_numpy(Ax).cuda()
        dB = torch.from_numpy(np.asfortranarray(B4)).cuda().t().contiguous().t()
        dX = torch.empty((4, n), dtype=torch.float64, device="cuda").t()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        barrier()
        ts, extra = [], None
        for _ in range(steps):
            flush.fill_(1.0)
            barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            extra = fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(allmax(e0.elapsed_time(e1)))
        return statistics.mean(ts), extra

    def step32():
        if S is None:
            return np.zeros(0), 0
        S.factor(dAx, FP32, stream=sptr)
        return S.refine_device(dB, dX, tol=1e-14, maxit=30, stream=sptr)

    def step64():
        if S is None:
            return np.zeros(0), 0
        S.factor(dAx, FP64, stream=sptr)
        return S.refine_device(dB, dX, tol=1e-14, maxit=0, stream=sptr)

    sampler = ClockSampler(local)
    sampler.start()
    ms32, (be32, it32) = timed(step32, args.steps, args.warmup)
    clocks = sampler.stop()
    ms64, (be64, _) = timed(step64, max(1, min(args.steps, 3)), 1)
    be32 = allmax(float(np.max(be32)) if np.size(be32) else 0.0)
    be64 = allmax(float(np.max(be64)) if np.size(be64) else 0.0)
    it32 = int(allmax(float(it32)))
    loads = SB.load()
    if rank == 0:
        line = {"metric": METRIC, "value": flops / (ms32 * 1e-3) / 1e9, "unit": UNIT,
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms32, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None,
                "dtype": "f32 factor (tf32 tensor-core Schur) + f64 refinement",
                "data": "synthetic",
                "config": {"workload": "1024 systems: 512 2D 5-point (side U[16,96]) + 512 3D "
                                       "7-point (side U[8,32]), lognormal(0,0.5), shift 1e-2, "
                                       "AMD each, 4 RHS U(-1,1), one handle per GPU",
                           "n_total": int(sum(s[0] for s in syss)), "n_rank0": n,
                           "nsuper_rank0": S.info("nsuper") if S is not None else 0,
                           "flops_per_step": flops, "analyze_s_rank0": t_an,
                           "partition": "longest processing time first by estimated flops",
                           "load_gflop_per_rank": [float(v) / 1e9 for v in loads],
                           "autotuned_shapes_rank0": tuned,
                           "l2": "flushed between steps (256 MiB write)"},
                "backward_error": be32, "ir_iterations": it32,
                "fp64": {"ms_per_step": ms64, "value": flops / (ms64 * 1e-3) / 1e9,
                         "backward_error": be64,
                         "speedup_fp32_ir_over_fp64": ms64 / ms32},
                "clocks": clocks}
        print(json.dumps(line), flush=True)
    if dist is not None:
        barrier()
        dist.destroy_process_group()


def run_adjoint_arm(args):
    """loss = log det A(theta) + b' A(theta)^-1 b on the 48^3 7-point grid,
    edge conductances theta lognormal(0, 1), diagonal shift 1e-2, b U(-1,1).
    Forward: FP64 factor + solve + log det; backward: selected inverse +
    gradient of the lower-triangle values, then d loss / d theta_e =
    G(i,i) + G(j,j) - G(i,j) (A(i,i), A(j,j) gain theta_e, A(i,j) = -theta_e).
    Checked by central differences (h = 1e-6 theta_e) on 64 random edges and
    against an FP64 reference gradient on the same edges computed by solves,
    u' A^-1 u - (x_i - x_j)^2 with u = e_i - e_j (no selected inverse)."""
    import torch

    import mdgpu_b200 as M
    from mdgpu_b200 import matgen as mg

    side = 48
    n, Ap, Ai, Ax, lo, hi, cond = mg.laplacian_grid_edges((side,) * 3, seed=0, sigma=1.0,
                                                          shift=1e-2)
    b = mg.rhs_uniform(n, seed=1)
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    free0, total = torch.cuda.mem_get_info()
    S = M.Solver(n, Ap, Ai)
    dAx = torch.from_numpy(Ax).cuda()
    db = torch.from_numpy(b).cuda()

    def forward(v=None):
        S.factor(dAx if v is None else torch.from_numpy(v).cuda(), M.FP64, stream=sptr)
        x = S.solve(db, stream=sptr)
        return S.logdet(stream=sptr) + float(torch.dot(db, x)), x

    def backward(x):
        S.selinv(stream=sptr)
        return S.grad_lower(x, stream=sptr)

    def timed(fn, steps, warmup):
        out = None
        for _ in range(warmup):
            out = fn()
        ts = []
        for _ in range(steps):
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            out = fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.mean(ts), out

    ms_f, (loss, x) = timed(forward, args.steps, args.warmup)
    free1, _ = torch.cuda.mem_get_info()
    ms_b, G = timed(lambda: backward(x), args.steps, args.warmup)
    free2, _ = torch.cuda.mem_get_info()
    G = G.cpu().numpy()

    def pos(r, c_):
        seg = Ai[Ap[c_]:Ap[c_ + 1]]
        return Ap[c_] + int(np.searchsorted(seg, r))

    rng = np.random.default_rng(2)
    picked = rng.choice(len(cond), 64, replace=False)
    # FP64 reference gradient by solves, independent of the selected inverse:
    # d loss / d theta_e = u' A^-1 u - (x_i - x_j)^2 with u = e_i - e_j (one
    # 64-column solve with the same FP64 factor)
    U = np.zeros((n, len(picked)))
    U[lo[picked], np.arange(len(picked))] = 1.0
    U[hi[picked], np.arange(len(picked))] = -1.0
    Zu = S.solve(U)
    xh = x.cpu().numpy()
    ref_worst = 0.0
    for k, e in enumerate(picked):
        i, j = int(lo[e]), int(hi[e])
        g = G[pos(i, i)] + G[pos(j, j)] - G[pos(j, i)]
        gref = Zu[i, k] - Zu[j, k] - (xh[i] - xh[j]) ** 2
        ref_worst = max(ref_worst, abs(g - gref) / max(abs(gref), 1e-300))
    worst = 0.0
    for e in picked:
        i, j = int(lo[e]), int(hi[e])
        pii, pjj, pij = pos(i, i), pos(j, j), pos(j, i)
        g = G[pii] + G[pjj] - G[pij]
        h = 1e-6 * cond[e]
        vals = []
        for sgn in (1.0, -1.0):
            v = Ax.copy()
            v[pii] += sgn * h
            v[pjj] += sgn * h
            v[pij] -= sgn * h
            vals.append(forward(v)[0])
        fd = (vals[0] - vals[1]) / (2 * h)
        worst = max(worst, abs(fd - g) / max(abs(g), 1e-300))
    line = {"metric": "adjoint: backward / forward time (FP64 factor+solve+logdet vs selected "
                      "inverse + gradient)",
            "value": ms_b / ms_f, "unit": "ratio", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": False, "data": "synthetic",
            "dtype": "f64",
            "config": {"workload": "3D 7-point Laplacian 48^3 (n=110592), edge conductances "
                                   "lognormal(0,1), shift 1e-2, AMD + supernodes, loss = "
                                   "log det A + b'A^-1 b, b U(-1,1)",
                       "n": n, "edges": int(len(cond)), "nsuper": S.info("nsuper"),
                       "lnz": S.info("lnz")},
            "forward_ms": ms_f, "backward_ms": ms_b, "loss": loss,
            "fd_edges": 64, "fd_max_rel_err": worst,
            "solve_reference_max_rel_err": ref_worst,
            "solve_reference": "u' A^-1 u - (x_i - x_j)^2, u = e_i - e_j, by FP64 solves on "
                               "the same 64 edges",
            "hbm_bytes": {"after_forward": int(free0 - free1),
                          "backward_extra": int(free1 - free2),
                          "zustore_bytes": int(S.info("zustore_bytes")),
                          "note": "the selected inverse's update parts have their own store, "
                                  "reused over their top-down lifetimes; nothing is "
                                  "recomputed"}}
    print(json.dumps(line), flush=True)


def run_elasticity_arm(args):
    """The multi-unknown system: 3 unknowns per node of a side^3 node grid
    (--elastic-side, 40 by default: n = 192000) with 27-point connectivity,
    blocks w (I + 0.5 e e'), w
    lognormal(0, 1), shift 1e-2, AMD on the node graph expanded to the
    unknowns.  One step = factor + solve to backward error 1e-14 of one
    right-hand side: BF16-update factor + GMRES-IR (the line's value), then
    FP32 factor + GMRES-IR, FP32 factor + plain refinement, FP64 factor +
    solve."""
    import torch

    import mdgpu_b200 as M
    from mdgpu_b200 import matgen as mg

    side = args.elastic_side
    n, Ap, Ai, Ax = mg.elasticity_3dof(side, seed=0, sigma=1.0, shift=1e-2)
    nn, gp, gi, _ = mg.node_graph_lower(side)
    perm = mg.expand_node_perm(M.Solver(nn, gp, gi, ordering=M.ORDER_AMD).array("perm"))
    n, Ap, Ai, Ax = mg.permute_lower(n, Ap, Ai, Ax, perm)
    t0 = time.perf_counter()
    S = M.Solver(n, Ap, Ai, ordering=M.ORDER_NATURAL)
    t_an = time.perf_counter() - t0
    flops = float(S.info("flops"))
    b = mg.rhs_uniform(n, seed=1)
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    dAx = torch.from_numpy(Ax).cuda()
    dB = torch.from_numpy(b).cuda()
    dX = torch.empty(n, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        ts, extra = [], None
        for _ in range(steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            extra = fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.mean(ts), extra

    def step_bf16_gmres():
        S.factor(dAx, M.BF16, stream=sptr)
        return S.gmres_ir_device(dB, dX, tol=1e-14, maxit=10, stream=sptr)

    def step_gmres():
        S.factor(dAx, M.FP32, stream=sptr)
        return S.gmres_ir_device(dB, dX, tol=1e-14, maxit=10, stream=sptr)

    def step_tf32_gmres():
        S.factor(dAx, M.TF32, stream=sptr)
        return S.gmres_ir_device(dB, dX, tol=1e-14, maxit=10, stream=sptr)

    def step_ir():
        S.factor(dAx, M.FP32, stream=sptr)
        return S.refine_device(dB, dX, tol=1e-14, maxit=30, stream=sptr)

    def step64():
        S.factor(dAx, M.FP64, stream=sptr)
        return S.refine_device(dB, dX, tol=1e-14, maxit=0, stream=sptr)

    A_full = mg.lower_to_full_scipy(n, Ap, Ai, Ax)
    a_inf = float(abs(A_full).sum(axis=1).max())

    def host_berr(x):
        return float(np.abs(b - A_full @ x).max() / (a_inf * np.abs(x).max() + np.abs(b).max()))

    sampler = ClockSampler(0)
    sampler.start()
    ms_b, (be_b, it_b, in_b) = timed(step_bf16_gmres, args.steps, args.warmup)
    clocks = sampler.stop()
    x_b = dX.cpu().numpy()
    prec_b = int(S.info("precision_used"))
    ms_g, (be_g, it_g, in_g) = timed(step_gmres, max(1, min(args.steps, 3)), 1)
    x_g = dX.cpu().numpy()
    ms_t, (be_t, it_t, in_t) = timed(step_tf32_gmres, max(1, min(args.steps, 3)), 1)
    x_t = dX.cpu().numpy()
    ms_ir, (be_ir, it_ir) = timed(step_ir, max(1, min(args.steps, 3)), 1)
    x_ir = dX.cpu().numpy()
    ms64, (be64, _) = timed(step64, max(1, min(args.steps, 3)), 1)
    x64 = dX.cpu().numpy()
    # where the time goes: the factor alone per precision, and the kernel
    # classes of one step of each precision mode
    factor_ms = {}
    for name, prec in (("bf16", M.BF16), ("tf32", M.TF32), ("fp32", M.FP32), ("fp64", M.FP64)):
        factor_ms[name], _ = timed(lambda: S.factor(dAx, prec, stream=sptr), 2, 1)
    kernels = {"bf16_gmres_ir": S.profile_step(step_bf16_gmres)["classes"],
               "fp32_gmres_ir": S.profile_step(step_gmres)["classes"]}

    def fwd(x):
        return float(np.abs(x - x64).max() / np.abs(x64).max())

    line = {"metric": METRIC, "value": flops / (ms_b * 1e-3) / 1e9, "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_b,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 factor with bf16 tensor-core Schur updates + f64 GMRES-IR",
            "data": "synthetic",
            "config": {"workload": "3 unknowns per node, %d^3 node grid, 27-point, blocks "
                                   "w(I+0.5ee'), w lognormal(0,1), shift 1e-2, node-graph AMD, "
                                   "1 RHS U(-1,1)" % side,
                       "n": n, "nsuper": S.info("nsuper"), "lnz": S.info("lnz"),
                       "flops_per_step": flops, "analyze_s": t_an,
                       "l2": "flushed between steps (256 MiB write)"},
            "backward_error": float(np.max(be_b)), "backward_error_host": host_berr(x_b),
            "forward_error": fwd(x_b), "corrections": int(np.max(it_b)),
            "gmres_steps": int(np.sum(in_b)),
            "precision_used": {0: "fp64", 1: "fp32 (bf16 fell back)", 2: "bf16"}[prec_b],
            "tf32_gmres_ir": {"ms_per_step": ms_t, "backward_error": float(np.max(be_t)),
                              "backward_error_host": host_berr(x_t), "forward_error": fwd(x_t),
                              "corrections": int(np.max(it_t)),
                              "gmres_steps": int(np.sum(in_t))},
            "fp32_gmres_ir": {"ms_per_step": ms_g, "backward_error": float(np.max(be_g)),
                              "backward_error_host": host_berr(x_g), "forward_error": fwd(x_g),
                              "corrections": int(np.max(it_g)),
                              "gmres_steps": int(np.sum(in_g))},
            "fp32_plain_ir": {"ms_per_step": ms_ir, "backward_error": float(np.max(be_ir)),
                              "backward_error_host": host_berr(x_ir), "forward_error": fwd(x_ir),
                              "corrections": int(it_ir)},
            "fp64": {"ms_per_step": ms64, "value": flops / (ms64 * 1e-3) / 1e9,
                     "backward_error": float(np.max(be64)), "backward_error_host": host_berr(x64),
                     "speedup_bf16_gmres_ir_over_fp64": ms64 / ms_b},
            "fp64_diag_tiles": int(S.info("fp64_diag_tiles")),
            "factor_ms": factor_ms, "kernels": kernels,
            "clocks": clocks}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.workload == "batch" and args.impl != "reference":
        run_batch_arm(args)
        return
    if args.workload == "adjoint" and args.impl != "reference":
        run_adjoint_arm(args)
        return
    if args.workload == "elasticity" and args.impl != "reference":
        run_elasticity_arm(args)
        return
    if args.impl == "reference" and args.workload in ("batch", "elasticity"):
        run_reference_workload_arm(args)
    elif args.impl == "reference":
        run_reference_arm(args)
    else:
        run_gpu_arm(args)


if __name__ == "__main__":
    main()
