#!/usr/bin/env python3
"""AMG-PCG time-to-1e-8 on the 128³ heterogeneous-diffusion system, B200.

Workload (one "step" = one full solve from x0 = 0 to a relative residual
of 1e-8, checked in FP64):
  3-D 7-point finite-volume diffusion on a 128³ grid, permeability
  κ = exp(g), g a seeded Gaussian random field (σ = 3, correlation length 8
  cells), harmonic-mean face transmissibilities, Dirichlet faces; b ~ U(-1,1).
  Hierarchy: hypre_default_config(agg_trunc_factor=0.2) with l1-Jacobi
  (HMIS θ=0.5, aggressive HMIS on level 1, extended+i interpolation),
  V(1,1).  Solver: conjugate gradients preconditioned by one AMG cycle.
  `value` = mean time of the FP64 solve (FP64 hierarchy, cycle and outer
  CG: the reference's arithmetic); the mixed-precision solve (FP32
  hierarchy and cycle, FP64 outer residual / products / dots / updates) is
  timed beside it ("mixed", "speedup_mixed_vs_fp64").  Inputs stay in HBM;
  the finest matrix alone (175 MB) exceeds the 126 MB L2, so no L2 flush is
  needed between steps.  `e2e` is the FP64 solve through the C ABI
  (draugr_b200_pcg) with pinned host x and b.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

--impl reference times the reference's CPU solve (the oracle restatement of
Draugr.jl's cycle inside a textbook PCG, all host cores) on the same
system and hierarchy structure; the structure is built by a child process
(--write-structure) so that the timed process loads only the oracle.
"""

from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "draugr.jl_b200"))

METRIC = ("AMG-PCG time-to-1e-8 (s) at 128³, mixed vs FP64 on B200; V-cycle HBM GB/s")
TOL = 1e-8
MAXITER = 500


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=128, help="grid side (128 = the quoted workload)")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--kernel-only", action="store_true",
                    help="only time one level kernel (for profiling): --level --op --precision --reps")
    ap.add_argument("--level", type=int, default=0)
    ap.add_argument("--op", type=int, default=2, help="2 = smoother sweep, 0 = SpMV")
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--resetup", action="store_true",
                    help="the 27-point coefficient-update workload: time GPU partial resetups "
                         "(numeric Galerkin products) at --n^3 nodes, then PCG on the result")
    ap.add_argument("--updates", type=int, default=20)
    ap.add_argument("--profile-block", action="store_true",
                    help="run exactly one block PCG solve (3D Poisson 96^3, 32 right-hand sides, mixed)")
    ap.add_argument("--profile-resetup", action="store_true",
                    help="run two partial resetups (27-point anisotropic diffusion on --n^3 nodes)")
    ap.add_argument("--batch", action="store_true",
                    help="the batching workload: 64 independent 3D Poisson systems (sides 16..64) "
                         "solved concurrently, and one 96^3 operator with 32 right-hand sides")
    ap.add_argument("--systems", type=int, default=64)
    ap.add_argument("--workers", type=int, default=16)
    ap.add_argument("--profile-solve", choices=["fp64", "mixed"], default=None,
                    help="run exactly one PCG solve in this precision (for profiling)")
    ap.add_argument("--profile-batch", action="store_true",
                    help="run exactly one segmented batched solve of the batching workload's 64 systems")
    ap.add_argument("--write-structure", default=None, metavar="PATH",
                    help="build the workload's hierarchy structure on the host (no GPU) and write "
                         "it with the right-hand side to PATH (.npz) for the reference arm")
    return ap.parse_args()


def workload(n, seed):
    from draugr import problems
    import draugr

    A = problems.heterogeneous_diffusion_3d(n, sigma=3.0, corr_len=8.0, seed=seed)
    b = problems.rhs(A.shape[0], seed + 1)
    cfg = draugr.hypre_default_config(agg_trunc_factor=0.2, smoother=draugr.L1JacobiSmootherType(),
                                      seed=seed)
    return A, b, cfg


def workload_config(n, rows, nnz, h=None):
    d = {"workload": f"3D 7-point heterogeneous diffusion {n}^3 (kappa=exp(g), sigma=3, "
                     "corr. length 8), hypre_default_config(agg_trunc_factor=0.2) + l1-Jacobi "
                     "V(1,1), AMG-PCG to 1e-8 from x0=0",
         "n": int(rows), "nnz": int(nnz), "tol": TOL,
         "l2": "inputs larger than L2 (finest matrix alone 175 MB > 126 MB); no flush"}
    if h is not None:
        nl = h.nlevels
        rows = [int(h.level_info(l)[0]) for l in range(nl)] + [int(h.level_info(-1)[0])]
        nnzs = [int(h.level_info(l)[1]) for l in range(nl)]
        d.update(levels=nl + 1, level_rows=rows, level_nnz=nnzs,
                 level_nnzP=[int(h.level_info(l)[3]) for l in range(nl)],
                 operator_complexity=round(sum(nnzs) / nnzs[0], 3) if nnzs else None)
    return d


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(name):
    """Per-launch DRAM bytes of a kernel from a committed ncu summary line
    'traffic_bytes_per_launch <name> <bytes>' under profiles/, else None."""
    for f in sorted((ROOT / "profiles").glob("*.md")):
        for line in f.read_text().splitlines():
            parts = line.strip().strip("`").split()
            if len(parts) == 3 and parts[0] == "traffic_bytes_per_launch" and parts[1] == name:
                return float(parts[2])
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = pathlib.Path(f"/tmp/draugr_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}", "--format=csv,noheader",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1].split()[0]))
                smax.append(float(f[2].split()[0]))
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        self.path.unlink(missing_ok=True)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = "nccl" if args.impl == "ours" else "gloo"
        if args.impl == "ours":
            import torch

            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def max_over_ranks(v, world):
    """The largest of every rank's v (a device tensor under NCCL, a host one
    under gloo)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def repo_libraries():
    """Shared objects under this repository mapped into this process."""
    try:
        maps = pathlib.Path("/proc/self/maps").read_text().splitlines()
    except OSError:
        return None
    root = str(ROOT)
    return sorted({ln.split()[-1][len(root) + 1:] for ln in maps
                   if ln.split()[-1].startswith(root) and ".so" in ln.split()[-1]})


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# --------------------------------------------------------------------- ours
def run_ours(args, world, rank, local):
    import torch

    import draugr

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    A, b, cfg = workload(args.n, args.seed)
    n = A.shape[0]
    # setup for the device, its Galerkin products on the CPU and then on the
    # GPU (the offload), after a small setup has loaded the kernels
    from draugr import problems as _pb
    draugr.amg_setup(_pb.poisson3d(16), cfg).free()
    os.environ["DRAUGR_B200_GPU_SETUP"] = "0"
    t0 = time.time()
    hh = draugr.amg_setup(A, cfg)
    setup_host_s = time.time() - t0
    hh.free()
    os.environ.pop("DRAUGR_B200_GPU_SETUP", None)
    t0 = time.time()
    h = draugr.amg_setup(A, cfg)
    setup_s = time.time() - t0
    stream = torch.cuda.current_stream()
    h.set_stream(stream)
    bd = torch.tensor(b, dtype=torch.float64, device=dev)
    xd = torch.zeros(n, dtype=torch.float64, device=dev)
    bnorm = np.linalg.norm(b)

    def solve(mode):
        xd.zero_()
        return draugr.pcg(xd, bd, h, cfg, tol=TOL, maxiter=MAXITER, precision=mode)

    def timed(mode, steps):
        times, its = [], []
        for _ in range(steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            xd.zero_()
            e0.record(stream)
            _, it, _ = draugr.pcg(xd, bd, h, cfg, tol=TOL, maxiter=MAXITER, precision=mode)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
            its.append(it)
        return times, its

    res = {}
    for mode in ("fp64", "mixed"):
        for _ in range(args.warmup):
            solve(mode)
        torch.cuda.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        if mode == "fp64":  # the headline value: the reference's arithmetic, FP64 throughout
            launches0 = draugr.load().draugr_b200_kernel_launches()
            with ClockSampler(local) as cs:
                times, its = timed(mode, args.steps)
            launches = draugr.load().draugr_b200_kernel_launches() - launches0
            clocks = cs.summary()
        else:
            times, its = timed(mode, args.steps)
        torch.cuda.synchronize()
        barrier(world)
        x = xd.cpu().numpy()
        rr = float(np.linalg.norm(b - A @ x) / bnorm)
        res[mode] = {"time_s": max_over_ranks(float(np.mean(times)), world),
                     "time_s_min": float(np.min(times)), "iterations": int(its[-1]),
                     "relres_fp64_verified": rr}
        if rr >= TOL:
            raise SystemExit(f"{mode} solve did not reach {TOL}: {rr}")

    # end-to-end through the C ABI with host buffers (pinned host memory):
    # H2D of x0 and b, D2H of x, all inside the timed region
    xh = torch.zeros(n, dtype=torch.float64, pin_memory=True).numpy()
    bh = torch.zeros(n, dtype=torch.float64, pin_memory=True).numpy()
    bh[:] = b

    def e2e_time(mode):
        ts = []
        for k in range(args.warmup + args.steps):
            xh[:] = 0.0
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            draugr.pcg(xh, bh, h, cfg, tol=TOL, maxiter=MAXITER, precision=mode)
            e1.record(stream)
            e1.synchronize()
            if k >= args.warmup:
                ts.append(e0.elapsed_time(e1) / 1e3)
        rr = float(np.linalg.norm(b - A @ xh) / bnorm)
        if rr >= TOL:
            raise SystemExit(f"{mode} solve through the C ABI did not reach {TOL}: {rr}")
        return max_over_ranks(float(np.mean(ts)), world)

    # the other Krylov forms on the same system: FGMRES(30) with the FP32
    # cycle, and iterative refinement (FP64 residual, mixed PCG to 1e-4 inside)
    def other(fn, key):
        for _ in range(2):
            xd.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = fn()
            e1.record(stream)
            e1.synchronize()
        x = xd.cpu().numpy()
        d = {"time_s": e0.elapsed_time(e1) / 1e3, "relres_fp64_verified": float(np.linalg.norm(b - A @ x) / bnorm)}
        d.update(key(r))
        return d

    krylov = {
        "fgmres_mixed": other(lambda: draugr.fgmres(xd, bd, h, cfg, tol=TOL, maxiter=MAXITER, restart=30,
                                                    precision="mixed"),
                              lambda r: {"iterations": int(r[1])}),
        "refine_mixed_pcg": other(lambda: draugr.refine(xd, bd, h, cfg, tol=TOL, inner_tol=1e-4,
                                                        inner="pcg", precision="mixed"),
                                  lambda r: {"steps": int(r[1]), "inner_iterations": int(r[2])}),
    }

    e2e = {"value": e2e_time("fp64"), "unit": "s",
           "h2d_bytes_per_step": 2 * n * 8, "d2h_bytes_per_step": n * 8,
           "path": "draugr_b200_pcg, precision 0 (C ABI, pinned host x and b, FP64 cycle)",
           "mixed": e2e_time("mixed")}

    # roofline of the dominant kernels: finest-level Jacobi sweep and SpMV
    nnz = A.nnz
    kern = {}
    for name, op, prec, byts in (
            ("l1_jacobi_fp64_level1", 2, 0, 12 * nnz + 4 * (n + 1) + 32 * n),
            ("l1_jacobi_fp32_level1", 2, 1, 8 * nnz + 4 * (n + 1) + 16 * n),
            ("spmv_fp64_level1", 0, 0, 12 * nnz + 4 * (n + 1) + 16 * n),
            ("spmv_fp32_level1", 0, 1, 8 * nnz + 4 * (n + 1) + 8 * n)):
        ms = h.time_level_op(0, op, prec, reps=50)
        kern[name] = {"bytes": int(byts), "ms": ms, "GBps": byts / (ms * 1e-3) / 1e9}
    peak, peak_kind = peaks()
    dom = kern["l1_jacobi_fp64_level1"]
    roofline = {"bound": "hbm", "kernel": "l1_jacobi_fp64_level1 (k_tile_rows: one lane per row, 256 threads, EpJacobi; finest level)",
                "achieved": round(dom["GBps"], 1), "peak": peak, "unit": "GB/s",
                "frac": round(dom["GBps"] / peak, 3),
                "traffic": profiled_traffic("l1_jacobi_fp64_level1"),
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                else "fallback 6.65 TB/s",
                "algorithmic_bytes_per_launch": dom["bytes"],
                "timing": "CUDA events on the hierarchy's stream, 50 launches after 3 warm-up, "
                          "run after the timed solves",
                "kernels": {k: {kk: (round(vv, 4) if isinstance(vv, float) else vv)
                                for kk, vv in v.items()} for k, v in kern.items()}}

    # the whole V-cycle: algorithmic bytes of the kernels one FP64 V(1,1)
    # cycle launches, per level, against the cycle's event-timed duration
    vc_bytes = vcycle_bytes(h)
    xc = torch.zeros(n, dtype=torch.float64, device=dev)
    for _ in range(3):
        draugr.amg_cycle(xc, bd, h, cfg)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ncyc = 20
    e0.record(stream)
    for _ in range(ncyc):
        draugr.amg_cycle(xc, bd, h, cfg)
    e1.record(stream)
    e1.synchronize()
    vc_ms = e0.elapsed_time(e1) / ncyc
    vcycle = {"precision": "fp64", "ms": round(vc_ms, 4), "algorithmic_bytes": int(vc_bytes),
              "GBps": round(vc_bytes / (vc_ms * 1e-3) / 1e9, 1),
              "frac": round(vc_bytes / (vc_ms * 1e-3) / 1e9 / peak, 3),
              "note": "V(1,1) through draugr_b200_cycle_device, 20 cycles after 3 warm-up; bytes: "
                      "per level the residual (12 nnz + 4 (n+1) + 24 n), restriction, prolongation and "
                      "the Jacobi sweep formulas (two sweeps on the finest level, whose pre-smoothing "
                      "starts from a given x; the coarser levels' first sweep is formed in the "
                      "restriction), shared-memory tail levels included at their global-memory size"}

    out = {"metric": METRIC, "value": res["fp64"]["time_s"], "unit": "s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": res["fp64"]["time_s"] * 1e3, "higher_is_better": False,
           "scaling": "weak", "vs_baseline": None,
           "dtype": "f64 (value, e2e: FP64 cycle and outer CG); 'mixed': f32 hierarchy and cycle "
                    "inside f64 CG",
           "data": "synthetic (seeded log-normal permeability field, b ~ U(-1,1))",
           "config": dict(workload_config(args.n, n, A.nnz, h),
                          parallelism=f"replicas x{world}" if world > 1 else "1 GPU"),
           "setup_s": round(setup_s, 3), "setup_s_galerkin_on_cpu": round(setup_host_s, 3),
           "fp64": res["fp64"], "mixed": res["mixed"],
           "speedup_mixed_vs_fp64": res["fp64"]["time_s"] / res["mixed"]["time_s"],
           "krylov": krylov,
           "e2e": e2e, "roofline": roofline, "vcycle": vcycle, "clocks": clocks,
           "loaded_repo_libraries": repo_libraries(),
           "gpu_launches": int(launches)}

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(h, b, cfg)
    h.set_stream(None)
    return out


def vcycle_bytes(h):
    """Algorithmic bytes of one FP64 V(1,1) cycle (the reference's passes):
    per level the residual (12 nnz + 4 (n+1) + 24 n), restriction,
    prolongation and Jacobi sweep formulas, two sweeps on the finest level."""
    total = 0
    for l in range(h.nlevels):
        info = h.level_info(l)
        ln, lnnz, lnc, lnnzp = int(info[0]), int(info[1]), int(info[2]), int(info[3])
        resid = lnnz * 12 + 4 * (ln + 1) + 3 * ln * 8
        total += resid + op_bytes(3, 0, ln, lnnz, lnc, lnnzp) + op_bytes(4, 0, ln, lnnz, lnc, lnnzp)
        total += op_bytes(2, 0, ln, lnnz, lnc, lnnzp) * (2 if l == 0 else 1)
    return total


def cpu_vcycle(h, b, cfg, reps=3):
    """The oracle's FP64 V(1,1) cycle on the host cores: mean seconds per
    cycle (one warm-up) and the same algorithmic GB/s as the GPU cycle."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    O = oracle.OracleHierarchy(h)
    x0 = np.random.default_rng(7).uniform(-1, 1, len(b))
    O.cycle(x0, b, cfg.pre_smoothing_steps, cfg.post_smoothing_steps, cfg.cycle_type == "W")
    t0 = time.perf_counter()
    for _ in range(reps):
        O.cycle(x0, b, cfg.pre_smoothing_steps, cfg.post_smoothing_steps, cfg.cycle_type == "W")
    t = (time.perf_counter() - t0) / reps
    return t, vcycle_bytes(h) / t / 1e9


def cpu_solve_time(h, b, cfg, reps=1):
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    O = oracle.OracleHierarchy(h)
    n = len(b)
    ts = []
    its = 0
    for _ in range(reps):
        t0 = time.perf_counter()
        x, its, rel = O.pcg(np.zeros(n), b, cfg.pre_smoothing_steps, cfg.post_smoothing_steps,
                            cfg.cycle_type == "W", TOL, MAXITER)
        ts.append(time.perf_counter() - t0)
    return float(np.mean(ts)), its


def cpu_baseline(h, b, cfg):
    t, its = cpu_solve_time(h, b, cfg)
    vt, vg = cpu_vcycle(h, b, cfg)
    return {"value": t, "unit": "s", "cores": os.cpu_count(), "kind": "port",
            "iterations": its, "vcycle_ms": round(vt * 1e3, 2), "vcycle_GBps": round(vg, 1),
            "sample": "one full AMG-PCG solve (FP64 cycle) of the same system and hierarchy "
                      "to 1e-8, oracle restatement of the reference's CPU kernels, OpenMP "
                      "static/64-row chunks on all host threads"}


# --------------------------------------------------------------- reference
def write_structure(args):
    """--write-structure: the workload's hierarchy structure, built on the
    host by the library's setup (no GPU is touched), written with b for
    the reference arm, which then loads only the oracle."""
    import draugr

    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    A, b, cfg = workload(args.n, args.seed)
    t0 = time.time()
    h = draugr.amg_setup(A, cfg, on_device=False)
    oracle.save_structure(h, args.write_structure, b=b, setup_s=time.time() - t0,
                          pre=cfg.pre_smoothing_steps, post=cfg.post_smoothing_steps,
                          w=int(cfg.cycle_type == "W"))
    h.free()


def run_reference(args, world, rank):
    """The reference's CPU solve phase (the oracle's restatement of
    Draugr.jl's kernels, OpenMP on all host threads) on the same hierarchy
    structure.  The structure is built in a child process (the input, not
    the timed path); this process loads nothing but the oracle."""
    if rank != 0:
        return None
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    path = pathlib.Path(f"/tmp/draugr_structure_n{args.n}_s{args.seed}_{os.getpid()}.npz")
    subprocess.run([sys.executable, str(ROOT / "bench.py"), "--write-structure", str(path),
                    "--n", str(args.n), "--seed", str(args.seed)], check=True)
    try:
        S = oracle.StructureFile(path)
    finally:
        path.unlink(missing_ok=True)
    b = S.extra("b")
    pre, post, w = int(S.extra("pre")), int(S.extra("post")), bool(int(S.extra("w")))
    O = oracle.OracleHierarchy(S)
    nrows = len(b)
    times = []
    its = 0
    x = None
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        x, its, rel = O.pcg(np.zeros(nrows), b, pre, post, w, TOL, MAXITER)
        if k >= args.warmup:
            times.append(time.perf_counter() - t0)
    rp, ci, av = S.export(0, "A_rowptr"), S.export(0, "A_colval"), S.export(0, "A_nzval")
    rr = float(np.linalg.norm(oracle.residual(nrows, rp, ci, av, x, b)) / np.linalg.norm(b))
    v = float(np.mean(times))
    # one V-cycle on the host cores, with the GPU cycle's algorithmic bytes
    x0 = np.random.default_rng(7).uniform(-1, 1, nrows)
    O.cycle(x0, b, pre, post, w)
    t0 = time.perf_counter()
    for _ in range(3):
        O.cycle(x0, b, pre, post, w)
    vt = (time.perf_counter() - t0) / 3
    sample = ("full AMG-PCG solve per step (FP64 cycle), oracle restatement of Draugr.jl's "
              "CPU kernels (Julia is not available), OpenMP on all host threads")
    return {"metric": METRIC, "impl": "reference", "value": v, "unit": "s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded log-normal permeability field, b ~ U(-1,1))",
            "config": dict(workload_config(args.n, nrows, len(ci), S),
                           parallelism=f"replicas x{world}" if world > 1 else "1 GPU"),
            "setup_s_cpu": round(float(S.extra("setup_s")), 3),
            "iterations": its, "relres_fp64_verified": rr,
            "structure": "hierarchy structure built by the library's host setup in a child "
                         "process (bench.py --write-structure); this process loads only the oracle",
            "loaded_repo_libraries": repo_libraries(),
            "cpu_baseline": {"value": v, "unit": "s", "cores": os.cpu_count(), "kind": "port",
                             "sample": sample, "vcycle_ms": round(vt * 1e3, 2),
                             "vcycle_GBps": round(vcycle_bytes(S) / vt / 1e9, 1)},
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


OPS = {0: "spmv", 2: "jacobi", 3: "restrict", 4: "prolong", 6: "zero_jacobi_residual"}


def op_bytes(op, prec, n, nnz, nc, nnzp):
    """Algorithmic bytes of one level kernel: every operand counted once,
    the x gather once per vector entry (ideal reuse), int32 indices, and
    V = 8 bytes per value and vector entry in FP64, 4 in FP32."""
    V = 8 if prec == 0 else 4
    if op == 0:
        return nnz * (4 + V) + 4 * (n + 1) + 2 * n * V
    if op in (2, 6):
        return nnz * (4 + V) + 4 * (n + 1) + 4 * n * V
    if op == 3:
        return nnzp * (4 + V) + 4 * (nc + 1) + n * V + nc * V
    if op == 4:
        return nnzp * (4 + V) + 4 * (n + 1) + nc * V + 2 * n * V
    raise ValueError(op)


def level_table(h, reps=20, precisions=(0, 1), ops=(2, 6, 3, 4)):
    peak, _ = peaks()
    rows = []
    for l in range(h.nlevels):
        info = h.level_info(l)
        n, nnz, nc, nnzp, G = (int(info[0]), int(info[1]), int(info[2]), int(info[3]), int(info[7]))
        for prec in precisions:
            for op in ops:
                ms = h.time_level_op(l, op, prec, reps=reps)
                byts = op_bytes(op, prec, n, nnz, nc, nnzp)
                rows.append({"level": l + 1, "op": OPS[op], "prec": "fp64" if prec == 0 else "fp32",
                             "rows": n, "nnz": nnz, "nnzP": nnzp, "lanes": G, "us": round(ms * 1e3, 2),
                             "GBps": round(byts / (ms * 1e-3) / 1e9, 1),
                             "frac": round(byts / (ms * 1e-3) / 1e9 / peak, 3)})
    return rows


def run_kernel_only(args):
    import torch

    import draugr

    torch.cuda.set_device(0)
    A, b, cfg = workload(args.n, args.seed)
    h = draugr.amg_setup(A, cfg)
    if args.level < 0:
        reps = max(args.reps, 10)
        # the V(1,1) cycle from each level down (coarse tail included): the
        # differences between consecutive starts are each level's share
        cyc = [{"from_level": l + 1, "prec": "fp64" if prec == 0 else "fp32",
                "us": round(h.time_level_op(l, 8, prec, reps=reps) * 1e3, 2)}
               for prec in (0, 1) for l in range(1, h.nlevels)]
        return {"kernel_only": True, "levels": level_table(h, reps=reps), "cycles": cyc}
    ms = h.time_level_op(args.level, args.op, args.precision, reps=args.reps)
    info = h.level_info(args.level)
    return {"kernel_only": True, "level": args.level, "op": args.op, "precision": args.precision,
            "rows": int(info[0]), "nnz": int(info[1]), "ms_per_launch": ms}


def rap_bytes(h):
    """Algorithmic bytes of one partial resetup's numeric Galerkin products,
    summed over levels (each operand once, int32 indices): per level
    12 nnz_A + 4 (n+1) + 2 (12 nnz_P + 4 (n+1)) + 4 (n_c+1) + 12 nnz_Ac."""
    total = 0
    nl = h.nlevels
    for l in range(nl):
        info = h.level_info(l)
        n, nnz, nc, nnzp = int(info[0]), int(info[1]), int(info[2]), int(info[3])
        nnz_c = int(h.level_info(l + 1)[1]) if l + 1 < nl else int(h.level_info(-1)[1])
        total += 12 * nnz + 4 * (n + 1) + 2 * (12 * nnzp + 4 * (n + 1)) + 4 * (nc + 1) + 12 * nnz_c
    return total


def run_resetup(args):
    """27-point anisotropic diffusion (Q1, eps_z = 1e-3) on n^3 nodes with
    the headline configuration; coefficient updates kappa <- kappa *
    exp(0.5 N(0,1)) per element on the same pattern.  A few updated value
    arrays are prepared on the host and kept on the device; each timed step
    is one partial resetup from device-resident values (CUDA events on the
    hierarchy's stream)."""
    import torch

    import draugr
    from draugr import problems

    torch.cuda.set_device(0)
    m = args.n
    rng = np.random.default_rng(args.seed)
    kappa = np.ones((m + 1,) * 3)
    A = problems.anisotropic_27pt(m, 1e-3, kappa)
    cfg = draugr.hypre_default_config(agg_trunc_factor=0.2, smoother=draugr.L1JacobiSmootherType(),
                                      seed=args.seed)
    t0 = time.time()
    h = draugr.amg_setup(A, cfg)
    setup_s = time.time() - t0
    stream = torch.cuda.current_stream()
    h.set_stream(stream)
    n = A.shape[0]
    b = problems.rhs(n, args.seed + 1)
    bd = torch.tensor(b, device="cuda")
    xd = torch.zeros(n, dtype=torch.float64, device="cuda")
    draugr.pcg(xd, bd, h, cfg, tol=TOL, maxiter=MAXITER, precision="mixed")  # FP32 copies exist
    vals = []
    for _ in range(3):
        kappa = kappa * np.exp(0.5 * rng.standard_normal(kappa.shape))
        vals.append(torch.tensor(problems.anisotropic_27pt(m, 1e-3, kappa).data, device="cuda"))
    A_last = problems.anisotropic_27pt(m, 1e-3, kappa)
    def time_updates():
        for k in range(args.warmup):
            draugr.amg_resetup(h, vals[k % 3], cfg)
        ts = []
        for k in range(args.updates):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            draugr.amg_resetup(h, vals[(args.warmup + k) % 3], cfg)
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1) / 1e3)
        return ts

    h.set_resetup_precision(-1)
    times_fp64 = time_updates()
    # the configuration's precision split: FP64 Galerkin products on the top
    # two levels, FP32 below
    h.set_resetup_precision(2)
    times = time_updates()
    draugr.amg_resetup(h, vals[2], cfg)  # the solve below uses the last update
    res = {}
    for mode in ("fp64", "mixed"):
        xd.zero_()
        draugr.pcg(xd, bd, h, cfg, tol=TOL, maxiter=MAXITER, precision=mode)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        xd.zero_()
        e0.record(stream)
        _, it, _ = draugr.pcg(xd, bd, h, cfg, tol=TOL, maxiter=MAXITER, precision=mode)
        e1.record(stream)
        e1.synchronize()
        rr = float(np.linalg.norm(b - A_last @ xd.cpu().numpy()) / np.linalg.norm(b))
        res[mode] = {"time_s": e0.elapsed_time(e1) / 1e3, "iterations": int(it),
                     "relres_fp64_verified": rr}
    h.set_stream(None)
    byts = rap_bytes(h)
    t = float(np.mean(times))
    peak, peak_kind = peaks()
    nl = h.nlevels
    return {"workload": f"27-point Q1 anisotropic diffusion (eps_z=1e-3) {m}^3 nodes, "
                        "hypre_default_config(agg_trunc_factor=0.2) + l1-Jacobi; coefficient updates "
                        "kappa <- kappa*exp(0.5 N(0,1)) per element, partial resetup from device values",
            "metric": "partial resetup time (s)", "value": t, "unit": "s", "higher_is_better": False,
            "updates": args.updates, "warmup": args.warmup, "n": n, "nnz": int(A.nnz),
            "levels": nl + 1, "level_nnz": [int(h.level_info(l)[1]) for l in range(nl)],
            "setup_s_cpu": round(setup_s, 2), "resetup_s_min": float(np.min(times)),
            "precision": "Galerkin products of the top two levels in FP64, the rest in FP32",
            "resetup_s_all_fp64": float(np.mean(times_fp64)),
            "galerkin_algorithmic_bytes": byts,
            "galerkin_GBps_lower_bound": byts / t / 1e9,
            "note": "GB/s counts only the Galerkin products' bytes against the whole resetup time "
                    "(which also copies the values, recomputes every smoother diagonal, the coarsest "
                    "LU and the FP32 copies)",
            "peak_GBps": peak, "peak_source": peak_kind,
            "pcg_after_resetup": res}


def run_batch(args):
    """Batching workload: `systems` independent 3D 7-point constant-coefficient
    Poisson systems with sides ~ U{16..64} (seeded), each with its own
    hierarchy (hypre_default_config(agg_trunc_factor=0.2) + l1-Jacobi) and
    CUDA stream, mixed-precision PCG to 1e-8 from x0 = 0: solved one after
    another, then concurrently from `workers` host threads (solves/s, p50
    and p99 latency); and a 96^3 operator with 32 U(-1,1) right-hand sides
    solved back to back on one hierarchy."""
    import torch

    import draugr
    from draugr import problems

    torch.cuda.set_device(0)
    rng = np.random.default_rng(args.seed)
    cfg = draugr.hypre_default_config(agg_trunc_factor=0.2, smoother=draugr.L1JacobiSmootherType(),
                                      seed=args.seed)
    sides = rng.integers(16, 65, size=args.systems)
    mats = [problems.poisson3d(int(s)) for s in sides]
    t0 = time.time()
    hs = [draugr.amg_setup(A, cfg) for A in mats]
    setup_s = time.time() - t0
    bs = [torch.tensor(rng.uniform(-1, 1, A.shape[0]), device="cuda") for A in mats]
    xs = [torch.zeros_like(b) for b in bs]
    torch.cuda.synchronize()

    def run(workers):
        for x in xs:
            x.zero_()
        torch.cuda.synchronize()
        t = time.perf_counter()
        out = draugr.pcg_batch(hs, xs, bs, cfg, tol=TOL, maxiter=MAXITER, precision="mixed", workers=workers)
        torch.cuda.synchronize()
        return time.perf_counter() - t, out

    for _ in range(args.warmup):
        run(args.workers)
    seq_wall, seq = run(1)
    walls, lat = [], []
    for _ in range(args.steps):
        w, out = run(args.workers)
        walls.append(w)
        lat += [o[2] for o in out]
    worst = 0.0
    for A, b, x in zip(mats, bs, xs):
        bn = b.cpu().numpy()
        worst = max(worst, float(np.linalg.norm(bn - A @ x.cpu().numpy()) / np.linalg.norm(bn)))
    # the same systems merged into one batch: one launch per cycle stage for all
    t0 = time.time()
    batch = draugr.batch_setup(hs, cfg)
    merge_s = time.time() - t0
    bcat = torch.cat(bs)
    xcat = torch.zeros_like(bcat)
    for _ in range(args.warmup):
        xcat.zero_()
        draugr.pcg_batched(xcat, bcat, batch, cfg, tol=TOL, maxiter=MAXITER, precision="mixed")
    seg_t, seg_lat = [], []
    for _ in range(args.steps):
        xcat.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        _, sits, srel = draugr.pcg_batched(xcat, bcat, batch, cfg, tol=TOL, maxiter=MAXITER, precision="mixed")
        e1.record()
        e1.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        seg_t.append(t)
        # a system's latency: the iterations it needed at the batch's time per iteration
        seg_lat += [t * int(k) / max(1, int(sits.max())) for k in sits]
    xh = xcat.cpu().numpy()
    seg_worst = 0.0
    for k, (A, b) in enumerate(zip(mats, bs)):
        lo, hi = int(batch.offsets[k]), int(batch.offsets[k + 1])
        bn = b.cpu().numpy()
        seg_worst = max(seg_worst, float(np.linalg.norm(bn - A @ xh[lo:hi]) / np.linalg.norm(bn)))
    segmented = {"path": "draugr_b200_batch_pcg_device (hierarchies merged level by level; one launch per "
                         "cycle stage, dot product and update for all systems; one iteration per CUDA graph)",
                 "solves_per_s": args.systems / float(np.mean(seg_t)), "ms_per_batch": 1e3 * float(np.mean(seg_t)),
                 "latency_s": {"p50": float(np.percentile(seg_lat, 50)), "p99": float(np.percentile(seg_lat, 99))},
                 "iterations": [int(sits.min()), int(sits.max())], "worst_relres_fp64_verified": seg_worst,
                 "merge_s_cpu": round(merge_s, 2),
                 "timing": "CUDA events around each batched solve (device-resident vectors)"}
    batch.free()
    # one operator, many right-hand sides
    A96 = problems.poisson3d(96)
    h96 = draugr.amg_setup(A96, cfg)
    B = [torch.tensor(rng.uniform(-1, 1, A96.shape[0]), device="cuda") for _ in range(32)]
    X = torch.zeros(A96.shape[0], dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        X.zero_()
        torch.cuda.synchronize()
        draugr.pcg(X, B[0], h96, cfg, tol=TOL, maxiter=MAXITER, precision="mixed")
    t = time.perf_counter()
    its = []
    for b in B:
        X.zero_()
        torch.cuda.synchronize()
        _, it, _ = draugr.pcg(X, b, h96, cfg, tol=TOL, maxiter=MAXITER, precision="mixed")
        its.append(it)
    torch.cuda.synchronize()
    rhs_wall = time.perf_counter() - t
    # the same 32 right-hand sides as one block solve
    Bm = torch.stack(B, dim=1).contiguous()
    Xm = torch.zeros_like(Bm)
    for _ in range(args.warmup):
        Xm.zero_()
        torch.cuda.synchronize()
        draugr.pcg_multi(Xm, Bm, h96, cfg, tol=TOL, maxiter=MAXITER, precision="mixed")
    blk = []
    for _ in range(args.steps):
        Xm.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        _, bits, brel = draugr.pcg_multi(Xm, Bm, h96, cfg, tol=TOL, maxiter=MAXITER, precision="mixed")
        e1.record()
        e1.synchronize()
        blk.append(e0.elapsed_time(e1) / 1e3)
    Xh = Xm.cpu().numpy()
    Bh = Bm.cpu().numpy()
    blk_rr = max(float(np.linalg.norm(Bh[:, c] - A96 @ Xh[:, c]) / np.linalg.norm(Bh[:, c])) for c in range(32))
    n_tot = int(sum(A.shape[0] for A in mats))
    return {"workload": f"{args.systems} independent 3D 7-point Poisson systems, sides U{{16..64}} "
                        f"({n_tot} unknowns in all), hypre_default_config(agg_trunc_factor=0.2) + "
                        "l1-Jacobi, mixed-precision PCG to 1e-8; one hierarchy and stream per system",
            "metric": "solves/s", "value": args.systems / float(np.mean(walls)), "unit": "solves/s",
            "higher_is_better": True, "workers": args.workers, "steps": args.steps, "warmup": args.warmup,
            "sequential_solves_per_s": args.systems / seq_wall,
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "worst_relres_fp64_verified": worst, "setup_s_cpu": round(setup_s, 2),
            "segmented": segmented,
            "timing": "host wall clock around each batch (device synchronised on both sides); "
                      "latency = each solve's call from a pool thread",
            "multi_rhs": {"workload": "3D 7-point Poisson 96^3, 32 right-hand sides, mixed PCG to 1e-8, "
                                      "solved back to back on one hierarchy",
                          "solves_per_s": 32 / rhs_wall, "ms_per_solve": 1e3 * rhs_wall / 32,
                          "iterations": [int(min(its)), int(max(its))],
                          "block": {"path": "draugr_b200_pcg_block_device (32 columns, one pass over each "
                                            "level matrix per block product)",
                                    "solves_per_s": 32 / float(np.mean(blk)),
                                    "ms_per_block": 1e3 * float(np.mean(blk)),
                                    "iterations": [int(min(bits)), int(max(bits))],
                                    "worst_relres_fp64_verified": blk_rr}}}


def run_profile_block(args):
    import torch

    import draugr
    from draugr import problems

    torch.cuda.set_device(0)
    A = problems.poisson3d(96)
    cfg = draugr.hypre_default_config(agg_trunc_factor=0.2, smoother=draugr.L1JacobiSmootherType(),
                                      seed=args.seed)
    h = draugr.amg_setup(A, cfg)
    B = torch.tensor(np.random.default_rng(args.seed).uniform(-1, 1, (A.shape[0], 32)), device="cuda")
    X = torch.zeros_like(B)
    torch.cuda.synchronize()
    _, its, rel = draugr.pcg_multi(X, B, h, cfg, tol=TOL, maxiter=MAXITER, precision="mixed")
    return {"profile_block": True, "iterations": [int(min(its)), int(max(its))], "relres_max": max(rel)}


def run_profile_resetup(args):
    import torch

    import draugr
    from draugr import problems

    torch.cuda.set_device(0)
    m = args.n
    rng = np.random.default_rng(args.seed)
    kappa = np.ones((m + 1,) * 3)
    A = problems.anisotropic_27pt(m, 1e-3, kappa)
    cfg = draugr.hypre_default_config(agg_trunc_factor=0.2, smoother=draugr.L1JacobiSmootherType(),
                                      seed=args.seed)
    h = draugr.amg_setup(A, cfg)
    kappa = kappa * np.exp(0.5 * rng.standard_normal(kappa.shape))
    v = torch.tensor(problems.anisotropic_27pt(m, 1e-3, kappa).data, device="cuda")
    torch.cuda.synchronize()
    for _ in range(2):  # the first also records the Galerkin product lists
        draugr.amg_resetup(h, v, cfg)
    torch.cuda.synchronize()
    return {"profile_resetup": True, "n": int(A.shape[0]), "nnz": int(A.nnz), "levels": h.nlevels + 1}


def run_profile_batch(args):
    import torch

    import draugr
    from draugr import problems

    torch.cuda.set_device(0)
    rng = np.random.default_rng(args.seed)
    cfg = draugr.hypre_default_config(agg_trunc_factor=0.2, smoother=draugr.L1JacobiSmootherType(),
                                      seed=args.seed)
    sides = rng.integers(16, 65, size=args.systems)
    mats = [problems.poisson3d(int(s)) for s in sides]
    hs = [draugr.amg_setup(A, cfg) for A in mats]
    batch = draugr.batch_setup(hs, cfg)
    b = torch.tensor(np.concatenate([rng.uniform(-1, 1, A.shape[0]) for A in mats]), device="cuda")
    x = torch.zeros_like(b)
    torch.cuda.synchronize()
    _, its, rel = draugr.pcg_batched(x, b, batch, cfg, tol=TOL, maxiter=MAXITER, precision="mixed")
    return {"profile_batch": True, "systems": int(args.systems), "rows": int(b.numel()),
            "iterations": [int(its.min()), int(its.max())], "relres_max": float(rel.max())}


def run_profile_solve(args):
    import torch

    import draugr

    torch.cuda.set_device(0)
    A, b, cfg = workload(args.n, args.seed)
    h = draugr.amg_setup(A, cfg)
    x = np.zeros(A.shape[0])
    _, it, rel = draugr.pcg(x, b, h, cfg, tol=TOL, maxiter=MAXITER, precision=args.profile_solve)
    return {"profile_solve": args.profile_solve, "iterations": it, "relres": rel,
            "relres_fp64_verified": float(np.linalg.norm(b - A @ x) / np.linalg.norm(b))}


def main():
    args = parse()
    if args.resetup:
        print(json.dumps(run_resetup(args)), flush=True)
        return
    if args.batch:
        print(json.dumps(run_batch(args)), flush=True)
        return
    if args.profile_block:
        print(json.dumps(run_profile_block(args)), flush=True)
        return
    if args.profile_resetup:
        print(json.dumps(run_profile_resetup(args)), flush=True)
        return
    if args.profile_solve:
        print(json.dumps(run_profile_solve(args)), flush=True)
        return
    if args.profile_batch:
        print(json.dumps(run_profile_batch(args)), flush=True)
        return
    if args.kernel_only:
        print(json.dumps(run_kernel_only(args)), flush=True)
        return
    if args.write_structure:
        write_structure(args)
        return
    world, rank, local = dist_init(args)
    if args.impl == "reference":
        out = run_reference(args, world, rank)
    else:
        out = run_ours(args, world, rank, local)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
