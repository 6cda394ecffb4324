"""Throughput of the SIMP loop on B200: SIMP iterations/s and DOF*CG-iterations/s.

Workload (default, one GPU): the 128x64x64 cantilever with a protected-void
cylinder (radius 12, axis y, centre x=64, z=32), a protected-solid slab
x in [0, 4), volfrac 0.3, penal 3, rmin 3, beta 1, eta 0.5, move 0.2,
unit-cube elements, total unit -z load on the x=nelx, z=0 edge.  A "step" is
one iteration of the loop body: multigrid-PCG solve, sensitivities, OC
bisection, re-projection.  Synthetic inputs, no dataset.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision mixed|fp64]
    python bench.py --impl reference ...   # the reference algorithm on the host cores

Under torchrun every rank runs an independent replica (the path has no data
exchange); ``value`` is the whole-job rate (sum over ranks at the max-over-ranks
time).
"""

from __future__ import annotations

import argparse
import contextlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NELX, NELY, NELZ = 128, 64, 64
VOLFRAC, PENAL, RMIN, BETA, ETA, MOVE = 0.3, 3.0, 3.0, 1.0, 0.5, 0.2


def workload(nelx=NELX, nely=NELY, nelz=NELZ):
    """Masks and loads of the 128x64x64 configuration (scaled for other sizes)."""
    from pytopo3d_b200.assembly import build_force_vector, build_supports

    shape = (nely, nelx, nelz)
    yy, xx, zz = np.ogrid[:nely, :nelx, :nelz]
    r = 12 * nelx // 128
    void = np.broadcast_to((xx - nelx // 2) ** 2 + (zz - nelz // 2) ** 2 <= r * r, shape).copy()
    solid = np.zeros(shape, bool)
    solid[:, : max(1, 4 * nelx // 128), :] = True
    solid[:, -1, 0] = True  # load strip (optimizer.py:366-369)
    solid[:, 0, :] = True  # support face (optimizer.py:378-390)
    solid &= ~void
    ndof = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
    F = build_force_vector(nelx, nely, nelz, ndof) / (nely + 1)  # total unit load
    free, _ = build_supports(nelx, nely, nelz, ndof)
    fixed = np.ones(ndof, np.uint8)
    fixed[free] = 0
    return shape, solid, void, F, fixed


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region.

    The sampler is started before the warm-up (nvidia-smi takes a moment to
    start); ``timed()`` brackets the timed region and only samples taken inside
    it (or, for a region shorter than the sampling interval, the one nearest to
    it) enter the summary."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self.proc = None
        self.window = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.perf_counter(), [c.strip() for c in line.split(",")]))

    @contextlib.contextmanager
    def timed(self):
        t0 = time.perf_counter()
        yield
        self.window = (t0, time.perf_counter())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = list(self.rows)
        if self.window and rows:
            t0, t1 = self.window
            inside = [r for t, r in rows if t0 <= t <= t1 + 0.05]
            rows = inside or [min(rows, key=lambda tr: abs(tr[0] - 0.5 * (t0 + t1)))[1]]
        else:
            rows = [r for _, r in rows]
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) >= 9:
                for n, v in zip(names, r[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_loop(precision, x0=None, solver_options=None, dims=None, volfrac=VOLFRAC, rmin=RMIN, masks=True):
    """The cantilever loop at `dims` (default: the 128x64x64 workload).  masks=False:
    the plain cantilever (default load strip and support face only, no cylinder or
    slab), the configuration the reference's own CPU path runs at 32x16x16."""
    from pytopo3d_b200.optimizer import SimpLoop
    from pytopo3d_b200.stiffness import lk_H8

    nelx, nely, nelz = dims or (NELX, NELY, NELZ)
    shape, solid, void, F, fixed = workload(nelx, nely, nelz) if masks else plain_cantilever(nelx, nely, nelz)
    loop = SimpLoop(nelx, nely, nelz, volfrac, PENAL, rmin, lk_H8(elem_size=1.0), F, fixed, solid, void,
                    projection_eta=ETA, move=MOVE, precision=precision, x0=x0, solver_options=solver_options)
    loop.set_beta(BETA)
    return loop


def plain_cantilever(nelx, nely, nelz):
    """The reference's default cantilever: load strip and support face protected
    (optimizer.py:366-390), no obstacles, total unit -z load on the x = nelx, z = 0 edge."""
    from pytopo3d_b200.assembly import build_force_vector, build_supports

    shape = (nely, nelx, nelz)
    solid = np.zeros(shape, bool)
    solid[:, -1, 0] = True
    solid[:, 0, :] = True
    void = np.zeros(shape, bool)
    ndof = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
    F = build_force_vector(nelx, nely, nelz, ndof) / (nely + 1)
    free, _ = build_supports(nelx, nely, nelz, ndof)
    fixed = np.ones(ndof, np.uint8)
    fixed[free] = 0
    return shape, solid, void, F, fixed


def e2e_rate_of(loop_factory, warm, steps, dist, world):
    """SIMP it/s through SimpLoop.step_host (pinned H2D of the design, D2H of the
    new design and the compliance every step), wall clock around `steps` steps
    after `warm` steps, max over ranks."""
    import torch

    loop = loop_factory()
    x_host = loop.design().permute(2, 1, 0).contiguous().reshape(-1).cpu().numpy()
    for _ in range(warm):
        x_host, _ = loop.step_host(x_host)
    barrier(dist)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        x_host, _ = loop.step_host(x_host)
    torch.cuda.synchronize()
    dt = max_over_ranks(time.perf_counter() - t0, dist)
    loop.close()
    return job_rate(steps, dt, world)


def time_device_steps(loop, steps, dist):
    import torch

    L = __import__("pytopo3d_b200._lib", fromlist=["lib"]).lib()
    cg = 0
    barrier(dist)
    torch.cuda.synchronize()
    n0 = L.tp3d_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    cs = []
    for _ in range(steps):
        st = loop.step()
        cg += loop.last["cg_iterations"]
        cs.append(st[:1])
    e1.record()
    torch.cuda.synchronize()
    barrier(dist)
    ms = e0.elapsed_time(e1)
    launches = L.tp3d_launch_count() - n0
    c = float(cs[-1].item())
    return ms, cg, launches, c


def accuracy_vs_fp64(loop, precision):
    """Relative compliance (u'Ku) and displacement errors of one solve of the
    loop's own solver on its current design and warm start, against an FP64
    solve of the same system to relative residual 1e-12 (or its floor)."""
    from pytopo3d_b200.solver import HexSolver
    from pytopo3d_b200.stiffness import lk_H8

    S = loop.S
    rho, F, U0 = S.rho_p.clone(), S.F[0], S.U[0].clone()
    fixed = workload(NELX, NELY, NELZ)[4]
    ref = HexSolver(NELX, NELY, NELZ, lk_H8(elem_size=1.0), fixed, precision="fp64", rtol=1e-12,
                    max_iterations=10000)
    ref.set_density(rho, PENAL)
    Ur = ref.solve(F, U0.clone(), raise_on_fail=False)
    loop.solver.set_density(rho, PENAL)
    Um = loop.solver.solve(F, U0.clone())
    c_r = float(Ur @ ref.apply(Ur))
    c_m = float(Um @ ref.apply(Um))
    out = {"precision": precision, "rtol": loop.solver.opts.rtol, "iterations": loop.solver.last_iterations,
           "compliance_rel_err": abs(c_m - c_r) / abs(c_r),
           "displacement_rel_err": float((Um - Ur).norm() / Ur.norm()),
           "reference": {"precision": "fp64", "rtol": 1e-12, "relres": ref.last_relres,
                         "iterations": ref.last_iterations}}
    ref.close()
    return out


def barrier(dist):
    if dist is not None:
        dist.barrier()


def max_over_ranks(v, dist):
    """Largest value over the ranks (the job's time is its slowest replica's)."""
    if dist is None:
        return v
    import torch

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, seconds, world):
    """Whole-job throughput of `world` independent replicas at the max-over-ranks time."""
    return world * units_per_rank / seconds


def cpu_reference_sample(steps=1):
    """The reference algorithm (oracle restatement: COO/CSR assembly, SuperLU spsolve,
    element energy, chain rule, OC bisection) timed on the host cores.  The
    128x64x64 direct solve does not fit (SuperLU fill on 1.6 M DOF), so the
    sample is the same loop body at 32x16x16, where the reference runs."""
    from oracle import simp_oracle as O

    nelx, nely, nelz = 32, 16, 16
    shape = (nely, nelx, nelz)
    solid, void, free = O.prepare_masks(nelx, nely, nelz)
    ndof = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
    F = O.build_force_vector(nelx, nely, nelz, ndof) / (nely + 1)
    freedofs, _ = O.build_supports(nelx, nely, nelz, ndof)
    KE = O.lk_H8(elem_size=1.0)
    H, Hs = O.build_filter(nelx, nely, nelz, RMIN)
    x = np.full(shape, VOLFRAC)
    x[solid], x[void] = 1.0, 0.0
    target = VOLFRAC * int(free.sum())
    t0 = time.perf_counter()
    for _ in range(steps):
        _, rho, dp = O.build_physical_density(x, H, Hs, BETA, ETA, solid, void)
        it = O.simp_iteration(x, rho, dp, BETA, ETA, PENAL, MOVE, target, H, Hs, KE, F, freedofs, solid, void,
                              free, nelx, nely, nelz)
        x = it["x_new"]
    dt = time.perf_counter() - t0
    return steps / dt, dt


def run_reference(args, rank):
    if rank != 0:
        return 0
    steps = max(1, args.steps)
    warm = max(3, args.warmup)  # the same warm-up rule as the B200 arm
    cpu_reference_sample(warm)
    rate, dt = cpu_reference_sample(steps)
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    line = {
        "impl": "reference", "metric": "SIMP iterations/s", "value": rate, "unit": "iter/s", "n_gpus": 0,
        "steps": steps, "warmup": warm, "ms_per_step": 1e3 * dt / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "cantilever 32x16x16 (reference CPU path: SuperLU spsolve); the 128x64x64 "
                               "workload does not fit the reference's direct solve; the B200 line's "
                               "same_config_as_reference object times this same workload", "beta": BETA,
                   "rmin": RMIN, "volfrac": VOLFRAC},
        "cpu_baseline": {"value": rate, "unit": "iter/s", "cores": 1, "kind": "port",
                         "sample": f"{steps} loop bodies of the oracle restatement at 32x16x16 "
                                   f"(single-threaded SuperLU), {cores} cores visible"},
        "e2e": {"value": rate, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-large", action="store_true", help="skip the 256x128x128 design")
    ap.add_argument("--mode", default="bench", choices=["bench", "step", "apply", "batch", "large"],
                    help="step: warm-up + --steps loop bodies only (for launch lists); "
                         "apply: fine-operator launches only (for kernel captures)")
    ap.add_argument("--size", type=int, default=NELX, help="nelx for --mode step/apply (nely = nelz = nelx/2)")
    ap.add_argument("--fine-operator", type=int, default=0,
                    help="solver option fine_operator for --mode step/apply (0 timed choice)")
    ap.add_argument("--solver-opt", action="append", default=[], metavar="KEY=VALUE",
                    help="further solver options for --mode step/apply/batch (integers or floats)")
    args = ap.parse_args()
    if args.mode == "batch":
        return run_batch(args)
    if args.mode == "large":
        return run_large(args)
    if args.mode != "bench":
        return run_probe(args)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        return run_reference(args, rank)

    import torch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = dist_mod

    from pytopo3d_b200 import _lib

    L = _lib.lib()
    W = max(3, args.warmup)
    results = {}
    for prec in ([args.precision] + [p for p in ("fp64", "mixed") if p != args.precision]):
        # both precisions: the same warm-up, the same number of timed steps
        loop = make_loop(prec)
        with ClockSampler(local) as clk:
            for _ in range(W):
                loop.step()
            torch.cuda.synchronize()
            with clk.timed():
                ms, cg, launches, c = time_device_steps(loop, args.steps, dist)
        if prec == args.precision:
            clocks = clk.summary()
        steps = args.steps
        ms = max_over_ranks(ms, dist)
        apply_ms = (ctypes_time_apply(loop.solver, fp32=(prec == "mixed")))
        results[prec] = dict(ms=ms, steps=steps, cg=cg, launches=launches, c=c, apply_ms=apply_ms,
                             loop=loop, stats=loop.solver.stats(), clocks=clk.summary())
        results[prec]["accuracy"] = accuracy_vs_fp64(loop, prec)
        if prec != args.precision:
            loop.close()

    # the autotuner: the same loop with the smoothing degrees searched on this
    # grid at its first solve (the fine operator's shape and slab depth are
    # searched at the first set_density either way), same warm-up and steps
    tl = make_loop(args.precision, solver_options={"autotune": True})
    for _ in range(W):
        tl.step()
    torch.cuda.synchronize()
    tms, tcg, _, _ = time_device_steps(tl, args.steps, dist)
    tms = max_over_ranks(tms, dist)
    autotune = {"value": job_rate(args.steps, tms / 1e3, world), "unit": "iter/s",
                "ms_per_step": tms / args.steps, "cg_iterations_per_step": tcg / args.steps,
                "search": tl.solver.tuning,
                "chosen": {k: v for k, v in tl.solver.stats().items()
                           if k in ("degree_fine", "degree_level1", "degree_level2", "fine_slab_depth",
                                    "fine_threads", "tile_y", "tile_x")}}
    tl.close()

    main_r = results[args.precision]
    loop = main_r["loop"]
    ndof = 3 * (NELX + 1) * (NELY + 1) * (NELZ + 1)
    nele = NELX * NELY * NELZ
    steps = main_r["steps"]
    rate = job_rate(steps, main_r["ms"] / 1e3, world)

    # end-to-end through the public API with host buffers (pinned H2D of x, D2H of x_new + c):
    # a fresh loop from the same start, the same warm-up and the same number of
    # steps as the device-timed run, so both follow the same trajectory
    e2e_rate = e2e_rate_of(lambda: make_loop(args.precision), W, steps, dist, world)

    # the reference's own CPU workload (the plain 32x16x16 cantilever, which its
    # direct solve can run) on the B200, both precisions, same warm-up and steps:
    # the like-for-like partner of the --impl reference line
    same = {"workload": "cantilever 32x16x16, no obstacles, beta 1 (the --impl reference workload)"}
    for prec in ("fp64", "mixed"):
        mk = lambda: make_loop(prec, dims=(32, 16, 16), masks=False)
        sl = mk()
        for _ in range(W):
            sl.step()
        torch.cuda.synchronize()
        sms, scg, _, _ = time_device_steps(sl, args.steps, dist)
        sl.close()
        same[prec] = {"value": job_rate(args.steps, max_over_ranks(sms, dist) / 1e3, world), "unit": "iter/s",
                      "cg_iterations_per_step": scg / args.steps,
                      "e2e": e2e_rate_of(mk, W, args.steps, dist, world)}

    # roofline of the dominant kernel (fine-level operator apply)
    peak, peak_kind = peaks()
    fp32 = args.precision == "mixed"
    # u read + y write per DOF, one modulus read per element (FP32 moduli in the
    # mixed form unless the solver runs on BF16 densities)
    bf16 = bool(getattr(loop.solver.opts, "inner_density", 0))
    alg_bytes = (8 * ndof + (2 if bf16 else 4) * nele) if fp32 else (16 * ndof + 8 * nele)
    achieved = alg_bytes / (main_r["apply_ms"] * 1e-3) / 1e9
    nnode = (NELX + 1) * (NELY + 1) * (NELZ + 1)
    form = main_r["stats"].get("fine_form_fp32" if fp32 else "fine_form_fp64", 0)
    # fine_form is 1 + the Walsh-Hadamard shape (0 the dense form); FP32 shapes
    # 6 and 7 run Apply in the one-barrier kernel
    kname = ("wht1_apply" if fp32 and form >= 7 else "wht_apply") if form and form >= 1 else "fine_apply"
    # floating-point operations the kernel executes per node (FMA = 2): the
    # Walsh-Hadamard block form does 99 FMAs and 81 adds per node and plane; the
    # dense-KE form the dense 576 FMAs per element
    flops_node = 1152.0 if kname == "fine_apply" else 279.0
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf):
        try:
            traffic = json.load(open(tf)).get(kname + ("_f32" if fp32 else "_f64"))
        except Exception:
            traffic = None
    # the largest coarse-level kernel (level 1, packed stencil), cold L2
    c_ms, c_bytes = loop.solver.time_level(1, fp32, 10)
    c_gbs = c_bytes / (c_ms * 1e-3) / 1e9
    # step level: the CG loop's algorithmic bytes (summed over the kernels of one
    # captured iteration) times the iterations per step, over the whole step time
    bpi = main_r["stats"].get("bytes_per_cg_iteration", 0.0)
    step_gbs = bpi * (main_r["cg"] / steps) / (main_r["ms"] / steps * 1e-3) / 1e9

    # the large single design (256x128x128, volfrac 0.2, rmin 4.5, beta 1, mixed):
    # a short device-timed run of the same loop body
    large = None
    if not args.no_large:
        ll = make_loop("mixed", dims=(256, 128, 128), volfrac=0.2, rmin=4.5)
        for _ in range(W):
            ll.step()
        torch.cuda.synchronize()
        lsteps = max(3, args.steps // 2)
        lms, lcg, _, _ = time_device_steps(ll, lsteps, dist)
        lms = max_over_ranks(lms, dist)
        l_ndof = 3 * 257 * 129 * 129
        l_apply = ctypes_time_apply(ll.solver, fp32=True)
        l_bytes = 8 * l_ndof + 4 * 256 * 128 * 128
        large = {"workload": "cantilever 256x128x128, volfrac 0.2, rmin 4.5, beta 1, mixed", "steps": lsteps,
                 "warmup": W, "value": job_rate(lsteps, lms / 1e3, world), "unit": "iter/s",
                 "dof_cg_iters_per_s": world * l_ndof * lcg / (lms / 1e3), "cg_iterations_per_step": lcg / lsteps,
                 "fine_operator": {"launch_ms": l_apply, "bytes_per_launch": l_bytes,
                                   "achieved": l_bytes / (l_apply * 1e-3) / 1e9, "frac": l_bytes / (l_apply * 1e-3) / 1e9 / peak}}
        ll.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        crate, cdt = cpu_reference_sample(1)
        cpu = {"value": crate, "unit": "iter/s", "cores": 1, "kind": "port",
               "sample": "1 loop body of the oracle restatement at 32x16x16 (SuperLU spsolve, single "
                         "thread); the 128x64x64 direct solve does not fit the reference's CPU path"}

    other = [p for p in results if p != args.precision]
    line = {
        "metric": "SIMP iterations/s", "value": rate, "unit": "iter/s", "n_gpus": world, "steps": steps,
        "warmup": W, "ms_per_step": main_r["ms"] / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+bf16 inner / f64 refinement" if fp32 else "f64",
        "data": "synthetic",
        "config": {"workload": "cantilever 128x64x64, void cylinder r12 (axis y), solid slab x<4, beta 1",
                   "nele": nele, "ndof": ndof, "precision": args.precision, "rmin": RMIN,
                   "volfrac": VOLFRAC, "l2": "SIMP step working set (multigrid hierarchy + vectors) > 126 MB L2; roofline kernel timed back to back over rotating input vectors totalling > 256 MiB",
                   "parallelism": f"replicas x{world}"},
        "dof_cg_iters_per_s": world * ndof * main_r["cg"] / (main_r["ms"] / 1e3),
        "cg_iterations_per_step": main_r["cg"] / steps,
        "compliance": main_r["c"],
        "solver": {k: v for k, v in main_r["stats"].items()},
        "accuracy_vs_fp64": main_r["accuracy"],
        "other_precision": {p: {"value": world * results[p]["steps"] / (results[p]["ms"] / 1e3),
                                "ms_per_step": results[p]["ms"] / results[p]["steps"],
                                "cg_iterations_per_step": results[p]["cg"] / results[p]["steps"],
                                "apply_ms": results[p]["apply_ms"], "accuracy_vs_fp64": results[p]["accuracy"],
                                "steps": results[p]["steps"], "warmup": W,
                                "bytes_per_cg_iteration": results[p]["stats"].get("bytes_per_cg_iteration"),
                                "kernels_per_cg_iteration": results[p]["stats"].get("kernels_per_cg_iteration"),
                                "clocks": results[p]["clocks"]}
                            for p in other},
        "e2e": {"value": e2e_rate, "unit": "iter/s", "h2d_bytes_per_step": 8 * nele,
                "d2h_bytes_per_step": 8 * nele + 8},
        "same_config_as_reference": same,
        "roofline": {"bound": "hbm", "kernel": kname + "_kernel<" + ("float" if fp32 else "double") + ">",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "traffic": traffic, "bytes_per_launch": alg_bytes,
                     "launch_ms": main_r["apply_ms"],
                     "executed_flops_per_node": flops_node,
                     "executed_tflops": flops_node * nnode / (main_r["apply_ms"] * 1e-3) / 1e12},
        "roofline_coarse": {"bound": "hbm", "kernel": ("nm3_apply_kernel (level 1, node-major bf16 stencil, cold L2)"
                                                      if fp32 and getattr(loop.solver.opts, "coarse_node_major", 0)
                                                      else "stencil_apply_kernel (level 1, packed "
                                                      + ("bf16" if fp32 else "fp64") + " stencil, cold L2)"),
                            "achieved": c_gbs, "peak": peak, "unit": "GB/s", "frac": c_gbs / peak,
                            "bytes_per_launch": c_bytes, "launch_ms": c_ms},
        "roofline_step": {"bound": "hbm", "what": "algorithmic bytes of the CG loop's kernels per step / step time",
                          "bytes_per_cg_iteration": bpi,
                          "kernels_per_cg_iteration": main_r["stats"].get("kernels_per_cg_iteration"),
                          "achieved": step_gbs, "peak": peak, "unit": "GB/s", "frac": step_gbs / peak},
        "large_design": large,
        "autotune": autotune,
        "cpu_baseline": cpu,
        "gpu_launches": main_r["launches"],
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    loop.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def run_batch(args):
    """The batched workload: 64 seeded cantilevers of uneven sizes, each an
    independent loop on its own stream, 8 host threads; --steps loop bodies per
    design after --warmup.  The same designs one after another on the default
    stream are timed beside it.  Prints one JSON line (not the headline bench
    line)."""
    # the designs' streams run side by side only over as many hardware queues as
    # the context has (CUDA_DEVICE_MAX_CONNECTIONS, 8 by default): 32 measured
    # 174 SIMP it/s against 144-150 for the stream runner (the graph runner is
    # unaffected); read when the context is created, so set before any CUDA call
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    import torch

    from pytopo3d_b200.batch import BatchRunner, batched_cantilevers

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    specs = batched_cantilevers(64, seed=0)
    opts = solver_opts_of(args)
    tuned = {}
    for crit in ("bytes", "time"):
        t0 = time.perf_counter()
        br = BatchRunner(specs, precision=args.precision, workers=8, tune=crit, solver_options=opts)
        setup_s = time.perf_counter() - t0
        br.run(max(1, args.warmup))
        r = br.run(args.steps)
        r["autotune_setup_s"] = setup_s
        r["degrees"] = [(t["degree_fine"], t["degree_level1"], t["degree_deep"]) for t in br.tuning]
        tuned[crit] = r
        br.close()
    # the same position on each design's trajectory as the tuned runs (three
    # loop bodies of tuning plus the warm-up)
    br = BatchRunner(specs, precision=args.precision, workers=8, tune=None, solver_options=opts)
    br.run(3 + max(1, args.warmup))
    conc_default = br.run(args.steps)
    br.close()
    # every design advanced by one graph launch per call (no host thread per design)
    br = BatchRunner(specs, precision=args.precision, workers=8, tune="bytes", solver_options=opts)
    br.run_graph(max(1, args.warmup))
    graph_tuned = br.run_graph(args.steps)
    br.close()
    seq = BatchRunner(specs, precision=args.precision, workers=1, tune=None, solver_options=opts)
    seq.run(3 + max(1, args.warmup))
    one = seq.run(args.steps)
    seq.close()
    nele = [s.nelx * s.nely * s.nelz for s in specs]
    print(json.dumps({"mode": "batch", "designs": len(specs), "precision": args.precision, "steps": args.steps,
                      "elements_total": int(sum(nele)), "elements_min": int(min(nele)),
                      "elements_max": int(max(nele)),
                      "concurrent_8_threads_autotuned_bytes": tuned["bytes"],
                      "concurrent_8_threads_autotuned_time": tuned["time"],
                      "concurrent_8_threads_default_degrees": conc_default,
                      "one_graph_launch_autotuned_bytes": graph_tuned,
                      "speedup_graph_over_threads": graph_tuned["simp_iterations_per_s"]
                      / tuned["bytes"]["simp_iterations_per_s"],
                      "one_after_another_default_degrees": one,
                      "speedup_concurrent": conc_default["simp_iterations_per_s"] / one["simp_iterations_per_s"],
                      "speedup_autotune_bytes": tuned["bytes"]["simp_iterations_per_s"]
                      / conc_default["simp_iterations_per_s"],
                      "speedup_autotune_time": tuned["time"]["simp_iterations_per_s"]
                      / conc_default["simp_iterations_per_s"]}))
    return 0


def run_large(args):
    """The large single design in full: 256x128x128 (4.19 M elements, 12.8 M
    DOFs), volfrac 0.2, rmin 4.5, penal 3, beta 1, 2, 4, 8 with --steps loop
    bodies per stage (default schedule: 100), mixed precision.  Each stage is
    timed on the device with CUDA events; the compliance of the final design is
    checked against an FP64 solve.  Prints one JSON line (not the headline bench
    line)."""
    import torch

    from pytopo3d_b200.solver import HexSolver
    from pytopo3d_b200.stiffness import lk_H8

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dims = (256, 128, 128)
    ndof = 3 * 257 * 129 * 129
    per_stage = args.steps
    loop = make_loop("mixed", dims=dims, volfrac=0.2, rmin=4.5)
    stages = []
    total_ms, total_cg = 0.0, 0
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        with clk.timed():
            for beta in (1.0, 2.0, 4.0, 8.0):
                loop.set_beta(beta)
                torch.cuda.synchronize()
                ms, cg, launches, c = time_device_steps(loop, per_stage, None)
                total_ms += ms
                total_cg += cg
                stages.append({"beta": beta, "iterations": per_stage, "ms": ms, "simp_iterations_per_s":
                               per_stage / (ms / 1e3), "cg_iterations_per_step": cg / per_stage, "compliance": c,
                               "kernel_launches": launches})
    # the final design: one mixed solve against an FP64 solve to 1e-12
    S = loop.S
    fixed = workload(*dims)[4]
    ref = HexSolver(*dims, lk_H8(elem_size=1.0), fixed, precision="fp64", rtol=1e-12, max_iterations=20000)
    ref.set_density(S.rho_p, PENAL)
    Ur = ref.solve(S.F[0], S.U[0].clone(), raise_on_fail=False)
    loop.solver.set_density(S.rho_p, PENAL)
    Um = loop.solver.solve(S.F[0], S.U[0].clone())
    c_r, c_m = float(Ur @ ref.apply(Ur)), float(Um @ ref.apply(Um))
    apply_ms = ctypes_time_apply(loop.solver, fp32=True)
    peak, peak_kind = peaks()
    fbytes = 8 * ndof + 4 * dims[0] * dims[1] * dims[2]
    n_it = 4 * per_stage
    print(json.dumps({
        "mode": "large", "workload": "cantilever 256x128x128, void cylinder r24 (axis y), solid slab x<8, volfrac "
                                     "0.2, rmin 4.5, beta 1/2/4/8, mixed", "iterations_per_stage": per_stage,
        "simp_iterations_per_s": n_it / (total_ms / 1e3), "dof_cg_iters_per_s": ndof * total_cg / (total_ms / 1e3),
        "cg_iterations_per_step": total_cg / n_it, "stages": stages,
        "final_compliance_rel_err_vs_fp64": abs(c_m - c_r) / abs(c_r),
        "final_displacement_rel_err_vs_fp64": float((Um - Ur).norm() / Ur.norm()),
        "fp64_reference": {"relres": ref.last_relres, "iterations": ref.last_iterations},
        "fine_operator": {"launch_ms": apply_ms, "bytes_per_launch": fbytes,
                          "achieved_gbs": fbytes / (apply_ms * 1e-3) / 1e9,
                          "frac": fbytes / (apply_ms * 1e-3) / 1e9 / peak, "peak": peak, "peak_source": peak_kind},
        "solver": loop.solver.stats(), "clocks": clk.summary(),
        "device_memory_in_use_gb": (lambda fm: (fm[1] - fm[0]) / 1e9)(torch.cuda.mem_get_info())}))
    ref.close()
    loop.close()
    return 0


def solver_opts_of(args):
    """Solver options given as --solver-opt KEY=VALUE (integers or floats)."""
    opts = {}
    for kv in args.solver_opt:
        k, v = kv.split("=", 1)
        opts[k] = float(v) if any(ch in v for ch in ".e") else int(v)
    return opts


def run_probe(args):
    """Small fixed workloads for profiler captures (no timing printed as a bench value)."""
    global NELX, NELY, NELZ
    import torch

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    NELX, NELY, NELZ = args.size, args.size // 2, args.size // 2
    opts = {"fine_operator": args.fine_operator, **solver_opts_of(args)}
    loop = make_loop(args.precision, solver_options=opts)
    if args.mode == "step":
        for _ in range(max(1, args.warmup)):
            loop.step()
        torch.cuda.synchronize()
        oc_steps, cg = [], 0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            oc_steps.append(loop.step()[3:4])
            cg += loop.last["cg_iterations"]
        e1.record()
        torch.cuda.synchronize()
        print(json.dumps({"mode": "step", "size": [NELX, NELY, NELZ], "steps": args.steps,
                          "ms_per_step": e0.elapsed_time(e1) / args.steps, "cg_per_step": cg / args.steps,
                          "options": opts, "bisection_steps": [float(t.item()) for t in oc_steps],
                          "solver": loop.solver.stats()}))
    else:
        # moduli + hierarchy only (no solve), so the first launches of the
        # operator kernel in this process are the timed ones
        loop.solver.set_density(loop.S.rho_p, PENAL)
        ms = ctypes_time_apply(loop.solver, fp32=(args.precision == "mixed"))
        print(json.dumps({"mode": "apply", "size": [NELX, NELY, NELZ], "precision": args.precision,
                          "apply_ms": ms, "solver": loop.solver.stats()}))
    loop.close()
    return 0


def ctypes_time_apply(solver, fp32):
    import ctypes

    from pytopo3d_b200 import _lib

    ms = ctypes.c_double(0)
    _lib.check(_lib.lib().tp3d_solver_time_apply(solver._h, 1 if fp32 else 0, 20, ctypes.byref(ms)),
               "time_apply")
    return ms.value


if __name__ == "__main__":
    sys.exit(main())
