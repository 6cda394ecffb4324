"""Many independent SIMP designs at once on one GPU.

A batch of designs of uneven grid sizes (the batched workload: 64 seeded
cantilevers with random sizes, volume fractions, filter radii, void
cylinders and load positions) is run as one ``SimpLoop`` per design, each on
its own CUDA stream, driven by a small pool of host threads.  Every design
is an independent problem, so nothing is shared between them but the GPU:
the small designs' launches, which would leave most of the 148 SMs idle one
at a time, overlap across streams.  (The library calls release the GIL, so
the host threads run concurrently too.)

The reference runs designs one after another (runners/experiment.py); this
module has no reference counterpart beyond the per-design loop body, which
is ``SimpLoop.step`` (optimizer.py:578-696).
"""

from __future__ import annotations

import ctypes as C
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import torch

from ._tensors import device
from .assembly import build_force_vector, build_supports
from ._tensors import to_flat_mask
from .obstacles import cylinder_elements, obstacle_mask_flat
from .optimizer import SimpLoop, _elements_at_loaded_nodes
from .stiffness import lk_H8


@dataclass
class DesignSpec:
    """One cantilever of the batch: grid, volume fraction, filter radius, void
    cylinders ``(axis, centre_a, centre_b, radius)`` in element units (centre in
    the two axes perpendicular to ``axis``, in x, y, z order), and the load edge
    (``load_mid``: the x = nelx edge at z = nelz // 2 instead of z = 0)."""

    nelx: int
    nely: int
    nelz: int
    volfrac: float
    rmin: float
    cylinders: List[tuple] = field(default_factory=list)
    load_mid: bool = False
    penal: float = 3.0


def batched_cantilevers(n: int = 64, seed: int = 0) -> List[DesignSpec]:
    """The seeded batch: nelx ~ U{24..96}, nely = nelx // 2, nelz ~ U{12..48},
    volfrac ~ U[0.15, 0.4], rmin ~ U[1.5, 3.5], 0-3 void cylinders of radius
    U{2..8} with random axis and centre, load on the z = 0 or z = nelz // 2 edge
    by coin flip."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nelx = int(rng.integers(24, 97))
        nely = nelx // 2
        nelz = int(rng.integers(12, 49))
        dims = (nelx, nely, nelz)
        cyl = []
        for _ in range(int(rng.integers(0, 4))):
            axis = int(rng.integers(0, 3))
            a, b = [i for i in range(3) if i != axis]
            cyl.append((axis, int(rng.integers(0, dims[a])), int(rng.integers(0, dims[b])),
                        int(rng.integers(2, 9))))
        out.append(DesignSpec(nelx, nely, nelz, float(rng.uniform(0.15, 0.4)), float(rng.uniform(1.5, 3.5)),
                              cyl, bool(rng.integers(0, 2))))
    return out


def design_problem(spec: DesignSpec):
    """Masks, total-unit load, fixed DOFs of one design: clamped at x = 0, the
    -z load on the chosen x = nelx edge; elements at the clamped face and at the
    loaded nodes are protected solid (optimizer.py:366-390), void wins over
    solid (:392-399).  The masks are flat uint8 device tensors: the void
    cylinders are built by the obstacle-mask kernel on the current stream."""
    nelx, nely, nelz = spec.nelx, spec.nely, spec.nelz
    shape = (nely, nelx, nelz)
    dims = (nelx, nely, nelz)
    ndof = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
    void = obstacle_mask_flat(shape, [cylinder_elements(axis, ca, cb, r, dims[axis])
                                      for axis, ca, cb, r in spec.cylinders])
    F = np.zeros(ndof)
    iz = nelz // 2 if spec.load_mid else 0
    for iy in range(nely + 1):
        F[3 * (iy + (nely + 1) * (nelx + (nelx + 1) * iz)) + 2] = -1.0 / (nely + 1)
    solid = _elements_at_loaded_nodes(F[None, :], nelx, nely, nelz)
    solid[:, 0, :] = True
    solid = to_flat_mask(solid) & (void == 0).to(torch.uint8)
    free, _ = build_supports(nelx, nely, nelz, ndof)
    fixed = np.ones(ndof, np.uint8)
    fixed[free] = 0
    return shape, solid, void, F, fixed


class BatchRunner:
    """One ``SimpLoop`` per design on its own stream; ``run(iterations)``
    advances every design by that many loop bodies with ``workers`` host
    threads (design i is always driven by thread i % workers).  With ``tune``
    ("bytes", the default, or "time"; None: off) every design first runs three
    loop bodies alone, the third of which autotunes its smoothing degrees on its
    own grid (``HexSolver.autotune``).  The designs then share the GPU, where
    throughput counts, so the default criterion is the solve's traffic.

    The designs' streams run concurrently only over as many hardware queues as
    the CUDA context has: set ``CUDA_DEVICE_MAX_CONNECTIONS=32`` in the
    environment before the process's first CUDA call (the default 8 cost about
    15% on the 64-design workload; ``run_graph`` does not depend on it)."""

    def __init__(self, specs: List[DesignSpec], precision: str = "mixed", beta: float = 1.0, eta: float = 0.5,
                 move: float = 0.2, workers: int = 8, solver_options: Optional[dict] = None,
                 tune: Optional[str] = "bytes"):
        self.specs = list(specs)
        self.workers = max(1, min(int(workers), len(self.specs)))
        # the designs already run side by side: each solver's set-up keeps its
        # power iterations on its own stream (fewer host calls per design)
        solver_options = {"spectra_streams": 0, **(solver_options or {})}
        self.streams = [torch.cuda.Stream(device=device()) for _ in self.specs]
        self.loops: List[SimpLoop] = [None] * len(self.specs)
        self.ndof = [3 * (s.nelx + 1) * (s.nely + 1) * (s.nelz + 1) for s in self.specs]
        KE = lk_H8(elem_size=1.0)

        def build(i):
            spec = self.specs[i]
            with torch.cuda.stream(self.streams[i]):
                shape, solid, void, F, fixed = design_problem(spec)
                loop = SimpLoop(spec.nelx, spec.nely, spec.nelz, spec.volfrac, spec.penal, spec.rmin, KE, F,
                                fixed, solid, void, projection_eta=eta, move=move, precision=precision,
                                solver_options=solver_options)
                loop.set_beta(beta)
                self.loops[i] = loop

        self._each(build)
        torch.cuda.synchronize()
        if tune:
            # smoothing degrees per design, searched at each design's third loop
            # body, one design at a time so that no other design's work disturbs
            # the timings (cached per grid)
            self.tuning = []
            for i, loop in enumerate(self.loops):
                loop.solver.autotune_at = 3
                loop.solver.autotune_pending = True
                loop.solver.autotune_criterion = tune
                with torch.cuda.stream(self.streams[i]):
                    for _ in range(3):
                        loop.step()
                torch.cuda.synchronize()
                self.tuning.append(loop.solver.tuning)
        self.cg_iterations = [0] * len(self.specs)
        self.compliance = [float("nan")] * len(self.specs)

    def _each(self, fn):
        """fn(i) for every design, design i on thread i % workers; re-raises."""
        def worker(w):
            for i in range(w, len(self.specs), self.workers):
                fn(i)

        with ThreadPoolExecutor(self.workers) as ex:
            for f in [ex.submit(worker, w) for w in range(self.workers)]:
                f.result()

    def run(self, iterations: int) -> dict:
        """Advance every design; returns wall time, SIMP iterations/s and
        DOF * CG-iterations/s of the whole batch."""
        torch.cuda.synchronize()
        cg0 = list(self.cg_iterations)
        lock = threading.Lock()

        def advance(i):
            loop = self.loops[i]
            with torch.cuda.stream(self.streams[i]):
                cg = 0
                st = None
                for _ in range(iterations):
                    st = loop.step()
                    cg += loop.last["cg_iterations"]
                c = float(st[0]) if st is not None else float("nan")
            with lock:
                self.cg_iterations[i] += cg
                self.compliance[i] = c

        t0 = time.perf_counter()
        self._each(advance)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        n = len(self.specs)
        dof_cg = sum(self.ndof[i] * (self.cg_iterations[i] - cg0[i]) for i in range(n))
        return {"seconds": dt, "designs": n, "iterations": iterations,
                "simp_iterations_per_s": n * iterations / dt, "dof_cg_iterations_per_s": dof_cg / dt}

    def run_graph(self, iterations: int) -> dict:
        """Advance every design by ``iterations`` loop bodies with ONE graph
        launch (``tp3d_batch_*``): each design's loop body in a WHILE node of its
        own, all designs parallel branches of the graph, no host thread per
        design.  Captured at the first call (every design must have run a loop
        body on the host path, which the autotuning steps or ``run`` provide);
        later calls relaunch it.  A design whose solve the host path would have
        finished differently (the mixed form's FP64 fallback) is handed back:
        its iteration is rerun on the host path and its remaining iterations
        run there.  Returns the same figures as ``run``."""
        from . import _lib
        from .optimizer import stage_desc

        n = len(self.specs)
        if any(loop.S.n_iter == 0 for loop in self.loops):
            self.run(1)
        if getattr(self, "_graph", None) is None or iterations > self._graph_cap:
            self._close_graph()
            cap = max(int(iterations), 1)
            self._graph_cap = cap
            self._g_counters = torch.zeros((n, 8), dtype=torch.int32, device=device())
            self._g_record = torch.zeros((n, cap, 8), dtype=torch.float64, device=device())
            self._g_hold = []
            descs = (_lib.StageDesc * n)()
            handles = (C.c_void_p * n)()
            for i, loop in enumerate(self.loops):
                S = loop.S
                loop.copy_mode = True
                U_bak, rho_new = torch.empty_like(S.U), torch.empty_like(loop.x)
                self._g_hold.append((U_bak, rho_new))
                descs[i] = stage_desc(S, loop.x, loop.beta, loop.eta, loop.move, loop.target, -1.0,
                                      self._g_counters[i], self._g_record[i], U_bak, rho_new)
                handles[i] = S.solver._h
            torch.cuda.synchronize()
            h = C.c_void_p()
            _lib.check(_lib.lib().tp3d_batch_capture(handles, descs, n, _lib.stream_ptr(), C.byref(h)),
                       "batch_capture")
            self._graph, self._g_descs = h, descs
        torch.cuda.synchronize()
        cg0 = list(self.cg_iterations)
        t0 = time.perf_counter()
        rows = [[0, 0, 0, int(iterations), loop.S.n_solved, 0, 0, 0] for loop in self.loops]
        self._g_counters.copy_(torch.tensor(rows, dtype=torch.int32))
        _lib.check(_lib.lib().tp3d_batch_run(self._graph, _lib.stream_ptr()), "batch_run")
        ctr = self._g_counters.cpu().numpy()
        rec = self._g_record.cpu().numpy()
        passes = (C.c_longlong * n)()
        cgs = (C.c_longlong * n)()
        handed_back = 0
        for i, loop in enumerate(self.loops):
            it, ab = int(ctr[i, 0]), int(ctr[i, 1])
            S = loop.S
            S.n_solved += it
            S.n_iter += it
            cg = int(rec[i, :it, 5].sum())
            passes[i], cgs[i] = it + ab, cg
            c = float(rec[i, it - 1, 0]) if it else float("nan")
            if ab:
                handed_back += 1
                with torch.cuda.stream(self.streams[i]):
                    S.U.copy_(self._g_hold[i][0])
                    st = loop.step(rerun=True)
                    cg += loop.last["cg_iterations"]
                    for _ in range(iterations - it - 1):
                        st = loop.step()
                        cg += loop.last["cg_iterations"]
                    c = float(st[0])
            self.cg_iterations[i] += cg
            self.compliance[i] = c
        _lib.lib().tp3d_batch_count_launches(self._graph, passes, cgs)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        dof_cg = sum(self.ndof[i] * (self.cg_iterations[i] - cg0[i]) for i in range(n))
        return {"seconds": dt, "designs": n, "iterations": iterations, "handed_back": handed_back,
                "simp_iterations_per_s": n * iterations / dt, "dof_cg_iterations_per_s": dof_cg / dt}

    def _close_graph(self):
        from . import _lib

        if getattr(self, "_graph", None) is not None:
            _lib.lib().tp3d_batch_destroy(self._graph)
            self._graph = None

    def design(self, i: int) -> torch.Tensor:
        torch.cuda.synchronize()
        return self.loops[i].design()

    def close(self):
        self._close_graph()
        for loop in self.loops:
            if loop is not None:
                loop.close()
