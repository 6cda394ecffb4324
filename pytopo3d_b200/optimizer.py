"""``top3d`` on the B200: drop-in for pytopo3d/core/optimizer.py.

Same signature, defaults, validation messages, exception types, return tuple
and ``diagnostics_out`` keys as the reference ``top3d`` (optimizer.py:283-839)
and ``evaluate_fixed_geometry_metrics`` / ``_compliance`` (:54-279).  The loop
body runs on the device with the design kept as flat Fortran-ordered CUDA
vectors; the host sees two scalars per iteration (compliance and change)
plus the logging metrics.

Extensions (keyword-only): ``F`` — an explicit nodal load vector, or a 2-D
array of load cases whose compliances are summed; ``precision`` — "fp64"
(default) or "mixed"; ``solver_options`` — HexSolver options;
``record`` — a list receiving per-iteration stats (and the iteration's new
design as a flat device tensor, key ``x``, for iterations run on the host
path); ``stage_graph`` — run each projection stage's loop bodies as one CUDA
graph launch, the stage's loop condition decided on the device
(``StageGraph``; not with ``save_history``).
"""

from __future__ import annotations

import ctypes as C
import logging
import time
from typing import Any, Dict, MutableMapping, Optional, Sequence, Tuple, Union

import numpy as np
import torch

from . import _lib
from ._tensors import device, from_flat, to_flat, to_flat_mask, vec
from .assembly import build_force_vector, build_supports
from .filter import ConeFilter, build_filter, project_flat, transpose_flat
from .oc_update import OCWorkspace, oc_update_flat
from .solver import HexSolver
from .stiffness import lk_H8

logger = logging.getLogger(__name__)

EMIN = 1.0e-9
EVAL_RTOL = 1.0e-12  # fixed-geometry evaluations (optimizer.py:54-279 solve directly)


def _fixed_dof_mask(nelx, nely, nelz, support_mask):
    ndof = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
    free, _ = build_supports(nelx, nely, nelz, ndof, support_mask)
    fixed = np.ones(ndof, dtype=np.uint8)
    fixed[free] = 0
    return fixed


def _elements_at_loaded_nodes(F2, nelx, nely, nelz):
    """Elements touching a loaded node: the explicit-load analogue of the default
    load strip protection (optimizer.py:366-369)."""
    loaded = np.any(F2.reshape(F2.shape[0], -1, 3) != 0.0, axis=(0, 2))
    node = loaded.reshape(nelz + 1, nelx + 1, nely + 1)  # [iz, ix, iy]
    el = np.zeros((nelz, nelx, nely), dtype=bool)
    for oz in (0, 1):
        for ox in (0, 1):
            for oy in (0, 1):
                el |= node[oz:oz + nelz, ox:ox + nelx, oy:oy + nely]
    return el.transpose(2, 1, 0)


def _ke(material_params, elem_size):
    return lk_H8(elem_size=elem_size) if material_params is None else lk_H8(*material_params,
                                                                              elem_size=elem_size)


def resolve_masks(nelx, nely, nelz, obstacle_mask=None, protected_zone_mask=None, force_field=None,
                  support_mask=None, F=None):
    """Protected-solid, protected-void and free masks of a run (optimizer.py:346-405).

    Same precedence, validation messages and warning as the reference: the
    default load strip ``[:, -1, 0]`` (or the elements carrying a non-zero
    force field) and the support elements (or the ``x = 0`` face when no or an
    empty support mask is given) are protected solid; a protected-void element
    wins where the two overlap.  With an explicit nodal ``F`` (an extension of
    this package) the elements touching a loaded node take the place of the
    default load strip.  Returns ``(solid, void, free)`` boolean
    ``(nely, nelx, nelz)`` arrays; raises ``ValueError`` when no element is free.
    """
    expected_shape = (nely, nelx, nelz)
    obstacle_mask = (np.zeros(expected_shape, dtype=bool) if obstacle_mask is None
                     else np.asarray(obstacle_mask, dtype=bool).copy())
    protected_zone_mask = (np.zeros(expected_shape, dtype=bool) if protected_zone_mask is None
                           else np.asarray(protected_zone_mask, dtype=bool).copy())
    if obstacle_mask.shape != expected_shape:
        raise ValueError(f"obstacle_mask has shape {obstacle_mask.shape}, expected {expected_shape}")
    if protected_zone_mask.shape != expected_shape:
        raise ValueError("protected_zone_mask has shape "
                         f"{protected_zone_mask.shape}, expected {expected_shape}")
    if force_field is None:
        if F is None:
            protected_zone_mask[:, -1, 0] = True
        else:
            protected_zone_mask |= _elements_at_loaded_nodes(np.atleast_2d(F), nelx, nely, nelz)
    else:
        if force_field.shape != expected_shape + (3,):
            raise ValueError(f"force_field has shape {force_field.shape}, "
                             f"expected {expected_shape + (3,)}")
        protected_zone_mask |= np.any(force_field != 0.0, axis=-1)
    if support_mask is None:
        protected_zone_mask[:, 0, :] = True
    else:
        if support_mask.shape != expected_shape:
            raise ValueError(f"support_mask has shape {support_mask.shape}, expected {expected_shape}")
        if np.any(support_mask):
            protected_zone_mask |= np.asarray(support_mask, dtype=bool)
        else:
            protected_zone_mask[:, 0, :] = True
    overlap = obstacle_mask & protected_zone_mask
    if np.any(overlap):
        logger.warning("Protected-solid and protected-void masks overlap at %d elements; "
                       "protected void takes precedence.", int(np.sum(overlap)))
        protected_zone_mask[overlap] = False
    free_mask = ~(obstacle_mask | protected_zone_mask)
    if not np.any(free_mask):
        raise ValueError("optimization requires at least one free design element")
    return protected_zone_mask, obstacle_mask, free_mask


class SimpState:
    """Device buffers of one SIMP loop: flat Fortran-ordered element vectors."""

    def __init__(self, H: ConeFilter, Hs, solid, void, free, KE, F, solver: HexSolver, penal):
        self.H, self.Hs = H, Hs
        self.solid, self.void, self.free = solid, void, free
        self.KE = np.ascontiguousarray(KE)
        self.F = F  # (ncases, ndof)
        self.solver = solver
        self.penal = float(penal)
        n = H.nelx * H.nely * H.nelz
        z = lambda: torch.empty(n, dtype=torch.float64, device=device())
        self.rho_f, self.rho_p, self.dproj = z(), z(), z()
        self.x_new, self.rho_new = z(), z()
        self.dc_dx, self.dv_dx, self.ce = z(), z(), z()
        self.dc_acc = z()
        self.c_dev = torch.zeros(2, dtype=torch.float64, device=device())
        self.U = torch.zeros_like(F)
        self.U_prev = torch.zeros_like(F)  # last solutions, for the extrapolated initial guess
        self.n_solved = 0
        self.n_iter = 0  # loop bodies run (not reset between stages)
        self.sens_scratch = torch.empty(
            _lib.lib().tp3d_sensitivity_scratch_bytes(H.nelx, H.nely, H.nelz), dtype=torch.uint8,
            device=device())
        self.ws = OCWorkspace(H)

    def project(self, x, beta, eta, rho_f=None, rho_p=None, dproj=None):
        return project_flat(self.H, x, self.Hs, beta, eta, self.solid, self.void,
                            self.rho_f if rho_f is None else rho_f,
                            self.rho_p if rho_p is None else rho_p,
                            self.dproj if dproj is None else dproj)

    def new_stage(self):
        """A projection change moves the physical design at once: the next solve
        starts from the last solution, not from an extrapolation across the jump."""
        self.n_solved = min(self.n_solved, 1)

    def sensitivities(self, rho_p, dproj, rerun=False):
        """Solve every load case, then fused energy / compliance / chain rule.
        ``rerun``: the iteration that a stage graph handed back after its set-up
        and warm start, so U already holds the initial guesses and the solver
        the hierarchy of rho_p."""
        L = _lib.lib()
        H = self.H
        if not rerun:
            self.solver.set_density(rho_p, self.penal)
        iters = 0
        for k in range(self.F.shape[0]):
            if not rerun:
                have_prev = 1 if self.n_solved >= 2 else 0
                if self.solver.opts.ritz_start:
                    # the best combination of the last two solutions under the new operator
                    _lib.check(L.tp3d_solver_ritz_start(self.solver._h, self.F[k].data_ptr(), self.U[k].data_ptr(),
                                                        self.U_prev[k].data_ptr(), have_prev), "ritz_start")
                else:
                    _lib.check(L.tp3d_warm_start(self.U[k].data_ptr(), self.U_prev[k].data_ptr(), self.U.shape[1],
                                                 have_prev, _lib.stream_ptr()), "warm_start")
            dst_dc = self.dc_dx if k == 0 else self.dc_acc
            if k == 0 and self.solver.autotune_pending and self.n_iter + 1 >= self.solver.autotune_at:
                self.solver.autotune(self.F[k], self.U[k])

            def sens():
                _lib.check(L.tp3d_sensitivity(
                    H.nelx, H.nely, H.nelz, H.rmin, self.U[k].data_ptr(), self.KE.ctypes.data,
                    rho_p.data_ptr(), dproj.data_ptr(), self.Hs.data_ptr(), self.free.data_ptr(), self.penal,
                    self.ce.data_ptr(), dst_dc.data_ptr(), self.dv_dx.data_ptr(),
                    self.c_dev[min(k, 1)].data_ptr(), self.sens_scratch.data_ptr(), _lib.stream_ptr()),
                    "sensitivity")

            # the sensitivities are queued behind the solve before the host waits
            # for it; a mixed solve finished in FP64 replaces U, and they are redone
            self.solver.solve_begin(self.F[k], self.U[k])
            sens()
            if self.solver.solve_end():
                sens()
            iters += self.solver.last_iterations
            if k > 0:
                self.dc_dx += self.dc_acc
                self.c_dev[0] += self.c_dev[1]
        self.n_solved += 1
        self.n_iter += 1
        return iters


def stage_desc(S: "SimpState", x, beta, eta, move, target, tolx, counters, record, U_bak, rho_new,
               max_bisection=80, bisection_tol=1e-8) -> "_lib.StageDesc":
    """The tp3d_stage_desc of a loop state: its device buffers and the stage's
    projection, OC and stopping parameters."""
    d = _lib.StageDesc()
    d.ncases = S.F.shape[0]
    d.rmin, d.beta, d.eta, d.penal, d.move = float(S.H.rmin), float(beta), float(eta), S.penal, float(move)
    d.target_free_volume, d.tolx = float(target), float(tolx)
    d.max_bisection, d.bisection_tol = int(max_bisection), float(bisection_tol)
    d.F, d.U, d.U_prev, d.U_bak = S.F.data_ptr(), S.U.data_ptr(), S.U_prev.data_ptr(), U_bak.data_ptr()
    d.x, d.x_new = x.data_ptr(), S.x_new.data_ptr()
    d.rho_f, d.rho_p, d.dproj, d.rho_new = S.rho_f.data_ptr(), S.rho_p.data_ptr(), S.dproj.data_ptr(), rho_new.data_ptr()
    d.dc_dx, d.dc_acc, d.dv_dx, d.ce = S.dc_dx.data_ptr(), S.dc_acc.data_ptr(), S.dv_dx.data_ptr(), S.ce.data_ptr()
    d.c = S.c_dev.data_ptr()
    d.Hs = S.Hs.data_ptr()
    d.solid, d.void_, d.free_mask = _lib.ptr(S.solid), _lib.ptr(S.void), S.free.data_ptr()
    d.KE_host = S.KE.ctypes.data
    d.sens_scratch, d.oc_scratch = S.sens_scratch.data_ptr(), S.ws.scratch.data_ptr()
    d.oc_stats = S.ws.stats.data_ptr()
    d.record, d.counters = record.data_ptr(), counters.data_ptr()
    return d


class StageGraph:
    """One projection stage of the loop body as a CUDA graph (tp3d_stage_*).

    Captured for the state ``S`` and the stage's projection parameters; ``x``
    is updated in place (the host path must then copy, not swap, the new
    design).  ``run(limit)`` launches it once: up to ``limit`` loop bodies,
    ending early when change <= tolx; returns (records, aborted), a record per
    completed iteration [c, lambda, volume, steps, change, CG iterations, lo,
    hi].  After an abort, each case's warm-started initial guess is in
    ``U_bak``: the caller reruns that iteration on the host path from there.
    """

    def __init__(self, S: "SimpState", x, beta, eta, move, target, tolx, capacity,
                 max_bisection=80, bisection_tol=1e-8):
        self.S = S
        self.capacity = int(capacity)
        self.counters = torch.zeros(8, dtype=torch.int32, device=device())
        self.record = torch.zeros((self.capacity, 8), dtype=torch.float64, device=device())
        self.U_bak = torch.empty_like(S.U)
        self.rho_new = torch.empty(x.numel(), dtype=torch.float64, device=device())
        self._desc = stage_desc(S, x, beta, eta, move, target, tolx, self.counters, self.record, self.U_bak,
                                self.rho_new, max_bisection, bisection_tol)
        self._x = x
        h = C.c_void_p()
        _lib.check(_lib.lib().tp3d_stage_capture(S.solver._h, C.byref(self._desc), _lib.stream_ptr(), C.byref(h)),
                   "stage_capture")
        self._h = h

    def run(self, limit: int):
        limit = min(int(limit), self.capacity)
        self.counters.copy_(torch.tensor([0, 0, 0, limit, self.S.n_solved, 0, 0, 0], dtype=torch.int32))
        it, ab = C.c_int(0), C.c_int(0)
        _lib.check(_lib.lib().tp3d_stage_run(self._h, _lib.stream_ptr(), C.byref(it), C.byref(ab)), "stage_run")
        rec = self.record[:it.value].cpu().numpy().copy()
        _lib.lib().tp3d_stage_count_launches(self._h, it.value + ab.value, int(rec[:, 5].sum()) if len(rec) else 0)
        self.S.n_solved += it.value
        self.S.n_iter += it.value
        return rec, bool(ab.value)

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().tp3d_stage_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SimpLoop:
    """Stateful SIMP loop on the device: set up once, then one ``step()`` per
    iteration of the loop body (optimizer.py:578-696).

    ``step()`` works on device-resident state; ``step_host(x)`` takes and
    returns host arrays (pinned copies in both directions) for callers that keep
    the design on the host.
    """

    def __init__(self, nelx, nely, nelz, volfrac, penal, rmin, KE, F, fixed_dofs, protected_solid,
                 protected_void, projection_eta=0.5, move=0.2, precision="fp64", solver_options=None,
                 x0=None):
        self.shape = (nely, nelx, nelz)
        if isinstance(protected_solid, torch.Tensor) or isinstance(protected_void, torch.Tensor):
            # flat uint8 device masks (Fortran element order), e.g. built by obstacle_mask_flat
            solid_d = torch.as_tensor(protected_solid).to(device(), torch.uint8).reshape(-1)
            void_d = torch.as_tensor(protected_void).to(device(), torch.uint8).reshape(-1)
            free_d = ((solid_d | void_d) == 0).to(torch.uint8)
            nfree = int(free_d.sum())
        else:
            solid = np.asarray(protected_solid, bool)
            void = np.asarray(protected_void, bool)
            solid_d, void_d, free_d = to_flat_mask(solid), to_flat_mask(void), to_flat_mask(~(solid | void))
            nfree = int((~(solid | void)).sum())
        self.target = float(volfrac * nfree)
        self.eta, self.move, self.penal = float(projection_eta), float(move), float(penal)
        H, Hs = build_filter(nelx, nely, nelz, rmin)
        self.solver = HexSolver(nelx, nely, nelz, KE, fixed_dofs, precision=precision,
                                **(solver_options or {}))
        Fd = torch.as_tensor(np.atleast_2d(np.asarray(F, dtype=np.float64))).to(device()).contiguous()
        self.S = SimpState(H, Hs, solid_d, void_d, free_d, KE, Fd, self.solver, penal)
        if x0 is None:
            # volfrac on free elements, 1 on protected solid, 0 on protected void (void wins)
            x = torch.full((nelx * nely * nelz,), float(volfrac), dtype=torch.float64, device=device())
            x[solid_d.bool()] = 1.0
            x[void_d.bool()] = 0.0
            self.x = x
        else:
            self.x = to_flat(x0)
        self.beta = None
        self.last = {}
        self.copy_mode = False  # a captured graph holds x's address: copy the new design, do not swap
        n = self.x.numel()
        self._pin_in = torch.empty(n, dtype=torch.float64, pin_memory=True)
        self._pin_out = torch.empty(n + 1, dtype=torch.float64, pin_memory=True)

    def set_beta(self, beta):
        self.beta = float(beta)
        self.S.project(self.x, self.beta, self.eta)
        self.S.new_stage()

    def step(self, rerun=False):
        """One loop body: solve, sensitivities, OC update, re-projection.
        Returns the device stats tensor [c, lambda, volume, steps, change, ...].
        ``rerun``: the iteration a graph handed back (see SimpState.sensitivities)."""
        S = self.S
        cg = S.sensitivities(S.rho_p, S.dproj, rerun=rerun)
        stats = oc_update_flat(S.H, self.x, S.dc_dx, S.dv_dx, S.Hs, S.solid, S.void, self.move, self.target,
                               self.beta, self.eta, S.x_new, S.rho_new, S.ws)
        if self.copy_mode:
            self.x.copy_(S.x_new)
        else:
            self.x, S.x_new = S.x_new, self.x
        S.project(self.x, self.beta, self.eta)
        self.last = dict(cg_iterations=cg, relres=self.solver.last_relres)
        return torch.cat([S.c_dev[:1], stats])

    def step_host(self, x_host: np.ndarray):
        """Host design in (Fortran-flat or (nely, nelx, nelz)), host (x_new, compliance) out."""
        xf = np.asarray(x_host, dtype=np.float64)
        if xf.ndim == 3:
            xf = xf.transpose(2, 1, 0).reshape(-1)
        self._pin_in.numpy()[:] = xf
        self.x.copy_(self._pin_in, non_blocking=True)
        self.S.project(self.x, self.beta, self.eta)
        st = self.step()
        self._pin_out[:-1].copy_(self.x, non_blocking=True)
        self._pin_out[-1:].copy_(st[:1], non_blocking=True)
        torch.cuda.current_stream().synchronize()
        out = self._pin_out.numpy()
        return out[:-1].copy(), float(out[-1])

    def design(self):
        return from_flat(self.x, self.shape)

    def physical(self):
        return from_flat(self.S.rho_p, self.shape)

    def close(self):
        self.solver.close()


def _free_stats(rho: torch.Tensor, free: torch.Tensor):
    f = free.bool()
    r = rho[f]
    return float(r.mean()), float(((r > 0.05) & (r < 0.95)).double().mean())


def top3d(
    nelx: int,
    nely: int,
    nelz: int,
    volfrac: float,
    penal: float,
    rmin: float,
    disp_thres: float,
    material_params: Optional[Sequence[float]] = None,
    elem_size: float = 0.01,
    obstacle_mask: Optional[np.ndarray] = None,
    force_field: Optional[np.ndarray] = None,
    support_mask: Optional[np.ndarray] = None,
    tolx: float = 0.01,
    maxloop: int = 2000,
    save_history: bool = False,
    history_frequency: int = 10,
    use_gpu: bool = False,
    protected_zone_mask: Optional[np.ndarray] = None,
    beta_schedule: Sequence[float] = (1.0, 2.0, 4.0, 8.0),
    projection_eta: float = 0.5,
    move: float = 0.2,
    diagnostics_out: Optional[MutableMapping[str, Any]] = None,
    *,
    F: Optional[np.ndarray] = None,
    precision: str = "fp64",
    solver_options: Optional[Dict[str, Any]] = None,
    record: Optional[list] = None,
    stage_graph: bool = False,
) -> Tuple[np.ndarray, Optional[Dict[str, list]], float, None]:
    """Density-filtered SIMP with Heaviside continuation (optimizer.py:283-839).

    ``maxloop`` caps each beta stage.  Returns ``(xPhys, history, compliance,
    None)`` with xPhys the projected physical density (numpy, (nely, nelx, nelz)).
    ``use_gpu`` is accepted for signature compatibility; the path is always the B200.
    """
    # ---- validation (optimizer.py:313-341) ----
    if min(nelx, nely, nelz) < 1:
        raise ValueError("nelx, nely, and nelz must all be positive")
    expected_shape = (nely, nelx, nelz)
    if not 0.0 < volfrac <= 1.0:
        raise ValueError(f"volfrac must be in (0, 1], got {volfrac}")
    if not np.isfinite(penal) or penal <= 0:
        raise ValueError(f"penal must be positive, got {penal}")
    if not np.isfinite(maxloop) or maxloop < 1:
        raise ValueError(f"maxloop must be at least 1, got {maxloop}")
    if not np.isfinite(tolx) or tolx <= 0:
        raise ValueError(f"tolx must be positive, got {tolx}")
    if not np.isfinite(history_frequency) or history_frequency < 1:
        raise ValueError(f"history_frequency must be at least 1, got {history_frequency}")
    if not np.isfinite(move) or move <= 0:
        raise ValueError(f"move must be positive, got {move}")
    if not 0.0 < projection_eta < 1.0:
        raise ValueError(f"projection_eta must be between 0 and 1, got {projection_eta}")
    beta_schedule = tuple(float(b) for b in beta_schedule)
    if not beta_schedule:
        raise ValueError("beta_schedule must contain at least one value")
    if any(not np.isfinite(b) or b <= 0.0 for b in beta_schedule):
        raise ValueError(f"all beta_schedule values must be finite and positive, got {beta_schedule}")

    ndof = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
    if F is not None:
        F = np.atleast_2d(np.asarray(F, dtype=np.float64))
        if F.ndim != 2 or F.shape[1] != ndof:
            raise ValueError(f"F must have {ndof} entries per load case")

    # ---- masks (optimizer.py:346-405) ----
    protected_zone_mask, obstacle_mask, free_mask = resolve_masks(
        nelx, nely, nelz, obstacle_mask, protected_zone_mask, force_field, support_mask, F)
    design_nele = int(np.sum(free_mask))
    target_free_volume = float(volfrac * design_nele)

    # ---- setup (optimizer.py:427-463) on the device ----
    Fh = build_force_vector(nelx, nely, nelz, ndof, force_field)[None, :] if F is None else F
    KE = _ke(material_params, elem_size)
    H, Hs = build_filter(nelx, nely, nelz, rmin)
    solid, void, free = (to_flat_mask(protected_zone_mask), to_flat_mask(obstacle_mask),
                         to_flat_mask(free_mask))
    solver = HexSolver(nelx, nely, nelz, KE, _fixed_dof_mask(nelx, nely, nelz, support_mask),
                       precision=precision, **(solver_options or {}))
    Fd = torch.as_tensor(Fh, dtype=torch.float64).to(device()).contiguous()
    S = SimpState(H, Hs, solid, void, free, KE, Fd, solver, penal)

    x0 = np.full(expected_shape, volfrac, dtype=float)
    x0[protected_zone_mask] = 1.0
    x0[obstacle_mask] = 0.0
    x = to_flat(x0)
    history = ({"density_history": [], "iteration_history": [], "compliance_history": [],
                "beta_history": []} if save_history else None)

    def bounds(beta):
        lo = np.zeros(expected_shape)
        lo[protected_zone_mask] = 1.0
        hi = np.ones(expected_shape)
        hi[obstacle_mask] = 0.0
        out = []
        for d in (lo, hi):
            _, rp, _ = S.project(to_flat(d), beta, projection_eta, torch.empty_like(x),
                                 torch.empty_like(x), torch.empty_like(x))
            out.append(float(rp[free.bool()].mean()))
        return out

    # one CUDA graph launch per projection stage (after the run's first loop body,
    # which sets the solver up); per-iteration densities are not kept on the
    # device, so a run that saves its history stays on the host path
    use_graph = bool(stage_graph) and not save_history
    total_loop = 0
    c = float("nan")
    snap = torch.empty(nelx * nely * nelz, dtype=torch.float64, pin_memory=True) if save_history else None
    stage_summaries = []
    for beta in beta_schedule:
        logger.info("Starting projection stage: beta=%g", beta)
        change, stage_loop, c_prev = float("inf"), 0, float("nan")
        S.project(x, beta, projection_eta)
        S.new_stage()
        vmin, vmax = bounds(beta)
        within = vmin - 1.0e-10 <= volfrac <= vmax + 1.0e-10
        if volfrac < vmin - 1.0e-10:
            raise ValueError(
                "projected free-volume target is infeasible at "
                f"beta={beta:g}: target={volfrac:.6f}, minimum achievable="
                f"{vmin:.6f}. Protected-solid density "
                "spreads into the free region through the density filter.")
        if volfrac > vmax + 1.0e-10:
            logger.warning("Projected free-volume target %.6f exceeds the maximum achievable %.6f at "
                           "beta=%g; the volume upper bound is inactive at the all-solid free design.",
                           volfrac, vmax, beta)
        graph = None
        rerun = False  # the next host iteration reruns one that the stage graph handed back
        while change > tolx and stage_loop < maxloop:
            if use_graph and not rerun and not solver.autotune_pending and total_loop > 0:
                # the rest of the stage as one graph launch (until change <= tolx,
                # maxloop, or a solve that the host path has to finish)
                if graph is None:
                    try:
                        graph = StageGraph(S, x, beta, projection_eta, move, target_free_volume, tolx, maxloop)
                    except _lib.Topo3dError as e:
                        logger.warning("stage graph unavailable (%s); the loop runs on the host path", e)
                        use_graph = False
                        continue
                t0 = time.time()
                rec_arr, aborted = graph.run(maxloop - stage_loop)
                dt = (time.time() - t0) / max(1, len(rec_arr))
                for r in rec_arr:
                    stage_loop += 1
                    total_loop += 1
                    c, change = float(r[0]), float(r[4])
                    if not np.isfinite(r[3]):
                        raise _lib.Topo3dError("OC bisection did not finish (bounded device wait expired)")
                    c_delta = c - c_prev if np.isfinite(c_prev) else float("nan")
                    c_prev = c
                    if record is not None:
                        record.append(dict(beta=beta, c=c, change=change, cg_iterations=int(r[5]),
                                           relres=float("nan"), bisection_steps=int(r[3]), lam=float(r[1]),
                                           stage_graph=True))
                    logger.info("beta=%4.1f iter=%4d total=%4d C=%.6e dC=%.3e change=%.5e time=%.4fs cg=%d "
                                "(stage graph)", beta, stage_loop, total_loop, c, c_delta, change, dt, int(r[5]))
                if aborted:
                    # a solve that the host path finishes differently: rerun that
                    # iteration from its warm-started initial guesses
                    S.U.copy_(graph.U_bak)
                    rerun = True
                continue
            stage_loop += 1
            total_loop += 1
            t0 = time.time()
            if save_history:
                # the design this iteration solves on, copied to pinned host memory
                # while the iteration runs (read only if the iteration is recorded)
                snap.copy_(S.rho_p, non_blocking=True)
            cg_iters = S.sensitivities(S.rho_p, S.dproj, rerun=rerun)
            rerun = False
            stats = oc_update_flat(H, x, S.dc_dx, S.dv_dx, Hs, solid, void, move, target_free_volume, beta,
                                   projection_eta, S.x_new, S.rho_new, S.ws)
            host = torch.cat([S.c_dev[:1], stats]).cpu().numpy()
            c, change = float(host[0]), float(host[4])
            if not np.isfinite(host[3]):
                raise _lib.Topo3dError("OC bisection did not finish (bounded device wait expired)")
            if use_graph:
                x.copy_(S.x_new)  # the stage graph holds x's address
            else:
                x, S.x_new = S.x_new, x
            c_delta = c - c_prev if np.isfinite(c_prev) else float("nan")
            c_prev = c
            if record is not None:
                record.append(dict(beta=beta, c=c, change=change, cg_iterations=cg_iters,
                                   relres=solver.last_relres, bisection_steps=int(host[3]),
                                   lam=float(host[1]), x=x.clone()))
            if save_history and ((total_loop - 1) % history_frequency == 0 or change <= tolx
                                 or stage_loop == maxloop):
                history["density_history"].append(snap.numpy().reshape(nelz, nelx, nely).transpose(2, 1, 0).copy())
                history["iteration_history"].append(total_loop - 1)
                history["compliance_history"].append(c)
                history["beta_history"].append(beta)
            if logger.isEnabledFor(logging.INFO):
                vol, gray = _free_stats(S.rho_new, free)
                logger.info("beta=%4.1f iter=%4d total=%4d C=%.6e dC=%.3e vol=%.5f gray=%.5f "
                            "change=%.5e time=%.2fs cg=%d", beta, stage_loop, total_loop, c, c_delta, vol,
                            gray, change, time.time() - t0, cg_iters)
            S.project(x, beta, projection_eta)
        if graph is not None:
            graph.close()
        vol, gray = _free_stats(S.rho_p, free)
        converged = change <= tolx
        if not converged:
            logger.warning("Projection stage beta=%g reached maxloop=%d without converging: final change "
                           "%.6e exceeds tolx %.6e.", beta, maxloop, change, tolx)
        stage_summaries.append({
            "beta": float(beta), "iterations": int(stage_loop), "converged": bool(converged),
            "physical_density_fraction": vol, "volume_fraction_error": vol - float(volfrac),
            "gray_fraction_005_095": gray, "final_change": float(change),
            "minimum_achievable_physical_fraction": vmin, "maximum_achievable_physical_fraction": vmax,
            "target_within_achievable_range": within})

    final_beta = beta_schedule[-1]
    S.project(x, final_beta, projection_eta)
    final_x = from_flat(x, expected_shape).cpu().numpy()
    final_rho_filtered = from_flat(S.rho_f, expected_shape).cpu().numpy()
    final_xPhys = from_flat(S.rho_p, expected_shape).cpu().numpy()

    solver.close()
    # Final and binary designs are evaluated by a tight FP64 solve: thresholded
    # designs with 1e-9 voids are far worse conditioned than the loop's iterates.
    eval_solver = HexSolver(nelx, nely, nelz, KE, _fixed_dof_mask(nelx, nely, nelz, support_mask),
                            precision="fp64", rtol=EVAL_RTOL, max_iterations=20000)
    ev = dict(penal=penal, material_params=material_params, elem_size=elem_size, force_field=force_field,
              support_mask=support_mask, obstacle_mask=obstacle_mask,
              protected_zone_mask=protected_zone_mask, _solver=eval_solver, _F=Fd)
    final_compliance = evaluate_fixed_geometry_compliance(xPhys=final_xPhys, **ev)
    if save_history:
        history["density_history"].append(final_xPhys.copy())
        history["iteration_history"].append(total_loop)
        history["compliance_history"].append(float(final_compliance))
        history["beta_history"].append(float(final_beta))
    rho_binary = (final_xPhys >= 0.5).astype(float)
    rho_binary[protected_zone_mask] = 1.0
    rho_binary[obstacle_mask] = 0.0
    binary_compliance = evaluate_fixed_geometry_compliance(xPhys=rho_binary, **ev)
    delta = ((binary_compliance - final_compliance) / final_compliance if final_compliance != 0.0 else None)
    fv = final_xPhys[free_mask]
    gray_mask = (fv > 0.05) & (fv < 0.95)
    metrics = {
        "projection_enabled": True,
        "projection_beta": float(final_beta),
        "projection_beta_schedule": [float(b) for b in beta_schedule],
        "projection_eta": float(projection_eta),
        "penal": float(penal),
        "design_variable_fraction": float(np.mean(final_x[free_mask])),
        "filtered_density_fraction": float(np.mean(final_rho_filtered[free_mask])),
        "physical_density_fraction": float(np.mean(fv)),
        "gray_fraction_005_095": float(np.mean(gray_mask.astype(float))),
        "projected_compliance": float(final_compliance),
        "binary_compliance": float(binary_compliance),
        "binary_compliance_delta": None if delta is None else float(delta),
        "binary_threshold": 0.5,
        "target_free_volume_fraction": float(volfrac),
        "physical_volume_fraction_error": float(np.mean(fv) - volfrac),
        "projection_total_iterations": int(total_loop),
        "projection_stage_summaries": stage_summaries,
        "projection_converged": all(s["converged"] for s in stage_summaries),
        "projection_target_within_achievable_range": all(
            s["target_within_achievable_range"] for s in stage_summaries),
    }
    logger.info("Final projection: beta=%.1f eta=%.3f vol=%.5f gray=%.5f C_projected=%.6e C_binary=%.6e",
                final_beta, projection_eta, metrics["physical_density_fraction"],
                metrics["gray_fraction_005_095"], final_compliance, binary_compliance)
    if diagnostics_out is not None:
        diagnostics_out.clear()
        diagnostics_out.update(metrics)
    eval_solver.close()
    return final_xPhys, history, final_compliance, None


def evaluate_fixed_geometry_metrics(xPhys, penal, material_params=None, elem_size=0.01, force_field=None,
                                    support_mask=None, obstacle_mask=None, protected_zone_mask=None,
                                    use_gpu=False, *, F=None, precision="fp64", _solver=None, _F=None):
    """One device solve on a fixed design plus load-patch metrics (optimizer.py:54-252)."""
    xPhys = np.asarray(xPhys, dtype=float)
    nely, nelx, nelz = xPhys.shape
    ndof = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
    x_eval = xPhys.copy()
    if protected_zone_mask is not None:
        x_eval[np.asarray(protected_zone_mask, bool)] = 1.0
    if obstacle_mask is not None:
        x_eval[np.asarray(obstacle_mask, bool)] = 0.0
    if _F is not None:
        Fd = _F
        Fh = _F.cpu().numpy()
    else:
        Fh = (build_force_vector(nelx, nely, nelz, ndof, force_field) if F is None
              else np.asarray(F, dtype=np.float64))
        Fh = np.atleast_2d(Fh)
        Fd = torch.as_tensor(Fh).to(device())
    KE = _ke(material_params, elem_size)
    solver = _solver
    if solver is None:
        solver = HexSolver(nelx, nely, nelz, KE, _fixed_dof_mask(nelx, nely, nelz, support_mask),
                           precision=precision, rtol=EVAL_RTOL, max_iterations=20000)
    rho = to_flat(x_eval)
    solver.set_density(rho, penal)
    E = EMIN + (1.0 - EMIN) * rho ** penal
    total = 0.0
    U_all = []
    ce = torch.empty_like(rho)
    for k in range(Fd.shape[0]):
        U = solver.solve(Fd[k])
        _lib.check(_lib.lib().tp3d_element_compliance(nelx, nely, nelz, U.data_ptr(),
                                                      np.ascontiguousarray(KE).ctypes.data, ce.data_ptr(),
                                                      _lib.stream_ptr()), "element_compliance")
        total += float(torch.dot(E, ce))
        U_all.append(U)
    U = U_all[0].cpu().numpy()
    F0 = Fh[0]
    loaded = np.flatnonzero(np.abs(F0) > 0.0)
    nodes = np.unique(loaded // 3)
    out = {"compliance": float(total)}
    tot = {}
    for ci, ax in enumerate("xyz"):
        d = 3 * nodes + ci
        tot[ax] = float(np.sum(np.abs(F0[d]))) if d.size else 0.0
        out[f"u{ax}_avg_load_patch"] = float(np.mean(U[d])) if d.size else None
    for ax in "xyz":
        u = out[f"u{ax}_avg_load_patch"]
        out[f"k_avg_{ax}"] = (float(tot[ax] / abs(u)) if u is not None and u != 0.0 and tot[ax] > 0.0
                              else None)
    dom = max((("x", tot["x"]), ("y", tot["y"]), ("z", tot["z"])), key=lambda t: t[1])[0]
    out["k_avg"] = out[f"k_avg_{dom}"]
    out["F_total"] = float(np.sum(np.abs(F0[loaded]))) if loaded.size else 0.0
    for ax in "xyz":
        out[f"F_total_{ax}"] = tot[ax]
    for ax in "xyz":
        out[f"loaded_{ax}_dof_count"] = int(nodes.size)
    if _solver is None:
        solver.close()
    return out


def evaluate_fixed_geometry_compliance(xPhys, penal, material_params=None, elem_size=0.01,
                                       force_field=None, support_mask=None, obstacle_mask=None,
                                       protected_zone_mask=None, use_gpu=False, **kw) -> float:
    """Compliance only (optimizer.py:255-279)."""
    return float(evaluate_fixed_geometry_metrics(xPhys, penal, material_params, elem_size, force_field,
                                                 support_mask, obstacle_mask, protected_zone_mask, use_gpu,
                                                 **kw)["compliance"])
