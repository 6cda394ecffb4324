"""Matrix-free multigrid-preconditioned CG for K(rho) U = F on the B200.

Replaces the reference's solve boundary: the per-iteration CSR assembly and
``solver_func(Kff, F[free])`` from ``get_solver`` (pytopo3d/utils/solver.py:
15-73, called at pytopo3d/core/optimizer.py:584-594).  Two forms:

* ``precision="fp64"``: FP64 operator, FP64 multigrid V-cycle, PCG to the
  relative residual ``rtol`` (default 1e-10);
* ``precision="mixed"``: CG whose operator, multigrid V-cycle and vectors are
  FP32 (fine operator from FP32 moduli, or BF16 densities with
  ``inner_density=1``), FP64 dot products, and FP64 reliable updates: the FP32
  iterate is folded into the FP64 solution and the FP64 residual ``f - K u``
  replaces the FP32 one whenever the latter has fallen by ``reliable_delta``;
  convergence is decided on the FP64 residual, by default at ``rtol`` 1e-6
  (``MIXED_RTOL``).  That stopping rule is chosen for the compliance: on the
  128x64x64 cantilever it leaves the compliance (u'Ku, what the loop reports)
  within about 1e-8 of the FP64 solution at 1e-13 and the displacements
  within about 2e-7, against a 1e-6 compliance budget; the reference's own
  GPU path stops CuPy's CG at its default 1e-5 (pytopo3d/utils/solver.py:56).

Non-convergence raises ``RuntimeError`` like the reference's CuPy path
(solver.py:57-58).
"""

from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._tensors import device, vec


# Default relative-residual target of the mixed form (see the module docstring).
MIXED_RTOL = 1e-6


class HexSolver:
    """Solver handle for one grid, one support set and one stream."""

    def __init__(self, nelx: int, nely: int, nelz: int, KE, fixed_dofs, precision: str = "fp64",
                 **opts):
        self.grid = (int(nelx), int(nely), int(nelz))
        self.ndof = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
        self.nele = nelx * nely * nelz
        self.precision = precision
        # autotune=k: a SIMP loop searches the smoothing degrees at its k-th
        # iteration (True: the third), on that iteration's design and warm start
        # (tp3d_solver_autotune); the choice is cached per grid and precision
        at = opts.pop("autotune", 0)
        self.autotune_at = 3 if at is True else int(at or 0)
        self.autotune_pending = self.autotune_at > 0
        # "time": fastest solve alone on the GPU; "bytes": least solve traffic
        # (designs that share the GPU, where throughput rather than latency counts)
        self.autotune_criterion = opts.pop("autotune_criterion", "time")
        self.tuning = None
        L = _lib.lib()
        o = _lib.SolverOpts()
        L.tp3d_solver_default_opts(C.byref(o))
        o.precision = {"fp64": _lib.PRECISION_FP64, "mixed": _lib.PRECISION_MIXED}[precision]
        if precision == "mixed" and "rtol" not in opts:
            o.rtol = MIXED_RTOL
        for k, v in opts.items():
            if not hasattr(o, k):
                raise TypeError(f"unknown solver option {k}")
            setattr(o, k, v)
        self.opts = o
        self.KE = np.ascontiguousarray(np.asarray(KE, dtype=np.float64))
        if self.KE.shape != (24, 24):
            raise ValueError("KE must be 24x24")
        fx = torch.as_tensor(np.asarray(fixed_dofs) if isinstance(fixed_dofs, np.ndarray) else fixed_dofs)
        fx = fx.to(device=device(), dtype=torch.uint8).contiguous()
        if fx.numel() != self.ndof:
            raise ValueError(f"fixed_dofs must have {self.ndof} entries")
        self.fixed = fx
        h = C.c_void_p()
        _lib.check(L.tp3d_solver_create(nelx, nely, nelz, self.KE.ctypes.data, fx.data_ptr(), C.byref(o),
                                        _lib.stream_ptr(), C.byref(h)), "tp3d_solver_create")
        self._h = h
        self.last_iterations = 0
        self.last_relres = float("nan")

    @classmethod
    def from_freedofs(cls, nelx, nely, nelz, KE, freedofs, **kw):
        ndof = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
        fixed = np.ones(ndof, dtype=np.uint8)
        fixed[np.asarray(freedofs, dtype=np.int64)] = 0
        return cls(nelx, nely, nelz, KE, fixed, **kw)

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().tp3d_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_density(self, rho_flat: torch.Tensor, penal: float):
        """Moduli E = 1e-9 + (1 - 1e-9) rho^penal and the multigrid hierarchy."""
        self._rho = rho_flat  # keep alive while the handle may read it
        _lib.check(_lib.lib().tp3d_solver_set_density(self._h, rho_flat.data_ptr(), float(penal)),
                   "set_density")

    def solve(self, F: torch.Tensor, U: Optional[torch.Tensor] = None, raise_on_fail: bool = True):
        """U (warm start if given, updated in place) solving K U = F on the free DOFs."""
        F = vec(F)
        U = torch.zeros_like(F) if U is None else U
        it, rr = C.c_int(0), C.c_double(0)
        rc = _lib.check(_lib.lib().tp3d_solver_solve(self._h, F.data_ptr(), U.data_ptr(), C.byref(it),
                                                     C.byref(rr)), "solve")
        self.last_iterations, self.last_relres = it.value, rr.value
        if rc == _lib.TP3D_NOT_CONVERGED and raise_on_fail:
            raise RuntimeError(f"CG failed to converge: iterations={it.value}, relres={rr.value:.3e}")
        return U

    def solve_begin(self, F: torch.Tensor, U: torch.Tensor):
        """Queue the solve of K U = F (U: warm start, updated in place in stream
        order) without waiting for it; ``solve_end`` completes it."""
        self._pending_F = vec(F)
        _lib.check(_lib.lib().tp3d_solver_solve_begin(self._h, self._pending_F.data_ptr(), U.data_ptr()),
                   "solve")

    def solve_end(self, raise_on_fail: bool = True) -> bool:
        """Wait for the queued solve; True when the mixed form finished it with
        the FP64 solver after the work queued since ``solve_begin`` (which then
        read a U that has since been replaced)."""
        it, rr, rep = C.c_int(0), C.c_double(0), C.c_int(0)
        rc = _lib.check(_lib.lib().tp3d_solver_solve_end(self._h, C.byref(it), C.byref(rr), C.byref(rep)),
                        "solve")
        self._pending_F = None
        self.last_iterations, self.last_relres = it.value, rr.value
        if rc == _lib.TP3D_NOT_CONVERGED and raise_on_fail:
            raise RuntimeError(f"CG failed to converge: iterations={it.value}, relres={rr.value:.3e}")
        return bool(rep.value)

    def apply(self, u: torch.Tensor) -> torch.Tensor:
        y = torch.empty_like(u)
        fn = _lib.lib().tp3d_solver_apply_f64 if u.dtype == torch.float64 else _lib.lib().tp3d_solver_apply_f32
        _lib.check(fn(self._h, u.data_ptr(), y.data_ptr()), "apply")
        return y

    def apply_level(self, level: int, u: torch.Tensor) -> torch.Tensor:
        """Coarse level ``level``'s operator as the mixed form's V-cycle applies it
        (tp3d_solver_apply_level_f32); u: FP32, 3 x the level's nodes."""
        y = torch.empty_like(u)
        _lib.check(_lib.lib().tp3d_solver_apply_level_f32(self._h, int(level), u.data_ptr(), y.data_ptr()),
                   "apply_level")
        return y

    def stats(self) -> dict:
        buf = (C.c_double * 40)()
        n = _lib.lib().tp3d_solver_stats(self._h, buf, 40)
        keys = ["levels", "iterations", "reliable_updates", "relres", "restarts", "coarsest_dofs",
                "tile_y", "tile_x", "z_chunk", "coarse_fallback", "lambda_max_fine", "residual_floor",
                "fp64_fallback", "fine_form_fp64", "fine_form_fp32", "fused_cycle_level", "device_loop",
                "pdl", "coarse_bf16", "coarsest_status", "deep_cta_level", "bytes_per_cg_iteration",
                "kernels_per_cg_iteration", "autotuned", "degree_fine", "degree_level1", "degree_level2",
                "fine_slab_depth", "fine_threads", "cluster_level", "cluster_ctas", "fine_tile_y", "fine_tile_x"]
        return {k: buf[i] for i, k in enumerate(keys[:n])}

    def autotune(self, F: torch.Tensor, U0: Optional[torch.Tensor] = None, criterion: Optional[str] = None) -> dict:
        """Search the smoothing degrees on this grid (tp3d_solver_autotune) with
        K U = F from U0; criterion "time" (default) or "bytes"; returns the choice
        and the costs (ms for "time", GB for "bytes")."""
        F = vec(F)
        U0 = torch.zeros_like(F) if U0 is None else U0
        crit = {"time": 0, "bytes": 1}[criterion or self.autotune_criterion]
        rep = (C.c_double * 10)()
        _lib.check(_lib.lib().tp3d_solver_autotune(self._h, F.data_ptr(), U0.data_ptr(), crit, rep, 10),
                   "autotune")
        self.autotune_pending = False
        self.tuning = {"degree_fine": int(rep[0]), "degree_level1": int(rep[1]), "degree_deep": int(rep[2]),
                       "best": rep[3], "start": rep[4], "tried": int(rep[5]), "from_cache": bool(rep[6]),
                       "criterion": ("time", "bytes")[crit], "last_iterations": int(rep[8]),
                       "last_bytes_per_iteration": rep[9]}
        return self.tuning

    def time_level(self, level: int, fp32: bool, launches: int = 10):
        """(ms per launch, algorithmic bytes per launch) of the level's operator
        with cold L2 (tp3d_solver_time_level)."""
        ms, nb = C.c_double(0), C.c_double(0)
        _lib.check(_lib.lib().tp3d_solver_time_level(self._h, int(level), 1 if fp32 else 0, int(launches),
                                                     C.byref(ms), C.byref(nb)), "time_level")
        return ms.value, nb.value


def get_solver(use_gpu: bool = True):
    """``(solver_factory, name)`` — the B200 counterpart of solver.py:69-73.

    The reference returns a function of an assembled matrix; the B200 path is
    matrix-free, so the factory returned here builds a :class:`HexSolver`.
    """
    return HexSolver, "B200 matrix-free multigrid PCG"
