"""Projected-volume optimality-criteria update on the B200 (drop-in for pytopo3d/utils/oc_update.py).

The reference bisects the Lagrange multiplier on the host; every one of its
up to 80 steps re-filters and re-projects a candidate and syncs the volume
back (oc_update.py:70-122).  ``optimality_criteria_update_projected`` runs
the same sequence of midpoints, comparisons, best-candidate choice and stop
rule inside one cooperative CUDA launch (``tp3d_oc_update``).
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from ._tensors import device, like_input, to_flat, to_flat_mask, vec
from .filter import ConeFilter, _as_filter


class OCWorkspace:
    """Device scratch and stats of the OC kernel for one grid (reused across calls)."""

    def __init__(self, H: ConeFilter):
        n = _lib.lib().tp3d_oc_scratch_bytes(H.nelx, H.nely, H.nelz, float(H.rmin))
        self.scratch = torch.empty(n, dtype=torch.uint8, device=device())
        self.stats = torch.empty(8, dtype=torch.float64, device=device())


def oc_update_flat(H: ConeFilter, x, dc_dx, dv_dx, Hs, solid, void, move, target, beta, eta,
                   x_new, rho_new, ws: OCWorkspace, max_bisection_iterations=80,
                   bisection_tolerance=1e-8):
    """Flat-vector form used on the hot path; returns the device stats tensor
    [lambda_best, volume_best, steps, change, ratio_scale, lo, hi, best_error]."""
    _lib.check(_lib.lib().tp3d_oc_update(
        H.nelx, H.nely, H.nelz, float(H.rmin), x.data_ptr(), dc_dx.data_ptr(), dv_dx.data_ptr(),
        Hs.data_ptr(), _lib.ptr(solid), _lib.ptr(void), float(move), float(target), float(beta),
        float(eta), int(max_bisection_iterations), float(bisection_tolerance), x_new.data_ptr(),
        rho_new.data_ptr(), ws.stats.data_ptr(), ws.scratch.data_ptr(), _lib.stream_ptr()),
        "optimality_criteria_update_projected")
    return ws.stats


def optimality_criteria_update_projected(x, dc_dx, dv_dx, move: float, target_free_volume: float, H, Hs,
                                         beta: float, eta: float, free_mask, protected_solid,
                                         protected_void, xp=None, max_bisection_iterations: int = 80,
                                         bisection_tolerance: float = 1e-8):
    """``(best_x, best_rho)`` of the projected OC update (oc_update.py:25-124).

    ``free_mask`` must be the complement of the protected masks, as in every
    reference call site (optimizer.py:401, 627-641).
    """
    if not np.isfinite(move) or move <= 0:
        raise ValueError(f"move must be positive, got {move}")
    if max_bisection_iterations < 1:
        raise ValueError("max_bisection_iterations must be at least 1")
    H = _as_filter(H)
    shape = tuple(x.shape)
    solid, void = to_flat_mask(protected_solid), to_flat_mask(protected_void)
    free = to_flat_mask(free_mask)
    if solid is not None and void is not None:
        if not torch.equal(free.bool(), ~(solid.bool() | void.bool())):
            raise ValueError("free_mask must equal ~(protected_solid | protected_void)")
    xf = to_flat(x)
    x_new, rho_new = torch.empty_like(xf), torch.empty_like(xf)
    ws = OCWorkspace(H)
    stats = oc_update_flat(H, xf, to_flat(dc_dx), to_flat(dv_dx), vec(Hs), solid, void, move,
                           target_free_volume, beta, eta, x_new, rho_new, ws,
                           max_bisection_iterations, bisection_tolerance)
    st = stats.cpu().numpy()
    if not np.isfinite(st[2]):
        raise _lib.Topo3dError("OC bisection did not finish (bounded device wait expired)")
    best_rho = like_input(rho_new, shape, x) if np.isfinite(st[0]) else None
    return like_input(x_new, shape, x), best_rho


oc_update_projected = optimality_criteria_update_projected
