"""Density filter and Heaviside projection on the B200 (drop-ins for pytopo3d/utils/filter.py).

The reference forms a sparse cone-weight matrix H with a KD-tree and a Python
loop (filter.py:122-228) and applies it with SpMV.  Here ``build_filter``
returns a :class:`ConeFilter` descriptor in place of H: the weights
``rmin - |d|`` (integer offsets, kept when > 1e-9, truncated at the domain
boundary) are applied as a shared-memory stencil by the CUDA kernels, and
``Hs`` (the row sums) is computed on the device by the same stencil.  Because
H is symmetric, ``H.T @ v`` is the same stencil.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._tensors import device, like_input, to_flat, to_flat_mask, vec

FLOAT_EPSILON = 1e-9


@dataclass(frozen=True)
class ConeFilter:
    """Matrix-free stand-in for the reference's filter matrix H."""

    nelx: int
    nely: int
    nelz: int
    rmin: float

    @property
    def shape(self):
        n = self.nelx * self.nely * self.nelz
        return (n, n)

    @property
    def T(self):  # H is symmetric
        return self

    def taps(self):
        """(dx, dy, dz, w) offsets of the stencil, as the reference's threshold keeps them."""
        R = int(math.ceil(self.rmin)) + 1
        out = []
        for dz in range(-R, R + 1):
            for dx in range(-R, R + 1):
                for dy in range(-R, R + 1):
                    w = self.rmin - math.sqrt(float(dx * dx + dy * dy + dz * dz))
                    if w > FLOAT_EPSILON:
                        out.append((dx, dy, dz, w))
        return out

    def __matmul__(self, v):
        """H @ v for a flat Fortran-ordered vector (divides by nothing)."""
        v = vec(v)
        out = torch.empty_like(v)
        ones = torch.ones_like(v)
        _lib.check(_lib.lib().tp3d_filter_transpose(self.nelx, self.nely, self.nelz, float(self.rmin),
                                                    v.data_ptr(), None, ones.data_ptr(), out.data_ptr(),
                                                    _lib.stream_ptr()), "filter")
        return out


def _validate_grid(nelx, nely, nelz, rmin):
    if min(nelx, nely, nelz) < 1:
        raise ValueError("nelx, nely, and nelz must all be positive")
    if not np.isfinite(rmin) or rmin <= 0.0:
        raise ValueError(f"rmin must be finite and positive, got {rmin}")
    if rmin - 7.0 > 1e-9:
        # the stencil reaches offsets d with rmin - d > 1e-9; its shared-memory
        # tile holds offsets up to 6 per axis
        raise ValueError(f"rmin too large for the stencil filter (max 7), got {rmin}")


def filter_rowsum(H: ConeFilter) -> torch.Tensor:
    Hs = torch.empty(H.nelx * H.nely * H.nelz, dtype=torch.float64, device=device())
    _lib.check(_lib.lib().tp3d_filter_rowsum(H.nelx, H.nely, H.nelz, float(H.rmin), Hs.data_ptr(),
                                             _lib.stream_ptr()), "build_filter")
    return Hs


def build_filter(nelx: int, nely: int, nelz: int, rmin: float):
    """``(H, Hs)``: a :class:`ConeFilter` and the device row sums (filter.py:122-228)."""
    _validate_grid(nelx, nely, nelz, rmin)
    H = ConeFilter(int(nelx), int(nely), int(nelz), float(rmin))
    return H, filter_rowsum(H)


def _check_projection(beta, eta):
    if not np.isfinite(beta) or beta <= 0:
        raise ValueError(f"beta must be positive, got {beta}")
    if not 0.0 < eta < 1.0:
        raise ValueError(f"eta must be between 0 and 1, got {eta}")


def heaviside_projection(rho_filtered, beta: float, eta: float = 0.5, xp=None):
    """Projected density (clipped to [0, 1]) and its unclipped derivative (filter.py:26-60)."""
    _check_projection(beta, eta)
    is_np = isinstance(rho_filtered, np.ndarray)
    t = torch.as_tensor(np.asarray(rho_filtered) if is_np else rho_filtered)
    shape = t.shape
    r = t.to(device=device(), dtype=torch.float64).contiguous().reshape(-1)
    out, der = torch.empty_like(r), torch.empty_like(r)
    _lib.check(_lib.lib().tp3d_heaviside(r.data_ptr(), r.numel(), float(beta), float(eta), out.data_ptr(),
                                         der.data_ptr(), _lib.stream_ptr()), "heaviside_projection")
    out, der = out.reshape(shape), der.reshape(shape)
    if is_np:
        return out.cpu().numpy(), der.cpu().numpy()
    return out, der


def _as_filter(H) -> ConeFilter:
    if not isinstance(H, ConeFilter):
        raise TypeError("H must be the ConeFilter returned by pytopo3d_b200.build_filter")
    return H


def project_flat(H: ConeFilter, x: torch.Tensor, Hs: torch.Tensor, beta, eta, solid, void,
                 rho_f=None, rho_p=None, dproj=None):
    """Flat-vector form used on the hot path; outputs may be preallocated."""
    rho_p = torch.empty_like(x) if rho_p is None else rho_p
    _lib.check(_lib.lib().tp3d_filter_project(
        H.nelx, H.nely, H.nelz, float(H.rmin), x.data_ptr(), Hs.data_ptr(), float(beta), float(eta),
        _lib.ptr(solid), _lib.ptr(void), _lib.ptr(rho_f), rho_p.data_ptr(), _lib.ptr(dproj),
        _lib.stream_ptr()), "build_physical_density")
    return rho_f, rho_p, dproj


def build_physical_density(x, H, Hs, beta: float, eta: float, protected_solid, protected_void, xp=None):
    """``(rho_filtered, rho_physical, projection_derivative)`` (filter.py:63-100)."""
    H = _as_filter(H)
    _check_projection(beta, eta)
    shape = tuple(x.shape)
    xf = to_flat(x)
    Hs_d = vec(Hs)
    rf, rp, dp = torch.empty_like(xf), torch.empty_like(xf), torch.empty_like(xf)
    project_flat(H, xf, Hs_d, beta, eta, to_flat_mask(protected_solid), to_flat_mask(protected_void),
                 rf, rp, dp)
    return like_input(rf, shape, x), like_input(rp, shape, x), like_input(dp, shape, x)


def transpose_flat(H: ConeFilter, g: torch.Tensor, dproj, Hs: torch.Tensor, out=None):
    out = torch.empty_like(g) if out is None else out
    _lib.check(_lib.lib().tp3d_filter_transpose(H.nelx, H.nely, H.nelz, float(H.rmin), g.data_ptr(),
                                                _lib.ptr(dproj), Hs.data_ptr(), out.data_ptr(),
                                                _lib.stream_ptr()), "apply_density_filter_chain_rule")
    return out


def apply_density_filter_chain_rule(physical_derivative, projection_derivative, H, Hs):
    """``H^T (g * dproj / Hs)`` with the input's shape (filter.py:103-119)."""
    H = _as_filter(H)
    shape = tuple(physical_derivative.shape)
    out = transpose_flat(H, to_flat(physical_derivative), to_flat(projection_derivative), vec(Hs))
    return like_input(out, shape, physical_derivative)
