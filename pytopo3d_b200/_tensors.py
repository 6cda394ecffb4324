"""Conversions between the reference's (nely, nelx, nelz) arrays and the flat
Fortran-ordered device vectors the kernels use (e = y + nely*(x + nelx*z))."""

from __future__ import annotations

import numpy as np
import torch


def device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("pytopo3d_b200 needs a CUDA device (B200, sm_100a); no CPU fallback")
    return torch.device("cuda", torch.cuda.current_device())


def to_flat(a, dtype=torch.float64) -> torch.Tensor:
    """(nely, nelx, nelz) array/tensor -> contiguous flat device vector in Fortran order."""
    t = torch.as_tensor(np.asarray(a) if isinstance(a, np.ndarray) else a)
    if t.dim() == 3:
        t = t.permute(2, 1, 0)
    t = t.to(device=device(), dtype=dtype)
    return t.contiguous().reshape(-1)


def to_flat_mask(m) -> torch.Tensor | None:
    if m is None:
        return None
    return to_flat(m, torch.uint8)


def from_flat(v: torch.Tensor, shape) -> torch.Tensor:
    """Flat Fortran-ordered vector -> (nely, nelx, nelz) view."""
    nely, nelx, nelz = shape
    return v.reshape(nelz, nelx, nely).permute(2, 1, 0)


def like_input(v: torch.Tensor, shape, template):
    """Return a result shaped like the reference (numpy in -> numpy out)."""
    out = from_flat(v, shape)
    if isinstance(template, np.ndarray):
        return out.cpu().numpy()
    return out


def vec(a, dtype=torch.float64) -> torch.Tensor:
    """1-D array/tensor -> contiguous device vector."""
    t = torch.as_tensor(np.asarray(a) if isinstance(a, np.ndarray) else a)
    return t.to(device=device(), dtype=dtype).contiguous().reshape(-1)
