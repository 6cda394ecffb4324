"""Element strain energy on the B200 (drop-in for pytopo3d/core/compliance.py:18-75)."""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from ._tensors import device, vec
from .assembly import grid_from_edof


def element_compliance(U, edofMat, KE):
    """``ce[e] = u_e^T KE u_e`` for every element, Fortran element order.

    ``edofMat`` only identifies the structured grid (the kernel derives the
    element's DOFs from its coordinates); numpy in -> numpy out.
    """
    nelx, nely, nelz = _grid(edofMat)
    u = vec(U)
    ke = np.ascontiguousarray(np.asarray(KE.cpu() if isinstance(KE, torch.Tensor) else KE, dtype=np.float64))
    ce = torch.empty(nelx * nely * nelz, dtype=torch.float64, device=device())
    _lib.check(_lib.lib().tp3d_element_compliance(nelx, nely, nelz, u.data_ptr(), ke.ctypes.data,
                                                  ce.data_ptr(), _lib.stream_ptr()), "element_compliance")
    return ce.cpu().numpy() if isinstance(U, np.ndarray) else ce


def _grid(edofMat):
    e = edofMat.cpu().numpy() if isinstance(edofMat, torch.Tensor) else np.asarray(edofMat)
    nelx, nely, nelz = grid_from_edof(e)
    if e.shape[0] != nelx * nely * nelz:
        raise ValueError("edofMat does not describe a full structured grid")
    return nelx, nely, nelz
