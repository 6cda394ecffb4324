"""Compliance of a design as a ``torch.autograd.Function`` with a hand-written adjoint.

``compliance(rho_design)`` = sum over load cases of F_k^T U_k with
K(rho_phys) U_k = F_k, rho_phys = project(H rho_design / Hs).  The backward
pass is the adjoint of that chain, the same math the reference tests use for
their gradient check (tests/test_projected_optimizer.py:24-80):

* the compliance problem is self-adjoint, so dc/drho_phys = -p (1 - Emin)
  rho^(p-1) u_e^T KE u_e per load case (optimizer.py:607-612);
* the Heaviside derivative and the filter transpose map it back to the design
  variables (filter.py:103-119).

Both run in the fused ``tp3d_sensitivity`` kernel.  Displacements are kept
from the forward pass on the autograd context (``recompute=False``), or they
are re-solved per load case in backward when device memory is short
(``recompute=True``).
"""

from __future__ import annotations

from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._tensors import device, from_flat, to_flat, to_flat_mask
from .filter import build_filter, project_flat
from .optimizer import _fixed_dof_mask
from .solver import HexSolver
from .stiffness import lk_H8


class ComplianceProblem:
    """Grid, loads, supports, filter and projection settings of a compliance objective."""

    def __init__(self, nelx, nely, nelz, F, rmin, beta, eta=0.5, penal=3.0, KE=None, support_mask=None,
                 protected_solid=None, protected_void=None, precision="fp64", recompute=True,
                 solver_options=None):
        self.shape = (nely, nelx, nelz)
        self.nele = nelx * nely * nelz
        self.beta, self.eta, self.penal = float(beta), float(eta), float(penal)
        self.KE = np.ascontiguousarray(lk_H8(elem_size=1.0) if KE is None else KE)
        self.H, self.Hs = build_filter(nelx, nely, nelz, rmin)
        self.F = torch.as_tensor(np.atleast_2d(np.asarray(F, dtype=np.float64))).to(device()).contiguous()
        self.solid = to_flat_mask(protected_solid)
        self.void = to_flat_mask(protected_void)
        free = np.ones(self.shape, bool)
        if protected_solid is not None:
            free &= ~np.asarray(protected_solid, bool)
        if protected_void is not None:
            free &= ~np.asarray(protected_void, bool)
        self.free = to_flat_mask(free)
        self.solver = HexSolver(nelx, nely, nelz, self.KE, _fixed_dof_mask(nelx, nely, nelz, support_mask),
                                precision=precision, **(solver_options or {}))
        self.recompute = recompute
        n = self.nele
        mk = lambda: torch.empty(n, dtype=torch.float64, device=device())
        self.rho_f, self.rho_p, self.dproj = mk(), mk(), mk()
        self.dc, self.dv, self.dc_acc, self.ce = mk(), mk(), mk(), mk()
        self.c = torch.zeros(1, dtype=torch.float64, device=device())
        self.scratch = torch.empty(_lib.lib().tp3d_sensitivity_scratch_bytes(nelx, nely, nelz),
                                   dtype=torch.uint8, device=device())
        self.U = torch.zeros_like(self.F)

    def forward(self, x_flat: torch.Tensor, keep: bool = False):
        """Summed compliance of the flat design; with ``keep`` also the state the
        adjoint needs (physical density, projection derivative, one displacement
        field per load case) as fresh tensors owned by the caller."""
        project_flat(self.H, x_flat, self.Hs, self.beta, self.eta, self.solid, self.void, self.rho_f,
                     self.rho_p, self.dproj)
        self.solver.set_density(self.rho_p, self.penal)
        total = torch.zeros((), dtype=torch.float64, device=device())
        U = torch.zeros_like(self.F) if keep else self.U
        for k in range(self.F.shape[0]):
            U[k].zero_()
            self.solver.solve(self.F[k], U[k])
            total = total + torch.dot(self.F[k], U[k])
        state = (self.rho_p.clone(), self.dproj.clone(), U) if keep else None
        return total, state

    def gradient(self, x_flat: torch.Tensor, state=None) -> torch.Tensor:
        """d compliance / d x (flat): from the saved ``state`` of the forward pass,
        or with the displacements recomputed per load case when ``state`` is None."""
        L = _lib.lib()
        H = self.H
        if state is None:
            project_flat(self.H, x_flat, self.Hs, self.beta, self.eta, self.solid, self.void, self.rho_f,
                         self.rho_p, self.dproj)
            self.solver.set_density(self.rho_p, self.penal)
            rho_p, dproj, U = self.rho_p, self.dproj, self.U
        else:
            rho_p, dproj, U = state
        out = torch.zeros(self.nele, dtype=torch.float64, device=device())
        for k in range(self.F.shape[0]):
            if state is None:
                U[k].zero_()
                self.solver.solve(self.F[k], U[k])
            _lib.check(L.tp3d_sensitivity(
                H.nelx, H.nely, H.nelz, H.rmin, U[k].data_ptr(), self.KE.ctypes.data,
                rho_p.data_ptr(), dproj.data_ptr(), self.Hs.data_ptr(), self.free.data_ptr(),
                self.penal, self.ce.data_ptr(), self.dc.data_ptr(), self.dv.data_ptr(), self.c.data_ptr(),
                self.scratch.data_ptr(), _lib.stream_ptr()), "sensitivity")
            out += self.dc
        return out

    def close(self):
        self.solver.close()


class _Compliance(torch.autograd.Function):
    """The forward pass's state lives on ``ctx``: with ``recompute=False`` each
    call saves its own physical density, projection derivative and
    displacements, so several forwards before their backwards each get the
    gradient of their own design.  With ``recompute=True`` only the design is
    saved and backward re-solves every load case."""

    @staticmethod
    def forward(ctx, rho_design: torch.Tensor, problem: ComplianceProblem):
        x = rho_design.detach()
        shape = tuple(x.shape)
        xf = x.permute(2, 1, 0).contiguous().reshape(-1) if x.dim() == 3 else x.contiguous()
        xf = xf.to(torch.float64)
        c, state = problem.forward(xf, keep=not problem.recompute)
        ctx.problem, ctx.shape, ctx.dim = problem, shape, x.dim()
        if state is None:
            ctx.save_for_backward(xf)
        else:
            ctx.save_for_backward(xf, *state)
        return c.to(rho_design.dtype)

    @staticmethod
    def backward(ctx, grad_out):
        saved = ctx.saved_tensors
        state = None if len(saved) == 1 else tuple(saved[1:])
        g = ctx.problem.gradient(saved[0], state) * grad_out.to(torch.float64)
        if ctx.dim == 3:
            g = from_flat(g, ctx.shape)
        return g, None


def compliance(rho_design: torch.Tensor, problem: ComplianceProblem) -> torch.Tensor:
    """Summed compliance of ``rho_design`` ((nely, nelx, nelz) or flat Fortran order)."""
    return _Compliance.apply(rho_design, problem)
