"""Summed compliance of several load cases as a torch.autograd.Function.

Mirrors the differentiation workload: a cantilever with three load cases
(-z edge load at x = nelx, z = 0; +y edge load at x = nelx, z = nelz; -z
point load at the centre of face x = nelx), design densities uniform in
[0.05, 1] from a seed, filter radius 2.5, Heaviside beta 4, eta 0.5, the
displacements recomputed per load case in backward.  The gradient is checked

* against the oracle's restatement of the reference sensitivities
  (optimizer.py:596-625: element energies, SIMP derivative, projection and
  filter chain rule, with spsolve displacements) at 1e-8 relative, and
* against FP64 central finite differences (h = 1e-6) of the compliance on
  random elements at 1e-5 relative (the FD error at this h and a 1e-12
  solve).

The grid is 24x12x12 (the workload's 48x24x24 takes minutes in the oracle's
direct solve); the FD check uses the B200 FP64 solver, as the reference's own
gradient test does with its solver (tests/test_projected_optimizer.py:83-125).
"""

import numpy as np
import pytest
import torch

from oracle import simp_oracle as O

pytestmark = pytest.mark.gpu

NX, NY, NZ = 24, 12, 12
RMIN, BETA, ETA, PENAL = 2.5, 4.0, 0.5, 3.0


def _nid(ix, iy, iz):
    return iy + (NY + 1) * (ix + (NX + 1) * iz)


def _load_cases():
    ndof = 3 * (NX + 1) * (NY + 1) * (NZ + 1)
    F = np.zeros((3, ndof))
    for iy in range(NY + 1):
        F[0, 3 * _nid(NX, iy, 0) + 2] = -1.0 / (NY + 1)      # -z edge load at x = nelx, z = 0
        F[1, 3 * _nid(NX, iy, NZ) + 1] = 1.0 / (NY + 1)      # +y edge load at x = nelx, z = nelz
    F[2, 3 * _nid(NX, NY // 2, NZ // 2) + 2] = -1.0          # -z point load, centre of face x = nelx
    return F


@pytest.fixture(scope="module")
def setup():
    import pytopo3d_b200 as P
    from pytopo3d_b200 import _lib
    from pytopo3d_b200.autograd import ComplianceProblem

    _lib.lib()
    F = _load_cases()
    prob = ComplianceProblem(NX, NY, NZ, F, RMIN, BETA, eta=ETA, penal=PENAL, precision="fp64",
                             recompute=True, solver_options={"rtol": 1e-12, "max_iterations": 5000})
    rng = np.random.default_rng(5)
    x = rng.uniform(0.05, 1.0, size=(NY, NX, NZ))
    yield P, prob, F, x
    prob.close()


def test_gradient_matches_reference_sensitivities(setup):
    from pytopo3d_b200.autograd import compliance

    P, prob, F, x = setup
    xt = torch.tensor(x, device="cuda", requires_grad=True)
    c = compliance(xt, prob)
    c.backward()
    g = xt.grad.detach().cpu().numpy()

    # oracle: the reference's sensitivity chain with spsolve displacements
    ndof = F.shape[1]
    shape = (NY, NX, NZ)
    free = np.ones(shape, bool)
    none = np.zeros(shape, bool)
    H, Hs = O.build_filter(NX, NY, NZ, RMIN)
    _, rho, dproj = O.build_physical_density(x, H, Hs, BETA, ETA, none, none)
    freedofs, _ = O.build_supports(NX, NY, NZ, ndof)
    KE = O.lk_H8(elem_size=1.0)
    c_ref, dc_sum = 0.0, np.zeros(shape)
    for k in range(3):
        U, edof = O.solve_displacement(rho, KE, PENAL, F[k], freedofs, NX, NY, NZ)
        ck, _, dck = O.sensitivities(rho, U, edof, KE, PENAL)
        c_ref += ck
        dc_sum += dck
    g_ref = O.apply_density_filter_chain_rule(dc_sum, dproj, H, Hs)
    assert float(c.detach()) == pytest.approx(c_ref, rel=1e-9)
    np.testing.assert_allclose(g, g_ref, rtol=0, atol=1e-8 * np.abs(g_ref).max())
    assert free.all()


def test_gradient_matches_central_differences(setup):
    from pytopo3d_b200.autograd import compliance

    P, prob, F, x = setup
    xt = torch.tensor(x, device="cuda", requires_grad=True)
    compliance(xt, prob).backward()
    g = xt.grad.detach().cpu().numpy()
    rng = np.random.default_rng(11)
    h = 1e-6
    flat = rng.choice(x.size, size=20, replace=False)
    for f in flat:
        idx = np.unravel_index(f, x.shape)
        xp, xm = x.copy(), x.copy()
        xp[idx] += h
        xm[idx] -= h
        cp = float(compliance(torch.tensor(xp, device="cuda"), prob))
        cm = float(compliance(torch.tensor(xm, device="cuda"), prob))
        fd = (cp - cm) / (2 * h)
        assert g[idx] == pytest.approx(fd, rel=1e-5, abs=1e-7 * np.abs(g).max()), (idx, g[idx], fd)
