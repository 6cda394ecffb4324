"""Summed compliance of several load cases as a torch.autograd.Function.

The differentiation workload at its full size: a 48x24x24 cantilever with
three load cases (-z edge load at x = nelx, z = 0; +y edge load at x = nelx,
z = nelz; -z point load at the centre of face x = nelx), design densities
uniform in [0.05, 1] from a seed, filter radius 2.5, Heaviside beta 4, eta 0.5.
The gradient is checked

* against the reference's own sensitivities: ``golden_sensitivities_48x24x24.npz``
  holds the summed compliance and d compliance / d x computed by the
  reference's functions with its direct solve (element energies, SIMP
  derivative, projection and filter chain rule: optimizer.py:584-625,
  filter.py:103-119), at 1e-8 of the largest entry;
* against FP64 central finite differences (h = 1e-6) of the compliance on 200
  random elements, with the B200 FP64 solver at a relative residual of 1e-13,
  as the reference's own gradient test does with its solver
  (tests/test_projected_optimizer.py:83-125), at 1e-5 relative (the FD error
  at this h);
* with the displacements recomputed per load case in backward
  (``recompute=True``) and kept on the autograd context (``recompute=False``,
  two forwards before their backwards).
"""

import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def gs():
    return np.load(os.path.join(ROOT, "golden", "golden_sensitivities_48x24x24.npz"))


@pytest.fixture(scope="module")
def setup(gs):
    from golden.make_golden import sensitivity_load_cases
    from pytopo3d_b200 import _lib
    from pytopo3d_b200.autograd import ComplianceProblem

    _lib.lib()
    nx, ny, nz = (int(v) for v in gs["dims"])
    rmin, beta, eta, penal, _ = gs["params"]
    F = sensitivity_load_cases(nx, ny, nz)
    opts = {"rtol": 1e-13, "max_iterations": 20000}
    probs = {rc: ComplianceProblem(nx, ny, nz, F, rmin, beta, eta=eta, penal=penal, precision="fp64",
                                   recompute=rc, solver_options=opts) for rc in (True, False)}
    yield probs, gs["x"]
    for p in probs.values():
        p.close()


@pytest.mark.parametrize("recompute", [True, False])
def test_gradient_matches_reference_sensitivities(setup, gs, recompute):
    from pytopo3d_b200.autograd import compliance

    probs, x = setup
    xt = torch.tensor(x, device="cuda", requires_grad=True)
    c = compliance(xt, probs[recompute])
    c.backward()
    g = xt.grad.detach().cpu().numpy()
    g_ref = gs["grad"]
    assert float(c.detach()) == pytest.approx(float(gs["c_cases"].sum()), rel=1e-9)
    err = np.abs(g - g_ref).max() / np.abs(g_ref).max()
    print(f"recompute={recompute}: gradient error {err:.2e} of max |g|")
    assert err <= 1e-8


def test_saved_state_belongs_to_each_forward(setup, gs):
    """recompute=False: two forwards, then their backwards in reverse order;
    each gradient is that of its own design."""
    from pytopo3d_b200.autograd import compliance

    probs, x = setup
    x2 = np.clip(x * 0.8 + 0.1, 0.05, 1.0)
    a = torch.tensor(x, device="cuda", requires_grad=True)
    b = torch.tensor(x2, device="cuda", requires_grad=True)
    ca = compliance(a, probs[False])
    cb = compliance(b, probs[False])
    cb.backward()
    ca.backward()
    ga, gb = a.grad.cpu().numpy(), b.grad.cpu().numpy()
    np.testing.assert_allclose(ga, gs["grad"], rtol=0, atol=1e-8 * np.abs(gs["grad"]).max())
    ref_b = torch.tensor(x2, device="cuda", requires_grad=True)
    compliance(ref_b, probs[True]).backward()
    np.testing.assert_allclose(gb, ref_b.grad.cpu().numpy(), rtol=0, atol=1e-10 * np.abs(gb).max())
    assert np.abs(ga - gb).max() > 1e-3 * np.abs(ga).max()


def test_gradient_matches_central_differences(setup, gs):
    from pytopo3d_b200.autograd import compliance

    probs, x = setup
    prob = probs[True]
    g = gs["grad"]
    rng = np.random.default_rng(11)
    h = 1e-6
    flat = rng.choice(x.size, size=200, replace=False)
    worst = 0.0
    for f in flat:
        idx = np.unravel_index(f, x.shape)
        xp, xm = x.copy(), x.copy()
        xp[idx] += h
        xm[idx] -= h
        cp = float(compliance(torch.tensor(xp, device="cuda"), prob))
        cm = float(compliance(torch.tensor(xm, device="cuda"), prob))
        fd = (cp - cm) / (2 * h)
        worst = max(worst, abs(g[idx] - fd) / max(abs(fd), 1e-2 * np.abs(g).max()))
        assert g[idx] == pytest.approx(fd, rel=1e-5, abs=1e-7 * np.abs(g).max()), (idx, g[idx], fd)
    print(f"worst FD mismatch {worst:.2e}")
