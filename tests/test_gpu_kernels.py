"""CUDA filter / projection / chain-rule / element-energy / OC kernels against the oracle
and the reference's golden vectors (FP64, tolerance 1e-12 unless stated)."""

import numpy as np
import pytest
import torch

from oracle import simp_oracle as O

pytestmark = pytest.mark.gpu

GRIDS = [(3, 2, 4, 1.6), (5, 4, 6, 2.5), (6, 5, 4, 3.0), (7, 6, 5, 4.5), (4, 3, 3, 1.5), (9, 33, 5, 0.9),
         (37, 3, 2, 1.0), (17, 40, 9, 2.2), (1, 1, 1, 3.0)]


@pytest.fixture(scope="module")
def P():
    import pytopo3d_b200 as P
    from pytopo3d_b200 import _lib

    _lib.lib()
    return P


@pytest.mark.parametrize("g", GRIDS)
def test_filter_rowsums_match_oracle(P, g):
    nx, ny, nz, r = g
    _, Hs = P.build_filter(nx, ny, nz, r)
    _, Hso = O.build_filter(nx, ny, nz, r)
    np.testing.assert_allclose(Hs.cpu().numpy(), Hso, rtol=1e-14, atol=0)


@pytest.mark.parametrize("g", GRIDS)
def test_filter_projection_and_transpose_match_oracle(P, g):
    nx, ny, nz, r = g
    rng = np.random.default_rng(nx * 100 + ny)
    shape = (ny, nx, nz)
    x = rng.uniform(size=shape)
    solid = rng.uniform(size=shape) < 0.15
    void = (rng.uniform(size=shape) < 0.15) & ~solid
    H, Hs = P.build_filter(nx, ny, nz, r)
    Ho, Hso = O.build_filter(nx, ny, nz, r)
    for beta in (1.0, 8.0):
        rf, rp, dp = P.build_physical_density(x, H, Hs, beta, 0.5, solid, void)
        rfo, rpo, dpo = O.build_physical_density(x, Ho, Hso, beta, 0.5, solid, void)
        np.testing.assert_allclose(rf, rfo, rtol=1e-13, atol=1e-14)
        np.testing.assert_allclose(rp, rpo, rtol=1e-12, atol=1e-13)
        np.testing.assert_allclose(dp, dpo, rtol=1e-12, atol=1e-13)
        gph = rng.normal(size=shape)
        out = P.apply_density_filter_chain_rule(gph, dp, H, Hs)
        np.testing.assert_allclose(out, O.apply_density_filter_chain_rule(gph, dpo, Ho, Hso), rtol=1e-12,
                                   atol=1e-13 * np.abs(gph).max())


def test_projection_matches_golden(P, golden):
    nx, ny, nz, r = golden["bpd_dims"]
    H, Hs = P.build_filter(int(nx), int(ny), int(nz), float(r))
    x, solid, void = golden["bpd_x"], golden["bpd_solid"], golden["bpd_void"]
    for beta in (1.0, 4.0, 8.0):
        rf, rp, dp = P.build_physical_density(x, H, Hs, beta, 0.5, solid, void)
        np.testing.assert_allclose(rf, golden[f"bpd_rf_b{beta}"], rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(rp, golden[f"bpd_rp_b{beta}"], rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(dp, golden[f"bpd_dp_b{beta}"], rtol=1e-12, atol=1e-14)
        out = P.apply_density_filter_chain_rule(golden[f"chain_g_b{beta}"], dp, H, Hs)
        np.testing.assert_allclose(out, golden[f"chain_out_b{beta}"], rtol=1e-12, atol=1e-14)
    out, der = P.heaviside_projection(golden["hv_rho"], 6.0, 0.4)
    np.testing.assert_allclose(out, golden["hv_out"], rtol=1e-14, atol=1e-15)
    np.testing.assert_allclose(der, golden["hv_der"], rtol=1e-14, atol=1e-15)


def test_projection_derivative_matches_central_difference(P):
    # mirrors the reference's tests/test_projection.py:14-30
    rho = np.linspace(0.01, 0.99, 50)
    _, d = P.heaviside_projection(rho, beta=8.0, eta=0.5)
    up, _ = P.heaviside_projection(rho + 1e-7, 8.0, 0.5)
    lo, _ = P.heaviside_projection(rho - 1e-7, 8.0, 0.5)
    np.testing.assert_allclose(d, (up - lo) / 2e-7, rtol=1e-5, atol=1e-7)


@pytest.mark.parametrize("beta,eta", [(0.0, 0.5), (-1.0, 0.5), (np.nan, 0.5), (np.inf, 0.5), (1.0, 0.0),
                                      (1.0, 1.0)])
def test_projection_rejects_invalid_parameters(P, beta, eta):
    with pytest.raises(ValueError):
        P.heaviside_projection(np.array([0.5]), beta=beta, eta=eta)


def test_chain_rule_matches_finite_difference(P):
    # the reference's transpose test (tests/test_projection.py:119-184) with a cone filter
    nx, ny, nz = 3, 2, 2
    shape = (ny, nx, nz)
    rng = np.random.default_rng(3)
    x = rng.uniform(0.2, 0.8, size=shape)
    w = rng.normal(size=shape)
    H, Hs = P.build_filter(nx, ny, nz, 1.5)
    fixed = np.zeros(shape, bool)

    def obj(c):
        return float(np.sum(w * P.build_physical_density(c, H, Hs, 3.0, 0.5, fixed, fixed)[1]))

    _, _, dp = P.build_physical_density(x, H, Hs, 3.0, 0.5, fixed, fixed)
    an = P.apply_density_filter_chain_rule(w, dp, H, Hs).ravel(order="F")
    fd = np.empty(x.size)
    for i in range(x.size):
        u, l = x.ravel(order="F").copy(), x.ravel(order="F").copy()
        u[i] += 1e-7
        l[i] -= 1e-7
        fd[i] = (obj(u.reshape(shape, order="F")) - obj(l.reshape(shape, order="F"))) / 2e-7
    np.testing.assert_allclose(an, fd, rtol=1e-6, atol=1e-8)


def test_element_compliance_matches_golden(P, golden):
    edof = P.build_edof(4, 3, 2)[0]
    ce = P.element_compliance(golden["ce_U"], edof, golden["KE_default_h1"])
    np.testing.assert_allclose(ce, golden["ce_out"], rtol=1e-13)


def test_fused_sensitivity_matches_oracle(P):
    from pytopo3d_b200 import _lib
    from pytopo3d_b200._tensors import to_flat, to_flat_mask, from_flat

    nx, ny, nz, r, penal = 9, 5, 4, 2.5, 3.0
    shape = (ny, nx, nz)
    rng = np.random.default_rng(5)
    rho = rng.uniform(0.0, 1.0, size=shape)
    dp = rng.uniform(0.0, 2.0, size=shape)
    free = rng.uniform(size=shape) < 0.8
    U = rng.normal(size=3 * (nx + 1) * (ny + 1) * (nz + 1))
    KE = P.lk_H8(elem_size=1.0)
    H, Hs = P.build_filter(nx, ny, nz, r)
    Ho, Hso = O.build_filter(nx, ny, nz, r)
    c, ce, dc = O.sensitivities(rho, U, O.build_edof(nx, ny, nz), KE, penal)
    dc_o = O.apply_density_filter_chain_rule(dc, dp, Ho, Hso)
    dv_o = O.apply_density_filter_chain_rule(free.astype(float), dp, Ho, Hso)
    n = nx * ny * nz
    out = {k: torch.empty(n, dtype=torch.float64, device="cuda") for k in ("ce", "dc", "dv")}
    comp = torch.zeros(1, dtype=torch.float64, device="cuda")
    scratch = torch.empty(_lib.lib().tp3d_sensitivity_scratch_bytes(nx, ny, nz), dtype=torch.uint8,
                          device="cuda")
    Ud, rd, dpd, fd = torch.as_tensor(U).cuda(), to_flat(rho), to_flat(dp), to_flat_mask(free)
    rc = _lib.lib().tp3d_sensitivity(nx, ny, nz, r, Ud.data_ptr(), KE.ctypes.data, rd.data_ptr(),
                                     dpd.data_ptr(), Hs.data_ptr(), fd.data_ptr(), penal,
                                     out["ce"].data_ptr(), out["dc"].data_ptr(), out["dv"].data_ptr(),
                                     comp.data_ptr(), scratch.data_ptr(), _lib.stream_ptr())
    assert rc == 0
    np.testing.assert_allclose(from_flat(out["ce"], shape).cpu().numpy(), ce, rtol=1e-12)
    assert float(comp) == pytest.approx(c, rel=1e-12)
    np.testing.assert_allclose(from_flat(out["dc"], shape).cpu().numpy(), dc_o, rtol=1e-11,
                               atol=1e-13 * np.abs(dc_o).max())
    np.testing.assert_allclose(from_flat(out["dv"], shape).cpu().numpy(), dv_o, rtol=1e-12, atol=1e-14)


def test_oc_update_matches_golden(P, golden):
    nx, ny, nz, r = golden["oc_dims"]
    H, Hs = P.build_filter(int(nx), int(ny), int(nz), float(r))
    solid, void = golden["oc_solid"], golden["oc_void"]
    free = ~(solid | void)
    bx, brho = P.optimality_criteria_update_projected(golden["oc_x"], golden["oc_dc_dx"], golden["oc_dv_dx"],
                                                      0.2, float(golden["oc_target"]), H, Hs, 2.0, 0.5, free,
                                                      solid, void)
    np.testing.assert_allclose(bx, golden["oc_best_x"], rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(brho, golden["oc_best_rho"], rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("tag", ["8x4x4", "32x16x16"])
def test_oc_update_on_reference_iteration(P, golden, tag):
    nx, ny, nz, volfrac, penal, rmin, beta, eta, move, _ = golden[f"it{tag}_dims"]
    nx, ny, nz = int(nx), int(ny), int(nz)
    solid, void = golden[f"it{tag}_solid"], golden[f"it{tag}_void"]
    H, Hs = P.build_filter(nx, ny, nz, rmin)
    bx, brho = P.optimality_criteria_update_projected(golden[f"it{tag}_x"], golden[f"it{tag}_dc_dx"],
                                                      golden[f"it{tag}_dv_dx"], move,
                                                      float(golden[f"it{tag}_target"]), H, Hs, beta, eta,
                                                      ~(solid | void), solid, void)
    np.testing.assert_allclose(bx, golden[f"it{tag}_x_new"], rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(brho, golden[f"it{tag}_rho_new"], rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("scale", (1.0, 1.0e-18, 1.0e18))
def test_oc_preserves_free_volume_and_fixed_regions(P, scale):
    # reference tests/test_projection.py:213-272; rmin 0.9 keeps only the centre tap (H = 0.9 I)
    shape = (1, 6, 1)
    x = np.full(shape, 0.5)
    solid = np.zeros(shape, bool)
    void = np.zeros(shape, bool)
    solid[0, 0, 0] = True
    void[0, -1, 0] = True
    free = ~(solid | void)
    x[solid], x[void] = 1.0, 0.0
    H, Hs = P.build_filter(6, 1, 1, 0.9)
    _, _, dp = P.build_physical_density(x, H, Hs, 4.0, 0.5, solid, void)
    dc = P.apply_density_filter_chain_rule(-scale * np.ones(shape), dp, H, Hs)
    dv = P.apply_density_filter_chain_rule(free.astype(float), dp, H, Hs)
    xn, rn = P.optimality_criteria_update_projected(x, dc, dv, 0.2, 0.4 * int(free.sum()), H, Hs, 4.0, 0.5,
                                                    free, solid, void)
    assert xn[solid].item() == 1.0 and xn[void].item() == 0.0
    assert rn[solid].item() == 1.0 and rn[void].item() == 0.0
    assert np.mean(rn[free]) == pytest.approx(0.4, abs=1e-7)


def test_oc_rejects_bad_arguments(P):
    H, Hs = P.build_filter(2, 2, 2, 1.5)
    z = np.zeros((2, 2, 2))
    m = np.zeros((2, 2, 2), bool)
    with pytest.raises(ValueError):
        P.optimality_criteria_update_projected(z, z, z, 0.0, 1.0, H, Hs, 1.0, 0.5, ~m, m, m)
    with pytest.raises(ValueError):
        P.optimality_criteria_update_projected(z, z, z, 0.2, 1.0, H, Hs, 1.0, 0.5, ~m, m, m,
                                               max_bisection_iterations=0)


def _oracle_bisection(tag_inputs, max_iter, tol):
    """(steps, best lambda, final lo, final hi) of the reference bisection, replayed from the oracle trace."""
    x, dc, dv, move, target, H, Hs, beta, eta, free, solid, void = tag_inputs
    trace = []
    O.oc_update_projected(x, dc, dv, move, target, H, Hs, beta, eta, free, solid, void,
                          max_bisection_iterations=max_iter, bisection_tolerance=tol, trace=trace)
    lo, hi, best, best_err = 0.0, 1.0e12, None, float("inf")
    for lam, vol in trace:
        err = abs(vol - target)
        if err < best_err:
            best, best_err = lam, err
        if vol > target:
            lo = lam
        else:
            hi = lam
    return len(trace), best, lo, hi


@pytest.mark.parametrize("tag", ["8x4x4", "32x16x16"])
@pytest.mark.parametrize("max_iter,tol", [(80, 1e-8), (30, 1e-8), (12, 1e-8), (80, 1e-3), (80, 1.5)])
def test_oc_bisection_path_matches_reference(P, golden, tag, max_iter, tol):
    # the multiplier sequence is exact binary fractions of 1e12: same path, same numbers
    from pytopo3d_b200.oc_update import OCWorkspace, oc_update_flat
    from pytopo3d_b200._tensors import to_flat, to_flat_mask, vec

    nx, ny, nz, volfrac, penal, rmin, beta, eta, move, _ = golden[f"it{tag}_dims"]
    nx, ny, nz = int(nx), int(ny), int(nz)
    solid, void = golden[f"it{tag}_solid"], golden[f"it{tag}_void"]
    x, dc, dv = golden[f"it{tag}_x"], golden[f"it{tag}_dc_dx"], golden[f"it{tag}_dv_dx"]
    target = float(golden[f"it{tag}_target"])
    Ho, Hso = O.build_filter(nx, ny, nz, rmin)
    steps, best, lo, hi = _oracle_bisection((x, dc, dv, move, target, Ho, Hso, beta, eta, ~(solid | void), solid,
                                             void), max_iter, tol)
    H, Hs = P.build_filter(nx, ny, nz, rmin)
    xf = to_flat(x)
    xn, rn = torch.empty_like(xf), torch.empty_like(xf)
    st = oc_update_flat(H, xf, to_flat(dc), to_flat(dv), vec(Hs), to_flat_mask(solid), to_flat_mask(void), move,
                        target, beta, eta, xn, rn, OCWorkspace(H), max_iter, tol).cpu().numpy()
    assert int(st[2]) == steps
    assert st[0] == best and st[5] == lo and st[6] == hi


@pytest.mark.parametrize("max_iter", [39, 40, 80])
def test_oc_bisection_ties_keep_the_first_step(P, max_iter):
    """A volume plateau: every free design value is 0.5 and the move limit 0.2,
    so for every multiplier above about 2.8 each candidate sits at its lower
    move limit and the projected volume is the same.  With the target just
    above that volume, the reference's first 38 midpoints tie, and it keeps the
    FIRST of them (strict <, oc_update.py:106); the reported multiplier must be
    that one, with the same steps and final bracket."""
    from pytopo3d_b200.oc_update import OCWorkspace, oc_update_flat
    from pytopo3d_b200._tensors import to_flat, to_flat_mask, vec

    nx, ny, nz, rmin, beta, eta, move = 8, 5, 4, 2.0, 2.0, 0.5, 0.2
    shape = (ny, nx, nz)
    rng = np.random.default_rng(21)
    solid = np.zeros(shape, bool)
    solid[:, 0, :] = True
    void = np.zeros(shape, bool)
    void[2, 4, 1:3] = True
    free = ~(solid | void)
    x = np.full(shape, 0.5)
    x[solid], x[void] = 1.0, 0.0
    Ho, Hso = O.build_filter(nx, ny, nz, rmin)
    _, _, dp = O.build_physical_density(x, Ho, Hso, beta, eta, solid, void)
    dc = O.apply_density_filter_chain_rule(-np.abs(rng.normal(size=shape)), dp, Ho, Hso)
    dv = O.apply_density_filter_chain_rule(free.astype(float), dp, Ho, Hso)
    low = x.copy()
    low[free] = x[free] - move
    _, rho_low, _ = O.build_physical_density(low, Ho, Hso, beta, eta, solid, void)
    target = float(rho_low[free].sum()) + 1e-6
    steps, best, lo, hi = _oracle_bisection((x, dc, dv, move, target, Ho, Hso, beta, eta, free, solid, void),
                                            max_iter, 1e-8)
    H, Hs = P.build_filter(nx, ny, nz, rmin)
    xf = to_flat(x)
    xn, rn = torch.empty_like(xf), torch.empty_like(xf)
    st = oc_update_flat(H, xf, to_flat(dc), to_flat(dv), vec(Hs), to_flat_mask(solid), to_flat_mask(void), move,
                        target, beta, eta, xn, rn, OCWorkspace(H), max_iter, 1e-8).cpu().numpy()
    if max_iter == 39:
        assert best == 5.0e11  # the tie is real: the reference keeps step 1
    assert int(st[2]) == steps
    assert st[0] == best and st[5] == lo and st[6] == hi


def test_expired_barrier_wait_reaches_the_host(P, golden):
    """Every grid-barrier wait of the OC kernel is bounded.  The wait-expiry hook
    makes the barrier wait for a block that never arrives, with a short poll
    limit: the launch must end by itself, the drop-in must raise Topo3dError,
    and the context must stay usable (the same update then completes and
    matches the reference)."""
    from pytopo3d_b200 import _lib

    L = _lib.lib()
    nx, ny, nz, r = golden["oc_dims"]
    H, Hs = P.build_filter(int(nx), int(ny), int(nz), float(r))
    solid, void = golden["oc_solid"], golden["oc_void"]
    free = ~(solid | void)
    args = (golden["oc_x"], golden["oc_dc_dx"], golden["oc_dv_dx"], 0.2, float(golden["oc_target"]), H, Hs, 2.0,
            0.5, free, solid, void)
    assert L.tp3d_debug_expire_oc_waits(4096, 1) == 0
    try:
        with pytest.raises(_lib.Topo3dError, match="bounded device wait"):
            P.optimality_criteria_update_projected(*args)
    finally:
        assert L.tp3d_debug_expire_oc_waits(0, 0) == 0
    torch.cuda.synchronize()
    bx, brho = P.optimality_criteria_update_projected(*args)
    np.testing.assert_allclose(bx, golden["oc_best_x"], rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(brho, golden["oc_best_rho"], rtol=1e-12, atol=1e-13)
