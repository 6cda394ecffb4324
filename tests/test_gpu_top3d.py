"""The B200 SIMP loop against the reference's loop body and full top3d runs.

Per-iteration parity from identical inputs (loop body of optimizer.py:584-642):
densities 1e-12, U 1e-8 of max|U| (solver rtol 1e-10 vs direct solve),
compliance 1e-9, new design 1e-8.  Whole runs: 1e-6 (OC decisions on a
trajectory amplify round-off).
"""

import numpy as np
import pytest
import torch

from oracle import simp_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def P():
    import pytopo3d_b200 as P
    from pytopo3d_b200 import _lib

    _lib.lib()
    return P


@pytest.mark.parametrize("tag", ["8x4x4", "32x16x16"])
def test_loop_body_matches_reference(P, golden, tag):
    from pytopo3d_b200._tensors import from_flat, to_flat, to_flat_mask
    from pytopo3d_b200.oc_update import oc_update_flat
    from pytopo3d_b200.optimizer import SimpState, _fixed_dof_mask
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz, volfrac, penal, rmin, beta, eta, move, _ = golden[f"it{tag}_dims"]
    nx, ny, nz = int(nx), int(ny), int(nz)
    shape = (ny, nx, nz)
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    x, solid, void = golden[f"it{tag}_x"], golden[f"it{tag}_solid"], golden[f"it{tag}_void"]
    free = ~(solid | void)
    KE = P.lk_H8(elem_size=1.0)
    H, Hs = P.build_filter(nx, ny, nz, rmin)
    sd, vd, fd = to_flat_mask(solid), to_flat_mask(void), to_flat_mask(free)
    solver = HexSolver(nx, ny, nz, KE, _fixed_dof_mask(nx, ny, nz, None))
    F = torch.as_tensor(O.build_force_vector(nx, ny, nz, ndof)[None]).cuda()
    S = SimpState(H, Hs, sd, vd, fd, KE, F, solver, penal)
    xd = to_flat(x)
    S.project(xd, beta, eta)
    np.testing.assert_allclose(from_flat(S.rho_p, shape).cpu().numpy(), golden[f"it{tag}_rho_p"], rtol=1e-12,
                               atol=1e-13)
    S.sensitivities(S.rho_p, S.dproj)
    Uref = golden[f"it{tag}_U"]
    np.testing.assert_allclose(S.U[0].cpu().numpy(), Uref, rtol=0, atol=1e-8 * np.abs(Uref).max())
    assert float(S.c_dev[0]) == pytest.approx(float(golden[f"it{tag}_c"]), rel=1e-9)
    dref = golden[f"it{tag}_dc_dx"]
    np.testing.assert_allclose(from_flat(S.dc_dx, shape).cpu().numpy(), dref, rtol=0,
                               atol=1e-8 * np.abs(dref).max())
    oc_update_flat(H, xd, S.dc_dx, S.dv_dx, Hs, sd, vd, move, float(golden[f"it{tag}_target"]), beta, eta,
                   S.x_new, S.rho_new, S.ws)
    np.testing.assert_allclose(from_flat(S.x_new, shape).cpu().numpy(), golden[f"it{tag}_x_new"], rtol=0,
                               atol=1e-8)
    np.testing.assert_allclose(from_flat(S.rho_new, shape).cpu().numpy(), golden[f"it{tag}_rho_new"], rtol=0,
                               atol=1e-8)
    solver.close()


def test_top3d_run_matches_reference(P, golden):
    diag = {}
    xphys, hist, comp, failure = P.top3d(nelx=6, nely=3, nelz=3, volfrac=0.4, penal=3.0, rmin=1.5,
                                         disp_thres=0.5, elem_size=1.0, tolx=0.01, maxloop=4,
                                         beta_schedule=(1.0, 2.0), save_history=True, history_frequency=1,
                                         diagnostics_out=diag)
    assert failure is None
    np.testing.assert_allclose(xphys, golden["top3d_xphys"], rtol=0, atol=1e-6)
    assert comp == pytest.approx(float(golden["top3d_compliance"]), rel=1e-6)
    np.testing.assert_allclose(hist["compliance_history"], golden["top3d_hist_c"], rtol=1e-6)
    # The thresholded design is nearly a mechanism (C ~ 3.4e10, carried by 1e-9
    # void material): its FP64 CG residual has an attainable floor, so the
    # iterative solve matches the reference's direct solve to ~1e-5 here.
    assert diag["binary_compliance"] == pytest.approx(float(golden["top3d_binary_compliance"]), rel=2e-5)
    assert diag["projection_total_iterations"] == int(golden["top3d_total_iterations"])


def test_top3d_matches_oracle_trajectory(P):
    rec = []
    x, rho, hist = O.top3d(12, 6, 6, 0.3, 3.0, 2.0, tolx=0.01, maxloop=6, beta_schedule=(1.0, 2.0))
    xphys, _, comp, _ = P.top3d(nelx=12, nely=6, nelz=6, volfrac=0.3, penal=3.0, rmin=2.0, disp_thres=0.5,
                                elem_size=1.0, tolx=0.01, maxloop=6, beta_schedule=(1.0, 2.0), record=rec)
    np.testing.assert_allclose([r["c"] for r in rec], hist, rtol=1e-7)
    np.testing.assert_allclose(xphys, rho, rtol=0, atol=1e-6)


def test_continuation_returns_one_physical_field_and_records_metrics(P):
    # mirrors tests/test_projected_optimizer.py:184-249 of the reference
    n = 2
    shape = (n, n, n)
    support = np.zeros(shape, bool)
    support[:, 0, :] = True
    ff = np.zeros(shape + (3,))
    ff[0, 1, 0, 0] = 1.0
    obstacle = np.zeros(shape, bool)
    obstacle[1, 1, 1] = True
    diag = {}
    rho, history, comp, _ = P.top3d(nelx=n, nely=n, nelz=n, volfrac=0.5, penal=3.0, rmin=1.0, disp_thres=0.5,
                                    force_field=ff, support_mask=support, obstacle_mask=obstacle, tolx=1e-12,
                                    maxloop=1, save_history=True, history_frequency=1, beta_schedule=(1.0, 2.0),
                                    diagnostics_out=diag)
    prot = support | np.any(ff != 0.0, axis=-1)
    assert np.all(rho[prot] == 1.0)
    assert rho[obstacle].item() == 0.0
    np.testing.assert_allclose(history["density_history"][-1], rho)
    assert history["iteration_history"] == [0, 1, 2]
    assert history["beta_history"] == [1.0, 2.0, 2.0]
    assert history["compliance_history"][-1] == pytest.approx(comp)
    for d, c in zip(history["density_history"], history["compliance_history"]):
        rc = P.evaluate_fixed_geometry_compliance(xPhys=d, penal=3.0, force_field=ff, support_mask=support,
                                                  obstacle_mask=obstacle)
        assert c == pytest.approx(rc, rel=1e-9)
    assert diag["projection_beta_schedule"] == [1.0, 2.0]
    assert diag["projection_total_iterations"] == 2
    assert diag["projection_converged"] is False
    for st in diag["projection_stage_summaries"]:
        assert st["volume_fraction_error"] == pytest.approx(0.0, abs=1e-7)
    assert diag["physical_density_fraction"] == pytest.approx(0.5, abs=1e-7)


def test_default_boundary_attachments_are_protected(P):
    nx, ny, nz = 3, 2, 2
    diag = {}
    rho, _, _, _ = P.top3d(nelx=nx, nely=ny, nelz=nz, volfrac=0.5, penal=3.0, rmin=1.5, disp_thres=0.5,
                           support_mask=np.zeros((ny, nx, nz), bool), maxloop=1, beta_schedule=(1.0,),
                           diagnostics_out=diag)
    assert np.all(rho[:, 0, :] == 1.0) and np.all(rho[:, -1, 0] == 1.0)
    st = diag["projection_stage_summaries"][0]
    assert st["minimum_achievable_physical_fraction"] > 0.0 and st["target_within_achievable_range"] is True
    assert diag["physical_density_fraction"] == pytest.approx(0.5, abs=1e-7)


def test_infeasible_target_is_reported_before_fea(P):
    with pytest.raises(ValueError, match="minimum achievable"):
        P.top3d(nelx=2, nely=2, nelz=2, volfrac=0.3, penal=3.0, rmin=1.5, disp_thres=0.5, maxloop=1,
                beta_schedule=(1.0,))


def test_symmetric_tensile_update_preserves_symmetry(P):
    nx, ny, nz = 4, 12, 2
    ff = P.build_force_field(nx, ny, nz, 0, nx, ny - 1, ny, 0, nz, 0.0, 1.0, 0.0)
    sm = P.build_support_mask(nx, ny, nz, 0, nx, 0, 1, 0, nz)
    prot = np.zeros((ny, nx, nz), bool)
    prot[:3] = True
    prot[-3:] = True
    rho, _, _, _ = P.top3d(nelx=nx, nely=ny, nelz=nz, volfrac=0.5, penal=3.0, rmin=2.0, disp_thres=0.5,
                           force_field=ff, support_mask=sm, protected_zone_mask=prot, tolx=1e-12, maxloop=1,
                           beta_schedule=(1.0,))
    f = rho[3:-3]
    np.testing.assert_allclose(f, f[::-1], rtol=0, atol=1e-3)


def test_fixed_geometry_metrics_match_reference(P, golden):
    m = P.evaluate_fixed_geometry_metrics(golden["top3d_xphys"], 3.0, elem_size=1.0)
    for k, v in m.items():
        ref = float(golden[f"metrics_{k}"])
        if v is None:
            assert np.isnan(ref), k
        else:
            assert v == pytest.approx(ref, rel=1e-8, abs=1e-8 * abs(m["uz_avg_load_patch"])), k


def test_mixed_precision_top3d_tracks_fp64(P):
    kw = dict(nelx=24, nely=12, nelz=12, volfrac=0.3, penal=3.0, rmin=2.0, disp_thres=0.5, elem_size=1.0,
              tolx=1e-9, maxloop=5, beta_schedule=(1.0,))
    r64, r32 = [], []
    x64, _, c64, _ = P.top3d(**kw, record=r64)
    x32, _, c32, _ = P.top3d(**kw, record=r32, precision="mixed")
    assert abs(r32[0]["c"] - r64[0]["c"]) <= 1e-6 * abs(r64[0]["c"])
    assert abs(c32 - c64) <= 1e-5 * abs(c64)


@pytest.mark.parametrize("precision,opts", [("fp64", {}), ("mixed", {}),
                                            ("mixed", {"max_iterations": 16, "rtol": 1e-5})])
def test_stage_graph_matches_host_path(P, precision, opts):
    """Each projection stage as one CUDA graph launch (the loop condition
    decided on the device) reproduces the host-driven loop bit for bit (FP64
    and mixed: measured 23 of 24 iterations in graphs, the first on the host
    path).  With an iteration cap of 16 every mixed solve stops short, the graph
    hands each such iteration back, and the host path finishes it with its FP64
    fallback: the trajectory is still the host path's, bit for bit."""
    kw = dict(nelx=16, nely=8, nelz=8, volfrac=0.3, penal=3.0, rmin=1.5, disp_thres=0.5, elem_size=1.0,
              tolx=0.01, maxloop=8, beta_schedule=(1.0, 2.0, 4.0), precision=precision, solver_options=opts)
    r_host, r_graph, d_host, d_graph = [], [], {}, {}
    x_host, _, c_host, _ = P.top3d(**kw, record=r_host, diagnostics_out=d_host)
    x_graph, _, c_graph, _ = P.top3d(**kw, record=r_graph, diagnostics_out=d_graph, stage_graph=True)
    n_graph = sum(1 for r in r_graph if r.get("stage_graph"))
    print(f"{precision} {opts}: {n_graph} of {len(r_graph)} iterations in stage graphs")
    assert [r["c"] for r in r_graph] == [r["c"] for r in r_host]
    assert [r["change"] for r in r_graph] == [r["change"] for r in r_host]
    assert [r["lam"] for r in r_graph] == [r["lam"] for r in r_host]
    assert [r["cg_iterations"] for r in r_graph] == [r["cg_iterations"] for r in r_host]
    np.testing.assert_array_equal(x_graph, x_host)
    assert c_graph == c_host
    assert d_graph["projection_total_iterations"] == d_host["projection_total_iterations"]
    if opts:
        assert any(not r.get("stage_graph") for r in r_graph[1:])  # handed back to the host path
    else:
        assert n_graph >= len(r_graph) - 3  # all but the run's first body and rare hand-backs


@pytest.fixture(scope="module")
def cantilever_run(P):
    """The 32x16x16 cantilever in full (beta 1, 2, 4, 8; maxloop 200 per stage;
    tolx 0.01; volfrac 0.3; penal 3; rmin 3; the reference's default load and
    supports) with the FP64 solver at a relative residual of 1e-12."""
    import os

    from pytopo3d_b200._tensors import from_flat

    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                             "golden_cantilever_32x16x16.npz"))
    rec, diag = [], {}
    xphys, hist, comp, failure = P.top3d(nelx=32, nely=16, nelz=16, volfrac=0.3, penal=3.0, rmin=3.0,
                                         disp_thres=0.5, elem_size=1.0, tolx=0.01, maxloop=200,
                                         beta_schedule=(1.0, 2.0, 4.0, 8.0), save_history=True,
                                         history_frequency=1, diagnostics_out=diag, record=rec,
                                         solver_options={"rtol": 1e-12, "max_iterations": 20000})
    shape = (16, 32, 16)
    x = [from_flat(e["x"], shape).cpu().numpy() for e in rec]
    return g, dict(xphys=xphys, hist=hist, comp=comp, failure=failure, diag=diag, rec=rec, x=x)


def test_cantilever_full_run_matches_reference(cantilever_run):
    """The whole 800-iteration run against the reference's own run of the same
    problem (``golden_cantilever_32x16x16.npz``, recorded by
    tests/golden/make_golden.py from pytopo3d/core/optimizer.py:537-836 with
    its direct solve): the same stage lengths and stopping, the first ten
    designs, the design at the end of every stage, the compliance of every
    iteration, the final physical density and compliance, and the stage
    diagnostics.  The B200 solves iteratively (FP64 CG to relres 1e-12) and
    sums the filter and the volume in another order, so the runs start
    1e-12 apart and the OC bisection carries the difference along the
    trajectory.  Measured on a B200: first ten designs 1.1e-11, stage-end
    designs 1.6e-9 / 9.1e-9 / 6.4e-9 / 2.2e-8, compliance of every iteration
    7.8e-10 relative (9.5e-12 over the first ten), change 4.2e-8, final
    physical density 2.9e-9, final compliance 1.3e-10; the bounds are about
    ten times those (the test prints them)."""
    g, r = cantilever_run
    diag, rec, hist = r["diag"], r["rec"], r["hist"]
    assert r["failure"] is None
    st = diag["projection_stage_summaries"]
    np.testing.assert_array_equal([s["iterations"] for s in st], g["cl_stage_iterations"])
    assert diag["projection_total_iterations"] == int(g["cl_total_iterations"]) == len(rec)
    err_first = np.abs(np.stack(r["x"][:10]) - g["cl_first_x"]).max()
    ends = np.cumsum(g["cl_stage_iterations"]) - 1
    err_ends = [float(np.abs(r["x"][i] - g["cl_stage_end_x"][k]).max()) for k, i in enumerate(ends)]
    c = np.array(hist["compliance_history"])
    c_ref = g["cl_hist_c"]
    assert c.shape == c_ref.shape
    err_c = np.abs(c / c_ref - 1.0)
    err_change = np.abs(np.array([e["change"] for e in rec]) - g["cl_change"])
    err_xphys = np.abs(r["xphys"] - g["cl_xphys"]).max()
    err_comp = abs(r["comp"] / float(g["cl_compliance"]) - 1.0)
    print(f"first 10 designs {err_first:.2e}; stage-end designs {['%.2e' % e for e in err_ends]}; "
          f"compliance per iteration: first 10 {err_c[:10].max():.2e}, stage 1 {err_c[:200].max():.2e}, "
          f"all {err_c.max():.2e}; change {err_change.max():.2e}; xphys {err_xphys:.2e}; "
          f"final compliance {err_comp:.2e}")
    assert err_first <= 1e-10
    assert err_c[:10].max() <= 1e-10
    assert err_c.max() <= 1e-8
    assert max(err_ends) <= 3e-7
    assert err_change.max() <= 5e-7
    assert err_xphys <= 3e-8
    assert err_comp <= 2e-9
    np.testing.assert_allclose([s["physical_density_fraction"] for s in st], g["cl_stage_vol"], atol=1e-10)
    # a count of elements: at most one element's density may sit on 0.05 or 0.95 differently
    np.testing.assert_allclose([s["gray_fraction_005_095"] for s in st], g["cl_stage_gray"], atol=1.0 / 8192)
    np.testing.assert_allclose([s["minimum_achievable_physical_fraction"] for s in st], g["cl_stage_vmin"],
                               atol=1e-8)
    np.testing.assert_allclose([s["maximum_achievable_physical_fraction"] for s in st], g["cl_stage_vmax"],
                               atol=1e-12)
    np.testing.assert_allclose([s["final_change"] for s in st], g["cl_stage_final_change"], atol=5e-7)
    assert diag["binary_compliance"] == pytest.approx(float(g["cl_binary_compliance"]), rel=1e-6)


def test_step_host_matches_device_loop(P):
    """SimpLoop.step_host (host design in, host design and compliance out, the
    path bench.py's end-to-end figure times) gives the device loop's trajectory
    bit for bit, for flat and (nely, nelx, nelz) host designs."""
    import bench
    from pytopo3d_b200.optimizer import SimpLoop

    nelx, nely, nelz = 24, 12, 12
    shape, solid, void, F, fixed = bench.workload(nelx, nely, nelz)
    loops = [SimpLoop(nelx, nely, nelz, 0.3, 3.0, 2.0, P.lk_H8(elem_size=1.0), F, fixed, solid, void,
                      precision="fp64") for _ in range(2)]
    for lp in loops:
        lp.set_beta(1.0)
    x_host = loops[1].design().permute(2, 1, 0).contiguous().reshape(-1).cpu().numpy()
    for it in range(4):
        st = loops[0].step()
        if it % 2 == 0:
            x_host, c = loops[1].step_host(x_host)
        else:  # the 3D layout of the reference's arrays
            x3 = x_host.reshape(nelz, nelx, nely).transpose(2, 1, 0)
            x_host, c = loops[1].step_host(x3)
        assert c == float(st[0])
        ref = loops[0].design().permute(2, 1, 0).contiguous().reshape(-1).cpu().numpy()
        assert np.array_equal(x_host, ref)
    for lp in loops:
        lp.close()
