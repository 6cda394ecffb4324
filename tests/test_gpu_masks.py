"""Obstacle masks on the device and top3d runs through every mask path, against the reference.

* The obstacle-mask kernel (tp3d_obstacle_mask) against the reference's own
  cube, sphere and cylinder masks and a JSON obstacle list
  (pytopo3d/utils/obstacles.py:12-269): bit for bit.
* top3d (FP64) on the three recorded mask runs of ``golden_masks.npz``
  (obstacle cylinder + force field + partial supports + protected zone; empty
  support mask + default load strip + overlapping obstacle; the 128x64x64
  workload's masks at 32x16x16): the per-iteration designs and physical
  densities within 1e-11 (measured: 2e-12 at most), compliances within 1e-10
  relative (measured: 3e-12), the same stage iteration counts and the same
  stage diagnostics.  The reference solves
  directly; the B200 solves iteratively to a relative residual of 1e-12.
"""

import json
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def gm():
    return np.load(os.path.join(ROOT, "golden", "golden_masks.npz"))


@pytest.fixture(scope="module")
def P():
    import pytopo3d_b200 as P
    from pytopo3d_b200 import _lib

    _lib.lib()
    return P


def test_primitives_match_reference(P, gm):
    from pytopo3d_b200 import obstacles as ob
    from test_masks_golden import PRIMITIVES

    for key, (kind, shape, args) in PRIMITIVES.items():
        fn = {"cube": ob.create_cube_obstacle, "sphere": ob.create_sphere_obstacle,
              "cylinder": ob.create_cylinder_obstacle}[kind]
        m = fn(shape, *args)
        assert m.dtype == bool and m.shape == shape
        np.testing.assert_array_equal(m, gm[key], err_msg=key)


def test_obstacle_config_file_matches_reference(P, gm, tmp_path):
    from pytopo3d_b200 import obstacles as ob

    f = tmp_path / "obstacles.json"
    f.write_text(str(gm["prim_config_json"]))
    np.testing.assert_array_equal(ob.parse_obstacle_config_file(str(f), (16, 24, 12)), gm["prim_config_mask"])
    cfg = json.loads(str(gm["prim_config_json"]))["obstacles"]
    with pytest.raises(ValueError, match="Unknown obstacle type"):
        ob.create_obstacle_from_config((4, 4, 4), {"type": "torus"})
    m = ob.create_obstacle_from_config((16, 24, 12), cfg[1])
    assert m.any() and not m.all()


def test_cylinders_of_the_golden_set(P, golden):
    from pytopo3d_b200.obstacles import create_cylinder_obstacle

    np.testing.assert_array_equal(create_cylinder_obstacle((16, 32, 16), (0.5, 0.5, 0.5), 0.25, 1.0, 1),
                                  golden["cyl_y"])
    np.testing.assert_array_equal(create_cylinder_obstacle((10, 12, 14), (0.3, 0.6, 0.5), 0.3, 0.5, 0),
                                  golden["cyl_x"])


def test_long_obstacle_lists_and_flat_layout(P):
    """More primitives than one launch takes (chunks OR-ed together), on a grid
    whose element count is not a multiple of 16, in the kernels' flat order."""
    from test_host_setup import primitive_mask
    from pytopo3d_b200 import obstacles as ob
    from pytopo3d_b200._tensors import from_flat

    shape = (13, 27, 11)
    rng = np.random.default_rng(3)
    prims = []
    for i in range(75):
        c = rng.uniform(0, 1, 3)
        k = i % 3
        if k == 0:
            prims.append(ob.cube_params(shape, c, tuple(rng.uniform(0.05, 0.3, 3))))
        elif k == 1:
            prims.append(ob.sphere_params(shape, c, rng.uniform(0.05, 0.2)))
        else:
            prims.append(ob.cylinder_params(shape, c, rng.uniform(0.05, 0.2), rng.uniform(0.2, 1.0),
                                            int(rng.integers(0, 3))))
    want = np.zeros(shape, bool)
    for o in prims:
        want |= primitive_mask(shape, o)
    flat = ob.obstacle_mask_flat(shape, prims)
    assert flat.dtype == torch.uint8 and flat.numel() == np.prod(shape)
    np.testing.assert_array_equal(from_flat(flat, shape).cpu().numpy().astype(bool), want)
    # an empty list clears the mask
    np.testing.assert_array_equal(ob.obstacle_mask_flat(shape, [], out=flat).cpu().numpy(), 0)


RUNS = {
    "m1": dict(nelx=10, nely=6, nelz=5, volfrac=0.35, rmin=1.5, maxloop=3, beta_schedule=(1.0, 2.0),
               inputs=dict(obstacle_mask="m1_obstacle", force_field="m1_force_field", support_mask="m1_support",
                           protected_zone_mask="m1_zone")),
    "m2": dict(nelx=8, nely=4, nelz=4, volfrac=0.3, rmin=1.5, maxloop=3, beta_schedule=(1.0, 4.0),
               inputs=dict(obstacle_mask="m2_obstacle", support_mask="empty")),
    "m3": dict(nelx=32, nely=16, nelz=16, volfrac=0.3, rmin=3.0, maxloop=3, beta_schedule=(1.0,),
               inputs=dict(obstacle_mask="m3_obstacle", protected_zone_mask="m3_zone")),
}


@pytest.mark.parametrize("tag", sorted(RUNS))
def test_top3d_mask_paths_match_reference(P, gm, tag):
    r = RUNS[tag]
    kw = {k: v for k, v in r.items() if k != "inputs"}
    shape = (r["nely"], r["nelx"], r["nelz"])
    for name, key in r["inputs"].items():
        kw[name] = np.zeros(shape, bool) if key == "empty" else gm[key]
    rec, diag = [], {}
    xphys, hist, comp, _ = P.top3d(penal=3.0, disp_thres=0.5, elem_size=1.0, tolx=0.01, save_history=True,
                                   history_frequency=1, diagnostics_out=diag, record=rec,
                                   solver_options={"rtol": 1e-12, "max_iterations": 20000}, **kw)
    n = len(gm[f"{tag}_change"])
    assert len(rec) == n
    np.testing.assert_array_equal([s["iterations"] for s in diag["projection_stage_summaries"]],
                                  gm[f"{tag}_stage_iterations"])
    x_ref = gm[f"{tag}_x_new"]
    from pytopo3d_b200._tensors import from_flat

    x_b200 = np.stack([from_flat(e["x"], shape).cpu().numpy() for e in rec])
    err_x = np.abs(x_b200 - x_ref).max()
    err_rho = np.abs(np.stack(hist["density_history"]) - gm[f"{tag}_hist_rho"]).max()
    c_ref = gm[f"{tag}_hist_c"]
    err_c = np.abs(np.array(hist["compliance_history"][:-1]) / c_ref[:-1] - 1.0).max()
    print(f"{tag}: max |x - x_ref| {err_x:.2e}, max |rho - rho_ref| {err_rho:.2e}, "
          f"max rel compliance error {err_c:.2e}")
    assert err_x <= 1e-11 and err_rho <= 1e-11 and err_c <= 1e-10
    np.testing.assert_allclose([e["change"] for e in rec], gm[f"{tag}_change"], rtol=0, atol=1e-10)
    np.testing.assert_allclose(xphys, gm[f"{tag}_xphys"], rtol=0, atol=1e-10)
    assert comp == pytest.approx(float(gm[f"{tag}_compliance"]), rel=1e-8)
    assert diag["projection_total_iterations"] == int(gm[f"{tag}_total_iterations"])
    st = diag["projection_stage_summaries"]
    np.testing.assert_allclose([s["physical_density_fraction"] for s in st], gm[f"{tag}_stage_vol"], atol=1e-10)
    np.testing.assert_allclose([s["gray_fraction_005_095"] for s in st], gm[f"{tag}_stage_gray"], atol=1e-12)
    np.testing.assert_allclose([s["minimum_achievable_physical_fraction"] for s in st], gm[f"{tag}_stage_vmin"],
                               atol=1e-12)
    np.testing.assert_allclose([s["maximum_achievable_physical_fraction"] for s in st], gm[f"{tag}_stage_vmax"],
                               atol=1e-12)
    np.testing.assert_allclose([s["final_change"] for s in st], gm[f"{tag}_stage_final_change"], atol=1e-10)
    # the binary design can be nearly a mechanism (1e-9 void material carries load),
    # whose iterative solve has an attainable residual floor
    assert diag["binary_compliance"] == pytest.approx(float(gm[f"{tag}_binary_compliance"]), rel=1e-4)
