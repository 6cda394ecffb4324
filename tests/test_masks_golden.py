"""Mask handling, loads and supports of top3d against what the reference built (CPU only).

``tests/golden/golden_masks.npz`` records, for three top3d runs of the
reference (``make_golden.py --set masks``), the protected-solid, protected-void
and free masks its loop received, its force vector and its free DOFs
(optimizer.py:346-405, 427-428).  The runs cover:

* m1: an obstacle cylinder, an explicit force field, a partial support mask and
  a protected zone that overlaps the cylinder (protected void wins);
* m2: an all-false support mask (falls back to the x = 0 face), the default
  load strip, an obstacle that cuts into both protected strips;
* m3: the 128x64x64 workload's masks at 32x16x16 (void cylinder along y, solid
  slab x < 1).

Everything here is host code and must match bit for bit.
"""

import logging
import os

import numpy as np
import pytest

import pytopo3d_b200 as P
from pytopo3d_b200.optimizer import _fixed_dof_mask, resolve_masks

ROOT = os.path.dirname(os.path.abspath(__file__))

# (nelx, nely, nelz) and the inputs of each recorded run
RUNS = {
    "m1": dict(dims=(10, 6, 5), obstacle="m1_obstacle", force_field="m1_force_field", support="m1_support",
               zone="m1_zone"),
    "m2": dict(dims=(8, 4, 4), obstacle="m2_obstacle", force_field=None, support="empty", zone=None),
    "m3": dict(dims=(32, 16, 16), obstacle="m3_obstacle", force_field=None, support=None, zone="m3_zone"),
}


@pytest.fixture(scope="module")
def gm():
    return np.load(os.path.join(ROOT, "golden", "golden_masks.npz"))


def _inputs(gm, tag):
    r = RUNS[tag]
    nx, ny, nz = r["dims"]
    get = lambda k: None if k is None else gm[k]
    support = np.zeros((ny, nx, nz), bool) if r["support"] == "empty" else get(r["support"])
    return nx, ny, nz, get(r["obstacle"]), get(r["zone"]), get(r["force_field"]), support


@pytest.mark.parametrize("tag", sorted(RUNS))
def test_masks_bit_exact(gm, tag, caplog):
    nx, ny, nz, obstacle, zone, ff, support = _inputs(gm, tag)
    with caplog.at_level(logging.WARNING):
        solid, void, free = resolve_masks(nx, ny, nz, obstacle, zone, ff, support)
    np.testing.assert_array_equal(solid, gm[f"{tag}_solid"])
    np.testing.assert_array_equal(void, gm[f"{tag}_void"])
    np.testing.assert_array_equal(free, gm[f"{tag}_free"])
    overlap = obstacle is not None and bool(np.any(obstacle & ~void))
    assert not overlap
    # m1 and m2 have protected-void elements inside a protected-solid region
    assert ("protected void takes precedence" in caplog.text) == (tag != "m3")


@pytest.mark.parametrize("tag", sorted(RUNS))
def test_loads_and_supports_bit_exact(gm, tag):
    nx, ny, nz, _, _, ff, support = _inputs(gm, tag)
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    F = P.build_force_vector(nx, ny, nz, ndof, ff)
    idx = np.flatnonzero(F)
    np.testing.assert_array_equal(idx, gm[f"{tag}_F_idx"])
    np.testing.assert_array_equal(F[idx], gm[f"{tag}_F_val"])
    free, _ = P.build_supports(nx, ny, nz, ndof, support)
    np.testing.assert_array_equal(free, gm[f"{tag}_freedofs"])
    fixed = _fixed_dof_mask(nx, ny, nz, support)
    np.testing.assert_array_equal(np.flatnonzero(fixed == 0), gm[f"{tag}_freedofs"])


PRIMITIVES = {
    "prim_cube_a": ("cube", (6, 10, 5), ((0.3, 0.6, 0.5), 0.4)),
    "prim_cube_b": ("cube", (7, 9, 11), ((0.9, 0.1, 0.45), (0.2, 0.5, 0.9))),
    "prim_sphere_a": ("sphere", (12, 20, 10), ((0.5, 0.5, 0.5), 0.3)),
    "prim_sphere_b": ("sphere", (9, 13, 17), ((0.05, 0.7, 0.95), 0.45)),
    "prim_cyl_0": ("cylinder", (11, 14, 9), ((0.4, 0.55, 0.3), 0.35, 0.6, 0)),
    "prim_cyl_1": ("cylinder", (11, 14, 9), ((0.4, 0.55, 0.3), 0.35, 0.6, 1)),
    "prim_cyl_2": ("cylinder", (11, 14, 9), ((0.4, 0.55, 0.3), 0.35, 0.6, 2)),
    "m3_obstacle": ("cylinder", (16, 32, 16), ((0.5, 0.5, 0.5), 3.0 / 16.0, 1.0, 1)),
}


@pytest.mark.parametrize("key", sorted(PRIMITIVES))
def test_obstacle_parameters_reproduce_reference_masks(gm, key):
    """The integer parameters handed to the mask kernel, evaluated element by
    element on the host, give the reference's masks (obstacles.py:12-193)."""
    from test_host_setup import primitive_mask
    from pytopo3d_b200 import obstacles as ob

    kind, shape, args = PRIMITIVES[key]
    o = {"cube": ob.cube_params, "sphere": ob.sphere_params, "cylinder": ob.cylinder_params}[kind](shape, *args)
    np.testing.assert_array_equal(primitive_mask(shape, o), gm[key])


def test_mask_validation_messages():
    shape = (2, 3, 2)
    with pytest.raises(ValueError, match="obstacle_mask has shape"):
        resolve_masks(3, 2, 2, obstacle_mask=np.zeros((1, 1, 1), bool))
    with pytest.raises(ValueError, match="protected_zone_mask has shape"):
        resolve_masks(3, 2, 2, protected_zone_mask=np.zeros((2, 2, 2), bool))
    with pytest.raises(ValueError, match="force_field has shape"):
        resolve_masks(3, 2, 2, force_field=np.zeros(shape, float))
    with pytest.raises(ValueError, match="support_mask has shape"):
        resolve_masks(3, 2, 2, support_mask=np.zeros((3, 2, 2), bool))
    with pytest.raises(ValueError, match="at least one free design element"):
        resolve_masks(3, 2, 2, protected_zone_mask=np.ones(shape, bool))


def test_cantilever_masks_loads_and_supports_bit_exact():
    """The 32x16x16 cantilever run in full (``golden_cantilever_32x16x16.npz``):
    default masks, load and supports as the reference built them."""
    g = np.load(os.path.join(ROOT, "golden", "golden_cantilever_32x16x16.npz"))
    nx, ny, nz = 32, 16, 16
    solid, void, free = resolve_masks(nx, ny, nz)
    np.testing.assert_array_equal(solid, g["cl_solid"])
    np.testing.assert_array_equal(void, g["cl_void"])
    np.testing.assert_array_equal(free, g["cl_free"])
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    F = P.build_force_vector(nx, ny, nz, ndof)
    idx = np.flatnonzero(F)
    np.testing.assert_array_equal(idx, g["cl_F_idx"])
    np.testing.assert_array_equal(F[idx], g["cl_F_val"])
    free_dofs, _ = P.build_supports(nx, ny, nz, ndof)
    np.testing.assert_array_equal(free_dofs, g["cl_freedofs"])
