"""Host-side setup of the product package against the reference's golden vectors (CPU only)."""

import numpy as np
import pytest

import pytopo3d_b200 as P
from pytopo3d_b200.assembly import grid_from_edof
from pytopo3d_b200.obstacles import CUBE, SPHERE, cylinder_params

ORTHO = (10.0, 20.0, 30.0, 4.0, 5.0, 6.0, 0.10, 0.12, 0.08)


def test_stiffness_matches_reference(golden):
    np.testing.assert_allclose(P.lk_H8(elem_size=1.0), golden["KE_default_h1"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(P.lk_H8(elem_size=0.01), golden["KE_default_h001"], rtol=0, atol=1e-16)
    np.testing.assert_allclose(P.lk_H8(*ORTHO, elem_size=0.7), golden["KE_ortho_h07"], rtol=1e-13, atol=1e-12)
    np.testing.assert_allclose(P.make_C_matrix(*ORTHO), golden["C_ortho"], rtol=1e-14)


def test_connectivity_and_boundary_conditions_bit_exact(golden):
    edof, iK, jK = P.build_edof(3, 2, 4)
    np.testing.assert_array_equal(edof, golden["edof_3x2x4"])
    np.testing.assert_array_equal(iK, golden["iK_3x2x4"])
    np.testing.assert_array_equal(jK, golden["jK_3x2x4"])
    ndof = 180
    np.testing.assert_array_equal(P.build_force_vector(3, 2, 4, ndof), golden["F_default_3x2x4"])
    ff = P.build_force_field(3, 2, 4, 1, 3, 0, 2, 2, 4, 0.5, -1.0, 2.0)
    np.testing.assert_array_equal(ff, golden["force_field_3x2x4"])
    np.testing.assert_allclose(P.build_force_vector(3, 2, 4, ndof, ff), golden["F_field_3x2x4"], atol=1e-15)
    free, fixed = P.build_supports(3, 2, 4, ndof)
    np.testing.assert_array_equal(free, golden["free_default_3x2x4"])
    np.testing.assert_array_equal(fixed, golden["fixed_default_3x2x4"])
    sm = P.build_support_mask(3, 2, 4, 0, 1, 0, 2, 1, 3)
    free, fixed = P.build_supports(3, 2, 4, ndof, sm)
    np.testing.assert_array_equal(free, golden["free_mask_3x2x4"])
    np.testing.assert_array_equal(fixed, golden["fixed_mask_3x2x4"])


def test_corner_order_is_the_reference_one():
    edof, _, _ = P.build_edof(1, 1, 1)
    np.testing.assert_array_equal((edof[0, ::3] + 2) // 3, [1, 2, 4, 3, 5, 6, 8, 7])


@pytest.mark.parametrize("dims", [(1, 1, 1), (3, 2, 4), (7, 5, 3), (2, 9, 1)])
def test_grid_recovered_from_edof(dims):
    assert grid_from_edof(P.build_edof(*dims)[0]) == dims


def test_out_of_range_boxes_raise():
    with pytest.raises(ValueError):
        P.build_force_field(3, 2, 4, 0, 4, 0, 1, 0, 1, 1, 0, 0)
    with pytest.raises(ValueError):
        P.build_support_mask(3, 2, 4, 2, 2, 0, 1, 0, 1)
    with pytest.raises(ValueError):
        P.build_supports(3, 2, 4, 180, np.zeros((1, 1, 1), bool))


def primitive_mask(shape, o):
    """Test-side evaluation of one tp3d_obstacle's integer parameters, element by
    element, as the mask kernel's inside() does."""
    nely, nelx, nelz = shape
    yy, xx, zz = np.ogrid[:nely, :nelx, :nelz]
    c = [xx, yy, zz]
    if o.kind == CUBE:
        m = np.ones(shape, bool)
        for k in range(3):
            m &= (c[k] >= o.lo[k]) & (c[k] < o.hi[k])
        return m
    d2 = sum((c[k] - o.center[k]) ** 2 for k in range(3) if o.kind == SPHERE or k != o.axis)
    m = d2 <= o.r2
    if o.kind != SPHERE:
        m = m & (c[o.axis] >= o.lo[o.axis]) & (c[o.axis] < o.hi[o.axis])
    return np.broadcast_to(m, shape)


def test_cylinder_parameters_reproduce_reference_masks(golden):
    # the integer parameters the mask kernel receives (obstacles.py:137-160)
    for shape, args, key in (((16, 32, 16), ((0.5, 0.5, 0.5), 0.25, 1.0, 1), "cyl_y"),
                             ((10, 12, 14), ((0.3, 0.6, 0.5), 0.3, 0.5, 0), "cyl_x")):
        np.testing.assert_array_equal(primitive_mask(shape, cylinder_params(shape, *args)), golden[key])


def test_top3d_validation_happens_before_any_device_work():
    from pytopo3d_b200.optimizer import top3d

    bad = [dict(nelx=0), dict(volfrac=0.0), dict(penal=-1.0), dict(maxloop=0), dict(tolx=0.0),
           dict(history_frequency=0), dict(move=0.0), dict(projection_eta=1.0), dict(beta_schedule=()),
           dict(beta_schedule=(1.0, -2.0)), dict(obstacle_mask=np.zeros((1, 1, 1), bool)),
           dict(support_mask=np.zeros((1, 1, 1), bool))]
    for b in bad:
        kw = dict(nelx=4, nely=2, nelz=2, volfrac=0.3, penal=3.0, rmin=1.5, disp_thres=0.5)
        kw.update(b)
        with pytest.raises(ValueError):
            top3d(**kw)


def test_filter_radius_limit_is_reported_before_device_work():
    from pytopo3d_b200.filter import _validate_grid

    _validate_grid(4, 4, 4, 7.0)  # offsets up to 6: supported
    with pytest.raises(ValueError, match="max 7"):
        _validate_grid(4, 4, 4, 7.5)
