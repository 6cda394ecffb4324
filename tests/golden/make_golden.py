"""Generate golden vectors by running the reference PyTopo3D itself.

Run once in a container that has the reference checked out:

    python tests/golden/make_golden.py --reference <path of the PyTopo3D checkout> [--set NAME ...]

(or set PYTOPO3D_REFERENCE instead of passing --reference).  Each set writes
its own ``.npz`` next to this script:

* ``base``          -> golden.npz: kernels, set-up, loop bodies, a small top3d run;
* ``masks``         -> golden_masks.npz: top3d runs through every mask path
                       (obstacle, support, force field, protected zone, overlaps)
                       with the masks, loads and supports the reference built;
* ``cantilever``    -> golden_cantilever_32x16x16.npz: the full beta 1/2/4/8
                       schedule (maxloop 200, tolx 0.01) of the 32x16x16
                       cantilever with the reference's direct solve (about an
                       hour of single-threaded SuperLU);
* ``sensitivities`` -> golden_sensitivities_48x24x24.npz: summed compliance and
                       its design gradient for three load cases at 48x24x24
                       (three SuperLU solves of about two minutes each).

It imports the reference package (pure Python) with a headless stand-in for
matplotlib and for the reference's plotting module (both are imported by
pytopo3d/core/optimizer.py:20,34 but unused on the optimisation path), calls
the reference functions on small seeded inputs and writes ``golden.npz`` next
to this script.  The tests only read the ``.npz``; nothing at test time needs
the reference.
"""

from __future__ import annotations

import argparse
import os
import sys
import types

import numpy as np


def _import_reference(path):
    for name in ("matplotlib", "matplotlib.pyplot"):
        sys.modules.setdefault(name, types.ModuleType(name))
    disp = types.ModuleType("pytopo3d.visualization.display")
    disp.display_3D = lambda *a, **k: None
    sys.modules["pytopo3d.visualization.display"] = disp
    sys.path.insert(0, path)
    import pytopo3d.core.compliance as compliance
    import pytopo3d.core.optimizer as optimizer
    import pytopo3d.utils.assembly as assembly
    import pytopo3d.utils.filter as filt
    import pytopo3d.utils.obstacles as obstacles
    import pytopo3d.utils.oc_update as oc
    import pytopo3d.utils.stiffness as stiffness
    return types.SimpleNamespace(compliance=compliance, optimizer=optimizer, assembly=assembly,
                                 filt=filt, oc=oc, stiffness=stiffness, obstacles=obstacles)


ORTHO = (10.0, 20.0, 30.0, 4.0, 5.0, 6.0, 0.10, 0.12, 0.08)


def _one_iteration(ref, nelx, nely, nelz, volfrac, penal, rmin, beta, eta, move, seed,
                   obstacle=None):
    """One loop body of top3d from a seeded design, using reference functions only."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    rng = np.random.default_rng(seed)
    shape = (nely, nelx, nelz)
    ndof = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
    solid = np.zeros(shape, bool)
    solid[:, -1, 0] = True
    solid[:, 0, :] = True
    void = np.zeros(shape, bool) if obstacle is None else obstacle.copy()
    solid[void & solid] = False
    free = ~(solid | void)
    x = rng.uniform(0.1, 0.9, size=shape)
    x[solid] = 1.0
    x[void] = 0.0
    H, Hs = ref.filt.build_filter(nelx, nely, nelz, rmin)
    rf, rp, dp = ref.filt.build_physical_density(x, H, Hs, beta, eta, solid, void)
    KE = ref.stiffness.lk_H8(elem_size=1.0)
    edof, iK, jK = ref.assembly.build_edof(nelx, nely, nelz)
    F = ref.assembly.build_force_vector(nelx, nely, nelz, ndof)
    freedofs, _ = ref.assembly.build_supports(nelx, nely, nelz, ndof)
    E = 1e-9 + (1 - 1e-9) * rp.ravel(order="F") ** penal
    K = sp.coo_matrix((np.kron(E, KE.ravel()), (iK - 1, jK - 1)), shape=(ndof, ndof)).tocsr()
    U = np.zeros(ndof)
    U[freedofs] = spla.spsolve(K[freedofs, :][:, freedofs], F[freedofs])
    ce = ref.compliance.element_compliance(U, edof, KE).reshape(shape, order="F")
    c = float(np.sum((1e-9 + (1 - 1e-9) * rp ** penal) * ce))
    dc = -penal * (1 - 1e-9) * rp ** (penal - 1.0) * ce
    dc_dx = ref.filt.apply_density_filter_chain_rule(dc, dp, H, Hs)
    dv_dx = ref.filt.apply_density_filter_chain_rule(free.astype(float), dp, H, Hs)
    target = volfrac * int(free.sum())
    x_new, rho_new = ref.oc.optimality_criteria_update_projected(
        x, dc_dx, dv_dx, move, target, H, Hs, beta, eta, free, solid, void)
    return dict(x=x, solid=solid, void=void, rho_f=rf, rho_p=rp, dproj=dp, U=U, ce=ce, c=c,
                dc=dc, dc_dx=dc_dx, dv_dx=dv_dx, x_new=x_new, rho_new=rho_new, target=target)


def make_base(ref):
    g = {}

    # element stiffness (stiffness.py:12-197)
    g["KE_default_h1"] = ref.stiffness.lk_H8(elem_size=1.0)
    g["KE_default_h001"] = ref.stiffness.lk_H8(elem_size=0.01)
    g["KE_ortho_h07"] = ref.stiffness.lk_H8(*ORTHO, elem_size=0.7)
    g["C_ortho"] = ref.stiffness.make_C_matrix(*ORTHO)

    # connectivity, loads, supports (assembly.py)
    edof, iK, jK = ref.assembly.build_edof(3, 2, 4)
    g["edof_3x2x4"], g["iK_3x2x4"], g["jK_3x2x4"] = edof, iK, jK
    ndof = 3 * 4 * 3 * 5
    g["F_default_3x2x4"] = ref.assembly.build_force_vector(3, 2, 4, ndof)
    ff = ref.assembly.build_force_field(3, 2, 4, 1, 3, 0, 2, 2, 4, 0.5, -1.0, 2.0)
    g["force_field_3x2x4"] = ff
    g["F_field_3x2x4"] = ref.assembly.build_force_vector(3, 2, 4, ndof, ff)
    g["free_default_3x2x4"], g["fixed_default_3x2x4"] = ref.assembly.build_supports(3, 2, 4, ndof)
    sm = ref.assembly.build_support_mask(3, 2, 4, 0, 1, 0, 2, 1, 3)
    g["support_mask_3x2x4"] = sm
    g["free_mask_3x2x4"], g["fixed_mask_3x2x4"] = ref.assembly.build_supports(3, 2, 4, ndof, sm)

    # filter matrix (filter.py:122-228) on several grids / radii
    for (nx, ny, nz, r) in [(3, 2, 4, 1.6), (5, 4, 6, 2.5), (6, 5, 4, 3.0), (7, 6, 5, 4.5),
                            (4, 3, 3, 1.5)]:
        H, Hs = ref.filt.build_filter(nx, ny, nz, r)
        key = f"{nx}x{ny}x{nz}_r{r}"
        H = H.tocoo()
        g[f"H_{key}_row"], g[f"H_{key}_col"], g[f"H_{key}_val"] = H.row, H.col, H.data
        g[f"Hs_{key}"] = Hs

    # physical density / projection / chain rule on a random design
    rng = np.random.default_rng(7)
    nx, ny, nz, r = 9, 6, 5, 2.5
    shape = (ny, nx, nz)
    H, Hs = ref.filt.build_filter(nx, ny, nz, r)
    x = rng.uniform(0.0, 1.0, size=shape)
    solid = rng.uniform(size=shape) < 0.1
    void = (rng.uniform(size=shape) < 0.1) & ~solid
    x[solid], x[void] = 1.0, 0.0
    for beta in (1.0, 4.0, 8.0):
        rf, rp, dp = ref.filt.build_physical_density(x, H, Hs, beta, 0.5, solid, void)
        g[f"bpd_rf_b{beta}"], g[f"bpd_rp_b{beta}"], g[f"bpd_dp_b{beta}"] = rf, rp, dp
        gphys = rng.normal(size=shape)
        g[f"chain_g_b{beta}"] = gphys
        g[f"chain_out_b{beta}"] = ref.filt.apply_density_filter_chain_rule(gphys, dp, H, Hs)
    g["bpd_x"], g["bpd_solid"], g["bpd_void"] = x, solid, void
    g["bpd_dims"] = np.array([nx, ny, nz, r])
    rho_lin = np.linspace(-0.2, 1.2, 41)
    g["hv_rho"] = rho_lin
    g["hv_out"], g["hv_der"] = ref.filt.heaviside_projection(rho_lin, 6.0, 0.4)

    # element energy (compliance.py:18-75)
    nx, ny, nz = 4, 3, 2
    edof = ref.assembly.build_edof(nx, ny, nz)[0]
    U = rng.normal(size=3 * (nx + 1) * (ny + 1) * (nz + 1))
    g["ce_U"], g["ce_out"] = U, ref.compliance.element_compliance(U, edof, g["KE_default_h1"])

    # projected OC update (oc_update.py:25-124) on a filtered problem
    nx, ny, nz, r = 8, 5, 4, 2.0
    shape = (ny, nx, nz)
    H, Hs = ref.filt.build_filter(nx, ny, nz, r)
    x = rng.uniform(0.2, 0.8, size=shape)
    solid = np.zeros(shape, bool)
    solid[:, 0, :] = True
    void = np.zeros(shape, bool)
    void[2, 4, 1:3] = True
    free = ~(solid | void)
    x[solid], x[void] = 1.0, 0.0
    _, _, dp = ref.filt.build_physical_density(x, H, Hs, 2.0, 0.5, solid, void)
    dc = -np.abs(rng.normal(size=shape)) * 1e-3
    dc_dx = ref.filt.apply_density_filter_chain_rule(dc, dp, H, Hs)
    dv_dx = ref.filt.apply_density_filter_chain_rule(free.astype(float), dp, H, Hs)
    target = 0.35 * int(free.sum())
    bx, brho = ref.oc.optimality_criteria_update_projected(
        x, dc_dx, dv_dx, 0.2, target, H, Hs, 2.0, 0.5, free, solid, void)
    g.update(oc_x=x, oc_solid=solid, oc_void=void, oc_dc_dx=dc_dx, oc_dv_dx=dv_dx,
             oc_target=np.array(target), oc_best_x=bx, oc_best_rho=brho,
             oc_dims=np.array([nx, ny, nz, r]))

    # one full loop body from a seeded design (optimizer.py:584-642)
    for tag, dims in (("8x4x4", (8, 4, 4, 0.3, 3.0, 1.5, 2.0, 0.5, 0.2, 11)),
                      ("32x16x16", (32, 16, 16, 0.3, 3.0, 3.0, 1.0, 0.5, 0.2, 12))):
        it = _one_iteration(ref, *dims)
        for k, v in it.items():
            g[f"it{tag}_{k}"] = np.asarray(v)
        g[f"it{tag}_dims"] = np.array(dims, dtype=float)

    # a full top3d run (optimizer.py:283-839): two beta stages, capped iterations
    diag = {}
    xphys, hist, comp, _ = ref.optimizer.top3d(
        nelx=6, nely=3, nelz=3, volfrac=0.4, penal=3.0, rmin=1.5, disp_thres=0.5,
        elem_size=1.0, tolx=0.01, maxloop=4, beta_schedule=(1.0, 2.0), save_history=True,
        history_frequency=1, diagnostics_out=diag)
    g["top3d_xphys"], g["top3d_compliance"] = xphys, np.array(comp)
    g["top3d_hist_c"] = np.array(hist["compliance_history"])
    g["top3d_binary_compliance"] = np.array(diag["binary_compliance"])
    g["top3d_total_iterations"] = np.array(diag["projection_total_iterations"])

    # fixed-geometry metrics (optimizer.py:54-252)
    m = ref.optimizer.evaluate_fixed_geometry_metrics(xphys, 3.0, elem_size=1.0)
    for k, v in m.items():
        g[f"metrics_{k}"] = np.array(np.nan if v is None else v, dtype=float)

    # cylinder obstacle formula (obstacles.py:110-193)
    g["cyl_y"] = ref.obstacles.create_cylinder_obstacle((16, 32, 16), (0.5, 0.5, 0.5), 0.25, 1.0, 1)
    g["cyl_x"] = ref.obstacles.create_cylinder_obstacle((10, 12, 14), (0.3, 0.6, 0.5), 0.3, 0.5, 0)

    return g


def _run_top3d_recorded(ref, **kw):
    """Run the reference top3d and record what its loop saw.

    The optimizer module's own references to build_physical_density, the OC
    update, build_force_vector and build_supports are wrapped for the duration
    of the run, so the recorded masks, loads and supports are the ones the
    reference built from the arguments (optimizer.py:346-405, 427-428), and the
    per-iteration designs are the OC update's outputs (optimizer.py:627-642).
    """
    opt = ref.optimizer
    rec = dict(solid=None, void=None, free=None, F=None, freedofs=None, x_new=[], change=[])
    saved = {k: getattr(opt, k) for k in ("build_physical_density", "optimality_criteria_update_projected",
                                          "build_force_vector", "build_supports")}

    def bpd(*a, **k):
        if rec["solid"] is None:
            rec["solid"] = np.array(k["protected_solid"], dtype=bool)
            rec["void"] = np.array(k["protected_void"], dtype=bool)
        return saved["build_physical_density"](*a, **k)

    def oc(*a, **k):
        x_new, rho_new = saved["optimality_criteria_update_projected"](*a, **k)
        free = np.asarray(k["free_mask"], dtype=bool)
        if rec["free"] is None:
            rec["free"] = free.copy()
        rec["x_new"].append(np.array(x_new))
        rec["change"].append(float(np.max(np.abs(x_new[free] - k["x"][free]))))
        return x_new, rho_new

    def bfv(*a, **k):
        F = saved["build_force_vector"](*a, **k)
        if rec["F"] is None:
            rec["F"] = np.array(F)
        return F

    def bs(*a, **k):
        out = saved["build_supports"](*a, **k)
        if rec["freedofs"] is None:
            rec["freedofs"] = np.array(out[0])
        return out

    opt.build_physical_density, opt.optimality_criteria_update_projected = bpd, oc
    opt.build_force_vector, opt.build_supports = bfv, bs
    try:
        diag = {}
        xphys, hist, comp, _ = opt.top3d(save_history=True, history_frequency=1, diagnostics_out=diag, **kw)
    finally:
        for k, v in saved.items():
            setattr(opt, k, v)
    return xphys, hist, comp, diag, rec


def _store_run(g, tag, xphys, hist, comp, diag, rec, keep_designs=True):
    g[f"{tag}_xphys"] = xphys
    g[f"{tag}_compliance"] = np.array(comp)
    g[f"{tag}_hist_c"] = np.array(hist["compliance_history"])
    g[f"{tag}_hist_it"] = np.array(hist["iteration_history"])
    g[f"{tag}_hist_beta"] = np.array(hist["beta_history"])
    g[f"{tag}_binary_compliance"] = np.array(diag["binary_compliance"])
    g[f"{tag}_total_iterations"] = np.array(diag["projection_total_iterations"])
    st = diag["projection_stage_summaries"]
    g[f"{tag}_stage_iterations"] = np.array([s["iterations"] for s in st])
    g[f"{tag}_stage_final_change"] = np.array([s["final_change"] for s in st])
    g[f"{tag}_stage_vol"] = np.array([s["physical_density_fraction"] for s in st])
    g[f"{tag}_stage_gray"] = np.array([s["gray_fraction_005_095"] for s in st])
    g[f"{tag}_stage_vmin"] = np.array([s["minimum_achievable_physical_fraction"] for s in st])
    g[f"{tag}_stage_vmax"] = np.array([s["maximum_achievable_physical_fraction"] for s in st])
    g[f"{tag}_solid"], g[f"{tag}_void"], g[f"{tag}_free"] = rec["solid"], rec["void"], rec["free"]
    g[f"{tag}_F_idx"] = np.flatnonzero(rec["F"])
    g[f"{tag}_F_val"] = rec["F"][g[f"{tag}_F_idx"]]
    g[f"{tag}_freedofs"] = rec["freedofs"]
    g[f"{tag}_change"] = np.array(rec["change"])
    if keep_designs:
        g[f"{tag}_x_new"] = np.stack(rec["x_new"])
        g[f"{tag}_hist_rho"] = np.stack(hist["density_history"])


def make_masks(ref):
    """top3d runs through each mask path of optimizer.py:346-405."""
    g = {}
    # (1) obstacle cylinder, explicit force field, a partial support mask and a
    #     protected zone that overlaps the cylinder (void wins on the overlap)
    nx, ny, nz = 10, 6, 5
    shape = (ny, nx, nz)
    obstacle = ref.obstacles.create_cylinder_obstacle(shape, (0.5, 0.5, 0.5), 0.3, 1.0, 1)
    ff = ref.assembly.build_force_field(nx, ny, nz, nx - 1, nx, 0, ny, 0, 2, 0.0, 0.5, -1.0)
    sm = ref.assembly.build_support_mask(nx, ny, nz, 0, 1, 0, ny, 0, 3)
    pz = np.zeros(shape, bool)
    pz[1:3, 3:6, 1:4] = True
    kw = dict(nelx=nx, nely=ny, nelz=nz, volfrac=0.35, penal=3.0, rmin=1.5, disp_thres=0.5, elem_size=1.0,
              obstacle_mask=obstacle, force_field=ff, support_mask=sm, protected_zone_mask=pz, tolx=0.01,
              maxloop=3, beta_schedule=(1.0, 2.0))
    g.update(m1_obstacle=obstacle, m1_force_field=ff, m1_support=sm, m1_zone=pz)
    _store_run(g, "m1", *_run_top3d_recorded(ref, **kw))

    # (2) an all-false support mask (falls back to the x = 0 face), no force
    #     field (default load strip), an obstacle that cuts into both strips
    #     without leaving a loaded node on void elements only
    nx, ny, nz = 8, 4, 4
    shape = (ny, nx, nz)
    obstacle = np.zeros(shape, bool)
    obstacle[1:3, 0:2, 1:3] = True
    obstacle[1, nx - 1, 0] = True
    kw = dict(nelx=nx, nely=ny, nelz=nz, volfrac=0.3, penal=3.0, rmin=1.5, disp_thres=0.5, elem_size=1.0,
              obstacle_mask=obstacle, support_mask=np.zeros(shape, bool), tolx=0.01, maxloop=3,
              beta_schedule=(1.0, 4.0))
    g.update(m2_obstacle=obstacle)
    _store_run(g, "m2", *_run_top3d_recorded(ref, **kw))

    # (3) the masks of the 128x64x64 cantilever workload at a quarter of its
    #     size: a protected-void cylinder of radius 3 along y through
    #     (x, z) = (16, 8) and a protected-solid slab x < 1; beta 1, 3 iterations
    nx, ny, nz = 32, 16, 16
    shape = (ny, nx, nz)
    obstacle = ref.obstacles.create_cylinder_obstacle(shape, (0.5, 0.5, 0.5), 3.0 / 16.0, 1.0, 1)
    slab = np.zeros(shape, bool)
    slab[:, 0:1, :] = True
    kw = dict(nelx=nx, nely=ny, nelz=nz, volfrac=0.3, penal=3.0, rmin=3.0, disp_thres=0.5, elem_size=1.0,
              obstacle_mask=obstacle, protected_zone_mask=slab, tolx=0.01, maxloop=3, beta_schedule=(1.0,))
    g.update(m3_obstacle=obstacle, m3_zone=slab)
    _store_run(g, "m3", *_run_top3d_recorded(ref, **kw))

    # obstacle primitives (obstacles.py:12-193) and a JSON list of them (:237-269)
    import json
    import tempfile

    ob = ref.obstacles
    g["prim_cube_a"] = ob.create_cube_obstacle((6, 10, 5), (0.3, 0.6, 0.5), 0.4)
    g["prim_cube_b"] = ob.create_cube_obstacle((7, 9, 11), (0.9, 0.1, 0.45), (0.2, 0.5, 0.9))
    g["prim_sphere_a"] = ob.create_sphere_obstacle((12, 20, 10), (0.5, 0.5, 0.5), 0.3)
    g["prim_sphere_b"] = ob.create_sphere_obstacle((9, 13, 17), (0.05, 0.7, 0.95), 0.45)
    for axis in range(3):
        g[f"prim_cyl_{axis}"] = ob.create_cylinder_obstacle((11, 14, 9), (0.4, 0.55, 0.3), 0.35, 0.6, axis)
    cfg = {"obstacles": [{"type": "cube", "center": [0.2, 0.3, 0.4], "size": [0.3, 0.2, 0.5]},
                         {"type": "sphere", "center": [0.7, 0.6, 0.5], "radius": 0.25},
                         {"type": "cylinder", "center": [0.5, 0.5, 0.5], "radius": 0.15, "height": 0.8,
                          "axis": 0}]}
    with tempfile.NamedTemporaryFile("w", suffix=".json", delete=False) as f:
        json.dump(cfg, f)
    g["prim_config_json"] = np.array(json.dumps(cfg))
    g["prim_config_mask"] = ob.parse_obstacle_config_file(f.name, (16, 24, 12))
    os.unlink(f.name)
    return g


def make_cantilever(ref):
    """The 32x16x16 cantilever run in full: beta 1, 2, 4, 8, maxloop 200 per
    stage, tolx 0.01, volfrac 0.3, penal 3, rmin 3, unit-cube elements, the
    reference's default load and supports, no obstacles."""
    g = {}
    xphys, hist, comp, diag, rec = _run_top3d_recorded(
        ref, nelx=32, nely=16, nelz=16, volfrac=0.3, penal=3.0, rmin=3.0, disp_thres=0.5, elem_size=1.0,
        tolx=0.01, maxloop=200, beta_schedule=(1.0, 2.0, 4.0, 8.0))
    _store_run(g, "cl", xphys, hist, comp, diag, rec, keep_designs=False)
    # designs at the end of each stage (the whole trajectory is too large to keep)
    ends = np.cumsum(g["cl_stage_iterations"]) - 1
    g["cl_stage_end_x"] = np.stack([rec["x_new"][i] for i in ends])
    g["cl_first_x"] = np.stack(rec["x_new"][:10])
    return g


SENS_DIMS = (48, 24, 24)
SENS_RMIN, SENS_BETA, SENS_ETA, SENS_PENAL, SENS_SEED = 2.5, 4.0, 0.5, 3.0, 5


def sensitivity_load_cases(nx, ny, nz):
    """The three load cases of the differentiation workload: a -z edge load at
    x = nelx, z = 0; a +y edge load at x = nelx, z = nelz (each a unit total
    spread evenly over the edge's nodes); a unit -z point load at the centre node
    of face x = nelx."""
    nid = lambda ix, iy, iz: iy + (ny + 1) * (ix + (nx + 1) * iz)
    F = np.zeros((3, 3 * (nx + 1) * (ny + 1) * (nz + 1)))
    for iy in range(ny + 1):
        F[0, 3 * nid(nx, iy, 0) + 2] = -1.0 / (ny + 1)
        F[1, 3 * nid(nx, iy, nz) + 1] = 1.0 / (ny + 1)
    F[2, 3 * nid(nx, ny // 2, nz // 2) + 2] = -1.0
    return F


def _sens_case(args):
    """Compliance and dc/drho_physical of one load case with the reference's
    direct solve and element energies (the loop body's optimizer.py:584-612)."""
    path, k = args
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    ref = _import_reference(path)
    nx, ny, nz = SENS_DIMS
    shape = (ny, nx, nz)
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    x = np.random.default_rng(SENS_SEED).uniform(0.05, 1.0, size=shape)
    H, Hs = ref.filt.build_filter(nx, ny, nz, SENS_RMIN)
    none = np.zeros(shape, bool)
    _, rho, _ = ref.filt.build_physical_density(x, H, Hs, SENS_BETA, SENS_ETA, none, none)
    KE = ref.stiffness.lk_H8(elem_size=1.0)
    edof, iK, jK = ref.assembly.build_edof(nx, ny, nz)
    freedofs, _ = ref.assembly.build_supports(nx, ny, nz, ndof)
    F = sensitivity_load_cases(nx, ny, nz)[k]
    E = 1e-9 + (1 - 1e-9) * rho.ravel(order="F") ** SENS_PENAL
    K = sp.coo_matrix((np.kron(E, KE.ravel()), (iK - 1, jK - 1)), shape=(ndof, ndof)).tocsr()
    U = np.zeros(ndof)
    U[freedofs] = spla.spsolve(K[freedofs, :][:, freedofs], F[freedofs])
    ce = ref.compliance.element_compliance(U, edof, KE).reshape(shape, order="F")
    c = float(np.sum((1e-9 + (1 - 1e-9) * rho ** SENS_PENAL) * ce))
    dc = -SENS_PENAL * (1 - 1e-9) * rho ** (SENS_PENAL - 1.0) * ce
    return c, dc


def make_sensitivities(ref, path):
    """Summed compliance of the three load cases and its gradient with respect
    to the design variables through the Heaviside projection and the filter
    (apply_density_filter_chain_rule, filter.py:103-119)."""
    import multiprocessing as mp

    nx, ny, nz = SENS_DIMS
    shape = (ny, nx, nz)
    with mp.get_context("spawn").Pool(3) as pool:
        parts = pool.map(_sens_case, [(path, k) for k in range(3)])
    x = np.random.default_rng(SENS_SEED).uniform(0.05, 1.0, size=shape)
    H, Hs = ref.filt.build_filter(nx, ny, nz, SENS_RMIN)
    none = np.zeros(shape, bool)
    _, _, dproj = ref.filt.build_physical_density(x, H, Hs, SENS_BETA, SENS_ETA, none, none)
    dc_sum = sum(p[1] for p in parts)
    g = dict(x=x, c_cases=np.array([p[0] for p in parts]),
             grad=ref.filt.apply_density_filter_chain_rule(dc_sum, dproj, H, Hs),
             dims=np.array(SENS_DIMS), params=np.array([SENS_RMIN, SENS_BETA, SENS_ETA, SENS_PENAL, SENS_SEED]))
    return g


SETS = {"base": "golden.npz", "masks": "golden_masks.npz", "cantilever": "golden_cantilever_32x16x16.npz",
        "sensitivities": "golden_sensitivities_48x24x24.npz"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("PYTOPO3D_REFERENCE"),
                    help="path of the PyTopo3D checkout (default: $PYTOPO3D_REFERENCE)")
    ap.add_argument("--set", action="append", choices=sorted(SETS), dest="sets",
                    help="fixture set to write (repeatable; default: base)")
    args = ap.parse_args()
    if not args.reference:
        ap.error("give --reference or set PYTOPO3D_REFERENCE")
    ref = _import_reference(args.reference)
    here = os.path.dirname(os.path.abspath(__file__))
    for name in args.sets or ["base"]:
        if name == "sensitivities":
            g = make_sensitivities(ref, args.reference)
        else:
            g = {"base": make_base, "masks": make_masks, "cantilever": make_cantilever}[name](ref)
        out = os.path.join(here, SETS[name])
        np.savez_compressed(out, **g)
        print(f"wrote {len(g)} arrays to {out} ({os.path.getsize(out)/1024:.0f} KiB)")

if __name__ == "__main__":
    main()
