"""Generate golden vectors by running the reference PyTopo3D itself.

Run once in a container that has the reference checked out:

    python tests/golden/make_golden.py [--reference /root/reference]

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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                  "golden.npz"))
    args = ap.parse_args()
    ref = _import_reference(args.reference)
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

    np.savez_compressed(args.out, **g)
    print(f"wrote {len(g)} arrays to {args.out} ({os.path.getsize(args.out)/1024:.0f} KiB)")


if __name__ == "__main__":
    main()
