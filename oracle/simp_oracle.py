"""CPU oracle for PyTopo3D's per-iteration SIMP path (numpy / scipy, FP64).

TEST INFRASTRUCTURE ONLY.  This module restates, in plain numpy, the algorithm
of the reference hot path so that the CUDA path can be checked against it.  It
may be imported only by ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py``; the product package (``pytopo3d_b200``) never
imports it and has no CPU fallback.

Parity is pinned against golden vectors produced by the reference itself
(``tests/golden/make_golden.py`` imports pytopo3d and records its outputs;
``tests/test_oracle_golden.py`` checks this module against them).

Every function names the reference file:line range it restates.  Array
conventions follow the reference exactly:

* element arrays have shape ``(nely, nelx, nelz)`` and are flattened in Fortran
  order, ``e = y + nely * (x + nelx * z)``  (filter.py:85-87, 170-174);
* node ``nid = iy + ix*(nely+1) + iz*(nelx+1)*(nely+1)``, DOF ``3*nid + c``
  (assembly.py:121-129, 375-401);
* element-local corners follow ``H8_NODE_OFFSETS`` (assembly.py:17-26).
"""

from __future__ import annotations

import math
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

# (x, y, z) offset of each local corner from the element's minimum corner
# (assembly.py:17-26).  Shared by connectivity and element physics.
H8_NODE_OFFSETS = np.array(
    [
        [0, 0, 0],
        [0, 1, 0],
        [1, 1, 0],
        [1, 0, 0],
        [0, 0, 1],
        [0, 1, 1],
        [1, 1, 1],
        [1, 0, 1],
    ],
    dtype=np.int64,
)

E0 = 1.0
EMIN = 1.0e-9


# ---------------------------------------------------------------------------
# element stiffness (stiffness.py)
# ---------------------------------------------------------------------------
def make_C_matrix(E_x, E_y=None, E_z=None, G_xy=0.4, G_yz=None, G_zx=None,
                  nu_xy=0.3, nu_yz=None, nu_zx=None, normalize=False):
    """Orthotropic Voigt stiffness as the inverse of the compliance matrix.

    Restates stiffness.py:133-197: missing moduli default to the x / xy
    values, Voigt order is [xx, yy, zz, xy, yz, zx].
    """
    E_y = E_x if E_y is None else E_y
    E_z = E_x if E_z is None else E_z
    G_yz = G_xy if G_yz is None else G_yz
    G_zx = G_xy if G_zx is None else G_zx
    nu_yz = nu_xy if nu_yz is None else nu_yz
    nu_zx = nu_xy if nu_zx is None else nu_zx
    compliance = np.diag([1.0 / E_x, 1.0 / E_y, 1.0 / E_z,
                          1.0 / G_xy, 1.0 / G_yz, 1.0 / G_zx])
    compliance[0, 1] = compliance[1, 0] = -nu_xy / E_x
    compliance[1, 2] = compliance[2, 1] = -nu_yz / E_y
    compliance[0, 2] = compliance[2, 0] = -nu_zx / E_z
    C = np.linalg.inv(compliance)
    if normalize and E_x != 0:
        return C / E_x
    return C


def lk_H8(E_x=1, E_y=None, E_z=None, G_xy=0.4, G_yz=None, G_zx=None,
          nu_xy=0.3, nu_yz=None, nu_zx=None, elem_size=1.0):
    """24x24 trilinear-hexahedron stiffness, 2x2x2 Gauss rule.

    Restates stiffness.py:12-130 for a cube of side ``elem_size`` whose corners
    follow ``H8_NODE_OFFSETS``.  DOF order inside the element is
    (node 0: x,y,z), (node 1: x,y,z), ...
    """
    C = make_C_matrix(E_x, E_y, E_z, G_xy, G_yz, G_zx, nu_xy, nu_yz, nu_zx)
    signs = 2.0 * H8_NODE_OFFSETS.astype(float) - 1.0          # (8, 3) in {-1, 1}
    coords = 0.5 * elem_size * signs
    g = 1.0 / math.sqrt(3.0)
    KE = np.zeros((24, 24))
    for gz in (-g, g):
        for gy in (-g, g):
            for gx in (-g, g):
                p = np.array([gx, gy, gz])
                # dN_a/dxi_k = s_ak/8 * prod_{m != k} (1 + s_am p_m)
                lin = 1.0 + signs * p                            # (8, 3)
                dN = np.empty((8, 3))
                for k in range(3):
                    others = [m for m in range(3) if m != k]
                    dN[:, k] = 0.125 * signs[:, k] * lin[:, others[0]] * lin[:, others[1]]
                J = dN.T @ coords
                detJ = np.linalg.det(J)
                if detJ <= 0:
                    raise ValueError("Negative or zero Jacobian determinant.")
                dNx = np.linalg.solve(J.T, dN.T).T                 # (8, 3)
                B = np.zeros((6, 24))
                for a in range(8):
                    gx_, gy_, gz_ = dNx[a]
                    c = 3 * a
                    B[0, c] = gx_
                    B[1, c + 1] = gy_
                    B[2, c + 2] = gz_
                    B[3, c], B[3, c + 1] = gy_, gx_
                    B[4, c + 1], B[4, c + 2] = gz_, gy_
                    B[5, c], B[5, c + 2] = gz_, gx_
                KE += B.T @ C @ B * detJ
    return KE


# ---------------------------------------------------------------------------
# connectivity, loads, supports (assembly.py)
# ---------------------------------------------------------------------------
def node_id(ix, iy, iz, nelx, nely):
    return iy + ix * (nely + 1) + iz * (nelx + 1) * (nely + 1)


def element_coords(nelx, nely, nelz):
    """(y, x, z) integer coordinates of each element in Fortran order."""
    e = np.arange(nelx * nely * nelz)
    return e % nely, (e // nely) % nelx, e // (nelx * nely)


def build_edof(nelx, nely, nelz, with_coo=False):
    """1-based element-to-DOF table (assembly.py:351-408).

    Row ``e`` lists the 24 global DOFs of element ``e`` in local corner order;
    the COO index vectors are ``kron`` expansions of that table
    (assembly.py:404-406) and are only built when ``with_coo`` is set.
    """
    ey, ex, ez = element_coords(nelx, nely, nelz)
    base = node_id(ex, ey, ez, nelx, nely)                       # min-corner node
    off = node_id(H8_NODE_OFFSETS[:, 0], H8_NODE_OFFSETS[:, 1],
                  H8_NODE_OFFSETS[:, 2], nelx, nely)             # (8,)
    nodes = base[:, None] + off[None, :]                         # (nele, 8)
    edof = (3 * nodes[:, :, None] + np.arange(3)[None, None, :]).reshape(-1, 24) + 1
    if not with_coo:
        return edof
    iK = np.repeat(edof, 24, axis=1).ravel()
    jK = np.tile(edof, (1, 24)).ravel()
    return edof, iK, jK


def build_force_vector(nelx, nely, nelz, ndof, force_field=None):
    """Global nodal force vector (assembly.py:78-184).

    Default: -1 on the z-DOF of every node with ix=nelx, iz=0 (all iy).
    With a force field, each element's force is split evenly (1/8) between its
    eight corner nodes.
    """
    F = np.zeros(ndof)
    if force_field is None:
        iy = np.arange(nely + 1)
        nid = node_id(nelx, iy, 0, nelx, nely)
        F[3 * nid + 2] = -1.0
        return F
    expected = (nely, nelx, nelz, 3)
    if force_field.shape != expected:
        raise ValueError(
            f"force_field has shape {force_field.shape}, but expected {expected}")
    ff = np.asarray(force_field, dtype=float)
    # Fortran order over (y, x, z), per component
    per_node = ff / 8.0
    for dz in (0, 1):
        for dx in (0, 1):
            for dy in (0, 1):
                ey, ex, ez = np.meshgrid(np.arange(nely), np.arange(nelx),
                                         np.arange(nelz), indexing="ij")
                nid = node_id(ex + dx, ey + dy, ez + dz, nelx, nely)
                for c in range(3):
                    np.add.at(F, (3 * nid + c).ravel(), per_node[..., c].ravel())
    return F


def fixed_nodes_from_support(nelx, nely, nelz, support_mask=None):
    """Node ids whose three DOFs are clamped (assembly.py:224-348)."""
    if support_mask is not None:
        expected = (nely, nelx, nelz)
        if support_mask.shape != expected:
            raise ValueError(
                f"support_mask has shape {support_mask.shape}, but expected {expected}")
    if support_mask is None or not np.any(support_mask):
        iy, iz = np.meshgrid(np.arange(nely + 1), np.arange(nelz + 1), indexing="ij")
        return np.unique(node_id(0, iy, iz, nelx, nely).ravel())
    ys, xs, zs = np.nonzero(support_mask)
    nodes = [node_id(xs + o[0], ys + o[1], zs + o[2], nelx, nely) for o in H8_NODE_OFFSETS]
    return np.unique(np.concatenate(nodes))


def build_supports(nelx, nely, nelz, ndof, support_mask=None):
    """(freedofs0, fixeddof0), both sorted 0-based (assembly.py:224-348)."""
    nodes = fixed_nodes_from_support(nelx, nely, nelz, support_mask)
    fixed = np.unique(np.concatenate([3 * nodes, 3 * nodes + 1, 3 * nodes + 2]))
    fixed = fixed[(fixed >= 0) & (fixed < ndof)]
    is_fixed = np.zeros(ndof, dtype=bool)
    is_fixed[fixed] = True
    return np.nonzero(~is_fixed)[0], fixed


def build_force_field(nelx, nely, nelz, x1, x2, y1, y2, z1, z2, F_x, F_y, F_z):
    """Uniform element force field over a box (assembly.py:28-75)."""
    if not (0 <= x1 < x2 <= nelx and 0 <= y1 < y2 <= nely and 0 <= z1 < z2 <= nelz):
        raise ValueError("Specified index range is out of bounds")
    n = (x2 - x1) * (y2 - y1) * (z2 - z1)
    ff = np.zeros((nely, nelx, nelz, 3))
    ff[y1:y2, x1:x2, z1:z2] = np.array([F_x, F_y, F_z]) / n
    return ff


def build_support_mask(nelx, nely, nelz, x1, x2, y1, y2, z1, z2):
    """Boolean element box (assembly.py:186-221)."""
    if not (0 <= x1 < x2 <= nelx and 0 <= y1 < y2 <= nely and 0 <= z1 < z2 <= nelz):
        raise ValueError("Specified index range is out of bounds")
    m = np.zeros((nely, nelx, nelz), dtype=bool)
    m[y1:y2, x1:x2, z1:z2] = True
    return m


def cylinder_mask(shape, center, radius, height, axis=2):
    """Protected-void cylinder with integer-index distances (obstacles.py:110-193)."""
    nely, nelx, nelz = shape
    dims = [nelx, nely, nelz]
    c = [int(center[0] * nelx), int(center[1] * nely), int(center[2] * nelz)]
    perp = [dims[i] for i in range(3) if i != axis]
    r = int(radius * min(perp))
    half = int(height * dims[axis]) // 2
    lo, hi = max(0, c[axis] - half), min(dims[axis], c[axis] + half)
    yy, xx, zz = np.ogrid[:nely, :nelx, :nelz]
    d = [xx - c[0], yy - c[1], zz - c[2]]
    along = [xx, yy, zz][axis]
    p = [d[i] for i in range(3) if i != axis]
    m = (p[0] ** 2 + p[1] ** 2 <= r * r) & (along >= lo) & (along < hi)
    return np.broadcast_to(m, shape).copy()


# ---------------------------------------------------------------------------
# density filter and projection (filter.py)
# ---------------------------------------------------------------------------
FLOAT_EPSILON = 1e-9


def cone_taps(rmin):
    """Integer offsets (dx, dy, dz) and weights rmin - |d| > 1e-9 (filter.py:193-206)."""
    R = int(math.ceil(rmin)) + 1
    taps = []
    for dz in range(-R, R + 1):
        for dx in range(-R, R + 1):
            for dy in range(-R, R + 1):
                w = rmin - math.sqrt(float(dx * dx + dy * dy + dz * dz))
                if w > FLOAT_EPSILON:
                    taps.append((dx, dy, dz, w))
    return taps


def build_filter(nelx, nely, nelz, rmin):
    """Cone filter matrix H (CSR) and row sums Hs (filter.py:122-228).

    Same weights as the reference (integer-grid distance, threshold 1e-9,
    truncated at the boundary); built by offset instead of by KD-tree.
    """
    if min(nelx, nely, nelz) < 1:
        raise ValueError("nelx, nely, and nelz must all be positive")
    if not np.isfinite(rmin) or rmin <= 0.0:
        raise ValueError(f"rmin must be finite and positive, got {rmin}")
    ey, ex, ez = element_coords(nelx, nely, nelz)
    e = np.arange(nelx * nely * nelz)
    rows, cols, vals = [], [], []
    for dx, dy, dz, w in cone_taps(rmin):
        jx, jy, jz = ex + dx, ey + dy, ez + dz
        ok = (jx >= 0) & (jx < nelx) & (jy >= 0) & (jy < nely) & (jz >= 0) & (jz < nelz)
        rows.append(e[ok])
        cols.append((jy + nely * (jx + nelx * jz))[ok])
        vals.append(np.full(int(ok.sum()), w))
    n = nelx * nely * nelz
    H = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(n, n)).tocsr()
    Hs = np.asarray(H.sum(axis=1)).ravel()
    Hs[Hs == 0] = 1.0
    return H, Hs


def heaviside_projection(rho_filtered, beta, eta=0.5):
    """tanh projection and its (unclipped) derivative (filter.py:26-60)."""
    if not np.isfinite(beta) or beta <= 0:
        raise ValueError(f"beta must be positive, got {beta}")
    if not 0.0 < eta < 1.0:
        raise ValueError(f"eta must be between 0 and 1, got {eta}")
    den = np.tanh(beta * eta) + np.tanh(beta * (1.0 - eta))
    t = np.tanh(beta * (rho_filtered - eta))
    rho = (np.tanh(beta * eta) + t) / den
    return np.clip(rho, 0.0, 1.0), beta * (1.0 - t ** 2) / den


def build_physical_density(x, H, Hs, beta, eta, protected_solid, protected_void):
    """Filter, project, clamp protected regions (filter.py:63-100)."""
    shape = x.shape
    rf = ((H @ x.ravel(order="F")) / Hs).reshape(shape, order="F")
    rp, d = heaviside_projection(rf, beta, eta)
    rp = np.where(protected_solid, 1.0, rp)
    rp = np.where(protected_void, 0.0, rp)
    d = np.where(protected_solid | protected_void, 0.0, d)
    return rf, rp, d


def apply_density_filter_chain_rule(g, dproj, H, Hs):
    """H^T (g * dproj / Hs) in Fortran element order (filter.py:103-119)."""
    w = (g * dproj).ravel(order="F") / Hs
    return (H.T @ w).reshape(g.shape, order="F")


# ---------------------------------------------------------------------------
# element energy (compliance.py)
# ---------------------------------------------------------------------------
def element_compliance(U, edofMat, KE):
    """ce[e] = u_e^T KE u_e with a 1-based edof table (compliance.py:69-75)."""
    Ue = U[edofMat.astype(np.int64) - 1]
    return np.sum((Ue @ KE) * Ue, axis=1)


# ---------------------------------------------------------------------------
# OC update (oc_update.py)
# ---------------------------------------------------------------------------
def oc_update_projected(x, dc_dx, dv_dx, move, target_free_volume, H, Hs, beta, eta,
                        free_mask, protected_solid, protected_void,
                        max_bisection_iterations=80, bisection_tolerance=1e-8,
                        trace=None):
    """Projected-volume OC update by lambda bisection (oc_update.py:25-124).

    The multiplier search runs over [0, 1e12] with normalised ratios; each
    step re-filters and re-projects the candidate and the candidate with the
    smallest volume error is returned.  ``trace`` (a list) receives the
    (lambda_mid, volume) sequence when given.
    """
    if not np.isfinite(move) or move <= 0:
        raise ValueError(f"move must be positive, got {move}")
    if max_bisection_iterations < 1:
        raise ValueError("max_bisection_iterations must be at least 1")
    xf = x[free_mask]
    ratio = np.maximum(-dc_dx[free_mask] / np.maximum(dv_dx[free_mask], 1e-20), 0.0)
    scale = float(np.max(ratio)) if ratio.size else 0.0
    ratio = ratio / scale if scale > 0.0 else np.ones_like(ratio)
    lo, hi = 0.0, 1.0e12
    best_x, best_rho, best_err = x.copy(), None, float("inf")
    for _ in range(max_bisection_iterations):
        lam = 0.5 * (lo + hi)
        r = np.maximum(ratio / (lam + 1e-30), 1e-30)
        cf = np.clip(np.maximum(xf - move, np.minimum(xf + move, xf * np.sqrt(r))), 0.0, 1.0)
        cand = x.copy()
        cand[free_mask] = cf
        cand[protected_solid] = 1.0
        cand[protected_void] = 0.0
        _, rho, _ = build_physical_density(cand, H, Hs, beta, eta,
                                           protected_solid, protected_void)
        vol = float(np.sum(rho[free_mask]))
        if trace is not None:
            trace.append((lam, vol))
        err = abs(vol - target_free_volume)
        if err < best_err:
            best_x, best_rho, best_err = cand, rho, err
        if vol > target_free_volume:
            lo = lam
        else:
            hi = lam
        if (hi - lo) / max(hi + lo, np.finfo(float).tiny) < bisection_tolerance:
            break
    return best_x, best_rho


# ---------------------------------------------------------------------------
# FE solve (optimizer.py:584-594 with solver.py's CPU path)
# ---------------------------------------------------------------------------
def assemble_K(rho_physical, KE, penal, nelx, nely, nelz):
    """Global stiffness with SIMP moduli E = Emin + (E0-Emin) rho^p (optimizer.py:584-589)."""
    edof, iK, jK = build_edof(nelx, nely, nelz, with_coo=True)
    ndof = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
    E = EMIN + (E0 - EMIN) * rho_physical.ravel(order="F") ** penal
    vals = np.kron(E, KE.ravel())
    return sp.coo_matrix((vals, (iK - 1, jK - 1)), shape=(ndof, ndof)).tocsr(), edof


def solve_displacement(rho_physical, KE, penal, F, freedofs, nelx, nely, nelz,
                       solver: Optional[Callable] = None):
    """U with U[free] = Kff^{-1} F[free] (optimizer.py:591-594)."""
    K, edof = assemble_K(rho_physical, KE, penal, nelx, nely, nelz)
    Kff = K[freedofs, :][:, freedofs]
    solver = spla.spsolve if solver is None else solver
    U = np.zeros(K.shape[0])
    U[freedofs] = solver(Kff.tocsc() if solver is spla.spsolve else Kff, F[freedofs])
    return U, edof


def sensitivities(rho_physical, U, edof, KE, penal):
    """(c, ce, dc_drho) of optimizer.py:596-612."""
    shape = rho_physical.shape
    ce = element_compliance(U, edof, KE).reshape(shape, order="F")
    c = float(np.sum((EMIN + (E0 - EMIN) * rho_physical ** penal) * ce))
    dc = -penal * (E0 - EMIN) * rho_physical ** (penal - 1.0) * ce
    return c, ce, dc


# ---------------------------------------------------------------------------
# the SIMP loop (optimizer.py:283-839)
# ---------------------------------------------------------------------------
def prepare_masks(nelx, nely, nelz, obstacle_mask=None, protected_zone_mask=None,
                  force_field=None, support_mask=None, default_load_strip=True):
    """Protected-solid / protected-void / free masks (optimizer.py:346-405)."""
    shape = (nely, nelx, nelz)
    void = np.zeros(shape, bool) if obstacle_mask is None else np.asarray(obstacle_mask, bool).copy()
    solid = np.zeros(shape, bool) if protected_zone_mask is None else np.asarray(protected_zone_mask, bool).copy()
    if force_field is None:
        if default_load_strip:
            solid[:, -1, 0] = True
    else:
        solid |= np.any(force_field != 0.0, axis=-1)
    if support_mask is None or not np.any(support_mask):
        solid[:, 0, :] = True
    else:
        solid |= np.asarray(support_mask, bool)
    solid[void & solid] = False
    free = ~(void | solid)
    return solid, void, free


def simp_iteration(x, rho_physical, dproj, beta, eta, penal, move, target_free_volume,
                   H, Hs, KE, F, freedofs, solid, void, free, nelx, nely, nelz,
                   solver=None, U=None):
    """One pass of the loop body (optimizer.py:578-696): solve, sensitivities, OC.

    Returns a dict with every intermediate the CUDA path is checked against.
    ``U`` may be supplied to skip the solve (for decoupled checks).
    """
    if U is None:
        U, edof = solve_displacement(rho_physical, KE, penal, F, freedofs, nelx, nely, nelz, solver)
    else:
        edof = build_edof(nelx, nely, nelz)
    c, ce, dc = sensitivities(rho_physical, U, edof, KE, penal)
    dv = free.astype(float)
    dc_dx = apply_density_filter_chain_rule(dc, dproj, H, Hs)
    dv_dx = apply_density_filter_chain_rule(dv, dproj, H, Hs)
    trace: List[Tuple[float, float]] = []
    x_new, rho_new = oc_update_projected(x, dc_dx, dv_dx, move, target_free_volume, H, Hs,
                                         beta, eta, free, solid, void, trace=trace)
    change = float(np.max(np.abs(x_new[free] - x[free])))
    return dict(U=U, c=c, ce=ce, dc=dc, dc_dx=dc_dx, dv_dx=dv_dx, x_new=x_new,
                rho_new=rho_new, change=change, trace=trace)


def top3d(nelx, nely, nelz, volfrac, penal, rmin, KE=None, F=None, obstacle_mask=None,
          protected_zone_mask=None, force_field=None, support_mask=None, tolx=0.01,
          maxloop=2000, beta_schedule=(1.0, 2.0, 4.0, 8.0), projection_eta=0.5,
          move=0.2, elem_size=1.0, solver=None, max_total_iterations=None,
          record=None):
    """Restatement of the top3d loop (optimizer.py:283-696) with an optional nodal F.

    Returns ``(x, rho_physical, compliance_history)``; ``record`` (a list)
    receives the per-iteration dict of ``simp_iteration``.
    """
    shape = (nely, nelx, nelz)
    ndof = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
    solid, void, free = prepare_masks(nelx, nely, nelz, obstacle_mask, protected_zone_mask,
                                      force_field, support_mask)
    target = float(volfrac * int(free.sum()))
    if F is None:
        F = build_force_vector(nelx, nely, nelz, ndof, force_field)
    freedofs, _ = build_supports(nelx, nely, nelz, ndof, support_mask)
    KE = lk_H8(elem_size=elem_size) if KE is None else KE
    H, Hs = build_filter(nelx, nely, nelz, rmin)
    x = np.full(shape, volfrac)
    x[solid] = 1.0
    x[void] = 0.0
    history = []
    total = 0
    for beta in beta_schedule:
        _, rho, dproj = build_physical_density(x, H, Hs, beta, projection_eta, solid, void)
        change, loop = float("inf"), 0
        while change > tolx and loop < maxloop:
            if max_total_iterations is not None and total >= max_total_iterations:
                return x, rho, history
            loop += 1
            total += 1
            it = simp_iteration(x, rho, dproj, beta, projection_eta, penal, move, target, H, Hs,
                                KE, F, freedofs, solid, void, free, nelx, nely, nelz, solver)
            history.append(it["c"])
            if record is not None:
                record.append(it)
            change = it["change"]
            x = it["x_new"]
            _, rho, dproj = build_physical_density(x, H, Hs, beta, projection_eta, solid, void)
    return x, rho, history


def evaluate_fixed_geometry_metrics(xPhys, penal, KE, force_field=None, support_mask=None,
                                    obstacle_mask=None, protected_zone_mask=None, F=None):
    """One solve on a fixed design plus load-patch metrics (optimizer.py:54-252)."""
    nely, nelx, nelz = xPhys.shape
    ndof = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
    x = np.array(xPhys, dtype=float, copy=True)
    if protected_zone_mask is not None:
        x[protected_zone_mask] = 1.0
    if obstacle_mask is not None:
        x[obstacle_mask] = 0.0
    if F is None:
        F = build_force_vector(nelx, nely, nelz, ndof, force_field)
    freedofs, _ = build_supports(nelx, nely, nelz, ndof, support_mask)
    U, edof = solve_displacement(x, KE, penal, F, freedofs, nelx, nely, nelz)
    c, _, _ = sensitivities(x, U, edof, KE, penal)
    loaded = np.nonzero(np.abs(F) > 0.0)[0]
    nodes = np.unique(loaded // 3)
    out = {"compliance": float(c)}
    tot = {}
    for c_i, ax in enumerate("xyz"):
        d = 3 * nodes + c_i
        tot[ax] = float(np.sum(np.abs(F[d]))) if d.size else 0.0
        out[f"u{ax}_avg_load_patch"] = float(np.mean(U[d])) if d.size else None
    for ax in "xyz":
        u = out[f"u{ax}_avg_load_patch"]
        out[f"k_avg_{ax}"] = (float(tot[ax] / abs(u)) if u is not None and u != 0.0 and tot[ax] > 0.0
                              else None)
    dom = max((("x", tot["x"]), ("y", tot["y"]), ("z", tot["z"])), key=lambda t: t[1])[0]
    out["k_avg"] = out[f"k_avg_{dom}"]
    out["F_total"] = float(np.sum(np.abs(F[loaded]))) if loaded.size else 0.0
    for ax in "xyz":
        out[f"F_total_{ax}"] = tot[ax]
        out[f"loaded_{ax}_dof_count"] = int(nodes.size)
    return out
