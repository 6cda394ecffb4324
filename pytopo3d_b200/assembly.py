"""Structured-grid connectivity, loads and supports (host side).

Mirrors pytopo3d/utils/assembly.py: ``H8_NODE_OFFSETS`` (:17-26),
``build_force_field`` (:28-75), ``build_force_vector`` (:78-184),
``build_support_mask`` (:186-221), ``build_supports`` (:224-348) and
``build_edof`` (:351-408), with identical index conventions:
element e = y + nely*(x + nelx*z), node n = iy + (nely+1)*(ix + (nelx+1)*iz),
DOF 3n + c, 1-based edof table.  The loops of the reference are vectorised;
the solver itself never needs edof (the operator is matrix-free).
"""

from __future__ import annotations

from typing import Optional, Tuple

import numpy as np

H8_NODE_OFFSETS = (
    (0, 0, 0),
    (0, 1, 0),
    (1, 1, 0),
    (1, 0, 0),
    (0, 0, 1),
    (0, 1, 1),
    (1, 1, 1),
    (1, 0, 1),
)


def _nid(ix, iy, iz, nelx, nely):
    return iy + ix * (nely + 1) + iz * (nelx + 1) * (nely + 1)


def build_force_field(nelx, nely, nelz, x1, x2, y1, y2, z1, z2, F_x, F_y, F_z):
    """Element force field (nely, nelx, nelz, 3): the force spread evenly over a box."""
    if not (0 <= x1 < x2 <= nelx and 0 <= y1 < y2 <= nely and 0 <= z1 < z2 <= nelz):
        raise ValueError("Specified index range is out of bounds")
    n = (x2 - x1) * (y2 - y1) * (z2 - z1)
    ff = np.zeros((nely, nelx, nelz, 3), dtype=float)
    ff[y1:y2, x1:x2, z1:z2, 0] = F_x / n
    ff[y1:y2, x1:x2, z1:z2, 1] = F_y / n
    ff[y1:y2, x1:x2, z1:z2, 2] = F_z / n
    return ff


def build_force_vector(nelx: int, nely: int, nelz: int, ndof: int,
                       force_field: Optional[np.ndarray] = None) -> np.ndarray:
    """Nodal force vector: default -1 on the z-DOF of the ix=nelx, iz=0 edge nodes;
    with a force field, each element's force is shared 1/8 per corner."""
    F = np.zeros(ndof)
    if force_field is None:
        nid = _nid(nelx, np.arange(nely + 1), 0, nelx, nely)
        F[3 * nid + 2] = -1.0
        return F
    if force_field.shape != (nely, nelx, nelz, 3):
        raise ValueError(f"force_field has shape {force_field.shape}, "
                         f"but expected {(nely, nelx, nelz, 3)}")
    y, x, z = np.nonzero(np.any(force_field != 0, axis=-1))
    share = force_field[y, x, z] / 8.0
    for ox, oy, oz in H8_NODE_OFFSETS:
        nid = _nid(x + ox, y + oy, z + oz, nelx, nely)
        for c in range(3):
            np.add.at(F, 3 * nid + c, share[:, c])
    return F


def build_support_mask(nelx, nely, nelz, x1, x2, y1, y2, z1, z2):
    """Boolean element box (nely, nelx, nelz)."""
    if not (0 <= x1 < x2 <= nelx and 0 <= y1 < y2 <= nely and 0 <= z1 < z2 <= nelz):
        raise ValueError("Specified index range is out of bounds")
    m = np.zeros((nely, nelx, nelz), dtype=bool)
    m[y1:y2, x1:x2, z1:z2] = True
    return m


def fixed_node_ids(nelx, nely, nelz, support_mask=None) -> np.ndarray:
    """Sorted ids of clamped nodes: the x=0 face by default (or for an empty
    mask), else every corner of every supported element."""
    if support_mask is not None and support_mask.shape != (nely, nelx, nelz):
        raise ValueError(f"support_mask has shape {support_mask.shape}, "
                         f"but expected {(nely, nelx, nelz)}")
    if support_mask is None or not np.any(support_mask):
        iy, iz = np.meshgrid(np.arange(nely + 1), np.arange(nelz + 1), indexing="ij")
        return np.unique(_nid(0, iy, iz, nelx, nely).ravel())
    y, x, z = np.nonzero(support_mask)
    return np.unique(np.concatenate([_nid(x + ox, y + oy, z + oz, nelx, nely)
                                     for ox, oy, oz in H8_NODE_OFFSETS]))


def build_supports(nelx: int, nely: int, nelz: int, ndof: int,
                   support_mask: Optional[np.ndarray] = None) -> Tuple[np.ndarray, np.ndarray]:
    """(freedofs0, fixeddof0), sorted 0-based DOF indices."""
    nodes = fixed_node_ids(nelx, nely, nelz, support_mask)
    fixed = np.unique(np.concatenate([3 * nodes, 3 * nodes + 1, 3 * nodes + 2]))
    fixed = fixed[(fixed >= 0) & (fixed < ndof)]
    is_fixed = np.zeros(ndof, dtype=bool)
    is_fixed[fixed] = True
    return np.flatnonzero(~is_fixed), fixed


def build_edof(nelx: int, nely: int, nelz: int):
    """(edofMat (nele, 24) 1-based, iK, jK) as in the reference."""
    e = np.arange(nelx * nely * nelz)
    y, x, z = e % nely, (e // nely) % nelx, e // (nelx * nely)
    base = _nid(x, y, z, nelx, nely)
    off = np.array([_nid(ox, oy, oz, nelx, nely) for ox, oy, oz in H8_NODE_OFFSETS])
    nodes = base[:, None] + off[None, :]
    edof = (3 * nodes[:, :, None] + np.arange(3)).reshape(-1, 24) + 1
    iK = np.repeat(edof, 24, axis=1).ravel()
    jK = np.tile(edof, (1, 24)).ravel()
    return edof, iK, jK


def grid_from_edof(edofMat) -> Tuple[int, int, int]:
    """Recover (nelx, nely, nelz) from a structured edof table (compliance.py takes
    no grid arguments)."""
    e0 = np.asarray(edofMat[0], dtype=np.int64)
    nodes = (e0[0::3] - 1) // 3
    stride_x = int(nodes[3] - nodes[0])
    stride_z = int(nodes[4] - nodes[0])
    nely = stride_x - 1
    nelx = stride_z // stride_x - 1
    nele = int(np.asarray(edofMat).shape[0])
    if nely < 1 or nelx < 1 or nele % (nelx * nely):
        raise ValueError("edofMat is not a structured H8 connectivity table")
    return nelx, nely, nele // (nelx * nely)
