"""Protected-void cylinder masks (mirrors pytopo3d/utils/obstacles.py:110-193)."""

from __future__ import annotations

import numpy as np


def create_cylinder_obstacle(shape, center, radius, height, axis=2) -> np.ndarray:
    """Boolean (nely, nelx, nelz) cylinder; centre and sizes are domain fractions,
    distances are integer element-index distances compared with r^2."""
    nely, nelx, nelz = shape
    dims = [nelx, nely, nelz]
    c = [int(center[0] * nelx), int(center[1] * nely), int(center[2] * nelz)]
    r = int(radius * min(dims[i] for i in range(3) if i != axis))
    half = int(height * dims[axis]) // 2
    lo, hi = max(0, c[axis] - half), min(dims[axis], c[axis] + half)
    yy, xx, zz = np.ogrid[:nely, :nelx, :nelz]
    coords = [xx, yy, zz]
    p, q = [coords[i] - c[i] for i in range(3) if i != axis]
    m = (p ** 2 + q ** 2 <= r * r) & (coords[axis] >= lo) & (coords[axis] < hi)
    return np.broadcast_to(m, shape).copy()


def cylinder_mask_elements(shape, cx, cz_or_cy, radius, axis, c2=None):
    """Cylinder given directly in element units: axis 0/1/2, centre (a, b) in the
    two perpendicular axes (in x, y, z order), integer radius."""
    nely, nelx, nelz = shape
    yy, xx, zz = np.ogrid[:nely, :nelx, :nelz]
    coords = [xx, yy, zz]
    p, q = [coords[i] for i in range(3) if i != axis]
    m = (p - cx) ** 2 + (q - cz_or_cy) ** 2 <= radius * radius
    return np.broadcast_to(m, shape).copy()
