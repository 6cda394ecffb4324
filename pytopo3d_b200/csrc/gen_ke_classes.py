"""Generate tp3d_ke_classes.h: the signed value classes of the H8 element stiffness.

For a material with cubic symmetry (C11 = C22 = C33, C12 = C13 = C23,
C44 = C55 = C66; isotropic materials included) every entry of the 24x24
trilinear-hexahedron stiffness on a cube is +-(one of a few values): the entry
is a fixed linear combination of (C11, C12, C44) whose coefficients depend only
on the geometry and the corner order.  This script finds those combinations
with three unit materials and groups entries whose coefficient vectors agree up
to sign.  The kernel then keeps one register per class and folds the sign into
the FMA.  Usage: python gen_ke_classes.py > tp3d_ke_classes.h
"""

import math

import numpy as np

OFFSETS = np.array([[0, 0, 0], [0, 1, 0], [1, 1, 0], [1, 0, 0],
                    [0, 0, 1], [0, 1, 1], [1, 1, 1], [1, 0, 1]], dtype=float)


def stiffness_from_C(C):
    """2x2x2 Gauss integral of B^T C B on the unit cube (corner order OFFSETS)."""
    s = 2.0 * OFFSETS - 1.0
    g = 1.0 / math.sqrt(3.0)
    K = np.zeros((24, 24))
    for z in (-g, g):
        for y in (-g, g):
            for x in (-g, g):
                p = np.array([x, y, z])
                lin = 1.0 + s * p
                dN = np.empty((8, 3))
                dN[:, 0] = 0.125 * s[:, 0] * lin[:, 1] * lin[:, 2]
                dN[:, 1] = 0.125 * s[:, 1] * lin[:, 0] * lin[:, 2]
                dN[:, 2] = 0.125 * s[:, 2] * lin[:, 0] * lin[:, 1]
                G = dN * 2.0  # unit cube: d/dx = 2 d/dxi, detJ = 1/8
                B = np.zeros((6, 24))
                B[0, 0::3], B[1, 1::3], B[2, 2::3] = G[:, 0], G[:, 1], G[:, 2]
                B[3, 0::3], B[3, 1::3] = G[:, 1], G[:, 0]
                B[4, 1::3], B[4, 2::3] = G[:, 2], G[:, 1]
                B[5, 0::3], B[5, 2::3] = G[:, 2], G[:, 0]
                K += B.T @ C @ B * 0.125
    return K


def cubic_C(c11, c12, c44):
    C = np.zeros((6, 6))
    C[:3, :3] = c12
    np.fill_diagonal(C[:3, :3], c11)
    C[3, 3] = C[4, 4] = C[5, 5] = c44
    return C


def main():
    basis = [stiffness_from_C(cubic_C(*e)) for e in ((1, 0, 0), (0, 1, 0), (0, 0, 1))]
    coef = np.stack([b.ravel() for b in basis], axis=1)  # (576, 3)
    scale = np.abs(coef).max()
    key = np.round(coef / scale * 2 ** 20).astype(np.int64)
    classes = []
    table = []
    for v in key:
        if not v.any():
            table.append(0)
            continue
        for i, c in enumerate(classes):
            if np.array_equal(v, c):
                table.append(i + 1)
                break
            if np.array_equal(v, -c):
                table.append(-(i + 1))
                break
        else:
            classes.append(v)
            table.append(len(classes))
    print("// Generated by gen_ke_classes.py: signed value classes of the H8 element")
    print("// stiffness for cubic-symmetric materials (entry = sign * class value).")
    print("#pragma once")
    print(f"constexpr int kKEClasses = {len(classes)};")
    for decl in ("static __device__ constexpr signed char kKEClass[576]",
                 "static constexpr signed char kKEClassHost[576]"):
        print(decl + " = {")
        for r in range(24):
            print("    " + ", ".join(f"{t:3d}" for t in table[r * 24:(r + 1) * 24]) + ",")
        print("};")


if __name__ == "__main__":
    main()
