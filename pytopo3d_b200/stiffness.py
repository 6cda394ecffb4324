"""Element stiffness of the trilinear hexahedron (host side, FP64).

Mirrors pytopo3d/utils/stiffness.py (``lk_H8`` :12-130, ``make_C_matrix``
:133-197): same defaults (E=1, G_xy=0.4, nu=0.3, elem_size=1.0), same Voigt
order [xx, yy, zz, xy, yz, zx], same 2x2x2 Gauss rule and corner order.
KE is computed once on the host and handed to the device kernels.
"""

from __future__ import annotations

import math

import numpy as np

from .assembly import H8_NODE_OFFSETS


def make_C_matrix(E_x, E_y=None, E_z=None, G_xy=0.4, G_yz=None, G_zx=None,
                  nu_xy=0.3, nu_yz=None, nu_zx=None, normalize=False):
    """6x6 orthotropic stiffness in Voigt notation (inverse of the compliance)."""
    E_y = E_x if E_y is None else E_y
    E_z = E_x if E_z is None else E_z
    G_yz = G_xy if G_yz is None else G_yz
    G_zx = G_xy if G_zx is None else G_zx
    nu_yz = nu_xy if nu_yz is None else nu_yz
    nu_zx = nu_xy if nu_zx is None else nu_zx
    S = np.zeros((6, 6))
    S[0, 0], S[1, 1], S[2, 2] = 1.0 / E_x, 1.0 / E_y, 1.0 / E_z
    S[0, 1] = S[1, 0] = -nu_xy / E_x
    S[1, 2] = S[2, 1] = -nu_yz / E_y
    S[0, 2] = S[2, 0] = -nu_zx / E_z
    S[3, 3], S[4, 4], S[5, 5] = 1.0 / G_xy, 1.0 / G_yz, 1.0 / G_zx
    C = np.linalg.inv(S)
    return C / E_x if (normalize and E_x != 0) else C


def _shape_gradients(xi):
    """d N_a / d xi_k at natural point xi for the 8 corners (8, 3)."""
    s = 2.0 * np.asarray(H8_NODE_OFFSETS, dtype=float) - 1.0
    lin = 1.0 + s * np.asarray(xi)
    out = np.empty((8, 3))
    out[:, 0] = 0.125 * s[:, 0] * lin[:, 1] * lin[:, 2]
    out[:, 1] = 0.125 * s[:, 1] * lin[:, 0] * lin[:, 2]
    out[:, 2] = 0.125 * s[:, 2] * lin[:, 0] * lin[:, 1]
    return out


def lk_H8(E_x=1, E_y=None, E_z=None, G_xy=0.4, G_yz=None, G_zx=None,
          nu_xy=0.3, nu_yz=None, nu_zx=None, elem_size=1.0):
    """24x24 element stiffness by 2x2x2 Gauss quadrature on a cube of side elem_size."""
    C = make_C_matrix(E_x, E_y, E_z, G_xy, G_yz, G_zx, nu_xy, nu_yz, nu_zx)
    signs = 2.0 * np.asarray(H8_NODE_OFFSETS, dtype=float) - 1.0
    X = 0.5 * elem_size * signs
    g = 1.0 / math.sqrt(3.0)
    KE = np.zeros((24, 24))
    for z in (-g, g):
        for y in (-g, g):
            for x in (-g, g):
                dN = _shape_gradients((x, y, z))
                J = dN.T @ X
                det = np.linalg.det(J)
                if det <= 0:
                    raise ValueError("Negative or zero Jacobian determinant.")
                G = np.linalg.solve(J.T, dN.T).T
                B = np.zeros((6, 24))
                B[0, 0::3] = G[:, 0]
                B[1, 1::3] = G[:, 1]
                B[2, 2::3] = G[:, 2]
                B[3, 0::3], B[3, 1::3] = G[:, 1], G[:, 0]
                B[4, 1::3], B[4, 2::3] = G[:, 2], G[:, 1]
                B[5, 0::3], B[5, 2::3] = G[:, 2], G[:, 0]
                KE += B.T @ C @ B * det
    return KE
