"""Obstacle masks built on the device (drop-in for pytopo3d/utils/obstacles.py).

The reference converts each obstacle's fractional centre, size and radius to
element indices with ``int()`` truncation and tests every element with numpy
(obstacles.py:12-193); ``parse_obstacle_config_file`` ORs the masks of a JSON
list (:237-269).  Here the same integer parameters are computed on the host
(a handful of scalars per obstacle) and one kernel (``tp3d_obstacle_mask``)
tests every element of the grid against all of them, writing a flat uint8
mask in the kernels' Fortran element order.  ``obstacle_mask_flat`` keeps that
mask on the device (the batched runner feeds it straight to its loops); the
reference-named functions return the ``(nely, nelx, nelz)`` numpy array the
reference returns.
"""

from __future__ import annotations

import ctypes as C
import json
from typing import Dict, Iterable, List, Sequence, Tuple, Union

import numpy as np
import torch

from . import _lib
from ._tensors import device, from_flat

CUBE, SPHERE, CYLINDER = 0, 1, 2


class Obstacle(C.Structure):
    """``tp3d_obstacle`` of include/topo3d_b200.h: one primitive in element indices."""

    _fields_ = [("kind", C.c_int), ("axis", C.c_int), ("center", C.c_int * 3), ("lo", C.c_int * 3),
                ("hi", C.c_int * 3), ("r2", C.c_longlong)]


def _centre(shape, center):
    nely, nelx, nelz = shape
    return [int(center[0] * nelx), int(center[1] * nely), int(center[2] * nelz)]


def cube_params(shape, center, size) -> Obstacle:
    """Integer bounds of create_cube_obstacle (obstacles.py:36-57)."""
    nely, nelx, nelz = shape
    cx, cy, cz = _centre(shape, center)
    if isinstance(size, (int, float)):
        hx, hy, hz = int(size * nelx / 2), int(size * nely / 2), int(size * nelz / 2)
    else:
        hx, hy, hz = int(size[0] * nelx / 2), int(size[1] * nely / 2), int(size[2] * nelz / 2)
    o = Obstacle(kind=CUBE)
    lo = (max(0, cx - hx), max(0, cy - hy), max(0, cz - hz))
    hi = (min(nelx, cx + hx), min(nely, cy + hy), min(nelz, cz + hz))
    for k in range(3):
        o.center[k] = (cx, cy, cz)[k]
        o.lo[k], o.hi[k] = lo[k], hi[k]
    return o


def sphere_params(shape, center, radius) -> Obstacle:
    """Integer centre and squared radius of create_sphere_obstacle (obstacles.py:84-101)."""
    nely, nelx, nelz = shape
    c = _centre(shape, center)
    r = int(radius * min(nelx, nely, nelz))
    o = Obstacle(kind=SPHERE, r2=r * r)
    for k in range(3):
        o.center[k] = c[k]
    return o


def cylinder_params(shape, center, radius, height, axis=2) -> Obstacle:
    """Integer centre, squared radius and axial bounds of create_cylinder_obstacle
    (obstacles.py:137-160)."""
    nely, nelx, nelz = shape
    dims = [nelx, nely, nelz]
    c = _centre(shape, center)
    r = int(radius * min(dims[i] for i in range(3) if i != axis))
    half = int(height * dims[axis]) // 2
    o = Obstacle(kind=CYLINDER, axis=int(axis), r2=r * r)
    for k in range(3):
        o.center[k] = c[k]
        o.lo[k], o.hi[k] = 0, dims[k]
    o.lo[axis] = max(0, c[axis] - half)
    o.hi[axis] = min(dims[axis], c[axis] + half)
    return o


def cylinder_elements(axis, a, b, radius, length) -> Obstacle:
    """A cylinder given directly in element units: ``axis`` 0/1/2, centre (a, b)
    in the two axes perpendicular to it (in x, y, z order), integer radius,
    spanning the whole ``length`` of the grid along the axis."""
    o = Obstacle(kind=CYLINDER, axis=int(axis), r2=int(radius) * int(radius))
    perp = [i for i in range(3) if i != axis]
    o.center[perp[0]], o.center[perp[1]] = int(a), int(b)
    o.lo[axis], o.hi[axis] = 0, int(length)
    return o


def params_from_config(shape, config: Dict) -> Obstacle:
    """Primitive of one configuration entry (create_obstacle_from_config, obstacles.py:195-235)."""
    kind = config.get("type", "").lower()
    if kind == "cube":
        return cube_params(shape, config.get("center", [0.5, 0.5, 0.5]), config.get("size", 0.2))
    if kind == "sphere":
        return sphere_params(shape, config.get("center", [0.5, 0.5, 0.5]), config.get("radius", 0.2))
    if kind == "cylinder":
        return cylinder_params(shape, config.get("center", [0.5, 0.5, 0.5]), config.get("radius", 0.2),
                               config.get("height", 0.5), config.get("axis", 2))
    raise ValueError(f"Unknown obstacle type: {kind}")


def obstacle_mask_flat(shape, obstacles: Iterable[Obstacle], out: torch.Tensor = None) -> torch.Tensor:
    """Flat uint8 device mask (Fortran element order) of the union of ``obstacles``."""
    nely, nelx, nelz = shape
    obs = list(obstacles)
    arr = (Obstacle * max(1, len(obs)))(*obs)
    if out is None:
        out = torch.empty(nelx * nely * nelz, dtype=torch.uint8, device=device())
    _lib.check(_lib.lib().tp3d_obstacle_mask(nelx, nely, nelz, C.cast(arr, C.c_void_p), len(obs), out.data_ptr(),
                                             _lib.stream_ptr()), "obstacle_mask")
    return out


def _host(shape, obstacles) -> np.ndarray:
    return from_flat(obstacle_mask_flat(shape, obstacles), shape).bool().cpu().numpy()


def create_cube_obstacle(shape: Tuple[int, int, int], center: Sequence[float],
                         size: Union[float, Sequence[float]]) -> np.ndarray:
    """Boolean (nely, nelx, nelz) cube / cuboid mask (obstacles.py:12-61)."""
    return _host(shape, [cube_params(shape, center, size)])


def create_sphere_obstacle(shape: Tuple[int, int, int], center: Sequence[float], radius: float) -> np.ndarray:
    """Boolean (nely, nelx, nelz) sphere mask (obstacles.py:63-108)."""
    return _host(shape, [sphere_params(shape, center, radius)])


def create_cylinder_obstacle(shape: Tuple[int, int, int], center: Sequence[float], radius: float, height: float,
                             axis: int = 2) -> np.ndarray:
    """Boolean (nely, nelx, nelz) cylinder mask (obstacles.py:110-193)."""
    return _host(shape, [cylinder_params(shape, center, radius, height, axis)])


def create_obstacle_from_config(shape: Tuple[int, int, int], config: Dict) -> np.ndarray:
    """Mask of one configuration entry (obstacles.py:195-235)."""
    return _host(shape, [params_from_config(shape, config)])


def parse_obstacle_config_file(config_file: str, shape: Tuple[int, int, int]) -> np.ndarray:
    """Union of the obstacles listed in a JSON file (obstacles.py:237-269)."""
    with open(config_file, "r") as f:
        config = json.load(f)
    return _host(shape, [params_from_config(shape, c) for c in config.get("obstacles", [])])
