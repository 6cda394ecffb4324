"""B200-native SIMP hot path with PyTopo3D's optimizer API.

Drop-ins for the reference's hot-path functions (same names and argument
meaning) backed by hand-written sm_100a CUDA kernels in ``libtopo3d_b200.so``:

* ``top3d``, ``evaluate_fixed_geometry_metrics``, ``evaluate_fixed_geometry_compliance``
  (pytopo3d/core/optimizer.py)
* ``build_filter``, ``heaviside_projection``, ``build_physical_density``,
  ``apply_density_filter_chain_rule`` (pytopo3d/utils/filter.py)
* ``optimality_criteria_update_projected`` (pytopo3d/utils/oc_update.py)
* ``element_compliance`` (pytopo3d/core/compliance.py)
* ``HexSolver`` / ``get_solver`` (pytopo3d/utils/solver.py boundary)
* host setup: ``lk_H8``, ``make_C_matrix``, ``build_edof``, ``build_force_vector``,
  ``build_supports``, ``build_force_field``, ``build_support_mask``.
"""

from .assembly import (H8_NODE_OFFSETS, build_edof, build_force_field, build_force_vector,
                       build_support_mask, build_supports)
from .stiffness import lk_H8, make_C_matrix

__all__ = [
    "H8_NODE_OFFSETS", "build_edof", "build_force_field", "build_force_vector", "build_support_mask",
    "build_supports", "lk_H8", "make_C_matrix", "top3d", "evaluate_fixed_geometry_metrics",
    "evaluate_fixed_geometry_compliance", "build_filter", "heaviside_projection", "build_physical_density",
    "apply_density_filter_chain_rule", "optimality_criteria_update_projected", "element_compliance",
    "HexSolver", "get_solver", "ConeFilter",
]


def __getattr__(name):
    # device-backed modules import torch lazily
    if name in ("top3d", "evaluate_fixed_geometry_metrics", "evaluate_fixed_geometry_compliance"):
        from . import optimizer
        return getattr(optimizer, name)
    if name in ("build_filter", "heaviside_projection", "build_physical_density",
                "apply_density_filter_chain_rule", "ConeFilter"):
        from . import filter as _f
        return getattr(_f, name)
    if name in ("optimality_criteria_update_projected", "oc_update_projected"):
        from . import oc_update
        return getattr(oc_update, name)
    if name == "element_compliance":
        from .compliance import element_compliance
        return element_compliance
    if name in ("HexSolver", "get_solver"):
        from . import solver
        return getattr(solver, name)
    raise AttributeError(name)
