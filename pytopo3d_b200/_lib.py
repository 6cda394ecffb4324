"""ctypes binding of ``libtopo3d_b200.so`` (the C ABI in include/topo3d_b200.h).

The library is built in-tree by ``python -m pytopo3d_b200._build`` (or
``__graft_entry__.build()``).  There is no CPU fallback: every compute entry
point of this package goes through this library and raises if it is missing
or if no CUDA device is present.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libtopo3d_b200.so")

TP3D_OK = 0
TP3D_NOT_CONVERGED = 1
TP3D_ERR_ARG = -1
TP3D_ERR_CUDA = -2
TP3D_ERR_TIMEOUT = -3
TP3D_ERR_NONFINITE = -4
PRECISION_FP64 = 0
PRECISION_MIXED = 1

vp = C.c_void_p
i32 = C.c_int
f64 = C.c_double
i64 = C.c_longlong
sz = C.c_size_t


class SolverOpts(C.Structure):
    _fields_ = [
        ("precision", i32),
        ("max_iterations", i32),
        ("rtol", f64),
        ("pre_sweeps", i32),
        ("post_sweeps", i32),
        ("omega", f64),
        ("coarsest_max_dofs", i32),
        ("max_levels", i32),
        ("smoother", i32),
        ("cheb_ratio", f64),
        ("power_iterations", i32),
        ("inner_density", i32),
        ("reliable_delta", f64),
        ("max_restarts", i32),
        ("fine_operator", i32),
        ("fused_cycle_dofs", i32),
        ("galerkin", i32),
        ("coarse_sweeps", i32),
        ("device_loop", i32),
        ("deep_sweeps", i32),
        ("pdl", i32),
        ("coarse_bf16", i32),
        ("split_dofs", i32),
        ("deep_cta", i32),
        ("block_sweeps", i32),
        ("resid_restrict_dofs", i32),
        ("spectra_streams", i32),
        ("cluster_cycle", i32),
        ("fine_slab_depth", i32),
        ("coarse_node_major", i32),
        ("ritz_start", i32),
        ("cheb_ratio_coarse", C.c_double),
    ]


class StageDesc(C.Structure):
    """``tp3d_stage_desc`` of include/topo3d_b200.h."""

    _fields_ = [
        ("ncases", i32),
        ("rmin", f64), ("beta", f64), ("eta", f64), ("penal", f64), ("move", f64),
        ("target_free_volume", f64), ("tolx", f64),
        ("max_bisection", i32),
        ("bisection_tol", f64),
        ("F", vp), ("U", vp), ("U_prev", vp), ("U_bak", vp),
        ("x", vp), ("x_new", vp), ("rho_f", vp), ("rho_p", vp), ("dproj", vp), ("rho_new", vp),
        ("dc_dx", vp), ("dc_acc", vp), ("dv_dx", vp), ("ce", vp),
        ("c", vp),
        ("Hs", vp),
        ("solid", vp), ("void_", vp), ("free_mask", vp),
        ("KE_host", vp),
        ("sens_scratch", vp), ("oc_scratch", vp),
        ("oc_stats", vp),
        ("record", vp),
        ("counters", vp),
    ]


# name -> (restype, argtypes); must match include/topo3d_b200.h
SIGNATURES = {
    "tp3d_last_error": (C.c_char_p, []),
    "tp3d_abi_version": (i32, []),
    "tp3d_launch_count": (i64, []),
    "tp3d_filter_rowsum": (i32, [i32, i32, i32, f64, vp, vp]),
    "tp3d_filter_project": (i32, [i32, i32, i32, f64, vp, vp, f64, f64, vp, vp, vp, vp, vp, vp]),
    "tp3d_filter_transpose": (i32, [i32, i32, i32, f64, vp, vp, vp, vp, vp]),
    "tp3d_heaviside": (i32, [vp, i64, f64, f64, vp, vp, vp]),
    "tp3d_element_compliance": (i32, [i32, i32, i32, vp, vp, vp, vp]),
    "tp3d_sensitivity_scratch_bytes": (sz, [i32, i32, i32]),
    "tp3d_sensitivity": (i32, [i32, i32, i32, f64, vp, vp, vp, vp, vp, vp, f64, vp, vp, vp, vp, vp, vp]),
    "tp3d_oc_scratch_bytes": (sz, [i32, i32, i32, f64]),
    "tp3d_oc_update": (i32, [i32, i32, i32, f64, vp, vp, vp, vp, vp, vp, f64, f64, f64, f64, i32, f64, vp, vp,
                             vp, vp, vp]),
    "tp3d_oc_noalloc_max_elements": (i64, []),
    "tp3d_oc_update_noalloc": (i32, [i32, i32, i32, f64, vp, vp, vp, vp, vp, vp, f64, f64, f64, f64, i32, f64, vp,
                                     vp, vp, vp]),
    "tp3d_debug_expire_oc_waits": (i32, [i64, i32]),
    "tp3d_obstacle_mask": (i32, [i32, i32, i32, vp, i32, vp, vp]),
    "tp3d_solver_default_opts": (None, [C.POINTER(SolverOpts)]),
    "tp3d_solver_create": (i32, [i32, i32, i32, vp, vp, C.POINTER(SolverOpts), vp, C.POINTER(vp)]),
    "tp3d_solver_destroy": (i32, [vp]),
    "tp3d_solver_set_density": (i32, [vp, vp, f64]),
    "tp3d_solver_solve": (i32, [vp, vp, vp, C.POINTER(i32), C.POINTER(f64)]),
    "tp3d_solver_solve_begin": (i32, [vp, vp, vp]),
    "tp3d_solver_solve_end": (i32, [vp, C.POINTER(i32), C.POINTER(f64), C.POINTER(i32)]),
    "tp3d_solver_apply_f64": (i32, [vp, vp, vp]),
    "tp3d_solver_apply_f32": (i32, [vp, vp, vp]),
    "tp3d_solver_apply_level_f32": (i32, [vp, i32, vp, vp]),
    "tp3d_solver_ritz_start": (i32, [vp, vp, vp, vp, i32]),
    "tp3d_solver_time_apply": (i32, [vp, i32, i32, C.POINTER(f64)]),
    "tp3d_solver_autotune": (i32, [vp, vp, vp, i32, C.POINTER(f64), i32]),
    "tp3d_solver_time_level": (i32, [vp, i32, i32, i32, C.POINTER(f64), C.POINTER(f64)]),
    "tp3d_solver_stats": (i32, [vp, C.POINTER(f64), i32]),
    "tp3d_warm_start": (i32, [vp, vp, i64, i32, vp]),
    "tp3d_stage_capture": (i32, [vp, C.POINTER(StageDesc), vp, C.POINTER(vp)]),
    "tp3d_stage_run": (i32, [vp, vp, C.POINTER(i32), C.POINTER(i32)]),
    "tp3d_stage_count_launches": (i32, [vp, i64, i64]),
    "tp3d_stage_destroy": (i32, [vp]),
    "tp3d_batch_capture": (i32, [C.POINTER(vp), C.POINTER(StageDesc), i32, vp, C.POINTER(vp)]),
    "tp3d_batch_run": (i32, [vp, vp]),
    "tp3d_batch_count_launches": (i32, [vp, C.POINTER(i64), C.POINTER(i64)]),
    "tp3d_batch_destroy": (i32, [vp]),
}

_lib = None
_lock = threading.Lock()


class Topo3dError(RuntimeError):
    """Raised when a library call reports a CUDA error or a device-side timeout."""


def lib() -> C.CDLL:
    """Load the shared library (once); raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"{LIB_PATH} is missing: build it with `python -m pytopo3d_b200._build`")
            L = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def last_error() -> str:
    msg = lib().tp3d_last_error()
    return msg.decode() if msg else ""


def check(rc: int, what: str) -> int:
    """Map a status to the reference's exception types (ValueError / RuntimeError)."""
    if rc == TP3D_OK or rc == TP3D_NOT_CONVERGED:
        return rc
    msg = last_error()
    if rc == TP3D_ERR_ARG:
        raise ValueError(f"{what}: {msg or 'invalid argument'}")
    if rc == TP3D_ERR_NONFINITE:
        raise RuntimeError(f"{what}: {msg or 'non-finite value'}")
    if rc == TP3D_ERR_TIMEOUT:
        raise Topo3dError(f"{what}: bounded device wait expired")
    raise Topo3dError(f"{what}: CUDA error ({msg})")


def ptr(t) -> int | None:
    """Raw device pointer of a torch tensor (None passes NULL)."""
    if t is None:
        return None
    return t.data_ptr()


def stream_ptr():
    import torch

    return torch.cuda.current_stream().cuda_stream
