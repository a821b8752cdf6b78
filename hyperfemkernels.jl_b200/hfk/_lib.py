"""ctypes binding of ``libhfk.so`` (the C ABI declared in ``include/hfk.h``).

This is the Python stand-in for the ``ccall``s the Julia host makes. Vector arguments may be numpy
arrays (host memory) or CUDA tensors/arrays exposing ``data_ptr()`` (device memory); the library
detects which. There is no CPU fallback: loading fails loudly if the library is missing.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("HFK_LIB", os.path.join(_HERE, "libhfk.so"))

HFK_OK = 0
LAW_SVK = 1
LAW_LINEAR_ELASTIC = 2
MF_STORED = 0
MF_RECOMPUTE = 1
FP64 = 0
FP32 = 1
SCATTER_AUTO = 0
SCATTER_COLOURED = 1
SCATTER_ATOMIC = 2
COARSE_CHOLESKY = 0
COARSE_CG = 1
EIG_EUCLIDEAN = 0
EIG_PRECONDITIONED = 1
SLOT_LAGGED_ASSEMBLED = 0
SLOT_BLOCK_JACOBI = 1

_vp = ctypes.c_void_p
_i = ctypes.c_int
_i64 = ctypes.c_int64
_d = ctypes.c_double
_pi = ctypes.POINTER(ctypes.c_int)
_pi64 = ctypes.POINTER(ctypes.c_int64)
_pd = ctypes.POINTER(ctypes.c_double)

# name -> argtypes (every function returns int)
SIGNATURES = {
    "hfk_version": [],
    "hfk_problem_create": [ctypes.POINTER(_vp), _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _i, _vp, _i],
    "hfk_problem_destroy": [_vp],
    "hfk_problem_set_params": [_vp, _vp, _i],
    "hfk_problem_set_stream": [_vp, _vp],
    "hfk_problem_info": [_vp, _pi64, _pi, _pi, _pi, _pi64],
    "hfk_problem_set_scatter": [_vp, _i],
    "hfk_problem_set_launch": [_vp, _i, _i],
    "hfk_problem_set_assembly_kernel": [_vp, _i],
    "hfk_problem_set_solve_graph": [_vp, _i],
    "hfk_mf_apply_many": [_vp, _i, _vp, _vp],
    "hfk_problem_tuning": [_vp, _i, _i, _pi, _pi, _pi],
    "hfk_functional": [_vp, _vp, _vp, _i, _pd],
    "hfk_launch_count": [_vp, _pi64],
    "hfk_problem_set_timing": [_vp, _i],
    "hfk_problem_device_errors": [_vp, _pi],
    "hfk_problem_kernel_time": [_vp, _pd, _pi64],
    "hfk_device_peak_fp64": [_pd, _pd],
    "hfk_colors": [_vp, _vp],
    "hfk_pattern_build": [_vp, _pi64],
    "hfk_pattern_get": [_vp, _vp, _vp],
    "hfk_nonzero_positions": [_vp, _vp],
    "hfk_residual": [_vp, _vp, _vp, _vp],
    "hfk_jacobian": [_vp, _vp, _vp, _vp],
    "hfk_mf_prepare": [_vp, _vp, _vp, _i],
    "hfk_mf_apply": [_vp, _vp, _vp],
    "hfk_mf_apply_f32": [_vp, _vp, _vp],
    "hfk_blocks_update": [_vp, _pi],
    "hfk_blocks_apply": [_vp, _vp, _vp],
    "hfk_blocks_get": [_vp, _pi, _vp, _vp, _vp],
    "hfk_blocks_set": [_vp, _vp, _pi],
    "hfk_eigenvalue_bounds": [_vp, _i, _vp, _pd, _pd],
    "hfk_hessenberg_eigvals": [_i, _vp, _vp, _vp],
    "hfk_chebyshev_smooth": [_vp, _d, _d, _i, _vp, _vp, _i, _vp],
    "hfk_chebyshev_smooth_noalloc": [_vp, _d, _d, _i, _vp, _vp, _i, _vp],
    "hfk_transfer_create": [ctypes.POINTER(_vp), _vp, _vp, _vp, _vp],
    "hfk_transfer_destroy": [_vp],
    "hfk_transfer_set_multiplicity": [_vp, _vp],
    "hfk_prolongate": [_vp, _vp, _vp],
    "hfk_restrict": [_vp, _vp, _vp],
    "hfk_inject": [_vp, _vp, _vp, _vp, _vp],
    "hfk_pmg_create": [ctypes.POINTER(_vp), _i, _vp, _vp, _i, _d, _d, _i, _i, _i],
    "hfk_pmg_destroy": [_vp],
    "hfk_pmg_update": [_vp, _vp, _vp, _pi],
    "hfk_pmg_vcycle": [_vp, _vp, _vp],
    "hfk_pmg_level_info": [_vp, _i, _pd, _pd, _pd, _pd],
    "hfk_pmg_stats": [_vp, _vp],
    "hfk_pmg_status": [_vp, _pi, _pi],
    "hfk_solve_cg": [_vp, _vp, _vp, _vp, _d, _d, _i, _i, _pi, _pi, _pi, _pd],
    "hfk_solve_gmres": [_vp, _vp, _vp, _vp, _d, _d, _i, _i, _i, _pi, _pi, _pd],
    "hfk_slot_create": [ctypes.POINTER(_vp), _vp, _i, _i],
    "hfk_mlp_create": [ctypes.POINTER(_vp), ctypes.c_uint64],
    "hfk_mlp_destroy": [_vp],
    "hfk_mlp_num_params": [],
    "hfk_mlp_get_weights": [_vp, _vp],
    "hfk_mlp_set_weights": [_vp, _vp],
    "hfk_mlp_forward": [_vp, _vp, _i64, _vp],
    "hfk_mlp_grad": [_vp, _vp, _vp, _i64, _vp, _vp],
    "hfk_mlp_train": [_vp, _vp, _vp, _i64, _i, _i64, ctypes.c_float, _vp],
    "hfk_pmg_set_mlp": [_vp, _vp],
    "hfk_pmg_mlp_stats": [_vp, _pi64, _pi64],
    "hfk_pmg_mlp_sample": [_vp, _vp, _vp, _vp, _pi, _d],
    "hfk_pmg_set_coarse": [_vp, _i, _i],
    "hfk_pmg_test_coarse_wait": [_vp, _i, _i],
    "hfk_pmg_segment_bounds": [_vp, _i, _vp, _vp],
    "hfk_pmg_set_eig_inner": [_vp, _i],
    "hfk_oseen_create": [ctypes.POINTER(_vp), _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _vp, _i],
    "hfk_oseen_destroy": [_vp],
    "hfk_oseen_set_params": [_vp, _vp, _i],
    "hfk_oseen_set_scatter": [_vp, _i],
    "hfk_oseen_set_history": [_vp, _vp, _vp, _vp, _vp],
    "hfk_oseen_pattern": [_vp, _pi64],
    "hfk_oseen_pattern_get": [_vp, _vp, _vp],
    "hfk_oseen_residual": [_vp, _vp, _vp, _vp],
    "hfk_oseen_jacobian": [_vp, _vp],
    "hfk_oseen_launch_count": [_vp, _pi64],
    "hfk_oseen_set_outlet": [_vp, _i, _vp, _vp, _vp, _vp, _i, _vp, _vp, _d, _d],
    "hfk_problem_set_segments": [_vp, _i, _vp, _vp, _vp],
    "hfk_problem_segments": [_vp, _pi],
    "hfk_problem_set_cell_params": [_vp, _vp],
    "hfk_segment_dots": [_vp, _vp, _vp, _vp],
    "hfk_segment_scale": [_vp, _vp, _vp],
    "hfk_solve_cg_batched": [_vp, _vp, _vp, _vp, _d, _d, _i, _i, _vp, _vp, _vp, _vp, _pi],
}

_LIB = None


class HFKError(RuntimeError):
    """An error status from the library (message prefixed "HyperFEMKernels: ")."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


def lib():
    """The loaded library; raises if ``libhfk.so`` was not built (no silent fallback)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"HyperFEMKernels: {LIB_PATH} is missing; build it with __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        L.hfk_last_error.argtypes = []
        L.hfk_last_error.restype = ctypes.c_char_p
        _LIB = L
    return _LIB


# Destruction order of handles that refer to one another. A hierarchy (hfk_pmg) reads its level
# problems when it is destroyed, so every level problem must outlive the hierarchies built on it.
# Holding a reference does not guarantee that in Python: the cyclic garbage collector finalises the
# objects of a reference cycle (a test frame kept alive by a caught exception's traceback, say) in
# no particular order. The binding therefore orders it: a problem whose owner is finalised while
# hierarchies still use it is destroyed when the last of those hierarchies is.
_users: dict = {}     # problem handle (int) -> live hierarchies that use it
_pending: set = set()  # problem handles whose owner is gone, waiting for their hierarchies
_order_lock = threading.Lock()


def retain_problem(hv: int) -> None:
    """A hierarchy starts using problem handle ``hv``."""
    with _order_lock:
        _users[hv] = _users.get(hv, 0) + 1


def release_problem(hv: int) -> None:
    """A hierarchy that used ``hv`` is destroyed; destroy ``hv`` too if its owner already went."""
    with _order_lock:
        n = _users.get(hv, 0) - 1
        if n > 0:
            _users[hv] = n
            return
        _users.pop(hv, None)
        if hv not in _pending:
            return
        _pending.discard(hv)
    lib().hfk_problem_destroy(ctypes.c_void_p(hv))


def destroy_problem(hv: int) -> None:
    """The owner of problem handle ``hv`` is finalised: destroy it now, or once no hierarchy uses it."""
    with _order_lock:
        if _users.get(hv, 0) > 0:
            _pending.add(hv)
            return
    lib().hfk_problem_destroy(ctypes.c_void_p(hv))


def call(name, *args):
    """Call an ABI function and raise ``HFKError`` on a non-zero status."""
    L = lib()
    rc = getattr(L, name)(*args)
    if rc != HFK_OK:
        raise HFKError(rc, L.hfk_last_error().decode())
    return rc


def ptr(a, dtype=np.float64):
    """Address of a numpy array (checked dtype/contiguity) or a CUDA tensor (``data_ptr()``).

    The returned ``c_void_p`` holds a reference to the array, so a temporary passed straight into
    a call (``call(..., ptr(np.asfortranarray(x)))``) stays alive until the call returns; a bare
    address would let the temporary be freed, and its memory reused, before the library reads it.
    """
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        import torch  # only when a tensor is passed

        want = {np.float64: torch.float64, np.float32: torch.float32, np.int32: torch.int32,
                np.int64: torch.int64}[np.dtype(dtype).type]
        if a.dtype != want or not a.is_contiguous():
            raise TypeError(f"HyperFEMKernels: expected a contiguous {want} tensor")
        p = ctypes.c_void_p(a.data_ptr())
    else:
        if not isinstance(a, np.ndarray):
            raise TypeError("HyperFEMKernels: expected a numpy array or a CUDA tensor")
        if a.dtype != np.dtype(dtype):
            raise TypeError(f"HyperFEMKernels: expected dtype {np.dtype(dtype)}, got {a.dtype}")
        if not (a.flags.c_contiguous or a.flags.f_contiguous):
            raise TypeError("HyperFEMKernels: expected a contiguous array")
        p = ctypes.c_void_p(a.ctypes.data)
    p._owner = a
    return p
