"""ctypes binding of the C ABI declared in include/h3dg.h.

The shared library is built in-tree (``hermes3d_b200/libh3dg.so``, see
``hermes3d_b200.build``).  Loading fails loudly if it is missing: there is
no pure-Python or CPU fallback for the assembly path.
"""
from __future__ import annotations

import ctypes as C
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libh3dg.so")

H3DG_OK = 0
H3DG_ERR_INVALID_ARG = 1
H3DG_ERR_STATE = 6
H3DG_ERR_TIMEOUT = 7
H3DG_ERR_TOO_LARGE = 8
DEBUG_WAIT_GIVES_UP = 1
DEBUG_CORRUPT_POSITION = 2
STATUS = {
    0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of memory", 4: "unsupported form",
    5: "mesh error", 6: "call out of order", 7: "device wait timed out", 8: "size limit exceeded",
}

BC_ESSENTIAL, BC_NATURAL, BC_NONE = 0, 1, 2
BF_GRAD_GRAD, BF_GRAD_GRAD_MASS = 1, 2
LF_NONE, LF_CONST, LF_SIN = 0, 1, 2
SBF_U_V, SLF_G_V = 1, 1
QUAD_FIXED, QUAD_P_PLUS = 0, 1
QUAD_STOCK = 2
PREC_FP64 = 0
PREC_TF32X3 = 1
PREC_OZAKI = 2
NOALLOC_SCRATCH_DOUBLES = 2 << 20

BC_TYPE_FN = C.CFUNCTYPE(C.c_int, C.c_int, C.c_void_p)
BC_VALUE_FN = C.CFUNCTYPE(C.c_double, C.c_int, C.c_double, C.c_double, C.c_double, C.c_void_p)

_p = C.c_void_p
_i64 = C.c_int64
_i32 = C.c_int32
_pd = C.POINTER(C.c_double)
_pi64 = C.POINTER(C.c_int64)
_pi32 = C.POINTER(C.c_int32)

# name -> argtypes (restype is int status unless listed in _RESTYPES)
SIGNATURES = {
    "h3dg_version": [],
    "h3dg_status_string": [C.c_int],
    "h3dg_last_error": [],
    "h3dg_mesh_create": [C.POINTER(_p)],
    "h3dg_mesh_destroy": [_p],
    "h3dg_mesh_add_vertices": [_p, _pd, _i64],
    "h3dg_mesh_add_hexes": [_p, _pi64, _i64],
    "h3dg_mesh_add_quad_boundaries": [_p, _pi64, _pi32, _i64],
    "h3dg_mesh_finalize": [_p],
    "h3dg_mesh_counts": [_p, _pi64, _pi64, _pi64, _pi64],
    "h3dg_mesh_refine_element": [_p, _i64, C.c_int],
    "h3dg_disc_set_surface_forms": [_p, C.c_int, C.c_int, _pd, C.c_int],
    "h3dg_disc_norms": [_p, _p, C.c_int, _pd, _p],
    "h3dg_disc_solve_cg": [_p, _p, _p, _p, C.c_double, C.c_int, _pi32, _pd, _p],
    "h3dg_mesh_refine_elements": [_p, _pi64, _i64, C.c_int],
    "h3dg_mesh_get_arrays": [_p, _pd, _pi64, _pi64],
    "h3dg_space_create": [_p, C.POINTER(_p)],
    "h3dg_space_destroy": [_p],
    "h3dg_space_set_bc_types": [_p, BC_TYPE_FN, _p],
    "h3dg_space_set_bc_values": [_p, BC_VALUE_FN, _p],
    "h3dg_space_set_uniform_order": [_p, C.c_int, C.c_int, C.c_int],
    "h3dg_space_set_element_orders": [_p, _pi32, _i64],
    "h3dg_space_assign_dofs": [_p, C.c_int, C.c_int, _pi64],
    "h3dg_space_get_element_assembly_list": [_p, _i64, _pi64, _pi32, _pd, _i32, _pi32],
    "h3dg_disc_create": [C.POINTER(_p), C.c_int],
    "h3dg_disc_destroy": [_p],
    "h3dg_disc_set_space": [_p, _p],
    "h3dg_disc_set_test_space": [_p, _p],
    "h3dg_disc_set_bilinear_form": [_p, C.c_int, _pd, _i64],
    "h3dg_disc_set_linear_form": [_p, C.c_int, C.c_double],
    "h3dg_disc_set_quadrature": [_p, C.c_int, C.c_int],
    "h3dg_disc_create_pattern": [_p, _pi64, _pi64],
    "h3dg_disc_get_pattern": [_p, _pi64, _pi32],
    "h3dg_disc_assemble": [_p, C.c_int, _p, _p, _p],
    "h3dg_disc_assemble_host": [_p, C.c_int, _pd, _pd],
    "h3dg_disc_update_vertices": [_p, _pd, _i64],
    "h3dg_disc_update_coefficients": [_p, _pd, _i64],
    "h3dg_disc_update_coefficients_device": [_p, _p, _i64, _p],
    "h3dg_disc_last_launch_count": [_p, _pi32],
    "h3dg_disc_last_kernel": [_p, _pi32],
    "h3dg_disc_geometry": [_p, _p, _p, _p, _p],
    "h3dg_disc_adjoint": [_p, C.c_int, _p, _p, _p, _p, _p, _p],
    "h3dg_tc_selftest": [C.c_int, _p, _p, _p, C.c_int],
    "h3dg_disc_assemble_host_noalloc": [_p, C.c_int, _p, _p],
    "h3dg_disc_set_partition": [_p, C.c_int, C.c_int],
    "h3dg_disc_set_precision": [_p, C.c_int],
    "h3dg_disc_get_partition": [_p, _p, _p, _p, _p],
    "h3dg_disc_get_partition_elements": [_p, _p, C.c_int64],
    "h3dg_disc_enable_kernel_timing": [_p, _i32],
    "h3dg_disc_get_tuning": [_p, _pi32, _pi32, C.POINTER(C.c_float)],
    "h3dg_disc_tuned_scatter": [_p, _pi32],
    "h3dg_disc_seg_stats": [_p, C.POINTER(C.c_int64)],
    "h3dg_disc_kernel_times": [_p, C.POINTER(C.c_float), _i32, _pi32],
    "h3dg_disc_debug_inject": [_p, C.c_int],
}
_RESTYPES = {"h3dg_status_string": C.c_char_p, "h3dg_last_error": C.c_char_p}

_lib = None


class H3dgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s (%d): %s" % (STATUS.get(status, "?"), status, msg))
        self.status = status


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libh3dg.so not built: run `python -m hermes3d_b200.build` (no CPU fallback exists)")
        L = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = _RESTYPES.get(name, C.c_int)
        _lib = L
    return _lib


def check(status):
    if status != H3DG_OK:
        raise H3dgError(status, lib().h3dg_last_error().decode())
    return status


def call(name, *args):
    return check(getattr(lib(), name)(*args))


def ptr(arr, ctype):
    """ctypes pointer to a contiguous numpy array (or None)."""
    if arr is None:
        return None
    return arr.ctypes.data_as(C.POINTER(ctype))
