"""B200-native hp-FEM hexahedral assembly with the Hermes3D call surface.

Host objects (Mesh, H1Space, Discretization) run their one-time set-up in
C++ (libh3dg.so); assembly runs as sm_100a kernels.  See include/h3dg.h for
the C ABI.
"""
from . import _capi
from .discretization import (BC_ESSENTIAL, BC_NATURAL, BC_NONE, DF_HERMES_BIN, DF_MATLAB_SPARSE, DF_PLAIN_ASCII, Discretization, H1Space,
                             UMFPackMatrix,
                             UMFPackVector, UnsupportedForm, int_F_v, int_grad_u_grad_v,
                             int_grad_u_grad_v_plus_u_v, int_u_v, surf_int_G_v, surf_int_u_v,
                             SystemDiscretization)
from .mesh import Mesh, load_mesh3d, permute_vertices, unit_cube

H3dgError = _capi.H3dgError
PREC_FP64 = _capi.PREC_FP64
PREC_TF32X3 = _capi.PREC_TF32X3
PREC_OZAKI = _capi.PREC_OZAKI

__all__ = [
    "Mesh", "load_mesh3d", "unit_cube", "permute_vertices", "H1Space", "Discretization", "UMFPackMatrix",
    "UMFPackVector", "int_grad_u_grad_v", "int_grad_u_grad_v_plus_u_v", "int_F_v", "UnsupportedForm",
    "surf_int_u_v", "surf_int_G_v", "int_u_v", "SystemDiscretization",
    "BC_ESSENTIAL", "BC_NATURAL", "BC_NONE", "PREC_FP64", "PREC_TF32X3", "PREC_OZAKI", "H3dgError",
    "DF_HERMES_BIN", "DF_MATLAB_SPARSE", "DF_PLAIN_ASCII",
]
