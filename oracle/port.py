"""ctypes wrapper of the plain-C restatement oracle (oracle/port/h3d_port.c).

ORACLE / TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke()
and bench.py's CPU baseline as the checker, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "_ref", "libh3dport.so")
_lib = None


def build():
    src = os.path.join(HERE, "port", "h3d_port.c")
    if not os.path.exists(SO) or os.path.getmtime(SO) < os.path.getmtime(src):
        os.makedirs(os.path.dirname(SO), exist_ok=True)
        subprocess.run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-Wall", "-o", SO, src, "-lm"], check=True)
    return SO


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(SO)
        pd, pi64, pi32 = C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_int32)
        L.h3d_port_pattern.argtypes = [C.c_int64, pi64, pi32, C.c_int64, pi64, pi32, pi64]
        L.h3d_port_assemble.argtypes = [C.c_int64, pd, C.c_int64, pi64, pi32, pi64, pi64, pi32, pd, C.c_int, pd, C.c_int,
                                        C.c_double, C.c_int64, pi64, pi32, pd, pd]
        L.h3d_port_assemble_stock.argtypes = [C.c_int64, pd, C.c_int64, pi64, pi64, pi64, pi32, pd, C.c_int, pd, C.c_int,
                                              C.c_double, C.c_int64, pi64, pi32, pd, pd]
        L.h3d_port_element_matrix.argtypes = [pd, C.c_int, C.c_int, C.c_int, C.c_int, pi64, C.c_int, C.c_double, pd]
        L.h3d_port_element_rows.argtypes = [pd, C.c_int, C.c_int, C.c_int, C.c_int, pi64, C.c_int, pi32, C.c_int, C.c_double, pd]
        _lib = L
    return _lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def asmlists_from_space(space, ne):
    """Flatten the assembly lists of elements 1..ne (CSR over elements)."""
    ptr = [0]
    idx, dof, coef = [], [], []
    for e in range(1, ne + 1):
        i, d, c = space.get_element_assembly_list(e)
        idx.append(i)
        dof.append(d)
        coef.append(c)
        ptr.append(ptr[-1] + len(i))
    return (np.array(ptr, np.int64), np.concatenate(idx).astype(np.int64), np.concatenate(dof).astype(np.int32),
            np.concatenate(coef).astype(np.float64))


def asmlists_from_ref(ref_asm, ne):
    """Assembly lists dumped by the reference driver, reordered by element id."""
    by_id = {eid: (i, d, c) for eid, i, d, c in ref_asm}
    ptr = [0]
    idx, dof, coef = [], [], []
    for e in range(1, ne + 1):
        i, d, c = by_id[e]
        idx.append(i)
        dof.append(d)
        coef.append(c)
        ptr.append(ptr[-1] + len(i))
    return (np.array(ptr, np.int64), np.concatenate(idx).astype(np.int64), np.concatenate(dof).astype(np.int32),
            np.concatenate(coef).astype(np.float64))


def pattern(al_ptr, al_dof, ndof):
    ne = len(al_ptr) - 1
    nnz = C.c_int64()
    L = lib()
    if L.h3d_port_pattern(ne, _p(al_ptr, C.c_int64), _p(al_dof, C.c_int32), ndof, None, None, C.byref(nnz)) != 0:
        raise RuntimeError("port pattern failed")
    Ap = np.zeros(ndof + 1, np.int64)
    Ai = np.zeros(nnz.value, np.int32)
    L.h3d_port_pattern(ne, _p(al_ptr, C.c_int64), _p(al_dof, C.c_int32), ndof, _p(Ap, C.c_int64), _p(Ai, C.c_int32),
                       C.byref(nnz))
    return Ap, Ai


def assemble(xyz, hex0, nq, al, ndof, Ap, Ai, mass=False, gradcoef=None, lf=1, lf_value=1.0):
    """Numeric assembly.  hex0: ne x 8 zero-based; nq: ne x 3 points per direction
    (or a scalar / 3-tuple); al = (ptr, idx, dof, coef)."""
    xyz = np.ascontiguousarray(xyz, np.float64)
    hex0 = np.ascontiguousarray(hex0, np.int64)
    ne = len(hex0)
    nq = np.broadcast_to(np.asarray(nq, np.int32), (ne, 3)).copy()
    ptr, idx, dof, coef = al
    Ax = np.zeros(len(Ai), np.float64)
    rhs = np.zeros(ndof, np.float64)
    gc = None if gradcoef is None else np.ascontiguousarray(gradcoef, np.float64)
    r = lib().h3d_port_assemble(len(xyz), _p(xyz, C.c_double), ne, _p(hex0, C.c_int64), _p(nq, C.c_int32),
                                _p(ptr, C.c_int64), _p(idx, C.c_int64), _p(dof, C.c_int32), _p(coef, C.c_double),
                                int(mass), _p(gc, C.c_double), int(lf), float(lf_value), ndof, _p(Ap, C.c_int64),
                                _p(Ai, C.c_int32), _p(Ax, C.c_double), _p(rhs, C.c_double))
    if r != 0:
        raise RuntimeError("port assemble failed (%d)" % r)
    return Ax, rhs


def assemble_stock(xyz, hex0, al, ndof, Ap, Ai, mass=False, gradcoef=None, lf=1, lf_value=1.0):
    """Numeric assembly with the reference's stock per-pair quadrature."""
    xyz = np.ascontiguousarray(xyz, np.float64)
    hex0 = np.ascontiguousarray(hex0, np.int64)
    ptr, idx, dof, coef = al
    Ax = np.zeros(len(Ai), np.float64)
    rhs = np.zeros(ndof, np.float64)
    gc = None if gradcoef is None else np.ascontiguousarray(gradcoef, np.float64)
    r = lib().h3d_port_assemble_stock(len(xyz), _p(xyz, C.c_double), len(hex0), _p(hex0, C.c_int64),
                                      _p(ptr, C.c_int64), _p(idx, C.c_int64), _p(dof, C.c_int32), _p(coef, C.c_double),
                                      int(mass), _p(gc, C.c_double), int(lf), float(lf_value), ndof, _p(Ap, C.c_int64),
                                      _p(Ai, C.c_int32), _p(Ax, C.c_double), _p(rhs, C.c_double))
    if r != 0:
        raise RuntimeError("port assemble_stock failed (%d)" % r)
    return Ax, rhs


def element_matrix(X, nq, idx, mass=False, gradcoef=1.0):
    X = np.ascontiguousarray(X, np.float64).reshape(8, 3)
    idx = np.ascontiguousarray(idx, np.int64)
    n = len(idx)
    K = np.zeros((n, n), np.float64)
    nqx, nqy, nqz = (nq, nq, nq) if np.isscalar(nq) else nq
    lib().h3d_port_element_matrix(_p(X, C.c_double), nqx, nqy, nqz, n, _p(idx, C.c_int64), int(mass), float(gradcoef),
                                  _p(K, C.c_double))
    return K


def element_rows(X, nq, idx, rows, mass=False, gradcoef=1.0):
    """Rows (test indices into idx) of the element matrix, all columns."""
    X = np.ascontiguousarray(X, np.float64).reshape(8, 3)
    idx = np.ascontiguousarray(idx, np.int64)
    rows = np.ascontiguousarray(rows, np.int32)
    out = np.zeros((len(rows), len(idx)), np.float64)
    nqx, nqy, nqz = (nq, nq, nq) if np.isscalar(nq) else nq
    lib().h3d_port_element_rows(_p(X, C.c_double), nqx, nqy, nqz, len(idx), _p(idx, C.c_int64), len(rows),
                                _p(rows, C.c_int32), int(mass), float(gradcoef), _p(out, C.c_double))
    return out
