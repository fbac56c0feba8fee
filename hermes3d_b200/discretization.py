"""Reference-shaped host API over the C ABI: H1Space, weak-form descriptors,
Discretization, UMFPackMatrix / UMFPackVector.

Mirrors src/space.h, src/space/h1.h, src/discretization.h and
src/linsolver/umfpack.h of the reference: the same method names, argument
meaning and call order (set_* -> assign_dofs -> create -> assemble).  The
reference's forms are C function pointers evaluated on the CPU; here the
stock forms of src/integrals/h1.h are named by descriptor objects and run
on the GPU.  An unknown form raises UnsupportedForm; nothing falls back
to the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np

from . import _capi as capi

BC_ESSENTIAL = capi.BC_ESSENTIAL
BC_NATURAL = capi.BC_NATURAL
BC_NONE = capi.BC_NONE


class UnsupportedForm(capi.H3dgError):
    pass


class H1Space:
    """H1 space on hexahedra with the hierarchical Lobatto shapeset
    (H1Space + H1ShapesetLobattoHex, src/space/h1.h, src/shapeset/h1lobattohex.h)."""

    def __init__(self, mesh):
        if mesh.handle is None:
            mesh.ugh()
        self.mesh = mesh
        h = C.c_void_p()
        capi.call("h3dg_space_create", mesh.handle, C.byref(h))
        self.handle = h
        self._cb = []
        self.ndof = None

    def set_bc_types(self, fn: Optional[Callable[[int], int]]):
        """Space::set_bc_types; fn(marker) -> BC_ESSENTIAL / BC_NATURAL / BC_NONE."""
        if fn is None:
            capi.call("h3dg_space_set_bc_types", self.handle, capi.BC_TYPE_FN(), None)
            return
        cb = capi.BC_TYPE_FN(lambda marker, ctx: int(fn(marker)))
        self._cb.append(cb)
        capi.call("h3dg_space_set_bc_types", self.handle, cb, None)

    def set_bc_values(self, fn: Optional[Callable[[int, float, float, float], float]]):
        """Space::set_bc_values; fn(marker, x, y, z) -> Dirichlet value."""
        if fn is None:
            capi.call("h3dg_space_set_bc_values", self.handle, capi.BC_VALUE_FN(), None)
            return
        cb = capi.BC_VALUE_FN(lambda marker, x, y, z, ctx: float(fn(marker, x, y, z)))
        self._cb.append(cb)
        capi.call("h3dg_space_set_bc_values", self.handle, cb, None)

    def set_uniform_order(self, order):
        px, py, pz = (order, order, order) if np.isscalar(order) else order
        capi.call("h3dg_space_set_uniform_order", self.handle, int(px), int(py), int(pz))
        self.orders = ("uniform", (int(px), int(py), int(pz)))

    def set_element_orders(self, orders):
        o = np.ascontiguousarray(orders, dtype=np.int32).reshape(-1, 3)
        capi.call("h3dg_space_set_element_orders", self.handle, capi.ptr(o, C.c_int32), len(o))
        self.orders = ("elements", o.tobytes())

    def assign_dofs(self, first_dof=0, stride=1):
        n = C.c_int64()
        capi.call("h3dg_space_assign_dofs", self.handle, int(first_dof), int(stride), C.byref(n))
        self.ndof = n.value
        self.first_dof = int(first_dof)
        return n.value

    def get_dof_count(self):
        return self.ndof

    def get_element_assembly_list(self, elem_id):
        """AsmList of element ``elem_id`` (1-based): (idx, dof, coef) arrays."""
        cnt = C.c_int32()
        capi.call("h3dg_space_get_element_assembly_list", self.handle, int(elem_id), None, None, None, 0, C.byref(cnt))
        n = cnt.value
        idx = np.zeros(n, np.int64)
        dof = np.zeros(n, np.int32)
        coef = np.zeros(n, np.float64)
        capi.call("h3dg_space_get_element_assembly_list", self.handle, int(elem_id), capi.ptr(idx, C.c_int64),
                  capi.ptr(dof, C.c_int32), capi.ptr(coef, C.c_double), n, C.byref(cnt))
        return idx, dof, coef

    def __del__(self):
        if getattr(self, "handle", None) and capi._lib is not None:
            capi.lib().h3dg_space_destroy(self.handle)
            self.handle = None


# ---------------------------------------------------------------- form descriptors

@dataclass(frozen=True)
class BilinearForm:
    kind: int
    name: str


@dataclass(frozen=True)
class LinearForm:
    kind: int
    value: float
    name: str


int_grad_u_grad_v = BilinearForm(capi.BF_GRAD_GRAD, "int_grad_u_grad_v")
int_grad_u_grad_v_plus_u_v = BilinearForm(capi.BF_GRAD_GRAD_MASS, "int_grad_u_grad_v + int_u_v")
# int_u_v alone (src/integrals/h1.h:154-177): the grad.grad + mass kernels with a zero grad.grad coefficient
int_u_v = BilinearForm(-1, "int_u_v")


@dataclass(frozen=True)
class SurfaceBilinearForm:
    kind: int
    name: str


@dataclass(frozen=True)
class SurfaceLinearForm:
    kind: int
    g: tuple
    name: str


surf_int_u_v = SurfaceBilinearForm(capi.SBF_U_V, "surf_int_u_v")


def surf_int_G_v(g):
    """Surface linear form int G v on natural boundary faces, G constant per boundary
    marker: a dict {marker: value} or a sequence indexed by marker (markers 0..15)."""
    if isinstance(g, dict):
        vals = [0.0] * 16
        for m, v in g.items():
            if not 0 <= int(m) < 16:
                raise capi.H3dgError(1, "surface markers must be 0..15")
            vals[int(m)] = float(v)
    elif np.isscalar(g):
        vals = [float(g)] * 16
    else:
        vals = [float(v) for v in g]
        if len(vals) > 16:
            raise capi.H3dgError(1, "surface markers must be 0..15")
    return SurfaceLinearForm(capi.SLF_G_V, tuple(vals), "surf_int_G_v")


def int_F_v(F):
    """Linear form int F v for a constant F or F = "sin" (sin(pi x) sin(pi y) sin(pi z))."""
    if isinstance(F, str) and F == "sin":
        return LinearForm(capi.LF_SIN, 0.0, "int_F_v(sin)")
    if np.isscalar(F):
        return LinearForm(capi.LF_CONST, float(F), "int_F_v(%g)" % F)
    raise UnsupportedForm(capi.H3DG_OK + 4, "only constant or 'sin' sources run on the device")


# ---------------------------------------------------------------- matrix / vector sinks

# dump formats of Matrix::dump / Vector::dump (src/matrix.h:96-101)
DF_MATLAB_SPARSE, DF_PLAIN_ASCII, DF_HERMES_BIN = 0, 1, 2


def _open_for(file, mode):
    return (open(file, mode), True) if isinstance(file, (str, bytes, os.PathLike)) else (file, False)


class UMFPackMatrix:
    """CSC sink with the reference's arrays (src/linsolver/umfpack.h:26-47).
    Ap is int64 here (nnz may exceed INT_MAX)."""

    def __init__(self):
        self.Ap = None
        self.Ai = None
        self.Ax = None
        self.ndofs = 0

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csc_matrix((self.Ax, self.Ai, self.Ap), shape=(self.ndofs, self.ndofs))

    def dump(self, file, var_name, fmt=DF_MATLAB_SPARSE):
        """UMFPackMatrix::dump (src/linsolver/umfpack.cc:95-127): DF_HERMES_BIN
        writes "H2DX", the scalar size, ndofs, nnz, Ap, Ai (32-bit) and Ax;
        DF_MATLAB_SPARSE a MATLAB script of (row, column, value) triplets that
        spconvert()s into var_name.  file: a path or a file object."""
        n, nnz = int(self.ndofs), int(self.Ap[-1])
        if fmt == DF_HERMES_BIN:
            if nnz >= 2 ** 31:
                raise ValueError("H2DX stores 32-bit column pointers: nnz >= 2^31")
            f, own = _open_for(file, "wb")
            try:
                f.write(b"H2DX\x01\x00\x00\x00")
                f.write(np.array([8, n, nnz], np.int32).tobytes())
                f.write(np.asarray(self.Ap, np.int32).tobytes())
                f.write(np.asarray(self.Ai, np.int32).tobytes())
                f.write(np.asarray(self.Ax, np.float64).tobytes())
            finally:
                if own:
                    f.close()
            return True
        if fmt == DF_MATLAB_SPARSE:
            f, own = _open_for(file, "w")
            try:
                f.write("%% Size: %dx%d\n%% Nonzeros: %d\ntemp = zeros(%d, 3);\ntemp = [\n" % (n, n, nnz, nnz))
                cols = np.repeat(np.arange(n), np.diff(self.Ap))
                f.writelines("%d %d %f\n" % (i + 1, j + 1, x) for i, j, x in zip(self.Ai, cols, self.Ax))
                f.write("];\n%s = spconvert(temp);\n" % var_name)
            finally:
                if own:
                    f.close()
            return True
        if fmt == DF_PLAIN_ASCII:                # the reference exits with ERR_NOT_IMPLEMENTED
            raise NotImplementedError("DF_PLAIN_ASCII dump")
        return False

    @staticmethod
    def load(file):
        """Read an H2DX dump (the reference's or ours) back into a matrix."""
        f, own = _open_for(file, "rb")
        try:
            head = f.read(8)
            if head[:4] != b"H2DX":
                raise ValueError("not an H2DX dump")
            ssize, n, nnz = np.frombuffer(f.read(12), np.int32)
            if ssize != 8:
                raise ValueError("real (8-byte) scalars only")
            m = UMFPackMatrix()
            m.ndofs = int(n)
            m.Ap = np.frombuffer(f.read(4 * (n + 1)), np.int32).astype(np.int64)
            m.Ai = np.frombuffer(f.read(4 * nnz), np.int32).copy()
            m.Ax = np.frombuffer(f.read(8 * nnz), np.float64).copy()
            return m
        finally:
            if own:
                f.close()


class UMFPackVector:
    def __init__(self):
        self.v = None

    def dump(self, file, var_name, fmt=DF_MATLAB_SPARSE):
        """UMFPackVector::dump (src/linsolver/umfpack.cc:194-220): "H2DR", the
        scalar size, ndofs, v; or a MATLAB column vector."""
        n = len(self.v)
        if fmt == DF_HERMES_BIN:
            f, own = _open_for(file, "wb")
            try:
                f.write(b"H2DR\x01\x00\x00\x00")
                f.write(np.array([8, n], np.int32).tobytes())
                f.write(np.asarray(self.v, np.float64).tobytes())
            finally:
                if own:
                    f.close()
            return True
        if fmt == DF_MATLAB_SPARSE:
            f, own = _open_for(file, "w")
            try:
                f.write("%% Size: %dx1\n%s = [\n" % (n, var_name))
                f.writelines("%f\n" % x for x in self.v)
                f.write(" ];\n")
            finally:
                if own:
                    f.close()
            return True
        if fmt == DF_PLAIN_ASCII:                # the reference exits with ERR_NOT_IMPLEMENTED
            raise NotImplementedError("DF_PLAIN_ASCII dump")
        return False

    @staticmethod
    def load(file):
        """Read an H2DR dump back into a vector."""
        f, own = _open_for(file, "rb")
        try:
            head = f.read(8)
            if head[:4] != b"H2DR":
                raise ValueError("not an H2DR dump")
            ssize, n = np.frombuffer(f.read(8), np.int32)
            if ssize != 8:
                raise ValueError("real (8-byte) scalars only")
            vec = UMFPackVector()
            vec.v = np.frombuffer(f.read(8 * n), np.float64).copy()
            return vec
        finally:
            if own:
                f.close()


class Discretization:
    """Single-equation Discretization (src/discretization.h:39-101) on one GPU."""

    def __init__(self, device=0):
        h = C.c_void_p()
        capi.call("h3dg_disc_create", C.byref(h), int(device))
        self.handle = h
        self.device = device
        self.space = None
        self.ndof = None
        self.nnz = None
        self._quad = (capi.QUAD_P_PLUS, 2)

    def set_num_equations(self, neq):
        if neq != 1:
            raise capi.H3dgError(1, "only one equation is supported")

    def set_spaces(self, space):
        self.space = space
        capi.call("h3dg_disc_set_space", self.handle, space.handle)

    def set_test_space(self, space):
        """Block (m, n) of a system whose test space differs from the trial
        space set by set_spaces (no reference counterpart as a call: the
        reference's Discretization does this per block inside assemble).
        Rows then come from ``space``, each space counted from its own first
        DOF; FP64.  None: one space."""
        self._test_space = space
        capi.call("h3dg_disc_set_test_space", self.handle, None if space is None else space.handle)

    def set_pss(self, *args):
        pass  # the precalculated shapeset is the device's 1D tables

    def set_bilinear_form(self, form, coef=None, surf=None):
        """set_bilinear_form(0, 0, unsym, sym, surf): ``surf`` = surf_int_u_v or None."""
        if not isinstance(form, BilinearForm):
            raise UnsupportedForm(4, "bilinear form %r is not one of the device forms" % (form,))
        if surf is not None and not isinstance(surf, SurfaceBilinearForm):
            raise UnsupportedForm(4, "surface form %r is not one of the device forms" % (surf,))
        c = None if coef is None else np.ascontiguousarray(coef, dtype=np.float64)
        kind = form.kind
        if form is int_u_v:
            if self.space is None:
                raise capi.H3dgError(6, "set_spaces() before set_bilinear_form(int_u_v)")
            kind, c = capi.BF_GRAD_GRAD_MASS, np.zeros(self.space.mesh.num_elements, np.float64)
        capi.call("h3dg_disc_set_bilinear_form", self.handle, kind,
                  capi.ptr(c, C.c_double), 0 if c is None else len(c))
        self._coef = c
        self._bf_kind = kind
        self._sbf = surf
        self._set_surface()

    def set_linear_form(self, form, surf=None):
        """set_linear_form(0, lf, surf): ``surf`` = surf_int_G_v(g) or None."""
        if surf is not None and not isinstance(surf, SurfaceLinearForm):
            raise UnsupportedForm(4, "surface form %r is not one of the device forms" % (surf,))
        self._lf = form
        self._slf = surf
        self._set_surface()
        if form is None:
            capi.call("h3dg_disc_set_linear_form", self.handle, capi.LF_NONE, 0.0)
            return
        if not isinstance(form, LinearForm):
            raise UnsupportedForm(4, "linear form %r is not one of the device forms" % (form,))
        capi.call("h3dg_disc_set_linear_form", self.handle, form.kind, form.value)

    def _set_surface(self):
        sbf, slf = getattr(self, "_sbf", None), getattr(self, "_slf", None)
        g = np.ascontiguousarray(slf.g if slf is not None else [], dtype=np.float64)
        capi.call("h3dg_disc_set_surface_forms", self.handle, capi.SBF_U_V if sbf is not None else 0,
                  capi.SLF_G_V if slf is not None else 0, capi.ptr(g, C.c_double) if len(g) else None, len(g))

    def solve(self, Ax, rhs, x=None, rtol=1e-12, maxit=10000, stream=None):
        """Jacobi-preconditioned CG on the device for the assembled system (torch CUDA
        float64 tensors Ax, rhs in the plan's layout); returns (x, iterations, relres)."""
        import torch
        if x is None:
            x = torch.zeros_like(rhs)
        if stream is None:
            stream = torch.cuda.current_stream(rhs.device)
        it = C.c_int32()
        rr = C.c_double()
        capi.call("h3dg_disc_solve_cg", self.handle, C.c_void_p(Ax.data_ptr()), C.c_void_p(rhs.data_ptr()),
                  C.c_void_p(x.data_ptr()), float(rtol), int(maxit), C.byref(it), C.byref(rr),
                  C.c_void_p(stream.cuda_stream))
        return x, it.value, rr.value

    def norms(self, sol, exact=None, stream=None):
        """L2 / H1 error against an exact solution (None, "quadratic" = x^2+y^2+z^2,
        "sin") and L2 / H1 norm of the finite-element function with coefficients
        ``sol`` (calc_error / calc_norm, src/norm.cc:33-180), on the device."""
        import torch
        kinds = {None: 0, "quadratic": 1, "sin": 2}
        if exact not in kinds:
            raise capi.H3dgError(1, "exact solution must be None, 'quadratic' or 'sin'")
        t = sol if isinstance(sol, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(sol, dtype=np.float64))
        t = t.to(device="cuda:%d" % self.device, dtype=torch.float64).contiguous()
        if stream is None:
            stream = torch.cuda.current_stream(t.device)
        out = np.zeros(4, np.float64)
        capi.call("h3dg_disc_norms", self.handle, C.c_void_p(t.data_ptr()), kinds[exact], capi.ptr(out, C.c_double),
                  C.c_void_p(stream.cuda_stream))
        return {"l2_error": out[0], "h1_error": out[1], "l2_norm": out[2], "h1_norm": out[3]}

    def set_quadrature(self, points=None, p_plus=None, stock=False):
        """Fixed Gauss points per direction, p_d + p_plus per direction, or
        (stock=True) the rule the reference's stock forms pick: each pair
        with order(u) + order(v) + 1 per direction, the load vector with
        order 24 (src/integrals/h1.h:115-177; uniform orders 1..3, FP64)."""
        if stock:
            self._quad = (capi.QUAD_STOCK, 0)
        elif points is not None:
            self._quad = (capi.QUAD_FIXED, int(points))
        else:
            self._quad = (capi.QUAD_P_PLUS, int(p_plus))
        capi.call("h3dg_disc_set_quadrature", self.handle, *self._quad)

    def set_precision(self, precision: int):
        """Precision the next ``create`` plans for (no reference counterpart):
        with PREC_TF32X3 order-4 spaces already take the tensor-core path."""
        capi.call("h3dg_disc_set_precision", self.handle, int(precision))

    def set_partition(self, nparts: int, part: int):
        """Multi-GPU sharding without communication (no reference
        counterpart): the next ``create`` builds part ``part`` of ``nparts``
        z-slabs -- its slab of elements plus a one-element halo -- and
        ``assemble`` then yields the full CSC columns of the DOFs it owns
        (equal to the whole-mesh assembly's) with empty columns elsewhere."""
        capi.call("h3dg_disc_set_partition", self.handle, int(nparts), int(part))

    def partition(self):
        """Owned-DOF mask and element counts of the current plan's part."""
        owned = np.zeros(self.ndof, np.uint8)
        ns, nh, no = C.c_int64(), C.c_int64(), C.c_int64()
        capi.call("h3dg_disc_get_partition", self.handle, owned.ctypes.data_as(C.c_void_p), C.byref(ns), C.byref(nh),
                  C.byref(no))
        ne = self.space.mesh.num_elements
        elems = np.zeros(ne, np.uint8)
        capi.call("h3dg_disc_get_partition_elements", self.handle, elems.ctypes.data_as(C.c_void_p), ne)
        return {"owned": owned.astype(bool), "elements": elems.astype(bool), "slab_elements": ns.value,
                "halo_elements": nh.value, "owned_dofs": no.value}

    def create(self, matrix: Optional[UMFPackMatrix] = None, rhs: Optional[UMFPackVector] = None):
        """Discretization::create: sparsity pattern (+ device plan)."""
        capi.call("h3dg_disc_set_quadrature", self.handle, *self._quad)
        nd, nz = C.c_int64(), C.c_int64()
        capi.call("h3dg_disc_create_pattern", self.handle, C.byref(nd), C.byref(nz))
        self.ndof, self.nnz = nd.value, nz.value
        if matrix is not None:
            matrix.Ap = np.zeros(self.ndof + 1, np.int64)
            matrix.Ai = np.zeros(self.nnz, np.int32)
            capi.call("h3dg_disc_get_pattern", self.handle, capi.ptr(matrix.Ap, C.c_int64), capi.ptr(matrix.Ai, C.c_int32))
            matrix.Ax = np.zeros(self.nnz, np.float64)
            matrix.ndofs = self.ndof
        if rhs is not None:
            rhs.v = np.zeros(self.nrows, np.float64)

    @property
    def nrows(self):
        """Rows of the plan: the test space's DOFs (== ndof for one space)."""
        ts = getattr(self, "_test_space", None)
        return ts.ndof if ts is not None and ts is not self.space else self.ndof

    def assemble(self, matrix: Optional[UMFPackMatrix] = None, rhs: Optional[UMFPackVector] = None,
                 precision: int = capi.PREC_FP64):
        """Discretization::assemble into the host sinks (copies inside).
        ``precision``: PREC_FP64 (default, the reference's arithmetic) or
        PREC_TF32X3 (tensor-core split precision for the high-order path,
        normwise relative error below 1e-6)."""
        ax = None if matrix is None else matrix.Ax
        rv = None if rhs is None else rhs.v
        capi.call("h3dg_disc_assemble_host", self.handle, precision, capi.ptr(ax, C.c_double), capi.ptr(rv, C.c_double))

    def assemble_noalloc(self, matrix: Optional[UMFPackMatrix] = None, rhs: Optional[UMFPackVector] = None,
                         precision: int = capi.PREC_FP64):
        """``assemble`` without any device allocation (no reference
        counterpart): stages Ax and rhs in the library's fixed 16 MiB device
        array, so it serves callers that cannot allocate device memory (a
        pool holds it all, or cudaFree's device-wide synchronisation is not
        acceptable).  Raises H3dgError TOO_LARGE above that size and STATE
        unless one ``assemble`` with the same precision came first.
        Overlapping calls on one device race on the array."""
        ax = None if matrix is None else matrix.Ax
        rv = None if rhs is None else rhs.v
        capi.call("h3dg_disc_assemble_host_noalloc", self.handle, precision, capi.ptr(ax, C.c_double),
                  capi.ptr(rv, C.c_double))

    def assemble_device(self, Ax, rhs=None, stream=None, precision: int = capi.PREC_FP64):
        """Assemble into device tensors (torch CUDA float64) on ``stream``
        (default: torch's current stream)."""
        import torch
        if stream is None:
            stream = torch.cuda.current_stream(Ax.device if Ax is not None else rhs.device)
        sp = C.c_void_p(stream.cuda_stream)
        capi.call("h3dg_disc_assemble", self.handle, precision,
                  C.c_void_p(Ax.data_ptr()) if Ax is not None else None,
                  C.c_void_p(rhs.data_ptr()) if rhs is not None else None, sp)

    def geometry(self, jac=None, irm=None, xyz=None, stream=None):
        import torch
        t = jac if jac is not None else (irm if irm is not None else xyz)
        if stream is None:
            stream = torch.cuda.current_stream(t.device)
        capi.call("h3dg_disc_geometry", self.handle,
                  *[C.c_void_p(x.data_ptr()) if x is not None else None for x in (jac, irm, xyz)],
                  C.c_void_p(stream.cuda_stream))

    def adjoint(self, logcoef, u, lam, S=None, grad=None, stream=None):
        """Element sensitivities of L_k = lam_k^T K(exp(g_k)) u_k - lam_k^T f(exp(g_k)).

        logcoef (nf x ne, element-id order, or None), u and lam (nf x ndof) are
        torch CUDA float64 tensors; returns (S, grad), both nf x ne, with
        grad = exp(logcoef) * S = dL/dg."""
        import torch
        u = u.reshape(-1, self.ndof)
        lam = lam.reshape(-1, self.ndof)
        nf = u.shape[0]
        ne = self.space.mesh.num_elements
        dev = u.device
        if S is None:
            S = torch.empty(nf, ne, dtype=torch.float64, device=dev)
        if grad is None:
            grad = torch.empty(nf, ne, dtype=torch.float64, device=dev)
        if stream is None:
            stream = torch.cuda.current_stream(dev)
        lg = None if logcoef is None else logcoef.reshape(nf, ne).contiguous()
        u, lam = u.contiguous(), lam.contiguous()
        capi.call("h3dg_disc_adjoint", self.handle, nf, None if lg is None else C.c_void_p(lg.data_ptr()),
                  C.c_void_p(u.data_ptr()), C.c_void_p(lam.data_ptr()), C.c_void_p(S.data_ptr()),
                  C.c_void_p(grad.data_ptr()), C.c_void_p(stream.cuda_stream))
        return S, grad

    def update_vertices(self, xyz):
        a = np.ascontiguousarray(xyz, dtype=np.float64)
        capi.call("h3dg_disc_update_vertices", self.handle, capi.ptr(a, C.c_double), len(a.reshape(-1, 3)))

    def update_coefficients(self, coef):
        a = np.ascontiguousarray(coef, dtype=np.float64)
        capi.call("h3dg_disc_update_coefficients", self.handle, capi.ptr(a, C.c_double), len(a))

    def update_coefficients_device(self, coef, stream=None):
        """Per-element coefficients from a CUDA float64 tensor (element-id
        order), ordered on ``stream``; no host round trip."""
        import torch
        coef = coef.contiguous()
        if stream is None:
            stream = torch.cuda.current_stream(coef.device)
        capi.call("h3dg_disc_update_coefficients_device", self.handle, C.c_void_p(coef.data_ptr()), coef.numel(),
                  C.c_void_p(stream.cuda_stream))

    def enable_kernel_timing(self, n):
        capi.call("h3dg_disc_enable_kernel_timing", self.handle, int(n))

    def kernel_times(self, cap=4096):
        buf = (C.c_float * cap)()
        n = C.c_int32()
        capi.call("h3dg_disc_kernel_times", self.handle, buf, cap, C.byref(n))
        return [buf[i] for i in range(n.value)]

    def tuning(self):
        t, e, ms = C.c_int32(), C.c_int32(), C.c_float()
        capi.call("h3dg_disc_get_tuning", self.handle, C.byref(t), C.byref(e), C.byref(ms))
        sg = C.c_int32()
        capi.call("h3dg_disc_tuned_scatter", self.handle, C.byref(sg))
        scatter = {1: "segmented", 0: "colour sweeps"}.get(sg.value, "not tuned")
        return {"threads": t.value, "elems_per_cta": e.value, "ms": ms.value, "scatter": scatter}

    def seg_stats(self):
        """Wait statistics of the last segmented assembly (measurement hook)."""
        out = (C.c_int64 * 8)()
        capi.call("h3dg_disc_seg_stats", self.handle, out)
        keys = ("element_items_waited", "element_polls", "column_items_waited", "column_polls", "items",
                "ring_windows", "ctas", "span_windows")
        return dict(zip(keys, list(out)))

    def last_launch_count(self):
        n = C.c_int32()
        capi.call("h3dg_disc_last_launch_count", self.handle, C.byref(n))
        return n.value

    def last_kernel(self):
        """Element-matrix kernel family of the last volume assembly: "other"
        (low / mixed orders, stock rule), "ho_fp64_fma", "ho_fp64_dmma" (FP64
        tensor cores), "ho_tf32x3", "ho_ozaki"."""
        n = C.c_int32()
        capi.call("h3dg_disc_last_kernel", self.handle, C.byref(n))
        return ("other", "ho_fp64_fma", "ho_fp64_dmma", "ho_tf32x3", "ho_ozaki")[n.value]

    def debug_inject(self, what: int):
        """Test hook (no reference counterpart): DEBUG_WAIT_GIVES_UP makes the
        next FP64 low-order assembly's bounded wait give up (H3dgError
        TIMEOUT from ``assemble``); DEBUG_CORRUPT_POSITION points one position
        of the device scatter map past its column (H3dgError STATE until
        ``create`` rebuilds the plan).  Neither faults the device."""
        capi.call("h3dg_disc_debug_inject", self.handle, int(what))

    def __del__(self):
        if getattr(self, "handle", None) and capi._lib is not None:
            capi.lib().h3dg_disc_destroy(self.handle)
            self.handle = None


class SystemDiscretization:
    """Discretization with several equations (src/discretization.h:39-101 with
    neq > 1; assembly src/discretization.cc:232-343).  Space i is numbered
    after the spaces before it (assign_dofs(first_dof = sum of their DOF
    counts)), as in the reference's system tests.  Block (m, n) holds the form
    of test space m and trial space n; the Dirichlet lifting of the trial
    space goes to the rows of the test space; equation m's RHS is written only
    when it has a linear form.  Each block is assembled by the device kernels
    and placed into the system arrays on the device:
      * identical spaces (same orders and DOF counts; the caller gives them the
        same boundary conditions): every block on the first space's pattern,
        with any kernel the single space allows (mixed orders, refinement);
      * spaces that differ (orders): block (m, n) as a two-space plan (rows of
        space m, columns of space n, FP64; uniform orders per space)."""

    def __init__(self, device=0):
        self.device = device
        self.neq = 1
        self.spaces = []
        self.forms = {}
        self.lforms = {}
        self._quad = ("p_plus", 2)
        self.ndof = None
        self.nnz = None

    def set_num_equations(self, neq):
        if not 1 <= int(neq) <= 8:
            raise capi.H3dgError(1, "1..8 equations")
        self.neq = int(neq)

    def set_spaces(self, *spaces):
        if len(spaces) != self.neq:
            raise capi.H3dgError(1, "one space per equation")
        off = 0
        for sp in spaces:
            if sp.mesh is not spaces[0].mesh or getattr(sp, "first_dof", None) != off:
                raise capi.H3dgError(1, "the spaces share one mesh and are numbered one after another")
            off += sp.ndof
        self.spaces = list(spaces)
        self.identical = all(sp.ndof == spaces[0].ndof and getattr(sp, "orders", None) == getattr(spaces[0], "orders", None)
                             for sp in spaces)

    def set_bilinear_form(self, i, j, form, coef=None):
        if not isinstance(form, BilinearForm):
            raise UnsupportedForm(4, "bilinear form %r is not one of the device forms" % (form,))
        self.forms[(int(i), int(j))] = (form, coef)

    def set_linear_form(self, i, form):
        if form is not None and not isinstance(form, LinearForm):
            raise UnsupportedForm(4, "linear form %r is not one of the device forms" % (form,))
        self.lforms[int(i)] = form

    def set_quadrature(self, points=None, p_plus=None):
        self._quad = ("points", int(points)) if points is not None else ("p_plus", int(p_plus))

    def _base(self, m, n, form, coef, lf):
        """Single-space discretisation of block (m, n) (n < 0: a linear form
        alone) and its pattern, in the block's own numbering."""
        d = Discretization(self.device)
        if self.identical:
            d.set_spaces(self.spaces[0])
        else:
            d.set_spaces(self.spaces[n if n >= 0 else m])
            if n >= 0 and n != m:
                d.set_test_space(self.spaces[m])
        d.set_bilinear_form(form, coef)
        d.set_linear_form(lf)
        if self._quad[0] == "points":
            d.set_quadrature(points=self._quad[1])
        else:
            d.set_quadrature(p_plus=self._quad[1])
        bm = UMFPackMatrix()
        d.create(bm, UMFPackVector())
        return d, bm

    def create(self, matrix=None, rhs=None):
        """Discretization::create: the pattern of every block with a form.
        System column (n, j) holds the rows of the blocks (m, n), m ascending."""
        if not self.identical and any(getattr(sp, "orders", ("uniform",))[0] != "uniform" for sp in self.spaces):
            raise capi.H3dgError(1, "spaces that differ need uniform orders")
        offs = [sp.first_dof for sp in self.spaces]
        nds = [sp.ndof for sp in self.spaces]
        self._offs, self._nds = offs, nds
        # one discretisation per block; the first block of row m carries F_m,
        # the others contribute their lifting only (F = 0)
        self._blocks = []
        pats = {}
        for m in range(self.neq):
            row = [n for n in range(self.neq) if (m, n) in self.forms]
            lf = self.lforms.get(m)
            for k, n in enumerate(row):
                form, coef = self.forms[(m, n)]
                blf = (lf if k == 0 else int_F_v(0.0)) if lf is not None else None
                d, bm = self._base(m, n, form, coef, blf)
                self._blocks.append((m, n, d))
                pats[(m, n)] = (bm.Ap, bm.Ai)
            if lf is not None and not row:
                d, bm = self._base(m, -1, int_grad_u_grad_v, None, lf)
                self._blocks.append((m, -1, d))
        ntot = int(sum(nds))
        colcnt = np.zeros(ntot, np.int64)
        for (m, n), (Apb, Aib) in pats.items():
            colcnt[offs[n]:offs[n] + nds[n]] += np.diff(Apb)
        Ap = np.zeros(ntot + 1, np.int64)
        np.cumsum(colcnt, out=Ap[1:])
        Ai = np.zeros(Ap[-1], np.int32)
        self._pos = {}
        for n in range(self.neq):
            off = np.zeros(nds[n], np.int64)
            for m in range(self.neq):
                if (m, n) not in pats:
                    continue
                Apb, Aib = pats[(m, n)]
                counts = np.diff(Apb)
                start = Ap[offs[n]:offs[n] + nds[n]] + off
                idx = np.repeat(start - Apb[:-1], counts) + np.arange(Apb[-1])
                Ai[idx] = Aib + offs[m]
                self._pos[(m, n)] = idx
                off += counts
        self.ndof, self.nnz = ntot, int(Ap[-1])
        self.Ap, self.Ai = Ap, Ai
        if matrix is not None:
            matrix.Ap, matrix.Ai = Ap.copy(), Ai.copy()
            matrix.Ax = np.zeros(self.nnz, np.float64)
            matrix.ndofs = self.ndof
        if rhs is not None:
            rhs.v = np.zeros(self.ndof, np.float64)

    def assemble_device(self, Ax, rhs=None):
        """Assemble into torch CUDA float64 tensors (system layout), block by block."""
        import torch
        dev = Ax.device if Ax is not None else rhs.device
        if Ax is not None:
            Ax.zero_()
        if rhs is not None:
            rhs.zero_()
        for m, n, d in self._blocks:
            ax_b = torch.empty(d.nnz, dtype=torch.float64, device=dev) if (Ax is not None and n >= 0) else None
            rhs_b = (torch.empty(self._nds[m], dtype=torch.float64, device=dev)
                     if (rhs is not None and self.lforms.get(m) is not None) else None)
            if ax_b is None and rhs_b is None:
                continue
            d.assemble_device(ax_b, rhs_b)
            if ax_b is not None:
                key = ("t", m, n)
                if key not in self._pos:
                    self._pos[key] = torch.as_tensor(self._pos[(m, n)], device=dev)
                Ax.index_add_(0, self._pos[key], ax_b)     # each system entry belongs to one block
            if rhs_b is not None:
                rhs[self._offs[m]:self._offs[m] + self._nds[m]] += rhs_b

    def assemble(self, matrix=None, rhs=None):
        import torch
        dev = torch.device("cuda", self.device)
        Ax = torch.empty(self.nnz, dtype=torch.float64, device=dev) if matrix is not None else None
        r = torch.empty(self.ndof, dtype=torch.float64, device=dev) if rhs is not None else None
        self.assemble_device(Ax, r)
        if matrix is not None:
            matrix.Ax = Ax.cpu().numpy()
        if rhs is not None:
            rhs.v = r.cpu().numpy()
