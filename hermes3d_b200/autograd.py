"""torch.autograd binding of the assembly and its hand-written adjoint.

AssemblyEnergy computes, for nf coefficient fields g_k (per-element
log-coefficients, a = exp(g) multiplies int_grad_u_grad_v),

    L_k = lam_k^T K(a_k) u_k - lam_k^T f(a_k).

With f(a) = F - K(a) g (source minus the Dirichlet lifting) and the unit
element matrices K_e of the grad-grad form,

    L_k = sum_e a_{k,e} S_{k,e} - lam_k^T F,   S_{k,e} = lam_e^T K_e (u_e + d_e),

so the forward is matrix-free: one launch of the adjoint kernel for all
fields (S is also what the backward needs, dL_k/dg_{k,e} = a_{k,e} S_{k,e}),
plus the coefficient-free load vector F assembled once.  Forms with the mass
term take the assembled path (the adjoint kernel covers the coefficient-
weighted grad-grad term).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _capi as capi


def _csr_transpose_matvec(disc, Ax, x):
    """y = A^T x for the CSC matrix (Ap, Ai, Ax): the CSC arrays of A are the CSR arrays of A^T."""
    crow = disc._Ap_dev
    col = disc._Ai_dev
    AT = torch.sparse_csr_tensor(crow, col, Ax, size=(disc.ndof, disc.ndof), dtype=torch.float64,
                                 check_invariants=False)
    return AT @ x


def _ensure_pattern_on_device(disc, device):
    if getattr(disc, "_Ap_dev", None) is None:
        Ap = np.zeros(disc.ndof + 1, np.int64)
        Ai = np.zeros(disc.nnz, np.int32)
        capi.call("h3dg_disc_get_pattern", disc.handle, capi.ptr(Ap, capi.C.c_int64), capi.ptr(Ai, capi.C.c_int32))
        disc._Ap_dev = torch.from_numpy(Ap).to(device)
        disc._Ai_dev = torch.from_numpy(Ai.astype(np.int64)).to(device)


def energy_assembled(disc, g, u, lam):
    """L_k by assembling K(a_k) and f(a_k) for each field (the definition;
    an independent check of the matrix-free path and its adjoint)."""
    dev = u.device
    _ensure_pattern_on_device(disc, dev)
    nf = u.shape[0]
    Ax = torch.empty(disc.nnz, dtype=torch.float64, device=dev)
    rhs = torch.empty(disc.ndof, dtype=torch.float64, device=dev)
    out = torch.empty(nf, dtype=torch.float64, device=dev)
    for k in range(nf):
        a = torch.exp(g[k]).double()
        disc.update_coefficients_device(a)          # stream-ordered, no host round trip
        disc.assemble_device(Ax, rhs)
        ATl = _csr_transpose_matvec(disc, Ax, lam[k])
        out[k] = torch.dot(ATl, u[k]) - torch.dot(lam[k], rhs)
    return out


def _matrix_free(disc):
    return getattr(disc, "_bf_kind", capi.BF_GRAD_GRAD) == capi.BF_GRAD_GRAD


def _source_vector(disc, device):
    """F: the load vector without lifting (the source alone; it does not
    depend on the coefficients), assembled once per plan."""
    F = getattr(disc, "_F_dev", None)
    if F is None or F.device != device or F.numel() != disc.ndof:
        F = torch.empty(disc.ndof, dtype=torch.float64, device=device)
        disc.assemble_device(None, F)               # RHS alone: no lifting (as the reference)
        disc._F_dev = F
    return F


def energy_and_grad(disc, g, u, lam):
    """(L, dL/dg): matrix-free for the grad-grad form, else assembled +
    the adjoint kernel."""
    if not _matrix_free(disc):
        _, grad = disc.adjoint(g, u, lam)
        return energy_assembled(disc, g, u, lam), grad
    S, grad = disc.adjoint(g, u, lam)
    L = grad.sum(dim=1)
    if getattr(disc, "_lf", None) is not None:
        L = L - lam @ _source_vector(disc, u.device)
    return L, grad


def energy(disc, g, u, lam):
    """L_k for each field, g: nf x ne, u/lam: nf x ndof (CUDA float64)."""
    return energy_and_grad(disc, g, u, lam)[0]


class AssemblyEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, g, u, lam, disc):
        g = g.detach().double().contiguous()
        u = u.detach().double().contiguous()
        lam = lam.detach().double().contiguous()
        L, grad = energy_and_grad(disc, g, u, lam)
        ctx.save_for_backward(grad)
        return L

    @staticmethod
    def backward(ctx, gL):
        (grad,) = ctx.saved_tensors                   # from the forward's adjoint launch
        return gL[:, None] * grad, None, None, None


def assembly_energy(g, u, lam, disc):
    """Differentiable L(g) (nf values) for g: nf x ne log-coefficients."""
    return AssemblyEnergy.apply(g, u, lam, disc)
