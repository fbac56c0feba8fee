"""torch.autograd binding of the assembly and its hand-written adjoint.

AssemblyEnergy computes, for nf coefficient fields g_k (per-element
log-coefficients, a = exp(g) multiplies int_grad_u_grad_v),

    L_k = lam_k^T K(a_k) u_k - lam_k^T f(a_k)

forward by assembling K(a_k) and f(a_k) on the device (the same
Discretization::assemble path as everything else) and backward with the
adjoint kernel (dL_k/dg_{k,e} = a_{k,e} lam_e^T K_e (u_e + d_e)), never
differentiating through the assembly.
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


def energy(disc, g, u, lam):
    """L_k for each field (forward by assembly), g: nf x ne, u/lam: nf x ndof (CUDA float64)."""
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


class AssemblyEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, g, u, lam, disc):
        g = g.detach().double().contiguous()
        u = u.detach().double().contiguous()
        lam = lam.detach().double().contiguous()
        ctx.disc = disc
        ctx.save_for_backward(g, u, lam)
        return energy(disc, g, u, lam)

    @staticmethod
    def backward(ctx, gL):
        g, u, lam = ctx.saved_tensors
        _, grad = ctx.disc.adjoint(g, u, lam)
        return gL[:, None] * grad, None, None, None


def assembly_energy(g, u, lam, disc):
    """Differentiable L(g) (nf values) for g: nf x ne log-coefficients."""
    return AssemblyEnergy.apply(g, u, lam, disc)
