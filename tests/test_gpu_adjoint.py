"""Adjoint kernel: against central finite differences of the assembled
energy (h = 1e-6 on the log-coefficient) and against an FP64 reference
gradient built from the restatement oracle's element matrices."""
import numpy as np
import pytest

import hermes3d_b200 as h
from oracle import port

pytestmark = pytest.mark.gpu


def _problem(n=3, p=3, nq=5, lifting=False, seed=0):
    mesh = h.permute_vertices(h.unit_cube(n, 0.2, seed), seed=seed + 1)
    mesh.ugh()
    sp = h.H1Space(mesh)
    if lifting:
        sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    sp.set_uniform_order(p)
    sp.assign_dofs()
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v, np.ones(mesh.num_elements))
    d.set_linear_form(h.int_F_v(1.0))
    d.set_quadrature(points=nq)
    d.create()
    return mesh, sp, d


@pytest.mark.parametrize("lifting", [False, True])
def test_adjoint_matches_central_differences(gpu, lifting):
    import torch
    from hermes3d_b200.autograd import assembly_energy, energy, energy_assembled
    mesh, sp, d = _problem(lifting=lifting)
    nf, ne = 2, mesh.num_elements
    rng = np.random.default_rng(5)
    g = torch.tensor(rng.normal(0, 0.5, (nf, ne)), device="cuda", requires_grad=True)
    u = torch.tensor(rng.normal(0, 1, (nf, sp.ndof)), device="cuda")
    lam = torch.tensor(rng.normal(0, 1, (nf, sp.ndof)), device="cuda")
    L = assembly_energy(g, u, lam, d)
    # the matrix-free forward against the definition (K(a) and f(a) assembled)
    La = energy_assembled(d, g.detach(), u, lam)
    assert torch.allclose(L.detach(), La, rtol=1e-12, atol=1e-12 * float(La.abs().max()))
    assert torch.allclose(energy(d, g.detach(), u, lam), L.detach(), rtol=0, atol=0)
    L.sum().backward()
    grad = g.grad.detach().cpu().numpy()
    hstep = 1e-6
    for k in range(nf):
        for e in rng.choice(ne, 8, replace=False):
            gp = g.detach().clone()
            gm = g.detach().clone()
            gp[k, e] += hstep
            gm[k, e] -= hstep
            fd = (energy_assembled(d, gp, u, lam)[k] - energy_assembled(d, gm, u, lam)[k]).item() / (2 * hstep)
            assert abs(fd - grad[k, e]) <= 1e-6 * max(1.0, np.max(np.abs(grad[k]))), (k, e, fd, grad[k, e])


def test_adjoint_matches_fp64_reference_gradient(gpu):
    import torch
    mesh, sp, d = _problem(n=2, p=3, nq=5, lifting=True, seed=3)
    ne = mesh.num_elements
    rng = np.random.default_rng(7)
    g = rng.normal(0, 0.5, (1, ne))
    u = rng.normal(0, 1, (1, sp.ndof))
    lam = rng.normal(0, 1, (1, sp.ndof))
    S, grad = d.adjoint(torch.tensor(g, device="cuda"), torch.tensor(u, device="cuda"), torch.tensor(lam, device="cuda"))
    S = S.cpu().numpy()[0]
    ref = np.zeros(ne)
    for e in range(1, ne + 1):
        idx, dof, coef = sp.get_element_assembly_list(e)
        K = port.element_matrix(mesh.xyz[mesh.hexes[e - 1] - 1], 5, idx)    # K[i][j] = form(u_j, v_i)
        le = np.where(dof >= 0, coef * lam[0][np.maximum(dof, 0)], 0.0)
        we = np.where(dof >= 0, coef * u[0][np.maximum(dof, 0)], coef)
        ref[e - 1] = le @ K @ we
    assert np.max(np.abs(S - ref)) <= 1e-12 * np.max(np.abs(ref))
    assert np.allclose(grad.cpu().numpy()[0], np.exp(g[0]) * S, rtol=1e-14, atol=0)
