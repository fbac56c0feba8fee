"""Adjoint of mixed-order plans, hanging nodes included (k_adjoint_mixed):
against the uniform-order adjoint kernel on the same problem routed through
the mixed path, and against central finite differences of the assembled
energy on meshes with per-element order triples and with refinement (refined
parents, which hold no active element, get a zero gradient)."""
import os

import numpy as np
import pytest

import hermes3d_b200 as h
from helpers import load_refined, quad_of, refined_space_of

pytestmark = pytest.mark.gpu


def _disc(mesh, sp, qkind="pplus", qn=2):
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v, np.ones(mesh.num_elements))
    d.set_linear_form(h.int_F_v(1.0))
    if qkind == "fixed":
        d.set_quadrature(points=qn)
    else:
        d.set_quadrature(p_plus=qn)
    d.create()
    return d


def _uniform(p=3, force_mixed=False):
    mesh = h.permute_vertices(h.unit_cube(3, 0.2, 1), seed=2)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    sp.set_uniform_order(p)
    sp.assign_dofs()
    if force_mixed:
        os.environ["H3DG_FORCE_MIXED"] = "1"
    try:
        return mesh, sp, _disc(mesh, sp, "fixed", p + 2)
    finally:
        os.environ.pop("H3DG_FORCE_MIXED", None)


def test_mixed_adjoint_matches_uniform_kernel(gpu):
    import torch
    mesh, sp, du = _uniform()
    _, _, dm = _uniform(force_mixed=True)
    rng = np.random.default_rng(1)
    nf, ne = 3, mesh.num_elements
    g = torch.tensor(rng.normal(0, 0.5, (nf, ne)), device="cuda")
    u = torch.tensor(rng.normal(0, 1, (nf, sp.ndof)), device="cuda")
    lam = torch.tensor(rng.normal(0, 1, (nf, sp.ndof)), device="cuda")
    Su, Gu = du.adjoint(g, u, lam)
    Sm, Gm = dm.adjoint(g, u, lam)
    torch.cuda.synchronize()
    assert float((Sm - Su).abs().max()) <= 1e-12 * float(Su.abs().max())
    assert float((Gm - Gu).abs().max()) <= 1e-12 * float(Gu.abs().max())
    S2, _ = dm.adjoint(g, u, lam)
    assert torch.equal(S2, Sm)                       # bitwise reproducible


def _mixed_orders():
    mesh = h.permute_vertices(h.unit_cube(3, 0.2, 4), seed=5)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    orders = np.random.default_rng(7).integers(1, 5, size=(mesh.num_elements, 3)).astype(np.int32)
    sp.set_element_orders(orders)
    sp.assign_dofs()
    return mesh, sp, _disc(mesh, sp)


def _refined(name):
    g = load_refined(name)
    mesh, sp = refined_space_of(g)
    kind, n = quad_of(g)
    return mesh, sp, _disc(mesh, sp, kind, n)


CASES = {"mixed_orders": _mixed_orders, "refined_c3_like": lambda: _refined("ref_aniso_c3_like"),
         "refined_lifting_p3": lambda: _refined("ref_lifting_p3")}


@pytest.mark.parametrize("case", sorted(CASES))
def test_mixed_adjoint_matches_central_differences(gpu, case):
    import torch
    from hermes3d_b200.autograd import assembly_energy, energy_assembled
    mesh, sp, d = CASES[case]()
    nf, ne = 2, mesh.num_elements
    rng = np.random.default_rng(11)
    g = torch.tensor(rng.normal(0, 0.5, (nf, ne)), device="cuda", requires_grad=True)
    u = torch.tensor(rng.normal(0, 1, (nf, sp.ndof)), device="cuda")
    lam = torch.tensor(rng.normal(0, 1, (nf, sp.ndof)), device="cuda")
    L = assembly_energy(g, u, lam, d)
    La = energy_assembled(d, g.detach(), u, lam)
    assert torch.allclose(L.detach(), La, rtol=1e-12, atol=1e-12 * float(La.abs().max()))
    L.sum().backward()
    grad = g.grad.detach().cpu().numpy()
    active = mesh.active
    hstep = 1e-6
    for k in range(nf):
        for e in rng.choice(ne, 8, replace=False):
            gp = g.detach().clone()
            gm = g.detach().clone()
            gp[k, e] += hstep
            gm[k, e] -= hstep
            fd = (energy_assembled(d, gp, u, lam)[k] - energy_assembled(d, gm, u, lam)[k]).item() / (2 * hstep)
            assert abs(fd - grad[k, e]) <= 1e-6 * max(1.0, np.max(np.abs(grad[k]))), (k, e, fd, grad[k, e])
    # refined parents: no active element, no sensitivity
    assert (grad[:, ~active] == 0.0).all()
    if case.startswith("refined"):
        assert (~active).any()
