"""Mixed-order (anisotropic, per-element) FP64 path: bucketed kernel classes,
graph-replayed assembly.  Against the reference's own fixture, against the
restatement oracle on a jittered mesh with orders 1..6, and with uniform
fixtures routed through the mixed kernels; FP64 tolerance 1e-12."""
import numpy as np
import pytest

import hermes3d_b200 as h
from helpers import FP64_RTOL, disc_of, load, rel_err, space_of
from oracle import port

pytestmark = pytest.mark.gpu


def test_mixed_orders_reference_fixture(gpu):
    g = load("aniso_orders_lifting")
    sp = space_of(g)
    d = disc_of(g, sp)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)
    assert np.array_equal(M.Ap, g["Ap"]) and np.array_equal(M.Ai, g["Ai"])
    assert rel_err(M.Ax, g["Ax"]) < FP64_RTOL
    assert rel_err(V.v, g["rhs"]) < FP64_RTOL


@pytest.mark.parametrize("name", ["c1_small", "perm_p2_lifting", "perm_p3_mass_sin", "perm_p4_natural",
                                  "jitter_p3_mass_sin", "coef_p3"])
def test_uniform_fixtures_through_mixed_kernels(gpu, monkeypatch, name):
    monkeypatch.setenv("H3DG_FORCE_MIXED", "1")
    g = load(name)
    sp = space_of(g)
    d = disc_of(g, sp)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)
    assert rel_err(M.Ax, g["Ax"]) < FP64_RTOL
    assert rel_err(V.v, g["rhs"]) < FP64_RTOL


def _random_orders(ne, seed, lo=1, hi=6):
    return np.random.default_rng(seed).integers(lo, hi + 1, size=(ne, 3)).astype(np.int32)


@pytest.mark.parametrize("bc,mass", [("lifting", True), ("dirichlet0", False), ("natural", True)])
def test_mixed_orders_match_restatement(gpu, bc, mass):
    mesh = h.permute_vertices(h.unit_cube(3, 0.2, 7), seed=3)
    mesh.ugh()
    sp = h.H1Space(mesh)
    if bc == "natural":
        sp.set_bc_types(lambda m: h.BC_NATURAL)
    if bc == "lifting":
        sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    orders = _random_orders(mesh.num_elements, 11)
    sp.set_element_orders(orders)
    sp.assign_dofs()
    d = h.Discretization()
    d.set_spaces(sp)
    coef = np.random.default_rng(5).uniform(0.5, 2.0, mesh.num_elements)
    d.set_bilinear_form(h.int_grad_u_grad_v_plus_u_v if mass else h.int_grad_u_grad_v, coef)
    d.set_linear_form(h.int_F_v(-6.0 if bc == "lifting" else "sin"))
    d.set_quadrature(p_plus=2)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)
    al = port.asmlists_from_space(sp, mesh.num_elements)
    nq = orders + 2
    Ax, rhs = port.assemble(mesh.xyz, mesh.hexes - 1, nq, al, sp.ndof, M.Ap, M.Ai, mass=mass, gradcoef=coef,
                            lf=1 if bc == "lifting" else 2, lf_value=-6.0)
    assert rel_err(M.Ax, Ax) < FP64_RTOL
    assert rel_err(V.v, rhs) < FP64_RTOL


def test_mixed_replay_is_bitwise_reproducible(gpu):
    import torch
    mesh = h.unit_cube(4, 0.2, 2)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_element_orders(_random_orders(mesh.num_elements, 4))
    sp.assign_dofs()
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v)
    d.set_linear_form(h.int_F_v(1.0))
    d.set_quadrature(p_plus=2)
    d.create()
    A1 = torch.empty(d.nnz, dtype=torch.float64, device="cuda")
    A2 = torch.empty_like(A1)
    b1 = torch.empty(d.ndof, dtype=torch.float64, device="cuda")
    b2 = torch.empty_like(b1)
    d.assemble_device(A1, b1)
    d.assemble_device(A1, b1)            # replay of the cached graph
    d.assemble_device(A2, b2)            # other pointers: a new capture
    torch.cuda.synchronize()
    assert torch.equal(A1, A2) and torch.equal(b1, b2)
    assert d.last_launch_count() >= 1


def test_mixed_graph_follows_coefficient_updates(gpu):
    """The replayed graph must see coefficients set after its capture, from
    host or device memory."""
    import torch
    mesh = h.unit_cube(3, 0.2, 6)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_element_orders(_random_orders(mesh.num_elements, 8))
    sp.assign_dofs()
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v)
    d.set_linear_form(None)
    d.set_quadrature(p_plus=2)
    d.create()
    A = torch.empty(d.nnz, dtype=torch.float64, device="cuda")
    d.assemble_device(A)
    base = A.clone()
    d.update_coefficients_device(torch.full((mesh.num_elements,), 2.0, dtype=torch.float64, device="cuda"))
    d.assemble_device(A)
    torch.cuda.synchronize()
    assert torch.equal(A, 2.0 * base)             # a power-of-two coefficient scales exactly
    d.update_coefficients(np.full(mesh.num_elements, 3.0))
    d.assemble_device(A)
    torch.cuda.synchronize()
    assert float((A - 3.0 * base).abs().max()) <= 1e-13 * 3.0 * float(base.abs().max())
