"""Parity of the high-order FP64 kernel (orders whose element matrix does
not fit in shared memory; canonical tables, matrix-free lifting) against
the reference fixtures and the C restatement oracle."""
import os

import numpy as np
import pytest

import hermes3d_b200 as h
from helpers import FP64_RTOL, disc_of, load, rel_err, space_of
from oracle import port

pytestmark = pytest.mark.gpu


@pytest.fixture
def force_high_order():
    os.environ["H3DG_FORCE_HIGH_ORDER"] = "1"
    yield
    del os.environ["H3DG_FORCE_HIGH_ORDER"]


@pytest.mark.parametrize("name", ["c1_small", "jitter_p3_mass_sin", "perm_p3_mass_sin", "perm_p2_lifting",
                                  "coef_p3", "p2_c2_forms"])
def test_high_order_kernel_on_reference_fixtures(gpu, force_high_order, name):
    g = load(name)
    sp = space_of(g)
    d = disc_of(g, sp)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)
    assert rel_err(M.Ax, g["Ax"]) < FP64_RTOL
    assert rel_err(V.v, g["rhs"]) < FP64_RTOL


@pytest.mark.parametrize("p,bc", [(5, "lifting"), (6, "dirichlet0"), (5, "natural")])
def test_high_order_matches_restatement(gpu, p, bc):
    mesh = h.permute_vertices(h.unit_cube(2, 0.15, 3), seed=p)
    mesh.ugh()
    sp = h.H1Space(mesh)
    if bc == "natural":
        sp.set_bc_types(lambda m: h.BC_NATURAL)
    if bc == "lifting":
        sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    sp.set_uniform_order(p)
    sp.assign_dofs()
    d = h.Discretization()
    d.set_spaces(sp)
    coef = np.random.default_rng(p).uniform(0.5, 2.0, mesh.num_elements)
    d.set_bilinear_form(h.int_grad_u_grad_v_plus_u_v if bc != "dirichlet0" else h.int_grad_u_grad_v, coef)
    d.set_linear_form(h.int_F_v(-6.0 if bc == "lifting" else "sin"))
    d.set_quadrature(p_plus=2)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)
    al = port.asmlists_from_space(sp, mesh.num_elements)
    Ax, rhs = port.assemble(mesh.xyz, mesh.hexes - 1, p + 2, al, sp.ndof, M.Ap, M.Ai, mass=(bc != "dirichlet0"),
                            gradcoef=coef, lf=1 if bc == "lifting" else 2, lf_value=-6.0)
    assert rel_err(M.Ax, Ax) < FP64_RTOL
    assert rel_err(V.v, rhs) < FP64_RTOL


def test_p8_single_element_rows(gpu):
    """Order 8 with 10 points per direction (729 functions, 1000 points) on one
    jittered element with natural BCs: the assembled matrix is the element
    matrix; sampled rows against the restatement."""
    mesh = h.unit_cube(1)
    X = mesh.xyz + 0.08 * np.random.default_rng(8).uniform(-1, 1, mesh.xyz.shape)
    mesh = h.Mesh().set_arrays(X, mesh.hexes, mesh.bquads, mesh.bmarkers)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_bc_types(lambda m: h.BC_NATURAL)
    sp.set_uniform_order(8)
    assert sp.assign_dofs() == 729
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v, np.array([1.7]))
    d.set_quadrature(points=10)
    M = h.UMFPackMatrix()
    d.create(M)
    d.assemble(M)
    A = M.to_scipy().toarray()
    idx, dof, coef = sp.get_element_assembly_list(1)
    rows = np.random.default_rng(1).choice(len(idx), 12, replace=False).astype(np.int32)
    R = port.element_rows(X[mesh.hexes[0] - 1], 10, idx, rows, gradcoef=1.7) * np.outer(coef[rows], coef)
    got = np.array([[A[dof[r], dof[j]] for j in range(len(idx))] for r in rows])
    assert np.max(np.abs(got - R)) <= FP64_RTOL * np.max(np.abs(A))
