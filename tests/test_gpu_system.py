"""Two-equation systems on the GPU (block forms grad.grad, grad.grad + mass,
mass; coupling blocks with Dirichlet lifting; a source per equation) against
fixtures the reference itself produced; FP64 tolerance 1e-12.  Also int_u_v
as a single equation's form against the mass block of a fixture."""
import numpy as np
import pytest

import hermes3d_b200 as h
from helpers import FP64_RTOL, load_system, rel_err, system_names, system_problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", system_names())
def test_system_assembly_matches_reference(gpu, name):
    g = load_system(name)
    mesh, spaces, d = system_problem(g)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)
    assert np.array_equal(M.Ap, g["Ap"]) and np.array_equal(M.Ai, g["Ai"])
    assert rel_err(M.Ax, g["Ax"]) < FP64_RTOL
    assert rel_err(V.v, g["rhs"]) < FP64_RTOL


def test_mass_form_alone_matches_reference(gpu):
    g = load_system("sys_mass_blocks_p3")
    mesh, spaces, d = system_problem(g)
    n = spaces[0].ndof
    A = np.zeros((2 * n, 2 * n))
    for j in range(2 * n):
        A[g["Ai"][g["Ap"][j]:g["Ap"][j + 1]], j] = g["Ax"][g["Ap"][j]:g["Ap"][j + 1]]
    m = h.Discretization()
    m.set_spaces(spaces[0])
    m.set_bilinear_form(h.int_u_v)
    m.set_linear_form(None)
    m.set_quadrature(p_plus=2)
    Mm = h.UMFPackMatrix()
    m.create(Mm)
    m.assemble(Mm)
    B = np.zeros((n, n))
    for j in range(n):
        B[Mm.Ai[Mm.Ap[j]:Mm.Ap[j + 1]], j] = Mm.Ax[Mm.Ap[j]:Mm.Ap[j + 1]]
    # block (0, 1) of the fixture is the mass matrix
    assert np.max(np.abs(B - A[:n, n:])) < FP64_RTOL * np.max(np.abs(A[:n, n:]))
