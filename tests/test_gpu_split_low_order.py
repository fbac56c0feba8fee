"""Split precision (3xTF32) at low orders with the elements batched on the
tensor cores (stages 2+3 of the sum factorisation as one tcgen05 GEMM per
batch): against the reference's fixtures, the restatement oracle and the
FP64 kernel.  Tolerance 1e-6 of the largest matrix entry, entrywise and
normwise; the load vector is FP64 and keeps the FP64 tolerance."""
import numpy as np
import pytest

import hermes3d_b200 as h
from helpers import FP64_RTOL, disc_of, load, rel_err, space_of
from oracle import port

pytestmark = pytest.mark.gpu

SPLIT_RTOL = 1e-6


def _norm_err(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("name", ["p2_c2_forms", "perm_p2_lifting", "perm_p1_natural"])
def test_batched_split_on_reference_fixtures(gpu, name):
    g = load(name)
    sp = space_of(g)
    d = disc_of(g, sp)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V, precision=h.PREC_TF32X3)
    e_max, e_norm = rel_err(M.Ax, g["Ax"]), _norm_err(M.Ax, g["Ax"])
    print("%s: batched 3xTF32 error max %.2e norm %.2e" % (name, e_max, e_norm))
    assert e_max < SPLIT_RTOL and e_norm < SPLIT_RTOL
    assert rel_err(V.v, g["rhs"]) < FP64_RTOL


@pytest.mark.parametrize("p,nq,n", [(1, 2, 12), (1, 3, 12), (2, 3, 8), (2, 4, 10)])
def test_batched_split_matches_restatement_and_fp64(gpu, p, nq, n):
    mesh = h.permute_vertices(h.unit_cube(n, 0.2, 7), seed=p + nq)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    sp.set_uniform_order(p)
    sp.assign_dofs()
    coef = np.random.default_rng(n).uniform(0.5, 2.0, mesh.num_elements)
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v_plus_u_v, coef)
    d.set_linear_form(h.int_F_v("sin"))
    d.set_quadrature(points=nq)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V, precision=h.PREC_TF32X3)
    ax, v = M.Ax.copy(), V.v.copy()
    d.assemble(M, V, precision=h.PREC_TF32X3)          # bitwise reproducible
    assert np.array_equal(M.Ax, ax) and np.array_equal(V.v, v)
    al = port.asmlists_from_space(sp, mesh.num_elements)
    Ax, rhs = port.assemble(mesh.xyz, mesh.hexes - 1, nq, al, sp.ndof, M.Ap, M.Ai, mass=True, gradcoef=coef, lf=2)
    e_max, e_norm = rel_err(ax, Ax), _norm_err(ax, Ax)
    print("p=%d nq=%d: batched 3xTF32 error max %.2e norm %.2e" % (p, nq, e_max, e_norm))
    assert e_max < SPLIT_RTOL and e_norm < SPLIT_RTOL
    assert e_max > 0.0                                   # the split kernel ran, not the FP64 one
    # the RHS carries the Dirichlet lifting through the split matrix: its
    # error is the matrix's, relative to the RHS
    assert rel_err(v, rhs) < 1e-5
    d.assemble(M, V)                                      # FP64 on the same plan
    assert rel_err(M.Ax, Ax) < FP64_RTOL
