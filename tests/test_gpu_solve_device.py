"""The reference's exact-solution checks end to end on the device: assemble,
solve with the device CG (h3dg_disc_solve_cg), and measure the error with
h3dg_disc_norms; CG against scipy's direct solve; bitwise reproducibility."""
import numpy as np
import pytest

import hermes3d_b200 as h

pytestmark = pytest.mark.gpu


def _problem(refs=(), p=2, jitter=0.0, coef=None):
    mesh = h.unit_cube(3, jitter, 4)
    mesh.ugh()
    if refs:
        mesh.refine_elements(list(refs))
    sp = h.H1Space(mesh)
    sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    sp.set_element_orders(np.full((len(mesh.hexes), 3), p, np.int32))
    sp.assign_dofs()
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v, coef)
    d.set_linear_form(h.int_F_v(-6.0))
    d.set_quadrature(p_plus=2)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    return mesh, sp, d, M, V


def _device_assemble(d, M, V):
    import torch
    Ax = torch.empty(len(M.Ai), dtype=torch.float64, device="cuda")
    rhs = torch.empty(len(V.v) if V.v is not None else d.ndof, dtype=torch.float64, device="cuda")
    d.assemble_device(Ax, rhs)
    return Ax, rhs


@pytest.mark.parametrize("refs,p", [((), 2), ((), 3), ((14,), 2), ((1, 14, 27), 3)])
def test_exact_solution_on_device(gpu, refs, p):
    mesh, sp, d, M, V = _problem(refs, p)
    Ax, rhs = _device_assemble(d, M, V)
    x, it, rr = d.solve(Ax, rhs, rtol=1e-13)
    assert rr <= 1e-13 and it > 0
    r = d.norms(x, exact="quadratic")
    assert r["h1_error"] < 1e-9 * r["h1_norm"]


def test_cg_matches_direct_solve_and_is_reproducible(gpu):
    import scipy.sparse as sps
    import scipy.sparse.linalg as spl
    import torch
    coef = np.random.default_rng(3).uniform(0.5, 2.0, 27)
    mesh, sp, d, M, V = _problem((), 3, jitter=0.2, coef=coef)
    d.assemble(M, V)
    n = sp.ndof
    ref = spl.spsolve(sps.csc_matrix((M.Ax, M.Ai, M.Ap), shape=(n, n)), V.v)
    Ax, rhs = _device_assemble(d, M, V)
    x1, it1, _ = d.solve(Ax, rhs, rtol=1e-14)
    x2, it2, _ = d.solve(Ax, rhs, rtol=1e-14)
    torch.cuda.synchronize()
    assert it1 == it2 and torch.equal(x1, x2)
    assert np.max(np.abs(x1.cpu().numpy() - ref)) < 1e-10 * np.max(np.abs(ref))
