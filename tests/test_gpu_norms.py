"""Norms of a finite-element function on the GPU (h3dg_disc_norms; calc_error /
calc_norm with the H1 and L2 functions of src/norm.cc:33-180): against a
numpy evaluation from the assembly lists with the same rule (jittered mesh,
anisotropic orders, random coefficients, sin exact solution), the exact
reproduction of x^2+y^2+z^2 after a solve (uniform and refined meshes), the
analytic norms of that function, and bitwise reproducibility."""
import numpy as np
import pytest

import hermes3d_b200 as h
from test_gpu_solve_kat import _decode, _lobatto

pytestmark = pytest.mark.gpu

REF = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1], [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]])


def _norms_numpy(mesh, sp, sol, qplus, exact):
    tot = np.zeros(4)
    for e in np.nonzero(mesh.active)[0] + 1:
        idx, dof, coef = sp.get_element_assembly_list(int(e))
        X = mesh.xyz[mesh.hexes[e - 1] - 1]
        o = sp_orders[e - 1]
        rules = [np.polynomial.legendre.leggauss(int(o[d]) + qplus) for d in range(3)]
        for i0, (x0, w0) in enumerate(zip(*rules[0])):
            for x1, w1 in zip(*rules[1]):
                for x2, w2 in zip(*rules[2]):
                    xi = np.array([x0, x1, x2])
                    N = np.prod([(1 + REF[:, r] * xi[r]) / 2 for r in range(3)], axis=0)
                    dN = np.stack([REF[:, k] / 2 * np.prod([(1 + REF[:, r] * xi[r]) / 2 for r in range(3) if r != k], axis=0)
                                   for k in range(3)], axis=1)
                    J = X.T @ dN
                    det = np.linalg.det(J)
                    p = N @ X
                    u, g = 0.0, np.zeros(3)
                    for ii, dd, c in zip(idx, dof, coef):
                        ind, sg = _decode(int(ii))
                        v = [_lobatto(ind[r], xi[r]) for r in range(3)]
                        dv = [_dlobatto(ind[r], xi[r]) for r in range(3)]
                        w = c * sg * (sol[dd] if dd >= 0 else 1.0)
                        u += w * v[0] * v[1] * v[2]
                        g += w * np.array([dv[0] * v[1] * v[2], v[0] * dv[1] * v[2], v[0] * v[1] * dv[2]])
                    gx = np.linalg.solve(J.T, g)
                    ue, ge = exact(p)
                    wd = w0 * w1 * w2 * det
                    tot += wd * np.array([(u - ue) ** 2, (u - ue) ** 2 + np.sum((gx - ge) ** 2), u * u, u * u + gx @ gx])
    return np.where(tot > 10e-15, np.sqrt(tot), tot)


def _dlobatto(k, x):
    from numpy.polynomial import legendre as L
    if k == 0:
        return -0.5
    if k == 1:
        return 0.5
    c = np.zeros(k)
    c[k - 1] = 1.0
    return np.sqrt((2 * k - 1) / 2) * L.legval(x, c)


def _sin(p):
    s = np.sin(np.pi * p)
    c = np.cos(np.pi * p)
    return s[0] * s[1] * s[2], np.pi * np.array([c[0] * s[1] * s[2], s[0] * c[1] * s[2], s[0] * s[1] * c[2]])


sp_orders = None


def _disc(sp, qplus=2):
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v)
    d.set_linear_form(h.int_F_v(-6.0))
    d.set_quadrature(p_plus=qplus)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    return d, M, V


def test_norms_match_numpy_evaluation(gpu):
    global sp_orders
    mesh = h.permute_vertices(h.unit_cube(2, 0.2, 3), seed=2)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_bc_values(lambda m, x, y, z: x + 2 * y - z)
    sp_orders = np.random.default_rng(1).integers(1, 5, size=(8, 3)).astype(np.int32)
    sp.set_element_orders(sp_orders)
    sp.assign_dofs()
    d, M, V = _disc(sp)
    sol = np.random.default_rng(2).normal(size=sp.ndof)
    got = d.norms(sol, exact="sin")
    ref = _norms_numpy(mesh, sp, sol, 2, _sin)
    vals = np.array([got["l2_error"], got["h1_error"], got["l2_norm"], got["h1_norm"]])
    assert np.max(np.abs(vals - ref) / np.abs(ref)) < 1e-12
    again = d.norms(sol, exact="sin")
    assert again == got


@pytest.mark.parametrize("refs", [[], [1, 14, 27]])
def test_quadratic_solution_has_zero_error(gpu, refs):
    import scipy.sparse as sps
    import scipy.sparse.linalg as spl
    mesh = h.unit_cube(3)
    mesh.ugh()
    if refs:
        mesh.refine_elements(refs)
    sp = h.H1Space(mesh)
    sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    sp.set_element_orders(np.full((len(mesh.hexes), 3), 2, np.int32))
    sp.assign_dofs()
    d, M, V = _disc(sp)
    d.assemble(M, V)
    n = sp.ndof
    sol = spl.spsolve(sps.csc_matrix((M.Ax, M.Ai, M.Ap), shape=(n, n)), V.v)
    r = d.norms(sol, exact="quadratic")
    assert r["l2_error"] < 1e-9 and r["h1_error"] < 1e-9
    # int u^2 = 3/5 + 6/9, int |grad u|^2 = 4 over the unit cube
    assert abs(r["l2_norm"] - np.sqrt(3 / 5 + 6 / 9)) < 1e-10
    assert abs(r["h1_norm"] - np.sqrt(3 / 5 + 6 / 9 + 4)) < 1e-10
