"""Solve-based known-answer checks in the manner of the reference's calc/
and hang-nodes tests (u = x^2 + y^2 + z^2 is reproduced exactly by p >= 2):
the matrix and RHS assembled on the GPU for -Laplace(u) = -6 with Dirichlet
data u, solved on the host (scipy, test infrastructure), evaluated from the
assembly lists at random points of every active element.  Covers uniform,
anisotropic-order and refined (hanging-node) meshes (affine, so the integrals are exact)."""
import numpy as np
import pytest

import hermes3d_b200 as h

pytestmark = pytest.mark.gpu


def _lobatto(k, x):
    from numpy.polynomial import legendre as L
    if k == 0:
        return (1 - x) / 2
    if k == 1:
        return (1 + x) / 2
    c = np.zeros(k + 1)
    c[k] = 1.0
    c2 = np.zeros(k + 1)
    c2[k - 2] = 1.0
    return (L.legval(x, c) - L.legval(x, c2)) / np.sqrt(2 * (2 * k - 1))


def _decode(idx):
    ori = (idx >> 12) & 7
    ind = [(idx >> 8) & 15, (idx >> 4) & 15, idx & 15]
    flip = [0, 0, 0]
    n01 = sum(i < 2 for i in ind)
    if n01 == 2:
        for d in range(3):
            if ind[d] >= 2:
                flip[d] = ori & 1
    elif n01 == 1:
        ds = [d for d in range(3) if ind[d] >= 2]
        if ori % 2 == 1:
            flip[ds[0]] = 1
        if ori % 4 >= 2:
            flip[ds[1]] = 1
        if ori >= 4:
            ind[ds[0]], ind[ds[1]] = ind[ds[1]], ind[ds[0]]
            flip[ds[0]], flip[ds[1]] = flip[ds[1]], flip[ds[0]]
    sign = -1 if sum(1 for d in range(3) if flip[d] and ind[d] & 1) % 2 else 1
    return ind, sign


def _solve_and_check(mesh, sp, nq=2):
    import scipy.sparse as sps
    import scipy.sparse.linalg as spl
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v)
    d.set_linear_form(h.int_F_v(-6.0))
    d.set_quadrature(p_plus=nq)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)
    n = sp.ndof
    A = sps.csc_matrix((M.Ax, M.Ai, M.Ap), shape=(n, n))
    x = spl.spsolve(A, V.v)
    rng = np.random.default_rng(0)
    ref = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1], [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]])
    err = 0.0
    for e in np.nonzero(mesh.active)[0] + 1:
        idx, dof, coef = sp.get_element_assembly_list(int(e))
        X = mesh.xyz[mesh.hexes[e - 1] - 1]
        for _ in range(3):
            xi = rng.uniform(-1, 1, 3)
            N = np.prod([(1 + ref[:, r] * xi[r]) / 2 for r in range(3)], axis=0)
            p = N @ X
            uh = 0.0
            for i, dd, c in zip(idx, dof, coef):
                ind, sg = _decode(int(i))
                phi = sg * _lobatto(ind[0], xi[0]) * _lobatto(ind[1], xi[1]) * _lobatto(ind[2], xi[2])
                uh += c * phi * (x[dd] if dd >= 0 else 1.0)
            err = max(err, abs(uh - (p @ p)))
    return err


def _space(mesh, orders):
    sp = h.H1Space(mesh)
    sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    sp.set_element_orders(orders)
    sp.assign_dofs()
    return sp


def test_quadratic_reproduced_uniform(gpu):
    mesh = h.unit_cube(3)
    mesh.ugh()
    assert _solve_and_check(mesh, _space(mesh, np.full((27, 3), 2, np.int32))) < 1e-10


def test_quadratic_reproduced_anisotropic_orders(gpu):
    mesh = h.unit_cube(3)
    mesh.ugh()
    o = np.random.default_rng(5).integers(2, 5, size=(27, 3)).astype(np.int32)
    assert _solve_and_check(mesh, _space(mesh, o)) < 1e-10


@pytest.mark.parametrize("refs,p", [([14], 2), ([1, 14, 27], 3), ([2, 5, 13, 22], 2)])
def test_quadratic_reproduced_with_hanging_nodes(gpu, refs, p):
    mesh = h.unit_cube(3, 0.0)
    mesh.ugh()
    mesh.refine_elements(refs)
    sp = _space(mesh, np.full((len(mesh.hexes), 3), p, np.int32))
    assert _solve_and_check(mesh, sp) < 1e-10
