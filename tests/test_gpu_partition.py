"""z-slab parts assembled on the GPU (one after another on one device: the
parts never wait on each other): every owned CSC column and owned rhs entry
equals the whole-mesh assembly, for the low-order, high-order, split-precision
and mixed-order kernels."""
import numpy as np
import pytest

import hermes3d_b200 as h
from helpers import FP64_RTOL

pytestmark = pytest.mark.gpu


def _space(order, n=4, seed=3, refine=()):
    mesh = h.unit_cube(n, 0.2, seed)
    mesh.ugh()
    if refine:
        mesh.refine_elements(list(refine))
    sp = h.H1Space(mesh)
    sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    if isinstance(order, int):
        sp.set_uniform_order(order)
    else:
        sp.set_element_orders(np.random.default_rng(seed).integers(order[0], order[1] + 1,
                                                                   size=(mesh.num_elements, 3)))
    sp.assign_dofs()
    return mesh, sp


def _assemble(sp, nparts=1, part=0, precision=h.PREC_FP64):
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v_plus_u_v, np.linspace(0.5, 2.0, sp.mesh.num_elements))
    d.set_linear_form(h.int_F_v(-6.0))
    d.set_quadrature(p_plus=2)
    if nparts > 1:
        d.set_partition(nparts, part)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V, precision=precision)
    return d, M, V


@pytest.mark.parametrize("order,precision,tol", [(2, h.PREC_FP64, FP64_RTOL), (5, h.PREC_FP64, FP64_RTOL),
                                                 (5, h.PREC_TF32X3, 1e-6), ((1, 4), h.PREC_FP64, FP64_RTOL)])
def test_parts_match_whole_mesh(gpu, order, precision, tol):
    n = 3 if order == 5 else 4
    mesh, sp = _space(order, n)
    _, Mg, Vg = _assemble(sp, precision=precision)
    scale = np.abs(Mg.Ax).max()
    for part in range(2):
        d, M, V = _assemble(sp, 2, part, precision)
        owned = d.partition()["owned"]
        for j in np.flatnonzero(owned):
            a, b = M.Ax[M.Ap[j]:M.Ap[j + 1]], Mg.Ax[Mg.Ap[j]:Mg.Ap[j + 1]]
            assert np.max(np.abs(a - b)) <= tol * scale, j
        assert np.max(np.abs(V.v[owned] - Vg.v[owned])) <= FP64_RTOL * np.abs(Vg.v).max()


def test_parts_of_a_refined_mesh_match_whole_mesh(gpu):
    """Hanging nodes at and away from the slab cut, mixed orders: the owned
    columns and rhs entries of each part equal the whole mesh's."""
    mesh, sp = _space((1, 3), 4, refine=(6, 22, 27, 43))
    _, Mg, Vg = _assemble(sp)
    scale = np.abs(Mg.Ax).max()
    for part in range(2):
        d, M, V = _assemble(sp, 2, part)
        owned = d.partition()["owned"]
        for j in np.flatnonzero(owned):
            a, b = M.Ax[M.Ap[j]:M.Ap[j + 1]], Mg.Ax[Mg.Ap[j]:Mg.Ap[j + 1]]
            assert np.max(np.abs(a - b)) <= FP64_RTOL * scale, j
        assert np.max(np.abs(V.v[owned] - Vg.v[owned])) <= FP64_RTOL * np.abs(Vg.v).max()

