"""The reference's stock quadrature on the device (H3DG_QUAD_STOCK): every
pair integrated with order(u) + order(v) + 1 per direction and the load
vector with order 24, as the stock int_grad_u_grad_v / int_u_v / int_F_v do
(src/integrals/h1.h:115-177).  Checked against fixtures the reference made
with its stock forms on non-affine meshes (tests/golden/stock/), and against
the restatement of the rule on a larger mesh."""
import numpy as np
import pytest

import hermes3d_b200 as h
from hermes3d_b200 import _capi
from helpers import FP64_RTOL, disc_of, load_stock, rel_err, space_of, stock_names
from oracle import port

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", stock_names())
def test_stock_rule_matches_reference(gpu, name):
    g = load_stock(name)
    sp = space_of(g)
    d = disc_of(g, sp)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    assert np.array_equal(M.Ap, g["Ap"]) and np.array_equal(M.Ai, g["Ai"])
    d.assemble(M, V)
    assert rel_err(M.Ax, g["Ax"]) < FP64_RTOL
    assert rel_err(V.v, g["rhs"]) < FP64_RTOL


@pytest.mark.parametrize("p", [1, 2, 3])
def test_stock_rule_matches_restatement(gpu, p):
    mesh = h.permute_vertices(h.unit_cube(5 if p < 3 else 3, 0.2, 4), seed=p)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    sp.set_uniform_order(p)
    sp.assign_dofs()
    coef = np.random.default_rng(p).uniform(0.5, 2.0, mesh.num_elements)
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v_plus_u_v, coef)
    d.set_linear_form(h.int_F_v("sin"))
    d.set_quadrature(stock=True)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)
    ax, v = M.Ax.copy(), V.v.copy()
    d.assemble(M, V)
    assert np.array_equal(M.Ax, ax) and np.array_equal(V.v, v)      # bitwise reproducible
    al = port.asmlists_from_space(sp, mesh.num_elements)
    Ax, rhs = port.assemble_stock(mesh.xyz, mesh.hexes - 1, al, sp.ndof, M.Ap, M.Ai, mass=True, gradcoef=coef, lf=2)
    assert rel_err(ax, Ax) < FP64_RTOL and rel_err(v, rhs) < FP64_RTOL


def test_stock_rule_rejects_what_it_does_not_cover(gpu):
    mesh = h.unit_cube(2)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_uniform_order(4)
    sp.assign_dofs()
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v)
    d.set_quadrature(stock=True)
    with pytest.raises(_capi.H3dgError) as e:
        d.create(h.UMFPackMatrix(), h.UMFPackVector())
    assert e.value.status == _capi.H3DG_ERR_INVALID_ARG
