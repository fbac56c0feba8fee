"""h3dg_disc_assemble_host_noalloc: assembly into host sinks staged in the
library's fixed device array, without any device allocation.  Collected
last (file name) so it also runs after every other test in one process."""
import numpy as np
import pytest

import hermes3d_b200 as h
from hermes3d_b200 import _capi
from helpers import disc_of, load, space_of


def _disc(name):
    g = load(name)
    sp = space_of(g)
    return g, sp, disc_of(g, sp)


def _sinks_like(M, V):
    """Fresh host sinks on the same pattern (create() would build a new plan)."""
    M2, V2 = h.UMFPackMatrix(), h.UMFPackVector()
    M2.Ap, M2.Ai, M2.ndofs = M.Ap, M.Ai, M.ndofs
    M2.Ax = np.full_like(M.Ax, np.nan)
    V2.v = np.full_like(V.v, np.nan)
    return M2, V2


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c1_small", "perm_p2_lifting"])
def test_noalloc_matches_assemble_host_twice(gpu, name):
    g, sp, d = _disc(name)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)                      # the allocating call comes first
    for _ in range(2):                    # two calls in a row reuse the array
        M2, V2 = _sinks_like(M, V)
        d.assemble_noalloc(M2, V2)
        assert np.array_equal(M2.Ax, M.Ax)
        assert np.array_equal(V2.v, V.v)


@pytest.mark.gpu
def test_noalloc_split_precision_twice(gpu):
    mesh = h.unit_cube(2, 0.15, 5)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_uniform_order(5)
    sp.assign_dofs()
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v, np.random.default_rng(2).uniform(0.5, 2.0, mesh.num_elements))
    d.set_linear_form(h.int_F_v("sin"))
    d.set_quadrature(points=7)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V, precision=h.PREC_TF32X3)
    for _ in range(2):
        M2, V2 = _sinks_like(M, V)
        d.assemble_noalloc(M2, V2, precision=h.PREC_TF32X3)
        assert np.array_equal(M2.Ax, M.Ax)
        assert np.array_equal(V2.v, V.v)


@pytest.mark.gpu
def test_noalloc_needs_a_prior_allocating_call(gpu):
    g, sp, d = _disc("c1_small")
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    with pytest.raises(_capi.H3dgError) as e:
        d.assemble_noalloc(M, V)
    assert e.value.status == _capi.H3DG_ERR_STATE


def test_noalloc_rejects_oversize():
    mesh = h.unit_cube(12, 0.0, 0)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_uniform_order(3)
    sp.assign_dofs()
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v)
    d.set_linear_form(h.int_F_v(1.0))
    d.set_quadrature(points=5)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    assert d.nnz + d.ndof > _capi.NOALLOC_SCRATCH_DOUBLES
    with pytest.raises(_capi.H3dgError) as e:
        d.assemble_noalloc(M, V)
    assert e.value.status == _capi.H3DG_ERR_TOO_LARGE
    assert "16 MiB" in str(e.value)
