"""h3dg_disc_assemble_host_noalloc: assembly into host sinks staged in the
library's fixed device array, without any device allocation -- for callers
whose device memory is all held by their own pool, or who cannot accept the
device-wide synchronisation of cudaFree.  Collected last (file name) so it
also runs after every other test in one process.

Each case makes one allocating assembly first, then two no-allocation calls
in a row that must give the allocating call's bits while the device's free
memory (cudaMemGetInfo) stays exactly the same.  The cases are sized so that
any buffer the call could allocate (Ax, rhs, the split-precision work area)
is at least 2 MiB, the granularity at which cudaMemGetInfo moves."""
import numpy as np
import pytest

import hermes3d_b200 as h
from hermes3d_b200 import _capi
from helpers import (disc_of, load, load_refined, load_surface, refined_space_of, space_of, surface_problem)


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


def _free_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def _check_twice(d, M, V, precision=h.PREC_FP64, rhs_only=False):
    """Two no-allocation calls against the allocating call's result, with the
    free device memory unchanged around them.  An RHS-only call carries no
    Dirichlet lifting (the lifting reaches the RHS only with the matrix, as in
    the reference), so it is compared with an allocating RHS-only call."""
    if rhs_only:
        V = h.UMFPackVector()
        V.v = np.full(M.ndofs, np.nan)
        d.assemble(None, V, precision=precision)
    before = _free_bytes()
    for _ in range(2):
        M2, V2 = _sinks_like(M, V)
        d.assemble_noalloc(None if rhs_only else M2, V2, precision=precision)
        if not rhs_only:
            assert np.array_equal(M2.Ax, M.Ax)
        assert np.array_equal(V2.v, V.v)
    assert _free_bytes() == before


def _uniform(n, p, nq, jitter=0.15):
    mesh = h.permute_vertices(h.unit_cube(n, jitter, 5), seed=n)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    sp.set_uniform_order(p)
    sp.assign_dofs()
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v_plus_u_v, np.random.default_rng(2).uniform(0.5, 2.0, mesh.num_elements))
    d.set_linear_form(h.int_F_v("sin"))
    d.set_quadrature(points=nq)
    return mesh, sp, d


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c1_small", "perm_p2_lifting"])
def test_noalloc_matches_assemble_host_twice(gpu, name):
    g, sp, d = _disc(name)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)                      # the allocating call comes first
    _check_twice(d, M, V)


@pytest.mark.gpu
def test_noalloc_low_order_leaves_free_memory_unchanged(gpu):
    mesh, sp, d = _uniform(10, 2, 4)      # Ax ~ 4 MB: an allocation of it would show
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    assert 8 * d.nnz > (2 << 20)
    d.assemble(M, V)
    _check_twice(d, M, V)
    _check_twice(d, M, V, rhs_only=True)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [h.PREC_FP64, h.PREC_TF32X3, h.PREC_OZAKI])
def test_noalloc_split_precision_twice(gpu, prec):
    # p = 8, 10^3 points: the work area is ~9 MB; FP64 runs the tensor-core (DMMA)
    # kernel through the scatter stream the allocating call built
    mesh, sp, d = _uniform(2, 8, 10)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V, precision=prec)
    _check_twice(d, M, V, precision=prec)


@pytest.mark.gpu
def test_noalloc_mixed_orders_direct_launches(gpu, monkeypatch):
    """A mixed-order plan: the allocating call replays its CUDA graph, the
    no-allocation call launches the same kernels directly (instantiating a
    graph may allocate); same bits."""
    monkeypatch.setenv("H3DG_FORCE_MIXED", "1")
    g, sp, d = _disc("perm_p3_mass_sin")
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)
    _check_twice(d, M, V)


@pytest.mark.gpu
def test_noalloc_refined_mesh(gpu):
    g = load_refined("ref_aniso_c3_like")
    mesh, sp = refined_space_of(g)
    d = disc_of(g, sp)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)
    _check_twice(d, M, V)


@pytest.mark.gpu
def test_noalloc_surface_forms(gpu):
    mesh, sp, d = surface_problem(load_surface("surf_mixed_lifting_p3"))
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)
    _check_twice(d, M, V)


@pytest.mark.gpu
def test_noalloc_needs_an_allocating_call_with_the_same_precision(gpu):
    mesh, sp, d = _uniform(2, 5, 7)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    with pytest.raises(_capi.H3dgError) as e:          # nothing prepared yet
        d.assemble_noalloc(M, V)
    assert e.value.status == _capi.H3DG_ERR_STATE
    d.assemble(M, V, precision=h.PREC_TF32X3)
    for prec in (h.PREC_FP64, h.PREC_OZAKI):           # another precision was prepared
        with pytest.raises(_capi.H3dgError) as e:
            d.assemble_noalloc(M, V, precision=prec)
        assert e.value.status == _capi.H3DG_ERR_STATE
    d.create(M, V)                                      # a new plan forgets what was prepared
    with pytest.raises(_capi.H3dgError) as e:
        d.assemble_noalloc(M, V, precision=h.PREC_TF32X3)
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
