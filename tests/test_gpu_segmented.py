"""Segmented scatter (element matrices into an L2-resident ring, then every
CSC column summed in assembly order and written once) against the colour
sweeps: the same bits, on meshes large enough that the ring's slots are
reused many times, with Dirichlet lifting, per-element coefficients, the
matrix alone, the RHS alone, partitioned plans, and the corrupted-position
hook.  The colour sweeps themselves are pinned to the reference by the
parity tests."""
import numpy as np
import pytest

import hermes3d_b200 as h
from hermes3d_b200 import _capi
from helpers import FP64_RTOL, rel_err
from oracle import port

pytestmark = pytest.mark.gpu


def _space(n, p, jitter=0.2, seed=3, lifting=True):
    mesh = h.permute_vertices(h.unit_cube(n, jitter, seed), seed=seed)
    mesh.ugh()
    sp = h.H1Space(mesh)
    if lifting:
        sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    sp.set_uniform_order(p)
    sp.assign_dofs()
    return mesh, sp


def _assemble(monkeypatch, scatter, mesh, sp, nq, matrix=True, rhs=True, coef=True, nparts=1, part=0):
    monkeypatch.setenv("H3DG_SCATTER", scatter)
    d = h.Discretization()
    if nparts > 1:
        d.set_partition(nparts, part)
    d.set_spaces(sp)
    c = np.random.default_rng(5).uniform(0.5, 2.0, mesh.num_elements) if coef else None
    d.set_bilinear_form(h.int_grad_u_grad_v_plus_u_v, c)
    d.set_linear_form(h.int_F_v("sin"))
    d.set_quadrature(points=nq)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M if matrix else None, V if rhs else None)
    return d, M, V


@pytest.mark.parametrize("n,p,nq", [(24, 1, 3), (24, 2, 4), (12, 3, 5)])
def test_segmented_equals_colour_sweeps(gpu, monkeypatch, n, p, nq):
    mesh, sp = _space(n, p)
    ds, Ms, Vs = _assemble(monkeypatch, "segmented", mesh, sp, nq)
    assert ds.last_launch_count() == 1                  # one persistent launch
    dc, Mc, Vc = _assemble(monkeypatch, "colour", mesh, sp, nq)
    assert dc.last_launch_count() > 1
    assert np.array_equal(Ms.Ax, Mc.Ax)
    assert np.array_equal(Vs.v, Vc.v)
    # and again: bitwise reproducible run to run
    ds.assemble(Ms, Vs)
    assert np.array_equal(Ms.Ax, Mc.Ax) and np.array_equal(Vs.v, Vc.v)


def test_segmented_matches_restatement(gpu, monkeypatch):
    mesh, sp = _space(6, 2, seed=8)
    d, M, V = _assemble(monkeypatch, "segmented", mesh, sp, 4, coef=False)
    al = port.asmlists_from_space(sp, mesh.num_elements)
    Ax, rhs = port.assemble(mesh.xyz, mesh.hexes - 1, 4, al, sp.ndof, M.Ap, M.Ai, mass=True, lf=2)
    assert rel_err(M.Ax, Ax) < FP64_RTOL and rel_err(V.v, rhs) < FP64_RTOL


@pytest.mark.parametrize("matrix,rhs", [(True, False), (False, True)])
def test_segmented_matrix_or_rhs_alone(gpu, monkeypatch, matrix, rhs):
    mesh, sp = _space(16, 2)
    ds, Ms, Vs = _assemble(monkeypatch, "segmented", mesh, sp, 4, matrix=matrix, rhs=rhs)
    dc, Mc, Vc = _assemble(monkeypatch, "colour", mesh, sp, 4, matrix=matrix, rhs=rhs)
    if matrix:
        assert np.array_equal(Ms.Ax, Mc.Ax)
    if rhs:
        assert np.array_equal(Vs.v, Vc.v)


def test_segmented_partition_parts(gpu, monkeypatch):
    """Each part of a z-slab partition: its columns and its RHS entries
    (partial sums for DOFs it does not own) as the colour sweeps give them."""
    mesh, sp = _space(12, 2)
    for part in range(3):
        ds, Ms, Vs = _assemble(monkeypatch, "segmented", mesh, sp, 4, nparts=3, part=part)
        dc, Mc, Vc = _assemble(monkeypatch, "colour", mesh, sp, 4, nparts=3, part=part)
        assert np.array_equal(Ms.Ax, Mc.Ax) and np.array_equal(Vs.v, Vc.v)


def test_segmented_reports_a_corrupt_position(gpu, monkeypatch):
    mesh, sp = _space(8, 2)
    d, M, V = _assemble(monkeypatch, "segmented", mesh, sp, 4)
    good = M.Ax.copy()
    d.debug_inject(_capi.DEBUG_CORRUPT_POSITION)
    with pytest.raises(_capi.H3dgError) as e:
        d.assemble(M, V)
    assert e.value.status == _capi.H3DG_ERR_STATE
    d.create(M, V)                                 # a fresh plan
    d.assemble(M, V)
    assert np.array_equal(M.Ax, good)
