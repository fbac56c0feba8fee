"""Refined meshes with hanging nodes on the GPU: the batched path with the
constrained-element kernel (element matrix in the raised canonical basis,
then the constraint weights) against fixtures the reference itself produced;
FP64 tolerance 1e-12, pattern bit for bit, replay bitwise reproducible."""
import numpy as np
import pytest

import hermes3d_b200 as h
from helpers import FP64_RTOL, disc_of, load_refined, refined_names, refined_space_of, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", refined_names())
def test_refined_assembly_matches_reference(gpu, name):
    g = load_refined(name)
    mesh, sp = refined_space_of(g)
    d = disc_of(g, sp)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)
    assert np.array_equal(M.Ap, g["Ap"]) and np.array_equal(M.Ai, g["Ai"])
    assert rel_err(M.Ax, g["Ax"]) < FP64_RTOL
    assert rel_err(V.v, g["rhs"]) < FP64_RTOL


def test_refined_replay_is_bitwise_reproducible(gpu):
    g = load_refined("ref_aniso_c3_like")
    mesh, sp = refined_space_of(g)
    d = disc_of(g, sp)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)
    ax, v = M.Ax.copy(), V.v.copy()
    for _ in range(3):
        d.assemble(M, V)
        assert np.array_equal(M.Ax, ax) and np.array_equal(V.v, v)


def _parts(name):
    import torch
    g = load_refined(name)
    mesh, sp = refined_space_of(g)
    d = disc_of(g, sp)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)
    Ax = torch.zeros(len(M.Ax), dtype=torch.float64, device="cuda")
    rhs = torch.zeros(len(V.v), dtype=torch.float64, device="cuda")
    d.assemble_device(Ax, None)
    d.assemble_device(None, rhs)
    torch.cuda.synchronize()
    return M.Ax, V.v, Ax.cpu().numpy(), rhs.cpu().numpy()


def test_refined_rhs_only_and_matrix_only(gpu):
    """Matrix-only assembly gives the full assembly's matrix bit for bit; an
    RHS-only assembly has no Dirichlet lifting (the reference lifts inside the
    matrix loop, src/discretization.cc:296-317), so it equals the full RHS
    without non-homogeneous Dirichlet data and differs from it with."""
    ax, v, ax1, v1 = _parts("ref_lifting_p3")
    assert np.array_equal(ax1, ax)
    assert not np.allclose(v1, v)
    ax, v, ax1, v1 = _parts("ref_aniso_c3_like")
    assert np.array_equal(ax1, ax)
    assert np.array_equal(v1, v)
