"""FP64 high-order assembly on the FP64 tensor cores (k_assemble_fp64_dm):
stages 2 and 3 as DMMA GEMMs.  Checked against the reference's own fixtures
(p = 5..8), against the FMA kernel (H3DG_HO_FP64_FMA=1) on the same plan,
for bitwise reproducibility, and for the first-touch stores that replace the
zero-fill of Ax (the matrix is assembled into memory full of NaN)."""
import os

import numpy as np
import pytest
import torch

import hermes3d_b200 as h
from hermes3d_b200.mesh import unit_cube
from helpers import FP64_RTOL, highorder_names, highorder_problem, load_highorder, rel_err

pytestmark = pytest.mark.gpu


def _assemble(d, fma=False):
    if fma:
        os.environ["H3DG_HO_FP64_FMA"] = "1"
    try:
        M, V = h.UMFPackMatrix(), h.UMFPackVector()
        d.create(M, V)
        d.assemble(M, V)
        return M, V, d.last_kernel()
    finally:
        os.environ.pop("H3DG_HO_FP64_FMA", None)


@pytest.mark.parametrize("name", highorder_names())
def test_dmma_against_reference_and_fma(gpu, name):
    g = load_highorder(name)
    _, _, d = highorder_problem(g)
    M, V, kind = _assemble(d)
    assert kind == "ho_fp64_dmma"
    assert np.array_equal(M.Ap, g["Ap"]) and np.array_equal(M.Ai, g["Ai"])
    assert rel_err(M.Ax, g["Ax"]) < FP64_RTOL
    assert rel_err(V.v, g["rhs"]) < FP64_RTOL
    _, _, d2 = highorder_problem(g)
    Mf, Vf, kind_f = _assemble(d2, fma=True)
    assert kind_f == "ho_fp64_fma"
    e = rel_err(M.Ax, Mf.Ax)
    print("%s: DMMA vs FMA kernel %.2e" % (name, e))
    assert e < 1e-13
    assert np.array_equal(V.v, Vf.v)          # the load vector is the same code in both


@pytest.mark.parametrize("p", [4, 5, 6, 7, 8])
def test_dmma_reproducible_and_store_first(gpu, p):
    """Uniform order p on a jittered 3^3 mesh with Dirichlet lifting and mass:
    bitwise identical twice, and into NaN-filled device memory (every slot's
    first contribution is a store)."""
    mesh = unit_cube(3, jitter=0.15, seed=p)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    sp.set_uniform_order(p)
    sp.assign_dofs()
    d = h.Discretization(0)
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v_plus_u_v)
    d.set_linear_form(h.int_F_v("sin"))
    d.set_quadrature(p_plus=2)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    if p == 4:                                   # p = 4 takes the low-order path by default
        os.environ["H3DG_FORCE_HIGH_ORDER"] = "1"
    try:
        d.create(M, V)
    finally:
        os.environ.pop("H3DG_FORCE_HIGH_ORDER", None)
    ax = torch.full((len(M.Ai),), float("nan"), dtype=torch.float64, device="cuda")
    rhs = torch.zeros(sp.ndof, dtype=torch.float64, device="cuda")
    d.assemble_device(ax, rhs)
    assert d.last_kernel() == "ho_fp64_dmma"
    a1 = ax.cpu().numpy().copy()
    assert np.isfinite(a1).all()
    ax.fill_(float("nan"))
    d.assemble_device(ax, rhs)
    assert np.array_equal(a1.view(np.int64), ax.cpu().numpy().view(np.int64))
    os.environ["H3DG_HO_FP64_FMA"] = "1"
    try:
        ax.fill_(0.0)
        d.assemble_device(ax, rhs)
        assert d.last_kernel() == "ho_fp64_fma"
    finally:
        os.environ.pop("H3DG_HO_FP64_FMA", None)
    assert rel_err(a1, ax.cpu().numpy()) < 1e-13


def test_dmma_whole_and_half_elements(gpu):
    """12^3 elements at p = 5: colours of ~216 elements run one round of whole
    elements and a last round of half elements (trial z halves) over the SMs;
    the result matches the FMA kernel and repeats bit for bit."""
    mesh = unit_cube(12, jitter=0.1, seed=3)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_uniform_order(5)
    sp.assign_dofs()
    d = h.Discretization(0)
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v)
    d.set_linear_form(h.int_F_v(1.0))
    d.set_quadrature(p_plus=2)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    ax = torch.empty(len(M.Ai), dtype=torch.float64, device="cuda")
    rhs = torch.zeros(sp.ndof, dtype=torch.float64, device="cuda")
    d.assemble_device(ax, rhs)
    assert d.last_kernel() == "ho_fp64_dmma"
    a1, r1 = ax.cpu().numpy().copy(), rhs.cpu().numpy().copy()
    d.assemble_device(ax, rhs)
    assert np.array_equal(a1.view(np.int64), ax.cpu().numpy().view(np.int64))
    os.environ["H3DG_HO_FP64_FMA"] = "1"
    try:
        ax.zero_()
        d.assemble_device(ax, rhs)
        assert d.last_kernel() == "ho_fp64_fma"
    finally:
        os.environ.pop("H3DG_HO_FP64_FMA", None)
    assert rel_err(a1, ax.cpu().numpy()) < 1e-13
    assert np.array_equal(r1, rhs.cpu().numpy())


@pytest.mark.parametrize("p", [4, 5, 6])
def test_dmma_variants_give_the_same_bits(gpu, p):
    """The smaller-CTA variant (fewer pairs per iteration, two CTAs per SM)
    against the default: the same MMAs per pair and the same posts."""
    mesh = unit_cube(5, jitter=0.15, seed=p)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    sp.set_uniform_order(p)
    sp.assign_dofs()
    d = h.Discretization(0)
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v_plus_u_v)
    d.set_linear_form(h.int_F_v("sin"))
    d.set_quadrature(p_plus=2)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    out = []
    for var in ("0", "1"):
        os.environ["H3DG_DM_VARIANT"] = var
        try:
            d.assemble(M, V)
            assert d.last_kernel() == "ho_fp64_dmma"
            out.append((M.Ax.copy(), V.v.copy()))
        finally:
            os.environ.pop("H3DG_DM_VARIANT", None)
    assert np.array_equal(out[0][0].view(np.int64), out[1][0].view(np.int64))
    assert np.array_equal(out[0][1], out[1][1])
