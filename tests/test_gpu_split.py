"""Split precision on tcgen05 against the FP64 kernel, the reference
fixtures and the restatement oracle:
  PREC_TF32X3: FP32 z and y stages, 3xTF32 x stage; tolerance 1e-6;
  PREC_OZAKI:  FP64 z and y stages, x stage on int8 slices (7 per operand,
               exact int32 accumulation); tolerance 1e-12.
Tolerances are of the largest matrix entry, entrywise (max |dA| / max |A|),
and normwise (||dA||_2 / ||A||_2).  The load vector is FP64 throughout, so
it keeps the FP64 tolerance."""
import os

import numpy as np
import pytest

import hermes3d_b200 as h
from helpers import FP64_RTOL, disc_of, load, rel_err, space_of
from oracle import port

pytestmark = pytest.mark.gpu

SPLIT_RTOL = 1e-6
TOL = {h.PREC_TF32X3: 1e-6, h.PREC_OZAKI: 1e-12}
PRECS = [h.PREC_TF32X3, h.PREC_OZAKI]


def _norm_err(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture
def force_high_order():
    os.environ["H3DG_FORCE_HIGH_ORDER"] = "1"
    yield
    del os.environ["H3DG_FORCE_HIGH_ORDER"]


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("name", ["c1_small", "perm_p3_mass_sin", "perm_p2_lifting", "coef_p3"])
def test_split_on_reference_fixtures(gpu, force_high_order, name, prec):
    g = load(name)
    sp = space_of(g)
    d = disc_of(g, sp)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V, precision=prec)
    e_max, e_norm = rel_err(M.Ax, g["Ax"]), _norm_err(M.Ax, g["Ax"])
    print("%s prec %d: split error max %.2e norm %.2e" % (name, prec, e_max, e_norm))
    assert e_max < TOL[prec] and e_norm < TOL[prec]
    assert rel_err(V.v, g["rhs"]) < FP64_RTOL


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("p,bc,n", [(5, "lifting", 2), (6, "dirichlet0", 2), (7, "lifting", 1), (8, "natural", 1)])
def test_split_matches_restatement(gpu, p, bc, n, prec):
    mesh = h.permute_vertices(h.unit_cube(n, 0.15, 3), seed=p)
    mesh.ugh()
    sp = h.H1Space(mesh)
    if bc == "natural":
        sp.set_bc_types(lambda m: h.BC_NATURAL)
    if bc == "lifting":
        sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    sp.set_uniform_order(p)
    sp.assign_dofs()
    d = h.Discretization()
    d.set_spaces(sp)
    coef = np.random.default_rng(p).uniform(0.5, 2.0, mesh.num_elements)
    d.set_bilinear_form(h.int_grad_u_grad_v_plus_u_v if bc != "dirichlet0" else h.int_grad_u_grad_v, coef)
    d.set_linear_form(h.int_F_v(-6.0 if bc == "lifting" else "sin"))
    d.set_quadrature(p_plus=2)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V, precision=prec)
    al = port.asmlists_from_space(sp, mesh.num_elements)
    Ax, rhs = port.assemble(mesh.xyz, mesh.hexes - 1, p + 2, al, sp.ndof, M.Ap, M.Ai, mass=(bc != "dirichlet0"),
                            gradcoef=coef, lf=1 if bc == "lifting" else 2, lf_value=-6.0)
    e_max, e_norm = rel_err(M.Ax, Ax), _norm_err(M.Ax, Ax)
    print("p=%d %s prec %d: split error max %.2e norm %.2e" % (p, bc, prec, e_max, e_norm))
    assert e_max < TOL[prec] and e_norm < TOL[prec]
    assert rel_err(V.v, rhs) < FP64_RTOL


@pytest.mark.parametrize("prec", PRECS)
def test_split_is_deterministic_and_close_to_fp64(gpu, prec):
    import torch
    mesh = h.unit_cube(3, 0.2, 11)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_uniform_order(6)
    sp.assign_dofs()
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v, np.random.default_rng(1).uniform(0.5, 2.0, mesh.num_elements))
    d.set_linear_form(None)
    d.set_quadrature(points=8)
    d.create()
    A64 = torch.empty(d.nnz, dtype=torch.float64, device="cuda")
    A1, A2 = torch.empty_like(A64), torch.empty_like(A64)
    d.assemble_device(A64)
    d.assemble_device(A1, precision=prec)
    d.assemble_device(A2, precision=prec)
    torch.cuda.synchronize()
    assert torch.equal(A1, A2)
    a, b = A1.cpu().numpy(), A64.cpu().numpy()
    print("prec %d vs FP64: max %.2e norm %.2e" % (prec, rel_err(a, b), _norm_err(a, b)))
    assert rel_err(a, b) < TOL[prec] and _norm_err(a, b) < TOL[prec]
    # the split result is not the FP64 one (the tensor path really ran)
    assert not np.array_equal(a, b)


def test_split_order_3_uses_fp64(gpu):
    """p = 3 has no batched tensor-core kernel and is below the high-order
    threshold, where the FP64 kernels are the faster choice: PREC_TF32X3 then
    returns the FP64 matrix.  (p <= 2 takes the batched kernel,
    tests/test_gpu_split_low_order.py.)"""
    g = load("perm_p3_mass_sin")
    sp = space_of(g)
    d = disc_of(g, sp)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V, precision=h.PREC_TF32X3)
    M2, V2 = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M2, V2)
    d.assemble(M2, V2)
    assert np.array_equal(M.Ax, M2.Ax)


def test_precision_hint_puts_order_4_on_the_tensor_cores(gpu):
    """set_precision(PREC_TF32X3) before create(): p = 4 takes the tensor-core
    kernel (faster there), still within 1e-6 of the FP64 assembly."""
    def build(hint):
        mesh = h.unit_cube(3, 0.2, 4)
        mesh.ugh()
        sp = h.H1Space(mesh)
        sp.set_uniform_order(4)
        sp.assign_dofs()
        d = h.Discretization()
        d.set_spaces(sp)
        d.set_bilinear_form(h.int_grad_u_grad_v)
        d.set_linear_form(h.int_F_v(1.0))
        d.set_quadrature(points=6)
        if hint is not None:
            d.set_precision(hint)
        M, V = h.UMFPackMatrix(), h.UMFPackVector()
        d.create(M, V)
        return d, M, V
    d64, M64, V64 = build(None)
    d64.assemble(M64, V64)
    d, M, V = build(h.PREC_TF32X3)
    d.assemble(M, V, precision=h.PREC_TF32X3)
    assert np.array_equal(M.Ap, M64.Ap) and np.array_equal(M.Ai, M64.Ai)
    assert rel_err(M.Ax, M64.Ax) < SPLIT_RTOL and not np.array_equal(M.Ax, M64.Ax)
    assert rel_err(V.v, V64.v) < FP64_RTOL
