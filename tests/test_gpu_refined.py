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


def test_c3_sample_against_reference(gpu):
    """The mixed-order, hanging-node workload on the largest sample the
    reference assembles in a few minutes on one core, run live: 16^3 base
    hexahedra, 10 % of them (seeded) refined by REFT_HEX_XYZ (6966 active
    elements), orders p_d ~ U{1..6} per element and direction (seeded), p_d + 2
    Gauss points, grad.grad, f = 1, homogeneous Dirichlet.  DOF count and
    pattern bit for bit, Ax and rhs within 1e-12 of the largest entry."""
    from oracle import ref_driver
    if not ref_driver.available():
        pytest.skip("reference oracle binary not built")
    n = 16
    nb = n ** 3
    refs = np.sort(np.random.default_rng(2000).choice(nb, int(round(0.1 * nb)), replace=False) + 1)
    orders = np.random.default_rng(1000).integers(1, 7, size=(nb + 8 * len(refs), 3)).astype(np.int32)
    r = ref_driver.run(h.unit_cube(n), orders=orders, qmode="pplus:2", source="one", bc="dirichlet0",
                       refine=[(int(e), 7) for e in refs], timeout=3000)
    mesh = h.unit_cube(n)
    mesh.ugh()
    mesh.refine_elements(refs)
    sp = h.H1Space(mesh)
    sp.set_element_orders(orders)
    sp.assign_dofs()
    assert sp.ndof == r["ndof"]
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v)
    d.set_linear_form(h.int_F_v(1.0))
    d.set_quadrature(p_plus=2)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    assert np.array_equal(M.Ap, r["Ap"]) and np.array_equal(M.Ai, r["Ai"])
    d.assemble(M, V)
    e_ax, e_rhs = rel_err(M.Ax, r["Ax"]), rel_err(V.v, r["rhs"])
    print("C3 sample (16^3, 10%% refined) vs reference: Ax %.2e rhs %.2e" % (e_ax, e_rhs))
    assert e_ax < FP64_RTOL and e_rhs < FP64_RTOL
