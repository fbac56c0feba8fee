"""Parity of the sm_100a kernels against the reference (golden fixtures made
by the reference itself) and against the C restatement oracle, through the
C ABI."""
import numpy as np
import pytest

import hermes3d_b200 as h
from helpers import FP64_RTOL, disc_of, golden_names, lf_of, load, nq_of, rel_err, space_of
from oracle import port, ref_driver

pytestmark = pytest.mark.gpu

UNIFORM = [n for n in golden_names() if not n.startswith("aniso")]


@pytest.mark.parametrize("name", UNIFORM)
def test_assemble_matches_reference(gpu, name):
    g = load(name)
    sp = space_of(g)
    d = disc_of(g, sp)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)
    assert d.last_launch_count() >= 1
    assert rel_err(M.Ax, g["Ax"]) < FP64_RTOL
    assert rel_err(V.v, g["rhs"]) < FP64_RTOL


@pytest.mark.parametrize("name", ["jitter_p3_mass_sin", "perm_p2_lifting"])
def test_device_api_and_determinism(gpu, name):
    import torch
    g = load(name)
    sp = space_of(g)
    d = disc_of(g, sp)
    d.create()
    outs = []
    for _ in range(3):
        Ax = torch.full((d.nnz,), float("nan"), dtype=torch.float64, device="cuda")
        rhs = torch.full((d.ndof,), float("nan"), dtype=torch.float64, device="cuda")
        d.assemble_device(Ax, rhs)
        torch.cuda.synchronize()
        outs.append((Ax.cpu().numpy(), rhs.cpu().numpy()))
    for a, b in outs[1:]:
        assert np.array_equal(a, outs[0][0]) and np.array_equal(b, outs[0][1])   # bitwise reproducible
    assert rel_err(outs[0][0], g["Ax"]) < FP64_RTOL
    assert rel_err(outs[0][1], g["rhs"]) < FP64_RTOL


def test_geometry_kernel_matches_refmap(gpu):
    import torch
    g = load("perm_p3_mass_sin")
    sp = space_of(g)
    d = disc_of(g, sp)
    d.create()
    ne, nq = len(g["hexes"]), 5 ** 3
    jac = torch.zeros(ne * nq, dtype=torch.float64, device="cuda")
    irm = torch.zeros(ne * nq * 9, dtype=torch.float64, device="cuda")
    xyz = torch.zeros(ne * nq * 3, dtype=torch.float64, device="cuda")
    d.geometry(jac, irm, xyz)
    torch.cuda.synchronize()
    jac, irm, xyz = jac.cpu().numpy(), irm.cpu().numpy().reshape(ne, nq, 3, 3), xyz.cpu().numpy().reshape(ne, nq, 3)
    # reference: phys points are the trilinear map; the Jacobian volume integral equals the mesh volume
    w = np.polynomial.legendre.leggauss(5)[1]
    W = np.einsum("i,j,k->ijk", w, w, w).ravel()
    assert abs(float((jac.reshape(ne, nq) * W).sum()) - 1.0) < 1e-12
    X = g["xyz"][g["hexes"][0] - 1]
    pts = np.polynomial.legendre.leggauss(5)[0]
    x0 = pts[0]
    l0 = (1 - x0) / 2
    l1 = (1 + x0) / 2
    # first point of element 1 = (x0, x0, x0): weights of the 8 vertices
    wv = np.array([l0 * l0 * l0, l1 * l0 * l0, l1 * l1 * l0, l0 * l1 * l0, l0 * l0 * l1, l1 * l0 * l1, l1 * l1 * l1, l0 * l1 * l1])
    assert np.allclose(xyz[0, 0], wv @ X, rtol=0, atol=1e-14)
    # irm is the transposed inverse of the Jacobian: irm^T J = I with J from finite differences of the map
    assert np.all(np.isfinite(irm)) and np.all(jac > 0)


@pytest.mark.parametrize("n,p,nq,jit,mass,src", [(5, 2, 4, 0.2, True, "sin"), (4, 3, 5, 0.15, False, "one"),
                                                  (3, 1, 2, 0.1, True, "one")])
def test_matches_restatement_oracle(gpu, n, p, nq, jit, mass, src):
    mesh = h.permute_vertices(h.unit_cube(n, jit, 7), seed=n)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_uniform_order(p)
    sp.assign_dofs()
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v_plus_u_v if mass else h.int_grad_u_grad_v)
    d.set_linear_form(h.int_F_v("sin" if src == "sin" else 1.0))
    d.set_quadrature(points=nq)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)
    al = port.asmlists_from_space(sp, mesh.num_elements)
    Ax, rhs = port.assemble(mesh.xyz, mesh.hexes - 1, nq, al, sp.ndof, M.Ap, M.Ai, mass=mass,
                            lf=2 if src == "sin" else 1, lf_value=1.0)
    assert rel_err(M.Ax, Ax) < FP64_RTOL
    assert rel_err(V.v, rhs) < FP64_RTOL


@pytest.mark.skipif(not ref_driver.available(), reason="reference oracle binary not built")
def test_c1_full_size_against_reference(gpu):
    # Plain FP64 Poisson on the unit cube: 8^3 hexahedra, p=3, 5 points, homogeneous Dirichlet, f=1
    mesh = h.unit_cube(8)
    r = ref_driver.run(mesh, p=3, qmode="fixed:5", source="one", bc="dirichlet0")
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
    d.assemble(M, V)
    assert np.array_equal(M.Ap, r["Ap"]) and np.array_equal(M.Ai, r["Ai"])
    assert rel_err(M.Ax, r["Ax"]) < FP64_RTOL
    assert rel_err(V.v, r["rhs"]) < FP64_RTOL


@pytest.mark.skipif(not ref_driver.available(), reason="reference oracle binary not built")
def test_c2_full_size_against_reference(gpu):
    """The headline workload at full size against the reference itself, run
    live on the host (about 3 minutes on one core): 64^3 jittered (+-0.2h,
    seed 0) hexahedra, p=2, 4^3 Gauss points, grad.grad + mass,
    f = sin(pi x) sin(pi y) sin(pi z).  DOF count and CSC pattern bit for bit,
    Ax and rhs within 1e-12 of the largest entry."""
    mesh = h.unit_cube(64, 0.2, 0)
    r = ref_driver.run(mesh, p=2, qmode="fixed:4", mass=True, source="sin", bc="dirichlet0", timeout=3000)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_uniform_order(2)
    sp.assign_dofs()
    assert sp.ndof == r["ndof"] == 2048383
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v_plus_u_v)
    d.set_linear_form(h.int_F_v("sin"))
    d.set_quadrature(points=4)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    assert np.array_equal(M.Ap, r["Ap"]) and np.array_equal(M.Ai, r["Ai"])
    del r["Ai"]
    d.assemble(M, V)
    e_ax, e_rhs = rel_err(M.Ax, r["Ax"]), rel_err(V.v, r["rhs"])
    print("C2 64^3 vs reference: Ax %.2e rhs %.2e" % (e_ax, e_rhs))
    assert e_ax < FP64_RTOL and e_rhs < FP64_RTOL


def test_c2_full_size_properties(gpu):
    """64^3 jittered, p=2, 4 points, grad+mass, sin source: the matrix is
    symmetric and positive definite on random vectors; assembled twice it is
    bitwise identical; the RHS integrates the source against the basis."""
    import scipy.sparse as sps
    mesh = h.unit_cube(64, 0.2, 0)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_uniform_order(2)
    sp.assign_dofs()
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v_plus_u_v)
    d.set_linear_form(h.int_F_v("sin"))
    d.set_quadrature(points=4)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    assert d.ndof == 2048383 and d.nnz == 127263527
    d.assemble(M, V)
    A = M.to_scipy()
    x = np.random.default_rng(0).standard_normal(d.ndof)
    y = np.random.default_rng(1).standard_normal(d.ndof)
    assert abs(x @ (A @ y) - y @ (A @ x)) < 1e-10 * abs(x @ (A @ y))
    assert x @ (A @ x) > 0
    Ax1 = M.Ax.copy()
    d.assemble(M, V)
    assert np.array_equal(Ax1, M.Ax)
    assert np.all(np.isfinite(V.v)) and V.v.max() > 0


@pytest.mark.parametrize("p,nq", [(1, 3), (2, 4), (3, 5)])
def test_every_kernel_variant_is_bitwise_identical(gpu, monkeypatch, p, nq):
    """The autotuner may pick any variant (CTA-per-element batches or one
    element per warp): all of them must give the same bits."""
    mesh = h.permute_vertices(h.unit_cube(4, 0.2, 9), seed=2)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    sp.set_uniform_order(p)
    sp.assign_dofs()
    ref = None
    for v in range(20):                       # indices past the last candidate pin the last one
        monkeypatch.setenv("H3DG_FP64_VARIANT", str(v))
        d = h.Discretization()
        d.set_spaces(sp)
        d.set_bilinear_form(h.int_grad_u_grad_v_plus_u_v, np.linspace(0.5, 2.0, mesh.num_elements))
        d.set_linear_form(h.int_F_v("sin"))
        d.set_quadrature(points=nq)
        M, V = h.UMFPackMatrix(), h.UMFPackVector()
        d.create(M, V)
        d.assemble(M, V)
        if ref is None:
            ref = (M.Ax.copy(), V.v.copy())
            al = port.asmlists_from_space(sp, mesh.num_elements)
            Ax, rhs = port.assemble(mesh.xyz, mesh.hexes - 1, nq, al, sp.ndof, M.Ap, M.Ai, mass=True,
                                    gradcoef=np.linspace(0.5, 2.0, mesh.num_elements), lf=2)
            assert rel_err(M.Ax, Ax) < FP64_RTOL and rel_err(V.v, rhs) < FP64_RTOL
        else:
            assert np.array_equal(M.Ax, ref[0]) and np.array_equal(V.v, ref[1]), v


@pytest.mark.parametrize("name", ["hex1", "hex2", "hex4", "hex8", "hex27"])
def test_geometry_kernel_matches_reference_refmap_dumps(gpu, name):
    """k_geometry against the reference's own RefMap known answers
    (tests/refmap/dump/*.dump via tests/golden/kat/refmap_dumps.npz): Jacobian
    determinant, transposed inverse map and physical points at the 2x2x2
    Gauss points, printed to 6 decimals by the reference."""
    import os
    import torch
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "kat", "refmap_dumps.npz"))
    mesh = h.Mesh().set_arrays(z[name + "_xyz"], z[name + "_hexes"], z[name + "_bquads"], z[name + "_bmarkers"])
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_bc_types(lambda m: h.BC_NATURAL)
    sp.set_uniform_order(1)
    sp.assign_dofs()
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v)
    d.set_quadrature(points=2)
    d.create()
    ne, nq = mesh.num_elements, 8
    jac = torch.zeros(ne * nq, dtype=torch.float64, device="cuda")
    irm = torch.zeros(ne * nq * 9, dtype=torch.float64, device="cuda")
    xyz = torch.zeros(ne * nq * 3, dtype=torch.float64, device="cuda")
    d.geometry(jac, irm, xyz)
    torch.cuda.synchronize()
    tol = 1.5e-6                                  # 6 printed decimals
    assert np.max(np.abs(jac.cpu().numpy().reshape(ne, nq) - z[name + "_jac"])) < tol
    assert np.max(np.abs(irm.cpu().numpy().reshape(ne, nq, 3, 3) - z[name + "_irm"])) < tol
    assert np.max(np.abs(xyz.cpu().numpy().reshape(ne, nq, 3) - z[name + "_phys"])) < tol
