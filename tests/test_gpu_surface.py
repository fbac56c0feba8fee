"""Surface forms on natural boundary faces on the GPU (surf_int_u_v,
surf_int_G_v with g per marker; Newton, Neumann and mixed boundaries with
Dirichlet lifting through the surface form) against fixtures the reference
itself produced (tests/golden/make_surface_golden.py); FP64 tolerance 1e-12."""
import numpy as np
import pytest

import hermes3d_b200 as h
from helpers import FP64_RTOL, load_surface, rel_err, surface_names, surface_problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", surface_names())
def test_surface_forms_match_reference(gpu, name):
    g = load_surface(name)
    mesh, sp, d = surface_problem(g)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)
    assert sp.ndof == int(g["ndof"])
    assert np.array_equal(M.Ap, g["Ap"]) and np.array_equal(M.Ai, g["Ai"])
    assert rel_err(M.Ax, g["Ax"]) < FP64_RTOL
    assert rel_err(V.v, g["rhs"]) < FP64_RTOL


@pytest.mark.parametrize("force", ["H3DG_FORCE_MIXED", "H3DG_FORCE_HIGH_ORDER"])
def test_surface_forms_with_other_volume_kernels(gpu, monkeypatch, force):
    monkeypatch.setenv(force, "1")
    g = load_surface("surf_newton_p2")
    mesh, sp, d = surface_problem(g)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)
    assert rel_err(M.Ax, g["Ax"]) < FP64_RTOL
    assert rel_err(V.v, g["rhs"]) < FP64_RTOL
