"""Host DOF map of the product (C++ behind the C ABI) against the reference:
assembly lists and the CSC pattern must be bit-exact."""
import numpy as np
import pytest

import hermes3d_b200 as h
from helpers import disc_of, golden_names, highorder_names, highorder_problem, load, load_highorder, space_of


@pytest.mark.parametrize("name", golden_names())
def test_dof_count_and_assembly_lists(name):
    g = load(name)
    sp = space_of(g)
    assert sp.get_dof_count() == int(g["ndof"])
    ne = len(g["hexes"])
    for e in range(1, ne + 1):
        a, b = g["al_ptr"][e - 1], g["al_ptr"][e]
        idx, dof, coef = sp.get_element_assembly_list(e)
        assert np.array_equal(idx, g["al_idx"][a:b]), e
        assert np.array_equal(dof, g["al_dof"][a:b]), e
        assert np.allclose(coef, g["al_coef"][a:b], rtol=1e-12, atol=1e-12), e


@pytest.mark.parametrize("name", golden_names())
def test_pattern_bit_exact(name):
    g = load(name)
    sp = space_of(g)
    d = disc_of(g, sp)
    M = h.UMFPackMatrix()
    d.create(M, h.UMFPackVector())
    assert np.array_equal(M.Ap, g["Ap"])
    assert np.array_equal(M.Ai, g["Ai"])


@pytest.mark.parametrize("name", ["c1_small", "perm_p2_lifting", "perm_p4_natural"])
def test_mixed_plan_pattern_bit_exact(name, monkeypatch):
    """Uniform spaces routed through the mixed-order plan give the same pattern."""
    monkeypatch.setenv("H3DG_FORCE_MIXED", "1")
    g = load(name)
    sp = space_of(g)
    d = disc_of(g, sp)
    M = h.UMFPackMatrix()
    d.create(M, h.UMFPackVector())
    assert np.array_equal(M.Ap, g["Ap"])
    assert np.array_equal(M.Ai, g["Ai"])


def test_structured_counts_match_closed_form():
    # C1 sizes: 8^3 elements, p=3, homogeneous Dirichlet
    m = h.unit_cube(8)
    m.ugh()
    sp = h.H1Space(m)
    sp.set_uniform_order(3)
    assert sp.assign_dofs() == (3 * 8 - 1) ** 3
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v)
    d.set_quadrature(points=5)
    M = h.UMFPackMatrix()
    d.create(M)
    assert d.nnz == 1225043


def test_relabelling_changes_numbering_not_dof_count():
    base = h.unit_cube(3, 0.1, 4)
    counts = []
    for seed in range(3):
        m = h.permute_vertices(base, seed=seed)
        m.ugh()
        sp = h.H1Space(m)
        sp.set_uniform_order(4)
        counts.append(sp.assign_dofs())
    assert len(set(counts)) == 1


@pytest.mark.parametrize("name", highorder_names())
def test_high_order_dof_map_and_pattern_bit_exact(name):
    """Orders 5..8 with natural and Dirichlet faces mixed: assembly lists
    (indices, DOFs, lifting coefficients) and the CSC pattern."""
    g = load_highorder(name)
    mesh, sp, d = highorder_problem(g)
    assert sp.get_dof_count() == int(g["ndof"])
    for e in range(1, len(g["hexes"]) + 1):
        a, b = g["al_ptr"][e - 1], g["al_ptr"][e]
        idx, dof, coef = sp.get_element_assembly_list(e)
        assert np.array_equal(idx, g["al_idx"][a:b]), e
        assert np.array_equal(dof, g["al_dof"][a:b]), e
        assert np.allclose(coef, g["al_coef"][a:b], rtol=1e-12, atol=1e-12), e
    M = h.UMFPackMatrix()
    d.create(M, h.UMFPackVector())
    assert np.array_equal(M.Ap, g["Ap"]) and np.array_equal(M.Ai, g["Ai"])
