"""Two-equation systems (Discretization with neq = 2, identical spaces numbered
one after another, as the reference's calc/hex-h1-sys* tests): the block
pattern against fixtures the reference itself produced, and the checks on
the spaces."""
import numpy as np
import pytest

import hermes3d_b200 as h
from helpers import load_system, system_names, system_problem


@pytest.mark.parametrize("name", system_names())
def test_system_pattern_matches_reference(name):
    g = load_system(name)
    mesh, spaces, d = system_problem(g)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    assert d.ndof == int(g["ndof"])
    assert np.array_equal(M.Ap, g["Ap"]) and np.array_equal(M.Ai, g["Ai"])


def test_system_checks_its_spaces():
    mesh = h.unit_cube(2)
    mesh.ugh()
    a, b = h.H1Space(mesh), h.H1Space(mesh)
    a.set_uniform_order(2)
    b.set_uniform_order(2)
    a.assign_dofs()
    b.assign_dofs()                         # not numbered after the first space
    d = h.SystemDiscretization()
    d.set_num_equations(2)
    with pytest.raises(h.H3dgError):
        d.set_spaces(a, b)
