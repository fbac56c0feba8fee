"""Refined meshes (Mesh::refine_element, REFT_HEX_XYZ) and hanging nodes
(constrained vertex / edge / face functions), host side, against fixtures
the reference itself produced (tests/golden/make_refined_golden.py):
DOF numbering and every element's DOF set exactly, the CSC pattern bit for
bit, and the values the restatement oracle assembles from the expanded
assembly lists within the FP64 tolerance."""
import numpy as np
import pytest

import hermes3d_b200 as h
from helpers import FP64_RTOL, lf_of, load_refined, refined_names, refined_space_of, rel_err
from oracle import port


def _active_lists(mesh, sp):
    act = np.nonzero(mesh.active)[0] + 1
    ptr, idx, dof, coef = [0], [], [], []
    for e in act:
        i, d, c = sp.get_element_assembly_list(int(e))
        idx.append(i)
        dof.append(d)
        coef.append(c)
        ptr.append(ptr[-1] + len(i))
    return act, (np.array(ptr, np.int64), np.concatenate(idx).astype(np.int64), np.concatenate(dof).astype(np.int32),
                 np.concatenate(coef).astype(np.float64))


@pytest.mark.parametrize("name", refined_names())
def test_refined_dof_numbering_matches_reference(name):
    g = load_refined(name)
    mesh, sp = refined_space_of(g)
    assert sp.ndof == int(g["ndof"])
    act = np.nonzero(mesh.active)[0] + 1
    assert np.array_equal(act, g["act_ids"])
    for k, e in enumerate(act):
        _, d, _ = sp.get_element_assembly_list(int(e))
        ref = g["al_dof"][g["al_ptr"][k]:g["al_ptr"][k + 1]]
        assert sorted(set(d[d >= 0].tolist())) == sorted(set(ref[ref >= 0].tolist())), "element %d" % e


@pytest.mark.parametrize("name", refined_names())
def test_refined_pattern_and_values_match_reference(name):
    g = load_refined(name)
    mesh, sp = refined_space_of(g)
    act, al = _active_lists(mesh, sp)
    Ap, Ai = port.pattern(al[0], al[2], sp.ndof)
    assert np.array_equal(Ap, g["Ap"]) and np.array_equal(Ai, g["Ai"])
    lf, lv = lf_of(g)
    gc = g["gradcoef"][act - 1] if len(g["gradcoef"]) else None
    Ax, rhs = port.assemble(mesh.xyz, mesh.hexes[act - 1] - 1, g["orders"][act - 1] + 2, al, sp.ndof, Ap, Ai,
                            mass=g["params"].get("mass", False), gradcoef=gc, lf=lf, lf_value=lv)
    assert rel_err(Ax, g["Ax"]) < FP64_RTOL
    assert rel_err(rhs, g["rhs"]) < FP64_RTOL


def test_refine_element_structure():
    m = h.unit_cube(2)
    m.refine_element(1)
    assert len(m.hexes) == 16 and len(m.xyz) == 27 + 19
    assert list(m.parent[8:]) == [1] * 8 and not m.active[0] and m.active[1:].all()
    x = m.xyz
    # child i holds the parent's corner i; the centre vertex is shared by all children
    for i in range(8):
        assert m.hexes[8 + i][i] == m.hexes[0][i]
    ctr = set.intersection(*[set(m.hexes[8 + i]) for i in range(8)])
    assert len(ctr) == 1 and np.allclose(x[ctr.pop() - 1], [0.25, 0.25, 0.25])
    # an edge midpoint is the average of its end points
    a, b = m.hexes[0][0] - 1, m.hexes[0][1] - 1
    assert np.array_equal(x[m.hexes[8][1] - 1], (x[a] + x[b]) / 2.0)
    # a neighbour refined later reuses the shared midpoints
    nv = len(m.xyz)
    m.refine_element(2)
    assert len(m.xyz) == nv + 19 - 5      # the shared face: 4 edge midpoints and its centre


def test_refine_element_errors():
    m = h.unit_cube(2)
    m.refine_element(1)
    with pytest.raises(h.H3dgError):
        m.refine_element(1)          # not active any more
    with pytest.raises(h.H3dgError):
        m.refine_element(9)          # a child: one refinement level
    with pytest.raises(h.H3dgError):
        m.refine_element(2, 1)       # REFT_HEX_X is not supported


def test_partition_of_refined_mesh_is_planned():
    """A refined mesh cut into two z-slab parts: each DOF owned once, the
    refined parent in neither part (its children are)."""
    m = h.unit_cube(3)
    m.refine_element(14)
    sp = h.H1Space(m)
    sp.set_uniform_order(2)
    sp.assign_dofs()
    owner = np.zeros(sp.ndof, np.int32)
    for part in range(2):
        d = h.Discretization()
        d.set_spaces(sp)
        d.set_bilinear_form(h.int_grad_u_grad_v)
        d.set_linear_form(h.int_F_v(1.0))
        d.set_partition(2, part)
        d.create(h.UMFPackMatrix(), h.UMFPackVector())
        info = d.partition()
        owner += info["owned"]
        assert not info["elements"][13]          # element 14, refined
    assert np.all(owner == 1)
