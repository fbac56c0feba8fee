"""C ABI: every symbol declared in include/h3dg.h is exported, error paths
return status codes (never abort), and the assembly path refuses to run
without a device instead of falling back to the CPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import hermes3d_b200 as h
from hermes3d_b200 import _capi as capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    out = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            out += re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(h3dg_[a-z_0-9]+)\s*\(", src, re.M)
    return sorted(set(out))


def test_library_exports_every_declared_symbol():
    L = C.CDLL(capi.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 30
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) <= set(capi.SIGNATURES), set(syms) - set(capi.SIGNATURES)


def test_status_strings():
    L = capi.lib()
    for s in range(9):
        assert L.h3dg_status_string(s)
    assert L.h3dg_version() >= 1


def _mesh_with(hexes, bq, bm, xyz=None):
    if xyz is None:
        xyz = h.unit_cube(1).xyz
    return h.Mesh().set_arrays(xyz, hexes, bq, bm)


def test_invalid_vertex_index_is_an_error():
    m = h.unit_cube(1)
    hexes = m.hexes.copy()
    hexes[0, 3] = 99
    with pytest.raises(capi.H3dgError, match="Invalid vertex index"):
        _mesh_with(hexes, m.bquads, m.bmarkers).ugh()


def test_missing_boundary_is_an_error():
    m = h.unit_cube(2)
    with pytest.raises(capi.H3dgError, match="outer faces"):
        _mesh_with(m.hexes, m.bquads[:-1], m.bmarkers[:-1], m.xyz).ugh()


def test_order_out_of_range():
    m = h.unit_cube(1)
    m.ugh()
    sp = h.H1Space(m)
    with pytest.raises(capi.H3dgError):
        sp.set_uniform_order(11)
    with pytest.raises(capi.H3dgError):
        sp.set_element_orders(np.array([[0, 1, 1]]))


def test_calls_out_of_order():
    m = h.unit_cube(1)
    m.ugh()
    sp = h.H1Space(m)
    with pytest.raises(capi.H3dgError, match="assign_dofs"):
        sp.get_element_assembly_list(1)
    d = h.Discretization()
    with pytest.raises(capi.H3dgError):
        d.create(h.UMFPackMatrix())
    with pytest.raises(capi.H3dgError):
        d.assemble(h.UMFPackMatrix())


def test_unsupported_forms_are_rejected():
    d = h.Discretization()
    with pytest.raises(h.UnsupportedForm):
        d.set_bilinear_form(lambda fu, fv, ru, rv: 0.0)
    with pytest.raises(h.UnsupportedForm):
        d.set_linear_form(lambda fv, rv: 0.0)
    with pytest.raises(capi.H3dgError):
        capi.call("h3dg_disc_set_bilinear_form", d.handle, 77, None, 0)


@pytest.mark.skipif(__import__("conftest").has_gpu(), reason="checks the no-device path")
def test_assembly_without_device_fails_loudly():
    m = h.unit_cube(2)
    m.ugh()
    sp = h.H1Space(m)
    sp.set_uniform_order(2)
    sp.assign_dofs()
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v)
    d.set_linear_form(h.int_F_v(1.0))
    d.set_quadrature(points=4)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    with pytest.raises(capi.H3dgError) as ei:
        d.assemble(M, V)
    assert ei.value.status == 2


def test_non_finite_dirichlet_values_are_an_error():
    """A boundary projection that cannot be solved (here: Dirichlet values
    that are not finite) fails assign_dofs, as choldc's exit does in the
    reference, instead of leaving NaN lifting coefficients."""
    mesh = h.unit_cube(2)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_bc_values(lambda m, x, y, z: float("nan") if m == 3 else 1.0)
    sp.set_uniform_order(3)
    with pytest.raises(capi.H3dgError) as e:
        sp.assign_dofs()
    assert e.value.status == capi.H3DG_ERR_STATE
    assert "not finite" in str(e.value)
