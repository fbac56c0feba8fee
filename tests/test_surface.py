"""Surface forms, host side: the fixtures differ from the volume-only
assembly (so the GPU test checks the surface terms), the device form objects
and their argument checks."""
import numpy as np
import pytest

import hermes3d_b200 as h
from helpers import load_surface, surface_names
from oracle import ref_driver


@pytest.mark.skipif(not ref_driver.available(), reason="reference driver not built")
def test_surface_terms_are_present_in_the_fixtures():
    g = load_surface("surf_newton_p2")
    p = g["params"]
    mesh = h.Mesh().set_arrays(g["xyz"], g["hexes"], g["bquads"], g["bmarkers"])
    r = ref_driver.run(mesh, p=p["p"], qmode="pplus:2", bc="natural", mass=True, source="one")
    assert np.array_equal(r["Ap"], g["Ap"])
    assert np.abs(r["Ax"] - g["Ax"]).max() > 1e-3 * np.abs(g["Ax"]).max()
    assert np.abs(r["rhs"] - g["rhs"]).max() > 1e-3 * np.abs(g["rhs"]).max()


def test_surface_form_objects():
    f = h.surf_int_G_v({1: 2.0, 6: -1.0})
    assert f.g[1] == 2.0 and f.g[6] == -1.0 and f.g[0] == 0.0 and len(f.g) == 16
    assert h.surf_int_G_v(3.0).g == (3.0,) * 16
    with pytest.raises(h.H3dgError):
        h.surf_int_G_v({16: 1.0})
    d = h.Discretization()
    with pytest.raises(h.UnsupportedForm):
        d.set_bilinear_form(h.int_grad_u_grad_v, surf="surf_int_u_v")
    with pytest.raises(h.UnsupportedForm):
        d.set_linear_form(h.int_F_v(1.0), surf=h.surf_int_u_v)


def test_surface_forms_on_refined_mesh_are_rejected():
    mesh = h.unit_cube(2)
    mesh.refine_element(1)
    sp = h.H1Space(mesh)
    sp.set_bc_types(lambda m: h.BC_NATURAL)
    sp.set_uniform_order(2)
    sp.assign_dofs()
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v, surf=h.surf_int_u_v)
    d.set_linear_form(h.int_F_v(1.0))
    with pytest.raises(h.H3dgError):
        d.create(h.UMFPackMatrix(), h.UMFPackVector())


def test_surface_fixture_list():
    assert len(surface_names()) >= 5
