"""Shared test helpers: golden fixtures and building the product objects
from a fixture's parameters."""
import ast
import glob
import os

import numpy as np

import hermes3d_b200 as h

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# relative tolerance of FP64 values vs the reference (sum order and the
# reference's 14-digit Gauss tables differ at ~1e-14)
FP64_RTOL = 1e-12


def golden_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False)
    d = {k: z[k] for k in z.files}
    d["params"] = ast.literal_eval(str(d["params"]))
    return d


def mesh_of(g):
    return h.Mesh().set_arrays(g["xyz"], g["hexes"], g["bquads"], g["bmarkers"])


def space_of(g, mesh=None):
    p = g["params"]
    mesh = mesh or mesh_of(g)
    mesh.ugh()
    sp = h.H1Space(mesh)
    bc = p.get("bc", "dirichlet0")
    if bc == "natural":
        sp.set_bc_types(lambda m: h.BC_NATURAL)
    if bc == "dirichlet_poly":
        sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    if len(g["orders"]):
        sp.set_element_orders(g["orders"])
    else:
        sp.set_uniform_order(p["p"])
    sp.assign_dofs()
    return sp


def quad_of(g):
    q = g["params"]["qmode"]
    kind, n = q.split(":")
    return kind, int(n)


def disc_of(g, sp, device=0):
    p = g["params"]
    d = h.Discretization(device)
    d.set_spaces(sp)
    form = h.int_grad_u_grad_v_plus_u_v if p.get("mass") else h.int_grad_u_grad_v
    d.set_bilinear_form(form, g["gradcoef"] if len(g["gradcoef"]) else None)
    src = p.get("source", "one")
    if src == "one":
        d.set_linear_form(h.int_F_v(1.0))
    elif src == "sin":
        d.set_linear_form(h.int_F_v("sin"))
    elif src == "poly":
        d.set_linear_form(h.int_F_v(-6.0))
    if p["qmode"] == "ref":                         # the reference's stock per-pair rule
        d.set_quadrature(stock=True)
        return d
    kind, n = quad_of(g)
    if kind == "fixed":
        d.set_quadrature(points=n)
    else:
        d.set_quadrature(p_plus=n)
    return d


def lf_of(g):
    src = g["params"].get("source", "one")
    return {"one": (1, 1.0), "sin": (2, 0.0), "poly": (1, -6.0), "none": (0, 0.0)}[src]


def nq_of(g):
    kind, n = quad_of(g)
    ne = len(g["hexes"])
    if kind == "fixed":
        return np.full((ne, 3), n, np.int32)
    o = g["orders"] if len(g["orders"]) else np.full((ne, 3), g["params"]["p"], np.int32)
    return (np.asarray(o) + n).astype(np.int32)


def rel_err(a, b):
    s = max(float(np.max(np.abs(b))) if len(b) else 0.0, 1e-300)
    return float(np.max(np.abs(a - b))) / s if len(a) else 0.0


REFINED = os.path.join(GOLDEN, "refined")


def refined_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(REFINED, "*.npz")))


def load_refined(name):
    z = np.load(os.path.join(REFINED, name + ".npz"), allow_pickle=False)
    d = {k: z[k] for k in z.files}
    d["params"] = ast.literal_eval(str(d["params"]))
    return d


def refined_space_of(g):
    """Base mesh of a refined fixture, its refinements (REFT_HEX_XYZ) and the space."""
    p = g["params"]
    mesh = mesh_of(g)
    mesh.ugh()
    for e in g["refine"]:
        mesh.refine_element(int(e))
    sp = h.H1Space(mesh)
    bc = p.get("bc", "dirichlet0")
    if bc == "natural":
        sp.set_bc_types(lambda m: h.BC_NATURAL)
    if bc == "dirichlet_poly":
        sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    sp.set_element_orders(g["orders"])
    sp.assign_dofs()
    return mesh, sp


SURFACE = os.path.join(GOLDEN, "surface")


def surface_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(SURFACE, "*.npz")))


def load_surface(name):
    z = np.load(os.path.join(SURFACE, name + ".npz"), allow_pickle=False)
    d = {k: z[k] for k in z.files}
    d["params"] = ast.literal_eval(str(d["params"]))
    return d


def surface_problem(g, device=0):
    """Space and discretization of a surface-form fixture: BC types per marker,
    surf_int_u_v and / or surf_int_G_v with the fixture's g per marker 1..6."""
    p = g["params"]
    mesh = mesh_of(g)
    mesh.ugh()
    sp = h.H1Space(mesh)
    nat = set(p.get("natural_markers") or [])
    all_nat = p.get("bc") == "natural"
    sp.set_bc_types(lambda m: h.BC_NATURAL if (all_nat or m in nat) else h.BC_ESSENTIAL)
    if p.get("bc") == "dirichlet_poly":
        sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    if len(g["orders"]):
        sp.set_element_orders(g["orders"])
    else:
        sp.set_uniform_order(p["p"])
    sp.assign_dofs()
    d = h.Discretization(device)
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v_plus_u_v if p.get("mass") else h.int_grad_u_grad_v,
                        surf=h.surf_int_u_v if p.get("surf_uv") else None)
    src = p.get("source", "one")
    lf = {"one": h.int_F_v(1.0), "sin": h.int_F_v("sin"), "poly": h.int_F_v(-6.0)}[src]
    sg = p.get("surf_g")
    d.set_linear_form(lf, surf=h.surf_int_G_v([0.0] + list(sg)) if sg is not None else None)
    kind, n = quad_of(g)
    d.set_quadrature(p_plus=n) if kind == "pplus" else d.set_quadrature(points=n)
    return mesh, sp, d


SYSTEM = os.path.join(GOLDEN, "system")


def system_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(SYSTEM, "*.npz")))


def load_system(name):
    z = np.load(os.path.join(SYSTEM, name + ".npz"), allow_pickle=False)
    d = {k: z[k] for k in z.files}
    d["params"] = ast.literal_eval(str(d["params"]))
    return d


def system_problem(g, device=0):
    """Two spaces (identical, or the second of uniform order p2) and the
    block forms / sources / rule of a system fixture."""
    p = g["params"]
    mesh = mesh_of(g)
    mesh.ugh()
    spaces = []
    nd = 0
    for i in range(2):
        sp = h.H1Space(mesh)
        if p.get("bc") == "natural":
            sp.set_bc_types(lambda m: h.BC_NATURAL)
        if p.get("bc") == "dirichlet_poly":
            sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
        sp.set_uniform_order(p.get("p2") or p["p"] if i == 1 else p["p"])
        nd += sp.assign_dofs(nd)
        spaces.append(sp)
    d = h.SystemDiscretization(device)
    d.set_num_equations(2)
    d.set_spaces(*spaces)
    kinds = {"gg": h.int_grad_u_grad_v, "ggm": h.int_grad_u_grad_v_plus_u_v, "mass": h.int_u_v}
    for b, k in enumerate(p["sys"]):
        if k != "none":
            d.set_bilinear_form(b // 2, b % 2, kinds[k])
    src = {"one": h.int_F_v(1.0), "sin": h.int_F_v("sin"), "poly": h.int_F_v(-6.0), "none": None}
    d.set_linear_form(0, src[p.get("source", "one")])
    d.set_linear_form(1, src[p.get("source2", "none")])
    kind, n = p.get("qmode", "pplus:2").split(":")
    if kind == "fixed":
        d.set_quadrature(points=int(n))
    else:
        d.set_quadrature(p_plus=int(n))
    return mesh, spaces, d


HIGHORDER = os.path.join(GOLDEN, "highorder")


def highorder_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(HIGHORDER, "*.npz")))


def load_highorder(name):
    z = np.load(os.path.join(HIGHORDER, name + ".npz"), allow_pickle=False)
    d = {k: z[k] for k in z.files}
    d["params"] = ast.literal_eval(str(d["params"]))
    return d


def highorder_problem(g, device=0):
    """Space (BC type per marker, Dirichlet x^2+y^2+z^2) and discretization
    (a_e grad.grad [+ mass], source) of a high-order fixture."""
    p = g["params"]
    mesh = mesh_of(g)
    mesh.ugh()
    sp = h.H1Space(mesh)
    nat = set(p.get("natural_markers") or [])
    all_nat = p.get("bc") == "natural"
    sp.set_bc_types(lambda m: h.BC_NATURAL if (all_nat or m in nat) else h.BC_ESSENTIAL)
    if p.get("bc") == "dirichlet_poly":
        sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    sp.set_uniform_order(p["p"])
    sp.assign_dofs()
    d = h.Discretization(device)
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v_plus_u_v if p.get("mass") else h.int_grad_u_grad_v, g["gradcoef"])
    src = p.get("source", "one")
    d.set_linear_form({"one": h.int_F_v(1.0), "sin": h.int_F_v("sin"), "poly": h.int_F_v(-6.0)}[src])
    kind, n = quad_of(g)
    d.set_quadrature(p_plus=n) if kind == "pplus" else d.set_quadrature(points=n)
    return mesh, sp, d


def stock_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "stock", "*.npz")))


def load_stock(name):
    z = np.load(os.path.join(GOLDEN, "stock", name + ".npz"), allow_pickle=False)
    d = {k: z[k] for k in z.files}
    d["params"] = ast.literal_eval(str(d["params"]))
    return d

