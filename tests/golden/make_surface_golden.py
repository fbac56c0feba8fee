"""Generate the surface-form fixtures under tests/golden/surface/ by running
the Hermes3D reference itself (built from its sources by oracle/Makefile; needs
the reference tree, so this runs only where it is present).

    make -C oracle REF=/path/to/hermes3d && python tests/golden/make_surface_golden.py

Natural boundary faces with surf_int_u_v and / or surf_int_G_v (g constant per
boundary marker 1..6), integrated with the element's rule on the face, through
the reference's Discretization::assemble.  Each fixture holds the mesh, the
parameters and the reference's ndof, pattern, Ax and rhs.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from hermes3d_b200.mesh import permute_vertices, unit_cube  # noqa: E402
from oracle import ref_driver  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "surface")
G = [0.5, -1.0, 2.0, 0.25, 1.5, -0.75]

# name: (mesh builder, run kwargs)
CASES = {
    "surf_newton_p2": (lambda: unit_cube(3, 0.2, 1),
                       dict(p=2, bc="natural", mass=True, source="one", surf_uv=True, surf_g=G)),
    "surf_perm_newton_p3": (lambda: permute_vertices(unit_cube(3, 0.2, 4), seed=6),
                            dict(p=3, bc="natural", source="sin", surf_uv=True, surf_g=G)),
    "surf_mixed_lifting_p3": (lambda: unit_cube(3, 0.1, 2),
                              dict(p=3, bc="dirichlet_poly", natural_markers=[1, 3, 6], source="poly", surf_uv=True,
                                   surf_g=G)),
    "surf_uv_only_lifting_p2": (lambda: permute_vertices(unit_cube(3, 0.1, 3), seed=2),
                                dict(p=2, bc="dirichlet_poly", natural_markers=[2, 5], source="poly", surf_uv=True)),
    "surf_neumann_aniso": (lambda: unit_cube(3, 0.2, 5),
                           dict(orders=np.random.default_rng(4).integers(1, 7, size=(27, 3)).astype(np.int32),
                                bc="dirichlet0", natural_markers=[2, 4, 6], source="one", surf_g=G)),
}


def main():
    if not ref_driver.available():
        ref_driver.build()
    os.makedirs(OUT, exist_ok=True)
    for name, (mk, kw) in CASES.items():
        mesh = mk()
        kw = dict(kw)
        orders = kw.pop("orders", None)
        r = ref_driver.run(mesh, orders=orders, qmode="pplus:2", **kw)
        params = {k: v for k, v in kw.items()}
        params["qmode"] = "pplus:2"
        np.savez_compressed(
            os.path.join(OUT, name + ".npz"), xyz=mesh.xyz, hexes=mesh.hexes, bquads=mesh.bquads,
            bmarkers=mesh.bmarkers, params=np.array(repr(params)),
            orders=orders if orders is not None else np.zeros((0, 3), np.int32), gradcoef=np.zeros(0),
            ndof=r["ndof"], Ap=r["Ap"], Ai=r["Ai"], Ax=r["Ax"], rhs=r["rhs"])
        print(name, "ndof", r["ndof"], "nnz", r["nnz"])


if __name__ == "__main__":
    main()
