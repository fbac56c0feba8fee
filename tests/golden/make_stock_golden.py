"""Fixtures for the reference's stock quadrature (the per-pair rule of
int_grad_u_grad_v / int_u_v and the order-24 rule of int_F_v,
src/integrals/h1.h:115-177), made by running the Hermes3D reference itself
(oracle/_ref, `--qmode ref`) on jittered, vertex-relabelled meshes where the
rule matters (non-affine maps).  Needs the reference build:

    make -C oracle && python tests/golden/make_stock_golden.py

Writes tests/golden/stock/<name>.npz in the layout of make_golden.py.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

from hermes3d_b200.mesh import permute_vertices, unit_cube  # noqa: E402
from make_golden import flatten_asm  # noqa: E402
from oracle import ref_driver  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "stock")

CASES = {
    "stock_p2_mass_sin": (lambda: permute_vertices(unit_cube(3, 0.2, 5), seed=5),
                          dict(p=2, qmode="ref", mass=True, source="sin", bc="dirichlet0")),
    "stock_p3_lifting_coef": (lambda: permute_vertices(unit_cube(2, 0.15, 2), seed=6),
                              dict(p=3, qmode="ref", source="poly", bc="dirichlet_poly",
                                   gradcoef=np.random.default_rng(4).uniform(0.5, 2.0, 8))),
    "stock_p1_natural": (lambda: permute_vertices(unit_cube(3, 0.2, 7), seed=7),
                         dict(p=1, qmode="ref", source="one", bc="natural")),
    "stock_p2_lifting_mass": (lambda: permute_vertices(unit_cube(2, 0.2, 9), seed=9),
                              dict(p=2, qmode="ref", mass=True, source="one", bc="dirichlet_poly")),
}


def main():
    if not ref_driver.available():
        ref_driver.build()
    os.makedirs(OUT, exist_ok=True)
    for name, (mk, kw) in CASES.items():
        mesh = mk()
        r = ref_driver.run(mesh, **kw)
        ptr, idx, dof, coef = flatten_asm(r["asm"], len(mesh.hexes))
        params = {k: v for k, v in kw.items() if k not in ("orders", "gradcoef")}
        np.savez_compressed(
            os.path.join(OUT, name + ".npz"), xyz=mesh.xyz, hexes=mesh.hexes, bquads=mesh.bquads, bmarkers=mesh.bmarkers,
            params=np.array(repr(params)), orders=kw.get("orders", np.zeros((0, 3), np.int32)),
            gradcoef=kw.get("gradcoef", np.zeros(0)), ndof=r["ndof"], Ap=r["Ap"], Ai=r["Ai"], Ax=r["Ax"], rhs=r["rhs"],
            al_ptr=ptr, al_idx=idx, al_dof=dof, al_coef=coef)
        print(name, "ndof", r["ndof"], "nnz", r["nnz"])


if __name__ == "__main__":
    main()
