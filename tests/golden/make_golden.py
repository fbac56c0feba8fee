"""Generate the golden fixtures under tests/golden/ by running the Hermes3D
reference itself (built from its sources by oracle/Makefile; needs the
reference tree, so this runs only where it is present).

    make -C oracle REF=/path/to/hermes3d && python tests/golden/make_golden.py

Each fixture is an .npz holding the mesh, the space/forms parameters and
what the reference produced: ndof, the CSC pattern (Ap, Ai), Ax, rhs and the
assembly list of every element (element-id order).
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from hermes3d_b200.mesh import permute_vertices, unit_cube  # noqa: E402
from oracle import ref_driver  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# name: (mesh builder, run kwargs)
CASES = {
    "c1_small": (lambda: unit_cube(2), dict(p=3, qmode="fixed:5", source="one", bc="dirichlet0")),
    "jitter_p3_mass_sin": (lambda: unit_cube(3, 0.2, 1), dict(p=3, qmode="fixed:5", mass=True, source="sin")),
    "perm_p3_mass_sin": (lambda: permute_vertices(unit_cube(3, 0.2, 1), seed=4),
                         dict(p=3, qmode="fixed:5", mass=True, source="sin")),
    "perm_p2_lifting": (lambda: permute_vertices(unit_cube(3, 0.1, 2), seed=5),
                        dict(p=2, qmode="fixed:4", bc="dirichlet_poly", source="poly")),
    "perm_p4_natural": (lambda: permute_vertices(unit_cube(2, 0.1, 2), seed=6),
                        dict(p=4, qmode="fixed:6", bc="natural", mass=True, source="one")),
    "perm_p1_natural": (lambda: permute_vertices(unit_cube(3, 0.2, 9), seed=8),
                        dict(p=1, qmode="fixed:3", bc="natural", source="one")),
    "aniso_orders_lifting": (lambda: permute_vertices(unit_cube(3, 0.1, 2), seed=7),
                             dict(orders=np.random.default_rng(1).integers(1, 7, size=(27, 3)).astype(np.int32),
                                  qmode="pplus:2", bc="dirichlet_poly", source="poly")),
    "coef_p3": (lambda: unit_cube(3, 0.2, 3),
                dict(p=3, qmode="fixed:5", gradcoef=np.random.default_rng(2).uniform(0.5, 2.0, 27), source="one")),
    "p2_c2_forms": (lambda: unit_cube(4, 0.2, 11), dict(p=2, qmode="fixed:4", mass=True, source="sin")),
}


def flatten_asm(asm, ne):
    by_id = {eid: (i, d, c) for eid, i, d, c in asm}
    ptr, idx, dof, coef = [0], [], [], []
    for e in range(1, ne + 1):
        i, d, c = by_id[e]
        idx.append(i)
        dof.append(d)
        coef.append(c)
        ptr.append(ptr[-1] + len(i))
    return np.array(ptr, np.int64), np.concatenate(idx), np.concatenate(dof), np.concatenate(coef)


def main():
    if not ref_driver.available():
        ref_driver.build()
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
