"""Generate the two-equation system fixtures under tests/golden/system/ by
running the Hermes3D reference itself (built from its sources by
oracle/Makefile; needs the reference tree, so this runs only where it is
present).

    make -C oracle REF=/path/to/hermes3d && python tests/golden/make_system_golden.py

Two H1 spaces numbered one after another (the pattern of the reference's
calc/hex-h1-sys* tests) -- identical, or of different uniform orders (p, p2)
--, block forms grad.grad, grad.grad + mass or mass alone, a source per
equation; ndof, pattern, Ax and rhs of the reference's Discretization with
neq = 2.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from hermes3d_b200.mesh import permute_vertices, unit_cube  # noqa: E402
from oracle import ref_driver  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "system")

CASES = {
    "sys_uncoupled_p2": (lambda: unit_cube(3, 0.1, 1),
                         dict(p=2, bc="dirichlet0", source="one", sys=["gg", "none", "none", "gg"], source2="sin")),
    "sys_coupled_lifting_p2": (lambda: permute_vertices(unit_cube(3, 0.1, 2), seed=3),
                               dict(p=2, bc="dirichlet_poly", source="poly", sys=["gg", "mass", "mass", "gg"],
                                    source2="one")),
    "sys_mass_blocks_p3": (lambda: unit_cube(2, 0.2, 5),
                           dict(p=3, bc="natural", source="sin", sys=["ggm", "mass", "none", "gg"], source2="none")),
    # spaces of different orders, as the reference's calc/hex-h1-sys* tests (orders 2 and 4)
    "sys_diff_coupled_p2p4": (lambda: permute_vertices(unit_cube(2, 0.1, 4), seed=5),
                              dict(p=2, p2=4, bc="dirichlet0", source="sin", sys=["gg", "mass", "mass", "gg"],
                                   source2="one", qmode="fixed:6")),
    "sys_diff_lifting_p2p3": (lambda: permute_vertices(unit_cube(2, 0.15, 6), seed=7),
                              dict(p=2, p2=3, bc="dirichlet_poly", source="poly", sys=["gg", "mass", "mass", "gg"],
                                   source2="one", qmode="fixed:5")),
    "sys_diff_ggm_p3p2": (lambda: unit_cube(2, 0.2, 8),
                          dict(p=3, p2=2, bc="natural", source="one", sys=["ggm", "mass", "none", "gg"],
                               source2="sin", qmode="fixed:5")),
}


def main():
    if not ref_driver.available():
        ref_driver.build()
    os.makedirs(OUT, exist_ok=True)
    for name, (mk, kw) in CASES.items():
        mesh = mk()
        kw = dict(kw)
        kw.setdefault("qmode", "pplus:2")
        r = ref_driver.run(mesh, **kw)
        params = dict(kw)
        np.savez_compressed(
            os.path.join(OUT, name + ".npz"), xyz=mesh.xyz, hexes=mesh.hexes, bquads=mesh.bquads,
            bmarkers=mesh.bmarkers, params=np.array(repr(params)), orders=np.zeros((0, 3), np.int32),
            gradcoef=np.zeros(0), ndof=r["ndof"], Ap=r["Ap"], Ai=r["Ai"], Ax=r["Ax"], rhs=r["rhs"])
        print(name, "ndof", r["ndof"], "nnz", r["nnz"])


if __name__ == "__main__":
    main()
