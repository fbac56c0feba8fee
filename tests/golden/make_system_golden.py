"""Generate the two-equation system fixtures under tests/golden/system/ by
running the Hermes3D reference itself (built from its sources by
oracle/Makefile; needs the reference tree, so this runs only where it is
present).

    make -C oracle REF=/path/to/hermes3d && python tests/golden/make_system_golden.py

Two identical H1 spaces numbered one after another (the pattern of the
reference's calc/hex-h1-sys* tests), block forms grad.grad, grad.grad + mass
or mass alone, a source per equation; ndof, pattern, Ax and rhs of the
reference's Discretization with neq = 2.
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
}


def main():
    if not ref_driver.available():
        ref_driver.build()
    os.makedirs(OUT, exist_ok=True)
    for name, (mk, kw) in CASES.items():
        mesh = mk()
        r = ref_driver.run(mesh, qmode="pplus:2", **kw)
        params = dict(kw)
        params["qmode"] = "pplus:2"
        np.savez_compressed(
            os.path.join(OUT, name + ".npz"), xyz=mesh.xyz, hexes=mesh.hexes, bquads=mesh.bquads,
            bmarkers=mesh.bmarkers, params=np.array(repr(params)), orders=np.zeros((0, 3), np.int32),
            gradcoef=np.zeros(0), ndof=r["ndof"], Ap=r["Ap"], Ai=r["Ai"], Ax=r["Ax"], rhs=r["rhs"])
        print(name, "ndof", r["ndof"], "nnz", r["nnz"])


if __name__ == "__main__":
    main()
