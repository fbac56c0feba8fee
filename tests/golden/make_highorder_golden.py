"""Generate the high-order fixtures under tests/golden/highorder/ by running
the Hermes3D reference itself (built from its sources by oracle/Makefile; needs
the reference tree, so this runs only where it is present).

    make -C oracle REF=/path/to/hermes3d && python tests/golden/make_highorder_golden.py

Orders p = 5, 6, 7, 8 on one or two hexahedra whose every vertex (boundary
ones included, so the maps are non-affine even on one element) is moved by a
seeded U(+-0.12h) offset, with the forms of the split-precision workload
(a_e grad.grad, a_e ~ U[0.5, 2] per element) and n = p + 2 Gauss points per
direction (10^3 at p = 8).  Natural and non-homogeneous Dirichlet faces are
mixed so that every kind of function pair (vertex, edge, face, bubble) is in
the matrix or, through the lifting, in the rhs.  Each fixture holds the mesh,
the parameters and the reference's ndof, pattern (Ap, Ai), Ax, rhs and the
assembly list of every element (element-id order).
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from hermes3d_b200.mesh import Mesh, permute_vertices, unit_cube  # noqa: E402
from oracle import ref_driver  # noqa: E402
from make_golden import flatten_asm  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "highorder")


def jittered_all(nx, seed, amp=0.12):
    """nx x 1 x 1 elements on [0, nx] x [0, 1]^2 scaled to the unit cube in x,
    every vertex moved by U(-amp h, amp h) per coordinate."""
    m = unit_cube(1, nx=nx)
    h = np.array([1.0 / nx, 1.0, 1.0])
    X = m.xyz + amp * h * np.random.default_rng(seed).uniform(-1.0, 1.0, m.xyz.shape)
    return Mesh().set_arrays(X, m.hexes, m.bquads, m.bmarkers)


# name: (mesh builder, number of elements, run kwargs)
CASES = {
    # two elements sharing a face (random orientations), every face natural: the whole
    # element matrices of both elements and their sum on the shared face
    "hp5_2el_natural": (lambda: permute_vertices(jittered_all(2, 5), seed=15), 2,
                        dict(p=5, qmode="fixed:7", bc="natural", mass=True, source="sin")),
    # one element, Dirichlet x^2+y^2+z^2 on markers 2, 4, 6 (lifting), natural on 1, 3, 5
    "hp6_1el_mixed": (lambda: jittered_all(1, 6), 1,
                      dict(p=6, qmode="fixed:8", bc="dirichlet_poly", natural_markers=[1, 3, 5], source="poly")),
    # one element, Dirichlet on every face: bubbles in the matrix, everything else lifted
    "hp7_1el_lifting": (lambda: permute_vertices(jittered_all(1, 7), seed=17), 1,
                        dict(p=7, qmode="fixed:9", bc="dirichlet_poly", source="poly")),
    # the split-precision workload's element: p = 8, 10^3 points
    "hp8_1el_mixed": (lambda: permute_vertices(jittered_all(1, 8), seed=18), 1,
                      dict(p=8, qmode="fixed:10", bc="dirichlet_poly", natural_markers=[1, 4, 5], source="sin")),
}


def main():
    if not ref_driver.available():
        ref_driver.build()
    os.makedirs(OUT, exist_ok=True)
    for name, (mk, ne, kw) in CASES.items():
        mesh = mk()
        coef = np.random.default_rng(100 + kw["p"]).uniform(0.5, 2.0, ne)
        r = ref_driver.run(mesh, gradcoef=coef, **kw)
        ptr, idx, dof, cf = flatten_asm(r["asm"], len(mesh.hexes))
        np.savez_compressed(
            os.path.join(OUT, name + ".npz"), xyz=mesh.xyz, hexes=mesh.hexes, bquads=mesh.bquads,
            bmarkers=mesh.bmarkers, params=np.array(repr(kw)), orders=np.zeros((0, 3), np.int32), gradcoef=coef,
            ndof=r["ndof"], Ap=r["Ap"], Ai=r["Ai"], Ax=r["Ax"], rhs=r["rhs"], al_ptr=ptr, al_idx=idx, al_dof=dof,
            al_coef=cf)
        print(name, "ndof", r["ndof"], "nnz", r["nnz"], "t_assemble %.1fs" % r["timing"]["t_assemble"])


if __name__ == "__main__":
    main()
