"""Generate the refined-mesh (hanging-node) fixtures under tests/golden/refined/
by running the Hermes3D reference itself (built from its sources by
oracle/Makefile; needs the reference tree, so this runs only where it is
present).

    make -C oracle REF=/path/to/hermes3d && python tests/golden/make_refined_golden.py

Each fixture holds the base mesh, the refinements (element id, REFT_HEX_XYZ)
applied with Mesh::refine_element, the per-element-id orders, the space and
form parameters, and what the reference produced: ndof, the CSC pattern,
Ax, rhs and the DOFs of every active element's assembly list.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from hermes3d_b200.mesh import permute_vertices, unit_cube  # noqa: E402
from oracle import ref_driver  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "refined")
XYZ = 7   # REFT_HEX_XYZ


def _orders(n_ids, p=None, seed=None):
    if seed is None:
        return np.full((n_ids, 3), p, np.int32)
    return np.random.default_rng(seed).integers(1, 7, size=(n_ids, 3)).astype(np.int32)


def _c3_like():
    rng = np.random.default_rng(3)
    refs = sorted(int(e) for e in rng.choice(64, 6, replace=False) + 1)
    return refs, rng.integers(1, 7, size=(64 + 8 * len(refs), 3)).astype(np.int32)


_C3_REFS, _C3_ORDERS = _c3_like()

# name: (base mesh builder, refined element ids, run kwargs)
CASES = {
    "ref_center_p2": (lambda: unit_cube(3), [14], dict(p=2, source="one", bc="dirichlet0")),
    "ref_perm_p2_mass_sin": (lambda: permute_vertices(unit_cube(3, 0.2, 1), seed=4), [14],
                             dict(p=2, mass=True, source="sin", bc="dirichlet0")),
    "ref_perm_p3_natural": (lambda: permute_vertices(unit_cube(3, 0.2, 1), seed=5), [1, 14, 27],
                            dict(p=3, mass=True, source="one", bc="natural")),
    "ref_lifting_p3": (lambda: unit_cube(3, 0.1, 2), [5, 14], dict(p=3, source="poly", bc="dirichlet_poly")),
    "ref_coef_p3": (lambda: unit_cube(3, 0.2, 3), [13],
                    dict(p=3, source="one", bc="dirichlet0",
                         gradcoef=np.random.default_rng(2).uniform(0.5, 2.0, 27 + 8))),
    "ref_aniso_c3_like": (lambda: unit_cube(4), _C3_REFS, dict(orders=_C3_ORDERS, source="one", bc="dirichlet0")),
}


def main():
    if not ref_driver.available():
        ref_driver.build()
    os.makedirs(OUT, exist_ok=True)
    for name, (mk, refs, kw) in CASES.items():
        mesh = mk()
        n_ids = len(mesh.hexes) + 8 * len(refs)
        kw = dict(kw)
        orders = kw.pop("orders", None)
        if orders is None:
            orders = _orders(n_ids, p=kw["p"])
        kw.setdefault("p", 1)
        r = ref_driver.run(mesh, orders=orders, qmode="pplus:2", refine=[(e, XYZ) for e in refs], **kw)
        act_ids = sorted(eid for eid, _, _, _ in r["asm"])
        by_id = {eid: d for eid, _, d, _ in r["asm"]}
        ptr, dofs = [0], []
        for eid in act_ids:
            dofs.append(by_id[eid])
            ptr.append(ptr[-1] + len(by_id[eid]))
        params = {k: v for k, v in kw.items() if k not in ("gradcoef",)}
        params["qmode"] = "pplus:2"
        np.savez_compressed(
            os.path.join(OUT, name + ".npz"), xyz=mesh.xyz, hexes=mesh.hexes, bquads=mesh.bquads,
            bmarkers=mesh.bmarkers, refine=np.array(refs, np.int64), params=np.array(repr(params)), orders=orders,
            gradcoef=kw.get("gradcoef", np.zeros(0)), ndof=r["ndof"], Ap=r["Ap"], Ai=r["Ai"], Ax=r["Ax"], rhs=r["rhs"],
            act_ids=np.array(act_ids, np.int64), al_ptr=np.array(ptr, np.int64), al_dof=np.concatenate(dofs))
        print(name, "ndof", r["ndof"], "nnz", r["nnz"], "active", len(act_ids))


if __name__ == "__main__":
    main()
