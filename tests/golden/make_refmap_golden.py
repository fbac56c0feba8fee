"""Fixture from the reference's own RefMap known-answer dumps.

Reads, as text, the meshes meshes/mesh3d/hex{1,2,4,8,27}.mesh3d and the dumps
tests/refmap/dump/hex*.dump of the reference (tests/refmap/main.cc:49-95
prints, per element, the Jacobian determinant, the Jacobian matrix and the
transposed inverse at the 2 x 2 x 2 Gauss points of order (2,2,2), and the
physical coordinates, to 6 decimals) and writes tests/golden/kat/refmap_dumps.npz.
Run in the build container (the reference tree is not on the GPU box):
    python tests/golden/make_refmap_golden.py /root/reference
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_mesh3d(path):
    """vertices, hexes (1-based), boundary quads (1-based) and markers of a mesh3d file"""
    toks = []
    with open(path) as f:
        for line in f:
            line = line.split("#")[0].strip()
            if line:
                toks.append(line.split())
    it = iter(toks)
    nv = int(next(it)[0])
    xyz = np.array([[float(v) for v in next(it)] for _ in range(nv)])
    nt = int(next(it)[0])
    for _ in range(nt):
        next(it)
    nh = int(next(it)[0])
    hexes = np.array([[int(v) for v in next(it)] for _ in range(nh)])
    npr = int(next(it)[0])
    for _ in range(npr):
        next(it)
    ntri = int(next(it)[0])
    for _ in range(ntri):
        next(it)
    nq = int(next(it)[0])
    quads = [next(it) for _ in range(nq)]
    bq = np.array([[int(v) for v in q[:4]] for q in quads])
    bm = np.array([int(q[4]) for q in quads])
    return xyz, hexes, bq, bm


def read_dump(path):
    num = r"[-+]?\d+\.\d+"
    elems = []
    cur = None
    mode = None
    with open(path) as f:
        for line in f:
            if line.startswith("Element #"):
                cur = {"jac": [], "rm": [], "irm": [], "phys": []}
                elems.append(cur)
                mode = None
            elif line.startswith(" - jacobian:"):
                cur["jac"] = [float(v) for v in re.findall(num, line)]
            elif line.startswith(" - refmap | inv ref map"):
                mode = "rm"
            elif line.startswith(" - phys coords"):
                mode = "phys"
            elif line.startswith(" * Face"):
                mode = None
            elif mode == "rm" and "|" in line:
                a, b = line.split("|")
                cur["rm"].append([float(v) for v in re.findall(num, a)])
                cur["irm"].append([float(v) for v in re.findall(num, b)])
            elif mode == "phys" and line.strip():
                cur["phys"].append([float(v) for v in re.findall(num, line)])
    for e in elems:
        e["rm"] = np.array(e["rm"]).reshape(-1, 3, 3)
        e["irm"] = np.array(e["irm"]).reshape(-1, 3, 3)
        e["phys"] = np.array(e["phys"]).reshape(-1, 3)
        e["jac"] = np.array(e["jac"])
    return elems


def main(ref):
    out = {}
    for name in ["hex1", "hex2", "hex4", "hex8", "hex27"]:
        xyz, hexes, bq, bm = read_mesh3d(os.path.join(ref, "meshes", "mesh3d", name + ".mesh3d"))
        el = read_dump(os.path.join(ref, "tests", "refmap", "dump", name + ".dump"))
        assert len(el) == len(hexes)
        out[name + "_xyz"], out[name + "_hexes"], out[name + "_bquads"], out[name + "_bmarkers"] = xyz, hexes, bq, bm
        out[name + "_jac"] = np.stack([e["jac"] for e in el])
        out[name + "_rm"] = np.stack([e["rm"] for e in el])
        out[name + "_irm"] = np.stack([e["irm"] for e in el])
        out[name + "_phys"] = np.stack([e["phys"] for e in el])
    np.savez_compressed(os.path.join(HERE, "kat", "refmap_dumps.npz"), **out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HERMES3D_REF", "/root/reference"))
