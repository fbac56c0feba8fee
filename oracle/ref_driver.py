"""Run the Hermes3D reference (built from its sources into oracle/_ref/ by
oracle/Makefile) on a mesh and read back what it assembled.

ORACLE / TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg; never by the product package.
"""
from __future__ import annotations

import json
import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = os.path.join(HERE, "_ref", "h3d_ref_driver")


def available():
    return os.path.exists(DRIVER)


def build(ref=None):
    """Compile the reference + shim + driver (needs the reference sources;
    their location: HERMES3D_REF, see oracle.REFERENCE_DIR)."""
    if ref is None:
        from oracle import REFERENCE_DIR as ref
    if not os.path.isdir(ref):
        return available()
    subprocess.run(["make", "-C", HERE, "-j8", "REF=" + ref, "all"], check=True, capture_output=True)
    return available()


def run(mesh, p=2, orders=None, qmode="pplus:2", mass=False, gradcoef=None, source="one", bc="dirichlet0",
        repeat=1, elem_dump=False, assemble=True, refine=None, surf_uv=False, surf_g=None, natural_markers=None,
        sys=None, source2="none", p2=0, dump=None, timeout=3600):
    """Assemble ``mesh`` (hermes3d_b200.Mesh with arrays) with the reference.

    Returns dict(ndof, nnz, Ap, Ai, Ax, rhs, asm=[(id, idx, dof, coef)...],
    blocks=[...] (with elem_dump), timing=dict).
    """
    if not available():
        raise RuntimeError("reference oracle not built (make -C oracle)")
    with tempfile.TemporaryDirectory() as td:
        mf = os.path.join(td, "m.bin")
        of = os.path.join(td, "o.bin")
        mesh.save_bin(mf)
        cmd = [DRIVER, "--mesh", mf, "--out", of, "--p", str(p), "--qmode", qmode, "--source", source, "--bc", bc,
               "--repeat", str(repeat)]
        if orders is not None:
            o = np.ascontiguousarray(orders, dtype=np.int32).reshape(-1, 3)
            fn = os.path.join(td, "ord.bin")
            with open(fn, "wb") as f:
                f.write(struct.pack("<q", len(o)))
                f.write(o.tobytes())
            cmd += ["--orders", fn]
        if gradcoef is not None:
            c = np.ascontiguousarray(gradcoef, dtype=np.float64)
            fn = os.path.join(td, "coef.bin")
            with open(fn, "wb") as f:
                f.write(struct.pack("<q", len(c)))
                f.write(c.tobytes())
            cmd += ["--gradcoef", fn]
        if refine is None and getattr(mesh, "refinements", None):
            refine = mesh.refinements
        if refine is not None:
            r = np.ascontiguousarray(refine, dtype=np.int64).reshape(-1, 2)
            fn = os.path.join(td, "ref.bin")
            with open(fn, "wb") as f:
                f.write(struct.pack("<q", len(r)))
                f.write(r.tobytes())
            cmd += ["--refine", fn]
        if mass:
            cmd.append("--mass")
        if sys is not None:
            cmd += ["--sys", ",".join(sys), "--source2", source2]
            if p2:
                cmd += ["--p2", str(p2)]
        if dump:
            cmd += ["--dump", dump]
        if surf_uv:
            cmd.append("--surf-uv")
        if surf_g is not None:
            cmd += ["--surf-g", ",".join(repr(float(x)) for x in surf_g)]
        if natural_markers:
            cmd += ["--natural-markers", ",".join(str(int(m)) for m in natural_markers)]
        if elem_dump:
            cmd.append("--elem-dump")
        if not assemble:
            cmd.append("--no-asm")
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError("reference driver failed (%d): %s" % (r.returncode, r.stderr[-2000:]))
        timing = json.loads(r.stdout.strip().splitlines()[-1])
        return _parse(of, elem_dump) | {"timing": timing}


def _parse(path, elem_dump):
    with open(path, "rb") as f:
        buf = f.read()
    assert buf[:8] == b"H3DOUT01"
    pos = 8

    def take(dtype, n):
        nonlocal pos
        a = np.frombuffer(buf, dtype=dtype, count=n, offset=pos)
        pos += a.nbytes
        return a.copy()

    ndof, nnz = take(np.int64, 2)
    out = {"ndof": int(ndof), "nnz": int(nnz)}
    if ndof > 0:
        out["Ap"] = take(np.int32, ndof + 1).astype(np.int64)
        out["Ai"] = take(np.int32, nnz)
        out["Ax"] = take(np.float64, nnz)
        out["rhs"] = take(np.float64, ndof)
    nel = int(take(np.int64, 1)[0])
    asm = []
    rec = np.dtype([("idx", "<i8"), ("dof", "<i4"), ("coef", "<f8")])
    for _ in range(nel):
        eid, cnt = take(np.int64, 2)
        r = np.frombuffer(buf, dtype=rec, count=int(cnt), offset=pos)
        pos += r.nbytes
        asm.append((int(eid), r["idx"].copy(), r["dof"].copy(), r["coef"].copy()))
    out["asm"] = asm
    if elem_dump:
        nb = int(take(np.int64, 1)[0])
        blocks = []
        for _ in range(nb):
            n = int(take(np.int64, 1)[0])
            blocks.append(take(np.float64, n))
        out["blocks"] = blocks
    return out
