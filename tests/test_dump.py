"""Dumps of the assembled system in the reference's formats
(UMFPackMatrix::dump / UMFPackVector::dump, src/linsolver/umfpack.cc:95-127,
194-220), pinned byte for byte by dumps the reference itself wrote for the
c1_small problem (tests/golden/dump, made by make_dump_golden.py)."""
import io
import os

import numpy as np
import pytest

import hermes3d_b200 as h
from helpers import FP64_RTOL, GOLDEN, disc_of, load, rel_err, space_of

DUMP = os.path.join(GOLDEN, "dump")


def _sinks(g):
    m, v = h.UMFPackMatrix(), h.UMFPackVector()
    m.ndofs, m.Ap, m.Ai, m.Ax = int(g["ndof"]), g["Ap"], g["Ai"], g["Ax"]
    v.v = g["rhs"]
    return m, v


def _ref(ext, mode="rb"):
    with open(os.path.join(DUMP, "c1_small." + ext), mode) as f:
        return f.read()


def test_binary_dumps_match_reference_bytes():
    m, v = _sinks(load("c1_small"))
    b = io.BytesIO()
    assert m.dump(b, "A", h.DF_HERMES_BIN)
    assert b.getvalue() == _ref("h2dx")
    b = io.BytesIO()
    assert v.dump(b, "b", h.DF_HERMES_BIN)
    assert b.getvalue() == _ref("h2dr")


def test_matlab_dump_matches_reference_text():
    m, v = _sinks(load("c1_small"))
    s = io.StringIO()
    assert m.dump(s, "A", h.DF_MATLAB_SPARSE) and v.dump(s, "b", h.DF_MATLAB_SPARSE)
    assert s.getvalue() == _ref("m", "r")


def test_load_reads_reference_dumps(tmp_path):
    g = load("c1_small")
    m = h.UMFPackMatrix.load(os.path.join(DUMP, "c1_small.h2dx"))
    v = h.UMFPackVector.load(os.path.join(DUMP, "c1_small.h2dr"))
    assert m.ndofs == g["ndof"]
    assert np.array_equal(m.Ap, g["Ap"]) and np.array_equal(m.Ai, g["Ai"])
    assert np.array_equal(m.Ax, g["Ax"]) and np.array_equal(v.v, g["rhs"])
    # our dump of what we loaded is the file we read
    p = tmp_path / "again.h2dx"
    m.dump(str(p), "A", h.DF_HERMES_BIN)
    assert p.read_bytes() == _ref("h2dx")


def test_unsupported_format_and_bad_files(tmp_path):
    m, v = _sinks(load("c1_small"))
    with pytest.raises(NotImplementedError):                     # the reference: ERR_NOT_IMPLEMENTED
        m.dump(io.StringIO(), "A", h.DF_PLAIN_ASCII)
    with pytest.raises(NotImplementedError):
        v.dump(io.StringIO(), "b", h.DF_PLAIN_ASCII)
    assert not m.dump(io.StringIO(), "A", 7) and not v.dump(io.StringIO(), "b", 7)
    with pytest.raises(ValueError):
        h.UMFPackMatrix.load(io.BytesIO(_ref("h2dr")))
    with pytest.raises(ValueError):
        h.UMFPackVector.load(io.BytesIO(_ref("h2dx")))


def test_empty_system_dump_round_trip():
    m, v = h.UMFPackMatrix(), h.UMFPackVector()
    m.ndofs, m.Ap, m.Ai, m.Ax = 0, np.zeros(1, np.int64), np.zeros(0, np.int32), np.zeros(0)
    v.v = np.zeros(0)
    b = io.BytesIO()
    m.dump(b, "A", h.DF_HERMES_BIN)
    b.seek(0)
    r = h.UMFPackMatrix.load(b)
    assert r.ndofs == 0 and len(r.Ai) == 0 and list(r.Ap) == [0]
    b = io.BytesIO()
    v.dump(b, "b", h.DF_HERMES_BIN)
    b.seek(0)
    assert len(h.UMFPackVector.load(b).v) == 0


@pytest.mark.gpu
def test_device_assembly_dumps_like_reference(tmp_path):
    """Assemble c1_small on the GPU, dump, load back: the same pattern bytes as
    the reference's dump and values within the FP64 tolerance."""
    g = load("c1_small")
    d = disc_of(g, space_of(g))
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)
    pm, pv = tmp_path / "A.h2dx", tmp_path / "b.h2dr"
    assert M.dump(str(pm), "A", h.DF_HERMES_BIN) and V.dump(str(pv), "b", h.DF_HERMES_BIN)
    mine, ref = pm.read_bytes(), _ref("h2dx")
    n, nnz = int(g["ndof"]), int(g["Ap"][-1])
    head = 20 + 4 * (n + 1) + 4 * nnz                       # magic, sizes, Ap, Ai
    assert len(mine) == len(ref) and mine[:head] == ref[:head]
    m2, v2 = h.UMFPackMatrix.load(str(pm)), h.UMFPackVector.load(str(pv))
    assert np.array_equal(m2.Ax, M.Ax) and np.array_equal(v2.v, V.v)
    r = h.UMFPackMatrix.load(os.path.join(DUMP, "c1_small.h2dx"))
    assert rel_err(m2.Ax, r.Ax) < FP64_RTOL
    assert rel_err(v2.v, h.UMFPackVector.load(os.path.join(DUMP, "c1_small.h2dr")).v) < FP64_RTOL
