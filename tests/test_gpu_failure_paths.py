"""Failure paths of the device assembly, driven without any device fault:
a bounded wait that gives up (the kernel records a timeout, drains its copy
and leaves; the host reports H3DG_ERR_TIMEOUT) and a scatter position that
falls outside its CSC column (the bounds check skips the store; the host
reports H3DG_ERR_STATE).  After each, the next assembly is bit for bit the
one before."""
import numpy as np
import pytest

import hermes3d_b200 as h
from hermes3d_b200 import _capi
from helpers import disc_of, load, space_of

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["colour", "segmented"])
def scatter(request, monkeypatch):
    monkeypatch.setenv("H3DG_SCATTER", request.param)
    return request.param


def _problem():
    g = load("perm_p2_lifting")
    sp = space_of(g)
    d = disc_of(g, sp)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    d.assemble(M, V)
    return d, M, V, M.Ax.copy(), V.v.copy()


def test_wait_that_gives_up_reports_timeout_and_recovers(gpu, scatter):
    d, M, V, ax, v = _problem()
    d.debug_inject(_capi.DEBUG_WAIT_GIVES_UP)
    with pytest.raises(_capi.H3dgError) as e:
        d.assemble(M, V)
    assert e.value.status == _capi.H3DG_ERR_TIMEOUT
    if scatter == "colour":
        assert not np.array_equal(M.Ax, ax)        # every CTA left before its scatter
    d.assemble(M, V)
    assert np.array_equal(M.Ax, ax) and np.array_equal(V.v, v)


def test_position_outside_column_reports_state_and_rebuild_recovers(gpu, scatter):
    d, M, V, ax, v = _problem()
    d.debug_inject(_capi.DEBUG_CORRUPT_POSITION)
    for _ in range(2):                             # the corrupt plan keeps failing, nothing is written out of bounds
        with pytest.raises(_capi.H3dgError) as e:
            d.assemble(M, V)
        assert e.value.status == _capi.H3DG_ERR_STATE
        assert "outside its column" in str(e.value)
    d.create(M, V)                                 # a fresh plan
    d.assemble(M, V)
    assert np.array_equal(M.Ax, ax) and np.array_equal(V.v, v)
