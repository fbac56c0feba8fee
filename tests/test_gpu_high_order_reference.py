"""Orders 5..8 on the GPU against fixtures the reference itself assembled
(tests/golden/make_highorder_golden.py: jittered elements, a_e grad.grad,
p + 2 points per direction, 10^3 at p = 8, natural and Dirichlet faces).

FP64: the high-order kernel, entrywise within 1e-12 of the largest entry.
Split precision, with the error measured against the reference (not against
this library's own FP64 kernel): 3xTF32 within 1e-6 and the int8-sliced
(Ozaki) kernel within 1e-12, both entrywise-over-max and normwise.  The rhs
is FP64 in every precision."""
import numpy as np
import pytest

import hermes3d_b200 as h
from helpers import FP64_RTOL, highorder_names, highorder_problem, load_highorder, rel_err

pytestmark = pytest.mark.gpu

TOL = {h.PREC_FP64: FP64_RTOL, h.PREC_TF32X3: 1e-6, h.PREC_OZAKI: 1e-12}


def _norm_err(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("prec", [h.PREC_FP64, h.PREC_TF32X3, h.PREC_OZAKI])
@pytest.mark.parametrize("name", highorder_names())
def test_high_order_against_reference(gpu, name, prec):
    g = load_highorder(name)
    mesh, sp, d = highorder_problem(g)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    assert np.array_equal(M.Ap, g["Ap"]) and np.array_equal(M.Ai, g["Ai"])
    d.assemble(M, V, precision=prec)
    e_max, e_norm = rel_err(M.Ax, g["Ax"]), _norm_err(M.Ax, g["Ax"])
    print("%s precision %d: error vs reference max %.2e norm %.2e" % (name, prec, e_max, e_norm))
    assert e_max < TOL[prec] and e_norm < TOL[prec]
    assert rel_err(V.v, g["rhs"]) < FP64_RTOL
