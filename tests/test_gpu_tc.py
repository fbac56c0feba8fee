"""tcgen05 layer self-test: one 128 x 128 MMA tile through the C-ABI with
integer-valued operands (exact in tf32 and bf16), compared bit-for-bit with
the numpy product.  Checks shared-memory descriptors, the instruction
descriptor, TMEM allocation and the accumulator read-back layout."""
import numpy as np
import pytest
import torch

from hermes3d_b200 import _capi

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,K,lim", [(2, 32, 4), (1, 64, 4), (8, 64, 127)])
def test_tc_selftest_exact(gpu, kind, K, lim):
    rng = np.random.default_rng(kind)
    A = rng.integers(-lim, lim + 1, size=(128, K)).astype(np.float32)
    B = rng.integers(-lim, lim + 1, size=(128, K)).astype(np.float32)
    if kind == 8:
        A[0, :8] = -128                       # int8 extremes
        B[0, :8] = -128
    # distinct row / column signatures so a permuted read-back cannot pass
    A[:, 0] = np.arange(128) % 7 - 3
    B[:, 1] = np.arange(128) % 5 - 2
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    dC = torch.full((128, 128), float("nan"), dtype=torch.float32, device="cuda")
    _capi.call("h3dg_tc_selftest", kind, dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), 0)
    C = dC.cpu().numpy()
    np.testing.assert_array_equal(C, (A.astype(np.float64) @ B.T.astype(np.float64)).astype(np.float32))
