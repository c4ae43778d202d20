"""
The tensor-core primitives (slipcam_b200/csrc/tc.cuh) against a host GEMM: shared-memory
descriptors in both major orders, the instruction descriptor's shape and negation, TMEM
allocation, MMA completion through an mbarrier, and TMEM loads (b200_tc_selftest). Small integer
operands make every product and sum exact in FP16 x FP16 -> FP32.
"""

import numpy as np
import pytest

from slipcam_b200 import _lib

pytestmark = pytest.mark.gpu
torch = pytest.importorskip('torch')


@pytest.mark.parametrize('a_mn', [0, 1])
@pytest.mark.parametrize('b_mn', [0, 1])
@pytest.mark.parametrize('neg_b', [0, 1])
@pytest.mark.parametrize('n, k', [(16, 16), (96, 64), (160, 160), (256, 32), (112, 192)])
def test_mma(a_mn, b_mn, neg_b, n, k):
    rng = np.random.default_rng(n * 1000 + k + 7 * a_mn + 3 * b_mn + neg_b)
    a = rng.integers(-8, 9, (128, k)).astype(np.float16)
    b = rng.integers(-8, 9, (n, k)).astype(np.float16)
    da, db = torch.as_tensor(a).cuda(), torch.as_tensor(b).cuda()
    d = torch.empty((128, n), dtype=torch.float32, device='cuda')
    rc = _lib.lib().b200_tc_selftest(da.data_ptr(), db.data_ptr(), d.data_ptr(), n, k, a_mn, b_mn, neg_b,
                                     torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.OK
    ref = a.astype(np.float64) @ b.astype(np.float64).T * (-1 if neg_b else 1)
    assert np.array_equal(d.cpu().numpy(), ref.astype(np.float32))
