"""tcgen05 tile path: BF16 operands in the no-swizzle K-major layout, FP32 accumulation in TMEM."""
import numpy as np
import pytest

from nnpengine_b200 import _lib

pytestmark = pytest.mark.gpu


def bf16(a):
    """Round-to-nearest-even to bfloat16, returned as float64."""
    u = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
@pytest.mark.parametrize("N,K", [(64, 64), (128, 32), (256, 128), (16, 16), (192, 96)])
def test_tcgen05_tile_gemm(mode, N, K):
    """mode 0: K-major operands; 1: MN-major B; 2: A whose rows repeat every 8 (zero group stride);
    3: both."""
    rng = np.random.default_rng(N * 1000 + K + mode)
    A = rng.standard_normal((128, K)).astype(np.float32)
    if mode in (2, 3):
        A = np.tile(A[:8], (16, 1))
    B = rng.standard_normal((N, K)).astype(np.float32)
    D = np.zeros((128, N), np.float32)
    rc = _lib.load().nnpe_tc_selftest(0, mode, N, K, A.ravel(), B.ravel(), D.ravel())
    assert rc == 0
    ref = bf16(A) @ bf16(B).T
    np.testing.assert_allclose(D, ref, rtol=1e-5, atol=1e-4)
