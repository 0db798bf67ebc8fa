"""The FP64 path's correctly rounded pow/exp (awfl_pow.cuh).

The reference's CPU build evaluates every pow with glibc. The library evaluates pow to
~2^-75 relative in double-double arithmetic and rounds once, so its results are the
correctly rounded ones; they agree with glibc's except where glibc itself misrounds
(measured here against 200-bit mpmath values). The CUDA math library's pow is counted
beside it for reference only.
"""
import math

import mpmath as mp
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from awflcloud_b200 import capi  # noqa: E402

GAMMA = 1.40027894002789400278940027894
mp.mp.prec = 200


def _device(x, y, mode):
    L = capi.lib()
    d_x = torch.from_numpy(x).cuda()
    d_o = torch.empty_like(d_x)
    rc = L.awfl_selftest_pow(d_x.data_ptr(), y, d_o.data_ptr(), x.size, mode,
                             torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    torch.cuda.synchronize()
    return d_o.cpu().numpy()


def _cr_pow(x, y):
    return float(mp.power(mp.mpf(float(x)), mp.mpf(float(y))))


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("lo,hi,y", [
    (10.0, 2000.0, GAMMA),               # (rho*theta)^gamma: every pow on the hot path
    (0.3, 1.0, 1004.0 / 287.0),          # exner^(cp/rd) in the hydrostatic profile
    (1e2, 1e5, 1.0 / GAMMA),             # (p/C0)^(1/gamma)
    (1e-3, 1.0, 1.0),                    # bubble shape power
])
def test_pow_correctly_rounded(lo, hi, y):
    rng = np.random.default_rng(7)
    x = np.exp(rng.uniform(math.log(lo), math.log(hi), 200_000))
    mine = _device(x, y, 0)
    glibc = np.array([math.pow(v, y) for v in x])
    cuda = _device(x, y, 1)
    # every disagreement with glibc must be glibc's misrounding
    idx = np.nonzero(mine != glibc)[0]
    for i in idx:
        assert mine[i] == _cr_pow(x[i], y), (x[i], y)
    # and a random sample is correctly rounded
    for i in rng.integers(0, x.size, 300):
        assert mine[i] == _cr_pow(x[i], y), (x[i], y)
    print("pow y=%.6g over %d inputs: library != glibc %d (all glibc misroundings); "
          "CUDA math library != glibc %d" % (y, x.size, idx.size, int((cuda != glibc).sum())))


def test_exp_correctly_rounded():
    rng = np.random.default_rng(8)
    x = rng.uniform(-5.0, 5.0, 100_000)
    mine = _device(x, 0.0, 2)
    glibc = np.array([math.exp(v) for v in x])
    for i in np.nonzero(mine != glibc)[0]:
        assert mine[i] == float(mp.exp(mp.mpf(float(x[i])))), x[i]
    for i in rng.integers(0, x.size, 300):
        assert mine[i] == float(mp.exp(mp.mpf(float(x[i])))), x[i]
