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


def _hard_quotients(rng, n):
    """Operand pairs whose quotient lies within ~2^-53 ulp of a rounding midpoint, where a
    division that is not correctly rounded would show: with integer significands B (odd,
    53 bits) and M (odd, 54 bits: the midpoint), B*M = A*2^53 +- 1 makes A/B = M/2^53
    -+ 1/(B*2^53), so M = +-B^-1 mod 2^53 and A = (B*M -+ 1)/2^53 must fit 53 bits."""
    a, b = [], []
    P = 1 << 53
    while len(a) < n:
        B = int(rng.integers(1 << 52, 1 << 53)) | 1
        s = 1 if len(a) % 2 else -1
        M = (s * pow(B, -1, P)) % P
        lo = (1 << 105) // B + 1
        M += ((lo - M + P - 1) // P) * P  # smallest M >= lo in the class
        if M >= (1 << 54) or B * M >= (1 << 106) or M % 2 == 0:
            continue
        A, r = divmod(B * M - s, P)
        assert r == 0 and (1 << 52) <= A < (1 << 53)
        ea, eb = int(rng.integers(-30, 30)), int(rng.integers(-30, 30))
        a.append(math.ldexp(A, ea - 52))
        b.append(math.ldexp(B, eb - 52))
    return np.array(a), np.array(b)


def test_shared_reciprocal_division_is_ieee():
    """The FP64 kernels divide by a shared divisor through its correctly rounded reciprocal
    plus two Markstein corrections (awfl_div.cuh); that must be the IEEE quotient bit for
    bit, signed zeros included."""
    rng = np.random.default_rng(11)
    n = 400_000
    a = np.exp(rng.uniform(-46.0, 46.0, n)) * rng.choice([-1.0, 1.0], n)
    b = np.exp(rng.uniform(-46.0, 46.0, n)) * rng.choice([-1.0, 1.0], n)
    # physical ranges of the path and edge cases: significands of all ones, b = 1, a = b,
    # signed zeros, operands one ulp apart, the constant divisors 3 and 5
    a[:4000] = rng.uniform(0.5, 2.0, 4000)
    b[:4000] = rng.uniform(0.5, 2.0, 4000)
    ones = np.nextafter(np.array([2.0, 4.0, 1.0, 0.5]), 0.0)
    b[4000:4004] = ones
    a[4004:4010] = [0.0, -0.0, 0.0, -0.0, 1.0, 3.0]
    b[4004:4010] = [3.0, 3.0, -7.0, -7.0, 1.0, 3.0]
    b[4010:4020] = 3.0
    b[4020:4030] = 5.0
    a[4030:4040] = np.nextafter(b[4030:4040], np.inf)
    ha, hb = _hard_quotients(rng, 20_000)
    a[4040:4040 + ha.size] = ha
    b[4040:4040 + hb.size] = hb
    x = np.concatenate([a, b])
    mine = _device_pairs(x, 3)
    ieee = _device_pairs(x, 4)
    host = a / b
    assert np.array_equal(ieee.view(np.int64), host.view(np.int64))
    bad = np.nonzero(mine.view(np.int64) != ieee.view(np.int64))[0]
    assert bad.size == 0, [(a[i], b[i], mine[i], ieee[i]) for i in bad[:5]]


def _device_pairs(x, mode):
    L = capi.lib()
    n = x.size // 2
    d_x = torch.from_numpy(x).cuda()
    d_o = torch.empty(n, dtype=torch.float64, device="cuda")
    rc = L.awfl_selftest_pow(d_x.data_ptr(), 0.0, d_o.data_ptr(), n, mode, torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    torch.cuda.synchronize()
    return d_o.cpu().numpy()
