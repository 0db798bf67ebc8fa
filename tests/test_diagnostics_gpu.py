"""Diagnostics and the precision configuration: FP64 conservation sums (awfl_state_sums),
the device-side state check (awfl_check_state, failures injected on the host), normal
(Box-Muller) initial noise, and the FP32 form against the FP64 path on the 512x512x128
precision configuration (amp 2 K, radius 1.5 km, N(0, 0.05 K) theta noise, 100 steps)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from awflcloud_b200 import capi  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def interior(c, a):
    h = c.hs
    return a[..., h:h + c.nz, h:h + c.ny, h:h + c.nx]


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
def test_state_sums_match_a_direct_sum_and_repeat_exactly(prec):
    c = capi.Context(48, 40, 24, precision=prec)
    s = c.new_state()
    c.init_state(s, kind=capi.INIT_BUBBLE, noise_amp=0.01)
    dt = c.cfl(s, 0.8)
    for _ in range(3):
        c.step(s, dt)
    a = c.state_sums(s)
    b = c.state_sums(s)
    assert np.array_equal(a, b)
    x = interior(c, s[:5]).double() - (interior(c, s[5:]).double() if prec == capi.FP32 else 0)
    dv = (20000.0 / 48) * (20000.0 / 40) * (10000.0 / 24)
    ref = x.sum(dim=(1, 2, 3)).cpu().numpy() * dv
    scale = (x.abs().sum(dim=(1, 2, 3)).cpu().numpy() * dv) + 1e-300
    assert np.all(np.abs(a - ref) <= 1e-12 * scale), (a, ref)


def test_mass_is_conserved_to_rounding():
    c = capi.Context(64, 64, 32)  # periodic x/y, walls in z: no mass crosses the boundary
    s = c.new_state()
    c.init_state(s, kind=capi.INIT_BUBBLE, noise_amp=0.01)
    m0 = c.state_sums(s)[0]
    dt = c.cfl(s, 0.8)
    for _ in range(20):
        c.step(s, dt)
    m1 = c.state_sums(s)[0]
    total = float(np.sum(c.background()["hyDensCells"][c.hs:-c.hs])) * 64 * 64 * (20000.0 / 64) ** 2 * (10000.0 / 32)
    assert abs(m1 - m0) <= 1e-13 * total, (m0, m1, total)


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
def test_check_state_counts_injected_failures(prec):
    c = capi.Context(32, 24, 16, precision=prec)
    s = c.new_state()
    c.init_state(s, kind=capi.INIT_BUBBLE)
    assert c.check_state(s) == 0
    h = c.hs
    s[3, h + 2, h + 3, h + 4] = float("nan")          # a NaN momentum
    s[0, h + 5, h + 1, h + 1] = -10.0                 # total density 1.1 - 10 < 0
    s[4, h + 7, h + 7, h + 7] = float("inf")
    assert c.check_state(s) == 3
    rc = c.L.awfl_check_state(c.h, capi._ptr(s), None, None)
    assert rc == -4  # AWFL_ERR_STATE
    s[:, :h] = float("nan")                           # halo cells are not checked
    s[3, h + 2, h + 3, h + 4] = 0.0
    s[0, h + 5, h + 1, h + 1] = 0.0
    s[4, h + 7, h + 7, h + 7] = 0.0
    assert c.check_state(s) == 0


def test_normal_noise_has_the_requested_moments():
    c = capi.Context(128, 128, 64)
    s0, s1 = c.new_state(), c.new_state()
    c.init_state(s0, kind=capi.INIT_BUBBLE, amp=0.0)
    c.init_state(s1, kind=capi.INIT_BUBBLE, amp=0.0, noise_amp=0.05, noise_seed=11, noise_kind=capi.NOISE_NORMAL)
    dens = torch.tensor(c.background()["hyDensCells"][c.hs:-c.hs], device=s0.device)[:, None, None]
    n = (interior(c, s1[4]) - interior(c, s0[4])) / dens
    assert abs(n.mean().item()) < 3 * 0.05 / np.sqrt(n.numel())
    assert abs(n.std().item() / 0.05 - 1) < 0.01
    s2 = c.new_state()
    c.init_state(s2, kind=capi.INIT_BUBBLE, amp=0.0, noise_amp=0.05, noise_seed=11, noise_kind=capi.NOISE_NORMAL)
    assert torch.equal(s1, s2)


def test_precision_configuration_512():
    """512x512x128, amp 2 K, radius 1.5 km, N(0, 0.05 K) noise, 100 steps: the FP32 form
    stays within 1e-5 relative L2 of the FP64 path in every variable, and neither form
    changes the total mass beyond rounding."""
    n = (512, 512, 128)
    spec = dict(kind=capi.INIT_BUBBLE, xrad=1500.0, yrad=1500.0, zrad=1500.0, amp=2.0, noise_amp=0.05,
                noise_seed=20261203, noise_kind=capi.NOISE_NORMAL)
    c64, c32 = capi.Context(*n), capi.Context(*n, precision=capi.FP32)
    s64, s32 = c64.new_state(), c32.new_state()
    c64.init_state(s64, **spec)
    c32.init_state(s32, **spec)
    dt = c64.cfl(s64, 0.8)
    m64, m32 = c64.state_sums(s64)[0], c32.state_sums(s32)[0]
    for _ in range(100):
        c64.step(s64, dt)
        c32.step(s32, dt)
    assert c64.check_state(s64) == 0 and c32.check_state(s32) == 0
    for v in range(5):
        x, y = interior(c32, s32[v]).double(), interior(c64, s64[v])
        err = (torch.linalg.vector_norm(x - y) / torch.linalg.vector_norm(y)).item()
        assert err <= 1e-5, (v, err)
    bg = c64.background()["hyDensCells"][c64.hs:-c64.hs]
    total = float(np.sum(bg)) * n[0] * n[1] * (20000.0 / 512) ** 2 * (10000.0 / 128)
    assert abs(c64.state_sums(s64)[0] - m64) <= 1e-12 * total
    assert abs(c32.state_sums(s32)[0] - m32) <= 1e-7 * total
