"""FP32 precision form (perturbation form + Kahan-compensated stage updates).

Bar: relative L2 <= 1e-5 in rho*theta after 100 steps at 256x256x128 against
the FP64 path (itself bit-identical to the reference arithmetic, test_parity_gpu.py).
Smaller grids and every variable are checked as well, with the measured accuracy of
single precision as the bound.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from awflcloud_b200 import capi  # noqa: E402

BUBBLE = dict(kind=capi.INIT_BUBBLE, noise_amp=0.01)


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def rel_l2(a, b):
    return (torch.linalg.vector_norm((a - b).double()) / torch.linalg.vector_norm(b.double())).item()


def pair(n, ord_=5, bc=("periodic", "periodic", "wall")):
    c64 = capi.Context(*n, ord_=ord_, bc=bc)
    c32 = capi.Context(*n, ord_=ord_, bc=bc, precision=capi.FP32)
    s64 = c64.new_state()
    c64.init_state(s64, **BUBBLE)
    s32 = c32.new_state()
    assert s32.shape[0] == 10  # value plane + Kahan plane
    c32.init_state(s32, **BUBBLE)
    return c64, c32, s64, s32


def interior(st, hs, nplane=5):
    return st[:nplane, hs:-hs, hs:-hs, hs:-hs]


@pytest.mark.parametrize("d", [0, 1, 2])
@pytest.mark.parametrize("ord_", [5, 9])
def test_single_split_tendencies_close_to_fp64(d, ord_):
    n = (48, 40, 24)
    c64, c32, s64, s32 = pair(n, ord_)
    # start both from the same (FP32-representable) state
    s64[:5] = s32[:5].double()
    dt = c64.cfl(s64, 0.8 if ord_ == 5 else 0.4)
    for spl in range(2):  # develop winds first
        c64.split(s64, dt, spl)
    s32[:5] = s64.float()
    s32[5:] = 0
    s64[:5] = s32[:5].double()
    t64, t32 = c64.new_tend(), c32.new_tend()
    c64.compute_tendencies(s64, t64, dt, d)
    c32.compute_tendencies(s32, t32, dt, d)
    torch.cuda.synchronize()
    for v in range(5):
        ref = t64[v].abs().max().item()
        if ref == 0.0:  # e.g. rho*w after x/y splits from rest: both must stay exactly zero
            assert t32[v].abs().max().item() == 0.0, (d, v)
            continue
        e = rel_l2(t32[v].double(), t64[v])
        assert e < 2e-4, (d, v, e)


@pytest.mark.parametrize("ord_,cfl,steps", [(5, 0.8, 50), (9, 0.4, 20)])
def test_rising_bubble_fp32_vs_fp64(ord_, cfl, steps):
    n = (64, 64, 32)
    c64, c32, s64, s32 = pair(n, ord_)
    dt = c64.cfl(s64, cfl)
    assert abs(c32.cfl(s32, cfl) - dt) <= 1e-6 * dt
    for _ in range(steps):
        c64.step(s64, dt)
        c32.step(s32, dt)
    hs = c64.hs
    a, b = interior(s32, hs).double(), interior(s64, hs)
    errs = [rel_l2(a[v], b[v]) for v in range(5)]
    print("FP32 vs FP64 rel L2 per variable after %d steps (ord %d):" % (steps, ord_), errs)
    assert errs[4] <= 1e-5
    assert max(errs) <= 1e-3


def test_fused_equals_unfused_fp32():
    n = (40, 36, 20)
    c32 = capi.Context(*n, precision=capi.FP32, bc=("wall", "periodic", "wall"))
    a = c32.new_state()
    c32.init_state(a, **BUBBLE)
    b = a.clone()
    tend = c32.new_tend()
    dt = c32.cfl(a, 0.8)
    for d in (0, 1, 2, 2, 1, 0):
        c32.split(a, dt, d)
        c32.compute_tendencies(b, tend, dt, d)
        c32.apply_tendencies(b, tend, dt)
    torch.cuda.synchronize()
    assert torch.equal(a, b)


def test_fp32_mass_conservation():
    c32 = capi.Context(128, 128, 64, precision=capi.FP32)
    st = c32.new_state()
    c32.init_state(st, **BUBBLE)
    dt = c32.cfl(st, 0.8)
    hs = c32.hs
    m0 = (st[0, hs:-hs, hs:-hs, hs:-hs].double() - st[5, hs:-hs, hs:-hs, hs:-hs].double()).sum().item()
    for _ in range(10):
        c32.step(st, dt)
    rho = st[0, hs:-hs, hs:-hs, hs:-hs].double() - st[5, hs:-hs, hs:-hs, hs:-hs].double()
    m1 = rho.sum().item()
    assert torch.isfinite(st).all()
    assert abs(m1 - m0) <= 1e-6 * rho.abs().sum().item()


def test_fp32_full_size_rhotheta_bar():
    """The accuracy bar: 256x256x128, ord 5, 100 steps, rel L2 <= 1e-5 in rho*theta."""
    c64, c32, s64, s32 = pair((256, 256, 128))
    dt = c64.cfl(s64, 0.8)
    for _ in range(100):
        c64.step(s64, dt)
        c32.step(s32, dt)
    hs = c64.hs
    e = rel_l2(interior(s32, hs)[4].double(), interior(s64, hs)[4])
    print("256x256x128 x 100 steps: FP32 vs FP64 rel L2 (rho*theta) = %.3e" % e)
    assert e <= 1e-5


@pytest.mark.parametrize("ord_", [5, 9])
@pytest.mark.parametrize("bc", [("periodic", "periodic", "wall"), ("wall", "wall", "wall")])
def test_tma_staging_matches_cp_async_staging(ord_, bc):
    """Interior chunks of the FP32 sweeps arrive by tiled TMA when the state is 16-byte
    aligned with a row pitch that is a multiple of 16 bytes; the same state two floats
    further on (8-byte aligned, as the C ABI requires) takes the per-thread cp.async path
    in every chunk. Both stage the same values into the ring; the two kernels (separate
    instantiations, compiled with multiply-add contraction) may still round a few
    operations differently, so the bound is FP32 rounding: relative L2 <= 1e-6 per
    variable after 4 steps (a staging fault would show as O(1) differences). The grid
    leaves partial tiles (missing lines inside a box) and a partial last chunk in every
    direction, and no bounded TMA wait may have given up
    (awfl_check_state would report AWFL_ERR_TIMEOUT). Each state has its own context: a
    context alternates the split order from one step to the next."""
    n = (60, 44, 36)  # nx + 2hs = 64 (ord 5) / 68 (ord 9): a multiple of 4 floats
    ca = capi.Context(*n, ord_=ord_, bc=bc, precision=capi.FP32)
    cb = capi.Context(*n, ord_=ord_, bc=bc, precision=capi.FP32)
    s = ca.new_state()
    ca.init_state(s, **BUBBLE)
    dt = ca.cfl(s, 0.8 if ord_ == 5 else 0.4)
    buf = torch.empty(s.numel() + 2, dtype=torch.float32, device=s.device)
    u = buf[2:].view(s.shape)
    u.copy_(s)
    assert s.data_ptr() % 16 == 0 and u.data_ptr() % 16 == 8
    for _ in range(4):
        ca.step(s, dt)
        cb.step(u, dt)
    torch.cuda.synchronize()
    assert torch.isfinite(s).all()
    for v in range(5):
        x, y = interior(s, ca.hs, 10)[v].double(), interior(u, cb.hs, 10)[v].double()
        err = (torch.linalg.vector_norm(x - y) / torch.linalg.vector_norm(y)).item()
        assert err <= 1e-6, (v, err)
    assert ca.check_state(s) == 0 and cb.check_state(u) == 0
