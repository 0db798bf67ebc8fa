"""FP64 CUDA path (libawfl.so, sm_100a) against the reference and the CPU oracle.

Two bars:

1. BIT-EXACT against the reference arithmetic with a correctly rounded pow. The FP64
   kernels evaluate every pow correctly rounded (awfl_pow.cuh). The CPU oracle variant
   ``crpow`` does the same and is itself bit-identical to the reference's own code built
   with a correctly rounded pow (tests/test_oracle_golden.py). So GPU == oracle(crpow)
   exactly, split by split, tendencies, halos and states, and over the 64x64x32 x 50-step
   rising-bubble run.

2. Against the reference's glibc build (golden fixtures): glibc's pow is not correctly
   rounded in ~0.08% of calls, and the scheme amplifies those last-bit differences: the
   reference's own code with glibc's pow and with a correctly rounded pow differ by up to
   3.0e-12 relative L2 per variable after 50 steps at 64x64x32, and by up to 1.2e-11 on
   the tiny noise-dominated golden grids (measured). States are held to 5e-12 on the
   64x64x32 run and 2e-11 on the golden grids; per-split tendencies, where a difference
   of O(rho*cs) mass fluxes amplifies any last bit ~1e4-fold, to 1e-9.
"""
import glob
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from awflcloud_b200 import capi  # noqa: E402
from oracle.pyoracle import Oracle, build as build_oracle  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(os.path.basename(p)[5:-4] for p in glob.glob(os.path.join(GOLDEN, "case_*.npz")))
RTOL = 5e-12
GOLDEN_RTOL = 2e-11
TEND_RTOL = 1e-9


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def assert_close_vars(a, b, tol=RTOL, what=""):
    """Per variable: relative L2 and max error relative to the variable's max."""
    for v in range(a.shape[0]):
        av, bv = np.asarray(a[v]), np.asarray(b[v])
        scale = max(np.abs(bv).max(), 1e-300)
        assert np.abs(av - bv).max() <= tol * scale * 10, (what, v, np.abs(av - bv).max(), scale)
        assert rel_l2(av, bv) <= tol, (what, v, rel_l2(av, bv))


def ctx_for(g):
    ord_, nx, ny, nz, bx, by, bz, ws, ww = [int(v) for v in g["config"]]
    return capi.Context(nx, ny, nz, bc=(bx, by, bz), weno_scalars=bool(ws), weno_winds=bool(ww),
                        data=str(g["data"]), ord_=ord_)


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    build_oracle()


@pytest.mark.parametrize("case", CASES)
def test_golden_splits_unfused(case):
    """compute_tendencies + apply_tendencies, split by split, vs the reference."""
    g = np.load(os.path.join(GOLDEN, "case_%s.npz" % case))
    c = ctx_for(g)
    st = torch.from_numpy(np.array(g["state0"])).cuda()
    tend = c.new_tend()
    dt = float(g["dt"])
    assert abs(c.cfl(st, 0.8) - dt) <= 1e-15 * dt
    nsteps = len([k for k in g.files if k.startswith("state_s") and "_p" not in k])
    for step in range(min(2, nsteps)):
        order = [0, 1, 2] if step == 0 else [2, 1, 0]
        for spl, d in enumerate(order):
            c.compute_tendencies(st, tend, dt, d)
            torch.cuda.synchronize()
            assert_close_vars(tend.cpu().numpy(), g["tend_s%d_p%d" % (step, spl)], tol=TEND_RTOL,
                              what=(case, step, spl))
            c.apply_tendencies(st, tend, dt)
            if step == 0:
                assert_close_vars(st.cpu().numpy(), g["state_s0_p%d" % spl], tol=GOLDEN_RTOL,
                                  what=(case, "state", spl))
        assert_close_vars(st.cpu().numpy(), g["state_s%d" % step], tol=GOLDEN_RTOL, what=(case, "step", step))


@pytest.mark.parametrize("case", CASES)
def test_golden_fused_steps(case):
    """awfl_step (three fused split kernels, dimSwitch alternation) vs the reference."""
    g = np.load(os.path.join(GOLDEN, "case_%s.npz" % case))
    c = ctx_for(g)
    st = torch.from_numpy(np.array(g["state0"])).cuda()
    dt = float(g["dt"])
    nsteps = len([k for k in g.files if k.startswith("state_s") and "_p" not in k])
    for step in range(nsteps):
        c.step(st, dt)
        assert_close_vars(st.cpu().numpy(), g["state_s%d" % step], tol=GOLDEN_RTOL, what=(case, step))


@pytest.mark.parametrize("case", CASES)
def test_golden_init_state(case):
    """awfl_init_state (device quadrature) vs the reference's initState (+ bubble/noise)."""
    g = np.load(os.path.join(GOLDEN, "case_%s.npz" % case))
    c = ctx_for(g)
    st = c.new_state()
    kw = {}
    if "bubble" in g:
        b = g["bubble"]
        kw = dict(kind=capi.INIT_BUBBLE, shape=int(b[0]), x0=b[1], y0=b[2], z0=b[3], xrad=b[4],
                  yrad=b[5], zrad=b[6], amp=b[7], pwr=b[8])
    if "noise" in g:
        kw.update(noise_seed=int(g["noise"][0]), noise_amp=float(g["noise"][1]))
    c.init_state(st, **kw)
    h = c.hs
    got = st.cpu().numpy()[:, h:-h, h:-h, h:-h]
    ref = np.array(g["state0"])[:, h:-h, h:-h, h:-h]
    # pow/exp are correctly rounded on both sides; the bubble shapes' cos/sin are CUDA's,
    # which differ from glibc's in the last bit, hence a tolerance.
    for v in range(5):
        scale = max(np.abs(ref[v]).max(), 1e-300)
        assert np.abs(got[v] - ref[v]).max() <= 1e-12 * scale, (case, v)


def _bubble_case(o, nx, ny, nz, bc=(0, 0, 1), noise=0.01, crpow=False):
    O = Oracle(nx, ny, nz, bc=bc, ord_=o, crpow=crpow)
    st = O.new_state()
    O.init_state(st)
    O.set_bubble(st, 1, 10000.0, 10000.0, 2000.0, 2000.0, 2000.0, 2000.0, 3.0, 1.0)
    O.add_theta_noise(st, 20261203, noise)
    return O, st


@pytest.mark.parametrize("o,n,steps,cfl", [(5, (64, 64, 32), 50, 0.8), (9, (32, 32, 16), 10, 0.4)])
def test_rising_bubble_bit_exact(o, n, steps, cfl):
    """The parity configuration: 64x64x32 bubble + noise, 50 steps (ord 5): bit-identical
    to the reference arithmetic with a correctly rounded pow. ord 9 runs at CFL 0.4: at the
    driver's CFL 0.8 the reference's own ord-9 scheme diverges (NaN)."""
    O, st = _bubble_case(o, *n, crpow=True)
    dt = O.compute_dt(st, cfl)
    c = capi.Context(*n, ord_=o)
    d = torch.from_numpy(st.copy()).cuda()
    assert c.cfl(d, cfl) == dt
    for _ in range(steps):
        O.time_step(st, dt)
        c.step(d, dt)
    assert np.array_equal(d.cpu().numpy(), st)
    assert np.array_equal(d.cpu().numpy().view(np.int64), st.view(np.int64))  # signs of zero too


@pytest.mark.parametrize("o,n,steps,cfl", [(5, (64, 64, 32), 50, 0.8)])
def test_rising_bubble_vs_glibc_build(o, n, steps, cfl):
    """Same run against the oracle with glibc's pow (the reference's CPU build): within the
    reference's own glibc-vs-correctly-rounded spread."""
    O, st = _bubble_case(o, *n)
    dt = O.compute_dt(st, cfl)
    c = capi.Context(*n, ord_=o)
    d = torch.from_numpy(st.copy()).cuda()
    for _ in range(steps):
        O.time_step(st, dt)
        c.step(d, dt)
    got = d.cpu().numpy()
    h = c.hs
    for v in range(5):
        e = rel_l2(got[v, h:-h, h:-h, h:-h], st[v, h:-h, h:-h, h:-h])
        assert e <= RTOL, (v, e)


@pytest.mark.parametrize("o,n,steps,cfl", [(5, (64, 64, 32), 50, 0.8), (9, (32, 32, 16), 10, 0.4)])
def test_each_step_vs_glibc_build_same_inputs(o, n, steps, cfl):
    """Against the reference's glibc build on the same inputs: every one of the run's steps
    starts from the glibc build's own state (the oracle with glibc's pow, bit-identical to
    the reference's CPU build) and must land within 1e-12 relative L2 per variable of that
    build's next state. Only the rounding of glibc's pow separates the two; over many steps
    the scheme amplifies it (test_rising_bubble_vs_glibc_build), one step from the same
    input it stays far below the bar."""
    O, st = _bubble_case(o, *n)
    dt = O.compute_dt(st, cfl)
    c = capi.Context(*n, ord_=o)
    h = c.hs
    d = torch.from_numpy(st.copy()).cuda()
    worst = [0.0] * 5
    for _ in range(steps):
        d.copy_(torch.from_numpy(st))
        c.dimswitch = O.dimswitch
        O.time_step(st, dt)
        c.step(d, dt)
        got = d.cpu().numpy()
        for v in range(5):
            worst[v] = max(worst[v], rel_l2(got[v, h:-h, h:-h, h:-h], st[v, h:-h, h:-h, h:-h]))
    print("worst per-step relative L2 vs the glibc build:", ["%.2e" % e for e in worst])
    assert max(worst) <= 1e-12, worst


@pytest.mark.parametrize("case", CASES)
def test_splits_bit_exact_vs_crpow_oracle(case):
    """Every split (tendencies, halos, states) of steps 1-2 and the fused steps, from the
    reference's initial state: GPU == oracle(crpow) bit for bit."""
    g = np.load(os.path.join(GOLDEN, "case_%s.npz" % case))
    ord_, nx, ny, nz, bx, by, bz, ws, ww = [int(v) for v in g["config"]]
    O = Oracle(nx, ny, nz, bc=(bx, by, bz), weno_scalars=bool(ws), weno_winds=bool(ww),
               data=str(g["data"]), ord_=ord_, crpow=True)
    c = ctx_for(g)
    st = np.array(g["state0"])
    d = torch.from_numpy(st.copy()).cuda()
    fused = d.clone()
    tend = c.new_tend()
    dt = O.compute_dt(st, 0.8)
    assert c.cfl(d, 0.8) == dt
    for step in range(3):
        for spl in range(3):
            t_o = np.zeros(O.tend_shape)
            O.compute_tendencies(st, t_o, dt, spl)
            dd = (spl if step % 2 == 0 else 2 - spl)
            c.compute_tendencies(d, tend, dt, dd)
            torch.cuda.synchronize()
            assert np.array_equal(tend.cpu().numpy(), t_o), (step, spl)
            assert np.array_equal(tend.cpu().numpy().view(np.int64), t_o.view(np.int64)), (step, spl)
            O.apply(st, t_o, dt)
            c.apply_tendencies(d, tend, dt)
            assert np.array_equal(d.cpu().numpy(), st), (step, spl)
            assert np.array_equal(d.cpu().numpy().view(np.int64), st.view(np.int64)), (step, spl)
        c.step(fused, dt)
        assert np.array_equal(fused.cpu().numpy(), st), step
        assert np.array_equal(fused.cpu().numpy().view(np.int64), st.view(np.int64)), step


def test_fused_equals_unfused_bitwise():
    O, st = _bubble_case(5, 40, 36, 20, bc=(1, 0, 1))
    c = capi.Context(40, 36, 20, bc=(1, 0, 1))
    a = torch.from_numpy(st.copy()).cuda()
    b = a.clone()
    tend = c.new_tend()
    dt = c.cfl(a, 0.8)
    for d in (0, 1, 2, 2, 1, 0):
        c.split(a, dt, d)
        c.compute_tendencies(b, tend, dt, d)
        c.apply_tendencies(b, tend, dt)
    torch.cuda.synchronize()
    assert torch.equal(a, b)


def test_mass_conservation_full_size():
    """256x256x128, periodic x/y, walls in z: the flux-form update conserves total mass."""
    c = capi.Context(256, 256, 128)
    st = c.new_state()
    c.init_state(st, kind=capi.INIT_BUBBLE, noise_amp=0.01)
    dt = c.cfl(st, 0.8)
    h = c.hs
    m0 = st[0, h:-h, h:-h, h:-h].sum().item()
    for _ in range(3):
        c.step(st, dt)
    m1 = st[0, h:-h, h:-h, h:-h].sum().item()
    scale = st[0, h:-h, h:-h, h:-h].abs().sum().item()  # the density perturbation grows from 0
    assert torch.isfinite(st).all()
    assert scale > 0
    assert abs(m1 - m0) <= 1e-9 * scale, (m0, m1, scale)


def test_resting_atmosphere_stays_at_rest():
    """Hydrostatic balance: no perturbation -> tendencies at round-off level."""
    c = capi.Context(32, 32, 32)
    st = c.new_state()
    tend = c.new_tend()
    c.compute_tendencies(st, tend, 0.5, 2)
    torch.cuda.synchronize()
    assert tend.abs().max().item() < 1e-8
