"""Batching form: an ensemble of members with uneven grid sizes advanced by one
persistent kernel per split stage (CUDA graph), with autotuned tile shapes. FP64 members
must be bit-identical to stepping that member alone (awfl_step); FP32 members agree to
FP32 rounding (the FP32 form is compiled with multiply-add contraction, which the
compiler may place differently in the persistent kernel)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from awflcloud_b200 import capi  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def member_configs(prec, ord_):
    return [
        dict(nx=32, ny=32, nz=32, precision=prec, ord_=ord_),
        dict(nx=48, ny=40, nz=24, precision=prec, ord_=ord_),
        dict(nx=64, ny=64, nz=32, precision=prec, ord_=ord_),
        dict(nx=20, ny=36, nz=16, precision=prec, ord_=ord_, bc=("wall", "wall", "wall")),
        dict(nx=64, ny=1, nz=32, ylen=20000.0 / 64, precision=prec, ord_=ord_),  # sim2d: no y stage
        dict(nx=24, ny=24, nz=40, precision=prec, ord_=ord_, bc=("periodic", "wall", "wall")),
        # row pitch nx + 2hs not a multiple of 4 floats: an FP32 member TMA cannot address,
        # staged by cp.async inside the same persistent kernels as the TMA members
        dict(nx=30, ny=28, nz=20, precision=prec, ord_=ord_),
    ]


def init_member(ctx, i):
    s = ctx.new_state()
    rng = np.random.default_rng(100 + i)
    ctx.init_state(s, kind=capi.INIT_BUBBLE, x0=float(rng.uniform(5e3, 15e3)), y0=float(rng.uniform(5e3, 15e3)),
                   z0=float(rng.uniform(1.5e3, 3e3)), xrad=2000.0, yrad=2000.0, zrad=2000.0,
                   amp=float(rng.uniform(1, 4)), noise_amp=0.01, noise_seed=7 + i)
    return s


def make(prec, ord_):
    cfgs = member_configs(prec, ord_)
    E = capi.Ensemble(cfgs)
    states, dts = [], []
    for i, m in enumerate(E.members):
        s = init_member(m, i)
        dt = m.cfl(s, 0.8 if ord_ == 5 else 0.4)
        E.bind(i, s, dt)
        states.append(s)
        dts.append(dt)
    return E, cfgs, states, dts


def interior(ctx, a):
    h = ctx.hs
    return a[..., h:-h, h:-h, h:-h] if ctx.ny > 1 else a[..., h:-h, :, h:-h]


def mismatch(ctx, a, b):
    """0 when the interiors agree: bit for bit for FP64; for FP32 the largest per-variable
    relative L2 difference of the value plane if it exceeds 1e-5 (a few FP32 roundings
    amplified over a handful of steps), else 0."""
    x, y = interior(ctx, a), interior(ctx, b)
    if ctx.precision == capi.FP64:
        return 0.0 if torch.equal(x, y) else float("inf")
    worst = 0.0
    for v in range(5):
        d = torch.linalg.vector_norm((x[v] - y[v]).double()).item()
        n = torch.linalg.vector_norm(y[v].double()).item()
        worst = max(worst, d / n if n > 0 else d)
    return worst if worst > 1e-5 else 0.0


def alone(cfgs, states0, dts, nsteps):
    out = []
    for kw, s0, dt in zip(cfgs, states0, dts):
        kw = dict(kw)
        nx, ny, nz = kw.pop("nx"), kw.pop("ny"), kw.pop("nz")
        c = capi.Context(nx, ny, nz, **kw)
        s = s0.clone()
        for _ in range(nsteps):
            c.step(s, dt)
        out.append(s)
    return out


@pytest.mark.parametrize("prec,ord_", [(capi.FP32, 5), (capi.FP64, 5), (capi.FP32, 9), (capi.FP64, 9)])
def test_ensemble_members_bit_identical_to_single_steps(prec, ord_):
    E, cfgs, states, dts = make(prec, ord_)
    s0 = [s.clone() for s in states]
    E.step(5)  # two graph replays + one direct step
    ref = alone(cfgs, s0, dts, 5)
    torch.cuda.synchronize()
    for i, (a, b) in enumerate(zip(states, ref)):
        assert mismatch(E.members[i], a, b) == 0.0, (i, mismatch(E.members[i], a, b))
    assert E.dimswitch == 0


def test_autotuner_picks_a_candidate_and_keeps_results_exact():
    E, cfgs, states, dts = make(capi.FP32, 5)
    s0 = [s.clone() for s in states]
    table = E.tune(reps=2)
    torch.cuda.synchronize()
    for s, t in zip(states, s0):  # tuning runs on scratch copies
        assert torch.equal(s, t)
    for d in range(3):
        rows = table[d]
        assert len(rows) >= 2 and all(ms > 0 for _, _, ms in rows)
        idx, C, W, grid = E.shape(d)
        assert (C, W) == rows[idx][:2]
        assert rows[idx][2] == min(ms for _, _, ms in rows)
        assert grid >= 1
    E.step(4)
    E.step(1)
    ref = alone(cfgs, s0, dts, 5)
    torch.cuda.synchronize()
    for i, (a, b) in enumerate(zip(states, ref)):
        assert mismatch(E.members[i], a, b) == 0.0, (i, mismatch(E.members[i], a, b))


@pytest.mark.parametrize("d,shape", [(0, 2), (1, 1), (2, 3)])
def test_every_tile_shape_gives_the_same_result(d, shape):
    E, cfgs, states, dts = make(capi.FP64, 5)
    s0 = [s.clone() for s in states]
    E.set_shape(d, shape)
    E.step(2)
    ref = alone(cfgs, s0, dts, 2)
    torch.cuda.synchronize()
    for i, (a, b) in enumerate(zip(states, ref)):
        assert mismatch(E.members[i], a, b) == 0.0, (i, mismatch(E.members[i], a, b))


def test_ensemble_rejects_bad_use():
    with pytest.raises(capi.AwflError):
        capi.Ensemble([dict(nx=16, ny=16, nz=16, ord_=5), dict(nx=16, ny=16, nz=16, ord_=9)])
    E = capi.Ensemble([dict(nx=16, ny=16, nz=16), dict(nx=24, ny=16, nz=16)])
    s = E.members[0].new_state()
    E.bind(0, s, 1.0)
    with pytest.raises(capi.AwflError):  # member 1 not bound
        E.step(1)
    with pytest.raises(capi.AwflError):
        E.set_shape(0, 99)


@pytest.mark.parametrize("world", [2, 3])
def test_rank_shares_equal_single_steps(world):
    """The members split over ranks (awflcloud_b200.members): each share is its own
    ensemble -- here every rank's share held in this one process on one GPU, none waiting
    on another -- and every member still equals stepping it alone, bit for bit (FP64)."""
    from awflcloud_b200.members import RankEnsemble
    cfgs = member_configs(capi.FP64, 5)
    parts = [RankEnsemble(cfgs, r, world) for r in range(world)]
    assert sorted(i for p in parts for i in p.share) == list(range(len(cfgs)))
    states, dts = [None] * len(cfgs), [None] * len(cfgs)
    for p in parts:
        for i in p.share:
            m = p.member(i)
            states[i] = init_member(m, i)
            dts[i] = m.cfl(states[i], 0.8)
            p.bind(i, states[i], dts[i])
    s0 = [s.clone() for s in states]
    for p in parts:
        p.step(3)
    ref = alone(cfgs, s0, dts, 3)
    torch.cuda.synchronize()
    for p in parts:
        for i in p.share:
            assert mismatch(p.member(i), states[i], ref[i]) == 0.0, i
        p.close()
