"""Tracer transport in the FP32 precision form (awfl_split_tracers / awfl_step_tracers on an
FP32 context): the reference applies tracer tendencies in every precision
(Temporal_ader.h:67-69). The FP32 form reconstructs, fluxes and limits the tracers in FP32
next to its FP32 state split and keeps the tracers as FP64 arrays (division by the density
and the update in FP64).

Checks: against the FP64 path's tracer transport from the same initial data, the tracers
agree to the precision form's accuracy; the state advanced with tracers equals the FP32
state advanced without them (to FP32 rounding: the recording sweep is compiled apart); the
uniform tracer stays uniform; positive-definite tracers stay non-negative."""
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


def inner(x, hs):
    return x[..., hs:-hs, hs:-hs, hs:-hs]


@pytest.mark.parametrize("ord_,cfl,bc,n", [(5, 0.8, ("periodic", "periodic", "wall"), (64, 64, 32)),
                                           (5, 0.8, ("wall", "wall", "wall"), (64, 64, 32)),
                                           (9, 0.4, ("periodic", "periodic", "wall"), (64, 64, 32)),
                                           (5, 0.8, ("periodic", "periodic", "wall"), (64, 1, 32))])  # sim2d
def test_fp32_tracers_follow_fp64(ord_, cfl, bc, n):
    steps = 20
    kw = dict(ylen=20000.0 / 64) if n[1] == 1 else {}
    c64 = capi.Context(*n, ord_=ord_, bc=bc, **kw)
    c32 = capi.Context(*n, ord_=ord_, bc=bc, precision=capi.FP32, **kw)
    s64, s32 = c64.new_state(), c32.new_state()
    c64.init_state(s64, **BUBBLE)
    c32.init_state(s32, **BUBBLE)
    t64, t32 = c64.new_tracers(3), c32.new_tracers(3)
    c64.init_tracers(t64)
    c32.init_tracers(t32)
    assert torch.equal(t64, t32)
    plain = s32.clone()
    cp = capi.Context(*n, ord_=ord_, bc=bc, precision=capi.FP32, **kw)  # its own split order (dimSwitch)
    dt = c64.cfl(s64, cfl)
    for _ in range(steps):
        c64.step_tracers(s64, t64, dt)
        c32.step_tracers(s32, t32, dt)
        cp.step(plain, dt)
    torch.cuda.synchronize()
    hs = c64.hs
    errs = [rel_l2(inner(t32[t], hs), inner(t64[t], hs)) for t in range(3)]
    print("tracer rel L2 FP32 vs FP64", ord_, bc, errs)
    assert max(errs) <= 1e-6, errs  # measured 2e-10 .. 2e-9: FP32 fluxes, FP64 tracers
    # the state: equal to the FP32 split without tracers to FP32 rounding
    for v in range(5):
        a, b = inner(s32[v], hs), inner(plain[v], hs)
        assert (a - b).abs().max().item() <= 2e-6 * b.abs().max().item(), v
    # the uniform tracer (rho * 1) divided by the density stays 1; the limited ones stay
    # non-negative up to the rounding of the update (q*rho + dt*tend), as in the FP64 path
    q = c32.output_tracer_fields(s32, t32)
    assert (q[0] - 1).abs().max().item() <= 1e-5
    for t in (1, 2):
        assert inner(t32[t], hs).min().item() >= -1e-12 * inner(t32[t], hs).max().item()
        assert inner(t64[t], hs).min().item() >= -1e-12 * inner(t64[t], hs).max().item()


def test_fp32_split_tracers_one_direction_each():
    """Each split on its own, both halo conventions: the directions' tracer halos hold
    tracer/density as in the FP64 path."""
    n = (24, 20, 16)
    c64 = capi.Context(*n)
    c32 = capi.Context(*n, precision=capi.FP32)
    for d in range(3):
        s64, s32 = c64.new_state(), c32.new_state()
        c64.init_state(s64, **BUBBLE)
        c32.init_state(s32, **BUBBLE)
        t64, t32 = c64.new_tracers(3), c32.new_tracers(3)
        c64.init_tracers(t64)
        c32.init_tracers(t32)
        dt = c64.cfl(s64, 0.8)
        c64.split_tracers(s64, t64, dt, d)
        c32.split_tracers(s32, t32, dt, d)
        torch.cuda.synchronize()
        # whole arrays, halos included (relative to each tracer's range)
        for t in range(3):
            assert (t32[t] - t64[t]).abs().max().item() <= 1e-5 * t64[t].abs().max().item(), (d, t)
