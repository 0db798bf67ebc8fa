"""Tracer transport on the device (awfl_step_tracers / awfl_split_tracers; the reference's
tracer code, compiled out there by NO_TRACERS, built in): bit for bit against the
reference's own tracer code (tests/golden/tracer_transport.npz, made by the reference built
with NO_TRACERS blanked), and against the oracle's restatement of the same code, tracers
and their halos, for several configurations.

FP64 with no contracted multiply-add on both sides and the correctly rounded pow (the
oracle's crpow build) in the state's reconstruction, so equality is exact. The state
advanced with tracers is bit-identical to the state advanced without them."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from awflcloud_b200 import capi  # noqa: E402
from oracle.pyoracle import Oracle  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


BCN = {0: "periodic", 1: "wall"}
# (ord, nx, ny, nz, bc, weno_scalars, weno_winds, cfl, steps)
CASES = [
    (5, 24, 20, 12, (0, 0, 1), True, True, 0.8, 4),
    (5, 20, 16, 12, (1, 1, 1), True, True, 0.8, 3),
    (5, 16, 12, 10, (0, 0, 0), False, True, 0.8, 3),
    (5, 24, 1, 16, (0, 0, 1), True, True, 0.8, 3),
    (9, 20, 18, 16, (0, 1, 1), True, False, 0.4, 2),
    (5, 1, 12, 8, (1, 0, 1), True, True, 0.8, 2),   # a wall direction of one cell
]


@pytest.mark.parametrize("case", CASES)
def test_step_tracers_bit_exact(case):
    o, nx, ny, nz, bc, ws, ww, cfl, nsteps = case
    O = Oracle(nx, ny, nz, bc=bc, weno_scalars=ws, weno_winds=ww, ord_=o, crpow=True)
    st = O.new_state()
    O.init_state(st)
    O.set_bubble(st, 1, 10000, 10000 if ny > 1 else 10000, 2000, 3000, 3000, 3000, 3.0, 1.0)
    O.add_theta_noise(st, 11, 0.01)
    tr = O.new_tracers(4)
    O.init_tracers(tr)
    h = O.hs
    tr[3][h:h + nz, h:h + ny, h:h + nx] = -0.5 * tr[2][h:h + nz, h:h + ny, h:h + nx]
    pos = [1, 1, 1, 0]
    dt = O.compute_dt(st, cfl)

    c = capi.Context(nx, ny, nz, bc=tuple(BCN[b] for b in bc), weno_scalars=ws, weno_winds=ww, ord_=o)
    dst = torch.from_numpy(st).cuda()
    dtr = torch.from_numpy(tr).cuda()
    dst_plain = dst.clone()
    for _ in range(nsteps):
        O.time_step_tracers(st, tr, dt, pos=pos)
        c.step_tracers(dst, dtr, dt, pos=pos)
    c2 = capi.Context(nx, ny, nz, bc=tuple(BCN[b] for b in bc), weno_scalars=ws, weno_winds=ww, ord_=o)
    for _ in range(nsteps):
        c2.step(dst_plain, dt)
    got_tr = dtr.cpu().numpy()
    assert np.array_equal(dst.cpu().numpy(), st)
    assert np.array_equal(dst.cpu().numpy(), dst_plain.cpu().numpy())
    assert np.array_equal(dst.cpu().numpy().view(np.int64), st.view(np.int64))
    for t in range(4):
        assert np.array_equal(got_tr[t], tr[t]), (t, np.abs(got_tr[t] - tr[t]).max())
        # bit patterns too: the signs of zero (tracers absent from most cells) included
        assert np.array_equal(got_tr[t].view(np.int64), tr[t].view(np.int64)), t
    # the theta and block tracers have moved (the block is empty on a grid of fewer than
    # 3 cells in x: its x range is [4nx/10, 6nx/10))
    O0 = Oracle(nx, ny, nz, bc=bc, ord_=o)
    t0 = O0.new_tracers(3)
    O0.init_tracers(t0)
    for t in ((1, 2) if nx >= 3 else (1,)):
        assert np.abs(got_tr[t] - t0[t])[h:h + nz, h:h + ny, h:h + nx].max() > 1e-6, t


def _chained_case(nx, ny, nz, bc, d, seed):
    """A state whose velocity along d changes sign cell by cell at random (many cells
    empty through both faces) and positive tracers with nearly empty cells: there the
    limiter scales a face that the next face reads, the places where the reference's
    serial face order decides the result."""
    O = Oracle(nx, ny, nz, bc=bc, weno_scalars=True, weno_winds=True, crpow=True)
    st = O.new_state()
    O.init_state(st)
    rng = np.random.default_rng(seed)
    h = O.hs
    inner = (slice(h, h + nz), slice(h, h + ny), slice(h, h + nx))
    sh = (nz, ny, nx)
    st[(1 + d,) + inner] = rng.choice([-1., 1.], size=sh) * rng.uniform(10, 40, size=sh)
    tr = O.new_tracers(3)
    for t in range(3):
        tr[(t,) + inner] = np.where(rng.uniform(size=sh) > 0.4, rng.uniform(0.5, 1.5, sh), rng.uniform(0, 1e-2, sh))
    return O, st, tr


@pytest.mark.parametrize("d", [0, 1, 2])
@pytest.mark.parametrize("bc", [(0, 0, 1), (1, 1, 1)])
def test_limiter_serial_chains(d, bc):
    """The device limits every face at once and redoes in face order only the lines where
    a scaled face feeds another: on a case with hundreds of such faces (counted by the
    oracle) one split matches the oracle's serial limiter bit for bit."""
    nx, ny, nz = 24, 20, 16
    O, st, tr = _chained_case(nx, ny, nz, bc, d, 7 + d)
    pos = [1, 1, 0]
    dt = O.compute_dt(st, 0.8)
    c = capi.Context(nx, ny, nz, bc=tuple(BCN[b] for b in bc), weno_scalars=True, weno_winds=True, ord_=5)
    dst = torch.from_numpy(st).cuda()
    dtr = torch.from_numpy(tr).cuda()
    O.split_tracers(st, tr, dt, d, pos=pos)
    assert O.limiter_chained_faces() > 100
    c.split_tracers(dst, dtr, dt, d, pos=pos)
    got = dtr.cpu().numpy()
    for t in range(3):
        assert np.array_equal(got[t], tr[t]), (t, np.abs(got[t] - tr[t]).max())
    assert np.array_equal(dst.cpu().numpy(), st)


def test_split_tracers_rejects_bad_args():
    c64 = capi.Context(16, 12, 10)
    st64 = c64.new_state()
    tr = c64.new_tracers(2)
    with pytest.raises(ValueError):
        c64.step_tracers(st64, tr, 0.5, pos=[1])
    with pytest.raises(ValueError):
        c64.step_tracers(st64, tr.float(), 0.5)  # tracers are FP64 arrays in every precision
    with pytest.raises(capi.AwflError):
        c64.split_tracers(st64, tr, 0.5, 3)


def test_split_tracers_equal_reference_tracer_code(golden_dir):
    """Every split of the reference-made cases that use the correctly rounded pow: tracers
    (halos included) after each split and the final state, bit for bit."""
    import os
    z = np.load(os.path.join(golden_dir, "tracer_transport.npz"))
    names = sorted({k[:-len("_config")] for k in z.files if k.endswith("_config")})
    done = 0
    for name in names:
        o, nx, ny, nz, bcx, bcy, bcz, crpow = (int(v) for v in z[name + "_config"])
        if not crpow:
            continue  # glibc's pow: pinned through the oracle on the CPU
        pos = [int(p) for p in z[name + "_pos"]]
        c = capi.Context(nx, ny, nz, bc=(BCN[bcx], BCN[bcy], BCN[bcz]), ord_=o)
        dst = torch.from_numpy(z[name + "_state0"].copy()).cuda()
        dtr = torch.from_numpy(z[name + "_tracers0"].copy()).cuda()
        dt = float(z[name + "_dt"])
        for s, d in enumerate(z[name + "_splits"]):
            c.split_tracers(dst, dtr, dt, int(d), pos=pos)
            got = dtr.cpu().numpy()
            want = z[name + "_tracers%d" % (s + 1)]
            assert np.array_equal(got, want), (name, s, int(d), np.abs(got - want).max())
            assert np.array_equal(got.view(np.int64), np.ascontiguousarray(want).view(np.int64)), (name, s, int(d))
        assert np.array_equal(dst.cpu().numpy(), z[name + "_state_end"]), name
        assert np.array_equal(dst.cpu().numpy().view(np.int64),
                              np.ascontiguousarray(z[name + "_state_end"]).view(np.int64)), name
        done += 1
    assert done >= 7
