"""The oracle's restatement of the reference's tracer transport (its code under
#ifndef NO_TRACERS, Spatial_euler3d_cons_expl_cart_fv_Agrid.h:624-955 and the y/z
equivalents), which the reference compiles out (NO_TRACERS, :10).

Pinned to the reference's own tracer code: tests/golden/tracer_transport.npz comes from
the reference built with that one line blanked (oracle/Makefile, serially), and the
restatement must reproduce every split of it bit for bit -- x, y and z splits, periodic
and wall boundaries, ord 5 and 9, limited (positive-definite) tracers in x and z, glibc's
and a correctly rounded pow. (The reference's y limiter reads faces of another direction
for v < 0, :1285-1286; the y splits of the fixtures carry no positive-definite tracer.)

The properties the scheme has are checked as well: the state is
untouched by the tracers, a uniform mixing ratio stays uniform, tracer mass is conserved
where the mass flux through the boundary is zero (periodic x/y; a z wall, where the
reconstruction zeroes w -- an x or y wall copies the edge state without zeroing the normal
momentum, Spatial:826-835, so mass crosses it, for the state too), and the limiter keeps
positive tracers non-negative up to round-off-sized undershoots (the flux direction comes
from the Riemann velocity, the limiter's upwind cell from the averaged momentum).""" 
import numpy as np
import pytest

from oracle.pyoracle import Oracle, build


@pytest.fixture(scope="module", autouse=True)
def _built():
    build()


@pytest.mark.parametrize("ord_,bc,ws", [(5, (0, 0, 1), True), (5, (1, 1, 1), True), (5, (0, 0, 0), False),
                                        (9, (0, 1, 1), True)])
def test_tracer_transport_properties(ord_, bc, ws):
    nx, ny, nz = (16, 12, 10) if ord_ == 5 else (20, 18, 16)
    O = Oracle(nx, ny, nz, bc=bc, weno_scalars=ws, ord_=ord_)
    O2 = Oracle(nx, ny, nz, bc=bc, weno_scalars=ws, ord_=ord_)
    st = O.new_state()
    O.init_state(st)
    O.set_bubble(st, 1, 10000, 10000, 2000, 3000, 3000, 3000, 3.0, 1.0)
    O.add_theta_noise(st, 7, 0.01)
    st2 = st.copy()
    tr = O.new_tracers(4)
    O.init_tracers(tr)
    h = O.hs
    I = (slice(None), slice(h, h + nz), slice(h, h + ny), slice(h, h + nx))
    tr[3][I[1:]] = -tr[2][I[1:]]  # a negative, not positive-definite tracer
    m0 = tr[I].sum(axis=(1, 2, 3))
    dt = O.compute_dt(st, 0.8 if ord_ == 5 else 0.4)
    for _ in range(6):
        O.time_step_tracers(st, tr, dt, pos=[1, 1, 1, 0])
        O2.time_step(st2, dt)
    assert np.array_equal(st, st2)
    r = st[0][I[1:]] + O.background()["hyDensCells"][h:h + nz, None, None]
    assert np.abs(tr[0][I[1:]] / r - 1).max() < 1e-13  # free-stream: uniform mixing ratio
    m1 = tr[I].sum(axis=(1, 2, 3))
    if bc[0] == 0 and bc[1] == 0:
        np.testing.assert_allclose(m1, m0, rtol=1e-13, atol=1e-13 * np.abs(m0).max())
    for t in (1, 2):
        assert tr[t][I[1:]].min() > -1e-6 * tr[t][I[1:]].max()
    assert np.abs(tr[1][I[1:]] - O.new_tracers(4)[1][I[1:]]).max() > 0  # it moved


def _transport_cases(golden_dir):
    import os
    z = np.load(os.path.join(golden_dir, "tracer_transport.npz"))
    names = sorted({k[:-len("_config")] for k in z.files if k.endswith("_config")})
    return z, names


def test_restatement_equals_reference_tracer_transport(golden_dir):
    z, names = _transport_cases(golden_dir)
    assert len(names) >= 8
    for name in names:
        ord_, nx, ny, nz, bcx, bcy, bcz, crpow = (int(v) for v in z[name + "_config"])
        pos = [int(p) for p in z[name + "_pos"]]
        O = Oracle(nx, ny, nz, bc=(bcx, bcy, bcz), ord_=ord_, crpow=bool(crpow))
        st = z[name + "_state0"].copy()
        tr = z[name + "_tracers0"].copy()
        dt = float(z[name + "_dt"])
        for s, d in enumerate(z[name + "_splits"]):
            O.split_tracers(st, tr, dt, int(d), pos=pos)
            want = z[name + "_tracers%d" % (s + 1)]
            assert np.array_equal(tr, want), (name, s, int(d), np.abs(tr - want).max())
        assert np.array_equal(st, z[name + "_state_end"]), name
