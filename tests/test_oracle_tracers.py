"""The oracle's restatement of the reference's tracer transport (its code under
#ifndef NO_TRACERS, Spatial_euler3d_cons_expl_cart_fv_Agrid.h:624-955 and the y/z
equivalents). The reference defines NO_TRACERS unconditionally (:10), so no output of the
reference pins this part; these are the properties the scheme has instead: the state is
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
