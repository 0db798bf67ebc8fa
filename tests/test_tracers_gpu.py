"""Tracer initial data and tracer output fields on the device (Spatial::initTracers,
Spatial_euler3d_cons_expl_cart_fv_Agrid.h:505-560; Spatial::output's tracer_<name> fields,
:1778-1783). The reference runs both although its tracer transport is compiled out
(NO_TRACERS, :10), and its driver registers three tracers (driver.cpp:27-29).

The device evaluates the hydrostatic density at the quadrature points with the correctly
rounded pow; the reference (and the oracle, which equals it bit for bit:
tests/test_oracle_golden.py) with glibc's, which misrounds about 0.08% of calls by one ulp.
Where that happens the tracer's cell average differs in its last bit (e.g. 32x24x16, cell
(k, j, i) = (6, 11, 16) of the theta tracer: glibc's pow(exner, cp/rd) at the second
quadrature level is one ulp above the correctly rounded value, checked with 300-bit mpmath).
So: bit-identical in all but a few cells, and within 1e-15 relative everywhere."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from awflcloud_b200 import capi  # noqa: E402
from oracle.pyoracle import Oracle  # noqa: E402

netcdf = pytest.importorskip("scipy.io").netcdf_file


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


GRIDS = [(20, 20, 10, ("periodic", "periodic", "wall"), 5),
         (30, 1, 20, ("periodic", "periodic", "wall"), 5),
         (20, 10, 10, ("wall", "wall", "wall"), 9),
         (64, 64, 32, ("periodic", "periodic", "wall"), 5)]


@pytest.mark.parametrize("grid", GRIDS)
def test_init_tracers_bit_exact(grid):
    nx, ny, nz, bc, o = grid
    c = capi.Context(nx, ny, nz, bc=bc, ord_=o)
    tr = c.new_tracers(4)
    tr.fill_(-7.0)  # halos must stay as they were
    c.init_tracers(tr)
    got = tr.cpu().numpy()
    O = Oracle(nx, ny, nz, bc=tuple(0 if b == "periodic" else 1 for b in bc), ord_=o)
    ref = O.new_tracers(4)
    ref[:] = -7.0
    O.init_tracers(ref)
    np.testing.assert_allclose(got, ref, rtol=1e-15, atol=0)
    assert np.count_nonzero(got != ref) <= max(1, got.size // 1000)
    assert np.array_equal(got[3], ref[3]) and np.array_equal(got[0][:2], ref[0][:2])  # zero tracer, halos


def test_init_tracers_last_bit_is_the_correctly_rounded_one():
    """The one differing cell of the 32x24x16 grid: the device value is the per-operation
    IEEE evaluation with a correctly rounded pow (written here with 300-bit mpmath)."""
    mp = pytest.importorskip("mpmath")
    import math
    mp.mp.prec = 300
    c = capi.Context(32, 24, 16, bc=("periodic", "wall", "wall"))
    tr = c.new_tracers(2)
    c.init_tracers(tr)
    T = c.tables()
    pts, wts = T["gll_pts_ord"], T["gll_wts_ord"]
    C0, GAMMA = 27.5629410929725921310572974482, 1.40027894002789400278940027894
    crpow = lambda x, y: float(mp.power(mp.mpf(x), mp.mpf(y)))  # noqa: E731
    dx, dy, dz = 20000 / 32, 20000 / 24, 10000 / 16
    k, j, i = 6, 11, 16
    acc = 0.0
    for kk in range(5):
        for jj in range(5):
            for ii in range(5):
                z = (k + 0.5) * dz + pts[kk] * dz
                y = (j + 0.5) * dy + pts[jj] * dy
                x = (i + 0.5) * dx + pts[ii] * dx
                wt = wts[kk] * wts[jj] * wts[ii]
                p = crpow(1. - 9.81 * z / (1004. * 300.), 1004. / 287.) * 1.0e5
                rh = crpow(p / C0, 1. / GAMMA) / 300.
                xn, yn, zn = (x - 10000.) / 2000., (y - 10000.) / 2000., (z - 2000.) / 2000.
                tv = 2. * max(1. - math.sqrt(xn * xn + yn * yn + zn * zn), 0.)
                acc += rh * tv * wt
    h = c.hs
    assert float(tr[1, h + k, h + j, h + i]) == acc


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
def test_tracer_output_fields_and_file(tmp_path, prec):
    c = capi.Context(24, 16, 12, precision=prec)
    st = c.new_state()
    c.init_state(st, kind=capi.INIT_BUBBLE, noise_amp=0.01)
    tr = c.new_tracers(3)
    c.init_tracers(tr)
    dt = c.cfl(st, 0.8)
    c.step(st, dt)
    f = c.output_tracer_fields(st, tr).cpu().numpy()
    h = c.hs
    s = st.cpu().double().numpy()
    if prec == capi.FP32:
        s = s[:5] - s[5:]
    r = s[0, h:h + c.nz, h:h + c.ny, h:h + c.nx] + c.background()["hyDensCells"][h:h + c.nz, None, None]
    t = tr.cpu().numpy()[:, h:h + c.nz, h:h + c.ny, h:h + c.nx]
    np.testing.assert_array_equal(f, t / r)
    names = ["uniform", "theta", "block"]
    path = str(tmp_path / "tr.nc")
    c.write_netcdf_tracers(path, st, tr, names, 0.0)
    c.write_netcdf_tracers(path, st, tr, names, dt)
    diag = c.output_fields(st).cpu().numpy()
    with netcdf(path, "r", mmap=False) as nc:
        for i, n in enumerate(names):
            np.testing.assert_array_equal(nc.variables["tracer_" + n][1], f[i])
        np.testing.assert_array_equal(nc.variables["u"][1], diag[1])
        # uniform tracer / density ~ rho_h / (rho_h + rho'): close to 1
        assert abs(float(nc.variables["tracer_uniform"][0].mean()) - 1.0) < 1e-3
