"""The CPU oracle (oracle/awfl_oracle.c) against the reference's own outputs.

The fixtures in tests/golden/ were produced by the reference's unmodified headers
(tests/golden/make_golden.py). The oracle restates the same arithmetic in the same
order, so the comparison is bit-exact (np.array_equal), split by split.
"""
import glob
import os

import numpy as np
import pytest

from oracle.pyoracle import Oracle, build

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(os.path.basename(p)[5:-4] for p in glob.glob(os.path.join(GOLDEN, "case_*.npz")))
BC = {0: 0, 1: 1}


@pytest.fixture(scope="module", autouse=True)
def _built():
    build()


def _oracle_for(g):
    ord_, nx, ny, nz, bx, by, bz, ws, ww = [int(v) for v in g["config"]]
    return Oracle(nx, ny, nz, bc=(bx, by, bz), weno_scalars=bool(ws), weno_winds=bool(ww),
                  data=str(g["data"]), ord_=ord_)


def _initial_state(O, g):
    st = O.new_state()
    O.init_state(st)
    if "bubble" in g:
        b = g["bubble"]
        O.set_bubble(st, int(b[0]), *[float(v) for v in b[1:]])
    if "noise" in g:
        seed, amp = g["noise"]
        O.add_theta_noise(st, int(seed), float(amp))
    return st


def test_cases_present():
    assert len(CASES) >= 10


@pytest.mark.parametrize("case", CASES)
def test_background_and_init(case):
    g = np.load(os.path.join(GOLDEN, "case_%s.npz" % case))
    O = _oracle_for(g)
    bg = O.background()
    for k, v in bg.items():
        assert np.array_equal(v, g[k]), k
    st = _initial_state(O, g)
    assert np.array_equal(st, g["state0"])
    assert O.compute_dt(st, 0.8) == float(g["dt"])


@pytest.mark.parametrize("case", CASES)
def test_splits_bit_exact(case):
    """Every split's tendencies and the state after it, steps 1-2 (X,Y,Z then Z,Y,X)."""
    g = np.load(os.path.join(GOLDEN, "case_%s.npz" % case))
    O = _oracle_for(g)
    st = np.array(g["state0"])
    dt = float(g["dt"])
    nsteps = len([k for k in g.files if k.startswith("state_s") and "_p" not in k])
    for step in range(nsteps):
        if step < 2:
            for spl in range(3):
                tend = np.zeros(O.tend_shape)
                O.compute_tendencies(st, tend, dt, spl)
                assert np.array_equal(tend, g["tend_s%d_p%d" % (step, spl)]), (step, spl)
                O.apply(st, tend, dt)
                if step == 0:
                    assert np.array_equal(st, g["state_s0_p%d" % spl]), spl
        else:
            O.time_step(st, dt)
        assert np.array_equal(st, g["state_s%d" % step]), step


@pytest.mark.parametrize("ord_", [5, 9])
def test_weno_and_tv_probes(ord_):
    p = np.load(os.path.join(GOLDEN, "probes_o%d.npz" % ord_))
    O = Oracle(10, 8, 6, ord_=ord_)
    for a, v in zip(p["tv_lo_in"], p["tv_lo"]):
        assert O.coefs_to_tv(a) == v
    for a, v in zip(p["tv_hi_in"], p["tv_hi"]):
        assert O.coefs_to_tv(a) == v
    for s, v in zip(p["weno_in"], p["weno"]):
        assert np.array_equal(O.weno_coefs(s), v)


@pytest.mark.parametrize("ord_", [5, 9])
def test_derived_tables(ord_):
    """sten_to_gll, derivMatrix, idl, sigma as built at init (Spatial...h:274-315)."""
    t = np.load(os.path.join(GOLDEN, "tables_o%d.npz" % ord_))
    O = Oracle(10, 8, 6, ord_=ord_)
    mine = O.tables()
    assert np.array_equal(mine["sten_to_gll"], t["sten_to_gll"])
    assert np.array_equal(mine["idl"], t["idl"])
    assert np.array_equal(mine["sigma"], t["sigma"])
    # derivMatrix: exact-math tables vs the reference's Sage literals, which carry
    # 129-bit round-off (gll_to_coefs<5>(2,1) = -2.35e-38 where the exact value is 0).
    assert np.max(np.abs(mine["deriv"] - t["deriv"])) <= 1e-37


@pytest.mark.skipif(not __import__("oracle.pyoracle", fromlist=["x"]).ref_available(5, True),
                    reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("ord_,bc,ws", [(5, (0, 0, 1), True), (5, (1, 1, 0), False), (9, (0, 0, 1), True)])
def test_crpow_oracle_equals_crpow_reference(ord_, bc, ws):
    """The oracle variant with a correctly rounded pow/exp is bit-identical to the
    reference's own code built with the same pow/exp (oracle/_ref/*_crpow.so)."""
    from oracle.pyoracle import RefHarness
    n = (12, 10, 8)
    R = RefHarness(*n, bc=bc, weno_scalars=ws, ord_=ord_, crpow=True)
    O = Oracle(*n, bc=bc, weno_scalars=ws, ord_=ord_, crpow=True)
    R.init_state()
    R.set_bubble(1, 10000.0, 10000.0, 2000.0, 2500.0, 2500.0, 2500.0, 3.0, 1.0)
    R.add_theta_noise(7, 0.01)
    st = O.new_state()
    O.init_state(st)
    O.set_bubble(st, 1, 10000.0, 10000.0, 2000.0, 2500.0, 2500.0, 2500.0, 3.0, 1.0)
    O.add_theta_noise(st, 7, 0.01)
    assert np.array_equal(st, R.get_state())
    dt = R.compute_dt(0.4)
    assert O.compute_dt(st, 0.4) == dt
    for _ in range(4):
        R.time_step(dt)
        O.time_step(st, dt)
    assert np.array_equal(st, R.get_state())


def test_glibc_pow_rounding_spread():
    """The reference's sensitivity to last-bit pow rounding: glibc pow vs a correctly
    rounded pow, same code, 32x32x16 bubble + noise, 20 steps. Documents the size of the
    spread the FP64 GPU parity tolerance against the glibc build is based on."""
    res = []
    for cr in (False, True):
        O = Oracle(32, 32, 16, crpow=cr)
        st = O.new_state()
        O.init_state(st)
        O.set_bubble(st, 1, 10000.0, 10000.0, 2000.0, 2000.0, 2000.0, 2000.0, 3.0, 1.0)
        O.add_theta_noise(st, 20261203, 0.01)
        dt = O.compute_dt(st, 0.8)
        for _ in range(20):
            O.time_step(st, dt)
        res.append(st[:, 2:-2, 2:-2, 2:-2])
    spread = [np.linalg.norm(res[0][v] - res[1][v]) / np.linalg.norm(res[1][v]) for v in range(5)]
    assert max(spread) > 0          # glibc's pow is not correctly rounded everywhere
    assert max(spread) < 5e-12      # ... but only in the last bit


def test_init_tracers_bit_exact():
    """initTracers (Spatial:505-560) of the driver's three tracers plus a fourth (zero)."""
    g = np.load(os.path.join(GOLDEN, "tracers_init.npz"))
    names = sorted({k.rsplit("_", 1)[0] for k in g.files})
    assert len(names) == 3
    for name in names:
        ord_, nx, ny, nz, bx, by, bz = [int(v) for v in g[name + "_config"]]
        O = Oracle(nx, ny, nz, bc=(bx, by, bz), data=str(g[name + "_data"]), ord_=ord_)
        tr = O.new_tracers(4)
        O.init_tracers(tr)
        ref = g[name + "_tracers"]
        assert np.array_equal(tr, ref), name
        h = O.hs
        assert np.all(ref[3] == 0)
        assert np.all(ref[0, h:h + nz, h:h + ny, h:h + nx] > 0)  # rho_h-weighted uniform tracer
