"""The reference's own driver.cpp, compiled unchanged against the drop-in operator headers
(awflcloud_b200/dropin/) and libawfl.so, run end to end from a YAML input on the GPU.

The binary is built where the reference sources are present (build()); it then travels
with the tree. The driver's final output (outFile *.bin: raw FP64 state) is compared with
the CPU oracle advanced through the same sequence of time steps (the driver clips the last
step to simTime, driver.cpp:45-48).
"""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from oracle.pyoracle import Oracle  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "awflcloud_b200", "dropin", "bin", "driver_o5")


def _yaml(path, out, sim_time, extra="", out_freq=None):
    with open(path, "w") as f:
        f.write("""---
simTime  : %r
nx       : 32
ny       : 24
nz       : 16
xlen     : 20000
ylen     : 20000
zlen     : 10000
bc_x   : periodic
bc_y   : wall
bc_z   : wall
weno_scalars : true
weno_winds   : true
initData : thermal
outFile  : %s
outFreq  : %r
perturb: false
%s""" % (sim_time, out, sim_time if out_freq is None else out_freq, extra))


def _oracle_run(sim_time):
    O = Oracle(32, 24, 16, bc=(0, 1, 1), crpow=True)
    st = O.new_state()
    O.init_state(st)
    dt0 = O.compute_dt(st, 0.8)
    etime, n = 0.0, 0
    while etime < sim_time:  # driver.cpp:45-48
        dt = dt0
        if etime + dt > sim_time:
            dt = sim_time - etime
        O.time_step(st, dt)
        etime += dt
        n += 1
    return st, dt0, n


@pytest.fixture(scope="module", autouse=True)
def _needs_binary():
    if not os.path.exists(BIN):
        pytest.skip("drop-in driver not built (needs the reference sources at build time)")


def _run(tmp_path, extra=""):
    O = Oracle(32, 24, 16, bc=(0, 1, 1), crpow=True)
    st = O.new_state()
    O.init_state(st)
    sim_time = 3.5 * O.compute_dt(st, 0.8)
    inp, out = str(tmp_path / "in.yaml"), str(tmp_path / "state.bin")
    _yaml(inp, out, sim_time, extra)
    p = subprocess.run([BIN, inp], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    assert "Walltime:" in p.stdout
    got = np.fromfile(out, dtype=np.float64).reshape(O.state_shape)
    ref, dt0, n = _oracle_run(sim_time)
    assert n == 4
    assert ("dt: %g" % dt0)[:8] in p.stdout.replace("dt: ", "dt: ")
    return got, ref


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_reference_driver_fp64(tmp_path):
    got, ref = _run(tmp_path)
    # initial data: the library's device quadrature (correctly rounded pow) against the
    # oracle's glibc profiles -> last-bit differences, then the same arithmetic
    for v in range(5):
        assert _rel(got[v], ref[v]) <= 5e-12, v


def test_reference_driver_fp32(tmp_path):
    got, ref = _run(tmp_path, "precision : fp32\n")
    h = 2
    for v in range(5):
        a, b = got[v, h:-h, h:-h, h:-h], ref[v, h:-h, h:-h, h:-h]
        if np.abs(b).max() == 0:
            assert np.abs(a).max() < 1e-6
        else:
            assert _rel(a, b) <= 1e-5, (v, _rel(a, b))


def test_reference_driver_netcdf_output(tmp_path):
    """outFile *.nc: the driver's output calls (driver.cpp:41, 55-59) write the reference's
    netCDF file (Spatial:1705-1791) -- records at etime 0, at the first step past outFreq
    and at the end -- whose last record holds the diagnostics of the oracle's final state."""
    from scipy.io import netcdf_file
    from awflcloud_b200 import capi
    O = Oracle(32, 24, 16, bc=(0, 1, 1), crpow=True)
    st = O.new_state()
    O.init_state(st)
    dt0 = O.compute_dt(st, 0.8)
    sim_time = 3.5 * dt0
    inp, out = str(tmp_path / "in.yaml"), str(tmp_path / "out.nc")
    _yaml(inp, out, sim_time, out_freq=sim_time / 2)
    p = subprocess.run([BIN, inp], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    ref, _, _ = _oracle_run(sim_time)
    c = capi.Context(32, 24, 16, bc=("periodic", "wall", "wall"), device=-1)
    bg = c.background()
    h = c.hs
    s = ref[:, h:-h, h:-h, h:-h]
    d = bg["hyDensCells"][h:-h, None, None]
    dt = bg["hyDensThetaCells"][h:-h, None, None]
    r = s[0] + d
    t = (s[4] + dt) / r
    want = [s[0], s[1] / r, s[2] / r, s[3] / r, t - dt / d]
    with netcdf_file(out, "r", mmap=False) as nc:
        tt = nc.variables["t"][:].copy()
        assert len(tt) == 3 and tt[0] == 0.0
        assert abs(tt[1] - 2 * dt0) <= 1e-12 * dt0 and abs(tt[2] - sim_time) <= 1e-12 * sim_time
        for i, name in enumerate(["dens_pert", "u", "v", "w", "pot_temp_pert"]):
            got = nc.variables[name][2]
            assert _rel(got, want[i]) <= 5e-12, name
        # the driver's three tracers (driver.cpp:27-29): initTracers (Spatial:505-560) on the
        # device, written as tracer / rho (Spatial:1778-1783); transport is compiled out in
        # the reference, so they keep their initial values
        tr = O.new_tracers(3)
        O.init_tracers(tr)
        tr = tr[:, h:-h, h:-h, h:-h]
        r0 = st[0, h:-h, h:-h, h:-h] + d
        for i, name in enumerate(["uniform", "theta", "block"]):
            v = nc.variables["tracer_" + name]
            assert v.dimensions == ("t", "z", "y", "x")
            # the device's profile pow is correctly rounded, glibc's (the oracle's) is not
            # always: last-bit differences in a few cells
            np.testing.assert_allclose(v[0], tr[i] / r0, rtol=1e-15, atol=0)
            assert _rel(v[2], tr[i] / r) <= 5e-12, name


def test_reference_driver_tracer_transport(tmp_path):
    """tracer_transport: true runs the reference's compiled-out tracer code through the
    unchanged driver (three posDef tracers, driver.cpp:27-29): the last record's tracer
    fields against the oracle's restatement of that code. The device's initial tracers
    differ from the oracle's (glibc profile pow) in the last bit of a few cells, hence a
    relative L2 bound instead of equality."""
    from scipy.io import netcdf_file
    from awflcloud_b200 import capi
    O = Oracle(32, 24, 16, bc=(0, 1, 1), crpow=True)
    st = O.new_state()
    O.init_state(st)
    tr = O.new_tracers(3)
    O.init_tracers(tr)
    dt0 = O.compute_dt(st, 0.8)
    sim_time = 3.5 * dt0
    inp, out = str(tmp_path / "in.yaml"), str(tmp_path / "out.nc")
    _yaml(inp, out, sim_time, extra="tracer_transport : true\n")
    p = subprocess.run([BIN, inp], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    etime = 0.0
    while etime < sim_time:
        dt = dt0 if etime + dt0 <= sim_time else sim_time - etime
        O.time_step_tracers(st, tr, dt)
        etime += dt
    c = capi.Context(32, 24, 16, bc=("periodic", "wall", "wall"), device=-1)
    h = c.hs
    r = st[0, h:-h, h:-h, h:-h] + c.background()["hyDensCells"][h:-h, None, None]
    t0 = O.new_tracers(3)
    O.init_tracers(t0)
    with netcdf_file(out, "r", mmap=False) as nc:
        for i, name in enumerate(["uniform", "theta", "block"]):
            got = nc.variables["tracer_" + name][-1]
            want = tr[i, h:-h, h:-h, h:-h] / r
            assert _rel(got, want) <= 1e-12, (name, _rel(got, want))
            # transported: differs from the initial field
            assert np.abs(got - t0[i, h:-h, h:-h, h:-h] / r).max() > 1e-8 or name == "uniform"


def test_reference_driver_tracer_transport_fp32(tmp_path):
    """The same driver run in the FP32 form (precision: fp32): its tracer transport (FP32
    reconstruction, fluxes and limiter, FP64 tracer arrays) against the oracle's FP64
    restatement, to the precision form's accuracy."""
    from scipy.io import netcdf_file
    from awflcloud_b200 import capi
    O = Oracle(32, 24, 16, bc=(0, 1, 1), crpow=True)
    st = O.new_state()
    O.init_state(st)
    tr = O.new_tracers(3)
    O.init_tracers(tr)
    dt0 = O.compute_dt(st, 0.8)
    sim_time = 3.5 * dt0
    inp, out = str(tmp_path / "in.yaml"), str(tmp_path / "out.nc")
    _yaml(inp, out, sim_time, extra="tracer_transport : true\nprecision : fp32\n")
    p = subprocess.run([BIN, inp], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    etime = 0.0
    while etime < sim_time:
        dt = dt0 if etime + dt0 <= sim_time else sim_time - etime
        O.time_step_tracers(st, tr, dt)
        etime += dt
    c = capi.Context(32, 24, 16, bc=("periodic", "wall", "wall"), device=-1)
    h = c.hs
    r = st[0, h:-h, h:-h, h:-h] + c.background()["hyDensCells"][h:-h, None, None]
    with netcdf_file(out, "r", mmap=False) as nc:
        for i, name in enumerate(["uniform", "theta", "block"]):
            got = nc.variables["tracer_" + name][-1]
            want = tr[i, h:-h, h:-h, h:-h] / r
            assert _rel(got, want) <= 1e-6, (name, _rel(got, want))
