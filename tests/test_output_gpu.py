"""Output diagnostics of Spatial::output (Spatial:1744-1778) on the device and the netCDF
file written from them, for both state forms.

Pinned to the reference's own output(): tests/golden/output_fields.npz holds every field
the reference computed (recorded by its netCDF stand-in) for two records of three
configurations; the device fields from the same states are bit-identical to them where
the reference's pow is correctly rounded, and within a few ulp of the ~1e5 Pa pressure in
pressure_pert against its glibc build. Also: the fields against the same formulas in numpy
FP64 on the copied state (bit for bit except pressure_pert, whose pow the device rounds
correctly and libm may not: 1e-9 Pa on ~1e5 Pa), and the file against the fields."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from awflcloud_b200 import capi  # noqa: E402

netcdf = pytest.importorskip("scipy.io").netcdf_file

C0 = 27.5629410929725921310572974482  # phys_params.h
GAMMA = 1.40027894002789400278940027894


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def reference_fields(c, st):
    """Spatial:1744-1778 in numpy on the interior of a copied state."""
    h = c.hs
    s = st.cpu().double().numpy()
    if c.precision == capi.FP32:
        s = s[:5] - s[5:]  # value minus the Kahan compensation
    s = s[:, h:h + c.nz, h:h + c.ny, h:h + c.nx]
    bg = c.background()
    d = bg["hyDensCells"][h:h + c.nz, None, None]
    dt = bg["hyDensThetaCells"][h:h + c.nz, None, None]
    p = bg["hyPressureCells"][h:h + c.nz, None, None]
    r = s[0] + d
    t = (s[4] + dt) / r
    return np.stack([s[0], s[1] / r, s[2] / r, s[3] / r, t - dt / d, C0 * np.power(r * t, GAMMA) - p])


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
def test_output_fields_and_file(tmp_path, prec):
    c = capi.Context(40, 24, 20, precision=prec, bc=("periodic", "wall", "wall"))
    st = c.new_state()
    c.init_state(st, kind=capi.INIT_BUBBLE, noise_amp=0.01)
    dt = c.cfl(st, 0.8)
    path = str(tmp_path / "out.nc")
    c.write_netcdf(path, st, 0.0)
    recs = []
    for n in range(1, 3):
        for _ in range(3):
            c.step(st, dt)
        f = c.output_fields(st).cpu().numpy()
        ref = reference_fields(c, st)
        for i in range(5):
            np.testing.assert_array_equal(f[i], ref[i], err_msg=str(i))
        np.testing.assert_allclose(f[5], ref[5], rtol=0, atol=1e-9)
        c.write_netcdf(path, st, 3.0 * n * dt)
        recs.append(f)
    with netcdf(path, "r", mmap=False) as nc:
        np.testing.assert_allclose(nc.variables["t"][:], [0.0, 3.0 * dt, 6.0 * dt], rtol=0, atol=0)
        for i, name in enumerate(["dens_pert", "u", "v", "w", "pot_temp_pert", "pressure_pert"]):
            for r, f in enumerate(recs):
                np.testing.assert_array_equal(nc.variables[name][r + 1], f[i])
        assert np.abs(nc.variables["w"][2]).max() > 0  # the bubble has started to rise


def test_output_fields_equal_reference_output(golden_dir):
    import os
    z = np.load(os.path.join(golden_dir, "output_fields.npz"))
    names = sorted({k[:-len("_config")] for k in z.files if k.endswith("_config")})
    fields = ["dens_pert", "u", "v", "w", "pot_temp_pert", "pressure_pert"]
    tr = ["uniform", "theta", "block"]
    bcn = {0: "periodic", 1: "wall"}
    for name in names:
        o, nx, ny, nz, bx, by, bz, crpow = (int(v) for v in z[name + "_config"])
        c = capi.Context(nx, ny, nz, bc=(bcn[bx], bcn[by], bcn[bz]), ord_=o)
        for rec in (0, 1):
            st = torch.from_numpy(z["%s_r%d_state" % (name, rec)].copy()).cuda()
            trs = torch.from_numpy(z["%s_r%d_tracers" % (name, rec)].copy()).cuda()
            got = c.output_fields(st).cpu().numpy()
            for i, v in enumerate(fields):
                want = z["%s_r%d_%s" % (name, rec, v)].reshape(nz, ny, nx)
                if crpow or v != "pressure_pert":
                    np.testing.assert_array_equal(got[i], want, err_msg=(name, rec, v))
                else:  # glibc's pow vs correctly rounded: a few ulp of the ~1e5 Pa pressure
                    np.testing.assert_allclose(got[i], want, rtol=0, atol=4 * np.spacing(1.2e5))
            gt = c.output_tracer_fields(st, trs).cpu().numpy()
            for t, n in enumerate(tr):
                np.testing.assert_array_equal(gt[t], z["%s_r%d_tracer_%s" % (name, rec, n)].reshape(nz, ny, nx),
                                              err_msg=(name, rec, n))
