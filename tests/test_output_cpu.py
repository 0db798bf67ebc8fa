"""Output file of Spatial::output (Spatial:1705-1791) from the library's own netCDF writer
(classic data model, 64-bit offset format), checked with an independent reader
(scipy.io.netcdf_file) on a host-only context: dimensions, the fixed variables (coordinates
and the background profiles, Spatial:1716-1734), records appended one per output time
(Spatial:1738-1741), and the refusal to append to another grid's file."""
import numpy as np
import pytest

from awflcloud_b200 import capi

netcdf = pytest.importorskip("scipy.io").netcdf_file


def _ctx(nx=12, ny=10, nz=8):
    return capi.Context(nx, ny, nz, 20000.0, 16000.0, 10000.0, device=-1)


def _fields(c, seed):
    return np.random.default_rng(seed).standard_normal((6, c.nz, c.ny, c.nx))


def test_file_layout_and_records(tmp_path):
    c = _ctx()
    path = str(tmp_path / "out.nc")
    f0, f1, f2 = _fields(c, 1), _fields(c, 2), _fields(c, 3)
    c.write_netcdf_fields(path, f0, 0.0)
    c.write_netcdf_fields(path, f1, 2.5)
    c.write_netcdf_fields(path, f2, 7.25)
    bg = c.background()
    h = c.hs
    with netcdf(path, "r", mmap=False) as nc:
        assert nc.version_byte == 2
        assert nc.dimensions == {"x": 12, "y": 10, "z": 8, "t": None}
        assert list(nc.variables) == ["x", "y", "z", "hyDens", "hyPressure", "hyTheta", "t", "dens_pert", "u",
                                      "v", "w", "pot_temp_pert", "pressure_pert"]
        np.testing.assert_array_equal(nc.variables["x"][:], (np.arange(12) + 0.5) * (20000.0 / 12))
        np.testing.assert_array_equal(nc.variables["y"][:], (np.arange(10) + 0.5) * (16000.0 / 10))
        np.testing.assert_array_equal(nc.variables["z"][:], (np.arange(8) + 0.5) * (10000.0 / 8))
        np.testing.assert_array_equal(nc.variables["hyDens"][:], bg["hyDensCells"][h:h + 8])
        np.testing.assert_array_equal(nc.variables["hyPressure"][:], bg["hyPressureCells"][h:h + 8])
        np.testing.assert_array_equal(nc.variables["hyTheta"][:], bg["hyThetaCells"][h:h + 8])
        np.testing.assert_array_equal(nc.variables["t"][:], [0.0, 2.5, 7.25])
        for i, name in enumerate(["dens_pert", "u", "v", "w", "pot_temp_pert", "pressure_pert"]):
            v = nc.variables[name]
            assert v.dimensions == ("t", "z", "y", "x")
            for r, f in enumerate((f0, f1, f2)):
                np.testing.assert_array_equal(v[r], f[i])


def test_etime_zero_starts_a_new_file(tmp_path):
    c = _ctx()
    path = str(tmp_path / "out.nc")
    c.write_netcdf_fields(path, _fields(c, 1), 0.0)
    c.write_netcdf_fields(path, _fields(c, 2), 1.0)
    f = _fields(c, 3)
    c.write_netcdf_fields(path, f, 0.0)
    with netcdf(path, "r", mmap=False) as nc:
        np.testing.assert_array_equal(nc.variables["t"][:], [0.0])
        np.testing.assert_array_equal(nc.variables["u"][0], f[1])


def test_append_refuses_missing_or_foreign_files(tmp_path):
    c = _ctx()
    with pytest.raises(capi.AwflError) as e:
        c.write_netcdf_fields(str(tmp_path / "absent.nc"), _fields(c, 1), 1.0)
    assert e.value.code == -7
    other = _ctx(14, 10, 8)
    path = str(tmp_path / "other.nc")
    other.write_netcdf_fields(path, _fields(other, 1), 0.0)
    with pytest.raises(capi.AwflError) as e:
        c.write_netcdf_fields(path, _fields(c, 2), 1.0)
    assert e.value.code == -7
    with pytest.raises(ValueError):
        c.write_netcdf_fields(path, np.zeros(5), 1.0)


def test_tracer_record_variables(tmp_path):
    """Spatial:1778-1783: one tracer_<name> record variable per tracer after the six fields."""
    c = _ctx()
    names = ["uniform", "theta", "block"]
    path = str(tmp_path / "tr.nc")
    rng = np.random.default_rng(7)
    f0 = rng.standard_normal((9, c.nz, c.ny, c.nx))
    f1 = rng.standard_normal((9, c.nz, c.ny, c.nx))
    c.write_netcdf_fields_tracers(path, f0, names, 0.0)
    c.write_netcdf_fields_tracers(path, f1, names, 1.5)
    with netcdf(path, "r", mmap=False) as nc:
        assert list(nc.variables)[-3:] == ["tracer_uniform", "tracer_theta", "tracer_block"]
        np.testing.assert_array_equal(nc.variables["t"][:], [0.0, 1.5])
        for i, name in enumerate(["dens_pert", "u", "v", "w", "pot_temp_pert", "pressure_pert"]
                                 + ["tracer_" + n for n in names]):
            assert nc.variables[name].dimensions == ("t", "z", "y", "x")
            np.testing.assert_array_equal(nc.variables[name][0], f0[i])
            np.testing.assert_array_equal(nc.variables[name][1], f1[i])
    # a file made without these tracers is another layout: appending is refused
    with pytest.raises(capi.AwflError) as e:
        c.write_netcdf_fields(path, f1[:6], 3.0)
    assert e.value.code == -7
    with pytest.raises(ValueError):
        c.write_netcdf_fields_tracers(path, f1[:8], names, 3.0)


def test_file_fixed_variables_equal_reference_output(tmp_path, golden_dir):
    """The coordinates and hydrostatic profiles the library writes are the ones the
    reference's own output() writes (tests/golden/output_fields.npz: its first record,
    recorded by the netCDF stand-in), bit for bit; the record fields written from the
    reference's own values read back unchanged."""
    import os
    z = np.load(os.path.join(golden_dir, "output_fields.npz"))
    names = sorted({k[:-len("_config")] for k in z.files if k.endswith("_config")})
    assert len(names) >= 3
    tr = ["uniform", "theta", "block"]
    fields = ["dens_pert", "u", "v", "w", "pot_temp_pert", "pressure_pert"] + ["tracer_" + n for n in tr]
    for name in names:
        o, nx, ny, nz, bx, by, bz, _ = (int(v) for v in z[name + "_config"])
        bcn = {0: "periodic", 1: "wall"}
        c = capi.Context(nx, ny, nz, bc=(bcn[bx], bcn[by], bcn[bz]), ord_=o, device=-1)
        path = str(tmp_path / (name + ".nc"))
        f = np.stack([z["%s_r0_%s" % (name, v)].reshape(nz, ny, nx) for v in fields])
        c.write_netcdf_fields_tracers(path, f, tr, 0.0)
        with netcdf(path, "r", mmap=False) as nc:
            for v in ("x", "y", "z", "hyDens", "hyPressure", "hyTheta"):
                np.testing.assert_array_equal(nc.variables[v][:], z["%s_r0_%s" % (name, v)], err_msg=(name, v))
            for i, v in enumerate(fields):
                np.testing.assert_array_equal(nc.variables[v][0], f[i], err_msg=(name, v))
