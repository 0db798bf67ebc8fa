"""C-ABI checks that need no GPU: the library loads, exports every declared symbol,
validates its arguments, and builds the reference's tables and background (host-only
context) bit-identically to the reference."""
import ctypes
import os

import numpy as np
import pytest

from awflcloud_b200 import capi

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_library_exports_every_header_symbol():
    L = capi.lib()
    syms = capi.header_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_version():
    assert b"sm_100a" in capi.lib().awfl_version()


@pytest.mark.parametrize("kw,code", [
    (dict(ord_=7), -1),
    (dict(bc=(2, 0, 1)), -1),
    (dict(nx=1), -1),            # periodic x narrower than the halo
    (dict(precision=5), -6),
    (dict(data=9), -1),
])
def test_create_rejects_bad_config(kw, code):
    args = dict(nx=10, ny=8, nz=6, device=-1)
    args.update(kw)
    with pytest.raises(capi.AwflError) as e:
        capi.Context(**args)
    assert e.value.code == code


def test_host_only_context_refuses_device_work():
    c = capi.Context(10, 8, 6, device=-1)
    with pytest.raises(capi.AwflError) as e:
        c.split(8, 0.1, 0)  # any aligned non-null pointer: refused before use
    assert e.value.code == -1


@pytest.mark.parametrize("ord_", [5, 9])
def test_tables_match_reference(ord_):
    t = np.load(os.path.join(GOLDEN, "tables_o%d.npz" % ord_))
    mine = capi.Context(10, 8, 6, ord_=ord_, device=-1).tables()
    for k in ("weno_recon", "coefs_to_gll", "sten_to_gll", "idl", "sigma", "gll_pts_ord",
              "gll_wts_ord", "gll_pts_ngll", "gll_wts_ngll"):
        assert np.array_equal(mine[k], t[k]), k
    # exact-math tables vs the reference's Sage literals (129-bit round-off of 2.4e-38 at
    # gll_to_coefs<5>(2,1) where the exact value is 0)
    assert np.max(np.abs(mine["deriv"] - t["deriv"])) <= 1e-37


@pytest.mark.parametrize("case", ["o5_pw_thermal", "o5_igw", "o9_pw_thermal"])
def test_background_matches_reference(case):
    g = np.load(os.path.join(GOLDEN, "case_%s.npz" % case))
    ord_, nx, ny, nz = [int(v) for v in g["config"][:4]]
    c = capi.Context(nx, ny, nz, ord_=ord_, data=str(g["data"]), device=-1)
    for k, v in c.background().items():
        assert np.array_equal(v, g[k]), k


def test_wrapper_rejects_wrong_buffers_before_any_device_call():
    import torch
    c = capi.Context(10, 8, 6, precision=capi.FP32, device=-1)
    assert c.state_shape[0] == 10  # values + Kahan compensation plane
    with pytest.raises(ValueError):
        c.step(torch.zeros((5,) + c.state_shape[1:], dtype=torch.float32), 0.1)  # one plane only, on the CPU
    with pytest.raises(ValueError):
        c.step(torch.zeros(c.state_shape, dtype=torch.float64), 0.1)  # wrong dtype


def test_split_tracers_argument_checks_before_any_device_call():
    """awfl_split_tracers refuses bad arguments on the host: FP32 contexts, more than 64
    tracers, a NULL flag array, a bad direction. A wall direction shorter than the stencil
    half-width is accepted (its stencil indices map to its cells); only the host-only
    context stops it. Periodic ones that short are refused when the context is made."""
    import ctypes
    L = capi.lib()
    pos = (ctypes.c_int * 2)(1, 1)
    short = capi.Context(1, 8, 6, bc=("wall", "periodic", "wall"), device=-1)
    assert L.awfl_split_tracers(short.h, 8, 8, 2, pos, 0.1, 0, None) == -1
    assert b"host-only" in L.awfl_last_error(short.h)
    with pytest.raises(capi.AwflError):
        capi.Context(1, 8, 6, bc=("periodic", "periodic", "wall"), device=-1)
    c = capi.Context(10, 8, 6, device=-1)
    assert L.awfl_split_tracers(c.h, 8, 8, 65, pos, 0.1, 0, None) == -1
    assert L.awfl_split_tracers(c.h, 8, 8, 2, None, 0.1, 0, None) == -1
    assert L.awfl_split_tracers(c.h, 8, 8, 2, pos, 0.1, 3, None) == -1
    # an FP32 context takes tracers too: its arguments pass, and the host-only context then
    # refuses the device work
    c32 = capi.Context(10, 8, 6, precision=capi.FP32, device=-1)
    assert L.awfl_split_tracers(c32.h, 8, 8, 2, pos, 0.1, 0, None) == -1
    assert b"host-only" in L.awfl_last_error(c32.h)
