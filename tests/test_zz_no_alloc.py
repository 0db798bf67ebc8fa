"""awfl_cfl_noalloc: the CFL time step for callers that cannot call cudaMalloc.

Such callers (a host whose device memory all comes from its own pool, or a loop that
cannot afford an allocation's device synchronisation) pass the state and the hydrostatic
background they already hold on the device; the entry point keeps its reduction scratch
in a static device array of the library instead of allocating. It must return the same
time step as awfl_cfl (the minimum is order independent: exact equality), on two calls in
a row with different states (the shared scratch keeps the previous call's values), and it
must reject grids larger than its scratch with a clear error.

Collected last on purpose (file name), so a stop-at-first-failure run has already run
every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from awflcloud_b200 import capi  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _noalloc(ctx, state, dens_c, denstheta_c, cfl):
    L = capi.lib()
    out = ctypes.c_double()
    rc = L.awfl_cfl_noalloc(ctypes.byref(ctx.cfg), state.data_ptr(), dens_c.data_ptr(), denstheta_c.data_ptr(),
                            cfl, ctypes.byref(out), torch.cuda.current_stream().cuda_stream)
    return rc, out.value


def test_cfl_noalloc_matches_cfl_twice():
    ctx = capi.Context(96, 80, 48)
    bg = ctx.background()
    dens_c = torch.from_numpy(bg["hyDensCells"]).cuda()
    denstheta_c = torch.from_numpy(bg["hyDensThetaCells"]).cuda()
    a = ctx.new_state()
    ctx.init_state(a, kind=capi.INIT_BUBBLE, noise_amp=0.01)
    b = ctx.new_state()
    ctx.init_state(b, kind=capi.INIT_BUBBLE, amp=1.0, xrad=3000.0, noise_amp=0.05, noise_seed=11)
    ctx.step(b, ctx.cfl(b, 0.8))          # give the second state non-zero winds
    expected = [ctx.cfl(a, 0.8), ctx.cfl(b, 0.7)]
    assert expected[0] != expected[1]
    for st, cfl, want in ((a, 0.8, expected[0]), (b, 0.7, expected[1])):
        rc, got = _noalloc(ctx, st, dens_c, denstheta_c, cfl)
        assert rc == 0, capi.lib().awfl_last_error(None)
        assert got == want


def test_cfl_noalloc_rejects_grids_beyond_its_scratch():
    ctx = capi.Context(16, 16, 8)
    bg = ctx.background()
    dens_c = torch.from_numpy(bg["hyDensCells"]).cuda()
    st = ctx.new_state()
    big = capi.AwflConfig(512, 512, 128, 20000.0, 20000.0, 10000.0, 0, 0, 1, 1, 1, 1, 5, capi.FP64)
    out = ctypes.c_double(-1.0)
    rc = capi.lib().awfl_cfl_noalloc(ctypes.byref(big), st.data_ptr(), dens_c.data_ptr(), dens_c.data_ptr(),
                                     0.8, ctypes.byref(out), torch.cuda.current_stream().cuda_stream)
    assert rc == -1
    assert b"exceed" in capi.lib().awfl_last_error(None)
    assert out.value == -1.0
