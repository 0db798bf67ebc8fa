"""x-slab decomposition on the device (awfl_create_slab / awfl_slab_pack / awfl_split_slab):
the slabs of one grid, held in one process on one GPU, trade their halo columns by copies
(awflcloud_b200.slab.route_columns, the same neighbour rule as the NCCL exchange of
SlabDomain) and advance; the gathered interior must equal the undivided grid's bit for bit
-- FP64 (the FP32 form: to FP32 rounding), periodic and wall x, even and uneven splits. Also: a slab's
initial data is its part of the grid's, the grid's time step is the minimum of the slabs',
and the entry points that cannot run on a slab refuse it."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from awflcloud_b200 import capi  # noqa: E402
from awflcloud_b200.slab import route_columns  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


BUBBLE = dict(kind=capi.INIT_BUBBLE, x0=10000.0, y0=10000.0, z0=2000.0, xrad=3000.0, yrad=3000.0, zrad=3000.0,
              amp=3.0, noise_amp=0.01)


def _interior(c, st):
    h = c.hs
    return st[:5, h:h + c.nz, h:h + c.ny, h:h + c.nx]


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
@pytest.mark.parametrize("nx,nslabs,bcx", [(48, 2, "periodic"), (50, 3, "periodic"), (45, 3, "wall"),
                                           (40, 4, "wall")])
def test_slabs_equal_the_undivided_grid(prec, nx, nslabs, bcx):
    ny, nz, steps = 20, 16, 4
    bc = (bcx, "periodic", "wall")
    g = capi.Context(nx, ny, nz, bc=bc, precision=prec)
    gs = g.new_state()
    g.init_state(gs, **BUBBLE)
    slabs = [capi.Context.slab(nx, ny, nz, nslabs, s, bc=bc, precision=prec) for s in range(nslabs)]
    assert sum(c.nx for c in slabs) == nx and [c.xoff for c in slabs] == list(np.cumsum([0] + [c.nx for c in slabs])[:-1])
    ss = []
    for c in slabs:
        st = c.new_state()
        c.init_state(st, **BUBBLE)
        ss.append(st)
        # the slab's initial data is its part of the grid's
        assert torch.equal(_interior(c, st), _interior(g, gs)[..., c.xoff:c.xoff + c.nx])
    dt = g.cfl(gs, 0.8)
    assert min(c.cfl(st, 0.8) for c, st in zip(slabs, ss)) == dt
    dtype = torch.float64 if prec == capi.FP64 else torch.float32
    sends = [torch.empty((2, c.halo_elems // 2), dtype=dtype, device="cuda") for c in slabs]
    ds = 1
    for _ in range(steps):
        g.step(gs, dt)
        for spl in range(3):
            d = spl if ds else 2 - spl
            if d == 0:
                for c, st, sd in zip(slabs, ss, sends):
                    c.slab_pack(st, sd)
                recvs = route_columns(sends, periodic=bcx == "periodic")
                for c, st, rv in zip(slabs, ss, recvs):
                    c.split_slab(st, rv, dt)
            else:
                for c, st in zip(slabs, ss):
                    c.split(st, dt, d)
        ds = 1 - ds
    torch.cuda.synchronize()
    whole = torch.cat([_interior(c, st) for c, st in zip(slabs, ss)], dim=3)
    ref = _interior(g, gs)
    if prec == capi.FP64:
        assert torch.equal(whole, ref), (whole - ref).abs().max().item()
    else:
        # FP32: the compiler places contracted multiply-adds per inlined copy of the
        # reconstruction, and a slab's boundary face takes its states from the prologue's
        # and epilogue's copies where the undivided grid uses the main loop's: the results
        # agree to FP32 rounding (relative to each variable's range)
        for v in range(5):
            scale = ref[v].abs().max().item()
            assert (whole[v] - ref[v]).abs().max().item() <= 2e-6 * scale, v


def test_slab_refusals():
    c = capi.Context.slab(32, 8, 8, 2, 0)
    st = c.new_state()
    with pytest.raises(capi.AwflError):
        c.step(st, 0.5)          # the x split needs the neighbours' columns
    with pytest.raises(capi.AwflError):
        c.split(st, 0.5, 0)
    c.split(st, 0.5, 1)          # y and z need nothing from other slabs
    c.split(st, 0.5, 2)
    tr = c.new_tracers(1)
    with pytest.raises(capi.AwflError):
        c.step_tracers(st, tr, 0.5)
    with pytest.raises(capi.AwflError):
        capi.Context.slab(8, 8, 8, 4, 0)  # slabs narrower than hs+1 cells
    one = capi.Context.slab(32, 8, 8, 1, 0)  # a single slab is the whole grid
    one.step(one.new_state(), 0.5)
