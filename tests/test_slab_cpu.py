"""x-slab decomposition of one grid over ranks (awflcloud_b200/slab.py), host side.

Ranks run as gloo processes on the CPU and compute with the oracle, exchanging halo
columns with the library's own exchange logic (neighbours, exchange_columns): each rank
owns one slab of a periodic grid, packs its first and last hs+1 interior columns in the
layout of awfl_slab_pack, trades them with its neighbours before every x split, and
advances its slab's x split on an array extended by the received columns (the neighbour's
edge cell reconstructed locally, so the face between two slabs sees the same states as in
the undivided grid); y and z splits need nothing from other ranks. The grid's time step is
the minimum of the slabs' (an all-reduce). After several steps the gathered slabs must equal
the undivided grid's oracle run bit for bit. The legacy MPI model does the same with hs
columns plus a separate exchange of edge values (qjrmsCode/Exchange.cpp:106-320)."""
import os
import socket
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from awflcloud_b200.slab import exchange_columns, neighbours, route_columns  # noqa: E402

BC_GIVEN = 2  # the oracle's x mode for halos supplied by the caller


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_neighbours():
    assert neighbours(0, 1, True) == (None, None)
    assert neighbours(0, 2, True) == (1, 1)
    assert neighbours(0, 3, True) == (2, 1)
    assert neighbours(2, 3, True) == (1, 0)
    assert neighbours(0, 3, False) == (None, 1)
    assert neighbours(2, 3, False) == (1, None)


def test_route_columns_in_one_process():
    sends = [torch.arange(8, dtype=torch.float64).reshape(2, 4) + 100 * s for s in range(3)]
    r = route_columns(sends, periodic=True)
    assert torch.equal(r[0][0], sends[2][1]) and torch.equal(r[0][1], sends[1][0])
    assert torch.equal(r[2][1], sends[0][0])
    r = route_columns(sends, periodic=False)
    assert torch.count_nonzero(r[0][0]) == 0 and torch.count_nonzero(r[2][1]) == 0


def _pack(st, hs):
    """awfl_slab_pack's layout: [2][5][nz][ny][hs+1], first / last interior columns."""
    w = hs + 1
    inner = st[:, hs:-hs, hs:-hs, hs:-hs]
    return np.ascontiguousarray(np.stack([inner[..., :w], inner[..., inner.shape[-1] - w:]]))


def _x_split(O_ext, O_loc, st, recv, dt, hs):
    """The slab's x split: the line extended by the received columns (positions
    -(hs+1) .. L+hs; its cells -1 and L are the neighbours' edge cells), tendencies of the
    extended line, the slab's own cells applied."""
    nz, ny, L = st.shape[1] - 2 * hs, st.shape[2] - 2 * hs, st.shape[3] - 2 * hs
    ext = np.zeros((5, nz + 2 * hs, ny + 2 * hs, L + 2 + 2 * hs))
    I = (slice(None), slice(hs, hs + nz), slice(hs, hs + ny))
    ext[I + (slice(0, hs + 1),)] = recv[0]
    ext[I + (slice(hs + 1, hs + 1 + L),)] = st[I + (slice(hs, hs + L),)]
    ext[I + (slice(hs + 1 + L, L + 2 + 2 * hs),)] = recv[1]
    tend = np.zeros((5, nz, ny, L + 2))
    O_ext.compute_tendencies_dir(ext, tend, dt, 0)
    own = np.ascontiguousarray(tend[..., 1:L + 1])
    O_loc.apply(st, own, dt)


def _slab_rank(rank, world, port, cfg, q):
    from oracle.pyoracle import Oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        nx, ny, nz, nsteps = cfg
        bc = (0, 0, 1)
        G = Oracle(nx, ny, nz, bc=bc)
        st = G.new_state()
        G.init_state(st)
        G.set_bubble(st, 1, 10000.0, 10000.0, 2000.0, 2000.0, 2000.0, 2000.0, 3.0, 1.0)
        G.add_theta_noise(st, 20261203, 0.01)
        hs = G.hs
        L = nx // world
        x0 = rank * L
        dx, dy, dz = 20000.0 / nx, 20000.0 / ny, 10000.0 / nz
        loc = Oracle(L, ny, nz, bc=bc)
        loc.set_spacing(dx, dy, dz)
        ext = Oracle(L + 2, ny, nz, bc=(BC_GIVEN, bc[1], bc[2]))
        ext.set_spacing(dx, dy, dz)
        sl = np.zeros((5, nz + 2 * hs, ny + 2 * hs, L + 2 * hs))
        sl[..., hs:hs + L] = st[..., hs + x0:hs + x0 + L]
        # the grid's time step: the minimum of the slabs'
        t = torch.tensor([loc.compute_dt(sl, 0.8)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        dt = t.item()
        recv = torch.zeros((2, 5 * nz * ny * (hs + 1)), dtype=torch.float64)
        tend = np.zeros((5, nz, ny, L))
        ds = 1
        for _ in range(nsteps):
            for spl in range(3):
                d = spl if ds else 2 - spl
                if d == 0:
                    send = torch.from_numpy(_pack(sl, hs).reshape(2, -1))
                    exchange_columns(send, recv, rank, world, periodic=True)
                    _x_split(ext, loc, sl, recv.numpy().reshape(2, 5, nz, ny, hs + 1), dt, hs)
                else:
                    loc.compute_tendencies_dir(sl, tend, dt, d)
                    loc.apply(sl, tend, dt)
            ds = 1 - ds
        out = [torch.zeros_like(torch.from_numpy(sl)) for _ in range(world)]
        dist.all_gather(out, torch.from_numpy(sl))
        if rank == 0:
            gdt = G.compute_dt(st, 0.8)
            for _ in range(nsteps):
                G.time_step(st, gdt)
            whole = np.concatenate([o.numpy()[:, hs:-hs, hs:-hs, hs:-hs] for o in out], axis=3)
            q.put((dt == gdt, bool(np.array_equal(whole, st[:, hs:-hs, hs:-hs, hs:-hs])),
                   float(np.abs(whole - st[:, hs:-hs, hs:-hs, hs:-hs]).max())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slabs_over_gloo_ranks_equal_the_undivided_grid(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    cfg = (8 * world, 10, 8, 4)  # nx, ny, nz, steps: 8 cells per slab
    procs = [ctx.Process(target=_slab_rank, args=(r, world, port, cfg, q)) for r in range(world)]
    for p in procs:
        p.start()
    same_dt, equal, maxdiff = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert same_dt
    assert equal, maxdiff
