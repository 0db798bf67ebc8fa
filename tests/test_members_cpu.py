"""Ensemble members spread over ranks (awflcloud_b200/members.py), host side.

Ranks run as gloo processes on the CPU: each takes its share of the members from
assign_members, advances them with the oracle (no communication while stepping, as the
ranks' awfl_ensembles do on their GPUs), and gather_states brings every member to every
rank. The gathered members must equal the same members stepped one after another in one
process, bit for bit; every member is held by exactly one rank and the shares' cell counts
are balanced."""
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
from awflcloud_b200.members import assign_members, gather_states  # noqa: E402

SIZES = [(8, 8, 8), (12, 8, 8), (16, 10, 8), (8, 12, 10), (10, 10, 8), (16, 16, 8), (8, 8, 12)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_assign_members_covers_and_balances():
    rng = np.random.default_rng(3)
    for world in (1, 2, 3, 5, 8):
        cells = [int(c) for c in rng.integers(1, 1000, size=23)]
        shares = assign_members(cells, world)
        flat = sorted(m for s in shares for m in s)
        assert flat == list(range(len(cells)))
        loads = [sum(cells[m] for m in s) for s in shares]
        # longest-processing-time bound: no rank exceeds the mean by more than the largest member
        assert max(loads) <= sum(cells) / world + max(cells)
        assert shares == assign_members(cells, world)  # deterministic
    assert assign_members([5, 5], 4) == [[0], [1], [], []]


def _member(i):
    """Oracle, state and time step of member i: its own size and bubble."""
    from oracle.pyoracle import Oracle
    nx, ny, nz = SIZES[i]
    O = Oracle(nx, ny, nz, bc=(0, 0, 1))
    st = O.new_state()
    O.init_state(st)
    O.set_bubble(st, 1, 6000.0 + 1000.0 * i, 10000.0, 2000.0, 2500.0, 2500.0, 2500.0, 1.0 + 0.5 * i, 1.0)
    O.add_theta_noise(st, 100 + i, 0.01)
    return O, st, O.compute_dt(st, 0.8)


def _rank(rank, world, port, nsteps, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cells = [nx * ny * nz for nx, ny, nz in SIZES]
        share = assign_members(cells, world)[rank]
        mine = []
        for i in share:
            O, st, dt = _member(i)
            for _ in range(nsteps):
                O.time_step(st, dt)
            mine.append(torch.from_numpy(st))
        got = gather_states(mine, share, len(SIZES), torch.float64, torch.device("cpu"))
        if rank == 0:
            ok = []
            for i in range(len(SIZES)):
                O, st, dt = _member(i)
                for _ in range(nsteps):
                    O.time_step(st, dt)
                ok.append(bool(np.array_equal(got[i].numpy(), st.reshape(-1))))
            q.put(ok)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_members_over_gloo_ranks_equal_one_process(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, 2, q)) for r in range(world)]
    for p in procs:
        p.start()
    ok = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(ok), ok
