"""Ensemble members spread over the ranks of a torch.distributed process group.

The members of an ensemble are independent grids. Each rank builds one awfl_ensemble of
its share on its own GPU and advances it with no communication. Only the timing (the
maximum over ranks) and, on request, the gathered member states cross ranks. The legacy
model has no ensemble; the reference's active model runs one domain per process, so a
rank holding whole members is the replica form of its data parallelism.

Shares are balanced by cell count with the longest-processing-time rule: the largest
member first, each onto the rank with the fewest cells so far, ties to the lower rank and,
among equal members, to the lower member index. Every rank derives the same assignment
from the member list alone, so no rank has to tell another what it holds.
"""
from __future__ import annotations

from . import capi


def assign_members(cells, world):
    """Member indices per rank (each list ascending) for members of the given cell counts."""
    if world < 1:
        raise ValueError("world must be at least 1")
    load = [0] * world
    share = [[] for _ in range(world)]
    for m in sorted(range(len(cells)), key=lambda i: (-cells[i], i)):
        r = min(range(world), key=lambda q: (load[q], q))
        share[r].append(m)
        load[r] += cells[m]
    return [sorted(s) for s in share]


def member_cells(configs):
    return [int(c["nx"]) * int(c["ny"]) * int(c["nz"]) for c in configs]


class RankEnsemble:
    """This rank's share of an ensemble: an awfl_ensemble of the members assigned to it on
    this rank's GPU (none when there are more ranks than members)."""

    def __init__(self, configs, rank, world, device=0):
        self.configs = list(configs)
        self.rank, self.world = rank, world
        self.shares = assign_members(member_cells(self.configs), world)
        self.share = self.shares[rank]
        self.ensemble = capi.Ensemble([self.configs[i] for i in self.share], device=device) if self.share else None

    def __len__(self):
        return len(self.share)

    def member(self, i):
        """The Context of global member i, which must be in this rank's share."""
        return self.ensemble.members[self.share.index(i)]

    def bind(self, i, state, dt):
        self.ensemble.bind(self.share.index(i), state, dt)

    def tune(self, reps=3, stream=None):
        return self.ensemble.tune(reps, stream) if self.ensemble else None

    def step(self, nsteps=1, stream=None):
        if self.ensemble:
            self.ensemble.step(nsteps, stream)

    def cells(self):
        c = member_cells(self.configs)
        return sum(c[i] for i in self.share)

    def close(self):
        if self.ensemble:
            self.ensemble.close()
            self.ensemble = None


def gather_states(local_states, share, nmembers, dtype, device, group=None):
    """Every member's state on every rank, in member order, as flat tensors: local_states[q]
    is the state of member share[q] on this rank. Each rank's share travels as one
    broadcast from that rank; the shares and their sizes travel first as objects, so the
    receivers can size their buffers. dtype and device are those of every state."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    me = dist.get_rank(group)
    shares = [None] * world
    dist.all_gather_object(shares, [list(share), [int(s.numel()) for s in local_states]], group=group)
    out = [None] * nmembers
    for r in range(world):
        members, lens = shares[r]
        n = sum(lens)
        if n == 0:
            continue
        if r == me:
            buf = torch.cat([s.reshape(-1) for s in local_states]).to(dtype)
        else:
            buf = torch.empty(n, dtype=dtype, device=device)
        dist.broadcast(buf, dist.get_global_rank(group, r) if group is not None else r, group=group)
        off = 0
        for m, k in zip(members, lens):
            out[m] = buf[off:off + k]
            off += k
    return out
