"""Ensembles across ranks: members partitioned by device footprint, tempering
ladders that span ranks.

The reference runs one chain per process on one adapter (src/device.rs:31-78),
so this has no counterpart there.  Each rank holds the members the partition
gives it, in an ensemble of its own on its own device; members never move.
Every `every` sweeps each rank measures the energies of the ladder members it
holds, one all-reduce (a sum over a vector of int64, one entry per ladder
member: a few KB) gives every rank all of them, and every rank runs the same
swap phase over the full slot tables -- plq_tempering_swap_phase, the rule of
the ensemble kernel's own swap phase, defined once for host and device -- and
then sets the betas of the members it holds.  The result does not depend on
the number of ranks: a member's sweeps depend only on its own state, seed,
sweep counter and beta, and every rank sees the same energies and makes the
same decisions.

An engine is what runs the members of one rank: `advance(sweeps)`,
`energy(m)` (the int64 bond, agreement or plaquette sum), `set_beta(m, beta)`
and `read(m)` over local member indices.  `EnsembleEngine` is the device one.
"""
from __future__ import annotations

import numpy as np

from . import GAUGE
from .ensemble import Ensemble, swap_phase


def member_footprint(desc) -> int:
    """Device bytes a member holds: its state (one byte per variable) and its
    decision tables (at most a few hundred KB; counted as a fixed 64 KiB)."""
    n = int(np.prod([desc.shape[i] for i in range(desc.d)]))
    return (n * desc.d if desc.model == GAUGE else n) + (64 << 10)


def partition(footprints, n_ranks: int) -> list[int]:
    """The rank of every member: largest first, each to the rank holding the
    fewest bytes so far (lowest rank on a tie) -- deterministic, so every
    rank computes the same plan."""
    load = [0] * n_ranks
    owner = [0] * len(footprints)
    for m in sorted(range(len(footprints)), key=lambda i: (-footprints[i], i)):
        r = min(range(n_ranks), key=lambda k: (load[k], k))
        owner[m] = r
        load[r] += footprints[m]
    return owner


class EnsembleEngine:
    """The device engine: this rank's members in one ensemble (no device
    ladders: the swaps are decided across ranks)."""

    def __init__(self, gpu, descs, starts):
        self.ens = Ensemble(gpu, descs, starts)

    def advance(self, sweeps: int) -> None:
        self.ens.advance(sweeps)

    def energies(self) -> list[int]:
        return [int(p[0]) for p in self.ens.primaries_all()]

    def set_beta(self, m: int, beta: float) -> None:
        self.ens.set_beta(m, beta)

    def read(self, m: int) -> np.ndarray:
        return self.ens.read(m)

    def close(self):
        self.ens.close()


class DistributedTempering:
    """Members `descs` (with `starts`) over `world` ranks; `ladders` as
    (global member ids, betas, seed) with slot i of a ladder starting at
    betas[i]; swaps every `every` sweeps.  `allreduce(x)` sums an int64
    vector over the ranks in place (identity at one rank); `make_engine(descs,
    starts)` builds this rank's engine."""

    def __init__(self, descs, starts, ladders, every: int, world: int, rank: int, allreduce, make_engine):
        if every <= 0:
            raise ValueError("the swap interval must be positive")
        self.every = every
        self.world, self.rank = world, rank
        self.allreduce = allreduce
        n = len(descs)
        self.owner = partition([member_footprint(d) for d in descs], world)
        self.local = [m for m in range(n) if self.owner[m] == rank]
        self.local_index = {m: k for k, m in enumerate(self.local)}
        self.beta = np.array([float(d.beta) for d in descs], dtype=np.float64)
        self.j = np.array([float(d.j) for d in descs], dtype=np.float64)
        self.ladders = []
        for ids, betas, seed in ladders:
            for m, b in zip(ids, betas):
                self.beta[m] = b
            self.ladders.append((np.array(ids, dtype=np.int32), int(seed)))
        self.in_ladder = sorted({int(m) for ids, _ in self.ladders for m in ids})
        local_descs = []
        for m in self.local:
            d = type(descs[m]).from_buffer_copy(descs[m])
            d.beta = self.beta[m]
            local_descs.append(d)
        self.engine = make_engine(local_descs, [starts[m] for m in self.local] if starts is not None else None)
        self.sweep = int(descs[0].sweep_offset) if n else 0
        self.accepted = 0

    def _energies(self) -> np.ndarray:
        e = np.zeros(len(self.beta), dtype=np.int64)
        mine = self.engine.energies()
        for m in self.in_ladder:
            if self.owner[m] == self.rank:
                e[m] = mine[self.local_index[m]]
        self.allreduce(e)
        return e

    def advance(self, sweeps: int) -> None:
        """`sweeps` sweeps of every member, with the swap phases they reach."""
        left = sweeps
        while left > 0:
            to_swap = self.every - self.sweep % self.every
            step = min(left, to_swap)
            self.engine.advance(step)
            self.sweep += step
            left -= step
            if self.ladders and self.sweep % self.every == 0:
                energy = self._energies()
                att = self.sweep // self.every - 1
                before = self.beta.copy()
                for slots, seed in self.ladders:
                    self.accepted += swap_phase(slots, self.beta, energy, self.j, seed, att)
                for m in np.flatnonzero(self.beta != before):
                    if self.owner[m] == self.rank:
                        self.engine.set_beta(self.local_index[int(m)], float(self.beta[m]))

    def betas(self) -> np.ndarray:
        return self.beta.copy()

    def read(self, m: int) -> np.ndarray:
        """A member this rank holds."""
        return self.engine.read(self.local_index[m])


def torch_allreduce(dist, device=None):
    """An `allreduce` over torch.distributed (a CPU tensor for gloo, a device
    tensor for NCCL)."""
    import torch

    def run(x: np.ndarray) -> None:
        t = torch.from_numpy(x.copy())
        if device is not None:
            t = t.to(device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        x[:] = t.cpu().numpy()

    return run
