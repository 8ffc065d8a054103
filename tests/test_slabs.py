"""A lattice split into slabs along its last axis (plaquette_b200/slabs.py), on
the CPU: slabs run by an engine built on the oracle (the reference WGSL site
update over a slab with halo planes, draws at whole-lattice indices), their
halos exchanged in one process or between gloo ranks.  For any number of
slabs the result must equal the oracle's whole-lattice keyed sweeps."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import oracle as o

SPECS = [  # (model, q, shape, kernel, beta, j, seed)
    ("ising", 2, (8, 6, 10), o.METROPOLIS, 0.2216544, 1.0, 3),
    ("ising", 2, (12, 10), o.HEATBATH, 0.4406868, 0.8, 4),
    ("potts", 3, (6, 6, 8), o.HEATBATH, 0.5505, 1.0, 5),
    ("potts", 4, (6, 4, 8), o.METROPOLIS, 0.62, 1.0, 6),
]


def _model(kind, q, j):
    return o.Model.ising(j) if kind == "ising" else o.Model.potts(q, j)


class OracleSlab:
    """One slab (planes [z0, z0 + nz)) advanced by the oracle's keyed slab pass."""

    def __init__(self, kind, q, shape, kernel, beta, j, seed32, z0, nz, planes):
        self.model = _model(kind, q, j)
        self.kernel, self.beta, self.seed32 = kernel, beta, seed32
        self.plane = int(np.prod(shape[:-1]))
        self.z0, self.nz = z0, nz
        self.lat = o.Lattice(tuple(shape[:-1]) + (nz + 2,))
        self.buf = np.zeros((nz + 2) * self.plane, dtype=np.uint8)
        self.buf[self.plane:(nz + 1) * self.plane] = planes
        self.sweep = 0

    def views(self):
        p, n = self.plane, self.nz
        return [self.buf[0:p], self.buf[p:2 * p], self.buf[n * p:(n + 1) * p], self.buf[(n + 1) * p:(n + 2) * p]]

    def sync(self):
        pass

    def colour_pass(self, colour):
        local = (colour + (self.z0 + 1)) & 1  # buffer plane 1 is lattice plane z0
        o.keyed_slab_pass(self.model, self.lat, self.buf, self.kernel, self.beta, self.seed32, self.sweep, local,
                          self.plane, (self.nz + 1) * self.plane, (self.z0 - 1) * self.plane)

    def end_sweep(self):
        self.sweep += 1

    def read(self):
        return self.buf[self.plane:(self.nz + 1) * self.plane].copy()


def _start(shape, q, seed):
    rng = o.PcgStream(seed)
    return o.hot_start(int(np.prod(shape)), q, rng)


def _whole(kind, q, shape, kernel, beta, j, seed32, start, sweeps):
    lat = o.Lattice(shape)
    cfg = start.copy()
    for t in range(sweeps):
        o.keyed_local_sweep(_model(kind, q, j), lat, cfg, kernel, beta, seed32, t)
    return cfg


def test_split_is_contiguous_and_balanced():
    from plaquette_b200.slabs import split

    for extent, world in ((10, 1), (10, 3), (24, 5), (7, 7)):
        parts = split(extent, world)
        assert parts[0][0] == 0 and sum(n for _, n in parts) == extent
        assert all(a + n == b for (a, n), (b, _) in zip(parts, parts[1:]))
        assert max(n for _, n in parts) - min(n for _, n in parts) <= 1
    with pytest.raises(ValueError):
        split(4, 5)


@pytest.mark.parametrize("spec", SPECS, ids=lambda s: f"{s[0]}{s[1]}-{len(s[2])}d-{'hb' if s[3] == o.HEATBATH else 'metro'}")
@pytest.mark.parametrize("world", [1, 2, 3])
def test_slabs_in_one_process_equal_the_whole_lattice(spec, world):
    from plaquette_b200.slabs import SlabChain, split

    kind, q, shape, kernel, beta, j, seed = spec
    seed32 = o.fold_seed(seed)
    start = _start(shape, q, seed)
    plane = int(np.prod(shape[:-1]))
    engines = [OracleSlab(kind, q, shape, kernel, beta, j, seed32, z0, nz, start[z0 * plane:(z0 + nz) * plane])
               for z0, nz in split(shape[-1], world)]
    chain = SlabChain(engines)
    chain.advance(3)
    assert np.array_equal(chain.read(), _whole(kind, q, shape, kernel, beta, j, seed32, start, 3))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, spec, q_out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from plaquette_b200.slabs import SlabChain, ring_exchange, split

    kind, q, shape, kernel, beta, j, seed = spec
    seed32 = o.fold_seed(seed)
    start = _start(shape, q, seed)
    plane = int(np.prod(shape[:-1]))
    z0, nz = split(shape[-1], world)[rank]
    engine = OracleSlab(kind, q, shape, kernel, beta, j, seed32, z0, nz, start[z0 * plane:(z0 + nz) * plane])
    chain = SlabChain([engine], ring_exchange(dist, rank, world))
    chain.advance(3)
    q_out.put((rank, chain.read()))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slabs_across_gloo_ranks_equal_the_whole_lattice(world):
    spec = SPECS[0]
    kind, q, shape, kernel, beta, j, seed = spec
    ctx = mp.get_context("spawn")
    q_out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, spec, q_out)) for r in range(world)]
    for p in procs:
        p.start()
    parts = dict(q_out.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = np.concatenate([parts[r] for r in range(world)])
    want = _whole(kind, q, shape, kernel, beta, j, o.fold_seed(seed), _start(shape, q, seed), 3)
    assert np.array_equal(got, want)
