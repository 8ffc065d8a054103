"""The N > 1 paths on the CPU, as gloo ranks.

* bench.py's timing arithmetic: every rank agrees on the slowest rank's time
  and on the whole-job rate (weak scaling).
* Ensembles across ranks (plaquette_b200/distributed.py): members partitioned
  by device footprint, tempering ladders spanning the ranks, energies
  all-reduced every swap interval and the swap phase (the library's host
  rule) run on every rank.  Two ranks must give exactly the one-rank result:
  the same betas on every rank and every member's configuration.  The
  members here run in an engine built on the oracle's keyed sweeps (the
  reference WGSL checkerboard restated), so no device is needed; on a GPU the
  engine is the ensemble itself (tests/test_gpu_distributed.py).
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench

    my_ms = 10.0 + 5.0 * rank
    m = bench.max_over_ranks(dist, my_ms, None)
    rate = bench.whole_job_rate(world, 1000, 7, m)
    q.put((rank, m, rate))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_two_gloo_ranks_aggregate(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    slowest = 10.0 + 5.0 * (world - 1)
    for rank, m, rate in out:
        assert m == slowest
        assert rate == pytest.approx(1000 * world * 7 / (slowest * 1e6))


# ------------------------------------------------------- ensembles across ranks

class OracleEngine:
    """Members advanced by the oracle's keyed sweeps at their current beta."""

    def __init__(self, descs, starts):
        from oracle import oracle as o

        import plaquette_b200 as plq

        self.o = o
        self.members = []
        for d, st in zip(descs, starts):
            shape = tuple(int(d.shape[i]) for i in range(d.d))
            gauge = d.model == plq.GAUGE
            lat = o.Lattice(shape, staples=gauge)
            model = o.Model.gauge(d.j) if gauge else o.Model.ising(d.j, d.h)
            kernel = o.HEATBATH if d.updater == plq.HEATBATH else o.METROPOLIS
            self.members.append([model, lat, st.copy(), kernel, float(d.beta), o.fold_seed(d.seed)])
        self.sweep = int(descs[0].sweep_offset) if descs else 0

    def advance(self, sweeps):
        for _ in range(sweeps):
            for model, lat, cfg, kernel, beta, s32 in self.members:
                self.o.keyed_local_sweep(model, lat, cfg, kernel, beta, s32, self.sweep)
            self.sweep += 1

    def energies(self):
        return [int(m[0].primaries(m[1], m[2])[0]) for m in self.members]

    def set_beta(self, m, beta):
        self.members[m][4] = beta

    def read(self, m):
        return self.members[m][2].copy()


def _workload():
    import plaquette_b200 as plq

    descs, starts, ladders = [], [], []
    ids = []
    for i, b in enumerate(np.geomspace(0.18, 0.26, 5)):  # one ladder of 3D Ising, Metropolis
        ids.append(len(descs))
        descs.append(plq.make_desc(plq.ISING, 2, (6, 6, 6), plq.METROPOLIS, beta=float(b), seed=100 + i,
                                   rng=plq.RNG_KEYED, batch=1))
    ladders.append((ids, [float(descs[m].beta) for m in ids], 17))
    ids = []
    for i, b in enumerate((0.40, 0.45, 0.50)):  # one of 2D Ising heat bath, larger lattices
        ids.append(len(descs))
        descs.append(plq.make_desc(plq.ISING, 2, (12, 10), plq.HEATBATH, beta=b, j=0.8, seed=200 + i,
                                   rng=plq.RNG_KEYED, batch=1))
    ladders.append((ids, [0.40, 0.45, 0.50], 23))
    descs.append(plq.make_desc(plq.GAUGE, 2, (4, 4, 4), plq.HEATBATH, beta=0.6, seed=300, rng=plq.RNG_KEYED,
                               batch=1))  # outside every ladder
    for d in descs:
        n = int(np.prod([d.shape[i] for i in range(d.d)])) * (d.d if d.model == plq.GAUGE else 1)
        starts.append(plq.hot_start(int(d.seed), 2, n)[0])
    return descs, starts, ladders


def _run(world, rank, allreduce, sweeps=(3, 4, 9)):
    from plaquette_b200.distributed import DistributedTempering

    descs, starts, ladders = _workload()
    dt = DistributedTempering(descs, starts, ladders, 2, world, rank, allreduce, OracleEngine)
    for s in sweeps:
        dt.advance(s)
    states = {m: dt.read(m) for m in dt.local}
    return dt.betas(), states, dt.owner, dt.accepted


def _dist_rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from plaquette_b200.distributed import torch_allreduce

    betas, states, owner, accepted = _run(world, rank, torch_allreduce(dist))
    q.put((rank, betas, states, owner, accepted))
    dist.barrier()
    dist.destroy_process_group()


def test_partition_is_deterministic_and_balanced():
    from plaquette_b200.distributed import partition

    sizes = [5, 9, 1, 1, 7, 3, 3, 8]
    owner = partition(sizes, 3)
    assert owner == partition(sizes, 3)
    loads = [sum(s for s, r in zip(sizes, owner) if r == k) for k in range(3)]
    assert max(loads) - min(loads) <= max(sizes)
    assert partition(sizes, 1) == [0] * len(sizes)


def test_tempering_across_two_gloo_ranks_equals_one_rank():
    want_betas, want_states, _, want_acc = _run(1, 0, lambda x: None)
    assert want_acc > 0
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dist_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    seen = set()
    for rank, betas, states, owner, accepted in out:
        assert np.array_equal(betas, want_betas), rank
        assert accepted == want_acc
        assert {m for m, r in enumerate(owner) if r == rank} == set(states)
        for m, st in states.items():
            assert np.array_equal(st, want_states[m]), (rank, m)
            seen.add(m)
    assert seen == set(want_states)  # every member is held by exactly one rank
    assert len({r for _, _, _, owner, _ in out[:1] for r in owner}) == 2  # both ranks hold members
