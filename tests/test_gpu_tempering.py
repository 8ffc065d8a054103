"""Parallel tempering on the device against an independent host replay.

The reference has no tempering (it is new in this backend), so the oracle
restates the swap rule on its own: each member's keyed sweeps
(src/wgsl/metropolis.wgsl:32-63, heat_bath.wgsl:28-62 restated in the
oracle) at the beta it currently holds, then every `every` sweeps the
energies E = -J * (bond or plaquette sum) from the oracle's primaries and
one swap phase per ladder (orc_pt_swap_phase: even pairs on even attempts,
odd pairs on odd ones, min(1, exp((b_k - b_k+1)(E_k - E_k+1))) from the
keyed uniform).  The device's betas, slot order and every member's
configuration must equal the replay's after every block of sweeps.
"""
import numpy as np
import pytest

import plaquette_b200 as plq
from plaquette_b200.ensemble import Ensemble

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = plq.Gpu.new()
    if g is None:
        pytest.fail("no CUDA device")
    return g


class Replay:
    """The oracle's run of the same ensemble: member configurations, the
    beta each member holds, and each ladder's slot table."""

    def __init__(self, oracle, specs, starts, ladders):
        self.o = oracle
        self.members = []
        for (kind, shape, kernel, beta, seed, j), start in zip(specs, starts):
            lat = oracle.Lattice(shape, staples=kind == plq.GAUGE)
            model = oracle.Model.gauge(j) if kind == plq.GAUGE else oracle.Model.ising(j, 0.0)
            self.members.append([model, lat, start.copy(), kernel, oracle.fold_seed(seed)])
        self.beta = np.array([s[3] for s in specs], dtype=np.float64)
        self.j = np.array([s[5] for s in specs], dtype=np.float64)
        self.ladders = []
        for ids, betas, seed in ladders:
            for m, b in zip(ids, betas):
                self.beta[m] = b
            self.ladders.append((np.array(ids, dtype=np.int32), oracle.fold_seed(seed)))
        self.sweep = 0
        self.accepted = 0
        self.attempted = 0

    def advance(self, sweeps, every):
        for _ in range(sweeps):
            for m, (model, lat, cfg, kernel, s32) in enumerate(self.members):
                self.o.keyed_local_sweep(model, lat, cfg, kernel, float(self.beta[m]), s32, self.sweep)
            self.sweep += 1
            if self.ladders and self.sweep % every == 0:
                att = self.sweep // every - 1
                energy = np.array([int(model.primaries(lat, cfg)[0]) for (model, lat, cfg, _, _) in self.members],
                                  dtype=np.int64)
                for slots, s32 in self.ladders:
                    self.accepted += self.o.pt_swap_phase(slots, self.beta, energy, self.j, s32, att)
                    self.attempted += (len(slots) - (att & 1)) // 2


def _build(gpu, oracle, specs, ladders, cold=()):
    descs, starts = [], []
    for m, (kind, shape, kernel, beta, seed, j) in enumerate(specs):
        n_vars = int(np.prod(shape)) * (len(shape) if kind == plq.GAUGE else 1)
        start = np.zeros(n_vars, dtype=np.uint8) if m in cold else plq.hot_start(seed, 2, n_vars)[0]
        descs.append(plq.make_desc(kind, 2, shape, kernel, beta=beta, j=j, seed=seed, rng=plq.RNG_KEYED,
                                   sweeps_between=1, batch=1))
        starts.append(start)
    return descs, starts, Replay(oracle, specs, starts, ladders)


def _ladder_specs():
    specs, ladders = [], []
    # ladder 0: five 3D Ising replicas, Metropolis, geometric betas
    b0 = list(np.geomspace(0.20, 0.24, 5))
    ids = []
    for i, b in enumerate(b0):
        ids.append(len(specs))
        specs.append((plq.ISING, (8, 8, 8), plq.METROPOLIS, 0.3, 200 + i, 1.0))
    ladders.append((ids, b0, 7))
    # ladder 1: four 2D Ising replicas, heat bath, J = 0.8
    b1 = [0.45, 0.5, 0.55, 0.6]
    ids = []
    for i, b in enumerate(b1):
        ids.append(len(specs))
        specs.append((plq.ISING, (16, 12), plq.HEATBATH, 0.3, 300 + i, 0.8))
    ladders.append((ids, b1, 9))
    # ladder 2: three 4D Z2 gauge lattices, heat bath on links
    b2 = [0.40, 0.44, 0.48]
    ids = []
    for i, b in enumerate(b2):
        ids.append(len(specs))
        specs.append((plq.GAUGE, (4, 4, 4, 4), plq.HEATBATH, 0.4, 400 + i, 1.0))
    ladders.append((ids, b2, 11))
    # a member outside every ladder keeps its own beta
    specs.append((plq.ISING, (6, 6, 6), plq.METROPOLIS, 0.25, 500, 1.0))
    return specs, ladders


@pytest.mark.parametrize("batched", [True, False], ids=["batched", "per-lattice"])
def test_tempering_equals_host_replay(gpu, oracle, batched):
    specs, ladders = _ladder_specs()
    every = 2
    descs, starts, replay = _build(gpu, oracle, specs, ladders)
    ens = Ensemble(gpu, descs, starts)
    for ids, betas, seed in ladders:
        ens.add_ladder(ids, betas, every, seed=seed)
    step = ens.advance if batched else ens.advance_unbatched
    for block in (6, 1, 13, 20):  # 40 sweeps, blocks that do and do not end on a swap sweep
        step(block)
        replay.advance(block, every)
        assert np.array_equal(ens.betas(), replay.beta), replay.sweep
        for m in range(len(specs)):
            assert np.array_equal(ens.read(m), replay.members[m][2]), (replay.sweep, m)
    # the replay saw both outcomes, so the comparison constrains the rule
    assert 0 < replay.accepted < replay.attempted


def test_a_favourable_swap_is_always_taken(gpu, oracle):
    """Both betas in the ordered phase: after one sweep the cold lattice at
    the lower beta (0.3) still has by far the lower energy (bond sum ~ 10900
    of 12288 against ~ 4300 for the random one at 0.4), so
    (b_0 - b_1)(E_0 - E_1) ~ +600 > 0 and the first attempt must swap them
    (a sign error in the rule would keep them: exp(-600) is 0)."""
    specs = [(plq.ISING, (16, 16, 16), plq.METROPOLIS, 0.3, 61, 1.0),
             (plq.ISING, (16, 16, 16), plq.METROPOLIS, 0.4, 62, 1.0)]
    ladders = [([0, 1], [0.3, 0.4], 5)]
    descs, starts, replay = _build(gpu, oracle, specs, ladders, cold=(0,))
    ens = Ensemble(gpu, descs, starts)
    ens.add_ladder([0, 1], [0.3, 0.4], 1, seed=5)
    ens.advance(1)
    replay.advance(1, 1)
    assert replay.accepted == 1
    assert list(ens.betas()) == [0.4, 0.3]
    assert np.array_equal(ens.betas(), replay.beta)
