"""Tempering decided on the host (the path of ladders that span ranks) gives
exactly the device ladder's results: at one rank, DistributedTempering over
the ensemble engine -- energies read back, plq_tempering_swap_phase on the
host, betas set member by member -- against one ensemble whose kernel runs
the swap phase itself.  Betas and every member's configuration must agree,
which pins the host and device evaluations of the rule to each other."""
import numpy as np
import pytest

import plaquette_b200 as plq
from plaquette_b200.distributed import DistributedTempering, EnsembleEngine
from plaquette_b200.ensemble import Ensemble

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = plq.Gpu.new()
    if g is None:
        pytest.fail("no CUDA device")
    return g


def test_host_decided_tempering_equals_the_device_ladder(gpu):
    descs, starts, ladders = [], [], []
    for L, k, lo, hi, base in ((8, 6, 0.19, 0.25, 500), (16, 4, 0.20, 0.23, 600)):
        ids = []
        betas = [float(b) for b in np.geomspace(lo, hi, k)]
        for i, b in enumerate(betas):
            ids.append(len(descs))
            descs.append(plq.make_desc(plq.ISING, 2, (L, L, L), plq.METROPOLIS, beta=b, seed=base + i,
                                       rng=plq.RNG_KEYED, batch=1))
            starts.append(plq.hot_start(base + i, 2, L ** 3)[0])
        ladders.append((ids, betas, base))
    descs.append(plq.make_desc(plq.GAUGE, 2, (6, 6, 6, 6), plq.HEATBATH, beta=0.44, seed=700, rng=plq.RNG_KEYED,
                               batch=1))
    starts.append(plq.hot_start(700, 2, 4 * 6 ** 4)[0])
    every = 2

    dev = Ensemble(gpu, descs, starts)
    for ids, betas, seed in ladders:
        dev.add_ladder(ids, betas, every, seed=seed)
    host = DistributedTempering(descs, starts, ladders, every, 1, 0, lambda x: None,
                                lambda d, s: EnsembleEngine(gpu, d, s))
    for block in (5, 1, 14):
        dev.advance(block)
        host.advance(block)
        assert np.array_equal(dev.betas(), host.betas())
        for m in range(len(descs)):
            assert np.array_equal(dev.read(m), host.read(m)), m
    assert host.accepted > 0
