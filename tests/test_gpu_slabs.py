"""Slabs on the device (plq_slab_*): a lattice split along its last axis into
1, 2, 3 or 5 slabs, run in one process with the halos copied between them
before every colour pass, equals the whole-lattice keyed chain bit for bit.
(Ranks on separate devices exchange the same planes over torch.distributed;
that exchange is tested with gloo ranks on the CPU, tests/test_slabs.py.)"""
import numpy as np
import pytest

import plaquette_b200 as plq

pytestmark = pytest.mark.gpu

SPECS = [  # (model, q, shape, updater, beta, j, seed)
    (plq.ISING, 2, (64, 48, 40), plq.METROPOLIS, 0.2216544, 1.0, 21),
    (plq.ISING, 2, (256, 96), plq.HEATBATH, 0.4406868, 0.8, 22),
    (plq.POTTS, 3, (32, 32, 24), plq.HEATBATH, 0.5505, 1.0, 23),
    (plq.POTTS, 4, (32, 16, 24), plq.METROPOLIS, 0.62, 1.0, 24),
]


@pytest.fixture(scope="module")
def gpu():
    g = plq.Gpu.new()
    if g is None:
        pytest.fail("no CUDA device")
    return g


@pytest.mark.parametrize("spec", SPECS, ids=lambda s: f"q{s[1]}-{len(s[2])}d-{'hb' if s[3] == plq.HEATBATH else 'metro'}")
@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_device_slabs_equal_the_whole_chain(gpu, spec, world):
    from plaquette_b200.slabs import DeviceSlab, SlabChain, split

    kind, q, shape, upd, beta, j, seed = spec
    n = int(np.prod(shape))
    start, off = plq.hot_start(seed, q, n)
    desc = plq.make_desc(kind, q, shape, upd, beta=beta, j=j, seed=seed, rng=plq.RNG_KEYED, stream_offset=off,
                         sweeps_between=1, batch=1)
    whole = plq.GpuChain(gpu, desc, start)
    whole.advance(4)
    want = whole.read()
    plane = n // shape[-1]
    engines = [DeviceSlab(gpu, desc, z0, nz, start[z0 * plane:(z0 + nz) * plane])
               for z0, nz in split(shape[-1], world)]
    chain = SlabChain(engines)
    chain.advance(4)
    assert np.array_equal(chain.read(), want)
    for e in engines:
        e.close()


def test_slab_refuses_what_it_does_not_run(gpu):
    from plaquette_b200.slabs import DeviceSlab

    desc = plq.make_desc(plq.ISING, 2, (8, 8, 8), plq.METROPOLIS, beta=0.22, seed=1, rng=plq.RNG_STREAM, batch=1)
    with pytest.raises(plq.UnsupportedError):
        DeviceSlab(gpu, desc, 0, 4, np.zeros(256, dtype=np.uint8))
    desc = plq.make_desc(plq.ISING, 2, (8, 8, 8), plq.METROPOLIS, beta=0.22, seed=1, rng=plq.RNG_KEYED, batch=1)
    with pytest.raises(plq.ContractError):
        DeviceSlab(gpu, desc, 6, 4, np.zeros(256, dtype=np.uint8))  # planes 6..9 of 8
    with pytest.raises(plq.ContractError):
        DeviceSlab(gpu, desc, 0, 4, np.full(256, 2, dtype=np.uint8))  # a state >= q
