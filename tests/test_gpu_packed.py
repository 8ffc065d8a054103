"""Bit-packed passes of one q = 2 keyed site lattice (plq_packed3d.cu): the
chain's states and primaries equal the oracle's keyed sweeps (the reference
WGSL checkerboard) on small lattices -- rows of one, two and three 64-bit
words, 2D and 3D, Ising Metropolis and heat bath with a field, Potts q = 2 --
and the fused byte sweep on larger ones; sweeps split over several advance
calls continue the keyed sweep counter.  Each case runs twice: with the
per-site first-hash array filled at creation and with both hash rounds
computed in the passes."""
import numpy as np
import pytest

import plaquette_b200 as plq
from tests.test_gpu_local import run_pair

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = plq.Gpu.new()
    if g is None:
        pytest.fail("no CUDA device")
    return g


CASES = [  # kind, q, shape, kernel, beta, extra
    (plq.ISING, 2, (64, 4, 6), plq.METROPOLIS, 0.2216544, {}),
    (plq.ISING, 2, (128, 6, 4), plq.HEATBATH, 0.2216544, {"j": 0.9, "h": 0.1}),
    (plq.ISING, 2, (192, 4, 2), plq.METROPOLIS, 0.25, {"h": -0.2}),
    (plq.ISING, 2, (64, 10), plq.METROPOLIS, 0.4406868, {}),
    (plq.ISING, 2, (128, 6), plq.HEATBATH, 0.4406868, {}),
    (plq.POTTS, 2, (64, 8, 4), plq.HEATBATH, 0.9, {}),
    (plq.POTTS, 2, (128, 4, 4), plq.METROPOLIS, 0.7, {}),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{'ising' if c[0] == plq.ISING else 'potts2'}-"
                                                     f"{'x'.join(map(str, c[2]))}-{'hb' if c[3] == plq.HEATBATH else 'metro'}")
@pytest.mark.parametrize("flags", [0, plq.FLAG_NO_FIRST_HASH], ids=["first-hash-array", "hashed"])
def test_packed_matches_oracle(oracle, gpu, case, flags):
    kind, q, shape, kernel, beta, extra = case
    got, want, chain, model, lat = run_pair(oracle, gpu, kind, q, shape, kernel, plq.RNG_KEYED, beta, 5,
                                            flags=flags, **extra)
    assert chain.path == "packed"
    assert np.array_equal(got, want)
    assert list(chain.primaries()) == list(model.primaries(lat, want))


@pytest.mark.parametrize("kernel", [plq.METROPOLIS, plq.HEATBATH], ids=["metro", "hb"])
def test_packed_equals_fused_sweep(gpu, kernel):
    shape = (512, 64, 32)
    n = int(np.prod(shape))
    start, _ = plq.hot_start(41, 2, n)
    outs = []
    for flags in (0, plq.FLAG_NO_FIRST_HASH, plq.FLAG_NO_PACKED):
        d = plq.make_desc(plq.ISING, 2, shape, kernel, beta=0.2216544, seed=41, rng=plq.RNG_KEYED, sweeps_between=7,
                          batch=1, flags=flags)
        c = plq.GpuChain(gpu, d, start)
        assert c.path == ("fused3d" if flags == plq.FLAG_NO_PACKED else "packed")
        outs.append(next(c))
        c.close()
    assert np.array_equal(outs[0], outs[1])
    assert np.array_equal(outs[0], outs[2])


def test_sweeps_split_over_advance_calls(gpu):
    shape = (128, 16, 8)
    n = int(np.prod(shape))
    start, _ = plq.hot_start(43, 2, n)
    d = plq.make_desc(plq.ISING, 2, shape, plq.METROPOLIS, beta=0.22, seed=43, rng=plq.RNG_KEYED, batch=1)
    one = plq.GpuChain(gpu, d, start)
    one.advance(6)
    split = plq.GpuChain(gpu, d, start)
    for k in (1, 2, 3):
        split.advance(k)
    assert one.sweeps_done == split.sweeps_done == 6
    assert np.array_equal(one.read(), split.read())
