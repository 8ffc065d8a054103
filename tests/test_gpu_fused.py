"""The fused two-colour 3D sweep: bit-exact with the oracle on small
lattices, and identical to the per-colour pass kernels on larger ones."""
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


MODES = [
    (plq.POTTS, 3, plq.HEATBATH, plq.RNG_STREAM),
    (plq.POTTS, 3, plq.HEATBATH, plq.RNG_KEYED),
    (plq.ISING, 2, plq.HEATBATH, plq.RNG_STREAM),
    (plq.ISING, 2, plq.HEATBATH, plq.RNG_KEYED),
    (plq.ISING, 2, plq.METROPOLIS, plq.RNG_KEYED),
    (plq.POTTS, 2, plq.HEATBATH, plq.RNG_STREAM),
]
IDS = ["potts3-hb-stream", "potts3-hb-keyed", "ising-hb-stream", "ising-hb-keyed", "ising-metro-keyed",
       "potts2-hb-stream"]


@pytest.mark.parametrize("shape", [(128, 64, 16), (256, 32, 24), (512, 16, 8), (512, 32, 16)], ids=str)
@pytest.mark.parametrize("mode", MODES, ids=IDS)
def test_fused_matches_oracle(oracle, gpu, shape, mode):
    kind, q, kernel, rng = mode
    beta = {plq.ISING: 0.2216544, plq.POTTS: 0.5505}[kind]
    # (q = 2 keyed chains would take the bit-packed passes: kept on the fused sweep here)
    got, want, chain, model, lat = run_pair(oracle, gpu, kind, q, shape, kernel, rng, beta, 5,
                                            flags=plq.FLAG_NO_PACKED)
    assert chain.path == "fused3d"
    assert np.array_equal(got, want)
    assert list(chain.primaries()) == list(model.primaries(lat, want))


@pytest.mark.parametrize("mode", MODES, ids=IDS)
def test_fused_equals_pass_kernels(gpu, mode):
    kind, q, kernel, rng = mode
    shape = (256, 64, 64)
    n = 256 * 64 * 64
    start, off = plq.hot_start(99, q, n)
    outs = []
    for flags in (plq.FLAG_NO_PACKED, plq.FLAG_NO_FUSED):
        d = plq.make_desc(kind, q, shape, kernel, beta=0.4, seed=99, rng=rng, stream_offset=off,
                          sweeps_between=6, batch=1, flags=flags)
        c = plq.GpuChain(gpu, d, start)
        assert c.path == ("fused3d" if flags == plq.FLAG_NO_PACKED else ("lookback" if kernel == plq.METROPOLIS and rng == plq.RNG_STREAM else "words"))
        outs.append(next(c))
        if rng == plq.RNG_STREAM:
            outs.append(c.stream_position())
    assert np.array_equal(outs[0], outs[2 if rng == plq.RNG_STREAM else 1])
    if rng == plq.RNG_STREAM:
        assert outs[1] == outs[3] == off + 6 * n


@pytest.mark.parametrize("shape,beta", [((512, 64, 32), 0.2216544), ((1024, 512), 0.4406868), ((48, 32, 16), 0.3)],
                         ids=str)
def test_vector_scan_pass_equals_generic_lookback(gpu, shape, beta):
    """The vectorised stream-Metropolis pass (plq_scan.cu) against the
    generic look-back pass: same configurations, same stream position."""
    n = int(np.prod(shape))
    start, off = plq.hot_start(5, 2, n)
    outs = []
    for flags in (0, plq.FLAG_NO_FUSED):
        d = plq.make_desc(plq.ISING, 2, shape, plq.METROPOLIS, beta=beta, h=0.05, seed=5, rng=plq.RNG_STREAM,
                          stream_offset=off, sweeps_between=4, batch=1, flags=flags)
        c = plq.GpuChain(gpu, d, start)
        outs.append((next(c), c.stream_position()))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert outs[0][1] == outs[1][1]


def test_tile_copy_wait_limit_reports_and_context_survives(oracle, gpu):
    # every tile waits for a z-plane whose copies are never issued: the bounded
    # wait runs out, the launch reports status bit 16, and the device stays usable
    shape = (128, 64, 16)
    start = np.zeros(int(np.prod(shape)), dtype=np.uint8)
    d = plq.make_desc(plq.ISING, 2, shape, plq.METROPOLIS, beta=0.3, seed=3, rng=plq.RNG_KEYED, batch=1,
                      flags=plq.FLAG_TEST_COPY_STALL | plq.FLAG_NO_PACKED)
    chain = plq.GpuChain(gpu, d, start)
    assert chain.path == "fused3d"
    with pytest.raises(plq.PlaquetteError, match="16 = tile copy wait limit") as info:
        next(chain)
    assert info.value.code == plq.PLQ_EDEVICE
    chain.close()
    got, want, *_ = run_pair(oracle, gpu, plq.ISING, 2, shape, plq.METROPOLIS, plq.RNG_KEYED, 0.3, 2,
                             flags=plq.FLAG_NO_PACKED)
    assert np.array_equal(got, want)


def test_never_cut_point_leaves_the_fused_sweep(oracle, gpu):
    # at beta = 40 some heat-bath probabilities round to 1 in f64, so a cut point is
    # 2^53 ("never"), which the fused sweep's shifted table cannot hold: the chain
    # runs the per-colour passes and still equals the oracle
    shape = (128, 64, 8)
    got, want, chain, *_ = run_pair(oracle, gpu, plq.POTTS, 3, shape, plq.HEATBATH, plq.RNG_STREAM, 40.0, 2)
    assert chain.path == "words"
    assert np.array_equal(got, want)
    got, want, chain, *_ = run_pair(oracle, gpu, plq.POTTS, 3, shape, plq.HEATBATH, plq.RNG_STREAM, 0.5505, 2)
    assert chain.path == "fused3d"
    assert np.array_equal(got, want)
