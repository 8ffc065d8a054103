"""Device measurements against the oracle, integer for integer:
axis_pair_sums (src/models/mod.rs:44-61), Z2Gauge::polyakov_loop
(gauge/mod.rs:179-212) and Z2Gauge::wilson_rectangles (gauge/mod.rs:226-274),
on random and evolved configurations, word path (extent 0 a multiple of 4)
and byte path."""
import numpy as np
import pytest

import plaquette_b200 as plq

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = plq.Gpu.new()
    if g is None:
        pytest.fail("no CUDA device")
    return g


@pytest.mark.parametrize("shape", [(16,), (12, 8), (6, 10), (16, 12, 8), (4, 6, 2, 4), (10, 6, 6)],
                         ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("kind,q", [("ising", 2), ("potts", 3), ("potts", 7)])
def test_axis_pair_sums_match_oracle(oracle, gpu, shape, kind, q):
    n = int(np.prod(shape))
    lat = oracle.Lattice(shape)
    model = oracle.Model.ising(1.0, 0.0) if kind == "ising" else oracle.Model.potts(q, 1.0)
    mk = plq.ISING if kind == "ising" else plq.POTTS
    rng = np.random.default_rng(q * 100 + n)
    d = plq.make_desc(mk, q, shape, plq.METROPOLIS, beta=0.5, seed=3, rng=plq.RNG_KEYED, sweeps_between=2, batch=1)
    for start in (np.zeros(n, np.uint8), rng.integers(0, q, n).astype(np.uint8)):
        chain = plq.GpuChain(gpu, d, start)
        for _ in range(2):
            got = chain.axis_pair_sums()
            want = oracle.axis_pair_sums(model, lat, chain.read())
            assert [list(x) for x in got] == [list(x) for x in want]
            next(chain)
        chain.close()


def test_axis_pair_sums_large_lattice(oracle, gpu):
    # many CTAs per (axis, displacement) pair; oracle on a slice of the pairs via numpy
    shape = (64, 48, 32)
    n = int(np.prod(shape))
    start = np.random.default_rng(5).integers(0, 2, n).astype(np.uint8)
    d = plq.make_desc(plq.ISING, 2, shape, plq.METROPOLIS, beta=0.2, seed=3, rng=plq.RNG_KEYED, batch=1)
    chain = plq.GpuChain(gpu, d, start)
    got = chain.axis_pair_sums()
    g = start.reshape(tuple(reversed(shape))).astype(np.int64)
    s = 1 - 2 * g
    for mu in range(3):
        for r in range(shape[mu] // 2 + 1):
            assert got[mu][r] == int((s * np.roll(s, -r, axis=2 - mu)).sum()), (mu, r)


@pytest.mark.parametrize("shape", [(8, 8), (4, 6, 4), (4, 4, 4, 4), (6, 4, 8, 4), (8, 8, 8, 8), (6, 10, 6)],
                         ids=lambda s: "x".join(map(str, s)))
def test_gauge_loops_match_oracle(oracle, gpu, shape):
    dd = len(shape)
    n = int(np.prod(shape))
    lat = oracle.Lattice(shape)
    rng = np.random.default_rng(n)
    d = plq.make_desc(plq.GAUGE, 2, shape, plq.HEATBATH, beta=0.5, seed=9, rng=plq.RNG_KEYED, sweeps_between=3,
                      batch=1)
    for start in (np.zeros(n * dd, np.uint8), rng.integers(0, 2, n * dd).astype(np.uint8)):
        chain = plq.GpuChain(gpu, d, start)
        for _ in range(2):
            cfg = chain.read()
            for direction in range(dd):
                assert chain.polyakov(direction) == oracle.polyakov_sum(lat, cfg, direction)
            for max_side in (1, 3, 8):
                got, gpl = chain.wilson(max_side)
                want, wpl = oracle.wilson_totals(lat, cfg, max_side)
                assert gpl == wpl
                want = want.copy()
                want[0, :] = wpl
                want[:, 0] = wpl
                assert np.array_equal(got, want), (max_side,)
            next(chain)
        chain.close()


def test_measurement_contracts(gpu):
    site = plq.GpuChain(gpu, plq.make_desc(plq.ISING, 2, (8, 8), plq.METROPOLIS, beta=0.5, rng=plq.RNG_KEYED), None)
    with pytest.raises(plq.PlaquetteError, match="gauge measurement"):
        site.polyakov(0)
    with pytest.raises(plq.PlaquetteError, match="gauge measurement"):
        site.wilson(2)
    link = plq.GpuChain(gpu, plq.make_desc(plq.GAUGE, 2, (4, 4), plq.HEATBATH, beta=0.5, rng=plq.RNG_KEYED), None)
    with pytest.raises(plq.PlaquetteError, match="site-model measurement"):
        link.axis_pair_sums()
    with pytest.raises(plq.PlaquetteError, match="direction out of range"):
        link.polyakov(2)
