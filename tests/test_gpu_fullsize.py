"""Every benchmarked configuration checked against the oracle at its own size.

The benchmark times these lattices, so each is compared bit for bit with the
oracle's restatement of the reference at exactly that size (all tiles, every
z-step of the fused kernel's plane ring, indices up to 2^27, stream
positions up to several 2^27):

* 3D q=3 Potts 512^3, checkerboard heat bath on the PCG stream from the
  seed-20260718 hot start (the fused two-colour kernel), 2 sweeps --
  src/updater.rs:283-348 (LocalUpdate::sweep), heat_bath_step :135-167;
* 3D Ising 512^3 checkerboard Metropolis, keyed stream (fused kernel), 2
  sweeps -- src/wgsl/metropolis.wgsl:32-63 restated in the oracle;
* 3D Ising 512^3 checkerboard Metropolis on the PCG stream (device-wide
  look-back scan per colour pass), 1 sweep -- src/updater.rs:77-96;
* 2D Ising Swendsen-Wang 4096^2 at beta_c, keyed stream, 2 sweeps with the
  canonical labels and the cluster-size histogram -- cluster_prelude.wgsl,
  cluster_relabel.wgsl:39-90;
* 3D Ising Wolff 128^3 at beta = 0.2216544, keyed stream, 20 single-cluster
  updates one at a time (configuration and cluster size after each) against
  the seeded filter of the full decomposition -- src/gpu_cluster.rs:35-44.

The oracle's 512^3 lattice holds a 6.4 GB neighbour table on the host; one
lattice serves the three 512^3 cases.
"""
import numpy as np
import pytest

import plaquette_b200 as plq

pytestmark = pytest.mark.gpu

SEED = 20260718
SHAPE3 = (512, 512, 512)
N3 = 512 ** 3


@pytest.fixture(scope="module")
def gpu():
    g = plq.Gpu.new()
    if g is None:
        pytest.fail("no CUDA device")
    return g


@pytest.fixture(scope="module")
def lat512(oracle):
    lat = oracle.Lattice(SHAPE3)
    yield lat
    del lat


def _stream_case(oracle, gpu, lat, kind, q, kernel, beta, sweeps):
    start, off = plq.hot_start(SEED, q, N3)
    d = plq.make_desc(kind, q, SHAPE3, kernel, beta=beta, seed=SEED, rng=plq.RNG_STREAM, stream_offset=off,
                      sweeps_between=sweeps, batch=1)
    chain = plq.GpuChain(gpu, d, start)
    got, prims = chain.next_sample()
    path = chain.path
    pos = chain.stream_position()
    chain.close()
    model = oracle.Model.potts(q, 1.0) if kind == plq.POTTS else oracle.Model.ising(1.0, 0.0)
    r = oracle.PcgStream(SEED)
    r.advance(off)
    want = start
    oracle.local_sweeps(model, lat, want, kernel, beta, r, sweeps)
    return got, want, list(prims), list(model.primaries(lat, want)), path, pos, r.draws


def test_potts3_512cubed_heat_bath_stream(oracle, gpu, lat512):
    got, want, gp, wp, path, pos, draws = _stream_case(oracle, gpu, lat512, plq.POTTS, 3, plq.HEATBATH, 0.5505, 2)
    assert path == "fused3d"
    assert pos == draws
    assert gp == wp
    assert np.array_equal(got, want)


def test_ising_512cubed_metropolis_stream(oracle, gpu, lat512):
    got, want, gp, wp, path, pos, draws = _stream_case(oracle, gpu, lat512, plq.ISING, 2, plq.METROPOLIS,
                                                       0.2216544, 1)
    assert path == "lookback"
    assert pos == draws
    assert gp == wp
    assert np.array_equal(got, want)


def test_ising_512cubed_metropolis_keyed(oracle, gpu, lat512):
    beta = 0.2216544
    start, _ = plq.hot_start(SEED, 2, N3)
    d = plq.make_desc(plq.ISING, 2, SHAPE3, plq.METROPOLIS, beta=beta, seed=SEED, rng=plq.RNG_KEYED,
                      sweeps_between=2, batch=1)
    chain = plq.GpuChain(gpu, d, start)
    got, prims = chain.next_sample()
    assert chain.path == "packed"
    chain.close()
    model = oracle.Model.ising(1.0, 0.0)
    s32 = oracle.fold_seed(SEED)
    want = start
    for t in range(2):
        oracle.keyed_local_sweep(model, lat512, want, plq.METROPOLIS, beta, s32, t)
    assert list(prims) == list(model.primaries(lat512, want))
    assert np.array_equal(got, want)


def test_sw_4096sq_keyed(oracle, gpu):
    shape, beta = (4096, 4096), 0.4406868
    lat = oracle.Lattice(shape)
    model = oracle.Model.ising(1.0)
    start, _ = plq.hot_start(SEED, 2, lat.n_sites)
    d = plq.make_desc(plq.ISING, 2, shape, plq.CLUSTER, beta=beta, seed=SEED, rng=plq.RNG_KEYED,
                      sweeps_between=1, batch=1, extent=plq.EXTENT_ALL, relabel=plq.RELABEL_REDRAW)
    chain = plq.GpuClusterChain(gpu, d, start)
    s32 = oracle.fold_seed(SEED)
    want = start.copy()
    for sweep in range(2):
        roots = oracle.keyed_cluster_sweep(model, lat, want, oracle.ALL, oracle.REDRAW, beta, s32, sweep,
                                           want_roots=True)
        got = next(chain)
        assert np.array_equal(got, want), sweep
        gl = chain.labels()
        assert np.array_equal(gl, roots), sweep
        sizes = np.bincount(roots)
        sizes = sizes[sizes > 0]
        want_hist = np.bincount(np.floor(np.log2(sizes)).astype(int), minlength=32)[:32]
        assert np.array_equal(chain.size_histogram(32), want_hist), sweep


def test_wolff_128cubed_keyed(oracle, gpu):
    shape, beta = (128, 128, 128), 0.2216544
    lat = oracle.Lattice(shape)
    model = oracle.Model.ising(1.0)
    start, _ = plq.hot_start(SEED, 2, lat.n_sites)
    d = plq.make_desc(plq.ISING, 2, shape, plq.CLUSTER, beta=beta, seed=SEED, rng=plq.RNG_KEYED,
                      sweeps_between=1, batch=1, extent=plq.EXTENT_SEEDED, relabel=plq.RELABEL_FORCED)
    chain = plq.GpuClusterChain(gpu, d, start)
    s32 = oracle.fold_seed(SEED)
    want = start.copy()
    sizes = []
    for update in range(20):
        before = want.copy()
        oracle.keyed_cluster_sweep(model, lat, want, oracle.SEEDED, oracle.FORCED, beta, s32, update)
        got = next(chain)
        assert np.array_equal(got, want), update
        # with a forced relabel of a two-state model every member of the cluster flips
        size = int((before != want).sum())
        sizes.append(size)
        hist = chain.size_histogram(32)
        assert hist.sum() == 1 and hist[int(np.floor(np.log2(size)))] == 1, update
    assert max(sizes) > 1
