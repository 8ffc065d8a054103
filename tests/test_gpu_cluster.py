"""Swendsen-Wang and Wolff on the device against the oracle, bit for bit.

PCG stream: ClusterUpdate::sweep (src/updater.rs:541-613) with the same
stream; the decomposition's canonical labels, ranked, equal site_clusters'
compacted labels (src/cluster.rs:44-62,199-226).  Keyed stream: the reference
GPU cluster kernels (cluster_prelude.wgsl, cluster_relabel.wgsl) restated in
the oracle; Wolff's frontier BFS equals the seeded filter of the full
decomposition.  Limits and the pass-cap error path follow
src/gpu_cluster.rs:650-1056.
"""
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


def _model(oracle, kind, q, j=1.0):
    return oracle.Model.ising(j) if kind == plq.ISING else oracle.Model.potts(q, j)


def _chain(gpu, kind, q, shape, extent, relabel, beta, seed, start, rng, offset=0, flags=0, j=1.0):
    d = plq.make_desc(kind, q, shape, plq.CLUSTER, beta=beta, j=j, seed=seed, rng=rng, stream_offset=offset,
                      sweeps_between=1, batch=1, extent=extent, relabel=relabel, flags=flags)
    return plq.GpuClusterChain(gpu, d, start)


def _compact(labels):
    """Min-site labels -> first-encounter compaction (site_clusters' numbering)."""
    _, first = np.unique(labels, return_index=True)
    order = np.argsort(first)
    remap = np.empty(len(order), dtype=np.int64)
    uniq = np.unique(labels)
    remap[order] = np.arange(len(order))
    lut = dict(zip(uniq.tolist(), remap.tolist()))
    return np.array([lut[v] for v in labels.tolist()], dtype=np.int64)


SW_STREAM = [
    (plq.ISING, 2, (16, 16), plq.RELABEL_REDRAW, 0.4406868),
    (plq.ISING, 2, (7, 9), plq.RELABEL_REDRAW, 0.6),
    (plq.ISING, 2, (6, 4, 8), plq.RELABEL_REDRAW, 0.2216544),
    (plq.POTTS, 3, (12, 10), plq.RELABEL_REDRAW, 1.0050),
    (plq.POTTS, 3, (8, 6, 4), plq.RELABEL_FORCED, 0.7),
    (plq.POTTS, 5, (10, 10), plq.RELABEL_REDRAW, 1.2),
    (plq.ISING, 2, (2, 2, 2, 2), plq.RELABEL_REDRAW, 0.3),
    # 64-site tiles spanning whole rows and columns (both wraps inside one tile)
    (plq.ISING, 2, (64, 64), plq.RELABEL_REDRAW, 0.4406868),
    # 32-site tile rows that split the rows, 8-row tiles
    (plq.POTTS, 3, (96, 40), plq.RELABEL_REDRAW, 1.0050),
]


@pytest.mark.parametrize("case", SW_STREAM, ids=lambda c: f"{c[0]}-{c[1]}-{'x'.join(map(str, c[2]))}-{c[3]}")
def test_sw_stream_bit_exact(oracle, gpu, case):
    kind, q, shape, relabel, beta = case
    lat = oracle.Lattice(shape)
    model = _model(oracle, kind, q)
    n = lat.n_sites
    seed = 20260811
    start, off = plq.hot_start(seed, q, n)
    chain = _chain(gpu, kind, q, shape, plq.EXTENT_ALL, relabel, beta, seed, start, plq.RNG_STREAM, off)
    r = oracle.PcgStream(seed)
    r.advance(off)
    want = start.copy()
    for sweep in range(6):
        # the decomposition the CPU makes this sweep, on a copy of its stream
        probe = oracle.PcgStream(state=r.r.state, inc=r.r.inc)
        labels, sizes = oracle.site_clusters(lat, want, model.bond_probability(beta), probe)
        oracle.cluster_sweep(model, lat, want, oracle.ALL, relabel, beta, r)
        got = next(chain)
        assert np.array_equal(got, want), sweep
        assert chain.stream_position() == r.draws
        assert np.array_equal(_compact(chain.labels()), labels)
        hist = chain.size_histogram(24)
        want_hist = np.bincount(np.floor(np.log2(sizes)).astype(int), minlength=24)[:24]
        assert np.array_equal(hist, want_hist)


@pytest.mark.parametrize("relabel,seed", [(plq.RELABEL_REDRAW, 4), (plq.RELABEL_FORCED, 6)])
def test_sw_stream_second_draw_events(oracle, gpu, relabel, seed):
    """rand's range sampler takes a second draw when the low word of x * range
    lands in its rejection zone: probability (range - 1) / 2^32 per draw, and never
    for a power-of-two range.  At beta = 0 every site is its own cluster, so a
    4096^2 lattice draws 2^24 labels per sweep.  With q = 63 these seeds make two
    such draws in the first sweep, so the device re-runs the label draws twice with
    the events known.  States and stream positions stay bit-exact with the CPU."""
    q, shape = 63, (4096, 4096)
    lat = oracle.Lattice(shape)
    model = oracle.Model.potts(q, 1.0)
    n = lat.n_sites
    start, off = plq.hot_start(seed, q, n)
    chain = _chain(gpu, plq.POTTS, q, shape, plq.EXTENT_ALL, relabel, 0.0, seed, start, plq.RNG_STREAM, off)
    r = oracle.PcgStream(seed)
    r.advance(off)
    want = start.copy()
    for sweep in range(2):
        g = want.reshape(shape[1], shape[0]).astype(np.int16)
        agreeing = int((g == np.roll(g, -1, 1)).sum() + (g == np.roll(g, -1, 0)).sum())
        d0 = r.draws
        oracle.cluster_sweep(model, lat, want, oracle.ALL, relabel, 0.0, r)
        if sweep == 0:
            assert r.draws - d0 - agreeing - n == 2  # the two second draws
        got = next(chain)
        assert np.array_equal(got, want), sweep
        assert chain.stream_position() == r.draws


SW_KEYED = [
    (plq.ISING, 2, (16, 16), plq.RELABEL_REDRAW, 0.4406868),
    (plq.ISING, 2, (5, 7), plq.RELABEL_REDRAW, 0.5),
    (plq.ISING, 2, (6, 8, 4), plq.RELABEL_REDRAW, 0.2216544),
    (plq.POTTS, 3, (10, 12), plq.RELABEL_FORCED, 1.0),
    (plq.POTTS, 4, (8, 8, 6), plq.RELABEL_REDRAW, 0.6),
    # tile extents 64 and 32 (whole warps per mask word), with and without wraps inside a tile
    (plq.ISING, 2, (64, 48), plq.RELABEL_REDRAW, 0.4406868),
    (plq.ISING, 2, (128, 64), plq.RELABEL_REDRAW, 0.4406868),
    (plq.ISING, 2, (96, 32, 4), plq.RELABEL_REDRAW, 0.2216544),
    (plq.ISING, 2, (128,), plq.RELABEL_REDRAW, 1.5),
    (plq.POTTS, 3, (64, 96), plq.RELABEL_FORCED, 1.0),
]


@pytest.mark.parametrize("case", SW_KEYED, ids=lambda c: f"{c[0]}-{c[1]}-{'x'.join(map(str, c[2]))}-{c[3]}")
def test_sw_keyed_bit_exact(oracle, gpu, case):
    kind, q, shape, relabel, beta = case
    lat = oracle.Lattice(shape)
    model = _model(oracle, kind, q)
    seed = 77
    start, _ = plq.hot_start(seed, q, lat.n_sites)
    chain = _chain(gpu, kind, q, shape, plq.EXTENT_ALL, relabel, beta, seed, start, plq.RNG_KEYED)
    want = start.copy()
    s32 = oracle.fold_seed(seed)
    for sweep in range(5):
        roots = oracle.keyed_cluster_sweep(model, lat, want, oracle.ALL, relabel, beta, s32, sweep, want_roots=True)
        got = next(chain)
        assert np.array_equal(chain.labels(), roots), sweep
        assert np.array_equal(got, want), sweep


@pytest.mark.parametrize("kind,q,shape,relabel,beta", [
    (plq.ISING, 2, (16, 16), plq.RELABEL_FORCED, 0.4406868),
    (plq.ISING, 2, (8, 8, 8), plq.RELABEL_FORCED, 0.2216544),
    (plq.POTTS, 3, (12, 12), plq.RELABEL_FORCED, 1.0050),
    (plq.POTTS, 3, (9, 7), plq.RELABEL_REDRAW, 0.9),
    (plq.ISING, 2, (2, 4, 2), plq.RELABEL_FORCED, 0.8),
])
def test_wolff_keyed_bit_exact(oracle, gpu, kind, q, shape, relabel, beta):
    lat = oracle.Lattice(shape)
    model = _model(oracle, kind, q)
    seed = 5
    start, _ = plq.hot_start(seed, q, lat.n_sites)
    chain = _chain(gpu, kind, q, shape, plq.EXTENT_SEEDED, relabel, beta, seed, start, plq.RNG_KEYED)
    want = start.copy()
    s32 = oracle.fold_seed(seed)
    for sweep in range(40):
        oracle.keyed_cluster_sweep(model, lat, want, oracle.SEEDED, relabel, beta, s32, sweep)
    chain.advance(40)
    assert np.array_equal(chain.read(), want)


def test_wolff_one_update_at_a_time_equals_batched(gpu):
    start, _ = plq.hot_start(9, 2, 32 * 32)
    a = _chain(gpu, plq.ISING, 2, (32, 32), plq.EXTENT_SEEDED, plq.RELABEL_FORCED, 0.44, 9, start, plq.RNG_KEYED)
    b = _chain(gpu, plq.ISING, 2, (32, 32), plq.EXTENT_SEEDED, plq.RELABEL_FORCED, 0.44, 9, start, plq.RNG_KEYED)
    for _ in range(25):
        next(a)
    b.advance(25)
    assert np.array_equal(a.read(), b.read())
    h = a.size_histogram(16)
    assert h.sum() == 1


@pytest.mark.parametrize("rng", [plq.RNG_STREAM, plq.RNG_KEYED])
def test_beta_zero_opens_no_bond(gpu, rng):
    # gpu_cluster.rs:676-720: at beta = 0 every site is its own cluster
    start, off = plq.hot_start(3, 2, 64 * 64)
    c = _chain(gpu, plq.ISING, 2, (64, 64), plq.EXTENT_ALL, plq.RELABEL_REDRAW, 0.0, 3, start, rng, off)
    next(c)
    assert np.array_equal(c.labels(), np.arange(64 * 64, dtype=np.int32))


def test_large_beta_uniform_field_is_one_cluster(gpu):
    # gpu_cluster.rs:722-770: cold field at large beta -> one cluster, min site 0
    start = np.zeros(128 * 128, dtype=np.uint8)
    c = _chain(gpu, plq.ISING, 2, (128, 128), plq.EXTENT_ALL, plq.RELABEL_REDRAW, 40.0, 1, start, plq.RNG_KEYED)
    out = next(c)
    assert not c.labels().any()
    assert len(np.unique(out)) == 1


def test_pass_cap_error_path(gpu):
    start = np.zeros(64 * 64, dtype=np.uint8)
    c = _chain(gpu, plq.ISING, 2, (64, 64), plq.EXTENT_ALL, plq.RELABEL_REDRAW, 10.0, 1, start, plq.RNG_KEYED,
               flags=plq.FLAG_TINY_PASS_CAP)
    with pytest.raises(plq.PlaquetteError, match="did not converge") as info:
        next(c)
    assert info.value.code == plq.PLQ_ECAP


def test_contracts_on_device(gpu):
    start = np.zeros(16, dtype=np.uint8)
    with pytest.raises(plq.ContractError, match="invariant under relabeling"):
        plq.GpuClusterChain(gpu, plq.make_desc(plq.ISING, 2, (4, 4), plq.CLUSTER, beta=0.4, h=0.1), start)
    with pytest.raises(plq.UnsupportedError):
        _chain(gpu, plq.ISING, 2, (4, 4), plq.EXTENT_SEEDED, plq.RELABEL_FORCED, 0.4, 1, start, plq.RNG_STREAM)


def test_sw_4096sq_stream_matches_oracle(oracle, gpu):
    """Config 3 size: 2D Ising SW on 4096^2 at beta_c from a random start,
    bit-exact with the CPU ClusterUpdate over two sweeps, canonical labels
    and cluster-size histogram included."""
    shape, beta, seed = (4096, 4096), 0.4406868, 20260718
    lat = oracle.Lattice(shape)
    model = oracle.Model.ising(1.0)
    start, off = plq.hot_start(seed, 2, lat.n_sites)
    chain = _chain(gpu, plq.ISING, 2, shape, plq.EXTENT_ALL, plq.RELABEL_REDRAW, beta, seed, start,
                   plq.RNG_STREAM, off)
    r = oracle.PcgStream(seed)
    r.advance(off)
    want = start.copy()
    for sweep in range(2):
        probe = oracle.PcgStream(state=r.r.state, inc=r.r.inc)
        labels, sizes = oracle.site_clusters(lat, want, model.bond_probability(beta), probe)
        oracle.cluster_sweep(model, lat, want, oracle.ALL, oracle.REDRAW, beta, r)
        got = next(chain)
        assert np.array_equal(got, want)
        assert chain.stream_position() == r.draws
        gl = chain.labels()
        # ranks of the canonical roots reproduce the compaction
        roots = np.flatnonzero(gl == np.arange(lat.n_sites))
        rank = np.empty(lat.n_sites, dtype=np.int64)
        rank[roots] = np.arange(len(roots))
        assert np.array_equal(rank[gl], labels)
        want_hist = np.bincount(np.floor(np.log2(sizes)).astype(int), minlength=32)[:32]
        assert np.array_equal(chain.size_histogram(32), want_hist)
