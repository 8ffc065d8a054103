"""Parity of the CUDA checkerboard sweeps with the oracle, bit for bit.

Stream mode: configurations after N sweeps equal the reference CPU
``LocalUpdate`` checkerboard (src/updater.rs:283-348) driven by the same
PCG64 stream, and the chain consumed exactly as many draws.  Keyed mode:
configurations equal the reference WGSL sweep (src/wgsl/*.wgsl) restated in
the oracle.  Plus the reference's own GPU goldens (src/models/ising/gpu.rs:116-192).
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


def _models(oracle, kind, q, j, h, offsets):
    if kind == plq.ISING:
        return oracle.Model.ising(j, h)
    if kind == plq.POTTS:
        return oracle.Model.potts(q, j, offsets)
    return oracle.Model.gauge(j)


def run_pair(oracle, gpu, kind, q, shape, kernel, rng_mode, beta, sweeps, *, j=1.0, h=0.0, offsets=None,
             seed=20260718, start="hot", sweeps_between=None, flags=0):
    lat = oracle.Lattice(shape, staples=kind == plq.GAUGE)
    model = _models(oracle, kind, q, j, h, offsets)
    n_vars = model.n_vars(lat)
    if start == "hot":
        cfg, offset = plq.hot_start(seed, q, n_vars)
    else:
        cfg, offset = np.zeros(n_vars, dtype=np.uint8), 0
    d = plq.make_desc(kind, q, shape, kernel, beta=beta, j=j, h=h, offsets=offsets, seed=seed, rng=rng_mode,
                      stream_offset=offset, sweeps_between=sweeps_between or sweeps, batch=1, flags=flags)
    chain = plq.GpuChain(gpu, d, cfg)
    got = next(chain)
    want = cfg.copy()
    if rng_mode == plq.RNG_STREAM:
        r = oracle.PcgStream(seed)
        r.advance(offset)
        oracle.local_sweeps(model, lat, want, kernel, beta, r, sweeps)
        assert chain.stream_position() == r.draws
    else:
        s32 = oracle.fold_seed(seed)
        for t in range(sweeps):
            oracle.keyed_local_sweep(model, lat, want, kernel, beta, s32, t)
    return got, want, chain, model, lat


CASES = [
    # kind, q, shape, beta, extra
    (plq.ISING, 2, (16, 16), 0.4406868, {}),
    (plq.ISING, 2, (8, 6), 0.3, {"h": 0.25}),
    (plq.ISING, 2, (32,), 0.7, {}),
    (plq.ISING, 2, (4, 6, 8), 0.2216544, {}),
    (plq.ISING, 2, (4, 4, 4, 4), 0.15, {"j": 0.75, "h": -0.1}),
    (plq.ISING, 2, (2, 2, 2, 2, 2, 2), 0.1, {}),
    (plq.POTTS, 2, (10, 8), 0.9, {}),
    (plq.POTTS, 3, (12, 10), 1.0050, {}),
    (plq.POTTS, 3, (8, 8, 6), 0.5505, {}),
    (plq.POTTS, 3, (6, 4), 0.8, {"offsets": [0.3, -0.2, 0.1]}),
    (plq.POTTS, 4, (6, 6, 4), 0.62, {}),
    (plq.POTTS, 4, (8, 6, 4), 0.62, {"offsets": [0.1, 0.0, -0.2, 0.05]}),
    (plq.POTTS, 5, (8, 8), 1.1, {"j": 1.5}),
    (plq.GAUGE, 2, (8, 8), 0.7, {}),
    (plq.GAUGE, 2, (4, 4, 6), 0.6, {}),
    (plq.GAUGE, 2, (4, 4, 4, 4), 0.4407, {}),
    (plq.GAUGE, 2, (2, 4, 2), 0.9, {"j": 1.25}),
]


@pytest.mark.parametrize("rng_mode", [plq.RNG_STREAM, plq.RNG_KEYED], ids=["stream", "keyed"])
@pytest.mark.parametrize("kernel", [plq.METROPOLIS, plq.HEATBATH], ids=["metropolis", "heatbath"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{['ising','potts','gauge'][c[0]]}{c[1]}-{'x'.join(map(str, c[2]))}")
def test_sweeps_bit_exact(oracle, gpu, case, kernel, rng_mode):
    kind, q, shape, beta, extra = case
    got, want, *_ = run_pair(oracle, gpu, kind, q, shape, kernel, rng_mode, beta, 7, **extra)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("rng_mode", [plq.RNG_STREAM, plq.RNG_KEYED], ids=["stream", "keyed"])
def test_config1_64sq_cold_critical_10k_sweeps(oracle, gpu, rng_mode):
    """2D Ising 64x64, cold, J=1, h=0, beta_c, checkerboard Metropolis, 10^4
    sweeps (10^3 thermalisation), E and |M| every 10 sweeps: every sample's
    integer primaries and the final configuration bit-exact."""
    beta, seed = 0.4406868, 20260718
    lat = oracle.Lattice((64, 64))
    model = oracle.Model.ising(1.0, 0.0)
    d = plq.make_desc(plq.ISING, 2, (64, 64), plq.METROPOLIS, beta=beta, seed=seed, rng=rng_mode,
                      sweeps_between=10, batch=64)
    cfg = np.zeros(4096, dtype=np.uint8)
    chain = plq.GpuChain(gpu, d, cfg)
    chain.advance(1000)
    states, prims = chain.next_batch(900, states=False)
    want = cfg.copy()
    r = oracle.PcgStream(seed)
    s32 = oracle.fold_seed(seed)
    sweep = 0

    def sweeps(n):
        nonlocal sweep
        if rng_mode == plq.RNG_STREAM:
            oracle.local_sweeps(model, lat, want, plq.METROPOLIS, beta, r, n)
        else:
            for _ in range(n):
                oracle.keyed_local_sweep(model, lat, want, plq.METROPOLIS, beta, s32, sweep)
                sweep += 1

    sweeps(1000)
    for k in range(900):
        sweeps(10)
        assert list(prims[k]) == list(model.primaries(lat, want)), k
    assert np.array_equal(chain.read(), want)
    if rng_mode == plq.RNG_STREAM:
        assert chain.stream_position() == r.draws


@pytest.mark.parametrize("rng_mode", [plq.RNG_STREAM, plq.RNG_KEYED])
def test_a_launch_spanning_many_chunks_reaches_every_site(gpu, rng_mode):
    # src/models/ising/gpu.rs:160-192: j = 0, h = -1, cold, one sweep => M = -N.
    shape = (2048, 2048)
    d = plq.make_desc(plq.ISING, 2, shape, plq.METROPOLIS, beta=1.0, j=0.0, h=-1.0, seed=7, rng=rng_mode,
                      sweeps_between=1, batch=1)
    chain = plq.GpuChain(gpu, d, np.zeros(2048 * 2048, dtype=np.uint8))
    _, prim = chain.next_sample()
    assert prim[1] == -(2048 * 2048)


def test_zero_sweep_round_trip(gpu):
    # src/models/ising/gpu.rs:116-140
    start, _ = plq.hot_start(0, 2, 16)
    chain = plq.ising.gpu_chain(gpu, (4, 4), 1.0, 0.0, 0.5, 7, start, 0, 1, plq.METROPOLIS)
    assert np.array_equal(next(chain), start)
    links = (np.arange(4 * 4 * 3 * 2) % 2).astype(np.uint8)
    gchain = plq.gauge.gpu_chain(gpu, (4, 4, 2), 1.0, 0.5, 7, links[: 4 * 4 * 2 * 3], 0, 1, plq.HEATBATH)
    assert np.array_equal(next(gchain), links[: 4 * 4 * 2 * 3])


def test_odd_extent_rejected(gpu):
    # src/models/potts/gpu.rs:427-449
    with pytest.raises(plq.ContractError, match="even lattice extents"):
        plq.potts.gpu_chain(gpu, (5, 4), 3, 1.0, None, 0.5, 1, np.zeros(20, np.uint8), 1, 1, plq.HEATBATH)


def test_primaries_match_oracle(oracle, gpu):
    for kind, q, shape in [(plq.ISING, 2, (6, 4, 2)), (plq.POTTS, 4, (8, 6)), (plq.GAUGE, 2, (4, 2, 4, 2))]:
        got, want, chain, model, lat = run_pair(oracle, gpu, kind, q, shape, plq.HEATBATH, plq.RNG_STREAM, 0.5, 3)
        assert np.array_equal(got, want)
        assert list(chain.primaries()) == list(model.primaries(lat, want))


@pytest.mark.parametrize("shape", [(32, 6), (16, 4, 6), (48, 2, 2)])
@pytest.mark.parametrize("q", [0, 2, 3, 4, 5, 6, 7, 8])
def test_vector_primaries_match_oracle(oracle, gpu, q, shape):
    # extent 0 a multiple of 16: the 16-site vector counting path, every label count
    n = int(np.prod(shape))
    rng = np.random.default_rng(100 + q)
    for trial in range(3):
        if q == 0:
            kind, qq, model = plq.ISING, 2, oracle.Model.ising(1.0, 0.0)
        else:
            kind, qq, model = plq.POTTS, q, oracle.Model.potts(q, 1.0)
        start = rng.integers(0, qq, n).astype(np.uint8) if trial else np.full(n, qq - 1, np.uint8)
        d = plq.make_desc(kind, qq, shape, plq.METROPOLIS, beta=0.5, seed=1, rng=plq.RNG_KEYED)
        chain = plq.GpuChain(gpu, d, start)
        assert list(chain.primaries()) == list(model.primaries(oracle.Lattice(shape), start)), (q, shape, trial)
        chain.close()


def test_energy_matches_oracle_energy(oracle, gpu):
    # E from the integer primaries, as Ising::energy forms it (ising/mod.rs:116)
    got, want, chain, model, lat = run_pair(oracle, gpu, plq.ISING, 2, (12, 8), plq.METROPOLIS, plq.RNG_STREAM, 0.3,
                                            5, j=1.5, h=0.25)
    bond, spin = chain.primaries()
    assert -1.5 * float(bond) - 0.25 * float(spin) == model.energy(lat, want)


@pytest.mark.parametrize("kernel", [plq.METROPOLIS, plq.HEATBATH])
def test_large_lattice_stream_parity(oracle, gpu, kernel):
    got, want, *_ = run_pair(oracle, gpu, plq.ISING, 2, (256, 128, 8), kernel, plq.RNG_STREAM, 0.2216544, 3)
    assert np.array_equal(got, want)


def test_batch_samples_equal_sequential(oracle, gpu):
    d = plq.make_desc(plq.POTTS, 3, (16, 16), plq.HEATBATH, beta=1.0, seed=3, rng=plq.RNG_STREAM,
                      sweeps_between=2, batch=8)
    start, off = plq.hot_start(3, 3, 256)
    d.stream_offset = off
    a = plq.GpuChain(gpu, d, start)
    samples = [next(a) for _ in range(10)]
    lat = oracle.Lattice((16, 16))
    model = oracle.Model.potts(3, 1.0)
    r = oracle.PcgStream(3)
    r.advance(off)
    want = start.copy()
    for s in samples:
        oracle.local_sweeps(model, lat, want, plq.HEATBATH, 1.0, r, 2)
        assert np.array_equal(s, want)


WORD_CASES = [
    (plq.ISING, 2, (256, 128), plq.METROPOLIS, plq.RNG_KEYED, 0.4406868),
    (plq.ISING, 2, (32, 24, 16), plq.HEATBATH, plq.RNG_STREAM, 0.2216544),
    (plq.ISING, 2, (12, 8, 6, 4), plq.HEATBATH, plq.RNG_KEYED, 0.15),
    (plq.ISING, 2, (4, 6, 8), plq.METROPOLIS, plq.RNG_KEYED, 0.3),
    (plq.POTTS, 3, (40, 36), plq.HEATBATH, plq.RNG_STREAM, 1.0050),
    (plq.POTTS, 3, (24, 16, 10), plq.HEATBATH, plq.RNG_KEYED, 0.5505),
    (plq.POTTS, 3, (8, 6, 4, 4), plq.HEATBATH, plq.RNG_STREAM, 0.4),
    (plq.POTTS, 2, (128,), plq.HEATBATH, plq.RNG_STREAM, 0.9),
    (plq.POTTS, 4, (16, 12), plq.HEATBATH, plq.RNG_STREAM, 1.1),
    (plq.POTTS, 4, (8, 8, 8), plq.HEATBATH, plq.RNG_KEYED, 0.62),
    (plq.POTTS, 4, (4, 4, 4, 4), plq.HEATBATH, plq.RNG_STREAM, 0.5),
    (plq.GAUGE, 2, (16, 12), plq.HEATBATH, plq.RNG_STREAM, 0.7),
    (plq.GAUGE, 2, (12, 8, 6), plq.METROPOLIS, plq.RNG_KEYED, 0.6),
    (plq.GAUGE, 2, (16, 16, 16, 16), plq.HEATBATH, plq.RNG_STREAM, 0.4407),
    (plq.GAUGE, 2, (12, 4, 6, 8), plq.HEATBATH, plq.RNG_KEYED, 0.5),
    (plq.GAUGE, 2, (4, 4, 4, 4), plq.METROPOLIS, plq.RNG_KEYED, 0.44),
]


@pytest.mark.parametrize("case", WORD_CASES, ids=lambda c: f"{['ising','potts','gauge'][c[0]]}{c[1]}-"
                         f"{'x'.join(map(str, c[2]))}-{'metro' if c[3] == plq.METROPOLIS else 'hb'}-"
                         f"{'stream' if c[4] == plq.RNG_STREAM else 'keyed'}")
def test_word_passes_equal_generic(gpu, case):
    # four sites at a time (extent 0 a multiple of 4) == one variable per rank, bit for bit
    kind, q, shape, kernel, rng_mode, beta = case
    n_vars = int(np.prod(shape)) * (len(shape) if kind == plq.GAUGE else 1)
    start, off = plq.hot_start(77, q, n_vars)
    outs = []
    # (q = 2 keyed sites with extent 0 a multiple of 64 would take the bit-packed passes)
    for flags in (plq.FLAG_NO_PACKED, plq.FLAG_GENERIC_PASS):
        d = plq.make_desc(kind, q, shape, kernel, beta=beta, seed=77, rng=rng_mode, stream_offset=off,
                          sweeps_between=5, batch=1, flags=flags)
        c = plq.GpuChain(gpu, d, start)
        assert c.path == ("words" if flags == plq.FLAG_NO_PACKED else "pass")
        outs.append((next(c), c.stream_position() if rng_mode == plq.RNG_STREAM else 0, list(c.primaries())))
        c.close()
    assert np.array_equal(outs[0][0], outs[1][0])
    assert outs[0][1:] == outs[1][1:]


@pytest.mark.parametrize("pos", [0, 7, 63, 64, 65, 1000, 4095])
@pytest.mark.parametrize("bad", [2, 3, 127, 128, 255])
def test_out_of_range_start_state_refused(gpu, pos, bad):
    # State::new refuses an index >= q: the first offending variable is named
    start = np.ones(64 * 64, dtype=np.uint8)
    start[pos] = bad
    if pos + 3 < start.size:
        start[pos + 3] = 200  # a later offender does not mask the first
    d = plq.make_desc(plq.ISING, 2, (64, 64), plq.METROPOLIS, beta=0.4, seed=1, rng=plq.RNG_KEYED)
    with pytest.raises(plq.PlaquetteError, match=f"start variable {pos} holds state {bad}, not below q = 2"):
        plq.GpuChain(gpu, d, start)
    ok = np.ones(64 * 64, dtype=np.uint8)
    plq.GpuChain(gpu, d, ok).close()


def test_chain_outlives_its_context():
    """A garbage collector may finalize a context before a chain made from it
    (a chain kept alive by a traceback cycle, say).  The chain copies the
    context's record when it is created, so it keeps running after the
    context is destroyed, and a new context's chains run cleanly after it."""
    g = plq.Gpu.new()
    d = plq.make_desc(plq.ISING, 2, (64, 64), plq.METROPOLIS, beta=0.44, seed=1, rng=plq.RNG_KEYED,
                      sweeps_between=1, batch=1)
    c = plq.GpuChain(g, d, None)
    c.advance(2)
    plq.lib().plq_ctx_destroy(g._h)  # the context goes first
    g._h = None
    c.advance(2)
    first = next(c)
    c.close()
    g2 = plq.Gpu.new()
    c2 = plq.GpuChain(g2, d, None)
    c2.advance(4)
    assert np.array_equal(next(c2), first)  # same seed, same keyed sweeps
    c2.close()


def test_potts_stream_metropolis_second_draw(oracle, gpu):
    """Potts Metropolis on the PCG stream draws its proposal with
    next_below(q - 1) (src/updater.rs:659-668), which takes a second draw when
    the first lands in rand's rejection zone (probability (q - 2) / 2^32).  At
    seed 13 the draw at stream position 7064085 does so for q = 64, so a chain
    starting there must consume it on its first proposal -- and stay bit-exact
    with the CPU walk, configurations and stream position."""
    q, shape, seed, offset, beta = 64, (8, 8), 13, 7064085, 0.9
    probe = oracle.PcgStream(seed)
    probe.advance(offset)
    probe.next_below(q - 1)
    assert probe.draws == offset + 2  # the first proposal takes two draws
    lat = oracle.Lattice(shape)
    model = oracle.Model.potts(q, 1.0)
    start = np.random.default_rng(5).integers(0, q, 64).astype(np.uint8)
    d = plq.make_desc(plq.POTTS, q, shape, plq.METROPOLIS, beta=beta, seed=seed, rng=plq.RNG_STREAM,
                      stream_offset=offset, sweeps_between=3, batch=1)
    chain = plq.GpuChain(gpu, d, start)
    got = next(chain)
    r = oracle.PcgStream(seed)
    r.advance(offset)
    want = start.copy()
    oracle.local_sweeps(model, lat, want, plq.METROPOLIS, beta, r, 3)
    assert np.array_equal(got, want)
    assert chain.stream_position() == r.draws


@pytest.mark.parametrize("q,shape", [(3, (64, 32)), (4, (16, 8, 8)), (7, (6, 6, 4, 4))], ids=str)
def test_potts_stream_metropolis_larger_lattices(oracle, gpu, q, shape):
    """The sequential walk over groups of 32 ranks, with a partial last group,
    across many sweeps; the q = 3 heat bath beside it is unchanged."""
    got, want, chain, *_ = run_pair(oracle, gpu, plq.POTTS, q, shape, plq.METROPOLIS, plq.RNG_STREAM, 0.8, 5)
    assert chain.path == "lookback"
    assert np.array_equal(got, want)
