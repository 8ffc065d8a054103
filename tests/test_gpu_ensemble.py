"""Batched ensembles: every member evolves exactly as its own chain would,
batched (one persistent graph-captured launch) or unbatched (one launch per
member per colour pass); parallel tempering gives identical results on both
paths; the autotuner leaves the ensemble's state untouched."""
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


def _members():
    specs = [
        (plq.ISING, 2, (16, 16, 16), plq.METROPOLIS, plq.RNG_KEYED, 0.2216544, 1),
        (plq.ISING, 2, (24, 24, 24), plq.HEATBATH, plq.RNG_KEYED, 0.21, 2),
        (plq.POTTS, 3, (8, 8, 8), plq.HEATBATH, plq.RNG_STREAM, 0.5505, 3),
        (plq.GAUGE, 2, (4, 4, 4, 4), plq.HEATBATH, plq.RNG_KEYED, 0.44, 4),
        (plq.GAUGE, 2, (6, 6, 6, 6), plq.HEATBATH, plq.RNG_STREAM, 0.40, 5),
        (plq.ISING, 2, (32, 16), plq.METROPOLIS, plq.RNG_KEYED, 0.4406868, 6),
        (plq.POTTS, 4, (8, 6, 4), plq.METROPOLIS, plq.RNG_KEYED, 0.62, 7),
    ]
    descs, starts = [], []
    for kind, q, shape, upd, rng, beta, seed in specs:
        n = int(np.prod(shape)) * (len(shape) if kind == plq.GAUGE else 1)
        start, off = plq.hot_start(seed, q, n)
        descs.append(plq.make_desc(kind, q, shape, upd, beta=beta, seed=seed, rng=rng, stream_offset=off,
                                   sweeps_between=1, batch=1))
        starts.append(start)
    return descs, starts


def test_members_match_their_own_chains(gpu):
    descs, starts = _members()
    ens = Ensemble(gpu, descs, starts)
    chains = [plq.GpuChain(gpu, d, s) for d, s in zip(descs, starts)]
    ens.advance(7)
    for c in chains:
        c.advance(7)
    for m, c in enumerate(chains):
        assert np.array_equal(ens.read(m), c.read()), m
        assert list(ens.primaries(m)) == list(c.primaries()), m
    ens.advance_unbatched(5)
    for c in chains:
        c.advance(5)
    for m, c in enumerate(chains):
        assert np.array_equal(ens.read(m), c.read()), m
    ens.advance(3)
    ens.advance(3)  # graph replay
    for c in chains:
        c.advance(6)
    for m, c in enumerate(chains):
        assert np.array_equal(ens.read(m), c.read()), m


def _ladder_ensemble(gpu, L=8, k=8, every=2):
    betas = list(np.geomspace(0.20, 0.24, k))
    descs, starts = [], []
    for i in range(k):
        start, _ = plq.hot_start(100 + i, 2, L ** 3)
        descs.append(plq.make_desc(plq.ISING, 2, (L, L, L), plq.METROPOLIS, beta=betas[i], seed=100 + i,
                                   rng=plq.RNG_KEYED, sweeps_between=1, batch=1))
        starts.append(start)
    ens = Ensemble(gpu, descs, starts)
    ens.add_ladder(list(range(k)), betas, every, seed=42)
    return ens, betas


def test_tempering_batched_equals_unbatched(gpu):
    a, betas = _ladder_ensemble(gpu)
    b, _ = _ladder_ensemble(gpu)
    a.advance(20)
    b.advance_unbatched(20)
    assert np.array_equal(a.betas(), b.betas())
    for m in range(8):
        assert np.array_equal(a.read(m), b.read(m)), m
    ba = a.betas()
    assert sorted(ba.tolist()) == sorted(betas)
    assert not np.array_equal(ba, np.array(betas)), "no swap was accepted in 10 attempts"


def test_tune_keeps_state(gpu):
    descs, starts = _members()
    ens = Ensemble(gpu, descs, starts)
    ens.advance(2)
    before = [ens.read(m) for m in range(len(descs))]
    r, c, ms = ens.tune(3)
    assert r in (2, 4, 8) and c >= 1 and ms > 0
    after = [ens.read(m) for m in range(len(descs))]
    for x, y in zip(before, after):
        assert np.array_equal(x, y)
    chains = [plq.GpuChain(gpu, d, s) for d, s in zip(descs, starts)]
    ens.advance(4)
    for m, ch in enumerate(chains):
        ch.advance(6)
        assert np.array_equal(ens.read(m), ch.read()), m


def test_four_site_members_match_their_own_chains(gpu):
    # every member eligible for the four-sites-at-a-time body: the ensemble runs its
    # words-only kernel, and each member still equals its own chain
    specs = [
        (plq.ISING, 2, (16, 16, 16), plq.METROPOLIS, plq.RNG_KEYED, 0.2216544, 11),
        (plq.ISING, 2, (24, 12, 8), plq.HEATBATH, plq.RNG_STREAM, 0.21, 12),
        (plq.POTTS, 3, (12, 8, 8), plq.HEATBATH, plq.RNG_KEYED, 0.5505, 13),
        (plq.GAUGE, 2, (8, 8, 8, 8), plq.HEATBATH, plq.RNG_KEYED, 0.44, 14),
        (plq.GAUGE, 2, (12, 4, 4, 8), plq.HEATBATH, plq.RNG_STREAM, 0.40, 15),
        (plq.GAUGE, 2, (4, 6, 6), plq.METROPOLIS, plq.RNG_KEYED, 0.7, 16),
    ]
    descs, starts = [], []
    for kind, q, shape, upd, rng, beta, seed in specs:
        n = int(np.prod(shape)) * (len(shape) if kind == plq.GAUGE else 1)
        start, off = plq.hot_start(seed, q, n)
        descs.append(plq.make_desc(kind, q, shape, upd, beta=beta, seed=seed, rng=rng, stream_offset=off,
                                   sweeps_between=1, batch=1))
        starts.append(start)
    ens = Ensemble(gpu, descs, starts)
    chains = [plq.GpuChain(gpu, d, s) for d, s in zip(descs, starts)]
    for c in chains:
        assert c.path == "words"
    ens.advance(6)
    for c in chains:
        c.advance(6)
    for m, c in enumerate(chains):
        assert np.array_equal(ens.read(m), c.read()), m
    for r, k in ((2, 1), (4, 2), (8, 1)):
        ens.set_config(r, k)
        ens.advance(2)
    for c in chains:
        c.advance(6)
    for m, c in enumerate(chains):
        assert np.array_equal(ens.read(m), c.read()), m


def test_primaries_of_every_member_at_once(gpu):
    descs, starts = _members()
    # members larger than one measurement work item (16384 sites): several items each
    for kind, q, shape, seed in ((plq.ISING, 2, (64, 64, 8), 8), (plq.POTTS, 3, (40, 40, 20), 9),
                                 (plq.GAUGE, 2, (12, 12, 12, 12), 10)):
        n = int(np.prod(shape)) * (len(shape) if kind == plq.GAUGE else 1)
        start, off = plq.hot_start(seed, q, n)
        descs.append(plq.make_desc(kind, q, shape, plq.HEATBATH, beta=0.3, seed=seed, rng=plq.RNG_KEYED,
                                   stream_offset=off, sweeps_between=1, batch=1))
        starts.append(start)
    ens = Ensemble(gpu, descs, starts)
    for sweeps in (0, 4, 3):
        ens.advance(sweeps) if sweeps else None
        every = ens.primaries_all()
        assert len(every) == ens.n
        for m in range(ens.n):
            assert list(every[m]) == list(ens.primaries(m)), (sweeps, m)


def test_tuner_chooses_a_shape_per_member_shape(gpu):
    """The autotuner picks four-site words per thread for every member shape
    (timed alone), records them in the process-wide table, and a later
    ensemble of those shapes starts from them; results stay those of each
    member's own chain."""
    from plaquette_b200.ensemble import tune_entries

    specs = [((16, 16, 16), plq.ISING, plq.METROPOLIS, 0.22), ((8, 8, 8, 8), plq.GAUGE, plq.HEATBATH, 0.44),
             ((32, 32), plq.ISING, plq.HEATBATH, 0.44)]
    names = {plq.ISING: "ising", plq.GAUGE: "gauge"}
    upds = {plq.METROPOLIS: "metropolis", plq.HEATBATH: "heatbath"}
    descs, starts = [], []
    for i, (shape, kind, upd, beta) in enumerate(specs * 2):
        n = int(np.prod(shape)) * (len(shape) if kind == plq.GAUGE else 1)
        starts.append(plq.hot_start(70 + i, 2, n)[0])
        descs.append(plq.make_desc(kind, 2, shape, upd, beta=beta, seed=70 + i, rng=plq.RNG_KEYED, batch=1))
    ens = Ensemble(gpu, descs, starts)
    ens.tune(3)
    table = {(e["model"], tuple(e["shape"]), e["updater"]): e for e in tune_entries()}
    for shape, kind, upd, _ in specs:
        key = (names[kind], shape, upds[upd])
        assert key in table, key
        assert table[key]["words_per_thread"] in (1, 2, 4, 8) and table[key]["members"] == 2
        assert table[key]["ms_per_sweep_alone"] > 0
    for m, d in enumerate(descs):
        key = (names[d.model], tuple(d.shape[: d.d]), upds[d.updater])
        assert ens.member_config(m) == table[key]["words_per_thread"]
    later = Ensemble(gpu, descs, starts)
    assert [later.member_config(m) for m in range(len(descs))] == [ens.member_config(m) for m in range(len(descs))]
    chains = [plq.GpuChain(gpu, d, s) for d, s in zip(descs, starts)]
    ens.advance(5)
    later.advance(5)
    for m, c in enumerate(chains):
        c.advance(5)
        assert np.array_equal(ens.read(m), c.read()), m
        assert np.array_equal(later.read(m), c.read()), m
    # after a batched launch, tuning: its trial launches move the packed rows and it restores the
    # bytes, so the primaries of every member at once must come from the bytes again
    later.tune(3)
    every = later.primaries_all()
    for m in range(later.n):
        assert list(every[m]) == list(later.primaries(m)), m


@pytest.mark.parametrize("spec", [
    (plq.ISING, 2, (48, 16, 8), plq.METROPOLIS, 0.2216544),   # 64-bit rows
    (plq.ISING, 2, (64, 64), plq.HEATBATH, 0.44),             # 64-bit rows, 2D
    (plq.POTTS, 2, (40, 12, 6), plq.HEATBATH, 0.9),           # Potts at q = 2: agreement energy
    (plq.ISING, 2, (2, 6, 4), plq.METROPOLIS, 0.5),           # rows of two sites
    (plq.GAUGE, 2, (2, 4, 2, 4), plq.HEATBATH, 0.6),          # rows of two links
    (plq.GAUGE, 2, (32, 4, 4), plq.METROPOLIS, 0.8),          # full 32-bit rows
], ids=lambda s: f"{s[0]}-{'x'.join(map(str, s[2]))}")
def test_packed_members_match_their_own_chains(gpu, spec):
    """Keyed q = 2 sites and Z2 links run as packed rows inside the persistent
    launch (the per-member chain runs the byte passes): identical
    configurations and primaries, and the same under a tempering ladder,
    whose energies the launch reads from the packed rows."""
    kind, q, shape, upd, beta = spec
    n = int(np.prod(shape)) * (len(shape) if kind == plq.GAUGE else 1)
    descs, starts = [], []
    for k in range(3):
        starts.append(plq.hot_start(90 + k, q, n)[0])
        descs.append(plq.make_desc(kind, q, shape, upd, beta=beta * (1 + 0.05 * k), seed=90 + k, rng=plq.RNG_KEYED,
                                   batch=1))
    ens = Ensemble(gpu, descs, starts)
    chains = [plq.GpuChain(gpu, d, s) for d, s in zip(descs, starts)]
    ens.advance(7)
    for m, c in enumerate(chains):
        c.advance(7)
        assert np.array_equal(ens.read(m), c.read()), m
        assert list(ens.primaries(m)) == list(c.primaries()), m
    # a ladder over the same members: batched (packed, energies from packed rows) == per-lattice (bytes)
    a = Ensemble(gpu, descs, starts)
    b = Ensemble(gpu, descs, starts)
    for e in (a, b):
        e.add_ladder([0, 1, 2], [beta, beta * 1.05, beta * 1.1], 2, seed=3)
    a.advance(12)
    b.advance_unbatched(12)
    assert np.array_equal(a.betas(), b.betas())
    for m in range(3):
        assert np.array_equal(a.read(m), b.read(m)), m
    # primaries of every member at once: a's from the packed rows its launch left, b's from the
    # bytes the per-lattice launches wrote; both equal the byte scan of each member
    pa, pb = a.primaries_all(), b.primaries_all()
    for m in range(3):
        assert list(pa[m]) == list(pb[m]) == list(a.primaries(m)), m


def test_out_of_range_start_is_refused(gpu):
    """A start state >= q in any member (checked on the host threads before
    anything is allocated) refuses the whole ensemble."""
    descs, starts = [], []
    for k, shape in enumerate(((16, 16, 16), (8, 8, 8), (32, 16))):
        n = int(np.prod(shape))
        starts.append(plq.hot_start(200 + k, 2, n)[0])
        descs.append(plq.make_desc(plq.ISING, 2, shape, plq.METROPOLIS, beta=0.3, seed=200 + k, rng=plq.RNG_KEYED,
                                   batch=1))
    Ensemble(gpu, descs, starts).close()
    bad = [s.copy() for s in starts]
    bad[1][37] = 2
    with pytest.raises(plq.PlaquetteError, match="start state out of range"):
        Ensemble(gpu, descs, bad)
