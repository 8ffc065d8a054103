"""Checkpoint and resume on the keyed stream.

A keyed chain's RNG key is its sweep counter (src/device.rs:216-217, the
`sweeps_done` passed to every sweep).  A run of 10 sweeps must equal a run
of 5, a read-back of the configuration (the checkpoint), a new chain made
from it with sweep_offset = 5, and 5 more sweeps -- for local chains (fused
and per-colour paths), Swendsen-Wang and Wolff cluster chains, ensembles and
server jobs.  On the PCG stream the checkpoint is (configuration, stream
position), which stream_offset already resumes.
"""
import numpy as np
import pytest

import plaquette_b200 as plq
from plaquette_b200.ensemble import Ensemble
from plaquette_b200.serving import JOB_DONE, Server

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = plq.Gpu.new()
    if g is None:
        pytest.fail("no CUDA device")
    return g


LOCAL = [
    (plq.ISING, 2, (128, 64, 16), plq.METROPOLIS, 0.2216544, 0),   # fused 3D
    (plq.POTTS, 3, (40, 24), plq.HEATBATH, 1.005, 0),               # per-colour passes
    (plq.GAUGE, 2, (6, 6, 6, 6), plq.HEATBATH, 0.44, 0),            # links
    (plq.ISING, 2, (64, 32), plq.METROPOLIS, 0.44, plq.FLAG_GENERIC_PASS),
]


@pytest.mark.parametrize("case", LOCAL, ids=lambda c: f"{c[0]}-{c[1]}-{'x'.join(map(str, c[2]))}-{c[5]}")
def test_keyed_local_chain_resumes(gpu, case):
    kind, q, shape, kernel, beta, flags = case
    n_vars = int(np.prod(shape)) * (len(shape) if kind == plq.GAUGE else 1)
    start, _ = plq.hot_start(31, q, n_vars)

    def chain(st, offset):
        d = plq.make_desc(kind, q, shape, kernel, beta=beta, seed=31, rng=plq.RNG_KEYED, sweeps_between=1, batch=1,
                          flags=flags, sweep_offset=offset)
        return plq.GpuChain(gpu, d, st)

    whole = chain(start, 0)
    whole.advance(10)
    want = whole.read()
    assert whole.sweeps_done == 10

    first = chain(start, 0)
    first.advance(5)
    checkpoint = first.read()
    first.close()
    second = chain(checkpoint, 5)
    assert second.sweeps_done == 5
    second.advance(5)
    assert second.sweeps_done == 10
    assert np.array_equal(second.read(), want)
    assert list(second.primaries()) == list(whole.primaries())


@pytest.mark.parametrize("extent", [plq.EXTENT_ALL, plq.EXTENT_SEEDED], ids=["sw", "wolff"])
def test_keyed_cluster_chain_resumes(gpu, extent):
    shape = (64, 64)
    start, _ = plq.hot_start(8, 2, 64 * 64)
    relabel = plq.RELABEL_REDRAW if extent == plq.EXTENT_ALL else plq.RELABEL_FORCED

    def chain(st, offset):
        d = plq.make_desc(plq.ISING, 2, shape, plq.CLUSTER, beta=0.44, seed=8, rng=plq.RNG_KEYED, sweeps_between=1,
                          batch=1, extent=extent, relabel=relabel, sweep_offset=offset)
        return plq.GpuClusterChain(gpu, d, st)

    whole = chain(start, 0)
    whole.advance(10)
    first = chain(start, 0)
    first.advance(5)
    second = chain(first.read(), 5)
    second.advance(5)
    assert np.array_equal(second.read(), whole.read())


def _members():
    descs, starts = [], []
    for m, (shape, beta) in enumerate([((16, 16, 16), 0.22), ((12, 12, 12), 0.21), ((8, 8, 8, 8), 0.45)]):
        gauge = len(shape) == 4
        n_vars = int(np.prod(shape)) * (4 if gauge else 1)
        descs.append(((plq.GAUGE if gauge else plq.ISING), shape, beta, 40 + m))
        starts.append(plq.hot_start(40 + m, 2, n_vars)[0])
    return descs, starts


def _ens(gpu, descs, starts, offset):
    ds = [plq.make_desc(k, 2, shape, plq.HEATBATH if k == plq.GAUGE else plq.METROPOLIS, beta=beta, seed=seed,
                        rng=plq.RNG_KEYED, sweeps_between=1, batch=1, sweep_offset=offset)
          for (k, shape, beta, seed) in descs]
    return Ensemble(gpu, ds, starts)


def test_ensemble_resumes(gpu):
    descs, starts = _members()
    whole = _ens(gpu, descs, starts, 0)
    whole.advance(10)
    first = _ens(gpu, descs, starts, 0)
    first.advance(5)
    checkpoint = [first.read(m) for m in range(first.n)]
    second = _ens(gpu, descs, checkpoint, 5)
    second.advance(5)
    for m in range(whole.n):
        assert np.array_equal(second.read(m), whole.read(m)), m


def test_ensemble_refuses_unequal_offsets(gpu):
    ds = [plq.make_desc(plq.ISING, 2, (8, 8), plq.METROPOLIS, beta=0.4, seed=1, rng=plq.RNG_KEYED, batch=1,
                        sweep_offset=o) for o in (0, 3)]
    with pytest.raises(plq.ContractError, match="share one sweep counter"):
        Ensemble(gpu, ds, [None, None])


def test_server_job_resumes(gpu):
    shape, beta, seed = (32, 32, 32), 0.2216544, 77
    start, _ = plq.hot_start(seed, 2, 32 ** 3)

    def desc(offset):
        return plq.make_desc(plq.ISING, 2, shape, plq.METROPOLIS, beta=beta, seed=seed, rng=plq.RNG_KEYED,
                             batch=1, sweep_offset=offset)

    s = Server(gpu)
    try:
        j_whole = s.submit(desc(0), start, 10, want_states=True)
        j_first = s.submit(desc(0), start, 5, want_states=True)
        assert s.wait(j_whole, 60.0) == JOB_DONE and s.wait(j_first, 60.0) == JOB_DONE
        whole = s.result(j_whole, states=True)[0]
        checkpoint = s.result(j_first, states=True)[0]
        j_second = s.submit(desc(5), checkpoint, 5, want_states=True)
        assert s.wait(j_second, 60.0) == JOB_DONE
        assert np.array_equal(s.result(j_second, states=True)[0], whole)
    finally:
        s.close()
