"""Serving: continuous batching of jobs.  Every job's result is the same as
running it alone (bit for bit: its keyed sweep counter and stream position
are its own), jobs that arrive while others run are admitted as memory and
slots free up, admission respects the memory budget, queued jobs cancel."""
import threading
import time

import numpy as np
import pytest

import plaquette_b200 as plq
from plaquette_b200.serving import JOB_CANCELLED, JOB_DONE, Server

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = plq.Gpu.new()
    if g is None:
        pytest.fail("no CUDA device")
    return g


def _jobs():
    specs = [
        (plq.ISING, 2, (64, 64), plq.METROPOLIS, plq.RNG_KEYED, 0.44, 11, 300),
        (plq.ISING, 2, (32, 32, 32), plq.METROPOLIS, plq.RNG_KEYED, 0.2216544, 12, 120),
        (plq.POTTS, 3, (16, 16, 16), plq.HEATBATH, plq.RNG_KEYED, 0.5505, 13, 77),
        (plq.POTTS, 4, (12, 12, 12), plq.HEATBATH, plq.RNG_STREAM, 0.6286, 14, 50),
        (plq.GAUGE, 2, (8, 8, 8, 8), plq.HEATBATH, plq.RNG_KEYED, 0.4407, 15, 40),
        (plq.GAUGE, 2, (6, 6, 6, 6), plq.METROPOLIS, plq.RNG_KEYED, 0.45, 16, 0),
        (plq.ISING, 2, (256, 128), plq.HEATBATH, plq.RNG_STREAM, 0.4406868, 17, 25),
        # generic-body jobs (q = 5; an extent that is not a multiple of four) beside the four-site
        # ones: every tick then makes two launches, the second over item lists that continue the
        # first's
        (plq.POTTS, 5, (10, 10, 10), plq.HEATBATH, plq.RNG_KEYED, 0.62, 18, 90),
        (plq.GAUGE, 2, (6, 6, 6, 6), plq.HEATBATH, plq.RNG_KEYED, 0.45, 19, 60),
    ]
    out = []
    for kind, q, shape, upd, rng, beta, seed, sweeps in specs:
        n = int(np.prod(shape)) * (len(shape) if kind == plq.GAUGE else 1)
        start, off = plq.hot_start(seed, q, n)
        d = plq.make_desc(kind, q, shape, upd, beta=beta, seed=seed, rng=rng, stream_offset=off, sweeps_between=1,
                          batch=1)
        out.append((d, start, sweeps))
    return out


def test_results_alone_equal_results_in_the_mix(gpu):
    jobs = _jobs()
    srv = Server(gpu, 0, 64, 2.0)
    ids = []
    # staggered arrivals: later jobs join while earlier ones are on the GPU
    for d, start, sweeps in jobs:
        ids.append(srv.submit(d, start, sweeps, want_states=True))
        time.sleep(0.002)
    for (d, start, sweeps), jid in zip(jobs, ids):
        assert srv.wait(jid, 120.0) == JOB_DONE
        states, prim, timing = srv.result(jid, states=True)
        alone = plq.GpuChain(gpu, d, start)
        alone.advance(sweeps)
        assert np.array_equal(states, alone.read())
        assert list(prim) == list(alone.primaries())
        assert timing["latency_ms"] >= timing["queue_ms"] >= 0.0
    st = srv.stats()
    assert st["completed"] == len(jobs) and st["p99_ms"] >= st["p50_ms"] > 0
    srv.close()


def test_budget_queues_and_admits_as_memory_frees(gpu):
    jobs = _jobs()
    # room for roughly one 32^3 job at a time: everything still completes
    srv = Server(gpu, 400_000, 64, 2.0)
    ids = [srv.submit(d, s, sw) for d, s, sw in jobs[:4]]
    for jid in ids:
        assert srv.wait(jid, 120.0) == JOB_DONE
    big = plq.make_desc(plq.ISING, 2, (1024, 1024), plq.METROPOLIS, beta=0.44, rng=plq.RNG_KEYED)
    with pytest.raises(plq.PlaquetteError) as info:
        srv.submit(big, None, 10)
    assert info.value.code == plq.PLQ_ENOMEM
    srv.close()


def test_cancel_a_queued_job(gpu):
    srv = Server(gpu, 0, 1, 5.0)  # one slot: the second job waits in the queue
    long = plq.make_desc(plq.ISING, 2, (256, 256, 64), plq.METROPOLIS, beta=0.22, rng=plq.RNG_KEYED)
    a = srv.submit(long, None, 400)
    b = srv.submit(long, None, 5)
    srv.cancel(b)
    assert srv.wait(b, 10.0) == JOB_CANCELLED
    assert srv.wait(a, 120.0) == JOB_DONE
    srv.close()


def test_concurrent_clients(gpu):
    srv = Server(gpu, 0, 16, 2.0)
    results = {}

    def client(k):
        d = plq.make_desc(plq.ISING, 2, (32, 32), plq.METROPOLIS, beta=0.44, seed=k, rng=plq.RNG_KEYED)
        jid = srv.submit(d, None, 20 + k)
        srv.wait(jid, 60.0)
        results[k] = srv.result(jid)[1]

    threads = [threading.Thread(target=client, args=(k,)) for k in range(8)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for k in range(8):
        d = plq.make_desc(plq.ISING, 2, (32, 32), plq.METROPOLIS, beta=0.44, seed=k, rng=plq.RNG_KEYED)
        c = plq.GpuChain(gpu, d, None)
        c.advance(20 + k)
        assert list(results[k]) == list(c.primaries())
    srv.close()
