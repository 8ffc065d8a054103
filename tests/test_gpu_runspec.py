"""A run configuration in the reference's TOML vocabulary executed on the
device: the CPU-backend checkerboard run equals the oracle's chain from the
same seed (hot start drawn first, the generator continuing into the chain),
sample for sample; a GPU-backend run submitted to the serving loop ends where
its own chain ends."""
import numpy as np
import pytest

import plaquette_b200 as plq
from plaquette_b200 import runspec
from plaquette_b200.serving import Server

pytestmark = pytest.mark.gpu

TEXT = """
shape = [16, 12]
j = 1.0
h = 0.1
beta = 0.44
schedule = "checkerboard"
thermalize = 20
sweeps_between = 3
n_samples = 6
seed = 20260718
start = "hot"
description = "16x12 near the critical coupling"
"""


@pytest.fixture(scope="module")
def gpu():
    g = plq.Gpu.new()
    if g is None:
        pytest.fail("no CUDA device")
    return g


@pytest.mark.parametrize("updater", ["metropolis", "heat_bath"])
def test_cpu_backend_run_equals_oracle_chain(oracle, gpu, updater):
    spec = runspec.parse(TEXT + f'updater = "{updater}"\n', plq.ISING)
    samples, prims = runspec.run(gpu, spec)
    lat = oracle.Lattice((16, 12))
    model = oracle.Model.ising(1.0, 0.1)
    r = oracle.PcgStream(20260718)
    cfg = oracle.hot_start(16 * 12, 2, r)
    kernel = plq.METROPOLIS if updater == "metropolis" else plq.HEATBATH
    oracle.local_sweeps(model, lat, cfg, kernel, 0.44, r, 20)
    for k in range(6):
        oracle.local_sweeps(model, lat, cfg, kernel, 0.44, r, 3)
        assert np.array_equal(samples[k], cfg), k
        assert list(prims[k]) == list(model.primaries(lat, cfg)), k


def test_gpu_backend_run_through_the_serving_loop(gpu):
    spec = runspec.parse(TEXT.replace('schedule = "checkerboard"', 'schedule = "checkerboard"\nbackend = "gpu"'),
                         plq.ISING)
    srv = Server(gpu, 0, 8, 5.0)
    job = srv.submit_run(spec, want_states=True)
    assert srv.wait(job) == 2  # done
    final, prim, _ = srv.result(job, states=True)
    srv.release(job)
    srv.close()
    chain = runspec.build_chain(gpu, runspec.parse(TEXT.replace('schedule = "checkerboard"',
                                                               'schedule = "checkerboard"\nbackend = "gpu"'),
                                                  plq.ISING))
    chain.advance(spec.total_sweeps)
    assert np.array_equal(final, chain.read())
    assert list(prim) == list(chain.primaries())
