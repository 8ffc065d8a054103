"""The device reproduces the committed golden runs (tests/golden/runs.json):
final configuration (SHA-256), integer primaries and PCG stream position,
without running the oracle."""
import hashlib
import json
import os

import numpy as np
import pytest

import plaquette_b200 as plq

pytestmark = pytest.mark.gpu
RUNS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "runs.json")))


@pytest.fixture(scope="module")
def gpu():
    g = plq.Gpu.new()
    if g is None:
        pytest.fail("no CUDA device")
    return g


@pytest.mark.parametrize("run", RUNS, ids=lambda r: r["name"])
@pytest.mark.parametrize("flags", [0, plq.FLAG_GENERIC_PASS], ids=["default", "generic"])
def test_device_reproduces_golden_run(gpu, run, flags):
    shape = tuple(run["shape"])
    n = int(np.prod(shape)) * (len(shape) if run["model"] == plq.GAUGE else 1)
    if run["start"] == "cold":
        start = np.zeros(n, np.uint8)
    else:
        start, offset = plq.hot_start(run["seed"], run["q"], n)
        assert offset == run["stream_offset"]
    rng = plq.RNG_STREAM if run["rng"] == 0 else plq.RNG_KEYED
    d = plq.make_desc(run["model"], run["q"], shape, run["kernel"], beta=run["beta"], seed=run["seed"], rng=rng,
                      stream_offset=run["stream_offset"], sweeps_between=run["sweeps"], batch=1, flags=flags)
    chain = plq.GpuChain(gpu, d, start)
    cfg = next(chain)
    assert hashlib.sha256(cfg.tobytes()).hexdigest() == run["sha256"]
    assert [int(x) for x in chain.primaries()] == run["primaries"]
    if rng == plq.RNG_STREAM:
        assert chain.stream_position() == run["stream_position"]
    chain.close()
