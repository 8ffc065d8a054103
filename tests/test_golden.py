"""The oracle reproduces the committed golden runs (tests/golden/runs.json,
written by tests/golden/make_golden.py): a regression pin on the checker."""
import json
import os

import pytest

HERE = os.path.dirname(__file__)
RUNS = json.load(open(os.path.join(HERE, "golden", "runs.json")))


@pytest.mark.parametrize("run", RUNS, ids=lambda r: r["name"])
def test_oracle_reproduces_golden_run(oracle, run):
    import sys

    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden

    got = make_golden.run_case(run["name"], run["model"], run["q"], tuple(run["shape"]), run["kernel"], run["rng"],
                               run["beta"], run["sweeps"], run["seed"], run["start"])
    assert got == run
