"""bench.py's reference arm runs on the host cores alone, so its JSON line is
checked here: the keys the benchmark contract asks for, a CPU baseline that
describes the run, an end-to-end figure with no host-device copies, and the
cluster workloads timed on one thread (the reference is sequential), the
ensemble's members spread over the host threads."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _line(*args, timeout=300):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                       timeout=timeout, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    return json.loads(lines[0])


def _common(d, steps, warmup, unit):
    assert d["impl"] == "reference"
    assert d["metric"] == unit and d["unit"] == unit and d["higher_is_better"] is True
    assert d["steps"] == steps and d["warmup"] == warmup and d["n_gpus"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"] and cb["unit"] == unit
    assert d["e2e"] == {"value": d["value"], "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_default_workload_is_the_ensemble():
    d = _line("--impl", "reference", "--steps", "1", "--warmup", "1")
    _common(d, 1, 1, "site updates/ns")
    assert d["config"]["name"] == "ensemble-config4"


def test_reference_arm_single_lattice():
    d = _line("--impl", "reference", "--workload", "potts3-512-hb-stream", "--steps", "3", "--warmup", "3")
    _common(d, 3, 3, "site updates/ns")
    assert d["config"]["name"] == "potts3-512-hb-stream"


def test_gpus_flag_spawns_the_ranks_itself():
    """`--gpus 2` outside torchrun relaunches itself as two ranks; rank 0
    alone prints the reference arm's line."""
    d = _line("--impl", "reference", "--gpus", "2", "--workload", "wolff-128-keyed", "--steps", "2", "--warmup",
              "1", timeout=600)
    assert d["n_gpus"] == 2 and d["config"]["name"] == "wolff-128-keyed"


@pytest.mark.parametrize("workload,steps,unit", [("wolff-128-keyed", 3, "cluster updates/s"),
                                                 ("sw-4096-stream", 1, "SW sweeps/s"),
                                                 ("sw-4096-keyed", 1, "SW sweeps/s")])
def test_reference_arm_cluster_workloads(workload, steps, unit):
    d = _line("--impl", "reference", "--workload", workload, "--steps", str(steps), "--warmup", "1")
    _common(d, steps, 1, unit)
    assert d["cpu_baseline"]["cores"] == 1  # the reference's cluster moves are sequential
    assert d["config"]["name"] == workload


def test_reference_arm_ensemble():
    d = _line("--impl", "reference", "--workload", "ensemble-config4", "--steps", "2", "--warmup", "1")
    _common(d, 2, 1, "site updates/ns")
    assert d["config"]["members"] == 320 and d["config"]["variables"] == 48615936
