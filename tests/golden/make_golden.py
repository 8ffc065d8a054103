"""Writes tests/golden/runs.json: fixed seeded runs of the oracle (the C
restatement of the reference CPU path and of the reference GPU kernels) with
the SHA-256 of every final configuration, its integer primaries and the PCG
stream position.

The reference itself is a Rust crate that cannot be built here (no cargo),
so these fixtures are not outputs of the reference: they freeze the oracle's
answers (which the oracle tests pin against the PCG reference vectors, numpy's
PCG64 and the reference's own known answers) so that the device tests can be
checked against committed numbers and any later change to the oracle shows.

Run from the repository root:  python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)
from oracle import oracle as o  # noqa: E402

ISING, POTTS, GAUGE = 0, 1, 2
METRO, HB = 0, 1
STREAM, KEYED = 0, 1

# name, model, q, shape, kernel, rng, beta, sweeps, seed, start
CASES = [
    ("ising2d-64-cold-metro-stream", ISING, 2, (64, 64), METRO, STREAM, 0.4406868, 100, 20260718, "cold"),
    ("ising2d-64-cold-metro-keyed", ISING, 2, (64, 64), METRO, KEYED, 0.4406868, 100, 20260718, "cold"),
    ("ising3d-16-hot-hb-stream", ISING, 2, (16, 16, 16), HB, STREAM, 0.2216544, 20, 7, "hot"),
    ("potts3-3d-16-hot-hb-stream", POTTS, 3, (16, 16, 16), HB, STREAM, 0.5505, 20, 11, "hot"),
    ("potts3-3d-16-hot-hb-keyed", POTTS, 3, (16, 16, 16), HB, KEYED, 0.5505, 20, 11, "hot"),
    ("potts4-2d-32-hot-metro-keyed", POTTS, 4, (32, 32), METRO, KEYED, 1.1, 20, 13, "hot"),
    ("gauge4d-6-hot-hb-stream", GAUGE, 2, (6, 6, 6, 6), HB, STREAM, 0.44, 10, 17, "hot"),
    ("gauge3d-8-hot-metro-keyed", GAUGE, 2, (8, 8, 8), METRO, KEYED, 0.7, 10, 19, "hot"),
]


def model_of(kind, q):
    if kind == ISING:
        return o.Model.ising(1.0, 0.0)
    if kind == POTTS:
        return o.Model.potts(q, 1.0)
    return o.Model.gauge(1.0)


def run_case(name, kind, q, shape, kernel, rng_mode, beta, sweeps, seed, start):
    lat = o.Lattice(shape, staples=kind == GAUGE)
    model = model_of(kind, q)
    n = model.n_vars(lat)
    r = o.PcgStream(seed)
    cfg = np.zeros(n, np.uint8) if start == "cold" else o.hot_start(n, q, r)
    offset = r.draws
    if rng_mode == STREAM:
        o.local_sweeps(model, lat, cfg, kernel, beta, r, sweeps)
    else:
        s32 = o.fold_seed(seed)
        for t in range(sweeps):
            o.keyed_local_sweep(model, lat, cfg, kernel, beta, s32, t)
    return {"name": name, "model": kind, "q": q, "shape": list(shape), "kernel": kernel, "rng": rng_mode,
            "beta": beta, "sweeps": sweeps, "seed": seed, "start": start, "stream_offset": offset,
            "stream_position": r.draws if rng_mode == STREAM else None,
            "sha256": hashlib.sha256(cfg.tobytes()).hexdigest(),
            "primaries": [int(x) for x in model.primaries(lat, cfg)]}


def main():
    out = [run_case(*c) for c in CASES]
    path = os.path.join(os.path.dirname(__file__), "runs.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {len(out)} runs to {path}")


if __name__ == "__main__":
    main()
