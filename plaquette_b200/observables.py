"""Observables of a sample formed from the device's exact integer primaries.

The device reduces each configuration to integers (``plq_chain_primaries``):
Ising ``[bond_sum, spin_sum]``, Potts ``[agree, N_0, ..., N_{q-1}]``, Z2 gauge
``[plaquette_sum]``.  These functions apply the reference's final scalings to
them, in the reference's order of operations, so the floats equal what the
reference computes from a read-back configuration:

* Ising energy ``-J*bond_sum - h*spin_sum`` and magnetisation ``spin_sum``
  (src/models/ising/mod.rs:67-71, 98-117);
* Potts energy ``-J*agree - sum_a h_a N_a`` (src/models/potts/mod.rs:238-271),
  order parameter ``(Q f_max - 1)/(Q - 1)`` and its simplex form
  (src/models/potts/mod.rs:141-164);
* gauge energy ``-J*plaquette_sum`` (src/models/gauge/mod.rs:276-285).

``histogram`` bins a series of per-sample values (E/N, m) into fixed-width
bins, the per-sweep histograms of the 512^3 Potts benchmark.
"""
from __future__ import annotations

import math

import numpy as np

ISING, POTTS, GAUGE = 0, 1, 2


def energy(model: int, prims, *, j: float = 1.0, h: float = 0.0, offsets=None) -> float:
    """Energy of one sample from its primaries."""
    p = [int(v) for v in prims]
    if model == ISING:
        return -j * float(p[0]) - h * float(p[1])
    if model == POTTS:
        offset = 0.0
        if offsets is not None and any(o != 0.0 for o in offsets):
            offset = sum(float(ha) * float(na) for ha, na in zip(offsets, p[1:]))
        return -j * float(p[0]) - offset
    if model == GAUGE:
        return -j * float(p[0])
    raise ValueError(f"unknown model {model}")


def magnetization(prims) -> float:
    """Ising spin sum (ising/mod.rs:67-71)."""
    return float(int(prims[1]))


def potts_order(counts, n_vars: int) -> float:
    """(Q * f_max - 1) / (Q - 1), f_max the most common label's fraction."""
    q = len(counts)
    f_max = float(max(int(c) for c in counts)) / float(n_vars)
    return (q * f_max - 1.0) / (q - 1.0)


def potts_simplex_order(counts, n_vars: int) -> float:
    """sqrt[(Q * sum_a f_a^2 - 1) / (Q - 1)], clamped at zero under the root."""
    q = len(counts)
    squares = sum(int(c) * int(c) for c in counts)  # exact integer
    n = float(n_vars)
    sum_f2 = float(squares) / (n * n)
    return math.sqrt(max((q * sum_f2 - 1.0) / (q - 1.0), 0.0))


def series(model: int, prims: np.ndarray, n_vars: int, *, j: float = 1.0, h: float = 0.0,
           offsets=None) -> dict[str, np.ndarray]:
    """Per-sample energy per variable and order parameter (|M|/N for Ising) of
    a batch of primaries; element-wise the same operations as `energy` and
    `potts_order`."""
    p = np.asarray(prims, dtype=np.int64)
    if model == ISING:
        e = -j * p[:, 0].astype(np.float64) - h * p[:, 1].astype(np.float64)
        m = np.abs(p[:, 1].astype(np.float64)) / n_vars
    elif model == POTTS:
        e = -j * p[:, 0].astype(np.float64)
        if offsets is not None and any(o != 0.0 for o in offsets):
            off = np.zeros(len(p), dtype=np.float64)
            for a, ha in enumerate(offsets):
                off = off + float(ha) * p[:, 1 + a].astype(np.float64)
            e = e - off
        q = p.shape[1] - 1
        m = (q * (p[:, 1:].max(axis=1).astype(np.float64) / float(n_vars)) - 1.0) / (q - 1.0)
    elif model == GAUGE:
        e = -j * p[:, 0].astype(np.float64)
        m = np.zeros(len(p), dtype=np.float64)
    else:
        raise ValueError(f"unknown model {model}")
    return {"e": e / n_vars, "m": m}


def histogram(values, bins: int = 1024, lo: float = -3.0, hi: float = 3.0) -> np.ndarray:
    """Counts of `values` in `bins` equal-width bins over [lo, hi); values outside are clamped to the end bins."""
    v = np.asarray(values, dtype=np.float64)
    idx = np.floor((v - lo) / (hi - lo) * bins).astype(np.int64)
    np.clip(idx, 0, bins - 1, out=idx)
    return np.bincount(idx, minlength=bins).astype(np.int64)


def correlator(model: int, pair_sums, n_vars: int, q: int = 2) -> list[np.ndarray]:
    """Per-config correlator rows from ``axis_pair_sums``: Ising C_r = sum / N
    (ising/mod.rs:84-95); Potts C_r = agree / N - 1/Q (potts/mod.rs:218-234)."""
    n = float(n_vars)
    if model == ISING:
        return [np.array([float(int(c)) / n for c in row]) for row in pair_sums]
    floor = 1.0 / float(q)
    return [np.array([float(int(c)) / n - floor for c in row]) for row in pair_sums]


def polyakov_loop(total: int, lines: int) -> float:
    """Z2Gauge::polyakov_loop (gauge/mod.rs:179-212): signed line average."""
    return float(total) / float(lines)


def wilson_table(totals, placements: int) -> np.ndarray:
    """Z2Gauge::wilson_rectangles (gauge/mod.rs:226-274): totals / placements,
    row and column 0 the 1.0 anchor."""
    t = np.asarray(totals, dtype=np.int64)
    out = t.astype(np.float64) / float(placements)
    out[0, :] = 1.0
    out[:, 0] = 1.0
    return out
