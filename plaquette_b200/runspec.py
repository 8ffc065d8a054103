"""Run configurations in the reference's TOML vocabulary, turned into device
jobs.

The reference describes a run in a TOML file read by `IsingRunConfig`,
`PottsRunConfig` and `GaugeRunConfig` (src/models/*/run_config.rs): the
physics (shape, j, h, beta), the driver controls (updater, schedule, backend,
thermalize, sweeps_between, n_samples), the seed and start, and a free-form
description.  Unknown keys are rejected and `validate` refuses runs that
would panic or record nothing; the rules are restated here with the
reference's messages (src/config.rs:189-249, src/models/ising/run_config.rs:
168-200, potts/run_config.rs:221-262, gauge/run_config.rs:183-215).

`parse` returns a `RunSpec`: a chain descriptor plus the sampling plan.
`backend = "cpu"` maps to the PCG64 stream (bit-exact with the reference CPU
`Chain` under the checkerboard schedule, hot start drawn from the seeded
generator first); `backend = "gpu"` maps to the keyed stream of the reference
GPU kernels.  What this device path cannot run is refused with a reason: the
random schedule (a sequential walk) and Wolff on the PCG stream (the FIFO draw
order of `grow_cluster`).  Potts Metropolis at q >= 3 on the PCG stream runs
as a sequential walk on one warp (exact, at one thread's speed).
"""
from __future__ import annotations

import math
import tomllib
from dataclasses import dataclass, field

import numpy as np

from . import (CLUSTER, EXTENT_ALL, EXTENT_SEEDED, GAUGE, HEATBATH, ISING, METROPOLIS, POTTS, RELABEL_FORCED,
               RELABEL_REDRAW, RNG_KEYED, RNG_STREAM, ChainDesc, GpuChain, GpuClusterChain, hot_start, make_desc)


class ConfigError(ValueError):
    """A run configuration that does not parse, does not validate, or names a
    run this device path does not execute."""


_COMMON = {"shape", "j", "beta", "updater", "schedule", "backend", "thermalize", "sweeps_between", "n_samples",
           "seed", "start", "description"}
_KEYS = {ISING: _COMMON | {"h"}, POTTS: _COMMON | {"h"}, GAUGE: set(_COMMON)}
_REQUIRED = ("shape", "j", "beta", "thermalize", "sweeps_between", "n_samples", "seed")
_UPDATERS = {"metropolis", "heat_bath", "swendsen_wang", "wolff"}
_MIN_DIMENSION = {ISING: 1, POTTS: 1, GAUGE: 2}
_SCORES = {ISING: "nearest-neighbor bonds", POTTS: "nearest-neighbor bonds", GAUGE: "plaquettes"}
_UPDATER_NAME = {"metropolis": "Metropolis", "heat_bath": "HeatBath", "swendsen_wang": "SwendsenWang",
                 "wolff": "Wolff"}


@dataclass
class RunSpec:
    model: int
    q: int
    shape: tuple
    j: float
    h: object          # Ising: float; Potts: list of per-label offsets
    beta: float
    updater: str
    schedule: str | None
    backend: str
    thermalize: int
    sweeps_between: int
    n_samples: int
    seed: int
    start: str
    description: str | None = None
    desc: ChainDesc | None = field(default=None, repr=False)

    @property
    def n_vars(self) -> int:
        n = int(np.prod(self.shape))
        return n * len(self.shape) if self.model == GAUGE else n

    @property
    def total_sweeps(self) -> int:
        """Sweeps of the whole run: thermalisation plus every sample's gap."""
        return self.thermalize + self.sweeps_between * self.n_samples


def _nonneg_int(cfg, key):
    v = cfg[key]
    if isinstance(v, bool) or not isinstance(v, int) or v < 0:
        raise ConfigError(f"{key} must be a non-negative integer, got {v!r}")
    return v


def _float(cfg, key, default=None):
    v = cfg.get(key, default)
    if isinstance(v, bool) or not isinstance(v, (int, float)):
        raise ConfigError(f"{key} must be a number, got {v!r}")
    return float(v)


def _check_updater(updater, schedule, backend, shape):
    """check_updater (src/config.rs:222-249)."""
    name = _UPDATER_NAME[updater]
    clusters = updater in ("swendsen_wang", "wolff")
    if clusters and schedule is not None:
        raise ConfigError(f"{name} builds clusters rather than walking variables, so it takes no schedule; "
                          "remove the schedule field")
    if backend == "gpu" and not clusters:
        if (schedule or "random") != "checkerboard":
            raise ConfigError(f"the gpu backend runs {name} as parallel color passes, which needs "
                              'schedule = "checkerboard"')
        odd = [i for i, L in enumerate(shape) if L % 2]
        if odd:
            raise ConfigError(f"the gpu checkerboard colors in parallel, which needs even extents, but "
                              f"shape{list(shape)} is odd on axis {odd[0]}")


def parse(text: str, model: int, q: int | None = None) -> RunSpec:
    """Parse and validate a run configuration for `model` (ISING, POTTS or
    GAUGE).  Potts files do not name Q (the reference fixes it in the driver's
    source), so the caller passes `q`."""
    try:
        cfg = tomllib.loads(text)
    except tomllib.TOMLDecodeError as e:
        raise ConfigError(f"not valid TOML: {e}") from e
    unknown = sorted(set(cfg) - _KEYS[model])
    if unknown:
        raise ConfigError(f"unknown field `{unknown[0]}`")
    missing = [k for k in _REQUIRED if k not in cfg]
    if missing:
        raise ConfigError(f"missing field `{missing[0]}`")
    if model == POTTS:
        if q is None or not 2 <= q <= 64:
            raise ConfigError("a Potts run needs q in 2..64 from the caller")
    else:
        q = 2
    shape = cfg["shape"]
    if not isinstance(shape, list) or not all(isinstance(x, int) and not isinstance(x, bool) and x >= 0
                                              for x in shape):
        raise ConfigError(f"shape must be a list of non-negative integers, got {shape!r}")
    # check_shape (src/config.rs:189-207)
    if len(shape) < _MIN_DIMENSION[model]:
        raise ConfigError(f"this run scores {_SCORES[model]}, which need at least {_MIN_DIMENSION[model]} "
                          f"dimensions, but shape{shape} names {len(shape)}")
    if 0 in shape:
        raise ConfigError(f"every lattice extent must be positive, but shape{shape} is 0 on axis "
                          f"{shape.index(0)}")
    beta = _float(cfg, "beta")
    if not math.isfinite(beta) or beta <= 0.0:
        raise ConfigError(f"beta must be positive and finite, got {beta}")
    j = _float(cfg, "j")
    if not math.isfinite(j):
        raise ConfigError(f"j must be finite, got {j}")
    if model == ISING:
        h = _float(cfg, "h", 0.0)
        if not math.isfinite(h):
            raise ConfigError(f"h must be finite, got {h}")
    elif model == POTTS:
        h = cfg.get("h", [])
        if not isinstance(h, list) or not all(isinstance(x, (int, float)) and not isinstance(x, bool) for x in h):
            raise ConfigError(f"h must be a list of numbers, got {h!r}")
        h = [float(x) for x in h]
        bad = [i for i, v in enumerate(h) if not math.isfinite(v)]
        if bad:
            raise ConfigError(f"every entry of h must be finite, but entry {bad[0]} is {h[bad[0]]}")
        if h and len(h) != q:  # the reference checks the count in build(), against Q
            raise ConfigError(f"h names {len(h)} offsets but the run has q = {q} labels")
    else:
        h = 0.0
    updater = cfg.get("updater", "metropolis")
    if updater not in _UPDATERS:
        raise ConfigError(f"unknown updater {updater!r}")
    schedule = cfg.get("schedule")
    if schedule is not None and schedule not in ("random", "checkerboard"):
        raise ConfigError(f"unknown schedule {schedule!r}")
    backend = cfg.get("backend", "cpu")
    if backend not in ("cpu", "gpu"):
        raise ConfigError(f"unknown backend {backend!r}")
    start = cfg.get("start", "cold")
    if start not in ("cold", "hot"):
        raise ConfigError(f"unknown start {start!r}")
    clusters = updater in ("swendsen_wang", "wolff")
    if model == GAUGE and clusters:
        raise ConfigError("the gauge action scores plaquettes, which have no pairwise bond graph for a cluster "
                          "update to build on")
    _check_updater(updater, schedule, backend, shape)
    if clusters and model == ISING and h != 0.0:
        raise ConfigError(f"{_UPDATER_NAME[updater]} relabels whole clusters at once, which needs the spin-flip "
                          f"symmetry an external field breaks, but h is {h}")
    if clusters and model == POTTS and any(v != 0.0 for v in h):
        raise ConfigError(f"{_UPDATER_NAME[updater]} relabels whole clusters at once, which needs the label "
                          f"symmetry a per-label offset breaks, but h{h} is not all zero")
    thermalize = _nonneg_int(cfg, "thermalize")
    sweeps_between = _nonneg_int(cfg, "sweeps_between")
    n_samples = _nonneg_int(cfg, "n_samples")
    if n_samples == 0:
        raise ConfigError("n_samples must be positive, or the run records nothing")
    seed = cfg["seed"]
    if isinstance(seed, bool) or not isinstance(seed, int) or not 0 <= seed < 2 ** 64:
        raise ConfigError(f"seed must be an unsigned 64-bit integer, got {seed!r}")
    description = cfg.get("description")

    # ---- what this device path runs
    rng = RNG_KEYED if backend == "gpu" else RNG_STREAM
    if not clusters and (schedule or "random") != "checkerboard":
        raise ConfigError("this device path runs checkerboard colour passes; the random schedule is a "
                          "sequential walk (set schedule = \"checkerboard\")")
    if not clusters and any(L % 2 for L in shape):
        raise ConfigError(f"the device checkerboard needs even extents, but shape{shape} has an odd one")
    if updater == "wolff" and rng == RNG_STREAM:
        raise ConfigError("Wolff on the CPU stream draws in grow_cluster's sequential FIFO order; run it with "
                          'backend = "gpu" (the keyed stream)')
    kernel = {"metropolis": METROPOLIS, "heat_bath": HEATBATH}.get(updater, CLUSTER)
    extent = EXTENT_SEEDED if updater == "wolff" else EXTENT_ALL
    relabel = RELABEL_FORCED if updater == "wolff" else RELABEL_REDRAW
    spec = RunSpec(model=model, q=q, shape=tuple(shape), j=j, h=h, beta=beta, updater=updater, schedule=schedule,
                   backend=backend, thermalize=thermalize, sweeps_between=sweeps_between, n_samples=n_samples,
                   seed=seed, start=start, description=description)
    spec.desc = make_desc(model, q, spec.shape, kernel, beta=beta, j=j, h=h if model == ISING else 0.0,
                          offsets=h if model == POTTS and h else None, seed=seed, rng=rng,
                          sweeps_between=max(1, sweeps_between), batch=1, extent=extent, relabel=relabel)
    return spec


def start_configuration(spec: RunSpec) -> tuple[np.ndarray, int]:
    """The run's start configuration and the stream draws it consumed: cold is
    every variable in state 0; hot is drawn from the seeded generator
    (Configuration::hot), which then continues into the chain."""
    if spec.start == "cold":
        return np.zeros(spec.n_vars, dtype=np.uint8), 0
    return hot_start(spec.seed, spec.q, spec.n_vars)


def build_chain(gpu, spec: RunSpec):
    """A device chain for the run, positioned where the reference's chain starts."""
    start, offset = start_configuration(spec)
    desc = spec.desc
    if desc.rng == RNG_STREAM:
        desc.stream_offset = offset
    cls = GpuClusterChain if desc.updater == CLUSTER else GpuChain
    return cls(gpu, desc, start)


def run(gpu, spec: RunSpec):
    """The whole run on the device: thermalise, then n_samples samples
    sweeps_between apart.  Returns (samples, primaries) with samples the
    configurations (n_samples x n_vars uint8)."""
    chain = build_chain(gpu, spec)
    try:
        chain.advance(spec.thermalize)
        samples = np.empty((spec.n_samples, spec.n_vars), dtype=np.uint8)
        prims = []
        for k in range(spec.n_samples):
            chain.advance(spec.sweeps_between)
            samples[k] = chain.read()
            prims.append(chain.primaries())
        return samples, np.array(prims)
    finally:
        chain.close()
