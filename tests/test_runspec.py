"""Run configurations in the reference's TOML vocabulary: parsing, the
reference's validation rules and messages (src/config.rs:189-249,
src/models/*/run_config.rs validate), defaults, and the mapping onto device
chain descriptors."""
import pytest

import plaquette_b200 as plq
from plaquette_b200 import runspec
from plaquette_b200.runspec import ConfigError

BASE = """
shape = [16, 16]
j = 1.0
beta = 0.44
schedule = "checkerboard"
thermalize = 10
sweeps_between = 2
n_samples = 5
seed = 7
"""


def _cfg(extra="", base=BASE, drop=()):
    lines = [ln for ln in base.strip().splitlines() if ln.split("=")[0].strip() not in drop]
    return "\n".join(lines) + "\n" + extra


def test_defaults_and_mapping():
    s = runspec.parse(_cfg(), plq.ISING)
    assert (s.updater, s.backend, s.start, s.h) == ("metropolis", "cpu", "cold", 0.0)
    assert s.total_sweeps == 10 + 2 * 5 and s.n_vars == 256
    d = s.desc
    assert (d.model, d.q, d.d, d.updater, d.rng) == (plq.ISING, 2, 2, plq.METROPOLIS, plq.RNG_STREAM)
    g = runspec.parse(_cfg('backend = "gpu"\nupdater = "heat_bath"\nstart = "hot"\nh = 0.25'), plq.ISING)
    assert (g.desc.rng, g.desc.updater, g.start, g.desc.h) == (plq.RNG_KEYED, plq.HEATBATH, "hot", 0.25)
    sw = runspec.parse(_cfg('updater = "swendsen_wang"', drop=("schedule",)), plq.ISING)
    assert (sw.desc.updater, sw.desc.extent, sw.desc.relabel) == (plq.CLUSTER, plq.EXTENT_ALL, plq.RELABEL_REDRAW)
    w = runspec.parse(_cfg('updater = "wolff"\nbackend = "gpu"', drop=("schedule",)), plq.ISING)
    assert (w.desc.extent, w.desc.relabel) == (plq.EXTENT_SEEDED, plq.RELABEL_FORCED)
    p = runspec.parse(_cfg('h = [0.1, 0.0, -0.1]\nupdater = "heat_bath"'), plq.POTTS, q=3)
    assert p.desc.q == 3 and list(p.desc.offsets)[:3] == [0.1, 0.0, -0.1]
    ga = runspec.parse(_cfg(base=BASE.replace("[16, 16]", "[4, 4, 4, 4]")), plq.GAUGE)
    assert ga.n_vars == 4 * 256 and ga.desc.model == plq.GAUGE


@pytest.mark.parametrize("text,model,msg", [
    (_cfg("updatr = \"metropolis\""), plq.ISING, "unknown field `updatr`"),
    (_cfg("h = 0.1", base=BASE.replace("[16, 16]", "[4, 4]")), plq.GAUGE, "unknown field `h`"),
    (_cfg(drop=("seed",)), plq.ISING, "missing field `seed`"),
    (_cfg(base=BASE.replace("[16, 16]", "[]")), plq.ISING,
     "this run scores nearest-neighbor bonds, which need at least 1 dimensions, but shape[] names 0"),
    (_cfg(base=BASE.replace("[16, 16]", "[16]")), plq.GAUGE,
     "this run scores plaquettes, which need at least 2 dimensions, but shape[16] names 1"),
    (_cfg(base=BASE.replace("[16, 16]", "[16, 0]")), plq.ISING,
     "every lattice extent must be positive, but shape[16, 0] is 0 on axis 1"),
    (_cfg(base=BASE.replace("beta = 0.44", "beta = 0.0")), plq.ISING, "beta must be positive and finite, got 0.0"),
    (_cfg(base=BASE.replace("beta = 0.44", "beta = nan")), plq.ISING, "beta must be positive and finite, got nan"),
    (_cfg(base=BASE.replace("j = 1.0", "j = inf")), plq.ISING, "j must be finite, got inf"),
    (_cfg("h = [0.0, nan, 0.0]"), plq.POTTS, "every entry of h must be finite, but entry 1 is nan"),
    (_cfg('updater = "swendsen_wang"'), plq.ISING,
     "SwendsenWang builds clusters rather than walking variables, so it takes no schedule"),
    (_cfg('backend = "gpu"', drop=("schedule",)), plq.ISING,
     'the gpu backend runs Metropolis as parallel color passes, which needs schedule = "checkerboard"'),
    (_cfg('backend = "gpu"', base=BASE.replace("[16, 16]", "[16, 15]")), plq.ISING,
     "the gpu checkerboard colors in parallel, which needs even extents, but shape[16, 15] is odd on axis 1"),
    (_cfg('updater = "wolff"\nh = 0.5', drop=("schedule",)), plq.ISING,
     "Wolff relabels whole clusters at once, which needs the spin-flip symmetry an external field breaks"),
    (_cfg('updater = "swendsen_wang"\nh = [0.0, 0.2, 0.0]', drop=("schedule",)), plq.POTTS,
     "label symmetry a per-label offset breaks"),
    (_cfg('updater = "swendsen_wang"', drop=("schedule",), base=BASE.replace("[16, 16]", "[4, 4]")), plq.GAUGE,
     "the gauge action scores plaquettes, which have no pairwise bond graph"),
    (_cfg(base=BASE.replace("n_samples = 5", "n_samples = 0")), plq.ISING,
     "n_samples must be positive, or the run records nothing"),
    # what this device path refuses, with its reason
    (_cfg(drop=("schedule",)), plq.ISING, "the random schedule is a sequential walk"),
    (_cfg('updater = "wolff"', drop=("schedule",)), plq.ISING, "Wolff on the CPU stream"),
    (_cfg("h = [0.1, 0.2]"), plq.POTTS, "h names 2 offsets but the run has q = 3 labels"),
])
def test_validation_messages(text, model, msg):
    with pytest.raises(ConfigError, match=msg.replace("[", r"\[").replace("]", r"\]").replace("(", r"\(")
                       .replace(")", r"\)")):
        runspec.parse(text, model, q=3 if model == plq.POTTS else None)


def test_zero_warmup_and_gap_are_legitimate():
    s = runspec.parse(_cfg(base=BASE.replace("thermalize = 10", "thermalize = 0")
                           .replace("sweeps_between = 2", "sweeps_between = 0")), plq.ISING)
    assert s.total_sweeps == 0


def test_hot_start_is_drawn_from_the_seeded_generator(oracle):
    s = runspec.parse(_cfg('start = "hot"'), plq.ISING)
    cfg, off = runspec.start_configuration(s)
    r = oracle.PcgStream(7)
    want = oracle.hot_start(256, 2, r)
    assert (cfg == want).all() and off == r.draws


def test_potts_metropolis_on_the_cpu_stream_is_accepted():
    s = runspec.parse(_cfg(), plq.POTTS, q=3)
    assert s.desc.rng == plq.RNG_STREAM and s.desc.updater == plq.METROPOLIS and s.desc.q == 3
