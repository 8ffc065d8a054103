"""Observables formed from integer primaries equal the oracle's energies
(src/models/ising/mod.rs:98-117, potts/mod.rs:238-271, gauge/mod.rs:276-285),
and the order parameters follow potts/mod.rs:141-164."""
import math

import numpy as np
import pytest

from plaquette_b200 import observables as obs


@pytest.mark.parametrize("kind,q,shape,kw", [
    (obs.ISING, 2, (6, 4, 2), {"j": 1.5, "h": -0.25}),
    (obs.POTTS, 3, (8, 6), {"j": 0.75, "offsets": [0.3, -0.2, 0.1]}),
    (obs.POTTS, 5, (4, 4, 4), {"j": 1.0}),
    (obs.GAUGE, 2, (4, 4, 2), {"j": 1.25}),
])
def test_energy_from_primaries_equals_oracle(oracle, kind, q, shape, kw):
    lat = oracle.Lattice(shape, staples=kind == obs.GAUGE)
    if kind == obs.ISING:
        model = oracle.Model.ising(kw["j"], kw["h"])
    elif kind == obs.POTTS:
        model = oracle.Model.potts(q, kw["j"], kw.get("offsets"))
    else:
        model = oracle.Model.gauge(kw["j"])
    rng = np.random.default_rng(7)
    for _ in range(5):
        cfg = rng.integers(0, q, model.n_vars(lat)).astype(np.uint8)
        prims = model.primaries(lat, cfg)
        assert obs.energy(kind, prims, **kw) == model.energy(lat, cfg)


def test_potts_order_parameters():
    n = 12
    assert obs.potts_order([4, 4, 4], n) == 0.0
    assert obs.potts_order([12, 0, 0], n) == 1.0
    assert obs.potts_order([6, 3, 3], n) == pytest.approx((3 * 0.5 - 1) / 2)
    assert obs.potts_simplex_order([4, 4, 4], n) == 0.0
    assert obs.potts_simplex_order([0, 12, 0], n) == 1.0
    f = np.array([6, 3, 3]) / n
    assert obs.potts_simplex_order([6, 3, 3], n) == pytest.approx(math.sqrt((3 * (f * f).sum() - 1) / 2))


def test_histogram_bins_and_clamps():
    h = obs.histogram([-4.0, -3.0, 0.0, 2.999, 3.0, 10.0], bins=6, lo=-3.0, hi=3.0)
    assert h.tolist() == [2, 0, 0, 1, 0, 3]
    assert obs.histogram(np.linspace(-1, 1, 1000), bins=1024, lo=-1.0, hi=1.0).sum() == 1000


def test_series_shapes():
    prims = np.array([[10, 4, 3, 5], [12, 6, 3, 3]], dtype=np.int64)
    s = obs.series(obs.POTTS, prims, 12)
    assert s["e"].tolist() == [-10 / 12, -1.0]
    assert s["m"][1] == pytest.approx(0.25)


def test_series_equals_per_sample_functions():
    rng = np.random.default_rng(3)
    counts = rng.integers(0, 100, (50, 4))
    prims = np.concatenate([rng.integers(0, 500, (50, 1)), counts], axis=1)
    n = 400
    s = obs.series(obs.POTTS, prims, n, j=0.8, offsets=[0.1, 0.0, -0.3, 0.2])
    for k in range(50):
        assert s["e"][k] == obs.energy(obs.POTTS, prims[k], j=0.8, offsets=[0.1, 0.0, -0.3, 0.2]) / n
        assert s["m"][k] == obs.potts_order(prims[k, 1:], n)
    ip = np.stack([rng.integers(-500, 500, 50), rng.integers(-400, 400, 50)], axis=1)
    s = obs.series(obs.ISING, ip, n, j=1.5, h=0.25)
    for k in range(50):
        assert s["e"][k] == obs.energy(obs.ISING, ip[k], j=1.5, h=0.25) / n


def test_correlator_and_loop_formulas():
    rows = [np.array([16, 8, -4]), np.array([16, 0, 16])]
    c = obs.correlator(obs.ISING, rows, 16)
    assert c[0].tolist() == [1.0, 0.5, -0.25] and c[1].tolist() == [1.0, 0.0, 1.0]
    p = obs.correlator(obs.POTTS, [np.array([12, 6])], 12, q=3)
    assert p[0].tolist() == [1.0 - 1.0 / 3.0, 0.5 - 1.0 / 3.0]
    assert obs.polyakov_loop(-3, 12) == -0.25
    t = obs.wilson_table(np.array([[48, 48], [48, 12]]), 48)
    assert t.tolist() == [[1.0, 1.0], [1.0, 0.25]]
