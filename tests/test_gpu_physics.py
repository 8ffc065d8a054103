"""Physics anchors with stated error bars.

* 2D Ising 64^2 at beta_c: <E>/N from the device against Kaufman's exact
  finite-torus value (tests/exact_ising.py, itself checked against
  enumeration) -- Swendsen-Wang (tight) and the config-1 Metropolis run.
* Binder cumulant U4 from the device SW chain against the oracle's CPU SW
  chain (independent streams), within the combined jackknife error.
* 2D Z2 gauge: mean plaquette = tanh(beta) (gauge_e2e.rs:220-235).
* 2D q=3 Potts at its critical point: E/N near -(1 + 1/sqrt q) within 0.06
  (potts_e2e.rs:981-1011).
Errors: blocked standard error (blocks much longer than the autocorrelation).
"""
import math

import numpy as np
import pytest

import plaquette_b200 as plq
from tests.exact_ising import energy_per_site

pytestmark = pytest.mark.gpu

BETA_C = 0.5 * math.log(1 + math.sqrt(2))


@pytest.fixture(scope="module")
def gpu():
    g = plq.Gpu.new()
    if g is None:
        pytest.fail("no CUDA device")
    return g


def blocked(x, n_blocks=20):
    x = np.asarray(x, dtype=np.float64)
    b = len(x) // n_blocks
    means = x[: b * n_blocks].reshape(n_blocks, b).mean(axis=1)
    return float(x.mean()), float(means.std(ddof=1) / math.sqrt(n_blocks))


def binder_jackknife(m, n_blocks=20):
    m = np.asarray(m, dtype=np.float64)
    b = len(m) // n_blocks
    m = m[: b * n_blocks]
    m2, m4 = m ** 2, m ** 4

    def u4(a2, a4):
        return 1.0 - a4 / (3.0 * a2 * a2)

    full = u4(m2.mean(), m4.mean())
    s2 = m2.reshape(n_blocks, b).sum(axis=1)
    s4 = m4.reshape(n_blocks, b).sum(axis=1)
    T2, T4 = s2.sum(), s4.sum()
    jk = np.array([u4((T2 - s2[i]) / (len(m) - b), (T4 - s4[i]) / (len(m) - b)) for i in range(n_blocks)])
    err = math.sqrt((n_blocks - 1) / n_blocks * ((jk - jk.mean()) ** 2).sum())
    return full, err


def _ising_samples(gpu, updater, rng, n_samples, between, therm, seed=20260718, extent=plq.EXTENT_ALL):
    L = 64
    d = plq.make_desc(plq.ISING, 2, (L, L), updater, beta=BETA_C, seed=seed, rng=rng, sweeps_between=between,
                      batch=plq.GPU_BATCH, extent=extent)
    cls = plq.GpuClusterChain if updater == plq.CLUSTER else plq.GpuChain
    chain = cls(gpu, d, np.zeros(L * L, dtype=np.uint8))
    chain.advance(therm)
    if updater == plq.CLUSTER:
        prims = []
        for _ in range(n_samples):
            next(chain)
            prims.append(chain.primaries())
        prims = np.array(prims)
    else:
        _, prims = chain.next_batch(n_samples, states=False)
    return prims[:, 0].astype(np.float64), prims[:, 1].astype(np.float64), L * L


def test_sw_energy_matches_kaufman(gpu):
    bond, spin, N = _ising_samples(gpu, plq.CLUSTER, plq.RNG_KEYED, 4000, 1, 200)
    e, err = blocked(-bond / N)
    exact = energy_per_site(BETA_C, 64, 64)
    assert abs(e - exact) < 4 * err + 1e-4, (e, err, exact)


def test_config1_metropolis_energy_matches_kaufman(gpu):
    # 64^2, cold, beta_c, 10^4 sweeps with the first 10^3 discarded, E every 10 sweeps
    bond, spin, N = _ising_samples(gpu, plq.METROPOLIS, plq.RNG_STREAM, 900, 10, 1000)
    e, err = blocked(-bond / N, n_blocks=10)
    exact = energy_per_site(BETA_C, 64, 64)
    assert abs(e - exact) < 5 * err + 2e-3, (e, err, exact)


def test_binder_cumulant_matches_cpu_chain(gpu, oracle):
    _, spin, N = _ising_samples(gpu, plq.CLUSTER, plq.RNG_KEYED, 4000, 1, 200, seed=11)
    u_gpu, e_gpu = binder_jackknife(spin / N)
    lat = oracle.Lattice((64, 64))
    model = oracle.Model.ising(1.0)
    cfg = np.zeros(64 * 64, dtype=np.uint8)
    r = oracle.PcgStream(99)
    for _ in range(200):
        oracle.cluster_sweep(model, lat, cfg, oracle.ALL, oracle.REDRAW, BETA_C, r)
    ms = []
    for _ in range(4000):
        oracle.cluster_sweep(model, lat, cfg, oracle.ALL, oracle.REDRAW, BETA_C, r)
        ms.append(model.primaries(lat, cfg)[1] / N)
    u_cpu, e_cpu = binder_jackknife(ms)
    assert abs(u_gpu - u_cpu) < 4 * math.hypot(e_gpu, e_cpu) + 1e-3, (u_gpu, e_gpu, u_cpu, e_cpu)
    assert 0.5 < u_gpu < 0.7  # near the universal 2D value 0.61


def test_gauge_2d_plaquette_is_tanh_beta(gpu):
    L, beta = 32, 0.7
    d = plq.make_desc(plq.GAUGE, 2, (L, L), plq.HEATBATH, beta=beta, seed=5, rng=plq.RNG_KEYED, sweeps_between=2,
                      batch=plq.GPU_BATCH)
    chain = plq.GpuChain(gpu, d, None)
    chain.advance(200)
    _, prims = chain.next_batch(2000, states=False)
    p, err = blocked(prims[:, 0] / (L * L))
    assert abs(p - math.tanh(beta)) < 4 * err + 1e-3, (p, err, math.tanh(beta))


def test_potts_2d_critical_energy(gpu):
    q, L = 3, 64
    beta = math.log(1 + math.sqrt(q))
    d = plq.make_desc(plq.POTTS, q, (L, L), plq.CLUSTER, beta=beta, seed=3, rng=plq.RNG_KEYED, sweeps_between=1,
                      batch=1)
    chain = plq.GpuClusterChain(gpu, d, None)
    chain.advance(300)
    es = []
    for _ in range(2000):
        next(chain)
        es.append(-chain.primaries()[0] / (L * L))
    e, err = blocked(es)
    assert abs(e + (1 + 1 / math.sqrt(q))) < 0.06, (e, err)
