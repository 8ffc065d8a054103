"""The oracle's restatement of the tempering swap rule, checked on the CPU.

orc_pt_exp is the e^x the swap decision uses (basic IEEE operations only, so
host and device agree bit for bit); it must agree with libm's exp to within
a couple of units in the last place over the whole range the decision
reaches.  orc_pt_swap_phase is checked against a plain-Python statement of
the rule: even pairs on even attempts, odd pairs on odd ones, a favourable
exchange always taken, and the keyed uniform of each pair.
"""
import math

import numpy as np


def test_pt_exp_is_close_to_libm(oracle):
    rng = np.random.default_rng(3)
    xs = np.concatenate([-rng.exponential(3.0, 20000), -rng.uniform(0, 707.9, 20000),
                         [0.0, -1e-300, -1e-12, -0.5, -math.log(2), -1.0, -700.0, -707.99]])
    for x in xs:
        got, want = oracle.pt_exp(float(x)), math.exp(float(x))
        assert abs(got - want) <= 3 * math.ulp(want), x
    assert oracle.pt_exp(0.0) == 1.0
    assert oracle.pt_exp(-708.0) == 0.0 and oracle.pt_exp(-1e4) == 0.0


def _lowbias32(x):
    x ^= x >> 16
    x = (x * 0x7FEB352D) & 0xFFFFFFFF
    x ^= x >> 15
    x = (x * 0x846CA68B) & 0xFFFFFFFF
    x ^= x >> 16
    return x


def _keyed24(seed, var, sweep):
    k = _lowbias32((seed ^ var) & 0xFFFFFFFF)
    k = _lowbias32(k ^ ((sweep * 0x9E3779B9) & 0xFFFFFFFF))
    return k >> 8


def _python_phase(slots, beta, energy, j, seed32, att, exp):
    slots, beta = list(slots), list(beta)
    for k in range(att & 1, len(slots) - 1, 2):
        m1, m2 = slots[k], slots[k + 1]
        delta = (beta[m1] - beta[m2]) * (-(j[m1] * energy[m1]) - -(j[m2] * energy[m2]))
        h1 = _keyed24(seed32 ^ 0x6A09E667, k, att & 0xFFFFFFFF)
        h2 = _keyed24(seed32 ^ 0xBB67AE85, k, att & 0xFFFFFFFF)
        u = (h1 + h2 * 2.0 ** -24) * 2.0 ** -24
        if delta >= 0.0 or u < exp(delta):
            beta[m1], beta[m2] = beta[m2], beta[m1]
            slots[k], slots[k + 1] = m2, m1
    return slots, beta


def test_swap_phase_matches_a_python_statement(oracle):
    rng = np.random.default_rng(11)
    for trial in range(300):
        k = int(rng.integers(2, 9))
        n = k + 2
        slots = rng.permutation(n)[:k].astype(np.int32)
        beta = rng.uniform(0.1, 0.6, n)
        energy = rng.integers(-3000, 3000, n).astype(np.int64)
        j = rng.choice([1.0, 0.75, 1.25], n)
        seed32, att = int(rng.integers(0, 2 ** 32)), int(rng.integers(0, 50))
        want_slots, want_beta = _python_phase(slots, beta, energy, j, seed32, att, oracle.pt_exp)
        got_slots, got_beta = slots.copy(), beta.copy()
        oracle.pt_swap_phase(got_slots, got_beta, energy, j, seed32, att)
        assert list(got_slots) == want_slots, trial
        assert list(got_beta) == want_beta, trial


def test_favourable_exchange_is_always_taken_and_pairs_alternate(oracle):
    # slot 0 (beta 0.1) holds the low energy: (b0 - b1)(E0 - E1) > 0 -> always swapped
    for att in (0, 2, 4, 6):
        slots = np.array([0, 1], dtype=np.int32)
        beta = np.array([0.1, 0.5])
        assert oracle.pt_swap_phase(slots, beta, np.array([3000, 0], dtype=np.int64), np.ones(2), 9, att) == 1
        assert list(beta) == [0.5, 0.1] and list(slots) == [1, 0]
    # odd attempts pair slots (1, 2) only: slot 0 is never touched
    slots = np.array([0, 1, 2], dtype=np.int32)
    beta = np.array([0.1, 0.2, 0.3])
    oracle.pt_swap_phase(slots, beta, np.array([5000, 3000, 0], dtype=np.int64), np.ones(3), 9, 1)
    assert slots[0] == 0 and beta[0] == 0.1 and list(slots[1:]) == [2, 1]
    # a hopeless exchange (delta = -(0.4)(3000)) is never taken
    slots = np.array([0, 1], dtype=np.int32)
    beta = np.array([0.1, 0.5])
    assert oracle.pt_swap_phase(slots, beta, np.array([0, 3000], dtype=np.int64), np.ones(2), 9, 0) == 0


def test_library_host_rule_equals_the_oracle(oracle):
    """plq_tempering_swap_phase (the rule the device kernel uses, evaluated
    on the host for tempering across ranks) against the oracle's
    restatement, with the ladder seed folded as plq_ensemble_add_ladder
    folds it."""
    import plaquette_b200 as plq
    from plaquette_b200.ensemble import swap_phase

    rng = np.random.default_rng(29)
    for trial in range(300):
        k = int(rng.integers(2, 10))
        n = k + 3
        slots = rng.permutation(n)[:k].astype(np.int32)
        beta = rng.uniform(0.1, 0.7, n)
        energy = rng.integers(-5000, 5000, n).astype(np.int64)
        j = rng.choice([1.0, 0.8, 1.3], n)
        seed, att = int(rng.integers(0, 2 ** 63)), int(rng.integers(0, 100))
        a_slots, a_beta = slots.copy(), beta.copy()
        b_slots, b_beta = slots.copy(), beta.copy()
        na = swap_phase(a_slots, a_beta, energy, j, seed, att)
        nb = oracle.pt_swap_phase(b_slots, b_beta, energy, j, plq.fold_seed(seed), att)
        assert na == nb and list(a_slots) == list(b_slots) and list(a_beta) == list(b_beta), trial
