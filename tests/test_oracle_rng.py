"""Pins the oracle's randomness against independent implementations.

* PCG64 core (rand_pcg ``Lcg128Xsl64``): the PCG reference known-answer
  vectors for ``pcg64(42, 54)`` and numpy's ``PCG64`` bit generator (a
  third-party implementation of the same LCG128/XSL-RR generator).
* ``seed_from_u64`` and the ``f64`` / ``random_range`` conversions of rand
  0.10: restated from the crates' published algorithms, re-derived here in
  pure Python (parity with the real crate is unpinned: no cargo here).
* ``lowbias32`` / ``keyed_uniform`` (src/wgsl/rng.wgsl:34-52), re-derived here.
"""
import numpy as np
import pytest

M128 = (1 << 128) - 1
M64 = (1 << 64) - 1
MULT = 0x2360ED051FC65DA44385DF649FCCF645


def _pcg_c_seed(initstate, initseq):
    """pcg_setseq_128_srandom_r from the PCG C reference."""
    inc = ((initseq << 1) | 1) & M128
    s = inc
    s = (s + initstate) & M128
    s = (s * MULT + inc) & M128
    return s, inc


def _xsl_rr(s):
    rot = s >> 122
    x = ((s >> 64) ^ s) & M64
    return ((x >> rot) | (x << (64 - rot))) & M64 if rot else x


def test_pcg64_known_answer_vectors(oracle):
    s, inc = _pcg_c_seed(42, 54)
    r = oracle.PcgStream(state=s, inc=inc)
    got = [r.next_u64() for _ in range(6)]
    assert got == [
        0x86B1DA1D72062B68,
        0x1304AA46C9853D39,
        0xA3670E9E0DD50358,
        0xF9090E529A7DAE00,
        0xC85B9FD837996F2C,
        0x606121F8E3919196,
    ]


@pytest.mark.parametrize("seed", [0, 1, 7, 20260718, 2**63 + 12345])
def test_pcg64_matches_numpy(oracle, seed):
    ref = oracle.PcgStream(seed)
    g = np.random.PCG64()
    g.state = {"bit_generator": "PCG64", "state": {"state": ref.r.state, "inc": ref.r.inc},
               "has_uint32": 0, "uinteger": 0}
    want = [int(x) for x in g.random_raw(257)]
    got = [ref.next_u64() for _ in range(257)]
    assert got == want


def test_advance_equals_stepping(oracle):
    a = oracle.PcgStream(99)
    b = oracle.PcgStream(99)
    for delta in [0, 1, 2, 3, 17, 1000, 123457]:
        a.advance(delta)
        for _ in range(delta):
            b.next_u64()
        assert a.next_u64() == b.next_u64()
    # and against numpy's own advance
    c = oracle.PcgStream(5)
    g = np.random.PCG64()
    g.state = {"bit_generator": "PCG64", "state": {"state": c.r.state, "inc": c.r.inc},
               "has_uint32": 0, "uinteger": 0}
    c.advance(2**40 + 77)
    g.advance(2**40 + 77)
    assert c.next_u64() == int(g.random_raw())


def _seed_from_u64_py(seed):
    st = seed
    words = []
    for _ in range(8):
        st = (st * 6364136223846793005 + 11634580027462260723) & M64
        xs = (((st >> 18) ^ st) >> 27) & 0xFFFFFFFF
        rot = st >> 59
        x = ((xs >> rot) | (xs << (32 - rot))) & 0xFFFFFFFF if rot else xs
        words.append(x)
    raw = b"".join(w.to_bytes(4, "little") for w in words)
    state = int.from_bytes(raw[:16], "little")
    inc = int.from_bytes(raw[16:], "little") | 1
    state = (state + inc) & M128
    state = (state * MULT + inc) & M128
    return state, inc


@pytest.mark.parametrize("seed", [0, 1, 42, 20260718, M64])
def test_seed_from_u64_restatement(oracle, seed):
    r = oracle.PcgStream(seed)
    assert (r.r.state, r.r.inc) == _seed_from_u64_py(seed)


def test_same_seed_reproduces_stream(oracle):
    # src/rng.rs:56-64
    a, b = oracle.PcgStream(42), oracle.PcgStream(42)
    assert [a.next_f64() for _ in range(16)] == [b.next_f64() for _ in range(16)]


def test_f64_is_53_high_bits(oracle):
    a, b = oracle.PcgStream(3), oracle.PcgStream(3)
    for _ in range(1000):
        x = a.next_f64()
        assert 0.0 <= x < 1.0
        assert x == (b.next_u64() >> 11) * 2.0**-53


def _next_below_py(u64s, n):
    """rand 0.10 UniformUsize via the u32 widening-multiply sampler."""
    rng = iter(u64s)
    rng_range = n & 0xFFFFFFFF
    x = next(rng) & 0xFFFFFFFF
    m = x * rng_range
    result, lo = m >> 32, m & 0xFFFFFFFF
    used = 1
    if lo > ((-rng_range) & 0xFFFFFFFF):
        x2 = next(rng) & 0xFFFFFFFF
        used = 2
        if lo + ((x2 * rng_range) >> 32) > 0xFFFFFFFF:
            result += 1
    return result, used


@pytest.mark.parametrize("n", [2, 3, 5, 20, 4096, 3 * 2**30])
def test_next_below_restatement(oracle, n):
    a, b = oracle.PcgStream(11), oracle.PcgStream(11)
    for _ in range(2000):
        before = a.draws
        v = a.next_below(n)
        used = a.draws - before
        assert 0 <= v < n
        raw = [b.next_u64() for _ in range(used)]
        want, want_used = _next_below_py(raw + [0], n)
        assert (v, used) == (want, want_used)


def test_next_below_power_of_two_takes_one_draw(oracle):
    # range a power of two never lands in the bias zone: one u64 per call.
    r = oracle.PcgStream(123)
    for n in (2, 4, 64, 2**20):
        before = r.draws
        for _ in range(500):
            r.next_below(n)
        assert r.draws - before == 500


def test_next_below_second_draw_path(oracle):
    # Find a stream position whose u32 lands in the bias zone for a large
    # range, and check the extra draw is taken there.
    n = 3 * 2**30 + 1
    r = oracle.PcgStream(77)
    probe = oracle.PcgStream(77)
    found = False
    for _ in range(20000):
        x = probe.next_u64() & 0xFFFFFFFF
        lo = (x * n) & 0xFFFFFFFF
        before = r.draws
        r.next_below(n)
        if lo > ((-n) & 0xFFFFFFFF):
            assert r.draws - before == 2
            probe.next_u64()
            found = True
            break
        assert r.draws - before == 1
    assert found


def _lowbias32_py(x):
    x &= 0xFFFFFFFF
    x ^= x >> 16
    x = (x * 0x7FEB352D) & 0xFFFFFFFF
    x ^= x >> 15
    x = (x * 0x846CA68B) & 0xFFFFFFFF
    x ^= x >> 16
    return x


def test_keyed_uniform_restatement(oracle):
    rs = np.random.default_rng(0)
    for _ in range(500):
        seed, var, sweep = (int(v) for v in rs.integers(0, 2**32, 3, dtype=np.uint64))
        assert oracle.lowbias32(seed) == _lowbias32_py(seed)
        k = _lowbias32_py(seed ^ var)
        k = _lowbias32_py(k ^ ((sweep * 0x9E3779B9) & 0xFFFFFFFF))
        want = np.float32(k >> 8) * np.float32(1.0 / 16777216.0)
        got = oracle.keyed_uniform(seed, var, sweep)
        assert np.float32(got) == want
        assert 0.0 <= got < 1.0


def test_keyed_draw_split_form():
    """The device composes a keyed draw lowbias32(lowbias32(a) ^ m) as
    tail(head(a) ^ m ^ (m >> 16)), head/tail being lowbias32 without its last /
    first xorshift by 16: x -> x ^ (x >> 16) is linear over xor and its own
    inverse on 32 bits, so the two middle xorshifts cancel.  Checked here at
    random and at the edge values of both words."""
    M = 0xFFFFFFFF

    def head(x):
        x ^= x >> 16
        x = (x * 0x7FEB352D) & M
        x ^= x >> 15
        return (x * 0x846CA68B) & M

    def tail(y):
        y = (y * 0x7FEB352D) & M
        y ^= y >> 15
        y = (y * 0x846CA68B) & M
        return y ^ (y >> 16)

    rs = np.random.default_rng(7)
    pairs = [(int(a), int(t)) for a, t in rs.integers(0, 2**32, (4000, 2), dtype=np.uint64)]
    pairs += [(a, t) for a in (0, 1, 0xFFFF, 0x10000, M) for t in (0, 1, 0x10000, M)]
    for a, sweep in pairs:
        m = (sweep * 0x9E3779B9) & M
        assert _lowbias32_py(_lowbias32_py(a) ^ m) == tail(head(a) ^ m ^ (m >> 16))


def test_fold_seed(oracle):
    # src/device.rs:761-763
    for s in [0, 1, 2**32, 2**64 - 1, 20260718, 0xDEADBEEF_12345678]:
        assert oracle.fold_seed(s) == ((s ^ (s >> 32)) & 0xFFFFFFFF)
