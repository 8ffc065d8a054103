// plq_tables.cpp -- decision tables, PCG64 seeding and jump tables (host).
//
// Compiled with -ffp-contract=off: every f64/f32 operation below must round on
// its own, in the order the reference writes it, because the cut points are
// only exact if the arithmetic that defines them is the reference's.
#include "plq_tables.h"

#include <cmath>
#include <cstring>

#include "../../include/plaquette.h"

namespace plq {

using u128h = unsigned __int128;

static inline int decode(int s) { return 1 - 2 * s; }

int64_t env_key_count(const ModelParams &p) {
    if (p.model == PLQ_GAUGE) return 2 * (2 * (p.d - 1) + 1);
    int64_t base = 2 * p.d + 1, packed = 1;
    for (int s = 0; s < p.q - 1; ++s) {
        packed *= base;
        if (packed > kMaxTableEntries) return kMaxTableEntries + 1;
    }
    return packed * p.q;
}

int64_t potts_metro_key_count(const ModelParams &p) {
    int64_t b = 2 * p.d + 1;
    return (int64_t)p.q * p.q * b * b;
}

// Neighbour-state counts of a site environment; false if the packed index
// names no composition of 2d neighbours.  State 0 is the implied one:
// packed = sum over s >= 1 of c_s * (2d+1)^(s-1).
static bool unpack_counts(const ModelParams &p, int64_t packed, int *c) {
    int64_t base = 2 * p.d + 1;
    int rest = 2 * p.d;
    for (int s = 1; s < p.q; ++s) {
        c[s] = (int)(packed % base);
        packed /= base;
        rest -= c[s];
    }
    if (rest < 0) return false;
    c[0] = rest;
    return true;
}

// ---- reference f64 energy deltas -------------------------------------
// Ising::energy_delta (src/models/ising/mod.rs:119-143)
static double ising_delta64(const ModelParams &p, int cur, int prop, int nsum) {
    int64_t ds = (int64_t)(decode(prop) - decode(cur));
    if (ds == 0) return 0.0;
    return -(double)ds * (p.j * (double)nsum + p.h);
}
// Potts::energy_delta (src/models/potts/mod.rs:273-308)
static double potts_delta64(const ModelParams &p, int cur, int prop, int change) {
    if (prop == cur) return 0.0;
    double offset = p.offsets[prop] - p.offsets[cur];
    return -p.j * (double)change - offset;
}
// Z2Gauge::energy_delta (src/models/gauge/mod.rs:287-328)
static double gauge_delta64(const ModelParams &p, int cur, int prop, int staple_sum) {
    int64_t ds = (int64_t)(decode(prop) - decode(cur));
    if (ds == 0) return 0.0;
    return -p.j * (double)(ds * (int64_t)staple_sum);
}

// ---- reference GPU f32 energy deltas (params narrowed to f32) ---------
// ising/model.wgsl:32-38
static float ising_delta32(const ModelParams &p, int cur, int nsum) {
    float j32 = (float)p.j, h32 = (float)p.h;
    float t = j32 * (float)nsum;
    t = t + h32;
    float a = 2.0f * (float)decode(cur);
    return a * t;
}
// potts/model.wgsl:54-67
static float potts_delta32(const ModelParams &p, int cur, int prop, int change) {
    float j32 = (float)p.j;
    float offset = (float)p.offsets[prop] - (float)p.offsets[cur];
    float t = (-j32) * (float)change;
    return t - offset;
}
// gauge/model.wgsl:31-42
static float gauge_delta32(const ModelParams &p, int cur, int staple_sum) {
    float a = 2.0f * (float)p.j;
    a = a * (float)decode(cur);
    return a * (float)staple_sum;
}

// Environment -> per-state deltas (f64 and f32) for every state.
static bool env_deltas(const ModelParams &p, int64_t key, int &cur, double *d64, float *d32) {
    int q = p.model == PLQ_POTTS ? p.q : 2;
    cur = (int)(key % q);
    int64_t rest = key / q;
    if (p.model == PLQ_GAUGE) {
        int staple_sum = 2 * (int)rest - 2 * (p.d - 1);
        for (int s = 0; s < 2; ++s) {
            d64[s] = s == cur ? 0.0 : gauge_delta64(p, cur, s, staple_sum);
            d32[s] = s == cur ? 0.0f : gauge_delta32(p, cur, staple_sum);
        }
        return true;
    }
    int c[64];
    if (!unpack_counts(p, rest, c)) return false;
    if (p.model == PLQ_ISING) {
        int nsum = c[0] - c[1];
        for (int s = 0; s < 2; ++s) {
            d64[s] = s == cur ? 0.0 : ising_delta64(p, cur, s, nsum);
            d32[s] = s == cur ? 0.0f : ising_delta32(p, cur, nsum);
        }
        return true;
    }
    for (int s = 0; s < q; ++s) {
        int change = c[s] - c[cur];
        d64[s] = s == cur ? 0.0 : potts_delta64(p, cur, s, change);
        d32[s] = s == cur ? 0.0f : potts_delta32(p, cur, s, change);
    }
    return true;
}

// Smallest k in [0, hi] for which pred(k) is false (pred true on a prefix).
template <class Pred>
static uint64_t first_false(uint64_t hi, Pred pred) {
    uint64_t lo = 0;
    while (lo < hi) {
        uint64_t mid = lo + (hi - lo) / 2;
        if (pred(mid))
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

static const double kTwoM53 = 1.0 / 9007199254740992.0;  // 2^-53
static const float kTwoM24 = 1.0f / 16777216.0f;          // 2^-24

// heat_bath_step (src/updater.rs:109-167) in f64: cut points on k (53 bits).
static void hb_cuts64(const ModelParams &p, double beta, int q, const double *deltas, uint64_t *cut) {
    double floor_ = INFINITY;
    for (int s = 0; s < q; ++s) floor_ = std::fmin(floor_, deltas[s]);
    double w[64];
    double total = 0.0;
    for (int s = 0; s < q; ++s) {
        w[s] = std::exp(-beta * (deltas[s] - floor_));
        total += w[s];
    }
    double cumulative = 0.0;
    for (int s = 0; s < q - 1; ++s) {
        cumulative += w[s];
        const double cum = cumulative;
        cut[s] = first_false(1ULL << 53, [&](uint64_t k) {
            double u = (double)k * kTwoM53;
            return u * total < cum;
        });
    }
    (void)p;
}

// heat_bath.wgsl:28-62 in f32: cut points on k (24 bits).
static void hb_cuts32(float beta32, int q, const float *deltas, uint32_t *cut) {
    float lowest = 0.0f;
    for (int s = 0; s < q; ++s) lowest = std::fmin(lowest, deltas[s]);
    float w[64];
    float total = 0.0f;
    for (int s = 0; s < q; ++s) {
        float t = deltas[s] - lowest;
        float x = (-beta32) * t;
        w[s] = (float)std::exp((double)x);
        total = total + w[s];
    }
    float cumulative = 0.0f;
    for (int s = 0; s + 1 < q; ++s) {
        cumulative = cumulative + w[s];
        const float cum = cumulative;
        cut[s] = (uint32_t)first_false(1ULL << 24, [&](uint64_t k) {
            float u = (float)k * kTwoM24;
            float threshold = u * total;
            return threshold < cum;
        });
    }
}

// step (src/updater.rs:77-96): accept iff dE <= 0 (no draw) or next_f64 < exp(-beta dE).
static uint64_t metro_cut64(double beta, double delta) {
    if (delta <= 0.0) return kAlways53;
    double t = std::exp(-beta * delta);
    return first_false(1ULL << 53, [&](uint64_t k) { return (double)k * kTwoM53 < t; });
}

// metropolis.wgsl:57-62: accept iff dE <= 0 or u < exp(-beta dE), f32.
static uint32_t metro_cut32(float beta32, float delta) {
    if (delta <= 0.0f) return kAlways24;
    float x = (-beta32) * delta;
    float t = (float)std::exp((double)x);
    return (uint32_t)first_false(1ULL << 24, [&](uint64_t k) { return (float)k * kTwoM24 < t; });
}

bool build_tables(const ModelParams &p, int updater, int rng, Tables &out, std::string &err) {
    int q = p.model == PLQ_POTTS ? p.q : 2;
    float beta32 = (float)p.beta;
    out = Tables();
    if (updater == PLQ_HEATBATH || (updater == PLQ_METROPOLIS && q == 2)) {
        int64_t keys = env_key_count(p);
        int64_t entries = updater == PLQ_HEATBATH ? keys * (q - 1) : keys;
        if (keys > kMaxTableEntries || entries > kMaxTableEntries) {
            err = "the exact decision table for q = " + std::to_string(q) + " in " +
                  std::to_string(p.d) + " dimensions has more than " +
                  std::to_string(kMaxTableEntries) + " entries; this device path supports smaller q*d";
            return false;
        }
        if (updater == PLQ_HEATBATH) {
            if (rng == PLQ_RNG_STREAM) out.hb53.assign((size_t)entries, 0);
            else out.hb24.assign((size_t)entries, 0);
        } else {
            if (rng == PLQ_RNG_STREAM) out.metro53.assign((size_t)keys, kAlways53);
            else out.metro24.assign((size_t)keys, kAlways24);
        }
        for (int64_t key = 0; key < keys; ++key) {
            int cur;
            double d64[64];
            float d32[64];
            if (!env_deltas(p, key, cur, d64, d32)) continue;
            if (updater == PLQ_HEATBATH) {
                if (rng == PLQ_RNG_STREAM) hb_cuts64(p, p.beta, q, d64, &out.hb53[key * (q - 1)]);
                else hb_cuts32(beta32, q, d32, &out.hb24[key * (q - 1)]);
            } else {
                int prop = 1 - cur;
                if (rng == PLQ_RNG_STREAM) out.metro53[key] = metro_cut64(p.beta, d64[prop]);
                else out.metro24[key] = metro_cut32(beta32, d32[prop]);
            }
        }
        return true;
    }
    if (updater == PLQ_METROPOLIS) {  // Potts, q >= 3: keyed by (cur, prop, c_prop, c_cur)
        int64_t b = 2 * p.d + 1;
        int64_t keys = potts_metro_key_count(p);
        if (keys > kMaxTableEntries) {
            err = "the Potts Metropolis table is too large for this q and d";
            return false;
        }
        if (rng == PLQ_RNG_STREAM) out.metro53.assign((size_t)keys, kAlways53);
        else out.metro24.assign((size_t)keys, kAlways24);
        for (int cur = 0; cur < q; ++cur)
            for (int prop = 0; prop < q; ++prop)
                for (int cp = 0; cp < b; ++cp)
                    for (int cc = 0; cc < b; ++cc) {
                        int64_t key = (((int64_t)cur * q + prop) * b + cp) * b + cc;
                        if (prop == cur || cp + cc > 2 * p.d) continue;
                        int change = cp - cc;
                        if (rng == PLQ_RNG_STREAM)
                            out.metro53[key] = metro_cut64(p.beta, potts_delta64(p, cur, prop, change));
                        else
                            out.metro24[key] = metro_cut32(beta32, potts_delta32(p, cur, prop, change));
                    }
        return true;
    }
    err = "no decision table for this updater";
    return false;
}

// ---------------------------------------------------------------- PCG64
static const u128h kMult = ((u128h)0x2360ED051FC65DA4ULL << 64) | (u128h)0x4385DF649FCCF645ULL;

static uint64_t rotr64h(uint64_t x, unsigned r) {
    r &= 63u;
    return r ? (x >> r) | (x << (64u - r)) : x;
}

uint64_t HostPcg::next_u64() {
    state = state * kMult + inc;
    ++draws;
    return rotr64h((uint64_t)(state >> 64) ^ (uint64_t)state, (unsigned)(state >> 122));
}

// rand 0.10 random_range(0..n) for usize (UniformUsize -> u32 or u64
// widening-multiply sampler with one bias-reducing draw).
uint64_t HostPcg::next_below(uint64_t n) {
    uint64_t high = n - 1;
    if (high <= 0xFFFFFFFFULL) {
        uint32_t range = (uint32_t)(high + 1);
        if (range == 0) return (uint32_t)next_u64();
        uint32_t x = (uint32_t)next_u64();
        uint64_t m = (uint64_t)x * range;
        uint32_t result = (uint32_t)(m >> 32), lo = (uint32_t)m;
        if (lo > (uint32_t)(0u - range)) {
            uint32_t x2 = (uint32_t)next_u64();
            uint32_t hi2 = (uint32_t)(((uint64_t)x2 * range) >> 32);
            if ((uint64_t)lo + hi2 > 0xFFFFFFFFULL) result += 1;
        }
        return result;
    }
    uint64_t range = high + 1;
    if (range == 0) return next_u64();
    uint64_t x = next_u64();
    u128h m = (u128h)x * range;
    uint64_t result = (uint64_t)(m >> 64), lo = (uint64_t)m;
    if (lo > (0ULL - range)) {
        uint64_t x2 = next_u64();
        uint64_t hi2 = (uint64_t)(((u128h)x2 * range) >> 64);
        if (lo + hi2 < lo) result += 1;
    }
    return result;
}

// rand_core SeedableRng::seed_from_u64: PCG32 fills the 32-byte seed;
// Lcg128Xsl64::from_seed takes state = bytes[0..16] (LE), increment =
// bytes[16..32] (LE) | 1, then from_state_incr adds the increment and steps.
void pcg_seed_from_u64(uint64_t seed, uint64_t &s_lo, uint64_t &s_hi, uint64_t &i_lo,
                       uint64_t &i_hi) {
    uint32_t words[8];
    uint64_t st = seed;
    for (int c = 0; c < 8; ++c) {
        st = st * 6364136223846793005ULL + 11634580027462260723ULL;
        uint32_t xs = (uint32_t)(((st >> 18) ^ st) >> 27);
        unsigned rot = (unsigned)(st >> 59);
        words[c] = rot ? (xs >> rot) | (xs << (32u - rot)) : xs;
    }
    // little-endian words -> little-endian 128-bit integers
    u128h state = 0, incr = 0;
    for (int c = 3; c >= 0; --c) state = (state << 32) | words[c];
    for (int c = 7; c >= 4; --c) incr = (incr << 32) | words[c];
    incr |= 1u;
    state = state + incr;
    state = state * kMult + incr;
    s_lo = (uint64_t)state;
    s_hi = (uint64_t)(state >> 64);
    i_lo = (uint64_t)incr;
    i_hi = (uint64_t)(incr >> 64);
}

HostPcg host_pcg_from_seed(uint64_t seed) {
    uint64_t a, b, c, d;
    pcg_seed_from_u64(seed, a, b, c, d);
    HostPcg r;
    r.state = ((u128h)b << 64) | a;
    r.inc = ((u128h)d << 64) | c;
    r.draws = 0;
    return r;
}

struct AffH {
    u128h m, p;
};
static AffH comp(const AffH &f, const AffH &g) { return {g.m * f.m, g.m * f.p + g.p}; }

void build_jump_table(uint64_t inc_lo, uint64_t inc_hi, std::vector<AffineHost> &out) {
    const int digits = 8, radix = 256;
    out.resize((size_t)digits * radix);
    AffH base = {kMult, ((u128h)inc_hi << 64) | inc_lo};  // one step
    for (int d = 0; d < digits; ++d) {
        AffH acc = {1, 0};
        for (int v = 0; v < radix; ++v) {
            AffineHost &e = out[(size_t)d * radix + v];
            e.m_lo = (uint64_t)acc.m;
            e.m_hi = (uint64_t)(acc.m >> 64);
            e.p_lo = (uint64_t)acc.p;
            e.p_hi = (uint64_t)(acc.p >> 64);
            acc = comp(acc, base);
        }
        // next digit's unit = base^256 (acc is base^256 after the loop)
        base = acc;
    }
}

// Heap-free builders for callers that must not allocate: the q = 2
// Metropolis cut points of every environment key, and the jump table, each
// written into a caller-provided array.
int64_t q2_metro53_into(const ModelParams &p, uint64_t *out, int64_t capacity) {
    int64_t keys = env_key_count(p);
    if (keys > capacity) return -1;
    for (int64_t key = 0; key < keys; ++key) {
        int cur;
        double d64[2];
        float d32[2];
        out[key] = kAlways53;
        if (env_deltas(p, key, cur, d64, d32)) out[key] = metro_cut64(p.beta, d64[1 - cur]);
    }
    return keys;
}

void jump_table_into(uint64_t inc_lo, uint64_t inc_hi, AffineHost *out) {
    AffH base = {kMult, ((u128h)inc_hi << 64) | inc_lo};
    for (int d = 0; d < 8; ++d) {
        AffH acc = {1, 0};
        for (int v = 0; v < 256; ++v) {
            AffineHost &e = out[(size_t)d * 256 + v];
            e.m_lo = (uint64_t)acc.m;
            e.m_hi = (uint64_t)(acc.m >> 64);
            e.p_lo = (uint64_t)acc.p;
            e.p_hi = (uint64_t)(acc.p >> 64);
            acc = comp(acc, base);
        }
        base = acc;
    }
}

AffineHost affine_steps(const std::vector<AffineHost> &table, uint64_t n) {
    AffH acc = {1, 0};
    for (int d = 0; d < 8 && n; ++d) {
        unsigned v = (unsigned)(n & 255u);
        if (v) {
            const AffineHost &e = table[(size_t)d * 256 + v];
            AffH f = {((u128h)e.m_hi << 64) | e.m_lo, ((u128h)e.p_hi << 64) | e.p_lo};
            acc = comp(acc, f);
        }
        n >>= 8;
    }
    return {(uint64_t)acc.m, (uint64_t)(acc.m >> 64), (uint64_t)acc.p, (uint64_t)(acc.p >> 64)};
}

}  // namespace plq
