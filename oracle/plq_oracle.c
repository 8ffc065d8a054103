/*
 * plq_oracle.c -- CPU restatement of the reference's lattice Monte Carlo hot
 * path.  TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline);
 * see plq_oracle.h for the pinning status of each part.
 *
 * Floating point: built with -ffp-contract=off and SSE2 scalar arithmetic so
 * every f64/f32 operation is rounded on its own, in the order the reference
 * writes it.  exp is glibc's, the same libm Rust's f64::exp calls on Linux.
 */
#include "plq_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* ================================================================== RNG */

/* rand_pcg 0.10.2 pcg128.rs: MULTIPLIER of Lcg128Xsl64 (the PCG paper's
 * default 128-bit multiplier). */
static const u128 PCG_MULT =
    ((u128)0x2360ED051FC65DA4ULL << 64) | (u128)0x4385DF649FCCF645ULL;

static u128 rng_state(const orc_rng *r) { return ((u128)r->state_hi << 64) | r->state_lo; }
static u128 rng_inc(const orc_rng *r) { return ((u128)r->inc_hi << 64) | r->inc_lo; }
static void rng_set_state(orc_rng *r, u128 s) {
    r->state_lo = (uint64_t)s;
    r->state_hi = (uint64_t)(s >> 64);
}

static uint64_t rotr64(uint64_t x, unsigned r) {
    r &= 63u;
    return r ? (x >> r) | (x << (64u - r)) : x;
}
static uint32_t rotr32(uint32_t x, unsigned r) {
    r &= 31u;
    return r ? (x >> r) | (x << (32u - r)) : x;
}

/* Lcg128Xsl64::from_state_incr: state += incr, then one LCG step. */
static void rng_from_state_incr(orc_rng *r, u128 state, u128 incr) {
    r->inc_lo = (uint64_t)incr;
    r->inc_hi = (uint64_t)(incr >> 64);
    state = state + incr;
    state = state * PCG_MULT + incr;
    rng_set_state(r, state);
    r->draws = 0;
}

/* rand_core 0.10.1 SeedableRng::seed_from_u64 (default method): a PCG32
 * stream (advance first, XSH-RR output) fills the 32-byte seed in 4-byte
 * little-endian chunks; Lcg128Xsl64::from_seed reads state = bytes[0..16],
 * increment = bytes[16..32] | 1, both little-endian. */
void orc_rng_seed_from_u64(orc_rng *r, uint64_t seed) {
    const uint64_t MUL = 6364136223846793005ULL;
    const uint64_t INC = 11634580027462260723ULL;
    uint8_t bytes[32];
    uint64_t st = seed;
    for (int c = 0; c < 8; ++c) {
        st = st * MUL + INC;
        uint32_t xorshifted = (uint32_t)(((st >> 18) ^ st) >> 27);
        uint32_t rot = (uint32_t)(st >> 59);
        uint32_t x = rotr32(xorshifted, rot);
        bytes[4 * c + 0] = (uint8_t)(x);
        bytes[4 * c + 1] = (uint8_t)(x >> 8);
        bytes[4 * c + 2] = (uint8_t)(x >> 16);
        bytes[4 * c + 3] = (uint8_t)(x >> 24);
    }
    u128 state = 0, incr = 0;
    for (int b = 15; b >= 0; --b) state = (state << 8) | bytes[b];
    for (int b = 31; b >= 16; --b) incr = (incr << 8) | bytes[b];
    rng_from_state_incr(r, state, incr | 1u);
}

void orc_rng_from_state(orc_rng *r, uint64_t slo, uint64_t shi, uint64_t ilo, uint64_t ihi) {
    r->state_lo = slo;
    r->state_hi = shi;
    r->inc_lo = ilo;
    r->inc_hi = ihi;
    r->draws = 0;
}

/* Lcg128Xsl64::next_u64: step the LCG, then XSL-RR of the new state. */
uint64_t orc_rng_next_u64(orc_rng *r) {
    u128 s = rng_state(r) * PCG_MULT + rng_inc(r);
    rng_set_state(r, s);
    r->draws++;
    unsigned rot = (unsigned)(s >> 122);
    uint64_t xsl = (uint64_t)(s >> 64) ^ (uint64_t)s;
    return rotr64(xsl, rot);
}

/* rand 0.10.2 StandardUniform for f64: 53 high bits times 2^-53. */
double orc_rng_next_f64(orc_rng *r) {
    uint64_t v = orc_rng_next_u64(r) >> 11;
    return (double)v * (1.0 / 9007199254740992.0);
}

/* rand 0.10.2 `random_range(0..n)` for usize: UniformUsize samples through
 * the u32 sampler when the inclusive high fits a u32, else through u64; both
 * use the widening-multiply method with one bias-reducing extra draw
 * (sample_single_inclusive).  u32 draws are next_u64 truncated. */
uint64_t orc_rng_next_below(orc_rng *r, uint64_t n) {
    uint64_t high = n - 1;
    if (high <= 0xFFFFFFFFULL) {
        uint32_t range = (uint32_t)(high + 1);
        if (range == 0) return (uint32_t)orc_rng_next_u64(r);
        uint32_t x = (uint32_t)orc_rng_next_u64(r);
        uint64_t m = (uint64_t)x * range;
        uint32_t result = (uint32_t)(m >> 32);
        uint32_t lo = (uint32_t)m;
        if (lo > (uint32_t)(0u - range)) {
            uint32_t x2 = (uint32_t)orc_rng_next_u64(r);
            uint32_t new_hi = (uint32_t)(((uint64_t)x2 * range) >> 32);
            if ((uint64_t)lo + new_hi > 0xFFFFFFFFULL) result += 1;
        }
        return result;
    } else {
        uint64_t range = high + 1;
        if (range == 0) return orc_rng_next_u64(r);
        uint64_t x = orc_rng_next_u64(r);
        u128 m = (u128)x * range;
        uint64_t result = (uint64_t)(m >> 64);
        uint64_t lo = (uint64_t)m;
        if (lo > (0ULL - range)) {
            uint64_t x2 = orc_rng_next_u64(r);
            uint64_t new_hi = (uint64_t)(((u128)x2 * range) >> 64);
            if (lo + new_hi < lo) result += 1;
        }
        return result;
    }
}

/* Jump-ahead by `delta` LCG steps (Brown, "Random number generation with
 * arbitrary strides", 1994), as PCG's advance. */
void orc_rng_advance(orc_rng *r, uint64_t delta) {
    u128 cur_mult = PCG_MULT, cur_plus = rng_inc(r);
    u128 acc_mult = 1, acc_plus = 0;
    uint64_t d = delta;
    while (d > 0) {
        if (d & 1u) {
            acc_mult *= cur_mult;
            acc_plus = acc_plus * cur_mult + cur_plus;
        }
        cur_plus = (cur_mult + 1) * cur_plus;
        cur_mult *= cur_mult;
        d >>= 1;
    }
    rng_set_state(r, acc_mult * rng_state(r) + acc_plus);
    r->draws += delta;
}

void orc_hot_start(orc_rng *r, int32_t q, int64_t n, uint8_t *out) {
    for (int64_t i = 0; i < n; ++i) out[i] = (uint8_t)orc_rng_next_below(r, (uint64_t)q);
}

/* src/wgsl/rng.wgsl:34-42 */
uint32_t orc_lowbias32(uint32_t x) {
    uint32_t v = x;
    v ^= v >> 16;
    v *= 0x7feb352du;
    v ^= v >> 15;
    v *= 0x846ca68bu;
    v ^= v >> 16;
    return v;
}

/* src/wgsl/rng.wgsl:47-52 */
float orc_keyed_uniform(uint32_t seed, uint32_t variable, uint32_t sweep) {
    uint32_t k = seed;
    k = orc_lowbias32(k ^ variable);
    k = orc_lowbias32(k ^ (sweep * 0x9e3779b9u));
    return (float)(k >> 8) * (1.0f / 16777216.0f);
}

/* src/device.rs:761-763 */
uint32_t orc_fold_seed(uint64_t seed) { return (uint32_t)(seed ^ (seed >> 32)); }

/* ============================================================== lattice */

/* src/lattice.rs:55-122: mixed-radix packing, direction 0 fastest; neighbour
 * rows +0,-0,+1,-1,...; coordinate-sum parity. */
int orc_lattice_init(orc_lattice *lat, int32_t d, const int64_t *shape) {
    memset(lat, 0, sizeof(*lat));
    if (d <= 0 || d > ORC_MAX_D) return -1;
    lat->d = d;
    int64_t n = 1;
    for (int mu = 0; mu < d; ++mu) {
        if (shape[mu] <= 0) return -1;
        lat->shape[mu] = shape[mu];
        lat->stride[mu] = n;
        n *= shape[mu];
    }
    lat->n_sites = n;
    lat->neighbors = (int64_t *)malloc(sizeof(int64_t) * (size_t)n * 2 * (size_t)d);
    lat->parity = (uint8_t *)malloc((size_t)n);
    if (!lat->neighbors || !lat->parity) return -2;
    for (int64_t site = 0; site < n; ++site) {
        int64_t coord_sum = 0;
        for (int mu = 0; mu < d; ++mu) {
            int64_t l = lat->shape[mu], s = lat->stride[mu];
            int64_t coord = (site / s) % l;
            int64_t base = site - coord * s;
            coord_sum += coord;
            lat->neighbors[site * 2 * d + 2 * mu] = base + ((coord + 1) % l) * s;
            lat->neighbors[site * 2 * d + 2 * mu + 1] = base + ((coord + l - 1) % l) * s;
        }
        lat->parity[site] = (uint8_t)(coord_sum % 2);
    }
    return 0;
}

/* src/lattice.rs:278-292 (dir_pair). */
static void dir_pair(int d, int64_t pair, int *mu_out, int *nu_out) {
    int64_t rest = pair;
    int mu = 0;
    for (;;) {
        int64_t in_group = d - 1 - mu;
        if (rest < in_group) {
            *mu_out = mu;
            *nu_out = (int)(mu + 1 + rest);
            return;
        }
        rest -= in_group;
        mu += 1;
    }
}

/* src/lattice.rs:455-466 (plaquette_links): [(s,mu),(s+mu,nu),(s+nu,mu),(s,nu)] */
static void plaquette_links(const orc_lattice *lat, int64_t plaquette, int64_t links[4]) {
    int d = lat->d;
    int64_t n_pairs = (int64_t)d * (d - 1) / 2;
    int64_t site = plaquette / n_pairs;
    int mu, nu;
    dir_pair(d, plaquette % n_pairs, &mu, &nu);
    int64_t site_mu = lat->neighbors[site * 2 * d + 2 * mu];
    int64_t site_nu = lat->neighbors[site * 2 * d + 2 * nu];
    links[0] = site * d + mu;
    links[1] = site_mu * d + nu;
    links[2] = site_nu * d + mu;
    links[3] = site * d + nu;
}

/* src/lattice.rs:136-163 (build_staples): plaquettes in index order, each of
 * a plaquette's links gets the other three as one group. */
int orc_lattice_build_staples(orc_lattice *lat) {
    int d = lat->d;
    if (d < 2) return -1;
    int64_t stride = 6 * (int64_t)(d - 1);
    int64_t n_links = lat->n_sites * d;
    int64_t n_plaq = lat->n_sites * (int64_t)d * (d - 1) / 2;
    lat->staples = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n_links * stride));
    int64_t *filled = (int64_t *)calloc((size_t)n_links, sizeof(int64_t));
    if (!lat->staples || !filled) {
        free(filled);
        return -2;
    }
    for (int64_t p = 0; p < n_plaq; ++p) {
        int64_t links[4];
        plaquette_links(lat, p, links);
        for (int i = 0; i < 4; ++i) {
            int64_t link = links[i];
            int64_t base = link * stride + filled[link] * 3;
            int slot = 0;
            for (int j = 0; j < 4; ++j)
                if (j != i) lat->staples[base + slot++] = links[j];
            filled[link] += 1;
        }
    }
    free(filled);
    return 0;
}

void orc_lattice_free(orc_lattice *lat) {
    free(lat->neighbors);
    free(lat->parity);
    free(lat->staples);
    memset(lat, 0, sizeof(*lat));
}

/* =============================================================== models */

/* src/models/mod.rs:30-32 */
static int decode(int s) { return 1 - 2 * s; }

static int potts_symmetric(const orc_model *m) {
    for (int a = 0; a < m->q; ++a)
        if (m->offsets[a] != 0.0) return 0;
    return 1;
}

static int64_t gauge_plaquette_sum(const orc_lattice *lat, const uint8_t *cfg) {
    int d = lat->d;
    int64_t n_plaq = lat->n_sites * (int64_t)d * (d - 1) / 2;
    int64_t sum = 0;
    for (int64_t p = 0; p < n_plaq; ++p) {
        int64_t links[4];
        plaquette_links(lat, p, links);
        int32_t prod = 1;
        for (int k = 0; k < 4; ++k) prod *= decode(cfg[links[k]]);
        sum += prod;
    }
    return sum;
}

/* Ising::energy (src/models/ising/mod.rs:98-117), Potts::energy
 * (src/models/potts/mod.rs:238-271), Z2Gauge::energy (gauge/mod.rs:276-285). */
double orc_energy(const orc_model *m, const orc_lattice *lat, const uint8_t *cfg) {
    int d = lat->d;
    int64_t n = lat->n_sites;
    if (m->model == ORC_ISING) {
        int64_t bond_sum = 0, spin_sum = 0;
        for (int64_t site = 0; site < n; ++site) {
            int s_i = decode(cfg[site]);
            spin_sum += s_i;
            for (int mu = 0; mu < d; ++mu)
                bond_sum += (int64_t)(s_i * decode(cfg[lat->neighbors[site * 2 * d + 2 * mu]]));
        }
        return -m->j * (double)bond_sum - m->h * (double)spin_sum;
    } else if (m->model == ORC_POTTS) {
        int64_t agree = 0;
        for (int64_t site = 0; site < n; ++site)
            for (int mu = 0; mu < d; ++mu)
                agree += cfg[lat->neighbors[site * 2 * d + 2 * mu]] == cfg[site];
        double offset = 0.0;
        if (!potts_symmetric(m)) {
            int64_t counts[ORC_MAX_Q] = {0};
            for (int64_t site = 0; site < n; ++site) counts[cfg[site]]++;
            offset = -0.0;
            for (int a = 0; a < m->q; ++a) offset = offset + m->offsets[a] * (double)counts[a];
        }
        return -m->j * (double)agree - offset;
    } else {
        return -m->j * (double)gauge_plaquette_sum(lat, cfg);
    }
}

/* Ising::energy_delta (ising/mod.rs:119-143), Potts::energy_delta
 * (potts/mod.rs:273-308), Z2Gauge::energy_delta (gauge/mod.rs:287-328). */
double orc_energy_delta(const orc_model *m, const orc_lattice *lat, const uint8_t *cfg,
                        int64_t var, int32_t proposed) {
    int d = lat->d;
    int cur = cfg[var];
    if (m->model == ORC_ISING) {
        int64_t ds = (int64_t)(decode(proposed) - decode(cur));
        if (ds == 0) return 0.0;
        int64_t nsum = 0;
        for (int k = 0; k < 2 * d; ++k) nsum += decode(cfg[lat->neighbors[var * 2 * d + k]]);
        return -(double)ds * (m->j * (double)nsum + m->h);
    } else if (m->model == ORC_POTTS) {
        if (proposed == cur) return 0.0;
        int64_t change = 0;
        for (int k = 0; k < 2 * d; ++k) {
            int s = cfg[lat->neighbors[var * 2 * d + k]];
            change += (int64_t)(s == proposed) - (int64_t)(s == cur);
        }
        double offset = m->offsets[proposed] - m->offsets[cur];
        return -m->j * (double)change - offset;
    } else {
        int64_t ds = (int64_t)(decode(proposed) - decode(cur));
        if (ds == 0) return 0.0;
        int64_t stride = 6 * (int64_t)(d - 1);
        int64_t staple_sum = 0;
        const int64_t *row = lat->staples + var * stride;
        for (int g = 0; g < 2 * (d - 1); ++g) {
            int32_t prod = 1;
            for (int k = 0; k < 3; ++k) prod *= decode(cfg[row[3 * g + k]]);
            staple_sum += prod;
        }
        return -m->j * (double)(ds * staple_sum);
    }
}

int orc_primaries(const orc_model *m, const orc_lattice *lat, const uint8_t *cfg, int64_t *out) {
    int d = lat->d;
    int64_t n = lat->n_sites;
    if (m->model == ORC_ISING) {
        int64_t bond_sum = 0, spin_sum = 0;
        for (int64_t site = 0; site < n; ++site) {
            int s_i = decode(cfg[site]);
            spin_sum += s_i;
            for (int mu = 0; mu < d; ++mu)
                bond_sum += s_i * decode(cfg[lat->neighbors[site * 2 * d + 2 * mu]]);
        }
        out[0] = bond_sum;
        out[1] = spin_sum;
        return 2;
    } else if (m->model == ORC_POTTS) {
        int64_t agree = 0;
        for (int a = 0; a < m->q; ++a) out[1 + a] = 0;
        for (int64_t site = 0; site < n; ++site) {
            out[1 + cfg[site]]++;
            for (int mu = 0; mu < d; ++mu) agree += cfg[lat->neighbors[site * 2 * d + 2 * mu]] == cfg[site];
        }
        out[0] = agree;
        return 1 + m->q;
    } else {
        out[0] = gauge_plaquette_sum(lat, cfg);
        return 1;
    }
}

/* ============================================ CPU reference: local update */

static int model_q(const orc_model *m) { return m->model == ORC_POTTS ? m->q : 2; }

/* propose (src/updater.rs:659-668) */
static int propose(int q, int cur, orc_rng *r) {
    if (q == 2) return 1 - cur;
    int draw = (int)orc_rng_next_below(r, (uint64_t)(q - 1));
    return draw + (draw >= cur);
}

/* step (src/updater.rs:77-96) */
static double step(const orc_model *m, const orc_lattice *lat, uint8_t *cfg, int64_t var,
                   double beta, orc_rng *r) {
    int proposed = propose(model_q(m), cfg[var], r);
    double delta = orc_energy_delta(m, lat, cfg, var, proposed);
    if (delta <= 0.0 || orc_rng_next_f64(r) < exp(-beta * delta)) {
        cfg[var] = (uint8_t)proposed;
        return delta;
    }
    return 0.0;
}

/* heat_bath_step (src/updater.rs:109-167) */
static double heat_bath_step(const orc_model *m, const orc_lattice *lat, uint8_t *cfg,
                             int64_t var, double beta, orc_rng *r) {
    int q = model_q(m);
    int cur = cfg[var];
    double deltas[ORC_MAX_Q];
    for (int s = 0; s < q; ++s) deltas[s] = (s == cur) ? 0.0 : orc_energy_delta(m, lat, cfg, var, s);
    double floor_ = INFINITY;
    for (int s = 0; s < q; ++s) floor_ = fmin(floor_, deltas[s]);
    double weights[ORC_MAX_Q];
    double total = 0.0;
    for (int s = 0; s < q; ++s) {
        weights[s] = exp(-beta * (deltas[s] - floor_));
        total += weights[s];
    }
    double target = orc_rng_next_f64(r) * total;
    int chosen = q - 1;
    double cumulative = 0.0;
    for (int s = 0; s < q - 1; ++s) {
        cumulative += weights[s];
        if (target < cumulative) {
            chosen = s;
            break;
        }
    }
    cfg[var] = (uint8_t)chosen;
    return deltas[chosen];
}

static double apply(const orc_model *m, const orc_lattice *lat, uint8_t *cfg, int32_t kernel,
                    int64_t var, double beta, orc_rng *r) {
    return kernel == ORC_METROPOLIS ? step(m, lat, cfg, var, beta, r)
                                    : heat_bath_step(m, lat, cfg, var, beta, r);
}

/* LocalUpdate::sweep (src/updater.rs:283-348) */
double orc_local_sweep(const orc_model *m, const orc_lattice *lat, uint8_t *cfg, int32_t kernel,
                       int32_t schedule, double beta, orc_rng *r) {
    int d = lat->d;
    int64_t n = lat->n_sites;
    int64_t n_vars = m->model == ORC_GAUGE ? n * d : n;
    double net = 0.0;
    if (schedule == ORC_SCHED_RANDOM) {
        for (int64_t i = 0; i < n_vars; ++i) {
            int64_t var = (int64_t)orc_rng_next_below(r, (uint64_t)n_vars);
            net += apply(m, lat, cfg, kernel, var, beta, r);
        }
    } else if (m->model != ORC_GAUGE) {
        for (int color = 0; color < 2; ++color)
            for (int64_t site = 0; site < n; ++site)
                if (lat->parity[site] == color) net += apply(m, lat, cfg, kernel, site, beta, r);
    } else {
        for (int dir = 0; dir < d; ++dir)
            for (int color = 0; color < 2; ++color)
                for (int64_t site = 0; site < n; ++site)
                    if (lat->parity[site] == color)
                        net += apply(m, lat, cfg, kernel, site * d + dir, beta, r);
    }
    return net;
}

double orc_local_sweeps(const orc_model *m, const orc_lattice *lat, uint8_t *cfg, int32_t kernel,
                        int32_t schedule, double beta, orc_rng *r, int64_t n_sweeps) {
    double net = 0.0;
    for (int64_t t = 0; t < n_sweeps; ++t) net += orc_local_sweep(m, lat, cfg, kernel, schedule, beta, r);
    return net;
}

double orc_local_site_slice(const orc_model *m, const orc_lattice *lat, uint8_t *cfg,
                            int32_t kernel, double beta, orc_rng *r, int32_t color, int64_t lo,
                            int64_t hi, int64_t *updates) {
    double net = 0.0;
    int64_t count = 0;
    for (int64_t site = lo; site < hi; ++site)
        if (lat->parity[site] == color) {
            net += apply(m, lat, cfg, kernel, site, beta, r);
            count++;
        }
    if (updates) *updates = count;
    return net;
}

/* ========================================== CPU reference: cluster update */

/* BondAction::bond_energy_gap: Ising 2j (ising/mod.rs:152-154), Potts j
 * (potts/mod.rs:314-316); ClusterUpdate::bond_probability (updater.rs:499-501) */
double orc_bond_probability(const orc_model *m, double beta) {
    double gap = m->model == ORC_ISING ? 2.0 * m->j : m->j;
    return 1.0 - exp(-beta * gap);
}

/* Forest (src/cluster.rs:151-227): union by size, path halving. */
typedef struct {
    int64_t *parent, *size;
} forest;

static int64_t forest_find(forest *f, int64_t site) {
    int64_t cur = site;
    while (f->parent[cur] != cur) {
        f->parent[cur] = f->parent[f->parent[cur]];
        cur = f->parent[cur];
    }
    return cur;
}

static void forest_union(forest *f, int64_t a, int64_t b) {
    int64_t big = forest_find(f, a), small = forest_find(f, b);
    if (big == small) return;
    if (f->size[big] < f->size[small]) {
        int64_t t = big;
        big = small;
        small = t;
    }
    f->parent[small] = big;
    f->size[big] += f->size[small];
}

int64_t orc_site_clusters(const orc_lattice *lat, const uint8_t *cfg, double p, orc_rng *r,
                          int64_t *labels, int64_t *sizes) {
    int d = lat->d;
    int64_t n = lat->n_sites;
    forest f;
    f.parent = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    f.size = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        f.parent[i] = i;
        f.size[i] = 1;
    }
    for (int64_t site = 0; site < n; ++site)
        for (int mu = 0; mu < d; ++mu) {
            int64_t partner = lat->neighbors[site * 2 * d + 2 * mu];
            if (cfg[site] == cfg[partner] && orc_rng_next_f64(r) < p) forest_union(&f, site, partner);
        }
    /* into_clusters: first encounter names the cluster. */
    int64_t *label_of_root = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    for (int64_t i = 0; i < n; ++i) label_of_root[i] = -1;
    int64_t n_clusters = 0;
    for (int64_t site = 0; site < n; ++site) {
        int64_t root = forest_find(&f, site);
        if (label_of_root[root] < 0) {
            label_of_root[root] = n_clusters;
            if (sizes) sizes[n_clusters] = 0;
            n_clusters++;
        }
        labels[site] = label_of_root[root];
        if (sizes) sizes[labels[site]]++;
    }
    free(label_of_root);
    free(f.parent);
    free(f.size);
    return n_clusters;
}

int64_t orc_grow_cluster(const orc_lattice *lat, const uint8_t *cfg, int64_t seed, double p,
                         orc_rng *r, int64_t *members) {
    int d = lat->d;
    int64_t n = lat->n_sites;
    uint8_t *member = (uint8_t *)calloc((size_t)n, 1);
    member[seed] = 1;
    int64_t len = 0;
    members[len++] = seed;
    int64_t next = 0;
    while (next < len) {
        int64_t site = members[next++];
        for (int k = 0; k < 2 * d; ++k) {
            int64_t partner = lat->neighbors[site * 2 * d + k];
            if (!member[partner] && cfg[site] == cfg[partner] && orc_rng_next_f64(r) < p) {
                member[partner] = 1;
                members[len++] = partner;
            }
        }
    }
    free(member);
    return len;
}

/* ClusterUpdate::fresh_label (src/updater.rs:507-521) */
static int fresh_label(int q, int32_t relabel, int current, orc_rng *r) {
    if (relabel == ORC_RELABEL_REDRAW) return (int)orc_rng_next_below(r, (uint64_t)q);
    return propose(q, current, r);
}

double orc_cluster_sweep(const orc_model *m, const orc_lattice *lat, uint8_t *cfg, int32_t extent,
                         int32_t relabel, double beta, orc_rng *r) {
    int q = model_q(m);
    int64_t n = lat->n_sites;
    double before = orc_energy(m, lat, cfg);
    double p = orc_bond_probability(m, beta);
    if (extent == ORC_EXTENT_ALL) {
        int64_t *labels = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
        int64_t n_clusters = orc_site_clusters(lat, cfg, p, r, labels, NULL);
        int *current = (int *)malloc(sizeof(int) * (size_t)(n_clusters > 0 ? n_clusters : 1));
        int64_t seen = 0;
        for (int64_t site = 0; site < n; ++site)
            if (labels[site] == seen) current[seen++] = cfg[site];
        for (int64_t c = 0; c < n_clusters; ++c) current[c] = fresh_label(q, relabel, current[c], r);
        for (int64_t site = 0; site < n; ++site) cfg[site] = (uint8_t)current[labels[site]];
        free(current);
        free(labels);
    } else {
        int64_t seed = (int64_t)orc_rng_next_below(r, (uint64_t)n);
        int64_t *members = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
        int64_t len = orc_grow_cluster(lat, cfg, seed, p, r, members);
        int fresh = fresh_label(q, relabel, cfg[seed], r);
        for (int64_t i = 0; i < len; ++i) cfg[members[i]] = (uint8_t)fresh;
        free(members);
    }
    return orc_energy(m, lat, cfg) - before;
}

/* ============================== reference GPU semantics (keyed stream) */

/* src/wgsl/metropolis.wgsl:26, cluster_prelude.wgsl:29, cluster_relabel.wgsl:41-45 */
#define PROPOSAL_KEY 0x85ebca6bu
#define BOND_KEY 0x27d4eb2fu
#define ROOT_SALT 0x85ebca6bu
#define SEED_SALT 0xc2b2ae35u

static float exp32(float x) { return (float)exp((double)x); }
static int spin_pm(int s) { return 1 - 2 * s; }

/* ising/model.wgsl:32-38, potts/model.wgsl:54-67, gauge/model.wgsl:31-42,
 * with params narrowed to f32 as the per-model gpu.rs constructors do. */
static float keyed_energy_delta(const orc_model *m, const orc_lattice *lat, const uint8_t *cfg,
                                int64_t v, int cur, int prop) {
    int d = lat->d;
    float j32 = (float)m->j;
    if (m->model == ORC_ISING) {
        int32_t nsum = 0;
        for (int k = 0; k < 2 * d; ++k) nsum += spin_pm(cfg[lat->neighbors[v * 2 * d + k]]);
        float h32 = (float)m->h;
        float t = j32 * (float)nsum;
        t = t + h32;
        float a = 2.0f * (float)spin_pm(cur);
        return a * t;
    } else if (m->model == ORC_POTTS) {
        int32_t change = 0;
        for (int k = 0; k < 2 * d; ++k) {
            int s = cfg[lat->neighbors[v * 2 * d + k]];
            if (s == prop) change += 1;
            if (s == cur) change -= 1;
        }
        float offset = (float)m->offsets[prop] - (float)m->offsets[cur];
        float t = (-j32) * (float)change;
        return t - offset;
    } else {
        int64_t stride = 6 * (int64_t)(d - 1);
        const int64_t *row = lat->staples + v * stride;
        int32_t staple_sum = 0;
        for (int g = 0; g < 2 * (d - 1); ++g) {
            int32_t prod = 1;
            for (int k = 0; k < 3; ++k) prod *= spin_pm(cfg[row[3 * g + k]]);
            staple_sum += prod;
        }
        float a = 2.0f * j32;
        a = a * (float)spin_pm(cur);
        return a * (float)staple_sum;
    }
}

/* metropolis.wgsl:32-63 and heat_bath.wgsl:28-62 */
/* v indexes cfg and the lattice's tables; key_var is the variable index the
 * keyed draws are taken at (v itself, except for a slab of a larger lattice,
 * whose variables keep their indices in the whole lattice). */
static void keyed_update(const orc_model *m, const orc_lattice *lat, uint8_t *cfg, int32_t kernel,
                         float beta32, uint32_t seed32, uint32_t sweep, int64_t v, int64_t key_var) {
    int q = model_q(m);
    int cur = cfg[v];
    if (kernel == ORC_METROPOLIS) {
        int prop;
        if (q == 2) {
            prop = 1 - cur;
        } else {
            uint32_t alternatives = (uint32_t)(q - 1);
            float u = orc_keyed_uniform(seed32 ^ PROPOSAL_KEY, (uint32_t)key_var, sweep);
            float scaled = u * (float)alternatives;
            uint32_t draw = (uint32_t)scaled;
            if (draw >= alternatives) draw = alternatives - 1;
            prop = (int)draw;
            if (prop >= cur) prop += 1;
        }
        float dE = keyed_energy_delta(m, lat, cfg, v, cur, prop);
        float u = orc_keyed_uniform(seed32, (uint32_t)key_var, sweep);
        float x = (-beta32) * dE;
        if (dE <= 0.0f || u < exp32(x)) cfg[v] = (uint8_t)prop;
    } else {
        float deltas[ORC_MAX_Q];
        float lowest = 0.0f;
        for (int s = 0; s < q; ++s) {
            float dE = 0.0f;
            if (s != cur) dE = keyed_energy_delta(m, lat, cfg, v, cur, s);
            deltas[s] = dE;
            lowest = fminf(lowest, dE);
        }
        float weights[ORC_MAX_Q];
        float total = 0.0f;
        for (int s = 0; s < q; ++s) {
            float t = deltas[s] - lowest;
            float x = (-beta32) * t;
            weights[s] = exp32(x);
            total = total + weights[s];
        }
        float threshold = orc_keyed_uniform(seed32, (uint32_t)key_var, sweep) * total;
        int chosen = q - 1;
        float cumulative = 0.0f;
        for (int s = 0; s + 1 < q; ++s) {
            cumulative = cumulative + weights[s];
            if (threshold < cumulative) {
                chosen = s;
                break;
            }
        }
        cfg[v] = (uint8_t)chosen;
    }
}

/* site_schedule.wgsl:15-31 / link_schedule.wgsl:23-40, encode_sweep
 * (src/device.rs:417-430): colour passes in order, one shared sweep index. */
void orc_keyed_local_sweep(const orc_model *m, const orc_lattice *lat, uint8_t *cfg,
                           int32_t kernel, double beta, uint32_t seed32, uint32_t sweep) {
    int d = lat->d;
    int64_t n = lat->n_sites;
    float beta32 = (float)beta;
    int colors = m->model == ORC_GAUGE ? 2 * d : 2;
    for (int color = 0; color < colors; ++color)
        for (int64_t site = 0; site < n; ++site) {
            if (lat->parity[site] != (color & 1)) continue;
            int64_t v = m->model == ORC_GAUGE ? site * d + (color >> 1) : site;
            keyed_update(m, lat, cfg, kernel, beta32, seed32, sweep, v, v);
        }
}

/* One keyed colour pass of a site model over sites [first, last) of a slab:
 * `slab` is the lattice of the slab's planes with one halo plane on each side
 * (periodic along its last axis, which the interior sites never cross), its
 * site s is site s + var_offset of the whole lattice, and local_color is the
 * pass's colour in the slab's own parity. */
void orc_keyed_slab_pass(const orc_model *m, const orc_lattice *slab, uint8_t *cfg, int32_t kernel, double beta,
                         uint32_t seed32, uint32_t sweep, int32_t local_color, int64_t first, int64_t last,
                         int64_t var_offset) {
    float beta32 = (float)beta;
    for (int64_t site = first; site < last; ++site) {
        if (slab->parity[site] != local_color) continue;
        keyed_update(m, slab, cfg, kernel, beta32, seed32, sweep, site, site + var_offset);
    }
}

static int64_t root_find(int64_t *parent, int64_t x) {
    while (parent[x] != x) {
        parent[x] = parent[parent[x]];
        x = parent[x];
    }
    return x;
}

/* cluster_prelude.wgsl:61-147 + cluster_relabel.wgsl:39-90.  The propagation
 * fixed point is the minimum site index of each component; computed here by
 * union-find followed by a min per component. */
void orc_keyed_cluster_sweep(const orc_model *m, const orc_lattice *lat, uint8_t *cfg,
                             int32_t extent, int32_t relabel, double beta, uint32_t seed32,
                             uint32_t sweep, int64_t *root_out) {
    int d = lat->d;
    int64_t n = lat->n_sites;
    int q = model_q(m);
    float p32 = (float)orc_bond_probability(m, beta);
    int64_t *parent = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    int64_t *minsite = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    for (int64_t i = 0; i < n; ++i) parent[i] = i;
    for (int64_t bond = 0; bond < n * d; ++bond) {
        int64_t site = bond / d;
        int axis = (int)(bond % d);
        int64_t partner = lat->neighbors[site * 2 * d + 2 * axis];
        int agree = cfg[site] == cfg[partner];
        int drawn = orc_keyed_uniform(seed32 ^ BOND_KEY, (uint32_t)bond, sweep) < p32;
        if (agree && drawn) {
            int64_t a = root_find(parent, site), b = root_find(parent, partner);
            if (a != b) parent[a < b ? b : a] = a < b ? a : b;
        }
    }
    for (int64_t i = 0; i < n; ++i) minsite[i] = INT64_MAX;
    for (int64_t i = 0; i < n; ++i) {
        int64_t r = root_find(parent, i);
        if (i < minsite[r]) minsite[r] = i;
    }
    int64_t *root = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    for (int64_t i = 0; i < n; ++i) root[i] = minsite[root_find(parent, i)];
    if (root_out) memcpy(root_out, root, sizeof(int64_t) * (size_t)n);

    int64_t seed_root = -1;
    if (extent == ORC_EXTENT_SEEDED) {
        float u = orc_keyed_uniform(seed32 ^ SEED_SALT, 0u, sweep);
        uint32_t seed_site = (uint32_t)(u * (float)(uint32_t)n);
        if (seed_site >= (uint32_t)n) seed_site = (uint32_t)n - 1u;
        seed_root = root[seed_site];
    }
    for (int64_t site = 0; site < n; ++site) {
        if (extent == ORC_EXTENT_SEEDED && root[site] != seed_root) continue;
        float u = orc_keyed_uniform(seed32 ^ ROOT_SALT, (uint32_t)root[site], sweep);
        if (relabel == ORC_RELABEL_FORCED) {
            uint32_t stp = (uint32_t)(u * (float)(uint32_t)(q - 1));
            if (stp >= (uint32_t)(q - 1)) stp = (uint32_t)(q - 2);
            cfg[site] = (uint8_t)((cfg[site] + 1u + stp) % (uint32_t)q);
        } else {
            uint32_t draw = (uint32_t)(u * (float)(uint32_t)q);
            if (draw >= (uint32_t)q) draw = (uint32_t)(q - 1);
            cfg[site] = (uint8_t)draw;
        }
    }
    free(root);
    free(minsite);
    free(parent);
}

/* ===================================================== measurements */

/* Lattice::site_shift (src/lattice.rs:353-361) */
static int64_t site_shift(const orc_lattice *lat, int64_t site, int dir, int64_t delta) {
    int64_t st = lat->stride[dir], l = lat->shape[dir];
    int64_t coord = (site / st) % l;
    int64_t base = site - coord * st;
    return base + ((coord + delta % l) % l) * st;
}

int64_t orc_axis_pair_sums(const orc_model *m, const orc_lattice *lat, const uint8_t *cfg, int64_t *out) {
    int d = lat->d;
    int64_t off = 0;
    for (int mu = 0; mu < d; ++mu) {
        int64_t half = lat->shape[mu] / 2;
        for (int64_t r = 0; r <= half; ++r) {
            int64_t sum = 0;
            for (int64_t site = 0; site < lat->n_sites; ++site) {
                int a = cfg[site], b = cfg[site_shift(lat, site, mu, r)];
                if (m->model == ORC_ISING)
                    sum += (int64_t)(decode(a) * decode(b));
                else
                    sum += a == b;
            }
            out[off + r] = sum;
        }
        off += half + 1;
    }
    return off;
}

/* Lattice::loop_links (src/lattice.rs:467-486) over the steps (dir, +1 / -1),
 * as a product of the link signs; links are cfg[site * d + dir]. */
static int loop_product(const orc_lattice *lat, const uint8_t *cfg, int64_t base, const int *dirs,
                        const int *signs, int n_steps) {
    int d = lat->d;
    int64_t site = base;
    int prod = 1;
    for (int k = 0; k < n_steps; ++k) {
        int dir = dirs[k];
        int64_t link;
        if (signs[k] > 0) {
            link = site * d + dir;
            site = site_shift(lat, site, dir, 1);
        } else {
            site = site_shift(lat, site, dir, lat->shape[dir] - 1);
            link = site * d + dir;
        }
        prod *= decode(cfg[link]);
    }
    return prod;
}

int64_t orc_polyakov_sum(const orc_lattice *lat, const uint8_t *cfg, int32_t dir, int64_t *lines) {
    int l = (int)lat->shape[dir];
    int *dirs = (int *)malloc(sizeof(int) * (size_t)l), *signs = (int *)malloc(sizeof(int) * (size_t)l);
    for (int k = 0; k < l; ++k) {
        dirs[k] = dir;
        signs[k] = 1;
    }
    int64_t total = 0, count = 0;
    for (int64_t site = 0; site < lat->n_sites; ++site) {
        if ((site / lat->stride[dir]) % lat->shape[dir] != 0) continue;
        total += loop_product(lat, cfg, site, dirs, signs, l);
        ++count;
    }
    free(dirs);
    free(signs);
    *lines = count;
    return total;
}

int32_t orc_wilson_totals(const orc_lattice *lat, const uint8_t *cfg, int32_t max_side, int64_t *totals,
                          int64_t *placements) {
    int d = lat->d;
    int64_t shortest = lat->shape[0];
    for (int mu = 1; mu < d; ++mu)
        if (lat->shape[mu] < shortest) shortest = lat->shape[mu];
    int32_t mx = max_side < shortest / 2 ? max_side : (int32_t)(shortest / 2);
    int *dirs = (int *)malloc(sizeof(int) * (size_t)(4 * mx + 4));
    int *signs = (int *)malloc(sizeof(int) * (size_t)(4 * mx + 4));
    for (int64_t i = 0; i < (int64_t)(mx + 1) * (mx + 1); ++i) totals[i] = 0;
    for (int r = 1; r <= mx; ++r)
        for (int t = 1; t <= mx; ++t) {
            int64_t total = 0;
            for (int mu = 0; mu < d; ++mu)
                for (int nu = 0; nu < d; ++nu) {
                    if (mu == nu) continue;
                    /* Loop::rectangle (src/lattice.rs:532-555): r x (mu,+), t x (nu,+), r x (mu,-), t x (nu,-) */
                    int n = 0;
                    for (int k = 0; k < r; ++k) dirs[n] = mu, signs[n++] = 1;
                    for (int k = 0; k < t; ++k) dirs[n] = nu, signs[n++] = 1;
                    for (int k = 0; k < r; ++k) dirs[n] = mu, signs[n++] = -1;
                    for (int k = 0; k < t; ++k) dirs[n] = nu, signs[n++] = -1;
                    for (int64_t site = 0; site < lat->n_sites; ++site)
                        total += loop_product(lat, cfg, site, dirs, signs, n);
                }
            totals[r * (mx + 1) + t] = total;
        }
    free(dirs);
    free(signs);
    *placements = (int64_t)d * (d - 1) * lat->n_sites;
    return mx;
}

/* ================================================== parallel tempering */

/* ln2 = PT_LN2_HI + PT_LN2_LO, PT_LN2_HI with 32 significant bits (so n * PT_LN2_HI
 * is exact for |n| < 2^21); 1/k! rounded to double. */
#define PT_INV_LN2 1.4426950408889634
#define PT_LN2_HI 0.6931471803691238
#define PT_LN2_LO 1.9082149292705877e-10

double orc_pt_exp(double x) {
    static const double inv_fact[15] = {
        1.0, 1.0, 0.5, 0.16666666666666666, 0.041666666666666664, 0.008333333333333333,
        0.001388888888888889, 0.0001984126984126984, 2.48015873015873e-05, 2.7557319223985893e-06,
        2.755731922398589e-07, 2.505210838544172e-08, 2.08767569878681e-09, 1.6059043836821613e-10,
        1.1470745597729725e-11};
    if (!(x > -708.0)) return 0.0;
    double t = x * PT_INV_LN2;
    double n = floor(t + 0.5);
    double hi = n * PT_LN2_HI;
    double lo = n * PT_LN2_LO;
    double r = (x - hi) - lo;
    double p = inv_fact[14];
    for (int k = 13; k >= 0; --k) p = p * r + inv_fact[k];
    uint64_t bits = (uint64_t)((int64_t)n + 1023) << 52;
    double scale;
    memcpy(&scale, &bits, sizeof scale);
    return p * scale;
}

static uint32_t keyed24(uint32_t seed, uint32_t variable, uint32_t sweep) {
    uint32_t k = orc_lowbias32(seed ^ variable);
    k = orc_lowbias32(k ^ (sweep * 0x9e3779b9u));
    return k >> 8;
}

int32_t orc_pt_swap_phase(int32_t k_slots, int32_t *member_of_slot, double *beta_of_member,
                          const int64_t *energy, const double *j_of_member, uint32_t seed32, uint64_t att) {
    int32_t accepted = 0;
    for (int32_t k = (int32_t)(att & 1u); k + 1 < k_slots; k += 2) {
        int32_t m1 = member_of_slot[k], m2 = member_of_slot[k + 1];
        double b1 = beta_of_member[m1], b2 = beta_of_member[m2];
        double e1 = -(j_of_member[m1] * (double)energy[m1]);
        double e2 = -(j_of_member[m2] * (double)energy[m2]);
        double delta = (b1 - b2) * (e1 - e2);
        uint32_t h1 = keyed24(seed32 ^ 0x6a09e667u, (uint32_t)k, (uint32_t)att);
        uint32_t h2 = keyed24(seed32 ^ 0xbb67ae85u, (uint32_t)k, (uint32_t)att);
        double u = ((double)h1 + (double)h2 * 5.9604644775390625e-8) * 5.9604644775390625e-8;
        if (delta >= 0.0 || u < orc_pt_exp(delta)) {
            beta_of_member[m1] = b2;
            beta_of_member[m2] = b1;
            member_of_slot[k] = m2;
            member_of_slot[k + 1] = m1;
            ++accepted;
        }
    }
    return accepted;
}
