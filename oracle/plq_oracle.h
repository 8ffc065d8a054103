/*
 * plq_oracle.h -- CPU restatement of swvasquez/plaquette's lattice Monte Carlo
 * hot path.  TEST INFRASTRUCTURE ONLY: this library is the checker that the
 * CUDA product is compared against (and the timed CPU baseline).  Nothing in
 * the product links, loads or calls it.
 *
 * Two randomness back-ends, matching the two streams the reference uses:
 *
 *   STREAM  the reference CPU `Rng` (src/rng.rs:30-50): rand_pcg 0.10.2
 *           `Pcg64` (= Lcg128Xsl64) seeded by rand_core 0.10.1
 *           `seed_from_u64`, with rand 0.10.2's `random::<f64>()` and
 *           `random_range(0..n)` conversions.  Those crates are NOT vendored
 *           in the reference (Cargo.lock:681-701); their published algorithms
 *           are restated here.  The LCG128/XSL-RR core is pinned against
 *           numpy's PCG64 and the PCG paper's known-answer vectors; the
 *           seeding and the two conversions are restated from the crates'
 *           documented algorithms and are PARITY UNPINNED (no cargo here).
 *
 *   KEYED   the reference GPU stream: `lowbias32` / `keyed_uniform`
 *           (src/wgsl/rng.wgsl:34-52), fully specified by reference source.
 *
 * Every update rule is restated from the reference file:line named beside it.
 */
#ifndef PLQ_ORACLE_H
#define PLQ_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ----------------------------------------------------------------- RNG */

/* PCG64 state as four 64-bit words plus a draw counter (next_u64 calls). */
typedef struct {
    uint64_t state_lo, state_hi;
    uint64_t inc_lo, inc_hi;
    uint64_t draws;
} orc_rng;

void     orc_rng_seed_from_u64(orc_rng *r, uint64_t seed);
void     orc_rng_from_state(orc_rng *r, uint64_t slo, uint64_t shi,
                            uint64_t ilo, uint64_t ihi);
uint64_t orc_rng_next_u64(orc_rng *r);
double   orc_rng_next_f64(orc_rng *r);
uint64_t orc_rng_next_below(orc_rng *r, uint64_t n);
/* Advance by `delta` next_u64 steps (O(log delta) jump-ahead). */
void     orc_rng_advance(orc_rng *r, uint64_t delta);

uint32_t orc_lowbias32(uint32_t x);
float    orc_keyed_uniform(uint32_t seed, uint32_t variable, uint32_t sweep);
uint32_t orc_fold_seed(uint64_t seed);

/* Configuration::hot (src/configuration.rs:82-87): n draws of next_below(q). */
void     orc_hot_start(orc_rng *r, int32_t q, int64_t n, uint8_t *out);

/* ------------------------------------------------------------- lattice */

#define ORC_MAX_D 16

typedef struct {
    int32_t  d;
    int64_t  shape[ORC_MAX_D];
    int64_t  n_sites;
    int64_t  stride[ORC_MAX_D];
    int64_t *neighbors;   /* n_sites * 2d, row +0,-0,+1,-1,... */
    uint8_t *parity;      /* n_sites */
    int64_t *staples;     /* n_links * 6(d-1), or NULL until built */
} orc_lattice;

int  orc_lattice_init(orc_lattice *lat, int32_t d, const int64_t *shape);
int  orc_lattice_build_staples(orc_lattice *lat);
void orc_lattice_free(orc_lattice *lat);

/* -------------------------------------------------------------- models */

enum { ORC_ISING = 0, ORC_POTTS = 1, ORC_GAUGE = 2 };
enum { ORC_METROPOLIS = 0, ORC_HEATBATH = 1 };
enum { ORC_SCHED_RANDOM = 0, ORC_SCHED_CHECKERBOARD = 1 };
enum { ORC_EXTENT_ALL = 0, ORC_EXTENT_SEEDED = 1 };
enum { ORC_RELABEL_REDRAW = 0, ORC_RELABEL_FORCED = 1 };

#define ORC_MAX_Q 64

typedef struct {
    int32_t model;
    int32_t q;
    double  j;
    double  h;                 /* Ising field */
    double  offsets[ORC_MAX_Q];/* Potts per-label offsets */
} orc_model;

double orc_energy(const orc_model *m, const orc_lattice *lat, const uint8_t *cfg);
double orc_energy_delta(const orc_model *m, const orc_lattice *lat,
                        const uint8_t *cfg, int64_t var, int32_t proposed);
/* Integer primaries: Ising {bond_sum, spin_sum}; Potts {agree, counts[q]};
 * gauge {plaquette_sum}.  Returns how many int64 were written. */
int    orc_primaries(const orc_model *m, const orc_lattice *lat,
                     const uint8_t *cfg, int64_t *out);

/* -------------------------------------------------- CPU reference path */

/* LocalUpdate::sweep (src/updater.rs:283-348).  Returns the net dE. */
double orc_local_sweep(const orc_model *m, const orc_lattice *lat, uint8_t *cfg,
                       int32_t kernel, int32_t schedule, double beta, orc_rng *r);
double orc_local_sweeps(const orc_model *m, const orc_lattice *lat, uint8_t *cfg,
                        int32_t kernel, int32_t schedule, double beta, orc_rng *r,
                        int64_t n_sweeps);
/* A bounded slice of a checkerboard site sweep: the colour-`color` sites with
 * index in [lo, hi), in index order (used to time a fixed update budget). */
double orc_local_site_slice(const orc_model *m, const orc_lattice *lat, uint8_t *cfg,
                            int32_t kernel, double beta, orc_rng *r,
                            int32_t color, int64_t lo, int64_t hi, int64_t *updates);

/* ClusterUpdate::bond_probability (src/updater.rs:499-501). */
double orc_bond_probability(const orc_model *m, double beta);
/* site_clusters (src/cluster.rs:44-62) with the ClusterUpdate predicate
 * `peek(i)==peek(j) && next_f64() < p`; writes compacted labels (n_sites)
 * and returns the cluster count.  sizes may be NULL. */
int64_t orc_site_clusters(const orc_lattice *lat, const uint8_t *cfg, double p,
                          orc_rng *r, int64_t *labels, int64_t *sizes);
/* grow_cluster (src/cluster.rs:88-111) with the same predicate; returns the
 * member count, members in the order reached. */
int64_t orc_grow_cluster(const orc_lattice *lat, const uint8_t *cfg, int64_t seed,
                         double p, orc_rng *r, int64_t *members);
/* ClusterUpdate::sweep (src/updater.rs:541-613).  Returns the net dE. */
double orc_cluster_sweep(const orc_model *m, const orc_lattice *lat, uint8_t *cfg,
                         int32_t extent, int32_t relabel, double beta, orc_rng *r);

/* ----------------------------------------- reference GPU (keyed) path */

/* One sweep of the WGSL checkerboard (metropolis.wgsl / heat_bath.wgsl under
 * site_schedule.wgsl / link_schedule.wgsl) keyed by (seed32, var, sweep).
 * Arithmetic is f32 with each operation rounded separately in source order;
 * exp is evaluated as (float)exp((double)x). */
void orc_keyed_local_sweep(const orc_model *m, const orc_lattice *lat, uint8_t *cfg,
                           int32_t kernel, double beta, uint32_t seed32, uint32_t sweep);
/* One keyed colour pass of a site model over sites [first, last) of a slab of
 * a larger lattice (its planes with a halo plane on each side): draws at
 * variable index site + var_offset, colour in the slab's own parity. */
void orc_keyed_slab_pass(const orc_model *m, const orc_lattice *slab, uint8_t *cfg, int32_t kernel, double beta,
                         uint32_t seed32, uint32_t sweep, int32_t local_color, int64_t first, int64_t last,
                         int64_t var_offset);
/* One keyed cluster sweep (cluster_prelude.wgsl + cluster_relabel.wgsl):
 * bonds keyed by bond index, clusters rooted at their minimum site index,
 * relabel keyed on the root.  root_out (n_sites, may be NULL) receives the
 * canonical min-site label of every site before relabelling. */
void orc_keyed_cluster_sweep(const orc_model *m, const orc_lattice *lat, uint8_t *cfg,
                             int32_t extent, int32_t relabel, double beta,
                             uint32_t seed32, uint32_t sweep, int64_t *root_out);

/* ------------------------------------------------------ measurements */
/* axis_pair_sums (src/models/mod.rs:44-61) with Ising's product of signs
 * (ising/mod.rs:84-95) or Potts's equality (potts/mod.rs:218-234): entry
 * off_mu + r for r = 0..L_mu/2, off_mu = sum over nu < mu of (L_nu/2 + 1).
 * Returns the number of entries written. */
int64_t orc_axis_pair_sums(const orc_model *m, const orc_lattice *lat, const uint8_t *cfg, int64_t *out);
/* Z2Gauge::polyakov_loop (gauge/mod.rs:179-212) before the final division:
 * the sum of the line products along `dir`; *lines gets the divisor. */
int64_t orc_polyakov_sum(const orc_lattice *lat, const uint8_t *cfg, int32_t dir, int64_t *lines);
/* Z2Gauge::wilson_rectangles (gauge/mod.rs:226-274) before the divisions:
 * totals[r * (max + 1) + t] = sum of the rectangle products over every
 * ordered plane and site (r, t >= 1), *placements the divisor.  Returns max. */
int32_t orc_wilson_totals(const orc_lattice *lat, const uint8_t *cfg, int32_t max_side, int64_t *totals,
                          int64_t *placements);

/* -------------------------------------------------- parallel tempering */
/* The reference has no tempering; this restates the batched-ensemble swap
 * rule of this backend so its decisions are checked independently.
 *
 * orc_pt_exp: e^x for x <= 0 from IEEE basic operations only, each rounded
 * on its own: x = n ln2 + r (n = floor(x/ln2 + 1/2), ln2 split in a 32-bit
 * high part and a low part after Cody and Waite), e^r by its Taylor
 * polynomial to degree 14 in Horner form, times 2^n; 0 below x = -708. */
double orc_pt_exp(double x);
/* One swap phase of one ladder, attempt `att`: for slots k = att & 1,
 * att & 1 + 2, ... with k + 1 < k_slots, members m1 = slot[k] and
 * m2 = slot[k + 1] at betas b1, b2 with energies E = -J * energy (the bond,
 * agreement or plaquette sum; no field) exchange betas and slots when
 * delta = (b1 - b2)(E1 - E2) >= 0 or u < orc_pt_exp(delta), where
 * u = (h1 + h2 2^-24) 2^-24 with h1, h2 the 24-bit keyed hashes of
 * (seed32 ^ 0x6a09e667, k, att) and (seed32 ^ 0xbb67ae85, k, att).
 * Returns the number of accepted swaps. */
int32_t orc_pt_swap_phase(int32_t k_slots, int32_t *member_of_slot, double *beta_of_member,
                          const int64_t *energy, const double *j_of_member, uint32_t seed32, uint64_t att);

#ifdef __cplusplus
}
#endif
#endif
