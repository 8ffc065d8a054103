/*
 * plaquette.h -- C ABI of the B200 lattice Monte Carlo backend.
 *
 * This library replaces the reference's wgpu device path (src/device.rs,
 * src/gpu_cluster.rs, src/models/{ising,potts,gauge}/gpu.rs, the src/wgsl/ shaders)
 * behind the same chain semantics: a chain owns all device state, `advance`
 * runs sweeps without waiting, `next` runs `sweeps_between` sweeps and hands
 * back an owned copy of the configuration.  Plain C types only; the library
 * owns device memory, callers own host buffers.
 *
 * Two randomness modes:
 *   PLQ_RNG_STREAM  the reference CPU stream (src/rng.rs:30-50, PCG64 from
 *                   seed_from_u64): a sweep is bit-identical to
 *                   `LocalUpdate::sweep` with `Schedule::Checkerboard`
 *                   (src/updater.rs:283-348) or `ClusterUpdate::sweep`
 *                   (src/updater.rs:541-613) on the CPU.
 *   PLQ_RNG_KEYED   the reference GPU stream keyed by (seed, variable, sweep)
 *                   (src/wgsl/rng.wgsl:47-52), order-independent.
 *
 * Error handling: every entry point returns PLQ_OK or an error code; the
 * message of the last failure on the calling thread is plq_last_error().
 * Contract violations use the reference's panic wording.
 */
#ifndef PLAQUETTE_H
#define PLAQUETTE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ codes */
#define PLQ_OK 0
#define PLQ_ENODEV 1        /* no CUDA device: the reference's Gpu::new() == None */
#define PLQ_EINVAL 2        /* contract violation (message in plq_last_error) */
#define PLQ_EUNSUPPORTED 3  /* valid for the reference, outside this device path */
#define PLQ_ECUDA 4         /* a CUDA runtime call failed */
#define PLQ_ENOMEM 5        /* device or pinned-host allocation failed / over budget */
#define PLQ_ECAP 6          /* cluster labelling hit its pass cap (gpu_cluster.rs:512-518) */
#define PLQ_EDEVICE 7       /* a kernel reported a fault in its status word */
#define PLQ_EBUSY 8         /* serving: no slot or memory free right now */

#define PLQ_MAX_D 8
#define PLQ_MAX_Q 64

enum plq_model { PLQ_ISING = 0, PLQ_POTTS = 1, PLQ_GAUGE = 2 };
/* Kernel (src/updater.rs:179-190) or a cluster move (updater.rs:357-445). */
enum plq_updater { PLQ_METROPOLIS = 0, PLQ_HEATBATH = 1, PLQ_CLUSTER = 2 };
enum plq_extent { PLQ_EXTENT_ALL = 0, PLQ_EXTENT_SEEDED = 1 };       /* updater.rs:358-373 */
enum plq_relabel { PLQ_RELABEL_REDRAW = 0, PLQ_RELABEL_FORCED = 1 }; /* updater.rs:377-395 */
enum plq_rng { PLQ_RNG_STREAM = 0, PLQ_RNG_KEYED = 1 };
/* Force the per-colour pass kernels even where the fused two-colour sweep or
 * the bit-packed passes apply (all give identical results; used to check one
 * against the other). */
#define PLQ_FLAG_NO_FUSED 1
/* Cap every cluster-labelling find and union at one step, so any real merge
 * trips the cap: exercises the PLQ_ECAP path (gpu_cluster.rs:512-518) on the
 * host side without any device fault. */
#define PLQ_FLAG_TINY_PASS_CAP 2
/* Fused 3D sweep only: never issue the tile copies of one z-plane and wait
 * for them at most 1024 polls, so every tile's bounded wait runs out and the
 * launch reports PLQ_EDEVICE (status bit 16) -- exercises the copy-wait limit
 * without any device fault.  No reference counterpart (the reference has no
 * staged tiles). */
#define PLQ_FLAG_TEST_COPY_STALL 4
/* Run every colour pass one variable per rank (the generic pass body) even
 * where the four-sites-at-a-time body applies (both give identical results;
 * used to check one against the other). */
#define PLQ_FLAG_GENERIC_PASS 8
/* Keep a q = 2 keyed site chain on its byte passes (the fused sweep or the
 * four-sites-at-a-time body) where the bit-packed passes apply (identical
 * results; used to test the byte paths). */
#define PLQ_FLAG_NO_PACKED 16
/* Bit-packed chains only: hash both keyed rounds in every pass instead of
 * reading each site's sweep-independent first round from the array filled at
 * creation (identical results; used to test the hashing passes, which also
 * serve lattices of 2^31 sites and more and chains whose array found no room). */
#define PLQ_FLAG_NO_FIRST_HASH 32

typedef struct plq_ctx plq_ctx;
typedef struct plq_chain plq_chain;

/* Everything a chain needs; the union of the per-model `gpu_chain` argument
 * lists (src/models/ising/gpu.rs:57-68, potts/gpu.rs:93-103,
 * gauge/gpu.rs:54-64) and GpuClusterChain::new (src/gpu_cluster.rs:209-221). */
typedef struct plq_chain_desc {
    int32_t model;              /* enum plq_model */
    int32_t q;                  /* states per variable: 2 for Ising and gauge */
    int32_t d;                  /* lattice dimension, 1..PLQ_MAX_D */
    int32_t updater;            /* enum plq_updater */
    int64_t shape[PLQ_MAX_D];   /* extents, direction 0 fastest (lattice.rs:73-99) */
    int32_t extent;             /* enum plq_extent (PLQ_CLUSTER only) */
    int32_t relabel;            /* enum plq_relabel (PLQ_CLUSTER only) */
    int32_t rng;                /* enum plq_rng */
    int32_t flags;              /* PLQ_FLAG_* bits, normally 0 */
    double beta;
    double j;                   /* coupling J */
    double h;                   /* Ising field h */
    double offsets[PLQ_MAX_Q];  /* Potts per-label offsets h[a] */
    uint64_t seed;              /* keyed: folded as in device.rs:761-763; stream: seed_from_u64 */
    uint64_t stream_offset;     /* stream: next_u64 draws already consumed (e.g. the hot start) */
    int64_t sweeps_between;     /* sweeps per `next` (device.rs:590-701) */
    int64_t batch;              /* samples per device round-trip (GPU_BATCH, device.rs:501) */
    uint64_t sweep_offset;      /* sweeps already run: the keyed stream's sweep counter (the RNG key
                                   `sweeps_done`, device.rs:216-217) starts here, so a keyed chain
                                   re-created from a read-back configuration with sweep_offset = its
                                   sweeps so far continues bit-identically; counted in
                                   plq_chain_sweeps_done on both streams.  Normally 0. */
} plq_chain_desc;

/* ------------------------------------------------------- library */
const char *plq_version(void);
const char *plq_strerror(int code);
/* Message of the last failure on this thread (empty string if none). */
const char *plq_last_error(void);
int plq_device_count(int *count);

/* Gpu::new (src/device.rs:42-78): PLQ_ENODEV when no device is present. */
int plq_ctx_create(int device_ordinal, plq_ctx **out);
/* Chains, ensembles and servers copy the context's record when they are
   created, so a context may be destroyed before them (a garbage collector may
   finalize a Gpu before the chains made from it). */
void plq_ctx_destroy(plq_ctx *ctx);

/* ------------------------------------------------ host-side helpers */
/* Contract checks of GpuChain::build (device.rs:609-646), assert_even_extents
 * (device.rs:714-719), GpuClusterChain::new (gpu_cluster.rs:209-300) and
 * ClusterUpdate::new (updater.rs:447-483); no device needed. */
int plq_chain_validate(const plq_chain_desc *desc);
/* ClusterUpdate::bond_probability (updater.rs:499-501) for the model's gap. */
double plq_bond_probability(int32_t model, double j, double beta);
/* fold_seed (device.rs:761-763). */
uint32_t plq_fold_seed(uint64_t seed);
/* RandRng::seed_from_u64(seed) then Configuration::hot (configuration.rs:82-87):
 * n_vars draws of next_below(q).  *draws_out = next_u64 calls consumed, i.e.
 * the stream offset at which a chain continuing that rng starts. */
int plq_hot_start(uint64_t seed, int32_t q, int64_t n_vars, uint8_t *out, uint64_t *draws_out);

/* ------------------------------------------------------------ chains */
/* GpuChain::build (device.rs:609-681) / GpuClusterChain::new
 * (gpu_cluster.rs:209-300): uploads `start` (n_vars bytes, one state index
 * per variable in the reference's linear order; links are site*d+dir). */
int plq_chain_create(plq_ctx *ctx, const plq_chain_desc *desc, const uint8_t *start,
                     plq_chain **out);
/* GpuChain::advance (device.rs:387-399) / GpuClusterChain::advance
 * (gpu_cluster.rs:477-481): enqueue sweeps, return without waiting. */
int plq_chain_advance(plq_chain *chain, uint64_t sweeps);
/* Iterator::next (device.rs:692-700, gpu_cluster.rs:627-637): run
 * sweeps_between sweeps, then copy the configuration (n_vars bytes, may be
 * NULL) and its integer primaries (may be NULL; see plq_chain_primaries). */
int plq_chain_next(plq_chain *chain, uint8_t *out_states, int64_t *out_primaries);
/* run_batch (device.rs:435-484): `count` samples, one device round-trip. */
int plq_chain_next_batch(plq_chain *chain, int64_t count, uint8_t *out_states,
                         int64_t *out_primaries);
/* Copy the current configuration without sweeping. */
int plq_chain_read(plq_chain *chain, uint8_t *out_states);
/* Exact integer primaries of the current configuration, summed in int64 on
 * the device: Ising {bond_sum, spin_sum} (ising/mod.rs:67-117); Potts
 * {agree, count[0..q)} (potts/mod.rs:125-271); gauge {plaquette_sum}
 * (gauge/mod.rs:99-124).  Returns the count written via *n_out (may be NULL). */
int plq_chain_primaries(plq_chain *chain, int64_t *out, int32_t *n_out);
/* Ising / Potts chains: axis_pair_sums (src/models/mod.rs:44-61) of the current
 * configuration -- for each axis mu (row by row) and displacement r = 0..L_mu/2,
 * the sum over sites of s_i * s_{i+r mu} (Ising, ising/mod.rs:84-95) or of
 * [s_i == s_{i+r mu}] (Potts, potts/mod.rs:218-234).  `capacity` entries of
 * `out` must hold sum over mu of (L_mu/2 + 1); the correlators divide by N. */
int plq_chain_axis_pair_sums(plq_chain *chain, int64_t *out, int64_t capacity);
/* Gauge chains: Z2Gauge::polyakov_loop (gauge/mod.rs:179-212) of the current
 * configuration along `dir` as *sum (of the +1/-1 line products) / *lines. */
int plq_chain_polyakov(plq_chain *chain, int32_t dir, int64_t *sum, int64_t *lines);
/* Gauge chains: Z2Gauge::wilson_rectangles (gauge/mod.rs:226-274) of the
 * current configuration as totals[r * (m + 1) + t] / *placements for r, t in
 * 0..m, m = min(max_side, shortest extent / 2) returned via *m_out (row and
 * column 0 hold *placements: the 1.0 anchor).  m above 32 is refused
 * (PLQ_EUNSUPPORTED); `capacity` entries of totals must hold (m + 1)^2. */
int plq_chain_wilson(plq_chain *chain, int32_t max_side, int64_t *totals, int64_t capacity, int64_t *placements,
                     int32_t *m_out);
int plq_chain_sync(plq_chain *chain);
/* Device status word: PLQ_OK, or PLQ_ECAP / PLQ_EDEVICE after a fault. */
int plq_chain_status(plq_chain *chain);
/* Sweeps run so far, sweep_offset included (the keyed stream's next sweep key). */
uint64_t plq_chain_sweeps_done(plq_chain *chain);
/* Stream mode: next_u64 draws consumed so far (stream_offset included). */
int plq_chain_stream_position(plq_chain *chain, uint64_t *out);
int64_t plq_chain_n_vars(plq_chain *chain);
/* The chain's cudaStream_t, for callers that time or order work around it. */
void *plq_chain_cuda_stream(plq_chain *chain);
/* Cluster chains (Swendsen-Wang extent): the canonical label of every site in
 * the most recent decomposition -- the minimum site index of its cluster, the
 * fixed point of cluster_prelude.wgsl:113-147; ranked in site order it is
 * site_clusters' compaction (cluster.rs:199-226).  n_sites int32 values. */
int plq_chain_cluster_labels(plq_chain *chain, int32_t *out);
/* Cluster sizes of the most recent decomposition as a histogram: bin k counts
 * clusters with 2^k <= size < 2^(k+1) (the last bin takes the rest).  Wolff
 * chains: the cluster of the most recent update. */
int plq_chain_cluster_histogram(plq_chain *chain, int64_t *hist, int32_t nbins);
/* Which device path the chain's sweeps take: "fused3d" (both colours in one
 * pass), "pass" (one launch per colour), "lookback" (stream Metropolis with
 * the device-wide scan), "cluster". */
const char *plq_chain_path(plq_chain *chain);
/* Kernels this chain has launched so far. */
uint64_t plq_chain_launches(plq_chain *chain);
void plq_chain_destroy(plq_chain *chain);

/* -------------------------------------------------------- ensembles */
/* No counterpart in the reference (which runs one chain per GpuChain): many
 * chains -- any mix of models, dimensions <= 4, uneven shapes, betas and
 * seeds, local updaters on the keyed stream or heat bath on the PCG stream --
 * advanced together.  Member m evolves exactly as plq_chain_create(desc[m],
 * starts[m]) would; starts may be NULL (all members cold) or hold NULLs.
 * Members share one sweep counter, so their sweep_offset must be equal. */
typedef struct plq_ensemble plq_ensemble;
int plq_ensemble_create(plq_ctx *ctx, int32_t n, const plq_chain_desc *members, const uint8_t *const *starts,
                        plq_ensemble **out);
/* Parallel tempering over k members of identical model, shape and updater
 * (no field, no offsets): slot i runs at betas[i] (member member_ids[i]
 * starts there); every `every` sweeps adjacent slots attempt swaps (even
 * pairs, then odd pairs) with min(1, exp((b_i - b_i+1)(E_i - E_i+1))). */
int plq_ensemble_add_ladder(plq_ensemble *e, int32_t k, const int32_t *member_ids, const double *betas,
                            int32_t every, uint64_t seed);
/* Member m runs at `beta` from its next sweep (its decision tables rebuilt in
 * place); refused for members of a ladder, whose betas the ladder moves.
 * Used where tempering spans ranks: every rank decides the swaps with
 * plq_tempering_swap_phase and sets the betas of the members it holds. */
int plq_ensemble_set_beta(plq_ensemble *e, int32_t member, double beta);
/* The ladder's swap rule on the host, identical bit for bit to the device's
 * (one header defines both): one phase of attempt `attempt` over k_slots
 * slots -- pairs (k, k+1) from k = attempt & 1 in steps of 2 -- given every
 * member's energy integer (bond, agreement or plaquette sum) and coupling;
 * accepted pairs exchange their betas in beta_of_member and their members in
 * member_of_slot.  `ladder_seed` is folded as plq_ensemble_add_ladder folds
 * it.  *accepted_out (may be NULL) = the swaps taken. */
int plq_tempering_swap_phase(int32_t k_slots, int32_t *member_of_slot, double *beta_of_member,
                             const int64_t *energy, const double *j_of_member, uint64_t ladder_seed,
                             uint64_t attempt, int32_t *accepted_out);
/* `sweeps` sweeps of every member (and the swaps they reach) in one
 * persistent cooperative launch, captured once into a CUDA graph and replayed. */
int plq_ensemble_advance(plq_ensemble *e, uint64_t sweeps);
/* The same sweeps with one launch per member per colour pass (the
 * per-lattice baseline); identical results. */
int plq_ensemble_advance_unbatched(plq_ensemble *e, uint64_t sweeps);
/* Launch shape of the persistent kernel: ranks per thread of the generic
 * pass body (2, 4, 8) and CTAs per SM. */
int plq_ensemble_set_config(plq_ensemble *e, int32_t ranks_per_thread, int32_t ctas_per_sm);
/* The autotuner (the reference has one fixed shape, a workgroup of 64,
 * src/device.rs:96-106).  On a snapshot of the ensemble (restored
 * afterwards): (1) for every member shape -- (model, q, d, extents,
 * updater, stream) -- the members of that shape alone at 1, 2, 4 and 8
 * four-site words per thread, the fastest kept for them and recorded in a
 * process-wide table that later ensembles and served jobs of that shape
 * use; (2) the whole ensemble over the generic body's ranks per thread and
 * CTAs per SM.  Returns the launch shape chosen in (2) and its time per
 * sweep. */
int plq_ensemble_tune(plq_ensemble *e, int32_t trial_sweeps, int32_t *ranks_out, int32_t *ctas_out,
                      double *ms_per_sweep_out);
/* Member m's work-item shape: four-site words per thread (0: the generic body). */
int plq_ensemble_member_config(plq_ensemble *e, int32_t member, int32_t *words_per_thread);
/* The process-wide tuning table, one entry per member shape tuned so far;
 * *n_out = the number of entries (at most `capacity` are written). */
typedef struct plq_tune_entry {
    int32_t model, q, d, updater, rng;
    int32_t words_per_thread;   /* the fastest measured */
    int64_t shape[4];
    int32_t members;            /* members of this shape in the tuned ensemble */
    int32_t pad;
    double ms_per_sweep;        /* those members alone, at that shape */
} plq_tune_entry;
int plq_tune_entries(plq_tune_entry *out, int32_t capacity, int32_t *n_out);
int plq_ensemble_sync(plq_ensemble *e);
int plq_ensemble_read(plq_ensemble *e, int32_t member, uint8_t *out_states);
int plq_ensemble_primaries(plq_ensemble *e, int32_t member, int64_t *out, int32_t *n_out);
/* Every member's primaries at once (one replayed launch sequence and one
 * copy): member m's int64 primaries, as plq_chain_primaries, at
 * out[m * stride ...]; counts[m] (may be NULL) receives how many. */
int plq_ensemble_primaries_all(plq_ensemble *e, int64_t *out, int32_t stride, int32_t *counts);
/* Current beta of every member (parallel tempering moves them). */
int plq_ensemble_betas(plq_ensemble *e, double *beta_of_member);
int64_t plq_ensemble_n_vars(plq_ensemble *e);
void *plq_ensemble_cuda_stream(plq_ensemble *e);
uint64_t plq_ensemble_launches(plq_ensemble *e);
void plq_ensemble_destroy(plq_ensemble *e);

/* ---------------------------------------------------------- serving */
/* No counterpart in the reference.  A request loop for simulation jobs
 * (model, shape, beta, sweeps, ...): a worker thread admits queued jobs
 * first-fit while their device footprint fits `budget_bytes` (0 = 80 % of
 * free device memory) and fewer than `max_slots` run; keeps each job's state
 * resident on the device; and batches every running job into one persistent
 * launch per tick (about `tick_ms` of work), so jobs that arrive while others
 * run join at the next tick and share its launches.  A job's result is the
 * same alone or in any mix (its keyed sweep counter and stream position are
 * its own).  Jobs: local updaters, d <= 4, keyed or heat bath on the PCG stream. */
typedef struct plq_server plq_server;
enum plq_job_state { PLQ_JOB_QUEUED = 0, PLQ_JOB_ACTIVE = 1, PLQ_JOB_DONE = 2, PLQ_JOB_FAILED = 3,
                     PLQ_JOB_CANCELLED = 4 };
int plq_server_create(plq_ctx *ctx, uint64_t budget_bytes, int32_t max_slots, double tick_ms, plq_server **out);
/* Queue a job of `sweeps` sweeps from `start` (NULL = cold); returns at once.
 * PLQ_ENOMEM if it could never fit the budget. */
int plq_server_submit(plq_server *s, const plq_chain_desc *desc, const uint8_t *start, uint64_t sweeps,
                      int32_t want_states, int64_t *job_id);
/* Wait until the job left the queue and the device (timeout_s < 0: forever). */
int plq_server_wait(plq_server *s, int64_t job_id, double timeout_s, int32_t *state_out);
int plq_server_cancel(plq_server *s, int64_t job_id);
/* Final configuration (if submitted with want_states), int64 primaries as
 * plq_chain_primaries, timing {queue ms, latency ms} (each may be NULL). */
int plq_server_result(plq_server *s, int64_t job_id, uint8_t *out_states, int64_t *out_primaries,
                      double *timing_out);
int plq_server_release(plq_server *s, int64_t job_id);
/* {completed, p50 ms, p99 ms, site updates/ns while busy, ticks, queued,
 * running, device bytes in use}; returns a device error if one occurred. */
int plq_server_stats(plq_server *s, double *out8);
void plq_server_destroy(plq_server *s);

/* ------------------------------------------- allocation-free sweep */
/* No counterpart in the reference.  For callers that cannot call cudaMalloc
 * (a host that owns the device memory and lends this library one buffer, or
 * a loop that must not risk cudaMalloc's implicit synchronisation): `sweeps`
 * checkerboard Metropolis sweeps of an Ising lattice on the PCG stream, in
 * place on `spins` -- device memory the caller owns, n_sites bytes in the
 * reference's site order -- with exactly the results of a PLQ_ISING /
 * PLQ_METROPOLIS / PLQ_RNG_STREAM chain.  Allocates no device memory: its
 * scratch is a fixed 384 KiB array that every GPU loading the library holds
 * until exit, which limits the lattice to PLQ_NOALLOC_MAX_SITES sites (larger
 * lattices are refused with PLQ_EINVAL).  All calls share that array, so calls
 * that overlap on the GPU race and must not be issued.  The first call on a
 * device looks up the array's device address.  Runs on `cuda_stream` (NULL =
 * the default stream) and returns after it drained; *stream_position_out (may
 * be NULL) receives stream_offset plus the draws consumed.  The array keeps
 * the jump table of the last seed and the decision table of the last
 * couplings used on that device: a call with another seed or other couplings
 * copies those tables (about 64 KiB) from pageable host memory, which waits
 * for the work already queued on `cuda_stream`; a repeated call with the same
 * seed and couplings copies nothing. */
#define PLQ_NOALLOC_MAX_SITES 134217728
int plq_ising_metropolis_noalloc(uint8_t *spins, int32_t d, const int64_t *shape, double j, double h,
                                 double beta, uint64_t seed, uint64_t stream_offset, uint64_t sweeps,
                                 void *cuda_stream, uint64_t *stream_position_out);

/* ----------------------------------------------------------- slabs */
/* No counterpart in the reference (one chain per adapter, src/device.rs:31-78).
 * One lattice split across devices along its last axis: a slab holds planes
 * [z0, z0 + nz) of the site lattice `desc` describes (Ising or Potts, d = 2 or
 * 3, keyed stream, Metropolis or heat bath) plus one halo plane on each side.
 * Before each colour pass the caller fills the halos with the neighbouring
 * slabs' boundary planes (the previous slab's last plane into the low halo,
 * the next slab's first plane into the high one; the ring is periodic); the
 * pass then updates that colour (global parity) on the slab's planes with the
 * whole lattice's draws, so the slabs together equal the single chain.
 * `start` holds the slab's nz planes in the reference's site order.  A slab's
 * handle is not thread-safe; its work runs on a stream of its own. */
typedef struct plq_slab plq_slab;
#define PLQ_SLAB_LOW_HALO 0
#define PLQ_SLAB_FIRST_PLANE 1
#define PLQ_SLAB_LAST_PLANE 2
#define PLQ_SLAB_HIGH_HALO 3
int plq_slab_create(plq_ctx *ctx, const plq_chain_desc *desc, int64_t z0, int64_t nz, const uint8_t *start,
                    plq_slab **out);
/* Device address and size in bytes of one of the four exchange planes. */
int plq_slab_plane(plq_slab *s, int32_t which, void **device_ptr, int64_t *bytes);
/* One colour pass (0 or 1: the parity of the site's coordinate sum) at the
 * slab's sweep index, queued on its stream. */
int plq_slab_pass(plq_slab *s, int32_t colour);
/* The sweep is complete: later passes draw at the next sweep index. */
int plq_slab_end_sweep(plq_slab *s);
/* Waits for the slab's queued work (before its planes are exchanged). */
int plq_slab_sync(plq_slab *s);
/* The slab's nz planes to host memory (blocks). */
int plq_slab_read(plq_slab *s, uint8_t *out);
void plq_slab_destroy(plq_slab *s);

#ifdef __cplusplus
}
#endif
#endif
