// plq_abi.cu -- the C ABI: contexts, chains, validation, pass scheduling.
//
// Host-side counterpart of the reference's DeviceSweeper / GpuChain
// (src/device.rs:198-701) and GpuClusterChain (src/gpu_cluster.rs:144-637):
// the chain owns all device state, one CUDA stream per chain, `advance`
// enqueues sweeps without waiting, `next` hands back an owned copy.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/plaquette.h"
#include "plq_abi_internal.h"
#include "plq_cluster.h"
#include "plq_device.cuh"
#include "plq_fused.h"
#include "plq_local.h"
#include "plq_measure.h"
#include "plq_scan.h"
#include "plq_tables.h"
#include "plq_words.cuh"

using namespace plq;

static thread_local std::string g_last_error;

int plq_fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

static int cuda_fail(cudaError_t e, const char *what) {
    return plq_fail(e == cudaErrorMemoryAllocation ? PLQ_ENOMEM : PLQ_ECUDA,
                    std::string(what) + ": " + cudaGetErrorString(e));
}

#define PLQ_CUDA(call, what)                         \
    do {                                             \
        cudaError_t _e = (call);                     \
        if (_e != cudaSuccess) return cuda_fail(_e, what); \
    } while (0)

extern "C" const char *plq_version(void) { return "plaquette-b200 0.1 (sm_100a)"; }

extern "C" const char *plq_strerror(int code) {
    switch (code) {
        case PLQ_OK: return "ok";
        case PLQ_ENODEV: return "no CUDA device";
        case PLQ_EINVAL: return "invalid argument";
        case PLQ_EUNSUPPORTED: return "unsupported on this device path";
        case PLQ_ECUDA: return "CUDA runtime error";
        case PLQ_ENOMEM: return "out of memory";
        case PLQ_ECAP: return "cluster labeling did not converge within its pass cap";
        case PLQ_EDEVICE: return "a device kernel reported a fault";
        case PLQ_EBUSY: return "no slot or memory free";
        default: return "unknown error";
    }
}

extern "C" const char *plq_last_error(void) { return g_last_error.c_str(); }

extern "C" int plq_device_count(int *count) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) n = 0;
    if (count) *count = n;
    return PLQ_OK;
}

extern "C" int plq_ctx_create(int device_ordinal, plq_ctx **out) {
    if (!out) return plq_fail(PLQ_EINVAL, "out is NULL");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return plq_fail(PLQ_ENODEV, "no CUDA device is available");
    }
    if (device_ordinal < 0 || device_ordinal >= n)
        return plq_fail(PLQ_ENODEV, "device ordinal out of range");
    PLQ_CUDA(cudaSetDevice(device_ordinal), "cudaSetDevice");
    cudaDeviceProp prop;
    PLQ_CUDA(cudaGetDeviceProperties(&prop, device_ordinal), "cudaGetDeviceProperties");
    plq_ctx *c = new plq_ctx();
    c->device = device_ordinal;
    c->sm_count = prop.multiProcessorCount;
    c->mem_total = prop.totalGlobalMem;
    c->cc_major = prop.major;
    *out = c;
    return PLQ_OK;
}

extern "C" void plq_ctx_destroy(plq_ctx *ctx) { delete ctx; }

// ------------------------------------------------------------ helpers
extern "C" uint32_t plq_fold_seed(uint64_t seed) { return (uint32_t)(seed ^ (seed >> 32)); }

static double bond_gap(int32_t model, double j) { return model == PLQ_ISING ? 2.0 * j : j; }

extern "C" double plq_bond_probability(int32_t model, double j, double beta) {
    return 1.0 - std::exp(-beta * bond_gap(model, j));
}

extern "C" int plq_hot_start(uint64_t seed, int32_t q, int64_t n_vars, uint8_t *out,
                             uint64_t *draws_out) {
    if (q < 2 || q > PLQ_MAX_Q || n_vars < 0 || (!out && n_vars > 0))
        return plq_fail(PLQ_EINVAL, "plq_hot_start: bad arguments");
    HostPcg r = host_pcg_from_seed(seed);
    for (int64_t i = 0; i < n_vars; ++i) out[i] = (uint8_t)r.next_below((uint64_t)q);
    if (draws_out) *draws_out = r.draws;
    return PLQ_OK;
}

std::string shape_string(const plq_chain_desc *d) {
    std::string s = "[";
    for (int i = 0; i < d->d; ++i) {
        if (i) s += ", ";
        s += std::to_string(d->shape[i]);
    }
    return s + "]";
}

static std::string fmt_gap(double g) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%g", g);
    return buf;
}

extern "C" int plq_chain_validate(const plq_chain_desc *d) {
    if (!d) return plq_fail(PLQ_EINVAL, "desc is NULL");
    if (d->model < PLQ_ISING || d->model > PLQ_GAUGE) return plq_fail(PLQ_EINVAL, "unknown model");
    if (d->d < 1 || d->d > PLQ_MAX_D)
        return plq_fail(PLQ_EINVAL, "lattice dimension must be in 1..=" + std::to_string(PLQ_MAX_D));
    if (d->model == PLQ_GAUGE && d->d < 2)
        return plq_fail(PLQ_EINVAL,
                        "the Z2 gauge action scores plaquettes, which need at least two dimensions");
    if (d->model == PLQ_POTTS && d->q < 2)
        return plq_fail(PLQ_EINVAL,
                        "the Potts action scores agreement between labels, which needs at least two states");
    if (d->model != PLQ_POTTS && d->q != 2)
        return plq_fail(PLQ_EINVAL, "Ising spins and gauge links have q = 2");
    if (d->q > PLQ_MAX_Q) return plq_fail(PLQ_EINVAL, "q above the supported maximum");
    int64_t n = 1;
    for (int i = 0; i < d->d; ++i) {
        if (d->shape[i] <= 0) return plq_fail(PLQ_EINVAL, "every extent must be positive");
        if (n > (int64_t(1) << 31) / d->shape[i])
            return plq_fail(PLQ_EINVAL, "shape" + shape_string(d) + " names more variables than this device path indexes (2^31)");
        n *= d->shape[i];
    }
    int64_t n_vars = d->model == PLQ_GAUGE ? n * d->d : n;
    if (n_vars > (int64_t(1) << 31))
        return plq_fail(PLQ_EINVAL, "too many variables for this device path (2^31)");
    if (d->batch <= 0) return plq_fail(PLQ_EINVAL, "batch size must be positive");
    if (d->sweeps_between < 0) return plq_fail(PLQ_EINVAL, "sweeps_between must be non-negative");
    if (d->rng != PLQ_RNG_STREAM && d->rng != PLQ_RNG_KEYED) return plq_fail(PLQ_EINVAL, "unknown rng mode");
    if (d->updater == PLQ_METROPOLIS || d->updater == PLQ_HEATBATH) {
        for (int i = 0; i < d->d; ++i)
            if (d->shape[i] % 2 != 0)
                return plq_fail(PLQ_EINVAL, std::string("the parallel ") +
                                                (d->model == PLQ_GAUGE ? "link" : "site") +
                                                " checkerboard needs even lattice extents, got " +
                                                shape_string(d));
        return PLQ_OK;
    }
    if (d->updater == PLQ_CLUSTER) {
        if (d->model == PLQ_GAUGE)
            return plq_fail(PLQ_EINVAL,
                            "the cluster update bonds nearest-neighbor sites, so the start must be a site field");
        bool invariant = d->model == PLQ_ISING ? d->h == 0.0 : true;
        if (d->model == PLQ_POTTS)
            for (int a = 0; a < d->q; ++a)
                if (d->offsets[a] != 0.0) invariant = false;
        if (!invariant)
            return plq_fail(PLQ_EINVAL,
                            "the cluster move relabels a whole cluster at once, which is only weight-preserving "
                            "when the energy is invariant under relabeling; this model has a per-label offset "
                            "or an external field set");
        if (d->extent != PLQ_EXTENT_ALL && d->extent != PLQ_EXTENT_SEEDED)
            return plq_fail(PLQ_EINVAL, "unknown extent");
        if (d->relabel != PLQ_RELABEL_REDRAW && d->relabel != PLQ_RELABEL_FORCED)
            return plq_fail(PLQ_EINVAL, "unknown relabel rule");
        if (d->q == 2 && d->extent == PLQ_EXTENT_ALL && d->relabel == PLQ_RELABEL_FORCED)
            return plq_fail(PLQ_EINVAL,
                            "at Q = 2 a forced change of every cluster is the deterministic global flip on any "
                            "uniform configuration, so the chain falls into a two-cycle and stops being ergodic; "
                            "use Relabel::Redraw for the all-clusters extent, or the seeded extent for a forced change");
        double gap = bond_gap(d->model, d->j);
        if (!std::isfinite(gap) || gap < 0.0)
            return plq_fail(PLQ_EINVAL,
                            "the bond probability 1 - exp(-beta * gap) needs a finite, non-negative gap, got " +
                                fmt_gap(gap) +
                                "; an antiferromagnetic coupling is frustrated rather than merely inverted and "
                                "needs a different construction");
        return cluster_validate(d);
    }
    return plq_fail(PLQ_EINVAL, "unknown updater");
}

// ------------------------------------------------------------ chains
static ModelParams model_params(const plq_chain_desc *d) {
    ModelParams p;
    std::memset(&p, 0, sizeof p);
    p.model = d->model;
    p.q = d->model == PLQ_POTTS ? d->q : 2;
    p.d = d->d;
    p.beta = d->beta;
    p.j = d->j;
    p.h = d->h;
    for (int a = 0; a < PLQ_MAX_Q; ++a) p.offsets[a] = d->offsets[a];
    return p;
}

template <class T>
static int upload(std::vector<T> &host, T **dev, cudaStream_t s) {
    if (host.empty()) return PLQ_OK;
    PLQ_CUDA(cudaMalloc((void **)dev, host.size() * sizeof(T)), "cudaMalloc(table)");
    PLQ_CUDA(cudaMemcpyAsync(*dev, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice, s),
             "cudaMemcpyAsync(table)");
    return PLQ_OK;
}

static u128 to_u128(uint64_t lo, uint64_t hi) {
    u128 r;
    r.lo = lo;
    r.hi = hi;
    return r;
}

void chain_free(plq_chain *c) {
    if (!c) return;
    if (c->ctx) plq_enter_device(c->ctx->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->obs_stream) cudaStreamSynchronize(c->obs_stream);
    cluster_free(c);
    void *ptrs[] = {c->d_state, c->d_state_alt, c->d_io, c->d_hb53, c->d_hb24, c->d_metro53, c->d_metro24,
                    c->d_jump, c->d_ctrl, c->d_desc, c->d_obs, c->d_snap, c->d_snap_obs, c->d_loop_bits,
                    c->d_meas, c->d_pairs, c->d_hb53_fused, c->d_packed, c->d_first_hash};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (c->h_pinned) cudaFreeHost(c->h_pinned);
    if (c->obs_stream) cudaStreamDestroy(c->obs_stream);
    if (c->swept) cudaEventDestroy(c->swept);
    for (cudaEvent_t ev : c->measured)
        if (ev) cudaEventDestroy(ev);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

// Index of the first byte >= q (q <= 64) in a[0, n), or -1.  Sixty-four bytes per
// step: a byte b is flagged when b >= 128 or b + (128 - q) reaches 128; a carry
// out of a byte happens only when that byte is flagged already, so a clean
// block is clean byte for byte.  The flagged block is then scanned bytewise.
static int64_t first_state_at_least_serial(const uint8_t *a, int64_t n, int q) {
    const uint64_t H = 0x8080808080808080ull, add = 0x0101010101010101ull * (uint64_t)(128 - q);
    int64_t i = 0;
    for (; i + 64 <= n; i += 64) {
        uint64_t bad = 0;
        for (int k = 0; k < 8; ++k) {
            uint64_t w;
            std::memcpy(&w, a + i + 8 * k, 8);
            bad |= (w | (w + add)) & H;
        }
        if (bad) break;
    }
    for (; i < n; ++i)
        if (a[i] >= q) return i;
    return -1;
}

// The start checks run on several host threads: the scan is memory-bound at a few GB/s per
// thread, and a 512^3 start (134 MB) or a whole ensemble's starts (tens of MB) would otherwise
// take several milliseconds of creation.  Work is dealt out in increasing order and a thread
// stops taking pieces past the earliest failure found, so the result is the serial scan's.
static int scan_threads(int64_t pieces) {
    const unsigned hw = std::thread::hardware_concurrency();
    return (int)std::min<int64_t>(pieces, std::min(16u, hw ? hw : 1u));
}

template <class F>
static int64_t first_failing(int64_t pieces, F scan_piece) {
    const int T = scan_threads(pieces);
    if (T <= 1) {
        for (int64_t p = 0; p < pieces; ++p)
            if (scan_piece(p)) return p;
        return -1;
    }
    std::atomic<int64_t> next{0}, first_bad{pieces};
    auto work = [&]() {
        for (;;) {
            const int64_t p = next.fetch_add(1);
            if (p >= first_bad.load()) return;
            if (scan_piece(p)) {
                int64_t cur = first_bad.load();
                while (p < cur && !first_bad.compare_exchange_weak(cur, p)) {
                }
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < T; ++t) pool.emplace_back(work);
    work();
    for (std::thread &t : pool) t.join();
    const int64_t b = first_bad.load();
    return b < pieces ? b : -1;
}

int64_t first_state_at_least(const uint8_t *a, int64_t n, int q) {
    constexpr int64_t kPiece = int64_t(1) << 22;  // 4 MiB
    const int64_t pieces = (n + kPiece - 1) / kPiece;
    if (pieces <= 2) return first_state_at_least_serial(a, n, q);
    const int64_t p = first_failing(pieces, [&](int64_t k) {
        return first_state_at_least_serial(a + k * kPiece, std::min(kPiece, n - k * kPiece), q) >= 0;
    });
    if (p < 0) return -1;
    return p * kPiece + first_state_at_least_serial(a + p * kPiece, std::min(kPiece, n - p * kPiece), q);
}

int32_t first_bad_start(int32_t n, const uint8_t *const *starts, const int64_t *n_vars, const int *q) {
    const int64_t m = first_failing(n, [&](int64_t k) {
        return starts[k] && first_state_at_least_serial(starts[k], n_vars[k], q[k]) >= 0;
    });
    return (int32_t)m;
}

extern "C" int plq_chain_create(plq_ctx *ctx, const plq_chain_desc *desc, const uint8_t *start,
                                plq_chain **out) {
    if (!ctx || !desc || !out) return plq_fail(PLQ_EINVAL, "NULL argument");
    *out = nullptr;
    int rc = plq_chain_validate(desc);
    if (rc != PLQ_OK) return rc;
    {
        // State::new (src/state.rs) refuses an index >= Q; the kernels index
        // their tables by state, so a bad start is refused here.
        int q = desc->model == PLQ_POTTS ? desc->q : 2;
        int64_t n = 1;
        for (int i = 0; i < desc->d; ++i) n *= desc->shape[i];
        int64_t n_vars = desc->model == PLQ_GAUGE ? n * desc->d : n;
        if (start) {
            const int64_t i = first_state_at_least(start, n_vars, q);
            if (i >= 0)
                return plq_fail(PLQ_EINVAL, "start variable " + std::to_string(i) + " holds state " +
                                                std::to_string(start[i]) + ", not below q = " + std::to_string(q));
        }
    }
    PLQ_CUDA(plq_enter_device(ctx->device), "cudaSetDevice");

    plq_chain *c = new plq_chain();
    c->ctx_copy = *ctx;
    c->ctx = &c->ctx_copy;
    c->desc = *desc;
    c->sweeps_done = desc->sweep_offset;  // the keyed stream's sweep key resumes here
    c->q = desc->model == PLQ_POTTS ? desc->q : 2;
    c->d = desc->d;
    c->link = desc->model == PLQ_GAUGE;
    c->cluster = desc->updater == PLQ_CLUSTER;
    c->g.d = desc->d;
    int64_t n = 1;
    for (int i = 0; i < kMaxD; ++i) {
        c->g.L[i] = i < desc->d ? (int32_t)desc->shape[i] : 1;
        c->g.stride[i] = n;
        if (i < desc->d) n *= desc->shape[i];
    }
    c->g.n_sites = n;
    geom_init(c->g, desc->d, desc->shape);
    c->n_sites = n;
    c->n_vars = c->link ? n * desc->d : n;
    c->seed32 = plq_fold_seed(desc->seed);

    auto fail = [&](int code) {
        chain_free(c);
        return code;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaStreamCreate"));
    e = cudaMalloc((void **)&c->d_state, (size_t)c->n_vars);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMalloc(state)"));
    e = cudaMalloc((void **)&c->d_ctrl, sizeof(Control));
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMalloc(control)"));
    cudaMemsetAsync(c->d_ctrl, 0, sizeof(Control), c->stream);
    e = cudaMalloc((void **)&c->d_obs, sizeof(long long) * (PLQ_MAX_Q + 2));
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMalloc(observables)"));

    // start configuration
    if (start) {
        if (c->link) {
            e = cudaMalloc((void **)&c->d_io, (size_t)c->n_vars);
            if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMalloc(io)"));
            e = cudaMemcpyAsync(c->d_io, start, (size_t)c->n_vars, cudaMemcpyHostToDevice, c->stream);
            if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMemcpyAsync(start)"));
            e = launch_links_to_planes(c->d_io, c->d_state, n, c->d, c->stream);
            c->launches++;
        } else {
            e = cudaMemcpyAsync(c->d_state, start, (size_t)c->n_vars, cudaMemcpyHostToDevice, c->stream);
        }
        if (e != cudaSuccess) return fail(cuda_fail(e, "upload start"));
    } else {
        cudaMemsetAsync(c->d_state, 0, (size_t)c->n_vars, c->stream);
    }

    // PCG stream: base state such that draw n = xsl_rr(jump(base, n))
    if (desc->rng == PLQ_RNG_STREAM) {
        uint64_t slo, shi, ilo, ihi;
        pcg_seed_from_u64(desc->seed, slo, shi, ilo, ihi);
        std::vector<AffineHost> tab;
        build_jump_table(ilo, ihi, tab);
        c->inc = to_u128(ilo, ihi);
        // host-side jump to stream_offset + 1 steps
        u128 s = to_u128(slo, shi);
        uint64_t steps = desc->stream_offset;
        const Affine *T = reinterpret_cast<const Affine *>(tab.data());
        s = jump(T, s, steps);
        s = pcg_step(s, c->inc);
        c->base = s;
        AffineHost *dj = nullptr;
        int r2 = upload(tab, &dj, c->stream);
        if (r2 != PLQ_OK) return fail(r2);
        c->d_jump = reinterpret_cast<Affine *>(dj);
        c->h_jump = tab;
    }

    if (!c->cluster) {
        ModelParams p = model_params(desc);
        Tables t;
        std::string err;
        if (!build_tables(p, desc->updater, desc->rng, t, err)) return fail(plq_fail(PLQ_EUNSUPPORTED, err));
        int r2 = upload(t.hb53, &c->d_hb53, c->stream);
        if (r2 == PLQ_OK) r2 = upload(t.hb24, &c->d_hb24, c->stream);
        if (r2 == PLQ_OK) r2 = upload(t.metro53, &c->d_metro53, c->stream);
        if (r2 == PLQ_OK) r2 = upload(t.metro24, &c->d_metro24, c->stream);
        if (r2 != PLQ_OK) return fail(r2);
        // packing weights of the site environment key
        int32_t w = 1;
        for (int s = 0; s < 64; ++s) c->pw[s] = 0;
        for (int s = 1; s < c->q; ++s) {
            c->pw[s] = w;
            w *= 2 * desc->d + 1;
        }
        c->lookback = desc->rng == PLQ_RNG_STREAM && desc->updater == PLQ_METROPOLIS;
        c->words = !c->lookback && !(desc->flags & PLQ_FLAG_GENERIC_PASS) &&
                   words_eligible(desc->model, c->q, c->d, c->g.L, desc->updater, desc->rng);
        // the fused two-colour sweep where a variable's draw is a closed form
        size_t table_bytes = desc->updater == PLQ_HEATBATH
                                 ? (desc->rng == PLQ_RNG_STREAM ? t.hb53.size() * 8 : t.hb24.size() * 4)
                                 : t.metro24.size() * 4;
        // The fused stream heat bath compares the full 64-bit XSL-RR output with cut points
        // shifted left by 11 (k >= c  <=>  out >= c * 2^11 for c < 2^53), which needs every
        // cut below 2^53; a "never" cut of 2^53 (a probability that rounds to 1) sends the
        // chain to the per-colour passes instead.
        bool shifted_ok = true;
        std::vector<uint64_t> hb53_shifted;
        if (desc->rng == PLQ_RNG_STREAM && desc->updater == PLQ_HEATBATH) {
            hb53_shifted.reserve(t.hb53.size());
            for (uint64_t cut : t.hb53) {
                if (cut >= (uint64_t(1) << 53)) shifted_ok = false;
                hb53_shifted.push_back(cut << 11);
            }
        }
        if (!(desc->flags & (PLQ_FLAG_NO_FUSED | PLQ_FLAG_GENERIC_PASS | PLQ_FLAG_NO_PACKED)) && !c->link &&
            packed_chain_eligible(desc->model, c->q, c->d, c->g.L, desc->updater, desc->rng)) {
            c->packed = true;
            e = cudaMalloc((void **)&c->d_packed, (size_t)(c->n_sites / 64) * sizeof(uint64_t));
            if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMalloc(packed state)"));
            // every site's sweep-independent first keyed round lowbias32_head(seed ^ site) (4 B/site):
            // the passes hash only the sweep's round.  Optional: without it (2^31 sites and more, or
            // the array would take over a quarter of the free memory, or its allocation fails) the
            // passes hash both rounds, with identical results.
            size_t free_b = 0, total_b = 0;
            const size_t hb_bytes = first_hash_bytes(c->n_sites / 64);
            if (c->n_sites < (int64_t(1) << 31) && !(desc->flags & PLQ_FLAG_NO_FIRST_HASH) &&
                cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && hb_bytes <= free_b / 4) {
                if (cudaMalloc(&c->d_first_hash, hb_bytes) == cudaSuccess) {
                    e = launch_first_hash(c->d_first_hash, c->n_sites / 64, c->g.L[0], c->g.L[1], c->d, c->seed32,
                                          c->ctx->sm_count, c->stream);
                    if (e != cudaSuccess) return fail(cuda_fail(e, "first-hash launch"));
                    c->launches++;
                } else {
                    c->d_first_hash = nullptr;
                    (void)cudaGetLastError();  // the failed allocation's error; the chain hashes in its passes
                }
            }
        }
        if (!c->packed && !(desc->flags & PLQ_FLAG_NO_FUSED) &&
            fused3d_eligible(desc->model, c->q, c->d, c->g.L, desc->updater, desc->rng) &&
            table_bytes <= (size_t)fused3d_table_limit_bytes() && shifted_ok) {
            c->fused = true;
            if (!hb53_shifted.empty()) {
                int r3 = upload(hb53_shifted, &c->d_hb53_fused, c->stream);
                if (r3 != PLQ_OK) return fail(r3);
            }
            c->fused_tz = fused3d_default_tz(c->g.L[2]);
            e = cudaMalloc((void **)&c->d_state_alt, (size_t)c->n_vars);
            if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMalloc(state_alt)"));
            for (int k = 0; k < 2; ++k) {
                c->fused_map_buf[k] = k ? c->d_state_alt : c->d_state;
                e = fused3d_make_maps(c->fused_map_buf[k], c->g.L[0], c->g.L[1], c->g.L[2], &c->fused_maps[k]);
                if (e != cudaSuccess) return fail(cuda_fail(e, "tensor map of the state buffer"));
            }
            e = cudaStreamCreateWithFlags(&c->obs_stream, cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->swept, cudaEventDisableTiming);
            for (int k = 0; k < 2 && e == cudaSuccess; ++k)
                e = cudaEventCreateWithFlags(&c->measured[k], cudaEventDisableTiming);
            if (e != cudaSuccess) return fail(cuda_fail(e, "measurement stream"));
        }
        if (c->lookback) {
            c->n_chunks = local_chunks(n);
            // descriptors for the larger chunk count of the two look-back pass kernels
            const int64_t n_desc = std::max<int64_t>(c->n_chunks, scan_chunks(n));
            e = cudaMalloc((void **)&c->d_desc, sizeof(unsigned long long) * (size_t)n_desc);
            if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMalloc(lookback)"));
            cudaMemsetAsync(c->d_desc, 0, sizeof(unsigned long long) * (size_t)n_desc, c->stream);
        }
    } else {
        int r2 = cluster_create(c);
        if (r2 != PLQ_OK) return fail(r2);
    }
    e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return fail(cuda_fail(e, "chain setup"));
    *out = c;
    return PLQ_OK;
}

static LocalArgs local_args(plq_chain *c) {
    LocalArgs a;
    std::memset(&a, 0, sizeof a);
    a.state = c->d_state;
    a.g = c->g;
    a.q = c->q;
    a.kernel = c->desc.updater;
    a.model = c->desc.model;
    for (int s = 0; s < 64; ++s) a.pw[s] = c->pw[s];
    a.hb53 = c->d_hb53;
    a.hb24 = c->d_hb24;
    a.metro53 = c->d_metro53;
    a.metro24 = c->d_metro24;
    a.seed32 = c->seed32;
    a.jump = c->d_jump;
    a.base = c->base;
    a.inc = c->inc;
    a.ctrl = c->d_ctrl;
    a.desc = c->d_desc;
    a.n_chunks = c->n_chunks;
    a.words = c->words ? 1 : 0;
    return a;
}

static Affine to_affine(const AffineHost &h) {
    Affine f;
    f.m.lo = h.m_lo;
    f.m.hi = h.m_hi;
    f.p.lo = h.p_lo;
    f.p.hi = h.p_hi;
    return f;
}

// One fused two-colour sweep (out of place; the buffers swap).
static int fused_sweep(plq_chain *c) {
    FusedArgs f;
    std::memset(&f, 0, sizeof f);
    f.src = c->d_state;
    f.dst = c->d_state_alt;
    f.L0 = c->g.L[0];
    f.L1 = c->g.L[1];
    f.L2 = c->g.L[2];
    f.tz = c->fused_tz;
    const bool stream = c->desc.rng == PLQ_RNG_STREAM;
    const bool hb = c->desc.updater == PLQ_HEATBATH;
    if (hb) {
        if (stream) {
            f.table = c->d_hb53_fused;
            f.table_words = (int)(env_key_count(model_params(&c->desc)) * (c->q - 1) * 2);
        } else {
            f.table = c->d_hb24;
            f.table_words = (int)(env_key_count(model_params(&c->desc)) * (c->q - 1));
        }
    } else {
        f.table = c->d_metro24;
        f.table_words = (int)env_key_count(model_params(&c->desc));
    }
    f.seed32 = c->seed32;
    f.sweep32 = (uint32_t)c->sweeps_done;
    if (stream) {
        f.jump = c->d_jump;
        f.base = c->base;
        f.inc = c->inc;
        f.off0 = c->host_pos;
        f.off1 = c->host_pos + (uint64_t)(c->n_sites / 2);
        f.plane = to_affine(affine_steps(c->h_jump, (uint64_t)f.L0 * (uint64_t)f.L1 / 2));
    }
    f.status = &c->d_ctrl->status;
    const int dst_k = f.dst == c->fused_map_buf[0] ? 0 : 1;
    if (c->measuring[dst_k]) {  // a sample of this buffer is still being measured
        PLQ_CUDA(cudaStreamWaitEvent(c->stream, c->measured[dst_k], 0), "wait for measurement");
        c->measuring[dst_k] = false;
    }
    f.stall = (c->desc.flags & PLQ_FLAG_TEST_COPY_STALL) ? 1 : 0;
    f.wait_limit = f.stall ? 1024 : (1 << 21);
    const FusedMaps &maps = c->fused_maps[f.src == c->fused_map_buf[0] ? 0 : 1];
    cudaError_t e = launch_fused3d(f, maps, c->q, stream, hb, c->stream);
    c->launches++;
    if (e != cudaSuccess) return cuda_fail(e, "fused sweep launch");
    std::swap(c->d_state, c->d_state_alt);
    if (stream) c->host_pos += (uint64_t)c->n_vars;
    c->sweeps_done++;
    return PLQ_OK;
}

// `sweeps` sweeps of a packed chain: the bytes packed once, two colour passes
// per sweep on the words (the keyed sweep index as the byte passes use it),
// the words unpacked at the end.
static int packed_sweeps(plq_chain *c, uint64_t sweeps) {
    if (!sweeps) return PLQ_OK;
    const int64_t n_words = c->n_sites / 64;
    const int sm = c->ctx->sm_count;
    PLQ_CUDA(launch_pack64(c->d_state, c->d_packed, n_words, sm, c->stream), "pack launch");
    c->launches++;
    PackedPassArgs a;
    std::memset(&a, 0, sizeof a);
    a.words = c->d_packed;
    a.n_words = n_words;
    a.L0 = c->g.L[0];
    a.L1 = c->g.L[1];
    a.seed32 = c->seed32;
    const bool hb = c->desc.updater == PLQ_HEATBATH;
    a.table = hb ? c->d_hb24 : c->d_metro24;
    a.n_keys = 2 + 4 * c->d;  // keys cur + 2 * count, count <= 2d
    a.first_hash = c->d_first_hash;
    for (uint64_t t = 0; t < sweeps; ++t) {
        a.sweep32 = (uint32_t)c->sweeps_done;
        for (int colour = 0; colour < 2; ++colour) {
            a.colour = colour;
            PLQ_CUDA(launch_packed_pass(a, c->d, hb, sm, c->stream), "packed pass launch");
            c->launches++;
        }
        c->sweeps_done++;
    }
    PLQ_CUDA(launch_unpack64(c->d_packed, c->d_state, n_words, sm, c->stream), "unpack launch");
    c->launches++;
    return PLQ_OK;
}

// One sweep of local passes, in the reference's colour order
// (updater.rs:316-343; device.rs:417-430 for the keyed sweep index).
int local_sweep(plq_chain *c) {
    if (c->fused) return fused_sweep(c);
    if (c->packed) return packed_sweeps(c, 1);
    LocalArgs a = local_args(c);
    a.sweep32 = (uint32_t)c->sweeps_done;
    const int64_t half = c->n_sites / 2;
    const int passes = c->link ? 2 * c->d : 2;
    for (int pass = 0; pass < passes; ++pass) {
        a.dir = c->link ? pass >> 1 : 0;
        a.color = pass & 1;
        if (c->lookback) {
            a.epoch = (uint32_t)(c->lookback_passes + 1);
            a.ticket_base = c->tickets_issued;
            a.pos_in = (int)(c->lookback_passes & 1);
            c->lookback_passes++;
        } else if (c->desc.rng == PLQ_RNG_STREAM) {
            a.pass_offset = c->host_pos + (uint64_t)pass * (uint64_t)half;
        }
        cudaError_t e;
        if (c->lookback && !c->link && c->q == 2 && !(c->desc.flags & PLQ_FLAG_NO_FUSED) &&
            scan_metro_eligible(c->d, c->g.L)) {
            // q = 2 sites in 2D/3D: the vectorised look-back pass (same draws, same result)
            ScanArgs s;
            std::memset(&s, 0, sizeof s);
            s.state = c->d_state;
            s.n_sites = c->n_sites;
            s.L0 = c->g.L[0];
            s.L1 = c->g.L[1];
            s.L2 = c->g.L[2];
            s.dm0 = c->g.dm[0];
            s.dl0 = c->g.dl[0];
            s.dm1 = c->g.dm[1];
            s.dl1 = c->g.dl[1];
            s.color = a.color;
            s.metro53 = c->d_metro53;
            s.table_entries = (int)env_key_count(model_params(&c->desc));
            s.jump = c->d_jump;
            s.base = c->base;
            s.inc = c->inc;
            s.ctrl = c->d_ctrl;
            s.desc = c->d_desc;
            s.n_chunks = scan_chunks(c->n_sites);
            s.epoch = a.epoch;
            s.pos_in = a.pos_in;
            e = launch_scan_metro(s, c->d, c->stream);
        } else if (c->lookback && c->desc.model == PLQ_POTTS && c->q > 2) {
            // the proposal's draw count depends on its own value: a sequential walk
            e = launch_potts_metro_walk(a, c->stream);
        } else {
            e = launch_local_pass(a, c->link, c->lookback, c->stream);
            if (c->lookback) c->tickets_issued += (uint64_t)c->n_chunks;
        }
        c->launches++;
        if (e != cudaSuccess) return cuda_fail(e, "local pass launch");
    }
    if (c->desc.rng == PLQ_RNG_STREAM && !c->lookback) c->host_pos += (uint64_t)c->n_vars;
    c->sweeps_done++;
    return PLQ_OK;
}

static int run_sweeps(plq_chain *c, uint64_t sweeps) {
    if (c->cluster) return sweeps ? cluster_sweep_n(c, sweeps) : PLQ_OK;
    if (c->packed) return packed_sweeps(c, sweeps);
    for (uint64_t t = 0; t < sweeps; ++t) {
        int rc = c->cluster ? cluster_sweep(c) : local_sweep(c);
        if (rc != PLQ_OK) return rc;
    }
    return PLQ_OK;
}

extern "C" int plq_chain_advance(plq_chain *c, uint64_t sweeps) {
    if (!c) return plq_fail(PLQ_EINVAL, "chain is NULL");
    PLQ_CUDA(plq_enter_device(c->ctx->device), "cudaSetDevice");
    return run_sweeps(c, sweeps);
}

static int check_status(plq_chain *c) {
    unsigned int st = 0;
    PLQ_CUDA(cudaMemcpyAsync(&st, &c->d_ctrl->status, sizeof st, cudaMemcpyDeviceToHost, c->stream),
             "status read");
    PLQ_CUDA(cudaStreamSynchronize(c->stream), "stream sync");
    if (st & kStatusPassCap)
        return plq_fail(PLQ_ECAP, "cluster labeling did not converge in " + std::to_string(c->pass_cap) +
                                      " passes on " + std::to_string(c->n_sites) +
                                      " sites; the cap already allows many times the lattice diameter, "
                                      "so this is a bug rather than a hard lattice");
    if (st)
        return plq_fail(PLQ_EDEVICE, "device status word " + std::to_string(st) +
                                         " (1 = look-back wait limit, 4 = bounds, 8 = queue overflow, "
                                         "16 = tile copy wait limit)");
    return PLQ_OK;
}

// Configuration (host order) into a device buffer.
static int state_to_host_order(plq_chain *c, uint8_t *dst_dev) {
    if (c->link) {
        cudaError_t e = launch_planes_to_links(c->d_state, dst_dev, c->n_sites, c->d, c->stream);
        c->launches++;
        if (e != cudaSuccess) return cuda_fail(e, "planes_to_links");
    } else {
        PLQ_CUDA(cudaMemcpyAsync(dst_dev, c->d_state, (size_t)c->n_vars, cudaMemcpyDeviceToDevice, c->stream),
                 "snapshot copy");
    }
    return PLQ_OK;
}

static int ensure_io(plq_chain *c) {
    if (!c->d_io) PLQ_CUDA(cudaMalloc((void **)&c->d_io, (size_t)c->n_vars), "cudaMalloc(io)");
    return PLQ_OK;
}

extern "C" int plq_chain_read(plq_chain *c, uint8_t *out) {
    if (!c || !out) return plq_fail(PLQ_EINVAL, "NULL argument");
    PLQ_CUDA(plq_enter_device(c->ctx->device), "cudaSetDevice");
    if (c->link) {
        int rc = ensure_io(c);
        if (rc == PLQ_OK) rc = state_to_host_order(c, c->d_io);
        if (rc != PLQ_OK) return rc;
        PLQ_CUDA(cudaMemcpyAsync(out, c->d_io, (size_t)c->n_vars, cudaMemcpyDeviceToHost, c->stream), "read");
    } else {
        PLQ_CUDA(cudaMemcpyAsync(out, c->d_state, (size_t)c->n_vars, cudaMemcpyDeviceToHost, c->stream), "read");
    }
    return check_status(c);
}

// Measurement scratch of at least `entries` int64 (and the pair lists).
static int ensure_meas(plq_chain *c, int64_t entries) {
    if (c->meas_cap >= entries) return PLQ_OK;
    if (c->d_meas) cudaFree(c->d_meas);
    if (c->d_pairs) cudaFree(c->d_pairs);
    c->d_meas = nullptr;
    c->d_pairs = nullptr;
    c->meas_cap = 0;
    PLQ_CUDA(cudaMalloc((void **)&c->d_meas, sizeof(long long) * (size_t)entries), "cudaMalloc(measurements)");
    PLQ_CUDA(cudaMalloc((void **)&c->d_pairs, sizeof(int32_t) * 2 * (size_t)entries), "cudaMalloc(pairs)");
    c->meas_cap = entries;
    return PLQ_OK;
}

extern "C" int plq_chain_axis_pair_sums(plq_chain *c, int64_t *out, int64_t capacity) {
    if (!c || !out) return plq_fail(PLQ_EINVAL, "NULL argument");
    if (c->link) return plq_fail(PLQ_EINVAL, "axis pair sums are a site-model measurement");
    const int64_t entries = pair_sum_entries(c->g);
    if (capacity < entries)
        return plq_fail(PLQ_EINVAL, "output holds " + std::to_string(capacity) + " entries, " +
                                        std::to_string(entries) + " needed");
    PLQ_CUDA(plq_enter_device(c->ctx->device), "cudaSetDevice");
    int rc = ensure_meas(c, entries);
    if (rc != PLQ_OK) return rc;
    // the (mu, r >= 1) pairs: all mu values, then all r values
    std::vector<int32_t> pairs, rs;
    for (int mu = 0; mu < c->d; ++mu)
        for (int r = 1; r <= c->g.L[mu] / 2; ++r) {
            pairs.push_back(mu);
            rs.push_back(r);
        }
    const int n_pairs = (int)rs.size();
    pairs.insert(pairs.end(), rs.begin(), rs.end());
    std::vector<long long> differ(n_pairs, 0);
    if (n_pairs) {
        PLQ_CUDA(cudaMemcpyAsync(c->d_pairs, pairs.data(), sizeof(int32_t) * 2 * (size_t)n_pairs,
                                 cudaMemcpyHostToDevice, c->stream),
                 "pair lists");
        cudaError_t e = launch_pair_differ(c->d_state, c->g, c->d_pairs, c->d_pairs + n_pairs, n_pairs, c->d_meas,
                                           c->stream);
        c->launches++;
        if (e != cudaSuccess) return cuda_fail(e, "pair sums");
        PLQ_CUDA(cudaMemcpyAsync(differ.data(), c->d_meas, sizeof(long long) * (size_t)n_pairs,
                                 cudaMemcpyDeviceToHost, c->stream),
                 "pair sums read");
    }
    rc = check_status(c);
    if (rc != PLQ_OK) return rc;
    // Ising: sum of s_i s_j = pairs - 2 * differing; Potts: agreeing = pairs - differing
    const int64_t n = c->n_sites;
    int64_t off = 0;
    int k = 0;
    for (int mu = 0; mu < c->d; ++mu) {
        out[off] = n;  // r = 0: every site with itself
        for (int r = 1; r <= c->g.L[mu] / 2; ++r, ++k)
            out[off + r] = c->desc.model == PLQ_ISING ? n - 2 * (int64_t)differ[k] : n - (int64_t)differ[k];
        off += c->g.L[mu] / 2 + 1;
    }
    return PLQ_OK;
}

extern "C" int plq_chain_polyakov(plq_chain *c, int32_t dir, int64_t *sum, int64_t *lines) {
    if (!c || !sum || !lines) return plq_fail(PLQ_EINVAL, "NULL argument");
    if (!c->link) return plq_fail(PLQ_EINVAL, "the Polyakov loop is a gauge measurement");
    if (dir < 0 || dir >= c->d) return plq_fail(PLQ_EINVAL, "direction out of range");
    PLQ_CUDA(plq_enter_device(c->ctx->device), "cudaSetDevice");
    int rc = ensure_meas(c, 1);
    if (rc != PLQ_OK) return rc;
    cudaError_t e = launch_polyakov(c->d_state, c->g, dir, c->d_meas, c->stream);
    c->launches++;
    if (e != cudaSuccess) return cuda_fail(e, "polyakov");
    long long s = 0;
    PLQ_CUDA(cudaMemcpyAsync(&s, c->d_meas, sizeof s, cudaMemcpyDeviceToHost, c->stream), "polyakov read");
    rc = check_status(c);
    if (rc != PLQ_OK) return rc;
    *sum = s;
    *lines = c->n_sites / c->g.L[dir];
    return PLQ_OK;
}

extern "C" int plq_chain_wilson(plq_chain *c, int32_t max_side, int64_t *totals, int64_t capacity,
                                int64_t *placements, int32_t *m_out) {
    if (!c || !totals || !placements) return plq_fail(PLQ_EINVAL, "NULL argument");
    if (!c->link) return plq_fail(PLQ_EINVAL, "Wilson loops are a gauge measurement");
    if (c->d < 2) return plq_fail(PLQ_EINVAL, "Wilson loops need at least two dimensions");
    if (max_side < 0) return plq_fail(PLQ_EINVAL, "max_side is negative");
    int32_t shortest = c->g.L[0];
    for (int mu = 1; mu < c->d; ++mu) shortest = std::min(shortest, c->g.L[mu]);
    const int32_t m = std::min(max_side, shortest / 2);
    if (m > wilson_max_supported())
        return plq_fail(PLQ_EUNSUPPORTED, "Wilson rectangles wider than " + std::to_string(wilson_max_supported()) +
                                              " are not supported on the device");
    const int64_t entries = (int64_t)(m + 1) * (m + 1);
    if (capacity < entries)
        return plq_fail(PLQ_EINVAL, "totals hold " + std::to_string(capacity) + " entries, " +
                                        std::to_string(entries) + " needed");
    PLQ_CUDA(plq_enter_device(c->ctx->device), "cudaSetDevice");
    int rc = ensure_meas(c, entries);
    if (rc != PLQ_OK) return rc;
    if (!c->d_loop_bits)
        PLQ_CUDA(cudaMalloc((void **)&c->d_loop_bits, sizeof(uint32_t) * (size_t)c->n_vars), "cudaMalloc(loop bits)");
    const int64_t pl = (int64_t)c->d * (c->d - 1) * c->n_sites;
    std::vector<unsigned long long> neg((size_t)entries, 0);
    if (m > 0) {
        cudaError_t e = launch_wilson(c->d_state, c->g, m, c->d_loop_bits,
                                      reinterpret_cast<unsigned long long *>(c->d_meas), c->stream);
        c->launches += 2;
        if (e != cudaSuccess) return cuda_fail(e, "wilson");
        PLQ_CUDA(cudaMemcpyAsync(neg.data(), c->d_meas, sizeof(unsigned long long) * (size_t)entries,
                                 cudaMemcpyDeviceToHost, c->stream),
                 "wilson read");
    }
    rc = check_status(c);
    if (rc != PLQ_OK) return rc;
    for (int r = 0; r <= m; ++r)
        for (int t = 0; t <= m; ++t)
            totals[r * (m + 1) + t] = (r == 0 || t == 0) ? pl : pl - 2 * (int64_t)neg[(size_t)(r * (m + 1) + t)];
    *placements = pl;
    if (m_out) *m_out = m;
    return PLQ_OK;
}

extern "C" int plq_chain_primaries(plq_chain *c, int64_t *out, int32_t *n_out) {
    if (!c) return plq_fail(PLQ_EINVAL, "NULL argument");
    PLQ_CUDA(plq_enter_device(c->ctx->device), "cudaSetDevice");
    int np = primaries_count(c->desc.model, c->q);
    cudaError_t e = launch_primaries(c->d_state, c->g, c->desc.model, c->q, c->d_obs, c->stream);
    c->launches++;
    if (e != cudaSuccess) return cuda_fail(e, "primaries");
    if (out)
        PLQ_CUDA(cudaMemcpyAsync(out, c->d_obs, sizeof(long long) * np, cudaMemcpyDeviceToHost, c->stream),
                 "primaries read");
    if (n_out) *n_out = np;
    return check_status(c);
}

extern "C" int plq_chain_next(plq_chain *c, uint8_t *out_states, int64_t *out_primaries) {
    return plq_chain_next_batch(c, 1, out_states, out_primaries);
}

extern "C" int plq_chain_next_batch(plq_chain *c, int64_t count, uint8_t *out_states, int64_t *out_primaries) {
    if (!c || count < 0) return plq_fail(PLQ_EINVAL, "bad arguments");
    PLQ_CUDA(plq_enter_device(c->ctx->device), "cudaSetDevice");
    const int np = primaries_count(c->desc.model, c->q);
    // snapshot capacity: the reference clamps its staging batch by the
    // device's buffer limit (device.rs:268-274); here by 1 GiB of snapshots.
    int64_t cap = out_states ? std::max<int64_t>(1, (int64_t(1) << 30) / std::max<int64_t>(1, c->n_vars)) : count;
    cap = std::min<int64_t>(cap, std::max<int64_t>(count, 1));
    if (out_states && c->snap_cap < cap) {
        if (c->d_snap) cudaFree(c->d_snap);
        c->d_snap = nullptr;
        PLQ_CUDA(cudaMalloc((void **)&c->d_snap, (size_t)(cap * c->n_vars)), "cudaMalloc(snapshots)");
        c->snap_cap = cap;
    }
    if (out_primaries && c->snap_obs_cap < cap) {
        if (c->d_snap_obs) cudaFree(c->d_snap_obs);
        c->d_snap_obs = nullptr;
        PLQ_CUDA(cudaMalloc((void **)&c->d_snap_obs, sizeof(long long) * (size_t)(cap * np)), "cudaMalloc(obs)");
        c->snap_obs_cap = cap;
    }
    int64_t done = 0;
    while (done < count) {
        int64_t m = std::min<int64_t>(cap, count - done);
        for (int64_t k = 0; k < m; ++k) {
            int rc = run_sweeps(c, (uint64_t)c->desc.sweeps_between);
            if (rc != PLQ_OK) return rc;
            if (out_states) {
                rc = state_to_host_order(c, c->d_snap + k * c->n_vars);
                if (rc != PLQ_OK) return rc;
            }
            if (out_primaries) {
                cudaError_t e;
                if (c->fused && !out_states) {
                    // measure this sample beside the next sweep, which writes the other buffer
                    const int k_buf = c->d_state == c->fused_map_buf[0] ? 0 : 1;
                    PLQ_CUDA(cudaEventRecord(c->swept, c->stream), "sample event");
                    PLQ_CUDA(cudaStreamWaitEvent(c->obs_stream, c->swept, 0), "sample wait");
                    e = launch_primaries(c->d_state, c->g, c->desc.model, c->q, c->d_snap_obs + k * np,
                                         c->obs_stream);
                    if (e == cudaSuccess) e = cudaEventRecord(c->measured[k_buf], c->obs_stream);
                    c->measuring[k_buf] = true;
                } else {
                    e = launch_primaries(c->d_state, c->g, c->desc.model, c->q, c->d_snap_obs + k * np,
                                         c->stream);
                }
                c->launches++;
                if (e != cudaSuccess) return cuda_fail(e, "primaries");
            }
        }
        for (int k = 0; k < 2; ++k)  // every measurement of this batch lands before the read-back
            if (c->measuring[k]) {
                PLQ_CUDA(cudaStreamWaitEvent(c->stream, c->measured[k], 0), "measurement wait");
                c->measuring[k] = false;
            }
        if (out_states)
            PLQ_CUDA(cudaMemcpyAsync(out_states + done * c->n_vars, c->d_snap, (size_t)(m * c->n_vars),
                                     cudaMemcpyDeviceToHost, c->stream),
                     "batch read-back");
        if (out_primaries)
            PLQ_CUDA(cudaMemcpyAsync(out_primaries + done * np, c->d_snap_obs, sizeof(long long) * (size_t)(m * np),
                                     cudaMemcpyDeviceToHost, c->stream),
                     "batch primaries read-back");
        int rc = check_status(c);
        if (rc != PLQ_OK) return rc;
        done += m;
    }
    return PLQ_OK;
}

extern "C" int plq_chain_sync(plq_chain *c) {
    if (!c) return plq_fail(PLQ_EINVAL, "chain is NULL");
    PLQ_CUDA(plq_enter_device(c->ctx->device), "cudaSetDevice");
    return check_status(c);
}

extern "C" int plq_chain_status(plq_chain *c) { return plq_chain_sync(c); }

extern "C" uint64_t plq_chain_sweeps_done(plq_chain *c) { return c ? c->sweeps_done : 0; }

extern "C" int plq_chain_stream_position(plq_chain *c, uint64_t *out) {
    if (!c || !out) return plq_fail(PLQ_EINVAL, "NULL argument");
    if (c->desc.rng != PLQ_RNG_STREAM) return plq_fail(PLQ_EINVAL, "not a PCG-stream chain");
    PLQ_CUDA(plq_enter_device(c->ctx->device), "cudaSetDevice");
    uint64_t rel = c->host_pos;
    if (c->lookback || c->cluster) {
        unsigned long long pos[2];
        PLQ_CUDA(cudaMemcpyAsync(pos, c->d_ctrl->pos, sizeof pos, cudaMemcpyDeviceToHost, c->stream), "pos read");
        PLQ_CUDA(cudaStreamSynchronize(c->stream), "sync");
        rel = c->cluster ? pos[c->cluster_pos_parity] : pos[c->lookback_passes & 1];
    }
    *out = c->desc.stream_offset + rel;
    return PLQ_OK;
}

extern "C" int64_t plq_chain_n_vars(plq_chain *c) { return c ? c->n_vars : 0; }
extern "C" void *plq_chain_cuda_stream(plq_chain *c) { return c ? (void *)c->stream : nullptr; }
extern "C" uint64_t plq_chain_launches(plq_chain *c) { return c ? c->launches : 0; }
extern "C" int plq_chain_cluster_labels(plq_chain *c, int32_t *out) {
    if (!c || !out) return plq_fail(PLQ_EINVAL, "NULL argument");
    if (!c->cluster) return plq_fail(PLQ_EINVAL, "not a cluster chain");
    PLQ_CUDA(plq_enter_device(c->ctx->device), "cudaSetDevice");
    int rc = cluster_labels(c, out);
    return rc == PLQ_OK ? check_status(c) : rc;
}

extern "C" int plq_chain_cluster_histogram(plq_chain *c, int64_t *hist, int32_t nbins) {
    if (!c || !hist) return plq_fail(PLQ_EINVAL, "NULL argument");
    if (!c->cluster) return plq_fail(PLQ_EINVAL, "not a cluster chain");
    PLQ_CUDA(plq_enter_device(c->ctx->device), "cudaSetDevice");
    int rc = cluster_size_histogram(c, hist, nbins);
    return rc == PLQ_OK ? check_status(c) : rc;
}

extern "C" const char *plq_chain_path(plq_chain *c) {
    if (!c) return "";
    if (c->cluster) return "cluster";
    if (c->fused) return "fused3d";
    if (c->packed) return "packed";
    return c->lookback ? "lookback" : (c->words ? "words" : "pass");
}
extern "C" void plq_chain_destroy(plq_chain *c) { chain_free(c); }
