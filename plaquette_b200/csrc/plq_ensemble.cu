// plq_ensemble.cu -- many lattices advanced by one persistent launch.
//
// An ensemble is a list of member lattices (any mix of Ising / Potts sites
// and Z2 gauge links, uneven sizes, their own beta and seed), each exactly a
// chain of the C ABI.  Advancing it by S sweeps is one cooperative launch
// (replayed from a CUDA graph): every CTA walks "super-phases" -- super-phase
// p holds colour pass p of every member that has one -- taking (member,
// chunk) work items round-robin, with a grid barrier between super-phases.
// A work item runs exactly the per-lattice pass body (plq_local_impl.cuh), so
// an ensemble sweep is bit-identical to sweeping each member with its own
// chain; what changes is that ~10^4 small launches become one.
//
// Parallel tempering: members can be grouped into ladders (same model and
// shape, one beta per slot).  Every `every` sweeps the kernel sums each
// ladder member's energy in int64, then attempts swaps of adjacent slots
// (even pairs, then odd pairs on the next attempt) with acceptance
// min(1, exp((beta_k - beta_k+1)(E_k - E_k+1))), the uniform keyed by (ladder
// seed, pair, attempt).  A swap exchanges the two members' beta slots (and so
// their decision tables), never their configurations.
//
// The autotuner times candidate (ranks per thread, CTAs per SM) pairs on a
// snapshot of the ensemble and keeps the fastest.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/plaquette.h"
#include "plq_abi_internal.h"
#include "plq_device.cuh"
#include "plq_geom.cuh"
#include "plq_local.h"
#include "plq_local_impl.cuh"
#include "plq_tables.h"

using namespace plq;

namespace {

constexpr int kEnsThreads = 256;
constexpr int kBarrierSpin = 1 << 24;
constexpr int kEnergyChunk = 2048;

struct TableSet {
    const uint64_t *hb53;
    const uint32_t *hb24;
    const uint64_t *metro53;
    const uint32_t *metro24;
    double beta;
};

struct EnsMember {
    LocalArgs a;       // the member's pass arguments (state, geometry, tables of its own beta)
    int link;          // variables on links
    int passes;        // colour passes per sweep
    int64_t n_vars;
    int64_t chunks[2]; // unused slot kept for alignment
    double j;
    int ladder;
};

struct LadderDev {
    int k;
    int every;
    uint32_t seed32;
    int32_t *member_of_slot;  // k entries
};

// Device-resident launch state, advanced by the kernel itself so a captured
// graph replays without new parameters.
struct LaunchState {
    unsigned long long sweep;       // sweeps done (keyed sweep index, PT schedule)
    unsigned long long pt_attempts; // per-ensemble attempt counter
    unsigned int bar_count;
    unsigned int bar_gen;
};

struct EnsArgs {
    EnsMember *members;
    int n_members;
    TableSet *tsets;
    int32_t *ts_of_member;
    unsigned long long *pos;  // stream heat bath: per-member stream position (relative)
    const int32_t *item_member;
    const int32_t *item_chunk;
    const int64_t *sp_begin;
    int n_sp;
    const int32_t *e_item_member;
    const int32_t *e_item_chunk;
    int64_t n_e_items;
    long long *energy;
    LadderDev *ladders;
    int n_ladders;
    int pt_every;
    LaunchState *ls;
    Control *ctrl;
    uint64_t sweeps;
    int ranks;  // ranks per thread of a work item
};

__device__ __forceinline__ unsigned int ld_volatile(const unsigned int *p) {
    return *reinterpret_cast<const volatile unsigned int *>(p);
}

// Sense-counting grid barrier; all CTAs are co-resident (cooperative launch).
// Bounded: a wait that runs out sets a status bit and lets the CTA go on.
__device__ void grid_barrier(const EnsArgs &e) {
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int gen = ld_volatile(&e.ls->bar_gen);
        __threadfence();
        unsigned int arrived = atomicAdd(&e.ls->bar_count, 1u);
        if (arrived == gridDim.x - 1) {
            atomicExch(&e.ls->bar_count, 0u);
            __threadfence();
            atomicAdd(&e.ls->bar_gen, 1u);
        } else {
            int spins = 0;
            while (ld_volatile(&e.ls->bar_gen) == gen) {
                if (++spins > kBarrierSpin) {
                    atomicOr(&e.ctrl->status, kStatusLookbackTimeout);
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

template <int R>
__device__ void run_item(const LocalArgs &a, int d, int link, int64_t chunk) {
    if (link) {
        switch (d) {
            case 2: local_chunk<2, true, false, R>(a, chunk); break;
            case 3: local_chunk<3, true, false, R>(a, chunk); break;
            case 4: local_chunk<4, true, false, R>(a, chunk); break;
            default: break;
        }
    } else {
        switch (d) {
            case 1: local_chunk<1, false, false, R>(a, chunk); break;
            case 2: local_chunk<2, false, false, R>(a, chunk); break;
            case 3: local_chunk<3, false, false, R>(a, chunk); break;
            case 4: local_chunk<4, false, false, R>(a, chunk); break;
            default: break;
        }
    }
}

// The member's pass arguments for super-phase sp of sweep index `sweep`.
__device__ void item_args(const EnsArgs &e, int m, int sp, unsigned long long sweep_in_launch, LocalArgs &sa) {
    const EnsMember &mem = e.members[m];
    sa = mem.a;
    const TableSet &ts = e.tsets[e.ts_of_member[m]];
    sa.hb53 = ts.hb53;
    sa.hb24 = ts.hb24;
    sa.metro53 = ts.metro53;
    sa.metro24 = ts.metro24;
    sa.dir = mem.link ? sp >> 1 : 0;
    sa.color = sp & 1;
    sa.sweep32 = (uint32_t)(e.ls->sweep + sweep_in_launch);
    if (sa.jump)
        sa.pass_offset = e.pos[m] + sweep_in_launch * (unsigned long long)mem.n_vars +
                         (unsigned long long)sp * (unsigned long long)(mem.a.g.n_sites / 2);
}

// int64 energy integer of a member chunk: Ising bond sum, Potts agreement,
// gauge plaquette sum (E = -J * X when the field and offsets vanish).
template <int D, bool LINK>
__device__ long long energy_chunk(const LocalArgs &a, int64_t chunk) {
    const int64_t n = a.g.n_sites;
    long long acc = 0;
    for (int64_t s = chunk * kEnergyChunk + threadIdx.x; s < n && s < (chunk + 1) * kEnergyChunk; s += blockDim.x) {
        int32_t x[D];
        site_coords<D>(a.g, s, x);
        if (LINK) {
#pragma unroll
            for (int mu = 0; mu < D; ++mu) {
                int64_t s_mu = nbr_plus(a.g, s, x, mu);
#pragma unroll
                for (int nu = mu + 1; nu < D; ++nu) {
                    int64_t s_nu = nbr_plus(a.g, s, x, nu);
                    int b = a.state[mu * n + s] ^ a.state[nu * n + s_mu] ^ a.state[mu * n + s_nu] ^ a.state[nu * n + s];
                    acc += 1 - 2 * b;
                }
            }
        } else {
            int si = a.state[s];
#pragma unroll
            for (int mu = 0; mu < D; ++mu) {
                int sj = a.state[nbr_plus(a.g, s, x, mu)];
                acc += a.model == PLQ_ISING ? (long long)((1 - 2 * si) * (1 - 2 * sj)) : (long long)(si == sj);
            }
        }
    }
    return acc;
}

__device__ long long energy_item(const LocalArgs &a, int d, int link, int64_t chunk) {
    if (link) {
        switch (d) {
            case 2: return energy_chunk<2, true>(a, chunk);
            case 3: return energy_chunk<3, true>(a, chunk);
            case 4: return energy_chunk<4, true>(a, chunk);
        }
    } else {
        switch (d) {
            case 1: return energy_chunk<1, false>(a, chunk);
            case 2: return energy_chunk<2, false>(a, chunk);
            case 3: return energy_chunk<3, false>(a, chunk);
            case 4: return energy_chunk<4, false>(a, chunk);
        }
    }
    return 0;
}

__device__ __forceinline__ long long block_sum(long long v) {
    __shared__ long long part[kEnsThreads / 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    long long t = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
    __syncthreads();
    return t;
}

// Energies of every ladder member: grid-stride over energy items.
__device__ void energy_phase(const EnsArgs &e) {
    __shared__ LocalArgs sa;
    for (int64_t i = blockIdx.x; i < e.n_e_items; i += gridDim.x) {
        int m = e.e_item_member[i];
        if (threadIdx.x == 0) sa = e.members[m].a;
        __syncthreads();
        long long part = energy_item(sa, sa.g.d, e.members[m].link, e.e_item_chunk[i]);
        long long tot = block_sum(part);
        if (threadIdx.x == 0 && tot) atomicAdd((unsigned long long *)&e.energy[m], (unsigned long long)tot);
        __syncthreads();
    }
}

// Swap attempts of every ladder (one thread per pair); attempt index `att`.
__device__ void swap_phase(const EnsArgs &e, unsigned long long att) {
    for (int l = 0; l < e.n_ladders; ++l) {
        const LadderDev &L = e.ladders[l];
        const int parity = (int)(att & 1ull);
        for (int k = parity + 2 * (int)threadIdx.x; k + 1 < L.k; k += 2 * (int)blockDim.x) {
            int m1 = L.member_of_slot[k], m2 = L.member_of_slot[k + 1];
            double b1 = e.tsets[e.ts_of_member[m1]].beta, b2 = e.tsets[e.ts_of_member[m2]].beta;
            double E1 = -e.members[m1].j * (double)e.energy[m1];
            double E2 = -e.members[m2].j * (double)e.energy[m2];
            double delta = (b1 - b2) * (E1 - E2);
            uint32_t h1 = keyed24(L.seed32 ^ 0x6a09e667u, (uint32_t)k, (uint32_t)att);
            uint32_t h2 = keyed24(L.seed32 ^ 0xbb67ae85u, (uint32_t)k, (uint32_t)att);
            double u = ((double)h1 + (double)h2 * 5.9604644775390625e-8) * 5.9604644775390625e-8;
            if (delta >= 0.0 || u < exp(delta)) {
                int32_t t1 = e.ts_of_member[m1];
                e.ts_of_member[m1] = e.ts_of_member[m2];
                e.ts_of_member[m2] = t1;
                L.member_of_slot[k] = m2;
                L.member_of_slot[k + 1] = m1;
            }
        }
    }
}

template <int R>
__global__ void __launch_bounds__(kEnsThreads) ensemble_kernel(EnsArgs e) {
    __shared__ LocalArgs sa;
    for (unsigned long long t = 0; t < e.sweeps; ++t) {
        for (int sp = 0; sp < e.n_sp; ++sp) {
            for (int64_t i = e.sp_begin[sp] + blockIdx.x; i < e.sp_begin[sp + 1]; i += gridDim.x) {
                int m = e.item_member[i];
                if (threadIdx.x == 0) item_args(e, m, sp, t, sa);
                __syncthreads();
                run_item<R>(sa, sa.g.d, e.members[m].link, e.item_chunk[i]);
                __syncthreads();
            }
            grid_barrier(e);
        }
        const unsigned long long done = e.ls->sweep + t + 1;
        if (e.n_ladders && e.pt_every > 0 && done % (unsigned long long)e.pt_every == 0) {
            if (blockIdx.x == 0)
                for (int m = threadIdx.x; m < e.n_members; m += blockDim.x) e.energy[m] = 0;
            grid_barrier(e);
            energy_phase(e);
            grid_barrier(e);
            if (blockIdx.x == 0) swap_phase(e, e.ls->pt_attempts + done / (unsigned long long)e.pt_every - 1);
            grid_barrier(e);
        }
    }
    // advance the device-resident launch state (block 0, after every CTA left the loop)
    grid_barrier(e);
    if (blockIdx.x == 0) {
        for (int m = threadIdx.x; m < e.n_members; m += blockDim.x)
            if (e.members[m].a.jump) e.pos[m] += e.sweeps * (unsigned long long)e.members[m].n_vars;
        __syncthreads();
        if (threadIdx.x == 0) e.ls->sweep += e.sweeps;
    }
}

// Unbatched path helpers: one member's energy, and one swap attempt.
__global__ void member_energy_kernel(EnsArgs e, int m) {
    __shared__ LocalArgs sa;
    if (threadIdx.x == 0) sa = e.members[m].a;
    __syncthreads();
    const int64_t n = sa.g.n_sites;
    for (int64_t c = blockIdx.x; c * kEnergyChunk < n; c += gridDim.x) {
        long long tot = block_sum(energy_item(sa, sa.g.d, e.members[m].link, c));
        if (threadIdx.x == 0 && tot) atomicAdd((unsigned long long *)&e.energy[m], (unsigned long long)tot);
    }
}
__global__ void swap_kernel(EnsArgs e, unsigned long long att) { swap_phase(e, att); }

}  // namespace

struct plq_ensemble {
    plq_ctx *ctx = nullptr;
    cudaStream_t stream = nullptr;
    std::vector<plq_chain_desc> descs;
    std::vector<EnsMember> members;            // host copies (device pointers inside)
    std::vector<int64_t> n_vars;
    std::vector<void *> allocs;                // everything to cudaFree
    std::vector<TableSet> tsets;
    std::vector<int32_t> ts_of_member;
    std::vector<std::vector<int32_t>> ladders;
    std::vector<LadderDev> ladder_dev;
    int pt_every = 0;
    EnsMember *d_members = nullptr;
    TableSet *d_tsets = nullptr;
    int32_t *d_ts = nullptr;
    unsigned long long *d_pos = nullptr;
    long long *d_energy = nullptr;
    LadderDev *d_ladders = nullptr;
    LaunchState *d_ls = nullptr;
    Control *d_ctrl = nullptr;
    // work items for the current configuration
    int ranks = 8;
    int ctas_per_sm = 2;
    int32_t *d_item_member = nullptr, *d_item_chunk = nullptr;
    int64_t *d_sp_begin = nullptr;
    int n_sp = 0;
    int32_t *d_e_member = nullptr, *d_e_chunk = nullptr;
    int64_t n_e_items = 0;
    uint64_t launches = 0;
    uint64_t sweeps_done = 0;
    uint64_t pt_attempts_host = 0;
    // graph cache
    cudaGraphExec_t graph = nullptr;
    uint64_t graph_sweeps = 0;
    int graph_ranks = 0, graph_ctas = 0;
};

namespace {

int ens_fail(cudaError_t e, const char *what) {
    return plq_fail(e == cudaErrorMemoryAllocation ? PLQ_ENOMEM : PLQ_ECUDA,
                    std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
cudaError_t dev_upload(plq_ensemble *E, const T *host, size_t count, T **out) {
    *out = nullptr;
    if (count == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc((void **)out, count * sizeof(T));
    if (e != cudaSuccess) return e;
    E->allocs.push_back(*out);
    return cudaMemcpyAsync(*out, host, count * sizeof(T), cudaMemcpyHostToDevice, E->stream);
}

void drop_graph(plq_ensemble *E) {
    if (E->graph) cudaGraphExecDestroy(E->graph);
    E->graph = nullptr;
}

int build_items(plq_ensemble *E) {
    std::vector<int32_t> im, ic;
    std::vector<int64_t> spb;
    int max_passes = 0;
    for (auto &m : E->members) max_passes = std::max(max_passes, m.passes);
    const int64_t chunk = (int64_t)kEnsThreads * E->ranks;
    for (int sp = 0; sp < max_passes; ++sp) {
        spb.push_back((int64_t)im.size());
        for (size_t m = 0; m < E->members.size(); ++m) {
            if (sp >= E->members[m].passes) continue;
            int64_t half = E->members[m].a.g.n_sites / 2;
            int64_t nc = (half + chunk - 1) / chunk;
            for (int64_t c = 0; c < nc; ++c) {
                im.push_back((int32_t)m);
                ic.push_back((int32_t)c);
            }
        }
    }
    spb.push_back((int64_t)im.size());
    std::vector<int32_t> em, ec;
    for (auto &l : E->ladders)
        for (int32_t m : l) {
            int64_t nc = (E->members[m].a.g.n_sites + kEnergyChunk - 1) / kEnergyChunk;
            for (int64_t c = 0; c < nc; ++c) {
                em.push_back(m);
                ec.push_back((int32_t)c);
            }
        }
    void *old[] = {E->d_item_member, E->d_item_chunk, E->d_sp_begin, E->d_e_member, E->d_e_chunk};
    for (void *p : old)
        if (p) {
            cudaFree(p);
            E->allocs.erase(std::remove(E->allocs.begin(), E->allocs.end(), p), E->allocs.end());
        }
    cudaError_t e = dev_upload(E, im.data(), im.size(), &E->d_item_member);
    if (e == cudaSuccess) e = dev_upload(E, ic.data(), ic.size(), &E->d_item_chunk);
    if (e == cudaSuccess) e = dev_upload(E, spb.data(), spb.size(), &E->d_sp_begin);
    if (e == cudaSuccess) e = dev_upload(E, em.data(), em.size(), &E->d_e_member);
    if (e == cudaSuccess) e = dev_upload(E, ec.data(), ec.size(), &E->d_e_chunk);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
    if (e != cudaSuccess) return ens_fail(e, "ensemble work items");
    E->n_sp = max_passes;
    E->n_e_items = (int64_t)em.size();
    drop_graph(E);
    return PLQ_OK;
}

EnsArgs ens_args(plq_ensemble *E, uint64_t sweeps) {
    EnsArgs a;
    std::memset(&a, 0, sizeof a);
    a.members = E->d_members;
    a.n_members = (int)E->members.size();
    a.tsets = E->d_tsets;
    a.ts_of_member = E->d_ts;
    a.pos = E->d_pos;
    a.item_member = E->d_item_member;
    a.item_chunk = E->d_item_chunk;
    a.sp_begin = E->d_sp_begin;
    a.n_sp = E->n_sp;
    a.e_item_member = E->d_e_member;
    a.e_item_chunk = E->d_e_chunk;
    a.n_e_items = E->n_e_items;
    a.energy = E->d_energy;
    a.ladders = E->d_ladders;
    a.n_ladders = (int)E->ladders.size();
    a.pt_every = E->pt_every;
    a.ls = E->d_ls;
    a.ctrl = E->d_ctrl;
    a.sweeps = sweeps;
    a.ranks = E->ranks;
    return a;
}

template <int R>
const void *kernel_for() {
    return (const void *)ensemble_kernel<R>;
}

const void *kernel_ptr(int ranks) {
    switch (ranks) {
        case 2: return kernel_for<2>();
        case 4: return kernel_for<4>();
        default: return kernel_for<8>();
    }
}

int max_ctas_per_sm(int ranks) {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel_ptr(ranks), kEnsThreads, 0);
    return n;
}

cudaError_t launch_persistent(plq_ensemble *E, uint64_t sweeps) {
    EnsArgs a = ens_args(E, sweeps);
    void *params[] = {&a};
    dim3 grid((unsigned)(E->ctx->sm_count * E->ctas_per_sm));
    return cudaLaunchCooperativeKernel(kernel_ptr(E->ranks), grid, dim3(kEnsThreads), params, 0, E->stream);
}

}  // namespace

extern "C" int plq_ensemble_create(plq_ctx *ctx, int32_t n, const plq_chain_desc *descs, const uint8_t *const *starts,
                                   plq_ensemble **out) {
    if (!ctx || !descs || !out || n <= 0) return plq_fail(PLQ_EINVAL, "bad arguments");
    *out = nullptr;
    for (int32_t m = 0; m < n; ++m) {
        const plq_chain_desc &d = descs[m];
        int rc = plq_chain_validate(&d);
        if (rc != PLQ_OK) return rc;
        if (d.updater == PLQ_CLUSTER) return plq_fail(PLQ_EUNSUPPORTED, "ensembles take local updaters only");
        if (d.d > 4) return plq_fail(PLQ_EUNSUPPORTED, "ensemble members have at most 4 dimensions");
        if (d.rng == PLQ_RNG_STREAM && d.updater == PLQ_METROPOLIS)
            return plq_fail(PLQ_EUNSUPPORTED,
                            "stream-mode Metropolis needs a device-wide scan per pass; ensembles run it keyed");
    }
    cudaError_t ce = cudaSetDevice(ctx->device);
    if (ce != cudaSuccess) return ens_fail(ce, "cudaSetDevice");
    plq_ensemble *E = new plq_ensemble();
    E->ctx = ctx;
    auto fail = [&](int code) {
        plq_ensemble_destroy(E);
        return code;
    };
    ce = cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) return fail(ens_fail(ce, "stream"));
    E->descs.assign(descs, descs + n);
    for (int32_t m = 0; m < n; ++m) {
        const plq_chain_desc &d = descs[m];
        EnsMember mem;
        std::memset(&mem, 0, sizeof mem);
        LocalArgs &a = mem.a;
        const int q = d.model == PLQ_POTTS ? d.q : 2;
        a.g.d = d.d;
        int64_t ns = 1;
        for (int i = 0; i < kMaxD; ++i) {
            a.g.L[i] = i < d.d ? (int32_t)d.shape[i] : 1;
            a.g.stride[i] = ns;
            if (i < d.d) ns *= d.shape[i];
        }
        a.g.n_sites = ns;
        mem.link = d.model == PLQ_GAUGE;
        mem.passes = mem.link ? 2 * d.d : 2;
        mem.n_vars = mem.link ? ns * d.d : ns;
        mem.j = d.j;
        mem.ladder = -1;
        a.q = q;
        a.kernel = d.updater;
        a.model = d.model;
        int32_t w = 1;
        for (int s = 1; s < q; ++s) {
            a.pw[s] = w;
            w *= 2 * d.d + 1;
        }
        a.seed32 = plq_fold_seed(d.seed);
        // state (links: direction planes)
        uint8_t *st = nullptr;
        ce = cudaMalloc((void **)&st, (size_t)mem.n_vars);
        if (ce != cudaSuccess) return fail(ens_fail(ce, "member state"));
        E->allocs.push_back(st);
        a.state = st;
        if (starts && starts[m]) {
            for (int64_t i = 0; i < mem.n_vars; ++i)
                if (starts[m][i] >= q) return fail(plq_fail(PLQ_EINVAL, "start state out of range"));
            if (mem.link) {
                uint8_t *tmp = nullptr;
                ce = cudaMalloc((void **)&tmp, (size_t)mem.n_vars);
                if (ce == cudaSuccess)
                    ce = cudaMemcpyAsync(tmp, starts[m], (size_t)mem.n_vars, cudaMemcpyHostToDevice, E->stream);
                if (ce == cudaSuccess) ce = launch_links_to_planes(tmp, st, ns, d.d, E->stream);
                if (ce == cudaSuccess) ce = cudaStreamSynchronize(E->stream);
                if (tmp) cudaFree(tmp);
            } else {
                ce = cudaMemcpyAsync(st, starts[m], (size_t)mem.n_vars, cudaMemcpyHostToDevice, E->stream);
            }
        } else {
            ce = cudaMemsetAsync(st, 0, (size_t)mem.n_vars, E->stream);
        }
        if (ce != cudaSuccess) return fail(ens_fail(ce, "member start"));
        if (d.rng == PLQ_RNG_STREAM) {
            uint64_t slo, shi, ilo, ihi;
            pcg_seed_from_u64(d.seed, slo, shi, ilo, ihi);
            std::vector<AffineHost> tab;
            build_jump_table(ilo, ihi, tab);
            a.inc = u128{ilo, ihi};
            u128 s = jump(reinterpret_cast<const Affine *>(tab.data()), u128{slo, shi}, d.stream_offset);
            a.base = pcg_step(s, a.inc);
            AffineHost *dj = nullptr;
            ce = dev_upload(E, tab.data(), tab.size(), &dj);
            if (ce != cudaSuccess) return fail(ens_fail(ce, "jump table"));
            a.jump = reinterpret_cast<const Affine *>(dj);
        }
        E->members.push_back(mem);
        E->n_vars.push_back(mem.n_vars);
        E->ts_of_member.push_back(-1);
    }
    // one table set per member at its own beta
    for (int32_t m = 0; m < n; ++m) {
        const plq_chain_desc &d = descs[m];
        ModelParams p;
        std::memset(&p, 0, sizeof p);
        p.model = d.model;
        p.q = d.model == PLQ_POTTS ? d.q : 2;
        p.d = d.d;
        p.beta = d.beta;
        p.j = d.j;
        p.h = d.h;
        for (int a = 0; a < PLQ_MAX_Q; ++a) p.offsets[a] = d.offsets[a];
        Tables t;
        std::string err;
        if (!build_tables(p, d.updater, d.rng, t, err)) return fail(plq_fail(PLQ_EUNSUPPORTED, err));
        TableSet ts;
        std::memset(&ts, 0, sizeof ts);
        ts.beta = d.beta;
        uint64_t *a53 = nullptr, *b53 = nullptr;
        uint32_t *a24 = nullptr, *b24 = nullptr;
        ce = dev_upload(E, t.hb53.data(), t.hb53.size(), &a53);
        if (ce == cudaSuccess) ce = dev_upload(E, t.hb24.data(), t.hb24.size(), &a24);
        if (ce == cudaSuccess) ce = dev_upload(E, t.metro53.data(), t.metro53.size(), &b53);
        if (ce == cudaSuccess) ce = dev_upload(E, t.metro24.data(), t.metro24.size(), &b24);
        if (ce != cudaSuccess) return fail(ens_fail(ce, "tables"));
        ts.hb53 = a53;
        ts.hb24 = a24;
        ts.metro53 = b53;
        ts.metro24 = b24;
        E->ts_of_member[m] = (int32_t)E->tsets.size();
        E->tsets.push_back(ts);
    }
    std::vector<unsigned long long> pos(n, 0);
    std::vector<long long> zeros(n, 0);
    LaunchState ls;
    std::memset(&ls, 0, sizeof ls);
    Control ctrl;
    std::memset(&ctrl, 0, sizeof ctrl);
    ce = dev_upload(E, E->members.data(), E->members.size(), &E->d_members);
    if (ce == cudaSuccess) ce = dev_upload(E, E->tsets.data(), E->tsets.size(), &E->d_tsets);
    if (ce == cudaSuccess) ce = dev_upload(E, E->ts_of_member.data(), E->ts_of_member.size(), &E->d_ts);
    if (ce == cudaSuccess) ce = dev_upload(E, pos.data(), pos.size(), &E->d_pos);
    if (ce == cudaSuccess) ce = dev_upload(E, zeros.data(), zeros.size(), &E->d_energy);
    if (ce == cudaSuccess) ce = dev_upload(E, &ls, 1, &E->d_ls);
    if (ce == cudaSuccess) ce = dev_upload(E, &ctrl, 1, &E->d_ctrl);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(E->stream);
    if (ce != cudaSuccess) return fail(ens_fail(ce, "ensemble set-up"));
    E->ctas_per_sm = std::max(1, std::min(2, max_ctas_per_sm(E->ranks)));
    int rc = build_items(E);
    if (rc != PLQ_OK) return fail(rc);
    *out = E;
    return PLQ_OK;
}

extern "C" int plq_ensemble_add_ladder(plq_ensemble *E, int32_t k, const int32_t *member_ids, const double *betas,
                                       int32_t every, uint64_t seed) {
    if (!E || k < 2 || !member_ids || !betas || every <= 0) return plq_fail(PLQ_EINVAL, "bad ladder arguments");
    if (E->pt_every && E->pt_every != every) return plq_fail(PLQ_EINVAL, "all ladders share one swap interval");
    const plq_chain_desc &d0 = E->descs[member_ids[0]];
    std::vector<int32_t> ids(member_ids, member_ids + k);
    for (int32_t i = 0; i < k; ++i) {
        int32_t m = ids[i];
        if (m < 0 || m >= (int32_t)E->members.size()) return plq_fail(PLQ_EINVAL, "ladder member out of range");
        if (E->members[m].ladder >= 0) return plq_fail(PLQ_EINVAL, "a member belongs to one ladder at most");
        const plq_chain_desc &d = E->descs[m];
        bool same = d.model == d0.model && d.q == d0.q && d.d == d0.d && d.updater == d0.updater && d.rng == d0.rng &&
                    d.j == d0.j && d.h == 0.0;
        for (int a = 0; a < d.d; ++a) same = same && d.shape[a] == d0.shape[a];
        for (int a = 0; a < PLQ_MAX_Q; ++a) same = same && d.offsets[a] == 0.0;
        if (!same)
            return plq_fail(PLQ_EINVAL, "ladder members must share model, shape, updater and coupling, with no field");
    }
    // slot i of the ladder runs at betas[i]: rebuild member i's table set at that beta
    for (int32_t i = 0; i < k; ++i) {
        int32_t m = ids[i];
        plq_chain_desc d = E->descs[m];
        d.beta = betas[i];
        ModelParams p;
        std::memset(&p, 0, sizeof p);
        p.model = d.model;
        p.q = d.model == PLQ_POTTS ? d.q : 2;
        p.d = d.d;
        p.beta = d.beta;
        p.j = d.j;
        Tables t;
        std::string err;
        if (!build_tables(p, d.updater, d.rng, t, err)) return plq_fail(PLQ_EUNSUPPORTED, err);
        TableSet &ts = E->tsets[E->ts_of_member[m]];
        ts.beta = betas[i];
        size_t bytes53 = t.hb53.size() * 8, bytes24 = t.hb24.size() * 4, m53 = t.metro53.size() * 8,
               m24 = t.metro24.size() * 4;
        cudaError_t ce = cudaSuccess;
        if (bytes53) ce = cudaMemcpyAsync((void *)ts.hb53, t.hb53.data(), bytes53, cudaMemcpyHostToDevice, E->stream);
        if (ce == cudaSuccess && bytes24)
            ce = cudaMemcpyAsync((void *)ts.hb24, t.hb24.data(), bytes24, cudaMemcpyHostToDevice, E->stream);
        if (ce == cudaSuccess && m53)
            ce = cudaMemcpyAsync((void *)ts.metro53, t.metro53.data(), m53, cudaMemcpyHostToDevice, E->stream);
        if (ce == cudaSuccess && m24)
            ce = cudaMemcpyAsync((void *)ts.metro24, t.metro24.data(), m24, cudaMemcpyHostToDevice, E->stream);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(E->stream);
        if (ce != cudaSuccess) return ens_fail(ce, "ladder tables");
        E->members[m].ladder = (int)E->ladders.size();
    }
    int32_t *d_slots = nullptr;
    cudaError_t ce = dev_upload(E, ids.data(), ids.size(), &d_slots);
    if (ce != cudaSuccess) return ens_fail(ce, "ladder slots");
    LadderDev L;
    L.k = k;
    L.every = every;
    L.seed32 = plq_fold_seed(seed);
    L.member_of_slot = d_slots;
    E->ladders.push_back(ids);
    E->ladder_dev.push_back(L);
    E->pt_every = every;
    if (E->d_ladders) {
        cudaFree(E->d_ladders);
        E->allocs.erase(std::remove(E->allocs.begin(), E->allocs.end(), (void *)E->d_ladders), E->allocs.end());
    }
    ce = dev_upload(E, E->ladder_dev.data(), E->ladder_dev.size(), &E->d_ladders);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(E->d_tsets, E->tsets.data(), E->tsets.size() * sizeof(TableSet),
                                                cudaMemcpyHostToDevice, E->stream);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(E->d_members, E->members.data(), E->members.size() * sizeof(EnsMember),
                             cudaMemcpyHostToDevice, E->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(E->stream);
    if (ce != cudaSuccess) return ens_fail(ce, "ladder upload");
    return build_items(E);
}

static int ens_status(plq_ensemble *E) {
    unsigned int st = 0;
    cudaError_t e = cudaMemcpyAsync(&st, &E->d_ctrl->status, sizeof st, cudaMemcpyDeviceToHost, E->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
    if (e != cudaSuccess) return ens_fail(e, "ensemble sync");
    if (st) return plq_fail(PLQ_EDEVICE, "ensemble status word " + std::to_string(st) + " (1 = barrier wait limit)");
    return PLQ_OK;
}

extern "C" int plq_ensemble_advance(plq_ensemble *E, uint64_t sweeps) {
    if (!E) return plq_fail(PLQ_EINVAL, "NULL ensemble");
    if (sweeps == 0) return PLQ_OK;
    cudaError_t e = cudaSetDevice(E->ctx->device);
    if (e != cudaSuccess) return ens_fail(e, "cudaSetDevice");
    // one persistent launch, captured once per (sweeps, configuration) and replayed
    if (!E->graph || E->graph_sweeps != sweeps || E->graph_ranks != E->ranks || E->graph_ctas != E->ctas_per_sm) {
        drop_graph(E);
        cudaGraph_t g = nullptr;
        e = cudaStreamBeginCapture(E->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t le = launch_persistent(E, sweeps);
            e = cudaStreamEndCapture(E->stream, &g);
            if (le != cudaSuccess) e = le;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&E->graph, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            cudaGetLastError();
            E->graph = nullptr;
            // capture refused: launch directly
            e = launch_persistent(E, sweeps);
            E->launches++;
            if (e != cudaSuccess) return ens_fail(e, "persistent launch");
            E->sweeps_done += sweeps;
            return PLQ_OK;
        }
        E->graph_sweeps = sweeps;
        E->graph_ranks = E->ranks;
        E->graph_ctas = E->ctas_per_sm;
    }
    e = cudaGraphLaunch(E->graph, E->stream);
    E->launches++;
    if (e != cudaSuccess) return ens_fail(e, "graph launch");
    E->sweeps_done += sweeps;
    return PLQ_OK;
}

extern "C" int plq_ensemble_advance_unbatched(plq_ensemble *E, uint64_t sweeps) {
    if (!E) return plq_fail(PLQ_EINVAL, "NULL ensemble");
    cudaError_t e = cudaSetDevice(E->ctx->device);
    if (e != cudaSuccess) return ens_fail(e, "cudaSetDevice");
    // host mirrors of the device-resident state the per-member launches need
    LaunchState ls;
    std::vector<unsigned long long> pos(E->members.size());
    std::vector<int32_t> ts(E->members.size());
    e = cudaMemcpyAsync(&ls, E->d_ls, sizeof ls, cudaMemcpyDeviceToHost, E->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(pos.data(), E->d_pos, pos.size() * sizeof(pos[0]), cudaMemcpyDeviceToHost, E->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ts.data(), E->d_ts, ts.size() * sizeof(ts[0]), cudaMemcpyDeviceToHost, E->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
    if (e != cudaSuccess) return ens_fail(e, "unbatched state read");
    EnsArgs ea = ens_args(E, 0);
    for (uint64_t t = 0; t < sweeps; ++t) {
        for (size_t m = 0; m < E->members.size(); ++m) {
            const EnsMember &mem = E->members[m];
            LocalArgs a = mem.a;
            const TableSet &tsm = E->tsets[ts[m]];
            a.hb53 = tsm.hb53;
            a.hb24 = tsm.hb24;
            a.metro53 = tsm.metro53;
            a.metro24 = tsm.metro24;
            a.sweep32 = (uint32_t)(ls.sweep + t);
            for (int pass = 0; pass < mem.passes; ++pass) {
                a.dir = mem.link ? pass >> 1 : 0;
                a.color = pass & 1;
                if (a.jump) a.pass_offset = pos[m] + (uint64_t)pass * (uint64_t)(a.g.n_sites / 2);
                e = launch_local_pass(a, mem.link, false, E->stream);
                E->launches++;
                if (e != cudaSuccess) return ens_fail(e, "member pass");
            }
            if (a.jump) pos[m] += (unsigned long long)mem.n_vars;
        }
        const unsigned long long done = ls.sweep + t + 1;
        if (!E->ladders.empty() && done % (unsigned long long)E->pt_every == 0) {
            cudaMemsetAsync(E->d_energy, 0, sizeof(long long) * E->members.size(), E->stream);
            for (auto &l : E->ladders)
                for (int32_t m : l) {
                    int64_t nc = (E->members[m].a.g.n_sites + kEnergyChunk - 1) / kEnergyChunk;
                    member_energy_kernel<<<(unsigned)std::min<int64_t>(nc, 1184), kEnsThreads, 0, E->stream>>>(ea, m);
                    E->launches++;
                }
            swap_kernel<<<1, kEnsThreads, 0, E->stream>>>(ea, ls.pt_attempts + done / E->pt_every - 1);
            E->launches++;
            e = cudaMemcpyAsync(ts.data(), E->d_ts, ts.size() * sizeof(ts[0]), cudaMemcpyDeviceToHost, E->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
            if (e != cudaSuccess) return ens_fail(e, "unbatched swaps");
        }
    }
    ls.sweep += sweeps;
    e = cudaMemcpyAsync(E->d_ls, &ls, sizeof ls, cudaMemcpyHostToDevice, E->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(E->d_pos, pos.data(), pos.size() * sizeof(pos[0]), cudaMemcpyHostToDevice, E->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
    if (e != cudaSuccess) return ens_fail(e, "unbatched state write");
    E->sweeps_done += sweeps;
    return PLQ_OK;
}

extern "C" int plq_ensemble_set_config(plq_ensemble *E, int32_t ranks_per_thread, int32_t ctas_per_sm) {
    if (!E) return plq_fail(PLQ_EINVAL, "NULL ensemble");
    if (ranks_per_thread != 2 && ranks_per_thread != 4 && ranks_per_thread != 8)
        return plq_fail(PLQ_EINVAL, "ranks per thread must be 2, 4 or 8");
    int maxc = max_ctas_per_sm(ranks_per_thread);
    if (ctas_per_sm < 1 || ctas_per_sm > maxc)
        return plq_fail(PLQ_EINVAL, "CTAs per SM must be in 1.." + std::to_string(maxc));
    E->ranks = ranks_per_thread;
    E->ctas_per_sm = ctas_per_sm;
    return build_items(E);
}

extern "C" int plq_ensemble_tune(plq_ensemble *E, int32_t trial_sweeps, int32_t *ranks_out, int32_t *ctas_out,
                                 double *ms_per_sweep_out) {
    if (!E || trial_sweeps <= 0) return plq_fail(PLQ_EINVAL, "bad arguments");
    cudaError_t e = cudaSetDevice(E->ctx->device);
    if (e != cudaSuccess) return ens_fail(e, "cudaSetDevice");
    // snapshot: member states, PT slots, positions, launch state
    int64_t total = 0;
    for (auto v : E->n_vars) total += v;
    uint8_t *backup = nullptr;
    e = cudaMalloc((void **)&backup, (size_t)total);
    if (e != cudaSuccess) return ens_fail(e, "tune snapshot");
    std::vector<int32_t> ts(E->members.size());
    std::vector<unsigned long long> pos(E->members.size());
    LaunchState ls;
    std::vector<std::vector<int32_t>> slots;
    auto snapshot = [&](bool save) {
        int64_t off = 0;
        for (size_t m = 0; m < E->members.size(); ++m) {
            if (save)
                cudaMemcpyAsync(backup + off, E->members[m].a.state, (size_t)E->n_vars[m], cudaMemcpyDeviceToDevice,
                                E->stream);
            else
                cudaMemcpyAsync(E->members[m].a.state, backup + off, (size_t)E->n_vars[m], cudaMemcpyDeviceToDevice,
                                E->stream);
            off += E->n_vars[m];
        }
        if (save) {
            cudaMemcpyAsync(ts.data(), E->d_ts, ts.size() * 4, cudaMemcpyDeviceToHost, E->stream);
            cudaMemcpyAsync(pos.data(), E->d_pos, pos.size() * 8, cudaMemcpyDeviceToHost, E->stream);
            cudaMemcpyAsync(&ls, E->d_ls, sizeof ls, cudaMemcpyDeviceToHost, E->stream);
            slots.clear();
            for (size_t l = 0; l < E->ladders.size(); ++l) {
                slots.emplace_back(E->ladders[l].size());
                cudaMemcpyAsync(slots.back().data(), E->ladder_dev[l].member_of_slot, slots.back().size() * 4,
                                cudaMemcpyDeviceToHost, E->stream);
            }
        } else {
            cudaMemcpyAsync(E->d_ts, ts.data(), ts.size() * 4, cudaMemcpyHostToDevice, E->stream);
            cudaMemcpyAsync(E->d_pos, pos.data(), pos.size() * 8, cudaMemcpyHostToDevice, E->stream);
            cudaMemcpyAsync(E->d_ls, &ls, sizeof ls, cudaMemcpyHostToDevice, E->stream);
            for (size_t l = 0; l < E->ladders.size(); ++l)
                cudaMemcpyAsync(E->ladder_dev[l].member_of_slot, slots[l].data(), slots[l].size() * 4,
                                cudaMemcpyHostToDevice, E->stream);
        }
        cudaStreamSynchronize(E->stream);
    };
    snapshot(true);
    int best_r = E->ranks, best_c = E->ctas_per_sm;
    double best = 1e300;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    for (int r : {2, 4, 8}) {
        int maxc = max_ctas_per_sm(r);
        for (int c = 1; c <= std::min(maxc, 4); c *= 2) {
            if (plq_ensemble_set_config(E, r, c) != PLQ_OK) continue;
            snapshot(false);
            if (plq_ensemble_advance(E, 1) != PLQ_OK) continue;  // warm-up (and graph build)
            snapshot(false);
            if (plq_ensemble_advance(E, (uint64_t)trial_sweeps) != PLQ_OK) continue;  // capture
            snapshot(false);
            cudaEventRecord(t0, E->stream);
            if (plq_ensemble_advance(E, (uint64_t)trial_sweeps) != PLQ_OK) continue;
            cudaEventRecord(t1, E->stream);
            cudaEventSynchronize(t1);
            float ms = 0;
            cudaEventElapsedTime(&ms, t0, t1);
            if (ms < best) {
                best = ms;
                best_r = r;
                best_c = c;
            }
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    snapshot(false);
    cudaFree(backup);
    E->sweeps_done = 0;
    int rc = plq_ensemble_set_config(E, best_r, best_c);
    if (rc != PLQ_OK) return rc;
    if (ranks_out) *ranks_out = best_r;
    if (ctas_out) *ctas_out = best_c;
    if (ms_per_sweep_out) *ms_per_sweep_out = best / trial_sweeps;
    return ens_status(E);
}

extern "C" int plq_ensemble_sync(plq_ensemble *E) {
    if (!E) return plq_fail(PLQ_EINVAL, "NULL ensemble");
    return ens_status(E);
}

extern "C" int plq_ensemble_read(plq_ensemble *E, int32_t m, uint8_t *out) {
    if (!E || !out || m < 0 || m >= (int32_t)E->members.size()) return plq_fail(PLQ_EINVAL, "bad arguments");
    const EnsMember &mem = E->members[m];
    cudaError_t e = cudaSuccess;
    if (mem.link) {
        uint8_t *tmp = nullptr;
        e = cudaMalloc((void **)&tmp, (size_t)mem.n_vars);
        if (e == cudaSuccess) e = launch_planes_to_links(mem.a.state, tmp, mem.a.g.n_sites, mem.a.g.d, E->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(out, tmp, (size_t)mem.n_vars, cudaMemcpyDeviceToHost, E->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
        if (tmp) cudaFree(tmp);
    } else {
        e = cudaMemcpyAsync(out, mem.a.state, (size_t)mem.n_vars, cudaMemcpyDeviceToHost, E->stream);
    }
    if (e != cudaSuccess) return ens_fail(e, "member read");
    return ens_status(E);
}

extern "C" int plq_ensemble_primaries(plq_ensemble *E, int32_t m, int64_t *out, int32_t *n_out) {
    if (!E || !out || m < 0 || m >= (int32_t)E->members.size()) return plq_fail(PLQ_EINVAL, "bad arguments");
    const EnsMember &mem = E->members[m];
    long long *d = nullptr;
    int np = primaries_count(mem.a.model, mem.a.q);
    cudaError_t e = cudaMalloc((void **)&d, sizeof(long long) * (size_t)np);
    if (e == cudaSuccess) e = launch_primaries(mem.a.state, mem.a.g, mem.a.model, mem.a.q, d, E->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, sizeof(long long) * (size_t)np, cudaMemcpyDeviceToHost, E->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
    if (d) cudaFree(d);
    if (e != cudaSuccess) return ens_fail(e, "member primaries");
    if (n_out) *n_out = np;
    return ens_status(E);
}

extern "C" int plq_ensemble_betas(plq_ensemble *E, double *beta_of_member) {
    if (!E || !beta_of_member) return plq_fail(PLQ_EINVAL, "bad arguments");
    std::vector<int32_t> ts(E->members.size());
    cudaError_t e = cudaMemcpyAsync(ts.data(), E->d_ts, ts.size() * 4, cudaMemcpyDeviceToHost, E->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
    if (e != cudaSuccess) return ens_fail(e, "betas read");
    for (size_t m = 0; m < ts.size(); ++m) beta_of_member[m] = E->tsets[ts[m]].beta;
    return PLQ_OK;
}

extern "C" int64_t plq_ensemble_n_vars(plq_ensemble *E) {
    int64_t t = 0;
    if (E)
        for (auto v : E->n_vars) t += v;
    return t;
}
extern "C" void *plq_ensemble_cuda_stream(plq_ensemble *E) { return E ? (void *)E->stream : nullptr; }
extern "C" uint64_t plq_ensemble_launches(plq_ensemble *E) { return E ? E->launches : 0; }

extern "C" void plq_ensemble_destroy(plq_ensemble *E) {
    if (!E) return;
    if (E->ctx) cudaSetDevice(E->ctx->device);
    if (E->stream) cudaStreamSynchronize(E->stream);
    drop_graph(E);
    for (void *p : E->allocs) cudaFree(p);
    if (E->stream) cudaStreamDestroy(E->stream);
    delete E;
}
