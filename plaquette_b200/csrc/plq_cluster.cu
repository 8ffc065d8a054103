// plq_cluster.cu -- Swendsen-Wang and Wolff chains on the device.
//
// One cluster sweep of ClusterUpdate::sweep (src/updater.rs:541-613) /
// GpuClusterChain::run_sweep (src/gpu_cluster.rs:492-526):
//
//  1. bonds  -- a forward bond (site, axis) opens iff the two sites agree and
//               the draw is below p = 1 - exp(-beta * gap) (the host computes
//               p as ClusterUpdate::bond_probability does).  Keyed stream: the
//               draw is keyed by the bond index (cluster_prelude.wgsl:61-80).
//               PCG stream: one draw per *agreeing* bond in site-major,
//               axis-minor order (cluster.rs:44-62), placed by a device-wide
//               exclusive scan (decoupled look-back) over agreeing bonds.
//  2. labels -- lock-free union-find: every open bond unites its ends by
//               hooking the larger root under the smaller with a CAS, first
//               inside 64x64 tiles in shared memory (tile_hook_kernel), then
//               for the bonds that leave a tile (boundary_hook_kernel); the
//               relabel pass walks each site to its root (a short walk: sites
//               point at their tile-local roots) and stores it.  Roots only
//               ever hook under smaller roots, so each component ends rooted
//               at its minimum site: the canonical min-site label of the
//               reference GPU (the fixed point of cluster_prelude.wgsl:113-147),
//               and, ranked, the reference CPU's first-encounter compaction
//               (cluster.rs:199-226).
//  3. relabel -- keyed: per-root keyed draw (cluster_relabel.wgsl:39-90).
//               PCG stream: clusters in root order draw next_below(q) (or the
//               forced-change proposal) at consecutive positions, inside the
//               rank scan; rand's range sampler occasionally takes a second
//               draw, which shifts every later cluster -- those rare events
//               are reported by the scan and fixed up by re-running the
//               (parallel) draw pass with the events known, in a short host
//               loop.
//
// Wolff on the keyed stream: the reference relabels the cluster of a keyed
// seed site in the full decomposition (cluster_relabel.wgsl:55-66).  Here a
// frontier BFS from the seed site over lazily evaluated keyed bonds finds the
// same component (work proportional to the cluster), its minimum site is the
// root the forced change is keyed on.  One CTA runs all requested updates in
// one launch.  Wolff on the PCG stream (draws in grow_cluster's FIFO order)
// is sequential by definition and is not run on the device.
//
// Every loop that waits or retries has an iteration cap; hitting one sets a
// status bit the host turns into PLQ_ECAP / PLQ_EDEVICE.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/plaquette.h"
#include "plq_cluster.h"
#include "plq_device.cuh"
#include "plq_geom.cuh"
#include "plq_local.h"
#include "plq_tables.h"

using namespace plq;

namespace {

constexpr int kThreads = 256;
constexpr int kSitesPerThread = 8;
constexpr int kChunk = kThreads * kSitesPerThread;
constexpr int kSpinLimit = 1 << 22;
constexpr int kMaxEvents = 64;
constexpr int kBfsThreads = 1024;
constexpr unsigned long long kDescAgg = 1ull, kDescPrefix = 2ull;

struct ClusterArgs {
    uint8_t *state;
    uint8_t *bonds;
    int32_t *parent;
    uint8_t *fresh;
    int32_t *rank;
    struct ChunkBase {     // stream relabel: per root_rank chunk, the state at the label draw of
        u128 st;           // the chunk's first root (no second draws before it) and that root's rank
        int64_t rank0, pad;
    } *chunk_base;
    uint32_t *stamp;
    int32_t *queue;
    Geom g;
    int q;
    int extent, relabel;
    uint32_t seed32, sweep32;
    uint32_t kp24;   // keyed: bond open iff k24 < kp24
    uint64_t kp53;   // stream: bond open iff k53 < kp53
    const Affine *jump;
    u128 base, inc;
    Control *ctrl;
    unsigned long long *desc;
    int64_t n_chunks;
    uint64_t ticket_base;
    uint32_t epoch;
    int cap;          // iteration cap of finds and unions
    const int32_t *events;  // sorted ranks of clusters that take two draws
    int n_events;
    int *first_new;   // device: smallest rank with an unknown second draw
    uint64_t updates; // Wolff: updates in this launch
};

__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int32_t ld_relaxed32(const int32_t *p) {
    int32_t v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long make_desc(uint32_t epoch, unsigned long long st, uint32_t value) {
    return ((unsigned long long)(epoch & 0x3FFFFFFFu) << 34) | (st << 32) | value;
}

// Block-wide exclusive scan of `v` with decoupled look-back across chunks
// (taken in ticket order).  Returns the thread's global exclusive prefix and,
// through block_total / ok, the chunk total and whether the wait completed.
__device__ uint64_t chunk_scan(const ClusterArgs &a, int64_t chunk, int v, int &block_total, bool &ok) {
    __shared__ int warp_tot[kThreads / 32];
    __shared__ unsigned long long s_excl;
    __shared__ int s_fail;
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += y;
    }
    if (lane == 31) warp_tot[wid] = incl;
    if (threadIdx.x == 0) s_fail = 0;
    __syncthreads();
    int warp_excl = 0, total = 0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) {
        int t = warp_tot[w];
        if (w < wid) warp_excl += t;
        total += t;
    }
    // Warp 0 looks back over 32 predecessors per round: the nearest one with an inclusive
    // prefix ends the walk, and the aggregates up to it are summed with one warp reduction.
    if (wid == 0) {
        unsigned long long excl = 0;
        bool fail = false;
        if (chunk == 0) {
            if (lane == 0) atomicExch(&a.desc[0], make_desc(a.epoch, kDescPrefix, (uint32_t)total));
        } else {
            if (lane == 0) atomicExch(&a.desc[chunk], make_desc(a.epoch, kDescAgg, (uint32_t)total));
            const uint32_t ep = a.epoch & 0x3FFFFFFFu;
            int64_t top = chunk - 1;
            int spins = 0;
            while (true) {
                const int64_t idx = top - lane;
                // before chunk 0: an inclusive prefix of 0
                const unsigned long long d = idx >= 0 ? ld_relaxed(&a.desc[idx]) : make_desc(a.epoch, kDescPrefix, 0u);
                const unsigned long long st = (uint32_t)(d >> 34) == ep ? (d >> 32) & 3ull : 0ull;
                const unsigned incl_lanes = __ballot_sync(0xffffffffu, st == kDescPrefix);
                const unsigned ready = __ballot_sync(0xffffffffu, st != 0ull);
                // lanes up to the nearest inclusive prefix (all 32 when none is in this window)
                const unsigned span = incl_lanes ? (((incl_lanes & (0u - incl_lanes)) << 1) - 1u) : 0xffffffffu;
                if ((ready & span) != span) {
                    if (++spins > kSpinLimit) {
                        fail = true;
                        break;
                    }
                    __nanosleep(32);
                    continue;
                }
                unsigned long long v = ((span >> lane) & 1u) ? (unsigned long long)(uint32_t)d : 0ull;
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
                excl += v;
                if (incl_lanes) break;
                top -= 32;
            }
            if (lane == 0 && !fail) atomicExch(&a.desc[chunk], make_desc(a.epoch, kDescPrefix, (uint32_t)(excl + total)));
        }
        if (lane == 0) {
            if (fail) {
                s_fail = 1;
                atomicOr(&a.ctrl->status, kStatusLookbackTimeout);
            }
            s_excl = excl;
        }
    }
    __syncthreads();
    ok = s_fail == 0;
    block_total = total;
    return s_excl + (uint64_t)(warp_excl + incl - v);
}

__device__ __forceinline__ int64_t take_chunk(const ClusterArgs &a, bool lookback) {
    if (!lookback) return blockIdx.x;
    __shared__ unsigned long long s_ticket;
    if (threadIdx.x == 0) s_ticket = atomicAdd(&a.ctrl->ticket, 1ull) - a.ticket_base;
    __syncthreads();
    return (int64_t)s_ticket;
}

// ------------------------------------------------------------- 1. bonds
static_assert(kSitesPerThread == 8, "the bonds pass loads and stores a thread's sites as one 8-byte word");

// High bit of each byte of the result set iff that byte of a equals that of b.
__device__ __forceinline__ uint64_t bytes_equal(uint64_t a, uint64_t b) {
    const uint64_t e = a ^ b, lo7 = 0x7F7F7F7F7F7F7F7Full;
    return ~(((e & lo7) + lo7) | e) & ~lo7;
}

template <int D, bool STREAM>
__global__ void __launch_bounds__(kThreads) bonds_kernel(ClusterArgs a) {
    const int64_t n = a.g.n_sites;
    const int64_t chunk = take_chunk(a, STREAM);
    if (chunk >= a.n_chunks) {
        if (threadIdx.x == 0) atomicOr(&a.ctrl->status, kStatusBounds);
        return;
    }
    const int64_t s0 = chunk * kChunk + (int64_t)threadIdx.x * kSitesPerThread;
    // With L0 % 8 == 0 a thread's 8 sites (s0 is a multiple of 8) lie in one row, and every
    // +mu neighbour row is 8-byte aligned: one vector load per direction, one vector store.
    const bool row8 = (a.g.L[0] & 7) == 0;
    uint8_t agree[kSitesPerThread];
    int count = 0;
    if (row8) {
#pragma unroll
        for (int i = 0; i < kSitesPerThread; ++i) agree[i] = 0;
        if (s0 < n) {
            int32_t x[D];
            site_coords<D>(a.g, s0, x);
            const uint64_t cv = *reinterpret_cast<const uint64_t *>(a.state + s0);
            // +x: bytes s0+1 .. s0+8, the last one wrapping to the row start
            const int64_t past = x[0] + kSitesPerThread < a.g.L[0] ? s0 + kSitesPerThread
                                                                   : s0 + kSitesPerThread - a.g.L[0];
            uint64_t eq[D];
            eq[0] = bytes_equal(cv, (cv >> 8) | ((uint64_t)a.state[past] << 56));
#pragma unroll
            for (int mu = 1; mu < D; ++mu)
                eq[mu] = bytes_equal(cv, *reinterpret_cast<const uint64_t *>(a.state + nbr_plus(a.g, s0, x, mu)));
#pragma unroll
            for (int i = 0; i < kSitesPerThread; ++i) {
                uint32_t m = 0;
#pragma unroll
                for (int mu = 0; mu < D; ++mu) m |= (uint32_t)((eq[mu] >> (8 * i + 7)) & 1u) << mu;
                agree[i] = (uint8_t)m;
                count += __popc(m);
            }
        }
    } else {
#pragma unroll
        for (int i = 0; i < kSitesPerThread; ++i) {
            int64_t s = s0 + i;
            agree[i] = 0;
            if (s >= n) continue;
            int32_t x[D];
            site_coords<D>(a.g, s, x);
            uint8_t cur = a.state[s];
            uint8_t m = 0;
#pragma unroll
            for (int mu = 0; mu < D; ++mu)
                if (a.state[nbr_plus(a.g, s, x, mu)] == cur) m |= (uint8_t)(1u << mu);
            agree[i] = m;
            count += __popc(m);
        }
    }
    u128 st{0, 0};
    if (STREAM) {
        int total;
        bool ok;
        uint64_t excl = chunk_scan(a, chunk, count, total, ok);
        if (!ok) return;
        // One full jump per chunk, to its first draw (thread 0's prefix is the chunk's); each
        // thread then applies the low digits of its offset inside the chunk (< kChunk * D draws).
        // Jump maps are iterates of one affine map, so they compose in any order.
        __shared__ unsigned long long s_base, s_excl0;
        __shared__ u128 s_state;
        if (threadIdx.x == 0) {
            s_base = a.ctrl->pos[0];
            if (chunk == a.n_chunks - 1) a.ctrl->pos[1] = s_base + excl + (unsigned long long)total;
            s_excl0 = excl;
            s_state = jump(a.jump, a.base, s_base + excl);
        }
        __syncthreads();
        if (count) st = jump(a.jump, s_state, excl - s_excl0);
    }
    uint64_t opened = 0;
#pragma unroll
    for (int i = 0; i < kSitesPerThread; ++i) {
        int64_t s = s0 + i;
        if (s >= n) continue;
        uint8_t open = 0;
#pragma unroll
        for (int mu = 0; mu < D; ++mu) {
            if (!((agree[i] >> mu) & 1u)) continue;
            bool drawn;
            if (STREAM) {
                uint64_t k = draw53(st);
                st = pcg_step(st, a.inc);
                drawn = k < a.kp53;
            } else {
                drawn = keyed24(a.seed32 ^ kBondKey, (uint32_t)(s * D + mu), a.sweep32) < a.kp24;
            }
            if (drawn) open |= (uint8_t)(1u << mu);
        }
        if (row8) opened |= (uint64_t)open << (8 * i);
        else a.bonds[s] = open;
    }
    if (row8 && s0 < n) *reinterpret_cast<uint64_t *>(a.bonds + s0) = opened;
}

// The keyed bond (s, mu) to the +mu neighbour `nb`, evaluated where it is
// used (no bond array on the keyed stream): open iff the two sites agree and
// the bond's keyed draw is below p (cluster_prelude.wgsl:61-80).
template <int D>
__device__ __forceinline__ bool keyed_bond(const ClusterArgs &a, int64_t s, int mu, int64_t nb) {
    return a.state[s] == a.state[nb] &&
           keyed24(a.seed32 ^ kBondKey, (uint32_t)(s * D + mu), a.sweep32) < a.kp24;
}

// ------------------------------------------------------------ 2. labels
__device__ __forceinline__ int32_t find_root(int32_t *parent, int32_t x, int cap, Control *ctrl) {
    int32_t p = ld_relaxed32(&parent[x]);
    int it = 0;
    while (p != x) {
        int32_t gp = ld_relaxed32(&parent[p]);
        if (gp != p) parent[x] = gp;  // path halving: gp is an ancestor, never a wrong set
        x = p;
        p = gp;
        if (++it > cap) {
            atomicOr(&ctrl->status, kStatusPassCap);
            break;
        }
    }
    return x;
}

__device__ __forceinline__ void unite(int32_t *parent, int32_t a, int32_t b, int cap, Control *ctrl) {
    for (int it = 0;; ++it) {
        a = find_root(parent, a, cap, ctrl);
        b = find_root(parent, b, cap, ctrl);
        if (a == b) return;
        if (a > b) {
            int32_t t = a;
            a = b;
            b = t;
        }
        if (atomicCAS(&parent[b], b, a) == b) return;  // b was still a root: hooked under a
        if (it > cap) {
            atomicOr(&ctrl->status, kStatusPassCap);
            return;
        }
    }
}

// ---- tile-local labelling: a CTA owns a T0 x T1 tile of (dims 0, 1), T0 and T1
// the largest power-of-two divisors of L0, L1 capped at 64.  It unites the
// open bonds inside the tile on a shared-memory parent array (same rule:
// larger root under smaller, so each local root is the tile component's
// minimum site; local and global index orders agree), then points every site
// at its local root -- this is also the label init (cluster_prelude.wgsl:83-93)
// of every site.  Only bonds that leave the tile go through the global
// union-find (boundary_hook_kernel): ~2 / 64 of the bonds of a 2D lattice.
constexpr int kTileMax = 64;
constexpr int kTileSites = kTileMax * kTileMax;

__device__ __forceinline__ int tile_extent(int L) {
    const int p2 = L & -L;  // largest power-of-two divisor
    return p2 < kTileMax ? p2 : kTileMax;
}

__device__ __forceinline__ int lfind(int32_t *p, int32_t x, int cap, Control *ctrl) {
    int32_t px = p[x];
    int it = 0;
    while (px != x) {
        // no path halving: the trees inside a tile are shallow (about 2.3 deep at beta_c),
        // and the halving stores cost more than the hops they save
        const int32_t gp = p[px];
        x = px;
        px = gp;
        if (++it > cap) {
            atomicOr(&ctrl->status, kStatusPassCap);
            break;
        }
    }
    return x;
}

__device__ __forceinline__ void lunite(int32_t *p, int32_t a, int32_t b, int cap, Control *ctrl) {
    for (int it = 0;; ++it) {
        a = lfind(p, a, cap, ctrl);
        b = lfind(p, b, cap, ctrl);
        if (a == b) return;
        if (a > b) {
            const int32_t t = a;
            a = b;
            b = t;
        }
        if (atomicCAS(&p[b], b, a) == b) return;
        if (it > cap) {
            atomicOr(&ctrl->status, kStatusPassCap);
            return;
        }
    }
}

template <int D, bool KEYED>
__global__ void __launch_bounds__(kThreads) tile_hook_kernel(ClusterArgs a) {
    __shared__ int32_t p[kTileSites];
    __shared__ uint8_t bs[kTileSites];  // the tile's bond bytes
    const int L0 = a.g.L[0], L1 = D >= 2 ? a.g.L[1] : 1;
    const int T0 = tile_extent(L0), T1 = D >= 2 ? tile_extent(L1) : 1;
    const int T = T0 * T1;
    const int tiles0 = L0 / T0, tiles1 = L1 / T1;
    // tile origin: (tx * T0, ty * T1, slab) with slab the index over dims >= 2
    const int64_t bid = blockIdx.x;
    const int tx = (int)(bid % tiles0);
    const int64_t r1 = bid / tiles0;
    const int ty = (int)(r1 % tiles1);
    const int64_t slab = r1 / tiles1;
    const int64_t base = slab * (int64_t)L0 * L1 + (int64_t)ty * T1 * L0 + (int64_t)tx * T0;
    const int cap = a.cap < kTileSites + 64 ? a.cap : kTileSites + 64;
    // T0 is a power of two: local index li = yl * T0 + xl splits by shift and mask (a runtime
    // division would cost ~20 instructions, several times per site)
    const int sh0 = __ffs(T0) - 1, m0 = T0 - 1;
    // x runs first: a warp holds 32 consecutive sites; each site points straight at
    // the start of its run of open +x bonds (the run's minimum), found with one ballot
    const int lane = threadIdx.x & 31;
    const int rounds = (T + (int)blockDim.x - 1) / (int)blockDim.x;
    for (int k = 0; k < rounds; ++k) {
        const int li = k * (int)blockDim.x + (int)threadIdx.x;
        const bool valid = li < T;
        const int xl = li & m0;
        uint32_t own = 0;
        if (valid) {
            const int64_t s = base + xl + (int64_t)(li >> sh0) * L0;
            if (KEYED) {
                // +x and +y bonds from the spins and the keyed draws (the bonds along
                // dims >= 2 all leave the tile: boundary_hook_kernel evaluates them)
                const int xg = tx * T0 + xl;
                own = keyed_bond<D>(a, s, 0, xg + 1 < L0 ? s + 1 : s + 1 - L0) ? 1u : 0u;
                if (D >= 2) {
                    const int yg = ty * T1 + (li >> sh0);
                    own |= keyed_bond<D>(a, s, 1, yg + 1 < L1 ? s + L0 : s - (int64_t)(L1 - 1) * L0) ? 2u : 0u;
                }
            } else {
                own = a.bonds[s];
            }
        }
        if (valid) bs[li] = (uint8_t)own;
        // the bond into this site from its -x neighbour (lane - 1), inside this warp's segment
        const uint32_t from_left = __shfl_up_sync(0xffffffffu, own, 1);
        const bool joined = valid && lane > 0 && xl > 0 && (from_left & 1u) != 0;
        const unsigned starts = __ballot_sync(0xffffffffu, !joined);
        const int start = 31 - __clz(starts & (0xffffffffu >> (31 - lane)));
        if (valid) p[li] = li - lane + start;
    }
    __syncthreads();
    // the remaining bonds inside the tile: +x across a warp segment or around the row, and +y.
    // (Skipping a +y bond that the x-1 bonds already imply saves 16 % of these unions at
    // criticality but measured slower: the extra shared-memory reads cost more.)
    for (int li = threadIdx.x; li < T; li += blockDim.x) {
        const int xl = li & m0, yl = li >> sh0;
        const uint32_t b = bs[li];
        if (b & 1u) {
            if (xl + 1 < T0) {
                if ((li & 31) == 31) lunite(p, li, li + 1, cap, a.ctrl);
            } else if (T0 == L0) {
                lunite(p, li, li - (T0 - 1), cap, a.ctrl);
            }
        }
        if (D >= 2 && (b & 2u)) {  // +y inside the tile
            if (yl + 1 < T1) lunite(p, li, li + T0, cap, a.ctrl);
            else if (T1 == L1) lunite(p, li, li - T0 * (T1 - 1), cap, a.ctrl);
        }
    }
    __syncthreads();
    // The forest is final: each site walks to its local root (read-only; trees at β_c are
    // about 2.3 deep on average, at most ~10, so this beats block-wide pointer-jumping rounds)
    // and points at it.
    for (int li = threadIdx.x; li < T; li += blockDim.x) {
        int32_t r = li;
        for (int it = 0; p[r] != r && it < kTileSites; ++it) r = p[r];
        const int64_t s = base + (li & m0) + (int64_t)(li >> sh0) * L0;
        a.parent[s] = (int32_t)(base + (r & m0) + (int64_t)(r >> sh0) * L0);
    }
}

// Global unions for the open bonds that leave their tile: +x bonds of the
// tile's last column (when tiles split the rows), +y bonds of its last row
// (when tiles split dim 1), and every bond along dims >= 2.  Thread t of the
// grid takes candidate site t of each family in turn.
template <int D, bool KEYED>
__global__ void __launch_bounds__(kThreads) boundary_hook_kernel(ClusterArgs a) {
    const int64_t n = a.g.n_sites;
    const int L0 = a.g.L[0], L1 = D >= 2 ? a.g.L[1] : 1;
    const int T0 = tile_extent(L0), T1 = D >= 2 ? tile_extent(L1) : 1;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    // the two families in one index space, so a thread makes at most one union of them:
    // candidates c < nx are sites with x = k*T0 + T0-1 (n / T0 of them), the rest the sites of
    // rows with y = k*T1 + T1-1 (n / T1)
    const int64_t nx = T0 < L0 ? n / T0 : 0;
    const int64_t ny = D >= 2 && T1 < L1 ? n / T1 : 0;
    const int64_t per_row = L0;
    for (int64_t c = t0; c < nx + ny; c += stride) {
        int64_t s;
        int mu;
        if (c < nx) {
            s = c * T0 + (T0 - 1);
            mu = 0;
        } else {
            const int64_t cy = c - nx;
            const int64_t row = fdiv((uint32_t)cy, a.g.dm[0], a.g.dl[0]);  // index among the selected rows
            s = (row * T1 + (T1 - 1)) * per_row + (cy - row * per_row);
            mu = 1;
        }
        if (!KEYED && !((a.bonds[s] >> mu) & 1u)) continue;
        int32_t x[D];
        site_coords<D>(a.g, s, x);
        // compile-time directions keep the coordinates in registers
        const int64_t nb = mu == 0 ? nbr_plus(a.g, s, x, 0) : nbr_plus(a.g, s, x, D >= 2 ? 1 : 0);
        if (KEYED && !keyed_bond<D>(a, s, mu, nb)) continue;
        unite(a.parent, (int32_t)s, (int32_t)nb, a.cap, a.ctrl);
    }
    if (D >= 3) {
        for (int64_t s = t0; s < n; s += stride) {
            uint8_t b = 0;
            int32_t x[D];
            if (KEYED) {
                site_coords<D>(a.g, s, x);
#pragma unroll
                for (int mu = 2; mu < D; ++mu)
                    if (keyed_bond<D>(a, s, mu, nbr_plus(a.g, s, x, mu))) b |= (uint8_t)(1u << (mu - 2));
            } else {
                b = (uint8_t)(a.bonds[s] >> 2);
                if (!b) continue;
                site_coords<D>(a.g, s, x);
            }
#pragma unroll
            for (int mu = 2; mu < D; ++mu)
                if ((b >> (mu - 2)) & 1u) unite(a.parent, (int32_t)s, (int32_t)nbr_plus(a.g, s, x, mu), a.cap, a.ctrl);
        }
    }
}

// Read-only find for the relabel pass: a compressing find could overwrite a
// site another thread has just set to its root with a non-root ancestor.
__device__ __forceinline__ int32_t find_root_ro(const int32_t *parent, int32_t x, int cap, Control *ctrl) {
    int32_t p = ld_relaxed32(&parent[x]);
    int it = 0;
    while (p != x) {
        x = p;
        p = ld_relaxed32(&parent[x]);
        if (++it > cap) {
            atomicOr(&ctrl->status, kStatusPassCap);
            break;
        }
    }
    return x;
}

// Sites a thread resolves at once (stride apart): the loads of all of them
// are issued before any is used, so their latencies overlap.
constexpr int kRootBatch = 4;

// The roots of sites s0, s0 + stride, ... after the boundary unions; also
// stores them, which leaves the parent array flat (every site holding its
// root) for the readers after the sweep.  tile_hook left every site pointing
// at its local root, and the boundary unions only re-point roots (or halve
// paths onto local roots), so the walk from a site's parent is short: at
// beta_c about 7 % of the local roots end up under another root, a few levels
// deep at most.  Every value stored is a final root, so concurrent walks stay
// correct.
__device__ __forceinline__ void take_roots(const ClusterArgs &a, int64_t s0, int64_t stride, int64_t n,
                                           int32_t *root) {
    int32_t p[kRootBatch], q[kRootBatch];
#pragma unroll
    for (int k = 0; k < kRootBatch; ++k) {
        const int64_t s = s0 + k * stride;
        p[k] = s < n ? a.parent[s] : 0;  // only this thread writes parent[s] here
    }
#pragma unroll
    for (int k = 0; k < kRootBatch; ++k) q[k] = s0 + k * stride < n ? ld_relaxed32(&a.parent[p[k]]) : 0;
#pragma unroll
    for (int k = 0; k < kRootBatch; ++k) {
        const int64_t s = s0 + k * stride;
        root[k] = 0;
        if (s >= n) continue;
        const int32_t r = q[k] == p[k] ? p[k] : find_root_ro(a.parent, q[k], a.cap, a.ctrl);
        if (r != p[k]) a.parent[s] = r;
        root[k] = r;
    }
}

// ----------------------------------------------------------- 3. relabel
// keyed (cluster_relabel.wgsl:72-89), every cluster
__global__ void relabel_keyed_kernel(ClusterArgs a) {
    const int64_t n = a.g.n_sites;
    const uint32_t q = (uint32_t)a.q;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t s0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s0 < n; s0 += stride * kRootBatch) {
        int32_t roots[kRootBatch];
        take_roots(a, s0, stride, n, roots);
#pragma unroll
        for (int k = 0; k < kRootBatch; ++k) {
            const int64_t s = s0 + k * stride;
            if (s >= n) continue;
            const uint32_t root = (uint32_t)roots[k];
            float u = __fmul_rn((float)keyed24(a.seed32 ^ kRootSalt, root, a.sweep32), 5.9604644775390625e-8f);
            if (a.relabel == PLQ_RELABEL_FORCED) {
                uint32_t step = __float2uint_rz(__fmul_rn(u, (float)(q - 1u)));
                if (step >= q - 1u) step = q - 2u;
                a.state[s] = (uint8_t)((a.state[s] + 1u + step) % q);
            } else {
                uint32_t draw = __float2uint_rz(__fmul_rn(u, (float)q));
                if (draw >= q) draw = q - 1u;
                a.state[s] = (uint8_t)draw;
            }
        }
    }
}

// rand 0.10 random_range(0..range) for range < 2^32 whose first draw is the
// output of state st: returns the value and whether a second draw was taken.
__device__ __forceinline__ uint32_t next_below_from(const ClusterArgs &a, u128 st, uint32_t range, bool &second) {
    uint32_t x = (uint32_t)xsl_rr(st);
    uint64_t m = (uint64_t)x * range;
    uint32_t result = (uint32_t)(m >> 32), lo = (uint32_t)m;
    second = lo > (uint32_t)(0u - range);
    if (second) {
        st = pcg_step(st, a.inc);
        uint32_t x2 = (uint32_t)xsl_rr(st);
        uint32_t hi2 = (uint32_t)(((uint64_t)x2 * range) >> 32);
        if ((uint64_t)lo + hi2 > 0xFFFFFFFFull) result += 1;
    }
    return result;
}

// The fresh label of a cluster (ClusterUpdate::fresh_label, updater.rs:507-521)
// whose first draw is the output of st: next_below(q), or with forced change the
// proposal of updater.rs:659-668 (q >= 3 there).
__device__ __forceinline__ uint32_t fresh_label(const ClusterArgs &a, u128 st, uint32_t cur, bool &second) {
    if (a.relabel == PLQ_RELABEL_REDRAW) return next_below_from(a, st, (uint32_t)a.q, second);
    const uint32_t d = next_below_from(a, st, (uint32_t)(a.q - 1), second);
    return d + (d >= cur ? 1u : 0u);
}

// stream: rank of each root among roots (first-encounter order), and each
// root's fresh label drawn with no second draws known: rank r draws at
// bond_end + r, so a thread steps the stream from one root to the next.  A root
// whose label takes a second draw reports its rank in first_new; the host then
// re-runs the draws (root_draw_kernel) with that event known.
template <int D>
__global__ void __launch_bounds__(kThreads) root_rank_kernel(ClusterArgs a) {
    const int64_t n = a.g.n_sites;
    const int64_t chunk = take_chunk(a, true);
    if (chunk >= a.n_chunks) {
        if (threadIdx.x == 0) atomicOr(&a.ctrl->status, kStatusBounds);
        return;
    }
    const int64_t s0 = chunk * kChunk + (int64_t)threadIdx.x * kSitesPerThread;
    int count = 0;
    uint32_t mask = 0;
    if (s0 + kSitesPerThread <= n) {  // s0 is a multiple of 8: two aligned 16-byte loads
        const int4 lo = *reinterpret_cast<const int4 *>(a.parent + s0);
        const int4 hi = *reinterpret_cast<const int4 *>(a.parent + s0 + 4);
        const int32_t par[kSitesPerThread] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
#pragma unroll
        for (int i = 0; i < kSitesPerThread; ++i)
            if (par[i] == (int32_t)(s0 + i)) mask |= 1u << i;
        count = __popc(mask);
    } else {
#pragma unroll
        for (int i = 0; i < kSitesPerThread; ++i) {
            int64_t s = s0 + i;
            if (s < n && a.parent[s] == (int32_t)s) {
                mask |= 1u << i;
                ++count;
            }
        }
    }
    int total;
    bool ok;
    uint64_t excl = chunk_scan(a, chunk, count, total, ok);
    if (!ok) return;
    __shared__ u128 s_state;
    __shared__ unsigned long long s_excl0;
    if (threadIdx.x == 0) {
        if (chunk == a.n_chunks - 1) a.ctrl->scratch[0] = excl + (unsigned long long)total;
        // labels are drawn from the end of the bond draws, in root rank order
        const u128 st0 = jump(a.jump, a.base, a.ctrl->pos[1] + excl);
        a.chunk_base[chunk].st = st0;
        a.chunk_base[chunk].rank0 = (int64_t)excl;
        s_state = st0;
        s_excl0 = excl;
    }
    __syncthreads();
    if (!count) return;
    u128 st = jump(a.jump, s_state, excl - s_excl0);
    int r = (int)excl;
#pragma unroll
    for (int i = 0; i < kSitesPerThread; ++i) {
        if (!((mask >> i) & 1u)) continue;
        const int64_t s = s0 + i;
        a.rank[s] = r;
        bool second;
        a.fresh[s] = (uint8_t)fresh_label(a, st, a.state[s], second);
        if (second) atomicMin(a.first_new, r);
        st = pcg_step(st, a.inc);
        ++r;
    }
}

// stream: each root draws its cluster's fresh label (ClusterUpdate::fresh_label,
// updater.rs:507-521) at bond_end + rank + (known second draws before it),
// jumping from its root_rank chunk's first label draw.
__global__ void root_draw_kernel(ClusterArgs a) {
    const int64_t n = a.g.n_sites;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
        if (a.parent[s] != (int32_t)s) continue;
        int32_t r = a.rank[s];
        int before = 0;
        bool known = false;
        for (int e = 0; e < a.n_events; ++e) {
            before += a.events[e] < r;
            known |= a.events[e] == r;
        }
        const ClusterArgs::ChunkBase &cb = a.chunk_base[s / kChunk];
        const u128 st = jump(a.jump, cb.st, (uint64_t)((int64_t)r - cb.rank0) + (uint64_t)before);
        bool second;
        a.fresh[s] = (uint8_t)fresh_label(a, st, a.state[s], second);
        if (second && !known) atomicMin(a.first_new, r);
    }
}

__global__ void apply_fresh_kernel(ClusterArgs a) {
    const int64_t n = a.g.n_sites;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t s0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s0 < n; s0 += stride * kRootBatch) {
        int32_t roots[kRootBatch];
        take_roots(a, s0, stride, n, roots);
        uint8_t f[kRootBatch];
#pragma unroll
        for (int k = 0; k < kRootBatch; ++k) f[k] = s0 + k * stride < n ? a.fresh[roots[k]] : 0;
#pragma unroll
        for (int k = 0; k < kRootBatch; ++k)
            if (s0 + k * stride < n) a.state[s0 + k * stride] = f[k];
    }
}

__global__ void finish_pos_kernel(Control *ctrl, int n_events) {
    ctrl->pos[0] = ctrl->pos[1] + ctrl->scratch[0] + (unsigned long long)n_events;
}

// ------------------------------------------------------- Wolff (keyed BFS)
template <int D>
__global__ void __launch_bounds__(kBfsThreads) wolff_bfs_kernel(ClusterArgs a) {
    __shared__ int s_tail, s_min;
    __shared__ int s_lvl_begin, s_lvl_end;
    const int64_t n = a.g.n_sites;
    const uint32_t q = (uint32_t)a.q;
    for (uint64_t up = 0; up < a.updates; ++up) {
        const uint32_t sweep = a.sweep32 + (uint32_t)up;
        const uint32_t epoch = sweep + 1u;
        // seed site (cluster_relabel.wgsl:55-61)
        float us = __fmul_rn((float)keyed24(a.seed32 ^ kSeedSalt, 0u, sweep), 5.9604644775390625e-8f);
        uint32_t seed_site = __float2uint_rz(__fmul_rn(us, (float)(uint32_t)n));
        if (seed_site >= (uint32_t)n) seed_site = (uint32_t)n - 1u;
        if (threadIdx.x == 0) {
            a.queue[0] = (int32_t)seed_site;
            a.stamp[seed_site] = epoch;
            s_tail = 1;
            s_min = (int32_t)seed_site;
            s_lvl_begin = 0;
            s_lvl_end = 1;
        }
        __syncthreads();
        const uint8_t cur = a.state[seed_site];
        while (true) {
            int begin = s_lvl_begin, end = s_lvl_end;
            if (begin >= end) break;
            for (int i = begin + threadIdx.x; i < end; i += blockDim.x) {
                int64_t u = a.queue[i];
                int32_t x[D];
                site_coords<D>(a.g, u, x);
                // the 2D neighbours' loads, then their stamp exchanges, each issued together so
                // their latencies overlap; the cluster (a set) does not depend on the order
                int64_t v[2 * D];
                uint8_t sv[2 * D];
#pragma unroll
                for (int k = 0; k < 2 * D; ++k) {
                    v[k] = (k & 1) == 0 ? nbr_plus(a.g, u, x, k >> 1) : nbr_minus(a.g, u, x, k >> 1);
                    sv[k] = a.state[v[k]];
                }
                bool join[2 * D];
#pragma unroll
                for (int k = 0; k < 2 * D; ++k) {
                    const uint32_t bond = (uint32_t)(((k & 1) == 0 ? u : v[k]) * D + (k >> 1));
                    join[k] = sv[k] == cur && keyed24(a.seed32 ^ kBondKey, bond, sweep) < a.kp24;
                }
#pragma unroll
                for (int k = 0; k < 2 * D; ++k)
                    if (join[k]) join[k] = atomicExch(&a.stamp[v[k]], epoch) != epoch;  // not yet a member
#pragma unroll
                for (int k = 0; k < 2 * D; ++k) {
                    if (!join[k]) continue;
                    int slot = atomicAdd(&s_tail, 1);
                    a.queue[slot] = (int32_t)v[k];
                    atomicMin(&s_min, (int32_t)v[k]);
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                s_lvl_begin = end;
                s_lvl_end = s_tail;
            }
            __syncthreads();
        }
        const int members = s_tail;
        const uint32_t root = (uint32_t)s_min;
        float u = __fmul_rn((float)keyed24(a.seed32 ^ kRootSalt, root, sweep), 5.9604644775390625e-8f);
        uint8_t next;
        if (a.relabel == PLQ_RELABEL_FORCED) {
            uint32_t step = __float2uint_rz(__fmul_rn(u, (float)(q - 1u)));
            if (step >= q - 1u) step = q - 2u;
            next = (uint8_t)((cur + 1u + step) % q);
        } else {
            uint32_t draw = __float2uint_rz(__fmul_rn(u, (float)q));
            if (draw >= q) draw = q - 1u;
            next = (uint8_t)draw;
        }
        for (int i = threadIdx.x; i < members; i += blockDim.x) a.state[a.queue[i]] = next;
        if (threadIdx.x == 0) a.ctrl->scratch[1] = (unsigned long long)members;
        __syncthreads();
    }
}

// ------------------------------------------------------------ sizes
// Cluster sizes: one atomic per distinct root among a warp's 32 sites (a big
// cluster's root would otherwise take one atomic per site).
__global__ void sizes_kernel(const int32_t *parent, int32_t *size, int64_t n) {
    const int64_t n_pad = (n + 31) & ~(int64_t)31;  // whole warps per iteration: the match below is warp-wide
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n_pad; s += (int64_t)gridDim.x * blockDim.x) {
        const int32_t r = s < n ? parent[s] : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, r);
        if (r >= 0 && (int)(threadIdx.x & 31u) == __ffs(peers) - 1) atomicAdd(&size[r], __popc(peers));
    }
}
// Clusters per size bin [2^k, 2^(k+1)): counted per CTA in shared memory (bins
// 0..31 cover every int32 size), one global atomic per bin per CTA.
__global__ void size_hist_kernel(const int32_t *parent, const int32_t *size, int64_t n, long long *hist, int nbins) {
    __shared__ unsigned int bins[32];
    if (threadIdx.x < 32) bins[threadIdx.x] = 0;
    __syncthreads();
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
        if (parent[s] != (int32_t)s) continue;
        atomicAdd(&bins[31 - __clz(size[s])], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 32 && bins[threadIdx.x]) {
        int bin = (int)threadIdx.x;
        if (bin >= nbins) bin = nbins - 1;
        atomicAdd((unsigned long long *)&hist[bin], (unsigned long long)bins[threadIdx.x]);
    }
}

// ------------------------------------------------------------ host side
struct ClusterDev {
    uint8_t *bonds = nullptr;
    int32_t *parent = nullptr;
    uint8_t *fresh = nullptr;
    int32_t *rank = nullptr;
    ClusterArgs::ChunkBase *chunk_base = nullptr;
    uint32_t *stamp = nullptr;
    int32_t *queue = nullptr;
    unsigned long long *desc = nullptr;
    int64_t n_chunks = 0;
    int64_t n_tiles = 0;  // CTAs of tile_hook_kernel
    int32_t *events = nullptr;
    int *first_new = nullptr;
    int32_t *sizes = nullptr;
    uint32_t kp24 = 0;
    uint64_t kp53 = 0;
    uint64_t lookback_launches = 0;
    std::vector<int32_t> host_events;
    bool decomposed = false;
};

unsigned grid_stride_blocks(int64_t n) {
    int64_t b = (n + kThreads - 1) / kThreads;
    if (b > 148 * 16) b = 148 * 16;
    return (unsigned)(b < 1 ? 1 : b);
}

ClusterArgs cluster_args(plq_chain *c) {
    ClusterDev *cd = static_cast<ClusterDev *>(c->cl);
    ClusterArgs a;
    std::memset(&a, 0, sizeof a);
    a.state = c->d_state;
    a.bonds = cd->bonds;
    a.parent = cd->parent;
    a.fresh = cd->fresh;
    a.rank = cd->rank;
    a.chunk_base = cd->chunk_base;
    a.stamp = cd->stamp;
    a.queue = cd->queue;
    a.g = c->g;
    a.q = c->q;
    a.extent = c->desc.extent;
    a.relabel = c->desc.relabel;
    a.seed32 = c->seed32;
    a.sweep32 = (uint32_t)c->sweeps_done;
    a.kp24 = cd->kp24;
    a.kp53 = cd->kp53;
    a.jump = c->d_jump;
    a.base = c->base;
    a.inc = c->inc;
    a.ctrl = c->d_ctrl;
    a.desc = cd->desc;
    a.n_chunks = cd->n_chunks;
    a.cap = (c->desc.flags & PLQ_FLAG_TINY_PASS_CAP) ? 1 : (int)std::min<int64_t>(c->n_sites + 64, 1 << 30);
    a.events = cd->events;
    a.first_new = cd->first_new;
    return a;
}

// The range of the per-cluster label draw: next_below(q) to redraw
// (src/updater.rs:512), propose's next_below(q - 1) for the forced change
// (:515, :659-668; a range of 1 at q = 2, which consumes nothing).
bool label_range_is_power_of_two(const plq_chain *c) {
    const uint32_t range = c->desc.relabel == PLQ_RELABEL_FORCED ? (uint32_t)c->q - 1u : (uint32_t)c->q;
    return (range & (range - 1u)) == 0u;
}

template <int D>
int sweep_d(plq_chain *c, uint64_t sweeps) {
    ClusterDev *cd = static_cast<ClusterDev *>(c->cl);
    const bool stream = c->desc.rng == PLQ_RNG_STREAM;
    const int64_t n = c->n_sites;
    const unsigned gs = grid_stride_blocks(n);
    if (c->desc.extent == PLQ_EXTENT_SEEDED) {
        ClusterArgs a = cluster_args(c);
        a.updates = sweeps;
        wolff_bfs_kernel<D><<<1, kBfsThreads, 0, c->stream>>>(a);
        c->launches++;
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return plq_fail(PLQ_ECUDA, std::string("wolff launch: ") + cudaGetErrorString(e));
        c->sweeps_done += sweeps;
        cd->decomposed = false;
        return PLQ_OK;
    }
    for (uint64_t t = 0; t < sweeps; ++t) {
        ClusterArgs a = cluster_args(c);
        auto lookback = [&](ClusterArgs &x) {
            x.epoch = (uint32_t)(cd->lookback_launches + 1);
            x.ticket_base = cd->lookback_launches * (uint64_t)cd->n_chunks;
            cd->lookback_launches++;
        };
        if (stream) {
            // PCG stream: the bond draws sit at scanned positions, so they are made in one pass
            lookback(a);
            bonds_kernel<D, true><<<(unsigned)cd->n_chunks, kThreads, 0, c->stream>>>(a);
            tile_hook_kernel<D, false><<<(unsigned)cd->n_tiles, kThreads, 0, c->stream>>>(a);
            boundary_hook_kernel<D, false><<<gs, kThreads, 0, c->stream>>>(a);
            c->launches += 3;
        } else {
            // keyed: each bond is a closed form of its index, evaluated where it is used
            tile_hook_kernel<D, true><<<(unsigned)cd->n_tiles, kThreads, 0, c->stream>>>(a);
            boundary_hook_kernel<D, true><<<gs, kThreads, 0, c->stream>>>(a);
            c->launches += 2;
        }
        if (!stream) {
            relabel_keyed_kernel<<<gs, kThreads, 0, c->stream>>>(a);
            c->launches++;
        } else if (label_range_is_power_of_two(c)) {
            // rand's range sampler never takes a second draw for a power-of-two range
            // (x * 2^k leaves its low word a multiple of 2^k, never inside the rejection
            // zone above 2^32 - 2^k): the labels drawn by the rank pass are final and the
            // sweep needs no round-trip to the host
            lookback(a);
            root_rank_kernel<D><<<(unsigned)cd->n_chunks, kThreads, 0, c->stream>>>(a);
            apply_fresh_kernel<<<gs, kThreads, 0, c->stream>>>(a);
            finish_pos_kernel<<<1, 1, 0, c->stream>>>(c->d_ctrl, 0);
            c->launches += 3;
        } else {
            lookback(a);
            const int none = 0x7FFFFFFF;
            cudaMemcpyAsync(cd->first_new, &none, sizeof none, cudaMemcpyHostToDevice, c->stream);
            // ranks, and the labels with no second draws known
            root_rank_kernel<D><<<(unsigned)cd->n_chunks, kThreads, 0, c->stream>>>(a);
            c->launches++;
            cd->host_events.clear();
            for (int round = 0;; ++round) {
                if (round > 0) {  // again, with the second draws found so far known
                    a.n_events = (int)cd->host_events.size();
                    cudaMemcpyAsync(cd->first_new, &none, sizeof none, cudaMemcpyHostToDevice, c->stream);
                    cudaMemcpyAsync(cd->events, cd->host_events.data(), sizeof(int32_t) * a.n_events,
                                    cudaMemcpyHostToDevice, c->stream);
                    root_draw_kernel<<<gs, kThreads, 0, c->stream>>>(a);
                    c->launches++;
                }
                int first = none;
                cudaMemcpyAsync(&first, cd->first_new, sizeof first, cudaMemcpyDeviceToHost, c->stream);
                cudaError_t e = cudaStreamSynchronize(c->stream);
                if (e != cudaSuccess) return plq_fail(PLQ_ECUDA, std::string("root draws: ") + cudaGetErrorString(e));
                if (first == none) break;
                if ((int)cd->host_events.size() >= kMaxEvents)
                    return plq_fail(PLQ_EDEVICE, "too many two-draw label events in one sweep");
                cd->host_events.insert(std::upper_bound(cd->host_events.begin(), cd->host_events.end(), first), first);
            }
            apply_fresh_kernel<<<gs, kThreads, 0, c->stream>>>(a);
            finish_pos_kernel<<<1, 1, 0, c->stream>>>(c->d_ctrl, (int)cd->host_events.size());
            c->launches += 2;
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return plq_fail(PLQ_ECUDA, std::string("cluster sweep: ") + cudaGetErrorString(e));
        c->sweeps_done++;
        cd->decomposed = true;
    }
    return PLQ_OK;
}

}  // namespace

int cluster_validate(const plq_chain_desc *d) {
    if (d->extent == PLQ_EXTENT_SEEDED && d->rng == PLQ_RNG_STREAM)
        return plq_fail(PLQ_EUNSUPPORTED,
                        "Wolff on the PCG stream draws in grow_cluster's sequential FIFO order; this device path "
                        "runs the seeded extent on the keyed stream only");
    return PLQ_OK;
}

int cluster_create(plq_chain *c) {
    ClusterDev *cd = new ClusterDev();
    c->cl = cd;
    const int64_t n = c->n_sites;
    double p = plq_bond_probability(c->desc.model, c->desc.j, c->desc.beta);
    // bond open iff u < p: keyed in f32 (cluster_prelude.wgsl:77), stream in f64 (updater.rs:570-572)
    float p32 = (float)p;
    uint32_t lo = 0, hi = 1u << 24;
    while (lo < hi) {
        uint32_t mid = lo + (hi - lo) / 2;
        if ((float)mid * (1.0f / 16777216.0f) < p32) lo = mid + 1;
        else hi = mid;
    }
    cd->kp24 = lo;
    uint64_t lo53 = 0, hi53 = 1ull << 53;
    while (lo53 < hi53) {
        uint64_t mid = lo53 + (hi53 - lo53) / 2;
        if ((double)mid * (1.0 / 9007199254740992.0) < p) lo53 = mid + 1;
        else hi53 = mid;
    }
    cd->kp53 = lo53;
    c->pass_cap = (c->desc.flags & PLQ_FLAG_TINY_PASS_CAP) ? 1 : std::min<int64_t>(n + 64, 1 << 30);
    cd->n_chunks = (n + kChunk - 1) / kChunk;
    {
        auto tile = [](int64_t L) { const int64_t p2 = L & -L; return p2 < kTileMax ? p2 : (int64_t)kTileMax; };
        const int64_t t0 = tile(c->g.L[0]), t1 = c->d >= 2 ? tile(c->g.L[1]) : 1;
        cd->n_tiles = n / (t0 * t1);
    }
    cudaError_t e = cudaSuccess;
    auto alloc = [&](void **p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes);
    };
    if (c->desc.extent == PLQ_EXTENT_SEEDED) {
        alloc((void **)&cd->stamp, sizeof(uint32_t) * (size_t)n);
        alloc((void **)&cd->queue, sizeof(int32_t) * (size_t)n);
        if (e == cudaSuccess) e = cudaMemsetAsync(cd->stamp, 0, sizeof(uint32_t) * (size_t)n, c->stream);
    } else {
        alloc((void **)&cd->bonds, (size_t)n);
        alloc((void **)&cd->parent, sizeof(int32_t) * (size_t)n);
        alloc((void **)&cd->desc, sizeof(unsigned long long) * (size_t)cd->n_chunks);
        if (e == cudaSuccess)
            e = cudaMemsetAsync(cd->desc, 0, sizeof(unsigned long long) * (size_t)cd->n_chunks, c->stream);
        if (c->desc.rng == PLQ_RNG_STREAM) {
            alloc((void **)&cd->fresh, (size_t)n);
            alloc((void **)&cd->rank, sizeof(int32_t) * (size_t)n);
            alloc((void **)&cd->chunk_base, sizeof(ClusterArgs::ChunkBase) * (size_t)cd->n_chunks);
            alloc((void **)&cd->events, sizeof(int32_t) * kMaxEvents);
            alloc((void **)&cd->first_new, sizeof(int));
        }
    }
    if (e != cudaSuccess)
        return plq_fail(e == cudaErrorMemoryAllocation ? PLQ_ENOMEM : PLQ_ECUDA,
                        std::string("cluster buffers: ") + cudaGetErrorString(e));
    return PLQ_OK;
}

int cluster_sweep_n(plq_chain *c, uint64_t sweeps) {
    switch (c->d) {
        case 1: return sweep_d<1>(c, sweeps);
        case 2: return sweep_d<2>(c, sweeps);
        case 3: return sweep_d<3>(c, sweeps);
        case 4: return sweep_d<4>(c, sweeps);
        case 5: return sweep_d<5>(c, sweeps);
        case 6: return sweep_d<6>(c, sweeps);
        case 7: return sweep_d<7>(c, sweeps);
        case 8: return sweep_d<8>(c, sweeps);
        default: return plq_fail(PLQ_EINVAL, "dimension out of range");
    }
}

int cluster_sweep(plq_chain *c) { return cluster_sweep_n(c, 1); }

void cluster_free(plq_chain *c) {
    ClusterDev *cd = static_cast<ClusterDev *>(c->cl);
    if (!cd) return;
    void *ptrs[] = {cd->bonds, cd->parent, cd->fresh, cd->rank, cd->chunk_base, cd->stamp, cd->queue,
                    cd->desc, cd->events, cd->first_new, cd->sizes};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    delete cd;
    c->cl = nullptr;
}

int cluster_labels(plq_chain *c, int32_t *out) {
    ClusterDev *cd = static_cast<ClusterDev *>(c->cl);
    if (!cd || !cd->decomposed) return plq_fail(PLQ_EINVAL, "no decomposition yet (run a Swendsen-Wang sweep first)");
    cudaError_t e = cudaMemcpyAsync(out, cd->parent, sizeof(int32_t) * (size_t)c->n_sites, cudaMemcpyDeviceToHost,
                                    c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return plq_fail(PLQ_ECUDA, std::string("labels read: ") + cudaGetErrorString(e));
    return PLQ_OK;
}

int cluster_size_histogram(plq_chain *c, int64_t *hist, int32_t nbins) {
    ClusterDev *cd = static_cast<ClusterDev *>(c->cl);
    if (!cd || nbins <= 0) return plq_fail(PLQ_EINVAL, "bad arguments");
    std::vector<long long> h((size_t)nbins, 0);
    if (c->desc.extent == PLQ_EXTENT_SEEDED) {
        unsigned long long members = 0;
        cudaMemcpyAsync(&members, &c->d_ctrl->scratch[1], sizeof members, cudaMemcpyDeviceToHost, c->stream);
        cudaError_t e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) return plq_fail(PLQ_ECUDA, cudaGetErrorString(e));
        if (members) {
            int bin = 63 - __builtin_clzll(members);
            h[(size_t)std::min(bin, nbins - 1)] = 1;
        }
    } else {
        if (!cd->decomposed) return plq_fail(PLQ_EINVAL, "no decomposition yet (run a Swendsen-Wang sweep first)");
        const int64_t n = c->n_sites;
        cudaError_t e = cudaSuccess;
        if (!cd->sizes) e = cudaMalloc((void **)&cd->sizes, sizeof(int32_t) * (size_t)n);
        long long *dh = nullptr;
        if (e == cudaSuccess) e = cudaMalloc((void **)&dh, sizeof(long long) * (size_t)nbins);
        if (e != cudaSuccess) return plq_fail(PLQ_ENOMEM, cudaGetErrorString(e));
        cudaMemsetAsync(cd->sizes, 0, sizeof(int32_t) * (size_t)n, c->stream);
        cudaMemsetAsync(dh, 0, sizeof(long long) * (size_t)nbins, c->stream);
        sizes_kernel<<<grid_stride_blocks(n), kThreads, 0, c->stream>>>(cd->parent, cd->sizes, n);
        size_hist_kernel<<<grid_stride_blocks(n), kThreads, 0, c->stream>>>(cd->parent, cd->sizes, n, dh, nbins);
        c->launches += 2;
        cudaMemcpyAsync(h.data(), dh, sizeof(long long) * (size_t)nbins, cudaMemcpyDeviceToHost, c->stream);
        e = cudaStreamSynchronize(c->stream);
        cudaFree(dh);
        if (e != cudaSuccess) return plq_fail(PLQ_ECUDA, cudaGetErrorString(e));
    }
    for (int i = 0; i < nbins; ++i) hist[i] = h[(size_t)i];
    return PLQ_OK;
}
