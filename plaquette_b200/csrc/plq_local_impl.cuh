// plq_local_impl.cuh -- the body of one colour-pass chunk, shared by the
// per-lattice pass kernels (plq_local.cu) and the batched ensemble kernel
// (plq_ensemble.cu).  See plq_local.cu for what a pass computes.
#pragma once
#include <cuda_runtime.h>

#include "../../include/plaquette.h"
#include "plq_device.cuh"

namespace plq {

constexpr int kThreads = 256;
constexpr int kRanksPerThread = 8;
constexpr int kChunk = kThreads * kRanksPerThread;
constexpr int kLookbackSpinLimit = 1 << 22;

// Look-back descriptor: [epoch:30 | status:2 | value:32].
constexpr unsigned long long kDescAgg = 1ull;
constexpr unsigned long long kDescPrefix = 2ull;

__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long make_desc(uint32_t epoch, unsigned long long st,
                                                        uint32_t value) {
    return ((unsigned long long)(epoch & 0x3FFFFFFFu) << 34) | (st << 32) | value;
}

template <int D>
__device__ __forceinline__ void coords_of(const Geom &g, int64_t s, int32_t *x) {
    uint32_t t = (uint32_t)s;
#pragma unroll
    for (int mu = 0; mu < D; ++mu) {
        uint32_t q = fdiv(t, g.dm[mu], g.dl[mu]);
        x[mu] = (int32_t)(t - q * (uint32_t)g.L[mu]);
        t = q;
    }
}

template <int D>
__device__ __forceinline__ int64_t step_plus(const Geom &g, int64_t s, const int32_t *x, int mu) {
    return x[mu] + 1 < g.L[mu] ? s + g.stride[mu] : s - (int64_t)(g.L[mu] - 1) * g.stride[mu];
}
template <int D>
__device__ __forceinline__ int64_t step_minus(const Geom &g, int64_t s, const int32_t *x, int mu) {
    return x[mu] > 0 ? s - g.stride[mu] : s + (int64_t)(g.L[mu] - 1) * g.stride[mu];
}

// Site of colour `color` with rank r among that colour in index order
// (extent 0 even): s = 2r + b, b fixed by the parity of the row.
template <int D>
__device__ __forceinline__ int64_t site_of_rank(const Geom &g, int64_t r, int color, int32_t *x) {
    const uint32_t even = 2u * (uint32_t)r;  // < 2^31: a site index
    const uint32_t row = fdiv(even, g.dm[0], g.dl[0]);
    int par = 0;
    uint32_t rr = row;
#pragma unroll
    for (int mu = 1; mu < D; ++mu) {
        uint32_t q = fdiv(rr, g.dm[mu], g.dl[mu]);
        int32_t c = (int32_t)(rr - q * (uint32_t)g.L[mu]);
        rr = q;
        x[mu] = c;
        par += c;
    }
    int b = (color ^ par) & 1;
    uint32_t s = even + (uint32_t)b;
    x[0] = (int32_t)(s - row * (uint32_t)g.L[0]);
    return (int64_t)s;
}

// Environment of a variable: key into the decision tables, plus the two
// neighbour counts a Potts Metropolis proposal needs (filled later).
struct Env {
    int64_t key;
    int cur;
    int prop;
    int cp, cc;
};

template <int D>
__device__ __forceinline__ void site_env(const LocalArgs &a, int64_t s, const int32_t *x, int cur,
                                         uint8_t *nb) {
#pragma unroll
    for (int mu = 0; mu < D; ++mu) {
        nb[2 * mu] = a.state[step_plus<D>(a.g, s, x, mu)];
        nb[2 * mu + 1] = a.state[step_minus<D>(a.g, s, x, mu)];
    }
    (void)cur;
}

template <int D>
__device__ __forceinline__ int link_staple_sum(const LocalArgs &a, int64_t s, const int32_t *x,
                                               int mu) {
    const int64_t n = a.g.n_sites;
    const uint8_t *U = a.state;
    int64_t s_mu = step_plus<D>(a.g, s, x, mu);
    int32_t xm[D];
#pragma unroll
    for (int k = 0; k < D; ++k) xm[k] = x[k];
    xm[mu] = x[mu] + 1 < a.g.L[mu] ? x[mu] + 1 : 0;
    int sum = 0;
#pragma unroll
    for (int nu = 0; nu < D; ++nu) {
        if (nu == mu) continue;
        int64_t s_nu = step_plus<D>(a.g, s, x, nu);
        int64_t s_mnu = step_minus<D>(a.g, s, x, nu);
        int64_t s_mu_mnu = step_minus<D>(a.g, s_mu, xm, nu);
        // forward plaquette: U_nu(x+mu) U_mu(x+nu) U_nu(x)
        int f = U[nu * n + s_mu] ^ U[mu * n + s_nu] ^ U[nu * n + s];
        // backward plaquette: U_nu(x+mu-nu) U_mu(x-nu) U_nu(x-nu)
        int bk = U[nu * n + s_mu_mnu] ^ U[mu * n + s_mnu] ^ U[nu * n + s_mnu];
        sum += (1 - 2 * f) + (1 - 2 * bk);
    }
    return sum;
}

// Heat-bath choice from cut points: number of cut points <= k.
template <class T>
__device__ __forceinline__ int hb_choose(const T *cut, int qm1, uint64_t k) {
    int chosen = 0;
    for (int s = 0; s < qm1; ++s) chosen += (uint64_t)cut[s] <= k ? 1 : 0;
    return chosen;
}

// One chunk of a colour pass: blockDim.x threads, each owning R consecutive
// ranks of the colour.  LINK selects link variables; LOOKBACK the
// stream-mode Metropolis (data-dependent draw positions).  Also the work item
// of the batched ensemble kernel (plq_ensemble.cu).
template <int D, bool LINK, bool LOOKBACK, int R>
__device__ __forceinline__ void local_chunk(const LocalArgs &a, int64_t chunk) {
    const int64_t half = a.g.n_sites / 2;
    const bool stream = a.jump != nullptr;
    const int q = a.q;
    const int64_t r0 = chunk * (int64_t)blockDim.x * R + (int64_t)threadIdx.x * R;
    constexpr int kRanksPerThread = R;

    int64_t vars[kRanksPerThread];
    uint8_t curs[kRanksPerThread];
    uint8_t props[kRanksPerThread];
    unsigned long long entry[kRanksPerThread];  // decision entry (metro) or key (hb)
    int need = 0;

#pragma unroll
    for (int i = 0; i < kRanksPerThread; ++i) {
        int64_t r = r0 + i;
        vars[i] = -1;
        entry[i] = 0;
        if (r >= half) continue;
        int32_t x[D];
        int64_t s = site_of_rank<D>(a.g, r, a.color, x);
        int64_t key;
        int cur;
        int prop = 0;
        int cp = 0, cc = 0;
        if (LINK) {
            int64_t v = (int64_t)a.dir * a.g.n_sites + s;
            cur = a.state[v];
            int S = link_staple_sum<D>(a, s, x, a.dir);
            key = cur + 2 * ((S + 2 * (D - 1)) / 2);
            vars[i] = s;  // site; the link is (s, dir)
            prop = 1 - cur;
        } else {
            cur = a.state[s];
            uint8_t nb[2 * D];
            site_env<D>(a, s, x, cur, nb);
            int64_t packed = 0;
#pragma unroll
            for (int k = 0; k < 2 * D; ++k) packed += a.pw[nb[k]];
            key = cur + (int64_t)q * packed;
            vars[i] = s;
            if (a.kernel == PLQ_METROPOLIS) {
                if (q == 2) {
                    prop = 1 - cur;
                } else {
                    // keyed proposal (metropolis.wgsl:45-55)
                    uint32_t k24 = keyed24(a.seed32 ^ kProposalKey, (uint32_t)s, a.sweep32);
                    float u = __fmul_rn((float)k24, 5.9604644775390625e-8f);
                    float scaled = __fmul_rn(u, (float)(q - 1));
                    uint32_t draw = __float2uint_rz(scaled);
                    if (draw >= (uint32_t)(q - 1)) draw = (uint32_t)(q - 2);
                    prop = (int)draw;
                    if (prop >= cur) prop += 1;
#pragma unroll
                    for (int k = 0; k < 2 * D; ++k) {
                        cp += nb[k] == prop;
                        cc += nb[k] == cur;
                    }
                    const int64_t B = 2 * D + 1;
                    key = (((int64_t)cur * q + prop) * B + cp) * B + cc;
                }
            }
        }
        curs[i] = (uint8_t)cur;
        props[i] = (uint8_t)prop;
        if (a.kernel == PLQ_METROPOLIS) {
            if (stream) {
                entry[i] = a.metro53[key];
                if (entry[i] != ~0ull) ++need;
            } else {
                entry[i] = a.metro24[key];
            }
        } else {
            entry[i] = (unsigned long long)key;
        }
    }

    // ---- draw positions on the PCG stream
    uint64_t my_pos = 0;
    bool ok = true;
    if (stream) {
        if (LOOKBACK) {
            // block exclusive scan of `need`
            __shared__ int warp_tot[kThreads / 32];
            __shared__ unsigned long long s_excl;
            __shared__ unsigned long long s_base;
            __shared__ int s_fail;
            int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
            int incl = need;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, incl, off);
                if (lane >= off) incl += y;
            }
            if (lane == 31) warp_tot[wid] = incl;
            if (threadIdx.x == 0) s_fail = 0;
            __syncthreads();
            int warp_excl = 0, block_total = 0;
#pragma unroll
            for (int w = 0; w < kThreads / 32; ++w) {
                int t = warp_tot[w];
                if (w < wid) warp_excl += t;
                block_total += t;
            }
            int thread_excl = warp_excl + incl - need;
            if (threadIdx.x == 0) {
                unsigned long long excl = 0;
                if (chunk == 0) {
                    atomicExch(&a.desc[0], make_desc(a.epoch, kDescPrefix, (uint32_t)block_total));
                } else {
                    atomicExch(&a.desc[chunk], make_desc(a.epoch, kDescAgg, (uint32_t)block_total));
                    int64_t j = chunk - 1;
                    int spins = 0;
                    while (j >= 0) {
                        unsigned long long v = ld_relaxed(&a.desc[j]);
                        uint32_t ep = (uint32_t)(v >> 34);
                        unsigned long long st = (v >> 32) & 3ull;
                        if (ep != (a.epoch & 0x3FFFFFFFu) || st == 0) {
                            if (++spins > kLookbackSpinLimit) {
                                s_fail = 1;
                                atomicOr(&a.ctrl->status, kStatusLookbackTimeout);
                                break;
                            }
                            __nanosleep(64);
                            continue;
                        }
                        excl += (uint32_t)v;
                        if (st == kDescPrefix) break;
                        --j;
                    }
                    if (!s_fail)
                        atomicExch(&a.desc[chunk],
                                   make_desc(a.epoch, kDescPrefix, (uint32_t)(excl + block_total)));
                }
                s_excl = excl;
                s_base = a.ctrl->pos[a.pos_in];
                if (chunk == a.n_chunks - 1 && !s_fail)
                    a.ctrl->pos[a.pos_in ^ 1] = s_base + excl + (unsigned long long)block_total;
            }
            __syncthreads();
            ok = s_fail == 0;
            my_pos = s_base + s_excl + (uint64_t)thread_excl;
        } else {
            my_pos = a.pass_offset + (uint64_t)r0;
        }
    }
    if (!ok) return;

    u128 st;
    if (stream) st = jump(a.jump, a.base, my_pos);

#pragma unroll
    for (int i = 0; i < kRanksPerThread; ++i) {
        if (vars[i] < 0) continue;
        int64_t s = vars[i];
        int64_t v = LINK ? (int64_t)a.dir * a.g.n_sites + s : s;
        uint32_t key_var = LINK ? (uint32_t)(s * D + a.dir) : (uint32_t)s;
        int out;
        if (a.kernel == PLQ_METROPOLIS) {
            bool accept;
            if (stream) {
                if (entry[i] == ~0ull) {
                    accept = true;
                } else {
                    uint64_t k = draw53(st);
                    st = pcg_step(st, a.inc);
                    accept = k < entry[i];
                }
            } else {
                uint32_t k = keyed24(a.seed32, key_var, a.sweep32);
                accept = entry[i] == 0xFFFFFFFFull || k < entry[i];
            }
            out = accept ? props[i] : curs[i];
        } else {
            int64_t key = (int64_t)entry[i];
            if (stream) {
                uint64_t k = draw53(st);
                st = pcg_step(st, a.inc);
                out = hb_choose(a.hb53 + key * (q - 1), q - 1, k);
            } else {
                uint32_t k = keyed24(a.seed32, key_var, a.sweep32);
                out = hb_choose(a.hb24 + key * (q - 1), q - 1, (uint64_t)k);
            }
        }
        a.state[v] = (uint8_t)out;
    }
}

}  // namespace plq
