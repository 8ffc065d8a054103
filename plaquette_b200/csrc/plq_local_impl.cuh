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

// Site of colour `color` with rank r among that colour in index order
// (extent 0 even): s = 2r + b, b fixed by the parity of the row.  Site
// indices are below 2^31 (chain validation), so all index math is 32-bit.
template <int D>
__device__ __forceinline__ uint32_t site_of_rank(const Geom &g, uint32_t r, int color, int32_t *x) {
    const uint32_t even = 2u * r;
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
    const int b = (color ^ par) & 1;
    const uint32_t s = even + (uint32_t)b;
    x[0] = (int32_t)(s - row * (uint32_t)g.L[0]);
    return s;
}

// Index offsets to the +mu and -mu neighbours of the site at x (periodic).
template <int D>
__device__ __forceinline__ void wrap_offsets(const Geom &g, const int32_t *x, int32_t *op, int32_t *om) {
#pragma unroll
    for (int mu = 0; mu < D; ++mu) {
        const int32_t st = (int32_t)g.stride[mu];
        const int32_t span = (g.L[mu] - 1) * st;
        op[mu] = x[mu] + 1 < g.L[mu] ? st : -span;
        om[mu] = x[mu] > 0 ? -st : span;
    }
}

// Staple sum of link (s, mu): over nu != mu, the forward plaquette
// U_nu(s+mu) U_mu(s+nu) U_nu(s) and the backward one U_nu(s+mu-nu) U_mu(s-nu)
// U_nu(s-nu), each +1 or -1 (Z2 states 0/1 multiply as XOR).  Links are
// stored as direction planes of n sites.
template <int D>
__device__ __forceinline__ int link_staple_sum(const uint8_t *U, uint32_t n, uint32_t s, const int32_t *op,
                                               const int32_t *om, int mu) {
    const uint8_t *Umu = U + (size_t)mu * n;
    const uint32_t s_mu = s + (uint32_t)op[mu];
    int unsat = 0;
#pragma unroll
    for (int nu = 0; nu < D; ++nu) {
        if (nu == mu) continue;
        const uint8_t *Unu = U + (size_t)nu * n;
        const uint32_t s_mnu = s + (uint32_t)om[nu];
        const int f = Unu[s_mu] ^ Umu[s + (uint32_t)op[nu]] ^ Unu[s];
        const int bk = Unu[s_mu + (uint32_t)om[nu]] ^ Umu[s_mnu] ^ Unu[s_mnu];
        unsat += f + bk;
    }
    return 2 * (D - 1) - 2 * unsat;  // sum of the 2(D-1) staple products, each +1 or -1
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
    const uint32_t n = (uint32_t)a.g.n_sites;
    const uint32_t half = n / 2;
    const bool stream = a.jump != nullptr;
    const int q = a.q;
    const uint32_t r0 = (uint32_t)(chunk * (int64_t)blockDim.x * R) + threadIdx.x * (uint32_t)R;
    constexpr int kRanksPerThread = R;
    uint8_t *plane = a.state + (LINK ? (size_t)a.dir * n : (size_t)0);  // the pass's variables

    int32_t vars[kRanksPerThread];
    uint8_t curs[kRanksPerThread];
    uint8_t props[kRanksPerThread];
    unsigned long long entry[kRanksPerThread];  // decision entry (metro) or key (hb)
    int need = 0;

#pragma unroll
    for (int i = 0; i < kRanksPerThread; ++i) {
        const uint32_t r = r0 + i;
        vars[i] = -1;
        entry[i] = 0;
        if (r >= half) continue;
        int32_t x[D], op[D], om[D];
        const uint32_t s = site_of_rank<D>(a.g, r, a.color, x);
        wrap_offsets<D>(a.g, x, op, om);
        int64_t key;
        int cur;
        int prop = 0;
        int cp = 0, cc = 0;
        if (LINK) {
            cur = plane[s];
            const int S = link_staple_sum<D>(a.state, n, s, op, om, a.dir);
            key = cur + 2 * ((S + 2 * (D - 1)) / 2);
            vars[i] = (int32_t)s;  // site; the link is (s, dir)
            prop = 1 - cur;
        } else {
            cur = a.state[s];
            uint8_t nb[2 * D];
#pragma unroll
            for (int mu = 0; mu < D; ++mu) {
                nb[2 * mu] = a.state[s + (uint32_t)op[mu]];
                nb[2 * mu + 1] = a.state[s + (uint32_t)om[mu]];
            }
            int64_t packed = 0;
#pragma unroll
            for (int k = 0; k < 2 * D; ++k) packed += a.pw[nb[k]];
            key = cur + (int64_t)q * packed;
            vars[i] = (int32_t)s;
            if (a.kernel == PLQ_METROPOLIS) {
                if (q == 2) {
                    prop = 1 - cur;
                } else {
                    // keyed proposal (metropolis.wgsl:45-55)
                    uint32_t k24 = keyed24(a.seed32 ^ kProposalKey, s, a.sweep32);
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
        const uint32_t s = (uint32_t)vars[i];
        const uint32_t key_var = LINK ? s * (uint32_t)D + (uint32_t)a.dir : s;
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
        plane[s] = (uint8_t)out;
    }
}

}  // namespace plq
