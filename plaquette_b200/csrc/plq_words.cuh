// plq_words.cuh -- colour passes four sites at a time, for lattices whose
// extent 0 is a multiple of 4 (the generic body of plq_local_impl.cuh does one
// variable per rank).  Same variables, same draws, same results; only the
// work per variable changes.
//
// A thread owns R consecutive 4-site words of the pass's plane (the state for
// sites, the direction-mu plane for links).  The neighbour words of a word sit
// at row-aligned offsets (directions >= 1) or are the word's row neighbours
// shifted by one byte (direction 0, funnel shifts with the row wrapping), so
// the table keys of all four sites come out of a few 32-bit SWAR additions
// (no byte ever carries), and the two sites of the pass's colour (bytes b and
// b+2, b the row's parity) draw and decide as in the generic body:
//
//  * sites, q <= 3: key = cur + q * sum of g(neighbour), g(0)=0, g(1)=1,
//    g(2)=2d+1 (the packing weights of the generic key); q = 4 (heat bath):
//    the same key in 16-bit lanes holding just the two colour sites;
//  * Z2 links: key = cur + 4(d-1) - 2 * (number of staples with product -1),
//    the generic cur + 2 * ((S + 2(d-1)) / 2) for the staple sum S.
//
// Draws: keyed by variable (order-free), or the PCG stream heat bath, where
// the colour rank of word w's two sites is 2w and 2w+1 (one jump per thread,
// then one LCG step per site).
#pragma once
#include <cuda_runtime.h>

#include "../../include/plaquette.h"
#include "plq_device.cuh"

namespace plq {

constexpr int kWordThreads = 256;
constexpr int kWordsPerThread = 4;

// The 4-byte word at site index `idx`.  Index arithmetic is modulo 2^32
// (offsets to earlier rows or words are stored as wrapped unsigned values), so
// every index is formed as a uint32_t before it meets the pointer.
__device__ __forceinline__ uint32_t ld_word(const uint8_t *p, uint32_t idx) {
    return *reinterpret_cast<const uint32_t *>(p + (size_t)idx);
}

// The word of sites displaced by dx in {-1, 0, +1} along x from the word at
// `base` (a word of the row starting at `base - x0`).
__device__ __forceinline__ uint32_t word_dx(const uint8_t *p, uint32_t base, int dx, uint32_t left,
                                            uint32_t right) {
    const uint32_t w = ld_word(p, base);
    if (dx == 0) return w;
    if (dx > 0) return __funnelshift_r(w, ld_word(p, base + right), 8);
    return __funnelshift_l(ld_word(p, base + left), w, 8);
}

struct WordPos {
    uint32_t s;       // first site of the word
    uint32_t x0;      // its coordinate along direction 0
    int32_t op[8], om[8];  // row-aligned offsets to the +mu / -mu rows (mu >= 1)
    uint32_t left, right;  // offsets to the previous / next word of the row (wrapping)
    int b;            // byte of the first colour site
};

template <int D>
__device__ __forceinline__ WordPos word_pos(const LocalArgs &a, uint32_t w) {
    WordPos P;
    const Geom &g = a.g;
    P.s = 4u * w;
    const uint32_t row = fdiv(P.s, g.dm[0], g.dl[0]);
    const uint32_t x0 = P.s - row * (uint32_t)g.L[0];
    const uint32_t L0 = (uint32_t)g.L[0];
    P.x0 = x0;
    P.left = x0 == 0 ? L0 - 4u : (uint32_t)-4;
    P.right = x0 + 4u == L0 ? (uint32_t)(4 - (int)L0) : 4u;
    int par = 0;
    uint32_t rr = row;
#pragma unroll
    for (int mu = 1; mu < D; ++mu) {
        const uint32_t q = fdiv(rr, g.dm[mu], g.dl[mu]);
        const int32_t c = (int32_t)(rr - q * (uint32_t)g.L[mu]);
        rr = q;
        par += c;
        const int32_t st = (int32_t)g.stride[mu];
        const int32_t span = (g.L[mu] - 1) * st;
        P.op[mu] = c + 1 < g.L[mu] ? st : -span;
        P.om[mu] = c > 0 ? -st : span;
    }
    P.b = (a.color ^ par) & 1;
    return P;
}

// The position of word w + 1 from that of word w: within a row only the site,
// x0 and the row-wrap offsets move (the offsets to other rows and the colour's
// byte do not); at a row's end everything is recomputed.
template <int D>
__device__ __forceinline__ void word_pos_next(const LocalArgs &a, uint32_t w_next, WordPos &P) {
    const uint32_t L0 = (uint32_t)a.g.L[0];
    if (P.x0 + 4u < L0) {
        P.s += 4u;
        P.x0 += 4u;
        P.left = (uint32_t)-4;
        P.right = P.x0 + 4u == L0 ? (uint32_t)(4 - (int)L0) : 4u;
    } else {
        P = word_pos<D>(a, w_next);
    }
}

// Decision of one colour site from its key; `k` is the draw (53-bit stream or
// 24-bit keyed), cut tables as the generic body reads them.
template <int Q, bool STREAM>
__device__ __forceinline__ uint32_t word_decide(const LocalArgs &a, uint32_t key, uint32_t cur, uint64_t k) {
    if (a.kernel == PLQ_METROPOLIS) {  // keyed, q = 2 (eligibility)
        const uint32_t e = a.metro24[key];
        const bool accept = e == 0xFFFFFFFFu || (uint32_t)k < e;
        return accept ? 1u - cur : cur;
    }
    uint32_t chosen = 0;
    if (STREAM) {
        const uint64_t *cut = a.hb53 + (size_t)key * (Q - 1);
#pragma unroll
        for (int j = 0; j < Q - 1; ++j) chosen += cut[j] <= k ? 1u : 0u;
    } else {
        const uint32_t *cut = a.hb24 + (size_t)key * (Q - 1);
#pragma unroll
        for (int j = 0; j < Q - 1; ++j) chosen += cut[j] <= (uint32_t)k ? 1u : 0u;
    }
    return chosen;
}

// Updates the two colour sites (bytes b, b+2) of word C with keys K.
// `var0` is the keyed variable index of site byte 0 (sites: the site; links:
// site * d + mu, so consecutive sites step by `vstep`).
template <int Q, bool STREAM>
__device__ __forceinline__ uint32_t word_update(const LocalArgs &a, uint32_t C, uint32_t K, int b, uint32_t var0,
                                                uint32_t vstep, u128 &st) {
    const uint32_t sh = 8u * (uint32_t)b;
    const uint32_t Cs = C >> sh, Ks = K >> sh;
    uint32_t delta = 0;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const uint32_t key = (Ks >> (16 * i)) & 0xFFu;
        const uint32_t cur = (Cs >> (16 * i)) & 0xFFu;
        uint64_t k;
        if (STREAM) {
            k = draw53(st);
            st = pcg_step(st, a.inc);
        } else {
            k = keyed24(a.seed32, var0 + vstep * (uint32_t)(b + 2 * i), a.sweep32);
        }
        delta |= (word_decide<Q, STREAM>(a, key, cur, k) ^ cur) << (16 * i);
    }
    return C ^ (delta << sh);
}

// Sites (Ising, Potts q <= 3, Potts q = 4 heat bath): one chunk of a colour pass, R words per thread.
template <int D, int Q, bool STREAM>
__device__ __forceinline__ void site_words_chunk(const LocalArgs &a, int64_t chunk, int R) {
    const uint32_t n_words = (uint32_t)(a.g.n_sites / 4);
    const uint32_t w0 = (uint32_t)(chunk * (int64_t)blockDim.x * R) + threadIdx.x * (uint32_t)R;
    if (w0 >= n_words) return;
    u128 st{0, 0};
    if (STREAM) st = jump(a.jump, a.base, a.pass_offset + 2ull * w0);
    const uint8_t *S = a.state;
    const uint32_t M1 = 0x01010101u;
    const uint32_t P2 = 2u * D + 1u;  // g(2)
    WordPos P = word_pos<D>(a, w0);
#pragma unroll 1
    for (int i = 0; i < R; ++i) {
        const uint32_t w = w0 + i;
        if (w >= n_words) break;
        if (i > 0) word_pos_next<D>(a, w, P);
        const uint32_t C = ld_word(S, P.s);
        uint32_t nb[2 * D];
        nb[0] = word_dx(S, P.s, +1, P.left, P.right);
        nb[1] = word_dx(S, P.s, -1, P.left, P.right);
#pragma unroll
        for (int mu = 1; mu < D; ++mu) {
            nb[2 * mu] = ld_word(S, P.s + (uint32_t)P.op[mu]);
            nb[2 * mu + 1] = ld_word(S, P.s + (uint32_t)P.om[mu]);
        }
        if (Q == 4) {
            // keys reach 4 + 4 * 2d * (2d+1)^2: two colour sites per word in 16-bit lanes
            // (bytes b and b+2 of each word); g(s) = pw[s] from the two state bits:
            // g = b0 + P b1 + (P^2 - 1 - P) b0 b1 with P = 2d + 1.
            const uint32_t sh = 8u * (uint32_t)P.b;
            const uint32_t LM = 0x00FF00FFu, L1 = 0x00010001u;
            uint32_t sum = 0;
#pragma unroll
            for (int k = 0; k < 2 * D; ++k) {
                const uint32_t x = (nb[k] >> sh) & LM;
                const uint32_t b0 = x & L1, b1 = (x >> 1) & L1;
                sum += b0 + P2 * b1 + (P2 * P2 - 1u - P2) * (b0 & b1);
            }
            const uint32_t Cl = (C >> sh) & LM;
            const uint32_t K16 = Cl + 4u * sum;
            uint32_t delta = 0;
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const uint32_t key = (K16 >> (16 * i)) & 0xFFFFu;
                const uint32_t cur = (Cl >> (16 * i)) & 0xFFu;
                uint64_t k;
                if (STREAM) {
                    k = draw53(st);
                    st = pcg_step(st, a.inc);
                } else {
                    k = keyed24(a.seed32, P.s + (uint32_t)(P.b + 2 * i), a.sweep32);
                }
                delta |= (word_decide<4, STREAM>(a, key, cur, k) ^ cur) << (16 * i);
            }
            *reinterpret_cast<uint32_t *>(a.state + (size_t)P.s) = C ^ (delta << sh);
            continue;
        }
        uint32_t raw = 0;
#pragma unroll
        for (int k = 0; k < 2 * D; ++k) raw += nb[k];
        uint32_t K;
        if (Q == 3) {
            uint32_t hi2 = 0;
#pragma unroll
            for (int k = 0; k < 2 * D; ++k) hi2 += nb[k] & (2u * M1);
            const uint32_t cnt2 = hi2 >> 1;  // state-2 neighbours per byte (each byte of hi2 is even)
            K = C + 3u * raw + 3u * (P2 - 2u) * cnt2;
        } else {
            K = C + (uint32_t)Q * raw;
        }
        const uint32_t out = word_update<Q, STREAM>(a, C, K, P.b, P.s, 1u, st);
        *reinterpret_cast<uint32_t *>(a.state + (size_t)P.s) = out;
    }
}

// Z2 links of direction a.dir: one chunk of a (direction, parity) pass, R words per thread.
template <int D, bool STREAM>
__device__ __forceinline__ void link_words_chunk(const LocalArgs &a, int64_t chunk, int R) {
    const uint32_t n = (uint32_t)a.g.n_sites;
    const uint32_t n_words = n / 4;
    const uint32_t w0 = (uint32_t)(chunk * (int64_t)blockDim.x * R) + threadIdx.x * (uint32_t)R;
    if (w0 >= n_words) return;
    const int mu = a.dir;
    u128 st{0, 0};
    if (STREAM) st = jump(a.jump, a.base, a.pass_offset + 2ull * w0);
    const uint8_t *Umu = a.state + (size_t)mu * n;
    WordPos P = word_pos<D>(a, w0);
#pragma unroll 1
    for (int i = 0; i < R; ++i) {
        const uint32_t w = w0 + i;
        if (w >= n_words) break;
        if (i > 0) word_pos_next<D>(a, w, P);
        // displacement of +mu: along x a byte shift, else a row offset
        const int dxm = mu == 0 ? 1 : 0;
        // P.op[mu] by compile-time indices: a runtime index would put P in local memory
        uint32_t om_mu = 0;
#pragma unroll
        for (int k = 1; k < D; ++k)
            if (k == mu) om_mu = (uint32_t)P.op[k];
        uint32_t unsat = 0;
#pragma unroll
        for (int nu = 0; nu < D; ++nu) {
            if (nu == mu) continue;
            const uint8_t *Unu = a.state + (size_t)nu * n;
            const int dxn = nu == 0 ? 1 : 0;
            const uint32_t opn = nu == 0 ? 0u : (uint32_t)P.op[nu];
            const uint32_t omn = nu == 0 ? 0u : (uint32_t)P.om[nu];
            // forward: U_nu(s+mu) U_mu(s+nu) U_nu(s)
            const uint32_t f = word_dx(Unu, P.s + om_mu, dxm, P.left, P.right) ^
                               word_dx(Umu, P.s + opn, dxn, P.left, P.right) ^
                               ld_word(Unu, P.s);
            // backward: U_nu(s+mu-nu) U_mu(s-nu) U_nu(s-nu)
            const uint32_t bk = word_dx(Unu, P.s + om_mu + omn, dxm - dxn, P.left, P.right) ^
                                word_dx(Umu, P.s + omn, -dxn, P.left, P.right) ^
                                word_dx(Unu, P.s + omn, -dxn, P.left, P.right);
            unsat += f + bk;
        }
        const uint32_t C = ld_word(Umu, P.s);
        const uint32_t K = C + (uint32_t)(4 * (D - 1)) * 0x01010101u - 2u * unsat;
        const uint32_t out = word_update<2, STREAM>(a, C, K, P.b, P.s * (uint32_t)D + (uint32_t)mu, (uint32_t)D, st);
        *reinterpret_cast<uint32_t *>(a.state + (size_t)mu * n + P.s) = out;
    }
}

// Whether a member's passes can run four sites at a time.
__host__ __device__ inline bool words_eligible(int model, int q, int d, const int32_t *L, int updater, int rng) {
    if (d < 1 || d > 4 || L[0] % 4 != 0) return false;
    if (updater == PLQ_METROPOLIS && !(rng == PLQ_RNG_KEYED && q == 2)) return false;
    if (updater != PLQ_METROPOLIS && updater != PLQ_HEATBATH) return false;
    if (model == PLQ_GAUGE) return d >= 2;
    return q == 2 || q == 3 || (q == 4 && updater == PLQ_HEATBATH);
}

}  // namespace plq
