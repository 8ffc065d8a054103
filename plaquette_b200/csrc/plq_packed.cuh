// plq_packed.cuh -- device helpers of the bit-packed row bodies (one bit per
// q = 2 variable, a row of them per 32- or 64-bit word): neighbour rows by
// rotation, the bit-sliced neighbour counter, and the decision of a row's
// variables of one parity from nibble keys (plq_ensemble.cu's packed members,
// plq_packed3d.cu's single lattices).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "plq_rng.cuh"

namespace plq {

template <class W>
__device__ __forceinline__ W row_xp(W w, uint32_t L0, W full) {  // bit x <- bit x+1
    return ((w >> 1) | (w << (L0 - 1))) & full;
}
template <class W>
__device__ __forceinline__ W row_xm(W w, uint32_t L0, W full) {  // bit x <- bit x-1
    return ((w << 1) | (w >> (L0 - 1))) & full;
}
// bit-sliced counter (c2 c1 c0) += v, per bit position (counts stay below 8)
template <class W>
__device__ __forceinline__ void count_add(W &c0, W &c1, W &c2, W v) {
    const W k0 = c0 & v;
    c0 ^= v;
    c2 |= c1 & k0;
    c1 ^= k0;
}
__device__ __forceinline__ int popc_w(uint32_t v) { return __popc(v); }
__device__ __forceinline__ int popc_w(uint64_t v) { return __popcll(v); }

// Decide the n = L0 / 2 variables of one row that a pass updates.  Cs, c0s,
// c1s, c2s: the row's state bits and the bits of each variable's count
// (c2 c1 c0 in binary: neighbours in state 1, or satisfied staples), all
// shifted so variable j of the pass sits at bit 2j.  Its table key is
// cur + 2 * count, a nibble: eight variables' keys are gathered into one word
// (pairs (cur, c0) and (c1, c2) interleaved at two-bit granularity, Hacker's
// Delight's outer perfect shuffle without its last stage), and the key times
// four is the byte offset of its entry in the shared-memory table tab, whose
// entries are at most 2^24 (the table's "always" sentinel clamped there, which
// every 24-bit draw is below).  The draw of variable j is the keyed stream's at
// index v0 + j * DV, composed as keyed24 does (mix = keyed_mix(sweep)).
// Returns the bits to flip, at 2j: Metropolis accepts when the draw is below
// the entry; heat bath sets the new state to (entry <= draw).
//
// A decision is k < e for k < 2^24 and e <= 2^24, so k - e lies in
// (-2^24, 2^24) and its top two bits are 11 exactly when k < e, 00 otherwise:
// a funnel shift moves them in below the decisions so far (variables taken
// from the last to the first, so variable i's pair lands at bits 2i, 2i + 1)
// and one mask keeps bit 2i.
__device__ __forceinline__ uint32_t table_entry(uint32_t e) { return e < (1u << 24) ? e : (1u << 24); }

// Eight (or, TAIL, the first m < 8) variables of a row from their key word x
// (nibble i: variable i's key): the flip or new-state bits at 2i.
template <int DV, bool HB, bool TAIL>
__device__ __forceinline__ uint32_t decide8(uint32_t x, int m, uint32_t vc, uint32_t seed32, uint32_t mix,
                                            const char *tb) {
    uint32_t o = 0;
#pragma unroll
    for (int i = 7; i >= 0; --i) {
        if (!TAIL || i < m) {
            const uint32_t key4 = i == 0 ? (x << 2) & 0x3Cu : (x >> (4 * i - 2)) & 0x3Cu;
            const uint32_t e = *reinterpret_cast<const uint32_t *>(tb + key4);
            const uint32_t k = lowbias32_tail(lowbias32_head(seed32 ^ (vc + (uint32_t)(i * DV))) ^ mix) >> 8;
            o = __funnelshift_l(k - e, o, 2);
        }
    }
    return HB ? ~o & (TAIL ? 0x5555u >> (16 - 2 * m) : 0x5555u) : o & 0x5555u;
}

// decide8 over eight (or, TAIL, the first m < 8) variables whose first rounds
// lowbias32_head(seed ^ index) are given (h1[i] for variable i): half a keyed
// draw's hashing per variable.
template <bool HB, bool TAIL = false>
__device__ __forceinline__ uint32_t decide8_h1(uint32_t x, const uint32_t (&h1)[8], uint32_t mix,
                                               const char *tb, int m = 8) {
    uint32_t o = 0;
#pragma unroll
    for (int i = 7; i >= 0; --i) {
        if (!TAIL || i < m) {
            const uint32_t key4 = i == 0 ? (x << 2) & 0x3Cu : (x >> (4 * i - 2)) & 0x3Cu;
            const uint32_t e = *reinterpret_cast<const uint32_t *>(tb + key4);
            const uint32_t k = lowbias32_tail(h1[i] ^ mix) >> 8;
            o = __funnelshift_l(k - e, o, 2);
        }
    }
    return HB ? ~o & (TAIL ? 0x5555u >> (16 - 2 * m) : 0x5555u) : o & 0x5555u;
}

// The key word of variables 8c .. 8c + 7: pairs (cur, c0) of P and (c1, c2)
// of Q interleaved at two-bit granularity.
template <class W>
__device__ __forceinline__ uint32_t key_word(W P, W Q, int c) {
    uint32_t x = __byte_perm((uint32_t)(P >> (16 * c)), (uint32_t)(Q >> (16 * c)), 0x5410);
    x = __byte_perm(x, 0, 0x3120);
    uint32_t t = (x ^ (x >> 4)) & 0x00F000F0u;
    x ^= t ^ (t << 4);
    t = (x ^ (x >> 2)) & 0x0C0C0C0Cu;
    x ^= t ^ (t << 2);
    return x;
}

template <class W, int DV, bool HB>
__device__ __forceinline__ W decide_row(W Cs, W c0s, W c1s, W c2s, int n, uint32_t v0, uint32_t seed32,
                                        uint32_t mix, const uint32_t *tab) {
    const W M = (W)0x5555555555555555ull;
    const W P = (Cs & M) | ((c0s << 1) & ~M);
    const W Q = (c1s & M) | ((c2s << 1) & ~M);
    const char *tb = reinterpret_cast<const char *>(tab);
    W out = 0;
    const int full = n >> 3;
#pragma unroll 1
    for (int c = 0; c < full; ++c)
        out |= (W)decide8<DV, HB, false>(key_word(P, Q, c), 8, v0 + (uint32_t)(8 * c * DV), seed32, mix, tb)
               << (16 * c);
    if (n & 7)
        out |= (W)decide8<DV, HB, true>(key_word(P, Q, full), n & 7, v0 + (uint32_t)(8 * full * DV), seed32,
                                        mix, tb)
               << (16 * full);
    if (HB) {  // new states -> flips, over the n variables
        const W valid = 2 * n >= (int)(8 * sizeof(W)) ? ~(W)0 : (((W)1 << (2 * n)) - 1);
        out ^= P & M & valid;
    }
    return out;
}

}  // namespace plq
