// plq_rng.cuh -- the two randomness streams, usable from host and device.
//
// STREAM: PCG64 = rand_pcg Lcg128Xsl64 (the reference CPU Rng, src/rng.rs:30-50).
// A 128-bit LCG state s_{n+1} = A*s_n + inc, output XSL-RR of the new state.
// Every position n of the stream is reachable directly: s_n = A^n s_0 + C_n,
// an affine map that composes, so the device jumps to a site's draw position
// instead of walking the stream.  Jumps use per-chain radix-256 tables of
// affine maps (8 digits x 256 entries).
//
// KEYED: lowbias32 / keyed_uniform of src/wgsl/rng.wgsl:34-52.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define PLQ_HD __host__ __device__ __forceinline__
#else
#define PLQ_HD inline
#endif

namespace plq {

struct u128 {
    uint64_t lo, hi;
};

PLQ_HD uint64_t mulhi64(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

PLQ_HD u128 add128(u128 a, u128 b) {
    u128 r;
    r.lo = a.lo + b.lo;
    r.hi = a.hi + b.hi + (r.lo < a.lo ? 1u : 0u);
    return r;
}

PLQ_HD u128 mul128(u128 a, u128 b) {
    u128 r;
    r.lo = a.lo * b.lo;
    r.hi = mulhi64(a.lo, b.lo) + a.lo * b.hi + a.hi * b.lo;
    return r;
}

// Multiplier of Lcg128Xsl64 (the PCG paper's 128-bit default).
PLQ_HD u128 pcg_mult() {
    u128 m;
    m.lo = 0x4385DF649FCCF645ULL;
    m.hi = 0x2360ED051FC65DA4ULL;
    return m;
}

// An affine map s -> m*s + p on Z/2^128.
struct Affine {
    u128 m, p;
};

PLQ_HD u128 apply(const Affine &f, u128 s) { return add128(mul128(f.m, s), f.p); }

// g after f: s -> g(f(s)).
PLQ_HD Affine compose(const Affine &f, const Affine &g) {
    Affine r;
    r.m = mul128(g.m, f.m);
    r.p = add128(mul128(g.m, f.p), g.p);
    return r;
}

PLQ_HD uint64_t rotr64(uint64_t x, unsigned r) {
    r &= 63u;
    return r ? (x >> r) | (x << (64u - r)) : x;
}

// XSL-RR output of a 128-bit state.
PLQ_HD uint64_t xsl_rr(u128 s) { return rotr64(s.hi ^ s.lo, (unsigned)(s.hi >> 58)); }

// One LCG step.
PLQ_HD u128 pcg_step(u128 s, u128 inc) { return add128(mul128(s, pcg_mult()), inc); }

// 53-bit integer behind rand's next_f64: the draw is (k * 2^-53).
PLQ_HD uint64_t draw53(u128 state_after_step) { return xsl_rr(state_after_step) >> 11; }

// Jump tables: 8 radix-256 digits; entry [digit][v] = the map for v*256^digit steps.
constexpr int kJumpDigits = 8;
constexpr int kJumpRadix = 256;

// The state reached after `n` steps from `s0` (n steps: position n draws
// next_u64 from state s_{n+1}; see stream_draw53 below).
PLQ_HD u128 jump(const Affine *table, u128 s0, uint64_t n) {
    u128 s = s0;
#pragma unroll 1
    for (int d = 0; d < kJumpDigits && n; ++d) {
        unsigned v = (unsigned)(n & 255u);
        if (v) s = apply(table[d * kJumpRadix + v], s);
        n >>= 8;
    }
    return s;
}

// ---------------------------------------------------------------- keyed
PLQ_HD uint32_t lowbias32(uint32_t x) {
    uint32_t v = x;
    v ^= v >> 16;
    v *= 0x7feb352du;
    v ^= v >> 15;
    v *= 0x846ca68bu;
    v ^= v >> 16;
    return v;
}

// The 24-bit integer k behind keyed_uniform: the float is k * 2^-24, exactly.
PLQ_HD uint32_t keyed24(uint32_t seed, uint32_t variable, uint32_t sweep) {
    uint32_t k = lowbias32(seed ^ variable);
    k = lowbias32(k ^ (sweep * 0x9e3779b9u));
    return k >> 8;
}

// Stream keys of the reference kernels (metropolis.wgsl:26,
// cluster_prelude.wgsl:29, cluster_relabel.wgsl:41-45).
constexpr uint32_t kProposalKey = 0x85ebca6bu;
constexpr uint32_t kBondKey = 0x27d4eb2fu;
constexpr uint32_t kRootSalt = 0x85ebca6bu;
constexpr uint32_t kSeedSalt = 0xc2b2ae35u;

}  // namespace plq
