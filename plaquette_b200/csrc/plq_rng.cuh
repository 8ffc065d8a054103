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

PLQ_HD u128 apply(const Affine &f, u128 s);

// g after f: s -> g(f(s)).
PLQ_HD Affine compose(const Affine &f, const Affine &g);

PLQ_HD uint64_t rotr64(uint64_t x, unsigned r) {
    r &= 63u;
    return r ? (x >> r) | (x << (64u - r)) : x;
}

#if defined(__CUDA_ARCH__)
// Device forms of the two per-draw operations, written on 32-bit limbs: the
// generic 64-bit expressions above compile to wide-multiply-high sequences and
// compare-based carries that load the integer ALU pipe.

// m*s + p (mod 2^128) as carry chains of 32-bit multiply-adds: the ten limb
// products s_i*m_j with i + j <= 3 (high halves where i + j <= 2), with p as
// the initial accumulator.
__device__ __forceinline__ u128 muladd128_limbs(u128 m, u128 s, u128 p) {
    const uint32_t s0 = (uint32_t)s.lo, s1 = (uint32_t)(s.lo >> 32), s2 = (uint32_t)s.hi,
                   s3 = (uint32_t)(s.hi >> 32);
    const uint32_t m0 = (uint32_t)m.lo, m1 = (uint32_t)(m.lo >> 32), m2 = (uint32_t)m.hi,
                   m3 = (uint32_t)(m.hi >> 32);
    const uint32_t i0 = (uint32_t)p.lo, i1 = (uint32_t)(p.lo >> 32), i2 = (uint32_t)p.hi,
                   i3 = (uint32_t)(p.hi >> 32);
    uint32_t r0, r1, r2, r3;
    asm("{\n\t"
        "mad.lo.cc.u32  %0, %4, %8, %12;\n\t"   // s0*m0 + p (cols 0..1), s0*m2 (cols 2..3)
        "madc.hi.cc.u32 %1, %4, %8, %13;\n\t"
        "madc.lo.cc.u32 %2, %4, %10, %14;\n\t"
        "madc.hi.u32    %3, %4, %10, %15;\n\t"
        "mad.lo.cc.u32  %1, %4, %9, %1;\n\t"    // s0*m1 (cols 1..2), s0*m3 (col 3)
        "madc.hi.cc.u32 %2, %4, %9, %2;\n\t"
        "madc.lo.u32    %3, %4, %11, %3;\n\t"
        "mad.lo.cc.u32  %1, %5, %8, %1;\n\t"    // s1*m0 (cols 1..2), s1*m2 (col 3)
        "madc.hi.cc.u32 %2, %5, %8, %2;\n\t"
        "madc.lo.u32    %3, %5, %10, %3;\n\t"
        "mad.lo.cc.u32  %2, %5, %9, %2;\n\t"    // s1*m1 (cols 2..3)
        "madc.hi.u32    %3, %5, %9, %3;\n\t"
        "mad.lo.cc.u32  %2, %6, %8, %2;\n\t"    // s2*m0 (cols 2..3)
        "madc.hi.u32    %3, %6, %8, %3;\n\t"
        "mad.lo.u32     %3, %6, %9, %3;\n\t"    // s2*m1 (col 3)
        "mad.lo.u32     %3, %7, %8, %3;\n\t"    // s3*m0 (col 3)
        "}"
        : "=&r"(r0), "=&r"(r1), "=&r"(r2), "=&r"(r3)
        : "r"(s0), "r"(s1), "r"(s2), "r"(s3), "r"(m0), "r"(m1), "r"(m2), "r"(m3), "r"(i0), "r"(i1), "r"(i2),
          "r"(i3));
    u128 r;
    r.lo = ((uint64_t)r1 << 32) | r0;
    r.hi = ((uint64_t)r3 << 32) | r2;
    return r;
}

// XSL-RR with the 64-bit rotation as two funnel shifts: rotating by r >= 32
// is a word swap followed by a rotation by r - 32.
__device__ __forceinline__ uint64_t xsl_rr_limbs(u128 s) {
    const uint32_t x0 = (uint32_t)s.lo ^ (uint32_t)s.hi;
    const uint32_t x1 = (uint32_t)(s.lo >> 32) ^ (uint32_t)(s.hi >> 32);
    const uint32_t r = (uint32_t)(s.hi >> 58);
    const bool swap = (r & 32u) != 0;
    const uint32_t a = swap ? x1 : x0, b = swap ? x0 : x1;
    const uint32_t o0 = __funnelshift_r(a, b, r), o1 = __funnelshift_r(b, a, r);
    return ((uint64_t)o1 << 32) | o0;
}
#endif

PLQ_HD u128 apply(const Affine &f, u128 s) {
#if defined(__CUDA_ARCH__)
    return muladd128_limbs(f.m, s, f.p);
#else
    return add128(mul128(f.m, s), f.p);
#endif
}

PLQ_HD Affine compose(const Affine &f, const Affine &g) {
    Affine r;
#if defined(__CUDA_ARCH__)
    const u128 zero{0, 0};
    r.m = muladd128_limbs(g.m, f.m, zero);
    r.p = muladd128_limbs(g.m, f.p, g.p);
#else
    r.m = mul128(g.m, f.m);
    r.p = add128(mul128(g.m, f.p), g.p);
#endif
    return r;
}

// XSL-RR output of a 128-bit state.
PLQ_HD uint64_t xsl_rr(u128 s) {
#if defined(__CUDA_ARCH__)
    return xsl_rr_limbs(s);
#else
    return rotr64(s.hi ^ s.lo, (unsigned)(s.hi >> 58));
#endif
}

// One LCG step.
PLQ_HD u128 pcg_step(u128 s, u128 inc) {
#if defined(__CUDA_ARCH__)
    return muladd128_limbs(pcg_mult(), s, inc);
#else
    return add128(mul128(s, pcg_mult()), inc);
#endif
}

// 53-bit integer behind rand's next_f64: the draw is (k * 2^-53).
PLQ_HD uint64_t draw53(u128 state_after_step) { return xsl_rr(state_after_step) >> 11; }

// Jump tables: 8 radix-256 digits; entry [digit][v] = the map for v*256^digit steps.
constexpr int kJumpDigits = 8;
constexpr int kJumpRadix = 256;

// The state reached after `n` steps from `s0` (the draw at stream position n
// is the output of the state one step further).
PLQ_HD u128 jump(const Affine *table, u128 s0, uint64_t n) {
    u128 s = s0;
#if defined(__CUDA_ARCH__)
#pragma unroll 1
#endif
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

// lowbias32 split at its xorshifts by 16: lowbias32(x) = y ^ (y >> 16) with
// y = lowbias32_head(x), and lowbias32(z) = lowbias32_tail(z ^ (z >> 16)).
PLQ_HD uint32_t lowbias32_head(uint32_t x) {
    uint32_t v = x;
    v ^= v >> 16;
    v *= 0x7feb352du;
    v ^= v >> 15;
    v *= 0x846ca68bu;
    return v;
}
PLQ_HD uint32_t lowbias32_tail(uint32_t v) {
    v *= 0x7feb352du;
    v ^= v >> 15;
    v *= 0x846ca68bu;
    v ^= v >> 16;
    return v;
}

// The sweep's term of a keyed draw, with the second round's opening xorshift
// applied: keyed_mix(t) = m ^ (m >> 16), m = t * 0x9e3779b9.
PLQ_HD uint32_t keyed_mix(uint32_t sweep) {
    const uint32_t m = sweep * 0x9e3779b9u;
    return m ^ (m >> 16);
}

// The 24-bit integer k behind keyed_uniform: the float is k * 2^-24, exactly.
// keyed_uniform is lowbias32(lowbias32(seed ^ variable) ^ m) >> 8.  The map
// x -> x ^ (x >> 16) is linear over xor and its own inverse on 32 bits, so the
// first round's closing xorshift and the second round's opening one cancel:
// lowbias32(lowbias32(a) ^ m) = lowbias32_tail(lowbias32_head(a) ^ m ^ (m >> 16)),
// four operations fewer per draw, the same bits.
PLQ_HD uint32_t keyed24(uint32_t seed, uint32_t variable, uint32_t sweep) {
    return lowbias32_tail(lowbias32_head(seed ^ variable) ^ keyed_mix(sweep)) >> 8;
}

// Stream keys of the reference kernels (metropolis.wgsl:26,
// cluster_prelude.wgsl:29, cluster_relabel.wgsl:41-45).
constexpr uint32_t kProposalKey = 0x85ebca6bu;
constexpr uint32_t kBondKey = 0x27d4eb2fu;
constexpr uint32_t kRootSalt = 0x85ebca6bu;
constexpr uint32_t kSeedSalt = 0xc2b2ae35u;

}  // namespace plq
