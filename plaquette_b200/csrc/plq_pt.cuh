// plq_pt.cuh -- the parallel-tempering swap rule, one definition for the
// device (the ensemble kernel's swap phase) and the host (tempering across
// ranks, where every rank applies the same decisions to the energies they
// all-reduced).  The reference has no tempering.
//
// The pair at slots (k, k+1), members at betas b1, b2 with energies
// E = -J * (bond, agreement or plaquette sum), exchanges betas when
// delta = (b1 - b2)(E1 - E2) >= 0 or a uniform u < e^delta, u built from two
// 24-bit keyed hashes of (ladder seed, k, attempt).  Only IEEE basic
// operations, each rounded on its own (explicit _rn intrinsics on the
// device, -ffp-contract=off on the host), and an exp of its own: the
// decision is a pure function, bit-identical wherever it is evaluated.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#include "plq_rng.cuh"

namespace plq {

PLQ_HD double pt_mul(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
PLQ_HD double pt_add(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
PLQ_HD double pt_sub(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}

// e^x for x <= 0: x = n ln2 + r with n = floor(x/ln2 + 1/2) and ln2 split
// after Cody and Waite into a 32-significant-bit high part (n * high is
// exact) and a low part; e^r (|r| <= 0.347) by its Taylor polynomial to
// degree 14 in Horner form (truncation below 2^-60 relative); then times
// 2^n.  Below x = -708 the result is 0 (2^n would leave the normal range).
PLQ_HD double pt_exp(double x) {
    if (!(x > -708.0)) return 0.0;
    const double n = floor(pt_add(pt_mul(x, 1.4426950408889634), 0.5));
    const double r = pt_sub(pt_sub(x, pt_mul(n, 0.6931471803691238)), pt_mul(n, 1.9082149292705877e-10));
    double p = 1.1470745597729725e-11;  // 1/14!
    p = pt_add(pt_mul(p, r), 1.6059043836821613e-10);
    p = pt_add(pt_mul(p, r), 2.08767569878681e-09);
    p = pt_add(pt_mul(p, r), 2.505210838544172e-08);
    p = pt_add(pt_mul(p, r), 2.755731922398589e-07);
    p = pt_add(pt_mul(p, r), 2.7557319223985893e-06);
    p = pt_add(pt_mul(p, r), 2.48015873015873e-05);
    p = pt_add(pt_mul(p, r), 0.0001984126984126984);
    p = pt_add(pt_mul(p, r), 0.001388888888888889);
    p = pt_add(pt_mul(p, r), 0.008333333333333333);
    p = pt_add(pt_mul(p, r), 0.041666666666666664);
    p = pt_add(pt_mul(p, r), 0.16666666666666666);
    p = pt_add(pt_mul(p, r), 0.5);
    p = pt_add(pt_mul(p, r), 1.0);
    p = pt_add(pt_mul(p, r), 1.0);
    const uint64_t bits = (uint64_t)((int64_t)n + 1023) << 52;
    double scale;
#if defined(__CUDA_ARCH__)
    scale = __longlong_as_double((long long)bits);
#else
    std::memcpy(&scale, &bits, sizeof scale);
#endif
    return pt_mul(p, scale);
}

// Whether the pair at slot k exchanges betas on attempt `att`.
PLQ_HD bool pt_accept(double b1, double b2, long long energy1, long long energy2, double j1, double j2,
                      uint32_t seed32, uint32_t k, uint32_t att) {
    const double E1 = -pt_mul(j1, (double)energy1);
    const double E2 = -pt_mul(j2, (double)energy2);
    const double delta = pt_mul(pt_sub(b1, b2), pt_sub(E1, E2));
    const uint32_t h1 = keyed24(seed32 ^ 0x6a09e667u, k, att);
    const uint32_t h2 = keyed24(seed32 ^ 0xbb67ae85u, k, att);
    const double u = pt_mul(pt_add((double)h1, pt_mul((double)h2, 5.9604644775390625e-8)), 5.9604644775390625e-8);
    return delta >= 0.0 || u < pt_exp(delta);
}

}  // namespace plq
