// plq_walk.cu -- Potts Metropolis at q >= 3 on the PCG stream: the sequential walk.
//
// The reference CPU step (src/updater.rs:77-96) first proposes a new state
// through propose (:659-668), which draws next_below(q - 1) -- one next_u64,
// and a second one when the first lands in the range sampler's rejection
// zone -- and then draws next_f64 only for an uphill move.  How many draws a
// variable consumes therefore depends on the value of its own first draw, so
// where a variable's draws sit in the stream depends on every earlier draw
// of the pass: the colour pass is one sequential walk of the stream, which a
// prefix scan cannot split (the stream-Metropolis passes of the other models
// can be scanned because their draw count is fixed before any draw is made).
//
// This kernel runs that walk on one warp.  For each group of 32 colour ranks
// the lanes gather, in parallel, each variable's site, state, neighbour
// states and the count of neighbours equal to its state; lane 0 then walks
// the group draw by draw with the LCG, exactly as the CPU does, and the
// lanes store the new states.  The pass reads its start position from the
// chain's control block and writes its end position back (the convention of
// the look-back passes), so positions stay on the device.  It is exact, and
// as fast as one thread: the keyed stream, whose draws are order-free, is the
// parallel path for Potts Metropolis.
#include <cuda_runtime.h>

#include "../../include/plaquette.h"
#include "plq_device.cuh"
#include "plq_local.h"
#include "plq_local_impl.cuh"

namespace plq {

namespace {

constexpr int kWalkLanes = 32;

template <int D>
__global__ void __launch_bounds__(kWalkLanes) potts_metro_walk_kernel(const LocalArgs a) {
    const int lane = threadIdx.x;
    const uint32_t half = (uint32_t)(a.g.n_sites / 2);
    const int q = a.q;
    const uint32_t range = (uint32_t)(q - 1);  // next_below(q - 1)
    const int B = 2 * D + 1;
    __shared__ uint32_t s_site[kWalkLanes];
    __shared__ uint8_t s_cur[kWalkLanes], s_cc[kWalkLanes], s_new[kWalkLanes];
    __shared__ uint8_t s_nb[kWalkLanes][2 * D];

    unsigned long long pos = 0;  // lane 0: draws consumed so far (relative to the chain's base)
    u128 st{0, 0};               // lane 0: the state whose output is the next draw
    if (lane == 0) {
        pos = a.ctrl->pos[a.pos_in];
        st = jump(a.jump, a.base, pos);
    }
    for (uint32_t r0 = 0; r0 < half; r0 += kWalkLanes) {
        const uint32_t r = r0 + (uint32_t)lane;
        if (r < half) {
            int32_t x[D], op[D], om[D];
            const uint32_t s = site_of_rank<D>(a.g, r, a.color, x);
            wrap_offsets<D>(a.g, x, op, om);
            const int cur = a.state[s];
            int cc = 0;
#pragma unroll
            for (int mu = 0; mu < D; ++mu) {
                const uint8_t up = a.state[s + (uint32_t)op[mu]], dn = a.state[s + (uint32_t)om[mu]];
                s_nb[lane][2 * mu] = up;
                s_nb[lane][2 * mu + 1] = dn;
                cc += (up == cur) + (dn == cur);
            }
            s_site[lane] = s;
            s_cur[lane] = (uint8_t)cur;
            s_cc[lane] = (uint8_t)cc;
        }
        __syncwarp();
        if (lane == 0) {
            const int n = half - r0 < (uint32_t)kWalkLanes ? (int)(half - r0) : kWalkLanes;
            for (int i = 0; i < n; ++i) {
                const int cur = s_cur[i];
                // propose: next_below(q - 1), rand's widening multiply on the low 32 bits
                const uint32_t x = (uint32_t)xsl_rr(st);
                st = pcg_step(st, a.inc);
                ++pos;
                const uint64_t m = (uint64_t)x * range;
                uint32_t draw = (uint32_t)(m >> 32);
                const uint32_t lo = (uint32_t)m;
                if (lo > 0u - range) {  // the rejection zone: one more draw settles the rounding
                    const uint32_t x2 = (uint32_t)xsl_rr(st);
                    st = pcg_step(st, a.inc);
                    ++pos;
                    const uint32_t new_hi = (uint32_t)(((uint64_t)x2 * range) >> 32);
                    if ((uint64_t)lo + new_hi > 0xFFFFFFFFull) draw += 1u;
                }
                const int prop = (int)draw + ((int)draw >= cur ? 1 : 0);
                int cp = 0;
#pragma unroll
                for (int k = 0; k < 2 * D; ++k) cp += s_nb[i][k] == prop;
                const int64_t key = (((int64_t)cur * q + prop) * B + cp) * B + s_cc[i];
                const uint64_t cut = a.metro53[key];
                bool accept = true;
                if (cut != ~0ull) {  // uphill: next_f64 < exp(-beta dE)
                    const uint64_t k = xsl_rr(st) >> 11;
                    st = pcg_step(st, a.inc);
                    ++pos;
                    accept = k < cut;
                }
                s_new[i] = (uint8_t)(accept ? prop : cur);
            }
        }
        __syncwarp();
        if (r < half) a.state[s_site[lane]] = s_new[lane];
        __syncwarp();
    }
    if (lane == 0) a.ctrl->pos[1 - a.pos_in] = pos;
}

}  // namespace

cudaError_t launch_potts_metro_walk(const LocalArgs &a, cudaStream_t stream) {
#define PLQ_CASE(DD)                                                           \
    case DD:                                                                   \
        potts_metro_walk_kernel<DD><<<1, kWalkLanes, 0, stream>>>(a);          \
        break;
    switch (a.g.d) {
        PLQ_CASE(1)
        PLQ_CASE(2)
        PLQ_CASE(3)
        PLQ_CASE(4)
        PLQ_CASE(5)
        PLQ_CASE(6)
        PLQ_CASE(7)
        PLQ_CASE(8)
        default:
            return cudaErrorInvalidValue;
    }
#undef PLQ_CASE
    return cudaGetLastError();
}

}  // namespace plq
