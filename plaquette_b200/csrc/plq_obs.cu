// plq_obs.cu -- exact integer primaries of a configuration, and the link
// layout conversion.
//
// The reference measures on the host after a read-back: Ising bond and spin
// sums (src/models/ising/mod.rs:67-117), Potts agreement and label counts
// (src/models/potts/mod.rs:125-271), gauge plaquette sum
// (src/models/gauge/mod.rs:99-124), all accumulated in integers.  Here one
// pass over the device-resident configuration produces the same integers:
// per-thread int64 partials, a warp-shuffle reduction, one 64-bit atomic per
// warp (per-block shared counters for the Potts label counts).
#include <cuda_runtime.h>

#include "../../include/plaquette.h"
#include "plq_device.cuh"
#include "plq_local.h"

namespace plq {

constexpr int kObsThreads = 256;

__device__ __forceinline__ long long warp_sum(long long v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    return v;
}

template <int D>
__global__ void __launch_bounds__(kObsThreads)
primaries_kernel(const uint8_t *state, Geom g, int model, int q, long long *out) {
    __shared__ int s_counts[64];
    if (model == PLQ_POTTS)
        for (int i = threadIdx.x; i < q; i += blockDim.x) s_counts[i] = 0;
    __syncthreads();
    long long acc0 = 0, acc1 = 0;
    const int64_t n = g.n_sites;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n;
         s += (int64_t)gridDim.x * blockDim.x) {
        int32_t x[D];
        uint32_t t = (uint32_t)s;
#pragma unroll
        for (int mu = 0; mu < D; ++mu) {
            uint32_t qq = fdiv(t, g.dm[mu], g.dl[mu]);
            x[mu] = (int32_t)(t - qq * (uint32_t)g.L[mu]);
            t = qq;
        }
        if (model == PLQ_GAUGE) {
            // plaquettes (s, mu, nu), mu < nu: U_mu(s) U_nu(s+mu) U_mu(s+nu) U_nu(s)
#pragma unroll
            for (int mu = 0; mu < D; ++mu) {
                int64_t s_mu = x[mu] + 1 < g.L[mu] ? s + g.stride[mu] : s - (int64_t)(g.L[mu] - 1) * g.stride[mu];
#pragma unroll
                for (int nu = mu + 1; nu < D; ++nu) {
                    int64_t s_nu = x[nu] + 1 < g.L[nu] ? s + g.stride[nu] : s - (int64_t)(g.L[nu] - 1) * g.stride[nu];
                    int b = state[mu * n + s] ^ state[nu * n + s_mu] ^ state[mu * n + s_nu] ^ state[nu * n + s];
                    acc0 += 1 - 2 * b;
                }
            }
        } else {
            int si = state[s];
            if (model == PLQ_ISING) acc1 += 1 - 2 * si;
            else atomicAdd(&s_counts[si], 1);
#pragma unroll
            for (int mu = 0; mu < D; ++mu) {
                int64_t s_mu = x[mu] + 1 < g.L[mu] ? s + g.stride[mu] : s - (int64_t)(g.L[mu] - 1) * g.stride[mu];
                int sj = state[s_mu];
                if (model == PLQ_ISING) acc0 += (1 - 2 * si) * (1 - 2 * sj);
                else acc0 += si == sj;
            }
        }
    }
    acc0 = warp_sum(acc0);
    acc1 = warp_sum(acc1);
    if ((threadIdx.x & 31) == 0) {
        if (acc0) atomicAdd((unsigned long long *)&out[0], (unsigned long long)acc0);
        if (model == PLQ_ISING && acc1) atomicAdd((unsigned long long *)&out[1], (unsigned long long)acc1);
    }
    if (model == PLQ_POTTS) {
        __syncthreads();
        for (int i = threadIdx.x; i < q; i += blockDim.x)
            if (s_counts[i]) atomicAdd((unsigned long long *)&out[1 + i], (unsigned long long)s_counts[i]);
    }
}

int primaries_count(int model, int q) {
    if (model == PLQ_ISING) return 2;
    if (model == PLQ_POTTS) return 1 + q;
    return 1;
}

cudaError_t launch_primaries(const uint8_t *state, const Geom &g, int model, int q, long long *out,
                             cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(long long) * primaries_count(model, q), stream);
    if (e != cudaSuccess) return e;
    int64_t blocks = (g.n_sites + kObsThreads - 1) / kObsThreads;
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
#define PLQ_CASE(DD)                                                                              \
    case DD:                                                                                      \
        primaries_kernel<DD><<<(unsigned)blocks, kObsThreads, 0, stream>>>(state, g, model, q, out); \
        break;
    switch (g.d) {
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

__global__ void links_to_planes_kernel(const uint8_t *in, uint8_t *out, int64_t n_sites, int d) {
    int64_t total = n_sites * d;
    for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < total;
         l += (int64_t)gridDim.x * blockDim.x) {
        int64_t site = l / d;
        int dir = (int)(l - site * d);
        out[dir * n_sites + site] = in[l];
    }
}

__global__ void planes_to_links_kernel(const uint8_t *in, uint8_t *out, int64_t n_sites, int d) {
    int64_t total = n_sites * d;
    for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < total;
         l += (int64_t)gridDim.x * blockDim.x) {
        int64_t site = l / d;
        int dir = (int)(l - site * d);
        out[l] = in[dir * n_sites + site];
    }
}

static unsigned grid_for(int64_t total) {
    int64_t b = (total + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    return (unsigned)(b < 1 ? 1 : b);
}

cudaError_t launch_links_to_planes(const uint8_t *in, uint8_t *out, int64_t n_sites, int d,
                                   cudaStream_t stream) {
    links_to_planes_kernel<<<grid_for(n_sites * d), 256, 0, stream>>>(in, out, n_sites, d);
    return cudaGetLastError();
}

cudaError_t launch_planes_to_links(const uint8_t *in, uint8_t *out, int64_t n_sites, int d,
                                   cudaStream_t stream) {
    planes_to_links_kernel<<<grid_for(n_sites * d), 256, 0, stream>>>(in, out, n_sites, d);
    return cudaGetLastError();
}

}  // namespace plq
