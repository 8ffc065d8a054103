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

#include <algorithm>

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

// One site's (or, gauge, one site's plaquettes') contribution to the
// primaries: acc0 the bond / agreement / plaquette sum, acc1 the Ising spin
// sum; Potts labels counted in the block's shared counters.
template <int D>
__device__ __forceinline__ void site_primaries(const uint8_t *state, const Geom &g, int model, int64_t s,
                                               long long &acc0, long long &acc1, int *s_counts) {
    const int64_t n = g.n_sites;
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

// The block's partial sums into out (one 64-bit atomic per warp; the Potts
// label counters after a barrier).
__device__ __forceinline__ void flush_primaries(long long acc0, long long acc1, int model, int q, int *s_counts,
                                                long long *out) {
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

template <int D>
__global__ void __launch_bounds__(kObsThreads)
primaries_kernel(const uint8_t *state, Geom g, int model, int q, long long *out) {
    __shared__ int s_counts[64];
    if (model == PLQ_POTTS)
        for (int i = threadIdx.x; i < q; i += blockDim.x) s_counts[i] = 0;
    __syncthreads();
    long long acc0 = 0, acc1 = 0;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < g.n_sites;
         s += (int64_t)gridDim.x * blockDim.x)
        site_primaries<D>(state, g, model, s, acc0, acc1, s_counts);
    flush_primaries(acc0, acc1, model, q, s_counts, out);
}

// Many configurations' primaries in one launch: work item i is sites
// [chunk * kPrimChunk, (chunk + 1) * kPrimChunk) of task item_task[i]; a CTA
// takes items grid-stride.  The outputs must be zero before the launch.
template <int D>
__device__ __forceinline__ void primaries_item(const PrimTask &t, int64_t chunk, int *s_counts) {
    long long acc0 = 0, acc1 = 0;
    const int64_t end = min(t.g.n_sites, (chunk + 1) * kPrimChunk);
    for (int64_t s = chunk * kPrimChunk + threadIdx.x; s < end; s += blockDim.x)
        site_primaries<D>(t.state, t.g, t.model, s, acc0, acc1, s_counts);
    flush_primaries(acc0, acc1, t.model, t.q, s_counts, t.out);
}

__global__ void __launch_bounds__(kObsThreads)
primaries_multi_kernel(const PrimTask *tasks, const int32_t *item_task, const int32_t *item_chunk, int64_t n_items) {
    __shared__ int s_counts[64];
    for (int64_t i = blockIdx.x; i < n_items; i += gridDim.x) {
        const PrimTask &t = tasks[item_task[i]];
        if (t.model == PLQ_POTTS) {
            for (int k = threadIdx.x; k < t.q; k += blockDim.x) s_counts[k] = 0;
            __syncthreads();
        }
        switch (t.g.d) {
            case 1: primaries_item<1>(t, item_chunk[i], s_counts); break;
            case 2: primaries_item<2>(t, item_chunk[i], s_counts); break;
            case 3: primaries_item<3>(t, item_chunk[i], s_counts); break;
            case 4: primaries_item<4>(t, item_chunk[i], s_counts); break;
            default: break;
        }
        __syncthreads();  // the counters and the task are reused by the next item
    }
}

cudaError_t launch_primaries_multi(const PrimTask *tasks, const int32_t *item_task, const int32_t *item_chunk,
                                   int64_t n_items, int sm_count, cudaStream_t stream) {
    if (n_items <= 0) return cudaSuccess;
    const int64_t blocks = std::min<int64_t>(n_items, (int64_t)sm_count * 8);
    primaries_multi_kernel<<<(unsigned)blocks, kObsThreads, 0, stream>>>(tasks, item_task, item_chunk, n_items);
    return cudaGetLastError();
}

// Fast path for site models with extent 0 a multiple of 16 and q <= 8: a
// thread takes 16 consecutive sites as one 16-byte vector and counts with
// SWAR popcounts -- disagreeing forward bonds, ones (Ising spin sum), and
// per-label counts -- in 32-bit per-thread registers (Q = 0: Ising; Q = 2..8:
// Potts with q = Q; the label counts come from the state bits for Q <= 4).
template <int Q>
__device__ __forceinline__ uint32_t differ_bytes(uint32_t a, uint32_t b) {
    const uint32_t t = a ^ b;
    if (Q <= 2) return t;                                  // states 0/1: bit 0 only
    if (Q <= 4) return (t | (t >> 1)) & 0x01010101u;       // states < 4
    return (t | (t >> 1) | (t >> 2)) & 0x01010101u;        // states < 8
}

template <int D, int Q>
__global__ void __launch_bounds__(kObsThreads) primaries_runs_kernel(const uint8_t *state, Geom g, long long *out) {
    constexpr int NC = Q == 0 ? 1 : Q;  // Ising: ones; Potts: one count per label
    __shared__ unsigned long long s_acc[1 + NC];
    if (threadIdx.x < 1 + NC) s_acc[threadIdx.x] = 0;
    __syncthreads();
    const int64_t runs = g.n_sites / 16;
    uint32_t disagree = 0;
    uint32_t cnt[NC];
#pragma unroll
    for (int a = 0; a < NC; ++a) cnt[a] = 0;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < runs; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = r * 16;
        int32_t x[D];
        uint32_t t = (uint32_t)s;
#pragma unroll
        for (int mu = 0; mu < D; ++mu) {
            uint32_t qq = fdiv(t, g.dm[mu], g.dl[mu]);
            x[mu] = (int32_t)(t - qq * (uint32_t)g.L[mu]);
            t = qq;
        }
        const uint4 C = *reinterpret_cast<const uint4 *>(state + s);
        // +x: the byte after the run wraps to the row start at the end of a row
        const int64_t nx = x[0] + 16 < g.L[0] ? s + 16 : s + 16 - g.L[0];
        const uint32_t N0 = *reinterpret_cast<const uint32_t *>(state + nx);
        const uint32_t w[5] = {C.x, C.y, C.z, C.w, N0};
        uint32_t dif = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) dif += __popc(differ_bytes<Q>(w[k], __funnelshift_r(w[k], w[k + 1], 8)));
#pragma unroll
        for (int mu = 1; mu < D; ++mu) {
            const int64_t sp = x[mu] + 1 < g.L[mu] ? s + g.stride[mu] : s - (int64_t)(g.L[mu] - 1) * g.stride[mu];
            const uint4 F = *reinterpret_cast<const uint4 *>(state + sp);
            dif += __popc(differ_bytes<Q>(C.x, F.x)) + __popc(differ_bytes<Q>(C.y, F.y)) +
                   __popc(differ_bytes<Q>(C.z, F.z)) + __popc(differ_bytes<Q>(C.w, F.w));
        }
        disagree += dif;
        const uint32_t M = 0x01010101u;
        if (Q <= 2) {  // Ising ones, or Potts q = 2 label 1; label 0 is the rest
            const uint32_t ones = __popc(C.x) + __popc(C.y) + __popc(C.z) + __popc(C.w);
            cnt[NC - 1] += ones;
            if (Q == 2) cnt[0] += 16u - ones;
        } else if (Q <= 4) {
            const uint32_t b0 = __popc(C.x & M) + __popc(C.y & M) + __popc(C.z & M) + __popc(C.w & M);
            const uint32_t b1 = __popc((C.x >> 1) & M) + __popc((C.y >> 1) & M) + __popc((C.z >> 1) & M) +
                                __popc((C.w >> 1) & M);
            uint32_t c3 = 0;
            if (Q == 4)
                c3 = __popc(C.x & (C.x >> 1) & M) + __popc(C.y & (C.y >> 1) & M) + __popc(C.z & (C.z >> 1) & M) +
                     __popc(C.w & (C.w >> 1) & M);
            cnt[1] += b0 - c3;
            cnt[2] += b1 - c3;
            if (Q == 4) cnt[3 % NC] += c3;
            cnt[0] += 16u - b0 - b1 + c3;
        } else {
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                const uint32_t A = M * (uint32_t)a;
                cnt[a] += 16u - __popc(differ_bytes<Q>(C.x, A)) - __popc(differ_bytes<Q>(C.y, A)) -
                          __popc(differ_bytes<Q>(C.z, A)) - __popc(differ_bytes<Q>(C.w, A));
            }
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) disagree += __shfl_down_sync(0xffffffffu, disagree, off);
#pragma unroll
    for (int a = 0; a < NC; ++a)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) cnt[a] += __shfl_down_sync(0xffffffffu, cnt[a], off);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&s_acc[0], (unsigned long long)disagree);
#pragma unroll
        for (int a = 0; a < NC; ++a) atomicAdd(&s_acc[1 + a], (unsigned long long)cnt[a]);
    }
    __syncthreads();
    if (threadIdx.x < 1 + NC) atomicAdd((unsigned long long *)&out[threadIdx.x], s_acc[threadIdx.x]);
}

template <int D>
static void launch_runs(unsigned blocks, cudaStream_t stream, const uint8_t *state, const Geom &g, int model, int q,
                        long long *out) {
    if (model == PLQ_ISING) {
        primaries_runs_kernel<D, 0><<<blocks, kObsThreads, 0, stream>>>(state, g, out);
        return;
    }
    switch (q) {
        case 2: primaries_runs_kernel<D, 2><<<blocks, kObsThreads, 0, stream>>>(state, g, out); break;
        case 3: primaries_runs_kernel<D, 3><<<blocks, kObsThreads, 0, stream>>>(state, g, out); break;
        case 4: primaries_runs_kernel<D, 4><<<blocks, kObsThreads, 0, stream>>>(state, g, out); break;
        case 5: primaries_runs_kernel<D, 5><<<blocks, kObsThreads, 0, stream>>>(state, g, out); break;
        case 6: primaries_runs_kernel<D, 6><<<blocks, kObsThreads, 0, stream>>>(state, g, out); break;
        case 7: primaries_runs_kernel<D, 7><<<blocks, kObsThreads, 0, stream>>>(state, g, out); break;
        default: primaries_runs_kernel<D, 8><<<blocks, kObsThreads, 0, stream>>>(state, g, out); break;
    }
}

// Raw counts -> the reference's integers: Ising bond_sum = bonds - 2*disagree,
// spin_sum = n - 2*ones; Potts agree = bonds - disagree.
__global__ void primaries_fixup_kernel(long long *out, int model, long long n_sites, int d) {
    const long long bonds = n_sites * d;
    if (model == PLQ_ISING) {
        out[0] = bonds - 2 * out[0];
        out[1] = n_sites - 2 * out[1];
    } else {
        out[0] = bonds - out[0];
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
    if (model != PLQ_GAUGE && q <= 8 && (g.d == 2 || g.d == 3) && g.L[0] % 16 == 0) {
        const int64_t runs = g.n_sites / 16;
        int64_t blocks = (runs + kObsThreads - 1) / kObsThreads;
        if (blocks > 148 * 16) blocks = 148 * 16;
        if (blocks < 1) blocks = 1;
        if (g.d == 2)
            launch_runs<2>((unsigned)blocks, stream, state, g, model, q, out);
        else
            launch_runs<3>((unsigned)blocks, stream, state, g, model, q, out);
        primaries_fixup_kernel<<<1, 1, 0, stream>>>(out, model, (long long)g.n_sites, g.d);
        return cudaGetLastError();
    }
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
