// plq_measure.cu -- per-configuration measurements beyond the primaries, on
// the device-resident configuration, as exact integers:
//
//  * axis_pair_sums (src/models/mod.rs:44-61): for every axis mu and
//    displacement r = 0..L_mu/2, the sum over sites of pair(s_i, s_{i+r mu}),
//    Ising's product of signs (ising/mod.rs:84-95) or Potts's equality
//    (potts/mod.rs:218-234).  Both follow from the count of *differing* pairs
//    D: Ising n - 2D, Potts n - D.  D is counted four sites per 32-bit word
//    (SWAR nonzero-byte test on the XOR) when extent 0 is a multiple of 4.
//  * Z2Gauge::polyakov_loop (gauge/mod.rs:179-212): the sum over lines along
//    `dir` of the product of the line's links (XOR of the 0/1 states).
//  * Z2Gauge::wilson_rectangles (gauge/mod.rs:226-274): for every r, t <= max,
//    the sum over ordered planes (mu, nu) and base sites of the rectangle
//    product.  A rectangle walked +mu r, +nu t, -mu r, -nu t from x multiplies
//    line_mu(x, r) line_nu(x + r mu, t) line_mu(x + t nu, r) line_nu(x, t),
//    line_mu(x, k) the product of the k links from x along mu; one pass stores
//    those line parities as bit masks (bit k-1 for length k), a second
//    combines them, counting the -1 rectangles per (r, t) with warp ballots
//    into shared-memory counters.
// The host applies the reference's final divisions.
#include <cuda_runtime.h>

#include "../../include/plaquette.h"
#include "plq_device.cuh"
#include "plq_measure.h"

namespace plq {

constexpr int kMeasThreads = 256;

__device__ __forceinline__ uint32_t nonzero_bytes(uint32_t t) {
    return ((((t & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | t) & 0x80808080u);
}

__device__ __forceinline__ uint32_t coord_of(const Geom &g, uint32_t s, int mu) {
    // (s / stride_mu) % L_mu with the invariant-divisor divisions of Geom
    uint32_t t = s;
    for (int k = 0; k < mu; ++k) t = fdiv(t, g.dm[k], g.dl[k]);
    return t - fdiv(t, g.dm[mu], g.dl[mu]) * (uint32_t)g.L[mu];
}

// Differing pairs (s, s + r e_mu) for the pair index blockIdx.y -> (mu, r).
__global__ void __launch_bounds__(kMeasThreads)
pair_differ_kernel(const uint8_t *cfg, Geom g, const int32_t *pair_mu, const int32_t *pair_r, long long *out) {
    const int mu = pair_mu[blockIdx.y];
    const uint32_t r = (uint32_t)pair_r[blockIdx.y];
    const uint32_t n = (uint32_t)g.n_sites;
    const uint32_t L = (uint32_t)g.L[mu];
    const uint32_t st = (uint32_t)g.stride[mu];
    const uint32_t L0 = (uint32_t)g.L[0];
    const uint32_t stride = gridDim.x * blockDim.x;
    uint32_t count = 0;
    if (L0 % 4 == 0) {
        for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < n / 4; w += stride) {
            const uint32_t s = 4u * w;
            const uint32_t a = *reinterpret_cast<const uint32_t *>(cfg + s);
            uint32_t b;
            if (mu == 0) {
                const uint32_t row = fdiv(s, g.dm[0], g.dl[0]);
                const uint32_t rs = row * L0, x0 = s - rs;
                uint32_t xs = x0 + r;
                if (xs >= L0) xs -= L0;
                const uint32_t lo = xs & ~3u, hi = lo + 4u == L0 ? 0u : lo + 4u;
                const uint32_t w1 = *reinterpret_cast<const uint32_t *>(cfg + rs + lo);
                const uint32_t w2 = *reinterpret_cast<const uint32_t *>(cfg + rs + hi);
                b = __funnelshift_r(w1, w2, 8u * (xs & 3u));
            } else {
                const uint32_t c = coord_of(g, s, mu);
                const uint32_t t = c + r < L ? s + r * st : s - (L - r) * st;
                b = *reinterpret_cast<const uint32_t *>(cfg + t);
            }
            count += __popc(nonzero_bytes(a ^ b));
        }
    } else {
        for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) {
            const uint32_t c = coord_of(g, s, mu);
            const uint32_t t = c + r < L ? s + r * st : s - (L - r) * st;
            count += cfg[s] != cfg[t] ? 1u : 0u;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) count += __shfl_down_sync(0xffffffffu, count, off);
    if ((threadIdx.x & 31) == 0 && count) atomicAdd((unsigned long long *)&out[blockIdx.y], (unsigned long long)count);
}

// Product of the L_dir links of each line along dir, summed as +1 / -1.
__global__ void __launch_bounds__(kMeasThreads) polyakov_kernel(const uint8_t *links, Geom g, int dir, long long *out) {
    const uint32_t n = (uint32_t)g.n_sites;
    const uint32_t L = (uint32_t)g.L[dir], st = (uint32_t)g.stride[dir];
    const uint8_t *U = links + (size_t)dir * n;
    long long acc = 0;
    for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < n / L; l += gridDim.x * blockDim.x) {
        const uint32_t base = (l % st) + (l / st) * st * L;  // the line's site with coordinate 0 along dir
        uint32_t par = 0;
        for (uint32_t k = 0; k < L; ++k) par ^= U[base + k * st];
        acc += 1 - 2 * (long long)(par & 1u);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0 && acc) atomicAdd((unsigned long long *)out, (unsigned long long)acc);
}

// Line parities: bits[mu * n + x] bit k-1 = parity of the k links from x along mu.
__global__ void __launch_bounds__(kMeasThreads) line_bits_kernel(const uint8_t *links, Geom g, int max_len,
                                                                 uint32_t *bits) {
    const uint32_t n = (uint32_t)g.n_sites;
    const uint32_t total = n * (uint32_t)g.d;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int mu = (int)(i / n);
        const uint32_t x = i - (uint32_t)mu * n;
        const uint32_t L = (uint32_t)g.L[mu], st = (uint32_t)g.stride[mu];
        const uint8_t *U = links + (size_t)mu * n;
        uint32_t c = coord_of(g, x, mu), y = x, acc = 0, out = 0;
        for (int k = 0; k < max_len; ++k) {
            acc ^= U[y];
            out |= (acc & 1u) << k;
            if (++c == L) {
                c = 0;
                y -= (L - 1) * st;
            } else {
                y += st;
            }
        }
        bits[i] = out;
    }
}

constexpr int kWilsonMax = 32;

// Counts of -1 rectangles per (r, t) into out[r * (max + 1) + t].
__global__ void __launch_bounds__(kMeasThreads) wilson_kernel(const uint32_t *bits, Geom g, int max_side,
                                                              unsigned long long *out) {
    __shared__ unsigned int cnt[(kWilsonMax + 1) * (kWilsonMax + 1)];
    const int M = max_side + 1;
    for (int i = threadIdx.x; i < M * M; i += blockDim.x) cnt[i] = 0;
    __syncthreads();
    const uint32_t n = (uint32_t)g.n_sites;
    const int d = g.d;
    const int lane = threadIdx.x & 31;
    // every thread of a warp runs the same loop trips (ballots need the whole warp)
    const uint32_t rounds = (n + gridDim.x * blockDim.x - 1) / (gridDim.x * blockDim.x);
    for (uint32_t k = 0; k < rounds; ++k) {
        const uint32_t x = (k * gridDim.x + blockIdx.x) * blockDim.x + threadIdx.x;
        const bool valid = x < n;
        const uint32_t xv = valid ? x : 0;
        for (int mu = 0; mu < d; ++mu)
            for (int nu = 0; nu < d; ++nu) {
                if (mu == nu) continue;
                const uint32_t pm = bits[(size_t)mu * n + xv], pn = bits[(size_t)nu * n + xv];
                const uint32_t cm = coord_of(g, xv, mu), cn = coord_of(g, xv, nu);
                const uint32_t Lm = (uint32_t)g.L[mu], Ln = (uint32_t)g.L[nu];
                const uint32_t sm = (uint32_t)g.stride[mu], sn = (uint32_t)g.stride[nu];
                for (int r = 1; r <= max_side; ++r) {
                    const uint32_t xr = cm + r < Lm ? xv + r * sm : xv - (Lm - r) * sm;  // x + r mu
                    const uint32_t a = bits[(size_t)nu * n + xr];                       // line_nu(x + r mu, .)
                    for (int t = 1; t <= max_side; ++t) {
                        const uint32_t xt = cn + t < Ln ? xv + t * sn : xv - (Ln - t) * sn;  // x + t nu
                        const uint32_t c = bits[(size_t)mu * n + xt];                       // line_mu(x + t nu, .)
                        const uint32_t w = ((pm >> (r - 1)) ^ (a >> (t - 1)) ^ (c >> (r - 1)) ^ (pn >> (t - 1))) & 1u;
                        const unsigned neg = __ballot_sync(0xffffffffu, valid && w);
                        if (lane == 0 && neg) atomicAdd(&cnt[r * M + t], (unsigned)__popc(neg));
                    }
                }
            }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < M * M; i += blockDim.x)
        if (cnt[i]) atomicAdd(&out[i], (unsigned long long)cnt[i]);
}

static unsigned blocks_for(int64_t work) {
    int64_t b = (work + kMeasThreads - 1) / kMeasThreads;
    if (b > 148 * 8) b = 148 * 8;
    return (unsigned)(b < 1 ? 1 : b);
}

int64_t pair_sum_entries(const Geom &g) {
    int64_t e = 0;
    for (int mu = 0; mu < g.d; ++mu) e += g.L[mu] / 2 + 1;
    return e;
}

cudaError_t launch_pair_differ(const uint8_t *cfg, const Geom &g, const int32_t *pair_mu, const int32_t *pair_r,
                               int n_pairs, long long *out, cudaStream_t stream) {
    if (n_pairs == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(long long) * (size_t)n_pairs, stream);
    if (e != cudaSuccess) return e;
    const int64_t units = g.L[0] % 4 == 0 ? g.n_sites / 4 : g.n_sites;
    int64_t bx = (units + kMeasThreads - 1) / kMeasThreads;
    const int64_t want = (148 * 16 + n_pairs - 1) / n_pairs;  // about 16 CTAs per SM in all
    if (bx > want) bx = want;
    if (bx < 1) bx = 1;
    pair_differ_kernel<<<dim3((unsigned)bx, (unsigned)n_pairs), kMeasThreads, 0, stream>>>(cfg, g, pair_mu, pair_r,
                                                                                          out);
    return cudaGetLastError();
}

cudaError_t launch_polyakov(const uint8_t *links, const Geom &g, int dir, long long *out, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(long long), stream);
    if (e != cudaSuccess) return e;
    polyakov_kernel<<<blocks_for(g.n_sites / g.L[dir]), kMeasThreads, 0, stream>>>(links, g, dir, out);
    return cudaGetLastError();
}

int wilson_max_supported() { return kWilsonMax; }

cudaError_t launch_wilson(const uint8_t *links, const Geom &g, int max_side, uint32_t *bits, unsigned long long *out,
                          cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(unsigned long long) * (size_t)(max_side + 1) * (max_side + 1),
                                    stream);
    if (e != cudaSuccess) return e;
    line_bits_kernel<<<blocks_for(g.n_sites * g.d), kMeasThreads, 0, stream>>>(links, g, max_side, bits);
    wilson_kernel<<<blocks_for(g.n_sites), kMeasThreads, 0, stream>>>(bits, g, max_side, out);
    return cudaGetLastError();
}

}  // namespace plq
