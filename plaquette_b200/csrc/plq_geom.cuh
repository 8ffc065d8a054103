// plq_geom.cuh -- periodic hypercubic geometry on the device (direction 0
// fastest, as src/lattice.rs:73-99 packs it).
#pragma once
#include <cstdint>

#include "plq_device.cuh"

namespace plq {

template <int D>
__device__ __forceinline__ void site_coords(const Geom &g, int64_t s, int32_t *x) {
    uint32_t t = (uint32_t)s;  // site indices are below 2^31
#pragma unroll
    for (int mu = 0; mu < D; ++mu) {
        uint32_t q = fdiv(t, g.dm[mu], g.dl[mu]);
        x[mu] = (int32_t)(t - q * (uint32_t)g.L[mu]);
        t = q;
    }
}

// The +mu / -mu neighbour of site s with coordinates x.
__device__ __forceinline__ int64_t nbr_plus(const Geom &g, int64_t s, const int32_t *x, int mu) {
    return x[mu] + 1 < g.L[mu] ? s + g.stride[mu] : s - (int64_t)(g.L[mu] - 1) * g.stride[mu];
}
__device__ __forceinline__ int64_t nbr_minus(const Geom &g, int64_t s, const int32_t *x, int mu) {
    return x[mu] > 0 ? s - g.stride[mu] : s + (int64_t)(g.L[mu] - 1) * g.stride[mu];
}

}  // namespace plq
