// plq_measure.h -- correlator pair sums, Polyakov loops and Wilson rectangles
// on the device (plq_measure.cu).
#pragma once
#include <cuda_runtime.h>

#include "plq_device.cuh"

namespace plq {

// Entries of axis_pair_sums: sum over mu of (L_mu / 2 + 1).
int64_t pair_sum_entries(const Geom &g);
// Differing pairs (s, s + r e_mu) for n_pairs (mu, r) pairs (device arrays) into out.
cudaError_t launch_pair_differ(const uint8_t *cfg, const Geom &g, const int32_t *pair_mu, const int32_t *pair_r,
                               int n_pairs, long long *out, cudaStream_t stream);
// Sum over the lines along dir of the line product (+1 / -1) into *out.
cudaError_t launch_polyakov(const uint8_t *links, const Geom &g, int dir, long long *out, cudaStream_t stream);
// Largest rectangle side the device table supports.
int wilson_max_supported();
// Counts of -1 rectangles per (r, t) into out[r * (max_side + 1) + t]; bits: n * d words of scratch.
cudaError_t launch_wilson(const uint8_t *links, const Geom &g, int max_side, uint32_t *bits, unsigned long long *out,
                          cudaStream_t stream);

}  // namespace plq
