// plq_scan.h -- the q = 2 stream-Metropolis colour pass for 2D/3D sites (plq_scan.cu).
#pragma once
#include <cuda_runtime.h>

#include "plq_device.cuh"

namespace plq {

struct ScanArgs {
    uint8_t *state;
    int64_t n_sites;
    int L0, L1, L2;
    uint32_t dm0, dm1;  // division by L0 and by L1 (Granlund-Montgomery, as Geom)
    int32_t dl0, dl1;
    int color;
    const uint64_t *metro53;  // decision table (q = 2 environment keys)
    int table_entries;
    const Affine *jump;
    u128 base, inc;
    Control *ctrl;
    unsigned long long *desc;
    int64_t n_chunks;
    uint32_t epoch;
    int pos_in;
};

bool scan_metro_eligible(int d, const int32_t *L);
// Chunks (thread blocks, look-back descriptors) of one pass.
int64_t scan_chunks(int64_t n_sites);
cudaError_t launch_scan_metro(const ScanArgs &a, int d, cudaStream_t stream);

}  // namespace plq
