// plq_fused.h -- the fused two-colour 3D site sweep (plq_fused.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "plq_device.cuh"

namespace plq {

struct FusedArgs {
    const uint8_t *src;
    uint8_t *dst;
    int L0, L1, L2, tz;
    int ty;              // rows per tile (set by the launcher)
    const void *table;   // decision table in global memory (copied to smem)
    int table_words;     // its size in 32-bit words
    uint32_t seed32, sweep32;
    const Affine *jump;  // PCG stream (null on the keyed stream)
    u128 base, inc;
    uint64_t off0, off1; // stream positions of rank 0 of colours 0 and 1
    Affine plane;        // stream jump by one z-plane of one colour (L0*L1/2 draws)
    unsigned int *status;  // chain status word (copy wait limit)
    int wait_limit;        // polls of a plane's barrier before the launch gives up
    int stall;             // test only: plane zfirst + 4 of every tile is never issued
};

// TMA descriptors of one state buffer viewed as u8 [L2][L1][L0/X][X] (X =
// min(L0, 256)): boxes of TY full rows (a tile's interior) and of 2 rows (a
// y halo), one z-plane deep.
struct FusedMaps {
    CUtensorMap rows, halo;
};

bool fused3d_eligible(int model, int q, int d, const int32_t *L, int updater, int rng);
int fused3d_default_tz(int L2);
size_t fused3d_smem_bytes(int L0, int slots);
int fused3d_table_limit_bytes();
cudaError_t fused3d_make_maps(const uint8_t *buf, int L0, int L1, int L2, FusedMaps *out);
cudaError_t launch_fused3d(const FusedArgs &a, const FusedMaps &maps, int q, bool stream, bool hb, cudaStream_t s);

}  // namespace plq
