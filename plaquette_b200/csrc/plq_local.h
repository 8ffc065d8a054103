// plq_local.h -- launchers of the local (single-variable) passes.
#pragma once
#include <cuda_runtime.h>

#include "plq_device.cuh"

namespace plq {

// Chunks (CTAs) one colour pass launches; also the look-back descriptor count.
int64_t local_chunks(int64_t n_sites);
// CTAs of one four-sites-at-a-time pass (a.words set).
int64_t word_chunks(int64_t n_sites);
// One colour pass: sites (link=false) or the links of direction a.dir.
cudaError_t launch_local_pass(const LocalArgs &a, bool link, bool lookback, cudaStream_t stream);
// One colour pass of Potts Metropolis (q >= 3) on the PCG stream: the
// sequential walk (plq_walk.cu); start and end positions in a.ctrl->pos.
cudaError_t launch_potts_metro_walk(const LocalArgs &a, cudaStream_t stream);

// Exact integer primaries of a configuration into out (int64, zeroed by the
// launcher): Ising {bond_sum, spin_sum}, Potts {agree, counts[q]}, gauge
// {plaquette_sum}.  Returns the number of values.
int primaries_count(int model, int q);
cudaError_t launch_primaries(const uint8_t *state, const Geom &g, int model, int q,
                             long long *out, cudaStream_t stream);

// Many configurations' primaries in one launch (d <= 4): task k's values go
// to tasks[k].out, which must be zero before the launch; work item i covers
// sites [item_chunk[i] * kPrimChunk, ...) of task item_task[i].
constexpr int64_t kPrimChunk = 16384;
struct PrimTask {
    const uint8_t *state;
    Geom g;
    int model, q;
    long long *out;
};
cudaError_t launch_primaries_multi(const PrimTask *tasks, const int32_t *item_task, const int32_t *item_chunk,
                                   int64_t n_items, int sm_count, cudaStream_t stream);

// Bit-packed colour passes of one q = 2 site lattice on the keyed stream
// (plq_packed3d.cu): 2D or 3D, extent 0 a multiple of 64; word g holds sites
// [64 g, 64 g + 64).  n_keys table entries (cur + 2 * count) are read.
struct PackedPassArgs {
    uint64_t *words;
    int64_t n_words;
    int L0, L1;  // L1: the 3D lattice's extent 1 (unused in 2D)
    int colour;
    uint32_t seed32, sweep32;
    const uint32_t *table;  // metro24 (Metropolis) or hb24 (heat bath)
    int n_keys;
    // Optional: every variable's sweep-independent first round lowbias32_head(seed ^ site)
    // (first_hash_bytes(n_words) bytes, filled by launch_first_hash); null = hash in the pass.
    const void *first_hash;
};
bool packed_chain_eligible(int model, int q, int d, const int32_t *L, int updater, int rng);
size_t first_hash_bytes(int64_t n_words);
cudaError_t launch_first_hash(void *first_hash, int64_t n_words, int L0, int L1, int d, uint32_t seed32,
                              int sm_count, cudaStream_t stream);
cudaError_t launch_pack64(const uint8_t *bytes, uint64_t *words, int64_t n_words, int sm_count, cudaStream_t stream);
cudaError_t launch_unpack64(const uint64_t *words, uint8_t *bytes, int64_t n_words, int sm_count,
                            cudaStream_t stream);
cudaError_t launch_packed_pass(const PackedPassArgs &a, int d, bool hb, int sm_count, cudaStream_t stream);

// Layout conversion of link variables: host order (site*d + dir) <-> device
// planes (dir*n_sites + site).
cudaError_t launch_links_to_planes(const uint8_t *in, uint8_t *out, int64_t n_sites, int d,
                                   cudaStream_t stream);
cudaError_t launch_planes_to_links(const uint8_t *in, uint8_t *out, int64_t n_sites, int d,
                                   cudaStream_t stream);

}  // namespace plq
