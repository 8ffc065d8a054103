// plq_packed3d.cu -- bit-packed colour passes of one q = 2 site lattice.
//
// A chain of an Ising (or q = 2 Potts) lattice on the keyed stream, 2D or 3D
// with extent 0 a multiple of 64, runs its sweeps on a packed copy of its
// state: word g holds sites [64 g, 64 g + 64) (64 consecutive sites of one
// row), one bit per site.  advance() packs the bytes once, runs every colour
// pass in place on the words and unpacks at the end.  A thread takes one word:
// the states of the +x / -x neighbours of its 64 sites are the word shifted by
// one with the end bit taken from the next / previous word of the row
// (periodic), the +-y and +-z neighbours are the same word of other rows; a
// bit-sliced counter sums the 2d neighbour words, and the 32 sites of the
// pass's parity decide exactly as the byte passes do -- key cur + 2 * count,
// the keyed draw of the site's index (rng.wgsl:34-52), the same cut-point
// table (metropolis.wgsl:32-63, heat_bath.wgsl:28-62) -- so the chain's states
// are bit-identical to the byte paths'.  A pass changes only its colour's
// bits, so a neighbour word read while another thread rewrites it yields the
// same bits of the other colour either way.
//
// The packed copy (1/8 B per site) stays in L2 and the passes are bound by
// the ALU pipe, mostly the keyed draws' hashing.  So a chain also keeps, where
// it has room, each site's sweep-independent first round of its draws (4 B per
// site, filled once at creation) and a pass streams its colour's half of that
// array from HBM instead of computing it: HBM bytes the packed passes do not
// otherwise use, traded for ALU work.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/plaquette.h"
#include "plq_device.cuh"
#include "plq_local.h"
#include "plq_packed.cuh"
#include "plq_rng.cuh"

namespace plq {

namespace {

constexpr int kPackedThreads = 256;

// bytes (0/1) -> bits: thread g packs sites [64 g, 64 g + 64)
__global__ void __launch_bounds__(kPackedThreads) pack64_kernel(const uint8_t *bytes, uint64_t *words, int64_t n_words) {
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n_words; g += (int64_t)gridDim.x * blockDim.x) {
        const uint4 *src = reinterpret_cast<const uint4 *>(bytes + 64 * g);
        uint64_t w = 0;
#pragma unroll
        for (int q4 = 0; q4 < 4; ++q4) {
            const uint4 v = src[q4];
            const uint32_t parts[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int k = 0; k < 4; ++k)  // four 0/1 bytes -> four bits (b_i * 2^(24 - 7 i) lands at bit 24 + i)
                w |= (uint64_t)(((parts[k] * 0x01020408u) >> 24) & 0xFu) << (16 * q4 + 4 * k);
        }
        words[g] = w;
    }
}

// bits -> bytes
__global__ void __launch_bounds__(kPackedThreads) unpack64_kernel(const uint64_t *words, uint8_t *bytes, int64_t n_words) {
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n_words; g += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t w = words[g];
        uint4 *dst = reinterpret_cast<uint4 *>(bytes + 64 * g);
#pragma unroll
        for (int q4 = 0; q4 < 4; ++q4) {
            uint32_t parts[4];
#pragma unroll
            for (int k = 0; k < 4; ++k)  // nibble -> four 0/1 bytes
                parts[k] = ((uint32_t)(w >> (16 * q4 + 4 * k)) & 0xFu) * 0x00204081u & 0x01010101u;
            dst[q4] = make_uint4(parts[0], parts[1], parts[2], parts[3]);
        }
    }
}

// The first-hash array, lowbias32_head(seed ^ site) of every site (the sweep-independent
// first round of its keyed draws, keyed24 in plq_rng.cuh): for colour c, word g and the
// pass's variables 4 jq .. 4 jq + 3 of
// that word (sites 64 g + x0 + 2 (4 jq + m)), one uint4 at ((c * nb + g / 32) * 8 + jq) * 32
// + g % 32, nb = ceil(n_words / 32): the 32 words of a warp read 512 contiguous bytes per load.
__global__ void __launch_bounds__(kPackedThreads) first_hash_kernel(uint4 *H, int64_t n_words, int64_t nb,
                                                                   uint32_t wpr, uint32_t L1, int d, uint32_t seed32) {
    const int64_t total = 2 * nb * 8 * 32;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t lane = (uint32_t)(i & 31);
        const int64_t t = i >> 5;
        const uint32_t jq = (uint32_t)(t & 7);
        const int64_t bc = t >> 3;
        const uint32_t colour = (uint32_t)(bc / nb);
        const int64_t g = (bc - (int64_t)colour * nb) * 32 + lane;
        if (g >= n_words) {
            H[i] = make_uint4(0, 0, 0, 0);
            continue;
        }
        const uint32_t r = (uint32_t)(g / wpr);
        const uint32_t y = d == 3 ? r % L1 : r;
        const uint32_t z = d == 3 ? r / L1 : 0;
        const uint32_t v = (uint32_t)(64 * g) + ((colour ^ y ^ z) & 1u) + 8 * jq;
        H[i] = make_uint4(lowbias32_head(seed32 ^ v), lowbias32_head(seed32 ^ (v + 2)),
                          lowbias32_head(seed32 ^ (v + 4)), lowbias32_head(seed32 ^ (v + 6)));
    }
}

template <int D, bool HB, bool CACHED>
__global__ void __launch_bounds__(kPackedThreads, 8) packed_pass_kernel(PackedPassArgs a) {
    __shared__ uint32_t s_tab[16];
    if (threadIdx.x < 16) s_tab[threadIdx.x] = threadIdx.x < (unsigned)a.n_keys ? table_entry(a.table[threadIdx.x]) : 0u;
    __syncthreads();
    const uint32_t wpr = (uint32_t)a.L0 / 64;  // words per row
    const uint32_t rows = (uint32_t)(a.n_words / wpr);
    const uint32_t sweep_mix = keyed_mix(a.sweep32);
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < a.n_words; g += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t r = (uint32_t)g / wpr;
        const uint32_t wi = (uint32_t)g - r * wpr;
        uint32_t y, z = 0;
        if (D == 3) {
            z = r / (uint32_t)a.L1;
            y = r - z * (uint32_t)a.L1;
        } else {
            y = r;
        }
        uint4 hv[8];
        if (CACHED) {  // this pass's 32 first hashes, issued before the neighbour loads
            const uint4 *hp = static_cast<const uint4 *>(a.first_hash) +
                              ((((int64_t)a.colour * ((a.n_words + 31) >> 5) + (g >> 5)) * 8) << 5) + (g & 31);
#pragma unroll
            for (int k = 0; k < 8; ++k) hv[k] = __ldcs(hp + 32 * k);
        }
        const uint64_t *w = a.words;
        const uint32_t rb = r * wpr;
        const uint64_t C = w[g];
        const uint64_t left = w[rb + (wi > 0 ? wi - 1 : wpr - 1)];
        const uint64_t right = w[rb + (wi + 1 < wpr ? wi + 1 : 0)];
        uint64_t c0 = 0, c1 = 0, c2 = 0;
        count_add(c0, c1, c2, (C >> 1) | (right << 63));  // +x
        count_add(c0, c1, c2, (C << 1) | (left >> 63));   // -x
        // +-y: rows r +- 1 within the plane (periodic)
        const uint32_t Ly = D == 3 ? (uint32_t)a.L1 : rows;
        const uint32_t ryp = y + 1 < Ly ? r + 1 : r - (Ly - 1);
        const uint32_t rym = y > 0 ? r - 1 : r + (Ly - 1);
        count_add(c0, c1, c2, w[ryp * wpr + wi]);
        count_add(c0, c1, c2, w[rym * wpr + wi]);
        if (D == 3) {  // +-z: rows r +- L1 (periodic)
            const uint32_t Lz = rows / (uint32_t)a.L1;
            const uint32_t rzp = z + 1 < Lz ? r + (uint32_t)a.L1 : r - (Lz - 1) * (uint32_t)a.L1;
            const uint32_t rzm = z > 0 ? r - (uint32_t)a.L1 : r + (Lz - 1) * (uint32_t)a.L1;
            count_add(c0, c1, c2, w[rzp * wpr + wi]);
            count_add(c0, c1, c2, w[rzm * wpr + wi]);
        }
        // the word's first site x = 64 wi is even: the pass's sites are at (colour + y + z) & 1 + 2j
        const uint32_t x0 = (uint32_t)((a.colour ^ y ^ z) & 1u);
        const uint32_t v0 = r * (uint32_t)a.L0 + 64u * wi + x0;  // keyed index of the word's first such site
        uint64_t flip;
        if (CACHED) {
            const uint64_t M = 0x5555555555555555ull;
            const uint64_t P = ((C >> x0) & M) | (((c0 >> x0) << 1) & ~M);
            const uint64_t Q = ((c1 >> x0) & M) | (((c2 >> x0) << 1) & ~M);
            const char *tb = reinterpret_cast<const char *>(s_tab);
            flip = 0;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const uint32_t h1[8] = {hv[2 * c].x,     hv[2 * c].y,     hv[2 * c].z,     hv[2 * c].w,
                                        hv[2 * c + 1].x, hv[2 * c + 1].y, hv[2 * c + 1].z, hv[2 * c + 1].w};
                flip |= (uint64_t)decide8_h1<HB>(key_word(P, Q, c), h1, sweep_mix, tb) << (16 * c);
            }
            if (HB) flip ^= P & M;  // new states -> flips
            (void)v0;
        } else {
            flip = decide_row<uint64_t, 2, HB>(C >> x0, c0 >> x0, c1 >> x0, c2 >> x0, 32, v0, a.seed32, sweep_mix,
                                               s_tab);
        }
        a.words[g] = C ^ (flip << x0);
    }
}

unsigned blocks_for(int64_t n_words, int sm_count) {
    const int64_t b = (n_words + kPackedThreads - 1) / kPackedThreads;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)sm_count * 16));
}

}  // namespace

bool packed_chain_eligible(int model, int q, int d, const int32_t *L, int updater, int rng) {
    return rng == PLQ_RNG_KEYED && (model == PLQ_ISING || (model == PLQ_POTTS && q == 2)) &&
           (updater == PLQ_METROPOLIS || updater == PLQ_HEATBATH) && (d == 2 || d == 3) && L[0] % 64 == 0;
}

cudaError_t launch_pack64(const uint8_t *bytes, uint64_t *words, int64_t n_words, int sm_count, cudaStream_t stream) {
    pack64_kernel<<<blocks_for(n_words, sm_count), kPackedThreads, 0, stream>>>(bytes, words, n_words);
    return cudaGetLastError();
}

cudaError_t launch_unpack64(const uint64_t *words, uint8_t *bytes, int64_t n_words, int sm_count, cudaStream_t stream) {
    unpack64_kernel<<<blocks_for(n_words, sm_count), kPackedThreads, 0, stream>>>(words, bytes, n_words);
    return cudaGetLastError();
}

size_t first_hash_bytes(int64_t n_words) { return (size_t)((n_words + 31) / 32) * 2 * 8 * 32 * sizeof(uint4); }

cudaError_t launch_first_hash(void *first_hash, int64_t n_words, int L0, int L1, int d, uint32_t seed32,
                              int sm_count, cudaStream_t stream) {
    if (d != 2 && d != 3) return cudaErrorInvalidValue;
    const int64_t nb = (n_words + 31) / 32;
    const int64_t total = nb * 2 * 8 * 32;
    first_hash_kernel<<<blocks_for(total, sm_count), kPackedThreads, 0, stream>>>(
        static_cast<uint4 *>(first_hash), n_words, nb, (uint32_t)L0 / 64, (uint32_t)L1, d, seed32);
    return cudaGetLastError();
}

template <int D, bool HB>
static void launch_pass_d(const PackedPassArgs &a, unsigned blocks, cudaStream_t stream) {
    if (a.first_hash) packed_pass_kernel<D, HB, true><<<blocks, kPackedThreads, 0, stream>>>(a);
    else packed_pass_kernel<D, HB, false><<<blocks, kPackedThreads, 0, stream>>>(a);
}

cudaError_t launch_packed_pass(const PackedPassArgs &a, int d, bool hb, int sm_count, cudaStream_t stream) {
    const unsigned blocks = blocks_for(a.n_words, sm_count);
    if (d == 3) {
        if (hb) launch_pass_d<3, true>(a, blocks, stream);
        else launch_pass_d<3, false>(a, blocks, stream);
    } else if (d == 2) {
        if (hb) launch_pass_d<2, true>(a, blocks, stream);
        else launch_pass_d<2, false>(a, blocks, stream);
    } else {
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace plq
