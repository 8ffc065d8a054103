// plq_device.cuh -- device-side structures shared by the kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "plq_rng.cuh"

namespace plq {

constexpr int kMaxD = 8;

// Status word bits a kernel may raise (host maps them to PLQ_EDEVICE/ECAP).
constexpr uint32_t kStatusLookbackTimeout = 1u << 0;
constexpr uint32_t kStatusPassCap = 1u << 1;
constexpr uint32_t kStatusBounds = 1u << 2;
constexpr uint32_t kStatusQueueOverflow = 1u << 3;
constexpr uint32_t kStatusCopyTimeout = 1u << 4;

// Lattice geometry by value: extents, strides, site count, and the magic
// numbers that divide a site index (< 2^31) by each extent.
struct Geom {
    int d;
    int32_t L[kMaxD];
    int64_t stride[kMaxD];
    int64_t n_sites;
    uint32_t dm[kMaxD];  // division by L[mu]: multiplier
    int32_t dl[kMaxD];   // ... and ceil(log2 L[mu])
};

// Division by an invariant integer with one multiply-high (Granlund and
// Montgomery, "Division by invariant integers using multiplication", 1994,
// the unsigned multiply-add form): exact for every 32-bit n.
PLQ_HD uint32_t fdiv(uint32_t n, uint32_t m, int l) {
    if (l == 0) return n;
#if defined(__CUDA_ARCH__)
    uint32_t t1 = __umulhi(m, n);
#else
    uint32_t t1 = (uint32_t)(((uint64_t)m * n) >> 32);
#endif
    return (t1 + ((n - t1) >> 1)) >> (l - 1);
}

// Fill extents, strides and division constants from a shape.
inline void geom_init(Geom &g, int d, const int64_t *shape) {
    g.d = d;
    int64_t n = 1;
    for (int i = 0; i < kMaxD; ++i) {
        g.L[i] = i < d ? (int32_t)shape[i] : 1;
        g.stride[i] = n;
        if (i < d) n *= shape[i];
        uint32_t L = (uint32_t)g.L[i];
        if (L <= 1) {
            g.dm[i] = 0;
            g.dl[i] = 0;
        } else {
            int l = 0;
            while ((1ull << l) < L) ++l;
            g.dm[i] = (uint32_t)((((1ull << 32) * ((1ull << l) - L)) / L) + 1);
            g.dl[i] = l;
        }
    }
    g.n_sites = n;
}

// Per-chain device control block (in device memory).
struct Control {
    unsigned long long pos[2];     // stream position ping-pong (data-dependent passes)
    unsigned long long ticket;     // chunk tickets for decoupled look-back
    unsigned int status;           // fault bits
    unsigned int pad;
    unsigned long long scratch[4]; // per-kernel small counters
};

// Everything a local (single-variable) pass needs.
struct LocalArgs {
    uint8_t *state;          // sites: n_sites; links: d planes of n_sites
    Geom g;
    int q;
    int kernel;              // PLQ_METROPOLIS / PLQ_HEATBATH
    int model;               // PLQ_ISING / PLQ_POTTS / PLQ_GAUGE
    int color;               // 0/1 (sites) ; link passes: parity
    int dir;                 // link passes: direction
    int32_t pw[64];          // packing weights of neighbour states (site env keys)
    // decision tables
    const uint64_t *hb53;
    const uint32_t *hb24;
    const uint64_t *metro53;
    const uint32_t *metro24;
    // keyed stream
    uint32_t seed32;
    uint32_t sweep32;
    // PCG stream
    const Affine *jump;      // radix-256 jump table for this chain's increment
    u128 base;               // state s.t. draw n = xsl_rr(jump(base, n))
    u128 inc;
    uint64_t pass_offset;    // deterministic passes: position of rank 0
    // look-back (data-dependent passes)
    Control *ctrl;
    unsigned long long *desc;  // per-chunk descriptors
    uint64_t ticket_base;
    uint32_t epoch;
    int pos_in;               // which ctrl->pos[] to read; the other is written
    int64_t n_chunks;
    int words;                // run the pass four sites at a time (plq_words.cuh)
};

}  // namespace plq
