// plq_tables.h -- host precompute of every accept/reject and heat-bath
// decision as integer cut points on the raw random integer.
//
// The reference decides with floating point:
//   Metropolis   next_f64() < exp(-beta*dE)           (src/updater.rs:90)
//   heat bath    next_f64()*total < cumulative_s      (src/updater.rs:151-164)
// in f64 on the CPU and in f32 with a 24-bit uniform on the GPU
// (metropolis.wgsl:59-60, heat_bath.wgsl:50-61).  For a fixed chain every
// quantity except the uniform is a function of a small "environment" (the
// variable's state and its neighbours' state counts, or its staple sum), so
// each decision is "k < K" for the raw integer k behind the uniform
// (53 bits from PCG64, 24 bits from the keyed hash).  K is found on the host
// by evaluating the reference arithmetic in the reference precision, so the
// device makes exactly the reference's decisions with no exp and no floating
// point at all.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace plq {

constexpr uint64_t kAlways53 = ~0ULL;     // dE <= 0: accept, consume no draw
constexpr uint32_t kAlways24 = 0xFFFFFFFFu;

struct ModelParams {
    int model;  // PLQ_ISING / PLQ_POTTS / PLQ_GAUGE
    int q;
    int d;
    double beta, j, h;
    double offsets[64];
};

// Environment keys (the device computes the same index):
//   site models: key = cur + q * packed, packed = sum over the 2d neighbours
//                of pw[state], pw[0] = 0 and pw[s] = (2d+1)^(s-1) for s >= 1
//                (for q = 2 the packed value is the neighbour state sum);
//   gauge links: key = cur + 2 * ((S + 2(d-1)) / 2), S the staple sum.
int64_t env_key_count(const ModelParams &p);
// Potts Metropolis key: ((cur*q + prop)*(2d+1) + c_prop)*(2d+1) + c_cur.
int64_t potts_metro_key_count(const ModelParams &p);

struct Tables {
    // Heat bath: (q-1) nondecreasing cut points per environment key;
    // chosen = number of cut points <= k.
    std::vector<uint64_t> hb53;
    std::vector<uint32_t> hb24;
    // Metropolis: one entry per environment key (q == 2) or Potts key;
    // kAlways* = accept without a draw, else accept iff k < K.
    std::vector<uint64_t> metro53;
    std::vector<uint32_t> metro24;
};

// Builds the tables for `updater` (PLQ_METROPOLIS / PLQ_HEATBATH) and `rng`.
// Returns false with a message when the table would be too large.
bool build_tables(const ModelParams &p, int updater, int rng, Tables &out, std::string &err);

// Largest table the builder accepts, in entries.
constexpr int64_t kMaxTableEntries = int64_t(1) << 24;

// Radix-256 jump tables for the PCG64 stream with increment `inc`
// (kJumpDigits * kJumpRadix affine maps).
struct AffineHost {
    uint64_t m_lo, m_hi, p_lo, p_hi;
};
void build_jump_table(uint64_t inc_lo, uint64_t inc_hi, std::vector<AffineHost> &out);
// Heap-free variants: q = 2 Metropolis cut points on the PCG stream for every
// environment key (returns the key count, or -1 if `capacity` is too small),
// and the jump table into `out` (kJumpDigits * kJumpRadix entries).
int64_t q2_metro53_into(const ModelParams &p, uint64_t *out, int64_t capacity);
void jump_table_into(uint64_t inc_lo, uint64_t inc_hi, AffineHost *out);
// The affine map of n LCG steps, composed from the jump table.
AffineHost affine_steps(const std::vector<AffineHost> &table, uint64_t n);

// rand_core seed_from_u64 + rand_pcg from_seed: the stream's state s_0
// (after construction) and increment.
void pcg_seed_from_u64(uint64_t seed, uint64_t &s_lo, uint64_t &s_hi, uint64_t &i_lo,
                       uint64_t &i_hi);

// Host reproduction of the reference's hot start draws.
struct HostPcg {
    unsigned __int128 state, inc;
    uint64_t draws = 0;
    uint64_t next_u64();
    uint64_t next_below(uint64_t n);
};
HostPcg host_pcg_from_seed(uint64_t seed);

}  // namespace plq
