// plq_abi_internal.h -- the objects behind the opaque C handles.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/plaquette.h"
#include "plq_device.cuh"
#include "plq_fused.h"
#include "plq_tables.h"

struct plq_ctx {
    int device = 0;
    int sm_count = 0;
    int cc_major = 0;
    size_t mem_total = 0;
};

// Makes `device` current and drops a non-sticky error that an unrelated
// earlier runtime call left on this thread, so that the launch checks after it
// report only their own launches.  A sticky (device) error cannot be cleared
// and still fails every later call.
inline cudaError_t plq_enter_device(int device) {
    (void)cudaGetLastError();
    return cudaSetDevice(device);
}

struct plq_chain {
    // The context's record, copied at creation: the chain stays valid if the
    // caller destroys the context first (a garbage collector may finalize the
    // two in either order).
    plq_ctx ctx_copy;
    plq_ctx *ctx = nullptr;  // = &ctx_copy
    plq_chain_desc desc;
    int q = 2, d = 1;
    bool link = false, cluster = false, lookback = false;
    bool words = false;  // passes four sites at a time (plq_words.cuh)
    int64_t n_sites = 0, n_vars = 0;
    plq::Geom g;
    uint32_t seed32 = 0;
    cudaStream_t stream = nullptr;

    uint8_t *d_state = nullptr;  // device layout (links as direction planes)
    uint8_t *d_state_alt = nullptr;  // second buffer of the out-of-place fused sweep
    bool fused = false;
    bool packed = false;          // q = 2 keyed sites: sweeps on a bit-packed copy (plq_packed3d.cu)
    uint64_t *d_packed = nullptr; // n_sites / 64 words
    void *d_first_hash = nullptr; // packed chains: lowbias32_head(seed ^ site) of every site (plq_packed3d.cu)
    int fused_tz = 0;
    plq::FusedMaps fused_maps[2];          // TMA descriptors of the two state buffers
    const uint8_t *fused_map_buf[2] = {nullptr, nullptr};
    // Fused chains measure a sample on a second stream while the next sweep (which
    // writes the other buffer) runs; a sweep about to overwrite a buffer waits for
    // the measurement still reading it.
    cudaStream_t obs_stream = nullptr;
    cudaEvent_t swept = nullptr, measured[2] = {nullptr, nullptr};
    bool measuring[2] = {false, false};
    std::vector<plq::AffineHost> h_jump;  // host copy of the jump table
    uint8_t *d_io = nullptr;     // host-order staging on the device
    uint64_t *d_hb53 = nullptr, *d_metro53 = nullptr;
    uint64_t *d_hb53_fused = nullptr;  // stream heat-bath cut points << 11 (the fused sweep's table)
    uint32_t *d_hb24 = nullptr, *d_metro24 = nullptr;
    int32_t pw[64];
    plq::Affine *d_jump = nullptr;
    plq::u128 base{0, 0}, inc{0, 0};
    plq::Control *d_ctrl = nullptr;
    unsigned long long *d_desc = nullptr;
    int64_t n_chunks = 0;
    long long *d_obs = nullptr;
    uint8_t *d_snap = nullptr;
    uint32_t *d_loop_bits = nullptr;   // Wilson line parities (n_sites * d words), on first use
    long long *d_meas = nullptr;       // measurement results (meas_cap int64)
    int32_t *d_pairs = nullptr;        // (mu, r) pair lists of the correlator (2 * meas_cap)
    int64_t meas_cap = 0;
    long long *d_snap_obs = nullptr;
    int64_t snap_cap = 0, snap_obs_cap = 0;
    void *h_pinned = nullptr;

    uint64_t sweeps_done = 0;
    uint64_t host_pos = 0;          // deterministic stream passes: draws consumed
    uint64_t lookback_passes = 0;   // data-dependent passes launched
    uint64_t tickets_issued = 0;    // look-back chunk tickets taken by those passes
    uint64_t launches = 0;

    // cluster state (plq_cluster.cu)
    void *cl = nullptr;
    int cluster_pos_parity = 0;
    int64_t pass_cap = 0;
};

int plq_fail(int code, const std::string &msg);
// Index of the first byte >= q (q <= 64) in a[0, n), or -1 (64 bytes per step).
int64_t first_state_at_least(const uint8_t *a, int64_t n, int q);
// The smallest member index m whose start (if not null) holds a state >= q[m], or -1.
int32_t first_bad_start(int32_t n, const uint8_t *const *starts, const int64_t *n_vars, const int *q);
std::string shape_string(const plq_chain_desc *d);
void chain_free(plq_chain *c);
int local_sweep(plq_chain *c);
