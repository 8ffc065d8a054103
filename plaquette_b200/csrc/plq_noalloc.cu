// plq_noalloc.cu -- an Ising Metropolis sweep on the PCG stream that
// allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host application that hands this
// library a device buffer it already owns and reserves the rest of the
// device's memory for itself (a framework with its own caching allocator, or
// a fixed memory budget agreed up front), or a latency-sensitive loop that
// must not risk the implicit device synchronisation cudaMalloc/cudaFree may
// perform.  For them, plq_ising_metropolis_noalloc runs the same colour passes
// as an Ising chain with PLQ_METROPOLIS on PLQ_RNG_STREAM, on a spin buffer
// the caller owns, and keeps every piece of scratch the passes need -- the
// PCG jump table, the decision table, the look-back control block and the
// per-chunk look-back descriptors -- in the file-scope array below.
//
// That array is kScratchBytes (384 KiB) of device memory held by every GPU
// that loads the library until the process exits.  Its size caps the lattice
// at PLQ_NOALLOC_MAX_SITES sites.  All calls share it and it keeps the last
// call's contents, so each call clears the parts that must start at zero
// (control block, descriptors); two calls that overlap on the GPU -- on
// different streams, or from different host threads -- race on it and must
// not be issued.  The first call on each device takes the array's device
// address (cudaGetSymbolAddress) with that device current.
//
// The host-side tables are built in a per-thread buffer (not on the caller's
// stack: the jump table is 64 KiB and embedding hosts often run small-stack
// worker threads).  The library remembers, per device, which seed's jump
// table and which couplings' decision table the array holds, and copies a
// table only when it differs: a repeated call with the same seed and
// couplings enqueues no host-to-device copy.  A copy that does happen comes
// from pageable memory, so it waits for the work already queued on the
// caller's stream.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/plaquette.h"
#include "plq_abi_internal.h"
#include "plq_device.cuh"
#include "plq_local.h"
#include "plq_tables.h"

using namespace plq;

namespace {

constexpr size_t kJumpBytes = (size_t)kJumpDigits * kJumpRadix * sizeof(Affine);  // 64 KiB
constexpr size_t kTableOffset = kJumpBytes;
constexpr int64_t kTableEntries = 64;  // q = 2 keys: 2(2d+1) <= 34 for d <= 8
constexpr size_t kControlOffset = kTableOffset + kTableEntries * sizeof(uint64_t);
constexpr size_t kDescOffset = kControlOffset + 256;
constexpr int64_t kMaxChunks = PLQ_NOALLOC_MAX_SITES / 2 / 2048;  // look-back chunks of 2048 ranks
constexpr size_t kScratchBytes = 384 * 1024;
static_assert(kDescOffset + kMaxChunks * sizeof(unsigned long long) <= kScratchBytes,
              "the scratch array must hold the largest lattice's descriptors");
static_assert(sizeof(Control) <= 256, "control block slot");

// The scratch every call of plq_ising_metropolis_noalloc shares.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;

// What the array on one device holds: its device address, and which jump
// table (by the stream's increment) and decision table (by its parameters)
// the last successful call left in it.
struct DeviceScratch {
    unsigned char *ptr;
    bool jump_valid;
    uint64_t inc_lo, inc_hi;
    bool table_valid;
    int32_t d;
    uint64_t j_bits, h_bits, beta_bits;
};
std::mutex g_setup_mu;
DeviceScratch g_dev[kMaxDevices] = {};

// The host-side jump table of the calling thread.
thread_local AffineHost t_jump_host[kJumpDigits * kJumpRadix];

uint64_t bits_of(double x) {
    uint64_t b;
    std::memcpy(&b, &x, sizeof b);
    return b;
}

// Once per device, with that device current: the array's device address.
int scratch_for_current_device(int *dev_out, unsigned char **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return plq_fail(PLQ_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return plq_fail(PLQ_ENODEV, "device ordinal above the supported range");
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_dev[dev].ptr) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr)
            return plq_fail(PLQ_ECUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_dev[dev].ptr = static_cast<unsigned char *>(p);
    }
    *dev_out = dev;
    *out = g_dev[dev].ptr;
    return PLQ_OK;
}

}  // namespace

extern "C" int plq_ising_metropolis_noalloc(uint8_t *spins, int32_t d, const int64_t *shape, double j, double h,
                                            double beta, uint64_t seed, uint64_t stream_offset, uint64_t sweeps,
                                            void *cuda_stream, uint64_t *stream_position_out) {
    if (!spins || !shape) return plq_fail(PLQ_EINVAL, "spins and shape must not be NULL");
    if (d < 1 || d > PLQ_MAX_D) return plq_fail(PLQ_EINVAL, "lattice dimension must be in 1..=8");
    int64_t n = 1;
    for (int i = 0; i < d; ++i) {
        if (shape[i] <= 0) return plq_fail(PLQ_EINVAL, "every extent must be positive");
        if (shape[i] % 2 != 0) {
            plq_chain_desc tmp;
            std::memset(&tmp, 0, sizeof tmp);
            tmp.d = d;
            for (int k = 0; k < d; ++k) tmp.shape[k] = shape[k];
            return plq_fail(PLQ_EINVAL,
                            "the parallel site checkerboard needs even lattice extents, got " + shape_string(&tmp));
        }
        if (n > PLQ_NOALLOC_MAX_SITES / shape[i])
            return plq_fail(PLQ_EINVAL, "the lattice exceeds the no-allocation limit of " +
                                            std::to_string((long long)PLQ_NOALLOC_MAX_SITES) +
                                            " sites (the size of its fixed scratch array)");
        n *= shape[i];
    }
    cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
    // the caller's current device; drop a non-sticky error an unrelated earlier
    // runtime call left on this thread, so the checks below see only our calls
    (void)cudaGetLastError();
    unsigned char *scratch = nullptr;
    int dev = 0;
    int rc = scratch_for_current_device(&dev, &scratch);
    if (rc != PLQ_OK) return rc;

    // host-side tables: the decision table (at most 64 entries) on the stack,
    // the 64 KiB jump table in this thread's buffer
    ModelParams p;
    std::memset(&p, 0, sizeof p);
    p.model = PLQ_ISING;
    p.q = 2;
    p.d = d;
    p.beta = beta;
    p.j = j;
    p.h = h;
    uint64_t metro[kTableEntries];
    if (q2_metro53_into(p, metro, kTableEntries) < 0) return plq_fail(PLQ_EINVAL, "decision table too large");
    AffineHost *jump_host = t_jump_host;
    uint64_t slo, shi, ilo, ihi;
    pcg_seed_from_u64(seed, slo, shi, ilo, ihi);
    jump_table_into(ilo, ihi, jump_host);
    const Affine *T = reinterpret_cast<const Affine *>(jump_host);
    u128 inc{ilo, ihi};
    u128 base = jump(T, u128{slo, shi}, stream_offset);
    base = pcg_step(base, inc);

    const int64_t n_chunks = local_chunks(n);
    // copy only the tables the array does not hold already; a table about to
    // be rewritten counts as absent until this call has succeeded
    bool need_jump, need_table;
    const uint64_t jb = bits_of(j), hb = bits_of(h), bb = bits_of(beta);
    {
        std::lock_guard<std::mutex> lock(g_setup_mu);
        DeviceScratch &r = g_dev[dev];
        need_jump = !(r.jump_valid && r.inc_lo == ilo && r.inc_hi == ihi);
        need_table = !(r.table_valid && r.d == d && r.j_bits == jb && r.h_bits == hb && r.beta_bits == bb);
        if (need_jump) r.jump_valid = false;
        if (need_table) r.table_valid = false;
    }
    cudaError_t e = cudaSuccess;
    if (need_jump) e = cudaMemcpyAsync(scratch, jump_host, kJumpBytes, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess && need_table)
        e = cudaMemcpyAsync(scratch + kTableOffset, metro, sizeof metro, cudaMemcpyHostToDevice, stream);
    // the parts that must start at zero: control block and descriptors
    if (e == cudaSuccess) e = cudaMemsetAsync(scratch + kControlOffset, 0, sizeof(Control), stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(scratch + kDescOffset, 0, (size_t)n_chunks * sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return plq_fail(PLQ_ECUDA, std::string("scratch set-up: ") + cudaGetErrorString(e));

    LocalArgs a;
    std::memset(&a, 0, sizeof a);
    a.state = spins;
    a.g.d = d;
    int64_t stride = 1;
    for (int i = 0; i < kMaxD; ++i) {
        a.g.L[i] = i < d ? (int32_t)shape[i] : 1;
        a.g.stride[i] = stride;
        if (i < d) stride *= shape[i];
    }
    a.g.n_sites = n;
    geom_init(a.g, d, shape);
    a.q = 2;
    a.kernel = PLQ_METROPOLIS;
    a.model = PLQ_ISING;
    a.pw[1] = 1;
    a.metro53 = reinterpret_cast<const uint64_t *>(scratch + kTableOffset);
    a.jump = reinterpret_cast<const Affine *>(scratch);
    a.base = base;
    a.inc = inc;
    a.ctrl = reinterpret_cast<Control *>(scratch + kControlOffset);
    a.desc = reinterpret_cast<unsigned long long *>(scratch + kDescOffset);
    a.n_chunks = n_chunks;
    uint64_t passes = 0;
    for (uint64_t t = 0; t < sweeps; ++t)
        for (int color = 0; color < 2; ++color, ++passes) {
            a.color = color;
            a.epoch = (uint32_t)(passes + 1);
            a.ticket_base = passes * (uint64_t)n_chunks;
            a.pos_in = (int)(passes & 1);
            e = launch_local_pass(a, false, true, stream);
            if (e != cudaSuccess) return plq_fail(PLQ_ECUDA, std::string("pass launch: ") + cudaGetErrorString(e));
        }

    Control host_ctrl;
    e = cudaMemcpyAsync(&host_ctrl, scratch + kControlOffset, sizeof host_ctrl, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return plq_fail(PLQ_ECUDA, std::string("read-back: ") + cudaGetErrorString(e));
    {
        std::lock_guard<std::mutex> lock(g_setup_mu);
        DeviceScratch &r = g_dev[dev];
        r.jump_valid = true;
        r.inc_lo = ilo;
        r.inc_hi = ihi;
        r.table_valid = true;
        r.d = d;
        r.j_bits = jb;
        r.h_bits = hb;
        r.beta_bits = bb;
    }
    if (host_ctrl.status)
        return plq_fail(PLQ_EDEVICE, "device status word " + std::to_string(host_ctrl.status));
    if (stream_position_out) *stream_position_out = stream_offset + host_ctrl.pos[passes & 1];
    return PLQ_OK;
}
