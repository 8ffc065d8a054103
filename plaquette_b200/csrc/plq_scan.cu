// plq_scan.cu -- one colour pass of q = 2 checkerboard Metropolis on the PCG
// stream for 2D/3D site lattices with extent 0 a multiple of 16.
//
// Same semantics as the generic look-back pass (plq_local_impl.cuh): a
// variable draws only when its move is uphill (src/updater.rs:90), so its draw
// position is the count of uphill variables of the colour before it in index
// order -- a device-wide exclusive scan, done in one pass with decoupled
// look-back over chunks in block order.  What this kernel changes is
// the cost per site:
//   * a thread owns 16 consecutive sites (one 16-byte vector, 8 of the pass's
//     colour); neighbour words come as vectors (+-y, +-z) and 4-byte words
//     (+-x across the vector's ends), and the table keys of all 16 sites are
//     computed four at a time in 32-bit words (SWAR: key = cur + 2 * sum of
//     neighbour states, no byte ever carries);
//   * the chunk's first thread jumps the PCG stream to the chunk's position
//     once (8 radix-256 digits); every thread then jumps from there by its
//     local exclusive count (< 2^16: at most 2 digits) and steps the LCG.
#include <cuda_runtime.h>

#include "../../include/plaquette.h"
#include "plq_device.cuh"
#include "plq_scan.h"

namespace plq {

constexpr int SThreads = 256;
constexpr int SSites = 16;  // sites per thread
constexpr int SChunkSites = SThreads * SSites;
constexpr int SSpinLimit = 1 << 22;

__device__ __forceinline__ unsigned long long s_ld_relaxed(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long s_make_desc(uint32_t epoch, unsigned long long st, uint32_t value) {
    return ((unsigned long long)(epoch & 0x3FFFFFFFu) << 34) | (st << 32) | value;
}

// jump by a small count (< 2^16): the two low radix-256 digits
__device__ __forceinline__ u128 jump_small(const Affine *table, u128 s, uint32_t n) {
    uint32_t v0 = n & 255u, v1 = (n >> 8) & 255u;
    if (v0) s = apply(table[v0], s);
    if (v1) s = apply(table[kJumpRadix + v1], s);
    return s;
}

template <int D>
__global__ void __launch_bounds__(SThreads, 8) scan_metro_kernel(ScanArgs a) {
    __shared__ uint64_t s_tab[64];
    __shared__ int warp_tot[SThreads / 32];
    __shared__ u128 s_chunk_state;
    __shared__ int s_fail;

    if (threadIdx.x < a.table_entries) s_tab[threadIdx.x] = a.metro53[threadIdx.x];
    __syncthreads();
    // Chunk = block index: blocks are dispatched in index order, so a chunk's
    // predecessors are running or done when it looks back (the waits are
    // bounded all the same).
    const int64_t chunk = (int64_t)blockIdx.x;
    if (chunk >= a.n_chunks) {
        if (threadIdx.x == 0) atomicOr(&a.ctrl->status, kStatusBounds);
        return;
    }
    const int64_t n = a.n_sites;
    const int64_t s0 = chunk * SChunkSites + (int64_t)threadIdx.x * SSites;
    const bool active = s0 < n;

    // ---- keys of the 16 sites
    uint32_t C[4] = {0, 0, 0, 0}, K[4] = {0, 0, 0, 0};
    uint32_t need_mask = 0;  // bit i: colour site i (0..7) draws
    int b = 0;
    if (active) {
        // coordinates of the vector's first site (x multiple of 16; site
        // indices are below 2^32 on this path, see scan_metro_eligible)
        const uint32_t row = fdiv((uint32_t)s0, a.dm0, a.dl0);
        const uint32_t x0 = (uint32_t)s0 - row * (uint32_t)a.L0;
        uint32_t y = row, z = 0;
        if (D == 3) {
            z = fdiv(row, a.dm1, a.dl1);
            y = row - z * (uint32_t)a.L1;
        }
        const uint4 c4 = *reinterpret_cast<const uint4 *>(a.state + s0);
        C[0] = c4.x;
        C[1] = c4.y;
        C[2] = c4.z;
        C[3] = c4.w;
        const int64_t rs = s0 - x0;  // row start
        const uint32_t Lw = *reinterpret_cast<const uint32_t *>(a.state + rs + (x0 == 0 ? a.L0 - 4 : x0 - 4));
        const uint32_t Rw = *reinterpret_cast<const uint32_t *>(a.state + rs + (x0 + 16 == (uint32_t)a.L0 ? 0 : x0 + 16));
        const int64_t sy = (int64_t)a.L0;
        const uint4 up = *reinterpret_cast<const uint4 *>(a.state + (y + 1 < (uint32_t)a.L1 ? s0 + sy : s0 - sy * (a.L1 - 1)));
        const uint4 dn = *reinterpret_cast<const uint4 *>(a.state + (y > 0 ? s0 - sy : s0 + sy * (a.L1 - 1)));
        uint32_t U[4] = {up.x, up.y, up.z, up.w}, Dn[4] = {dn.x, dn.y, dn.z, dn.w};
        uint32_t Zp[4] = {0, 0, 0, 0}, Zm[4] = {0, 0, 0, 0};
        if (D == 3) {
            const int64_t sz = (int64_t)a.L0 * a.L1;
            const uint4 zp = *reinterpret_cast<const uint4 *>(a.state + (z + 1 < (uint32_t)a.L2 ? s0 + sz : s0 - sz * (a.L2 - 1)));
            const uint4 zm = *reinterpret_cast<const uint4 *>(a.state + (z > 0 ? s0 - sz : s0 + sz * (a.L2 - 1)));
            Zp[0] = zp.x; Zp[1] = zp.y; Zp[2] = zp.z; Zp[3] = zp.w;
            Zm[0] = zm.x; Zm[1] = zm.y; Zm[2] = zm.z; Zm[3] = zm.w;
        }
        const uint32_t W[6] = {Lw, C[0], C[1], C[2], C[3], Rw};
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            uint32_t l = __funnelshift_l(W[w], W[w + 1], 8);
            uint32_t r = __funnelshift_r(W[w + 1], W[w + 2], 8);
            uint32_t s = l + r + U[w] + Dn[w] + Zp[w] + Zm[w];
            K[w] = C[w] + 2u * s;
        }
        // the pass's colour sits at byte offsets b, b+2, ... (x0 even)
        b = (int)((a.color + y + z) & 1u);
        // shift each word by b bytes: colour site i is byte 2*(i&1) of word i>>1
        const uint32_t sh = 8u * (uint32_t)b;
#pragma unroll
        for (int w = 0; w < 4; ++w) K[w] >>= sh;
#pragma unroll
        for (int i = 0; i < 8; ++i)
            if (s_tab[(K[i >> 1] >> (16 * (i & 1))) & 0xFFu] != ~0ull) need_mask |= 1u << i;
    }
    const int need = __popc(need_mask);

    // ---- block scan + decoupled look-back (warp 0 reads 32 predecessors at a time)
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = need;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        int v = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += v;
    }
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    int warp_excl = 0, total = 0;
#pragma unroll
    for (int w = 0; w < SThreads / 32; ++w) {
        int t = warp_tot[w];
        if (w < wid) warp_excl += t;
        total += t;
    }
    const int thread_excl = warp_excl + incl - need;
    if (wid == 0) {
        const uint32_t ep = a.epoch & 0x3FFFFFFFu;
        unsigned long long excl = 0;
        bool fail = false;
        if (chunk == 0) {
            if (lane == 0) atomicExch(&a.desc[0], s_make_desc(a.epoch, 2ull, (uint32_t)total));
        } else {
            if (lane == 0) atomicExch(&a.desc[chunk], s_make_desc(a.epoch, 1ull, (uint32_t)total));
            int64_t top = chunk - 1;  // lane l reads chunk top - l
            int spins = 0;
            while (true) {
                const int64_t idx = top - lane;
                const unsigned long long d = idx >= 0 ? s_ld_relaxed(&a.desc[idx]) : s_make_desc(a.epoch, 2ull, 0u);
                const unsigned long long st = (uint32_t)(d >> 34) == ep ? (d >> 32) & 3ull : 0ull;
                const unsigned incl_lanes = __ballot_sync(0xffffffffu, st == 2ull);
                const unsigned ready = __ballot_sync(0xffffffffu, st != 0ull);
                // lanes up to the nearest inclusive prefix (all 32 when none is in this window)
                const unsigned span = incl_lanes ? (((incl_lanes & (0u - incl_lanes)) << 1) - 1u) : 0xffffffffu;
                if ((ready & span) != span) {
                    if (++spins > SSpinLimit) {
                        fail = true;
                        break;
                    }
                    __nanosleep(32);
                    continue;
                }
                unsigned long long v = ((span >> lane) & 1u) ? (unsigned long long)(uint32_t)d : 0ull;
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
                excl += v;
                if (incl_lanes) break;
                top -= 32;
            }
            if (lane == 0 && !fail)
                atomicExch(&a.desc[chunk], s_make_desc(a.epoch, 2ull, (uint32_t)(excl + total)));
        }
        unsigned long long pass_pos = 0;
        if (lane == 0) {
            s_fail = fail ? 1 : 0;
            if (fail) atomicOr(&a.ctrl->status, kStatusLookbackTimeout);
            pass_pos = a.ctrl->pos[a.pos_in];
            if (chunk == a.n_chunks - 1 && !fail) a.ctrl->pos[a.pos_in ^ 1] = pass_pos + excl + (unsigned long long)total;
        }
        // the chunk's stream state: lanes 0..7 fetch one radix-256 digit's map each and the maps
        // (powers of the same LCG step, so they commute) are composed in a tree
        const unsigned long long n_pos = __shfl_sync(0xffffffffu, pass_pos, 0) + excl;
        Affine f;
        const unsigned dv = lane < kJumpDigits ? (unsigned)((n_pos >> (8 * lane)) & 255u) : 0u;
        if (dv) {
            f = a.jump[lane * kJumpRadix + dv];
        } else {
            f.m.lo = 1; f.m.hi = 0; f.p.lo = 0; f.p.hi = 0;
        }
#pragma unroll
        for (int off = 1; off < kJumpDigits; off <<= 1) {
            Affine g;
            g.m.lo = __shfl_down_sync(0xffffffffu, f.m.lo, off);
            g.m.hi = __shfl_down_sync(0xffffffffu, f.m.hi, off);
            g.p.lo = __shfl_down_sync(0xffffffffu, f.p.lo, off);
            g.p.hi = __shfl_down_sync(0xffffffffu, f.p.hi, off);
            f = compose(f, g);
        }
        if (lane == 0) s_chunk_state = apply(f, a.base);
    }
    __syncthreads();
    if (s_fail || !active) return;

    // ---- draws and decisions
    u128 st = jump_small(a.jump, s_chunk_state, (uint32_t)thread_excl);
    uint32_t flip[4] = {0, 0, 0, 0};  // in the shifted frame
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        bool accept = true;  // downhill: accept without a draw
        if ((need_mask >> i) & 1u) {
            const uint64_t k = draw53(st);
            st = pcg_step(st, a.inc);
            accept = k < s_tab[(K[i >> 1] >> (16 * (i & 1))) & 0xFFu];
        }
        flip[i >> 1] |= (accept ? 1u : 0u) << (16 * (i & 1));
    }
    const uint32_t fsh = 8u * (uint32_t)b;
    *reinterpret_cast<uint4 *>(a.state + s0) = make_uint4(C[0] ^ (flip[0] << fsh), C[1] ^ (flip[1] << fsh),
                                                          C[2] ^ (flip[2] << fsh), C[3] ^ (flip[3] << fsh));
}

bool scan_metro_eligible(int d, const int32_t *L) {
    int64_t n = 1;
    for (int mu = 0; mu < d; ++mu) n *= L[mu];
    return (d == 2 || d == 3) && L[0] % 16 == 0 && L[0] >= 16 && n < (int64_t(1) << 32);
}

int64_t scan_chunks(int64_t n_sites) { return (n_sites + SChunkSites - 1) / SChunkSites; }

cudaError_t launch_scan_metro(const ScanArgs &a, int d, cudaStream_t stream) {
    if (d == 2)
        scan_metro_kernel<2><<<(unsigned)a.n_chunks, SThreads, 0, stream>>>(a);
    else
        scan_metro_kernel<3><<<(unsigned)a.n_chunks, SThreads, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace plq
