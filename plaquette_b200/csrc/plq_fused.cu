// plq_fused.cu -- one launch per sweep: both checkerboard colours of a 3D
// site lattice in a single pass over HBM, out of place (src -> dst).
//
// Equivalent to the two colour passes of LocalUpdate::sweep with
// Schedule::Checkerboard (src/updater.rs:316-324) whenever a variable's draw
// is a closed form of its index: the heat bath on the PCG stream (exactly one
// draw per site, position = pass offset + site/2) and every keyed kernel.
//
// A CTA owns full x-rows (L0 = 128, 256 or 512, so x wraps inside
// shared memory) for TY = 8192/L0 rows of y, and marches along z through a
// ring of shared-memory planes with a y halo of 2.  At step z:
//   1. plane z+2 has landed (prefetched FPREF steps ahead as three TMA boxes
//      -- TY interior rows and two wrapped 2-row halos -- on the slot's mbarrier);
//   2. colour 0 of plane z+1 is updated in shared memory on the interior rows
//      and on the two ring rows y0-1 and y0+TY (recomputed by the
//      neighbouring tile too -- same inputs, same draws, same result);
//   3. colour 1 of plane z is updated on the interior from the new colour-0
//      values of planes z-1, z, z+1, and the final plane z goes to dst.
// HBM traffic: one read and one write of every site per sweep (halo re-reads
// hit L2), the 2 B/site-update floor.  Every thread does the same work: two
// interior runs of 16 sites per colour phase plus one 4-site word of ring.
//
// Neighbour keys are computed four sites per 32-bit word (SWAR): states are
// bytes and the per-byte neighbour sum of g(state) never carries (g = state
// for q = 2; g = 0,1,7 for q = 3), giving the table key cur + q*sum(g).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <climits>

#include "../../include/plaquette.h"
#include "plq_device.cuh"
#include "plq_fused.h"

namespace plq {

constexpr int FTHREADS = 256;
constexpr int FRUN = 16;                      // bytes per run
constexpr int FRUNS_PER_THREAD = 2;
constexpr int FPLANE_SITES = FTHREADS * FRUNS_PER_THREAD * FRUN;  // 8192 interior sites per plane
// Ring depth and CTAs per SM by kernel variant: planes are prefetched FPREF
// steps ahead into a ring of FPREF + 5 slots (planes z-1..z+2 in use, z+3..
// z+FPREF+3 in flight).  Three CTAs per SM (FPREF 2, 75 KB of shared memory
// each) measured faster for all but the keyed q = 3 heat bath (two CTAs, FPREF 3).
template <int Q, bool STREAM>
struct FusedCfg {
    static constexpr int ctas = (Q == 3 && !STREAM) ? 2 : 3;
    static constexpr int pref = ctas == 3 ? 2 : 3;
    static constexpr int slots = pref + 5;
};
constexpr int FTABLE_BYTES = 4096;
constexpr int FMAX_L0 = 512;  // 2 ring rows of L0/4 words: one word per thread

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// Waits for the phase of the given parity to complete; false after `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int limit) {
    for (int i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// One TMA box of full rows (x = 0, rows from y, plane z) into shared memory,
// completing on `bar` with its byte count.  No multicast.
__device__ __forceinline__ void tma_rows(void *dst, const CUtensorMap *map, int y, int z, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(0), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ int wrapi(int v, int L) { return v < 0 ? v + L : (v >= L ? v - L : v); }

// Per-byte g(state) of a word.
template <int Q>
__device__ __forceinline__ uint32_t gw(uint32_t w) {
    if (Q == 3) return w + ((w >> 1) & 0x01010101u) * 5u;
    return w;
}

// Keys of the 4 sites of word C given its six neighbour words.  For q = 3,
// sum g = raw + 5*hi with hi the per-byte count of state-2 neighbours; the
// masked bits (value 2 per state-2 neighbour) are summed first and the key is
// C + 3*raw + 15*hi2/2, where each byte of 15*hi2 is even and at most 180, so
// the final shift moves no bit across a byte boundary.
template <int Q>
__device__ __forceinline__ uint32_t key_word(uint32_t C, uint32_t l, uint32_t r, uint32_t u, uint32_t d,
                                             uint32_t m, uint32_t p) {
    const uint32_t raw = l + r + u + d + m + p;
    if (Q == 3) {
        const uint32_t M2 = 0x02020202u;
        const uint32_t hi2 = (l & M2) + (r & M2) + (u & M2) + (d & M2) + (m & M2) + (p & M2);
        return C + raw * 3u + ((hi2 * 15u) >> 1);
    }
    return C + raw * (uint32_t)Q;
}

// Table decision for one site; returns the new state.
template <int Q, bool STREAM, bool HB>
__device__ __forceinline__ uint32_t decide(const uint8_t *tab, uint32_t key, uint32_t cur, uint64_t k) {
    if (HB) {
        if (STREAM) {
            if (Q == 3) {  // both cut points of a key in one 16-byte load
                const ulonglong2 cut = reinterpret_cast<const ulonglong2 *>(tab)[key];
                return (k >= cut.x ? 1u : 0u) + (k >= cut.y ? 1u : 0u);
            }
            return k >= reinterpret_cast<const uint64_t *>(tab)[key] ? 1u : 0u;
        } else {
            const uint32_t *cut = reinterpret_cast<const uint32_t *>(tab) + key * (Q - 1);
            uint32_t k32 = (uint32_t)k;
            uint32_t ch = k32 >= cut[0] ? 1u : 0u;
            if (Q == 3) ch += k32 >= cut[1] ? 1u : 0u;
            return ch;
        }
    } else {  // keyed Metropolis, q = 2: kAlways24 exceeds every 24-bit k
        uint32_t e = reinterpret_cast<const uint32_t *>(tab)[key];
        return cur ^ ((uint32_t)k < e ? 1u : 0u);
    }
}

// Updates the colour-c sites (byte offsets b, b+2) of one 32-bit word in place:
// the word and its keys are shifted by b bytes once, so both sites sit at fixed
// byte offsets 0 and 2.
template <int Q, bool STREAM, bool HB>
__device__ __forceinline__ uint32_t update_word(const FusedArgs &a, const uint8_t *tab, uint32_t C, uint32_t K,
                                                int b, uint32_t var0, u128 &st) {
    const uint32_t sh = 8u * (uint32_t)b;
    const uint32_t Cs = C >> sh, Ks = K >> sh;
    uint32_t delta = 0;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const uint32_t key = (Ks >> (16 * i)) & 0xFFu;
        const uint32_t cur = (Cs >> (16 * i)) & 0xFFu;
        uint64_t k;
        if (STREAM) {
            k = xsl_rr(st);  // all 64 bits: the table holds the 53-bit cut points << 11
            st = pcg_step(st, a.inc);
        } else {
            k = keyed24(a.seed32, var0 + (uint32_t)(b + 2 * i), a.sweep32);
        }
        const uint32_t nv = decide<Q, STREAM, HB>(tab, key, cur, k);
        delta |= (nv ^ cur) << (16 * i);
    }
    return C ^ (delta << sh);
}

// A run of 16 bytes at x offset xr of smem row `row` (plane c, neighbours in
// planes m and p); rows are L0 bytes, x wraps.
template <int Q, bool STREAM, bool HB>
__device__ __forceinline__ uint4 update_run(const FusedArgs &a, const uint8_t *tab, const uint8_t *pc,
                                            const uint8_t *pm, const uint8_t *pp, int row, int xr, int L0,
                                            int b, uint32_t var0, u128 &st) {
    const int off = row * L0 + xr;
    uint4 C = *reinterpret_cast<const uint4 *>(pc + off);
    uint4 U = *reinterpret_cast<const uint4 *>(pc + off - L0);
    uint4 D = *reinterpret_cast<const uint4 *>(pc + off + L0);
    uint4 M = *reinterpret_cast<const uint4 *>(pm + off);
    uint4 P = *reinterpret_cast<const uint4 *>(pp + off);
    uint32_t Lw = *reinterpret_cast<const uint32_t *>(pc + row * L0 + ((xr - 4) & (L0 - 1)));
    uint32_t Rw = *reinterpret_cast<const uint32_t *>(pc + row * L0 + ((xr + 16) & (L0 - 1)));
    uint32_t K0 = key_word<Q>(C.x, __funnelshift_l(Lw, C.x, 8), __funnelshift_r(C.x, C.y, 8), U.x, D.x, M.x, P.x);
    uint32_t K1 = key_word<Q>(C.y, __funnelshift_l(C.x, C.y, 8), __funnelshift_r(C.y, C.z, 8), U.y, D.y, M.y, P.y);
    uint32_t K2 = key_word<Q>(C.z, __funnelshift_l(C.y, C.z, 8), __funnelshift_r(C.z, C.w, 8), U.z, D.z, M.z, P.z);
    uint32_t K3 = key_word<Q>(C.w, __funnelshift_l(C.z, C.w, 8), __funnelshift_r(C.w, Rw, 8), U.w, D.w, M.w, P.w);
    uint4 O;
    O.x = update_word<Q, STREAM, HB>(a, tab, C.x, K0, b, var0, st);
    O.y = update_word<Q, STREAM, HB>(a, tab, C.y, K1, b, var0 + 4, st);
    O.z = update_word<Q, STREAM, HB>(a, tab, C.z, K2, b, var0 + 8, st);
    O.w = update_word<Q, STREAM, HB>(a, tab, C.w, K3, b, var0 + 12, st);
    return O;
}

template <int Q, bool STREAM, bool HB>
__global__ void __launch_bounds__(FTHREADS, FusedCfg<Q, STREAM>::ctas)
    fused3d_kernel(const FusedArgs a, const __grid_constant__ CUtensorMap tm_rows,
                   const __grid_constant__ CUtensorMap tm_halo) {
    constexpr int FPREF = FusedCfg<Q, STREAM>::pref, FNS = FusedCfg<Q, STREAM>::slots;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // TMA destinations start on 128-byte boundaries: align the base here
    // (the launch reserves 128 bytes for it) rather than trust the window's.
    uint8_t *smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
    const int L0 = a.L0, L1 = a.L1, L2 = a.L2, TY = a.ty;
    const int plane_bytes = L0 * (TY + 4);
    uint8_t *ring = smem;
    uint8_t *tab = smem + FNS * plane_bytes;
    uint64_t *bars = reinterpret_cast<uint64_t *>(tab + FTABLE_BYTES);
    const int t = threadIdx.x;
    const int y0 = blockIdx.x * TY, z0 = blockIdx.y * a.tz;

    if (t == 0) {
        for (int i = 0; i < FNS; ++i) mbar_init(&bars[i], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(a.table);
        uint32_t *dst = reinterpret_cast<uint32_t *>(tab);
        for (int i = t; i < a.table_words; i += FTHREADS) dst[i] = src[i];
    }
    __syncthreads();

    // Plane zp (zfirst <= zp <= zlast) lives in ring slot (zp - zfirst) % FNS;
    // its fill is that slot's use number (zp - zfirst) / FNS, whose parity the
    // waits name.  Thread 0 issues every plane as three TMA boxes: the TY
    // interior rows and the two 2-row y halos (wrapped, so each is contiguous).
    const int zfirst = z0 - 2, zlast = z0 + a.tz + 1;
    auto slot = [&](int zp) { return (zp - zfirst) % FNS; };
    auto parity = [&](int zp) { return (uint32_t)(((zp - zfirst) / FNS) & 1); };
    auto issue = [&](int zp) {
        if (zp <= zlast && !(a.stall && zp == zfirst + 4)) {
            const int gz = wrapi(zp, L2);
            uint8_t *dst = ring + slot(zp) * plane_bytes;
            uint64_t *bar = &bars[slot(zp)];
            mbar_expect_tx(bar, (uint32_t)plane_bytes);
            tma_rows(dst + 2 * L0, &tm_rows, y0, gz, bar);
            tma_rows(dst, &tm_halo, wrapi(y0 - 2, L1), gz, bar);
            tma_rows(dst + (TY + 2) * L0, &tm_halo, wrapi(y0 + TY, L1), gz, bar);
        }
    };
    if (t == 0)
        for (int zp = zfirst; zp <= z0 + FPREF; ++zp) issue(zp);

    // interior runs u = t + 256k: smem row 2 + u / runs_per_row, x = 16 * (u % runs_per_row)
    const int runs_per_row = L0 / FRUN;
    int rrow[FRUNS_PER_THREAD], rx[FRUNS_PER_THREAD], rgy[FRUNS_PER_THREAD];
#pragma unroll
    for (int k = 0; k < FRUNS_PER_THREAD; ++k) {
        int u = t + FTHREADS * k;
        rrow[k] = 2 + u / runs_per_row;
        rx[k] = FRUN * (u % runs_per_row);
        rgy[k] = y0 + rrow[k] - 2;
    }
    // ring words: w = t < L0/2: smem row 1 or TY+2, x = 4 * (w % (L0/4))
    const bool has_ring = t < L0 / 2;
    const int wq = L0 / 4;
    const int ring_row = (t / wq) == 0 ? 1 : TY + 2;
    const int ring_x = 4 * (t % wq);
    const int ring_gy = wrapi(ring_row == 1 ? y0 - 1 : y0 + TY, L1);

    u128 st0[FRUNS_PER_THREAD], st1[FRUNS_PER_THREAD], stR;
    const size_t plane_sites = (size_t)L0 * L1;

    int z_abort = INT_MAX;
    for (int z = zfirst; z < z0 + a.tz; ++z) {
        // planes z and z+1 landed at earlier steps (both at the first), z+2 now
        bool landed = true;
        if (z == zfirst)
            landed = mbar_wait(&bars[slot(z)], parity(z), a.wait_limit) &&
                      mbar_wait(&bars[slot(z + 1)], parity(z + 1), a.wait_limit);
        landed = landed && mbar_wait(&bars[slot(z + 2)], parity(z + 2), a.wait_limit);
        if (__syncthreads_or(!landed)) {
            z_abort = z;
            break;
        }
        if (t == 0) {
            // every thread's reads and writes of the slot refilled next are done
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue(z + FPREF + 3);
        }

        const int gz1 = wrapi(z + 1, L2), gz0 = wrapi(z, L2);
        const uint8_t *sM = ring + slot(z) * plane_bytes;      // plane z
        uint8_t *sC = ring + slot(z + 1) * plane_bytes;        // plane z+1
        const uint8_t *sP = ring + slot(z + 2) * plane_bytes;  // plane z+2
        const size_t zoff1 = (size_t)gz1 * plane_sites;

        // ---- colour 0 of plane z+1: interior runs and the ring word
        if (STREAM) {
            bool fresh = z == z0 - 2 || gz1 == 0;
#pragma unroll
            for (int k = 0; k < FRUNS_PER_THREAD; ++k)
                st0[k] = fresh ? jump(a.jump, a.base, a.off0 + ((zoff1 + (size_t)rgy[k] * L0 + rx[k]) >> 1))
                               : apply(a.plane, st0[k]);
            if (has_ring)
                stR = fresh ? jump(a.jump, a.base, a.off0 + ((zoff1 + (size_t)ring_gy * L0 + ring_x) >> 1))
                            : apply(a.plane, stR);
        }
        uint4 out0[FRUNS_PER_THREAD];
#pragma unroll
        for (int k = 0; k < FRUNS_PER_THREAD; ++k) {
            u128 st = st0[k];
            out0[k] = update_run<Q, STREAM, HB>(a, tab, sC, sM, sP, rrow[k], rx[k], L0, (rgy[k] + gz1) & 1,
                                                (uint32_t)(zoff1 + (size_t)rgy[k] * L0 + rx[k]), st);
        }
        uint32_t outR = 0;
        if (has_ring) {
            const int off = ring_row * L0 + ring_x;
            uint32_t C = *reinterpret_cast<const uint32_t *>(sC + off);
            uint32_t Lw = *reinterpret_cast<const uint32_t *>(sC + ring_row * L0 + ((ring_x - 4) & (L0 - 1)));
            uint32_t Rw = *reinterpret_cast<const uint32_t *>(sC + ring_row * L0 + ((ring_x + 4) & (L0 - 1)));
            uint32_t K = key_word<Q>(C, __funnelshift_l(Lw, C, 8), __funnelshift_r(C, Rw, 8),
                                     *reinterpret_cast<const uint32_t *>(sC + off - L0),
                                     *reinterpret_cast<const uint32_t *>(sC + off + L0),
                                     *reinterpret_cast<const uint32_t *>(sM + off),
                                     *reinterpret_cast<const uint32_t *>(sP + off));
            u128 st = stR;
            outR = update_word<Q, STREAM, HB>(a, tab, C, K, (ring_gy + gz1) & 1,
                                              (uint32_t)(zoff1 + (size_t)ring_gy * L0 + ring_x), st);
        }
        __syncthreads();  // all colour-0 inputs read; publish
#pragma unroll
        for (int k = 0; k < FRUNS_PER_THREAD; ++k)
            *reinterpret_cast<uint4 *>(sC + rrow[k] * L0 + rx[k]) = out0[k];
        if (has_ring) *reinterpret_cast<uint32_t *>(sC + ring_row * L0 + ring_x) = outR;
        __syncthreads();

        // ---- colour 1 of plane z: interior runs, stored to dst
        if (z >= z0) {
            const size_t zoff0 = (size_t)gz0 * plane_sites;
            const uint8_t *zM = ring + slot(z - 1) * plane_bytes;
            // both runs first, then the stores: a store to dst between them would order the
            // second run's shared-memory reads after it and keep the two draw chains apart
            uint4 out1[FRUNS_PER_THREAD];
#pragma unroll
            for (int k = 0; k < FRUNS_PER_THREAD; ++k) {
                if (STREAM)
                    st1[k] = (z == z0 || gz0 == 0)
                                 ? jump(a.jump, a.base, a.off1 + ((zoff0 + (size_t)rgy[k] * L0 + rx[k]) >> 1))
                                 : apply(a.plane, st1[k]);
                u128 st = st1[k];
                out1[k] = update_run<Q, STREAM, HB>(a, tab, sM, zM, sC, rrow[k], rx[k], L0, (rgy[k] + gz0 + 1) & 1,
                                                    (uint32_t)(zoff0 + (size_t)rgy[k] * L0 + rx[k]), st);
            }
#pragma unroll
            for (int k = 0; k < FRUNS_PER_THREAD; ++k)
                *reinterpret_cast<uint4 *>(a.dst + zoff0 + (size_t)rgy[k] * L0 + rx[k]) = out1[k];
        }
    }
    if (z_abort != INT_MAX && t == 0) {
        // a plane never landed: report, and let the copies already issued finish (bounded) before exit
        atomicOr(a.status, kStatusCopyTimeout);
        const int last = min(zlast, z_abort + FPREF + 2);
        for (int zp = z_abort; zp <= last; ++zp) mbar_wait(&bars[slot(zp)], parity(zp), a.wait_limit);
    }
}

static int fused_ty(int L0) { return FPLANE_SITES / L0; }

bool fused3d_eligible(int model, int q, int d, const int32_t *L, int updater, int rng) {
    if (d != 3 || model == PLQ_GAUGE) return false;
    if (q != 2 && q != 3) return false;
    const int L0 = L[0];
    if (L0 < 128 || L0 > FMAX_L0 || (L0 & (L0 - 1))) return false;
    if (L[1] % fused_ty(L0) || L[2] % 8 || L[1] < fused_ty(L0)) return false;
    if (updater == PLQ_METROPOLIS && !(rng == PLQ_RNG_KEYED && q == 2)) return false;
    return true;
}

int fused3d_default_tz(int L2) {
    for (int tz : {32, 16, 8})
        if (L2 % tz == 0) return tz;
    return 0;
}

size_t fused3d_smem_bytes(int L0, int slots) {
    return 128 + (size_t)slots * (size_t)L0 * (size_t)(fused_ty(L0) + 4) + FTABLE_BYTES + slots * sizeof(uint64_t);
}
int fused3d_table_limit_bytes() { return FTABLE_BYTES; }

static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
        return nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
}

cudaError_t fused3d_make_maps(const uint8_t *buf, int L0, int L1, int L2, FusedMaps *out) {
    static const PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (!encode) return cudaErrorNotSupported;
    // u8 [L2][L1][L0/X][X]: rows of L0 bytes land densely in shared memory
    const cuuint32_t X = (cuuint32_t)(L0 < 256 ? L0 : 256);
    const cuuint64_t dims[4] = {X, (cuuint64_t)(L0 / (int)X), (cuuint64_t)L1, (cuuint64_t)L2};
    const cuuint64_t strides[3] = {X, (cuuint64_t)L0, (cuuint64_t)L0 * (cuuint64_t)L1};
    const cuuint32_t elem[4] = {1, 1, 1, 1};
    const cuuint32_t box_rows[4] = {X, (cuuint32_t)(L0 / (int)X), (cuuint32_t)fused_ty(L0), 1};
    const cuuint32_t box_halo[4] = {X, (cuuint32_t)(L0 / (int)X), 2, 1};
    for (int k = 0; k < 2; ++k) {
        CUresult r = encode(k ? &out->halo : &out->rows, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, const_cast<uint8_t *>(buf),
                            dims, strides, k ? box_halo : box_rows, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
                            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    }
    return cudaSuccess;
}

template <int Q, bool STREAM, bool HB>
static cudaError_t launch_t(FusedArgs a, const FusedMaps &m, cudaStream_t s) {
    auto kern = fused3d_kernel<Q, STREAM, HB>;
    size_t smem = fused3d_smem_bytes(a.L0, FusedCfg<Q, STREAM>::slots);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    a.ty = fused_ty(a.L0);
    dim3 grid(a.L1 / a.ty, a.L2 / a.tz);
    kern<<<grid, FTHREADS, smem, s>>>(a, m.rows, m.halo);
    return cudaGetLastError();
}

cudaError_t launch_fused3d(const FusedArgs &a, const FusedMaps &m, int q, bool stream, bool hb, cudaStream_t s) {
    if (q == 2) {
        if (hb) return stream ? launch_t<2, true, true>(a, m, s) : launch_t<2, false, true>(a, m, s);
        return launch_t<2, false, false>(a, m, s);
    }
    if (q == 3 && hb) return stream ? launch_t<3, true, true>(a, m, s) : launch_t<3, false, true>(a, m, s);
    return cudaErrorInvalidValue;
}

}  // namespace plq
