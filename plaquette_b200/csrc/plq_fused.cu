// plq_fused.cu -- one launch per sweep: both checkerboard colours of a 3D
// site lattice in a single pass over HBM, out of place (src -> dst).
//
// Equivalent to two colour passes of LocalUpdate::sweep with
// Schedule::Checkerboard (src/updater.rs:316-324) whenever a variable's draw
// is a closed form of its index: the heat bath on the PCG stream (exactly one
// draw per site, position = pass offset + site/2) and every keyed kernel.
//
// A CTA owns a 128 x 16 (x, y) column and marches along z through a ring of
// shared-memory planes, each holding the column with a halo of 2 (16 bytes
// of x halo so every copy is an aligned 16-byte cp.async).  At step z:
//   1. plane z+2 has landed (prefetched FPREF steps ahead);
//   2. colour 0 of plane z+1 is updated in shared memory on the interior and
//      on a one-site ring around it (the ring is recomputed by the
//      neighbouring column too -- same inputs, same draws, same result);
//   3. colour 1 of plane z is updated on the interior from the new colour-0
//      values of planes z-1, z, z+1, and the final plane z goes to dst.
// HBM traffic is one read and one write of every site per sweep (the halo
// re-reads hit L2), i.e. the 2 B/site-update floor.
//
// Neighbour keys are computed four sites at a time in 32-bit words (SWAR):
// states are bytes, and the per-byte neighbour sum of g(state) never
// carries (g = state for q = 2; g = 0,1,7 for q = 3), giving the table key
// cur + q * sum(g) of the host tables.
#include <cuda_runtime.h>

#include "../../include/plaquette.h"
#include "plq_device.cuh"
#include "plq_fused.h"

namespace plq {

constexpr int FX = 128, FY = 16;
constexpr int FPX = FX + 32, FPY = FY + 4, FPLANE = FPX * FPY;  // 3200 bytes
constexpr int FPREF = 3, FNS = FPREF + 5;                      // ring of 8 planes
constexpr int FTHREADS = 256;
constexpr int FCHUNKS = (FPX / 16) * FPY;                       // 200 copies per plane
constexpr int FTABLE_BYTES = 4096;

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_pref() {
    asm volatile("cp.async.wait_group %0;" ::"n"(FPREF) : "memory");
}

__device__ __forceinline__ int wrapi(int v, int L) { return v < 0 ? v + L : (v >= L ? v - L : v); }

// Per-byte sum of g(state) over the six neighbours of the 8-byte run at
// (row base `c` in the centre plane, same offsets in planes m and p), and the
// key word cur + q*sum.
template <int Q>
__device__ __forceinline__ void run_keys(const uint8_t *c, const uint8_t *m, const uint8_t *p, uint32_t &A,
                                         uint32_t &B, uint32_t &KA, uint32_t &KB) {
    uint2 ctr = *reinterpret_cast<const uint2 *>(c);
    A = ctr.x;
    B = ctr.y;
    uint32_t Lw = *reinterpret_cast<const uint32_t *>(c - 4);
    uint32_t Rw = *reinterpret_cast<const uint32_t *>(c + 8);
    uint2 up = *reinterpret_cast<const uint2 *>(c - FPX);
    uint2 dn = *reinterpret_cast<const uint2 *>(c + FPX);
    uint2 zm = *reinterpret_cast<const uint2 *>(m);
    uint2 zp = *reinterpret_cast<const uint2 *>(p);
    uint32_t lA = __funnelshift_l(Lw, A, 8), lB = __funnelshift_l(A, B, 8);
    uint32_t rA = __funnelshift_r(A, B, 8), rB = __funnelshift_r(B, Rw, 8);
    uint32_t sA = lA + rA + up.x + dn.x + zm.x + zp.x;
    uint32_t sB = lB + rB + up.y + dn.y + zm.y + zp.y;
    if (Q == 3) {
        const uint32_t M = 0x01010101u;
        uint32_t tA = ((lA >> 1) & M) + ((rA >> 1) & M) + ((up.x >> 1) & M) + ((dn.x >> 1) & M) +
                      ((zm.x >> 1) & M) + ((zp.x >> 1) & M);
        uint32_t tB = ((lB >> 1) & M) + ((rB >> 1) & M) + ((up.y >> 1) & M) + ((dn.y >> 1) & M) +
                      ((zm.y >> 1) & M) + ((zp.y >> 1) & M);
        sA += tA * 5u;
        sB += tB * 5u;
    }
    KA = A + sA * (uint32_t)Q;
    KB = B + sB * (uint32_t)Q;
}

template <int Q>
__device__ __forceinline__ int g_state(int s) {
    return Q == 3 ? s + 5 * (s >> 1) : s;
}

// One decision from the table in shared memory.
template <int Q, bool STREAM, bool HB>
__device__ __forceinline__ int decide(const void *tab, int key, int cur, uint64_t k) {
    if (HB) {
        if (STREAM) {
            const uint64_t *cut = reinterpret_cast<const uint64_t *>(tab) + key * (Q - 1);
            int ch = k >= cut[0] ? 1 : 0;
            if (Q == 3) ch += k >= cut[1] ? 1 : 0;
            return ch;
        } else {
            const uint32_t *cut = reinterpret_cast<const uint32_t *>(tab) + key * (Q - 1);
            uint32_t k32 = (uint32_t)k;
            int ch = k32 >= cut[0] ? 1 : 0;
            if (Q == 3) ch += k32 >= cut[1] ? 1 : 0;
            return ch;
        }
    } else {  // keyed Metropolis, q = 2
        uint32_t e = reinterpret_cast<const uint32_t *>(tab)[key];
        bool accept = e == 0xFFFFFFFFu || (uint32_t)k < e;
        return accept ? 1 - cur : cur;
    }
}

__device__ __forceinline__ int byte_of(uint32_t A, uint32_t B, int j) {
    return (int)(((j < 4 ? A : B) >> (8 * (j & 3))) & 0xFFu);
}
__device__ __forceinline__ void set_byte(uint32_t &A, uint32_t &B, int j, int v) {
    uint32_t sh = 8u * (uint32_t)(j & 3);
    uint32_t mask = ~(0xFFu << sh);
    if (j < 4)
        A = (A & mask) | ((uint32_t)v << sh);
    else
        B = (B & mask) | ((uint32_t)v << sh);
}

// Updates the four colour-c sites of an 8-site run (first site b of the run
// has colour c).  `st` is the PCG state of the run's first colour-c draw.
template <int Q, bool STREAM, bool HB>
__device__ __forceinline__ void update_run(const FusedArgs &a, const void *tab, uint32_t &A, uint32_t &B,
                                           uint32_t KA, uint32_t KB, int b, uint32_t var0, u128 st) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        int j = b + 2 * i;
        int key = byte_of(KA, KB, j);
        int cur = byte_of(A, B, j);
        uint64_t k;
        if (STREAM) {
            k = draw53(st);
            st = pcg_step(st, a.inc);
        } else {
            k = keyed24(a.seed32, var0 + (uint32_t)j, a.sweep32);
        }
        set_byte(A, B, j, decide<Q, STREAM, HB>(tab, key, cur, k));
    }
}

template <int Q, bool STREAM, bool HB>
__global__ void __launch_bounds__(FTHREADS, 2) fused3d_kernel(FusedArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint8_t *ring = smem;
    uint8_t *tab = smem + FNS * FPLANE;
    const int t = threadIdx.x;
    const int L0 = a.L0, L1 = a.L1, L2 = a.L2;
    const int x0 = blockIdx.x * FX, y0 = blockIdx.y * FY, z0 = blockIdx.z * a.tz;

    // decision table -> shared memory
    {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(a.table);
        uint32_t *dst = reinterpret_cast<uint32_t *>(tab);
        for (int i = t; i < a.table_words; i += FTHREADS) dst[i] = src[i];
    }

    const int zlast = z0 + a.tz + 1;  // last plane the column needs
    auto issue = [&](int zp) {
        if (zp <= zlast && t < FCHUNKS) {
            int row = t / (FPX / 16), cx = t - row * (FPX / 16);
            int gy = wrapi(y0 - 2 + row, L1);
            int gx = wrapi(x0 - 16 + 16 * cx, L0);
            int gz = wrapi(zp, L2);
            const uint8_t *g = a.src + ((size_t)gz * L1 + gy) * L0 + gx;
            uint8_t *s = ring + ((zp + 2 * FNS) % FNS) * FPLANE + row * FPX + 16 * cx;
            cp_async16(s, g);
        }
        cp_commit();
    };
    // prologue: planes z0-2 .. z0+FPREF
    for (int zp = z0 - 2; zp <= z0 + FPREF; ++zp) issue(zp);

    // thread roles
    const int row = t >> 4, r = t & 15;
    const int xo = 16 + 8 * r;           // smem x offset of the run
    const int gxr = x0 + 8 * r;          // global x of the run (even)
    const int gy = y0 + row;
    const bool ringrow = t < 32;
    const int ryy = t < 16 ? 1 : FY + 2; // smem row of the ring row
    const int rgy = wrapi(t < 16 ? y0 - 1 : y0 + FY, L1);
    const bool ringcol = t >= 32 && t < 64;
    const int cu = t - 32;
    const int cxo = cu < 16 ? 15 : 16 + FX;
    const int cgx = wrapi(cu < 16 ? x0 - 1 : x0 + FX, L0);
    const int cyy = 2 + (cu & 15);
    const int cgy = y0 + (cu & 15);

    u128 st0{0, 0}, stR{0, 0}, st1{0, 0};
    const size_t plane_sites = (size_t)L0 * L1;

    for (int z = z0 - 2; z < z0 + a.tz; ++z) {
        cp_wait_pref();
        __syncthreads();
        issue(z + FPREF + 3);

        const int gz1 = wrapi(z + 1, L2), gz0 = wrapi(z, L2);
        const uint8_t *sM = ring + ((z + 2 * FNS) % FNS) * FPLANE;      // plane z
        uint8_t *sC = ring + ((z + 1 + 2 * FNS) % FNS) * FPLANE;        // plane z+1
        const uint8_t *sP = ring + ((z + 2 + 2 * FNS) % FNS) * FPLANE;  // plane z+2
        const size_t zoff1 = (size_t)gz1 * plane_sites;

        // ---- colour 0 on plane z+1 (interior + ring)
        if (STREAM) {
            bool fresh = z == z0 - 2 || gz1 == 0;
            if (fresh) {
                st0 = jump(a.jump, a.base, a.off0 + ((zoff1 + (size_t)gy * L0 + gxr) >> 1));
                if (ringrow) stR = jump(a.jump, a.base, a.off0 + ((zoff1 + (size_t)rgy * L0 + gxr) >> 1));
                if (ringcol) stR = jump(a.jump, a.base, a.off0 + ((zoff1 + (size_t)cgy * L0 + cgx) >> 1));
            } else {
                st0 = apply(a.plane, st0);
                if (ringrow || ringcol) stR = apply(a.plane, stR);
            }
        }
        {
            uint32_t A, B, KA, KB;
            const int yy = row + 2;
            run_keys<Q>(sC + yy * FPX + xo, sM + yy * FPX + xo, sP + yy * FPX + xo, A, B, KA, KB);
            update_run<Q, STREAM, HB>(a, tab, A, B, KA, KB, (gy + gz1) & 1,
                                      (uint32_t)(zoff1 + (size_t)gy * L0 + gxr), st0);
            uint32_t RA = 0, RB = 0;
            if (ringrow) {
                uint32_t RKA, RKB;
                run_keys<Q>(sC + ryy * FPX + xo, sM + ryy * FPX + xo, sP + ryy * FPX + xo, RA, RB, RKA, RKB);
                update_run<Q, STREAM, HB>(a, tab, RA, RB, RKA, RKB, (rgy + gz1) & 1,
                                          (uint32_t)(zoff1 + (size_t)rgy * L0 + gxr), stR);
            }
            int cres = -1;
            if (ringcol && ((cgx + cgy + gz1) & 1) == 0) {
                const uint8_t *cc = sC + cyy * FPX + cxo;
                int cur = cc[0];
                int sum = g_state<Q>(cc[-1]) + g_state<Q>(cc[1]) + g_state<Q>(cc[-FPX]) + g_state<Q>(cc[FPX]) +
                          g_state<Q>(sM[cyy * FPX + cxo]) + g_state<Q>(sP[cyy * FPX + cxo]);
                uint64_t k;
                if (STREAM) k = draw53(stR);
                else k = keyed24(a.seed32, (uint32_t)(zoff1 + (size_t)cgy * L0 + cgx), a.sweep32);
                cres = decide<Q, STREAM, HB>(tab, cur + Q * sum, cur, k);
            }
            __syncthreads();  // every colour-0 input has been read; now publish
            *reinterpret_cast<uint2 *>(sC + yy * FPX + xo) = make_uint2(A, B);
            if (ringrow) *reinterpret_cast<uint2 *>(sC + ryy * FPX + xo) = make_uint2(RA, RB);
            if (cres >= 0) sC[cyy * FPX + cxo] = (uint8_t)cres;
        }
        __syncthreads();

        // ---- colour 1 on plane z (interior), store
        if (z >= z0) {
            const size_t zoff0 = (size_t)gz0 * plane_sites;
            if (STREAM) {
                if (z == z0 || gz0 == 0)
                    st1 = jump(a.jump, a.base, a.off1 + ((zoff0 + (size_t)gy * L0 + gxr) >> 1));
                else
                    st1 = apply(a.plane, st1);
            }
            const uint8_t *zM = ring + ((z - 1 + 2 * FNS) % FNS) * FPLANE;
            const uint8_t *zC = sM;
            const uint8_t *zP = sC;
            int yy = row + 2;
            uint32_t A, B, KA, KB;
            run_keys<Q>(zC + yy * FPX + xo, zM + yy * FPX + xo, zP + yy * FPX + xo, A, B, KA, KB);
            int b = (gy + gz0 + 1) & 1;
            update_run<Q, STREAM, HB>(a, tab, A, B, KA, KB, b, (uint32_t)(zoff0 + (size_t)gy * L0 + gxr), st1);
            *reinterpret_cast<uint2 *>(a.dst + zoff0 + (size_t)gy * L0 + gxr) = make_uint2(A, B);
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
}

bool fused3d_eligible(int model, int q, int d, const int32_t *L, int updater, int rng) {
    if (d != 3 || model == PLQ_GAUGE) return false;
    if (q != 2 && q != 3) return false;
    if (L[0] % FX || L[1] % FY || L[2] % 8) return false;
    if (updater == PLQ_METROPOLIS && !(rng == PLQ_RNG_KEYED && q == 2)) return false;
    return true;
}

int fused3d_default_tz(int L2) {
    for (int tz : {64, 32, 16, 8})
        if (L2 % tz == 0) return tz;
    return 0;
}

size_t fused3d_smem_bytes() { return (size_t)FNS * FPLANE + FTABLE_BYTES; }
int fused3d_table_limit_bytes() { return FTABLE_BYTES; }

template <int Q, bool STREAM, bool HB>
static cudaError_t launch_t(const FusedArgs &a, cudaStream_t s) {
    auto kern = fused3d_kernel<Q, STREAM, HB>;
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fused3d_smem_bytes());
        configured = true;
    }
    dim3 grid(a.L0 / FX, a.L1 / FY, a.L2 / a.tz);
    kern<<<grid, FTHREADS, fused3d_smem_bytes(), s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_fused3d(const FusedArgs &a, int q, bool stream, bool hb, cudaStream_t s) {
    if (q == 2) {
        if (hb) return stream ? launch_t<2, true, true>(a, s) : launch_t<2, false, true>(a, s);
        return launch_t<2, false, false>(a, s);
    }
    if (q == 3 && hb) return stream ? launch_t<3, true, true>(a, s) : launch_t<3, false, true>(a, s);
    return cudaErrorInvalidValue;
}

}  // namespace plq
