// plq_slab.cu -- one slab of a site lattice split along its last axis.
//
// A rank holds planes [z0, z0 + nz) of an Ising or Potts site lattice of
// dimension 2 or 3 (the split axis is the last one: y in 2D, z in 3D), in a
// buffer of nz + 2 planes: plane 0 is the low halo (the previous rank's last
// plane), planes 1..nz its own, plane nz + 1 the high halo (the next rank's
// first plane).  A colour pass updates the colour's sites of planes 1..nz
// exactly as the whole-lattice keyed pass does (plq_local_impl.cuh, the
// reference's site_schedule.wgsl:15-31 with metropolis.wgsl:32-63 or
// heat_bath.wgsl:28-62): the environment key cur + q * sum pw[neighbour]
// looked up in the same cut-point tables, the keyed draw of the site's index
// in the whole lattice and the shared sweep index.  Neighbours along the
// split axis are the adjacent planes (halos at the ends), along the other
// axes periodic within the plane.  The halos are filled by the caller
// between passes (plaquette_b200/slabs.py: neighbour send/recv over
// torch.distributed, or copies when the ring shares a process).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>

#include "../../include/plaquette.h"
#include "plq_abi_internal.h"
#include "plq_local_impl.cuh"
#include "plq_rng.cuh"
#include "plq_tables.h"

namespace {

using namespace plq;

constexpr int kSlabThreads = 256;

struct SlabArgs {
    uint8_t *state;          // nz + 2 planes
    int L0, L1;              // in-plane extents (L1 = 1 in 2D)
    int nz;
    int q, kernel;
    int32_t pw[64];
    const uint32_t *metro24;
    const uint32_t *hb24;
    uint32_t seed32, sweep32;
    int local_colour;        // the pass's colour in the buffer's parity (x + y + local plane)
    int64_t var_offset;      // whole-lattice index of buffer site 0
};

// One thread per site of the colour on the slab's own planes: rank r ->
// (local plane 1 + r / per_plane, in-plane colour rank), then x from the
// parity rule (L0 even).
__global__ void __launch_bounds__(kSlabThreads) slab_pass_kernel(SlabArgs a) {
    const int64_t plane = (int64_t)a.L0 * a.L1;
    const int64_t per_plane = plane / 2;
    const int64_t total = per_plane * a.nz;
    const int half0 = a.L0 / 2;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < total;
         r += (int64_t)gridDim.x * blockDim.x) {
        const int zl = 1 + (int)(r / per_plane);
        const int64_t rp = r - (int64_t)(zl - 1) * per_plane;
        const int y = (int)(rp / half0);
        const int x = 2 * (int)(rp - (int64_t)y * half0) + ((y + zl + a.local_colour) & 1);
        const int64_t row = ((int64_t)zl * a.L1 + y) * a.L0;
        const int64_t s = row + x;
        const int cur = a.state[s];
        uint8_t nb[6];
        int k = 0;
        nb[k++] = a.state[row + (x + 1 < a.L0 ? x + 1 : 0)];
        nb[k++] = a.state[row + (x > 0 ? x - 1 : a.L0 - 1)];
        if (a.L1 > 1) {
            const int64_t pbase = (int64_t)zl * a.L1 * a.L0;
            nb[k++] = a.state[pbase + (int64_t)(y + 1 < a.L1 ? y + 1 : 0) * a.L0 + x];
            nb[k++] = a.state[pbase + (int64_t)(y > 0 ? y - 1 : a.L1 - 1) * a.L0 + x];
        }
        nb[k++] = a.state[s + plane];
        nb[k++] = a.state[s - plane];
        int64_t packed = 0;
        for (int i = 0; i < k; ++i) packed += a.pw[nb[i]];
        const int64_t key = cur + (int64_t)a.q * packed;
        const uint32_t var = (uint32_t)(s + a.var_offset);
        int out;
        if (a.kernel == PLQ_METROPOLIS) {
            int prop;
            int64_t mkey = key;
            if (a.q == 2) {
                prop = 1 - cur;
            } else {
                // keyed proposal (metropolis.wgsl:45-55), then the Potts key
                const uint32_t k24 = keyed24(a.seed32 ^ kProposalKey, var, a.sweep32);
                const float u = __fmul_rn((float)k24, 5.9604644775390625e-8f);
                const float scaled = __fmul_rn(u, (float)(a.q - 1));
                uint32_t draw = __float2uint_rz(scaled);
                if (draw >= (uint32_t)(a.q - 1)) draw = (uint32_t)(a.q - 2);
                prop = (int)draw;
                if (prop >= cur) prop += 1;
                int cp = 0, cc = 0;
                for (int i = 0; i < k; ++i) {
                    cp += nb[i] == prop;
                    cc += nb[i] == cur;
                }
                const int64_t B = k + 1;
                mkey = (((int64_t)cur * a.q + prop) * B + cp) * B + cc;
            }
            const uint32_t e = a.metro24[mkey];
            const uint32_t kd = keyed24(a.seed32, var, a.sweep32);
            out = (e == 0xFFFFFFFFu || kd < e) ? prop : cur;
        } else {
            const uint32_t kd = keyed24(a.seed32, var, a.sweep32);
            out = hb_choose(a.hb24 + key * (a.q - 1), a.q - 1, (uint64_t)kd);
        }
        a.state[s] = (uint8_t)out;
    }
}

}  // namespace

struct plq_slab {
    plq_ctx ctx_copy;
    plq_chain_desc desc;
    int d = 3, q = 2;
    int L0 = 0, L1 = 1;
    int64_t z0 = 0, nz = 0, plane = 0;
    uint8_t *d_state = nullptr;  // nz + 2 planes
    uint32_t *d_metro24 = nullptr, *d_hb24 = nullptr;
    int32_t pw[64];
    uint32_t seed32 = 0;
    uint64_t sweep = 0;
    cudaStream_t stream = nullptr;
};

namespace {

void slab_free(plq_slab *s) {
    if (!s) return;
    cudaSetDevice(s->ctx_copy.device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    cudaFree(s->d_state);
    cudaFree(s->d_metro24);
    cudaFree(s->d_hb24);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

int slab_cuda(plq_slab *s, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return PLQ_OK;
    (void)s;
    return plq_fail(PLQ_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

extern "C" int plq_slab_create(plq_ctx *ctx, const plq_chain_desc *desc, int64_t z0, int64_t nz,
                               const uint8_t *start, plq_slab **out) {
    if (!ctx || !desc || !out || !start) return plq_fail(PLQ_EINVAL, "bad arguments");
    *out = nullptr;
    const int rc = plq_chain_validate(desc);
    if (rc != PLQ_OK) return rc;
    const plq_chain_desc &d = *desc;
    if (d.rng != PLQ_RNG_KEYED || (d.model != PLQ_ISING && d.model != PLQ_POTTS) ||
        (d.updater != PLQ_METROPOLIS && d.updater != PLQ_HEATBATH) || (d.d != 2 && d.d != 3))
        return plq_fail(PLQ_EUNSUPPORTED,
                        "a slab holds a 2D or 3D Ising or Potts site lattice on the keyed stream, "
                        "updated by Metropolis or heat bath");
    const int64_t Lz = d.shape[d.d - 1];
    if (z0 < 0 || nz < 1 || z0 + nz > Lz) return plq_fail(PLQ_EINVAL, "slab planes out of the lattice");
    plq_slab *s = new plq_slab();
    s->ctx_copy = *ctx;
    s->desc = d;
    s->d = d.d;
    s->q = d.model == PLQ_POTTS ? d.q : 2;
    s->L0 = (int)d.shape[0];
    s->L1 = d.d == 3 ? (int)d.shape[1] : 1;
    s->z0 = z0;
    s->nz = nz;
    s->plane = (int64_t)s->L0 * s->L1;
    s->seed32 = plq_fold_seed(d.seed);
    s->sweep = d.sweep_offset;
    if (first_state_at_least(start, nz * s->plane, s->q) >= 0) {
        delete s;
        return plq_fail(PLQ_EINVAL, "start state out of range");
    }
    // the decision tables of the whole lattice's model and beta (plq_tables.cpp)
    ModelParams p;
    std::memset(&p, 0, sizeof p);
    p.model = d.model;
    p.q = s->q;
    p.d = d.d;
    p.beta = d.beta;
    p.j = d.j;
    p.h = d.h;
    for (int k = 0; k < PLQ_MAX_Q; ++k) p.offsets[k] = d.offsets[k];
    Tables t;
    std::string err;
    if (!build_tables(p, d.updater, d.rng, t, err)) {
        delete s;
        return plq_fail(PLQ_EUNSUPPORTED, err);
    }
    int32_t w = 1;
    std::memset(s->pw, 0, sizeof s->pw);
    for (int k = 1; k < s->q; ++k) {
        s->pw[k] = w;
        w *= 2 * d.d + 1;
    }
    cudaError_t e = plq_enter_device(ctx->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc((void **)&s->d_state, (size_t)((nz + 2) * s->plane));
    if (e == cudaSuccess && !t.metro24.empty()) e = cudaMalloc((void **)&s->d_metro24, t.metro24.size() * 4);
    if (e == cudaSuccess && !t.hb24.empty()) e = cudaMalloc((void **)&s->d_hb24, t.hb24.size() * 4);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->d_state + s->plane, start, (size_t)(nz * s->plane), cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess && s->d_metro24)
        e = cudaMemcpyAsync(s->d_metro24, t.metro24.data(), t.metro24.size() * 4, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess && s->d_hb24)
        e = cudaMemcpyAsync(s->d_hb24, t.hb24.data(), t.hb24.size() * 4, cudaMemcpyHostToDevice, s->stream);
    // halos start as zeros; the first exchange fills them
    if (e == cudaSuccess) e = cudaMemsetAsync(s->d_state, 0, (size_t)s->plane, s->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->d_state + (nz + 1) * s->plane, 0, (size_t)s->plane, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) {
        slab_free(s);
        return plq_fail(PLQ_ECUDA, std::string("slab set-up: ") + cudaGetErrorString(e));
    }
    *out = s;
    return PLQ_OK;
}

extern "C" int plq_slab_plane(plq_slab *s, int32_t which, void **device_ptr, int64_t *bytes) {
    if (!s || !device_ptr || which < PLQ_SLAB_LOW_HALO || which > PLQ_SLAB_HIGH_HALO)
        return plq_fail(PLQ_EINVAL, "bad arguments");
    const int64_t index[4] = {0, 1, s->nz, s->nz + 1};
    *device_ptr = s->d_state + index[which] * s->plane;
    if (bytes) *bytes = s->plane;
    return PLQ_OK;
}

extern "C" int plq_slab_pass(plq_slab *s, int32_t colour) {
    if (!s || (colour != 0 && colour != 1)) return plq_fail(PLQ_EINVAL, "bad arguments");
    cudaError_t e = plq_enter_device(s->ctx_copy.device);
    if (e != cudaSuccess) return slab_cuda(s, e, "cudaSetDevice");
    SlabArgs a;
    std::memset(&a, 0, sizeof a);
    a.state = s->d_state;
    a.L0 = s->L0;
    a.L1 = s->L1;
    a.nz = (int)s->nz;
    a.q = s->q;
    a.kernel = s->desc.updater;
    std::memcpy(a.pw, s->pw, sizeof a.pw);
    a.metro24 = s->d_metro24;
    a.hb24 = s->d_hb24;
    a.seed32 = s->seed32;
    a.sweep32 = (uint32_t)s->sweep;
    // buffer plane 1 is plane z0 of the lattice: the buffer's parity differs by (z0 - 1) mod 2
    a.local_colour = (colour + (int)((s->z0 + 1) & 1)) & 1;
    a.var_offset = (s->z0 - 1) * s->plane;
    const int64_t sites = s->plane / 2 * s->nz;
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((sites + kSlabThreads - 1) / kSlabThreads,
                                                                  (int64_t)s->ctx_copy.sm_count * 16));
    slab_pass_kernel<<<(unsigned)blocks, kSlabThreads, 0, s->stream>>>(a);
    return slab_cuda(s, cudaGetLastError(), "slab pass");
}

extern "C" int plq_slab_end_sweep(plq_slab *s) {
    if (!s) return plq_fail(PLQ_EINVAL, "bad arguments");
    ++s->sweep;
    return PLQ_OK;
}

extern "C" int plq_slab_sync(plq_slab *s) {
    if (!s) return plq_fail(PLQ_EINVAL, "bad arguments");
    cudaError_t e = plq_enter_device(s->ctx_copy.device);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    return slab_cuda(s, e, "slab sync");
}

extern "C" int plq_slab_read(plq_slab *s, uint8_t *out) {
    if (!s || !out) return plq_fail(PLQ_EINVAL, "bad arguments");
    cudaError_t e = plq_enter_device(s->ctx_copy.device);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, s->d_state + s->plane, (size_t)(s->nz * s->plane), cudaMemcpyDeviceToHost,
                            s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    return slab_cuda(s, e, "slab read");
}

extern "C" void plq_slab_destroy(plq_slab *s) { slab_free(s); }
