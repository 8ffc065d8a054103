// plq_local.cu -- generic checkerboard colour passes (any D <= 8) for site
// and link variables, in both randomness modes.
//
// One launch = one colour pass of LocalUpdate::sweep with
// Schedule::Checkerboard (src/updater.rs:316-343): the sites of one parity
// (or, for links, one direction and base-site parity).  Within a pass no
// variable reads another of the same colour, so the pass is data-parallel;
// what the CPU does sequentially is reproduced by giving every variable the
// draw it would have had in the sequential walk:
//
//  * heat bath (any mode) and the keyed stream: the draw position/key of a
//    variable is a closed form of its index (one draw per variable in
//    colour order: rank = floor(site/2) when extent 0 is even);
//  * Metropolis on the PCG stream draws only uphill (updater.rs:90), so the
//    position of a variable's draw is the number of uphill variables before
//    it in the pass: a device-wide exclusive scan, done here with a
//    single-pass decoupled look-back over chunks taken in ticket order.
//
// Each thread owns R consecutive ranks of the colour, so on the PCG stream it
// jumps once and then steps the LCG.
#include <cuda_runtime.h>

#include "../../include/plaquette.h"
#include "plq_device.cuh"
#include "plq_local.h"
#include "plq_local_impl.cuh"
#include "plq_words.cuh"

namespace plq {

template <int D, bool LINK, int Q, bool STREAM>
__global__ void __launch_bounds__(kWordThreads) word_pass_kernel(LocalArgs a) {
    if (LINK)
        link_words_chunk<D, STREAM>(a, blockIdx.x, kWordsPerThread);
    else
        site_words_chunk<D, Q, STREAM>(a, blockIdx.x, kWordsPerThread);
}

int64_t word_chunks(int64_t n_sites) {
    const int64_t per = (int64_t)kWordThreads * kWordsPerThread;
    return (n_sites / 4 + per - 1) / per;
}

template <int D>
static cudaError_t launch_words_d(const LocalArgs &a, bool link, cudaStream_t stream) {
    const unsigned blocks = (unsigned)word_chunks(a.g.n_sites);
    const bool st = a.jump != nullptr;
    if (link) {
        if (st) word_pass_kernel<D, true, 2, true><<<blocks, kWordThreads, 0, stream>>>(a);
        else word_pass_kernel<D, true, 2, false><<<blocks, kWordThreads, 0, stream>>>(a);
    } else if (a.q == 3) {
        if (st) word_pass_kernel<D, false, 3, true><<<blocks, kWordThreads, 0, stream>>>(a);
        else word_pass_kernel<D, false, 3, false><<<blocks, kWordThreads, 0, stream>>>(a);
    } else if (a.q == 4) {
        if (st) word_pass_kernel<D, false, 4, true><<<blocks, kWordThreads, 0, stream>>>(a);
        else word_pass_kernel<D, false, 4, false><<<blocks, kWordThreads, 0, stream>>>(a);
    } else {
        if (st) word_pass_kernel<D, false, 2, true><<<blocks, kWordThreads, 0, stream>>>(a);
        else word_pass_kernel<D, false, 2, false><<<blocks, kWordThreads, 0, stream>>>(a);
    }
    return cudaGetLastError();
}

static cudaError_t launch_words(const LocalArgs &a, bool link, cudaStream_t stream) {
    switch (a.g.d) {
        case 1: return launch_words_d<1>(a, link, stream);
        case 2: return launch_words_d<2>(a, link, stream);
        case 3: return launch_words_d<3>(a, link, stream);
        case 4: return launch_words_d<4>(a, link, stream);
        default: return cudaErrorInvalidValue;
    }
}

template <int D, bool LINK, bool LOOKBACK>
__global__ void __launch_bounds__(kThreads) local_pass_kernel(LocalArgs a) {
    int64_t chunk;
    if (LOOKBACK) {
        __shared__ unsigned long long s_ticket;
        if (threadIdx.x == 0) s_ticket = atomicAdd(&a.ctrl->ticket, 1ull) - a.ticket_base;
        __syncthreads();
        chunk = (int64_t)s_ticket;
        if (chunk >= a.n_chunks) {  // host bookkeeping broke: refuse, never index out of range
            if (threadIdx.x == 0) atomicOr(&a.ctrl->status, kStatusBounds);
            return;
        }
    } else {
        chunk = blockIdx.x;
    }
    local_chunk<D, LINK, LOOKBACK, kRanksPerThread>(a, chunk);
}

// ------------------------------------------------------------ launchers
template <int D, bool LINK>
static void launch_d(const LocalArgs &a, bool lookback, cudaStream_t stream, int64_t blocks) {
    if (lookback)
        local_pass_kernel<D, LINK, true><<<(unsigned)blocks, kThreads, 0, stream>>>(a);
    else
        local_pass_kernel<D, LINK, false><<<(unsigned)blocks, kThreads, 0, stream>>>(a);
}

int64_t local_chunks(int64_t n_sites) { return (n_sites / 2 + kChunk - 1) / kChunk; }

cudaError_t launch_local_pass(const LocalArgs &a, bool link, bool lookback, cudaStream_t stream) {
    if (a.words && !lookback) return launch_words(a, link, stream);
    int64_t blocks = local_chunks(a.g.n_sites);
    if (blocks <= 0) return cudaSuccess;
#define PLQ_CASE(DD)                                              \
    case DD:                                                      \
        if (link) launch_d<DD, true>(a, lookback, stream, blocks); \
        else launch_d<DD, false>(a, lookback, stream, blocks);    \
        break;
    switch (a.g.d) {
        PLQ_CASE(1)
        PLQ_CASE(2)
        PLQ_CASE(3)
        PLQ_CASE(4)
        PLQ_CASE(5)
        PLQ_CASE(6)
        PLQ_CASE(7)
        PLQ_CASE(8)
        default:
            return cudaErrorInvalidValue;
    }
#undef PLQ_CASE
    return cudaGetLastError();
}

}  // namespace plq
