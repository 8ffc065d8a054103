// plq_ensemble.cu -- many lattices advanced by one persistent launch.
//
// An ensemble is a list of member lattices (any mix of Ising / Potts sites
// and Z2 gauge links, uneven sizes, their own beta and seed), each exactly a
// chain of the C ABI.  Advancing it by S sweeps is one cooperative launch
// (replayed from a CUDA graph): every CTA walks "super-phases" -- super-phase
// p holds colour pass p of every member that has one -- taking (member,
// chunk) work items round-robin, with a grid barrier between super-phases.
// A work item runs exactly the per-lattice pass body (plq_local_impl.cuh), so
// an ensemble sweep is bit-identical to sweeping each member with its own
// chain; what changes is that ~10^4 small launches become one.
//
// Parallel tempering: members can be grouped into ladders (same model and
// shape, one beta per slot).  Every `every` sweeps the kernel sums each
// ladder member's energy in int64, then attempts swaps of adjacent slots
// (even pairs, then odd pairs on the next attempt) with acceptance
// min(1, exp((beta_k - beta_k+1)(E_k - E_k+1))), the uniform keyed by (ladder
// seed, pair, attempt).  A swap exchanges the two members' beta slots (and so
// their decision tables), never their configurations.
//
// The autotuner times candidate (ranks per thread, CTAs per SM) pairs on a
// snapshot of the ensemble and keeps the fastest.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/plaquette.h"
#include "plq_abi_internal.h"
#include "plq_device.cuh"
#include "plq_geom.cuh"
#include "plq_local.h"
#include "plq_local_impl.cuh"
#include "plq_packed.cuh"
#include "plq_pt.cuh"
#include "plq_tables.h"
#include "plq_words.cuh"

using namespace plq;

namespace {

constexpr int kEnsThreads = 256;
constexpr int kBarrierSpin = 1 << 24;
constexpr int kEnergyChunk = 2048;

struct TableSet {
    const uint64_t *hb53;
    const uint32_t *hb24;
    const uint64_t *metro53;
    const uint32_t *metro24;
    double beta;
};

struct EnsMember {
    LocalArgs a;       // the member's pass arguments (state, geometry, tables of its own beta)
    int link;          // variables on links
    int passes;        // colour passes per sweep
    int64_t n_vars;
    int wpt;           // four-site or packed body: words (rows) per thread of a work item (the tuned shape)
    int pk_wide;       // packed rows are 64-bit words (sites with 32 < L0 <= 64)
    void *pk;          // packed variables: one row of L0 bits per word (links: d planes), or null
    double j;
    int ladder;
};

struct LadderDev {
    int k;
    int every;
    uint32_t seed32;
    int32_t *member_of_slot;  // k entries
};

// The autotuner's table: the work-item shape (four-site words per thread)
// measured fastest for each member shape -- (model, q, d, extents, updater,
// stream) -- in this process.  Ensembles and served jobs created later take
// their members' shapes from it (4 where a shape was never tuned).
struct ShapeKey {
    int32_t model, q, d, updater, rng;
    int32_t L[4];
    bool operator<(const ShapeKey &o) const { return std::memcmp(this, &o, sizeof *this) < 0; }
};
struct TuneEntry {
    int wpt;
    double ms_per_sweep;  // the members of this shape alone, at that shape
    int members;
};
std::mutex g_tune_mu;
std::map<ShapeKey, TuneEntry> g_tuned;

ShapeKey shape_key(const plq_chain_desc &d) {
    ShapeKey k;
    std::memset(&k, 0, sizeof k);
    k.model = d.model;
    k.q = d.model == PLQ_POTTS ? d.q : 2;
    k.d = d.d;
    k.updater = d.updater;
    k.rng = d.rng;
    for (int i = 0; i < d.d && i < 4; ++i) k.L[i] = (int32_t)d.shape[i];
    return k;
}

int tuned_wpt(const plq_chain_desc &d) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tuned.find(shape_key(d));
    return it == g_tuned.end() ? kWordsPerThread : it->second.wpt;
}

// Device-resident launch state, advanced by the kernel itself so a captured
// graph replays without new parameters.
struct LaunchState {
    unsigned long long sweep;       // sweeps done (keyed sweep index, PT schedule)
    unsigned long long pt_attempts; // per-ensemble attempt counter
    unsigned int bar_count;
    unsigned int bar_gen;
    unsigned long long ticket;      // next work-item ticket of the running launch (zero between launches)
};

// One work item: `count` consecutive chunks, from `chunk`, of one colour pass
// of one member (index relative to the launch's member array).  16 bytes:
// the kernel fetches it with one load.
struct alignas(16) WorkItem {
    int32_t member;
    int32_t chunk;
    int32_t count;
    int32_t pass;  // colour pass (link members: 2 * direction + parity)
};

struct EnsArgs {
    EnsMember *members;
    int n_members;
    TableSet *tsets;
    int32_t *ts_of_member;
    unsigned long long *pos;  // stream heat bath: per-member stream position (relative)
    unsigned long long *msweep;  // per-member sweep counters (serving), or null: all share ls->sweep
    const WorkItem *items;     // one sweep's items, super-phase by super-phase
    int64_t n_items;
    const int32_t *e_item_member;
    const int32_t *e_item_chunk;
    int64_t n_e_items;
    long long *energy;
    LadderDev *ladders;
    int n_ladders;
    int pt_every;
    LaunchState *ls;
    Control *ctrl;
    unsigned long long *done;  // per member: work items completed in this launch (zero between launches)
    uint64_t sweeps;
    int ranks;  // ranks per thread of a work item
};

__device__ __forceinline__ unsigned int ld_volatile(const unsigned int *p) {
    return *reinterpret_cast<const volatile unsigned int *>(p);
}

// Sense-counting grid barrier; all CTAs are co-resident (cooperative launch).
// Bounded: a wait that runs out sets a status bit and lets the CTA go on.
__device__ void grid_barrier(const EnsArgs &e) {
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int gen = ld_volatile(&e.ls->bar_gen);
        __threadfence();
        unsigned int arrived = atomicAdd(&e.ls->bar_count, 1u);
        if (arrived == gridDim.x - 1) {
            atomicExch(&e.ls->bar_count, 0u);
            __threadfence();
            atomicAdd(&e.ls->bar_gen, 1u);
        } else {
            int spins = 0;
            while (ld_volatile(&e.ls->bar_gen) == gen) {
                if (++spins > kBarrierSpin) {
                    atomicOr(&e.ctrl->status, kStatusLookbackTimeout);
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

template <int D>
__device__ void run_words(const LocalArgs &a, int link, int64_t chunk, int R) {
    const bool st = a.jump != nullptr;
    if (link) {
        if (D >= 2) {
            if (st) link_words_chunk<D, true>(a, chunk, R);
            else link_words_chunk<D, false>(a, chunk, R);
        }
    } else if (a.q == 3) {
        if (st) site_words_chunk<D, 3, true>(a, chunk, R);
        else site_words_chunk<D, 3, false>(a, chunk, R);
    } else if (a.q == 4) {
        if (st) site_words_chunk<D, 4, true>(a, chunk, R);
        else site_words_chunk<D, 4, false>(a, chunk, R);
    } else {
        if (st) site_words_chunk<D, 2, true>(a, chunk, R);
        else site_words_chunk<D, 2, false>(a, chunk, R);
    }
}

// WORDS_ONLY: every member runs four sites at a time, so the generic body is
// compiled out (far fewer registers, more CTAs per SM).
template <int R, bool WORDS_ONLY>
__device__ void run_item(const LocalArgs &a, int d, int link, int64_t chunk, int wpt) {
    if (WORDS_ONLY || a.words) {
        switch (d) {
            case 1: run_words<1>(a, link, chunk, wpt); break;
            case 2: run_words<2>(a, link, chunk, wpt); break;
            case 3: run_words<3>(a, link, chunk, wpt); break;
            case 4: run_words<4>(a, link, chunk, wpt); break;
            default: break;
        }
        return;
    }
    if (WORDS_ONLY) return;
    if (link) {
        switch (d) {
            case 2: local_chunk<2, true, false, R>(a, chunk); break;
            case 3: local_chunk<3, true, false, R>(a, chunk); break;
            case 4: local_chunk<4, true, false, R>(a, chunk); break;
            default: break;
        }
    } else {
        switch (d) {
            case 1: local_chunk<1, false, false, R>(a, chunk); break;
            case 2: local_chunk<2, false, false, R>(a, chunk); break;
            case 3: local_chunk<3, false, false, R>(a, chunk); break;
            case 4: local_chunk<4, false, false, R>(a, chunk); break;
            default: break;
        }
    }
}

// ---- Z2 gauge members with L0 <= 32 on the keyed stream: links bit-packed by rows.
// Inside a persistent launch such a member's links live in pk: word dir * rows + r
// holds bit x = U_dir(x, r) for row r (the site index over directions >= 1).  A
// work item takes rows of one (direction mu, parity) pass: the six staples of
// every link of a row come out of XORs of whole row words (a shift along
// direction 0 is a rotation of the row, along the others another row), their
// count of unsatisfied staples out of a bit-sliced counter, and each link of
// the pass's parity then decides exactly as the byte body does -- the same key
// cur + 4(d-1) - 2 * unsatisfied, the same keyed draw of variable site * d + mu,
// the same table -- so results are bit-identical.  The launch packs the bytes
// first and unpacks them at its end (pack_links_kernel).

// Rows of a lattice (sites over directions >= 1): L1 * L2 * ... (extents past
// d are 1), by multiplication.
__host__ __device__ __forceinline__ uint32_t row_count(const Geom &g) {
    uint32_t n = 1;
#pragma unroll
    for (int k = 1; k < kMaxD; ++k) n *= (uint32_t)g.L[k];
    return n;
}

// Row r's coordinates along directions 1..D-1: their parity and the row
// offsets to the +k / -k neighbour rows (periodic).  The row stride of
// direction k is L1 * ... * L(k-1).
template <int D>
__device__ __forceinline__ int row_geometry(const Geom &g, uint32_t r, int32_t *op, int32_t *om) {
    uint32_t rr = r;
    int par = 0;
    int32_t rs = 1;
#pragma unroll
    for (int k = 1; k < D; ++k) {
        const uint32_t q = fdiv(rr, g.dm[k], g.dl[k]);
        const int32_t c = (int32_t)(rr - q * (uint32_t)g.L[k]);
        rr = q;
        par += c;
        op[k] = c + 1 < g.L[k] ? rs : -(g.L[k] - 1) * rs;
        om[k] = c > 0 ? -rs : (g.L[k] - 1) * rs;
        rs *= g.L[k];
    }
    return par;
}

// q = 2 sites (Ising, or Potts at q = 2) packed by rows: the per-site count of
// neighbours in state 1 comes out of the bit-sliced counter over the 2d
// neighbour rows (d <= 3: at most 6), key cur + 2 * count as the byte body's.
template <int D, class W>
__device__ void packed_site_item(const LocalArgs &a, W *pk, int64_t chunk, int R, const uint32_t *tab) {
    const uint32_t L0 = (uint32_t)a.g.L[0];
    const uint32_t rows = row_count(a.g);
    const W full = L0 == 8 * sizeof(W) ? ~(W)0 : (((W)1 << L0) - 1);
    const uint32_t r0 = (uint32_t)(chunk * (int64_t)blockDim.x * R) + threadIdx.x * (uint32_t)R;
    const bool hb = a.kernel == PLQ_HEATBATH;
    const uint32_t sweep_mix = keyed_mix(a.sweep32);
#pragma unroll 1
    for (int i = 0; i < R; ++i) {
        const uint32_t r = r0 + (uint32_t)i;
        if (r >= rows) break;
        int32_t op[4] = {0, 0, 0, 0}, om[4] = {0, 0, 0, 0};
        const int par = row_geometry<D>(a.g, r, op, om);
        const W C = pk[r];
        W c0 = 0, c1 = 0, c2 = 0;
        count_add(c0, c1, c2, row_xp(C, L0, full));
        count_add(c0, c1, c2, row_xm(C, L0, full));
#pragma unroll
        for (int k = 1; k < D; ++k) {
            count_add(c0, c1, c2, pk[r + (uint32_t)op[k]]);
            count_add(c0, c1, c2, pk[r + (uint32_t)om[k]]);
        }
        const uint32_t x0 = (uint32_t)((a.color ^ par) & 1);
        const int n = (int)(L0 / 2);
        const uint32_t v0 = r * L0 + x0;  // the keyed stream's index of the row's first variable
        const W flip = hb ? decide_row<W, 2, true>(C >> x0, c0 >> x0, c1 >> x0, c2 >> x0, n, v0, a.seed32, sweep_mix, tab)
                          : decide_row<W, 2, false>(C >> x0, c0 >> x0, c1 >> x0, c2 >> x0, n, v0, a.seed32, sweep_mix, tab);
        pk[r] = C ^ (flip << x0);
    }
}

// Energy integer of packed rows [c * blockDim, (c + 1) * blockDim), one row per
// thread: sites -- the bond sum (Ising) or agreement count (Potts) over the
// +mu bonds; links -- the plaquette sum over mu < nu (as energy_chunk).
template <int D, class W>
__device__ long long packed_energy_rows(const LocalArgs &a, const W *pk, int link, int64_t c) {
    const uint32_t L0 = (uint32_t)a.g.L[0];
    const uint32_t rows = row_count(a.g);
    const W full = L0 == 8 * sizeof(W) ? ~(W)0 : (((W)1 << L0) - 1);
    const uint32_t r = (uint32_t)(c * (int64_t)blockDim.x) + threadIdx.x;
    if (r >= rows) return 0;
    int32_t op[4] = {0, 0, 0, 0}, om[4] = {0, 0, 0, 0};
    row_geometry<D>(a.g, r, op, om);
    long long acc = 0;
    if (!link) {
        const W C = pk[r];
        int diff = popc_w((C ^ row_xp(C, L0, full)) & full);
        long long pairs = L0;
#pragma unroll
        for (int k = 1; k < D; ++k) {
            diff += popc_w(C ^ pk[r + (uint32_t)op[k]]);
            pairs += L0;
        }
        acc = a.model == PLQ_ISING ? pairs - 2ll * diff : pairs - diff;
    } else {
#pragma unroll
        for (int mu = 0; mu < D; ++mu) {
#pragma unroll
            for (int nu = mu + 1; nu < D; ++nu) {
                const W *Pmu = pk + (uint32_t)mu * rows, *Pnu = pk + (uint32_t)nu * rows;
                const W umu = Pmu[r], unu = Pnu[r];
                // U_nu(s + mu): mu = 0 a rotation of the row, else the +mu row
                const W nu_smu = mu == 0 ? row_xp(unu, L0, full) : Pnu[r + (uint32_t)op[mu]];
                const W mu_snu = Pmu[r + (uint32_t)op[nu]];  // nu >= 1
                acc += (long long)L0 - 2ll * popc_w(umu ^ nu_smu ^ mu_snu ^ unu);
            }
        }
    }
    return acc;
}

// MU: the pass's direction (a compile-time constant, so the staple terms that
// are row rotations and those that are other rows are fixed per variant).
template <int D, int MU>
__device__ void packed_link_item(const LocalArgs &a, uint32_t *pk, int64_t chunk, int R, const uint32_t *tab) {
    // (rows of at most 32 links)
    const uint32_t L0 = (uint32_t)a.g.L[0];
    const uint32_t rows = row_count(a.g);
    constexpr int mu = MU;
    const uint32_t full = L0 == 32 ? 0xFFFFFFFFu : ((1u << L0) - 1u);
    const uint32_t r0 = (uint32_t)(chunk * (int64_t)blockDim.x * R) + threadIdx.x * (uint32_t)R;
    const bool hb = a.kernel == PLQ_HEATBATH;
    const uint32_t sweep_mix = keyed_mix(a.sweep32);
#pragma unroll 1
    for (int i = 0; i < R; ++i) {
        const uint32_t r = r0 + (uint32_t)i;
        if (r >= rows) break;
        int32_t op[4] = {0, 0, 0, 0}, om[4] = {0, 0, 0, 0};
        const int par = row_geometry<D>(a.g, r, op, om);
        const int32_t op_mu = mu > 0 ? op[mu] : 0;
        const uint32_t Umu = pk[(uint32_t)mu * rows + r];
        uint32_t c0 = 0, c1 = 0, c2 = 0;  // satisfied staples per link
#pragma unroll
        for (int nu = 0; nu < D; ++nu) {
            if (nu == mu) continue;
            const uint32_t *Pnu = pk + (uint32_t)nu * rows;
            const uint32_t *Pmu = pk + (uint32_t)mu * rows;
            // forward: U_nu(s+mu) U_mu(s+nu) U_nu(s)
            const uint32_t nu_s = Pnu[r];
            const uint32_t nu_smu = mu == 0 ? row_xp(nu_s, L0, full) : Pnu[r + (uint32_t)op_mu];
            const uint32_t mu_snu = nu == 0 ? row_xp(Umu, L0, full) : Pmu[r + (uint32_t)op[nu]];
            count_add(c0, c1, c2, ~(nu_smu ^ mu_snu ^ nu_s));
            // backward: U_nu(s+mu-nu) U_mu(s-nu) U_nu(s-nu)
            uint32_t nu_smn, mu_smn, nu_smumn;
            if (nu == 0) {
                nu_smn = row_xm(nu_s, L0, full);
                mu_smn = row_xm(Umu, L0, full);
                nu_smumn = row_xm(nu_smu, L0, full);
            } else {
                nu_smn = Pnu[r + (uint32_t)om[nu]];
                mu_smn = Pmu[r + (uint32_t)om[nu]];
                nu_smumn = mu == 0 ? row_xp(nu_smn, L0, full) : Pnu[r + (uint32_t)op_mu + (uint32_t)om[nu]];
            }
            count_add(c0, c1, c2, ~(nu_smumn ^ mu_smn ^ nu_smn));
        }
        // the links of the pass's parity: x with (x + par) % 2 == colour; the byte body's key
        // cur + 4(d-1) - 2 * unsatisfied is cur + 2 * satisfied
        const uint32_t x0 = (uint32_t)((a.color ^ par) & 1);
        const int n = (int)(L0 / 2);
        const uint32_t v0 = (r * L0 + x0) * (uint32_t)D + (uint32_t)mu;  // keyed index of link (x0, r, mu)
        const uint32_t flip = hb ? decide_row<uint32_t, 2 * D, true>(Umu >> x0, c0 >> x0, c1 >> x0, c2 >> x0, n, v0,
                                                                     a.seed32, sweep_mix, tab)
                                 : decide_row<uint32_t, 2 * D, false>(Umu >> x0, c0 >> x0, c1 >> x0, c2 >> x0, n, v0,
                                                                      a.seed32, sweep_mix, tab);
        pk[(uint32_t)mu * rows + r] = Umu ^ (flip << x0);
    }
}

// Packing entry of one member: its rows (of all d directions, for links)
// occupy [first, first + planes * rows) of the launch's packing index space.
struct PackEntry {
    uint8_t *state;   // byte planes (dir * n_sites + site)
    void *pk;
    uint32_t first;   // first index of this member
    uint32_t L0;
    int wide;         // 64-bit rows
    int pad;
};

// Bytes to bits (unpack = false) or back (unpack = true) for every packed
// member of the launch: one thread per row of one direction.
__global__ void pack_links_kernel(const PackEntry *tab, int n_tab, uint32_t total, bool unpack) {
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
        int lo = 0, hi = n_tab - 1;
        while (lo < hi) {  // the entry holding g
            const int mid = (lo + hi + 1) / 2;
            if (tab[mid].first <= g) lo = mid;
            else hi = mid - 1;
        }
        const PackEntry &t = tab[lo];
        const uint32_t idx = g - t.first;  // dir * rows + row: its bytes start at idx * L0
        uint8_t *bytes = t.state + (size_t)idx * t.L0;
        const bool quads = (t.L0 & 3u) == 0;  // the row's bytes come as aligned 32-bit words
        if (!unpack) {
            uint64_t w = 0;
            if (quads) {
                // four 0/1 bytes to four bits: b_i * 2^(8i) times 2^24 + 2^17 + 2^10 + 2^3 lands
                // b_i on bit 24 + i, every other product below bit 24 or beyond bit 31
                const uint32_t *q4 = reinterpret_cast<const uint32_t *>(bytes);
                for (uint32_t k = 0; k < t.L0 / 4; ++k)
                    w |= (uint64_t)((((q4[k] & 0x01010101u) * 0x01020408u) >> 24) & 0xFu) << (4 * k);
            } else {
                for (uint32_t x = 0; x < t.L0; ++x) w |= (uint64_t)(bytes[x] & 1u) << x;
            }
            if (t.wide) static_cast<uint64_t *>(t.pk)[idx] = w;
            else static_cast<uint32_t *>(t.pk)[idx] = (uint32_t)w;
        } else {
            const uint64_t w = t.wide ? static_cast<const uint64_t *>(t.pk)[idx] : static_cast<const uint32_t *>(t.pk)[idx];
            if (quads) {
                // four bits to four bytes: bit i times 2^0 + 2^7 + 2^14 + 2^21 has a copy on bit 8i
                uint32_t *q4 = reinterpret_cast<uint32_t *>(bytes);
                for (uint32_t k = 0; k < t.L0 / 4; ++k)
                    q4[k] = ((uint32_t)((w >> (4 * k)) & 0xFu) * 0x00204081u) & 0x01010101u;
            } else {
                for (uint32_t x = 0; x < t.L0; ++x) bytes[x] = (uint8_t)((w >> x) & 1u);
            }
        }
    }
}

// The pass-specific fields of member m's arguments for colour pass `sp` of
// sweep `sweep_in_launch`: loaded into registers (pass_fields), then written
// over the member's arguments in shared memory (apply).
struct PassFields {
    const uint64_t *hb53;
    const uint32_t *hb24;
    const uint64_t *metro53;
    const uint32_t *metro24;
    uint64_t pass_offset;
    uint32_t sweep32;
    int dir, color;
};

__device__ __forceinline__ PassFields pass_fields(const EnsArgs &e, int m, int sp,
                                                  unsigned long long sweep_in_launch) {
    const EnsMember &mem = e.members[m];
    const TableSet &ts = e.tsets[e.ts_of_member[m]];
    PassFields f;
    f.hb53 = ts.hb53;
    f.hb24 = ts.hb24;
    f.metro53 = ts.metro53;
    f.metro24 = ts.metro24;
    f.dir = mem.link ? sp >> 1 : 0;
    f.color = sp & 1;
    f.sweep32 = (uint32_t)((e.msweep ? e.msweep[m] : e.ls->sweep) + sweep_in_launch);
    f.pass_offset = mem.a.jump ? e.pos[m] + sweep_in_launch * (unsigned long long)mem.n_vars +
                                     (unsigned long long)sp * (unsigned long long)(mem.a.g.n_sites / 2)
                               : 0;
    return f;
}

__device__ __forceinline__ void apply(const PassFields &f, LocalArgs &sa) {
    sa.hb53 = f.hb53;
    sa.hb24 = f.hb24;
    sa.metro53 = f.metro53;
    sa.metro24 = f.metro24;
    sa.dir = f.dir;
    sa.color = f.color;
    sa.sweep32 = f.sweep32;
    if (sa.jump) sa.pass_offset = f.pass_offset;
}

// int64 energy integer of a member chunk: Ising bond sum, Potts agreement,
// gauge plaquette sum (E = -J * X when the field and offsets vanish).
template <int D, bool LINK>
__device__ long long energy_chunk(const LocalArgs &a, int64_t chunk) {
    const int64_t n = a.g.n_sites;
    long long acc = 0;
    for (int64_t s = chunk * kEnergyChunk + threadIdx.x; s < n && s < (chunk + 1) * kEnergyChunk; s += blockDim.x) {
        int32_t x[D];
        site_coords<D>(a.g, s, x);
        if (LINK) {
#pragma unroll
            for (int mu = 0; mu < D; ++mu) {
                int64_t s_mu = nbr_plus(a.g, s, x, mu);
#pragma unroll
                for (int nu = mu + 1; nu < D; ++nu) {
                    int64_t s_nu = nbr_plus(a.g, s, x, nu);
                    int b = a.state[mu * n + s] ^ a.state[nu * n + s_mu] ^ a.state[mu * n + s_nu] ^ a.state[nu * n + s];
                    acc += 1 - 2 * b;
                }
            }
        } else {
            int si = a.state[s];
#pragma unroll
            for (int mu = 0; mu < D; ++mu) {
                int sj = a.state[nbr_plus(a.g, s, x, mu)];
                acc += a.model == PLQ_ISING ? (long long)((1 - 2 * si) * (1 - 2 * sj)) : (long long)(si == sj);
            }
        }
    }
    return acc;
}

__device__ long long energy_item(const LocalArgs &a, int d, int link, int64_t chunk) {
    if (link) {
        switch (d) {
            case 2: return energy_chunk<2, true>(a, chunk);
            case 3: return energy_chunk<3, true>(a, chunk);
            case 4: return energy_chunk<4, true>(a, chunk);
        }
    } else {
        switch (d) {
            case 1: return energy_chunk<1, false>(a, chunk);
            case 2: return energy_chunk<2, false>(a, chunk);
            case 3: return energy_chunk<3, false>(a, chunk);
            case 4: return energy_chunk<4, false>(a, chunk);
        }
    }
    return 0;
}

__device__ __forceinline__ long long block_sum(long long v) {
    __shared__ long long part[kEnsThreads / 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    long long t = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
    __syncthreads();
    return t;
}

// Energies of every ladder member: grid-stride over energy items.
__device__ void energy_phase(const EnsArgs &e) {
    __shared__ LocalArgs sa;
    for (int64_t i = blockIdx.x; i < e.n_e_items; i += gridDim.x) {
        int m = e.e_item_member[i];
        if (threadIdx.x == 0) sa = e.members[m].a;
        __syncthreads();
        const EnsMember &mem = e.members[m];
        long long part = 0;
        if (!mem.pk) {
            part = energy_item(sa, sa.g.d, mem.link, e.e_item_chunk[i]);
        } else if (mem.pk_wide) {
            const uint64_t *pk = static_cast<const uint64_t *>(mem.pk);
            part = sa.g.d == 2 ? packed_energy_rows<2, uint64_t>(sa, pk, mem.link, e.e_item_chunk[i])
                               : packed_energy_rows<3, uint64_t>(sa, pk, mem.link, e.e_item_chunk[i]);
        } else {
            const uint32_t *pk = static_cast<const uint32_t *>(mem.pk);
            switch (sa.g.d) {
                case 2: part = packed_energy_rows<2, uint32_t>(sa, pk, mem.link, e.e_item_chunk[i]); break;
                case 3: part = packed_energy_rows<3, uint32_t>(sa, pk, mem.link, e.e_item_chunk[i]); break;
                case 4: part = packed_energy_rows<4, uint32_t>(sa, pk, mem.link, e.e_item_chunk[i]); break;
                default: break;
            }
        }
        long long tot = block_sum(part);
        if (threadIdx.x == 0 && tot) atomicAdd((unsigned long long *)&e.energy[m], (unsigned long long)tot);
        __syncthreads();
    }
}

// Primaries of packed members from their rows (the same integers as the byte
// scan, primaries_multi_kernel): item i is rows [c * blockDim, (c + 1) * blockDim)
// of member item_member[i]; out[0] gets the bond / agreement / plaquette sum
// (packed_energy_rows), sites also their counts of state 1 -- the Ising spin
// sum n - 2 * ones into out[1], Potts q = 2 label counts into out[1], out[2].
// The outputs must be zero before the launch.
__global__ void __launch_bounds__(kEnsThreads)
packed_primaries_kernel(const EnsMember *members, const int32_t *item_member, const int32_t *item_chunk,
                        int64_t n_items, long long *prims, const int64_t *prims_offset) {
    for (int64_t i = blockIdx.x; i < n_items; i += gridDim.x) {
        const int m = item_member[i];
        const EnsMember &mem = members[m];
        const LocalArgs &a = mem.a;
        const int64_t c = item_chunk[i];
        long long part = 0, ones = 0;
        const uint32_t rows = row_count(a.g);
        const uint32_t r = (uint32_t)(c * (int64_t)blockDim.x) + threadIdx.x;
        if (mem.pk_wide) {
            const uint64_t *pk = static_cast<const uint64_t *>(mem.pk);
            part = a.g.d == 2 ? packed_energy_rows<2, uint64_t>(a, pk, mem.link, c)
                              : packed_energy_rows<3, uint64_t>(a, pk, mem.link, c);
            if (!mem.link && r < rows) ones = popc_w(pk[r]);
        } else {
            const uint32_t *pk = static_cast<const uint32_t *>(mem.pk);
            switch (a.g.d) {
                case 2: part = packed_energy_rows<2, uint32_t>(a, pk, mem.link, c); break;
                case 3: part = packed_energy_rows<3, uint32_t>(a, pk, mem.link, c); break;
                case 4: part = packed_energy_rows<4, uint32_t>(a, pk, mem.link, c); break;
                default: break;
            }
            if (!mem.link && r < rows) ones = popc_w(pk[r]);
        }
        const long long tot = block_sum(part);
        const long long tot_ones = mem.link ? 0 : block_sum(ones);
        if (threadIdx.x == 0) {
            long long *out = prims + prims_offset[m];
            if (tot) atomicAdd((unsigned long long *)&out[0], (unsigned long long)tot);
            if (!mem.link) {
                const int64_t r0 = c * (int64_t)blockDim.x;
                const int64_t nr = min((int64_t)rows - r0, (int64_t)blockDim.x);
                const long long sites = nr * (long long)a.g.L[0];
                if (a.model == PLQ_ISING) {
                    atomicAdd((unsigned long long *)&out[1], (unsigned long long)(sites - 2 * tot_ones));
                } else {
                    atomicAdd((unsigned long long *)&out[1], (unsigned long long)(sites - tot_ones));
                    atomicAdd((unsigned long long *)&out[2], (unsigned long long)tot_ones);
                }
            }
        }
        __syncthreads();
    }
}

// Swap attempts of every ladder (one thread per pair); attempt index `att`.
// Energies E = -J * (bond, agreement or plaquette sum); the pair at slots
// (k, k+1) exchanges betas when (b_k - b_k+1)(E_k - E_k+1) >= 0 or a keyed
// uniform u < e^((b_k - b_k+1)(E_k - E_k+1)); even pairs on even attempts,
// odd pairs on odd ones.
__device__ void swap_phase(const EnsArgs &e, unsigned long long att) {
    for (int l = 0; l < e.n_ladders; ++l) {
        const LadderDev &L = e.ladders[l];
        const int parity = (int)(att & 1ull);
        for (int k = parity + 2 * (int)threadIdx.x; k + 1 < L.k; k += 2 * (int)blockDim.x) {
            int m1 = L.member_of_slot[k], m2 = L.member_of_slot[k + 1];
            const double b1 = e.tsets[e.ts_of_member[m1]].beta, b2 = e.tsets[e.ts_of_member[m2]].beta;
            if (pt_accept(b1, b2, e.energy[m1], e.energy[m2], e.members[m1].j, e.members[m2].j, L.seed32,
                          (uint32_t)k, (uint32_t)att)) {
                int32_t t1 = e.ts_of_member[m1];
                e.ts_of_member[m1] = e.ts_of_member[m2];
                e.ts_of_member[m2] = t1;
                L.member_of_slot[k] = m2;
                L.member_of_slot[k + 1] = m1;
            }
        }
    }
}

static_assert(sizeof(LocalArgs) % 4 == 0, "work items copy LocalArgs as 32-bit words");

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Work items per colour pass of member m (as append_items cuts them).
__device__ __forceinline__ unsigned long long member_chunks(const EnsArgs &e, int m) {
    const EnsMember &mem = e.members[m];
    // (32-bit: variables < 2^31, a chunk < 2^16)
    const uint32_t units = mem.pk ? row_count(mem.a.g)
                                  : (uint32_t)(mem.a.words ? mem.a.g.n_sites / 4 : mem.a.g.n_sites / 2);
    const uint32_t chunk = (uint32_t)kEnsThreads * (uint32_t)(mem.pk || mem.a.words ? mem.wpt : e.ranks);
    return (unsigned long long)((units + chunk - 1) / chunk);
}

// Thread 0: wait (bounded) until every work item of member m's passes before
// pass p of sweep t (in this launch) is complete.  The acquire makes the
// stores of those items -- run by any CTA -- visible to this CTA's threads
// after the next __syncthreads.
__device__ void wait_member(const EnsArgs &e, int m, unsigned long long t, int p) {
    const unsigned long long need = (t * (unsigned long long)e.members[m].passes + (unsigned long long)p) *
                                    member_chunks(e, m);
    int spins = 0;
    while (ld_acquire_u64(&e.done[m]) < need) {
        if (++spins > kBarrierSpin) {
            atomicOr(&e.ctrl->status, kStatusLookbackTimeout);
            break;
        }
        __nanosleep(64);
    }
}

// The persistent launch.  Work items are dealt out dynamically: ticket k is
// item k mod n_items of sweep k / n_items, and a CTA takes its next ticket
// (one atomic add) at the start of the current item, so the CTAs stay evenly
// loaded although items differ several-fold in work (each super-phase lists
// its items largest first).  There is no grid barrier between super-phases:
// before an item of member m's pass p the CTA waits until the member's
// previous passes are complete (per-member counters, released by the CTAs
// that ran them), so a pass of one member overlaps the tails of every other
// member's passes.  Tickets are taken in order and every wait is on items of
// lower tickets, all taken by resident CTAs (cooperative launch) that wait
// only on still lower ones, so the waits always end.  A CTA whose ticket lies
// past the end of a sweep with a tempering phase joins that phase's grid
// barriers (all its items of the sweep are done and released by then); every
// CTA crosses every sweep end, in order, so all take the same barriers.
//
// Between two items three warps work side by side: thread 0 takes the next
// ticket and waits for the member, threads 32-47 load the pass fields and (a
// packed member's) decision table, thread 64 releases the previous item; the
// next item's entry is loaded while this one runs.  An item is a run of
// chunks of one pass (more than one where a super-phase holds far more chunks
// than the grid has CTAs); the CTA runs them back to back and releases them
// together.
template <int R, bool WORDS_ONLY>
__global__ void __launch_bounds__(kEnsThreads, WORDS_ONLY ? 4 : 2) ensemble_kernel(EnsArgs e) {
    __shared__ LocalArgs sa;
    __shared__ unsigned long long s_ticket;
    __shared__ uint32_t s_tab[16];  // a packed member's decision table (keys cur + 2 * count < 16)
    const unsigned long long n_items = (unsigned long long)e.n_items;
    const unsigned long long total = n_items * e.sweeps;
    if (threadIdx.x == 0) s_ticket = atomicAdd(&e.ls->ticket, 1ull);
    __syncthreads();
    unsigned long long tk = s_ticket;
    unsigned long long r = 0;  // the ticket's sweep
    WorkItem it{0, 0, 0, 0};  // ... and item
    if (tk < total) {
        r = tk / n_items;
        it = e.items[tk - r * n_items];
    }
    unsigned long long round = 0;  // sweeps whose end this CTA has crossed
    int last_m = -1;               // the member whose arguments are in sa
    int pending = -1;              // member of the last item run, not yet released
    int pending_n = 0;             // ... and its chunks
    for (;;) {
        const unsigned long long r_at = tk < total ? r : e.sweeps;
        if (round < r_at) {
            if (pending >= 0) {  // release it before any tempering barrier
                if (threadIdx.x == 0) {
                    __threadfence();
                    atomicAdd(&e.done[pending], (unsigned long long)pending_n);
                }
                pending = -1;
            }
            for (; round < r_at; ++round) {  // past the end of sweep `round`: its tempering phase
                const unsigned long long swept = e.ls->sweep + round + 1;
                if (e.n_ladders && e.pt_every > 0 && swept % (unsigned long long)e.pt_every == 0) {
                    grid_barrier(e);  // every member's sweeps complete
                    energy_phase(e);
                    grid_barrier(e);
                    if (blockIdx.x == 0) {
                        swap_phase(e, e.ls->pt_attempts + swept / (unsigned long long)e.pt_every - 1);
                        __syncthreads();
                        for (int k = threadIdx.x; k < e.n_members; k += blockDim.x) e.energy[k] = 0;  // next phase
                    }
                    grid_barrier(e);
                }
            }
        }
        if (tk >= total) break;
        const int m = it.member, p = it.pass;
        PassFields pf;
        uint32_t tv = 0;
        const EnsMember &mem = e.members[m];
        if (threadIdx.x == 0) {
            const unsigned long long next = atomicAdd(&e.ls->ticket, 1ull);  // used after this item
            wait_member(e, m, r, p);
            s_ticket = next;
        } else if (threadIdx.x >= 32 && threadIdx.x < 48) {
            pf = pass_fields(e, m, p, r);
            const int k = (int)threadIdx.x - 32;
            const int nk = 2 + 4 * (mem.link ? mem.a.g.d - 1 : mem.a.g.d);  // keys of a q = 2 table
            if (mem.pk && k < nk) tv = table_entry((mem.a.kernel == PLQ_HEATBATH ? pf.hb24 : pf.metro24)[k]);
        } else if (threadIdx.x == 64 && pending >= 0) {
            __threadfence();
            atomicAdd(&e.done[pending], (unsigned long long)pending_n);
        }
        if (m != last_m) {  // the member's arguments into shared memory, one 32-bit word per thread
            const uint32_t *src = reinterpret_cast<const uint32_t *>(&e.members[m].a);
            uint32_t *dst = reinterpret_cast<uint32_t *>(&sa);
            for (int k = threadIdx.x; k < (int)(sizeof(LocalArgs) / 4); k += blockDim.x) dst[k] = src[k];
            last_m = m;
        }
        __syncthreads();  // the wait is over, the previous item released, the arguments loaded
        if (threadIdx.x == 32) apply(pf, sa);
        if (threadIdx.x >= 32 && threadIdx.x < 48) s_tab[threadIdx.x - 32] = tv;
        // the next item's entry, loaded while this one runs
        const unsigned long long tk_next = s_ticket;
        unsigned long long r_next = 0;
        WorkItem it_next{0, 0, 0, 0};
        if (tk_next < total) {
            r_next = tk_next / n_items;
            it_next = e.items[tk_next - r_next * n_items];
        }
        __syncthreads();
        for (int q = 0; q < it.count; ++q) {
            const int64_t chunk = (int64_t)it.chunk + q;
            if (mem.pk && mem.link) {
                uint32_t *pk = static_cast<uint32_t *>(mem.pk);
                switch (sa.g.d * 4 + sa.dir) {
                    case 8: packed_link_item<2, 0>(sa, pk, chunk, mem.wpt, s_tab); break;
                    case 9: packed_link_item<2, 1>(sa, pk, chunk, mem.wpt, s_tab); break;
                    case 12: packed_link_item<3, 0>(sa, pk, chunk, mem.wpt, s_tab); break;
                    case 13: packed_link_item<3, 1>(sa, pk, chunk, mem.wpt, s_tab); break;
                    case 14: packed_link_item<3, 2>(sa, pk, chunk, mem.wpt, s_tab); break;
                    case 16: packed_link_item<4, 0>(sa, pk, chunk, mem.wpt, s_tab); break;
                    case 17: packed_link_item<4, 1>(sa, pk, chunk, mem.wpt, s_tab); break;
                    case 18: packed_link_item<4, 2>(sa, pk, chunk, mem.wpt, s_tab); break;
                    case 19: packed_link_item<4, 3>(sa, pk, chunk, mem.wpt, s_tab); break;
                    default: break;
                }
            } else if (mem.pk) {
                if (mem.pk_wide) {
                    uint64_t *pk = static_cast<uint64_t *>(mem.pk);
                    if (sa.g.d == 2) packed_site_item<2, uint64_t>(sa, pk, chunk, mem.wpt, s_tab);
                    else packed_site_item<3, uint64_t>(sa, pk, chunk, mem.wpt, s_tab);
                } else {
                    uint32_t *pk = static_cast<uint32_t *>(mem.pk);
                    if (sa.g.d == 2) packed_site_item<2, uint32_t>(sa, pk, chunk, mem.wpt, s_tab);
                    else packed_site_item<3, uint32_t>(sa, pk, chunk, mem.wpt, s_tab);
                }
            } else {
                run_item<R, WORDS_ONLY>(sa, sa.g.d, mem.link, chunk, mem.wpt);
            }
        }
        __syncthreads();  // every thread's stores of the item are done (released by the next step)
        pending = m;
        pending_n = it.count;
        tk = tk_next;
        r = r_next;
        it = it_next;
    }
    if (pending >= 0 && threadIdx.x == 0) {
        __threadfence();
        atomicAdd(&e.done[pending], (unsigned long long)pending_n);
    }
    // advance the device-resident launch state (block 0, after every CTA left the loop)
    grid_barrier(e);
    if (blockIdx.x == 0) {
        for (int m = threadIdx.x; m < e.n_members; m += blockDim.x) {
            if (e.members[m].a.jump) e.pos[m] += e.sweeps * (unsigned long long)e.members[m].n_vars;
            if (e.msweep) e.msweep[m] += e.sweeps;
            e.done[m] = 0;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            e.ls->sweep += e.sweeps;
            e.ls->ticket = 0;
        }
    }
}

// Unbatched path helpers: one member's energy, and one swap attempt.
__global__ void member_energy_kernel(EnsArgs e, int m) {
    __shared__ LocalArgs sa;
    if (threadIdx.x == 0) sa = e.members[m].a;
    __syncthreads();
    const int64_t n = sa.g.n_sites;
    for (int64_t c = blockIdx.x; c * kEnergyChunk < n; c += gridDim.x) {
        long long tot = block_sum(energy_item(sa, sa.g.d, e.members[m].link, c));
        if (threadIdx.x == 0 && tot) atomicAdd((unsigned long long *)&e.energy[m], (unsigned long long)tot);
    }
}
__global__ void swap_kernel(EnsArgs e, unsigned long long att) { swap_phase(e, att); }

}  // namespace

struct plq_ensemble {
    plq_ctx ctx_copy;        // the context's record, copied at creation (outlives the caller's)
    plq_ctx *ctx = nullptr;  // = &ctx_copy
    cudaStream_t stream = nullptr;
    std::vector<plq_chain_desc> descs;
    std::vector<EnsMember> members;            // host copies (device pointers inside)
    std::vector<int64_t> n_vars;
    std::vector<void *> allocs;                // everything to cudaFree
    std::vector<TableSet> tsets;
    std::vector<int32_t> ts_of_member;
    std::vector<std::vector<int32_t>> ladders;
    std::vector<LadderDev> ladder_dev;
    int pt_every = 0;
    EnsMember *d_members = nullptr;
    TableSet *d_tsets = nullptr;
    int32_t *d_ts = nullptr;
    unsigned long long *d_pos = nullptr;
    unsigned long long *d_done = nullptr;  // per-member work-item counters of the persistent launch
    long long *d_energy = nullptr;
    LadderDev *d_ladders = nullptr;
    LaunchState *d_ls = nullptr;
    Control *d_ctrl = nullptr;
    // work items for the current configuration
    int ranks = 4;
    int ctas_per_sm = 2;
    bool words_only = false;  // every member runs four sites at a time
    WorkItem *d_items = nullptr;
    int64_t n_items = 0;
    int32_t *d_e_member = nullptr, *d_e_chunk = nullptr;
    int64_t n_e_items = 0;
    uint64_t launches = 0;
    uint64_t sweeps_done = 0;
    uint64_t pt_attempts_host = 0;
    // graph cache
    cudaGraphExec_t graph = nullptr;
    uint64_t graph_sweeps = 0;
    int graph_ranks = 0, graph_ctas = 0;
    // packed Z2 members: their packing table (device) and its index space
    PackEntry *d_pack = nullptr;
    int n_pack = 0;
    uint32_t pack_total = 0;
    // every member's primaries: one device buffer, the launches captured once
    long long *d_prims_all = nullptr;
    std::vector<int64_t> prims_offset;  // member m's first entry
    PrimTask *d_prim_tasks = nullptr;   // every member's measurement task (the states never move)
    int32_t *d_prim_task = nullptr, *d_prim_chunk = nullptr;
    int64_t n_prim_items = 0;
    // The same from the packed rows: after a batched launch every packed member's rows still
    // hold its configuration (unpacking leaves them), so its primaries are row popcounts.
    // pk_current: no byte state has been written since the last batched launch.
    bool pk_current = false;
    int32_t *d_prim_task_bytes = nullptr, *d_prim_chunk_bytes = nullptr;  // items of unpacked members
    int64_t n_prim_items_bytes = 0;
    int32_t *d_pk_prim_member = nullptr, *d_pk_prim_chunk = nullptr;     // row chunks of packed members
    int64_t n_pk_prim_items = 0;
    int64_t *d_prims_offset = nullptr;
};

namespace {

int ens_fail(cudaError_t e, const char *what) {
    return plq_fail(e == cudaErrorMemoryAllocation ? PLQ_ENOMEM : PLQ_ECUDA,
                    std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
cudaError_t dev_upload(plq_ensemble *E, const T *host, size_t count, T **out) {
    *out = nullptr;
    if (count == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc((void **)out, count * sizeof(T));
    if (e != cudaSuccess) return e;
    E->allocs.push_back(*out);
    return cudaMemcpyAsync(*out, host, count * sizeof(T), cudaMemcpyHostToDevice, E->stream);
}

void drop_graph(plq_ensemble *E) {
    if (E->graph) cudaGraphExecDestroy(E->graph);
    E->graph = nullptr;
}

// Estimated time of work item `c` of a member (arbitrary units: only the
// order of items matters): the units of its busiest thread -- packed rows,
// four-site words or colour ranks -- times their cost in instructions.
int64_t item_cost(const EnsMember &mem, int64_t c, int ranks) {
    const LocalArgs &a = mem.a;
    const bool shaped = a.words || mem.pk;
    const int64_t per_thread = shaped ? mem.wpt : ranks;
    const int64_t chunk = (int64_t)kEnsThreads * per_thread;
    const int64_t units = mem.pk ? a.g.n_sites / a.g.L[0] : (a.words ? a.g.n_sites / 4 : a.g.n_sites / 2);
    const int64_t in_item = std::min(chunk, units - c * chunk);
    const int64_t busiest = std::min(per_thread, (in_item + kEnsThreads - 1) / kEnsThreads);
    int64_t unit_cost;
    if (mem.pk) {  // a row: its staples or neighbour counts, then L0 / 2 updates
        const int64_t upd = a.g.L[0] / 2;
        unit_cost = mem.link ? 40 * upd + 35 * (a.g.d - 1) : 35 * upd + 12 * a.g.d;
    } else if (a.words) {
        unit_cost = 400;  // four sites of one colour in bytes
    } else {
        unit_cost = 150;  // one colour rank, generic body
    }
    return busiest * unit_cost;
}

// Work items of one sweep of members `ids`, by super-phase; member indices
// are relative to lo.  With S super-phases (the most colour passes of any
// member), pass p of a member with P passes runs in super-phases [p S / P,
// (p + 1) S / P), its chunks split evenly over them: a site lattice's two
// colours each spread over half the super-phases, a 4D gauge lattice's eight
// passes one per super-phase, so every super-phase holds a similar share of
// the sweep.  A chunk is 256 * wpt four-site words or packed rows (256 *
// ranks colour ranks in the generic body).  Where a super-phase holds more
// than 2 * min_items chunks, an item takes a run of g of a pass's consecutive
// chunks (g = chunks / min_items) to keep the per-item overhead small; else
// one.  Each super-phase lists its items largest first (item_cost times
// count), as the kernel deals them out in list order.  Returns S.
int append_items(const EnsMember *mems, const std::vector<size_t> &ids, size_t lo, int ranks, int64_t min_items,
                 std::vector<WorkItem> &items) {
    int S = 0;
    for (size_t m : ids) S = std::max(S, mems[m].passes);
    struct Span {
        size_t m;
        int p;
        int64_t c0, c1;
    };
    for (int sp = 0; sp < S; ++sp) {
        std::vector<Span> spans;
        int64_t chunks = 0;
        for (size_t m : ids) {
            const int P = mems[m].passes;
            const LocalArgs &ma = mems[m].a;
            const bool shaped = ma.words || mems[m].pk;
            const int64_t chunk = (int64_t)kEnsThreads * (shaped ? mems[m].wpt : ranks);
            const int64_t units = mems[m].pk ? (int64_t)row_count(ma.g) : (ma.words ? ma.g.n_sites / 4 : ma.g.n_sites / 2);
            const int64_t nc = (units + chunk - 1) / chunk;
            for (int p = 0; p < P; ++p) {
                const int p0 = p * S / P, p1 = (p + 1) * S / P;
                if (sp < p0 || sp >= p1) continue;
                const int64_t c0 = (int64_t)(sp - p0) * nc / (p1 - p0), c1 = (int64_t)(sp - p0 + 1) * nc / (p1 - p0);
                if (c1 > c0) spans.push_back(Span{m, p, c0, c1});
                chunks += c1 - c0;
            }
        }
        const int64_t g = min_items > 0 && chunks > 2 * min_items ? chunks / min_items : 1;
        const size_t first = items.size();
        for (const Span &sn : spans)
            for (int64_t c = sn.c0; c < sn.c1; c += g)
                items.push_back(WorkItem{(int32_t)(sn.m - lo), (int32_t)c, (int32_t)std::min(g, sn.c1 - c), sn.p});
        // largest first; equal costs keep member order
        const size_t n = items.size() - first;
        std::vector<int64_t> cost(n);
        for (size_t k = 0; k < n; ++k) {
            const WorkItem &w = items[first + k];
            cost[k] = item_cost(mems[(size_t)w.member + lo], w.chunk, ranks) * w.count;
        }
        std::vector<size_t> ord(n);
        for (size_t k = 0; k < n; ++k) ord[k] = k;
        std::stable_sort(ord.begin(), ord.end(), [&](size_t x, size_t y) { return cost[x] > cost[y]; });
        std::vector<WorkItem> sorted(n);
        for (size_t k = 0; k < n; ++k) sorted[k] = items[first + ord[k]];
        std::copy(sorted.begin(), sorted.end(), items.begin() + first);
    }
    return S;
}

// Items per super-phase below which chunks are not grouped into runs, per SM
// (about four per CTA at four CTAs per SM).
constexpr int64_t kItemsPerSm = 16;

// The launch's item list must name only its own members (the kernel indexes
// the member array with it unchecked).
bool items_in_range(const WorkItem *items, size_t n, size_t n_members) {
    for (size_t k = 0; k < n; ++k)
        if (items[k].member < 0 || (size_t)items[k].member >= n_members || items[k].count <= 0) return false;
    return true;
}

int build_items(plq_ensemble *E) {
    std::vector<WorkItem> items;
    std::vector<size_t> all(E->members.size());
    for (size_t m = 0; m < all.size(); ++m) all[m] = m;
    append_items(E->members.data(), all, 0, E->ranks, kItemsPerSm * E->ctx->sm_count, items);
    if (!items_in_range(items.data(), items.size(), E->members.size()))
        return plq_fail(PLQ_EINVAL, "ensemble work items name a member out of range");
    std::vector<int32_t> em, ec;
    for (auto &l : E->ladders)
        for (int32_t m : l) {
            const EnsMember &mem = E->members[m];
            // packed members: one row per thread; bytes: kEnergyChunk sites per item
            const int64_t nc = mem.pk ? (mem.a.g.n_sites / mem.a.g.L[0] + kEnsThreads - 1) / kEnsThreads
                                      : (mem.a.g.n_sites + kEnergyChunk - 1) / kEnergyChunk;
            for (int64_t c = 0; c < nc; ++c) {
                em.push_back(m);
                ec.push_back((int32_t)c);
            }
        }
    void *old[] = {E->d_items, E->d_e_member, E->d_e_chunk};
    for (void *p : old)
        if (p) {
            cudaFree(p);
            E->allocs.erase(std::remove(E->allocs.begin(), E->allocs.end(), p), E->allocs.end());
        }
    cudaError_t e = dev_upload(E, items.data(), items.size(), &E->d_items);
    if (e == cudaSuccess) e = dev_upload(E, em.data(), em.size(), &E->d_e_member);
    if (e == cudaSuccess) e = dev_upload(E, ec.data(), ec.size(), &E->d_e_chunk);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
    if (e != cudaSuccess) return ens_fail(e, "ensemble work items");
    E->n_items = (int64_t)items.size();
    E->n_e_items = (int64_t)em.size();
    drop_graph(E);
    return PLQ_OK;
}

EnsArgs ens_args(plq_ensemble *E, uint64_t sweeps) {
    EnsArgs a;
    std::memset(&a, 0, sizeof a);
    a.members = E->d_members;
    a.n_members = (int)E->members.size();
    a.tsets = E->d_tsets;
    a.ts_of_member = E->d_ts;
    a.pos = E->d_pos;
    a.done = E->d_done;
    a.items = E->d_items;
    a.n_items = E->n_items;
    a.e_item_member = E->d_e_member;
    a.e_item_chunk = E->d_e_chunk;
    a.n_e_items = E->n_e_items;
    a.energy = E->d_energy;
    a.ladders = E->d_ladders;
    a.n_ladders = (int)E->ladders.size();
    a.pt_every = E->pt_every;
    a.ls = E->d_ls;
    a.ctrl = E->d_ctrl;
    a.sweeps = sweeps;
    a.ranks = E->ranks;
    return a;
}

template <int R>
const void *kernel_for(bool words_only) {
    return words_only ? (const void *)ensemble_kernel<R, true> : (const void *)ensemble_kernel<R, false>;
}

const void *kernel_ptr(int ranks, bool words_only) {
    switch (ranks) {
        case 2: return kernel_for<2>(words_only);
        case 4: return kernel_for<4>(words_only);
        default: return kernel_for<8>(words_only);
    }
}

int max_ctas_per_sm(int ranks, bool words_only) {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel_ptr(ranks, words_only), kEnsThreads, 0);
    return n;
}

// One persistent launch with arguments `a`: packed members are packed before
// and unpacked after it, so outside a launch every member is in byte planes.
// `tab` (n entries, `total` rows) is the packing table: the ensemble's by default.
cudaError_t launch_ensemble(plq_ensemble *E, EnsArgs &a, const PackEntry *tab = nullptr, int n = -1,
                            uint32_t total = 0) {
    if (n < 0) {
        tab = E->d_pack;
        n = E->n_pack;
        total = E->pack_total;
    }
    const unsigned pack_blocks = (unsigned)std::min<uint32_t>((total + 255) / 256, 148u * 8u);
    cudaError_t e = cudaSuccess;
    if (n) {
        pack_links_kernel<<<pack_blocks, 256, 0, E->stream>>>(tab, n, total, false);
        e = cudaGetLastError();
    }
    void *params[] = {&a};
    dim3 grid((unsigned)(E->ctx->sm_count * E->ctas_per_sm));
    if (e == cudaSuccess)
        e = cudaLaunchCooperativeKernel(kernel_ptr(E->ranks, E->words_only), grid, dim3(kEnsThreads), params, 0,
                                        E->stream);
    if (e == cudaSuccess && n) {
        pack_links_kernel<<<pack_blocks, 256, 0, E->stream>>>(tab, n, total, true);
        e = cudaGetLastError();
    }
    return e;
}

cudaError_t launch_persistent(plq_ensemble *E, uint64_t sweeps) {
    EnsArgs a = ens_args(E, sweeps);
    return launch_ensemble(E, a);
}

// Members that run packed, on the keyed stream with Metropolis or heat bath:
// Z2 gauge links with 2 <= d <= 4 and rows of at most 32 links; q = 2 sites
// (Ising, Potts at q = 2) with 2 <= d <= 3 (at most 6 neighbours for the
// counter) and rows of at most 64 sites.
bool packed_eligible(const plq_chain_desc &d) {
    if (d.rng != PLQ_RNG_KEYED || (d.updater != PLQ_HEATBATH && d.updater != PLQ_METROPOLIS) ||
        (d.flags & PLQ_FLAG_GENERIC_PASS))
        return false;
    if (d.model == PLQ_GAUGE) return d.d >= 2 && d.d <= 4 && d.shape[0] <= 32;
    const int q = d.model == PLQ_POTTS ? d.q : 2;
    return q == 2 && d.d >= 2 && d.d <= 3 && d.shape[0] <= 64;
}

// Bytes of a packed member's rows (every direction of a link member).
size_t packed_bytes(const plq_chain_desc &d, int64_t n_vars) {
    const size_t rows = (size_t)n_vars / (size_t)d.shape[0];  // links: d planes of rows
    return rows * (d.model != PLQ_GAUGE && d.shape[0] > 32 ? 8 : 4);
}

// The packing table of members `ids` (those with pk set) on the host.
std::vector<PackEntry> pack_entries(const plq_ensemble *E, const std::vector<size_t> &ids, uint32_t &total) {
    std::vector<PackEntry> tab;
    total = 0;
    for (size_t m : ids) {
        const EnsMember &mem = E->members[m];
        if (!mem.pk) continue;
        PackEntry t;
        std::memset(&t, 0, sizeof t);
        t.state = mem.a.state;
        t.pk = mem.pk;
        t.first = total;
        t.L0 = (uint32_t)mem.a.g.L[0];
        t.wide = mem.pk_wide;
        const uint32_t planes = mem.link ? (uint32_t)mem.a.g.d : 1u;
        total += planes * (uint32_t)(mem.a.g.n_sites / mem.a.g.L[0]);
        tab.push_back(t);
    }
    return tab;
}

// The device packing table of every member with pk set.
cudaError_t build_pack_table(plq_ensemble *E) {
    std::vector<size_t> all(E->members.size());
    for (size_t m = 0; m < all.size(); ++m) all[m] = m;
    uint32_t total = 0;
    std::vector<PackEntry> tab = pack_entries(E, all, total);
    if (E->d_pack) {
        cudaFree(E->d_pack);
        E->allocs.erase(std::remove(E->allocs.begin(), E->allocs.end(), (void *)E->d_pack), E->allocs.end());
        E->d_pack = nullptr;
    }
    E->n_pack = (int)tab.size();
    E->pack_total = total;
    if (tab.empty()) return cudaSuccess;
    return dev_upload(E, tab.data(), tab.size(), &E->d_pack);
}

}  // namespace

extern "C" int plq_ensemble_create(plq_ctx *ctx, int32_t n, const plq_chain_desc *descs, const uint8_t *const *starts,
                                   plq_ensemble **out) {
    if (!ctx || !descs || !out || n <= 0) return plq_fail(PLQ_EINVAL, "bad arguments");
    *out = nullptr;
    for (int32_t m = 0; m < n; ++m) {
        const plq_chain_desc &d = descs[m];
        int rc = plq_chain_validate(&d);
        if (rc != PLQ_OK) return rc;
        if (d.updater == PLQ_CLUSTER) return plq_fail(PLQ_EUNSUPPORTED, "ensembles take local updaters only");
        if (d.d > 4) return plq_fail(PLQ_EUNSUPPORTED, "ensemble members have at most 4 dimensions");
        if (d.rng == PLQ_RNG_STREAM && d.updater == PLQ_METROPOLIS)
            return plq_fail(PLQ_EUNSUPPORTED,
                            "stream-mode Metropolis needs a device-wide scan per pass; ensembles run it keyed");
        if (d.sweep_offset != descs[0].sweep_offset)
            return plq_fail(PLQ_EINVAL, "ensemble members share one sweep counter: every sweep_offset must be equal");
    }
    if (starts) {  // every member's start below its q, checked on the host threads
        std::vector<int64_t> nv(n);
        std::vector<int> qs(n);
        for (int32_t m = 0; m < n; ++m) {
            const plq_chain_desc &d = descs[m];
            int64_t ns = 1;
            for (int i = 0; i < d.d; ++i) ns *= d.shape[i];
            nv[m] = d.model == PLQ_GAUGE ? ns * d.d : ns;
            qs[m] = d.model == PLQ_POTTS ? d.q : 2;
        }
        if (first_bad_start(n, starts, nv.data(), qs.data()) >= 0)
            return plq_fail(PLQ_EINVAL, "start state out of range");
    }
    cudaError_t ce = plq_enter_device(ctx->device);
    if (ce != cudaSuccess) return ens_fail(ce, "cudaSetDevice");
    plq_ensemble *E = new plq_ensemble();
    E->ctx_copy = *ctx;
    E->ctx = &E->ctx_copy;
    auto fail = [&](int code) {
        plq_ensemble_destroy(E);
        return code;
    };
    ce = cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) return fail(ens_fail(ce, "stream"));
    E->descs.assign(descs, descs + n);
    // 1. on the host: every member's geometry, decision tables and (PCG stream) jump table,
    //    then one device arena for all states and one for all tables -- a few allocations
    //    and one synchronisation for the whole ensemble rather than several per member
    auto align = [](size_t b) { return (b + 255) & ~(size_t)255; };
    std::vector<Tables> tables(n);
    std::map<std::string, int32_t> table_of;  // host build of each distinct parameter set
    std::vector<std::vector<AffineHost>> jumps(n);
    size_t state_bytes = 0, table_bytes = 0, stage_bytes = 0;
    for (int32_t m = 0; m < n; ++m) {
        const plq_chain_desc &d = descs[m];
        EnsMember mem;
        std::memset(&mem, 0, sizeof mem);
        LocalArgs &a = mem.a;
        const int q = d.model == PLQ_POTTS ? d.q : 2;
        a.g.d = d.d;
        int64_t ns = 1;
        for (int i = 0; i < kMaxD; ++i) {
            a.g.L[i] = i < d.d ? (int32_t)d.shape[i] : 1;
            a.g.stride[i] = ns;
            if (i < d.d) ns *= d.shape[i];
        }
        a.g.n_sites = ns;
        geom_init(a.g, d.d, d.shape);
        mem.link = d.model == PLQ_GAUGE;
        mem.passes = mem.link ? 2 * d.d : 2;
        mem.n_vars = mem.link ? ns * d.d : ns;
        mem.j = d.j;
        mem.ladder = -1;
        a.q = q;
        a.kernel = d.updater;
        a.model = d.model;
        int32_t w = 1;
        for (int s = 1; s < q; ++s) {
            a.pw[s] = w;
            w *= 2 * d.d + 1;
        }
        a.seed32 = plq_fold_seed(d.seed);
        a.words = !(d.flags & PLQ_FLAG_GENERIC_PASS) &&
                  words_eligible(d.model, q, d.d, a.g.L, d.updater, d.rng) ? 1 : 0;
        mem.wpt = tuned_wpt(d);
        ModelParams p;
        std::memset(&p, 0, sizeof p);
        p.model = d.model;
        p.q = q;
        p.d = d.d;
        p.beta = d.beta;
        p.j = d.j;
        p.h = d.h;
        for (int k = 0; k < PLQ_MAX_Q; ++k) p.offsets[k] = d.offsets[k];
        // members with the same model parameters, updater and stream share one host build (the
        // device copies stay per member: a member's tables are rewritten in place when its beta
        // changes)
        std::string key(reinterpret_cast<const char *>(&p), sizeof p);
        key.append(reinterpret_cast<const char *>(&d.updater), sizeof d.updater);
        key.append(reinterpret_cast<const char *>(&d.rng), sizeof d.rng);
        auto built = table_of.find(key);
        if (built != table_of.end()) {
            tables[m] = tables[built->second];
        } else {
            std::string err;
            if (!build_tables(p, d.updater, d.rng, tables[m], err)) return fail(plq_fail(PLQ_EUNSUPPORTED, err));
            table_of.emplace(std::move(key), m);
        }
        const Tables &t = tables[m];
        table_bytes += align(t.hb53.size() * 8) + align(t.hb24.size() * 4) + align(t.metro53.size() * 8) +
                       align(t.metro24.size() * 4);
        if (d.rng == PLQ_RNG_STREAM) {
            uint64_t slo, shi, ilo, ihi;
            pcg_seed_from_u64(d.seed, slo, shi, ilo, ihi);
            build_jump_table(ilo, ihi, jumps[m]);
            a.inc = u128{ilo, ihi};
            u128 s0 = jump(reinterpret_cast<const Affine *>(jumps[m].data()), u128{slo, shi}, d.stream_offset);
            a.base = pcg_step(s0, a.inc);
            table_bytes += align(jumps[m].size() * sizeof(AffineHost));
        }
        state_bytes += align((size_t)mem.n_vars);
        if (packed_eligible(d)) state_bytes += align(packed_bytes(d, mem.n_vars));
        if (mem.link && starts && starts[m]) stage_bytes = std::max(stage_bytes, (size_t)mem.n_vars);
        E->members.push_back(mem);
        E->n_vars.push_back(mem.n_vars);
        E->ts_of_member.push_back(-1);
    }
    uint8_t *state_arena = nullptr, *table_arena = nullptr, *stage = nullptr;
    ce = cudaMalloc((void **)&state_arena, std::max<size_t>(state_bytes, 256));
    if (ce == cudaSuccess) E->allocs.push_back(state_arena);
    if (ce == cudaSuccess) ce = cudaMalloc((void **)&table_arena, std::max<size_t>(table_bytes, 256));
    if (ce == cudaSuccess) E->allocs.push_back(table_arena);
    if (ce == cudaSuccess && stage_bytes) ce = cudaMalloc((void **)&stage, stage_bytes);
    if (ce != cudaSuccess) {
        if (stage) cudaFree(stage);
        return fail(ens_fail(ce, "ensemble arenas"));
    }
    // 2. the uploads, in stream order: starts (links through one staging buffer and the
    //    plane conversion), then every table and jump table laid out in one host image of the
    //    table arena and copied in one transfer
    size_t soff = 0, toff = 0;
    std::vector<uint8_t> table_image(std::max<size_t>(table_bytes, 256), 0);
    auto put = [&](const void *host, size_t bytes) -> void * {
        if (!bytes) return nullptr;
        void *dst = table_arena + toff;
        std::memcpy(table_image.data() + toff, host, bytes);
        toff += align(bytes);
        return dst;
    };
    for (int32_t m = 0; m < n && ce == cudaSuccess; ++m) {
        EnsMember &mem = E->members[m];
        LocalArgs &a = mem.a;
        uint8_t *st = state_arena + soff;
        soff += align((size_t)mem.n_vars);
        a.state = st;
        if (packed_eligible(descs[m])) {
            mem.pk = state_arena + soff;
            mem.pk_wide = descs[m].model != PLQ_GAUGE && descs[m].shape[0] > 32 ? 1 : 0;
            soff += align(packed_bytes(descs[m], mem.n_vars));
        }
        if (starts && starts[m]) {
            if (mem.link) {
                ce = cudaMemcpyAsync(stage, starts[m], (size_t)mem.n_vars, cudaMemcpyHostToDevice, E->stream);
                if (ce == cudaSuccess) ce = launch_links_to_planes(stage, st, a.g.n_sites, a.g.d, E->stream);
            } else {
                ce = cudaMemcpyAsync(st, starts[m], (size_t)mem.n_vars, cudaMemcpyHostToDevice, E->stream);
            }
        } else {
            ce = cudaMemsetAsync(st, 0, (size_t)mem.n_vars, E->stream);
        }
        if (!jumps[m].empty()) a.jump = reinterpret_cast<const Affine *>(put(jumps[m].data(),
                                                                             jumps[m].size() * sizeof(AffineHost)));
        const Tables &t = tables[m];
        TableSet ts;
        std::memset(&ts, 0, sizeof ts);
        ts.beta = descs[m].beta;
        ts.hb53 = (const uint64_t *)put(t.hb53.data(), t.hb53.size() * 8);
        ts.hb24 = (const uint32_t *)put(t.hb24.data(), t.hb24.size() * 4);
        ts.metro53 = (const uint64_t *)put(t.metro53.data(), t.metro53.size() * 8);
        ts.metro24 = (const uint32_t *)put(t.metro24.data(), t.metro24.size() * 4);
        E->ts_of_member[m] = (int32_t)E->tsets.size();
        E->tsets.push_back(ts);
    }
    if (ce == cudaSuccess && toff)
        ce = cudaMemcpyAsync(table_arena, table_image.data(), toff, cudaMemcpyHostToDevice, E->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(E->stream);
    if (stage) cudaFree(stage);
    if (ce != cudaSuccess) return fail(ens_fail(ce, "member set-up"));
    ce = build_pack_table(E);
    if (ce != cudaSuccess) return fail(ens_fail(ce, "packing table"));
    std::vector<unsigned long long> pos(n, 0);
    std::vector<long long> zeros(n, 0);
    LaunchState ls;
    std::memset(&ls, 0, sizeof ls);
    ls.sweep = descs[0].sweep_offset;  // the keyed sweep key resumes here
    E->sweeps_done = descs[0].sweep_offset;
    Control ctrl;
    std::memset(&ctrl, 0, sizeof ctrl);
    ce = dev_upload(E, E->members.data(), E->members.size(), &E->d_members);
    if (ce == cudaSuccess) ce = dev_upload(E, E->tsets.data(), E->tsets.size(), &E->d_tsets);
    if (ce == cudaSuccess) ce = dev_upload(E, E->ts_of_member.data(), E->ts_of_member.size(), &E->d_ts);
    if (ce == cudaSuccess) ce = dev_upload(E, pos.data(), pos.size(), &E->d_pos);
    if (ce == cudaSuccess) ce = dev_upload(E, pos.data(), pos.size(), &E->d_done);  // zeros
    if (ce == cudaSuccess) ce = dev_upload(E, zeros.data(), zeros.size(), &E->d_energy);
    if (ce == cudaSuccess) ce = dev_upload(E, &ls, 1, &E->d_ls);
    if (ce == cudaSuccess) ce = dev_upload(E, &ctrl, 1, &E->d_ctrl);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(E->stream);
    if (ce != cudaSuccess) return fail(ens_fail(ce, "ensemble set-up"));
    E->words_only = true;
    for (auto &m : E->members) E->words_only = E->words_only && m.a.words;
    E->ctas_per_sm = std::max(1, std::min(4, max_ctas_per_sm(E->ranks, E->words_only)));
    int rc = build_items(E);
    if (rc != PLQ_OK) return fail(rc);
    *out = E;
    return PLQ_OK;
}

namespace {

// Member m's current table set (the host copy) rebuilt at `beta`, in place:
// the table sizes depend on the model and shape only, so the device buffers
// (and every captured launch that reads them) stay.
int rebuild_tables(plq_ensemble *E, int32_t m, double beta, bool sync = true) {
    const plq_chain_desc &d = E->descs[m];
    ModelParams p;
    std::memset(&p, 0, sizeof p);
    p.model = d.model;
    p.q = d.model == PLQ_POTTS ? d.q : 2;
    p.d = d.d;
    p.beta = beta;
    p.j = d.j;
    p.h = d.h;
    for (int a = 0; a < PLQ_MAX_Q; ++a) p.offsets[a] = d.offsets[a];
    Tables t;
    std::string err;
    if (!build_tables(p, d.updater, d.rng, t, err)) return plq_fail(PLQ_EUNSUPPORTED, err);
    TableSet &ts = E->tsets[E->ts_of_member[m]];
    ts.beta = beta;
    const size_t bytes53 = t.hb53.size() * 8, bytes24 = t.hb24.size() * 4, m53 = t.metro53.size() * 8,
                 m24 = t.metro24.size() * 4;
    cudaError_t ce = cudaSuccess;
    if (bytes53) ce = cudaMemcpyAsync((void *)ts.hb53, t.hb53.data(), bytes53, cudaMemcpyHostToDevice, E->stream);
    if (ce == cudaSuccess && bytes24)
        ce = cudaMemcpyAsync((void *)ts.hb24, t.hb24.data(), bytes24, cudaMemcpyHostToDevice, E->stream);
    if (ce == cudaSuccess && m53)
        ce = cudaMemcpyAsync((void *)ts.metro53, t.metro53.data(), m53, cudaMemcpyHostToDevice, E->stream);
    if (ce == cudaSuccess && m24)
        ce = cudaMemcpyAsync((void *)ts.metro24, t.metro24.data(), m24, cudaMemcpyHostToDevice, E->stream);
    if (ce == cudaSuccess && E->d_tsets)
        ce = cudaMemcpyAsync(E->d_tsets + E->ts_of_member[m], &ts, sizeof ts, cudaMemcpyHostToDevice, E->stream);
    // the host tables are pageable: each copy is staged before cudaMemcpyAsync returns, so
    // they may go out of scope unsynchronised
    if (ce == cudaSuccess && sync) ce = cudaStreamSynchronize(E->stream);
    if (ce != cudaSuccess) return ens_fail(ce, "member tables");
    return PLQ_OK;
}

}  // namespace

extern "C" int plq_ensemble_set_beta(plq_ensemble *E, int32_t m, double beta) {
    if (!E || m < 0 || m >= (int32_t)E->members.size()) return plq_fail(PLQ_EINVAL, "bad arguments");
    if (E->members[m].ladder >= 0)
        return plq_fail(PLQ_EINVAL, "the beta of a member in a tempering ladder belongs to its ladder");
    cudaError_t ce = plq_enter_device(E->ctx->device);
    if (ce != cudaSuccess) return ens_fail(ce, "cudaSetDevice");
    const int rc = rebuild_tables(E, m, beta);
    if (rc != PLQ_OK) return rc;
    E->descs[m].beta = beta;
    return PLQ_OK;
}

extern "C" int plq_ensemble_add_ladder(plq_ensemble *E, int32_t k, const int32_t *member_ids, const double *betas,
                                       int32_t every, uint64_t seed) {
    if (!E || k < 2 || !member_ids || !betas || every <= 0) return plq_fail(PLQ_EINVAL, "bad ladder arguments");
    if (E->pt_every && E->pt_every != every) return plq_fail(PLQ_EINVAL, "all ladders share one swap interval");
    const plq_chain_desc &d0 = E->descs[member_ids[0]];
    std::vector<int32_t> ids(member_ids, member_ids + k);
    for (int32_t i = 0; i < k; ++i) {
        int32_t m = ids[i];
        if (m < 0 || m >= (int32_t)E->members.size()) return plq_fail(PLQ_EINVAL, "ladder member out of range");
        if (E->members[m].ladder >= 0) return plq_fail(PLQ_EINVAL, "a member belongs to one ladder at most");
        const plq_chain_desc &d = E->descs[m];
        bool same = d.model == d0.model && d.q == d0.q && d.d == d0.d && d.updater == d0.updater && d.rng == d0.rng &&
                    d.j == d0.j && d.h == 0.0;
        for (int a = 0; a < d.d; ++a) same = same && d.shape[a] == d0.shape[a];
        for (int a = 0; a < PLQ_MAX_Q; ++a) same = same && d.offsets[a] == 0.0;
        if (!same)
            return plq_fail(PLQ_EINVAL, "ladder members must share model, shape, updater and coupling, with no field");
    }
    // slot i of the ladder runs at betas[i]: rebuild member i's table set at that beta (unless
    // it already runs at it; members outside ladders keep their own table set)
    for (int32_t i = 0; i < k; ++i) {
        const int32_t m = ids[i];
        const int rc = E->tsets[E->ts_of_member[m]].beta == betas[i] ? PLQ_OK : rebuild_tables(E, m, betas[i], false);
        if (rc != PLQ_OK) return rc;
        E->members[m].ladder = (int)E->ladders.size();
    }
    int32_t *d_slots = nullptr;
    cudaError_t ce = dev_upload(E, ids.data(), ids.size(), &d_slots);
    if (ce != cudaSuccess) return ens_fail(ce, "ladder slots");
    cudaError_t pe = build_pack_table(E);
    if (pe != cudaSuccess) return ens_fail(pe, "packing table");
    LadderDev L;
    L.k = k;
    L.every = every;
    L.seed32 = plq_fold_seed(seed);
    L.member_of_slot = d_slots;
    E->ladders.push_back(ids);
    E->ladder_dev.push_back(L);
    E->pt_every = every;
    if (E->d_ladders) {
        cudaFree(E->d_ladders);
        E->allocs.erase(std::remove(E->allocs.begin(), E->allocs.end(), (void *)E->d_ladders), E->allocs.end());
    }
    ce = dev_upload(E, E->ladder_dev.data(), E->ladder_dev.size(), &E->d_ladders);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(E->d_tsets, E->tsets.data(), E->tsets.size() * sizeof(TableSet),
                                                cudaMemcpyHostToDevice, E->stream);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(E->d_members, E->members.data(), E->members.size() * sizeof(EnsMember),
                             cudaMemcpyHostToDevice, E->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(E->stream);
    if (ce != cudaSuccess) return ens_fail(ce, "ladder upload");
    return build_items(E);
}

static int ens_status(plq_ensemble *E) {
    unsigned int st = 0;
    cudaError_t e = cudaMemcpyAsync(&st, &E->d_ctrl->status, sizeof st, cudaMemcpyDeviceToHost, E->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
    if (e != cudaSuccess) return ens_fail(e, "ensemble sync");
    if (st) return plq_fail(PLQ_EDEVICE, "ensemble status word " + std::to_string(st) + " (1 = barrier wait limit)");
    return PLQ_OK;
}

extern "C" int plq_ensemble_advance(plq_ensemble *E, uint64_t sweeps) {
    if (!E) return plq_fail(PLQ_EINVAL, "NULL ensemble");
    if (sweeps == 0) return PLQ_OK;
    cudaError_t e = plq_enter_device(E->ctx->device);
    if (e != cudaSuccess) return ens_fail(e, "cudaSetDevice");
    // one persistent launch, captured once per (sweeps, configuration) and replayed
    if (!E->graph || E->graph_sweeps != sweeps || E->graph_ranks != E->ranks || E->graph_ctas != E->ctas_per_sm) {
        drop_graph(E);
        cudaGraph_t g = nullptr;
        e = cudaStreamBeginCapture(E->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t le = launch_persistent(E, sweeps);
            e = cudaStreamEndCapture(E->stream, &g);
            if (le != cudaSuccess) e = le;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&E->graph, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            cudaGetLastError();
            E->graph = nullptr;
            // capture refused: launch directly
            e = launch_persistent(E, sweeps);
            E->launches++;
            if (e != cudaSuccess) return ens_fail(e, "persistent launch");
            E->sweeps_done += sweeps;
            E->pk_current = true;
            return PLQ_OK;
        }
        E->graph_sweeps = sweeps;
        E->graph_ranks = E->ranks;
        E->graph_ctas = E->ctas_per_sm;
    }
    e = cudaGraphLaunch(E->graph, E->stream);
    E->launches++;
    if (e != cudaSuccess) return ens_fail(e, "graph launch");
    E->sweeps_done += sweeps;
    E->pk_current = true;
    return PLQ_OK;
}

extern "C" int plq_ensemble_advance_unbatched(plq_ensemble *E, uint64_t sweeps) {
    if (!E) return plq_fail(PLQ_EINVAL, "NULL ensemble");
    cudaError_t e = plq_enter_device(E->ctx->device);
    if (e != cudaSuccess) return ens_fail(e, "cudaSetDevice");
    if (sweeps) E->pk_current = false;  // the byte states move on without the packed rows
    // host mirrors of the device-resident state the per-member launches need
    LaunchState ls;
    std::vector<unsigned long long> pos(E->members.size());
    std::vector<int32_t> ts(E->members.size());
    e = cudaMemcpyAsync(&ls, E->d_ls, sizeof ls, cudaMemcpyDeviceToHost, E->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(pos.data(), E->d_pos, pos.size() * sizeof(pos[0]), cudaMemcpyDeviceToHost, E->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ts.data(), E->d_ts, ts.size() * sizeof(ts[0]), cudaMemcpyDeviceToHost, E->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
    if (e != cudaSuccess) return ens_fail(e, "unbatched state read");
    EnsArgs ea = ens_args(E, 0);
    for (uint64_t t = 0; t < sweeps; ++t) {
        for (size_t m = 0; m < E->members.size(); ++m) {
            const EnsMember &mem = E->members[m];
            LocalArgs a = mem.a;
            const TableSet &tsm = E->tsets[ts[m]];
            a.hb53 = tsm.hb53;
            a.hb24 = tsm.hb24;
            a.metro53 = tsm.metro53;
            a.metro24 = tsm.metro24;
            a.sweep32 = (uint32_t)(ls.sweep + t);
            for (int pass = 0; pass < mem.passes; ++pass) {
                a.dir = mem.link ? pass >> 1 : 0;
                a.color = pass & 1;
                if (a.jump) a.pass_offset = pos[m] + (uint64_t)pass * (uint64_t)(a.g.n_sites / 2);
                e = launch_local_pass(a, mem.link, false, E->stream);
                E->launches++;
                if (e != cudaSuccess) return ens_fail(e, "member pass");
            }
            if (a.jump) pos[m] += (unsigned long long)mem.n_vars;
        }
        const unsigned long long done = ls.sweep + t + 1;
        if (!E->ladders.empty() && done % (unsigned long long)E->pt_every == 0) {
            cudaMemsetAsync(E->d_energy, 0, sizeof(long long) * E->members.size(), E->stream);
            for (auto &l : E->ladders)
                for (int32_t m : l) {
                    int64_t nc = (E->members[m].a.g.n_sites + kEnergyChunk - 1) / kEnergyChunk;
                    member_energy_kernel<<<(unsigned)std::min<int64_t>(nc, 1184), kEnsThreads, 0, E->stream>>>(ea, m);
                    E->launches++;
                }
            swap_kernel<<<1, kEnsThreads, 0, E->stream>>>(ea, ls.pt_attempts + done / E->pt_every - 1);
            E->launches++;
            // energies start every phase at zero (the persistent launch relies on it too)
            cudaMemsetAsync(E->d_energy, 0, sizeof(long long) * E->members.size(), E->stream);
            e = cudaMemcpyAsync(ts.data(), E->d_ts, ts.size() * sizeof(ts[0]), cudaMemcpyDeviceToHost, E->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
            if (e != cudaSuccess) return ens_fail(e, "unbatched swaps");
        }
    }
    ls.sweep += sweeps;
    e = cudaMemcpyAsync(E->d_ls, &ls, sizeof ls, cudaMemcpyHostToDevice, E->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(E->d_pos, pos.data(), pos.size() * sizeof(pos[0]), cudaMemcpyHostToDevice, E->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
    if (e != cudaSuccess) return ens_fail(e, "unbatched state write");
    E->sweeps_done += sweeps;
    return PLQ_OK;
}

extern "C" int plq_ensemble_set_config(plq_ensemble *E, int32_t ranks_per_thread, int32_t ctas_per_sm) {
    if (!E) return plq_fail(PLQ_EINVAL, "NULL ensemble");
    if (ranks_per_thread != 2 && ranks_per_thread != 4 && ranks_per_thread != 8)
        return plq_fail(PLQ_EINVAL, "ranks per thread must be 2, 4 or 8");
    int maxc = max_ctas_per_sm(ranks_per_thread, E->words_only);
    if (ctas_per_sm < 1 || ctas_per_sm > maxc)
        return plq_fail(PLQ_EINVAL, "CTAs per SM must be in 1.." + std::to_string(maxc));
    E->ranks = ranks_per_thread;
    E->ctas_per_sm = ctas_per_sm;
    return build_items(E);
}

extern "C" int plq_ensemble_tune(plq_ensemble *E, int32_t trial_sweeps, int32_t *ranks_out, int32_t *ctas_out,
                                 double *ms_per_sweep_out) {
    if (!E || trial_sweeps <= 0) return plq_fail(PLQ_EINVAL, "bad arguments");
    cudaError_t e = plq_enter_device(E->ctx->device);
    if (e != cudaSuccess) return ens_fail(e, "cudaSetDevice");
    // snapshot: member states, PT slots, positions, launch state
    int64_t total = 0;
    for (auto v : E->n_vars) total += v;
    uint8_t *backup = nullptr;
    e = cudaMalloc((void **)&backup, (size_t)total);
    if (e != cudaSuccess) return ens_fail(e, "tune snapshot");
    std::vector<int32_t> ts(E->members.size());
    std::vector<unsigned long long> pos(E->members.size());
    LaunchState ls;
    std::vector<std::vector<int32_t>> slots;
    auto snapshot = [&](bool save) {
        // a restore rewrites the bytes; the trial launches (plq_ensemble_advance among them) left
        // the packed rows at their own states
        if (!save) E->pk_current = false;
        int64_t off = 0;
        for (size_t m = 0; m < E->members.size(); ++m) {
            if (save)
                cudaMemcpyAsync(backup + off, E->members[m].a.state, (size_t)E->n_vars[m], cudaMemcpyDeviceToDevice,
                                E->stream);
            else
                cudaMemcpyAsync(E->members[m].a.state, backup + off, (size_t)E->n_vars[m], cudaMemcpyDeviceToDevice,
                                E->stream);
            off += E->n_vars[m];
        }
        if (save) {
            cudaMemcpyAsync(ts.data(), E->d_ts, ts.size() * 4, cudaMemcpyDeviceToHost, E->stream);
            cudaMemcpyAsync(pos.data(), E->d_pos, pos.size() * 8, cudaMemcpyDeviceToHost, E->stream);
            cudaMemcpyAsync(&ls, E->d_ls, sizeof ls, cudaMemcpyDeviceToHost, E->stream);
            slots.clear();
            for (size_t l = 0; l < E->ladders.size(); ++l) {
                slots.emplace_back(E->ladders[l].size());
                cudaMemcpyAsync(slots.back().data(), E->ladder_dev[l].member_of_slot, slots.back().size() * 4,
                                cudaMemcpyDeviceToHost, E->stream);
            }
        } else {
            cudaMemcpyAsync(E->d_ts, ts.data(), ts.size() * 4, cudaMemcpyHostToDevice, E->stream);
            cudaMemcpyAsync(E->d_pos, pos.data(), pos.size() * 8, cudaMemcpyHostToDevice, E->stream);
            cudaMemcpyAsync(E->d_ls, &ls, sizeof ls, cudaMemcpyHostToDevice, E->stream);
            for (size_t l = 0; l < E->ladders.size(); ++l)
                cudaMemcpyAsync(E->ladder_dev[l].member_of_slot, slots[l].data(), slots[l].size() * 4,
                                cudaMemcpyHostToDevice, E->stream);
        }
        cudaStreamSynchronize(E->stream);
    };
    snapshot(true);
    const uint64_t done0 = E->sweeps_done;
    int best_r = E->ranks, best_c = E->ctas_per_sm;
    double best = 1e300;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);

    // 1. per member shape: the members of that shape alone at 1, 2, 4 and 8
    //    words per thread (one direct cooperative launch of trial_sweeps sweeps
    //    after a one-sweep warm-up, each from the snapshot); the fastest is kept
    std::map<ShapeKey, std::vector<size_t>> groups;
    for (size_t m = 0; m < E->members.size(); ++m)
        if (E->members[m].a.words || E->members[m].pk) groups[shape_key(E->descs[m])].push_back(m);
    for (auto &kv : groups) {
        const std::vector<size_t> &ids = kv.second;
        int best_w = E->members[ids[0]].wpt;
        double best_g = 1e300;
        for (int wpt : {1, 2, 4, 8}) {
            for (size_t m : ids) E->members[m].wpt = wpt;
            std::vector<WorkItem> items;
            append_items(E->members.data(), ids, 0, E->ranks, kItemsPerSm * E->ctx->sm_count, items);
            uint32_t g_total = 0;
            const std::vector<PackEntry> g_tab = pack_entries(E, ids, g_total);
            PackEntry *d_gtab = nullptr;
            WorkItem *d_items = nullptr;
            e = items_in_range(items.data(), items.size(), E->members.size()) ? cudaSuccess : cudaErrorInvalidValue;
            if (e == cudaSuccess && !g_tab.empty()) {
                e = cudaMalloc((void **)&d_gtab, g_tab.size() * sizeof(PackEntry));
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(d_gtab, g_tab.data(), g_tab.size() * sizeof(PackEntry), cudaMemcpyHostToDevice,
                                        E->stream);
            }
            if (e == cudaSuccess) e = cudaMalloc((void **)&d_items, items.size() * sizeof(WorkItem));
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(E->d_members, E->members.data(), E->members.size() * sizeof(EnsMember),
                                    cudaMemcpyHostToDevice, E->stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(d_items, items.data(), items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice,
                                    E->stream);
            float ms = 0;
            for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {  // warm-up, then timed
                snapshot(false);
                EnsArgs a = ens_args(E, rep == 0 ? 1 : (uint64_t)trial_sweeps);
                a.items = d_items;
                a.n_items = (int64_t)items.size();
                a.n_ladders = 0;
                a.pt_every = 0;
                cudaEventRecord(t0, E->stream);
                e = launch_ensemble(E, a, d_gtab, (int)g_tab.size(), g_total);
                cudaEventRecord(t1, E->stream);
                if (e == cudaSuccess) e = cudaEventSynchronize(t1);
                if (e == cudaSuccess) cudaEventElapsedTime(&ms, t0, t1);
            }
            if (d_items) cudaFree(d_items);
            if (d_gtab) cudaFree(d_gtab);
            if (e != cudaSuccess) break;
            if (ms < best_g) {
                best_g = ms;
                best_w = wpt;
            }
        }
        for (size_t m : ids) E->members[m].wpt = best_w;
        if (e != cudaSuccess) break;
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tuned[kv.first] = TuneEntry{best_w, best_g / trial_sweeps, (int)ids.size()};
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(E->d_members, E->members.data(), E->members.size() * sizeof(EnsMember),
                            cudaMemcpyHostToDevice, E->stream);
    if (e != cudaSuccess) {
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        snapshot(false);
        cudaFree(backup);
        return ens_fail(e, "tune");
    }

    // 2. the whole ensemble: ranks per thread of the generic body (none to choose
    //    when every member runs four sites at a time) and CTAs per SM
    std::vector<int> rs = E->words_only ? std::vector<int>{E->ranks} : std::vector<int>{2, 4, 8};
    for (int r : rs) {
        const int maxc = max_ctas_per_sm(r, E->words_only);
        std::vector<int> cs;
        for (int c : {1, 2, 4, maxc})
            if (c >= 1 && c <= maxc && std::find(cs.begin(), cs.end(), c) == cs.end()) cs.push_back(c);
        for (int c : cs) {
            if (plq_ensemble_set_config(E, r, c) != PLQ_OK) continue;
            snapshot(false);
            if (plq_ensemble_advance(E, 1) != PLQ_OK) continue;  // warm-up (and graph build)
            snapshot(false);
            if (plq_ensemble_advance(E, (uint64_t)trial_sweeps) != PLQ_OK) continue;  // capture
            snapshot(false);
            cudaEventRecord(t0, E->stream);
            if (plq_ensemble_advance(E, (uint64_t)trial_sweeps) != PLQ_OK) continue;
            cudaEventRecord(t1, E->stream);
            cudaEventSynchronize(t1);
            float ms = 0;
            cudaEventElapsedTime(&ms, t0, t1);
            if (ms < best) {
                best = ms;
                best_r = r;
                best_c = c;
            }
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    snapshot(false);
    cudaFree(backup);
    E->sweeps_done = done0;
    int rc = plq_ensemble_set_config(E, best_r, best_c);
    if (rc != PLQ_OK) return rc;
    if (ranks_out) *ranks_out = best_r;
    if (ctas_out) *ctas_out = best_c;
    if (ms_per_sweep_out) *ms_per_sweep_out = best / trial_sweeps;
    return ens_status(E);
}

extern "C" int plq_tempering_swap_phase(int32_t k_slots, int32_t *member_of_slot, double *beta_of_member,
                                        const int64_t *energy, const double *j_of_member, uint64_t ladder_seed,
                                        uint64_t attempt, int32_t *accepted_out) {
    if (k_slots < 0 || (k_slots > 0 && (!member_of_slot || !beta_of_member || !energy || !j_of_member)))
        return plq_fail(PLQ_EINVAL, "bad arguments");
    const uint32_t seed32 = plq_fold_seed(ladder_seed);
    int32_t accepted = 0;
    for (int32_t k = (int32_t)(attempt & 1u); k + 1 < k_slots; k += 2) {
        const int32_t m1 = member_of_slot[k], m2 = member_of_slot[k + 1];
        const double b1 = beta_of_member[m1], b2 = beta_of_member[m2];
        if (pt_accept(b1, b2, energy[m1], energy[m2], j_of_member[m1], j_of_member[m2], seed32, (uint32_t)k,
                      (uint32_t)attempt)) {
            beta_of_member[m1] = b2;
            beta_of_member[m2] = b1;
            member_of_slot[k] = m2;
            member_of_slot[k + 1] = m1;
            ++accepted;
        }
    }
    if (accepted_out) *accepted_out = accepted;
    return PLQ_OK;
}

extern "C" int plq_ensemble_member_config(plq_ensemble *E, int32_t m, int32_t *words_per_thread) {
    if (!E || !words_per_thread || m < 0 || m >= (int32_t)E->members.size())
        return plq_fail(PLQ_EINVAL, "bad arguments");
    *words_per_thread = E->members[m].a.words ? E->members[m].wpt : 0;
    return PLQ_OK;
}

extern "C" int plq_tune_entries(plq_tune_entry *out, int32_t capacity, int32_t *n_out) {
    if (!n_out || capacity < 0 || (capacity > 0 && !out)) return plq_fail(PLQ_EINVAL, "bad arguments");
    std::lock_guard<std::mutex> lock(g_tune_mu);
    int32_t n = 0;
    for (const auto &kv : g_tuned) {
        if (n < capacity) {
            plq_tune_entry &t = out[n];
            std::memset(&t, 0, sizeof t);
            t.model = kv.first.model;
            t.q = kv.first.q;
            t.d = kv.first.d;
            t.updater = kv.first.updater;
            t.rng = kv.first.rng;
            for (int i = 0; i < 4; ++i) t.shape[i] = kv.first.L[i];
            t.words_per_thread = kv.second.wpt;
            t.members = kv.second.members;
            t.ms_per_sweep = kv.second.ms_per_sweep;
        }
        ++n;
    }
    *n_out = n;
    return PLQ_OK;
}

extern "C" int plq_ensemble_sync(plq_ensemble *E) {
    if (!E) return plq_fail(PLQ_EINVAL, "NULL ensemble");
    return ens_status(E);
}

extern "C" int plq_ensemble_read(plq_ensemble *E, int32_t m, uint8_t *out) {
    if (!E || !out || m < 0 || m >= (int32_t)E->members.size()) return plq_fail(PLQ_EINVAL, "bad arguments");
    const EnsMember &mem = E->members[m];
    cudaError_t e = cudaSuccess;
    if (mem.link) {
        uint8_t *tmp = nullptr;
        e = cudaMalloc((void **)&tmp, (size_t)mem.n_vars);
        if (e == cudaSuccess) e = launch_planes_to_links(mem.a.state, tmp, mem.a.g.n_sites, mem.a.g.d, E->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(out, tmp, (size_t)mem.n_vars, cudaMemcpyDeviceToHost, E->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
        if (tmp) cudaFree(tmp);
    } else {
        e = cudaMemcpyAsync(out, mem.a.state, (size_t)mem.n_vars, cudaMemcpyDeviceToHost, E->stream);
    }
    if (e != cudaSuccess) return ens_fail(e, "member read");
    return ens_status(E);
}

extern "C" int plq_ensemble_primaries(plq_ensemble *E, int32_t m, int64_t *out, int32_t *n_out) {
    if (!E || !out || m < 0 || m >= (int32_t)E->members.size()) return plq_fail(PLQ_EINVAL, "bad arguments");
    const EnsMember &mem = E->members[m];
    long long *d = nullptr;
    int np = primaries_count(mem.a.model, mem.a.q);
    cudaError_t e = cudaMalloc((void **)&d, sizeof(long long) * (size_t)np);
    if (e == cudaSuccess) e = launch_primaries(mem.a.state, mem.a.g, mem.a.model, mem.a.q, d, E->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, sizeof(long long) * (size_t)np, cudaMemcpyDeviceToHost, E->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
    if (d) cudaFree(d);
    if (e != cudaSuccess) return ens_fail(e, "member primaries");
    if (n_out) *n_out = np;
    return ens_status(E);
}

extern "C" int plq_ensemble_primaries_all(plq_ensemble *E, int64_t *out, int32_t stride, int32_t *counts) {
    if (!E || !out || stride < 1) return plq_fail(PLQ_EINVAL, "bad arguments");
    const size_t n = E->members.size();
    cudaError_t e = plq_enter_device(E->ctx->device);
    if (e != cudaSuccess) return ens_fail(e, "cudaSetDevice");
    if (!E->d_prim_tasks) {
        // one buffer for all members, a task per member and its work items (built once)
        E->prims_offset.assign(n + 1, 0);
        for (size_t m = 0; m < n; ++m)
            E->prims_offset[m + 1] =
                E->prims_offset[m] + primaries_count(E->members[m].a.model, E->members[m].a.q);
        e = cudaMalloc((void **)&E->d_prims_all, sizeof(long long) * (size_t)E->prims_offset[n]);
        if (e != cudaSuccess) return ens_fail(e, "primaries buffer");
        E->allocs.push_back(E->d_prims_all);
        std::vector<PrimTask> tasks(n);
        std::vector<int32_t> it_task, it_chunk, itb_task, itb_chunk, pk_member, pk_chunk;
        for (size_t m = 0; m < n; ++m) {
            const EnsMember &mem = E->members[m];
            tasks[m] = PrimTask{mem.a.state, mem.a.g, mem.a.model, mem.a.q, E->d_prims_all + E->prims_offset[m]};
            for (int64_t c = 0; c * kPrimChunk < mem.a.g.n_sites; ++c) {
                it_task.push_back((int32_t)m);
                it_chunk.push_back((int32_t)c);
                if (!mem.pk) {
                    itb_task.push_back((int32_t)m);
                    itb_chunk.push_back((int32_t)c);
                }
            }
            if (mem.pk)
                for (int64_t c = 0; c * kEnsThreads < (int64_t)row_count(mem.a.g); ++c) {
                    pk_member.push_back((int32_t)m);
                    pk_chunk.push_back((int32_t)c);
                }
        }
        e = dev_upload(E, it_task.data(), it_task.size(), &E->d_prim_task);
        if (e == cudaSuccess) e = dev_upload(E, it_chunk.data(), it_chunk.size(), &E->d_prim_chunk);
        if (e == cudaSuccess) e = dev_upload(E, itb_task.data(), itb_task.size(), &E->d_prim_task_bytes);
        if (e == cudaSuccess) e = dev_upload(E, itb_chunk.data(), itb_chunk.size(), &E->d_prim_chunk_bytes);
        if (e == cudaSuccess) e = dev_upload(E, pk_member.data(), pk_member.size(), &E->d_pk_prim_member);
        if (e == cudaSuccess) e = dev_upload(E, pk_chunk.data(), pk_chunk.size(), &E->d_pk_prim_chunk);
        if (e == cudaSuccess) e = dev_upload(E, E->prims_offset.data(), E->prims_offset.size(), &E->d_prims_offset);
        if (e == cudaSuccess) e = dev_upload(E, tasks.data(), tasks.size(), &E->d_prim_tasks);
        if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
        if (e != cudaSuccess) {
            E->d_prim_tasks = nullptr;
            return ens_fail(e, "primaries tasks");
        }
        E->n_prim_items = (int64_t)it_task.size();
        E->n_prim_items_bytes = (int64_t)itb_task.size();
        E->n_pk_prim_items = (int64_t)pk_member.size();
    }
    for (size_t m = 0; m < n; ++m) {
        const int64_t np = E->prims_offset[m + 1] - E->prims_offset[m];
        if (np > stride) return plq_fail(PLQ_EINVAL, "stride is below a member's primaries count");
    }
    std::vector<long long> host((size_t)E->prims_offset[n]);
    e = cudaMemsetAsync(E->d_prims_all, 0, sizeof(long long) * host.size(), E->stream);
    if (E->pk_current && E->n_pk_prim_items) {
        // packed members from their rows, the rest from their bytes
        if (e == cudaSuccess && E->n_prim_items_bytes) {
            e = launch_primaries_multi(E->d_prim_tasks, E->d_prim_task_bytes, E->d_prim_chunk_bytes,
                                       E->n_prim_items_bytes, E->ctx->sm_count, E->stream);
            E->launches++;
        }
        if (e == cudaSuccess) {
            const unsigned blocks = (unsigned)std::min<int64_t>(E->n_pk_prim_items, (int64_t)E->ctx->sm_count * 8);
            packed_primaries_kernel<<<blocks, kEnsThreads, 0, E->stream>>>(
                E->d_members, E->d_pk_prim_member, E->d_pk_prim_chunk, E->n_pk_prim_items, E->d_prims_all,
                E->d_prims_offset);
            e = cudaGetLastError();
            E->launches++;
        }
    } else {
        if (e == cudaSuccess)
            e = launch_primaries_multi(E->d_prim_tasks, E->d_prim_task, E->d_prim_chunk, E->n_prim_items,
                                       E->ctx->sm_count, E->stream);
        E->launches++;
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(host.data(), E->d_prims_all, sizeof(long long) * host.size(), cudaMemcpyDeviceToHost,
                            E->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
    if (e != cudaSuccess) return ens_fail(e, "primaries of every member");
    for (size_t m = 0; m < n; ++m) {
        const int64_t np = E->prims_offset[m + 1] - E->prims_offset[m];
        for (int64_t i = 0; i < np; ++i) out[(int64_t)m * stride + i] = host[(size_t)(E->prims_offset[m] + i)];
        if (counts) counts[m] = (int32_t)np;
    }
    return ens_status(E);
}

extern "C" int plq_ensemble_betas(plq_ensemble *E, double *beta_of_member) {
    if (!E || !beta_of_member) return plq_fail(PLQ_EINVAL, "bad arguments");
    std::vector<int32_t> ts(E->members.size());
    cudaError_t e = cudaMemcpyAsync(ts.data(), E->d_ts, ts.size() * 4, cudaMemcpyDeviceToHost, E->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
    if (e != cudaSuccess) return ens_fail(e, "betas read");
    for (size_t m = 0; m < ts.size(); ++m) beta_of_member[m] = E->tsets[ts[m]].beta;
    return PLQ_OK;
}

extern "C" int64_t plq_ensemble_n_vars(plq_ensemble *E) {
    int64_t t = 0;
    if (E)
        for (auto v : E->n_vars) t += v;
    return t;
}
extern "C" void *plq_ensemble_cuda_stream(plq_ensemble *E) { return E ? (void *)E->stream : nullptr; }
extern "C" uint64_t plq_ensemble_launches(plq_ensemble *E) { return E ? E->launches : 0; }

extern "C" void plq_ensemble_destroy(plq_ensemble *E) {
    if (!E) return;
    if (E->ctx) plq_enter_device(E->ctx->device);
    if (E->stream) cudaStreamSynchronize(E->stream);
    drop_graph(E);
    for (void *p : E->allocs) cudaFree(p);
    if (E->stream) cudaStreamDestroy(E->stream);
    delete E;
}

// ====================================================================
// Serving: continuous batching of simulation jobs.
//
// A worker thread owns the device.  Each tick it (1) admits queued jobs,
// first-fit, while their device footprint fits the memory budget and a slot
// is free -- a job's lattice, tables and jump table are allocated once and
// stay resident until it finishes; (2) launches the persistent ensemble
// kernel over every active job for a quantum of sweeps sized so a tick takes
// about `tick_ms`; (3) retires finished jobs: final primaries (and, if asked,
// the configuration) are read back and their memory freed.  Jobs that arrive
// while others run join at the next tick; their sweeps share launches with
// whatever else is active.  Each job keeps its own keyed sweep counter and
// stream position, so its result is the same alone or in any mix.
// ====================================================================

struct ServerJob {
    int64_t id = 0;
    plq_chain_desc desc;
    std::vector<uint8_t> start;
    bool has_start = false;
    uint64_t sweeps = 0, done = 0;
    bool want_states = false;
    int state = PLQ_JOB_QUEUED;
    int error = PLQ_OK;
    std::string message;
    double t_submit = 0, t_admit = 0, t_finish = 0;
    uint64_t footprint = 0;
    // device state while active
    EnsMember mem;
    TableSet ts;
    std::vector<void *> allocs;
    unsigned long long pos = 0, msweep = 0;
    // results
    std::vector<uint8_t> final_states;
    std::vector<int64_t> primaries;
};

struct plq_server {
    plq_ctx ctx_copy;        // the context's record, copied at creation (outlives the caller's)
    plq_ctx *ctx = nullptr;  // = &ctx_copy
    uint64_t budget = 0, used = 0;
    int max_slots = 0;
    double tick_ms = 10.0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread worker;
    bool stop = false;
    int64_t next_id = 1;
    std::deque<ServerJob *> queue;
    std::vector<ServerJob *> active;
    std::map<int64_t, ServerJob *> jobs;
    // statistics
    std::vector<double> latencies_ms;
    double updates = 0, busy_s = 0;
    uint64_t ticks = 0, launches = 0;
    double last_ms_per_sweep = 1.0;
    int device_error = PLQ_OK;
    std::string device_message;
};

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Device bytes a job holds while active.
uint64_t job_footprint(const plq_chain_desc &d) {
    int64_t n = 1;
    for (int i = 0; i < d.d; ++i) n *= d.shape[i];
    int64_t n_vars = d.model == PLQ_GAUGE ? n * d.d : n;
    ModelParams p;
    std::memset(&p, 0, sizeof p);
    p.model = d.model;
    p.q = d.model == PLQ_POTTS ? d.q : 2;
    p.d = d.d;
    int64_t keys = d.updater == PLQ_METROPOLIS && p.q > 2 ? potts_metro_key_count(p) : env_key_count(p);
    uint64_t table = (uint64_t)keys * (uint64_t)std::max(1, p.q - 1) * 8ull;
    uint64_t jump = d.rng == PLQ_RNG_STREAM ? 65536ull : 0ull;
    return (uint64_t)n_vars + table + jump + 4096ull;
}

void job_release(ServerJob *j) {
    for (void *p : j->allocs) cudaFree(p);
    j->allocs.clear();
}

// Allocate and upload a job's resident state (worker thread, device current).
int job_admit(ServerJob *j, cudaStream_t stream) {
    const plq_chain_desc &d = j->desc;
    EnsMember &mem = j->mem;
    std::memset(&mem, 0, sizeof mem);
    LocalArgs &a = mem.a;
    const int q = d.model == PLQ_POTTS ? d.q : 2;
    a.g.d = d.d;
    int64_t ns = 1;
    for (int i = 0; i < kMaxD; ++i) {
        a.g.L[i] = i < d.d ? (int32_t)d.shape[i] : 1;
        a.g.stride[i] = ns;
        if (i < d.d) ns *= d.shape[i];
    }
    a.g.n_sites = ns;
    geom_init(a.g, d.d, d.shape);
    mem.link = d.model == PLQ_GAUGE;
    mem.passes = mem.link ? 2 * d.d : 2;
    mem.n_vars = mem.link ? ns * d.d : ns;
    mem.j = d.j;
    mem.ladder = -1;
    a.q = q;
    a.kernel = d.updater;
    a.model = d.model;
    int32_t w = 1;
    for (int s = 1; s < q; ++s) {
        a.pw[s] = w;
        w *= 2 * d.d + 1;
    }
    a.seed32 = plq_fold_seed(d.seed);
    a.words = !(d.flags & PLQ_FLAG_GENERIC_PASS) &&
              words_eligible(d.model, q, d.d, a.g.L, d.updater, d.rng) ? 1 : 0;
    mem.wpt = tuned_wpt(d);
    cudaError_t e = cudaSuccess;
    auto alloc = [&](void **p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes);
        if (e == cudaSuccess) j->allocs.push_back(*p);
    };
    uint8_t *st = nullptr;
    alloc((void **)&st, (size_t)mem.n_vars);
    a.state = st;
    if (e == cudaSuccess) {
        if (j->has_start) {
            if (mem.link) {
                uint8_t *tmp = nullptr;
                e = cudaMalloc((void **)&tmp, (size_t)mem.n_vars);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(tmp, j->start.data(), (size_t)mem.n_vars, cudaMemcpyHostToDevice, stream);
                if (e == cudaSuccess) e = launch_links_to_planes(tmp, st, ns, d.d, stream);
                if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
                if (tmp) cudaFree(tmp);
            } else {
                e = cudaMemcpyAsync(st, j->start.data(), (size_t)mem.n_vars, cudaMemcpyHostToDevice, stream);
            }
        } else {
            e = cudaMemsetAsync(st, 0, (size_t)mem.n_vars, stream);
        }
    }
    if (e == cudaSuccess && d.rng == PLQ_RNG_STREAM) {
        uint64_t slo, shi, ilo, ihi;
        pcg_seed_from_u64(d.seed, slo, shi, ilo, ihi);
        std::vector<AffineHost> tab;
        build_jump_table(ilo, ihi, tab);
        a.inc = u128{ilo, ihi};
        u128 s0 = jump(reinterpret_cast<const Affine *>(tab.data()), u128{slo, shi}, d.stream_offset);
        a.base = pcg_step(s0, a.inc);
        void *dj = nullptr;
        alloc(&dj, tab.size() * sizeof(AffineHost));
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(dj, tab.data(), tab.size() * sizeof(AffineHost), cudaMemcpyHostToDevice, stream);
        a.jump = reinterpret_cast<const Affine *>(dj);
    }
    if (e != cudaSuccess) {
        job_release(j);
        return plq_fail(e == cudaErrorMemoryAllocation ? PLQ_ENOMEM : PLQ_ECUDA, cudaGetErrorString(e));
    }
    ModelParams p;
    std::memset(&p, 0, sizeof p);
    p.model = d.model;
    p.q = q;
    p.d = d.d;
    p.beta = d.beta;
    p.j = d.j;
    p.h = d.h;
    for (int k = 0; k < PLQ_MAX_Q; ++k) p.offsets[k] = d.offsets[k];
    Tables t;
    std::string err;
    if (!build_tables(p, d.updater, d.rng, t, err)) {
        job_release(j);
        return plq_fail(PLQ_EUNSUPPORTED, err);
    }
    std::memset(&j->ts, 0, sizeof j->ts);
    j->ts.beta = d.beta;
    auto up = [&](const void *host, size_t bytes) -> void * {
        if (!bytes || e != cudaSuccess) return nullptr;
        void *p2 = nullptr;
        alloc(&p2, bytes);
        if (e == cudaSuccess) e = cudaMemcpyAsync(p2, host, bytes, cudaMemcpyHostToDevice, stream);
        return p2;
    };
    j->ts.hb53 = (const uint64_t *)up(t.hb53.data(), t.hb53.size() * 8);
    j->ts.hb24 = (const uint32_t *)up(t.hb24.data(), t.hb24.size() * 4);
    j->ts.metro53 = (const uint64_t *)up(t.metro53.data(), t.metro53.size() * 8);
    j->ts.metro24 = (const uint32_t *)up(t.metro24.data(), t.metro24.size() * 4);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        job_release(j);
        return plq_fail(e == cudaErrorMemoryAllocation ? PLQ_ENOMEM : PLQ_ECUDA, cudaGetErrorString(e));
    }
    return PLQ_OK;
}

// Device buffers of one tick's launch; grown, never shrunk.
struct TickBuffers {
    EnsMember *members = nullptr;
    TableSet *tsets = nullptr;
    int32_t *ts = nullptr;
    unsigned long long *pos = nullptr, *msweep = nullptr, *done = nullptr;
    WorkItem *items = nullptr;
    LaunchState *ls = nullptr;
    Control *ctrl = nullptr;
    size_t cap_members = 0, cap_items = 0;
    void release() {
        void *ps[] = {members, tsets, ts, pos, msweep, done, items, ls, ctrl};
        for (void *p : ps)
            if (p) cudaFree(p);
        *this = TickBuffers();
    }
};

int run_tick(plq_server *S, TickBuffers &B, cudaStream_t stream, uint64_t sweeps) {
    const size_t n = S->active.size();
    // members that run four sites at a time first: they go to the words-only kernel
    // (few registers, several CTAs per SM), the rest to a second launch of the full kernel
    std::vector<size_t> order;
    for (size_t m = 0; m < n; ++m)
        if (S->active[m]->mem.a.words) order.push_back(m);
    const size_t nw = order.size();
    for (size_t m = 0; m < n; ++m)
        if (!S->active[m]->mem.a.words) order.push_back(m);
    std::vector<EnsMember> mems(n);
    std::vector<TableSet> tss(n);
    std::vector<int32_t> ts(n);
    std::vector<unsigned long long> pos(n), msw(n);
    for (size_t k = 0; k < n; ++k) {
        const ServerJob *j = S->active[order[k]];
        mems[k] = j->mem;
        tss[k] = j->ts;
        ts[k] = (int32_t)k;
        pos[k] = j->pos;
        msw[k] = j->msweep;
    }
    // ranks per thread: 4 for the words-only kernel; 2 for the full kernel, whose generic
    // body needs the registers (2 CTAs per SM instead of 1)
    const int ranks_w = 4, ranks_g = 2;
    std::vector<WorkItem> items;
    std::vector<size_t> ids_w, ids_g;
    for (size_t k = 0; k < n; ++k) (k < nw ? ids_w : ids_g).push_back(k);
    const int64_t min_items = kItemsPerSm * S->ctx->sm_count;
    if (nw) append_items(mems.data(), ids_w, 0, ranks_w, min_items, items);
    const size_t n_w_items = items.size();  // the second group's items follow the first's
    if (n > nw) append_items(mems.data(), ids_g, nw, ranks_g, min_items, items);
    if (!items_in_range(items.data(), n_w_items, nw) ||
        !items_in_range(items.data() + n_w_items, items.size() - n_w_items, n - nw))
        return plq_fail(PLQ_EINVAL, "serving work items name a member out of range");
    cudaError_t e = cudaSuccess;
    if (!B.ls) {
        e = cudaMalloc((void **)&B.ls, sizeof(LaunchState));
        if (e == cudaSuccess) e = cudaMalloc((void **)&B.ctrl, sizeof(Control));
        if (e == cudaSuccess) e = cudaMemsetAsync(B.ls, 0, sizeof(LaunchState), stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(B.ctrl, 0, sizeof(Control), stream);
    }
    if (e == cudaSuccess && B.cap_members < n) {
        cudaFree(B.members);
        cudaFree(B.tsets);
        cudaFree(B.ts);
        cudaFree(B.pos);
        cudaFree(B.msweep);
        cudaFree(B.done);
        size_t c = std::max<size_t>(n, 2 * B.cap_members);
        e = cudaMalloc((void **)&B.members, c * sizeof(EnsMember));
        if (e == cudaSuccess) e = cudaMalloc((void **)&B.tsets, c * sizeof(TableSet));
        if (e == cudaSuccess) e = cudaMalloc((void **)&B.ts, c * sizeof(int32_t));
        if (e == cudaSuccess) e = cudaMalloc((void **)&B.pos, c * sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMalloc((void **)&B.msweep, c * sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMalloc((void **)&B.done, c * sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMemsetAsync(B.done, 0, c * sizeof(unsigned long long), stream);
        B.cap_members = c;
    }
    if (e == cudaSuccess && B.cap_items < items.size() + 1) {
        cudaFree(B.items);
        B.items = nullptr;
        size_t c = std::max<size_t>(items.size() + 1, 2 * B.cap_items);
        e = cudaMalloc((void **)&B.items, c * sizeof(WorkItem));
        B.cap_items = c;
    }
    if (e != cudaSuccess) return plq_fail(PLQ_ENOMEM, std::string("tick buffers: ") + cudaGetErrorString(e));
    cudaMemcpyAsync(B.members, mems.data(), n * sizeof(EnsMember), cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(B.tsets, tss.data(), n * sizeof(TableSet), cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(B.ts, ts.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(B.pos, pos.data(), n * sizeof(unsigned long long), cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(B.msweep, msw.data(), n * sizeof(unsigned long long), cudaMemcpyHostToDevice, stream);
    if (!items.empty())
        cudaMemcpyAsync(B.items, items.data(), items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice, stream);
    // one cooperative launch per member group, each over its own part of the item list
    // (member indices relative to the group's first member)
    auto launch = [&](size_t lo, size_t hi, size_t item_lo, size_t item_hi, bool words_only,
                      int ranks) -> cudaError_t {
        if (hi == lo || item_hi == item_lo) return cudaSuccess;
        EnsArgs a;
        std::memset(&a, 0, sizeof a);
        a.members = B.members + lo;
        a.n_members = (int)(hi - lo);
        a.tsets = B.tsets;
        a.ts_of_member = B.ts + lo;
        a.pos = B.pos + lo;
        a.msweep = B.msweep + lo;
        a.done = B.done + lo;
        a.items = B.items + item_lo;
        a.n_items = (int64_t)(item_hi - item_lo);
        a.ls = B.ls;
        a.ctrl = B.ctrl;
        a.sweeps = sweeps;
        a.ranks = ranks;
        void *params[] = {&a};
        const int ctas = std::max(1, std::min(4, max_ctas_per_sm(ranks, words_only)));
        dim3 grid((unsigned)(S->ctx->sm_count * ctas));
        S->launches++;
        return cudaLaunchCooperativeKernel(kernel_ptr(ranks, words_only), grid, dim3(kEnsThreads), params, 0, stream);
    };
    e = launch(0, nw, 0, n_w_items, true, ranks_w);
    if (e == cudaSuccess) e = launch(nw, n, n_w_items, items.size(), false, ranks_g);
    unsigned int status = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&status, &B.ctrl->status, sizeof status, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return plq_fail(PLQ_ECUDA, std::string("serving launch: ") + cudaGetErrorString(e));
    if (status) return plq_fail(PLQ_EDEVICE, "serving kernel status word " + std::to_string(status));
    for (size_t m = 0; m < n; ++m) {
        ServerJob *j = S->active[m];
        j->done += sweeps;
        j->msweep += sweeps;
        if (j->mem.a.jump) j->pos += sweeps * (unsigned long long)j->mem.n_vars;
    }
    return PLQ_OK;
}

void retire(plq_server *S, ServerJob *j, cudaStream_t stream) {
    const EnsMember &mem = j->mem;
    int np = primaries_count(mem.a.model, mem.a.q);
    std::vector<long long> prim((size_t)np, 0);
    long long *d = nullptr;
    cudaError_t e = cudaMalloc((void **)&d, sizeof(long long) * (size_t)np);
    if (e == cudaSuccess) e = launch_primaries(mem.a.state, mem.a.g, mem.a.model, mem.a.q, d, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(prim.data(), d, sizeof(long long) * (size_t)np, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && j->want_states) {
        j->final_states.resize((size_t)mem.n_vars);
        if (mem.link) {
            uint8_t *tmp = nullptr;
            e = cudaMalloc((void **)&tmp, (size_t)mem.n_vars);
            if (e == cudaSuccess) e = launch_planes_to_links(mem.a.state, tmp, mem.a.g.n_sites, mem.a.g.d, stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(j->final_states.data(), tmp, (size_t)mem.n_vars, cudaMemcpyDeviceToHost, stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
            if (tmp) cudaFree(tmp);
        } else {
            e = cudaMemcpyAsync(j->final_states.data(), mem.a.state, (size_t)mem.n_vars, cudaMemcpyDeviceToHost,
                                stream);
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (d) cudaFree(d);
    job_release(j);
    std::lock_guard<std::mutex> lock(S->mu);
    S->used -= j->footprint;
    j->t_finish = now_s();
    if (e != cudaSuccess) {
        j->state = PLQ_JOB_FAILED;
        j->error = PLQ_ECUDA;
        j->message = cudaGetErrorString(e);
    } else {
        j->primaries.assign(prim.begin(), prim.end());
        j->state = PLQ_JOB_DONE;
        S->latencies_ms.push_back((j->t_finish - j->t_submit) * 1e3);
    }
}

void worker_loop(plq_server *S) {
    plq_enter_device(S->ctx->device);
    cudaStream_t stream = nullptr;
    cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    TickBuffers B;
    for (;;) {
        // 1. admit (first fit by footprint and slots)
        std::vector<ServerJob *> admit;
        {
            std::unique_lock<std::mutex> lock(S->mu);
            S->cv_work.wait(lock, [&] { return S->stop || !S->queue.empty() || !S->active.empty(); });
            if (S->stop) break;
            for (auto it = S->queue.begin(); it != S->queue.end();) {
                ServerJob *j = *it;
                if ((int)(S->active.size() + admit.size()) >= S->max_slots) break;
                if (S->used + j->footprint <= S->budget) {
                    S->used += j->footprint;
                    admit.push_back(j);
                    it = S->queue.erase(it);
                } else {
                    ++it;
                }
            }
        }
        for (ServerJob *j : admit) {
            int rc = job_admit(j, stream);
            std::lock_guard<std::mutex> lock(S->mu);
            if (rc != PLQ_OK) {
                S->used -= j->footprint;
                j->state = PLQ_JOB_FAILED;
                j->error = rc;
                j->message = plq_last_error();
                j->t_finish = now_s();
                S->cv_done.notify_all();
            } else {
                j->state = PLQ_JOB_ACTIVE;
                j->t_admit = now_s();
                S->active.push_back(j);
            }
        }
        // jobs with nothing left to run (zero sweeps) retire before the tick
        {
            std::vector<ServerJob *> still;
            for (ServerJob *j : S->active) {
                if (j->done >= j->sweeps)
                    retire(S, j, stream);
                else
                    still.push_back(j);
            }
            S->active.swap(still);
            S->cv_done.notify_all();
        }
        if (S->active.empty()) continue;
        // 2. one tick: a quantum of sweeps for every active job
        uint64_t remaining = ~0ull;
        for (ServerJob *j : S->active) remaining = std::min(remaining, j->sweeps - j->done);
        uint64_t quantum = (uint64_t)std::max(1.0, S->tick_ms / std::max(1e-3, S->last_ms_per_sweep));
        quantum = std::max<uint64_t>(1, std::min(quantum, remaining));
        double t0 = now_s();
        int rc = remaining ? run_tick(S, B, stream, quantum) : PLQ_OK;
        double dt = now_s() - t0;
        if (remaining) S->last_ms_per_sweep = std::max(1e-3, dt * 1e3 / (double)quantum);
        {
            std::lock_guard<std::mutex> lock(S->mu);
            S->ticks++;
            S->busy_s += dt;
            if (rc != PLQ_OK) {
                S->device_error = rc;
                S->device_message = plq_last_error();
                for (ServerJob *j : S->active) {
                    j->state = PLQ_JOB_FAILED;
                    j->error = rc;
                    j->message = S->device_message;
                    S->used -= j->footprint;
                }
            } else if (remaining) {
                for (ServerJob *j : S->active) {
                    int64_t nv = j->mem.n_vars;
                    S->updates += (double)nv * (double)quantum;
                }
            }
        }
        if (rc != PLQ_OK) {
            for (ServerJob *j : S->active) job_release(j);
            S->active.clear();
            S->cv_done.notify_all();
            continue;
        }
        // 3. retire finished jobs
        std::vector<ServerJob *> still;
        for (ServerJob *j : S->active) {
            if (j->done >= j->sweeps)
                retire(S, j, stream);
            else
                still.push_back(j);
        }
        S->active.swap(still);
        S->cv_done.notify_all();
    }
    for (ServerJob *j : S->active) job_release(j);
    S->active.clear();
    B.release();
    cudaStreamDestroy(stream);
}

}  // namespace

extern "C" int plq_server_create(plq_ctx *ctx, uint64_t budget_bytes, int32_t max_slots, double tick_ms,
                                 plq_server **out) {
    if (!ctx || !out || max_slots <= 0) return plq_fail(PLQ_EINVAL, "bad server arguments");
    *out = nullptr;
    plq_server *S = new plq_server();
    S->ctx_copy = *ctx;
    S->ctx = &S->ctx_copy;
    S->max_slots = max_slots;
    S->tick_ms = tick_ms > 0 ? tick_ms : 10.0;
    if (budget_bytes == 0) {
        size_t free_b = 0, total_b = 0;
        plq_enter_device(ctx->device);
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
            delete S;
            return plq_fail(PLQ_ECUDA, "cudaMemGetInfo failed");
        }
        budget_bytes = (uint64_t)(0.8 * (double)free_b);
    }
    S->budget = budget_bytes;
    S->worker = std::thread(worker_loop, S);
    *out = S;
    return PLQ_OK;
}

extern "C" int plq_server_submit(plq_server *S, const plq_chain_desc *desc, const uint8_t *start, uint64_t sweeps,
                                 int32_t want_states, int64_t *job_id) {
    if (!S || !desc || !job_id) return plq_fail(PLQ_EINVAL, "bad arguments");
    int rc = plq_chain_validate(desc);
    if (rc != PLQ_OK) return rc;
    if (desc->updater == PLQ_CLUSTER || desc->d > 4 ||
        (desc->rng == PLQ_RNG_STREAM && desc->updater == PLQ_METROPOLIS))
        return plq_fail(PLQ_EUNSUPPORTED,
                        "served jobs are local updaters in at most 4 dimensions (keyed, or heat bath on the PCG "
                        "stream)");
    ServerJob *j = new ServerJob();
    j->desc = *desc;
    j->msweep = desc->sweep_offset;  // the job's keyed sweep key resumes here
    j->sweeps = sweeps;
    j->want_states = want_states != 0;
    j->footprint = job_footprint(*desc);
    int64_t n = 1;
    for (int i = 0; i < desc->d; ++i) n *= desc->shape[i];
    int64_t n_vars = desc->model == PLQ_GAUGE ? n * desc->d : n;
    const int q = desc->model == PLQ_POTTS ? desc->q : 2;
    if (start) {
        if (first_state_at_least(start, n_vars, q) >= 0) {
            delete j;
            return plq_fail(PLQ_EINVAL, "start state out of range");
        }
        j->start.assign(start, start + n_vars);
        j->has_start = true;
    }
    std::lock_guard<std::mutex> lock(S->mu);
    if (j->footprint > S->budget) {
        delete j;
        return plq_fail(PLQ_ENOMEM, "the job's device footprint exceeds the server's memory budget");
    }
    j->id = S->next_id++;
    j->t_submit = now_s();
    S->jobs[j->id] = j;
    if (sweeps == 0) {
        // nothing to run: still a job, resolved at the next tick with its start state
        j->sweeps = 0;
    }
    S->queue.push_back(j);
    *job_id = j->id;
    S->cv_work.notify_one();
    return PLQ_OK;
}

extern "C" int plq_server_wait(plq_server *S, int64_t job_id, double timeout_s, int32_t *state_out) {
    if (!S) return plq_fail(PLQ_EINVAL, "NULL server");
    std::unique_lock<std::mutex> lock(S->mu);
    auto it = S->jobs.find(job_id);
    if (it == S->jobs.end()) return plq_fail(PLQ_EINVAL, "unknown job");
    ServerJob *j = it->second;
    auto finished = [&] { return j->state == PLQ_JOB_DONE || j->state == PLQ_JOB_FAILED || j->state == PLQ_JOB_CANCELLED; };
    if (timeout_s < 0)
        S->cv_done.wait(lock, finished);
    else
        S->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), finished);
    if (state_out) *state_out = j->state;
    return PLQ_OK;
}

extern "C" int plq_server_cancel(plq_server *S, int64_t job_id) {
    if (!S) return plq_fail(PLQ_EINVAL, "NULL server");
    std::lock_guard<std::mutex> lock(S->mu);
    auto it = S->jobs.find(job_id);
    if (it == S->jobs.end()) return plq_fail(PLQ_EINVAL, "unknown job");
    ServerJob *j = it->second;
    if (j->state != PLQ_JOB_QUEUED) return plq_fail(PLQ_EBUSY, "only a queued job can be cancelled");
    S->queue.erase(std::remove(S->queue.begin(), S->queue.end(), j), S->queue.end());
    j->state = PLQ_JOB_CANCELLED;
    j->t_finish = now_s();
    S->cv_done.notify_all();
    return PLQ_OK;
}

extern "C" int plq_server_result(plq_server *S, int64_t job_id, uint8_t *out_states, int64_t *out_primaries,
                                 double *timing_out) {
    if (!S) return plq_fail(PLQ_EINVAL, "NULL server");
    std::lock_guard<std::mutex> lock(S->mu);
    auto it = S->jobs.find(job_id);
    if (it == S->jobs.end()) return plq_fail(PLQ_EINVAL, "unknown job");
    ServerJob *j = it->second;
    if (j->state == PLQ_JOB_FAILED) return plq_fail(j->error, j->message);
    if (j->state != PLQ_JOB_DONE) return plq_fail(PLQ_EBUSY, "job not finished");
    if (out_states) {
        if (!j->want_states) return plq_fail(PLQ_EINVAL, "the job was submitted without want_states");
        std::memcpy(out_states, j->final_states.data(), j->final_states.size());
    }
    if (out_primaries) std::copy(j->primaries.begin(), j->primaries.end(), out_primaries);
    if (timing_out) {
        timing_out[0] = (j->t_admit - j->t_submit) * 1e3;
        timing_out[1] = (j->t_finish - j->t_submit) * 1e3;
    }
    return PLQ_OK;
}

extern "C" int plq_server_release(plq_server *S, int64_t job_id) {
    if (!S) return plq_fail(PLQ_EINVAL, "NULL server");
    std::lock_guard<std::mutex> lock(S->mu);
    auto it = S->jobs.find(job_id);
    if (it == S->jobs.end()) return plq_fail(PLQ_EINVAL, "unknown job");
    ServerJob *j = it->second;
    if (j->state == PLQ_JOB_QUEUED || j->state == PLQ_JOB_ACTIVE) return plq_fail(PLQ_EBUSY, "job still running");
    S->jobs.erase(it);
    delete j;
    return PLQ_OK;
}

extern "C" int plq_server_stats(plq_server *S, double *out) {
    if (!S || !out) return plq_fail(PLQ_EINVAL, "bad arguments");
    std::lock_guard<std::mutex> lock(S->mu);
    std::vector<double> lat = S->latencies_ms;
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double p) {
        if (lat.empty()) return 0.0;
        size_t k = (size_t)std::min<double>((double)lat.size() - 1, std::ceil(p * (double)lat.size()) - 1);
        return lat[k];
    };
    out[0] = (double)lat.size();
    out[1] = pct(0.50);
    out[2] = pct(0.99);
    out[3] = S->busy_s > 0 ? S->updates / S->busy_s / 1e9 : 0.0;
    out[4] = (double)S->ticks;
    out[5] = (double)S->queue.size();
    out[6] = (double)S->active.size();
    out[7] = (double)S->used;
    return S->device_error;
}

extern "C" void plq_server_destroy(plq_server *S) {
    if (!S) return;
    {
        std::lock_guard<std::mutex> lock(S->mu);
        S->stop = true;
        S->cv_work.notify_all();
    }
    if (S->worker.joinable()) S->worker.join();
    for (auto &kv : S->jobs) delete kv.second;
    delete S;
}
