"""Batched ensembles: many chains advanced by one persistent launch.

``Ensemble`` wraps the ``plq_ensemble_*`` entry points of include/plaquette.h:
members are chain descriptors (any mix of models, shapes, betas, seeds),
optionally grouped into parallel-tempering ladders; ``advance`` runs every
member in one cooperative, graph-captured launch and ``advance_unbatched``
runs the same sweeps one launch per member per colour pass (the per-lattice
baseline, identical results).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import ChainDesc, check, extra_signatures, lib

_P = C.POINTER
extra_signatures({
    "plq_ensemble_create": ([C.c_void_p, C.c_int32, _P(ChainDesc), _P(C.c_void_p), _P(C.c_void_p)], C.c_int),
    "plq_ensemble_add_ladder": ([C.c_void_p, C.c_int32, _P(C.c_int32), _P(C.c_double), C.c_int32, C.c_uint64],
                                C.c_int),
    "plq_ensemble_advance": ([C.c_void_p, C.c_uint64], C.c_int),
    "plq_ensemble_advance_unbatched": ([C.c_void_p, C.c_uint64], C.c_int),
    "plq_ensemble_set_config": ([C.c_void_p, C.c_int32, C.c_int32], C.c_int),
    "plq_ensemble_tune": ([C.c_void_p, C.c_int32, _P(C.c_int32), _P(C.c_int32), _P(C.c_double)], C.c_int),
    "plq_ensemble_sync": ([C.c_void_p], C.c_int),
    "plq_ensemble_read": ([C.c_void_p, C.c_int32, C.c_void_p], C.c_int),
    "plq_ensemble_primaries": ([C.c_void_p, C.c_int32, C.c_void_p, _P(C.c_int32)], C.c_int),
    "plq_ensemble_primaries_all": ([C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p], C.c_int),
    "plq_ensemble_member_config": ([C.c_void_p, C.c_int32, _P(C.c_int32)], C.c_int),
    "plq_ensemble_set_beta": ([C.c_void_p, C.c_int32, C.c_double], C.c_int),
    "plq_tempering_swap_phase": ([C.c_int32, _P(C.c_int32), _P(C.c_double), _P(C.c_int64), _P(C.c_double),
                                  C.c_uint64, C.c_uint64, _P(C.c_int32)], C.c_int),
    "plq_tune_entries": ([C.c_void_p, C.c_int32, _P(C.c_int32)], C.c_int),
    "plq_ensemble_betas": ([C.c_void_p, C.c_void_p], C.c_int),
    "plq_ensemble_n_vars": ([C.c_void_p], C.c_int64),
    "plq_ensemble_cuda_stream": ([C.c_void_p], C.c_void_p),
    "plq_ensemble_launches": ([C.c_void_p], C.c_uint64),
    "plq_ensemble_destroy": ([C.c_void_p], None),
})


class Ensemble:
    def __init__(self, gpu, descs: list[ChainDesc], starts: list[np.ndarray | None] | None = None):
        self.gpu = gpu
        self.descs = list(descs)
        n = len(self.descs)
        arr = (ChainDesc * n)(*self.descs)
        self._keep = []
        ptrs = (C.c_void_p * n)()
        if starts is not None:
            for i, s in enumerate(starts):
                if s is not None:
                    s = np.ascontiguousarray(s, dtype=np.uint8)
                    self._keep.append(s)
                    ptrs[i] = s.ctypes.data
        self._h = C.c_void_p()
        # bound now: at interpreter exit the module's globals may already be gone
        self._destroy = lib().plq_ensemble_destroy
        check(lib().plq_ensemble_create(gpu._h, n, arr, ptrs, C.byref(self._h)))
        self.n = n

    def close(self):
        if getattr(self, "_h", None):
            self._destroy(self._h)
            self._h = None

    __del__ = close

    def add_ladder(self, member_ids, betas, every: int, seed: int = 0):
        k = len(member_ids)
        ids = (C.c_int32 * k)(*member_ids)
        bs = (C.c_double * k)(*betas)
        check(lib().plq_ensemble_add_ladder(self._h, k, ids, bs, every, seed))

    def advance(self, sweeps: int):
        check(lib().plq_ensemble_advance(self._h, sweeps))

    def advance_unbatched(self, sweeps: int):
        check(lib().plq_ensemble_advance_unbatched(self._h, sweeps))

    def set_config(self, ranks_per_thread: int, ctas_per_sm: int):
        check(lib().plq_ensemble_set_config(self._h, ranks_per_thread, ctas_per_sm))

    def tune(self, trial_sweeps: int = 10):
        r, c, ms = C.c_int32(), C.c_int32(), C.c_double()
        check(lib().plq_ensemble_tune(self._h, trial_sweeps, C.byref(r), C.byref(c), C.byref(ms)))
        return r.value, c.value, ms.value

    def set_beta(self, m: int, beta: float) -> None:
        """Member m runs at `beta` from its next sweep (members outside ladders)."""
        check(lib().plq_ensemble_set_beta(self._h, m, beta))

    def member_config(self, m: int) -> int:
        """Member m's four-site words per thread (0: the generic body)."""
        w = C.c_int32()
        check(lib().plq_ensemble_member_config(self._h, m, C.byref(w)))
        return w.value

    def sync(self):
        check(lib().plq_ensemble_sync(self._h))

    def n_vars(self, m: int | None = None) -> int:
        if m is None:
            return int(lib().plq_ensemble_n_vars(self._h))
        d = self.descs[m]
        n = int(np.prod([d.shape[i] for i in range(d.d)]))
        return n * d.d if d.model == 2 else n

    def read(self, m: int) -> np.ndarray:
        out = np.empty(self.n_vars(m), dtype=np.uint8)
        check(lib().plq_ensemble_read(self._h, m, out.ctypes.data))
        return out

    def primaries(self, m: int) -> np.ndarray:
        out = np.zeros(66, dtype=np.int64)
        n = C.c_int32()
        check(lib().plq_ensemble_primaries(self._h, m, out.ctypes.data, C.byref(n)))
        return out[: n.value].copy()

    def primaries_all(self) -> list[np.ndarray]:
        """Every member's primaries in one device round-trip."""
        stride = 66
        out = np.zeros((self.n, stride), dtype=np.int64)
        counts = np.zeros(self.n, dtype=np.int32)
        check(lib().plq_ensemble_primaries_all(self._h, out.ctypes.data, stride, counts.ctypes.data))
        return [out[m, : counts[m]].copy() for m in range(self.n)]

    def betas(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float64)
        check(lib().plq_ensemble_betas(self._h, out.ctypes.data))
        return out

    @property
    def cuda_stream(self) -> int:
        return lib().plq_ensemble_cuda_stream(self._h) or 0

    @property
    def launches(self) -> int:
        return int(lib().plq_ensemble_launches(self._h))


def swap_phase(member_of_slot: np.ndarray, beta_of_member: np.ndarray, energy: np.ndarray, j_of_member: np.ndarray,
               ladder_seed: int, attempt: int) -> int:
    """The ladder's swap rule on the host (plq_tempering_swap_phase), in place
    on the int32 slot table and the float64 betas; returns the swaps taken."""
    assert member_of_slot.dtype == np.int32 and beta_of_member.dtype == np.float64
    assert energy.dtype == np.int64 and j_of_member.dtype == np.float64
    acc = C.c_int32()
    check(lib().plq_tempering_swap_phase(len(member_of_slot), member_of_slot.ctypes.data_as(_P(C.c_int32)),
                                         beta_of_member.ctypes.data_as(_P(C.c_double)),
                                         energy.ctypes.data_as(_P(C.c_int64)),
                                         j_of_member.ctypes.data_as(_P(C.c_double)), ladder_seed, attempt,
                                         C.byref(acc)))
    return acc.value


class TuneEntry(C.Structure):
    _fields_ = [("model", C.c_int32), ("q", C.c_int32), ("d", C.c_int32), ("updater", C.c_int32),
                ("rng", C.c_int32), ("words_per_thread", C.c_int32), ("shape", C.c_int64 * 4),
                ("members", C.c_int32), ("pad", C.c_int32), ("ms_per_sweep", C.c_double)]


def tune_entries() -> list[dict]:
    """The process-wide tuning table: one entry per member shape tuned so far."""
    n = C.c_int32()
    check(lib().plq_tune_entries(None, 0, C.byref(n)))
    arr = (TuneEntry * max(1, n.value))()
    check(lib().plq_tune_entries(arr, n.value, C.byref(n)))
    names = {0: "ising", 1: "potts", 2: "gauge"}
    return [{"model": names.get(t.model, t.model), "q": t.q, "shape": list(t.shape)[: t.d],
             "updater": ["metropolis", "heatbath", "cluster"][t.updater], "rng": ["stream", "keyed"][t.rng],
             "words_per_thread": t.words_per_thread, "members": t.members,
             "ms_per_sweep_alone": round(t.ms_per_sweep, 5)} for t in arr[: n.value]]


def batched_workload_spec(seed: int = 20260718):
    """The batched-ensemble workload: 64 4D Z2 gauge lattices, L in {8, 12, 16,
    24} with 16 each, beta uniformly spaced over [0.40, 0.48], checkerboard heat
    bath on links; beside them 256 3D Ising replicas in five parallel-tempering
    ladders (L in {16, 24, 32, 48, 64}, 52 + 4 x 51 replicas), beta
    geometrically spaced over [0.20, 0.24] in each ladder, checkerboard
    Metropolis.  Keyed stream (the reference GPU kernels' randomness), hot
    starts from per-member seeds.  Returns (descs, starts, ladders) with
    ladders as (member ids, betas) pairs."""
    from . import GAUGE, HEATBATH, ISING, METROPOLIS, RNG_KEYED, hot_start, make_desc

    descs, starts, ladders = [], [], []
    s = seed
    for L in (8, 12, 16, 24):
        for beta in np.linspace(0.40, 0.48, 16):
            start, _ = hot_start(s, 2, 4 * L ** 4)
            descs.append(make_desc(GAUGE, 2, (L, L, L, L), HEATBATH, beta=float(beta), seed=s, rng=RNG_KEYED,
                                   sweeps_between=1, batch=1))
            starts.append(start)
            s += 1
    for L, k in ((16, 52), (24, 51), (32, 51), (48, 51), (64, 51)):
        betas = [float(b) for b in np.geomspace(0.20, 0.24, k)]
        ids = []
        for b in betas:
            start, _ = hot_start(s, 2, L ** 3)
            ids.append(len(descs))
            descs.append(make_desc(ISING, 2, (L, L, L), METROPOLIS, beta=b, seed=s, rng=RNG_KEYED,
                                   sweeps_between=1, batch=1))
            starts.append(start)
            s += 1
        ladders.append((ids, betas))
    return descs, starts, ladders


def build_ensemble(gpu, descs, starts, ladders, seed: int = 20260718, pt_every: int = 10) -> Ensemble:
    """An ensemble of `descs` from host `starts`, with its tempering ladders."""
    ens = Ensemble(gpu, descs, starts)
    for i, (ids, betas) in enumerate(ladders):
        ens.add_ladder(ids, betas, pt_every, seed=seed + 1000 + i)
    return ens
