"""ctypes wrapper over the C oracle (``plq_oracle.c``).

TEST INFRASTRUCTURE ONLY.  The oracle restates the reference's CPU update
path (``src/updater.rs``, ``src/cluster.rs``, ``src/models/*/mod.rs``,
``src/lattice.rs``) and its GPU keyed stream (``src/wgsl/*.wgsl``).  Only the
tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import
it; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libplq_oracle.so")

ISING, POTTS, GAUGE = 0, 1, 2
METROPOLIS, HEATBATH = 0, 1
RANDOM, CHECKERBOARD = 0, 1
ALL, SEEDED = 0, 1
REDRAW, FORCED = 0, 1
MAX_Q = 64
MAX_D = 16


class Rng(C.Structure):
    _fields_ = [
        ("state_lo", C.c_uint64),
        ("state_hi", C.c_uint64),
        ("inc_lo", C.c_uint64),
        ("inc_hi", C.c_uint64),
        ("draws", C.c_uint64),
    ]

    @property
    def state(self) -> int:
        return (self.state_hi << 64) | self.state_lo

    @property
    def inc(self) -> int:
        return (self.inc_hi << 64) | self.inc_lo


class _Lattice(C.Structure):
    _fields_ = [
        ("d", C.c_int32),
        ("shape", C.c_int64 * MAX_D),
        ("n_sites", C.c_int64),
        ("stride", C.c_int64 * MAX_D),
        ("neighbors", C.POINTER(C.c_int64)),
        ("parity", C.POINTER(C.c_uint8)),
        ("staples", C.POINTER(C.c_int64)),
    ]


class _Model(C.Structure):
    _fields_ = [
        ("model", C.c_int32),
        ("q", C.c_int32),
        ("j", C.c_double),
        ("h", C.c_double),
        ("offsets", C.c_double * MAX_Q),
    ]


def build() -> str:
    """Compile the oracle with its Makefile (gcc) if it is missing or stale."""
    src = os.path.join(_HERE, "plq_oracle.c")
    if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        L = _lib
        P = C.POINTER
        u8p = P(C.c_uint8)
        i64p = P(C.c_int64)
        L.orc_rng_seed_from_u64.argtypes = [P(Rng), C.c_uint64]
        L.orc_rng_from_state.argtypes = [P(Rng), C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64]
        L.orc_rng_next_u64.argtypes = [P(Rng)]
        L.orc_rng_next_u64.restype = C.c_uint64
        L.orc_rng_next_f64.argtypes = [P(Rng)]
        L.orc_rng_next_f64.restype = C.c_double
        L.orc_rng_next_below.argtypes = [P(Rng), C.c_uint64]
        L.orc_rng_next_below.restype = C.c_uint64
        L.orc_rng_advance.argtypes = [P(Rng), C.c_uint64]
        L.orc_hot_start.argtypes = [P(Rng), C.c_int32, C.c_int64, u8p]
        L.orc_lowbias32.argtypes = [C.c_uint32]
        L.orc_lowbias32.restype = C.c_uint32
        L.orc_keyed_uniform.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32]
        L.orc_keyed_uniform.restype = C.c_float
        L.orc_fold_seed.argtypes = [C.c_uint64]
        L.orc_fold_seed.restype = C.c_uint32
        L.orc_lattice_init.argtypes = [P(_Lattice), C.c_int32, i64p]
        L.orc_lattice_init.restype = C.c_int
        L.orc_lattice_build_staples.argtypes = [P(_Lattice)]
        L.orc_lattice_build_staples.restype = C.c_int
        L.orc_lattice_free.argtypes = [P(_Lattice)]
        L.orc_energy.argtypes = [P(_Model), P(_Lattice), u8p]
        L.orc_energy.restype = C.c_double
        L.orc_energy_delta.argtypes = [P(_Model), P(_Lattice), u8p, C.c_int64, C.c_int32]
        L.orc_energy_delta.restype = C.c_double
        L.orc_primaries.argtypes = [P(_Model), P(_Lattice), u8p, i64p]
        L.orc_primaries.restype = C.c_int
        L.orc_local_sweep.argtypes = [P(_Model), P(_Lattice), u8p, C.c_int32, C.c_int32, C.c_double, P(Rng)]
        L.orc_local_sweep.restype = C.c_double
        L.orc_local_sweeps.argtypes = [P(_Model), P(_Lattice), u8p, C.c_int32, C.c_int32, C.c_double,
                                       P(Rng), C.c_int64]
        L.orc_local_sweeps.restype = C.c_double
        L.orc_local_site_slice.argtypes = [P(_Model), P(_Lattice), u8p, C.c_int32, C.c_double, P(Rng),
                                           C.c_int32, C.c_int64, C.c_int64, i64p]
        L.orc_local_site_slice.restype = C.c_double
        L.orc_bond_probability.argtypes = [P(_Model), C.c_double]
        L.orc_bond_probability.restype = C.c_double
        L.orc_site_clusters.argtypes = [P(_Lattice), u8p, C.c_double, P(Rng), i64p, i64p]
        L.orc_site_clusters.restype = C.c_int64
        L.orc_grow_cluster.argtypes = [P(_Lattice), u8p, C.c_int64, C.c_double, P(Rng), i64p]
        L.orc_grow_cluster.restype = C.c_int64
        L.orc_cluster_sweep.argtypes = [P(_Model), P(_Lattice), u8p, C.c_int32, C.c_int32, C.c_double, P(Rng)]
        L.orc_cluster_sweep.restype = C.c_double
        L.orc_keyed_local_sweep.argtypes = [P(_Model), P(_Lattice), u8p, C.c_int32, C.c_double,
                                            C.c_uint32, C.c_uint32]
        L.orc_keyed_slab_pass.argtypes = [P(_Model), P(_Lattice), u8p, C.c_int32, C.c_double, C.c_uint32,
                                          C.c_uint32, C.c_int32, C.c_int64, C.c_int64, C.c_int64]
        L.orc_keyed_cluster_sweep.argtypes = [P(_Model), P(_Lattice), u8p, C.c_int32, C.c_int32, C.c_double,
                                              C.c_uint32, C.c_uint32, i64p]
        L.orc_axis_pair_sums.argtypes = [P(_Model), P(_Lattice), u8p, i64p]
        L.orc_axis_pair_sums.restype = C.c_int64
        L.orc_polyakov_sum.argtypes = [P(_Lattice), u8p, C.c_int32, i64p]
        L.orc_polyakov_sum.restype = C.c_int64
        L.orc_wilson_totals.argtypes = [P(_Lattice), u8p, C.c_int32, i64p, i64p]
        L.orc_wilson_totals.restype = C.c_int32
        L.orc_pt_exp.argtypes = [C.c_double]
        L.orc_pt_exp.restype = C.c_double
        L.orc_pt_swap_phase.argtypes = [C.c_int32, P(C.c_int32), P(C.c_double), i64p, P(C.c_double), C.c_uint32,
                                        C.c_uint64]
        L.orc_pt_swap_phase.restype = C.c_int32
    return _lib


def _u8(a: np.ndarray):
    assert a.dtype == np.uint8 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def _i64(a: np.ndarray):
    assert a.dtype == np.int64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_int64))


class PcgStream:
    """The reference ``RandRng`` (PCG64 from ``seed_from_u64``)."""

    def __init__(self, seed: int | None = None, *, state: int | None = None, inc: int | None = None):
        self.r = Rng()
        if seed is not None:
            lib().orc_rng_seed_from_u64(C.byref(self.r), C.c_uint64(seed))
        else:
            m = (1 << 64) - 1
            lib().orc_rng_from_state(C.byref(self.r), state & m, state >> 64, inc & m, inc >> 64)

    def next_u64(self) -> int:
        return lib().orc_rng_next_u64(C.byref(self.r))

    def next_f64(self) -> float:
        return lib().orc_rng_next_f64(C.byref(self.r))

    def next_below(self, n: int) -> int:
        return lib().orc_rng_next_below(C.byref(self.r), n)

    def advance(self, delta: int) -> None:
        lib().orc_rng_advance(C.byref(self.r), delta)

    @property
    def draws(self) -> int:
        return self.r.draws

    @property
    def ref(self):
        return C.byref(self.r)


def keyed_uniform(seed32: int, variable: int, sweep: int) -> float:
    return lib().orc_keyed_uniform(seed32 & 0xFFFFFFFF, variable & 0xFFFFFFFF, sweep & 0xFFFFFFFF)


def lowbias32(x: int) -> int:
    return lib().orc_lowbias32(x & 0xFFFFFFFF)


def fold_seed(seed: int) -> int:
    return lib().orc_fold_seed(seed)


class Lattice:
    """``Lattice<D>`` (src/lattice.rs): neighbour/parity tables, staples on demand."""

    def __init__(self, shape, staples: bool = False):
        self.shape = tuple(int(x) for x in shape)
        self.d = len(self.shape)
        self.lat = _Lattice()
        arr = (C.c_int64 * MAX_D)(*self.shape)
        rc = lib().orc_lattice_init(C.byref(self.lat), self.d, arr)
        if rc != 0:
            raise ValueError(f"bad lattice shape {shape}")
        self.n_sites = int(self.lat.n_sites)
        self.n_links = self.n_sites * self.d
        if staples:
            self.build_staples()

    def build_staples(self):
        if not self.lat.staples:
            if lib().orc_lattice_build_staples(C.byref(self.lat)) != 0:
                raise ValueError("staples need D >= 2")

    def neighbors(self) -> np.ndarray:
        n = self.n_sites * 2 * self.d
        return np.ctypeslib.as_array(self.lat.neighbors, shape=(n,)).reshape(self.n_sites, 2 * self.d).copy()

    def parity(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.lat.parity, shape=(self.n_sites,)).copy()

    def staples(self) -> np.ndarray:
        self.build_staples()
        n = self.n_links * 6 * (self.d - 1)
        return np.ctypeslib.as_array(self.lat.staples, shape=(n,)).reshape(self.n_links, 6 * (self.d - 1)).copy()

    def __del__(self):
        try:
            lib().orc_lattice_free(C.byref(self.lat))
        except Exception:
            pass


class Model:
    """One of ``Ising``, ``Potts<Q>``, ``Z2Gauge`` with its couplings."""

    def __init__(self, kind: int, q: int = 2, j: float = 1.0, h: float = 0.0, offsets=None):
        self.m = _Model()
        self.m.model = kind
        self.m.q = q if kind == POTTS else 2
        self.m.j = j
        self.m.h = h
        if offsets is not None:
            for a, v in enumerate(offsets):
                self.m.offsets[a] = v
        self.kind = kind
        self.q = self.m.q

    @classmethod
    def ising(cls, j=1.0, h=0.0):
        return cls(ISING, 2, j, h)

    @classmethod
    def potts(cls, q, j=1.0, offsets=None):
        return cls(POTTS, q, j, 0.0, offsets)

    @classmethod
    def gauge(cls, j=1.0):
        return cls(GAUGE, 2, j)

    @property
    def ref(self):
        return C.byref(self.m)

    def n_vars(self, lat: Lattice) -> int:
        return lat.n_links if self.kind == GAUGE else lat.n_sites

    def energy(self, lat: Lattice, cfg: np.ndarray) -> float:
        if self.kind == GAUGE:
            lat.build_staples()
        return lib().orc_energy(self.ref, C.byref(lat.lat), _u8(cfg))

    def energy_delta(self, lat: Lattice, cfg: np.ndarray, var: int, proposed: int) -> float:
        if self.kind == GAUGE:
            lat.build_staples()
        return lib().orc_energy_delta(self.ref, C.byref(lat.lat), _u8(cfg), var, proposed)

    def primaries(self, lat: Lattice, cfg: np.ndarray) -> np.ndarray:
        out = np.zeros(1 + MAX_Q, dtype=np.int64)
        n = lib().orc_primaries(self.ref, C.byref(lat.lat), _u8(cfg), _i64(out))
        return out[:n].copy()

    def bond_probability(self, beta: float) -> float:
        return lib().orc_bond_probability(self.ref, beta)


def local_sweeps(model: Model, lat: Lattice, cfg: np.ndarray, kernel: int, beta: float,
                 rng: PcgStream, n_sweeps: int = 1, schedule: int = CHECKERBOARD) -> float:
    """``LocalUpdate::sweep`` repeated (src/updater.rs:283-348), in place."""
    if model.kind == GAUGE:
        lat.build_staples()
    return lib().orc_local_sweeps(model.ref, C.byref(lat.lat), _u8(cfg), kernel, schedule, beta, rng.ref,
                                  n_sweeps)


def local_site_slice(model, lat, cfg, kernel, beta, rng, color, lo, hi) -> int:
    upd = np.zeros(1, dtype=np.int64)
    lib().orc_local_site_slice(model.ref, C.byref(lat.lat), _u8(cfg), kernel, beta, rng.ref, color, lo, hi,
                               _i64(upd))
    return int(upd[0])


def cluster_sweep(model: Model, lat: Lattice, cfg: np.ndarray, extent: int, relabel: int, beta: float,
                  rng: PcgStream) -> float:
    """``ClusterUpdate::sweep`` (src/updater.rs:541-613), in place."""
    return lib().orc_cluster_sweep(model.ref, C.byref(lat.lat), _u8(cfg), extent, relabel, beta, rng.ref)


def site_clusters(lat: Lattice, cfg: np.ndarray, p: float, rng: PcgStream):
    labels = np.zeros(lat.n_sites, dtype=np.int64)
    sizes = np.zeros(lat.n_sites, dtype=np.int64)
    n = lib().orc_site_clusters(C.byref(lat.lat), _u8(cfg), p, rng.ref, _i64(labels), _i64(sizes))
    return labels, sizes[:n].copy()


def grow_cluster(lat: Lattice, cfg: np.ndarray, seed: int, p: float, rng: PcgStream) -> np.ndarray:
    members = np.zeros(lat.n_sites, dtype=np.int64)
    n = lib().orc_grow_cluster(C.byref(lat.lat), _u8(cfg), seed, p, rng.ref, _i64(members))
    return members[:n].copy()


def keyed_local_sweep(model: Model, lat: Lattice, cfg: np.ndarray, kernel: int, beta: float, seed32: int,
                      sweep: int) -> None:
    """One sweep of the reference WGSL checkerboard (keyed stream), in place."""
    if model.kind == GAUGE:
        lat.build_staples()
    lib().orc_keyed_local_sweep(model.ref, C.byref(lat.lat), _u8(cfg), kernel, beta, seed32 & 0xFFFFFFFF,
                                sweep & 0xFFFFFFFF)


def keyed_slab_pass(model: Model, slab: Lattice, cfg: np.ndarray, kernel: int, beta: float, seed32: int,
                    sweep: int, local_color: int, first: int, last: int, var_offset: int) -> None:
    """One keyed colour pass (the reference WGSL site update) over sites
    [first, last) of a slab lattice -- the slab's planes with a halo plane on
    each side -- whose site s is site s + var_offset of the whole lattice; in
    place.  local_color is the pass's colour in the slab's own parity."""
    lib().orc_keyed_slab_pass(model.ref, C.byref(slab.lat), _u8(cfg), kernel, beta, seed32 & 0xFFFFFFFF,
                              sweep & 0xFFFFFFFF, local_color, first, last, var_offset)


def keyed_cluster_sweep(model: Model, lat: Lattice, cfg: np.ndarray, extent: int, relabel: int, beta: float,
                        seed32: int, sweep: int, want_roots: bool = False):
    roots = np.zeros(lat.n_sites, dtype=np.int64) if want_roots else None
    lib().orc_keyed_cluster_sweep(model.ref, C.byref(lat.lat), _u8(cfg), extent, relabel, beta,
                                  seed32 & 0xFFFFFFFF, sweep & 0xFFFFFFFF,
                                  _i64(roots) if roots is not None else None)
    return roots


def hot_start(n_vars: int, q: int, rng: PcgStream) -> np.ndarray:
    """``Configuration::hot`` (src/configuration.rs:82-87): next_below(Q) per variable."""
    out = np.empty(n_vars, dtype=np.uint8)
    lib().orc_hot_start(rng.ref, q, n_vars, _u8(out))
    return out


def axis_pair_sums(model: Model, lat: Lattice, cfg: np.ndarray) -> list[np.ndarray]:
    """``axis_pair_sums`` (src/models/mod.rs:44-61) with the model's pair:
    one int64 row per axis, displacements r = 0..L_mu/2."""
    shape = [int(lat.lat.shape[i]) for i in range(lat.lat.d)]
    out = np.zeros(sum(L // 2 + 1 for L in shape), dtype=np.int64)
    lib().orc_axis_pair_sums(model.ref, C.byref(lat.lat), _u8(cfg), _i64(out))
    rows, off = [], 0
    for L in shape:
        rows.append(out[off:off + L // 2 + 1].copy())
        off += L // 2 + 1
    return rows


def polyakov_sum(lat: Lattice, cfg: np.ndarray, direction: int) -> tuple[int, int]:
    """``Z2Gauge::polyakov_loop`` (gauge/mod.rs:179-212) as (sum, lines)."""
    lines = np.zeros(1, dtype=np.int64)
    total = lib().orc_polyakov_sum(C.byref(lat.lat), _u8(cfg), direction, _i64(lines))
    return int(total), int(lines[0])


def wilson_totals(lat: Lattice, cfg: np.ndarray, max_side: int) -> tuple[np.ndarray, int]:
    """``Z2Gauge::wilson_rectangles`` (gauge/mod.rs:226-274) as the integer
    totals table and the common divisor (placements)."""
    shortest = min(int(lat.lat.shape[i]) for i in range(lat.lat.d))
    mx = min(max_side, shortest // 2)
    totals = np.zeros((mx + 1) * (mx + 1), dtype=np.int64)
    placements = np.zeros(1, dtype=np.int64)
    got = lib().orc_wilson_totals(C.byref(lat.lat), _u8(cfg), max_side, _i64(totals), _i64(placements))
    assert got == mx
    return totals.reshape(mx + 1, mx + 1), int(placements[0])


def pt_exp(x: float) -> float:
    """The tempering decision's e^x (x <= 0) from basic operations only."""
    return lib().orc_pt_exp(x)


def pt_swap_phase(member_of_slot: np.ndarray, beta_of_member: np.ndarray, energy: np.ndarray,
                  j_of_member: np.ndarray, seed32: int, att: int) -> int:
    """One swap phase of one ladder (attempt `att`), in place on the int32
    slot table and the float64 betas; returns the swaps accepted."""
    assert member_of_slot.dtype == np.int32 and beta_of_member.dtype == np.float64
    assert energy.dtype == np.int64 and j_of_member.dtype == np.float64
    return lib().orc_pt_swap_phase(len(member_of_slot), member_of_slot.ctypes.data_as(C.POINTER(C.c_int32)),
                                   beta_of_member.ctypes.data_as(C.POINTER(C.c_double)), _i64(energy),
                                   j_of_member.ctypes.data_as(C.POINTER(C.c_double)), seed32 & 0xFFFFFFFF, att)
