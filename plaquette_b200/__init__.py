"""plaquette_b200 -- B200 (sm_100a) lattice Monte Carlo backend.

Python host mirror of the reference's device API (swvasquez/plaquette):

* ``Gpu.new()`` -- ``Gpu::new`` (src/device.rs:42-78); ``None`` without a device.
* ``GpuChain`` -- ``GpuChain<Q>`` (src/device.rs:590-701): ``advance`` and
  iteration yield owned configurations every ``sweeps_between`` sweeps.
* ``ising.gpu_chain`` / ``potts.gpu_chain`` / ``gauge.gpu_chain`` -- the
  per-model constructors (src/models/{ising,potts,gauge}/gpu.rs).
* ``GpuClusterChain`` -- ``GpuClusterChain<Q>`` with ``swendsen_wang`` and
  ``wolff`` (src/gpu_cluster.rs:144-637).

Everything runs through the C ABI of ``include/plaquette.h`` in
``_lib/libplaquette_b200.so``; there is no CPU fallback -- importing this
package fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from types import SimpleNamespace

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libplaquette_b200.so")

PLQ_OK, PLQ_ENODEV, PLQ_EINVAL, PLQ_EUNSUPPORTED, PLQ_ECUDA, PLQ_ENOMEM, PLQ_ECAP, PLQ_EDEVICE, PLQ_EBUSY = range(9)
ISING, POTTS, GAUGE = 0, 1, 2
METROPOLIS, HEATBATH, CLUSTER = 0, 1, 2
EXTENT_ALL, EXTENT_SEEDED = 0, 1
RELABEL_REDRAW, RELABEL_FORCED = 0, 1
RNG_STREAM, RNG_KEYED = 0, 1
FLAG_NO_FUSED = 1
FLAG_TINY_PASS_CAP = 2
FLAG_TEST_COPY_STALL = 4
FLAG_GENERIC_PASS = 8
FLAG_NO_PACKED = 16
FLAG_NO_FIRST_HASH = 32
MAX_D = 8
MAX_Q = 64
GPU_BATCH = 64  # src/device.rs:501

Kernel = SimpleNamespace(Metropolis=METROPOLIS, HeatBath=HEATBATH)
Extent = SimpleNamespace(All=EXTENT_ALL, Seeded=EXTENT_SEEDED)
Relabel = SimpleNamespace(Redraw=RELABEL_REDRAW, ForcedChange=RELABEL_FORCED)


class PlaquetteError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class ContractError(PlaquetteError, ValueError):
    """A contract violation: the reference panics with the same message."""


class UnsupportedError(PlaquetteError, NotImplementedError):
    pass


class ChainDesc(C.Structure):
    _fields_ = [
        ("model", C.c_int32),
        ("q", C.c_int32),
        ("d", C.c_int32),
        ("updater", C.c_int32),
        ("shape", C.c_int64 * MAX_D),
        ("extent", C.c_int32),
        ("relabel", C.c_int32),
        ("rng", C.c_int32),
        ("flags", C.c_int32),
        ("beta", C.c_double),
        ("j", C.c_double),
        ("h", C.c_double),
        ("offsets", C.c_double * MAX_Q),
        ("seed", C.c_uint64),
        ("stream_offset", C.c_uint64),
        ("sweeps_between", C.c_int64),
        ("batch", C.c_int64),
        ("sweep_offset", C.c_uint64),
    ]


_lib = None

# Every entry point of include/plaquette.h with its ctypes signature.
_SIGNATURES = {
    "plq_version": ([], C.c_char_p),
    "plq_strerror": ([C.c_int], C.c_char_p),
    "plq_last_error": ([], C.c_char_p),
    "plq_device_count": ([C.POINTER(C.c_int)], C.c_int),
    "plq_ctx_create": ([C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "plq_ctx_destroy": ([C.c_void_p], None),
    "plq_chain_validate": ([C.POINTER(ChainDesc)], C.c_int),
    "plq_bond_probability": ([C.c_int32, C.c_double, C.c_double], C.c_double),
    "plq_fold_seed": ([C.c_uint64], C.c_uint32),
    "plq_hot_start": ([C.c_uint64, C.c_int32, C.c_int64, C.c_void_p, C.POINTER(C.c_uint64)], C.c_int),
    "plq_chain_create": ([C.c_void_p, C.POINTER(ChainDesc), C.c_void_p, C.POINTER(C.c_void_p)], C.c_int),
    "plq_chain_advance": ([C.c_void_p, C.c_uint64], C.c_int),
    "plq_chain_next": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "plq_chain_next_batch": ([C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p], C.c_int),
    "plq_chain_read": ([C.c_void_p, C.c_void_p], C.c_int),
    "plq_chain_primaries": ([C.c_void_p, C.c_void_p, C.POINTER(C.c_int32)], C.c_int),
    "plq_chain_sync": ([C.c_void_p], C.c_int),
    "plq_chain_status": ([C.c_void_p], C.c_int),
    "plq_chain_sweeps_done": ([C.c_void_p], C.c_uint64),
    "plq_chain_stream_position": ([C.c_void_p, C.POINTER(C.c_uint64)], C.c_int),
    "plq_chain_n_vars": ([C.c_void_p], C.c_int64),
    "plq_chain_cuda_stream": ([C.c_void_p], C.c_void_p),
    "plq_chain_launches": ([C.c_void_p], C.c_uint64),
    "plq_chain_path": ([C.c_void_p], C.c_char_p),
    "plq_chain_axis_pair_sums": ([C.c_void_p, C.c_void_p, C.c_int64], C.c_int),
    "plq_chain_polyakov": ([C.c_void_p, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)], C.c_int),
    "plq_chain_wilson": ([C.c_void_p, C.c_int32, C.c_void_p, C.c_int64, C.POINTER(C.c_int64),
                          C.POINTER(C.c_int32)], C.c_int),
    "plq_chain_cluster_labels": ([C.c_void_p, C.c_void_p], C.c_int),
    "plq_chain_cluster_histogram": ([C.c_void_p, C.c_void_p, C.c_int32], C.c_int),
    "plq_chain_destroy": ([C.c_void_p], None),
    "plq_ising_metropolis_noalloc": ([C.c_void_p, C.c_int32, C.POINTER(C.c_int64), C.c_double, C.c_double,
                                      C.c_double, C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p,
                                      C.POINTER(C.c_uint64)], C.c_int),
}


def lib():
    """The loaded C-ABI library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m plaquette_b200.build` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def extra_signatures(table: dict) -> None:
    """Register signatures of entry points declared by other modules."""
    L = lib()
    for name, (args, res) in table.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
        _SIGNATURES[name] = (args, res)


def exported_symbols() -> list[str]:
    return sorted(_SIGNATURES)


def check(rc: int) -> None:
    if rc == PLQ_OK:
        return
    msg = lib().plq_last_error().decode() or lib().plq_strerror(rc).decode()
    if rc == PLQ_EINVAL:
        raise ContractError(rc, msg)
    if rc == PLQ_EUNSUPPORTED:
        raise UnsupportedError(rc, msg)
    raise PlaquetteError(rc, msg)


def version() -> str:
    return lib().plq_version().decode()


def device_count() -> int:
    n = C.c_int(0)
    lib().plq_device_count(C.byref(n))
    return n.value


def fold_seed(seed: int) -> int:
    return lib().plq_fold_seed(seed)


def bond_probability(model: int, j: float, beta: float) -> float:
    return lib().plq_bond_probability(model, j, beta)


def hot_start(seed: int, q: int, n_vars: int) -> tuple[np.ndarray, int]:
    """``RandRng::seed_from_u64(seed)`` + ``Configuration::hot``: (states, draws consumed)."""
    out = np.empty(n_vars, dtype=np.uint8)
    draws = C.c_uint64(0)
    check(lib().plq_hot_start(seed, q, n_vars, out.ctypes.data, C.byref(draws)))
    return out, draws.value


class Gpu:
    """``Gpu`` (src/device.rs:31-78): one CUDA device context."""

    def __init__(self, handle, device: int):
        self._h = handle
        self.device = device

    @classmethod
    def new(cls, device: int = 0):
        h = C.c_void_p()
        rc = lib().plq_ctx_create(device, C.byref(h))
        if rc == PLQ_ENODEV:
            return None
        check(rc)
        return cls(h, device)

    def __del__(self):
        try:
            if self._h:
                lib().plq_ctx_destroy(self._h)
                self._h = None
        except Exception:
            pass


def make_desc(model, q, shape, updater, *, beta, j=1.0, h=0.0, offsets=None, seed=0, rng=RNG_STREAM,
              stream_offset=0, sweeps_between=1, batch=GPU_BATCH, extent=EXTENT_ALL,
              relabel=RELABEL_REDRAW, flags=0, sweep_offset=0) -> ChainDesc:
    d = ChainDesc()
    d.model = model
    d.q = q
    d.d = len(shape)
    d.updater = updater
    for i, L in enumerate(shape):
        d.shape[i] = int(L)
    d.extent = extent
    d.relabel = relabel
    d.rng = rng
    d.beta = beta
    d.j = j
    d.h = h
    if offsets is not None:
        for a, v in enumerate(offsets):
            d.offsets[a] = v
    d.seed = seed
    d.stream_offset = stream_offset
    d.sweeps_between = sweeps_between
    d.batch = batch
    d.flags = flags
    d.sweep_offset = sweep_offset
    return d


def validate(desc: ChainDesc) -> None:
    check(lib().plq_chain_validate(C.byref(desc)))


class GpuChain:
    """A device chain (local or cluster) over a copy of ``start``.

    ``next()`` runs ``sweeps_between`` sweeps and returns an owned copy of the
    configuration (uint8 states in the reference's linear order), exactly as
    ``GpuChain::next`` / ``GpuClusterChain::next`` do.
    """

    def __init__(self, gpu: Gpu, desc: ChainDesc, start: np.ndarray | None):
        self.gpu = gpu
        self.desc = desc
        self._h = C.c_void_p()
        ptr = None
        if start is not None:
            start = np.ascontiguousarray(start, dtype=np.uint8)
            ptr = start.ctypes.data
        # bound now: at interpreter exit the module's globals may already be gone
        self._destroy = lib().plq_chain_destroy
        check(lib().plq_chain_create(gpu._h, C.byref(desc), ptr, C.byref(self._h)))
        self.n_vars = int(lib().plq_chain_n_vars(self._h))
        self.n_primaries = {ISING: 2, POTTS: 1 + desc.q, GAUGE: 1}[desc.model]
        self._buffer: list[np.ndarray] = []

    def close(self):
        if getattr(self, "_h", None):
            self._destroy(self._h)
            self._h = None

    __del__ = close

    def advance(self, sweeps: int) -> None:
        check(lib().plq_chain_advance(self._h, sweeps))

    def __iter__(self):
        return self

    def __next__(self) -> np.ndarray:
        if not self._buffer:
            batch = int(self.desc.batch)
            out = np.empty((batch, self.n_vars), dtype=np.uint8)
            check(lib().plq_chain_next_batch(self._h, batch, out.ctypes.data, None))
            self._buffer = list(out)
        return self._buffer.pop(0)

    def next_sample(self) -> tuple[np.ndarray, np.ndarray]:
        out = np.empty(self.n_vars, dtype=np.uint8)
        prim = np.empty(self.n_primaries, dtype=np.int64)
        check(lib().plq_chain_next(self._h, out.ctypes.data, prim.ctypes.data))
        return out, prim

    def next_batch(self, count: int, states: bool = True) -> tuple[np.ndarray | None, np.ndarray]:
        out = np.empty((count, self.n_vars), dtype=np.uint8) if states else None
        prim = np.empty((count, self.n_primaries), dtype=np.int64)
        check(lib().plq_chain_next_batch(self._h, count, out.ctypes.data if states else None, prim.ctypes.data))
        return out, prim

    def read(self) -> np.ndarray:
        out = np.empty(self.n_vars, dtype=np.uint8)
        check(lib().plq_chain_read(self._h, out.ctypes.data))
        return out

    def primaries(self) -> np.ndarray:
        out = np.empty(self.n_primaries, dtype=np.int64)
        n = C.c_int32(0)
        check(lib().plq_chain_primaries(self._h, out.ctypes.data, C.byref(n)))
        return out[: n.value]

    def axis_pair_sums(self) -> list[np.ndarray]:
        """``axis_pair_sums`` (src/models/mod.rs:44-61) of the current
        configuration: one int64 row per axis, displacements 0..L_mu/2."""
        shape = [int(self.desc.shape[i]) for i in range(self.desc.d)]
        out = np.zeros(sum(L // 2 + 1 for L in shape), dtype=np.int64)
        check(lib().plq_chain_axis_pair_sums(self._h, out.ctypes.data, out.size))
        rows, off = [], 0
        for L in shape:
            rows.append(out[off:off + L // 2 + 1].copy())
            off += L // 2 + 1
        return rows

    def polyakov(self, direction: int) -> tuple[int, int]:
        """Polyakov loop along `direction` as (sum of line products, lines)."""
        s, n = C.c_int64(0), C.c_int64(0)
        check(lib().plq_chain_polyakov(self._h, direction, C.byref(s), C.byref(n)))
        return s.value, n.value

    def wilson(self, max_side: int) -> tuple[np.ndarray, int]:
        """Wilson rectangle totals table (r, t = 0..m) and the placements divisor."""
        shortest = min(int(self.desc.shape[i]) for i in range(self.desc.d))
        m = min(max_side, shortest // 2)
        out = np.zeros((m + 1) * (m + 1), dtype=np.int64)
        pl, mo = C.c_int64(0), C.c_int32(0)
        check(lib().plq_chain_wilson(self._h, max_side, out.ctypes.data, out.size, C.byref(pl), C.byref(mo)))
        return out.reshape(mo.value + 1, mo.value + 1), pl.value

    def sync(self) -> None:
        check(lib().plq_chain_sync(self._h))

    @property
    def sweeps_done(self) -> int:
        return int(lib().plq_chain_sweeps_done(self._h))

    def stream_position(self) -> int:
        v = C.c_uint64(0)
        check(lib().plq_chain_stream_position(self._h, C.byref(v)))
        return v.value

    @property
    def cuda_stream(self) -> int:
        return lib().plq_chain_cuda_stream(self._h) or 0

    @property
    def path(self) -> str:
        return lib().plq_chain_path(self._h).decode()

    @property
    def launches(self) -> int:
        return int(lib().plq_chain_launches(self._h))


# --------------------------------------------------- per-model constructors
def _ising_gpu_chain(gpu, shape, j, h, beta, seed, start, sweeps_between, batch, kernel, *, rng=RNG_KEYED,
                     stream_offset=0):
    """``models::ising::gpu_chain`` (src/models/ising/gpu.rs:57-95)."""
    d = make_desc(ISING, 2, shape, kernel, beta=beta, j=j, h=h, seed=seed, rng=rng, stream_offset=stream_offset,
                  sweeps_between=sweeps_between, batch=batch)
    return GpuChain(gpu, d, start)


def _potts_gpu_chain(gpu, shape, q, j, offsets, beta, seed, start, sweeps_between, batch, kernel, *,
                     rng=RNG_KEYED, stream_offset=0):
    """``models::potts::gpu_chain`` (src/models/potts/gpu.rs:93-148)."""
    d = make_desc(POTTS, q, shape, kernel, beta=beta, j=j, offsets=offsets, seed=seed, rng=rng,
                  stream_offset=stream_offset, sweeps_between=sweeps_between, batch=batch)
    return GpuChain(gpu, d, start)


def _gauge_gpu_chain(gpu, shape, j, beta, seed, start, sweeps_between, batch, kernel, *, rng=RNG_KEYED,
                     stream_offset=0):
    """``models::gauge::gpu_chain`` (src/models/gauge/gpu.rs:54-107)."""
    d = make_desc(GAUGE, 2, shape, kernel, beta=beta, j=j, seed=seed, rng=rng, stream_offset=stream_offset,
                  sweeps_between=sweeps_between, batch=batch)
    return GpuChain(gpu, d, start)


ising = SimpleNamespace(gpu_chain=_ising_gpu_chain)
potts = SimpleNamespace(gpu_chain=_potts_gpu_chain)
gauge = SimpleNamespace(gpu_chain=_gauge_gpu_chain)


class GpuClusterChain(GpuChain):
    """``GpuClusterChain<Q>`` (src/gpu_cluster.rs:144-637)."""

    @classmethod
    def new(cls, gpu, shape, model, q, j, extent, relabel, beta, seed, start, sweeps_between, *,
            rng=RNG_KEYED, stream_offset=0):
        d = make_desc(model, q, shape, CLUSTER, beta=beta, j=j, seed=seed, rng=rng, stream_offset=stream_offset,
                      sweeps_between=sweeps_between, batch=1, extent=extent, relabel=relabel)
        return cls(gpu, d, start)

    @classmethod
    def swendsen_wang(cls, gpu, shape, model, q, j, beta, seed, start, sweeps_between, **kw):
        return cls.new(gpu, shape, model, q, j, EXTENT_ALL, RELABEL_REDRAW, beta, seed, start, sweeps_between, **kw)

    @classmethod
    def wolff(cls, gpu, shape, model, q, j, beta, seed, start, sweeps_between, **kw):
        return cls.new(gpu, shape, model, q, j, EXTENT_SEEDED, RELABEL_FORCED, beta, seed, start, sweeps_between,
                       **kw)

    def __next__(self) -> np.ndarray:
        out = np.empty(self.n_vars, dtype=np.uint8)
        check(lib().plq_chain_next(self._h, out.ctypes.data, None))
        return out

    def labels(self) -> np.ndarray:
        """Canonical (minimum-site) cluster label of every site, last decomposition."""
        out = np.empty(self.n_vars, dtype=np.int32)
        check(lib().plq_chain_cluster_labels(self._h, out.ctypes.data))
        return out

    def size_histogram(self, nbins: int = 32) -> np.ndarray:
        """Clusters per size bin [2^k, 2^(k+1)) of the last decomposition (Wolff: last cluster)."""
        out = np.zeros(nbins, dtype=np.int64)
        check(lib().plq_chain_cluster_histogram(self._h, out.ctypes.data, nbins))
        return out
