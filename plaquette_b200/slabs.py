"""One lattice split into slabs along its last axis, one slab per rank, with a
halo exchange before every colour pass.

The reference runs a chain on one adapter (src/device.rs:31-78); this splits
one lattice across devices.  A site lattice of shape (L0, ..., Lz) is cut
into contiguous ranges of planes along its last axis; rank r holds planes
[z0, z0 + nz) plus one halo plane on each side.  Before each colour pass the
ranks exchange boundary planes around the periodic ring (rank r's first plane
becomes rank r - 1's high halo, its last plane rank r + 1's low halo), then
every rank updates the colour on its own planes.  On the keyed stream every
draw is a closed form of (seed, global variable index, sweep) and a colour
pass reads only the other colour, so the slabs together reproduce the
single-device chain bit for bit, for any number of ranks.

An engine holds one slab: `views()` gives its four exchange planes (low halo,
first plane, last plane, high halo) as arrays or tensors the exchange can
copy into and out of, `sync()` waits for its device work, `colour_pass(c)`
runs colour c (global parity) over its planes, `end_sweep()` advances its
sweep counter and `read()` returns its planes.  `DeviceSlab` is the device
engine (plq_slab_* in the library); tests use one built on the oracle.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import ChainDesc, Gpu, check, extra_signatures, lib

LOW_HALO, FIRST_PLANE, LAST_PLANE, HIGH_HALO = 0, 1, 2, 3

_P = C.POINTER
extra_signatures({
    "plq_slab_create": ([C.c_void_p, _P(ChainDesc), C.c_int64, C.c_int64, C.c_void_p, _P(C.c_void_p)], C.c_int),
    "plq_slab_plane": ([C.c_void_p, C.c_int32, _P(C.c_void_p), _P(C.c_int64)], C.c_int),
    "plq_slab_pass": ([C.c_void_p, C.c_int32], C.c_int),
    "plq_slab_end_sweep": ([C.c_void_p], C.c_int),
    "plq_slab_sync": ([C.c_void_p], C.c_int),
    "plq_slab_read": ([C.c_void_p, C.c_void_p], C.c_int),
    "plq_slab_destroy": ([C.c_void_p], None),
})


def split(extent: int, world: int) -> list[tuple[int, int]]:
    """(z0, nz) of every rank: contiguous, sizes differing by at most one."""
    if world < 1 or world > extent:
        raise ValueError(f"cannot split {extent} planes over {world} ranks")
    return [(r * extent // world, (r + 1) * extent // world - r * extent // world) for r in range(world)]


class _DevicePlane:
    """A device plane as a CUDA array (for torch.as_tensor)."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "version": 3}


class DeviceSlab:
    """Planes [z0, z0 + nz) of the lattice `desc` names (keyed stream, Ising
    or Potts sites, d = 2 or 3) on one device; `start` holds those planes."""

    def __init__(self, gpu: Gpu, desc: ChainDesc, z0: int, nz: int, start: np.ndarray):
        start = np.ascontiguousarray(start, dtype=np.uint8)
        h = C.c_void_p()
        self._destroy = lib().plq_slab_destroy  # bound now: module globals may be gone at exit
        check(lib().plq_slab_create(gpu._h, C.byref(desc), z0, nz, start.ctypes.data_as(C.c_void_p), C.byref(h)))
        self._h = h
        self.nz = nz
        self.plane_bytes = start.size // nz

    def plane(self, which: int) -> tuple[int, int]:
        """(device address, bytes) of the low halo, first plane, last plane or high halo."""
        ptr, nbytes = C.c_void_p(), C.c_int64()
        check(lib().plq_slab_plane(self._h, which, C.byref(ptr), C.byref(nbytes)))
        return ptr.value, nbytes.value

    def views(self):
        import torch

        return [torch.as_tensor(_DevicePlane(*self.plane(w)), device="cuda") for w in range(4)]

    def sync(self) -> None:
        check(lib().plq_slab_sync(self._h))

    def colour_pass(self, colour: int) -> None:
        check(lib().plq_slab_pass(self._h, colour))

    def end_sweep(self) -> None:
        check(lib().plq_slab_end_sweep(self._h))

    def read(self) -> np.ndarray:
        out = np.empty(self.nz * self.plane_bytes, dtype=np.uint8)
        check(lib().plq_slab_read(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def local_exchange(engines) -> None:
    """All slabs of the ring in one process: halos copied from the neighbours'
    boundary planes (a single slab is its own neighbour on both sides)."""
    for e in engines:
        e.sync()
    views = [e.views() for e in engines]
    n = len(engines)
    for r in range(n):
        lo, hi = views[(r - 1) % n], views[(r + 1) % n]
        _copy(views[r][LOW_HALO], lo[LAST_PLANE])
        _copy(views[r][HIGH_HALO], hi[FIRST_PLANE])
    if views and not isinstance(views[0][0], np.ndarray):
        import torch

        torch.cuda.synchronize()


def _copy(dst, src) -> None:
    if isinstance(dst, np.ndarray):
        dst[:] = src
    else:
        dst.copy_(src)


def ring_exchange(dist, rank: int, world: int):
    """The halo exchange of one rank over torch.distributed (gloo on CPU
    arrays, NCCL on device planes): its first plane to rank - 1, its last
    plane to rank + 1, the halos from them.  One rank: its own planes."""

    def run(engine) -> None:
        engine.sync()
        v = engine.views()
        if world == 1:
            _copy(v[LOW_HALO], v[LAST_PLANE])
            _copy(v[HIGH_HALO], v[FIRST_PLANE])
            return
        import torch

        t = [torch.from_numpy(x) if isinstance(x, np.ndarray) else x for x in v]
        prev, nxt = (rank - 1) % world, (rank + 1) % world
        ops = [dist.P2POp(dist.isend, t[FIRST_PLANE].contiguous(), prev),
               dist.P2POp(dist.isend, t[LAST_PLANE].contiguous(), nxt),
               dist.P2POp(dist.irecv, t[HIGH_HALO], nxt),
               dist.P2POp(dist.irecv, t[LOW_HALO], prev)]
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        if t[0].is_cuda:
            torch.cuda.synchronize()

    return run


class SlabChain:
    """Sweeps of a slab-split lattice: before each colour pass the halos are
    exchanged (`exchange(engine)` for one rank's engine, or `local_exchange`
    over every engine of the ring when they share a process)."""

    def __init__(self, engines, exchange=None):
        self.engines = list(engines)
        self.exchange = exchange

    def advance(self, sweeps: int) -> None:
        for _ in range(sweeps):
            for colour in (0, 1):
                if self.exchange is None:
                    local_exchange(self.engines)
                else:
                    for e in self.engines:
                        self.exchange(e)
                for e in self.engines:
                    e.colour_pass(colour)
            for e in self.engines:
                e.end_sweep()

    def read(self) -> np.ndarray:
        """The planes of every engine held here, in order."""
        return np.concatenate([e.read() for e in self.engines])
