"""The allocation-free Ising Metropolis entry point.

Callers that cannot allocate device memory themselves (they lend this
library a buffer they own, or must not risk cudaMalloc's implicit
synchronisation) use plq_ising_metropolis_noalloc.  It must give exactly the
results of the allocating chain API on the same seed and stream position,
call after call, although every call reuses the same fixed scratch array.
Collected last so that a run stopping at its first failure has already run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

import plaquette_b200 as plq

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = plq.Gpu.new()
    if g is None:
        pytest.fail("no CUDA device")
    return g


def _noalloc(dev_ptr, shape, beta, seed, offset, sweeps, j=1.0, h=0.0):
    arr = (C.c_int64 * len(shape))(*shape)
    pos = C.c_uint64(0)
    rc = plq.lib().plq_ising_metropolis_noalloc(dev_ptr, len(shape), arr, j, h, beta, seed, offset, sweeps, None,
                                                C.byref(pos))
    plq.check(rc)
    return pos.value


@pytest.mark.parametrize("shape,beta,h", [((64, 32, 16), 0.2216544, 0.0), ((128, 128), 0.4406868, 0.1),
                                          ((16, 8, 8, 8), 0.15, 0.0), ((96,), 0.7, 0.05),
                                          ((4, 4, 4, 4, 4, 4), 0.1, 0.0)], ids=str)
def test_two_calls_match_the_chain_api(gpu, shape, beta, h):
    import torch

    n = int(np.prod(shape))
    seed = 20260718
    start, offset = plq.hot_start(seed, 2, n)
    spins = torch.from_numpy(start.copy()).cuda()
    # the allocating entry point: the same sweeps through a chain
    d = plq.make_desc(plq.ISING, 2, shape, plq.METROPOLIS, beta=beta, h=h, seed=seed, rng=plq.RNG_STREAM,
                      stream_offset=offset, sweeps_between=1, batch=1)
    chain = plq.GpuChain(gpu, d, start)

    pos1 = _noalloc(spins.data_ptr(), shape, beta, seed, offset, 4, h=h)
    torch.cuda.synchronize()
    chain.advance(4)
    assert np.array_equal(spins.cpu().numpy(), chain.read())
    assert pos1 == chain.stream_position()

    pos2 = _noalloc(spins.data_ptr(), shape, beta, seed, pos1, 3, h=h)
    torch.cuda.synchronize()
    chain.advance(3)
    assert np.array_equal(spins.cpu().numpy(), chain.read())
    assert pos2 == chain.stream_position()


def test_rejects_lattices_beyond_the_scratch_limit(gpu):
    shape = (1024, 1024, 256)  # 2^28 sites > PLQ_NOALLOC_MAX_SITES
    arr = (C.c_int64 * 3)(*shape)
    rc = plq.lib().plq_ising_metropolis_noalloc(C.c_void_p(1), 3, arr, 1.0, 0.0, 0.2, 1, 0, 1, None, None)
    assert rc == plq.PLQ_EINVAL
    assert "no-allocation limit of 134217728 sites" in plq.lib().plq_last_error().decode()


def _chain_result(gpu, shape, beta, seed, offset, start, sweeps, h=0.0):
    d = plq.make_desc(plq.ISING, 2, shape, plq.METROPOLIS, beta=beta, h=h, seed=seed, rng=plq.RNG_STREAM,
                      stream_offset=offset, sweeps_between=1, batch=1)
    chain = plq.GpuChain(gpu, d, start)
    chain.advance(sweeps)
    out = chain.read(), chain.stream_position()
    chain.close()
    return out


def test_earlier_calls_leave_nothing_behind(gpu):
    """Each call starts from whatever the previous call left in the shared
    array: a large lattice, then a small one with another seed and other
    couplings, then the large one again must each equal a fresh chain."""
    import torch

    cases = [((256, 128, 64), 0.2216544, 0.0, 11), ((32, 16), 0.9, 0.2, 12), ((256, 128, 64), 0.2216544, 0.0, 11)]
    for shape, beta, h, seed in cases:
        n = int(np.prod(shape))
        start, offset = plq.hot_start(seed, 2, n)
        spins = torch.from_numpy(start.copy()).cuda()
        pos = _noalloc(spins.data_ptr(), shape, beta, seed, offset, 3, h=h)
        torch.cuda.synchronize()
        want, want_pos = _chain_result(gpu, shape, beta, seed, offset, start, 3, h=h)
        assert np.array_equal(spins.cpu().numpy(), want), shape
        assert pos == want_pos, shape


def test_the_largest_accepted_lattice(gpu):
    """2^27 sites, the array's limit: the last look-back descriptor slot is
    used, and the call still equals the chain API."""
    import torch

    shape, beta, seed = (16384, 8192), 0.4406868, 5
    n = 16384 * 8192
    start, offset = plq.hot_start(seed, 2, n)
    spins = torch.from_numpy(start.copy()).cuda()
    pos = _noalloc(spins.data_ptr(), shape, beta, seed, offset, 1)
    torch.cuda.synchronize()
    want, want_pos = _chain_result(gpu, shape, beta, seed, offset, start, 1)
    assert pos == want_pos
    assert np.array_equal(spins.cpu().numpy(), want)
