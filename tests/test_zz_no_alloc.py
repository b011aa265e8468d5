"""gkm_index_score_noalloc through the C ABI: the scores of a caller that
cannot allocate device memory while scoring must equal gkm_index_score's.

The fixed scratch array is shared by every call and keeps the previous call's
contents, so the check runs two calls in a row (different rows) and compares
both.  This file is collected last: run alone or after the other tests, a
failure here leaves every other test already run.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-9, 1e-12


def _setup(tile_svs=0):
    import gkmsvm_lite_b200 as gk
    import gkmsvm_lite_b200.synthetic as syn
    from gkmsvm_lite_b200 import engine

    rng = np.random.default_rng(21)
    sv = syn.random_codes(rng, 300, 200)
    coef = rng.normal(size=300)
    m = gk.GkmSVM(sv, coef, 0.25, "gkmrbf", {"L": 11, "k": 7, "d": 3, "gamma": 2.0}).cuda()
    m.use_lmer_table = False
    if tile_svs:
        index = engine.DeviceIndex(m._spec(), *m._sv_packed(), m._masks(), tile_svs=tile_svs)
    else:
        index = m._sv_index()
    x = syn.random_codes(rng, 96, 260)
    lengths = rng.integers(40, 261, 96)
    fwd, rc, counts = engine.pack(m._spec(), torch.from_numpy(x).cuda(), lengths)
    dx = engine.self_kernel(m._spec(), fwd, rc, counts)
    inv_dx = 1.0 / torch.sqrt(torch.clamp(dx, min=1e-20))
    return m, index, fwd, counts, inv_dx


def _noalloc(m, index, fwd, counts, inv_dx, order=None, out=None):
    from gkmsvm_lite_b200 import _lib

    if out is None:
        out = torch.full((fwd.shape[0],), float("nan"), dtype=torch.float64, device=fwd.device)
    lib = _lib.load()
    st = lib.gkm_index_score_noalloc(index.handle, fwd.data_ptr(), counts.data_ptr(), fwd.shape[0],
                                     fwd.shape[1], inv_dx.data_ptr(), m._inv_ds().data_ptr(),
                                     m._sv_coef().data_ptr(), 2.0, 1, 0.25,
                                     None if order is None else order.data_ptr(), out.data_ptr(),
                                     _lib.stream_handle())
    _lib.check(st, "gkm_index_score_noalloc")
    return out


class _StreamPool:
    """The current device's stream-ordered memory pool (the one cudaMallocAsync
    draws on), through the driver API: its used / reserved high-water marks."""

    USED_HIGH, USED_CURRENT, RESERVED_HIGH, RESERVED_CURRENT = 8, 7, 6, 5

    def __init__(self):
        self.cu = ctypes.CDLL("libcuda.so.1")
        dev = ctypes.c_int()
        assert self.cu.cuDeviceGet(ctypes.byref(dev), torch.cuda.current_device()) == 0
        self.pool = ctypes.c_void_p()
        assert self.cu.cuDeviceGetMemPool(ctypes.byref(self.pool), dev) == 0

    def get(self, attr) -> int:
        v = ctypes.c_uint64()
        assert self.cu.cuMemPoolGetAttribute(self.pool, attr, ctypes.byref(v)) == 0
        return v.value

    def reset_highs(self):
        # setting a high-water mark to 0 resets it to the current value
        z = ctypes.c_uint64(0)
        for attr in (self.USED_HIGH, self.RESERVED_HIGH):
            assert self.cu.cuMemPoolSetAttribute(self.pool, attr, ctypes.byref(z)) == 0


def test_noalloc_scores_equal_allocating_entry_point_twice():
    m, index, fwd, counts, inv_dx = _setup()
    for rows in (slice(0, 96), slice(10, 50)):
        f, c, d = fwd[rows].contiguous(), counts[rows].contiguous(), inv_dx[rows].contiguous()
        want = index.score(f, c, d, m._inv_ds(), m._sv_coef(), 2.0, 1, 0.25)
        got = _noalloc(m, index, f, c, d)
        torch.cuda.synchronize()
        np.testing.assert_allclose(got.cpu().numpy(), want.cpu().numpy(), rtol=RTOL, atol=ATOL)


def test_noalloc_many_tiles_and_row_order():
    """Small SV tiles (several (row, tile) partials per row in the scratch) and
    a permuted hand-out order, two calls in a row."""
    m, index, fwd, counts, inv_dx = _setup(tile_svs=64)
    assert index.tiles >= 5
    rng = np.random.default_rng(5)
    for rows in (slice(0, 96), slice(7, 70)):
        f, c, d = fwd[rows].contiguous(), counts[rows].contiguous(), inv_dx[rows].contiguous()
        order = torch.from_numpy(rng.permutation(f.shape[0]).astype(np.int32)).cuda()
        want = index.score(f, c, d, m._inv_ds(), m._sv_coef(), 2.0, 1, 0.25)
        got = _noalloc(m, index, f, c, d, order=order)
        torch.cuda.synchronize()
        np.testing.assert_allclose(got.cpu().numpy(), want.cpu().numpy(), rtol=RTOL, atol=ATOL)
    index.close()


def test_noalloc_makes_no_device_allocation():
    """After its first call on the device, a call takes nothing from the
    stream-ordered pool or from torch's caching allocator."""
    m, index, fwd, counts, inv_dx = _setup()
    out = torch.empty(fwd.shape[0], dtype=torch.float64, device=fwd.device)
    _noalloc(m, index, fwd, counts, inv_dx, out=out)
    torch.cuda.synchronize()
    pool = _StreamPool()
    pool.reset_highs()
    torch.cuda.reset_peak_memory_stats()
    used0, res0 = pool.get(pool.USED_CURRENT), pool.get(pool.RESERVED_CURRENT)
    torch_before = torch.cuda.memory_allocated()
    _noalloc(m, index, fwd, counts, inv_dx, out=out)
    torch.cuda.synchronize()
    assert pool.get(pool.USED_HIGH) == used0
    assert pool.get(pool.RESERVED_HIGH) == res0
    assert torch.cuda.max_memory_allocated() == torch_before


def test_noalloc_rejects_rows_beyond_its_scratch():
    from gkmsvm_lite_b200 import _lib

    m, index, fwd, counts, inv_dx = _setup()
    lib = _lib.load()
    too_many = (1 << 19) // index.tiles + 1
    st = lib.gkm_index_score_noalloc(index.handle, fwd.data_ptr(), counts.data_ptr(), too_many,
                                     fwd.shape[1], inv_dx.data_ptr(), m._inv_ds().data_ptr(),
                                     m._sv_coef().data_ptr(), 2.0, 1, 0.25, None, inv_dx.data_ptr(),
                                     _lib.stream_handle())
    assert st == _lib.GKM_ERR_CAPACITY
    assert b"exceed its fixed scratch" in lib.gkm_last_error()
