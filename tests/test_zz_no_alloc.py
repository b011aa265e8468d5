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


def _setup():
    import gkmsvm_lite_b200 as gk
    import gkmsvm_lite_b200.synthetic as syn
    from gkmsvm_lite_b200 import engine

    rng = np.random.default_rng(21)
    sv = syn.random_codes(rng, 300, 200)
    coef = rng.normal(size=300)
    m = gk.GkmSVM(sv, coef, 0.25, "gkmrbf", {"L": 11, "k": 7, "d": 3, "gamma": 2.0}).cuda()
    m.use_lmer_table = False
    index = m._sv_index()
    x = syn.random_codes(rng, 96, 260)
    lengths = rng.integers(40, 261, 96)
    fwd, rc, counts = engine.pack(m._spec(), torch.from_numpy(x).cuda(), lengths)
    dx = engine.self_kernel(m._spec(), fwd, rc, counts)
    inv_dx = 1.0 / torch.sqrt(torch.clamp(dx, min=1e-20))
    return m, index, fwd, counts, inv_dx


def _noalloc(m, index, fwd, counts, inv_dx):
    from gkmsvm_lite_b200 import _lib

    out = torch.full((fwd.shape[0],), float("nan"), dtype=torch.float64, device=fwd.device)
    lib = _lib.load()
    st = lib.gkm_index_score_noalloc(index.handle, fwd.data_ptr(), counts.data_ptr(), fwd.shape[0],
                                     fwd.shape[1], inv_dx.data_ptr(), m._inv_ds().data_ptr(),
                                     m._sv_coef().data_ptr(), 2.0, 1, 0.25, None, out.data_ptr(),
                                     _lib.stream_handle())
    _lib.check(st, "gkm_index_score_noalloc")
    return out


def test_noalloc_scores_equal_allocating_entry_point_twice():
    m, index, fwd, counts, inv_dx = _setup()
    for rows in (slice(0, 96), slice(10, 50)):
        f, c, d = fwd[rows].contiguous(), counts[rows].contiguous(), inv_dx[rows].contiguous()
        want = index.score(f, c, d, m._inv_ds(), m._sv_coef(), 2.0, 1, 0.25)
        got = _noalloc(m, index, f, c, d)
        torch.cuda.synchronize()
        np.testing.assert_allclose(got.cpu().numpy(), want.cpu().numpy(), rtol=RTOL, atol=ATOL)


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
