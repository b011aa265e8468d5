"""The host SMO solver (gkm_smo_solve, C ABI) against LIBSVM's (sklearn SVC /
SVR on a precomputed kernel): same dual coefficients and bias on the same
kernel matrix, for C-SVC (with class weights) and epsilon-SVR, whatever the
column-cache size and prefetch.  Columns come from a NumPy kernel through the
callback, so no GPU is needed."""

import ctypes

import numpy as np
import pytest

from gkmsvm_lite_b200 import _lib


def _kernel(N, seed):
    rng = np.random.default_rng(seed)
    Z = rng.normal(size=(N, 5))
    d2 = ((Z[:, None, :] - Z[None, :, :]) ** 2).sum(-1)
    K = np.exp(-0.3 * d2)  # PSD, unit diagonal (a normalised kernel)
    return K, rng


def _smo(K, y, p, C, tol=1e-8, cache=None, prefetch=16, fail_after=None):
    N = K.shape[0]
    n = y.shape[0]
    calls = []

    def provider(count, idx_ptr, out_ptr, ctx):
        idx = np.ctypeslib.as_array(idx_ptr, shape=(count,)).copy()
        calls.append(len(idx))
        if fail_after is not None and len(calls) > fail_after:
            return 1
        out = np.ctypeslib.as_array(out_ptr, shape=(count * N,))
        out[:] = np.ascontiguousarray(K[:, idx].T).ravel()
        return 0

    cb = _lib.COLUMNS_CB(provider)
    y = np.ascontiguousarray(y, dtype=np.float64)
    p = np.ascontiguousarray(p, dtype=np.float64)
    diag = np.ascontiguousarray(np.diag(K))
    coef = np.zeros(n)
    bias = ctypes.c_double()
    iters = ctypes.c_int64()
    st = _lib.load().gkm_smo_solve(n, N, y.ctypes.data, p.ctypes.data, diag.ctypes.data, float(C[0]), float(C[1]),
                                   tol, 10_000_000, cache or N, prefetch, cb, None, coef.ctypes.data,
                                   ctypes.byref(bias), ctypes.byref(iters), 0)
    _lib.check(st, "gkm_smo_solve")
    return coef, bias.value, calls


@pytest.mark.parametrize("cache,prefetch", [(None, 16), (3, 1), (7, 4), (2, 256)])
def test_csvc_equals_libsvm(cache, prefetch):
    from sklearn.svm import SVC

    K, rng = _kernel(70, 1)
    y = np.where(rng.random(70) < 0.45, 1.0, -1.0)
    coef, bias, _ = _smo(K, y, -np.ones(70), (2.0, 1.0), cache=cache, prefetch=prefetch)
    ref = SVC(C=1.0, kernel="precomputed", tol=1e-8, class_weight={1: 2.0, -1: 1.0}).fit(K, y)
    want = np.zeros(70)
    want[ref.support_] = ref.dual_coef_[0]
    scale = np.abs(want).max()
    np.testing.assert_allclose(coef, want, atol=1e-5 * scale)
    np.testing.assert_allclose(bias, ref.intercept_[0], atol=1e-5)
    np.testing.assert_allclose(K @ coef + bias, ref.decision_function(K), atol=1e-5)


def test_svr_equals_libsvm():
    from sklearn.svm import SVR

    K, rng = _kernel(60, 2)
    z = rng.normal(size=60)
    N = 60
    signs = np.r_[np.ones(N), -np.ones(N)]
    coef, bias, _ = _smo(K, signs, np.r_[0.1 - z, 0.1 + z], (1.5, 1.5), cache=9, prefetch=8)
    coef = coef[:N] + coef[N:]
    ref = SVR(C=1.5, epsilon=0.1, kernel="precomputed", tol=1e-8).fit(K, z)
    want = np.zeros(N)
    want[ref.support_] = ref.dual_coef_[0]
    np.testing.assert_allclose(coef, want, atol=1e-5 * np.abs(want).max())
    np.testing.assert_allclose(K @ coef + bias, ref.predict(K), atol=1e-5)


def test_prefetch_batches_columns_and_provider_failure_stops():
    K, rng = _kernel(50, 3)
    y = np.where(rng.random(50) < 0.5, 1.0, -1.0)
    _, _, calls = _smo(K, y, -np.ones(50), (1.0, 1.0), cache=50, prefetch=32)
    assert max(calls) > 1  # a miss fetched likely next columns with it
    with pytest.raises(ValueError, match="column provider"):
        _smo(K, y, -np.ones(50), (1.0, 1.0), cache=4, prefetch=1, fail_after=2)


def test_shrinking_large_problems_equal_libsvm():
    """1,500 sequences (C-SVC) and 700 (SVR, 1,400 dual variables): many
    shrink rounds, the rebuild at 10 tol and the final full check."""
    from sklearn.svm import SVC, SVR

    K, rng = _kernel(1500, 3)
    y = np.where(rng.random(1500) < 0.5, 1.0, -1.0)
    y[rng.random(1500) < 0.1] *= -1  # label noise: bounded and free variables both
    coef, bias, _ = _smo(K, y, -np.ones(1500), (1.0, 1.0), tol=1e-6, cache=400, prefetch=32)
    ref = SVC(C=1.0, kernel="precomputed", tol=1e-6).fit(K, y)
    np.testing.assert_allclose(K @ coef + bias, ref.decision_function(K), atol=2e-4)
    want = np.zeros(1500)
    want[ref.support_] = ref.dual_coef_[0]
    assert np.abs(coef - want).max() < 1e-3
    K2, rng = _kernel(700, 4)
    z = np.sin(np.arange(700) / 30.0) + 0.1 * rng.normal(size=700)
    signs = np.r_[np.ones(700), -np.ones(700)]
    coef, bias, _ = _smo(K2, signs, np.r_[0.05 - z, 0.05 + z], (2.0, 2.0), tol=1e-6, cache=200, prefetch=16)
    ref = SVR(C=2.0, epsilon=0.05, kernel="precomputed", tol=1e-6).fit(K2, z)
    np.testing.assert_allclose(K2 @ (coef[:700] + coef[700:]) + bias, ref.predict(K2), atol=2e-4)
