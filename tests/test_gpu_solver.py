"""SMO training on the GPU column provider (solver.py of gkmsvm-lite): the
columns equal compute_gram's (index path and pairwise path), and smo_solve /
smo_svr_solve give LIBSVM's solution (sklearn on the same Gram matrix)."""

import numpy as np
import pytest

import gkmsvm_lite_b200 as gk
import gkmsvm_lite_b200.synthetic as syn

pytestmark = pytest.mark.gpu


def _data(n, seed):
    rng = np.random.default_rng(seed)
    lengths = syn.log_uniform_lengths(rng, n, 60, 300)
    return syn.ragged_codes(rng, lengths), lengths, rng


@pytest.mark.parametrize("kernel,uses_index", [
    (gk.CenterWeightedGkmKernel(11, 7, d=3), True),
    (gk.RbfGkmKernel(10, 6, d=3, gamma=2.0), True),
    (gk.DirectGkmKernel(11, 4), False),  # dmax 7: the index does not apply
])
def test_columns_equal_gram(kernel, uses_index):
    X, lengths, _ = _data(48, 1)
    gram = gk.compute_gram(kernel, X, lengths=lengths)
    cache = gk.KernelColumnCache(kernel, X, lengths)
    assert (cache.index is not None) == uses_index
    idx = [0, 5, 47, 5, 13]
    cols = cache.compute_columns(idx)
    for i in idx:
        np.testing.assert_allclose(cols[i], gram[:, i], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(cache.finished_diagonal(), np.diag(gram), rtol=1e-12)
    cache.close()


def test_smo_solve_equals_libsvm():
    from sklearn.svm import SVC, SVR

    X, lengths, rng = _data(80, 2)
    kernel = gk.RbfGkmKernel(10, 6, d=3, gamma=1.0)
    K = gk.compute_gram(kernel, X, lengths=lengths)
    y = np.where(rng.random(80) < 0.5, 1.0, -1.0)
    coef, bias = gk.smo_solve(kernel, X, y, C=1.0, tol=1e-8, lengths=lengths, cache_size=16)
    ref = SVC(C=1.0, kernel="precomputed", tol=1e-8).fit(K, y)
    np.testing.assert_allclose(K @ coef + bias, ref.decision_function(K), atol=1e-5)
    z = rng.normal(size=80)
    coef, bias = gk.smo_svr_solve(kernel, X, z, C=1.0, epsilon=0.1, tol=1e-8, lengths=lengths)
    ref = SVR(C=1.0, epsilon=0.1, kernel="precomputed", tol=1e-8).fit(K, z)
    np.testing.assert_allclose(K @ coef + bias, ref.predict(K), atol=1e-5)
