"""Size-independent properties at the benchmark sizes (72,000-SV models,
1,000 bp rows), after gkmsvm-lite's own property tests: reverse-complement
invariance (docs/scoring.md:140-151), ISM = f(mutant) - f(x) with the
reference base exactly 0 (tests/test_ism.py:132-140, 218-249), GkmExplain
completeness, sum of importance = f(x) - b (tests/test_explain.py:271-369),
Gram symmetry with unit diagonal (tests/test_gram.py:33-49), and padded =
chunked = per-row scoring (tests/test_variable_length.py:79-137)."""

import numpy as np
import pytest

import gkmsvm_lite_b200 as gk
import gkmsvm_lite_b200.synthetic as syn

pytestmark = pytest.mark.gpu
RTOL = 1e-9


@pytest.fixture(scope="module")
def svs():
    return syn.config3_model()


def _np(t):
    return t.detach().cpu().numpy()


def _acgt_rows(seed, lengths):
    """Ragged rows of A/C/G/T only (an N reads as A on both strands, which
    breaks strand symmetry by design)."""
    rng = np.random.default_rng(seed)
    lengths = np.asarray(lengths, dtype=np.int64)
    x = rng.integers(0, 4, (len(lengths), int(lengths.max())), dtype=np.uint8)
    for i, n in enumerate(lengths):
        x[i, n:] = 0
    return x, lengths


def _revcomp(x, lengths):
    r = np.zeros_like(x)
    for i, n in enumerate(lengths):
        r[i, :n] = 3 - x[i, :n][::-1]
    return r


@pytest.mark.parametrize("kt,params", [("gkm_esttrunc", {"L": 11, "k": 7, "d": 3}),
                                       ("gkmrbf", {"L": 11, "k": 7, "d": 3, "gamma": 2.0})])
def test_reverse_complement_invariance(svs, kt, params):
    sv, svl, coef = svs
    m = gk.GkmSVM(sv, coef, 0.1, kt, params, sv_lengths=svl).cuda()
    x, xl = _acgt_rows(21, np.random.default_rng(5).integers(50, 1500, 96))
    a = _np(m(x, lengths=xl))
    b = _np(m(_revcomp(x, xl), lengths=xl))
    np.testing.assert_allclose(b, a, rtol=RTOL, atol=1e-12)


def test_ism_equals_mutant_scores(svs):
    sv, svl, coef = svs
    m = gk.GkmSVM(sv, coef, 0.0, "gkm_esttrunc", {"L": 11, "k": 7, "d": 3}, sv_lengths=svl).cuda()
    x = syn.config4_queries()[:2]
    ism = _np(gk.ism(m, x))
    assert ism.shape == (2, 4, 1000)
    f0 = _np(m(x))[:, 0]
    rng = np.random.default_rng(8)
    for p in list(rng.integers(0, 1000, 6)) + [0, 999]:
        assert (ism[np.arange(2), x[:, p], p] == 0).all()  # the reference base: exactly 0
        muts = np.repeat(x, 4, axis=0)
        muts[:, p] = np.tile(np.arange(4, dtype=np.uint8), 2)
        want = _np(m(muts))[:, 0].reshape(2, 4) - f0[:, None]
        np.testing.assert_allclose(ism[:, :, p], want, rtol=RTOL, atol=1e-10 * np.abs(ism).max())


@pytest.mark.parametrize("use_table", [True, False])
def test_explain_completeness(svs, use_table):
    """sum over positions and bases of the importance attributions = f(x) - b
    (linear kernel; normalisation folded into the coefficients)."""
    sv, svl, coef = svs
    m = gk.GkmSVM(sv, coef, 0.3, "gkm_esttrunc", {"L": 11, "k": 7, "d": 3}, sv_lengths=svl).cuda()
    m.use_explain_table = use_table
    x = syn.config4_queries()[:4]
    imp = _np(gk.gkmexplain(m, x, mode="importance"))
    f = _np(m(x))[:, 0]
    total = imp.reshape(4, -1).sum(axis=1)
    scale = np.abs(imp).reshape(4, -1).sum(axis=1)
    np.testing.assert_allclose(total, f - 0.3, rtol=0, atol=1e-9 * scale.max() + 1e-12)


def test_gram_symmetric_with_unit_diagonal():
    x, xl = syn.config2(n=400)
    for k in (gk.CenterWeightedGkmKernel(11, 7, d=3), gk.KERNEL_BUILDERS["gkm_esttrunc"]({"L": 11, "k": 7, "d": 3})):
        g = gk.compute_gram(k, x, lengths=xl)
        assert g.shape == (400, 400)
        assert np.array_equal(g, g.T)
        np.testing.assert_allclose(np.diag(g), 1.0, rtol=0, atol=1e-12)
        assert (np.abs(g) <= 1.0 + 1e-12).all()


def test_padded_chunked_and_single_rows_agree(svs):
    sv, svl, coef = svs
    m = gk.GkmSVM(sv, coef, -0.2, "gkmrbf", {"L": 11, "k": 7, "d": 3, "gamma": 2.0}, sv_lengths=svl).cuda()
    x, xl = _acgt_rows(31, np.random.default_rng(6).integers(20, 2000, 40))
    full = _np(m(x, lengths=xl))
    chunked = _np(m(x, lengths=xl, batch_size=7))
    np.testing.assert_allclose(chunked, full, rtol=RTOL, atol=1e-12)
    for i in (0, 13, 39):
        alone = _np(m(x[i:i + 1, : xl[i]]))
        np.testing.assert_allclose(alone, full[i:i + 1], rtol=RTOL, atol=1e-12)
