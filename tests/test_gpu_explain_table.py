"""GPU explain table (explain/table.py of gkmsvm-lite): attributions read from
the [4^l, 4, l] table built by Walsh-Hadamard transforms equal the direct
l-mer path's (the reference's own check, tests/test_explain.py:609-634, at
rtol 1e-12); the "auto" rule builds it only for calls large enough to pay for
it, caches it per mode, and RBF models never get one."""

import numpy as np
import pytest
import torch

import gkmsvm_lite_b200 as gk

pytestmark = pytest.mark.gpu


def _model(kt, params, n_sv=40, L_sv=30, seed=9):
    rng = np.random.default_rng(seed)
    sv = rng.integers(0, 4, (n_sv, L_sv)).astype(np.uint8)
    return gk.GkmSVM(sv, rng.normal(size=n_sv), 0.2, kt, params).cuda(), rng


@pytest.mark.parametrize("mode", ["hypothetical", "perturbation", "importance"])
@pytest.mark.parametrize("kt,params", [
    ("gkm_esttrunc", {"L": 8, "k": 5, "d": 2}),
    ("gkm_esttrunc", {"L": 8, "k": 5, "d": 2, "include_rc": False}),
    ("gkm_estfull", {"L": 7, "k": 4, "d": 3}),
    ("gkm_cnt", {"L": 7, "k": 4}),
    ("wgkm", {"L": 8, "k": 5, "d": 2, "M": 20, "H": 5.0}),
])
def test_explain_table_matches_lmer_path(kt, params, mode):
    m, rng = _model(kt, params)
    x = rng.integers(0, 4, (4, 33)).astype(np.uint8)
    xl = np.array([33, 20, 8, 12])
    m.use_explain_table = False
    ref = gk.gkmexplain(m, x, lengths=xl, mode=mode).cpu().numpy()
    m.use_explain_table = True
    got = gk.gkmexplain(m, x, lengths=xl, mode=mode).cpu().numpy()
    assert m._explain_tables
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-14, equal_nan=True)


def test_explain_table_l11():
    """At l = 11 (4^11 l-mers) the transforms' rounding stays far inside the
    path's 1e-9 tolerance."""
    m, rng = _model("gkm_esttrunc", {"L": 11, "k": 7, "d": 3}, n_sv=300, L_sv=300, seed=4)
    x = rng.integers(0, 4, (6, 500)).astype(np.uint8)
    for mode in ("hypothetical", "perturbation"):
        m.use_explain_table = False
        ref = gk.gkmexplain(m, x, mode=mode).cpu().numpy()
        m.use_explain_table = True
        got = gk.gkmexplain(m, x, mode=mode).cpu().numpy()
        np.testing.assert_allclose(got, ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())
    m.clear_caches()
    assert m._explain_tables == {}


def test_explain_table_auto_and_caching(monkeypatch):
    from gkmsvm_lite_b200 import explain as ex

    m, rng = _model("gkm_esttrunc", {"L": 8, "k": 5, "d": 2}, n_sv=20)
    x = rng.integers(0, 4, (40, 30)).astype(np.uint8)
    # a table of 4^8 x 8 entries pays off after this many windows
    need = ex._TABLE_BUILD_S_PER_ENTRY * 4 ** 8 * 8 / ex._DIRECT_S_PER_WINDOW
    assert 2 * 23 < need < 40 * 23 * 10
    monkeypatch.setattr(ex, "_DIRECT_S_PER_WINDOW", ex._TABLE_BUILD_S_PER_ENTRY * 4 ** 8 * 8 / 100)
    gk.gkmexplain(m, x[:2], mode="hypothetical")  # 46 windows: direct
    assert m._explain_tables == {}
    full = gk.gkmexplain(m, x, mode="hypothetical").cpu().numpy()  # 920 windows: table
    assert list(m._explain_tables) == [False]
    again = gk.gkmexplain(m, x[:2], mode="hypothetical").cpu().numpy()  # cached table
    np.testing.assert_allclose(again, full[:2], rtol=1e-12, atol=1e-14)
    m.clear_caches()
    assert m._explain_tables == {}
    rbf, _ = _model("gkmrbf", {"L": 8, "k": 5, "d": 2, "gamma": 1.5}, n_sv=20)
    rbf.use_explain_table = True
    gk.gkmexplain(rbf, x, mode="hypothetical")
    assert rbf._explain_tables == {}
