"""Per-SV GkmExplain pair loop (gkm_explain_pairs; explain/cpu.py:14-66,
explain/core.py:170-247): against the reference's golden attributions with the
l-mer path switched off, and against the oracle's pair loop at l = 13..15
where no l-mer path exists."""

import warnings

import numpy as np
import pytest

import gkmsvm_lite_b200 as gk
from gkmsvm_lite_b200 import explain as ex
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
RTOL, ATOL = 1e-9, 1e-12
CASES = ["t2", "t2norc", "t0", "t0small", "t1", "t3", "t4", "t5", "t6"]
MODES = [("hypothetical", "explain_hyp"), ("importance", "explain_imp"), ("perturbation", "explain_pert")]


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("mode,key", MODES)
def test_pairs_match_reference_goldens(small, name, mode, key):
    c = small[name]
    m = gk.GkmSVM(c["sv"], c["coef"], float(c["bias"]), c["kernel_type"], c["params"],
                  sv_lengths=c["sv_lengths"]).cuda()
    m.use_lmer_index = False
    m.use_explain_table = False
    assert ex._explain_uses_pairs(m, mode == "perturbation")
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", UserWarning)
        got = gk.gkmexplain(m, c["x"], lengths=c["x_lengths"], mode=mode)
    np.testing.assert_allclose(_np(got), c[key], rtol=RTOL, atol=ATOL)


LONG = [
    ("gkm_esttrunc", {"L": 13, "k": 8, "d": 3}),
    ("gkm_esttrunc", {"L": 15, "k": 10, "d": 4, "include_rc": False}),
    ("wgkm", {"L": 13, "k": 8, "d": 3, "M": 20, "H": 10.0}),
    ("gkmrbf", {"L": 14, "k": 9, "d": 3, "gamma": 1.5}),
    ("wgkmrbf", {"L": 15, "k": 10, "d": 3, "gamma": 0.5}),
    ("gkm_cnt", {"L": 13, "k": 7}),
]


def _long_case(seed, kernel_type, params, S=24):
    rng = np.random.default_rng(seed)
    Ls, B, L = 70, 5, 64
    sv = rng.integers(0, 4, (S, Ls), dtype=np.uint8)
    # plant shared segments so that pairs within the cutoff occur
    motif = rng.integers(0, 4, 20, dtype=np.uint8)
    for s in range(0, S, 3):
        sv[s, 10:30] = motif
    sv_len = rng.integers(params["L"] - 1, Ls + 1, S)
    sv_len[0] = Ls
    x = rng.integers(0, 4, (B, L), dtype=np.uint8)
    x[1, 5:25] = motif
    x[2, 30:50] = motif
    x_len = np.array([L, L - 3, L - 20, params["L"], L])
    coef = rng.standard_normal(S)
    return sv, sv_len, coef, x, x_len


@pytest.mark.parametrize("case", range(len(LONG)))
@pytest.mark.parametrize("mode", ["hypothetical", "perturbation", "importance"])
def test_pairs_long_l_match_oracle(case, mode):
    kernel_type, params = LONG[case]
    sv, sv_len, coef, x, x_len = _long_case(100 + case, kernel_type, params)
    m = gk.GkmSVM(sv, coef, 0.25, kernel_type, params, sv_lengths=sv_len).cuda()
    assert ex._explain_uses_pairs(m, mode == "perturbation")
    got = _np(gk.gkmexplain(m, x, lengths=x_len, mode=mode))
    kd = orc.KernelDef.from_params(kernel_type, params)
    want = orc.gkmexplain(orc.OracleModel(sv, sv_len, coef, 0.25, kd), x, x_len, mode)
    assert np.abs(want).max() > 0
    np.testing.assert_allclose(got, want, rtol=RTOL, atol=1e-12 * np.abs(want).max())


def test_pairs_equal_lmer_path_l11():
    """The two GPU forms of the same attributions agree at l = 11."""
    sv, sv_len, coef, x, x_len = _long_case(7, "gkm_esttrunc", {"L": 11})
    params = {"L": 11, "k": 7, "d": 3}
    m = gk.GkmSVM(sv, coef, 0.0, "gkm_esttrunc", params, sv_lengths=sv_len).cuda()
    m.use_explain_table = False
    assert not ex._explain_uses_pairs(m, False)
    lmer = _np(gk.gkmexplain(m, x, lengths=x_len, mode="hypothetical"))
    m.use_lmer_index = False
    pairs = _np(gk.gkmexplain(m, x, lengths=x_len, mode="hypothetical"))
    np.testing.assert_allclose(pairs, lmer, rtol=1e-12, atol=1e-14 * np.abs(lmer).max())


def test_pairs_deterministic():
    kernel_type, params = LONG[3]
    sv, sv_len, coef, x, x_len = _long_case(11, kernel_type, params)
    m = gk.GkmSVM(sv, coef, 0.0, kernel_type, params, sv_lengths=sv_len).cuda()
    a = _np(gk.gkmexplain(m, x, lengths=x_len, mode="hypothetical"))
    b = _np(gk.gkmexplain(m, x, lengths=x_len, mode="hypothetical", batch_size=2))
    assert np.array_equal(a, b)


@pytest.mark.parametrize("kernel_type,params", [LONG[2], LONG[4]])
def test_pairs_sv_splits_match_oracle(kernel_type, params):
    """130 SVs: the SV range is split across blocks (5 splits)."""
    sv, sv_len, coef, x, x_len = _long_case(23, kernel_type, params, S=130)
    m = gk.GkmSVM(sv, coef, 0.0, kernel_type, params, sv_lengths=sv_len).cuda()
    got = _np(gk.gkmexplain(m, x, lengths=x_len, mode="perturbation"))
    kd = orc.KernelDef.from_params(kernel_type, params)
    want = orc.gkmexplain(orc.OracleModel(sv, sv_len, coef, 0.0, kd), x, x_len, "perturbation")
    np.testing.assert_allclose(got, want, rtol=RTOL, atol=1e-12 * np.abs(want).max())
