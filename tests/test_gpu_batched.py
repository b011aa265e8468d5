"""Bucketed, graph-captured ISM and GkmExplain (batch.BatchedIsm,
batch.BatchedExplain): results equal gkmsvm_lite_b200.ism / gkmexplain on
ragged batches, through the index path (RBF model: mutant window sets over the
persistent index query) and the l-mer table path, on first (captured) and
later (replayed) calls, with batches that share a bucket and ones that do
not."""

import numpy as np
import pytest
import torch

import gkmsvm_lite_b200 as gk
import gkmsvm_lite_b200.synthetic as syn
from gkmsvm_lite_b200.batch import BatchedExplain, BatchedIsm

pytestmark = pytest.mark.gpu
RTOL, ATOL = 1e-9, 1e-12


def _model(kt, params, seed=5, n_sv=300):
    rng = np.random.default_rng(seed)
    lengths = rng.integers(60, 200, n_sv)
    sv = syn.ragged_codes(rng, lengths)
    return gk.GkmSVM(sv, rng.normal(0, 0.3, n_sv), 0.1, kt, params, sv_lengths=lengths).cuda()


def _batches(seed=9):
    rng = np.random.default_rng(seed)
    out = []
    for n, lo, hi in ((5, 11, 120), (3, 90, 250), (6, 11, 120)):
        ln = rng.integers(lo, hi, n)
        ln[0] = max(ln[0], 30)
        out.append((syn.ragged_codes(rng, ln), ln))
    return out


def _close(got, want):
    got, want = got.cpu().numpy(), want.cpu().numpy()
    np.testing.assert_allclose(got, want, rtol=RTOL, atol=ATOL * max(1.0, np.abs(want).max()))


@pytest.mark.parametrize("kind", ["wgkmrbf", "gkm_esttrunc"])
def test_batched_ism_equals_ism(kind):
    params = {"L": 11, "k": 7, "d": 3, "gamma": 1.0} if kind == "wgkmrbf" else {"L": 11, "k": 7, "d": 3}
    m = _model(kind, params)
    if kind == "gkm_esttrunc":
        m.use_lmer_table = True
    runner = BatchedIsm(m)
    for x, ln in _batches():
        want = gk.ism(m, x, lengths=ln)
        got = runner(torch.from_numpy(x).cuda(), torch.from_numpy(ln).cuda())
        _close(got, want)
    assert len(runner._graphs) == 2  # the 1st and 3rd batches share a bucket


@pytest.mark.parametrize("mode", ["hypothetical", "importance", "perturbation"])
def test_batched_explain_equals_gkmexplain(mode):
    for kind, params in (("wgkmrbf", {"L": 10, "k": 6, "d": 3, "gamma": 1.0}),
                         ("gkm_esttrunc", {"L": 10, "k": 6, "d": 3})):
        m = _model(kind, params, seed=7)
        runner = BatchedExplain(m, mode)
        for x, ln in _batches(11):
            want = gk.gkmexplain(m, x, lengths=ln, mode=mode)
            got = runner(torch.from_numpy(x).cuda(), torch.from_numpy(ln).cuda())
            _close(got, want)
