"""Serving on the GPU: mixed predict / score_variants / ISM / GkmExplain
requests submitted concurrently give the same results as each call run alone
(rtol 1e-9, atol 1e-12)."""

import threading

import numpy as np
import pytest
import torch

import gkmsvm_lite_b200 as gk
import gkmsvm_lite_b200.synthetic as syn
from gkmsvm_lite_b200.serve import GkmServer, GpuBackend

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kt", ["wgkmrbf", "gkm_esttrunc"])
def test_results_same_alone_and_in_the_mix(kt):
    rng = np.random.default_rng(31)
    lens = rng.integers(150, 400, 250)
    sv = syn.ragged_codes(rng, lens)
    m = gk.GkmSVM(sv, rng.normal(size=250), 0.1, kt, {"L": 11, "k": 7, "d": 3, "gamma": 1.0},
                  sv_lengths=lens).cuda()
    m.use_lmer_table = False
    reqs = []
    for i in range(48):
        kind = ["predict", "predict", "score_variants", "ism", "explain"][i % 5]
        n = 1 if kind in ("ism", "explain") else int(rng.integers(1, 6))
        ql = syn.log_uniform_lengths(rng, n, 20, 600)
        ql[0] = max(ql[0], 12)
        x = syn.ragged_codes(rng, ql)
        req = {"kind": kind, "x": x, "lengths": ql}
        if kind == "score_variants":
            alt, al = syn.variant_pairs(rng, x, ql)
            req.update(alt=alt, alt_lengths=al)
        reqs.append(req)
    solo = []
    for r in reqs:
        if r["kind"] == "predict":
            solo.append(m(r["x"], lengths=r["lengths"]).cpu().numpy())
        elif r["kind"] == "score_variants":
            solo.append(m.score_variants(r["x"], r["alt"], ref_lengths=r["lengths"],
                                         alt_lengths=r["alt_lengths"]).cpu().numpy())
        elif r["kind"] == "ism":
            solo.append(gk.ism(m, r["x"], lengths=r["lengths"]).cpu().numpy())
        else:
            solo.append(gk.gkmexplain(m, r["x"], lengths=r["lengths"], mode="hypothetical").cpu().numpy())
    torch.cuda.synchronize()
    futs = [None] * len(reqs)
    with GkmServer(GpuBackend(m), max_batch_rows=64) as srv:
        def client(k):
            for i in range(k, len(reqs), 4):
                r = reqs[i]
                futs[i] = srv.submit(r["kind"], r["x"], lengths=r["lengths"], alt=r.get("alt"),
                                     alt_lengths=r.get("alt_lengths"))
        ts = [threading.Thread(target=client, args=(k,)) for k in range(4)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        got = [f.result(120) for f in futs]
        st = srv.stats()
    for r, a, b in zip(reqs, got, solo):
        np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-12, err_msg=r["kind"])
    assert st["all"]["n"] == len(reqs) and st["admitted"] > 0


@pytest.mark.parametrize("kt", ["gkmrbf", "wgkmrbf", "gkm_esttrunc"])
def test_direct_scorer_equals_model(kt):
    """Small serving batches skip the graphs: the same scores as model(x),
    also when a poly-A row's 16-bit carries force the exact rerun."""
    from gkmsvm_lite_b200.batch import DirectScorer

    rng = np.random.default_rng(21)
    sv = np.concatenate([np.zeros((6, 300), np.uint8), rng.integers(0, 4, (60, 300)).astype(np.uint8)])
    m = gk.GkmSVM(sv, rng.normal(0, 0.1, 66), 0.1, kt, {"L": 11, "k": 7, "d": 3, "gamma": 1.0}).cuda()
    m.use_lmer_table = False
    x = np.concatenate([np.zeros((1, 2000), np.uint8), rng.integers(0, 4, (3, 2000)).astype(np.uint8)])
    lengths = np.array([2000, 1500, 700, 11])
    want = m(x, lengths=lengths).cpu().numpy()[:, 0]
    ds = DirectScorer(m)
    got = ds.score(torch.from_numpy(x).cuda(), torch.from_numpy(lengths).cuda(), check=False)
    ds.check_flags()
    np.testing.assert_allclose(got.cpu().numpy(), want, rtol=1e-12, atol=1e-14)
