"""to_deltasvm weights (svm.py:664-785) on the GPU: the table route
(gkm_deltasvm_table) and the kernel route (every canonical l-mer scored)
against gkmsvm-lite's own weights (tests/golden/deltasvm.npz) and the oracle."""

import os

import numpy as np
import pytest
import torch

import gkmsvm_lite_b200 as gk
from conftest import GOLDEN
from gkmsvm_lite_b200 import deltasvm as dsv
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
RTOL = 1e-9
CASES = ["t2", "t2norc", "t0", "t0small", "t1", "t3", "t4", "t5", "t6"]


@pytest.fixture(scope="module")
def golden():
    z = np.load(os.path.join(GOLDEN, "deltasvm.npz"))
    return {k: z[k] for k in z.files}


def _model(c):
    return gk.GkmSVM(c["sv"], c["coef"], float(c["bias"]), c["kernel_type"], c["params"],
                     sv_lengths=c["sv_lengths"]).cuda()


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("key,qn", [("w", False), ("wq", True)])
def test_weights_match_reference(small, golden, name, key, qn):
    c = small[name]
    d = _model(c).to_deltasvm(query_norm=qn)
    assert (d.l, d.k, d.include_rc, d.bias) == (c["params"]["L"], c["params"]["L"], False, float(c["bias"]))
    w = d.weights
    assert isinstance(w, np.ndarray) and w.shape == (4 ** d.l,)
    want = golden[f"{name}/{key}"]
    scale = max(1.0, np.abs(want).max())
    np.testing.assert_allclose(w[golden[f"{name}/idx"]], want, rtol=RTOL, atol=1e-12 * scale)
    # every weight, through the sum
    np.testing.assert_allclose(w.sum(), golden[f"{name}/{key}_sum"], rtol=1e-8, atol=1e-12 * scale * w.size)


@pytest.mark.parametrize("name", ["t2", "t4", "t1"])
def test_table_route_equals_kernel_route(small, name):
    m = _model(small[name])
    assert m._build_lmer_table() is not None
    for qn in (False, True):
        table = dsv.deltasvm_weights(m, query_norm=qn)
        kern = dsv._weights_from_kernel(m, qn, False)
        scale = float(table.abs().max())
        torch.testing.assert_close(kern, table, rtol=1e-9, atol=1e-12 * scale)


def test_long_l_kernel_route_matches_oracle():
    """l = 13: no l-mer table, no index; every canonical l-mer goes through the
    pairwise forms."""
    rng = np.random.default_rng(3)
    sv = rng.integers(0, 4, (6, 40), dtype=np.uint8)
    coef = rng.standard_normal(6)
    params = {"L": 13, "k": 8, "d": 3}
    m = gk.GkmSVM(sv, coef, 0.3, "gkm_esttrunc", params).cuda()
    assert m._build_lmer_table() is None
    w = m.to_deltasvm(device="cuda").weights
    assert isinstance(w, torch.Tensor) and w.shape == (4 ** 13,)
    idx = np.sort(rng.choice(4 ** 13, 2048, replace=False))
    # l-mers near the SVs' own windows carry the large weights
    idx = np.unique(np.r_[idx, [int("".join(map(str, sv[s, i:i + 13])), 4) for s in range(6) for i in (0, 9, 27)]])
    want = orc.deltasvm_weights(orc.OracleModel(sv, None, coef, 0.3, orc.KernelDef.from_params("gkm_esttrunc", params)),
                                False, idx)
    got = w[torch.as_tensor(idx, device=w.device)].cpu().numpy()
    assert np.abs(want).max() > 0
    np.testing.assert_allclose(got, want, rtol=RTOL, atol=1e-12 * np.abs(want).max())


def test_too_long_l_raises():
    rng = np.random.default_rng(0)
    m = gk.GkmSVM(rng.integers(0, 4, (2, 30), dtype=np.uint8), np.ones(2), 0.0, "gkm_esttrunc",
                  {"L": 15, "k": 8, "d": 3}).cuda()
    with pytest.raises(ValueError, match="l <= 14"):
        m.to_deltasvm()
