"""GPU parity of the l-mer index query's row splits: a batch too small to fill
the GPU (rows x SV tiles items) has each row's windows cut into ranges whose
exact per-(SV, level) counts are summed on the device.  Profiles must stay
bit-exact against the oracle, and scores must match the same rows scored in a
batch large enough to need no split."""

import numpy as np
import pytest
import torch

from oracle import oracle as orc

import gkmsvm_lite_b200 as gk
from gkmsvm_lite_b200 import engine

pytestmark = pytest.mark.gpu
RTOL, ATOL = 1e-12, 1e-12


def _rows(rng, n, L, lengths=None):
    x = rng.integers(0, 4, size=(n, L), dtype=np.uint8)
    if lengths is not None:
        for i, m in enumerate(lengths):
            x[i, m:] = 0
    return x


@pytest.mark.parametrize("kt,params", [("gkm_esttrunc", dict(L=11, k=7, d=3)),
                                       ("wgkmrbf", dict(L=10, k=6, d=3, gamma=1.5, M=40, H=20.0))])
def test_split_profiles_bit_exact(kt, params):
    rng = np.random.default_rng(11)
    sv = _rows(rng, 150, 300)
    x = _rows(rng, 3, 1500, [1500, 900, 64])
    xl = np.array([1500, 900, 64])
    m = gk.GkmSVM(sv, np.linspace(-1, 1, 150), 0.0, kt, params).cuda()
    ix = m._sv_index()
    assert ix is not None
    spec = m._spec()
    fwd, _, counts = engine.pack(spec, torch.from_numpy(x).cuda(), xl)
    raw, prof = ix.pairwise(fwd, counts, profile=True)  # 3 rows x 1 tile: split
    kd = orc.KernelDef.from_params(kt, params)
    want = orc.profiles(x, xl, sv, None, kd)
    d = kd.dmax
    np.testing.assert_array_equal(prof.cpu().numpy()[..., : d + 1].astype(np.uint64), want[..., : d + 1])
    jraw, _ = engine.join_pairwise(spec, fwd, counts, *m._sv_packed())
    np.testing.assert_array_equal(raw.cpu().numpy(), jraw.cpu().numpy())


@pytest.mark.parametrize("kt,params", [("gkmrbf", dict(L=11, k=7, d=3, gamma=2.0)),
                                       ("wgkm", dict(L=11, k=7, d=3)),
                                       ("gkm_esttrunc", dict(L=11, k=7, d=3))])
def test_split_scores_equal_unsplit(kt, params):
    rng = np.random.default_rng(12)
    sv = _rows(rng, 400, 250)
    small = _rows(rng, 2, 2000, [2000, 700])
    sl = np.array([2000, 700])
    m = gk.GkmSVM(sv, rng.normal(0, 0.1, 400), 0.3, kt, params).cuda()
    m.use_lmer_table = False
    got = m(small, lengths=sl).cpu().numpy()[:, 0]  # 2 rows: split
    # the same rows among 1,022 others: enough items, no split
    big = np.zeros((1024, 2000), np.uint8)
    bl = np.full(1024, 150)
    big[:, :150] = _rows(rng, 1024, 150)
    big[:2] = small
    bl[:2] = sl
    want = m(big, lengths=bl).cpu().numpy()[:2, 0]
    np.testing.assert_allclose(got, want, rtol=RTOL, atol=ATOL)
