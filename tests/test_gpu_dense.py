"""GPU parity of the tensor-core pairwise kernel (gkm_dense_pairwise): mismatch
profiles bit-exact against the oracle, and K_raw bit-identical to the warp
join, on shapes that cross its tile edges -- query rows over several 128-window
tiles and over several 1,024-window staged segments, column sets over many
128-window tiles, SV counts that are not a multiple of its 16-SV chunk, rows
without windows, l from 1 to 15 and dmax up to
l - 1, weighted and unweighted, with and without reverse complements."""

import numpy as np
import pytest
import torch

from oracle import oracle as orc

import gkmsvm_lite_b200 as gk
from gkmsvm_lite_b200 import engine
from gkmsvm_lite_b200._lib import GkmError

pytestmark = pytest.mark.gpu

# (kernel type, params, query lengths, SV lengths)
CASES = {
    "esttrunc_l11_long": ("gkm_esttrunc", dict(L=11, k=7, d=3), [300, 11, 5, 129, 140],
                          [40, 300, 77, 11, 10, 180, 95, 60, 250, 33, 12, 200, 64]),
    "cnt_l15_d14": ("gkm_cnt", dict(L=15, k=1, d=14), [64, 200, 15], [15, 90, 150, 16, 70]),
    "cnt_l1": ("gkm_cnt", dict(L=1, k=1, d=0), [30, 1, 0], [5, 1, 17, 2]),
    "wgkm_l9_norc": ("wgkm", dict(L=9, k=6, d=2, include_rc=False, M=50, H=50.0), [400, 260, 9],
                     [120, 9, 300, 44, 45, 46, 47, 48, 49]),
    "wgkmrbf_l10": ("wgkmrbf", dict(L=10, k=6, d=3, gamma=2.0, M=30, H=10.0), [257, 130, 64],
                    [256, 129, 128, 127, 10, 260, 200, 64, 63, 140, 150, 160, 170, 180, 190, 120, 110]),
    "esttrunc_l11_segments": ("gkm_esttrunc", dict(L=11, k=7, d=3), [2500, 1100, 1034, 1035, 40],
                              [300, 64, 1030, 2100]),
    "estfull_l8_many": ("gkm_estfull", dict(L=8, k=4, d=2), [100, 100, 100, 100],
                        [50 + 7 * i for i in range(41)]),
}


def _codes(rng, lengths):
    L = max(max(lengths), 1)
    x = rng.integers(0, 4, size=(len(lengths), L), dtype=np.uint8)
    # a few N (code 4) bases: they pack as A
    x[rng.random(x.shape) < 0.01] = 4
    for i, n in enumerate(lengths):
        x[i, n:] = 0
    return x, np.asarray(lengths, np.int64)


@pytest.mark.parametrize("name", sorted(CASES))
def test_dense_profiles_bit_exact(name):
    kt, params, xl, yl = CASES[name]
    rng = np.random.default_rng(sum(map(ord, name)))
    x, xl = _codes(rng, xl)
    y, yl = _codes(rng, yl)
    L = params["L"]
    if x.shape[1] < L:
        x = np.pad(x, ((0, 0), (0, L - x.shape[1])))
    if y.shape[1] < L:
        y = np.pad(y, ((0, 0), (0, L - y.shape[1])))
    m = gk.GkmSVM(y, np.linspace(-1, 1, len(yl)), 0.25, kt, params, sv_lengths=yl).cuda()
    spec = m._spec()
    assert engine.dense_applies(spec)
    bx, _, cx = engine.pack(spec, torch.from_numpy(x).cuda(), xl)
    by, ry, cy = m._sv_packed()
    raw, prof = engine.dense_pairwise(spec, bx, cx, by, ry, cy, profile=True)
    kd = orc.KernelDef.from_params(kt, params)
    want = orc.profiles(x, xl, y, yl, kd)
    d = kd.dmax
    got = prof.cpu().numpy().astype(np.uint64)
    np.testing.assert_array_equal(got[..., : d + 1], want[..., : d + 1])
    assert not got[..., d + 1:].any()
    jraw, _ = engine.join_pairwise(spec, bx, cx, by, ry, cy)
    np.testing.assert_array_equal(raw.cpu().numpy(), jraw.cpu().numpy())


def test_dense_empty_and_unsupported():
    m = gk.GkmSVM(np.zeros((2, 20), np.uint8), np.ones(2), 0.0, "gkm_esttrunc", dict(L=11, k=7, d=3)).cuda()
    spec = m._spec()
    by, ry, cy = m._sv_packed()
    bx = torch.zeros((0, 10), dtype=torch.int32, device="cuda")
    cx = torch.zeros(0, dtype=torch.int32, device="cuda")
    raw, _ = engine.dense_pairwise(spec, bx, cx, by, ry, cy)
    assert raw.shape == (0, 2)
    # dmax = l (every pair counts; no kernel type reaches it, the ABI refuses it)
    spec.c.dmax = spec.base.l
    with pytest.raises(GkmError, match="dmax < l"):
        engine.dense_pairwise(spec, by, cy, by, ry, cy)


def test_auto_pairwise_uses_dense_on_long_rows(monkeypatch):
    """Model scores through the pairwise path agree whichever kernel auto picks."""
    rng = np.random.default_rng(7)
    y, yl = _codes(rng, [150] * 9)
    x, xl = _codes(rng, [500, 300, 90])
    m = gk.GkmSVM(y, np.linspace(-1, 1, 9), 0.1, "gkmrbf", dict(L=10, k=6, d=3, gamma=2.0), sv_lengths=yl).cuda()
    m.use_lmer_index = False
    m.use_lmer_table = False
    monkeypatch.setattr(engine, "PAIRWISE_METHOD", "join")
    a = m(x, lengths=xl).cpu().numpy()
    monkeypatch.setattr(engine, "PAIRWISE_METHOD", "dense")
    b = m(x, lengths=xl).cpu().numpy()
    np.testing.assert_array_equal(a, b)


def test_autotuner_times_once_per_class_and_changes_no_result(monkeypatch):
    """auto times both forms on the first call of a shape class, keeps the
    faster, and reuses it; every form gives the same K_raw and profiles."""
    monkeypatch.setattr(engine, "PAIRWISE_TUNED", {})
    monkeypatch.setattr(engine, "PAIRWISE_METHOD", "auto")
    rng = np.random.default_rng(11)
    y, yl = _codes(rng, [300] * 40)
    x, xl = _codes(rng, [280, 300, 120, 11])
    m = gk.GkmSVM(y, np.linspace(-1, 1, 40), 0.0, "gkm_esttrunc", dict(L=11, k=7, d=3), sv_lengths=yl).cuda()
    spec = m._spec()
    by, ry, cy = m._sv_packed()
    bx, _, cx = engine.pack(spec, torch.from_numpy(x).cuda(), xl)
    raw, prof = engine.pairwise(spec, bx, cx, by, ry, cy, profile=True)
    assert list(engine.PAIRWISE_TUNED.values()) in (["join"], ["dense"])
    for form in ("join", "dense"):
        r, p = engine.pairwise(spec, bx, cx, by, ry, cy, profile=True, method=form)
        assert torch.equal(r, raw) and torch.equal(p, prof)

    def timed_again(*a, **k):
        raise AssertionError("the autotuner timed a class it had already measured")

    monkeypatch.setattr(engine, "_time_form", timed_again)
    r2, _ = engine.pairwise(spec, bx, cx, by, ry, cy)
    assert torch.equal(r2, raw)


def test_role_wait_running_out_raises_and_next_call_is_exact():
    """A hand-off wait between the kernel's roles that runs out sets the
    call's error flag: the kernel's roles leave their loops, its copies and
    MMAs in flight are waited for (their own 1 s limit) and its tensor memory
    is freed, so the call raises GkmError and the next normal call on the same
    stream is bit-exact.  The role waits are shortened to 1 ns through the
    test hook, so the first hand-off not complete on its first poll runs out."""
    from gkmsvm_lite_b200._lib import call

    kt, params, xl, yl = CASES["esttrunc_l11_long"]
    rng = np.random.default_rng(3)
    x, xl = _codes(rng, xl)
    y, yl = _codes(rng, yl)
    m = gk.GkmSVM(y, np.linspace(-1, 1, len(yl)), 0.0, kt, params, sv_lengths=yl).cuda()
    spec = m._spec()
    bx, _, cx = engine.pack(spec, torch.from_numpy(x).cuda(), xl)
    by, ry, cy = m._sv_packed()
    want, wprof = engine.join_pairwise(spec, bx, cx, by, ry, cy, profile=True)
    call("gkm_dense_set_role_wait", 1)
    try:
        with pytest.raises(GkmError, match="wait limit"):
            engine.dense_pairwise(spec, bx, cx, by, ry, cy)
    finally:
        call("gkm_dense_set_role_wait", 0)
    raw, prof = engine.dense_pairwise(spec, bx, cx, by, ry, cy, profile=True)
    torch.cuda.synchronize()
    assert torch.equal(raw, want) and torch.equal(prof, wprof)
