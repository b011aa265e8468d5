"""Host-side logic without a GPU: kernel tables, neighbour masks and window
weights against the oracle; input handling; the C ABI library exports every
symbol include/gkm_b200.h declares."""

import ctypes
import os
import re
from math import comb

import numpy as np
import pytest

from conftest import ROOT
from oracle import oracle as orc

import gkmsvm_lite_b200 as gk
from gkmsvm_lite_b200 import kernels as K
from gkmsvm_lite_b200 import inputs

PARAMS = [
    ("gkm_esttrunc", {"L": 11, "k": 7, "d": 3}),
    ("gkm_estfull", {"L": 8, "k": 5, "d": 2}),
    ("gkm_cnt", {"L": 7, "k": 4}),
    ("gkm_cnt", {"L": 10, "k": 6, "d": 3}),
    ("gkmrbf", {"L": 10, "k": 6, "d": 3, "gamma": 2.0}),
    ("wgkm", {"L": 9, "k": 6, "d": 2, "M": 20, "H": 10.0}),
    ("wgkmrbf", {"L": 11, "k": 7, "d": 3}),
    ("gkm_cnt_rbf", {"L": 8, "k": 5, "d": 2, "gamma": 1.5}),
    ("gkm_esttrunc", {"L": 15, "k": 8, "d": 4}),
]


@pytest.mark.parametrize("kt,p", PARAMS)
def test_tables_equal_oracle(kt, p):
    kd = orc.KernelDef.from_params(kt, p)
    k = K.KERNEL_BUILDERS[K.resolve_kernel_type(kt)](p)
    np.testing.assert_array_equal(k.base._mismatch_table, kd.h)
    assert k.base.dmax == kd.dmax
    assert isinstance(k, K.RbfKernel) == kd.rbf


@pytest.mark.parametrize("kt,p", PARAMS[:8])
def test_neighbor_masks_equal_oracle(kt, p):
    kd = orc.KernelDef.from_params(kt, p)
    base = K.KERNEL_BUILDERS[K.resolve_kernel_type(kt)](p).base
    masks = base.masks()
    om, ol = orc.neighbor_masks(kd.l, kd.h, kd.dmax)
    np.testing.assert_array_equal(masks & 0x00FFFFFF, om)
    np.testing.assert_array_equal(masks >> 24, ol)


def test_mask_count_l11_d3():
    base = K.EstTruncGkmKernel(11, 7, d=3)
    assert len(base.masks()) == 4984 == K.neighbor_count(11, 3)
    assert base.index_applies() and base.has_table()


@pytest.mark.parametrize("M,H", [(50, 50.0), (20, 10.0), (255, 3.5), (1, 1.0)])
def test_window_weights_bit_identical(M, H):
    k = K.CenterWeightedGkmKernel(10, 6, M=M, H=H)
    for W in (1, 2, 7, 90, 91, 290, 1990):
        np.testing.assert_array_equal(k.window_weights(W), orc.window_weights(W, M, H))


def test_resolve_kernel_type():
    assert K.resolve_kernel_type(2) == "gkm_esttrunc"
    assert K.resolve_kernel_type("5") == "wgkmrbf"
    assert K.resolve_kernel_type("direct_rbf") == "gkm_cnt_rbf"
    with pytest.raises(ValueError):
        K.resolve_kernel_type(9)
    with pytest.raises(NotImplementedError):
        K.resolve_kernel_type("nope")


def test_kernel_argument_checks():
    with pytest.raises(ValueError):
        K.DirectGkmKernel(16, 4)
    with pytest.raises(ValueError):
        K.EstTruncGkmKernel(5, 7)
    with pytest.raises(ValueError):
        K.CenterWeightedGkmKernel(10, 6, M=0)


def test_as_batch_strings_and_one_hot():
    x, ln = inputs.as_batch(["ACGTN", "GG"])
    np.testing.assert_array_equal(x, [[0, 1, 2, 3, 0], [2, 2, 0, 0, 0]])
    np.testing.assert_array_equal(ln, [5, 2])
    oh = np.eye(4)[[[0, 1, 2, 3]]].transpose(0, 2, 1)
    oh[0, :, 1] = 0  # N reads as A
    np.testing.assert_array_equal(inputs.to_codes(oh), [[0, 0, 2, 3]])
    with pytest.raises(ValueError):
        inputs.as_batch(np.zeros((2, 5), np.uint8), lengths=[1, 9])
    assert inputs.as_batch(np.zeros((2, 5), np.uint8), lengths=[5, 5])[1] is None


def test_allele_batches_pad_indels():
    ref, alt = inputs.allele_batches(["ACGTA"], ["ACGTAAC"])
    assert ref.codes.shape == alt.codes.shape == (1, 7)
    np.testing.assert_array_equal(ref.lengths, [5])
    np.testing.assert_array_equal(alt.lengths, [7])


def test_seq_batch_rows_and_masks():
    import torch

    b = inputs.SeqBatch.read(["ACGTACGTACGT", "ACG", "TTTTTTTTTTTTTT"])
    assert (b.B, b.L) == (3, 14)
    np.testing.assert_array_equal(b.lengths, [12, 3, 14])
    assert b.n_windows(11) == 2 + 0 + 4
    with pytest.warns(UserWarning, match="fewer than l = 11"):
        short = b.short(11)
    np.testing.assert_array_equal(short, [False, True, False])
    p = b.part(1, 2)
    np.testing.assert_array_equal(p.lengths, [3, 14])
    both = inputs.SeqBatch.stacked(b.part(0, 1), b.part(2, 1))
    np.testing.assert_array_equal(both.lengths, [12, 14])
    out = torch.ones((3, 4, 14), dtype=torch.float64)
    m = inputs.per_position(out, b, short)
    assert torch.isnan(m[1]).all()
    assert m[0, :, :12].eq(1).all() and m[0, :, 12:].eq(0).all()
    assert m[2].eq(1).all()
    with pytest.raises(ValueError):
        inputs.encode_codes("ACGN")
    np.testing.assert_array_equal(inputs.encode_codes("ACGN", allow_n=True), [0, 1, 2, 0])
    with pytest.raises(ValueError):
        inputs.encode_codes("ACGX", allow_n=True)
    np.testing.assert_array_equal(inputs.encode_codes("acgx", allow_other=True), [0, 1, 2, 0])


def test_model_on_cpu_refuses_to_compute():
    m = gk.GkmSVM(np.zeros((3, 20), np.uint8), np.ones(3), 0.0, 2, {"L": 11, "k": 7, "d": 3})
    with pytest.raises(RuntimeError, match="CUDA only"):
        m(np.zeros((1, 20), np.uint8))


def test_lsgkm_loader_matches_oracle():
    from conftest import LSGKM

    p = os.path.join(LSGKM, "lsgkm_ragged_t4.model.txt.gz")
    m = gk.load_lsgkm_model(p)
    om = orc.load_lsgkm(p)
    np.testing.assert_array_equal(m.support_sequences, om.sv)
    np.testing.assert_array_equal(m.sv_lengths, om.sv_lengths)
    np.testing.assert_array_equal(m.coefficients, om.coef)
    assert m.bias == om.bias and m.kernel_type == "wgkm"


def _declared_symbols():
    src = open(os.path.join(ROOT, "include", "gkm_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gkm_[a-z0-9_]+)\s*\(", src)))


def test_abi_library_exports_every_declared_symbol():
    from gkmsvm_lite_b200 import _lib

    if not os.path.exists(_lib.LIB_PATH):
        from gkmsvm_lite_b200 import build
        build.build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = _declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) <= set(_lib.SIGNATURES) | {"gkm_last_error"}
    lib.gkm_version.restype = ctypes.c_int
    assert lib.gkm_version() >= 1


def test_thread_settings_refuse_negative_values():
    """The serving grid limit and the dense kernel's role-wait test hook are
    host-side, per-thread settings: negative values are refused, 0 restores
    the default (no device work is involved)."""
    from gkmsvm_lite_b200 import _lib

    lib = _lib.load()
    assert lib.gkm_set_thread_grid_limit(-1) == _lib.GKM_ERR_INVALID
    assert lib.gkm_set_thread_grid_limit(0) == _lib.GKM_OK
    assert lib.gkm_dense_set_role_wait(-5) == _lib.GKM_ERR_INVALID
    assert lib.gkm_dense_set_role_wait(0) == _lib.GKM_OK


def test_pairwise_forms_and_classes():
    """The forms the autotuner chooses between (the tensor-core product only
    where dmax < l <= 15), and its shape classes."""
    import torch

    from gkmsvm_lite_b200 import engine

    def spec(kt, p):
        m = gk.GkmSVM(np.zeros((2, 40), np.uint8), np.ones(2), 0.0, kt, p)
        return engine.Spec(m.kernel.base, torch.device("cpu"))

    from math import comb
    # exact: l-mers within 3 of a given one, over all 4^11
    want = sum(comb(11, m) * 3 ** m for m in range(4)) / 4 ** 11
    assert abs(engine.hit_rate(11, 3) - want) < 1e-15
    t2 = spec("gkm_esttrunc", dict(L=11, k=7, d=3))
    assert engine.pairwise_forms(t2) == ["join", "dense"]
    assert engine.pairwise_forms(spec("gkm_cnt", dict(L=15, k=5, d=10))) == ["join", "dense"]
    assert engine.pairwise_forms(spec("wgkm", dict(L=9, k=6, d=2))) == ["join", "dense"]
    # a kernel counting pairs at every mismatch level (dmax = l): the join only,
    # chosen without timing
    from types import SimpleNamespace
    full = SimpleNamespace(base=SimpleNamespace(l=7, dmax=7))
    assert engine.pairwise_forms(full) == ["join"]
    assert engine.choose_pairwise(full, torch.zeros((3, 5), dtype=torch.int32), None,
                                  torch.zeros((2, 8), dtype=torch.int32), None, None) == "join"
    c = engine.pairwise_class(t2, 100, 290, 72000, 490)
    assert c == (11, 3, False, True, 128, 512, 65536, 512)
    assert engine.pairwise_class(t2, 65, 257, 5000, 300) == (11, 3, False, True, 128, 512, 8192, 512)


def test_pairwise_autotuner_caches_per_class(monkeypatch):
    """The autotuner times each form once per shape class (here with a fake
    clock: the join is faster on short rows, the tensor-core form on long
    ones) and reuses the choice."""
    import torch

    from gkmsvm_lite_b200 import engine

    m = gk.GkmSVM(np.zeros((2, 40), np.uint8), np.ones(2), 0.0, "gkm_esttrunc", dict(L=11, k=7, d=3))
    spec = engine.Spec(m.kernel.base, torch.device("cpu"))
    timed = []

    def fake_time(form, spec_, bx, cx, by, ry, cy):
        timed.append((form, bx.shape[1]))
        return (1.0 if form == "join" else 2.0) if bx.shape[1] < 100 else (3.0 if form == "join" else 1.0)

    monkeypatch.setattr(engine, "_time_form", fake_time)
    monkeypatch.setattr(engine, "PAIRWISE_TUNED", {})
    i32 = lambda *s: torch.zeros(s, dtype=torch.int32)
    short, long_ = i32(10, 50), i32(10, 900)
    cols, ccount = i32(300, 290), i32(300)
    assert engine.choose_pairwise(spec, short, i32(10), cols, cols, ccount) == "join"
    assert engine.choose_pairwise(spec, short, i32(10), cols, cols, ccount) == "join"
    assert engine.choose_pairwise(spec, long_, i32(10), cols, cols, ccount) == "dense"
    assert engine.choose_pairwise(spec, i32(12, 1000), i32(12), cols, cols, ccount) == "dense"  # same class
    assert sorted(timed) == [("dense", 50), ("dense", 900), ("join", 50), ("join", 900)]
    assert len(engine.PAIRWISE_TUNED) == 2


def test_index_rule_past_the_reference_limit():
    """Neighbourhoods past the reference's limit (t=0 gkm_cnt l=11 k=7 with no
    d: 31,714 masks) take the index where its measured cost per query window
    is below the all-pairs forms' -- mid-size SV sets -- and not for a handful
    of SVs; the reference's own cases are unchanged."""
    k = K.DirectGkmKernel(11, 7)  # gkm_cnt, no d: dmax 4
    assert K.neighbor_count(11, k.dmax) == 31714
    assert not k.index_applies()
    assert not k.index_applies(100 * 290 * 2)       # 100 SVs x 300 bp: every pair is cheaper
    assert k.index_applies(4000 * 290 * 2)          # 4,000 SVs x 300 bp
    assert k.index_applies(72000 * 340 * 2)         # the reference's dense-neighbourhood case
    e = K.EstTruncGkmKernel(11, 7, d=3)             # 4,984 masks: always
    assert e.index_applies() and e.index_applies(10)


def test_mask_plan_matches_reference():
    """The masked-join plan (kernels/masked.py:45-69): mask sizes, coefficients
    and position subsets equal gkmsvm-lite's for every small kernel type and a
    few l = 10..12 kernels (tests/golden/maskplan.npz, made by make_golden.py),
    and a plan exists exactly where the kernel reports an l-mer table."""
    import ast

    from conftest import GOLDEN

    z = np.load(os.path.join(GOLDEN, "maskplan.npz"))
    n = len({k.split("/")[0] for k in z.files})
    assert n >= 10
    for i in range(n):
        kt, params = str(z[f"{i}/kernel"]).split(" ", 1)
        base = gk.KERNEL_BUILDERS[K.resolve_kernel_type(kt)](ast.literal_eval(params)).base
        plan = base.mask_plan()
        assert (plan is None) == bool(z[f"{i}/none"]), (kt, params)
        if plan is None:
            continue
        np.testing.assert_array_equal([j for j, _, _ in plan], z[f"{i}/sizes"])
        np.testing.assert_allclose([c for _, c, _ in plan], z[f"{i}/coefs"], rtol=1e-12, atol=1e-15)
        np.testing.assert_array_equal([int(p.sum()) for _, _, p in plan], z[f"{i}/positions_sum"])
        for j, _, pos in plan:
            assert pos.shape == (comb(base.l, j), j)
        assert base.has_table() == (base.l <= K.MAX_TABLE_L)
