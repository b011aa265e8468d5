"""GPU parity: the CUDA path against the oracle (bit-exact mismatch profiles)
and against gkmsvm-lite's own outputs (tests/golden) within the reference's
GPU tolerance, rtol 1e-9 / atol 1e-12 (its tests/test_gpu.py:100-104).
Every call goes through the C ABI (libgkm_b200.so)."""

import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN, LSGKM, codes_of, read_fasta, read_pred
from oracle import oracle as orc

import gkmsvm_lite_b200 as gk
from gkmsvm_lite_b200 import engine

pytestmark = pytest.mark.gpu
RTOL, ATOL = 1e-9, 1e-12
CASES = ["t2", "t2norc", "t0", "t0small", "t1", "t3", "t4", "t5", "t6"]
LINEAR = ["t2", "t2norc", "t0", "t0small", "t1", "t4"]


def _np(t):
    return t.detach().cpu().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)


def _model(c, **switches):
    m = gk.GkmSVM(c["sv"], c["coef"], float(c["bias"]), c["kernel_type"], c["params"],
                  sv_lengths=c["sv_lengths"]).cuda()
    for k, v in switches.items():
        setattr(m, k, v)
    return m


def _okd(c):
    return orc.KernelDef.from_params(c["kernel_type"], c["params"])


@pytest.mark.parametrize("name", CASES)
def test_pack_matches_oracle(small, name):
    c = small[name]
    m = _model(c)
    x, xl = c["x"], c["x_lengths"]
    fwd, rc, counts = engine.pack(m._spec(), torch.from_numpy(x).cuda(), xl)
    of, orr = orc.pack(x, xl, m.kernel.l)
    np.testing.assert_array_equal(_np(fwd).view(np.uint32), of)
    if rc is not None:
        np.testing.assert_array_equal(_np(rc).view(np.uint32), orr)
    np.testing.assert_array_equal(_np(counts), np.clip(xl - m.kernel.l + 1, 0, x.shape[1] - m.kernel.l + 1))


@pytest.mark.parametrize("name", CASES)
def test_self_profiles_bit_exact(small, name):
    c = small[name]
    m = _model(c)
    kd = _okd(c)
    fwd, rc, counts = m._sv_packed()
    diag, prof = engine.self_kernel(m._spec(), fwd, rc, counts, profile=True)
    want = orc.self_profiles(c["sv"], c["sv_lengths"], kd)
    d = kd.dmax
    np.testing.assert_array_equal(_np(prof)[:, : d + 1].astype(np.uint64), want[:, : d + 1])
    np.testing.assert_allclose(_np(diag), c["diag_sv"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("path", ["join", "dense", "index"])
def test_pairwise_profiles_bit_exact(small, name, path):
    c = small[name]
    m = _model(c)
    kd = _okd(c)
    spec = m._spec()
    bx, _, cx = engine.pack(spec, torch.from_numpy(c["x"]).cuda(), c["x_lengths"])
    by, ry, cy = m._sv_packed()
    if path == "join":
        raw, prof = engine.join_pairwise(spec, bx, cx, by, ry, cy, profile=True)
    elif path == "dense":
        if not engine.dense_applies(spec):
            pytest.skip("the tensor-core form needs dmax < l")
        raw, prof = engine.dense_pairwise(spec, bx, cx, by, ry, cy, profile=True)
    else:
        if not m.kernel.base.index_applies():
            pytest.skip("neighbourhood too large for the index")
        ix = engine.DeviceIndex(spec, by, ry, cy, m._masks(), tile_svs=5)  # several tiles
        raw, prof = ix.pairwise(bx, cx, profile=True)
        ix.close()
    want = orc.profiles(c["x"], c["x_lengths"], c["sv"], c["sv_lengths"], kd)
    d = kd.dmax
    np.testing.assert_array_equal(_np(prof)[..., : d + 1].astype(np.uint64), want[..., : d + 1])
    np.testing.assert_allclose(_np(raw), c["raw"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("switch", ["auto", "index", "join", "dense", "table"])
def test_scores_match_reference(small, name, switch, monkeypatch):
    c = small[name]
    pairs = dict(use_lmer_table=False, use_lmer_index=False)
    sw = {"index": dict(use_lmer_table=False), "join": pairs, "dense": pairs,
          "table": dict(use_lmer_table=True), "auto": {}}[switch]
    if switch in ("join", "dense"):
        monkeypatch.setattr(engine, "PAIRWISE_METHOD", switch)
    m = _model(c, **sw)
    with pytest.warns(UserWarning):
        got = m(c["x"], lengths=c["x_lengths"])
    np.testing.assert_allclose(_np(got), c["scores"], rtol=RTOL, atol=ATOL)
    assert np.isnan(_np(got)[-1, 0])


@pytest.mark.parametrize("name", CASES)
def test_variant_scores_match_reference(small, name):
    c = small[name]
    m = _model(c)
    ref, rl, alt, al = c["x"][:-1], c["x_lengths"][:-1], c["alt"], c["alt_lengths"]
    got = m.score_variants(ref, alt, ref_lengths=rl, alt_lengths=al)
    np.testing.assert_allclose(_np(got), c["variant_kernel"], rtol=RTOL, atol=ATOL)
    got = m.score_variants(ref, alt, method="gkmexplain", ref_lengths=rl, alt_lengths=al)
    np.testing.assert_allclose(_np(got), c["variant_impact"], rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("name", LINEAR)
@pytest.mark.parametrize("table", [True, False])
def test_ism_linear_matches_reference(small, name, table):
    c = small[name]
    m = _model(c, use_lmer_table=table)
    if not table and not m._index_applies():
        pytest.skip("no index for this kernel")
    with pytest.warns(UserWarning):
        got = gk.ism(m, c["x"], lengths=c["x_lengths"])
    np.testing.assert_allclose(_np(got), c["ism"], rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("name", CASES)
def test_ism_index_matches_reference(small, name):
    """ISM through the l-mer index (every kernel type, RBF included)."""
    c = small[name]
    m = _model(c, use_lmer_table=False)
    if not m._index_applies():
        pytest.skip("no index for this kernel")
    with pytest.warns(UserWarning):
        got = gk.ism(m, c["x"], lengths=c["x_lengths"])
    np.testing.assert_allclose(_np(got), c["ism"], rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("name", ["t3", "t5"])
def test_index_mutants_with_given_reference_scores(small, name):
    """gkm_index_mutants through the C ABI with the reference rows' scores
    passed in (index.score) and with a null ref_score (scored inside the call
    from ref_raw): the same ISM deltas, equal to gkmsvm-lite's."""
    from gkmsvm_lite_b200._lib import call, ptr, stream_handle
    from gkmsvm_lite_b200.ism import ism_workspace

    c = small[name]
    m = _model(c, use_lmer_table=False)
    spec, index = m._spec(), m._sv_index()
    x = torch.from_numpy(np.asarray(c["x"], np.uint8)).cuda()
    xl = None if c["x_lengths"] is None else torch.as_tensor(np.asarray(c["x_lengths"], np.int64)).cuda()
    fwd, rc, counts = engine.pack(spec, x, xl)
    B, W = fwd.shape
    L = x.shape[1]
    from gkmsvm_lite_b200.kernels import RbfKernel

    kernel = m.kernel
    rbf = isinstance(kernel, RbfKernel)
    gamma = kernel.gamma if rbf else 0.0
    diag = engine.self_kernel(spec, fwd, rc, counts)
    mut = engine.mutant_diag(spec, fwd, counts, L, diag)
    inv_dx = 1.0 / torch.sqrt(torch.clamp(diag, min=1e-20))
    inv_dmut = 1.0 / torch.sqrt(torch.clamp(mut, min=1e-20))
    ref_raw, _ = index.pairwise(fwd, counts)
    ref_score = index.score(fwd, counts, inv_dx, m._inv_ds(), m._sv_coef(), gamma, rbf, 0.0)
    work = ism_workspace(m, B, L, fwd.device)
    outs = []
    for given in (ref_score, None):
        out = torch.empty((B, 4, L), dtype=torch.float64, device=fwd.device)
        call("gkm_index_mutants", index.handle, ptr(fwd), ptr(counts), B, W, L, ptr(ref_raw), ptr(given),
             ptr(inv_dx), ptr(inv_dmut), ptr(m._inv_ds()), ptr(m._sv_coef()), float(gamma), int(rbf),
             ptr(out), ptr(work), int(work.numel()), stream_handle())
        torch.cuda.synchronize()
        outs.append(_np(out))
    want = np.asarray(c["ism"], np.float64)
    for got in outs:
        ok = np.isfinite(want)
        np.testing.assert_allclose(got[ok], want[ok], rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("mode,key", [("hypothetical", "explain_hyp"), ("importance", "explain_imp"),
                                      ("perturbation", "explain_pert")])
def test_explain_matches_reference(small, name, mode, key):
    c = small[name]
    m = _model(c)
    with pytest.warns(UserWarning):
        got = gk.gkmexplain(m, c["x"], lengths=c["x_lengths"], mode=mode)
    np.testing.assert_allclose(_np(got), c[key], rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("name", CASES)
def test_gram_matches_reference(small, name):
    c = small[name]
    m = _model(c)
    got = gk.compute_gram(m.kernel, c["sv"], lengths=c["sv_lengths"])
    np.testing.assert_allclose(got, c["gram"], rtol=RTOL, atol=ATOL)
    assert (got == got.T).all()


def test_mutant_diag_matches_oracle(small):
    """K(mutant, mutant) from the window-delta kernel equals the self-kernel of
    each mutant sequence."""
    c = small["t4"]
    m = _model(c)
    kd = _okd(c)
    x, xl = c["x"][:2], c["x_lengths"][:2]
    spec = m._spec()
    fwd, rc, counts = engine.pack(spec, torch.from_numpy(x).cuda(), xl)
    diag = engine.self_kernel(spec, fwd, rc, counts)
    L = x.shape[1]
    mut = _np(engine.mutant_diag(spec, fwd, counts, L, diag))
    for b in range(2):
        n = int(xl[b])
        mutants = np.repeat(x[b:b + 1, :n], 4 * n, axis=0)
        for p in range(n):
            for v in range(4):
                mutants[4 * p + v, p] = v
        want = orc.raw_from_profiles(orc.self_profiles(mutants, None, kd), kd).reshape(n, 4).T
        np.testing.assert_allclose(mut[:, :n, b], want, rtol=1e-12, atol=1e-12)


def test_config1_scores_match_reference():
    """Plain scoring workload: 2,000 SVs x 300 bp, 1,000 queries (t=2), every path."""
    import gkmsvm_lite_b200.synthetic as syn

    w = syn.config1()
    want = np.load(os.path.join(GOLDEN, "config1.npz"))["scores"]
    for sw in ({"use_lmer_table": False}, {"use_lmer_table": True}, {}):
        m = gk.GkmSVM(w.sv, w.coef, 0.0, "gkm_esttrunc", {"L": 11, "k": 7, "d": 3}).cuda()
        for k, v in sw.items():
            setattr(m, k, v)
        np.testing.assert_allclose(_np(m(w.x)), want, rtol=RTOL, atol=ATOL)


def test_config3_subsample_matches_reference():
    """72,000-SV model (SV lengths 200..500), queries 50..2000 bp with N: t=2
    (the first 256 queries) and t=3 gamma=2 (256 queries: the first 224 and
    the 32 longest of the first 20,000, 2,000 bp rows among them) against the
    reference."""
    import gkmsvm_lite_b200.synthetic as syn

    sv, svl, coef = syn.config3_model()
    xq, xl, _ = syn.config3_queries()
    z = np.load(os.path.join(GOLDEN, "config3.npz"))
    assert len(z["t3/rows"]) >= 256 and xl[z["t3/rows"]].max() >= 1990
    for name, kt, p in (("t2", "gkm_esttrunc", {"L": 11, "k": 7, "d": 3}),
                        ("t3", "gkmrbf", {"L": 11, "k": 7, "d": 3, "gamma": 2.0})):
        rows = z[f"{name}/rows"]
        m = gk.GkmSVM(sv, coef, 0.0, kt, p, sv_lengths=svl).cuda()
        m.use_lmer_table = False
        L = int(xl[rows].max())
        got = _np(m(xq[rows, :L], lengths=xl[rows]))
        np.testing.assert_allclose(got, z[f"{name}/scores"], rtol=RTOL, atol=ATOL)
        if name == "t2":
            np.testing.assert_allclose(_np(m._sv_diag())[:256], z["t2/diag_sv_head"], rtol=1e-12)
            m.use_lmer_table = True
            np.testing.assert_allclose(_np(m(xq[rows, :L], lengths=xl[rows])), z["t2/scores"], rtol=RTOL,
                                       atol=ATOL)


def _config4_model():
    import gkmsvm_lite_b200.synthetic as syn

    sv, svl, coef = syn.config3_model()
    return gk.GkmSVM(sv, coef, 0.0, "gkm_esttrunc", {"L": 11, "k": 7, "d": 3}, sv_lengths=svl).cuda()


def test_config4_ism_matches_reference():
    """16 x 1,000 bp through the l-mer table (fused mutant self-kernels) and
    through the index (mutant window sets)."""
    import gkmsvm_lite_b200.synthetic as syn

    x = syn.config4_queries()[:16]
    z = np.load(os.path.join(GOLDEN, "config4.npz"))
    assert z["ism"].shape[0] == 16
    m = _config4_model()
    for table in (True, False):
        m.use_lmer_table = table
        got = _np(gk.ism(m, x))
        np.testing.assert_allclose(got, z["ism"], rtol=RTOL, atol=1e-10 * np.abs(z["ism"]).max())


def test_config4_explain_matches_reference():
    """16 x 1,000 bp hypothetical attributions through the explain table and
    through the l-mer neighbour path."""
    import gkmsvm_lite_b200.synthetic as syn

    x = syn.config4_queries()[:16]
    z = np.load(os.path.join(GOLDEN, "config4.npz"))
    assert z["explain_hyp"].shape[0] == 16
    m = _config4_model()
    for table in ("auto", False):
        m.use_explain_table = table
        got = _np(gk.gkmexplain(m, x, mode="hypothetical", batch_size=16))
        np.testing.assert_allclose(got, z["explain_hyp"], rtol=RTOL, atol=1e-10 * np.abs(z["explain_hyp"]).max())


def test_encode_72k_model_matches_reference():
    """The reference benchmark's 72,145-SV ENCODE model (LS-GKM text, loaded by
    the native parser): gkmsvm-lite's scores of 64 x 300 bp queries for t2 (its
    l-mer table and the index) and for the same SVs as gkmrbf gamma=1."""
    z = np.load(os.path.join(GOLDEN, "encode.npz"))
    m = gk.load_lsgkm_model(os.path.join(LSGKM, "encode_ENCFF579AOX.model.txt.gz")).cuda()
    assert m.num_support_vectors == 72145
    # near-zero scores of 72,145 summed terms: atol relative to the largest
    # score (the reference's large-model tolerance, tests/test_gpu.py:783-784)
    for table in (True, False):
        m.use_lmer_table = table
        np.testing.assert_allclose(_np(m(z["x"])), z["t2"], rtol=RTOL, atol=1e-10 * np.abs(z["t2"]).max())
    r = gk.GkmSVM(m.support_sequences, m.coefficients, m.bias, "gkmrbf", {**m.kernel_params, "gamma": 1.0},
                  sv_lengths=m.sv_lengths).cuda()
    np.testing.assert_allclose(_np(r(z["x"])), z["t3"], rtol=RTOL, atol=1e-10 * np.abs(z["t3"]).max())


def test_config2_profiles_sampled_pairs_bit_exact():
    """Config 2 (4,000 sequences 100..1,000 bp, t=4 wgkm): mismatch profiles
    (levels 0..dmax, the ones with weight) of 10,000 sampled (row, column)
    pairs through the index, the tensor-core form and the join, and every
    diagonal (self-kernel), bit-exact against the oracle."""
    import gkmsvm_lite_b200.synthetic as syn

    X, xl = syn.config2()
    k = gk.CenterWeightedGkmKernel(11, 7, d=3)
    kd = orc.KernelDef.from_params("wgkm", {"L": 11, "k": 7, "d": 3})
    dev = torch.device("cuda")
    spec = engine.Spec(k.base, dev)
    bx, rx, cx = engine.pack(spec, torch.from_numpy(X).to(dev), xl)
    rng = np.random.default_rng(8)
    rows = np.sort(rng.choice(len(xl), 100, replace=False))
    cols = np.stack([np.sort(rng.choice(len(xl), 100, replace=False)) for _ in rows])
    want = np.stack([orc.profiles(X[r:r + 1], xl[r:r + 1], X[c], xl[c], kd)[0] for r, c in zip(rows, cols)])
    ri = torch.from_numpy(rows).to(dev)
    sub_x, sub_c = bx[ri].contiguous(), cx[ri].contiguous()
    ix = engine.DeviceIndex(spec, bx, rx, cx, engine.masks_tensor(k.base, dev))
    _, prof = ix.pairwise(sub_x, sub_c, raw=False, profile=True)
    ix.close()
    forms = {"index": _np(prof)}
    for method in engine.pairwise_forms(spec):
        forms[method] = _np(engine.pairwise(spec, sub_x, sub_c, bx, rx, cx, raw=False, profile=True,
                                            method=method)[1])
    # the GPU forms count the levels that carry weight, 0..dmax; the rest stay 0
    d = kd.dmax
    for name, p in forms.items():
        got = np.stack([p[i][cols[i]] for i in range(len(rows))]).astype(np.uint64)
        np.testing.assert_array_equal(got[..., : d + 1], want[..., : d + 1], err_msg=name)
        assert not got[..., d + 1:].any(), name
    _, diag = engine.self_kernel(spec, bx, rx, cx, profile=True)
    want_diag = orc.self_profiles(X, xl, kd, threads=os.cpu_count())
    np.testing.assert_array_equal(_np(diag).astype(np.uint64)[:, : d + 1], want_diag[:, : d + 1])


def test_config5_mixed_requests_match_reference():
    """72,000-SV t=5 (wgkmrbf) model: predict (with a row shorter than l),
    variant scores with indels, ISM and GkmExplain."""
    import gkmsvm_lite_b200.synthetic as syn

    sv, svl, coef = syn.config3_model()
    z = np.load(os.path.join(GOLDEN, "config5.npz"))
    m = gk.GkmSVM(sv, coef, 0.0, "wgkmrbf", {"L": 11, "k": 7, "d": 3, "gamma": 1.0}, sv_lengths=svl).cuda()
    with pytest.warns(UserWarning):
        got = _np(m(z["x"], lengths=z["x_lengths"]))
    np.testing.assert_allclose(got, z["scores"], rtol=RTOL, atol=ATOL)
    got = _np(m.score_variants(z["ref"], z["alt"], ref_lengths=z["ref_lengths"], alt_lengths=z["alt_lengths"]))
    np.testing.assert_allclose(got, z["variants"], rtol=RTOL, atol=ATOL)
    got = _np(gk.ism(m, z["ism_x"]))
    np.testing.assert_allclose(got, z["ism"], rtol=RTOL, atol=1e-10 * np.abs(z["ism"]).max())
    got = _np(gk.gkmexplain(m, z["ism_x"], mode="hypothetical"))
    np.testing.assert_allclose(got, z["explain_hyp"], rtol=RTOL, atol=1e-10 * np.abs(z["explain_hyp"]).max())


def test_config2_gram_matches_reference():
    import gkmsvm_lite_b200.synthetic as syn

    X, lengths = syn.config2()
    z = np.load(os.path.join(GOLDEN, "config2.npz"))
    k = gk.CenterWeightedGkmKernel(11, 7, d=3)
    rows = gk.compute_gram(k, X[:48], X, lengths=lengths[:48], y_lengths=lengths)
    np.testing.assert_allclose(rows, z["rows"], rtol=RTOL, atol=ATOL)
    sym = gk.compute_gram(k, X[:160], lengths=lengths[:160])
    np.testing.assert_allclose(sym, z["sym"], rtol=RTOL, atol=ATOL)


_WGKM = ["t0", "t1", "t2", "t2w2", "t3", "t4", "t4w05", "t5", "t6"]


@pytest.mark.parametrize("t", _WGKM)
def test_lsgkm_gkmpredict(t):
    m = gk.load_lsgkm_model(os.path.join(LSGKM, f"lsgkm_wgkm_{t}.model.txt.gz")).cuda()
    for n in (85, 100):
        _, seqs = read_fasta(os.path.join(LSGKM, f"lsgkm_wgkm_test{n}.fa"))
        want = read_pred(os.path.join(LSGKM, f"lsgkm_wgkm_{t}_test{n}.pred.txt"))
        np.testing.assert_allclose(_np(m(seqs))[:, 0], want, rtol=2e-5, atol=1e-5)


@pytest.mark.parametrize("t", ["t0", "t1", "t4", "t5", "t6"])
@pytest.mark.parametrize("lm,mode", [(0, "importance"), (1, "hypothetical"), (4, "perturbation")])
def test_lsgkm_gkmexplain(t, lm, mode):
    from conftest import read_lsgkm_explain

    m = gk.load_lsgkm_model(os.path.join(LSGKM, f"lsgkm_wgkm_{t}.model.txt.gz")).cuda()
    _, seqs = read_fasta(os.path.join(LSGKM, "lsgkm_wgkm_test85.fa"))
    want = read_lsgkm_explain(os.path.join(LSGKM, f"lsgkm_wgkm_{t}_test85.explain{lm}.txt.gz"))
    got = _np(gk.gkmexplain(m, seqs, mode=mode))
    np.testing.assert_allclose(got, want, rtol=2e-5, atol=5e-6 * np.abs(want).max())


@pytest.mark.parametrize("kind", ["est", "rbf"])
def test_lsgkm_mutation_impact(kind):
    m = gk.load_lsgkm_model(os.path.join(LSGKM, f"lsgkm_mode5_{kind}.model.txt.gz")).cuda()
    _, seqs = read_fasta(os.path.join(LSGKM, "lsgkm_mode5_test51.fa"))
    rows = [line.split("\t") for line in open(os.path.join(LSGKM, f"lsgkm_mode5_{kind}.txt"))]
    want = np.array([[float(v) for v in r[2].split(",")] for r in rows])
    c = len(seqs[0]) // 2
    ref, alt = [], []
    for s in seqs:
        for b in "ACGT":
            ref.append(s)
            alt.append(s[:c] + b + s[c + 1:])
    got = _np(gk.mutation_impact(m, ref, alt)).reshape(-1, 4)
    np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-6)


def test_encode_10sv_gkmpredict():
    m = gk.load_lsgkm_model(os.path.join(LSGKM, "encode_ENCFF579AOX_10sv.model.txt.gz")).cuda()
    rows = [line.rstrip("\n").split("\t") for line in open(os.path.join(LSGKM, "encode_10sv_gkmpredict.tsv"))]
    for i, (name, seq, want) in enumerate(rows):
        if name.startswith("sv"):
            n = m.sv_lengths[i] if m.sv_lengths is not None else m.support_sequences.shape[1]
            x = m.support_sequences[i:i + 1, :n]
        else:
            x = [seq]
        assert abs(float(_np(m(x))[0, 0]) - float(want)) < 1e-4


def test_counter_carries_are_exact():
    """Low-complexity rows push one (row, SV, level) count past 16 bits, and
    far past the narrow fields: counts stay exact whether the carries fit the
    log or a block outgrows it and the call reruns with 32-bit counters."""
    rng = np.random.default_rng(5)
    sv = np.concatenate([np.zeros((10, 500), np.uint8), rng.integers(0, 4, (30, 500)).astype(np.uint8)])
    coef = rng.normal(size=40)
    x = np.concatenate([np.zeros((1, 2000), np.uint8), rng.integers(0, 4, (2, 2000)).astype(np.uint8)])
    kd = orc.KernelDef.from_params("gkmrbf", {"L": 11, "k": 7, "d": 3, "gamma": 2.0})
    want_prof = orc.profiles(x, None, sv, None, kd)
    assert want_prof[0, 0, 0] > 65535
    m = gk.GkmSVM(sv, coef, 0.0, "gkmrbf", {"L": 11, "k": 7, "d": 3, "gamma": 2.0}).cuda()
    m.use_lmer_table = False
    index = m._sv_index()
    spec = m._spec()
    fwd, rc, counts = engine.pack(spec, torch.from_numpy(x).cuda(), None)
    # one poly-A SV per tile (exact through the log or the 32-bit rerun)
    ix1 = engine.DeviceIndex(spec, *m._sv_packed(), m._masks(), tile_svs=2)
    raw, prof = ix1.pairwise(fwd, counts, profile=True)
    np.testing.assert_array_equal(_np(prof)[..., :4].astype(np.uint64), want_prof[..., :4])
    ix1.close()
    # ten poly-A SVs in one tile, each row whole in one block (300 rows: enough
    # items that no row is split): the log overflows and the query reruns
    xr = np.repeat(x, 100, axis=0)
    fwd, rc, counts = engine.pack(spec, torch.from_numpy(xr).cuda(), None)
    inv_dx = 1.0 / torch.sqrt(engine.self_kernel(spec, fwd, rc, counts))
    before = index.counters()
    index.score(fwd, counts, inv_dx, m._inv_ds(), m._sv_coef(), 2.0, 1, 0.0, check=False)
    after = index.counters()
    torch.cuda.synchronize()
    assert int(after[0]) > int(before[0])
    got = _np(m(x))
    want = orc.scores(orc.OracleModel(sv, None, coef, 0.0, kd), x)
    np.testing.assert_allclose(got, want, rtol=RTOL, atol=ATOL)


def test_weighted_counts_past_32_bits_are_exact():
    """Window weights of 255 and poly-A rows push one (row, SV, level)
    weighted count past 2^32 (the reference sums these in float64): the 32-bit
    pass reports the wrap and the checked call reruns with 64-bit counters."""
    rng = np.random.default_rng(9)
    params = {"L": 11, "k": 7, "d": 3, "gamma": 1.0, "M": 255, "H": 1e6}
    sv = np.concatenate([np.zeros((4, 1000), np.uint8), rng.integers(0, 4, (20, 1000)).astype(np.uint8)])
    coef = rng.normal(size=24)
    x = np.concatenate([np.zeros((1, 1000), np.uint8), rng.integers(0, 4, (2, 1000)).astype(np.uint8)])
    kd = orc.KernelDef.from_params("wgkmrbf", params)
    want_prof = orc.profiles(x, None, sv, None, kd)
    assert want_prof[0, 0, 0] >= 2**32
    m = gk.GkmSVM(sv, coef, 0.0, "wgkmrbf", params).cuda()
    m.use_lmer_table = False
    index = m._sv_index()
    spec = m._spec()
    # 300 rows: enough items that no row is split, each row whole in one block
    xr = np.repeat(x, 100, axis=0)
    fwd, rc, counts = engine.pack(spec, torch.from_numpy(xr).cuda(), None)
    before = index.counters()
    index.pairwise(fwd, counts, check=False)
    after = index.counters()
    torch.cuda.synchronize()
    assert int(after[1]) > int(before[1])  # a 32-bit count wrapped
    raw, prof = index.pairwise(fwd, counts, profile=True)
    np.testing.assert_array_equal(_np(prof)[::100, :, :4].astype(np.uint64), want_prof[..., :4])
    want = orc.scores(orc.OracleModel(sv, None, coef, 0.0, kd), x)
    np.testing.assert_allclose(_np(m(xr))[::100], want, rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(_np(m(x)), want, rtol=RTOL, atol=ATOL)


def test_packed_counter_carries_are_logged_exactly():
    """Packed counters (every level of an SV in one 32-bit word, 4 bits for
    level 0): an 11-mer planted 5 times in 5 SVs and in the query rows makes
    level-0 counts of 25 (or more), past the field; the item's check sees the
    carry, the carry-logged retry corrects it within the log (no rerun), and
    the profiles equal the oracle's."""
    rng = np.random.default_rng(12)
    sv = rng.integers(0, 4, (40, 300)).astype(np.uint8)
    motif = rng.integers(0, 4, 11).astype(np.uint8)
    for r in range(5):
        for k in range(5):
            sv[r, 20 + 55 * k:31 + 55 * k] = motif
    x = rng.integers(0, 4, (300, 400)).astype(np.uint8)
    for k in range(5):
        x[:, 30 + 70 * k:41 + 70 * k] = motif
    kd = orc.KernelDef.from_params("gkmrbf", {"L": 11, "k": 7, "d": 3, "gamma": 2.0})
    want = orc.profiles(x[:3], None, sv, None, kd)
    assert want[:, :5, 0].min() >= 25
    m = gk.GkmSVM(sv, rng.normal(size=40), 0.0, "gkmrbf", {"L": 11, "k": 7, "d": 3, "gamma": 2.0}).cuda()
    m.use_lmer_table = False
    index = m._sv_index()
    spec = m._spec()
    # 300 rows: enough items that no row is split, each row whole in one block
    fwd, rc, counts = engine.pack(spec, torch.from_numpy(x).cuda(), None)
    before = index.counters()
    _, prof = index.pairwise(fwd, counts, raw=False, profile=True, check=False)
    after = index.counters()
    torch.cuda.synchronize()
    assert int(after[0]) == int(before[0])  # every carry fit the log
    np.testing.assert_array_equal(_np(prof)[:3, :, :4].astype(np.uint64), want[..., :4])


@pytest.mark.parametrize("name", ["t2", "t3", "t4", "t5", "t6", "t0"])
@pytest.mark.parametrize("graphs", [True, False])
def test_batched_scorer_equals_model(small, name, graphs):
    """Graph-captured batched scoring gives model(x)'s scores (short rows are
    masked by the caller, as model(x) does)."""
    from gkmsvm_lite_b200.batch import BatchedScorer

    c = small[name]
    m = _model(c, use_lmer_table=False)
    x, xl = c["x"][:-1], c["x_lengths"][:-1]
    bs = BatchedScorer(m, use_graphs=graphs)
    for _ in range(3):  # eager, capture + replay, replay
        got = _np(bs.score(torch.from_numpy(x).cuda(), torch.from_numpy(xl).cuda()))
        np.testing.assert_allclose(got, c["scores"][:-1, 0], rtol=RTOL, atol=ATOL)


def test_batched_scorer_config1_table_and_index():
    import gkmsvm_lite_b200.synthetic as syn
    from gkmsvm_lite_b200.batch import BatchedScorer

    w = syn.config1()
    want = np.load(os.path.join(GOLDEN, "config1.npz"))["scores"][:, 0]
    for table in (False, True):
        m = gk.GkmSVM(w.sv, w.coef, 0.0, "gkm_esttrunc", {"L": 11, "k": 7, "d": 3}).cuda()
        m.use_lmer_table = table
        bs = BatchedScorer(m)
        x = torch.from_numpy(w.x).cuda()
        for _ in range(3):  # eager, capture + replay, replay
            np.testing.assert_allclose(_np(bs.score(x)), want, rtol=RTOL, atol=ATOL)


def test_bucket_words_of_large_tiles():
    """48,000 SVs of 500 bp: an SV tile holds more than 2^24 index entries
    (one tile of 47M with packed counters), more bits of bucket begin than 24,
    so the bucket words keep fewer than 8 bits of length (a bucket that long
    reads its end from the offsets).  Profiles bit-exact to the all-pairs
    forms, scores equal to the oracle's."""
    import gkmsvm_lite_b200.synthetic as syn

    rng = np.random.default_rng(41)
    n_sv = 48000
    sv = syn.random_codes(rng, n_sv, 500)
    sv[:3] = 0  # poly-A SVs: one bucket of ~1,500 entries per tile
    coef = rng.normal(0, 0.1, n_sv)
    xl = np.array([500, 320, 75, 11])
    x = syn.ragged_codes(rng, xl)
    x[0, 100:200] = 0
    params = {"L": 11, "k": 7, "d": 3, "gamma": 2.0}
    m = gk.GkmSVM(sv, coef, 0.0, "gkmrbf", params).cuda()
    m.use_lmer_table = False
    index = m._sv_index()
    assert index.entries / index.tiles > 2**24
    spec = m._spec()
    fwd, rc, counts = engine.pack(spec, torch.from_numpy(x).cuda(), xl)
    _, p_index = index.pairwise(fwd, counts, raw=False, profile=True)
    by, ry, cy = m._sv_packed()
    _, p = engine.pairwise(spec, fwd, counts, by, ry, cy, raw=False, profile=True, method="dense")
    assert torch.equal(p, p_index)
    kd = orc.KernelDef.from_params("gkmrbf", params)
    want = orc.IndexBaseline(orc.OracleModel(sv, None, coef, 0.0, kd), threads=8).scores(x, xl, threads=8)
    np.testing.assert_allclose(_np(m(x, lengths=xl)).ravel(), want.ravel(), rtol=RTOL, atol=ATOL)


def test_large_neighbourhood_index_past_reference_limit():
    """t=0 gkm_cnt l=11 k=7 with no d (31,714 neighbour masks, read from global
    memory) on 1,500 SVs: the index serves it (its measured cost is below the
    all-pairs forms'), with profiles bit-exact to the tensor-core form and the
    join and scores equal to the oracle's."""
    import gkmsvm_lite_b200.synthetic as syn

    rng = np.random.default_rng(31)
    svl = rng.integers(200, 400, 1500)
    sv = syn.ragged_codes(rng, svl)
    coef = rng.normal(0, 0.2, 1500)
    xl = rng.integers(30, 600, 12)
    xl[0] = 599
    x = syn.ragged_codes(rng, xl)
    params = {"L": 11, "k": 7}
    m = gk.GkmSVM(sv, coef, 0.1, "gkm_cnt", params, sv_lengths=svl).cuda()
    m.use_lmer_table = False
    assert m._sv_index() is not None and m._sv_index().masks.numel() == 31714
    spec = m._spec()
    fwd, rc, counts = engine.pack(spec, torch.from_numpy(x).cuda(), xl)
    _, p_index = m._sv_index().pairwise(fwd, counts, raw=False, profile=True)
    by, ry, cy = m._sv_packed()
    for method in engine.pairwise_forms(spec):
        _, p = engine.pairwise(spec, fwd, counts, by, ry, cy, raw=False, profile=True, method=method)
        assert torch.equal(p, p_index), method
    kd = orc.KernelDef.from_params("gkm_cnt", params)
    want = orc.scores(orc.OracleModel(sv, svl, coef, 0.1, kd), x, xl)
    np.testing.assert_allclose(_np(m(x, lengths=xl)), want, rtol=RTOL, atol=ATOL)
