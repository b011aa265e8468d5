"""The CPU oracle against gkmsvm-lite's own outputs (tests/golden/small.npz,
config1.npz) and LS-GKM's gkmpredict / gkmexplain fixtures.  Pins the oracle
before any GPU result is compared with it."""

import os

import numpy as np
import pytest

from conftest import GOLDEN, LSGKM, codes_of, read_fasta, read_lsgkm_explain, read_pred
from oracle import oracle as orc

CASES = ["t2", "t2norc", "t0", "t0small", "t1", "t3", "t4", "t5", "t6"]


def _model(c):
    kd = orc.KernelDef.from_params(c["kernel_type"], c["params"])
    return orc.OracleModel(c["sv"], c["sv_lengths"], c["coef"], float(c["bias"]), kd)


def _rows(c):
    return c["x"], c["x_lengths"]


@pytest.mark.parametrize("name", CASES)
def test_raw_and_self_kernels(small, name):
    c = small[name]
    m = _model(c)
    x, xl = _rows(c)
    raw, dx, ds = orc.kernel_values(m, x, xl)
    np.testing.assert_allclose(raw, c["raw"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(dx, c["diag_x"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(ds, c["diag_sv"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("name", CASES)
def test_scores(small, name):
    c = small[name]
    m = _model(c)
    x, xl = _rows(c)
    got = orc.scores(m, x, xl)
    np.testing.assert_allclose(got, c["scores"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(got, c["scores_join"], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("name", CASES)
def test_variants_and_impact(small, name):
    c = small[name]
    m = _model(c)
    ref, rl = c["x"][:-1], c["x_lengths"][:-1]
    alt, al = c["alt"], c["alt_lengths"]
    L = max(ref.shape[1], alt.shape[1])
    ref = np.pad(ref, ((0, 0), (0, L - ref.shape[1])))
    alt = np.pad(alt, ((0, 0), (0, L - alt.shape[1])))
    np.testing.assert_allclose(orc.score_variants(m, ref, alt, rl, al), c["variant_kernel"],
                               rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(orc.mutation_impact(m, ref, alt, rl, al), c["variant_impact"],
                               rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("name", CASES)
def test_ism(small, name):
    c = small[name]
    m = _model(c)
    x, xl = _rows(c)
    got = orc.ism(m, x, xl)
    np.testing.assert_allclose(got, c["ism"], rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("mode,key", [("hypothetical", "explain_hyp"),
                                      ("importance", "explain_imp"),
                                      ("perturbation", "explain_pert")])
def test_explain(small, name, mode, key):
    c = small[name]
    m = _model(c)
    x, xl = _rows(c)
    got = orc.gkmexplain(m, x, xl, mode)
    np.testing.assert_allclose(got, c[key], rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("name", CASES)
def test_gram(small, name):
    c = small[name]
    m = _model(c)
    got = orc.gram(m.kd, c["sv"], c["sv_lengths"])
    np.testing.assert_allclose(got, c["gram"], rtol=1e-10, atol=1e-12)
    assert (got == got.T).all()


def test_esttrunc_table_is_lsgkm_weights():
    """h(m) of gkm_esttrunc l=11 k=7 d=3 equals the reference's table."""
    import ast
    z = np.load(os.path.join(GOLDEN, "small.npz"))
    kd = orc.KernelDef.from_params("gkm_esttrunc", ast.literal_eval(str(z["t2/params"])))
    assert kd.dmax == 3 and kd.h[4:].sum() == 0 and (kd.h[:4] > 0).all()


def test_config1_index_baseline():
    """The threaded index baseline gives the reference's scores for the first
    40 config-1 queries (2,000 SVs x 300 bp, t=2)."""
    import gkmsvm_lite_b200.synthetic as syn

    w = syn.config1()
    kd = orc.KernelDef.from_params("gkm_esttrunc", {"L": 11, "k": 7, "d": 3})
    m = orc.OracleModel(w.sv, None, w.coef, 0.0, kd)
    ib = orc.IndexBaseline(m)
    got = ib.scores(w.x[:40], None, threads=4)
    want = np.load(os.path.join(GOLDEN, "config1.npz"))["scores"][:40]
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-12)


_WGKM = ["t0", "t1", "t2", "t2w2", "t3", "t4", "t4w05", "t5", "t6"]


@pytest.mark.parametrize("t", _WGKM)
@pytest.mark.parametrize("n", [85, 100])
def test_lsgkm_gkmpredict(t, n):
    """Scores equal LS-GKM gkmpredict (6 significant digits printed)."""
    m = orc.load_lsgkm(os.path.join(LSGKM, f"lsgkm_wgkm_{t}.model.txt.gz"))
    _, seqs = read_fasta(os.path.join(LSGKM, f"lsgkm_wgkm_test{n}.fa"))
    x, xl = codes_of(seqs)
    want = read_pred(os.path.join(LSGKM, f"lsgkm_wgkm_{t}_test{n}.pred.txt"))
    got = orc.scores(m, x, xl if (xl != xl.max()).any() else None)[:, 0]
    np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-5)


@pytest.mark.parametrize("t", ["t2", "t4", "t5"])
def test_lsgkm_ragged_models(t):
    m = orc.load_lsgkm(os.path.join(LSGKM, f"lsgkm_ragged_{t}.model.txt.gz"))
    assert m.sv_lengths is not None
    _, seqs = read_fasta(os.path.join(LSGKM, "lsgkm_ragged_test.fa"))
    x, xl = codes_of(seqs)
    want = read_pred(os.path.join(LSGKM, f"lsgkm_ragged_{t}_test.pred.txt"))
    got = orc.scores(m, x, xl)[:, 0]
    np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-5)


@pytest.mark.parametrize("t", ["t0", "t1", "t4", "t5", "t6"])
@pytest.mark.parametrize("lm,mode", [(0, "importance"), (1, "hypothetical"), (4, "perturbation")])
def test_lsgkm_gkmexplain(t, lm, mode):
    m = orc.load_lsgkm(os.path.join(LSGKM, f"lsgkm_wgkm_{t}.model.txt.gz"))
    _, seqs = read_fasta(os.path.join(LSGKM, "lsgkm_wgkm_test85.fa"))
    x, xl = codes_of(seqs)
    want = read_lsgkm_explain(os.path.join(LSGKM, f"lsgkm_wgkm_{t}_test85.explain{lm}.txt.gz"))
    got = orc.gkmexplain(m, x, xl if (xl != xl.max()).any() else None, mode)
    np.testing.assert_allclose(got, want, rtol=2e-5, atol=5e-6 * np.abs(want).max())


@pytest.mark.parametrize("kind", ["est", "rbf"])
def test_lsgkm_mutation_impact(kind):
    """gkmexplain -m 5 on the centre base of each test51 sequence."""
    m = orc.load_lsgkm(os.path.join(LSGKM, f"lsgkm_mode5_{kind}.model.txt.gz"))
    _, seqs = read_fasta(os.path.join(LSGKM, "lsgkm_mode5_test51.fa"))
    rows = [line.split("\t") for line in open(os.path.join(LSGKM, f"lsgkm_mode5_{kind}.txt"))]
    want = np.array([[float(v) for v in r[2].split(",")] for r in rows])
    c = len(seqs[0]) // 2
    ref, alt = [], []
    for s in seqs:
        for b in "ACGT":
            ref.append(s)
            alt.append(s[:c] + b + s[c + 1:])
    rx, _ = codes_of(ref)
    ax, _ = codes_of(alt)
    got = orc.mutation_impact(m, rx, ax).reshape(-1, 4)
    np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-6)
    pred = read_pred(os.path.join(LSGKM, f"lsgkm_mode5_{kind}.pred.txt"))
    x, _ = codes_of(seqs)
    np.testing.assert_allclose(orc.scores(m, x)[:, 0], pred, rtol=1e-4, atol=1e-6)


def test_encode_10sv_gkmpredict():
    m = orc.load_lsgkm(os.path.join(LSGKM, "encode_ENCFF579AOX_10sv.model.txt.gz"))
    rows = [line.rstrip("\n").split("\t") for line in open(os.path.join(LSGKM, "encode_10sv_gkmpredict.tsv"))]
    for i, (name, seq, want) in enumerate(rows):
        if name.startswith("sv"):
            x = m.sv[i:i + 1, : (m.sv_lengths[i] if m.sv_lengths is not None else m.sv.shape[1])]
        else:
            x, _ = codes_of([seq])
        assert abs(orc.scores(m, x)[0, 0] - float(want)) < 1e-4


def test_encode_72k_model_index_baseline():
    """The full 72,145-SV ENCODE model: the oracle's CPU index path (the bench's
    CPU baseline) against gkmsvm-lite's t2 and gkmrbf gamma=1 scores of 64
    synthetic 300 bp queries."""
    z = np.load(os.path.join(GOLDEN, "encode.npz"))
    m = orc.load_lsgkm(os.path.join(LSGKM, "encode_ENCFF579AOX.model.txt.gz"))
    assert len(m.coef) == 72145
    threads = os.cpu_count() or 1
    for kt, params, key in (("gkm_esttrunc", {"L": 11, "k": 7, "d": 3}, "t2"),
                            ("gkmrbf", {"L": 11, "k": 7, "d": 3, "gamma": 1.0}, "t3")):
        mk = orc.OracleModel(m.sv, m.sv_lengths, m.coef, m.bias, orc.KernelDef.from_params(kt, params))
        got = orc.IndexBaseline(mk, threads=threads).scores(z["x"], threads=threads)
        # summing 72,145 terms in another order leaves ~1e-11 on near-zero
        # scores: atol relative to the largest score, as the reference's own
        # large-model GPU tests do (tests/test_gpu.py:783-784)
        np.testing.assert_allclose(got, z[key], rtol=1e-9, atol=1e-10 * np.abs(z[key]).max())


@pytest.fixture(scope="module")
def deltasvm_golden():
    z = np.load(os.path.join(GOLDEN, "deltasvm.npz"))
    return {k: z[k] for k in z.files}


@pytest.mark.parametrize("name", CASES)
def test_deltasvm_weights(small, deltasvm_golden, name):
    """to_deltasvm weights at the fixture's l-mers, with and without query_norm."""
    c, g = small[name], deltasvm_golden
    m = _model(c)
    idx = g[f"{name}/idx"]
    for key, qn in (("w", False), ("wq", True)):
        want = g[f"{name}/{key}"]
        got = orc.deltasvm_weights(m, qn, idx)
        np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-12 * max(1.0, np.abs(want).max()))
