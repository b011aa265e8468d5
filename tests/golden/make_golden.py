"""Generate the golden fixtures in this directory from gkmsvm-lite itself.

Run in a container that has the reference source tree (never on a GPU box):

    GKMSVM_LITE_ROOT=<gkmsvm-lite checkout> NUMBA_CACHE_DIR=/tmp/nbcache \
        python tests/golden/make_golden.py [groups...]

groups: small (every kernel type on small ragged inputs: raw kernel values,
self-kernels, scores, ISM, GkmExplain in three modes, variant scores, mutation
impact, Gram), config1, config2, config3, config4, config5 (subsamples of the
benchmark workloads), lsgkm (copies LS-GKM's gkmpredict / gkmexplain outputs
and their models from gkmsvm-lite's test fixtures), deltasvm (to_deltasvm
weights of the small models), gkmsvm (classic C++ / R gkmSVM models with the
gkmSVM tools' own scores, from gkmsvm-lite's test fixtures), files (model
files gkmsvm-lite's serialization writes).  Inputs are regenerated in
the tests from the same seeds through gkmsvm_lite_b200.synthetic, or stored
here when small.
"""

from __future__ import annotations

import os
import shutil
import sys
import time

import numpy as np

# the gkmsvm-lite source tree: GKMSVM_LITE_ROOT, else the read-only mount of
# the container the fixtures were made in
REF_ROOT = os.environ.get("GKMSVM_LITE_ROOT", "/root/reference")
REF_SRC = os.path.join(REF_ROOT, "src")
REF_FIXTURES = os.path.join(REF_ROOT, "tests", "fixtures")
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, REF_SRC)

import gkmsvm_lite_b200.synthetic as syn  # noqa: E402

from gkmsvm import ism as ref_ism  # noqa: E402
from gkmsvm.explain import gkmexplain, mutation_impact  # noqa: E402
from gkmsvm.gram import compute_gram  # noqa: E402
from gkmsvm.svm import GkmSVM  # noqa: E402

# (name, kernel_type, params, n_sv, sv length range, n_query, query length range, seed)
SMALL = [
    ("t2", "gkm_esttrunc", {"L": 11, "k": 7, "d": 3}, 14, (40, 70), 6, (30, 60), 11),
    ("t2norc", "gkm_esttrunc", {"L": 8, "k": 5, "d": 2, "include_rc": False}, 10, (25, 40), 5, (20, 45), 12),
    ("t0", "gkm_cnt", {"L": 7, "k": 4}, 9, (20, 30), 5, (15, 35), 13),
    ("t0small", "gkm_cnt", {"L": 3, "k": 2}, 5, (15, 15), 3, (15, 15), 14),
    ("t1", "gkm_estfull", {"L": 8, "k": 5, "d": 2}, 10, (30, 45), 5, (25, 50), 15),
    ("t3", "gkmrbf", {"L": 10, "k": 6, "d": 3, "gamma": 2.0}, 12, (40, 60), 5, (30, 70), 16),
    ("t4", "wgkm", {"L": 9, "k": 6, "d": 2, "M": 20, "H": 10.0}, 10, (30, 60), 5, (25, 60), 17),
    ("t5", "wgkmrbf", {"L": 10, "k": 6, "d": 3, "gamma": 1.0}, 12, (40, 70), 5, (30, 70), 18),
    ("t6", "gkm_cnt_rbf", {"L": 8, "k": 5, "d": 2, "gamma": 1.5}, 10, (30, 45), 5, (20, 45), 19),
]


def _ragged(rng, n, lo, hi):
    lengths = rng.integers(lo, hi + 1, n).astype(np.int64)
    return syn.ragged_codes(rng, lengths), lengths


def small():
    out = {}
    for name, kt, params, n_sv, svr, n_q, qr, seed in SMALL:
        t0 = time.time()
        rng = np.random.default_rng(seed)
        sv, svl = _ragged(rng, n_sv, *svr)
        coef = rng.normal(size=n_sv)
        x, xl = _ragged(rng, n_q, *qr)
        xl[-1] = params["L"] - 2  # one row shorter than l: NaN outputs
        x[-1, xl[-1]:] = 0
        alt, altl = syn.variant_pairs(rng, x[:-1], xl[:-1], indel_rate=0.4)
        m = GkmSVM(sv, coef, -0.15, kt, params, sv_lengths=svl)
        base = m.kernel.base
        bx, bx_rc = base.pack_both(x, xl)
        by, by_rc = base.pack_both(sv, svl)
        base.use_masked = False
        raw = base.raw_packed(bx, by, by_rc)
        base.use_masked = True
        d = {
            "kernel_type": kt, "params": repr(params), "sv": sv, "sv_lengths": svl,
            "coef": coef, "bias": -0.15, "x": x, "x_lengths": xl, "alt": alt,
            "alt_lengths": altl, "raw": raw,
            "diag_x": base.raw_diag_packed(bx, bx_rc), "diag_sv": base.raw_diag_packed(by, by_rc),
            "scores": m(x, lengths=xl),
            "ism": ref_ism(m, x, lengths=xl),
            "explain_hyp": gkmexplain(m, x, lengths=xl, mode="hypothetical"),
            "explain_imp": gkmexplain(m, x, lengths=xl, mode="importance"),
            "explain_pert": gkmexplain(m, x, lengths=xl, mode="perturbation"),
            "variant_kernel": m.score_variants(x[:-1], alt, ref_lengths=xl[:-1], alt_lengths=altl),
            "variant_impact": m.score_variants(
                x[:-1], alt, method="gkmexplain", ref_lengths=xl[:-1], alt_lengths=altl),
            "gram": compute_gram(m.kernel, sv, lengths=svl),
        }
        m2 = GkmSVM(sv, coef, -0.15, kt, params, sv_lengths=svl)
        m2.use_lmer_index = False
        m2.use_lmer_table = False
        d["scores_join"] = m2(x, lengths=xl)
        for k, v in d.items():
            out[f"{name}/{k}"] = np.asarray(v)
        print(f"small {name}: {time.time() - t0:.1f}s", flush=True)
    np.savez_compressed(os.path.join(HERE, "small.npz"), **out)


def config1():
    w = syn.config1()
    m = GkmSVM(w.sv, w.coef, 0.0, "gkm_esttrunc", {"L": 11, "k": 7, "d": 3})
    t = time.time()
    s = m(w.x)
    print(f"config1: {time.time() - t:.1f}s", flush=True)
    m.use_lmer_table = False
    np.savez_compressed(os.path.join(HERE, "config1.npz"), scores=s,
                        diag_sv=m._sv_diag())


def _model72k(kt, params):
    sv, svl, coef = syn.config3_model()
    return GkmSVM(sv, coef, 0.0, kt, params, sv_lengths=svl)


def config3_rows(xl, n_first=224, n_long=32, pool=20000):
    """The first n_first queries of the config-3 stream and the n_long
    longest of its first `pool` (2,000 bp rows included)."""
    longest = np.argsort(-xl[:pool], kind="stable")
    extra = [int(i) for i in longest if i >= n_first][:n_long]
    return np.concatenate([np.arange(n_first), np.asarray(extra, np.int64)])


def config3():
    xq, xl, _ = syn.config3_queries()
    out = {}
    for name, kt, params, rows in (
        ("t2", "gkm_esttrunc", {"L": 11, "k": 7, "d": 3}, np.arange(256)),
        ("t3", "gkmrbf", {"L": 11, "k": 7, "d": 3, "gamma": 2.0}, config3_rows(xl)),
    ):
        m = _model72k(kt, params)
        m.use_lmer_table = False
        t = time.time()
        L = int(xl[rows].max())
        out[f"{name}/scores"] = m(xq[rows, :L], lengths=xl[rows])
        out[f"{name}/rows"] = rows
        print(f"config3 {name} {len(rows)}: {time.time() - t:.1f}s", flush=True)
        if name == "t2":
            out["t2/diag_sv_head"] = np.asarray(m._sv_diag())[:256]
    np.savez_compressed(os.path.join(HERE, "config3.npz"), **out)


MASK_PLAN_KERNELS = [(kt, params) for _, kt, params, *_ in SMALL] + [
    ("gkm_esttrunc", {"L": 11, "k": 7, "d": 3}), ("gkm_cnt", {"L": 11, "k": 7}),
    ("gkm_estfull", {"L": 10, "k": 6}), ("gkm_cnt", {"L": 12, "k": 8, "d": 2})]


def maskplan():
    """gkmsvm-lite's masked-join plans (kernels/masked.py:45-69): mask sizes and
    coefficients of the small kernels and a few l = 10..12 ones."""
    from gkmsvm.kernels.masked import mask_plan

    out = {}
    for i, (kt, params) in enumerate(MASK_PLAN_KERNELS):
        base = GkmSVM(np.zeros((1, 20), np.uint8), np.ones(1), 0.0, kt, params).kernel.base
        plan = mask_plan(tuple(float(v) for v in base._mismatch_table), base.l, base._min_matches)
        out[f"{i}/kernel"] = np.array(f"{kt} {params!r}")
        out[f"{i}/none"] = np.array(plan is None)
        if plan is not None:
            out[f"{i}/sizes"] = np.array([j for j, _, _ in plan])
            out[f"{i}/coefs"] = np.array([c for _, c, _ in plan])
            out[f"{i}/positions_sum"] = np.array([int(p.sum()) for _, _, p in plan])
    np.savez_compressed(os.path.join(HERE, "maskplan.npz"), **out)


ENCODE_MODEL = "encode_ENCFF579AOX.model.txt.gz"


def encode():
    """The full 72,145-SV ENCODE model (t2, l=11 k=7 d=3) the reference's
    throughput benchmark scores (benchmarks/throughput_sweep.py:66-68), copied
    beside the LS-GKM fixtures, with gkmsvm-lite's scores of 64 synthetic
    300 bp queries (seed 6) for t2 and for the same SVs as gkmrbf gamma=1."""
    from gkmsvm import load_model

    dst = os.path.join(HERE, "lsgkm")
    shutil.copy(os.path.join(REF_FIXTURES, ENCODE_MODEL), os.path.join(dst, ENCODE_MODEL))
    x = syn.random_codes(np.random.default_rng(6), 64, 300)
    full = load_model(os.path.join(dst, ENCODE_MODEL))
    out = {"x": x}
    t = time.time()
    out["t2"] = full(x)
    rbf = GkmSVM(full.support_sequences, full.coefficients, full.bias, "gkmrbf",
                 {**full.kernel_params, "gamma": 1.0})
    out["t3"] = rbf(x)
    print(f"encode: {time.time() - t:.1f}s", flush=True)
    np.savez_compressed(os.path.join(HERE, "encode.npz"), **out)


def config4():
    x = syn.config4_queries()[:16]
    m = _model72k("gkm_esttrunc", {"L": 11, "k": 7, "d": 3})
    t = time.time()
    out = {"ism": ref_ism(m, x)}
    print(f"config4 ism: {time.time() - t:.1f}s", flush=True)
    t = time.time()
    out["explain_hyp"] = gkmexplain(m, x, mode="hypothetical")
    print(f"config4 explain: {time.time() - t:.1f}s", flush=True)
    np.savez_compressed(os.path.join(HERE, "config4.npz"), **out)


def config2():
    X, lengths = syn.config2()
    from gkmsvm.kernels.weighted import CenterWeightedGkmKernel

    k = CenterWeightedGkmKernel(11, 7, d=3)
    t = time.time()
    rows = compute_gram(k, X[:48], X, lengths=lengths[:48], y_lengths=lengths)
    sym = compute_gram(k, X[:160], lengths=lengths[:160])
    print(f"config2: {time.time() - t:.1f}s", flush=True)
    np.savez_compressed(os.path.join(HERE, "config2.npz"), rows=rows, sym=sym)


def config5():
    m = _model72k("wgkmrbf", {"L": 11, "k": 7, "d": 3, "gamma": 1.0})
    rng = np.random.default_rng(4)
    lengths = syn.log_uniform_lengths(rng, 24, 20, 2000)
    lengths[3] = 9  # shorter than l
    x = syn.ragged_codes(rng, lengths)
    t = time.time()
    out = {"x": x, "x_lengths": lengths, "scores": m(x, lengths=lengths)}
    ref = x[:6, :400]
    rl = np.minimum(lengths[:6], 400)
    rl[3] = 400
    ref[3, 9:] = syn.random_codes(rng, 1, 391)[0]
    alt, al = syn.variant_pairs(rng, ref, rl)
    out.update(ref=ref, ref_lengths=rl, alt=alt, alt_lengths=al,
               variants=m.score_variants(ref, alt, ref_lengths=rl, alt_lengths=al))
    xi = x[:1, :150]
    out["ism_x"] = xi
    out["ism"] = ref_ism(m, xi)
    out["explain_hyp"] = gkmexplain(m, xi, mode="hypothetical")
    print(f"config5: {time.time() - t:.1f}s", flush=True)
    np.savez_compressed(os.path.join(HERE, "config5.npz"), **out)


LSGKM_FILES = (
    [f"lsgkm_wgkm_{t}.model.txt.gz" for t in ("t0", "t1", "t2", "t2w2", "t3", "t4", "t4w05", "t5", "t6")]
    + [f"lsgkm_wgkm_{t}_test{n}.pred.txt" for t in ("t0", "t1", "t2", "t2w2", "t3", "t4", "t4w05", "t5", "t6") for n in (85, 100)]
    + ["lsgkm_wgkm_test85.fa", "lsgkm_wgkm_test100.fa"]
    + [f"lsgkm_wgkm_{t}_test85.explain{m}.txt.gz" for t in ("t0", "t1", "t4", "t5", "t6") for m in (0, 1, 4)]
    + [f"lsgkm_mode5_{k}{s}" for k in ("est", "rbf") for s in (".model.txt.gz", ".pred.txt", ".txt")]
    + ["lsgkm_mode5_test51.fa"]
    + [f"lsgkm_mode5_{k}.explain{m}.txt.gz" for k in ("est", "rbf") for m in (0, 1, 4)]
    + [f"lsgkm_ragged_{t}.model.txt.gz" for t in ("t2", "t4", "t5")]
    + [f"lsgkm_ragged_{t}_test.pred.txt" for t in ("t2", "t4", "t5")]
    + ["lsgkm_ragged_test.fa", "encode_ENCFF579AOX_10sv.model.txt.gz"]
)


def lsgkm():
    dst = os.path.join(HERE, "lsgkm")
    os.makedirs(dst, exist_ok=True)
    for f in LSGKM_FILES:
        shutil.copy(os.path.join(REF_FIXTURES, f), os.path.join(dst, f))
    # gkmpredict on the 10-SV ENCODE model (tests/test_importers/
    # test_encode_integration.py:119-124): the first three SVs and a random
    # 300 bp sequence from random.seed(42)
    import random

    random.seed(42)
    rand_seq = "".join(random.choice("ACGT") for _ in range(300))
    with open(os.path.join(dst, "encode_10sv_gkmpredict.tsv"), "w") as f:
        for name, v in (("sv0", 0.944171), ("sv1", 0.922764), ("sv2", 0.977893)):
            f.write(f"{name}\t\t{v}\n")
        f.write(f"random\t{rand_seq}\t-0.123703\n")


GKMSVM_PREFIXES = ["gkmsvm_classic_t0", "gkmsvm_classic_t1", "gkmsvm_classic_t2", "gkmsvm_r_t1", "gkmsvm_r_t2"]


def gkmsvm():
    """Copies the classic C++ and R gkmSVM models of gkmsvm-lite's fixtures
    (svalpha.out + svseq.fa, l=10 k=6 d=3) with gkmsvm_kernel's and
    gkmsvm_classify's scores of the 100 and 85 bp test sets (the test FASTA
    files are in lsgkm/)."""
    dst = os.path.join(HERE, "gkmsvm")
    os.makedirs(dst, exist_ok=True)
    for p in GKMSVM_PREFIXES:
        for suffix in ("_svalpha.out", "_svseq.fa", "_test100_kernel.txt", "_test85_kernel.txt",
                       "_test100_classify.txt", "_test85_classify.txt"):
            shutil.copy(os.path.join(REF_FIXTURES, p + suffix), os.path.join(dst, p + suffix))


def files():
    """Model files written by gkmsvm-lite itself (serialization.py): the t4
    and t2norc small models as npz and LS-GKM text (plain and gzip), and the
    t0small model's DeltaSVM weights as npz."""
    from gkmsvm.serialization import save_deltasvm_npz, save_lsgkm, save_npz

    dst = os.path.join(HERE, "files")
    os.makedirs(dst, exist_ok=True)
    for name, kt, params, n_sv, svr, n_q, qr, seed in SMALL:
        if name not in ("t4", "t2norc", "t0small"):
            continue
        rng = np.random.default_rng(seed)
        sv, svl = _ragged(rng, n_sv, *svr)
        coef = rng.normal(size=n_sv)
        m = GkmSVM(sv, coef, -0.15, kt, params, sv_lengths=svl)
        if name == "t0small":
            save_deltasvm_npz(m.to_deltasvm(), os.path.join(dst, f"{name}_deltasvm.npz"))
            continue
        save_npz(m, os.path.join(dst, f"{name}.npz"))
        save_lsgkm(m, os.path.join(dst, f"{name}.model.txt"))
        save_lsgkm(m, os.path.join(dst, f"{name}.model.txt.gz"))


DELTASVM_FULL = 4**7  # weights stored whole up to this many, else a sample
DELTASVM_SAMPLE = 8192


def deltasvm():
    """to_deltasvm weights (svm.py:706-785) of the small models, with and
    without query_norm: the whole array for l <= 7, else the weights at a
    seeded sample of l-mers and the sum of all of them."""
    out = {}
    for name, kt, params, n_sv, svr, n_q, qr, seed in SMALL:
        t0 = time.time()
        rng = np.random.default_rng(seed)
        sv, svl = _ragged(rng, n_sv, *svr)
        coef = rng.normal(size=n_sv)
        n = 4 ** params["L"]
        idx = (np.arange(n) if n <= DELTASVM_FULL
               else np.sort(np.random.default_rng(5).choice(n, DELTASVM_SAMPLE, replace=False)))
        out[f"{name}/idx"] = idx
        for key, qn in (("w", False), ("wq", True)):
            m = GkmSVM(sv, coef, -0.15, kt, params, sv_lengths=svl)
            w = np.asarray(m.to_deltasvm(query_norm=qn).weights, dtype=np.float64)
            out[f"{name}/{key}"] = w[idx]
            out[f"{name}/{key}_sum"] = w.sum()
        print(f"deltasvm {name}: {time.time() - t0:.1f}s", flush=True)
    np.savez_compressed(os.path.join(HERE, "deltasvm.npz"), **out)


if __name__ == "__main__":
    groups = sys.argv[1:] or ["small", "config1", "config2", "config3", "config4", "config5", "lsgkm", "deltasvm",
                              "gkmsvm", "files", "encode", "maskplan"]
    for g in groups:
        globals()[g]()
