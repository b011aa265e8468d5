"""Classic (C++) and R gkmSVM models as their tools wrote them, after
gkmsvm-lite's tests/test_importers/test_gkmsvm_tools.py: the importers on the
host, the oracle's scores against gkmsvm_kernel's own (a third-party pin of
the kernel at l=10 k=6 d=3 for the three filter types), and, on the GPU, the
model's scores against the same files."""

import os
import re

import numpy as np
import pytest

import gkmsvm_lite_b200 as gk
from conftest import GOLDEN, LSGKM, codes_of, read_fasta
from oracle import oracle as orc

TOOLS = os.path.join(GOLDEN, "gkmsvm")
# (fixture prefix, loader, gkmsvm_kernel -t / R useTgkm); l=10 k=6 d=3
MODELS = [
    ("gkmsvm_classic_t0", "classic", 0),
    ("gkmsvm_classic_t1", "classic", 1),
    ("gkmsvm_classic_t2", "classic", 2),
    ("gkmsvm_r_t1", "r", 1),
    ("gkmsvm_r_t2", "r", 2),
]


def _load(prefix, tool, filter_type):
    alpha = os.path.join(TOOLS, f"{prefix}_svalpha.out")
    with pytest.warns(UserWarning, match="other than ACGT, dropped"):
        if tool == "r":
            return gk.load_r_gkmsvm_model(alpha, useTgkm=filter_type)
        if filter_type == 1:  # the tools' default kernel
            return gk.load_classic_model(alpha)
        return gk.load_classic_model(alpha, filter_type=filter_type)


def _scores(path):
    return dict((line.split()[0], float(line.split()[1])) for line in open(path) if line.strip())


def _queries(test):
    names, seqs = read_fasta(os.path.join(LSGKM, f"lsgkm_wgkm_{test}.fa"))
    return [n.split()[0] for n in names], [re.sub("[^ACGT]", "", s) for s in seqs]


@pytest.mark.parametrize("prefix, tool, filter_type", MODELS)
@pytest.mark.parametrize("test", ["test100", "test85"])
def test_oracle_matches_gkmsvm_kernel(prefix, tool, filter_type, test):
    """The oracle's sum_i alpha_i K(x, sv_i) (normalised, no bias) equals
    gkmsvm_kernel's, printed to 7 significant digits; gkmsvm_classify's own
    output is within 3 % of it."""
    m = _load(prefix, tool, filter_type)
    assert m.bias == 0.0 and m.sv_lengths is not None  # N dropped: ragged SVs
    kd = orc.KernelDef.from_params(m.kernel_type, m.kernel_params)
    om = orc.OracleModel(m.support_sequences, m.sv_lengths, m.coefficients, 0.0, kd)
    names, seqs = _queries(test)
    x, xl = codes_of(seqs)
    got = orc.scores(om, x, xl).ravel()
    want = _scores(os.path.join(TOOLS, f"{prefix}_{test}_kernel.txt"))
    np.testing.assert_allclose(got, [want[n] for n in names], rtol=1e-5, atol=1e-6)
    classify = _scores(os.path.join(TOOLS, f"{prefix}_{test}_classify.txt"))
    assert np.abs(got - [classify[n] for n in names]).max() < 0.03


@pytest.mark.gpu
@pytest.mark.parametrize("prefix, tool, filter_type", MODELS)
@pytest.mark.parametrize("test", ["test100", "test85"])
def test_gpu_scores_match_gkmsvm_kernel(prefix, tool, filter_type, test):
    m = _load(prefix, tool, filter_type).cuda()
    names, seqs = _queries(test)
    got = m(seqs).cpu().numpy().ravel()
    want = _scores(os.path.join(TOOLS, f"{prefix}_{test}_kernel.txt"))
    np.testing.assert_allclose(got, [want[n] for n in names], rtol=1e-5, atol=1e-6)
    kd = orc.KernelDef.from_params(m.kernel_type, m.kernel_params)
    x, xl = codes_of(seqs)
    oracle = orc.scores(orc.OracleModel(m.support_sequences, m.sv_lengths, m.coefficients, 0.0, kd), x, xl).ravel()
    np.testing.assert_allclose(got, oracle, rtol=1e-9, atol=1e-12)


def _write(tmp_path, alphas, seqs):
    alpha = tmp_path / "m_svalpha.out"
    alpha.write_text("".join(f"{i}\t{a:e}\n" for i, a in alphas.items()))
    (tmp_path / "m_svseq.fa").write_text("".join(f">{i}\n{s}\n" for i, s in seqs.items()))
    return alpha


def test_svs_matched_by_id(tmp_path):
    """Each alpha picks its SV by id (extra FASTA records ignored, lower case
    read as upper case); an id missing from the FASTA is an error."""
    seqs = {"a": "ACGTTGCAAGGTC", "b": "ttgacgatcgaat", "c": "GGGCCCATATAGC"}
    m = gk.load_classic_model(_write(tmp_path, {"c": 0.5, "b": -0.3}, seqs), L=5, k=3)
    assert m.num_support_vectors == 2 and m.bias == 0.0
    np.testing.assert_array_equal(m.support_sequences,
                                  np.stack([gk.encode_codes(seqs[i].upper()) for i in ("c", "b")]))
    np.testing.assert_array_equal(m.coefficients, [0.5, -0.3])
    with pytest.raises(ValueError, match="not in"):
        gk.load_classic_model(_write(tmp_path, {"a": 1.0, "z": 1.0}, seqs), L=5, k=3)


def test_kernel_arguments(tmp_path):
    alpha = _write(tmp_path, {"a": 1.0}, {"a": "ACGTTGCAAGGTCAT"})
    m = gk.load_classic_model(alpha, L=6, k=4, d=2, filter_type=0, include_rc=False)
    assert m.kernel_type == "gkm_estfull"
    assert (m.kernel.l, m.kernel.k, m.kernel.d) == (6, 4, 2) and not m.kernel.include_rc
    r = gk.load_r_gkmsvm_model(alpha, L=6, K=4, maxnmm=2, useTgkm=0, addRC=False)
    assert r.kernel_params == m.kernel_params
    with pytest.raises(NotImplementedError, match="wildcard"):
        gk.load_classic_model(alpha, filter_type=3)


def test_malformed_alpha_file(tmp_path):
    alpha = tmp_path / "m_svalpha.out"
    alpha.write_text("svm_type c_svc\nrho 0.1 0.2\n")
    (tmp_path / "m_svseq.fa").write_text(">a\nACGT\n")
    with pytest.raises(ValueError):
        gk.load_classic_model(alpha)
    with pytest.raises(ValueError, match="give svseq_path"):
        gk.load_classic_model(tmp_path / "alphas.txt")
