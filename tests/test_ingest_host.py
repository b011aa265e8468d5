"""Model ingest on the host: the native LS-GKM SV parser (gkm_lsgkm_parse_svs)
behind load_lsgkm_model, and the npz / LS-GKM / DeltaSVM files of
serialization.py, after gkmsvm-lite's tests/test_importers/test_lsgkm.py and
tests/test_serialization.py.  No GPU: models stay on the host."""

import glob
import gzip
import os
import textwrap
import warnings

import numpy as np
import pytest

import gkmsvm_lite_b200 as gk
from conftest import LSGKM
from gkmsvm_lite_b200 import importers
from oracle import oracle as orc

SAMPLE = textwrap.dedent("""\
    svm_type c_svc
    kernel_type gkm_cnt
    L 3
    k 2
    d 3
    nr_class 2
    total_sv 3
    rho 0.25
    label 1 -1
    nr_sv 2 1
    SV
    0.5 ACGT
    0.3 AAAA
    -0.8 CCCC
""")


def _write(tmp_path, text, name="m.model.txt"):
    p = tmp_path / name
    if name.endswith(".gz"):
        with gzip.open(p, "wt") as f:
            f.write(text)
    else:
        p.write_text(text)
    return p


def test_header():
    h = importers._parse_header(SAMPLE.encode())[0]
    assert h["kernel_type"] == "gkm_cnt" and h["L"] == 3 and h["k"] == 2 and h["d"] == 3
    assert h["rho"] == [0.25] and h["label"] == [1, -1] and h["nr_sv"] == [2, 1] and h["norc"] == 0


@pytest.mark.parametrize("name", ["m.model.txt", "m.model.txt.gz"])
def test_basic(tmp_path, name):
    m = gk.load_lsgkm_model(_write(tmp_path, SAMPLE, name))
    assert m.bias == -0.25 and m.kernel.l == 3 and m.kernel.include_rc
    np.testing.assert_array_equal(m.coefficients, [0.5, 0.3, -0.8])
    np.testing.assert_array_equal(m.support_sequences, [[0, 1, 2, 3], [0, 0, 0, 0], [1, 1, 1, 1]])
    assert m.sv_lengths is None
    assert gk.parse_lsgkm_header(_write(tmp_path, SAMPLE, name))["total_sv"] == 3


def test_norc_and_blank_lines_and_case(tmp_path):
    text = SAMPLE.replace("nr_class 2", "norc 1\nnr_class 2").replace("0.3 AAAA", "\n  0.3\tacgn  \n")
    m = gk.load_lsgkm_model(_write(tmp_path, text))
    assert not m.kernel.include_rc
    np.testing.assert_array_equal(m.support_sequences[1], [0, 1, 2, 0])


def test_unsupported_kernel(tmp_path):
    with pytest.raises(NotImplementedError, match="totally_fake_kernel"):
        gk.load_lsgkm_model(_write(tmp_path, SAMPLE.replace("gkm_cnt", "totally_fake_kernel")))


def test_wrong_sv_count(tmp_path):
    with pytest.raises(ValueError, match="Expected 5"):
        gk.load_lsgkm_model(_write(tmp_path, SAMPLE.replace("total_sv 3", "total_sv 5")))


def test_missing_fields_and_malformed_lines(tmp_path):
    with pytest.raises(ValueError, match="rho"):
        gk.load_lsgkm_model(_write(tmp_path, SAMPLE.replace("rho 0.25\n", "")))
    with pytest.raises(ValueError, match="Malformed SV line 2"):
        gk.load_lsgkm_model(_write(tmp_path, SAMPLE.replace("0.3 AAAA", "0.3")))
    with pytest.raises(ValueError, match="Malformed coefficient on SV line 1"):
        gk.load_lsgkm_model(_write(tmp_path, SAMPLE.replace("0.5 ACGT", "0.5x ACGT")))
    with pytest.raises(NotImplementedError):
        gk.load_lsgkm_model(_write(tmp_path, SAMPLE.replace("nr_class 2", "nr_class 3")))


def test_variable_length_svs_load_padded(tmp_path):
    m = gk.load_lsgkm_model(_write(tmp_path, SAMPLE.replace("0.3 AAAA", "0.3 ACGTAC")))
    assert m.support_sequences.shape == (3, 6)
    np.testing.assert_array_equal(m.sv_lengths, [4, 6, 4])
    np.testing.assert_array_equal(m.support_sequences[0], [0, 1, 2, 3, 0, 0])


def test_other_letters_load_as_n(tmp_path):
    with pytest.warns(UserWarning, match="other than ACGTN"):
        m = gk.load_lsgkm_model(_write(tmp_path, SAMPLE.replace("0.3 AAAA", "0.3 ARYA")))
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        n = gk.load_lsgkm_model(_write(tmp_path, SAMPLE.replace("0.3 AAAA", "0.3 ANNA"), "n.model.txt"))
    np.testing.assert_array_equal(m.support_sequences, n.support_sequences)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(LSGKM, "*.model.txt.gz"))),
                         ids=os.path.basename)
def test_fixture_models_match_oracle_parser(path):
    """Every LS-GKM model fixture: coefficients bit-equal (strtod and float()
    both round correctly), codes and lengths equal to the oracle's parse."""
    m = gk.load_lsgkm_model(path)
    o = orc.load_lsgkm(path)
    assert np.array_equal(m.coefficients, o.coef)
    assert m.bias == o.bias
    lengths = m.sv_lengths if m.sv_lengths is not None else np.full(len(m.coefficients), m.support_sequences.shape[1])
    olen = o.sv_lengths if o.sv_lengths is not None else np.full(len(o.coef), o.sv.shape[1])
    np.testing.assert_array_equal(lengths, olen)
    for i in range(len(lengths)):
        np.testing.assert_array_equal(m.support_sequences[i, :lengths[i]], o.sv[i, :lengths[i]])
    assert (m.kernel.l, m.kernel.k, m.kernel.include_rc) == (o.kd.l, o.kd.k, o.kd.include_rc)


def _model(lengths=None):
    rng = np.random.default_rng(42)
    sv = rng.integers(0, 4, (5, 20), dtype=np.uint8)
    return gk.GkmSVM(sv, np.array([0.5, -0.3, 0.8, -0.1, 0.2]), 0.42, "gkm_esttrunc",
                     {"L": 7, "k": 5, "d": 3, "include_rc": True}, sv_lengths=lengths, sv_chunk_size=3)


@pytest.mark.parametrize("lengths", [None, [20, 12, 9, 20, 15]])
def test_npz_round_trip(tmp_path, lengths):
    m = _model(lengths)
    m.save(str(tmp_path / "model.npz"))
    got = gk.load_model(str(tmp_path / "model.npz"))
    assert got.kernel_type == m.kernel_type and got.bias == m.bias and got.sv_chunk_size == 3
    assert got._kernel_params == m._kernel_params
    np.testing.assert_array_equal(got.support_sequences, m.support_sequences)
    np.testing.assert_array_equal(got.coefficients, m.coefficients)
    if lengths is None:
        assert got.sv_lengths is None
    else:
        np.testing.assert_array_equal(got.sv_lengths, lengths)


@pytest.mark.parametrize("name", ["model.txt", "model.txt.gz"])
@pytest.mark.parametrize("lengths", [None, [20, 12, 9, 20, 15]])
def test_lsgkm_round_trip(tmp_path, name, lengths):
    m = _model(lengths)
    m.save(str(tmp_path / name))
    got = gk.load_model(str(tmp_path / name))
    assert got.bias == pytest.approx(m.bias) and got.kernel_type == m.kernel_type
    np.testing.assert_array_equal(got.coefficients, m.coefficients)
    n = got.support_sequences.shape[1]
    for i in range(5):
        k = 20 if lengths is None else lengths[i]
        np.testing.assert_array_equal(got.support_sequences[i, :k], m.support_sequences[i, :k])
        assert (got.sv_lengths is None and k == n) or got.sv_lengths[i] == k


@pytest.mark.parametrize("include_rc", [True, False])
def test_norc_only_when_rc_off(tmp_path, include_rc):
    m = gk.GkmSVM(np.zeros((2, 10), np.uint8), [1.0, -1.0], 0.0, "gkm_esttrunc",
                  {"L": 7, "k": 5, "d": 3, "include_rc": include_rc})
    m.save(str(tmp_path / "m.txt"))
    text = (tmp_path / "m.txt").read_text()
    assert ("norc 1" in text) == (not include_rc)
    assert [ln for ln in text.splitlines() if ln.startswith("rho")] == ["rho -0.0"]
    assert gk.load_model(str(tmp_path / "m.txt")).kernel.include_rc == include_rc


def test_format_override_and_invalid(tmp_path):
    m = _model()
    m.save(str(tmp_path / "model.bin"), fmt="npz")
    assert gk.load_model(str(tmp_path / "model.bin.npz")).kernel_type == m.kernel_type
    with pytest.raises(ValueError, match="Unknown format"):
        m.save(str(tmp_path / "x"), fmt="pickle")


def test_deltasvm_npz_round_trip(tmp_path):
    d = gk.DeltaSVMWeights(np.arange(4**3, dtype=np.float64) / 7, 3, 3, False, -0.5)
    gk.save_deltasvm_npz(d, tmp_path / "d.npz")
    got = gk.load_model(str(tmp_path / "d.npz"))
    assert (got.l, got.k, got.include_rc, got.bias) == (3, 3, False, -0.5)
    np.testing.assert_array_equal(got.weights, d.weights)


def test_parser_counts_then_fills():
    coef, codes, lengths, other = importers.parse_lsgkm_svs(b"1 AC\n\n-2.5e-3 gTXa\r\nSV\n3 A")
    np.testing.assert_array_equal(coef, [1.0, -2.5e-3, 3.0])
    np.testing.assert_array_equal(lengths, [2, 4, 1])
    np.testing.assert_array_equal(codes, [[0, 1, 0, 0], [2, 3, 0, 0], [0, 0, 0, 0]])
    assert other == 1
    coef, codes, lengths, other = importers.parse_lsgkm_svs(b"")
    assert coef.shape == (0,) and codes.shape == (0, 0)


FILES = os.path.join(os.path.dirname(LSGKM), "files")


@pytest.mark.parametrize("name", ["t4", "t2norc"])
@pytest.mark.parametrize("ext", [".npz", ".model.txt", ".model.txt.gz"])
def test_reads_files_gkmsvm_lite_wrote(small, name, ext):
    """npz and LS-GKM text written by gkmsvm-lite's own serialization load to
    the model they were written from."""
    c = small[name]
    m = gk.load_model(os.path.join(FILES, name + ext))
    assert m.kernel_type == c["kernel_type"]
    assert m.bias == pytest.approx(float(c["bias"]), abs=0 if ext == ".npz" else 1e-15)
    for key, value in c["params"].items():
        assert m.kernel_params.get(key, value) == value
    assert m.kernel.include_rc == c["params"].get("include_rc", True)
    np.testing.assert_array_equal(m.coefficients, c["coef"])
    lengths = np.asarray(c["sv_lengths"])
    np.testing.assert_array_equal(np.asarray(m.sv_lengths), lengths)
    for i, n in enumerate(lengths):
        np.testing.assert_array_equal(m.support_sequences[i, :n], c["sv"][i, :n])


def test_reads_deltasvm_npz_gkmsvm_lite_wrote():
    d = gk.load_model(os.path.join(FILES, "t0small_deltasvm.npz"))
    assert (d.l, d.k, d.include_rc) == (3, 3, False) and d.bias == -0.15
    assert d.weights.shape == (64,)
    z = np.load(os.path.join(os.path.dirname(LSGKM), "deltasvm.npz"))
    np.testing.assert_array_equal(d.weights, z["t0small/w"])
