"""LS-GKM model files (.model.txt / .model.txt.gz) -> GkmSVM, with the header
fields and conventions of gkmsvm-lite's importers/lsgkm.py:37-97: bias = -rho,
non-ACGT letters read as A, SVs of different lengths padded with lengths.  The
SV section (nearly all of a file) is parsed and encoded natively
(gkm_lsgkm_parse_svs); the few header lines in Python."""

from __future__ import annotations

import ctypes
import gzip
import re
import warnings

import numpy as np

from . import _lib
from .inputs import LSGKM_MAX_LENGTH, SeqBatch
from .kernels import KERNEL_ALIASES
from .model import GkmSVM

_INT = ("L", "k", "d", "M", "nr_class", "total_sv", "norc")
_FLOAT = ("gamma", "H")
_LIST = {"rho": float, "label": int, "nr_sv": int, "probA": float, "probB": float}


def _read_bytes(path) -> bytes:
    """The file's bytes, gunzipped when it is gzip (detected by content)."""
    with open(path, "rb") as f:
        data = f.read()
    if data[:2] == b"\x1f\x8b":
        data = gzip.decompress(data)
    return data


def _parse_header(data: bytes) -> tuple[dict, int]:
    """(typed header fields, offset of the SV section) of an LS-GKM file
    (importers/__init__.py:31-50 parse_header_value)."""
    header = {"norc": 0}
    pos = 0
    while pos < len(data):
        eol = data.find(b"\n", pos)
        if eol < 0:
            eol = len(data)
        line = data[pos:eol].decode("ascii", errors="replace").strip()
        pos = eol + 1
        if line.startswith("SV"):
            return header, pos
        parts = line.split(None, 1)
        if len(parts) < 2:
            continue
        key, value = parts
        if key == "kernel_type":
            header[key] = KERNEL_ALIASES.get(int(value), value) if value.isdigit() else value
        elif key in _INT:
            header[key] = int(value)
        elif key in _FLOAT:
            header[key] = float(value)
        elif key in _LIST:
            header[key] = [_LIST[key](v) for v in value.split()]
        elif key == "svm_type":
            header[key] = value
    return header, len(data)


def parse_lsgkm_header(path) -> dict:
    """Header fields of an LS-GKM model file (importers/lsgkm.py:23-34)."""
    return _parse_header(_read_bytes(str(path)))[0]


def parse_lsgkm_svs(text: bytes):
    """(coefficients [n] float64, codes [n, L_max] uint8, lengths [n] int64,
    SVs with letters other than ACGTN) of an SV section, parsed natively
    (gkm_lsgkm_parse_svs)."""
    lib = _lib.load()
    buf = ctypes.c_char_p(text)
    n, width, other, bad = (ctypes.c_int64() for _ in range(4))
    _lib.check(lib.gkm_lsgkm_parse_svs(buf, len(text), 0, 0, None, None, None, ctypes.byref(n),
                                       ctypes.byref(width), None, ctypes.byref(bad)), "gkm_lsgkm_parse_svs")
    n, width = n.value, width.value
    coef = np.empty(n, dtype=np.float64)
    lengths = np.empty(n, dtype=np.int64)
    codes = np.empty((n, width), dtype=np.uint8)
    got, longest = ctypes.c_int64(), ctypes.c_int64()
    if n:
        _lib.check(lib.gkm_lsgkm_parse_svs(buf, len(text), n, width, coef.ctypes.data, lengths.ctypes.data,
                                           codes.ctypes.data, ctypes.byref(got), ctypes.byref(longest),
                                           ctypes.byref(other), ctypes.byref(bad)), "gkm_lsgkm_parse_svs")
    return coef, codes, lengths, other.value


def load_lsgkm_model(path, *, sv_chunk_size=None, device="cpu") -> GkmSVM:
    """GkmSVM of an LS-GKM model file, plain or gzip (importers/lsgkm.py:37-97):
    bias = -rho; SVs of different lengths padded, with sv_lengths; letters
    other than ACGTN read as N, with a warning."""
    data = _read_bytes(str(path))
    header, start = _parse_header(data)
    for key in ("kernel_type", "total_sv", "rho"):
        if header.get(key) is None:
            raise ValueError(f"Model file missing {key} field")
    if header.get("nr_class", 2) != 2:
        raise NotImplementedError(
            f"Only binary classification (nr_class=2) is supported, got {header.get('nr_class')}")
    coef, sv, lengths, other = parse_lsgkm_svs(data[start:])
    if len(coef) == 0:
        raise ValueError("No support vector sequences found")
    if len(coef) != header["total_sv"]:
        raise ValueError(f"Expected {header['total_sv']} support vectors, got {len(coef)}")
    if other:
        warnings.warn(f"{other} support vectors contain letters other than ACGTN; "
                      "reading them as N (scored as A, as LS-GKM does)", stacklevel=2)
    longest = int(lengths.max())
    if longest > LSGKM_MAX_LENGTH:
        warnings.warn(f"sequences up to {longest} bp: LS-GKM reads only the first "
                      f"{LSGKM_MAX_LENGTH} bases of longer ones", stacklevel=2)
    params = {"L": header["L"], "k": header["k"], "include_rc": header.get("norc", 0) == 0}
    for key in ("d", "gamma", "M", "H"):
        if key in header:
            params[key] = header[key]
    return GkmSVM(sv, coef, -header["rho"][0], header["kernel_type"], params,
                  sv_lengths=None if (lengths == longest).all() else lengths, sv_chunk_size=sv_chunk_size,
                  device=device)


# gkmsvm_kernel -t (R useTgkm) filter types as kernel types, each cut at d
# mismatches (importers/classic.py:23-26); 3 (wildcard) and 4 (mismatch
# kernel) have no counterpart
GKMSVM_FILTERS = {0: "gkm_estfull", 1: "gkm_esttrunc", 2: "gkm_cnt"}


def read_fasta(path) -> list:
    """(name, sequence) records of a FASTA file, gzip or plain (fasta.py:19-44)."""
    records, name, seq = [], None, []
    for line in _read_bytes(str(path)).decode("ascii", errors="replace").splitlines():
        line = line.strip()
        if not line:
            continue
        if line.startswith(">"):
            if name is not None:
                records.append((name, "".join(seq)))
            name, seq = line[1:].strip(), []
        else:
            seq.append(line)
    if name is not None:
        records.append((name, "".join(seq)))
    return records


def load_classic_model(alpha_path, svseq_path=None, *, L: int = 10, k: int = 6, d: int = 3, filter_type: int = 1,
                       include_rc: bool = True, sv_chunk_size=None, device="cpu") -> GkmSVM:
    """GkmSVM of a model the classic gkmSVM tools (C++ or R) wrote
    (importers/classic.py:29-120): PREFIX_svalpha.out ("id <TAB> alpha") and
    PREFIX_svseq.fa, SVs matched to alphas by id with every letter other than
    ACGT dropped, as the tools read them; the kernel comes from the arguments
    (gkmsvm_kernel -l/-k/-d/-t, -R for no RC); bias 0."""
    alpha_path = str(alpha_path)
    if svseq_path is None:
        if not alpha_path.endswith("svalpha.out"):
            raise ValueError(f"give svseq_path for {alpha_path}")
        svseq_path = alpha_path[: -len("svalpha.out")] + "svseq.fa"
    ids, coefs = [], []
    for line in _read_bytes(alpha_path).decode("ascii", errors="replace").splitlines():
        parts = line.split()
        if not parts:
            continue
        if len(parts) != 2:
            raise ValueError(f"Expected 'id <TAB> alpha', got: {line.strip()[:80]}")
        ids.append(parts[0])
        coefs.append(float(parts[1]))
    by_id = {name.split()[0]: seq for name, seq in read_fasta(svseq_path) if name.split()}
    missing = [i for i in ids if i not in by_id]
    if missing:
        raise ValueError(f"{len(missing)} SV ids of {alpha_path} are not in {svseq_path}, e.g. {missing[0]}")
    seqs = [re.sub("[^ACGTacgt]", "", by_id[i]).upper() for i in ids]
    dropped = sum(len(by_id[i]) != len(s) for i, s in zip(ids, seqs))
    if dropped:
        warnings.warn(f"{dropped} support vectors hold letters other than ACGT, dropped as gkmSVM reads them "
                      "(queries with N score as in gkmsvm_classify only with those letters dropped too)",
                      stacklevel=2)
    if filter_type not in GKMSVM_FILTERS:
        raise NotImplementedError(f"gkmSVM filter type {filter_type} (wildcard/mismatch kernels) is not "
                                  f"supported; use {sorted(GKMSVM_FILTERS)}")
    if not seqs:
        raise ValueError("No support vector sequences found")
    svb = SeqBatch.read(seqs)
    sv, lengths = svb.codes, svb.lengths
    params = {"L": L, "k": k, "d": d, "include_rc": bool(include_rc)}
    return GkmSVM(sv, np.array(coefs, dtype=np.float64), 0.0, GKMSVM_FILTERS[filter_type], params,
                  sv_lengths=lengths, sv_chunk_size=sv_chunk_size, device=device)


def load_r_gkmsvm_model(path, svseq_path=None, *, L: int = 10, K: int = 6, maxnmm: int = 3, useTgkm: int = 1,
                        addRC: bool = True, sv_chunk_size=None, device="cpu") -> GkmSVM:
    """GkmSVM of a model R gkmSVM's gkmsvm_train wrote, the classic tools'
    files, with the R package's argument names (importers/r_gkmsvm.py:17-53)."""
    return load_classic_model(path, svseq_path, L=L, k=K, d=maxnmm, filter_type=useTgkm, include_rc=addRC,
                              sv_chunk_size=sv_chunk_size, device=device)
