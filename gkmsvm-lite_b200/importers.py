"""LS-GKM model files (.model.txt / .model.txt.gz) -> GkmSVM, with the header
fields and conventions of gkmsvm-lite's importers/lsgkm.py:37-97: bias = -rho,
non-ACGT letters read as A, SVs of different lengths padded with lengths."""

from __future__ import annotations

import gzip

import numpy as np

from .inputs import as_batch, encode_codes
from .kernels import KERNEL_ALIASES
from .model import GkmSVM

_INT = ("L", "k", "d", "M", "nr_class", "total_sv", "norc")
_FLOAT = ("gamma", "H")


def _open(path):
    try:
        f = gzip.open(path, "rt")
        f.readline()
        f.seek(0)
        return f
    except gzip.BadGzipFile:
        return open(path)


def load_lsgkm_model(path, *, sv_chunk_size=None, device="cpu") -> GkmSVM:
    header = {"norc": 0}
    coefs, seqs = [], []
    in_sv = False
    with _open(str(path)) as f:
        for line in f:
            line = line.strip()
            if not line:
                continue
            if line.startswith("SV"):
                in_sv = True
                continue
            parts = line.split()
            if not in_sv:
                if len(parts) < 2:
                    continue
                key, val = parts[0], parts[1:]
                if key == "kernel_type":
                    header[key] = KERNEL_ALIASES.get(int(val[0]), val[0]) if val[0].isdigit() else val[0]
                elif key in _INT:
                    header[key] = int(val[0])
                elif key in _FLOAT:
                    header[key] = float(val[0])
                elif key == "rho":
                    header[key] = [float(v) for v in val]
                continue
            if len(parts) < 2:
                raise ValueError(f"Malformed SV line: {line[:80]}")
            coefs.append(float(parts[0]))
            seqs.append(parts[1])
    for key in ("kernel_type", "total_sv", "rho"):
        if key not in header:
            raise ValueError(f"Model file missing {key} field")
    if header.get("nr_class", 2) != 2:
        raise NotImplementedError("Only binary classification (nr_class=2) is supported")
    if len(seqs) != header["total_sv"]:
        raise ValueError(f"Expected {header['total_sv']} support vectors, got {len(seqs)}")
    codes = [encode_codes(s, allow_n=True, allow_other=True) for s in seqs]
    sv, sv_lengths = as_batch(codes)
    params = {"L": header["L"], "k": header["k"], "include_rc": header.get("norc", 0) == 0}
    for key in ("d", "gamma", "M", "H"):
        if key in header:
            params[key] = header[key]
    return GkmSVM(sv, np.array(coefs, dtype=np.float64), -header["rho"][0], header["kernel_type"], params,
                  sv_lengths=sv_lengths, sv_chunk_size=sv_chunk_size, device=device)


load_model = load_lsgkm_model
