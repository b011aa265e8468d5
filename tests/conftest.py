"""Shared test set-up: the gpu marker, repository paths and golden loaders."""

import ast
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
LSGKM = os.path.join(GOLDEN, "lsgkm")
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def small_cases():
    """{name: {field: array}} of tests/golden/small.npz."""
    z = np.load(os.path.join(GOLDEN, "small.npz"), allow_pickle=False)
    out = {}
    for key in z.files:
        name, field = key.split("/", 1)
        out.setdefault(name, {})[field] = z[key]
    for d in out.values():
        d["kernel_type"] = str(d["kernel_type"])
        d["params"] = ast.literal_eval(str(d["params"]))
    return out


def read_fasta(path):
    names, seqs, cur = [], [], []
    with open(path) as f:
        for line in f:
            line = line.strip()
            if line.startswith(">"):
                if cur:
                    seqs.append("".join(cur))
                    cur = []
                names.append(line[1:])
            elif line:
                cur.append(line)
    if cur:
        seqs.append("".join(cur))
    return names, seqs


def codes_of(seqs):
    """[n, Lmax] uint8 codes (A C G T = 0..3, N and other letters 0) and lengths."""
    lut = np.zeros(256, np.uint8)
    for i, c in enumerate("ACGT"):
        lut[ord(c)] = i
        lut[ord(c.lower())] = i
    lens = np.array([len(s) for s in seqs], np.int64)
    x = np.zeros((len(seqs), lens.max()), np.uint8)
    for i, s in enumerate(seqs):
        x[i, : len(s)] = lut[np.frombuffer(s.encode(), np.uint8)]
    return x, lens


def read_lsgkm_explain(path):
    import gzip

    with gzip.open(path, "rt") as f:
        rows = [line.rstrip("\n").split("\t") for line in f]
    return np.stack([
        np.array([[float(v) for v in pos.split(",")] for pos in r[2].split(";")]).T
        for r in rows
    ])


def read_pred(path):
    return np.array([float(line.split("\t")[1]) for line in open(path) if line.strip()])


@pytest.fixture(scope="session")
def small():
    return small_cases()
