"""Seeded synthetic workloads with the shapes of the five benchmark configs.

The published benchmark used real ENCODE/GM12878 sequences, which are not
available offline; these generators give i.i.d. bases with P(A) = P(T) = 0.29
and P(C) = P(G) = 0.21 (GC = 0.42) and the stated length distributions, from
``numpy.random.default_rng(seed)`` draws that are stable across numpy
versions (uniform doubles and integers only).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

_CUM = np.array([0.29, 0.50, 0.71])  # A | C | G | T boundaries at GC = 0.42


def random_codes(rng, n: int, L: int) -> np.ndarray:
    """[n, L] uint8 base codes at GC 0.42."""
    return np.searchsorted(_CUM, rng.random((n, L)), side="right").astype(np.uint8)


def log_uniform_lengths(rng, n: int, lo: int, hi: int) -> np.ndarray:
    """[n] int64 lengths floor(exp(U(ln lo, ln hi)))."""
    return np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi), n))).astype(np.int64)


def ragged_codes(rng, lengths: np.ndarray) -> np.ndarray:
    """[n, max(lengths)] codes, zero (A) past each row's length."""
    lengths = np.asarray(lengths, np.int64)
    x = random_codes(rng, len(lengths), int(lengths.max()))
    x[np.arange(x.shape[1])[None, :] >= lengths[:, None]] = 0
    return x


@dataclass
class Workload:
    sv: np.ndarray
    sv_lengths: np.ndarray | None
    coef: np.ndarray
    x: np.ndarray
    x_lengths: np.ndarray | None


def config1(seed: int = 0) -> Workload:
    """Plain scoring: 2,000 SVs x 300 bp, alphas ~ U(-1, 1); 1,000 queries x 300 bp."""
    rng = np.random.default_rng(seed)
    sv = random_codes(rng, 2000, 300)
    coef = rng.uniform(-1.0, 1.0, 2000)
    x = random_codes(rng, 1000, 300)
    return Workload(sv, None, coef, x, None)


def config2(seed: int = 1, n: int = 4000) -> tuple[np.ndarray, np.ndarray]:
    """Gram: n sequences, lengths log-uniform in 100..1000 bp."""
    rng = np.random.default_rng(seed)
    lengths = log_uniform_lengths(rng, n, 100, 1000)
    return ragged_codes(rng, lengths), lengths


def config3_model(seed: int = 2, n_sv: int = 72000):
    """72,000 SVs with lengths uniform in 200..500 bp, alphas ~ N(0, 0.1^2)."""
    rng = np.random.default_rng(seed)
    lengths = rng.integers(200, 501, n_sv).astype(np.int64)
    sv = ragged_codes(rng, lengths)
    coef = rng.normal(0.0, 0.1, n_sv)
    return sv, lengths, coef


def config3_queries(seed: int = 102, n: int = 100000, n_rate: float = 0.005):
    """Queries with lengths log-uniform in 50..2000 bp and 0.5% N bases, given
    as codes (N stored as A, as every kernel reads it) plus an N mask."""
    rng = np.random.default_rng(seed)
    lengths = log_uniform_lengths(rng, n, 50, 2000)
    x = ragged_codes(rng, lengths)
    nmask = rng.random(x.shape) < n_rate
    nmask &= np.arange(x.shape[1])[None, :] < lengths[:, None]
    x[nmask] = 0
    return x, lengths, nmask


def config4_queries(seed: int = 3, n: int = 512, L: int = 1000) -> np.ndarray:
    """ISM / GkmExplain inputs: n x L bp."""
    return random_codes(np.random.default_rng(seed), n, L)


def variant_pairs(rng, ref: np.ndarray, lengths: np.ndarray, indel_rate: float = 0.2):
    """(alt codes, alt lengths): one SNV (1 - indel_rate) or an indel of
    U{1..10} bp at a uniform position of each row of ref."""
    n, L = ref.shape
    alts = []
    alen = np.empty(n, np.int64)
    for i in range(n):
        s = ref[i, : lengths[i]].copy()
        p = int(rng.integers(0, len(s)))
        if rng.random() >= indel_rate or len(s) < 12:
            s[p] = (s[p] + 1 + int(rng.integers(0, 3))) % 4
        elif rng.random() < 0.5:
            size = int(rng.integers(1, 11))
            s = np.concatenate([s[:p], random_codes(rng, 1, size)[0], s[p:]])
        else:
            size = int(rng.integers(1, 11))
            s = np.concatenate([s[:p], s[p + size:]])
        alts.append(s)
        alen[i] = len(s)
    out = np.zeros((n, max(L, int(alen.max()))), np.uint8)
    for i, s in enumerate(alts):
        out[i, : len(s)] = s
    return out, alen
