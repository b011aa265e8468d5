"""CPU oracle for the pairwise gapped-k-mer kernel path.

TEST INFRASTRUCTURE ONLY.  The parity tests, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` call this module as the checker; the
product package never imports it.

It restates, from gkmsvm-lite's source (paths relative to src/gkmsvm/), the
algorithm of the path on small inputs:

* pair weight tables h(m): kernels/direct.py:233-240 (gkm_cnt, C(l-m, k) cut at
  d; no cut when loaded without d, svm.py:96-97), kernels/esttrunc.py:40-110
  (LS-GKM's estimated l-mer weights, truncated, cut at d), RBF finish
  kernels/rbf.py:27-29;
* window weights kernels/weighted.py:38-43 and row weights kernels/packed.py:105-122;
* mismatch profiles by brute force over every window pair (gkm_oracle.c), whose
  sum through h is the raw kernel (kernels/direct.py:23-42);
* scores svm.py:368-451, variant scores svm.py:600-662, mutation impact
  explain/impact.py:22-48, ISM as f(mutant) - f(x) (ism.py; property checked by
  the reference's tests/test_ism.py:208-249), GkmExplain per-SV pair loop
  explain/cpu.py:14-66 with explain/core.py:116-247, Gram gram.py:21-164,
  DeltaSVM weights svm.py:664-785.

Parity is pinned by tests/golden (outputs of gkmsvm-lite itself, generated by
tests/golden/make_golden.py, plus LS-GKM fixtures from gkmsvm-lite's tests).
"""

from __future__ import annotations

import ctypes
import gzip
import os
import subprocess
from dataclasses import dataclass, field
from itertools import combinations, product
from math import comb

import numpy as np

PAD = np.uint32(0xFFFFFFFF)
_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libgkm_oracle.so")
_lib = None


def build() -> str:
    """Compile gkm_oracle.c into oracle/_build (make)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        I64 = ctypes.c_int64
        I = ctypes.c_int
        D = ctypes.c_double
        L.orc_pack.argtypes = [P, P, I64, I64, I, P, P]
        L.orc_profiles.argtypes = [P, P, I64, I64, P, P, I64, I64, I, P]
        L.orc_self_profiles.argtypes = [P, P, P, I64, I64, I, P]
        L.orc_self_profiles_mt.argtypes = [P, P, P, I64, I64, I, P, I]
        L.orc_index_build.argtypes = [P, P, P, P, I64, I64, I]
        L.orc_index_build.restype = P
        L.orc_index_free.argtypes = [P]
        L.orc_index_entries.argtypes = [P]
        L.orc_index_entries.restype = I64
        L.orc_index_reduce.argtypes = [P, P, P, I64, I64, P, P, I, P, P, P, D, I, P, I]
        L.orc_index_pairwise.argtypes = [P, P, P, I64, I64, P, P, I, I64, P]
        L.orc_explain_pairs.argtypes = [P, I64, I64, P, I64, I64, P, P, P, I, I, I64, I, P, P, P]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


# ---------------------------------------------------------------------------
# Pair weight tables and window weights
# ---------------------------------------------------------------------------


def _estimated_lmer_weights(l: int, k: int, truncate: bool) -> np.ndarray:
    """LS-GKM's estimated l-mer kernel weights by mismatch count (restating
    kernels/esttrunc.py:40-110, itself from LS-GKM's
    calc_gkm_kernel_lmerest_wt): a recursion over window length for the
    gapped-k-mer match weights wm, the expected l-mer kernel per mismatch
    count, optional truncation below 1e-50, then the convolution over pairs of
    mismatch counts that gives the weight at each mismatch count."""
    alphabet = 4
    prev = [[1.0] * (k + 1) for _ in range(k + 1)]
    cur = [[1.0] * (k + 1) for _ in range(k + 1)]
    for length in range(1, l + 1):
        for kk in range(1, k + 1):
            cur[kk][0] = prev[kk][0] + (alphabet - 1) * prev[kk - 1][0]
            for jm in range(1, kk + 1):
                cur[kk][jm] = (cur[kk - 1][jm - 1] * (kk - length)) / kk
        prev, cur = cur, prev
    norm = comb(l, k) * (alphabet**l)
    wm = [prev[k][i] / norm for i in range(k + 1)]
    est = []
    for m in range(l + 1):
        v = 0.0
        for i in range(min(m, k) + 1):
            if l - m >= k - i:
                v += wm[i] * comb(l - m, k - i) * comb(m, i)
        est.append(v)
    if truncate:
        live = True
        tr = []
        for v in est:
            if v < 1e-50:
                live = False
            tr.append(v if live else 0.0)
        est = tr
    out = [0.0] * (l + 1)
    for m in range(l + 1):
        acc = 0.0
        for m1 in range(l + 1):
            if est[m1] == 0.0:
                continue
            for m2 in range(l + 1):
                if est[m2] == 0.0:
                    continue
                for t in range(min(m, l) + 1):
                    r = m1 + m2 - 2 * t - l + m
                    diff = m1 - t
                    if r < 0 or diff > l - m or r > diff:
                        continue
                    c = (
                        comb(m, t)
                        * comb(l - m, diff)
                        * comb(diff, r)
                        * ((alphabet - 1) ** t)
                        * ((alphabet - 2) ** r)
                    )
                    acc += c * est[m1] * est[m2]
        out[l - m] = acc
    return np.array(out, dtype=np.float64)


_NAMES = {
    0: "gkm_cnt", 1: "gkm_estfull", 2: "gkm_esttrunc", 3: "gkmrbf", 4: "wgkm",
    5: "wgkmrbf", 6: "gkm_cnt_rbf", "direct": "gkm_cnt", "estimated": "gkm_esttrunc",
    "estimated_full": "gkm_estfull", "rbf": "gkmrbf", "weighted": "wgkm",
    "weighted_rbf": "wgkmrbf", "direct_rbf": "gkm_cnt_rbf",
}


@dataclass
class KernelDef:
    """A kernel type as KERNEL_BUILDERS (svm.py:95-106) builds it from params."""

    name: str
    l: int
    k: int
    d: int | None = 3
    gamma: float = 1.0
    M: int = 50
    H: float = 50.0
    include_rc: bool = True
    normalize: bool = True
    h: np.ndarray = field(default=None, repr=False)

    @classmethod
    def from_params(cls, kernel_type, p: dict) -> "KernelDef":
        if isinstance(kernel_type, str) and kernel_type.isdigit():
            kernel_type = int(kernel_type)
        name = _NAMES.get(kernel_type, kernel_type)
        # gkm_cnt params without d count every pair (svm.py:96-97)
        d = p.get("d", None if name == "gkm_cnt" else 3)
        kd = cls(name, p["L"], p["k"], d, p.get("gamma", 1.0), p.get("M", 50),
                 float(p.get("H", 50.0)), p.get("include_rc", True))
        kd.h = kd._table()
        return kd

    @property
    def rbf(self) -> bool:
        return self.name in ("gkmrbf", "wgkmrbf", "gkm_cnt_rbf")

    @property
    def weighted(self) -> bool:
        return self.name in ("wgkm", "wgkmrbf")

    def _table(self) -> np.ndarray:
        l, k, d = self.l, self.k, self.d
        if self.name in ("gkm_cnt", "gkm_cnt_rbf"):
            return np.array(
                [comb(l - m, k) if l - m >= k and (d is None or m <= d) else 0
                 for m in range(l + 1)], dtype=np.float64)
        h = _estimated_lmer_weights(l, k, self.name != "gkm_estfull")
        if d < l:
            h[d + 1:] = 0.0
        return h

    @property
    def dmax(self) -> int:
        nz = np.flatnonzero(self.h)
        return int(nz.max()) if len(nz) else -1


def window_weights(W: int, M: int, H: float) -> np.ndarray:
    """[W] uint8 (kernels/weighted.py:38-43)."""
    center = W // 2
    dist = np.abs(center - np.arange(W))
    wt = np.floor(M * np.exp(-1 * np.log(2) * dist / H) + 1)
    return np.minimum(wt, M).astype(np.uint8)


def row_weights(fwd: np.ndarray, kd: KernelDef) -> np.ndarray | None:
    """[R, W] uint8 forward weights from each row's window count, 0 on PAD."""
    if not kd.weighted:
        return None
    counts = (fwd != PAD).sum(axis=1)
    w = np.zeros(fwd.shape, dtype=np.uint8)
    for n in np.unique(counts[counts > 0]):
        w[counts == n, :n] = window_weights(int(n), kd.M, kd.H)
    return w


# ---------------------------------------------------------------------------
# Packing and profiles
# ---------------------------------------------------------------------------


def pack(codes: np.ndarray, lengths, l: int):
    codes = np.ascontiguousarray(codes, dtype=np.uint8)
    B, L = codes.shape
    W = L - l + 1
    fwd = np.empty((B, W), np.uint32)
    rc = np.empty((B, W), np.uint32)
    ln = None if lengths is None else np.ascontiguousarray(lengths, dtype=np.int64)
    lib().orc_pack(_p(codes), _p(ln), B, L, l, _p(fwd), _p(rc))
    return fwd, rc


def profiles(xc, xl, yc, yl, kd: KernelDef) -> np.ndarray:
    """[B, S, l+1] uint64 mismatch profiles of x rows against y's forward (and
    RC, when the kernel includes it) windows."""
    fx, _ = pack(xc, xl, kd.l)
    fy, ry = pack(yc, yl, kd.l)
    wx = row_weights(fx, kd)
    wy = row_weights(fy, kd)
    by = fy
    wby = wy
    if kd.include_rc:
        by = np.ascontiguousarray(np.concatenate([fy, ry], axis=1))
        if wy is not None:
            wby = np.ascontiguousarray(np.concatenate([wy, wy[:, ::-1]], axis=1))
            # a padded row's RC weights sit after its pads, reversed
            counts = (fy != PAD).sum(axis=1)
            W = fy.shape[1]
            for r, n in enumerate(counts):
                wby[r, W:] = 0
                wby[r, 2 * W - n:] = wy[r, :n][::-1]
    B, Wx = fx.shape
    S, Wy = by.shape
    out = np.zeros((B, S, kd.l + 1), np.uint64)
    lib().orc_profiles(_p(fx), _p(wx), B, Wx, _p(by), _p(wby), S, Wy, kd.l, _p(out))
    return out


def self_profiles(xc, xl, kd: KernelDef, threads: int = 1) -> np.ndarray:
    fx, rx = pack(xc, xl, kd.l)
    w = row_weights(fx, kd)
    B, W = fx.shape
    out = np.zeros((B, kd.l + 1), np.uint64)
    if threads > 1:
        lib().orc_self_profiles_mt(_p(fx), _p(rx if kd.include_rc else None), _p(w), B, W,
                                   kd.l, _p(out), int(threads))
    else:
        lib().orc_self_profiles(_p(fx), _p(rx if kd.include_rc else None), _p(w), B, W,
                                kd.l, _p(out))
    return out


def raw_from_profiles(prof: np.ndarray, kd: KernelDef) -> np.ndarray:
    return prof.astype(np.float64) @ kd.h


# ---------------------------------------------------------------------------
# Models and outputs
# ---------------------------------------------------------------------------


@dataclass
class OracleModel:
    sv: np.ndarray  # [S, L] uint8 codes
    sv_lengths: np.ndarray | None
    coef: np.ndarray  # [S] float64
    bias: float
    kd: KernelDef


def load_lsgkm(path: str) -> OracleModel:
    """LS-GKM model text (importers/lsgkm.py:37-97): bias = -rho; letters other
    than ACGT read as A."""
    op = gzip.open if str(path).endswith(".gz") else open
    header, coef, seqs, in_sv = {"norc": 0}, [], [], False
    with op(path, "rt") as f:
        for line in f:
            line = line.strip()
            if not line:
                continue
            if line.startswith("SV"):
                in_sv = True
                continue
            parts = line.split()
            if not in_sv:
                if len(parts) >= 2:
                    header[parts[0]] = parts[1:]
                continue
            coef.append(float(parts[0]))
            seqs.append(parts[1])
    lut = np.zeros(256, np.uint8)
    for i, c in enumerate("ACGT"):
        lut[ord(c)] = i
        lut[ord(c.lower())] = i
    lens = np.array([len(s) for s in seqs], np.int64)
    sv = np.zeros((len(seqs), lens.max()), np.uint8)
    for i, s in enumerate(seqs):
        sv[i, : len(s)] = lut[np.frombuffer(s.encode(), np.uint8)]
    kt = header["kernel_type"][0]
    p = {"L": int(header["L"][0]), "k": int(header["k"][0]),
         "include_rc": int(header["norc"][0] if isinstance(header["norc"], list) else 0) == 0}
    for key, typ in (("d", int), ("gamma", float), ("M", int), ("H", float)):
        if key in header:
            p[key] = typ(header[key][0])
    kd = KernelDef.from_params(kt, p)
    return OracleModel(sv, None if (lens == lens.max()).all() else lens,
                       np.array(coef), -float(header["rho"][0]), kd)


def _norms(diag):
    return np.sqrt(np.asarray(diag, np.float64))


def kernel_values(model: OracleModel, xc, xl) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(K_raw [B, S], K(x, x) [B], K(sv, sv) [S]) of the base kernel."""
    kd = model.kd
    raw = raw_from_profiles(profiles(xc, xl, model.sv, model.sv_lengths, kd), kd)
    dx = raw_from_profiles(self_profiles(xc, xl, kd), kd)
    ds = raw_from_profiles(self_profiles(model.sv, model.sv_lengths, kd), kd)
    return raw, dx, ds


def _finish(k, kd):
    return np.exp(kd.gamma * (k - 1.0)) if kd.rbf else k


def _short(lengths, l):
    if lengths is None:
        return None
    s = np.asarray(lengths) < l
    return s if s.any() else None


def scores(model: OracleModel, xc, xl=None) -> np.ndarray:
    """[B, 1] decision values (svm.py:368-451); NaN for rows shorter than l."""
    kd = model.kd
    raw, dx, ds = kernel_values(model, xc, xl)
    k = raw
    if kd.normalize:
        k = raw / np.maximum(np.sqrt(dx[:, None] * ds[None, :]), 1e-10)
    out = (_finish(k, kd) * model.coef).sum(axis=1) + model.bias
    short = _short(xl, kd.l)
    if short is not None:
        out[short] = np.nan
    return out[:, None]


def deltasvm_weights(model: OracleModel, query_norm: bool = False, idx=None) -> np.ndarray:
    """to_deltasvm weights (svm.py:706-785) at DeltaSVM indices idx (first
    base most significant; all 4^l when None): each l-mer scored alone, minus
    the bias, with its own normalisation undone unless query_norm (RBF keeps
    it).  With RC the canonical member of each l-mer/reverse-complement pair
    is the one scored (svm.py:771-785); the table route (svm.py:667-704) is the
    same sum read from the l-mer table."""
    kd = model.kd
    l = kd.l
    powers = 4 ** np.arange(l - 1, -1, -1, dtype=np.int64)
    idx = np.arange(4**l, dtype=np.int64) if idx is None else np.asarray(idx, dtype=np.int64)
    digits = (idx[:, None] // powers) % 4
    if kd.include_rc:
        rc = ((3 - digits[:, ::-1]) * powers).sum(axis=1)
        digits = (np.minimum(idx, rc)[:, None] // powers) % 4
    x = np.ascontiguousarray(digits.astype(np.uint8))
    w = scores(model, x)[:, 0] - model.bias
    if not query_norm and kd.normalize and not kd.rbf:
        dx = raw_from_profiles(self_profiles(x, None, kd), kd)
        w = w * np.sqrt(np.maximum(dx, 1e-10))
    return w


def _joint(L, n, a, b):
    if a is None and b is None:
        return None
    return np.concatenate([np.full(n, L) if a is None else a, np.full(n, L) if b is None else b])


def score_variants(model: OracleModel, ref, alt, ref_lengths=None, alt_lengths=None):
    """score(alt) - score(ref) (svm.py:632-647); ref/alt [n, L] codes of one L."""
    n, L = ref.shape
    s = scores(model, np.concatenate([alt, ref]), _joint(L, n, alt_lengths, ref_lengths))
    return s[:n] - s[n:]


def mutation_impact(model: OracleModel, ref, alt, ref_lengths=None, alt_lengths=None):
    """lsgkm gkmexplain -m 5 (explain/impact.py:22-48, 247-390) on [n, L] codes."""
    kd = model.kd
    n, L = ref.shape
    both = np.concatenate([ref, alt])
    bl = _joint(L, n, ref_lengths, alt_lengths)
    raw, dx, ds = kernel_values(model, both, bl)
    k = raw[:n]
    dk = raw[n:] - k
    if kd.normalize:
        z = np.maximum(np.sqrt(dx[:n, None] * ds[None, :]), 1e-10)
        k = k / z
        dk = dk / z
    if kd.rbf:
        pos = k > 0
        safe = np.where(pos, k, 1.0)
        dk = np.where(pos, dk * (np.exp(kd.gamma * (safe - 1)) - np.exp(-kd.gamma)) / safe, 0.0)
    out = (dk * model.coef).sum(axis=1)
    if bl is not None:
        short = (bl < kd.l).reshape(2, -1).any(axis=0)
        out[short] = np.nan
    return out[:, None]


def ism(model: OracleModel, xc, xl=None) -> np.ndarray:
    """[B, 4, L] f(mutant) - f(x) for every single-base substitution; 0 past a
    row's length; NaN rows shorter than l (ism.py:21-64; inputs.py:137-145)."""
    B, L = xc.shape
    lens = np.full(B, L) if xl is None else np.asarray(xl)
    out = np.zeros((B, 4, L))
    for b in range(B):
        n = int(lens[b])
        if n < model.kd.l:
            out[b] = np.nan
            continue
        x = xc[b : b + 1, :n].copy()
        mutants = np.repeat(x, 4 * n, axis=0)
        for p in range(n):
            for v in range(4):
                mutants[4 * p + v, p] = v
        s = scores(model, np.concatenate([x, mutants]))[:, 0]
        d = (s[1:] - s[0]).reshape(n, 4).T
        # the reference base keeps the reference windows: exactly 0
        for p in range(n):
            d[x[0, p], p] = 0.0
        out[b, :, :n] = d
    return out


def explain_tables(kd: KernelDef, mode: str):
    """(table_a, table_b) of explain/weights.py:19-57 for hypothetical or
    perturbation, and the minimum matches of a contributing pair."""
    l, h = kd.l, kd.h
    d = l if kd.d is None else kd.d
    a = np.zeros(l + 2)
    b = np.zeros(l + 2)
    if mode == "perturbation":
        for m in range(l + 1):
            now = h[m]
            more = h[m + 1] if m + 1 <= l else 0.0
            a[m] = more - now
            if m >= 1:
                b[m] = h[m - 1] - now
    else:
        for m in range(min(d, l) + 1):
            if l - m > 0:
                a[m] = h[m] / (l - m)
        for m in range(1, min(d, l) + 1):
            if l - m + 1 > 0:
                b[m] = h[m - 1] / (l - m + 1)
    nz = [m for m in range(l + 1) if a[m] != 0 or b[m] != 0]
    return a, b, l - max(nz, default=-1)


def gkmexplain(model: OracleModel, xc, xl=None, mode="hypothetical") -> np.ndarray:
    """[B, 4, L] GkmExplain attributions by the per-SV pair loop
    (explain/core.py:116-247, explain/cpu.py:14-66)."""
    kd = model.kd
    if mode == "importance":
        hyp = gkmexplain(model, xc, xl, "hypothetical")
        oh = np.eye(4)[xc].transpose(0, 2, 1)
        out = hyp * oh
    else:
        a, b, min_matches = explain_tables(kd, mode)
        fx, _ = pack(xc, xl, kd.l)
        fs, rs = pack(model.sv, model.sv_lengths, kd.l)
        wx = row_weights(fx, kd)
        ws = row_weights(fs, kd)
        py = fs
        wy = ws
        if kd.include_rc:
            py = np.concatenate([fs, rs], axis=1)
            if ws is not None:
                W = fs.shape[1]
                wr = np.zeros_like(ws)
                counts = (fs != PAD).sum(axis=1)
                for r, n in enumerate(counts):
                    wr[r, W - n:] = ws[r, :n][::-1]
                wy = np.concatenate([ws, wr], axis=1)
        raw, dx, ds = kernel_values(model, xc, xl)
        eff = np.broadcast_to(model.coef[None, :], raw.shape).astype(np.float64)
        if kd.normalize:
            eff = eff / np.maximum(np.sqrt(dx[:, None] * ds[None, :]), 1e-10)
        if kd.rbf:
            kn = raw / np.maximum(np.sqrt(dx[:, None] * ds[None, :]), 1e-10)
            pos = kn > 0
            safe = np.where(pos, kn, 1.0)
            eff = eff * np.where(pos, (np.exp(kd.gamma * (safe - 1)) - np.exp(-kd.gamma)) / safe, 0.0)
        B, W = fx.shape
        S, Wy = py.shape
        L = xc.shape[1]
        out = np.zeros((B, 4, L))
        fx, py = np.ascontiguousarray(fx), np.ascontiguousarray(py)
        eff = np.ascontiguousarray(eff)
        lib().orc_explain_pairs(
            _p(fx), B, W, _p(py), S, Wy, _p(a), _p(b), _p(eff), kd.l, min_matches, L,
            int(mode == "perturbation"), _p(None if wx is None else np.ascontiguousarray(wx)),
            _p(None if wy is None else np.ascontiguousarray(wy)), _p(out))
    if xl is not None:
        inside = np.arange(xc.shape[1])[None, None, :] < np.asarray(xl)[:, None, None]
        out = np.where(inside, out, 0.0)
        out[np.asarray(xl) < kd.l] = np.nan
    return out


def gram(kd: KernelDef, X, xl=None, Y=None, yl=None) -> np.ndarray:
    """Normalised, finished Gram matrix (gram.py:21-164), exactly symmetric for
    a self-Gram (the upper triangle mirrored, gram.py:101-105)."""
    sym = Y is None
    if sym:
        Y, yl = X, xl
    raw = raw_from_profiles(profiles(X, xl, Y, yl, kd), kd)
    k = raw
    if kd.normalize:
        dx = raw_from_profiles(self_profiles(X, xl, kd), kd)
        dy = dx if sym else raw_from_profiles(self_profiles(Y, yl, kd), kd)
        k = raw / np.maximum(np.sqrt(dx[:, None] * dy[None, :]), 1e-10)
    k = _finish(k, kd)
    if sym:
        k = np.triu(k) + np.triu(k, 1).T
    return k


# ---------------------------------------------------------------------------
# Neighbour masks and the index-based CPU baseline
# ---------------------------------------------------------------------------


def neighbor_masks(l: int, h: np.ndarray, dmax: int):
    """XOR masks of every l-mer within dmax mismatches whose h is non-zero,
    sorted by mask value, with their mismatch counts
    (kernels/lmer_index.py:67-87)."""
    masks, levels = [], []
    for m in range(dmax + 1):
        if h[m] == 0:
            continue
        for pos in combinations(range(l), m):
            for deltas in product((1, 2, 3), repeat=m):
                x = 0
                for p, dl in zip(pos, deltas):
                    x |= dl << (2 * p)
                masks.append(x)
                levels.append(m)
    masks = np.array(masks, np.uint32)
    levels = np.array(levels, np.int32)
    order = np.argsort(masks, kind="stable")
    return masks[order], levels[order]


class IndexBaseline:
    """The reference's CPU scoring path, restated in C with pthreads: an l-mer
    CSR over the SVs' windows (kernels/lmer_index.py:161-200) and the fused
    query + reduce (kernels/lmer_index_cpu.py:71-120)."""

    def __init__(self, model: OracleModel, sv_diag=None, threads: int = 1):
        kd = model.kd
        self.kd = kd
        self.model = model
        fs, rs = pack(model.sv, model.sv_lengths, kd.l)
        ws = row_weights(fs, kd)
        wr = None
        if ws is not None:
            W = fs.shape[1]
            wr = np.zeros_like(ws)
            counts = (fs != PAD).sum(axis=1)
            for r, n in enumerate(counts):
                wr[r, W - n:] = ws[r, :n][::-1]
        S, W = fs.shape
        self._keep = (fs, rs, ws, wr)
        self.h = lib().orc_index_build(_p(fs), _p(rs if kd.include_rc else None),
                                       _p(ws), _p(wr), S, W, kd.l)
        self.masks, lev = neighbor_masks(kd.l, kd.h, kd.dmax)
        self.weights = kd.h[lev].astype(np.float64)
        ds = sv_diag if sv_diag is not None else raw_from_profiles(
            self_profiles(model.sv, model.sv_lengths, kd, threads), kd)
        self.inv_ds = 1.0 / np.sqrt(np.clip(ds, 1e-20, None))

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().orc_index_free(self.h)
            except TypeError:  # interpreter shutdown: the module's globals are gone
                pass
            self.h = None

    def scores(self, xc, xl=None, threads: int = 1, diag_x=None) -> np.ndarray:
        kd = self.kd
        fx, _ = pack(xc, xl, kd.l)
        wx = row_weights(fx, kd)
        dx = diag_x if diag_x is not None else raw_from_profiles(self_profiles(xc, xl, kd, threads), kd)
        inv_dx = 1.0 / np.sqrt(np.clip(dx, 1e-20, None))
        B, W = fx.shape
        out = np.zeros(B)
        coef = np.ascontiguousarray(self.model.coef, np.float64)
        lib().orc_index_reduce(self.h, _p(fx), _p(wx), B, W, _p(self.masks), _p(self.weights),
                               len(self.masks), _p(inv_dx), _p(self.inv_ds), _p(coef),
                               float(kd.gamma), int(kd.rbf), _p(out), threads)
        return out[:, None] + self.model.bias
