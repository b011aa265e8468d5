"""Kernel types of the gapped-k-mer path: host-side descriptors.

Each kernel reduces to a pair weight h(m) by mismatch count m (zero past
dmax), optional centre window weights (-t 4/-t 5), reverse-complement and
normalisation flags, and for RBF kernels gamma.  The classes keep the names,
constructor arguments and attributes of gkmsvm-lite's kernel classes
(kernels/direct.py:209-253, kernels/esttrunc.py:9-38,
kernels/weighted.py:389-502, kernels/rbf.py:9-57) so that models, Gram calls
and tests built on them read the same; the computation happens on the device
(gkm_spec in include/gkm_b200.h).
"""

from __future__ import annotations

from functools import lru_cache
from itertools import combinations, product
from math import comb

import numpy as np

MAX_L = 15
# l-mer index limits (kernels/lmer_index.py:48-58)
INDEX_MAX_L = 12
MAX_NEIGHBORS = 8192
DENSE_MAX_NEIGHBORS = 32768
DENSE_WINDOWS_PER_LMER = 4
# l-mer table limit (lmer_table.py:31) and the masked-join plan size
# (kernels/masked.py:129) that decides whether a table exists
MAX_TABLE_L = 12
_MAX_PLAN_MASKS = 1000


def estimated_lmer_table(l: int, k: int, truncate: bool) -> np.ndarray:
    """LS-GKM's estimated l-mer kernel weights h(m), m = 0..l (the algorithm of
    kernels/esttrunc.py:40-110, LS-GKM's calc_gkm_kernel_lmerest_wt).

    1. wm[i]: the gapped-k-mer match weight of i mismatching informative
       positions, from a recursion over window length (normalised by
       C(l, k) 4^l);
    2. est[m] = sum_i wm[i] C(l-m, k-i) C(m, i), truncated to 0 from the first
       value below 1e-50 on when truncate;
    3. h(l - m) = sum over (m1, m2, t) of the number of ways two l-mers at
       distances m1, m2 from a third end m apart, times est[m1] est[m2].
    The floating-point operations follow the reference's order."""
    b = 4
    old = [[1.0] * (k + 1) for _ in range(k + 1)]
    new = [[1.0] * (k + 1) for _ in range(k + 1)]
    for il in range(1, l + 1):
        for ik in range(1, k + 1):
            new[ik][0] = old[ik][0] + (b - 1) * old[ik - 1][0]
            for jm in range(1, ik + 1):
                new[ik][jm] = (new[ik - 1][jm - 1] * (ik - il)) / ik
        old, new = new, old
    nnorm = comb(l, k) * (b**l)
    wm = [old[k][i] / nnorm for i in range(k + 1)]
    est = []
    for m in range(l + 1):
        s = 0.0
        for i in range(min(m, k) + 1):
            if l - m >= k - i:
                s += wm[i] * comb(l - m, k - i) * comb(m, i)
        est.append(s)
    if truncate:
        cut = next((i for i, v in enumerate(est) if v < 1e-50), l + 1)
        est = [v if i < cut else 0.0 for i, v in enumerate(est)]
    h = [0.0] * (l + 1)
    for m in range(l + 1):
        w = 0.0
        for m1 in range(l + 1):
            e1 = est[m1]
            if e1 == 0.0:
                continue
            for m2 in range(l + 1):
                e2 = est[m2]
                if e2 == 0.0:
                    continue
                for t in range(min(m, l) + 1):
                    r = m1 + m2 - 2 * t - l + m
                    diff = m1 - t
                    if r < 0 or diff > l - m or r > diff:
                        continue
                    w += (comb(m, t) * comb(l - m, diff) * comb(diff, r) * ((b - 1) ** t)
                          * ((b - 2) ** r)) * e1 * e2
        h[l - m] = w
    return np.array(h, dtype=np.float64)


@lru_cache(maxsize=64)
def mask_plan(table: tuple, l: int, min_matches: int):
    """The masked-join decomposition of a mismatch weight table (the
    reference's kernels/masked.py:45-69): with dmax = l - min_matches, the
    weights h(m), m <= dmax, as a sum over mask sizes j = l - dmax .. l of
    a_j C(l - m, j) -- the number of size-j position subsets on which two
    l-mers with m mismatches agree.  Returns [(j, a_j, positions [C(l, j), j]
    int64)] for the sizes with a non-zero coefficient, or None when there is no
    plan (no weight, or more than _MAX_PLAN_MASKS masks)."""
    dmax = l - min_matches
    if dmax < 0 or min_matches < 1:
        return None
    sizes = list(range(l - dmax, l + 1))
    if sum(comb(l, j) for j in sizes) > _MAX_PLAN_MASKS:
        return None
    system = np.array([[comb(l - m, j) for j in sizes] for m in range(dmax + 1)], dtype=np.float64)
    coef = np.linalg.solve(system, np.asarray(table, dtype=np.float64)[: dmax + 1])
    floor = 1e-12 * np.abs(coef).max()
    return [(j, float(c), np.array(list(combinations(range(l), j)), dtype=np.int64))
            for j, c in zip(sizes, coef) if abs(c) > floor]


def neighbor_count(l: int, dmax: int) -> int:
    return sum(comb(l, m) * 3**m for m in range(dmax + 1))


# Costs per query window on B200 (the fused index query and the pairwise
# forms, measured on the config-3 and t=0 workloads): an index lookup per SV
# tile (neighbour masks read from global memory past the 6,144 that fit in
# shared memory: about 3x), an index hit, and a window pair of the slower
# all-pairs form at dmax >= 4 (~2e12 pairs/s).  SV tiles hold about 16M windows.
_INDEX_LOOKUP_S = 2.6e-12
_INDEX_HIT_S = 1.7e-12
_PAIR_S = 5e-13
_STAGED_MASKS = 6144
_TILE_WINDOWS = 16_000_000


def index_cost_below_pairs(l: int, n_neighbors: int, n_windows: int) -> bool:
    """Whether the index costs less per query window than scoring every window
    pair, for n_windows indexed windows: lookups per tile plus hits (the
    expected share of windows within the neighbourhood, n_neighbors / 4^l, for
    uniform bases) against n_windows pairs."""
    tiles = 1 + n_windows // _TILE_WINDOWS
    lookup = _INDEX_LOOKUP_S * (3 if n_neighbors > _STAGED_MASKS else 1)
    index = n_neighbors * tiles * lookup + n_windows * (n_neighbors / 4**l) * _INDEX_HIT_S
    return index < n_windows * _PAIR_S


@lru_cache(maxsize=32)
def neighbor_masks(l: int, nonzero: tuple, dmax: int) -> np.ndarray:
    """XOR masks of every l-mer within dmax mismatches of a window, levels m
    with nonzero[m] only, sorted by mask (kernels/lmer_index.py:67-87), each
    packed as mask | m << 24 (uint32)."""
    out = []
    for m in range(dmax + 1):
        if not nonzero[m]:
            continue
        for pos in combinations(range(l), m):
            for deltas in product((1, 2, 3), repeat=m):
                x = 0
                for p, dl in zip(pos, deltas):
                    x |= dl << (2 * p)
                out.append((x, m))
    out.sort(key=lambda t: t[0])
    return np.array([x | (m << 24) for x, m in out], dtype=np.uint32)


def window_weight_table(M: int, H: float, n: int = 65537) -> np.ndarray:
    """[n] uint8 window weight by distance |W//2 - i| from the centre, with the
    reference's expression (kernels/weighted.py:38-43), so every weight is
    bit-identical to window_weights(W)[i]."""
    dist = np.arange(n)
    wt = np.floor(M * np.exp(-1 * np.log(2) * dist / H) + 1)
    return np.minimum(wt, M).astype(np.uint8)


class GkmKernel:
    """Base of every kernel type."""

    def __init__(self, l: int, k: int, *, normalize: bool = True, include_rc: bool = True):
        if k > l:
            raise ValueError(f"k ({k}) must be <= l ({l})")
        if l < 1:
            raise ValueError(f"l must be >= 1, got {l}")
        if k < 1:
            raise ValueError(f"k must be >= 1, got {k}")
        self.l = l
        self.k = k
        self.normalize = normalize
        self.include_rc = include_rc

    @property
    def base(self) -> "GkmKernel":
        return self

    @property
    def gamma_or_none(self):
        return None

    def finish(self, k_norm):
        return k_norm


class DirectGkmKernel(GkmKernel):
    """-t 0 gkm_cnt: h(m) = C(l - m, k), zero past d (every pair when d is None)."""

    use_masked = True

    def __init__(self, l, k, *, d=None, normalize=True, include_rc=True):
        if l > MAX_L:
            raise ValueError(f"l must be <= {MAX_L}, got {l}")
        super().__init__(l, k, normalize=normalize, include_rc=include_rc)
        self.d = d
        self._mismatch_table = np.array(
            [comb(l - m, k) if l - m >= k and (d is None or m <= d) else 0 for m in range(l + 1)],
            dtype=np.float64)
        self._min_matches = self._get_min_matches()

    def _get_min_matches(self) -> int:
        nz = np.flatnonzero(self._mismatch_table)
        return self.l - int(nz.max()) if len(nz) else self.l + 1

    @property
    def dmax(self) -> int:
        return self.l - self._min_matches

    def window_weights(self, W: int):
        return None

    @property
    def weighted(self) -> bool:
        return False

    def has_table(self) -> bool:
        """Whether an exact l-mer table exists: the masked-join plan does
        (kernels/masked.py:142-167)."""
        return self.l <= MAX_TABLE_L and self.mask_plan() is not None

    def mask_plan(self):
        """This kernel's masked-join plan (see mask_plan)."""
        return mask_plan(tuple(float(v) for v in self._mismatch_table), self.l, self._min_matches)

    def index_applies(self, n_windows: int | None = None) -> bool:
        """The reference's rule (kernels/lmer_index.py:97-109), and past it,
        neighbourhoods up to DENSE_MAX_NEIGHBORS wherever the index's cost
        per query window, measured on B200, is below the all-pairs forms'
        (index_cost_below_pairs).  Every form gives the same K_raw."""
        if self.dmax < 0 or self.l > INDEX_MAX_L:
            return False
        count = neighbor_count(self.l, self.dmax)
        dense = n_windows is not None and n_windows >= DENSE_WINDOWS_PER_LMER * 4**self.l
        if count <= (DENSE_MAX_NEIGHBORS if dense else MAX_NEIGHBORS):
            return True
        return count <= DENSE_MAX_NEIGHBORS and n_windows is not None and index_cost_below_pairs(
            self.l, count, n_windows)

    def masks(self) -> np.ndarray:
        t = self._mismatch_table
        return neighbor_masks(self.l, tuple(bool(v) for v in t), self.dmax)


class EstTruncGkmKernel(DirectGkmKernel):
    """-t 2 gkm_esttrunc (truncate) and -t 1 gkm_estfull, cut at d."""

    def __init__(self, l, k, *, d=3, normalize=True, include_rc=True, truncate=True):
        super().__init__(l, k, normalize=normalize, include_rc=include_rc)
        self.d = d
        self.truncate = truncate
        table = estimated_lmer_table(l, k, truncate)
        if d < l:
            table[d + 1:] = 0.0
        self._mismatch_table = table
        self._min_matches = self._get_min_matches()


class CenterWeightedGkmKernel(EstTruncGkmKernel):
    """-t 4 wgkm: the -t 2 table with centre window weights
    min(M, floor(M 2^(-|W/2 - i| / H) + 1))."""

    def __init__(self, l, k, *, d=3, M=50, H=50.0, normalize=True, include_rc=True):
        if not 1 <= M <= 255:
            raise ValueError(f"M must be in 1..255 (LS-GKM stores weights as uint8), got {M}")
        if H <= 0:
            raise ValueError(f"H must be positive, got {H}")
        super().__init__(l, k, d=d, normalize=normalize, include_rc=include_rc)
        self.M = int(M)
        self.H = float(H)
        self._wd = window_weight_table(self.M, self.H)

    @property
    def weighted(self) -> bool:
        return True

    def window_weights(self, W: int) -> np.ndarray:
        center = W // 2
        return self._wd[np.abs(center - np.arange(W))]


class RbfKernel(GkmKernel):
    """exp(gamma (K_norm - 1)) on a normalised base kernel (-t 3/5/6)."""

    def __init__(self, base: GkmKernel, gamma: float):
        super().__init__(base.l, base.k, normalize=True, include_rc=base.include_rc)
        self._base = base
        self.gamma = gamma

    @property
    def base(self) -> GkmKernel:
        return self._base

    @property
    def gamma_or_none(self):
        return self.gamma

    def finish(self, k_norm):
        import torch

        if isinstance(k_norm, torch.Tensor):
            return torch.exp(self.gamma * (k_norm - 1))
        return np.exp(self.gamma * (k_norm - 1))


class RbfGkmKernel(RbfKernel):
    """-t 3 gkmrbf."""

    def __init__(self, l, k, *, d=3, gamma=1.0, normalize=True, include_rc=True):
        super().__init__(EstTruncGkmKernel(l, k, d=d, normalize=True, include_rc=include_rc), gamma)
        self.d = d


class CenterWeightedRbfGkmKernel(RbfKernel):
    """-t 5 wgkmrbf."""

    def __init__(self, l, k, *, d=3, M=50, H=50.0, gamma=1.0, normalize=True, include_rc=True):
        super().__init__(CenterWeightedGkmKernel(l, k, d=d, M=M, H=H, normalize=True,
                                                 include_rc=include_rc), gamma)
        self.d = d
        self.M = M
        self.H = H


def _kernel_args(p, d=3, **extra):
    return dict(l=p["L"], k=p["k"], d=p.get("d", d), normalize=True,
                include_rc=p.get("include_rc", True), **extra)


def _gamma(p):
    return {"gamma": p.get("gamma", 1.0)}


def _weights(p):
    return {"M": p.get("M", 50), "H": p.get("H", 50.0)}


# The seven kernel modes (svm.py:64-106); gkm_cnt params without d count every pair
KERNEL_BUILDERS = {
    "gkm_cnt": lambda p: DirectGkmKernel(**_kernel_args(p, d=None)),
    "gkm_esttrunc": lambda p: EstTruncGkmKernel(**_kernel_args(p, truncate=True)),
    "gkm_estfull": lambda p: EstTruncGkmKernel(**_kernel_args(p, truncate=False)),
    "gkmrbf": lambda p: RbfGkmKernel(**_kernel_args(p, **_gamma(p))),
    "wgkm": lambda p: CenterWeightedGkmKernel(**_kernel_args(p, **_weights(p))),
    "wgkmrbf": lambda p: CenterWeightedRbfGkmKernel(**_kernel_args(p, **_weights(p), **_gamma(p))),
    "gkm_cnt_rbf": lambda p: RbfKernel(DirectGkmKernel(**_kernel_args(p)), **_gamma(p)),
}

KERNEL_ALIASES: dict = {
    "direct": "gkm_cnt", "estimated": "gkm_esttrunc", "estimated_full": "gkm_estfull",
    "rbf": "gkmrbf", "weighted": "wgkm", "weighted_rbf": "wgkmrbf", "direct_rbf": "gkm_cnt_rbf",
    0: "gkm_cnt", 1: "gkm_estfull", 2: "gkm_esttrunc", 3: "gkmrbf", 4: "wgkm", 5: "wgkmrbf",
    6: "gkm_cnt_rbf",
}


def resolve_kernel_type(kernel_type) -> str:
    """Internal name from a name, alias or LS-GKM -t integer (svm.py:126-152)."""
    if isinstance(kernel_type, str) and kernel_type.strip().isdigit():
        kernel_type = int(kernel_type)
    if isinstance(kernel_type, int):
        name = KERNEL_ALIASES.get(kernel_type)
        if name is None:
            raise ValueError(f"Unknown kernel type integer {kernel_type}. "
                             "Valid: 0-6 (LS-GKM -t flag; 6 from the kundajelab fork)")
        return name
    if kernel_type in KERNEL_BUILDERS:
        return kernel_type
    name = KERNEL_ALIASES.get(kernel_type)
    if name is not None:
        return name
    raise NotImplementedError(f"Unknown kernel type {kernel_type!r}")


# ---------------------------------------------------------------------------
# GkmExplain tables (explain/weights.py:9-57)
# ---------------------------------------------------------------------------


def explain_tables(base: DirectGkmKernel, perturbation: bool):
    """(table_a, table_b) [l + 2] float64 and the cutoff dmax of a contributing
    pair: alpha/kappa for importance and hypothetical, the perturbation
    deltas otherwise."""
    l, h = base.l, base._mismatch_table
    d = l if base.d is None else base.d
    a = np.zeros(l + 2)
    b = np.zeros(l + 2)
    if perturbation:
        for m in range(l + 1):
            now = float(h[m])
            a[m] = (float(h[m + 1]) if m + 1 <= l else 0.0) - now
            if m >= 1:
                b[m] = float(h[m - 1]) - now
    else:
        for m in range(min(d, l) + 1):
            if l - m > 0:
                a[m] = float(h[m]) / (l - m)
        for m in range(1, min(d, l) + 1):
            if l - m + 1 > 0:
                b[m] = float(h[m - 1]) / (l - m + 1)
    nz = [m for m in range(l + 1) if a[m] != 0 or b[m] != 0]
    return a, b, max(nz, default=-1)
