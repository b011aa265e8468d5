"""GkmExplain attributions and the GkmExplain mutation impact on the GPU
(explain/core.py:34-247, explain/lmer.py, explain/impact.py of gkmsvm-lite).

Attributions go through l-mer weights: each query window visits the l-mers
within the explain cutoff and adds alpha/kappa (or the perturbation deltas)
times the neighbour's weight to each of its positions.  The weight of a
neighbour v is V[v] = sum_s coef_s / sqrt(K(sv, sv)) (occurrences of v in sv_s
and its RC) for linear kernels, and for RBF kernels the per-query SV weights
summed over the l-mer index's entries of v (gkm_explain_lmer).

Linear kernels can instead read every window's attribution from the explain
table (explain/table.py): [4^l, 4, l] float64 built once per mode on the GPU by
Walsh-Hadamard transforms (gkm_explain_table_build) and cached on the model;
use_explain_table = True / False / "auto" (built once a call explains enough
rows to pay for it, and at most 2 GiB).
"""

from __future__ import annotations

import numpy as np
import torch

from . import engine
from ._lib import call, ptr, stream_handle
from .inputs import SeqBatch, allele_batches, device_codes, nan_rows, per_position
from .kernels import INDEX_MAX_L, MAX_NEIGHBORS, RbfKernel, explain_tables, neighbor_count, neighbor_masks

_MODE_ALIASES = {0: "importance", 1: "hypothetical", 2: "perturbation", "importance": "importance",
                 "hypothetical": "hypothetical", "perturbation": "perturbation"}


def _rbf_scale(k_norm: torch.Tensor, gamma: float) -> torch.Tensor:
    pos = k_norm > 0
    safe = torch.where(pos, k_norm, torch.ones_like(k_norm))
    return torch.where(pos, (torch.exp(gamma * (safe - 1)) - np.exp(-gamma)) / safe, torch.zeros_like(k_norm))


def _explain_masks(model, perturbation: bool, dev):
    base = model.kernel.base
    a, b, dmax = explain_tables(base, perturbation)
    key = ("explain_masks", perturbation)
    c = model._sv_cache
    if key not in c:
        nonzero = tuple(bool(a[m] != 0 or b[m] != 0) for m in range(base.l + 1))
        masks = neighbor_masks(base.l, nonzero, dmax)
        c[key] = (torch.from_numpy(masks.view(np.int32).copy()).to(dev),
                  torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev))
    return c[key]


def _explain_V(model) -> torch.Tensor:
    """V[v] = sum_s coef_s / sqrt(K(sv, sv)) over the window-weighted
    occurrences of l-mer v in each SV and its RC (explain/common.py:87-98)."""
    c = model._sv_cache
    if "explain_V" not in c:
        spec = model._spec()
        fwd, rc, counts = model._sv_packed()
        coef = model._sv_coef() * model._inv_ds()
        index = c.get("index")
        tmp = None
        if index is None:
            tmp = engine.DeviceIndex(spec, fwd, rc, counts, model._masks())
            index = tmp
        c["explain_V"] = index.lmer_weights(coef.contiguous())
        if tmp is not None:
            tmp.close()
    return c["explain_V"]


# SV windows a query window visits per l-mer neighbour before the per-SV pair
# loop is the cheaper form (explain/lmer.py:25)
_EXPLAIN_SV_WINDOWS_PER_NEIGHBOR = 6


def _explain_uses_pairs(model, perturbation: bool) -> bool:
    """Whether attributions go through the per-SV pair loop
    (explain/core.py:170-247) because the l-mer path does not apply
    (explain/lmer.py:60-85): the index is off, l > 12, no pair contributes,
    the neighbourhood outweighs the SV windows, or an RBF model has no index."""
    base = model.kernel.base
    _, _, dmax = explain_tables(base, perturbation)
    if not model.use_lmer_index or base.l > INDEX_MAX_L or dmax < 0:
        return True
    n = neighbor_count(base.l, dmax)
    if n > MAX_NEIGHBORS:
        fwd, rc, _ = model._sv_packed()
        sv_windows = fwd.numel() + (0 if rc is None else rc.numel())
        if n * _EXPLAIN_SV_WINDOWS_PER_NEIGHBOR > sv_windows:
            return True
    return isinstance(model.kernel, RbfKernel) and model._sv_index() is None


def _explain_pair_tables(model, perturbation: bool, dev):
    """Device (table_a, table_b) and the minimum matches of a contributing pair."""
    base = model.kernel.base
    key = ("explain_pair_tables", perturbation)
    c = model._sv_cache
    if key not in c:
        a, b, dmax = explain_tables(base, perturbation)
        c[key] = (torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev), base.l - dmax)
    return c[key]


# explain table limits and cost model ("auto"): build cost per entry of 4^l x l
# and the direct l-mer path's cost per query window, measured on B200 at l=11
# (a first call that builds V and the table: 0.17 s; the direct path: ~3e6
# windows/s, the table ~3e7), so a call of ~300k windows pays for it
_EXPLAIN_TABLE_MAX_L = 12
_EXPLAIN_TABLE_BYTES = 2 * 2**30
_TABLE_BUILD_S_PER_ENTRY = 1e-9
_DIRECT_S_PER_WINDOW = 1.5e-7


def _explain_table(model, n_windows: int, perturbation: bool, dev):
    """The cached explain table of this mode, built if use_explain_table calls
    for it, or None (RBF models have none)."""
    use = model.use_explain_table
    kernel = model.kernel
    base = kernel.base
    l = base.l
    if use is False or isinstance(kernel, RbfKernel) or l > _EXPLAIN_TABLE_MAX_L:
        return None
    tables = model._explain_tables
    if perturbation not in tables:
        n = 4 ** l
        if use == "auto" and (n * 4 * l * 8 > _EXPLAIN_TABLE_BYTES
                              or n_windows * _DIRECT_S_PER_WINDOW < _TABLE_BUILD_S_PER_ENTRY * n * l):
            return None
        _, ta, tb = _explain_masks(model, perturbation, dev)
        A = torch.empty((n, 4, l), dtype=torch.float64, device=dev)
        call("gkm_explain_table_build", model._spec().ref, ptr(_explain_V(model)), ptr(ta), ptr(tb), ptr(A),
             stream_handle())
        tables[perturbation] = A
    return tables[perturbation]


def gkmexplain(model, x, *, mode="importance", lengths=None, batch_size=50, verbose=False) -> torch.Tensor:
    """[B, 4, L] float64 attributions (explain/core.py:34-113): importance =
    hypothetical x one-hot (N credited to A), hypothetical, or perturbation."""
    resolved = _MODE_ALIASES.get(mode)
    if resolved is None:
        raise ValueError(f"mode must be 'importance', 'hypothetical', or 'perturbation' (or 0/1/2), got {mode!r}")
    dev = model._require_gpu()
    batch = SeqBatch.read(x, lengths)
    short = batch.short(model.kernel.base.l, "attributions")
    B = batch.B
    bs = max(1, int(batch_size)) if batch_size else B
    # the table (if any) is chosen for the whole call, as the reference does
    n_windows = batch.n_windows(model.kernel.base.l)
    table = _explain_table(model, n_windows, resolved == "perturbation", dev)
    parts = []
    it = range(0, B, bs)
    if verbose:
        from tqdm import tqdm
        it = tqdm(it, desc="GkmExplain")
    for s in it:
        p = batch.part(s, bs)
        parts.append(_explain_rows(model, p.codes, p.lengths, resolved, dev, table))
    out = parts[0] if len(parts) == 1 else torch.cat(parts)
    return per_position(out, batch, short)


def _explain_rows(model, x, lengths, mode, dev, table=None, check=True):
    """[B, 4, L] attributions of one pass (x: host or device codes).
    check=False: no host synchronisation (the index's exactness check is the
    caller's)."""
    kernel = model.kernel
    base = kernel.base
    spec = model._spec()
    L = x.shape[-1]
    if L < base.l:
        return torch.full((x.shape[0], 4, L), float("nan"), dtype=torch.float64, device=dev)
    xt = device_codes(x, dev)
    fwd, rc, counts = engine.pack(spec, xt, lengths)
    spec.check_rows(int(fwd.shape[1]))
    perturbation = mode == "perturbation"
    B, W = fwd.shape
    if base.normalize:
        dx = engine.self_kernel(spec, fwd, rc, counts)
        inv_dx = 1.0 / torch.sqrt(torch.clamp(dx, min=1e-20))
    else:
        inv_dx = torch.ones(B, dtype=torch.float64, device=dev)
    V = index = w = out = None
    if table is None and _explain_uses_pairs(model, perturbation):
        out = _explain_pairs(model, spec, fwd, counts, inv_dx, L, perturbation, dev)
    elif table is not None:
        out = torch.empty((B, 4, L), dtype=torch.float64, device=dev)
        call("gkm_explain_table", spec.ref, ptr(table), ptr(fwd), ptr(counts), B, W, L, ptr(inv_dx),
             int(perturbation), ptr(out), stream_handle())
    elif isinstance(kernel, RbfKernel):
        index = model._sv_index()  # not None: _explain_uses_pairs
        raw, _ = index.pairwise(fwd, counts, check=check)
        inv_ds = model._inv_ds()
        k_norm = raw * inv_dx[:, None] * inv_ds[None, :]
        w = (model._sv_coef() * inv_ds)[None, :] * _rbf_scale(k_norm, kernel.gamma)
        w = w.contiguous()
    else:
        V = _explain_V(model)
    if table is None and out is None:
        masks, ta, tb = _explain_masks(model, perturbation, dev)
        out = torch.empty((B, 4, L), dtype=torch.float64, device=dev)
        call("gkm_explain_lmer", spec.ref, ptr(fwd), ptr(counts), B, W, L, ptr(inv_dx), ptr(V),
             None if index is None else index.handle, ptr(w), ptr(masks), int(masks.numel()), ptr(ta), ptr(tb),
             int(perturbation), ptr(out), stream_handle())
    if mode == "importance":
        oh = torch.nn.functional.one_hot(xt.long(), 4).permute(0, 2, 1).to(out.dtype)
        out = out * oh
    return out


def _explain_pairs(model, spec, fwd, counts, inv_dx, L: int, perturbation: bool, dev) -> torch.Tensor:
    """[B, 4, L] attributions by the per-SV pair loop (gkm_explain_pairs):
    per-(row, SV) weights coef_s / sqrt(K(sv, sv)), RBF-scaled by the row's
    normalised kernel value with each SV (explain/core.py:207-226)."""
    kernel = model.kernel
    by, ry, cy = model._sv_packed()
    inv_ds = model._inv_ds()
    B, W = fwd.shape
    S = int(by.shape[0])
    w = (model._sv_coef() * inv_ds)[None, :].expand(B, S)
    if isinstance(kernel, RbfKernel):
        raw, _ = engine.pairwise(spec, fwd, counts, by, ry, cy)
        w = w * _rbf_scale(raw * inv_dx[:, None] * inv_ds[None, :], kernel.gamma)
    w = w.contiguous()
    ta, tb, min_matches = _explain_pair_tables(model, perturbation, dev)
    out = torch.empty((B, 4, L), dtype=torch.float64, device=dev)
    call("gkm_explain_pairs", spec.ref, ptr(fwd), ptr(counts), B, W, L, ptr(inv_dx), ptr(by), ptr(ry), ptr(cy), S,
         int(by.shape[1]), ptr(w), ptr(ta), ptr(tb), int(min_matches), int(perturbation), ptr(out), stream_handle())
    return out


def mutation_impact(model, ref, alt, *, ref_lengths=None, alt_lengths=None, batch_size=None,
                    verbose=False) -> torch.Tensor:
    """[B, 1] GkmExplain mutation impact (lsgkm gkmexplain -m 5,
    explain/impact.py:51-194): sum_j coef_j dK_j with K normalised by the
    reference allele's norm; RBF kernels scale each SV by
    (exp(g (K_j - 1)) - exp(-g)) / K_j."""
    dev = model._require_gpu()
    kernel = model.kernel
    base = kernel.base
    rb, ab = allele_batches(ref, alt, ref_lengths, alt_lengths)
    L, B = rb.L, rb.B
    # a variant whose reference or alternative allele has no window is NaN
    s = SeqBatch.stacked(rb, ab).short(base.l, "mutation impacts")
    short = None if s is None else s.reshape(2, -1).any(axis=0)
    W = max(L - base.l + 1, 0)
    model._plan_lmer_table(B * 2 * (min(base.l, W) if model._index_applies() else W))
    if L < base.l:
        return torch.full((B, 1), float("nan"), dtype=torch.float64, device=dev)
    spec = model._spec()
    bs = B if batch_size is None else max(1, batch_size)
    parts = []
    rbf = isinstance(kernel, RbfKernel)
    gamma = kernel.gamma if rbf else 0.0
    for s in range(0, B, bs):
        pair = SeqBatch.stacked(rb.part(s, bs), ab.part(s, bs))
        n = pair.B // 2
        fwd, rc, counts = engine.pack(spec, pair.on(dev), pair.lengths)
        spec.check_rows(int(fwd.shape[1]))
        table = model._lmer_table_for()
        if table is not None:
            _, raw, diag = engine.table_score(spec, table, fwd, rc, counts, 0.0, base.normalize,
                                              want_parts=True)
            dk = raw[n:] - raw[:n]
            if base.normalize:
                dk = dk / torch.sqrt(torch.clamp(diag[:n], min=1e-10))
            parts.append(dk)
            continue
        dr = engine.self_kernel(spec, fwd[:n], None if rc is None else rc[:n], counts[:n]) if base.normalize else None
        index = model._sv_index()
        if index is not None:
            kb, _ = index.pairwise(fwd, counts)
        else:
            by, ry, cy = model._sv_packed()
            kb, _ = engine.pairwise(spec, fwd, counts, by, ry, cy)
        ds = model._sv_diag() if base.normalize else None
        parts.append(engine.impact(kb, n, dr, ds, model._sv_coef(), gamma, rbf))
    out = torch.cat(parts)[:, None]
    return nan_rows(out, short)
