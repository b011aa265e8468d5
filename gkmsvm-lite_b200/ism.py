"""In silico mutagenesis (ism.py:21-320 of gkmsvm-lite) on the GPU.

Window-delta form: a substitution at p changes only the <= l windows that
cover p.  Kernels with an l-mer table read the changed windows' table weights
and the mutant self-kernels in one fused pass (gkm_ism_table); other kernels
(RBF) add the changed windows' index hits to the reference row's kernel
values and reduce over the SVs per mutant (gkm_index_mutants).
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import engine
from ._lib import call, ptr, stream_handle
from .inputs import SeqBatch, device_codes, per_position
from .kernels import RbfKernel

# Sequences per device pass: ISM outputs [B, 4, L] float64 per pass within this
_BLOCK_BYTES = 1 * 2**30
# Index-path ISM workspace (query rows and K_raw rows of a pass of positions)
_WORKSPACE_BYTES = 3 * 2**29


def ism(model, x, *, lengths=None, batch_size=None, verbose=False) -> torch.Tensor:
    """[B, 4, L] f(mutant) - f(x) for every single-base substitution; 0 past
    each row's length, NaN rows shorter than l (ism.py:21-64)."""
    dev = model._require_gpu()
    batch = SeqBatch.read(x, lengths)
    l = model.kernel.base.l
    short = batch.short(l, "ISM deltas")
    B, L = batch.B, batch.L
    model._plan_lmer_table(5 * l * B * L)
    bs = batch_size if batch_size is not None else max(1, _BLOCK_BYTES // (8 * 4 * L * 3))
    parts = []
    it = range(0, B, bs)
    if verbose:
        from tqdm import tqdm
        it = tqdm(it, desc="ISM")
    for s in it:
        p = batch.part(s, bs)
        parts.append(_ism_rows(model, p.codes, p.lengths, dev))
    out = parts[0] if len(parts) == 1 else torch.cat(parts)
    return per_position(out, batch, short)


def _ism_rows(model, x, lengths, dev, check=True, work=None):
    """[B, 4, L] deltas of one pass (x: host or device codes).  check=False:
    no host synchronisation (the index's exactness check is the caller's)."""
    base = model.kernel.base
    spec = model._spec()
    L = x.shape[-1]
    if L < base.l:
        return torch.full((x.shape[0], 4, L), float("nan"), dtype=torch.float64, device=dev)
    xt = device_codes(x, dev)
    fwd, rc, counts = engine.pack(spec, xt, lengths)
    spec.check_rows(int(fwd.shape[1]))
    table = model._lmer_table_for()
    if table is not None:
        _, raw, diag = engine.table_score(spec, table, fwd, rc, counts, 0.0, base.normalize, want_parts=True)
        return engine.ism_table(spec, table, fwd, counts, L, raw, diag, base.normalize)
    return _ism_index(model, fwd, rc, counts, L, check, work)


def _ism_index(model, fwd, rc, counts, L, check=True, work=None):
    kernel = model.kernel
    base = kernel.base
    spec = model._spec()
    index = model._sv_index()
    if index is None:
        raise NotImplementedError("ISM without an l-mer table needs the l-mer index "
                                  "(use_lmer_index=True and a neighbourhood it covers)")
    B, W = fwd.shape
    rbf = isinstance(kernel, RbfKernel)
    gamma = kernel.gamma if rbf else 0.0
    if base.normalize:
        diag = engine.self_kernel(spec, fwd, rc, counts)
        mut = engine.mutant_diag(spec, fwd, counts, L, diag)
        inv_dx = 1.0 / torch.sqrt(torch.clamp(diag, min=1e-20))
        inv_dmut = 1.0 / torch.sqrt(torch.clamp(mut, min=1e-20))
    else:
        inv_dx = torch.ones(B, dtype=torch.float64, device=fwd.device)
        inv_dmut = torch.ones((4, L, B), dtype=torch.float64, device=fwd.device)
    out = torch.empty((B, 4, L), dtype=torch.float64, device=fwd.device)
    if work is None:
        work = ism_workspace(model, B, L, fwd.device)

    def run():
        # the reference rows' K_raw; their scores come from it inside the call
        ref_raw, _ = index.pairwise(fwd, counts, check=False)
        call("gkm_index_mutants", index.handle, ptr(fwd), ptr(counts), B, W, L, ptr(ref_raw), None,
             ptr(inv_dx), ptr(inv_dmut), ptr(model._inv_ds()), ptr(model._sv_coef()), float(gamma), int(rbf),
             ptr(out), ptr(work), int(work.numel()), stream_handle())
        return out

    return index.checked(run) if check else run()


def ism_workspace_bytes(model, B: int, L: int, cap: int = None) -> int:
    """Bytes of an index-path ISM workspace for B rows x L positions: the query
    rows and K_raw rows of as many positions per chunk as fit in cap bytes
    (at least one position's)."""
    lo, hi = ctypes.c_int64(), ctypes.c_int64()
    call("gkm_index_mutants_workspace", model._sv_index().handle, B, L, ctypes.byref(lo), ctypes.byref(hi))
    return max(lo.value, min(hi.value, _WORKSPACE_BYTES if cap is None else cap))


def ism_pass_bytes(model, B: int, positions: int) -> int:
    """Workspace bytes of an index-path ISM pass over `positions` positions of
    B rows (a workspace of this size makes every pass that short)."""
    lo, hi = ctypes.c_int64(), ctypes.c_int64()
    call("gkm_index_mutants_workspace", model._sv_index().handle, B, max(1, int(positions)), ctypes.byref(lo),
         ctypes.byref(hi))
    return hi.value


def ism_workspace(model, B: int, L: int, device, cap: int = None) -> torch.Tensor:
    return torch.empty(ism_workspace_bytes(model, B, L, cap), dtype=torch.uint8, device=device)
