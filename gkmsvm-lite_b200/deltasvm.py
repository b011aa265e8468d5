"""DeltaSVM weights of a GkmSVM (svm.py:664-785 of gkmsvm-lite): one weight per
l-mer, the model's kernel sum on that l-mer alone, in DeltaSVM order (the
first base most significant).

Kernels with an exact l-mer table (-t 0/1/2/4, l <= 12) read the weights off
the table on the GPU (gkm_deltasvm_table, with the l-mer's own normalisation
when query_norm).  Other models (RBF, or no table) score every canonical l-mer
as a one-window row through the model's scoring path (the l-mer index, or the
pairwise forms) and copy each weight to the l-mer's reverse complement, as the
reference does.  The DeltaSVM scoring model itself is not part of this
package: to_deltasvm returns the weights with the fields DeltaSVM is built
from (deltasvm.py:75-98).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import engine
from ._lib import call, ptr, stream_handle
from .kernels import RbfKernel

# largest l accepted: 4^14 float64 weights = 2 GiB (svm.py:664-665)
_MAX_DELTASVM_L = 14
# l-mers scored per pass of the kernel route
_DELTASVM_CHUNK = 1 << 22


@dataclass
class DeltaSVMWeights:
    """What the reference's DeltaSVM(weights, l, k, include_rc=False, bias)
    is built from: weights [4^l] float64 in DeltaSVM order, k = l."""

    weights: torch.Tensor | np.ndarray
    l: int
    k: int
    include_rc: bool
    bias: float


def deltasvm_weights(model, *, query_norm: bool = False, verbose: bool = False) -> torch.Tensor:
    """[4^l] float64 device weights (svm.py:706-750): the kernel sum of each
    l-mer alone, without its own normalisation 1/sqrt(K(u, u)) unless
    query_norm (RBF models always keep it)."""
    kernel = model.kernel
    l = kernel.l
    if l > _MAX_DELTASVM_L:
        raise ValueError(
            f"to_deltasvm() requires l <= {_MAX_DELTASVM_L} "
            f"(4^{l} = {4**l:,} weights would use {4**l * 4 / 1e9:.1f} GB). Got l={l}.")
    dev = model._require_gpu()
    table = model._build_lmer_table()
    if table is not None:
        wt = kernel.window_weights(1)
        out = torch.empty(4**l, dtype=torch.float64, device=dev)
        call("gkm_deltasvm_table", model._spec().ref, ptr(table), 1.0 if wt is None else float(wt[0]),
             int(bool(query_norm) and kernel.normalize), ptr(out), stream_handle())
        return out
    return _weights_from_kernel(model, query_norm, verbose)


def _weights_from_kernel(model, query_norm: bool, verbose: bool) -> torch.Tensor:
    """Every canonical l-mer scored as a one-window row (svm.py:756-785)."""
    kernel = model.kernel
    base = kernel.base
    l = kernel.l
    dev = model._require_gpu()
    spec = model._spec()
    unnorm = not query_norm and base.normalize and not isinstance(kernel, RbfKernel)
    n_all = 4**l
    full = n_all - 1
    weights = torch.empty(n_all, dtype=torch.float64, device=dev)
    # DeltaSVM digit p (from the most significant end) -> packed position p
    down = torch.arange(l - 1, -1, -1, device=dev, dtype=torch.int64) * 2
    up = torch.arange(l, device=dev, dtype=torch.int64) * 2
    starts = range(0, n_all, _DELTASVM_CHUNK)
    if verbose:
        from tqdm import tqdm
        starts = tqdm(starts, desc="to_deltasvm")
    for start in starts:
        idx = torch.arange(start, min(start + _DELTASVM_CHUNK, n_all), dtype=torch.int64, device=dev)
        fwd = (((idx[:, None] >> down) & 3) << up).sum(dim=1)  # packed window of the l-mer
        # the reverse complement's DeltaSVM index is full - fwd, its packed window full - idx
        rc_idx = full - fwd
        if base.include_rc:
            keep = idx <= rc_idx
            idx, fwd, rc_idx = idx[keep], fwd[keep], rc_idx[keep]
        if idx.numel() == 0:
            continue
        fw = fwd.to(torch.int32)[:, None].contiguous()
        rw = (full - idx).to(torch.int32)[:, None].contiguous() if base.include_rc else None
        counts = torch.ones(idx.numel(), dtype=torch.int32, device=dev)
        w = model._score_packed(fw, rw, counts) - model.bias
        if unnorm:
            diag = engine.self_kernel(spec, fw, rw, counts)
            w = w * torch.sqrt(torch.clamp(diag, min=1e-10))
        weights[idx] = w
        if base.include_rc:
            weights[rc_idx] = w
    return weights


def to_deltasvm(model, *, device: str = "cpu", query_norm: bool = False, verbose: bool = False) -> DeltaSVMWeights:
    """The model as DeltaSVM weights (svm.py:706-750): k = l, no RC (the
    weights already hold both strands), the model's bias; weights on the host
    (device "cpu") or left on the GPU."""
    w = deltasvm_weights(model, query_norm=query_norm, verbose=verbose)
    if str(device) == "cpu":
        w = w.cpu().numpy()
    l = model.kernel.l
    return DeltaSVMWeights(w, l, l, False, float(model.bias))
