"""Gram matrix for training (gram.py:21-164 of gkmsvm-lite) on the GPU.

The columns Y are indexed once (or joined pair by pair when the index does not
apply) and the rows X queried in blocks; a self-Gram computes only the upper
triangle and mirrors it, so the result is exactly symmetric.  Normalisation
and the RBF finish run on the device (gkm_gram_finish); the matrix is
returned as host float64 NumPy, as the reference returns it.
"""

from __future__ import annotations

import numpy as np
import torch

from . import engine
from ._lib import require_cuda
from .inputs import SeqBatch
from .kernels import DirectGkmKernel, RbfKernel

_MAX_BLOCK_BYTES = 2 * 2**30


def compute_gram(kernel, X, Y=None, *, chunk_size=1000, verbose=False, out=None, lengths=None,
                 y_lengths=None, device=None) -> np.ndarray:
    """K(X, Y) [N, M] float64 (K(X, X) when Y is None), normalised and
    finished as the kernel defines; out: optional host array to fill."""
    require_cuda()
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    base = kernel.base
    symmetric = Y is None
    xb = SeqBatch.read(X, lengths)
    yb = xb if symmetric else SeqBatch.read(Y, y_lengths)
    N, M = xb.B, yb.B
    spec = engine.Spec(base, dev)
    bx, rx, cx = engine.pack(spec, xb.on(dev), xb.lengths)
    if symmetric:
        by, ry, cy = bx, rx, cx
    else:
        by, ry, cy = engine.pack(spec, yb.on(dev), yb.lengths)
    spec.check_rows(int(max(bx.shape[1], by.shape[1])))
    dx = dy = None
    if base.normalize:
        dx = engine.self_kernel(spec, bx, rx, cx)
        dy = dx if symmetric else engine.self_kernel(spec, by, ry, cy)
    n_windows = int(cy.sum().item()) * (2 if base.include_rc else 1)
    use_index = isinstance(base, DirectGkmKernel) and n_windows > 0 and base.index_applies(n_windows)
    raw = torch.zeros((N, M), dtype=torch.float64, device=dev)
    if use_index:
        index = engine.DeviceIndex(spec, by, ry, cy, engine.masks_tensor(base, dev))
        try:
            index.pairwise(bx, cx, diag_offset=0 if symmetric else None, out=raw)
        finally:
            index.close()
    else:
        step = max(1, _MAX_BLOCK_BYTES // (8 * M))
        for s in range(0, N, step):
            r, _ = engine.pairwise(spec, bx[s:s + step], cx[s:s + step], by, ry, cy)
            raw[s:s + step] = r
    rbf = isinstance(kernel, RbfKernel)
    gram = engine.gram_finish(raw, dx, dy, kernel.gamma if rbf else 0.0, rbf, symmetric)
    host = gram.cpu().numpy()
    if out is not None:
        out[...] = host
        return out
    return host
