"""Column-cached SMO training (solver.py of gkmsvm-lite): C-SVC and
epsilon-SVR duals solved on the host by gkm_smo_solve (second-order working-set
selection, LRU column cache), with every kernel column computed on the GPU.

KernelColumnCache packs the training sequences on the device once, with their
self-kernels, and -- when the neighbourhood allows -- indexes them all in one
l-mer index, so a batch of columns is one index query of those rows (row
splits keep a small batch's query across the whole GPU); otherwise columns go
through the pairwise kernels.  Columns are normalised and finished (RBF) on
the device and copied to the host, where the solver keeps them.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np
import torch

from . import _lib, engine
from .inputs import SeqBatch
from .kernels import DirectGkmKernel, RbfKernel

# most columns computed per column-cache miss: the requested one plus the
# likeliest next working-set members, while the cache has free slots
_SMO_PREFETCH = 256
# fraction of available host memory for the solver's column cache
_SMO_CACHE_RAM_FRACTION = 0.25


class KernelColumnCache:
    """Normalised kernel columns K(:, i) of the training set, from the GPU.

    kernel: a kernel object (``GkmSVM.kernel`` or a ``KERNEL_BUILDERS``
    entry); X: [N, L] codes, [N, 4, L] one-hot or strings; lengths: each
    sequence's length when they differ."""

    def __init__(self, kernel, X, lengths=None, device=None):
        _lib.require_cuda()
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.kernel = kernel
        base = kernel.base
        xb = SeqBatch.read(X, lengths)
        self.N = xb.B
        self.spec = engine.Spec(base, dev)
        self.fwd, self.rc, self.counts = engine.pack(self.spec, xb.on(dev), xb.lengths)
        self.spec.check_rows(int(self.fwd.shape[1]))
        self.diag = (engine.self_kernel(self.spec, self.fwd, self.rc, self.counts) if base.normalize
                     else torch.ones(self.N, dtype=torch.float64, device=dev))
        n_windows = int(self.counts.sum().item()) * (2 if base.include_rc else 1)
        self.index = None
        if isinstance(base, DirectGkmKernel) and n_windows > 0 and base.index_applies(n_windows):
            self.index = engine.DeviceIndex(self.spec, self.fwd, self.rc, self.counts,
                                            engine.masks_tensor(base, dev))
        self.rbf = isinstance(kernel, RbfKernel)
        self.gamma = kernel.gamma if self.rbf else 0.0

    def close(self):
        if self.index is not None:
            self.index.close()
            self.index = None

    def raw_columns(self, indices) -> torch.Tensor:
        """[len(indices), N] device K_raw rows of the given sequences (K is symmetric)."""
        sel = torch.as_tensor(np.asarray(indices, dtype=np.int64), device=self.fwd.device)
        bx, cx = self.fwd[sel].contiguous(), self.counts[sel].contiguous()
        if self.index is not None:
            raw, _ = self.index.pairwise(bx, cx)
            return raw
        raw, _ = engine.pairwise(self.spec, bx, cx, self.fwd, self.rc, self.counts)
        return raw

    def device_columns(self, indices) -> torch.Tensor:
        """[len(indices), N] device rows of the normalised, finished kernel."""
        indices = [int(i) for i in indices]
        raw = self.raw_columns(indices)
        sel = torch.as_tensor(np.asarray(indices, dtype=np.int64), device=raw.device)
        if not self.kernel.base.normalize and not self.rbf:
            return raw
        return engine.gram_finish(raw.contiguous(), self.diag[sel].contiguous(), self.diag, self.gamma, self.rbf,
                                  False)

    def finished_diagonal(self) -> np.ndarray:
        """[N] host K(i, i) after normalisation and finish: 1 except for
        sequences without windows."""
        d = self.diag.cpu().numpy()
        if not self.kernel.base.normalize:
            return d
        k = d / np.maximum(np.sqrt(d * d), 1e-10)
        return np.exp(self.gamma * (k - 1.0)) if self.rbf else k

    def compute_columns(self, indices) -> dict:
        """{i: K(:, i)} as host float64 [N] arrays (solver.py:47-81)."""
        indices = [int(i) for i in indices]
        if not indices:
            return {}
        host = self.device_columns(indices).cpu().numpy()
        return {i: np.ascontiguousarray(host[b]) for b, i in enumerate(indices)}


def auto_cache_columns(N: int) -> int:
    """Column-cache size from available host memory: all N columns if they fit."""
    try:
        avail = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
    except (ValueError, OSError, AttributeError):
        avail = 8 << 30
    cols = int(avail * _SMO_CACHE_RAM_FRACTION // (8 * max(N, 1)))
    return max(min(256, N), min(N, cols))


def _check_kernel(kernel):
    if not kernel.base.normalize:
        raise ValueError("smo_solve needs a normalized kernel")


_LAST_STATS: dict = {}


def last_solve_stats() -> dict:
    """Iterations, column-provider calls and columns of the last solve."""
    return dict(_LAST_STATS)


def _solve(cache: KernelColumnCache, y, p, C, tol, max_iter, cache_size, verbose):
    N = cache.N
    y = np.ascontiguousarray(y, dtype=np.float64)
    p = np.ascontiguousarray(p, dtype=np.float64)
    n = y.shape[0]
    diag = np.ascontiguousarray(cache.finished_diagonal(), dtype=np.float64)
    errors: list[BaseException] = []
    stats = {"calls": 0, "columns": 0}

    def provider(count, idx_ptr, out_ptr, ctx):
        try:
            stats["calls"] += 1
            stats["columns"] += count
            idx = np.ctypeslib.as_array(idx_ptr, shape=(count,)).copy()
            cols = cache.device_columns(idx).cpu().numpy()
            out = np.ctypeslib.as_array(out_ptr, shape=(count * N,))
            out[:] = np.ascontiguousarray(cols, dtype=np.float64).ravel()
            return 0
        except BaseException as exc:  # noqa: BLE001 - raised after the solver returns
            errors.append(exc)
            return 1

    cb = _lib.COLUMNS_CB(provider)
    coef = np.zeros(n, dtype=np.float64)
    bias = ctypes.c_double()
    iters = ctypes.c_int64()
    st = _lib.load().gkm_smo_solve(
        n, N, y.ctypes.data, p.ctypes.data, diag.ctypes.data, float(C[0]), float(C[1]), float(tol), int(max_iter),
        int(min(cache_size, N)), _SMO_PREFETCH, cb, None, coef.ctypes.data, ctypes.byref(bias),
        ctypes.byref(iters), int(bool(verbose)))
    if errors:
        raise RuntimeError("SMO kernel column computation failed") from errors[0]
    _lib.check(st, "gkm_smo_solve")
    _LAST_STATS.clear()
    _LAST_STATS.update(stats, iterations=int(iters.value), n=n, N=N)
    return coef, float(bias.value), int(iters.value)


def smo_solve(kernel, X, y, C: float = 1.0, tol: float = 1e-3, max_iter: int = 10_000_000, cache_size=None,
              verbose: bool = False, lengths=None, pos_weight: float = 1.0):
    """C-SVC by column-cached SMO (solver.py:84-132).  y: [N] labels +1/-1.
    Returns (coefficients [N] = alpha_i y_i, bias) with score = K coef + bias."""
    _check_kernel(kernel)
    y = np.asarray(y.cpu() if isinstance(y, torch.Tensor) else y, dtype=np.float64)
    cache = KernelColumnCache(kernel, X, lengths)
    try:
        N = cache.N
        if cache_size is None:
            cache_size = auto_cache_columns(N)
        coef, bias, _ = _solve(cache, y, -np.ones(N), (C * pos_weight, C), tol, max_iter, cache_size, verbose)
    finally:
        cache.close()
    return coef, bias


def smo_svr_solve(kernel, X, z, C: float = 1.0, epsilon: float = 0.1, tol: float = 1e-3,
                  max_iter: int = 10_000_000, cache_size=None, verbose: bool = False, lengths=None):
    """epsilon-SVR by column-cached SMO (solver.py:135-175), LIBSVM's 2N-variable
    form.  Returns (coefficients [N] = alpha_i - alpha*_i, bias)."""
    _check_kernel(kernel)
    z = np.asarray(z.cpu() if isinstance(z, torch.Tensor) else z, dtype=np.float64)
    cache = KernelColumnCache(kernel, X, lengths)
    try:
        N = cache.N
        if cache_size is None:
            cache_size = auto_cache_columns(N)
        signs = np.r_[np.ones(N), -np.ones(N)]
        p = np.r_[epsilon - z, epsilon + z]
        coef, bias, _ = _solve(cache, signs, p, (C, C), tol, max_iter, cache_size, verbose)
    finally:
        cache.close()
    return coef[:N] + coef[N:], bias
