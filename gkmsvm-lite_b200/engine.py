"""Device operations on torch tensors: thin wrappers over the C ABI.

Every function takes and returns CUDA tensors and enqueues its work on the
current torch stream; nothing here synchronises except index creation (which
reads the entry count back) and explicit capacity checks.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr

U32 = torch.int32  # uint32 words are stored in int32 tensors (bit patterns)


def _st():
    return _lib.stream_handle()


class Spec:
    """gkm_spec of a base kernel, with its window-weight table on the device."""

    def __init__(self, base, device: torch.device):
        self.base = base
        self.device = device
        s = _lib.GkmSpec()
        s.l = base.l
        s.include_rc = int(bool(base.include_rc))
        s.weighted = int(bool(base.weighted))
        s.dmax = base.dmax
        h = np.zeros(16)
        h[: base.l + 1] = base._mismatch_table
        for m in range(16):
            s.h[m] = float(h[m])
        self.wd = None
        if base.weighted:
            self.wd = torch.from_numpy(base._wd).to(device)
            s.wd = self.wd.data_ptr()
            s.wd_len = int(self.wd.numel())
        self.c = s
        self.ref = ctypes.byref(s)

    def check_rows(self, counts_max: int):
        if self.wd is not None and counts_max >= self.c.wd_len:
            raise ValueError(f"rows of {counts_max} windows exceed the weight table")


def pack(spec: Spec, codes: torch.Tensor, lengths) -> tuple:
    """(fwd [B, W], rc [B, W] or None, counts [B] int32)."""
    B, L = codes.shape
    l = spec.base.l
    if L < l:
        raise ValueError(f"Sequence length {L} is shorter than window length {l}")
    W = L - l + 1
    dev = codes.device
    fwd = torch.empty((B, W), dtype=U32, device=dev)
    rc = torch.empty((B, W), dtype=U32, device=dev) if spec.base.include_rc else None
    counts = torch.empty(B, dtype=torch.int32, device=dev)
    ln = None
    if isinstance(lengths, torch.Tensor):
        ln = lengths.to(device=dev, dtype=torch.int64)
    elif lengths is not None:
        ln = torch.as_tensor(np.asarray(lengths, dtype=np.int64)).to(dev, non_blocking=True)
    call("gkm_pack", spec.ref, ptr(codes), ptr(ln), B, L, ptr(fwd), ptr(rc), ptr(counts), _st())
    return fwd, rc, counts


def self_kernel(spec: Spec, fwd, rc, counts, profile: bool = False):
    B, W = fwd.shape
    diag = torch.empty(B, dtype=torch.float64, device=fwd.device)
    prof = torch.empty((B, spec.base.l + 1), dtype=torch.int64, device=fwd.device) if profile else None
    call("gkm_self_kernel", spec.ref, ptr(fwd), ptr(rc), ptr(counts), B, W, ptr(diag), ptr(prof), _st())
    return (diag, prof) if profile else diag


def join_pairwise(spec: Spec, bx, cx, by, ry, cy, raw: bool = True, profile: bool = False):
    B, Wx = bx.shape
    S, Wy = by.shape
    out = torch.empty((B, S), dtype=torch.float64, device=bx.device) if raw else None
    prof = torch.empty((B, S, spec.base.l + 1), dtype=torch.int64, device=bx.device) if profile else None
    call("gkm_join_pairwise", spec.ref, ptr(bx), ptr(cx), B, Wx, ptr(by), ptr(ry), ptr(cy), S, Wy,
         ptr(out), ptr(prof), _st())
    return out, prof


def dense_applies(spec: Spec) -> bool:
    """The tensor-core form needs 0 <= dmax < l <= 15."""
    b = spec.base
    return 0 <= b.dmax < b.l <= 15


def dense_pairwise(spec: Spec, bx, cx, by, ry, cy, raw: bool = True, profile: bool = False,
                   check: bool = True):
    """join_pairwise's results from the tensor-core kernel.  check: read the
    kernel's error flag back (synchronises) and raise if an MMA timed out."""
    B, Wx = bx.shape
    S, Wy = by.shape
    out = torch.empty((B, S), dtype=torch.float64, device=bx.device) if raw else None
    prof = torch.empty((B, S, spec.base.l + 1), dtype=torch.int64, device=bx.device) if profile else None
    err = torch.zeros(1, dtype=torch.int32, device=bx.device)
    call("gkm_dense_pairwise", spec.ref, ptr(bx), ptr(cx), B, Wx, ptr(by), ptr(ry), ptr(cy), S, Wy,
         ptr(out), ptr(prof), ptr(err), _st())
    if check and int(err.item()) != 0:
        raise _lib.GkmError(_lib.GKM_ERR_CUDA,
                            "tensor-core pairwise: a hand-off between the kernel's roles did not complete within "
                            "its wait limit")
    return out, prof


# Pairwise method: "join" (warp ballot/popc over window pairs), "dense"
# (tensor-core one-hot product), or "auto": per shape class, the faster of the
# forms that apply, measured on the first call of the class (the autotuner
# below).  The two forms give identical results, so the choice changes only
# the time.
PAIRWISE_METHOD = "auto"

# shape class -> "join" | "dense"; filled by the autotuner, read by bench/tests
PAIRWISE_TUNED: dict = {}
# rows and columns of the sample the autotuner times
_TUNE_ROWS = 64
_TUNE_COLS = 4096


def hit_rate(l: int, dmax: int) -> float:
    """Probability that two uniform random l-mers differ at <= dmax positions
    (the share of window pairs the dense epilogue counts)."""
    from math import comb
    return sum(comb(l, m) * 0.75 ** m * 0.25 ** (l - m) for m in range(dmax + 1))


def pairwise_forms(spec: Spec) -> list:
    """The pairwise forms that apply to the kernel: the join always, the
    tensor-core product for 0 <= dmax < l <= 15."""
    return ["join", "dense"] if dense_applies(spec) else ["join"]


def _pow2(n: int) -> int:
    return 1 << max(0, (int(n) - 1).bit_length())


def pairwise_class(spec: Spec, B: int, Wx: int, S: int, Wy: int) -> tuple:
    """The autotuner's shape class: the kernel's l, dmax, weighting and RC,
    and the row/column counts and window widths rounded up to powers of two
    (rows and columns capped where the per-pair cost has settled)."""
    b = spec.base
    return (b.l, b.dmax, bool(b.weighted), bool(b.include_rc), min(_pow2(B), 4096), _pow2(Wx),
            min(_pow2(S), 65536), _pow2(Wy))


def _time_form(form: str, spec: Spec, bx, cx, by, ry, cy) -> float:
    fn = dense_pairwise if form == "dense" else join_pairwise
    kw = {"check": False} if form == "dense" else {}
    fn(spec, bx, cx, by, ry, cy)  # warm-up (and, for the dense form, its error check)
    st = torch.cuda.current_stream()
    best = float("inf")
    for _ in range(2):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        fn(spec, bx, cx, by, ry, cy, **kw)
        b.record(st)
        b.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def choose_pairwise(spec: Spec, bx, cx, by, ry, cy) -> str:
    """The pairwise form for this call under "auto": the only one that
    applies, or the one that ran a sample of the call (up to 64 rows x 4,096
    columns) faster the first time its shape class was seen."""
    forms = pairwise_forms(spec)
    if len(forms) == 1:
        return forms[0]
    B, Wx = bx.shape
    S, Wy = by.shape
    key = pairwise_class(spec, B, Wx, S, Wy)
    got = PAIRWISE_TUNED.get(key)
    if got is None:
        nb, ns = min(B, _TUNE_ROWS), min(S, _TUNE_COLS)
        sample = (bx[:nb].contiguous(), cx[:nb].contiguous(), by[:ns].contiguous(),
                  None if ry is None else ry[:ns].contiguous(), cy[:ns].contiguous())
        times = {f: _time_form(f, spec, *sample) for f in forms}
        got = min(forms, key=lambda f: times[f])
        PAIRWISE_TUNED[key] = got
    return got


def pairwise(spec: Spec, bx, cx, by, ry, cy, raw: bool = True, profile: bool = False, method: str | None = None):
    """Pairwise K_raw / profiles through the join or the tensor-core kernel."""
    method = method or PAIRWISE_METHOD
    if method == "auto":
        method = choose_pairwise(spec, bx, cx, by, ry, cy)
    if method == "dense":
        return dense_pairwise(spec, bx, cx, by, ry, cy, raw, profile)
    if method != "join":
        raise ValueError(f"pairwise method must be 'auto', 'join' or 'dense', got {method!r}")
    return join_pairwise(spec, bx, cx, by, ry, cy, raw, profile)


def masks_tensor(base, device) -> torch.Tensor:
    m = base.masks()
    return torch.from_numpy(m.view(np.int32).copy()).to(device)


class DeviceIndex:
    """An l-mer index handle over packed columns (owned; freed on close)."""

    def __init__(self, spec: Spec, fwd, rc, counts, masks: torch.Tensor, tile_svs: int = 0):
        self.spec = spec
        self.S = fwd.shape[0]
        self.masks = masks
        h = ctypes.c_void_p()
        call("gkm_index_create", spec.ref, ptr(fwd), ptr(rc), ptr(counts), fwd.shape[0], fwd.shape[1],
             ptr(masks), int(masks.numel()), int(tile_svs), ctypes.byref(h), _st())
        self.handle = h
        e, t, ts, nb = ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
        call("gkm_index_info", h, ctypes.byref(e), ctypes.byref(t), ctypes.byref(ts), ctypes.byref(nb))
        self.entries, self.tiles, self.tile_svs, self.nbytes = e.value, t.value, ts.value, nb.value

    def close(self):
        if getattr(self, "handle", None) and self.handle.value:
            _lib.load().gkm_index_free(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def counters(self) -> torch.Tensor:
        """A pinned host snapshot of the index's event counts, copied in
        stream order (read it after the stream reaches this point)."""
        buf = torch.empty(2, dtype=torch.int32, pin_memory=True)
        call("gkm_index_status", self.handle, ptr(buf), -1, _st())
        return buf

    def set_wide(self, wide: int) -> None:
        """Counter width of later queries: unweighted 16-bit with the carry
        log (0) or 32-bit (1); weighted 32-bit (0, 1) or 64-bit (2)."""
        call("gkm_index_status", self.handle, None, int(wide), _st())

    def settle(self, before: torch.Tensor, rerun=None):
        """After a call bracketed by counters() snapshots: waits for the
        stream; if a query block's 16-bit carries outgrew its log anywhere in
        that window (this call's or a concurrent one's), reruns rerun() with
        32-bit counters, and if a weighted 32-bit count wrapped, with 64-bit
        counters (exact either way).  A wrapped unweighted 32-bit count (past
        2^32 matching window pairs of one row and one SV) raises.  Returns
        True when it reran."""
        after = self.counters()
        torch.cuda.current_stream().synchronize()
        reran = False
        wide = 0
        if rerun is not None:
            if self.spec.c.weighted and int(after[1]) != int(before[1]):
                wide = 2
            elif int(after[0]) != int(before[0]):
                wide = 1
        if wide:
            reran = True
            self.set_wide(wide)
            try:
                b2 = self.counters()
                rerun()
                after = self.counters()
                torch.cuda.current_stream().synchronize()
                before = b2
            finally:
                self.set_wide(0)
        if int(after[1]) != int(before[1]):
            raise _lib.GkmError(_lib.GKM_ERR_CAPACITY, "a weighted pair count passed 2^32 for one (row, SV) pair")
        return reran

    def checked(self, run):
        """run() through the index, exact: see settle()."""
        before = self.counters()
        out = run()
        self.settle(before, run)
        return out

    def pairwise(self, bx, cx, diag_offset=None, raw=True, profile=False, out=None, check=True):
        """(K_raw [B, S] or None, profiles [B, S, l+1] or None); check=False
        skips the exactness check (no synchronisation: the caller settles)."""
        B, W = bx.shape
        if raw and out is None:
            out = torch.zeros((B, self.S), dtype=torch.float64, device=bx.device)
        prof = (torch.zeros((B, self.S, self.spec.base.l + 1), dtype=torch.int64, device=bx.device)
                if profile else None)

        def run():
            call("gkm_index_pairwise", self.handle, ptr(bx), ptr(cx), B, W,
                 -1 if diag_offset is None else int(diag_offset), ptr(out if raw else None), ptr(prof), _st())
            return out, prof

        return self.checked(run) if check else run()

    def score(self, bx, cx, inv_dx, inv_ds, coef, gamma, rbf, bias, order=None, out=None, check=True):
        B, W = bx.shape
        if out is None:
            out = torch.empty(B, dtype=torch.float64, device=bx.device)

        def run():
            call("gkm_index_score", self.handle, ptr(bx), ptr(cx), B, W, ptr(inv_dx), ptr(inv_ds), ptr(coef),
                 float(gamma), int(rbf), float(bias), ptr(order), ptr(out), _st())
            return out

        return self.checked(run) if check else run()

    def count(self, bx, cx):
        """(lookups, hits) an index query over rows bx makes."""
        out = torch.zeros(2, dtype=torch.int64, device=bx.device)
        call("gkm_index_count", self.handle, ptr(bx), ptr(cx), bx.shape[0], bx.shape[1], ptr(out), _st())
        return [int(v) for v in out.cpu()]

    def lmer_weights(self, c_sv):
        n = 4**self.spec.base.l
        V = torch.empty(n, dtype=torch.float64, device=c_sv.device)
        call("gkm_index_lmer_weights", self.handle, ptr(c_sv), ptr(V), _st())
        return V


def lmer_table(spec: Spec, V, masks):
    table = torch.empty_like(V)
    call("gkm_lmer_table", spec.ref, ptr(V), ptr(masks), int(masks.numel()), ptr(table), _st())
    return table


def table_score(spec: Spec, table, fwd, rc, counts, bias, normalize, want_parts=False):
    B, W = fwd.shape
    dev = fwd.device
    scores = torch.empty(B, dtype=torch.float64, device=dev)
    raw = torch.empty(B, dtype=torch.float64, device=dev) if want_parts else None
    diag = torch.empty(B, dtype=torch.float64, device=dev) if want_parts else None
    call("gkm_table_score", spec.ref, ptr(table), ptr(fwd), ptr(rc), ptr(counts), B, W, float(bias),
         int(bool(normalize)), ptr(scores), ptr(raw), ptr(diag), _st())
    return (scores, raw, diag) if want_parts else scores


def raw_score(raw, dx, ds, coef, gamma, rbf, bias):
    B, S = raw.shape
    out = torch.empty(B, dtype=torch.float64, device=raw.device)
    call("gkm_raw_score", ptr(raw), B, S, ptr(dx), ptr(ds), ptr(coef), float(gamma), int(rbf), float(bias),
         ptr(out), _st())
    return out


def impact(raw, n, dr, ds, coef, gamma, rbf):
    S = raw.shape[1]
    out = torch.empty(n, dtype=torch.float64, device=raw.device)
    call("gkm_impact", ptr(raw), n, S, ptr(dr), ptr(ds), ptr(coef), float(gamma), int(rbf), ptr(out), _st())
    return out


def mutant_diag(spec: Spec, fwd, counts, L, diag):
    B, W = fwd.shape
    out = torch.empty((4, L, B), dtype=torch.float64, device=fwd.device)
    call("gkm_mutant_diag", spec.ref, ptr(fwd), ptr(counts), B, W, L, ptr(diag), ptr(out), _st())
    return out


def ism_table(spec: Spec, table, fwd, counts, L, ref_raw, diag, normalize, want_mut=False):
    B, W = fwd.shape
    out = torch.empty((B, 4, L), dtype=torch.float64, device=fwd.device)
    mut = torch.empty((4, L, B), dtype=torch.float64, device=fwd.device) if want_mut else None
    call("gkm_ism_table", spec.ref, ptr(table), ptr(fwd), ptr(counts), B, W, L, ptr(ref_raw),
         ptr(diag if normalize else None), ptr(mut), int(bool(normalize)), ptr(out), _st())
    return (out, mut) if want_mut else out


def gram_finish(raw, dx, dy, gamma, rbf, symmetric):
    N, M = raw.shape
    out = torch.empty_like(raw)
    call("gkm_gram_finish", ptr(raw), N, M, ptr(dx), ptr(dy), float(gamma), int(rbf), int(symmetric),
         ptr(out), _st())
    return out
