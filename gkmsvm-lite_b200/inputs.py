"""Sequence batches: every entry point (scoring, variants, ISM, GkmExplain,
Gram, training, serving) turns its input into one ``SeqBatch`` in a single
pass and asks the batch for what it needs afterwards -- row slices, the rows
shorter than l, device codes, and the masking of its outputs.

Interface semantics kept from gkmsvm-lite (inputs.py:27-145, codec.py:96-137):
bases are codes A=0 C=1 G=2 T=3; N (and, when allowed, any other letter) is
stored as A, which the kernels read as A forward and T on the reverse strand;
``lengths`` is None when every row is as long as the array; rows shorter than
l give NaN and positions past a row's length give 0; sequences longer than
LS-GKM's 2,047-base read limit draw a warning.
"""

from __future__ import annotations

import warnings
from dataclasses import dataclass

import numpy as np
import torch

# LS-GKM (libsvm_gkm.h MAX_SEQ_LENGTH 2048) reads at most this many bases
LSGKM_MAX_LENGTH = 2047

# byte -> code: ACGT/acgt 0..3, N/n 4 (stored as A), anything else 5
_BYTE_CODE = np.full(256, 5, dtype=np.uint8)
for _code, _letters in enumerate(("Aa", "Cc", "Gg", "Tt", "Nn")):
    for _ch in _letters:
        _BYTE_CODE[ord(_ch)] = _code


def _letters_to_codes(raw: np.ndarray, allow_n: bool, allow_other: bool) -> np.ndarray:
    """uint8 bytes -> codes, with N / other letters stored as A."""
    c = _BYTE_CODE[raw]
    worst = int(c.max()) if c.size else 0
    if worst == 4 and not (allow_n or allow_other):
        raise ValueError("sequence holds N; pass allow_n=True to read it (scored as A)")
    if worst == 5 and not allow_other:
        raise ValueError("sequence holds letters other than ACGTN; pass allow_other=True to read them as N")
    c[c > 3] = 0
    return c


def encode_codes(sequence: str, *, allow_n: bool = False, allow_other: bool = False) -> np.ndarray:
    """[L] uint8 codes of one DNA string (N stored as A when allowed)."""
    if not sequence:
        raise ValueError("Sequence must be non-empty")
    return _letters_to_codes(np.frombuffer(sequence.encode("ascii"), dtype=np.uint8), allow_n, allow_other)


def to_codes(x):
    """[B, L] uint8 codes of a [B, 4, L] one-hot batch (an all-zero column, N,
    reads as A) or of [B, L] integer codes; NumPy or torch, on x's device."""
    if isinstance(x, torch.Tensor):
        if x.ndim == 2:
            if x.dtype.is_floating_point or x.dtype.is_complex:
                raise ValueError(f"[B, L] base codes must be integers, got {x.dtype}")
            return x if x.dtype == torch.uint8 else x.to(torch.uint8)
        if x.ndim != 3 or x.shape[1] != 4:
            raise ValueError(f"expected a [B, 4, L] one-hot array or [B, L] base codes, got {list(x.shape)}")
        return x.argmax(dim=1).to(torch.uint8)
    a = np.asarray(x)
    if a.ndim == 2:
        if a.dtype.kind not in "iub":
            raise ValueError(f"[B, L] base codes must be integers, got {a.dtype}")
        return a if a.dtype == np.uint8 else a.astype(np.uint8)
    if a.ndim != 3 or a.shape[1] != 4:
        raise ValueError(f"expected a [B, 4, L] one-hot array or [B, L] base codes, got {list(a.shape)}")
    return a.argmax(axis=1).astype(np.uint8)


def _to_host(a):
    return a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)


@dataclass
class SeqBatch:
    """[B, L] uint8 codes (NumPy or torch, any device) and the rows' lengths
    as host int64, or None when every row is L long."""

    codes: np.ndarray | torch.Tensor
    lengths: np.ndarray | None = None

    # -- construction ---------------------------------------------------------

    @classmethod
    def read(cls, x, lengths=None) -> "SeqBatch":
        """A batch from a [B, 4, L] one-hot or [B, L] codes array / tensor (with
        the rows' lengths when they differ), or from a list of DNA strings,
        [4, L_i] one-hot or [L_i] code arrays."""
        if isinstance(x, (list, tuple)):
            if lengths is not None:
                raise ValueError("lengths go with a padded array, not a list")
            if not x:
                raise ValueError("no sequences")
            b = cls._from_strings(x) if isinstance(x[0], str) else cls._from_arrays(x)
        else:
            codes = to_codes(x)
            b = cls(codes, cls.checked_lengths(lengths, codes.shape))
        longest = b.longest
        if longest > LSGKM_MAX_LENGTH:
            warnings.warn(f"the longest sequence has {longest} bases; LS-GKM itself reads only the first "
                          f"{LSGKM_MAX_LENGTH}", stacklevel=3)
        return b

    @classmethod
    def _from_strings(cls, seqs) -> "SeqBatch":
        # every string in one buffer: one table lookup, one masked scatter
        lens = np.fromiter((len(s) for s in seqs), dtype=np.int64, count=len(seqs))
        if (lens == 0).any():
            raise ValueError("Sequence must be non-empty")
        flat = _letters_to_codes(np.frombuffer("".join(seqs).encode("ascii"), dtype=np.uint8), True, False)
        out = np.zeros((len(seqs), int(lens.max())), dtype=np.uint8)
        out[np.arange(out.shape[1])[None, :] < lens[:, None]] = flat
        return cls(out, lens)

    @classmethod
    def _from_arrays(cls, arrs) -> "SeqBatch":
        rows = [np.asarray(to_codes(_to_host(a)[None]))[0] for a in arrs]
        lens = np.array([r.shape[-1] for r in rows], dtype=np.int64)
        out = np.zeros((len(rows), int(lens.max())), dtype=np.uint8)
        out[np.arange(out.shape[1])[None, :] < lens[:, None]] = np.concatenate(rows)
        return cls(out, lens)

    @staticmethod
    def checked_lengths(lengths, shape):
        if lengths is None:
            return None
        n = np.asarray(_to_host(lengths), dtype=np.int64).reshape(-1)
        B, L = shape[0], shape[-1]
        if n.shape[0] != B or (n < 0).any() or (n > L).any():
            raise ValueError(f"lengths must be {B} values in 0..{L}")
        return None if (n == L).all() else n

    # -- shape ----------------------------------------------------------------

    @property
    def B(self) -> int:
        return int(self.codes.shape[0])

    @property
    def L(self) -> int:
        return int(self.codes.shape[-1])

    @property
    def longest(self) -> int:
        return self.L if self.lengths is None else int(self.lengths.max(initial=0))

    def row_lengths(self) -> np.ndarray:
        return np.full(self.B, self.L, dtype=np.int64) if self.lengths is None else self.lengths

    def n_windows(self, l: int) -> int:
        """l-mer windows over all rows."""
        return int(np.clip(self.row_lengths() - l + 1, 0, None).sum())

    # -- rows -----------------------------------------------------------------

    def part(self, start: int, n: int) -> "SeqBatch":
        return SeqBatch(self.codes[start:start + n], None if self.lengths is None else self.lengths[start:start + n])

    def widened(self, L: int) -> "SeqBatch":
        """The same rows zero-padded to L columns (lengths keep the real ones)."""
        if self.L == L:
            return self
        pad = L - self.L
        codes = (torch.nn.functional.pad(self.codes, (0, pad)) if isinstance(self.codes, torch.Tensor)
                 else np.pad(self.codes, ((0, 0), (0, pad))))
        return SeqBatch(codes, self.row_lengths())

    @staticmethod
    def stacked(*parts: "SeqBatch") -> "SeqBatch":
        """Rows of batches of one width, in order."""
        if any(isinstance(p.codes, torch.Tensor) for p in parts):
            codes = torch.cat([torch.as_tensor(p.codes) for p in parts])
        else:
            codes = np.concatenate([p.codes for p in parts])
        if all(p.lengths is None for p in parts):
            return SeqBatch(codes, None)
        return SeqBatch(codes, np.concatenate([p.row_lengths() for p in parts]))

    def short(self, l: int, what: str = "scores") -> np.ndarray | None:
        """[B] bool rows with no l-mer window (warns), or None if there are none."""
        if self.lengths is None:
            return None
        s = self.lengths < l
        if not s.any():
            return None
        warnings.warn(f"{int(s.sum())} of {self.B} sequences have fewer than l = {l} bases; "
                      f"their {what} are NaN", stacklevel=3)
        return s

    def on(self, device) -> torch.Tensor:
        """Codes as a contiguous uint8 tensor on device (pinned, asynchronous
        copy for host codes)."""
        return device_codes(self.codes, device)


def as_batch(x, lengths=None):
    """(codes [B, L_max], lengths or None): SeqBatch.read as a pair."""
    b = SeqBatch.read(x, lengths)
    return b.codes, b.lengths


def allele_batches(ref, alt, ref_lengths=None, alt_lengths=None) -> tuple[SeqBatch, SeqBatch]:
    """Reference and alternative alleles as batches of one common width (the
    shorter side zero-padded, its lengths kept), for indels of any size."""
    r = SeqBatch.read(ref, ref_lengths)
    a = SeqBatch.read(alt, alt_lengths)
    if r.B != a.B:
        raise ValueError(f"ref and alt hold {r.B} and {a.B} sequences")
    L = max(r.L, a.L)
    return r.widened(L), a.widened(L)


def nan_rows(out: torch.Tensor, short) -> torch.Tensor:
    """out with the rows flagged in short set to NaN."""
    if short is None:
        return out
    flag = torch.as_tensor(short, device=out.device).reshape(-1, *([1] * (out.ndim - 1)))
    return out.masked_fill(flag, float("nan"))


def per_position(out: torch.Tensor, batch: SeqBatch, short) -> torch.Tensor:
    """[B, 4, L] per-position outputs: 0 past each row's length, NaN rows in short."""
    if batch.lengths is None:
        return out
    past = (torch.arange(out.shape[2], device=out.device)[None, :]
            >= torch.as_tensor(batch.lengths, device=out.device)[:, None])
    return nan_rows(out.masked_fill(past[:, None, :], 0.0), short)


def device_codes(x, device) -> torch.Tensor:
    """Codes as a contiguous uint8 tensor on device (pinned + async for host input)."""
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=torch.uint8, non_blocking=True).contiguous()
    t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.uint8))
    if device.type == "cuda":
        t = t.pin_memory()
    return t.to(device, non_blocking=True)
