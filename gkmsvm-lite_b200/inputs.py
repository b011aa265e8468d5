"""Input handling: batches of base codes with per-row lengths, allele pairs,
and the NaN / zero masking of short rows and positions past a row's length
(the semantics of gkmsvm-lite's inputs.py:27-145 and codec.py:96-137)."""

from __future__ import annotations

import warnings

import numpy as np
import torch

LSGKM_MAX_LENGTH = 2047

_CODES = np.full(256, 5, dtype=np.uint8)
for _i, _b in enumerate("ACGT"):
    _CODES[ord(_b)] = _i
    _CODES[ord(_b.lower())] = _i
_CODES[ord("N")] = 4
_CODES[ord("n")] = 4


def encode_codes(sequence: str, *, allow_n: bool = True, allow_other: bool = False) -> np.ndarray:
    """[L] uint8 codes A=0 C=1 G=2 T=3 of a DNA string; N (and, with
    allow_other, any other letter) is stored as A, as the kernels read it."""
    if len(sequence) == 0:
        raise ValueError("Sequence must be non-empty")
    c = _CODES[np.frombuffer(sequence.encode("ascii"), dtype=np.uint8)]
    if (c == 4).any() and not allow_n:
        raise ValueError("Invalid base in sequence (pass allow_n=True for N)")
    if (c == 5).any() and not allow_other:
        raise ValueError("Invalid base in sequence (pass allow_other=True to read non-ACGTN letters as N)")
    return np.where(c > 3, 0, c).astype(np.uint8)


def to_codes(x):
    """[B, L] uint8 codes from [B, 4, L] one-hot (argmax: N, all zero, is A) or
    [B, L] integer codes; NumPy or torch, kept on its device."""
    if isinstance(x, torch.Tensor):
        if x.ndim == 2:
            if x.dtype.is_floating_point:
                raise ValueError(f"[B, L] base codes must be integers, got {x.dtype}")
            return x.to(torch.uint8)
        if x.ndim != 3 or x.shape[1] != 4:
            raise ValueError(f"expected a [B, 4, L] one-hot array or [B, L] base codes, got {list(x.shape)}")
        return torch.argmax(x, dim=1).to(torch.uint8)
    x = np.asarray(x)
    if x.ndim == 2:
        if x.dtype == np.uint8:
            return x
        if not (np.issubdtype(x.dtype, np.integer) or x.dtype == bool):
            raise ValueError(f"[B, L] base codes must be integers, got {x.dtype}")
        return x.astype(np.uint8)
    if x.ndim != 3 or x.shape[1] != 4:
        raise ValueError(f"expected a [B, 4, L] one-hot array or [B, L] base codes, got {list(x.shape)}")
    return np.argmax(x, axis=1).astype(np.uint8)


def _host(a):
    if a is None:
        return None
    if isinstance(a, torch.Tensor):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def uniform_or_lengths(lengths, shape):
    """lengths as host int64 [B], or None when every row is shape[-1] long."""
    if lengths is None:
        return None
    lengths = np.asarray(_host(lengths), dtype=np.int64).reshape(-1)
    B, L = shape[0], shape[-1]
    if lengths.shape[0] != B or (lengths < 0).any() or (lengths > L).any():
        raise ValueError(f"lengths must be {B} values in 0..{L}")
    return None if (lengths == L).all() else lengths


def as_batch(x, lengths=None):
    """(codes [B, L_max], lengths or None) from a one-hot/codes array or tensor
    or a list of strings / one-hot arrays / code arrays (inputs.py:27-61)."""
    if isinstance(x, (list, tuple)):
        if lengths is not None:
            raise ValueError("lengths go with a padded array, not a list")
        if not len(x):
            raise ValueError("no sequences")
        if isinstance(x[0], str):
            rows = [encode_codes(s, allow_n=True) for s in x]
        else:
            rows = [np.asarray(to_codes(_host(a)[None]))[0] for a in x]
        lens = np.array([r.shape[-1] for r in rows], dtype=np.int64)
        out = np.zeros((len(rows), int(lens.max())), dtype=np.uint8)
        for i, r in enumerate(rows):
            out[i, : r.shape[-1]] = r
        x, lengths = out, lens
    else:
        x = to_codes(x)
    lengths = uniform_or_lengths(lengths, x.shape)
    longest = int(x.shape[-1] if lengths is None else lengths.max())
    if longest > LSGKM_MAX_LENGTH:
        warnings.warn(f"sequences up to {longest} bp: LS-GKM reads only the first "
                      f"{LSGKM_MAX_LENGTH} bases of longer ones", stacklevel=3)
    return x, lengths


def allele_arrays(ref, alt, ref_lengths=None, alt_lengths=None):
    """(ref, alt, ref_lengths, alt_lengths) as code batches of one length L
    (inputs.py:64-85)."""
    ref, ref_lengths = as_batch(ref, ref_lengths)
    alt, alt_lengths = as_batch(alt, alt_lengths)
    if ref.shape[0] != alt.shape[0]:
        raise ValueError(f"ref and alt hold {ref.shape[0]} and {alt.shape[0]} sequences")
    L = max(ref.shape[-1], alt.shape[-1])

    def widen(a, n):
        if a.shape[-1] == L:
            return a, n
        n = np.full(a.shape[0], a.shape[-1], dtype=np.int64) if n is None else n
        if isinstance(a, torch.Tensor):
            return torch.nn.functional.pad(a, (0, L - a.shape[-1])), n
        return np.pad(a, ((0, 0), (0, L - a.shape[-1]))), n

    ref, ref_lengths = widen(ref, ref_lengths)
    alt, alt_lengths = widen(alt, alt_lengths)
    return ref, alt, ref_lengths, alt_lengths


def joint_lengths(L, *parts):
    if all(n is None for _, n in parts):
        return None
    return np.concatenate([np.full(rows, L, dtype=np.int64) if n is None else n for rows, n in parts])


def rows(lengths, start, n):
    return None if lengths is None else lengths[start : start + n]


def short_rows(lengths, l, what="scores"):
    if lengths is None:
        return None
    short = lengths < l
    if not short.any():
        return None
    warnings.warn(f"{int(short.sum())} sequences are shorter than l = {l}: their {what} are NaN",
                  stacklevel=3)
    return short


def nan_rows(out: torch.Tensor, short) -> torch.Tensor:
    if short is None:
        return out
    mask = torch.as_tensor(short, device=out.device).reshape(-1, *[1] * (out.ndim - 1))
    return torch.where(mask, torch.full_like(out, float("nan")), out)


def per_position(out: torch.Tensor, lengths, short) -> torch.Tensor:
    """[B, 4, L] with positions past each row's length 0 and short rows NaN."""
    if lengths is None:
        return out
    inside = torch.arange(out.shape[2], device=out.device)[None, None, :] < torch.as_tensor(
        lengths, device=out.device)[:, None, None]
    return nan_rows(torch.where(inside, out, torch.zeros_like(out)), short)


def device_codes(x, device) -> torch.Tensor:
    """Codes as a contiguous uint8 tensor on device (pinned + async for host input)."""
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=torch.uint8, non_blocking=True).contiguous()
    t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.uint8))
    if device.type == "cuda":
        t = t.pin_memory()
    return t.to(device, non_blocking=True)
