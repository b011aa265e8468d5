"""Model files (serialization.py of gkmsvm-lite): the native npz format, LS-GKM
text for interop, and DeltaSVM weight files, with the reference's layouts so
that files move between the two packages unchanged.

npz: support_sequences [S, L] uint8 codes, coefficients [S], sv_lengths [S]
(ragged SVs only) and metadata, a JSON object (bias, kernel_type,
kernel_params, sv_chunk_size) stored as bytes (serialization.py:15-32).
"""

from __future__ import annotations

import gzip
import json
from pathlib import Path

import numpy as np

_BASES = np.frombuffer(b"ACGT", dtype=np.uint8)


def _host(a):
    return a.cpu().numpy() if hasattr(a, "cpu") else np.asarray(a)


def save_npz(model, path) -> None:
    """serialization.py:15-32."""
    metadata = {"bias": float(model.bias), "kernel_type": model.kernel_type,
                "kernel_params": model._kernel_params}
    if model.sv_chunk_size is not None:
        metadata["sv_chunk_size"] = model.sv_chunk_size
    extra = {} if model.sv_lengths is None else {"sv_lengths": np.asarray(model.sv_lengths)}
    np.savez(path, support_sequences=_host(model.support_sequences), coefficients=_host(model.coefficients),
             metadata=np.void(json.dumps(metadata).encode("utf-8")), **extra)


def save_deltasvm_npz(model, path) -> None:
    """DeltaSVM weights (a DeltaSVMWeights or anything with weights, l, k,
    include_rc, bias) in the reference's DeltaSVM npz (serialization.py:35-49)."""
    metadata = {"model_type": "deltasvm", "l": int(model.l), "k": int(model.k),
                "include_rc": bool(model.include_rc), "bias": float(model.bias)}
    np.savez(path, weights=_host(model.weights), metadata=np.void(json.dumps(metadata).encode("utf-8")))


def _read_npz(path):
    data = np.load(path, allow_pickle=False)
    return data, json.loads(bytes(data["metadata"]))


def load_deltasvm_npz(path, *, device: str = "cpu"):
    """DeltaSVMWeights of a DeltaSVM npz (serialization.py:58-72); weights on
    the host, or on the GPU for device "cuda"."""
    from .deltasvm import DeltaSVMWeights

    data, metadata = _read_npz(path)
    w = np.asarray(data["weights"], dtype=np.float64)
    if str(device).startswith("cuda"):
        import torch

        w = torch.from_numpy(w).to(device)
    return DeltaSVMWeights(w, int(metadata["l"]), int(metadata["k"]), bool(metadata["include_rc"]),
                           float(metadata.get("bias", 0.0)))


def load_npz(path, *, device: str = "cpu"):
    """GkmSVM of a native npz (serialization.py:75-91)."""
    from .model import GkmSVM

    data, metadata = _read_npz(path)
    return GkmSVM(data["support_sequences"], data["coefficients"], metadata["bias"], metadata["kernel_type"],
                  metadata["kernel_params"],
                  sv_lengths=data["sv_lengths"] if "sv_lengths" in data.files else None,
                  sv_chunk_size=metadata.get("sv_chunk_size"), device=device)


def save_lsgkm(model, path) -> None:
    """LS-GKM text, gzip for a .gz name (serialization.py:94-140): rho = -bias,
    norc written only when RC is off, each SV without its padding."""
    path = Path(path)
    params = model._kernel_params
    coefs = _host(model.coefficients)
    svs = _host(model.support_sequences)
    lines = ["svm_type c_svc", f"kernel_type {model.kernel_type}", f"L {params['L']}", f"k {params['k']}"]
    for key in ("d", "gamma", "M", "H"):
        if key in params:
            lines.append(f"{key} {params[key]}")
    if not params.get("include_rc", True):
        lines.append("norc 1")
    lines += ["nr_class 2", f"total_sv {len(coefs)}", f"rho {-model.bias}", "label 1 -1",
              f"nr_sv {int((coefs > 0).sum())} {int((coefs <= 0).sum())}", "SV"]
    lengths = model.sv_lengths
    for i in range(len(coefs)):
        row = svs[i] if lengths is None else svs[i][: lengths[i]]
        lines.append(f"{coefs[i]} {_BASES[row].tobytes().decode('ascii')}")
    text = "\n".join(lines) + "\n"
    if str(path).endswith(".gz"):
        with gzip.open(path, "wt") as f:
            f.write(text)
    else:
        path.write_text(text)


def load_model(path, *, device: str = "cpu"):
    """A GkmSVM (or DeltaSVM weights) from .npz, else LS-GKM text
    (serialization.py:143-166)."""
    path = Path(path)
    if path.name.lower().endswith(".npz"):
        data, metadata = _read_npz(path)
        data.close()
        if metadata.get("model_type") == "deltasvm":
            return load_deltasvm_npz(path, device=device)
        return load_npz(path, device=device)
    from .importers import load_lsgkm_model

    return load_lsgkm_model(str(path), device=device)
