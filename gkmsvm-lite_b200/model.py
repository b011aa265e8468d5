"""GkmSVM: the gapped-k-mer SVM scoring model on a B200.

Mirrors gkmsvm-lite's GkmSVM (svm.py:155-662): the same constructor, switches
(use_lmer_index, use_lmer_table, use_explain_table, sv_chunk_size), __call__
and score_variants signatures and outputs.  The model holds its support
vectors on the host until .cuda(); from then on every call runs on the GPU
through libgkm_b200 and returns float64 torch CUDA tensors (where the
reference returns CuPy arrays).  There is no CPU path: calling a model that is
not on CUDA raises.
"""

from __future__ import annotations

import numpy as np
import torch

from . import engine
from ._lib import require_cuda
from .inputs import SeqBatch, allele_batches, device_codes, nan_rows, to_codes
from .kernels import KERNEL_BUILDERS, DirectGkmKernel, RbfKernel, neighbor_count, resolve_kernel_type

# Join-path [rows, S] float64 blocks stay within this (svm.py:475)
_MAX_SCORE_BYTES = 512 * 2**20
# Rows packed per device call, so packed windows stay within this
_MAX_PACK_BYTES = 2 * 2**30


class GkmSVM:
    """Gapped k-mer SVM: score = sum_i coef_i K(x, sv_i) + bias."""

    # "auto" builds the l-mer table when the index queries a call would make
    # cost more than building it: per (l-mer x neighbour) build cost, and per
    # (query window x neighbour) query cost a + b * (indexed windows per l-mer)
    _LMER_TABLE_BUILD_S = 2e-12
    _LMER_QUERY_S = (6e-12, 2e-12)

    def __init__(self, support_sequences, coefficients, bias, kernel_type, kernel_params, *,
                 sv_lengths=None, sv_chunk_size=None, device="cpu"):
        sv = support_sequences
        if isinstance(sv, torch.Tensor):
            sv = sv.detach().cpu().numpy()
        sv = np.asarray(sv)
        if sv.ndim == 3 and sv.shape[1] != 4:
            raise ValueError(f"support_sequences must be [S, 4, L] one-hot or [S, L] base codes, "
                             f"got {list(sv.shape)}")
        sv = np.ascontiguousarray(to_codes(sv))
        coef = coefficients.detach().cpu().numpy() if isinstance(coefficients, torch.Tensor) else np.asarray(coefficients)
        if coef.ndim != 1:
            raise ValueError(f"coefficients must be [S], got {list(coef.shape)}")
        if sv.shape[0] != coef.shape[0]:
            raise ValueError(f"Number of support sequences ({sv.shape[0]}) must match number of "
                             f"coefficients ({coef.shape[0]})")
        self.support_sequences = sv
        self.sv_lengths = SeqBatch.checked_lengths(sv_lengths, sv.shape)
        self.coefficients = coef.astype(np.float64)
        self.bias = float(bias)
        self.kernel_type = resolve_kernel_type(kernel_type)
        self._kernel_params = dict(kernel_params)
        self.kernel = KERNEL_BUILDERS[self.kernel_type](kernel_params)
        self.sv_chunk_size = sv_chunk_size
        self.use_lmer_index = True
        self.use_lmer_table: bool | str = "auto"
        self.use_explain_table: bool | str = "auto"
        self._device = torch.device("cpu")
        self._sv_cache: dict = {}
        self._lmer_table = None  # None: not built; False: none exists; tensor
        self._explain_tables: dict = {}
        if device != "cpu":
            self.to(device)

    # -- device placement ---------------------------------------------------

    @property
    def device(self) -> str:
        return self._device.type

    def to(self, device):
        device = torch.device("cuda" if device in ("auto",) else device)
        if device.type == "cuda":
            require_cuda()
            if device.index is None:
                device = torch.device("cuda", torch.cuda.current_device())
        elif device.type != "cpu":
            raise ValueError(f"device must be 'cpu' or 'cuda', got {device}")
        if device != self._device:
            self.clear_caches()
            self._device = device
        return self

    def cuda(self):
        return self.to("cuda")

    def cpu(self):
        return self.to("cpu")

    def _require_gpu(self):
        if self._device.type != "cuda":
            raise RuntimeError("this GkmSVM is on 'cpu': gkmsvm_lite_b200 computes on CUDA only; "
                               "call model.cuda() first")
        return self._device

    @property
    def num_support_vectors(self) -> int:
        return self.support_sequences.shape[0]

    @property
    def kernel_params(self) -> dict:
        return dict(self._kernel_params)

    def clear_caches(self) -> None:
        """Drop the device SV state (packed windows, self-kernels, index,
        l-mer table, explain tables); rebuilt on the next call."""
        idx = self._sv_cache.get("index")
        if idx is not None:
            idx.close()
        self._sv_cache = {}
        self._lmer_table = None
        self._explain_tables = {}

    # -- device SV state (svm.py:300-349) -------------------------------------

    def _spec(self) -> engine.Spec:
        c = self._sv_cache
        if "spec" not in c:
            c["spec"] = engine.Spec(self.kernel.base, self._require_gpu())
        return c["spec"]

    def _sv_packed(self):
        c = self._sv_cache
        if "packed" not in c:
            dev = self._require_gpu()
            codes = device_codes(self.support_sequences, dev)
            fwd, rc, counts = engine.pack(self._spec(), codes, self.sv_lengths)
            c["packed"] = (fwd, rc, counts)
            c["coef"] = torch.from_numpy(self.coefficients).to(dev)
            n = int(self.sv_lengths.max() if self.sv_lengths is not None else codes.shape[1])
            self._spec().check_rows(n)
        return c["packed"]

    def _sv_coef(self) -> torch.Tensor:
        self._sv_packed()
        return self._sv_cache["coef"]

    def _sv_diag(self) -> torch.Tensor:
        c = self._sv_cache
        if "diag" not in c:
            c["diag"] = engine.self_kernel(self._spec(), *self._sv_packed())
        return c["diag"]

    def _inv_ds(self) -> torch.Tensor:
        c = self._sv_cache
        if "inv_ds" not in c:
            if self.kernel.base.normalize:
                c["inv_ds"] = 1.0 / torch.sqrt(torch.clamp(self._sv_diag(), min=1e-20))
            else:
                c["inv_ds"] = torch.ones(self.num_support_vectors, dtype=torch.float64, device=self._device)
        return c["inv_ds"]

    def _masks(self) -> torch.Tensor:
        c = self._sv_cache
        if "masks" not in c:
            c["masks"] = engine.masks_tensor(self.kernel.base, self._require_gpu())
        return c["masks"]

    def _n_sv_windows(self) -> int:
        base = self.kernel.base
        L = self.support_sequences.shape[1]
        lens = self.sv_lengths if self.sv_lengths is not None else np.full(self.num_support_vectors, L)
        n = np.clip(lens - base.l + 1, 0, None).sum()
        return int(n * (2 if base.include_rc else 1))

    def _index_applies(self) -> bool:
        base = self.kernel.base
        n = self._n_sv_windows()
        return isinstance(base, DirectGkmKernel) and n > 0 and base.index_applies(n)

    def _sv_index(self):
        """The device l-mer index over the SVs, or None (use_lmer_index off or
        the neighbourhood too large); checked on every call."""
        if not self.use_lmer_index:
            return None
        c = self._sv_cache
        if "index" not in c:
            c["index"] = None
            if self._index_applies():
                fwd, rc, counts = self._sv_packed()
                c["index"] = engine.DeviceIndex(self._spec(), fwd, rc, counts, self._masks())
        return c["index"]

    # -- l-mer table (svm.py:485-557; lmer_table.py) --------------------------

    def _table_kernel_ok(self) -> bool:
        k = self.kernel
        return isinstance(k, DirectGkmKernel) and k.has_table()

    def _build_lmer_table(self):
        if self._lmer_table is None:
            if not self._table_kernel_ok():
                self._lmer_table = False
                return None
            base = self.kernel
            spec = self._spec()
            fwd, rc, counts = self._sv_packed()
            coef = self._sv_coef()
            if base.normalize:
                coef = coef / torch.sqrt(torch.clamp(self._sv_diag(), min=1e-10))
            index = self._sv_cache.get("index")
            tmp = None
            if index is None:
                tmp = engine.DeviceIndex(spec, fwd, rc, counts, self._masks())
                index = tmp
            V = index.lmer_weights(coef.contiguous())
            self._lmer_table = engine.lmer_table(spec, V, self._masks())
            if tmp is not None:
                tmp.close()
        return None if self._lmer_table is False else self._lmer_table

    def _plan_lmer_table(self, n_windows: int) -> None:
        k = self.kernel
        if (self.use_lmer_table != "auto" or self._lmer_table is not None
                or not self._table_kernel_ok()):
            return
        l = k.l
        nm = neighbor_count(l, k.dmax)
        per_lmer = self._n_sv_windows() / 4**l
        a, b = self._LMER_QUERY_S
        if n_windows * nm * (a + b * per_lmer) >= self._LMER_TABLE_BUILD_S * 4**l * nm:
            self._build_lmer_table()

    def _lmer_table_for(self):
        use = self.use_lmer_table
        if use is False or not self._table_kernel_ok():
            return None
        if use == "auto" and self._lmer_table is None:
            return None
        return self._build_lmer_table()

    # -- scoring ----------------------------------------------------------------

    def _score_packed(self, fwd, rc, counts) -> torch.Tensor:
        """[B] scores (bias included) of packed rows on the model's device."""
        kernel = self.kernel
        base = kernel.base
        spec = self._spec()
        spec.check_rows(int(fwd.shape[1]))
        table = self._lmer_table_for()
        if table is not None:
            return engine.table_score(spec, table, fwd, rc, counts, self.bias, base.normalize)
        rbf = isinstance(kernel, RbfKernel)
        gamma = kernel.gamma if rbf else 0.0
        dx = engine.self_kernel(spec, fwd, rc, counts) if base.normalize else None
        index = self._sv_index()
        if index is not None:
            if dx is None:
                inv_dx = torch.ones(fwd.shape[0], dtype=torch.float64, device=fwd.device)
            else:
                inv_dx = 1.0 / torch.sqrt(torch.clamp(dx, min=1e-20))
            order = torch.argsort(counts, descending=True).to(torch.int32)
            return index.score(fwd, counts, inv_dx, self._inv_ds(), self._sv_coef(), gamma, rbf,
                               self.bias, order)
        by, ry, cy = self._sv_packed()
        S = self.num_support_vectors
        step = max(1, _MAX_SCORE_BYTES // (8 * S))
        out = []
        ds = self._sv_diag() if base.normalize else None
        for s in range(0, fwd.shape[0], step):
            raw, _ = engine.pairwise(spec, fwd[s:s + step], counts[s:s + step], by, ry, cy)
            out.append(engine.raw_score(raw, None if dx is None else dx[s:s + step], ds, self._sv_coef(),
                                        gamma, rbf, self.bias))
        return torch.cat(out)

    def _score_codes(self, codes, lengths) -> torch.Tensor:
        dev = self._require_gpu()
        xt = device_codes(codes, dev)
        fwd, rc, counts = engine.pack(self._spec(), xt, lengths)
        return self._score_packed(fwd, rc, counts)

    def _score_unbatched(self, batch: SeqBatch) -> torch.Tensor:
        W = max(batch.L - self.kernel.l + 1, 1)
        step = max(1, _MAX_PACK_BYTES // (8 * W))
        parts = [self._score_codes(p.codes, p.lengths) for p in (batch.part(s, step) for s in range(0, batch.B, step))]
        return parts[0] if len(parts) == 1 else torch.cat(parts)

    def __call__(self, x, *, lengths=None, batch_size=None, verbose=False) -> torch.Tensor:
        """[B, 1] float64 decision values on the model's CUDA device; NaN for
        rows shorter than l (svm.py:407-451)."""
        dev = self._require_gpu()
        batch = x if isinstance(x, SeqBatch) else SeqBatch.read(x, lengths)
        l = self.kernel.l
        short = batch.short(l)
        B = batch.B
        if short is not None and short.all():
            return torch.full((B, 1), float("nan"), dtype=torch.float64, device=dev)
        self._plan_lmer_table(B * max(batch.L - l + 1, 0))
        if batch_size is not None and B > batch_size:
            it = range(0, B, batch_size)
            if verbose:
                from tqdm import tqdm
                it = tqdm(it, desc="Scoring")
            out = torch.cat([self._score_unbatched(batch.part(s, batch_size)) for s in it])
        else:
            out = self._score_unbatched(batch)
        return nan_rows(out[:, None], short)

    def score_variants(self, ref, alt, *, method="kernel", ref_lengths=None, alt_lengths=None,
                       batch_size=None, verbose=False) -> torch.Tensor:
        """[B, 1] variant effects (svm.py:600-662): score(alt) - score(ref), or
        GkmExplain mutation impact (lsgkm gkmexplain -m 5)."""
        if method == "kernel":
            r, a = allele_batches(ref, alt, ref_lengths, alt_lengths)
            scores = self(SeqBatch.stacked(a, r), batch_size=batch_size, verbose=verbose)
            return scores[:r.B] - scores[r.B:]
        if method == "gkmexplain":
            from .explain import mutation_impact

            return mutation_impact(self, ref, alt, ref_lengths=ref_lengths, alt_lengths=alt_lengths,
                                   batch_size=batch_size, verbose=verbose)
        raise ValueError(f"method must be 'kernel' or 'gkmexplain', got {method!r}")

    def to_deltasvm(self, *, device: str = "cpu", query_norm: bool = False, verbose: bool = False):
        """DeltaSVM weights, one per l-mer (svm.py:706-750); see
        deltasvm.to_deltasvm."""
        from .deltasvm import to_deltasvm

        return to_deltasvm(self, device=device, query_norm=query_norm, verbose=verbose)

    def save(self, path: str, *, fmt: str | None = None) -> None:
        """Save to disk (svm.py:273-298): "npz" (native) or "lsgkm" (text,
        gzip for .gz), from the extension unless fmt is given."""
        from .serialization import save_lsgkm, save_npz

        if fmt is None:
            fmt = "npz" if str(path).lower().endswith(".npz") else "lsgkm"
        if fmt == "npz":
            save_npz(self, path)
        elif fmt == "lsgkm":
            save_lsgkm(self, path)
        else:
            raise ValueError(f"Unknown format {fmt!r}. Use 'npz' or 'lsgkm'.")
