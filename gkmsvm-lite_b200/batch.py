"""Batched scoring: whole query batches in persistent, CUDA-graph-captured
launches.

A batch of queries of uneven length is packed into fixed device buffers whose
shape is rounded up to a bucket (rows to a multiple of 1,024, length to a power
of two), so a handful of CUDA graphs cover every batch.  Each graph holds the
whole scoring pass: packing, the query self-kernels, the longest-first row
order, and the persistent l-mer index query whose blocks (one per SM) take
(SV tile, row) items from a device work queue, tile-major, then the per-row
finish.  Replaying a graph costs one launch.

Linear kernels with an l-mer table score through the table instead (a
self-kernel plus W lookups per row), also captured.
"""

from __future__ import annotations

import gc
import weakref

import numpy as np
import torch

from . import engine
from .kernels import RbfKernel

_ROW_GRANULE = 1024


def _capture_graph(graph, fn, pool=None):
    """fn()'s CUDA work captured into graph in thread-local mode, on a capture
    stream of the graph's own.  torch.cuda.graph() is not used: it
    synchronises the whole device first (an error while another thread -- a
    server's other worker -- is capturing) and shares one capture stream per
    process between threads."""
    cs = torch.cuda.Stream()
    cs.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(cs):
        graph.capture_begin(pool=pool, capture_error_mode="thread_local")
        try:
            fn()
        finally:
            graph.capture_end()
    torch.cuda.current_stream().wait_stream(cs)


def _bucket_len(L: int) -> int:
    b = 64
    while b < L:
        b *= 2
    return b


def _bucket_rows(B: int) -> int:
    return max(_ROW_GRANULE, -(-B // _ROW_GRANULE) * _ROW_GRANULE)


class _Graph:
    def __init__(self, scorer, rows: int, L: int):
        m = scorer.model
        dev = m._device
        self.rows, self.L = rows, L
        self.codes = torch.zeros((rows, L), dtype=torch.uint8, device=dev)
        self.lengths = torch.zeros(rows, dtype=torch.int64, device=dev)
        self.out = torch.empty(rows, dtype=torch.float64, device=dev)
        self.graph = None
        self._scorer = weakref.ref(scorer)  # no cycle: graphs go with their scorer

    @property
    def scorer(self):
        return self._scorer()

    def _prep(self):
        s = self.scorer
        spec = s.model._spec()
        self.fwd, self.rc, self.counts = engine.pack(spec, self.codes, self.lengths)
        if s.table is not None:
            return
        if s.normalize:
            dx = engine.self_kernel(spec, self.fwd, self.rc, self.counts)
            self.inv_dx = 1.0 / torch.sqrt(torch.clamp(dx, min=1e-20))
        else:
            self.inv_dx = torch.ones(self.rows, dtype=torch.float64, device=self.fwd.device)
        self.order = torch.argsort(self.counts, descending=True).to(torch.int32)

    def _query(self):
        s = self.scorer
        m = s.model
        if s.table is not None:
            self.out.copy_(engine.table_score(m._spec(), s.table, self.fwd, self.rc, self.counts, m.bias,
                                              s.normalize))
            return
        s.index.score(self.fwd, self.counts, self.inv_dx, s.inv_ds, s.coef, s.gamma, s.rbf, m.bias, self.order,
                      out=self.out, check=False)

    def _body(self):
        self._prep()
        self._query()

    def _capture(self):
        # warm-up on a side stream, then capture the two phases (the work-queue
        # counter, the stream-ordered scratch and every kernel go into them)
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            self._body()
        torch.cuda.current_stream().wait_stream(side)
        # thread-local capture (_capture_graph): other threads may keep issuing CUDA
        # work meanwhile.  The cyclic garbage collector stays off
        # while a capture is open: freeing an unreachable object that holds
        # another CUDA graph or device memory is not permitted during capture
        # and would invalidate it (torch.cuda.graph collects just before).
        enabled = gc.isenabled()
        gc.disable()
        try:
            self.g_prep = torch.cuda.CUDAGraph()
            _capture_graph(self.g_prep, self._prep)
            self.g_query = torch.cuda.CUDAGraph()
            _capture_graph(self.g_query, self._query, pool=self.g_prep.pool())
        finally:
            if enabled:
                gc.enable()
        self.graph = True

    def run(self, events=None):
        """Replay; events (start, end): recorded around the query phase.  The
        bucket's first batch runs eagerly and the second captures, so a shape
        seen once pays no capture."""
        if self.graph is None:
            self.uses = getattr(self, "uses", 0) + 1
            if self.uses == 1:
                self._prep()
                if events:
                    events[0].record()
                self._query()
                if events:
                    events[1].record()
                return
            self._capture()
        self.g_prep.replay()
        if events:
            events[0].record()
        self.g_query.replay()
        if events:
            events[1].record()


class BatchedScorer:
    """Scores [B, L] code batches against model's SVs in graph-captured
    launches; results equal model(x) (same kernels, same order of sums)."""

    def __init__(self, model, use_graphs: bool = True):
        self.model = model
        kernel = model.kernel
        self.normalize = kernel.base.normalize
        self.rbf = isinstance(kernel, RbfKernel)
        self.gamma = kernel.gamma if self.rbf else 0.0
        self.table = model._lmer_table_for()
        self.index = None
        if self.table is None:
            self.index = model._sv_index()
            if self.index is None:
                raise ValueError("batched scoring needs the l-mer index or the l-mer table")
            self.inv_ds = model._inv_ds()
            self.coef = model._sv_coef()
        self.use_graphs = use_graphs
        self._graphs: dict = {}

    def _graph(self, B: int, L: int) -> _Graph:
        key = (_bucket_rows(B), _bucket_len(L))
        g = self._graphs.get(key)
        if g is None:
            g = self._graphs[key] = _Graph(self, *key)
        return g

    def score(self, codes: torch.Tensor, lengths: torch.Tensor | None = None, events=None,
              check: bool = True) -> torch.Tensor:
        """[B] float64 scores (bias included) of device codes [B, L] with
        device lengths [B] (None: every row L long).  events: optional CUDA
        events recorded around the query phase.  check=False skips the index
        flag read (no synchronisation); call check_flags() later."""
        B, L = codes.shape
        g = self._graph(B, L)
        self._last = g
        if self.index is not None:
            self._before = self.index.counters()
        g.codes[:B, :L].copy_(codes)
        if L < g.L:
            g.codes[:B, L:].zero_()
        if lengths is None:
            g.lengths[:B].fill_(L)
        else:
            g.lengths[:B].copy_(lengths)
        g.lengths[B:].zero_()
        if self.use_graphs:
            g.run(events)
        else:
            g._prep()
            if events:
                events[0].record()
            g._query()
            if events:
                events[1].record()
        if check:
            self.check_flags(g)
        return g.out[:B]

    def check_flags(self, g=None):
        """Waits for the last batch; reruns it eagerly with 32-bit counters if
        a query block's 16-bit carries outgrew its log meanwhile (the graph
        keeps the fast kernel).  Returns True when it reran."""
        if g is None:
            g = self._last
        if self.index is not None:
            return self.index.settle(self._before, g._body)
        return False


class DirectScorer:
    """BatchedScorer's interface without graphs or bucket padding, for small
    batches: the index query sees the batch's real rows, so a few long rows
    are cut into window ranges over the whole GPU (row splits) instead of
    keeping one SM per (row, SV tile).  Results equal model(x)'s."""

    def __init__(self, model):
        self.model = model
        kernel = model.kernel
        self.normalize = kernel.base.normalize
        self.rbf = isinstance(kernel, RbfKernel)
        self.gamma = kernel.gamma if self.rbf else 0.0
        self.table = model._lmer_table_for()
        self.index = None
        if self.table is None:
            self.index = model._sv_index()
            if self.index is None:
                raise ValueError("direct scoring needs the l-mer index or the l-mer table")
        self._rerun = None

    def score(self, codes: torch.Tensor, lengths: torch.Tensor | None = None, events=None,
              check: bool = True) -> torch.Tensor:
        m = self.model
        spec = m._spec()
        fwd, rc, counts = engine.pack(spec, codes, lengths)
        if events:
            events[0].record()
        if self.table is not None:
            out = engine.table_score(spec, self.table, fwd, rc, counts, m.bias, self.normalize)
        else:
            if self.normalize:
                dx = engine.self_kernel(spec, fwd, rc, counts)
                inv_dx = 1.0 / torch.sqrt(torch.clamp(dx, min=1e-20))
            else:
                inv_dx = torch.ones(fwd.shape[0], dtype=torch.float64, device=fwd.device)
            out = torch.empty(fwd.shape[0], dtype=torch.float64, device=fwd.device)

            def run():
                self.index.score(fwd, counts, inv_dx, m._inv_ds(), m._sv_coef(), self.gamma, self.rbf, m.bias,
                                 out=out, check=False)

            self._before = self.index.counters()
            run()
            self._rerun = run
        if events:
            events[1].record()
        if check:
            self.check_flags()
        return out

    def check_flags(self, g=None):
        """Waits for the last batch; reruns it with 32-bit counters if a query
        block's 16-bit carries outgrew its log.  Returns True when it reran."""
        if self.index is not None and self._rerun is not None:
            return self.index.settle(self._before, self._rerun)
        return False


class _PerRowGraph:
    """One bucket of a per-row pipeline (ISM, GkmExplain): fixed device
    buffers codes [rows, L] and lengths [rows] (rows past the batch get length
    0: no windows, no work) and one CUDA graph of the whole pass, captured on
    the first call after an eager warm-up."""

    def __init__(self, runner, rows: int, L: int):
        dev = runner.model._device
        self.rows, self.L = rows, L
        self.codes = torch.zeros((rows, L), dtype=torch.uint8, device=dev)
        self.lengths = torch.zeros(rows, dtype=torch.int64, device=dev)
        self.out = None
        self.graph = None
        self._runner = weakref.ref(runner)

    def _body(self):
        self.out = self._runner().body(self.codes, self.lengths)

    def run(self):
        if self.graph is None:
            side = torch.cuda.Stream()
            side.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(side):
                self._body()  # warm-up: builds SV caches, tunes pairwise forms
            torch.cuda.current_stream().wait_stream(side)
            enabled = gc.isenabled()
            gc.disable()
            try:
                self.graph = torch.cuda.CUDAGraph()
                _capture_graph(self.graph, self._body)
            finally:
                if enabled:
                    gc.enable()
        self.graph.replay()


class _PerRowRunner:
    """Shape-bucketed, graph-captured runs of a per-row pipeline: rows rounded
    up to a multiple of row_granule, length to a power of two >= 64, so a few
    graphs serve batches of uneven length; each replay is one launch of the
    whole pass (packing, self-kernels, the persistent index queries over the
    device work queue, the reductions).  A bucket runs eagerly on its first
    use and is captured on its second, so one-off shapes pay no capture.
    Results equal the eager pass's."""

    row_granule = 8
    capture_after = 1  # eager runs of a bucket before it is captured

    def __init__(self, model):
        self.model = model
        self._graphs: dict = {}
        self._uses: dict = {}

    def body(self, codes, lengths):  # [rows, 4, L] on the device, no host synchronisation
        raise NotImplementedError

    def __call__(self, codes: torch.Tensor, lengths: torch.Tensor | None = None) -> torch.Tensor:
        """[B, 4, L] of device codes [B, L] (lengths: device [B], None: all L);
        0 past each row's length, rows shorter than l all 0 (the caller
        marks them NaN)."""
        B, L = codes.shape
        key = (-(-B // self.row_granule) * self.row_granule, _bucket_len(max(L, self.model.kernel.l)))
        g = self._graphs.get(key)
        if g is None:
            g = self._graphs[key] = _PerRowGraph(self, *key)
        index = self.model._sv_index() if self.model.use_lmer_index else None
        before = index.counters() if index is not None else None
        g.codes[:B, :L].copy_(codes)
        g.codes[:B, L:].zero_()
        if lengths is None:
            g.lengths[:B].fill_(L)
        else:
            g.lengths[:B].copy_(lengths)
        g.lengths[B:].zero_()
        uses = self._uses.get(key, 0)
        self._uses[key] = uses + 1
        if uses < self.capture_after:
            g._body()
        else:
            g.run()
        if index is not None:
            # 16-bit counter carries that outgrew a block's log: rerun exactly
            index.settle(before, g._body)
        out = g.out[:B, :, :L]
        past = torch.arange(L, device=out.device)[None, None, :] >= g.lengths[:B, None, None]
        return out.masked_fill(past, 0.0)


class BatchedIsm(_PerRowRunner):
    """gkmsvm_lite_b200.ism of device code batches through bucket graphs."""

    def __init__(self, model, pass_positions: int = None):
        """pass_positions: on the index path, at most this many positions per
        pass (one short persistent query per pass, so that kernels of other
        streams get the SMs between passes); None: as many as 1.5 GiB of
        workspace holds."""
        super().__init__(model)
        self.pass_positions = pass_positions
        self._work = None
        self._works = []  # every workspace a captured graph refers to

    def body(self, codes, lengths):
        from .ism import _ism_rows, ism_pass_bytes, ism_workspace_bytes

        m = self.model
        work = None
        if m._lmer_table_for() is None:
            # the index path's workspace, shared by the buckets (their replays
            # are serial); grown for a bucket of more rows (the eager warm-up
            # allocates it, never the capture)
            B, L = codes.shape
            cap = None if self.pass_positions is None else ism_pass_bytes(m, B, self.pass_positions)
            need = ism_workspace_bytes(m, B, L, cap)
            if self._work is None or self._work.numel() < need:
                self._work = torch.empty(need, dtype=torch.uint8, device=codes.device)
                self._works.append(self._work)
            work = self._work[:need]  # the call sizes its passes by the bytes it is given
        return _ism_rows(m, codes, lengths, codes.device, check=False, work=work)


class BatchedExplain(_PerRowRunner):
    """gkmsvm_lite_b200.gkmexplain of device code batches through bucket
    graphs, for one mode ("importance", "hypothetical" or "perturbation")."""

    def __init__(self, model, mode: str = "hypothetical"):
        super().__init__(model)
        from .explain import _MODE_ALIASES

        self.mode = _MODE_ALIASES[mode]
        self._table = {}

    def body(self, codes, lengths):
        from .explain import _explain_rows, _explain_table

        m = self.model
        pert = self.mode == "perturbation"
        if pert not in self._table:
            # the explain table, if the model's switch calls for one, is chosen
            # once per runner (a large call's cost model)
            self._table[pert] = _explain_table(m, 1 << 62, pert, codes.device)
        return _explain_rows(m, codes, lengths, self.mode, codes.device, self._table[pert], check=False)
