"""Serving: a device-resident request loop with continuous batching.

GkmServer keeps one model's SV index in HBM and takes mixed requests --
predict, score_variants, ism, gkmexplain -- from any thread (submit returns a
Future).  A scheduler thread admits waiting requests into the next scoring
batch as long as the batch's row budget and the device's free memory allow
(requests that do not fit wait; a request larger than the whole budget is
refused), merges every predict and variant row of the batch into one
graph-captured scoring pass, and keeps up to max_inflight such passes in flight
(one by default) on separate streams; requests that arrive while a pass runs
join the next one.  ISM and GkmExplain requests run on their own worker
stream beside the scoring passes; the requests of one kind (and explain mode)
already waiting when the worker is free run as one batched call (up to
max_side_rows rows), so a burst of them shares the device.  Every request's
latency (submit to result) is recorded; stats() gives p50/p99 per request type
and sequences per second.

The scheduling is independent of the device work: a backend object runs the
batches (GpuBackend here; the tests drive the same loop with a host fake).
"""

from __future__ import annotations

import queue
import threading
import time
import warnings
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np

KINDS = ("predict", "score_variants", "ism", "explain")


class AdmissionError(RuntimeError):
    """The request can never be admitted (larger than the budget) or is malformed."""


@dataclass
class Request:
    kind: str
    x: object = None                # predict/ism/explain: codes [n, L] or list of strings
    lengths: object = None
    alt: object = None              # score_variants: alt alleles
    alt_lengths: object = None
    mode: str = "hypothetical"      # explain mode
    future: Future = field(default_factory=Future)
    t_submit: float = 0.0
    rows: int = 0                   # scoring rows it adds to a batch
    bytes: int = 0                  # device memory it needs while it runs
    t_start: float = 0.0


def _percentiles(v):
    if not v:
        return {"n": 0}
    a = np.asarray(v) * 1e3
    return {"n": len(a), "p50_ms": float(np.percentile(a, 50)), "p99_ms": float(np.percentile(a, 99)),
            "mean_ms": float(a.mean())}


class GkmServer:
    """Continuous-batching request loop over one model (see the module doc)."""

    def __init__(self, backend, *, max_batch_rows: int = 8192, max_inflight: int = 1,
                 memory_reserve: int = 2 << 30, max_wait_s: float = 0.002, max_side_rows: int = 4,
                 side_yield_s: float = 0.0):
        """max_inflight: scoring passes in flight at once.  One by default: the
        requests arriving during a pass then join one larger pass instead of
        a second small one beside it, which leaves more of the GPU to ISM /
        GkmExplain work (measured, config-5 mix, Poisson 300 and 400 req/s,
        two runs each: p99 77 - 157 ms with one pass in flight, 91 - 264 ms
        with two).

        side_yield_s > 0: before each ISM / GkmExplain call the side worker
        waits (at most this long) until no scoring pass is in flight or
        waiting, so the two kinds of work share the GPU in time: a scoring
        pass's index-query blocks take a whole SM's shared memory and can sit
        behind a side call's kernels until they finish.  Off by default: the
        GPU backend cuts ISM into short passes on a low-priority stream, so a
        scoring pass waits for one pass at most, and waiting before every side
        call starved side work whenever scoring stayed busy (measured, config-5
        mix at 50 % load: worst p99 over six runs 919 ms with a 50 ms yield,
        275 ms without)."""
        self.backend = backend
        self.max_batch_rows = max_batch_rows
        self.max_inflight = max_inflight
        self.memory_reserve = memory_reserve
        self.max_wait_s = max_wait_s
        self.max_side_rows = max_side_rows
        self.side_yield_s = side_yield_s
        self.side_memory_wait_s = 30.0
        self.side_batches: list[int] = []  # requests per side call
        self._in: queue.Queue = queue.Queue()
        self._side: queue.Queue = queue.Queue()
        self._waiting: list[Request] = []
        self._inflight: list = []  # (handle, [requests])
        self._side_load = 0  # ISM / GkmExplain requests waiting or running
        self._lat: dict = {k: [] for k in KINDS}
        self._seqs = 0
        self._t0 = None
        self._stop = threading.Event()
        self._threads: list[threading.Thread] = []
        self._lock = threading.Lock()
        self.admitted = 0
        self.deferred = 0
        self.rejected = 0

    # -- client side ---------------------------------------------------------

    def submit(self, kind: str, x=None, *, lengths=None, alt=None, alt_lengths=None, mode="hypothetical") -> Future:
        if kind not in KINDS:
            raise ValueError(f"kind must be one of {KINDS}, got {kind!r}")
        r = Request(kind, x, lengths, alt, alt_lengths, mode)
        r.t_submit = time.perf_counter()
        try:
            self.backend.prepare(r)
        except Exception as e:  # malformed request: fail it, never the loop
            self.rejected += 1
            r.future.set_exception(e)
            return r.future
        if r.kind in ("predict", "score_variants") and r.rows > self.max_batch_rows:
            self.rejected += 1
            r.future.set_exception(AdmissionError(
                f"{r.rows} rows exceed the batch budget of {self.max_batch_rows}; split the request"))
            return r.future
        (self._in if r.kind in ("predict", "score_variants") else self._side).put(r)
        return r.future

    # -- loop ------------------------------------------------------------------

    def start(self):
        self._t0 = time.perf_counter()
        self._stop.clear()
        self._threads = [threading.Thread(target=self._score_loop, daemon=True),
                         threading.Thread(target=self._side_loop, daemon=True)]
        for t in self._threads:
            t.start()
        return self

    def stop(self, timeout: float = 60.0):
        self._stop.set()
        for t in self._threads:
            t.join(timeout)
        self._threads = []

    def __enter__(self):
        return self.start()

    def __exit__(self, *a):
        self.stop()

    def _free_memory(self) -> int:
        return self.backend.free_memory() - self.memory_reserve

    def _score_loop(self):
        while not (self._stop.is_set() and not self._waiting and not self._inflight and self._in.empty()):
            # take everything that has arrived
            try:
                timeout = 0.0005 if (self._waiting or self._inflight) else 0.01
                self._waiting.append(self._in.get(timeout=timeout))
                while True:
                    self._waiting.append(self._in.get_nowait())
            except queue.Empty:
                pass
            # retire finished batches first: that frees slots and memory
            still = []
            for handle, reqs in self._inflight:
                if self.backend.done(handle):
                    self._finish_batch(handle, reqs)
                else:
                    still.append((handle, reqs))
            self._inflight = still
            if not self._waiting or len(self._inflight) >= self.max_inflight:
                continue
            # admit in arrival order while the row budget and free memory allow
            batch, rows, need = [], 0, 0
            free = self._free_memory()
            for r in list(self._waiting):
                if rows + r.rows > self.max_batch_rows or need + r.bytes > free:
                    self.deferred += 1
                    break
                batch.append(r)
                rows += r.rows
                need += r.bytes
            if not batch:
                if not self._inflight and self._waiting and self._waiting[0].bytes > free:
                    r = self._waiting.pop(0)  # can never fit: refuse it
                    self.rejected += 1
                    r.future.set_exception(AdmissionError("not enough free device memory for this request"))
                continue
            for r in batch:
                self._waiting.remove(r)
                r.t_start = time.perf_counter()
            self.admitted += len(batch)
            try:
                # tells the backend whether side work waits, so it may leave it SMs
                self.backend.side_busy = self._side_load > 0
                handle = self.backend.launch_scoring(batch)
            except Exception as e:
                for r in batch:
                    r.future.set_exception(e)
                continue
            self._inflight.append((handle, batch))

    def _finish_batch(self, handle, reqs):
        try:
            results = self.backend.collect_scoring(handle, reqs)
        except Exception as e:
            for r in reqs:
                r.future.set_exception(e)
            return
        now = time.perf_counter()
        with self._lock:
            for r, res in zip(reqs, results):
                self._lat[r.kind].append(now - r.t_submit)
                self._seqs += r.rows
                r.future.set_result(res)

    def _side_loop(self):
        pending: list[Request] = []
        batched = hasattr(self.backend, "run_side_batch")
        call_bytes = getattr(self.backend, "side_call_bytes", 0)
        while not (self._stop.is_set() and self._side.empty() and not pending):
            try:
                pending.append(self._side.get(timeout=0.01 if not pending else 0.0005))
                while True:
                    pending.append(self._side.get_nowait())
            except queue.Empty:
                pass
            self._side_load = len(pending)
            if not pending:
                continue
            # the oldest request's kind (and explain mode), with every waiting
            # request of the same kind that fits the row budget
            head = pending[0]
            free = self._free_memory()
            batch, rows, need = [], 0, call_bytes
            for r in list(pending):
                if r.kind != head.kind or r.mode != head.mode:
                    continue
                if batch and (not batched or rows + r.rows > self.max_side_rows or need + r.bytes > free):
                    break
                batch.append(r)
                rows += r.rows
                need += r.bytes
            for r in batch:
                pending.remove(r)
            # the oldest request alone may still need more than is free: wait
            # for memory (bounded), then refuse it
            deadline = time.perf_counter() + self.side_memory_wait_s
            while need > self._free_memory() and time.perf_counter() < deadline and not self._stop.is_set():
                time.sleep(0.001)
            if need > self._free_memory():
                self.rejected += len(batch)
                for r in batch:
                    r.future.set_exception(AdmissionError("not enough free device memory for this request"))
                continue
            if self.side_yield_s > 0:
                until = time.perf_counter() + self.side_yield_s
                while (self._inflight or self._waiting or not self._in.empty()) and time.perf_counter() < until:
                    time.sleep(0.0002)
            t = time.perf_counter()
            for r in batch:
                r.t_start = t
            try:
                results = self.backend.run_side_batch(batch) if batched else [self.backend.run_side(batch[0])]
            except Exception as e:
                for r in batch:
                    r.future.set_exception(e)
                continue
            now = time.perf_counter()
            with self._lock:
                self.side_batches.append(len(batch))
                for r in batch:
                    self._lat[r.kind].append(now - r.t_submit)
                    self._seqs += r.rows
            for r, res in zip(batch, results):
                r.future.set_result(res)

    def stats(self) -> dict:
        with self._lock:
            wall = time.perf_counter() - (self._t0 or time.perf_counter())
            out = {k: _percentiles(v) for k, v in self._lat.items()}
            allv = [x for v in self._lat.values() for x in v]
            out["all"] = _percentiles(allv)
            out["seqs_per_sec"] = self._seqs / wall if wall > 0 else 0.0
            out["admitted"], out["deferred"], out["rejected"] = self.admitted, self.deferred, self.rejected
            out["side_calls"] = len(self.side_batches)
            out["side_requests_per_call"] = (float(np.mean(self.side_batches)) if self.side_batches else 0.0)
            return out


class GpuBackend:
    side_call_bytes = 3 << 29  # an ISM / explain call's chunked scratch (1.5 GiB)

    """Runs a GkmServer's batches on the model's GPU: scoring rows through
    BatchedScorer (two instances, one per in-flight slot, each on its own
    high-priority stream), ISM and GkmExplain through BatchedIsm /
    BatchedExplain bucket graphs on a low-priority side stream whose persistent
    index queries take at most side_sm_share of the SMs."""

    # scoring batches of at most this many rows skip the graphs (DirectScorer):
    # the index query then splits their long rows over the whole GPU
    direct_rows = 64

    def __init__(self, model, slots: int = 2, side_sm_share: float = 1.0, side_graphs: bool = True,
                 side_pass_positions: int = 128, scoring_sm_share: float = 1.0):
        """side_sm_share: the share of the SMs the side worker's persistent
        index queries may take (1: all), so that a scoring pass launched
        meanwhile finds SMs free; side_graphs: ISM / GkmExplain through the
        bucketed graph runners (else direct ism() / gkmexplain() calls);
        side_pass_positions: index-path ISM passes of at most this many
        positions (None: as many as the workspace holds), so that a scoring
        pass waits for at most one short side kernel; scoring_sm_share: the
        share of the SMs a scoring pass's persistent index query may take
        while ISM / GkmExplain work waits (1: all; applies to the passes
        scored directly, not to the captured graphs of large batches)."""
        import torch

        from .batch import BatchedScorer, DirectScorer

        self.model = model
        self.torch = torch
        model._sv_index()
        model._sv_diag()
        self.scorers = [BatchedScorer(model) for _ in range(slots)]
        self.direct = [DirectScorer(model) for _ in range(slots)]
        # scoring passes are latency-bound requests: their streams get the
        # highest priority, so their blocks are dispatched before pending
        # blocks of the side stream's ISM / explain kernels
        p = torch.cuda.Stream.priority_range()  # a lower number is a higher priority
        self.streams = [torch.cuda.Stream(priority=min(p)) for _ in range(slots)]
        self.side_stream = torch.cuda.Stream(priority=max(p))
        props = torch.cuda.get_device_properties(model._device)
        self.side_blocks = 0 if side_sm_share >= 1 else max(1, int(props.multi_processor_count * side_sm_share))
        self.scoring_blocks = (0 if scoring_sm_share >= 1
                               else max(1, int(props.multi_processor_count * scoring_sm_share)))
        self.side_busy = False  # set by the server before each scoring launch
        self.side_graphs = side_graphs
        self.side_pass_positions = side_pass_positions
        # ISM / GkmExplain in bucket-shaped CUDA graphs, one runner per kind
        # (and explain mode), built by the side worker thread
        self.side_runners: dict = {}
        self._slot = 0
        self._busy = [False] * slots

    def warm(self, max_len: int = 2048, max_rows: int = 8192, explain_modes=("hypothetical",)) -> None:
        """Run and capture every graph bucket the loop can use (scoring rows in
        multiples of 1,024 up to max_rows, side calls of max_side_rows, lengths
        64..max_len) on rows of length 0, which have no windows and so almost
        no work: a bucket's first use and its capture then never fall inside
        a request's latency (the graphs do not depend on the rows' contents)."""
        torch = self.torch
        from .batch import BatchedExplain, BatchedIsm, _bucket_len

        dev = self.model._device
        lengths = [64]
        while lengths[-1] < _bucket_len(max_len):
            lengths.append(lengths[-1] * 2)
        for i, scorer in enumerate(self.scorers):
            with torch.cuda.stream(self.streams[i]):
                for rows in range(1024, max_rows + 1, 1024):
                    for L in lengths:
                        x = torch.zeros((rows, L), dtype=torch.uint8, device=dev)
                        ln = torch.zeros(rows, dtype=torch.int64, device=dev)
                        for _ in range(2):
                            scorer.score(x, ln)
        with torch.cuda.stream(self.side_stream):
            for key in ["ism"] + [("explain", m) for m in explain_modes]:
                runner = self.side_runners.get(key)
                if runner is None:
                    runner = self.side_runners[key] = (BatchedIsm(self.model, self.side_pass_positions)
                                                       if key == "ism" else BatchedExplain(self.model, key[1]))
                try:
                    for L in lengths:
                        x = torch.zeros((runner.row_granule, L), dtype=torch.uint8, device=dev)
                        ln = torch.zeros(runner.row_granule, dtype=torch.int64, device=dev)
                        for _ in range(2):
                            runner(x, ln)
                except NotImplementedError:
                    continue  # this model has no such path (its requests fail alone)
        torch.cuda.synchronize()

    def free_memory(self) -> int:
        """Bytes a new request can use: the device's free memory plus what
        torch's caching allocator holds but no tensor uses (it reuses that
        before asking the device; mem_get_info alone would count it as taken
        for as long as the cache keeps it)."""
        torch = self.torch
        free, _ = torch.cuda.mem_get_info()
        cached = torch.cuda.memory_reserved() - torch.cuda.memory_allocated()
        return int(free + max(cached, 0))

    def prepare(self, r: Request):
        from .inputs import SeqBatch, allele_batches

        if r.kind == "score_variants":
            rb, ab = allele_batches(r.x, r.alt, r.lengths, r.alt_lengths)
            r.x, r.alt, r.lengths, r.alt_lengths = rb.codes, ab.codes, rb.lengths, ab.lengths
            n, L = rb.B, rb.L
            r.rows = 2 * n
        else:
            b = SeqBatch.read(r.x, r.lengths)
            r.x, r.lengths = b.codes, b.lengths
            n, L = b.B, b.L
            r.rows = n
        # packed windows + scratch of its rows (ISM: mutant window sets too)
        # device memory while it runs: packed windows and float64 outputs; an
        # explain row also holds its [4, l] window parts and (RBF) its SV
        # weights.  A side call's own scratch (ISM mutant kernel rows, chunked
        # to about 1 GiB) is side_call_bytes, counted once per call.
        S = self.model.num_support_vectors
        per_row = {"predict": L * 16, "score_variants": L * 16, "ism": L * 48,
                   "explain": L * (48 + 8 * 4 * self.model.kernel.l) + 8 * S}[r.kind]
        r.bytes = r.rows * per_row

    def launch_scoring(self, batch):
        torch = self.torch
        slot = self._busy.index(False)
        self._busy[slot] = True
        rows, lens, spans = [], [], []
        L = 0
        for r in batch:
            if r.kind == "predict":
                parts = [(r.x, r.lengths)]
            else:
                parts = [(r.alt, r.alt_lengths), (r.x, r.lengths)]
            start = len(rows)
            for x, ln in parts:
                x = np.asarray(x)
                L = max(L, x.shape[1])
                for i in range(x.shape[0]):
                    rows.append(x[i])
                    lens.append(x.shape[1] if ln is None else int(ln[i]))
            spans.append((start, len(rows)))
        codes = np.zeros((len(rows), L), np.uint8)
        for i, x in enumerate(rows):
            codes[i, : len(x)] = x
        lens = np.asarray(lens, np.int64)
        stream = self.streams[slot]
        if self.scoring_blocks:
            from ._lib import call

            # this (scheduler) thread's index queries: leave SMs to side work that waits
            call("gkm_set_thread_grid_limit", int(self.scoring_blocks if self.side_busy else 0))
        with torch.cuda.stream(stream):
            xd = torch.from_numpy(codes).pin_memory().to(self.model._device, non_blocking=True)
            ld = torch.from_numpy(lens).pin_memory().to(self.model._device, non_blocking=True)
            scorer = self.direct[slot] if len(rows) <= self.direct_rows else self.scorers[slot]
            out = scorer.score(xd, ld, check=False)
            host = torch.empty(out.shape, dtype=out.dtype, pin_memory=True)
            host.copy_(out, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record()
        return (slot, ev, host, spans, lens, scorer, out)

    def done(self, handle) -> bool:
        return handle[1].query()

    def collect_scoring(self, handle, reqs):
        slot, ev, host, spans, lens, scorer, out = handle
        ev.synchronize()
        with self.torch.cuda.stream(self.streams[slot]):
            if scorer.check_flags():  # reran exactly: the first copy is stale
                host.copy_(out)
                self.torch.cuda.current_stream().synchronize()
        self._busy[slot] = False
        scores = host.numpy().copy()
        l = self.model.kernel.l
        scores[lens < l] = np.nan
        out = []
        for r, (a, b) in zip(reqs, spans):
            s = scores[a:b, None]
            if r.kind == "score_variants":
                n = (b - a) // 2
                s = s[:n] - s[n:]
            out.append(s)
        return out

    def run_side(self, r: Request):
        return self.run_side_batch([r])[0]

    def run_side_batch(self, reqs):
        """One ISM or GkmExplain call over every row of reqs (same kind and
        mode), rows padded to the widest; each request gets its own rows at its
        own width (a row's results do not depend on the rows beside it)."""
        torch = self.torch
        L = max(int(np.asarray(r.x).shape[1]) for r in reqs)
        xs, lens, spans, a = [], [], [], 0
        for r in reqs:
            x = np.asarray(r.x)
            n, w = x.shape
            pad = np.zeros((n, L), np.uint8)
            pad[:, :w] = x
            xs.append(pad)
            lens.append(np.full(n, w, np.int64) if r.lengths is None else np.asarray(r.lengths, np.int64))
            spans.append((a, n, w))
            a += n
        X, lengths = np.concatenate(xs), np.concatenate(lens)
        from ._lib import call
        from .batch import BatchedExplain, BatchedIsm

        call("gkm_set_thread_grid_limit", int(self.side_blocks))  # this (side worker) thread only
        key = "ism" if reqs[0].kind == "ism" else ("explain", reqs[0].mode)
        runner = self.side_runners.get(key)
        if runner is None:
            if not self.side_graphs:
                from .explain import gkmexplain
                from .ism import ism as ism_call

                runner = ((lambda x, ln: ism_call(self.model, x, lengths=ln)) if key == "ism" else
                          (lambda x, ln, mode=reqs[0].mode: gkmexplain(self.model, x, lengths=ln, mode=mode)))
            else:
                runner = (BatchedIsm(self.model, self.side_pass_positions) if key == "ism"
                          else BatchedExplain(self.model, reqs[0].mode))
            self.side_runners[key] = runner
        with torch.cuda.stream(self.side_stream):
            if self.side_graphs:
                xd = torch.from_numpy(X).pin_memory().to(self.model._device, non_blocking=True)
                ld = torch.from_numpy(lengths).pin_memory().to(self.model._device, non_blocking=True)
                res = runner(xd, ld)
            else:
                with warnings.catch_warnings():
                    warnings.simplefilter("ignore")  # short rows: marked NaN below
                    res = runner(X, lengths)
            host = res.cpu().numpy()
        host[lengths < self.model.kernel.l] = np.nan  # rows with no window
        return [host[a:a + n, :, :w] for a, n, w in spans]
