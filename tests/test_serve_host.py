"""The serving loop's scheduling on the host, with a fake backend: continuous
batching (requests arriving during a batch join the next one while it is still
in flight), admission by free device memory, refusal of requests that can
never fit, malformed requests failing alone, and latency statistics.  No GPU."""

import threading
import time

import numpy as np
import pytest

from gkmsvm_lite_b200.serve import AdmissionError, GkmServer


class FakeBackend:
    def __init__(self, free=1 << 40, delay=0.02):
        self.free = free
        self.delay = delay
        self.batches = []
        self.inflight = 0
        self.max_inflight_seen = 0
        self.lock = threading.Lock()

    def free_memory(self):
        return self.free

    def prepare(self, r):
        if r.x is None:
            raise ValueError("no sequences")
        x = np.asarray(r.x)
        r.rows = x.shape[0] * (2 if r.kind == "score_variants" else 1)
        r.bytes = r.rows * 1000

    def launch_scoring(self, batch):
        with self.lock:
            self.inflight += 1
            self.max_inflight_seen = max(self.max_inflight_seen, self.inflight)
            self.batches.append([id(r) for r in batch])
        return (time.perf_counter() + self.delay, batch)

    def done(self, h):
        return time.perf_counter() >= h[0]

    def collect_scoring(self, h, reqs):
        with self.lock:
            self.inflight -= 1
        return [np.asarray(r.x).sum(axis=1, keepdims=True).astype(float) for r in reqs]

    def run_side(self, r):
        time.sleep(self.delay)
        return np.asarray(r.x) * 2.0


def test_results_and_continuous_batching():
    be = FakeBackend(delay=0.05)
    with GkmServer(be, max_batch_rows=64, max_inflight=2, memory_reserve=0) as srv:
        futs = []
        for i in range(40):
            x = np.full((3, 5), i)
            futs.append((i, srv.submit("predict", x)))
            time.sleep(0.004)
        side = srv.submit("ism", np.ones((1, 4)))
        for i, f in futs:
            np.testing.assert_array_equal(f.result(10), np.full((3, 1), 5 * i))
        np.testing.assert_array_equal(side.result(10), np.full((1, 4), 2.0))
        st = srv.stats()
    assert len(be.batches) > 1 and max(len(b) for b in be.batches) > 1  # merged into batches
    assert be.max_inflight_seen == 2  # a second batch started while the first ran
    assert st["predict"]["n"] == 40 and st["predict"]["p99_ms"] >= st["predict"]["p50_ms"] > 0
    assert st["ism"]["n"] == 1 and st["seqs_per_sec"] > 0


def test_admission_waits_for_memory_and_refuses_what_never_fits():
    be = FakeBackend(free=10_000, delay=0.02)
    with GkmServer(be, max_batch_rows=1000, memory_reserve=0) as srv:
        small = [srv.submit("predict", np.zeros((4, 3))) for _ in range(6)]  # 4,000 B each
        huge = srv.submit("predict", np.zeros((20, 3)))  # 20,000 B > all free memory
        for f in small:
            assert f.result(10).shape == (4, 1)
        with pytest.raises(AdmissionError):
            huge.result(10)
        st = srv.stats()
    assert st["deferred"] > 0 and st["rejected"] == 1


def test_bad_requests_fail_alone():
    be = FakeBackend()
    with GkmServer(be, max_batch_rows=8, memory_reserve=0) as srv:
        with pytest.raises(ValueError):
            srv.submit("nope", np.zeros((1, 3)))
        bad = srv.submit("predict", None)
        too_big = srv.submit("predict", np.zeros((9, 3)))
        ok = srv.submit("predict", np.ones((2, 3)))
        with pytest.raises(ValueError):
            bad.result(5)
        with pytest.raises(AdmissionError):
            too_big.result(5)
        np.testing.assert_array_equal(ok.result(5), [[3.0], [3.0]])


class FakeBatchBackend(FakeBackend):
    """Side requests through run_side_batch: one call per batch, recorded."""

    def __init__(self, **kw):
        super().__init__(**kw)
        self.side_calls = []

    def run_side_batch(self, reqs):
        with self.lock:
            self.side_calls.append([(r.kind, r.rows) for r in reqs])
        time.sleep(self.delay)
        return [np.asarray(r.x) * 2.0 for r in reqs]


def test_waiting_side_requests_share_one_call():
    be = FakeBatchBackend(delay=0.05)
    srv = GkmServer(be, max_side_rows=8).start()
    rng = np.random.default_rng(3)
    xs = [rng.integers(0, 4, (1 + i % 2, 20 + i)) for i in range(12)]
    futs = [srv.submit("ism", x) for x in xs] + [srv.submit("explain", xs[0], mode="perturbation")]
    for x, f in zip(xs, futs):
        np.testing.assert_array_equal(f.result(10), x * 2.0)
    np.testing.assert_array_equal(futs[-1].result(10), xs[0] * 2.0)
    srv.stop()
    # the first call takes what waited then; later ones gather the burst
    assert max(len(c) for c in be.side_calls) > 1
    assert all(len({k for k, _ in c}) == 1 for c in be.side_calls)  # one kind per call
    assert all(sum(n for _, n in c) <= 8 or len(c) == 1 for c in be.side_calls)  # the row budget
    st = srv.stats()
    assert st["ism"]["n"] == 12 and st["explain"]["n"] == 1


def test_side_request_beyond_free_memory_is_refused():
    be = FakeBatchBackend(free=10_000, delay=0.01)
    srv = GkmServer(be, memory_reserve=0)
    srv.side_memory_wait_s = 0.2
    srv.start()
    huge = srv.submit("ism", np.zeros((20, 3)))  # 20,000 B > all free memory
    ok = srv.submit("ism", np.ones((2, 3)))
    with pytest.raises(AdmissionError):
        huge.result(10)
    np.testing.assert_array_equal(ok.result(10), np.full((2, 3), 2.0))
    srv.stop()
    assert srv.stats()["rejected"] == 1


def test_side_worker_yields_to_scoring_passes():
    """With side_yield_s, an ISM / explain call waits (bounded) until no
    scoring pass is in flight or waiting, so the two share the GPU in time."""

    class Recording(FakeBackend):
        def __init__(self):
            super().__init__(delay=0.15)
            self.side_started_with_inflight = []

        def run_side(self, r):
            with self.lock:
                self.side_started_with_inflight.append(self.inflight)
            return np.asarray(r.x) * 2.0

    be = Recording()
    with GkmServer(be, max_inflight=2, memory_reserve=0, side_yield_s=1.0) as srv:
        p = srv.submit("predict", np.ones((2, 5)))
        time.sleep(0.02)  # the scoring pass is in flight when the ISM arrives
        s = srv.submit("ism", np.ones((1, 5)))
        assert s.result(10).shape == (1, 5) and p.result(10).shape == (2, 1)
    assert be.side_started_with_inflight == [0]

    # bounded: a side call never waits past side_yield_s
    be = Recording()
    be.delay = 5.0
    with GkmServer(be, max_inflight=2, memory_reserve=0, side_yield_s=0.05) as srv:
        srv.submit("predict", np.ones((2, 5)))
        time.sleep(0.02)
        t0 = time.perf_counter()
        srv.submit("ism", np.ones((1, 5))).result(10)
        assert time.perf_counter() - t0 < 2.0
    assert be.side_started_with_inflight == [1]


def test_backend_told_when_side_work_waits():
    """Before each scoring launch the server sets backend.side_busy: True while
    ISM / GkmExplain requests wait or run, False when none do."""

    class Recording(FakeBackend):
        def __init__(self):
            super().__init__(delay=0.01)
            self.seen = []

        def launch_scoring(self, batch):
            self.seen.append(getattr(self, "side_busy", None))
            return super().launch_scoring(batch)

        def run_side(self, r):
            time.sleep(0.3)
            return np.asarray(r.x) * 2.0

    be = Recording()
    with GkmServer(be, memory_reserve=0) as srv:
        srv.submit("predict", np.ones((1, 5))).result(10)
        side = srv.submit("ism", np.ones((1, 5)))
        time.sleep(0.05)  # the side call is running
        srv.submit("predict", np.ones((1, 5))).result(10)
        side.result(10)
        time.sleep(0.05)
        srv.submit("predict", np.ones((1, 5))).result(10)
    assert be.seen == [False, True, False]
