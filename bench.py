"""Benchmark: batched scoring of 100,000 queries (50-2000 bp, 0.5% N) against a
72,000-SV l=11 k=7 d=3 model (the config-3 workload), one B200 per rank.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

A step scores every query of the rank's batch against the t=3 model (gkmrbf,
gamma=2) with the inputs already in HBM: pack, query self-kernels, and the
fused l-mer index query + RBF + alpha reduction.  Ranks score independent query
batches against full SV replicas (weak scaling, no collective on the data
path); the time is the max over ranks.  Rank 0 prints one JSON line.

--impl reference times the CPU restatement of the reference's index path
(oracle/gkm_oracle.c, pthreads over all host cores, rows handed out one at a
time) on bounded samples of the same query stream rank 0 scores.

With --gpus N > 1 and no torchrun environment, the script starts N ranks
itself under torch.distributed.run; under torchrun, WORLD_SIZE must equal N.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "seqs/sec vs 72k-SV l=11 k=7 d=3 model, batched vs plain; serving p50/p99 ms"
PARAMS_T3 = {"L": 11, "k": 7, "d": 3, "gamma": 2.0}
PARAMS_T2 = {"L": 11, "k": 7, "d": 3}
WORKLOAD = ("config3: 72,000 SVs (200-500 bp, alpha ~ N(0, 0.1^2)), t=3 gkmrbf gamma=2, "
            "queries 50-2000 bp log-uniform with 0.5% N")


# ncu on a 2,000-query launch of this workload (profiles/index_query_config3_t3_2000q.md):
# throughput fractions of the units that bind the index query
NCU_INDEX_QUERY = {"l1tex_data_pipe_frac": 0.762, "lts_throughput_frac": 0.291, "dram_bytes": 3.093e10,
                   "lts_sector_hit_frac": 0.901, "shared_atomic_wavefronts_frac": 0.319,
                   "global_load_wavefronts_frac": 0.253, "shared_atomic_bank_conflicts_per_wavefront": 0.57,
                   "issue_active_frac": 0.589, "warps_active_frac": 0.50}


def job_config(queries: int, world: int) -> dict:
    """The workload description both arms print (the same dict for both)."""
    return {"workload": WORKLOAD, "queries_per_rank": queries, "svs": 72000, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (100k packed queries: 1.6 GB; the 165 MB SV index with its bucket words also exceeds the 126 MB L2)"}


def shard_seed(rank: int, base: int = 102) -> int:
    """Each rank scores its own query batch: the config-3 stream of seed base + rank."""
    return base + rank


def launch_command(args, env) -> list[str] | None:
    """The torchrun command that starts --gpus ranks when this process is not
    a rank of one already (None: run here).  Raises when a torchrun world
    disagrees with --gpus."""
    world = env.get("WORLD_SIZE")
    if world is not None:
        if int(world) != args.gpus:
            raise SystemExit(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}; launch one rank per GPU")
        return None
    if args.gpus <= 1:
        return None
    import socket

    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
            "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__), *sys.argv[1:]]


def timed_region(step, steps: int, warmup: int, dist=None, sync=lambda: None, clock=None) -> float:
    """warmup untimed steps, then `steps` timed steps bracketed by a barrier and
    a device sync on both sides; this rank's seconds.  clock: a (start, stop)
    pair of callables returning seconds (default perf_counter); the GPU arm
    passes CUDA events."""
    for _ in range(warmup):
        step()
    sync()
    if dist is not None:
        dist.barrier()
    sync()
    if clock is None:
        t0 = time.perf_counter()
        for _ in range(steps):
            step()
        sync()
        return time.perf_counter() - t0
    start, stop = clock
    start()
    for _ in range(steps):
        step()
    return stop()


def job_throughput(seconds: float, units: float, dist=None, device=None) -> tuple[float, float, float]:
    """(max seconds over ranks, units summed over ranks, whole-job units/s)."""
    if dist is not None:
        import torch

        t = torch.tensor([seconds, float(units)], dtype=torch.float64, device=device)
        tmax, tsum = t[:1].clone(), t[1:].clone()
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
        dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
        seconds, units = float(tmax.item()), float(tsum.item())
    return seconds, units, units / seconds


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--queries", type=int, default=100000)
    ap.add_argument("--no-extras", action="store_true", help="skip t=2, plain-call and CPU legs")
    ap.add_argument("--leg", default="all",
                    choices=["all", "gram", "train", "explain", "explain-pairs", "serve", "encode", "pairwise-forms",
                             "weighted", "ism-index"],
                    help="gram / train / explain: run only the Gram-matrix, SMO training or config-4 ISM and "
                         "GkmExplain leg (one GPU), print its JSON")
    ap.add_argument("--gram-n", type=int, default=4000, help="sequences of the Gram-matrix leg")
    ap.add_argument("--weighted-n", type=int, default=20000, help="queries of the weighted (t=5) scoring leg")
    ap.add_argument("--ism-rows", type=int, default=32, help="1,000 bp rows of the index-path ISM leg")
    return ap.parse_args()


class Clocks:
    """nvidia-smi samples (SM clock, throttle reasons) during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}




class PortBaseline:
    """The oracle's C restatement of the reference's CPU index path (SV l-mer
    index, fused query + RBF + alpha reduce, query self-kernels) on every host
    thread, rows handed out one at a time.  Built once per process: the index
    and the SV self-kernels are the model caches the reference builds on its
    first call."""

    def __init__(self, sv, svl, coef):
        from oracle import oracle as orc

        self.threads = os.cpu_count() or 1
        kd = orc.KernelDef.from_params("gkmrbf", PARAMS_T3)
        t0 = time.perf_counter()
        self.ib = orc.IndexBaseline(orc.OracleModel(sv, svl, coef, 0.0, kd), threads=self.threads)
        self.build_s = time.perf_counter() - t0

    def scores(self, xq, xl, rows) -> np.ndarray:
        rows = np.asarray(rows)
        L = int(xl[rows].max())
        return self.ib.scores(xq[rows, :L], xl[rows], threads=self.threads)[:, 0]

    def time_rows(self, xq, xl, rows) -> float:
        t0 = time.perf_counter()
        self.scores(xq, xl, rows)
        return time.perf_counter() - t0


# rows of the query stream each reference-arm step times (and the cpu_baseline
# sample of the GPU arm): consecutive, so every length in the stream's mix
REF_ROWS_PER_STEP = 320


def parity_rows(xl, nmask, n=256, seed=7) -> np.ndarray:
    """Rows of a timed batch the oracle re-scores: the 16 longest, the 16 with
    the largest share of N bases, and random others."""
    nfrac = nmask.sum(axis=1) / np.maximum(xl, 1)
    pick = list(np.argsort(-xl, kind="stable")[:16]) + list(np.argsort(-nfrac, kind="stable")[:16])
    rest = np.setdiff1d(np.arange(len(xl)), pick)
    pick += list(np.random.default_rng(seed).choice(rest, n - len(set(pick)), replace=False))
    return np.unique(np.asarray(pick))


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    import gkmsvm_lite_b200.synthetic as syn

    sv, svl, coef = syn.config3_model()
    # the same stream rank 0 of the GPU arm scores
    xq, xl, _ = syn.config3_queries(seed=shard_seed(0), n=args.queries)
    t0 = time.perf_counter()
    base = PortBaseline(sv, svl, coef)
    first_rows = np.arange(REF_ROWS_PER_STEP)
    base.time_rows(xq, xl, first_rows)
    first_s = time.perf_counter() - t0  # caches built + the first call
    nsteps = max(1, (len(xl) - REF_ROWS_PER_STEP) // REF_ROWS_PER_STEP)
    times = []

    def step(k=[0]):
        lo = REF_ROWS_PER_STEP * (1 + k[0] % nsteps)
        times.append(base.time_rows(xq, xl, np.arange(lo, lo + REF_ROWS_PER_STEP)))
        k[0] += 1

    for _ in range(args.warmup):  # small calls, as the reference's own benchmark warms up
        base.time_rows(xq, xl, np.arange(8))
    total = timed_region(step, args.steps, 0)
    v = REF_ROWS_PER_STEP * args.steps / total
    sample = (f"{REF_ROWS_PER_STEP} consecutive queries of the seed-{shard_seed(0)} stream per step "
              f"(steady state); first call {first_s:.1f} s (SV index {base.build_s:.1f} s with the SV "
              f"self-kernels, then {REF_ROWS_PER_STEP} queries)")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "seqs/sec", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": job_config(args.queries, world),
            "cpu_baseline": {"value": v, "unit": "seqs/sec", "cores": base.threads, "kind": "port",
                             "sample": sample, "first_s": first_s,
                             "steady_s_per_step": float(np.mean(times))},
            "e2e": {"value": v, "unit": "seqs/sec", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def serving_leg(sv, svl, coef, n_requests=600, seed=4, backend_kw=None, server_kw=None):
    """Config 5: the 72k-SV t=5 (wgkmrbf, gamma=1) model served with continuous
    batching.  Mixed requests (60% predict, 25% score-variants, 10% ISM, 5%
    GkmExplain), lengths log-uniform 20..2000 bp, alt = one SNV (80%) or an
    indel of 1..10 bp.  First all requests at once (capacity: everything
    batches), then Poisson arrivals at 50% and at 70% of that rate for p50/p99
    latency (open arrivals batch less, so 70% of the closed-loop capacity is
    near saturation; the 50% point is the headline); beside it the plain
    per-call form (each request its own call, one after another)."""
    import torch

    import gkmsvm_lite_b200 as gk
    import gkmsvm_lite_b200.synthetic as syn
    from gkmsvm_lite_b200.serve import GkmServer, GpuBackend

    rng = np.random.default_rng(seed)
    model = gk.GkmSVM(sv, coef, 0.0, "wgkmrbf", {"L": 11, "k": 7, "d": 3, "gamma": 1.0}, sv_lengths=svl).cuda()
    kinds = rng.choice(["predict", "score_variants", "ism", "explain"], size=n_requests, p=[0.6, 0.25, 0.1, 0.05])
    reqs = []
    for kind in kinds:
        ln = syn.log_uniform_lengths(rng, 1, 20, 2000)
        ln[0] = max(int(ln[0]), 11)
        x = syn.ragged_codes(rng, ln)
        r = {"kind": str(kind), "x": x, "lengths": ln}
        if kind == "score_variants":
            r["alt"], r["alt_lengths"] = syn.variant_pairs(rng, x, ln)
        reqs.append(r)
    backend = GpuBackend(model, **(backend_kw or {}))
    t0 = time.perf_counter()
    backend.warm()  # every graph bucket captured before the first request
    warm_s = time.perf_counter() - t0

    def submit_all(srv, rate=None):
        futs = []
        t0 = time.perf_counter()
        gaps = rng.exponential(1.0 / rate, len(reqs)) if rate else np.zeros(len(reqs))
        t = t0
        for r, g in zip(reqs, gaps):
            t += g
            d = t - time.perf_counter()
            if d > 0:
                time.sleep(d)
            futs.append(srv.submit(r["kind"], r["x"], lengths=r["lengths"], alt=r.get("alt"),
                                   alt_lengths=r.get("alt_lengths")))
        for f in futs:
            f.result(300)
        return time.perf_counter() - t0

    warm = GkmServer(backend, **(server_kw or {})).start()
    for r in reqs[:24]:
        warm.submit(r["kind"], r["x"], lengths=r["lengths"], alt=r.get("alt"), alt_lengths=r.get("alt_lengths")).result(600)
    warm.stop()
    srv = GkmServer(backend, **(server_kw or {})).start()
    t_closed = submit_all(srv)
    cap = srv.stats()
    srv.stop()
    # Poisson arrivals: three runs at 50 % of the closed-loop rate (other
    # arrival draws), one at 70 %
    runs50 = []
    for _ in range(3):
        srv = GkmServer(backend, **(server_kw or {})).start()
        submit_all(srv, 0.5 * len(reqs) / t_closed)
        runs50.append(srv.stats())
        srv.stop()
    srv = GkmServer(backend, **(server_kw or {})).start()
    submit_all(srv, 0.7 * len(reqs) / t_closed)
    loads = {0.5: runs50[0], 0.7: srv.stats()}
    srv.stop()
    rate = 0.5 * len(reqs) / t_closed
    open_stats = max(runs50, key=lambda st: st["all"].get("p99_ms", 0.0))  # the worst of the three
    # plain per-call form: each request its own call, in order
    t0 = time.perf_counter()
    seqs = 0
    for r in reqs:
        if r["kind"] == "predict":
            model(r["x"], lengths=r["lengths"]).cpu()
            seqs += 1
        elif r["kind"] == "score_variants":
            model.score_variants(r["x"], r["alt"], ref_lengths=r["lengths"], alt_lengths=r["alt_lengths"]).cpu()
            seqs += 2
        elif r["kind"] == "ism":
            gk.ism(model, r["x"], lengths=r["lengths"]).cpu()
            seqs += 1
        else:
            gk.gkmexplain(model, r["x"], lengths=r["lengths"], mode="hypothetical").cpu()
            seqs += 1
    torch.cuda.synchronize()
    plain = seqs / (time.perf_counter() - t0)
    return {
        "workload": "config5: 72,000 SVs t=5 wgkmrbf gamma=1; 60/25/10/5% predict/variants/ISM/explain, "
                    f"{len(reqs)} requests, 20-2000 bp",
        "capacity_seqs_per_sec": cap["seqs_per_sec"], "capacity_requests_per_sec": len(reqs) / t_closed,
        "poisson_rate_requests_per_sec": rate,
        "p50_ms": open_stats["all"].get("p50_ms"), "p99_ms": open_stats["all"].get("p99_ms"),
        "backend_warm_s": warm_s,
        "runs_at_50pct": [{"p50_ms": st["all"].get("p50_ms"), "p99_ms": st["all"].get("p99_ms"),
                           "seqs_per_sec": st["seqs_per_sec"]} for st in runs50],
        "headline_run": "the run of the three at 50 % with the highest p99",
        "by_kind_ms": {k: open_stats[k] for k in ("predict", "score_variants", "ism", "explain")},
        "served_seqs_per_sec": open_stats["seqs_per_sec"],
        "at_70pct_load": {"rate_requests_per_sec": 0.7 * len(reqs) / t_closed,
                          "p50_ms": loads[0.7]["all"].get("p50_ms"), "p99_ms": loads[0.7]["all"].get("p99_ms")},
        "plain_per_call_seqs_per_sec": plain,
        "served_vs_plain": cap["seqs_per_sec"] / plain if plain else None,
    }


def ism_explain_leg(sv, svl, coef, n=512):
    """Config 4: ISM (all 3 x 1000 substitutions) and GkmExplain hypothetical
    attributions of n x 1,000 bp sequences on the 72k-SV t=2 model."""
    import torch

    import gkmsvm_lite_b200 as gk
    import gkmsvm_lite_b200.synthetic as syn

    model = gk.GkmSVM(sv, coef, 0.0, "gkm_esttrunc", PARAMS_T2, sv_lengths=svl).cuda()
    x = syn.config4_queries()[:n]
    out = {"workload": f"config4: {n} x 1,000 bp, 72,000-SV t=2 model"}
    for name, fn in (("ism", lambda xs: gk.ism(model, xs)),
                     ("explain_hypothetical", lambda xs: gk.gkmexplain(model, xs, mode="hypothetical",
                                                                      batch_size=n))):
        fn(x[:8])
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn(x)
        b.record()
        torch.cuda.synchronize()
        out[name] = {"value": n / (a.elapsed_time(b) / 1e3), "unit": "seqs/sec"}
    # the explain table's own build (1 + 4 + 4l Walsh-Hadamard transforms), V already built
    from gkmsvm_lite_b200 import explain as ex

    model._explain_tables.clear()
    torch.cuda.synchronize()
    a.record()
    ex._explain_table(model, 1 << 62, False, model._device)
    b.record()
    torch.cuda.synchronize()
    n_lmers = 4 ** model.kernel.base.l
    ms = a.elapsed_time(b)
    out["explain_table_build"] = {"ms": ms, "table_bytes": n_lmers * 4 * model.kernel.base.l * 8,
                                  "wht_pass_bytes_total": 2 * 8 * n_lmers * (5 + 4 * model.kernel.base.l)
                                  * model.kernel.base.l}
    # the per-SV pair loop (gkm_explain_pairs) on the same model and rows, the
    # form models the l-mer path does not take use (l > 12, no index)
    nps = 16
    model.use_lmer_index = False
    model.use_explain_table = False
    gk.gkmexplain(model, x[:2], mode="hypothetical")
    torch.cuda.synchronize()
    a.record()
    gk.gkmexplain(model, x[:nps], mode="hypothetical", batch_size=nps)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    fw, _, cy = model._sv_packed()
    pairs = nps * (x.shape[1] - model.kernel.base.l + 1) * int(cy.sum().item()) * 2
    out["explain_per_sv"] = {"value": nps / (ms / 1e3), "unit": "seqs/sec", "rows": nps,
                             "window_pairs_per_s": pairs / (ms / 1e3)}
    model.use_lmer_index = True
    model.use_explain_table = "auto"
    out["ism_path"] = "l-mer table + fused mutant self-kernels" if model._lmer_table is not None else "index"
    out["ism_index_t5"] = ism_index_leg(sv, svl, coef)
    out["explain_path"] = "explain table (GPU Walsh-Hadamard build, cached)" if model._explain_tables else "l-mer neighbours"
    return out


def ism_index_leg(sv, svl, coef, rows=32, L=1000, seed=13):
    """ISM through the l-mer index (the path RBF models take: mutant window
    sets over the persistent index query) on the 72k-SV t=5 model of the
    serving mix: rows x L bp through ism() and through the graph-captured
    BatchedIsm (second call, graphs captured)."""
    import torch

    import gkmsvm_lite_b200 as gk
    import gkmsvm_lite_b200.synthetic as syn
    from gkmsvm_lite_b200.batch import BatchedIsm

    model = gk.GkmSVM(sv, coef, 0.0, "wgkmrbf", {"L": 11, "k": 7, "d": 3, "gamma": 1.0}, sv_lengths=svl).cuda()
    x = syn.random_codes(np.random.default_rng(seed), rows, L)
    gk.ism(model, x)  # the same shape: workspace and caches allocated
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {"workload": f"{rows} x {L} bp, 72,000-SV t=5 wgkmrbf gamma=1 model (index path)"}
    torch.cuda.synchronize()
    a.record()
    want = gk.ism(model, x)
    b.record()
    torch.cuda.synchronize()
    out["ism"] = {"value": rows / (a.elapsed_time(b) / 1e3), "unit": "seqs/sec", "ms_per_row": a.elapsed_time(b) / rows}
    runner = BatchedIsm(model)
    xd = torch.from_numpy(x).cuda()
    for _ in range(2):  # the bucket's eager first use, then its capture
        runner(xd)
    torch.cuda.synchronize()
    a.record()
    got = runner(xd)
    b.record()
    torch.cuda.synchronize()
    out["batched_ism"] = {"value": rows / (a.elapsed_time(b) / 1e3), "unit": "seqs/sec",
                          "ms_per_row": a.elapsed_time(b) / rows,
                          "max_abs_diff_vs_ism": float((got - want).abs().max().item())}
    single = x[:1]
    gk.ism(model, single)
    torch.cuda.synchronize()
    a.record()
    gk.ism(model, single)
    b.record()
    torch.cuda.synchronize()
    out["single_row_ms"] = a.elapsed_time(b)
    return out


def deltasvm_leg(sv, svl, coef):
    """to_deltasvm weights of the 72k-SV models: t=2 off the exact l-mer table
    (built in the timed call), t=3 by scoring all 2.1M canonical 11-mers."""
    import torch

    import gkmsvm_lite_b200 as gk

    out = {}
    for name, kt, params in (("t2_table", "gkm_esttrunc", PARAMS_T2), ("t3_scored", "gkmrbf", PARAMS_T3)):
        model = gk.GkmSVM(sv, coef, 0.0, kt, params, sv_lengths=svl).cuda()
        model._sv_diag()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        w = model.to_deltasvm(device="cuda").weights
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        out[name] = {"s": dt, "lmers_per_s": w.numel() / dt, "weights": int(w.numel())}
        del model
    return out


def explain_pairs_leg(n_sv=2000, sv_len=300, rows=100, row_len=300, seed=9):
    """GkmExplain through the per-SV pair loop on an l = 13 model (no l-mer
    index or table exists past l = 12): n_sv random SVs, rows random queries."""
    import numpy as np
    import torch

    import gkmsvm_lite_b200 as gk

    rng = np.random.default_rng(seed)
    sv = rng.integers(0, 4, (n_sv, sv_len), dtype=np.uint8)
    x = rng.integers(0, 4, (rows, row_len), dtype=np.uint8)
    params = {"L": 13, "k": 8, "d": 3}
    model = gk.GkmSVM(sv, rng.normal(0.0, 0.1, n_sv), 0.0, "gkm_esttrunc", params).cuda()
    gk.gkmexplain(model, x[:2], mode="hypothetical")
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    gk.gkmexplain(model, x, mode="hypothetical", batch_size=rows)
    b.record()
    torch.cuda.synchronize()
    s = a.elapsed_time(b) / 1e3
    l = params["L"]
    pairs = rows * (row_len - l + 1) * n_sv * 2 * (sv_len - l + 1)
    return {"workload": f"l=13 k=8 d=3, {n_sv} SVs x {sv_len} bp, {rows} rows x {row_len} bp",
            "value": rows / s, "unit": "seqs/sec", "window_pairs_per_s": pairs / s}


ENCODE_MODEL = os.path.join(ROOT, "tests", "golden", "lsgkm", "encode_ENCFF579AOX.model.txt.gz")
# the reference's published steady-state seq/s for this shape (1,000 x 300 bp,
# 72,145 SVs), L40S / A100
ENCODE_PUBLISHED = {"t2": {"L40S": 45682, "A100": 35160}, "t3": {"L40S": 2202, "A100": 2261}}


def encode_leg(n=1000, L=300, seed=6):
    """The reference's scoring-throughput benchmark shape (its
    benchmarks/throughput_sweep.py): the 72,145-SV ENCODE model read by the
    native LS-GKM parser, as t2 (the file's gkm_esttrunc: the path "auto"
    picks for this call, and the l-mer table, the path the reference's own
    run took) and with the same SVs as gkmrbf gamma=1 (t3, the l-mer index);
    n synthetic L bp queries as host one-hot [n, 4, L]; model(X) read back to
    the host, timed on the first call (SV caches built) and the second."""
    import torch

    import gkmsvm_lite_b200 as gk
    import gkmsvm_lite_b200.synthetic as syn

    codes = syn.random_codes(np.random.default_rng(seed), n, L)
    X = np.eye(4, dtype=np.float32)[codes].transpose(0, 2, 1).copy()
    t0 = time.perf_counter()
    base = gk.load_lsgkm_model(ENCODE_MODEL)
    load_s = time.perf_counter() - t0
    # a small model warms the library and the allocator, as the reference's
    # benchmark warms its kernels
    gk.GkmSVM(base.support_sequences[:600], base.coefficients[:600], base.bias, "gkm_esttrunc",
              base.kernel_params).cuda()(X[:32]).cpu()
    out = {"workload": f"72,145-SV ENCODE model (ENCFF579AOX, l=11 k=7 d=3), {n} synthetic {L} bp one-hot queries",
           "model_load_s": load_s, "published_seqs_per_sec": ENCODE_PUBLISHED}
    for name, kt, extra, table in (("t2", "gkm_esttrunc", {}, "auto"), ("t2_table", "gkm_esttrunc", {}, True),
                                   ("t3", "gkmrbf", {"gamma": 1.0}, "auto")):
        m = gk.GkmSVM(base.support_sequences, base.coefficients, base.bias, kt, {**base.kernel_params, **extra},
                      sv_lengths=base.sv_lengths).cuda()
        m.use_lmer_table = table
        times = []
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            m(X).cpu()
            times.append(time.perf_counter() - t0)
        path = "l-mer table" if m._lmer_table is not None and m._lmer_table is not False else "l-mer index"
        pub = ENCODE_PUBLISHED[name.split("_")[0]]["L40S"]
        out[name] = {"first_s": times[0], "steady_s": min(times[1:]), "seqs_per_sec": n / min(times[1:]),
                     "path": path, "vs_L40S": n / min(times[1:]) / pub}
        del m
    return out


def weighted_leg(n=20000, steps=3):
    """Batched scoring with the weighted kernel of the serving mix: the 72k-SV
    config-3 SVs as t=5 wgkmrbf gamma=1 (M=50, H=50), n config-3 queries,
    through BatchedScorer; its index query counts in 32-bit shared counters
    (window weights up to 50 x 50 per pair), so an SV tile holds 12,000 SVs (6
    tiles, against 3 unweighted).  Roofline bytes: lookups x 8 B + hits x
    (4 B id + 1 B weight) + 12 B per window."""
    import torch

    import gkmsvm_lite_b200 as gk
    import gkmsvm_lite_b200.synthetic as syn
    from gkmsvm_lite_b200 import engine
    from gkmsvm_lite_b200.batch import BatchedScorer

    sv, svl, coef = syn.config3_model()
    xq, xl, _ = syn.config3_queries(n=n)
    m = gk.GkmSVM(sv, coef, 0.0, "wgkmrbf", {"L": 11, "k": 7, "d": 3, "gamma": 1.0}, sv_lengths=svl).cuda()
    index = m._sv_index()
    x, ln = torch.from_numpy(xq).cuda(), torch.from_numpy(xl).cuda()
    sc = BatchedScorer(m)
    for _ in range(3):  # eager, capture, replay
        sc.score(x, ln)
    torch.cuda.synchronize()
    ev = []
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        e = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        sc.score(x, ln, events=e, check=False)
        ev.append(e)
    b.record()
    torch.cuda.synchronize()
    sc.check_flags()
    step_ms = a.elapsed_time(b) / steps
    query_ms = float(np.mean([e0.elapsed_time(e1) for e0, e1 in ev]))
    fwd, _, counts = engine.pack(m._spec(), x, ln)
    n_win = int(counts.sum().item())
    look, hits_s = index.count(fwd[:4096], counts[:4096])
    hits = hits_s * n_win / max(int(counts[:4096].sum().item()), 1)
    alg = n_win * int(index.masks.numel()) * 8 + hits * 5 + 12 * n_win
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    return {"workload": f"config-3 SVs as t=5 wgkmrbf gamma=1, {n} config-3 queries, batched",
            "value": n / (step_ms / 1e3), "unit": "seqs/sec", "tiles": index.tiles, "tile_svs": index.tile_svs,
            "query_ms": query_ms, "roofline": {"achieved_GBs": alg / (query_ms / 1e3) / 1e9, "peak_GBs": peak,
                                               "frac": alg / (query_ms / 1e3) / 1e9 / peak, "hits": hits}}


def masked_join_hits(sv_windows: int, l: int, j: int, n_masks: int, q: float = 0.2564) -> float:
    """Expected exact-match hits per query window of the reference's masked
    join (kernels/masked.py:45-69, 265-310) with n_masks masks keeping j of l
    positions, over sv_windows indexed windows of i.i.d. bases with per-position
    match probability q (GC 0.42: 0.29^2 * 2 + 0.21^2 * 2)."""
    return n_masks * sv_windows * q**j


def pairwise_forms_leg(n_small=4000, rows=128, seed=12):
    """The shapes where the reference would take its masked join: t=0 gkm_cnt
    l=11 k=7 with no d (dmax 4, 31,714 neighbour masks).  At the 72k-SV config-3
    model the index applies (11.7 indexed windows per l-mer lift its limit to
    32,768 neighbours, as the reference's kernels/lmer_index.py:97-109); with
    n_small SVs of 300 bp the reference's rule would not, and the index is
    taken where its measured cost is below the all-pairs forms'
    (kernels.index_cost_below_pairs); the same rows also through the autotuned
    all-pairs form (the tensor-core product or the warp join), which scores
    every window pair.  Beside each: the masked join's own work, 330 masks of
    7 kept positions (its plan for h(m) = C(l - m, 7) is the single level j = 7)."""
    import torch

    import gkmsvm_lite_b200 as gk
    import gkmsvm_lite_b200.synthetic as syn
    from gkmsvm_lite_b200 import engine
    from math import comb

    params = {"L": 11, "k": 7}
    out = {"kernel": "t=0 gkm_cnt l=11 k=7 (no d: dmax 4, 31,714 neighbours)"}
    sv, svl, coef = syn.config3_model()
    xq, xl, _ = syn.config3_queries(n=2000)
    rowsel = np.arange(rows)
    L = int(xl[rowsel].max())
    cases = [("config3_72k", sv, svl, coef)]
    rng = np.random.default_rng(seed)
    small = syn.random_codes(rng, n_small, 300)
    cases.append((f"{n_small}_svs_300bp", small, None, rng.normal(0, 0.1, n_small)))
    cases.append((f"{n_small}_svs_300bp_all_pairs", small, None, cases[1][3]))
    for name, s_codes, s_len, s_coef in cases:
        m = gk.GkmSVM(s_codes, s_coef, 0.0, "gkm_cnt", params, sv_lengths=s_len).cuda()
        m.use_lmer_table = False
        m.use_lmer_index = not name.endswith("all_pairs")
        nwin = m._n_sv_windows()
        path = "index" if m._sv_index() is not None else "all-pairs (autotuned)"
        m(xq[rowsel, :L], lengths=xl[rowsel])  # builds the SV caches, tunes the pairwise form
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        m(xq[rowsel, :L], lengths=xl[rowsel])
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        qwin = int(np.clip(xl[rowsel] - 10, 0, None).sum())
        out[name] = {"path": path, "sv_windows": nwin, "query_windows": qwin, "ms": ms,
                     "seqs_per_sec": rows / (ms / 1e3),
                     "window_pairs_per_query_window": nwin,
                     "masked_join_hits_per_query_window": masked_join_hits(nwin, 11, 7, comb(11, 7)),
                     "pairwise_tuned": {str(k): v for k, v in engine.PAIRWISE_TUNED.items()}}
        del m
    return out


def gram_leg(n=4000, forms=("index", "dense", "join")):
    """Config 2: the normalised symmetric Gram matrix of n sequences (lengths
    log-uniform in 100..1000 bp), t=4 wgkm l=11 k=7 d=3, through
    gkmsvm_lite_b200.compute_gram (host codes in, host matrix out); beside it
    the raw pairwise kernel K_raw [n, n] of each device form on the same packed
    windows, with its pair count: the l-mer index (lookups and hits), the
    tensor-core one-hot product and the warp join (every window pair)."""
    import torch

    import gkmsvm_lite_b200 as gk
    import gkmsvm_lite_b200.synthetic as syn
    from gkmsvm_lite_b200 import engine

    x, xl = syn.config2(n=n)
    k = gk.CenterWeightedGkmKernel(11, 7, d=3)
    gk.compute_gram(k, x[:64], lengths=xl[:64])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    gk.compute_gram(k, x, lengths=xl)
    e2e = time.perf_counter() - t0
    dev = torch.device("cuda", torch.cuda.current_device())
    spec = engine.Spec(k.base, dev)
    bx, rx, cx = engine.pack(spec, torch.from_numpy(x).to(dev), xl)
    n_win = int(cx.sum().item())
    pairs = n_win * 2 * n_win
    out = {"workload": f"config2: {n} sequences 100-1000 bp log-uniform, t=4 wgkm l=11 k=7 d=3",
           "compute_gram_s": e2e, "compute_gram_path": "index" if k.base.index_applies(2 * n_win) else "pairwise",
           "windows": n_win, "window_pairs": pairs, "raw_ms": {}}
    ref = None
    for form in forms:
        if form == "index":
            ix = engine.DeviceIndex(spec, bx, rx, cx, engine.masks_tensor(k.base, dev))
            fn = lambda: ix.pairwise(bx, cx)[0]
        elif form == "dense":
            if not engine.dense_applies(spec):
                continue
            fn = lambda: engine.dense_pairwise(spec, bx, cx, bx, rx, cx, check=False)[0]
        else:
            fn = lambda: engine.join_pairwise(spec, bx, cx, bx, rx, cx)[0]
        if form == "dense":  # warm-up call reads its error flag back
            engine.dense_pairwise(spec, bx, cx, bx, rx, cx)
        else:
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        r = fn()
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        same = None
        if ref is None:
            ref = r
        else:
            same = bool(torch.equal(r, ref))
        out["raw_ms"][form] = {"ms": ms, "Gpairs_per_s": pairs / ms / 1e6, "identical_to_first": same}
        if form == "index":
            ix.close()
    # the form the pairwise autotuner picks for this shape (its first call
    # times both on a 64 x 4,096 sample)
    engine.PAIRWISE_TUNED.clear()
    engine.choose_pairwise(spec, bx, cx, bx, rx, cx)
    out["pairwise_autotuned"] = {str(key): form for key, form in engine.PAIRWISE_TUNED.items()}
    return out


def training_leg(n=4000, seed=5):
    """SMO C-SVC training (the reference's column-cached solver) on the config-2
    sequences (n, 100..1,000 bp log-uniform), t=4 wgkm l=11 k=7 d=3, C=1,
    tol=1e-3: a fixed 10 bp motif planted at a random position in half of the
    sequences makes the positive class.  Columns from the GPU l-mer index,
    solver on the host."""
    import torch

    import gkmsvm_lite_b200 as gk
    import gkmsvm_lite_b200.synthetic as syn
    from gkmsvm_lite_b200.solver import last_solve_stats

    x, xl = syn.config2(n=n)
    rng = np.random.default_rng(seed)
    motif = rng.integers(0, 4, 10).astype(np.uint8)
    y = np.where(rng.random(n) < 0.5, 1.0, -1.0)
    for i in np.flatnonzero(y > 0):
        p = rng.integers(0, max(1, int(xl[i]) - 10))
        x[i, p:p + 10] = motif
    k = gk.CenterWeightedGkmKernel(11, 7, d=3)
    gk.smo_solve(k, x[:64], y[:64], lengths=xl[:64])  # warm-up: library, graphs, allocator
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    coef, bias = gk.smo_solve(k, x, y, C=1.0, tol=1e-3, lengths=xl)
    dt = time.perf_counter() - t0
    st = last_solve_stats()
    # training accuracy from the Gram matrix (outside the timed region)
    acc = float((np.sign(gk.compute_gram(k, x, lengths=xl) @ coef + bias) == y).mean())
    return {"workload": f"config2 sequences: {n} x 100-1000 bp, t=4 wgkm l=11 k=7 d=3, C=1, tol=1e-3, "
                        "planted-motif labels",
            "train_s": dt, "iterations": st.get("iterations"), "column_calls": st.get("calls"),
            "columns": st.get("columns"), "support_vectors": int((np.abs(coef) > 0).sum()),
            "train_accuracy": acc}


def run_b200(args):
    import torch

    import gkmsvm_lite_b200 as gk
    import gkmsvm_lite_b200.synthetic as syn
    from gkmsvm_lite_b200 import engine

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)

    sv, svl, coef = syn.config3_model()
    xq, xl, nmask = syn.config3_queries(seed=shard_seed(rank), n=args.queries)
    model = gk.GkmSVM(sv, coef, 0.0, "gkmrbf", PARAMS_T3, sv_lengths=svl).cuda()
    model.use_lmer_table = False
    t0 = time.perf_counter()
    index = model._sv_index()
    torch.cuda.synchronize()
    index_build_s = time.perf_counter() - t0
    spec = model._spec()
    x_dev = torch.from_numpy(xq).to(dev)
    l_dev = torch.from_numpy(xl).to(dev)
    B = x_dev.shape[0]

    from gkmsvm_lite_b200.batch import BatchedScorer

    scorer = BatchedScorer(model)
    query_ev = []
    last = {}

    def step():
        e = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        last["scores"] = scorer.score(x_dev, l_dev, events=e, check=False)
        query_ev.append(e)

    def warm():
        for _ in range(args.warmup):
            step()
        scorer.check_flags()
        query_ev.clear()

    warm()
    before = index.counters()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def stop():
        ev1.record()
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1) / 1e3

    with Clocks(local) as clocks:
        elapsed = timed_region(step, args.steps, 0, dist=dist, sync=torch.cuda.synchronize,
                               clock=(ev0.record, stop))
    elapsed, units, value = job_throughput(elapsed, args.steps * B, dist=dist, device=dev)
    if dist is not None:
        dist.barrier()
    after = index.counters()
    torch.cuda.synchronize()
    # 16-bit counter carries never outgrew a block's log in the timed steps
    counts_exact = int(after[0]) == int(before[0]) and int(after[1]) == int(before[1])
    per_step = elapsed / args.steps
    query_ms = float(np.mean([a.elapsed_time(b) for a, b in query_ev]))
    timed_scores = last["scores"].cpu().numpy().copy()

    result = None
    if rank == 0:
        # roofline of the dominant kernel: the fused index query (algorithmic
        # bytes: lookups x 8 B (a bucket's two offsets) + hits x 4 B (an SV id)
        # + 12 B per query window; hits counted exactly on the first queries
        # and scaled by windows).  The index stores 2-byte ids (tiles of <=
        # 65,536 SVs, unweighted): that count is reported beside it.
        fwd, rc, counts = engine.pack(spec, x_dev, l_dev)
        n_win = int(counts.sum().item())
        nsample = min(B, 4096)
        look_s, hits_s = index.count(fwd[:nsample], counts[:nsample])
        win_s = int(counts[:nsample].sum().item())
        hits = hits_s * n_win / max(win_s, 1)
        lookups = n_win * int(index.masks.numel())
        entry_bytes = 2 if (not spec.base.weighted and index.tile_svs <= 65536) else 4
        alg_bytes = lookups * 8 + hits * 4 + 12 * n_win
        stored_bytes = lookups * 8 + hits * entry_bytes + 12 * n_win
        # DRAM traffic of the launch: ncu's dram__bytes_read.sum +
        # dram__bytes_write.sum on a 2,000-query launch of this workload
        # (NCU_INDEX_QUERY; the SV index stays in L2), scaled by queries
        traffic = NCU_INDEX_QUERY["dram_bytes"] * B / 2000
        achieved = alg_bytes / (query_ms / 1e3) / 1e9
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except OSError:
            pass
        peak = float(peaks.get("hbm_gbs", 6650.0))
        result = {
            "metric": METRIC, "value": value, "unit": "seqs/sec", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": per_step * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32 counts + f64 epilogue", "data": "synthetic",
            "config": job_config(B, world),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "traffic_source": "ncu dram bytes of a 2,000-query launch, scaled by queries",
                         "kernel": "index_query (fused SV-tile query + RBF + alpha reduce)",
                         "alg_bytes_per_launch": alg_bytes, "hits": hits, "lookups": lookups,
                         "frac_stored_entry_bytes": stored_bytes / (query_ms / 1e3) / 1e9 / peak,
                         "binding_unit": "the L1 data pipe (shared adds, bucket and entry gathers), "
                                         "instruction issue and L2 latency (90 % L2 hits; HBM carries "
                                         "~3 % of its bandwidth: not what binds it)",
                         "ncu_small_case": NCU_INDEX_QUERY,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback 6.65 TB/s"},
            "stages_ms": {"prep (pack, self-kernels, order)": per_step * 1e3 - query_ms,
                          "index_query + finish": query_ms},
            "form": "batched: CUDA-graph replay of pack + self-kernel + persistent work-queue index query",
            "index": {"build_s": index_build_s, "entries": index.entries, "tiles": index.tiles,
                      "tile_svs": index.tile_svs, "device_MB": index.nbytes / 1e6},
            "counts_exact": counts_exact,
            "gpu_launches": args.steps * 4,  # pack, self_kernel, index_query, finish_scores per step
            "clocks": clocks.summary(),
        }

    # e2e through the public API with host buffers, and the plain per-call form
    if not args.no_extras:
        if dist is not None:
            dist.barrier()
        nq = min(B, 20000)
        xh, lh = xq[:nq, : int(xl[:nq].max())], xl[:nq]
        model(xh[:64], lengths=lh[:64])
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        host_scores = model(xh, lengths=lh).cpu().numpy()
        b.record()
        torch.cuda.synchronize()
        e2e_s, e2e_n, e2e_v = job_throughput(a.elapsed_time(b) / 1e3, nq, dist=dist, device=dev)
        plain_n = min(nq, 5000)
        a.record()
        for s in range(0, plain_n, 1000):
            model(xh[s:s + 1000], lengths=lh[s:s + 1000]).cpu()
        b.record()
        torch.cuda.synchronize()
        plain_s = a.elapsed_time(b) / 1e3
        if rank == 0:
            result["e2e"] = {"value": e2e_v, "unit": "seqs/sec", "h2d_bytes_per_step": int(xh.nbytes + lh.nbytes),
                             "d2h_bytes_per_step": int(host_scores.nbytes), "queries_per_rank": nq}
            result["plain_per_call"] = {"value": plain_n / plain_s, "unit": "seqs/sec", "calls_of": 1000,
                                        "note": "model(x) per 1,000-query call with host inputs and output"}
            result["batched_vs_plain"] = value / world / result["plain_per_call"]["value"]
            # t=2 on the same SVs through the exact l-mer table
            m2 = gk.GkmSVM(sv, coef, 0.0, "gkm_esttrunc", PARAMS_T2, sv_lengths=svl).cuda()
            m2.use_lmer_table = True
            tb0 = time.perf_counter()
            m2._build_lmer_table()
            torch.cuda.synchronize()
            tb = time.perf_counter() - tb0
            for _ in range(2):
                m2._score_codes(x_dev, l_dev)
            a.record()
            for _ in range(3):
                m2._score_codes(x_dev, l_dev)
            b.record()
            torch.cuda.synchronize()
            result["t2_table"] = {"value": 3 * B / (a.elapsed_time(b) / 1e3), "unit": "seqs/sec",
                                  "table_build_s": tb}
            del m2
            if world == 1:
                result["serving"] = serving_leg(sv, svl, coef)
                result["ism_explain"] = ism_explain_leg(sv, svl, coef)
                result["deltasvm"] = deltasvm_leg(sv, svl, coef)
                result["gram"] = gram_leg(args.gram_n)
                result["encode"] = encode_leg()
                result["pairwise_forms"] = pairwise_forms_leg()
                result["weighted_t5"] = weighted_leg()
                result["training"] = training_leg(args.gram_n)
    if rank == 0:
        # the oracle re-scores rows of the timed batch (the longest, the most
        # N-heavy, random others) and, at N=1, times the reference's CPU path
        port = PortBaseline(sv, svl, coef)
        rows = parity_rows(xl, nmask)
        want = port.scores(xq, xl, rows)
        got = timed_scores[rows]
        rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-300)
        result["parity"] = {"rows": int(len(rows)), "of": "the last timed step's scores",
                            "max_rel_err": float(rel.max()), "max_abs_err": float(np.abs(got - want).max()),
                            "rtol": 1e-9, "atol": 1e-12,
                            "pass": bool(np.all(np.abs(got - want) <= 1e-12 + 1e-9 * np.abs(want))),
                            "longest_row_bp": int(xl[rows].max())}
        if world == 1 and not args.no_extras:
            sample = np.arange(REF_ROWS_PER_STEP, 2 * REF_ROWS_PER_STEP)
            port.time_rows(xq, xl, np.arange(8))
            sec = port.time_rows(xq, xl, sample)
            result["cpu_baseline"] = {"value": len(sample) / sec, "unit": "seqs/sec", "cores": port.threads,
                                      "kind": "port", "seconds": sec,
                                      "sample": f"{len(sample)} consecutive config-3 queries (rows "
                                                f"{sample[0]}..{sample[-1]} of the timed batch), steady state "
                                                f"(SV index and self-kernels built)"}
        result.setdefault("e2e", None)
        print(json.dumps(result), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    cmd = launch_command(args, os.environ)
    if cmd is not None:
        return subprocess.call(cmd)
    if args.impl == "reference":
        return run_reference(args)
    if args.leg == "gram":
        print(json.dumps(gram_leg(args.gram_n)), flush=True)
        return 0
    if args.leg == "train":
        print(json.dumps(training_leg(args.gram_n)), flush=True)
        return 0
    if args.leg == "serve":
        import gkmsvm_lite_b200.synthetic as syn

        print(json.dumps(serving_leg(*syn.config3_model())), flush=True)
        return 0
    if args.leg == "weighted":
        print(json.dumps(weighted_leg(args.weighted_n)), flush=True)
        return 0
    if args.leg == "ism-index":
        import gkmsvm_lite_b200.synthetic as syn

        print(json.dumps(ism_index_leg(*syn.config3_model(), rows=args.ism_rows)), flush=True)
        return 0
    if args.leg == "pairwise-forms":
        print(json.dumps(pairwise_forms_leg()), flush=True)
        return 0
    if args.leg == "encode":
        print(json.dumps(encode_leg()), flush=True)
        return 0
    if args.leg == "explain-pairs":
        print(json.dumps(explain_pairs_leg()), flush=True)
        return 0
    if args.leg == "explain":
        import gkmsvm_lite_b200.synthetic as syn

        sv, svl, coef = syn.config3_model()
        print(json.dumps({**ism_explain_leg(sv, svl, coef), "deltasvm": deltasvm_leg(sv, svl, coef)}), flush=True)
        return 0
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
