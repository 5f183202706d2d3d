"""Benchmark: DB residues x queries / s of blastp's two-hit word finding +
ungapped X-drop extension on a B200 (one query of a search counts once,
whatever its length; `residue_pairs_per_s` beside it weights each query by
its length: DB residues x query residues / s).

Workload (default): one 500-aa query vs 1,000,000 synthetic subjects
(~360M residues, HBM-resident), BLOSUM62, word 3, T 11, window 40,
x-drop 16 raw, cutoff 41 raw.  One step = one search of the query over the
whole database through the engine (scan kernel + ordering of the HSP set +
the count read-back).  The database (~0.36 GB) is larger than L2 (126 MB), so
no explicit flush is needed between steps.

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

With N > 1 (launched by torch.distributed.run) each rank scans its own
1,000,000-subject shard (weak scaling, no collective on the data path); the
timed region is bracketed by barriers and the max over ranks is reported.
`--impl reference` times the reference's own kernel code on the host cores:
gpu_blastp_kernel.cu host-compiled into oracle/_ref (one POSIX thread per
CUDA thread; its database layout built beforehand, as the reference's
database writer does), or, where oracle/_ref was not built, the oracle port.

Beside the headline the line carries: the 300-aa query against 10,000
subjects (the size the plain form's roofline target is quoted on), the scan
kernel's issue-rate roofline and its word-hit and extension rates, the
256-query batched workload with every query's result checked against its
plain search (device digests), and the serving loop with a sample of served
results checked the same way.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "blastp-cuda_b200"))
sys.path.insert(0, ROOT)

METRIC = "DB residues x queries / s (two-hit + ungapped X-drop, bit-exact HSPs)"
UNIT = "residues*queries/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--subjects", type=int, default=1_000_000)
    ap.add_argument("--qlen", type=int, default=500)
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--config1", type=int, default=1, help="also time one 300-aa query vs 10,000 subjects")
    ap.add_argument("--config1-reps", type=int, default=100)
    ap.add_argument("--gapped", type=int, default=1, help="also time the gapped stage on the headline search")
    ap.add_argument("--cpu-seconds", type=float, default=3.0, help="wall-clock budget of the CPU baseline sample")
    ap.add_argument("--batched", type=int, default=1, help="also measure the batched workload (1 GPU runs only)")
    ap.add_argument("--batch-subjects", type=int, default=2_000_000)
    ap.add_argument("--batch-queries", type=int, default=256)
    ap.add_argument("--batch-reps", type=int, default=1)
    ap.add_argument("--batch-autotune", type=int, default=1, help="run the autotuner (0: skip it)")
    ap.add_argument("--serve", type=int, default=1, help="also measure the serving loop (1 GPU runs only)")
    ap.add_argument("--serve-subjects", type=int, default=5_000_000)
    ap.add_argument("--serve-requests", type=int, default=256)
    ap.add_argument("--serve-rate", type=float, default=1000.0, help="offered load, queries/s (Poisson)")
    ap.add_argument("--serve-sustained-requests", type=int, default=384,
                    help="requests of each run at 80 %% of the measured capacity")
    ap.add_argument("--serve-check", type=int, default=32, help="served requests checked against plain searches")
    ap.add_argument("--serve-rate-high", type=float, default=5000.0, help="second offered load (0: skip)")
    ap.add_argument("--serve-lanes", type=int, default=1)
    ap.add_argument("--serve-depth", type=int, default=4, help="batches queued per lane")
    ap.add_argument("--serve-batch", type=int, default=1, help="queries per batch")
    ap.add_argument("--serve-max-wait-ms", type=int, default=250,
                    help="the wait after which a request goes first, in the capped preemptive run")
    ap.add_argument("--serve-segments", type=int, default=8,
                    help="subject ranges per request in the preemptive run (<= 1: no preemptive run)")
    ap.add_argument("--serve-schedule", default="dynamic", choices=["dynamic", "learned"],
                    help="item schedule of the served batches")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Ranks:
    """One process per GPU, as torchrun starts them: the process group, the
    barriers and the max-over-ranks reduction of the timing.  The GPU path
    uses NCCL and CUDA tensors; tests drive the same code with gloo on CPU."""

    def __init__(self, backend="nccl", device="cuda", timeout_s=300):
        import torch
        self.torch = torch
        self.rank, self.world, self.local = dist_env()
        self.device = device
        if self.world > 1:
            import datetime
            torch.distributed.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))

    def barrier(self, sync=None):
        if self.world > 1:
            self.torch.distributed.barrier()
        if sync:
            sync()

    def max(self, x):
        t = self.torch.tensor([float(x)], dtype=self.torch.float64, device=self.device)
        if self.world > 1:
            self.torch.distributed.all_reduce(t, op=self.torch.distributed.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.torch.distributed.destroy_process_group()


class EventTimer:
    """CUDA events on the stream the work is launched on."""

    def __init__(self, torch, stream):
        self.stream = stream
        self.e0 = torch.cuda.Event(enable_timing=True)
        self.e1 = torch.cuda.Event(enable_timing=True)

    def start(self):
        self.e0.record(self.stream)

    def mark(self):
        self.e1.record(self.stream)

    def ms(self):
        return self.e0.elapsed_time(self.e1)


class WallTimer:
    def start(self):
        self.t0 = time.perf_counter()

    def mark(self):
        self.t1 = time.perf_counter()

    def ms(self):
        return 1e3 * (self.t1 - self.t0)


def timed_steps(step, steps, warmup, ranks, timer, sync=None, during=None):
    """W untimed steps, a barrier, K timed steps between timer.start() and
    timer.mark(), a barrier (after which the device is idle), then the timed
    region's length as the max over ranks.  `during` (a context manager)
    brackets the timed steps (the clock sampler).  Returns (the steps'
    outputs, max ms, this rank's ms)."""
    import contextlib
    for _ in range(warmup):
        step()
    ranks.barrier(sync)
    outs = []
    with (during or contextlib.nullcontext()):
        timer.start()
        for _ in range(steps):
            outs.append(step())
        timer.mark()
        ranks.barrier(sync)
    local_ms = timer.ms()
    return outs, ranks.max(local_ms), local_ms


def load_workload(matrix, rank, n_subjects, qlen):
    from blastp_b200 import synth
    return synth.shape2(matrix, rep=rank, n_subjects=n_subjects, qlen=qlen)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.15)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.lines:
            return None
        sm, mx, reasons = [], 0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_per_residue(key):
    """A per-residue figure of the scan kernel (dram bytes, warp
    instructions) from the committed ncu summary
    (profiles/scan_kernel_q500_vs_1M.md), or None."""
    path = os.path.join(ROOT, "profiles", "scan_kernel_q500_vs_1M.md")
    try:
        for line in open(path):
            if line.startswith(key + ":"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


def reference_threads():
    """POSIX threads (= CUDA threads of one block) the reference kernel runs
    with on the host: a few per core, a multiple of 16 as its shared-memory
    layout requires."""
    n = 4 * (os.cpu_count() or 1)
    return max(64, min(1024, 16 * ((n + 15) // 16)))


def time_cpu_sample(matrix, q, res, off, prefer_reference=True):
    """One search of a sample on the host cores: the neighbour-word table
    build plus the reference's own kernel (oracle/_ref, kind "reference") --
    its kernel time alone, the interleaved layout being built beforehand as
    the reference's database writer does -- or else the oracle port (kind
    "port").  The reference requires length-sorted volumes
    (functions.cpp:433-438), so the sample is given to it sorted.
    Returns (seconds, kind, threads)."""
    import oracle
    from oracle import refkernel
    if prefer_reference and refkernel.available(2):
        t0 = time.perf_counter()
        table = oracle.build_table(q, matrix, 11)
        t_table = time.perf_counter() - t0
        tm = {}
        refkernel.two_hit(res, off, q, table, matrix, [(0, 16, 41)], slots=2, threads=reference_threads(),
                          timing=tm)
        return t_table + tm["kernel_s"], "reference", reference_threads()
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    table = oracle.build_table(q, matrix, 11)
    oracle.scan(res, off, q, table, matrix, [(0, 16, 41)], threads=threads)
    return time.perf_counter() - t0, "port", threads


def sorted_sample(w, n):
    """The first n subjects of a workload, sorted by length (ascending)."""
    off = w.db.offsets[:n + 1]
    lens = np.diff(off)
    order = np.argsort(lens, kind="stable")
    res = np.concatenate([w.db.residues[off[i]:off[i + 1]] for i in order]).astype(np.uint8)
    soff = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens[order], out=soff[1:])
    return res, soff


def cpu_baseline(matrix, w, budget_s):
    """The reference's kernel on the host cores (oracle/_ref; the oracle port
    where it was not built) on a bounded, length-sorted prefix of the same
    database, repeated until the budget is used; the port's rate on the same
    sample beside it."""
    q = w.queries[0]
    n = min(w.db.n_subjects, 100_000)
    res, off = sorted_sample(w, n)
    out = None
    for prefer in (True, False):
        done_res, busy, reps, t0 = 0, 0.0, 0, time.perf_counter()
        while True:
            dt, kind, threads = time_cpu_sample(matrix, q, res, off, prefer_reference=prefer)
            busy += dt
            done_res += int(off[-1])
            reps += 1
            if time.perf_counter() - t0 >= budget_s:
                break
        r = {"value": done_res / busy, "unit": UNIT, "cores": os.cpu_count() or 1, "threads": threads,
             "kind": kind, "residue_pairs_per_s": done_res * len(q) / busy,
             "sample": "first %d subjects (%d residues, sorted by length) x %d reps, query %d aa; "
                       "table build + %s" % (n, int(off[-1]), reps, len(q),
                                             "the reference's own kernel (gpu_blastp_kernel.cu host-compiled, "
                                             "one POSIX thread per CUDA thread)" if kind == "reference"
                                             else "the oracle port's scan on all host threads")}
        if out is None:
            out = r
            if kind != "reference":
                break
        else:
            out["port"] = {"value": r["value"], "threads": r["threads"],
                           "note": "the oracle's C restatement, tuned for CPUs, on the same sample"}
    return out


def run_config1(eng, matrix, args, torch, peak):
    """One 300-aa query against 10,000 subjects (3.6M residues, 3.6 MB): the
    workload the plain form's roofline target is quoted on.  Each search
    (scan + ordering pass + count read-back) is timed alone with CUDA events
    on the engine stream, L2 flushed before it by a 256 MB write; the scan
    kernel's own time comes from the engine's events around it."""
    from blastp_b200 import synth
    w = synth.shape1(matrix)
    db = eng.database(w.db.residues, w.db.offsets)
    qry = eng.query(w.queries[0])
    stream = torch.cuda.ExternalStream(eng.stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    search_ms, scan_ms = [], []
    launches0 = eng.launches
    for i in range(args.config1_reps + 5):
        flush.fill_(i & 0xff)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = eng.search(db, qry)
        e1.record(stream)
        r.wait()
        torch.cuda.synchronize()
        if i >= 5:
            search_ms.append(e0.elapsed_time(e1))
            scan_ms.append(eng.last_scan_ms)
        r.close()
    launches = (eng.launches - launches0) / (args.config1_reps + 5)
    res = eng.search(db, qry).fetch()
    qry.close()
    db.close()
    del flush
    n = w.db.n_subjects
    s_med = float(np.median(search_ms))
    k_med = float(np.median(scan_ms))
    alg = w.db.n_residues + 8 * (n + 1) + 12 * n
    return {"workload": w.name, "query_len": len(w.queries[0]), "subjects": n, "residues": w.db.n_residues,
            "reps": len(search_ms), "l2": "flushed before every search (256 MB write)",
            "search_us_median": 1e3 * s_med, "search_us_min": 1e3 * float(np.min(search_ms)),
            "scan_kernel_us_median": 1e3 * k_med,
            "overhead_us_median": 1e3 * (s_med - k_med),
            "launches_per_search": launches,
            "value": w.db.n_residues / (s_med / 1e3), "unit": UNIT,
            "scan_kernel_value": w.db.n_residues / (k_med / 1e3),
            "roofline": {"bound": "hbm", "algorithmic_bytes": alg, "achieved": alg / (k_med / 1e3) / 1e9,
                         "peak": peak, "unit": "GB/s", "frac": alg / (k_med / 1e3) / 1e9 / peak,
                         "hbm_floor_us": alg / (peak * 1e9) * 1e6},
            "hits": int(res.counters[:, 0].sum()), "extensions": int(res.counters[:, 2].sum()),
            "hsps": int(len(res.hsps))}


def run_gapped_stage(eng, db, qry, reps=5):
    """The gapped stage (bp_gapped_run) on the headline search's ungapped
    HSPs: device time of the stage (its own CUDA events), HSPs in and out."""
    import blastp_b200 as bp
    r = eng.search(db, qry)
    r.wait()
    times, g = [], None
    for _ in range(reps + 1):
        g = r.gapped(bp.gapped_params())
        times.append(g.ms)
    r.close()
    ms = float(np.median(times[1:]))
    n_ext = int(g.counters[:, 2].sum())
    return {"params": {"gap_open": 11, "gap_extend": 1, "x_dropoff": 38, "cutoff": 0},
            "ms": ms, "ungapped_hsps": int(g.counters[:, 0].sum()), "extensions": n_ext,
            "gapped_hsps": int(len(g.hsps)), "extensions_per_s": n_ext / (ms / 1e3),
            "subjects_with_hsps": int((g.counters[:, 0] > 0).sum())}


def run_batched(eng, matrix, args, torch):
    """256 queries (50-2000 aa) vs 2,000,000 subjects: the plain form (one
    search per query, back to back on the stream) against the batched
    persistent launch under each schedule, the autotuned configuration, and
    the learned schedule; device time with CUDA events on the engine stream."""
    from blastp_b200 import costmodel, synth
    from blastp_b200._lib import SCHED_COST_ORDER, SCHED_COSTS, SCHED_DYNAMIC, SCHED_NAMES, SCHED_STATIC
    w = synth.shape3(matrix, n_subjects=args.batch_subjects, n_queries=args.batch_queries)
    db = eng.database(w.db.residues, w.db.offsets)
    qs = [eng.query(q) for q in w.queries]
    qres = int(sum(len(q) for q in w.queries))
    work = float(w.db.n_residues) * len(qs)       # DB residues x queries
    pairs = float(w.db.n_residues) * qres         # DB residues x query residues
    stream = torch.cuda.ExternalStream(eng.stream)

    def timed(fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), out

    def plain_all():
        return [eng.search(db, q) for q in qs]

    for r in plain_all():                 # warm-up
        r.close()
    plain_ms, rs = timed(plain_all)
    plain_counts = []
    from blastp_b200._lib import lib
    for r in rs:
        r.wait()
        plain_counts.append(int(lib().bp_result_hsps(r.h)))
    # every query's plain result, as a device digest (counters, offsets, records)
    plain_digests = [r.digest() for r in rs]
    check_q = [0, len(qs) // 2, len(qs) - 1]
    plain_check = {i: eng.search(db, qs[i]).fetch() for i in check_q}
    for r in rs:
        r.close()
    out = {"workload": w.name, "queries": len(qs), "query_residues": qres, "subjects": w.db.n_subjects,
           "residues": w.db.n_residues, "unit": UNIT,
           "plain": {"ms": plain_ms, "value": work / (plain_ms / 1e3), "residue_pairs_per_s": pairs / (plain_ms / 1e3)}}
    model = costmodel.CostModel.load(eng)
    planted = 0.002
    variants = {"unpacked_dynamic": dict(chunk_residues=1 << 20, schedule=SCHED_DYNAMIC, pack_residues=0),
                "static": dict(chunk_residues=1 << 20, schedule=SCHED_STATIC),
                "dynamic": dict(chunk_residues=1 << 20, schedule=SCHED_DYNAMIC),
                "learned": dict(chunk_residues=1 << 20, schedule=SCHED_COSTS),
                "learned_order": dict(chunk_residues=1 << 20, schedule=SCHED_COST_ORDER),
                "plain_unpacked": dict(chunk_residues=1 << 20, schedule=SCHED_DYNAMIC, pack_residues=1024,
                                       plain_unpacked=1)}
    if args.batch_autotune:
        t0 = time.perf_counter()
        best, trials = eng.autotune(db, qs, model=model, planted_density=planted,
                                    sample_subjects=max(1, w.db.n_subjects // 16), reps=1)
        out["autotune"] = {"sample_subjects": max(1, w.db.n_subjects // 16), "seconds": time.perf_counter() - t0,
                           "best": dict(best, schedule=SCHED_NAMES[best["schedule"]]),
                           "trials": [[t["chunk_residues"], t["pack_residues"], SCHED_NAMES[t["schedule"]],
                                       t["max_warps"], t["plain_unpacked"], round(t["ms"], 3)] for t in trials],
                           "trial_fields": ["chunk_residues", "pack_residues", "schedule", "max_warps",
                                            "plain_unpacked", "ms"]}
        variants["autotuned"] = dict(best)
    identical = True
    identical_all = True
    res = {}
    for name, kw in variants.items():
        if kw["schedule"] in (SCHED_COSTS, SCHED_COST_ORDER):
            first = eng.plan_chunks(db, kw["chunk_residues"])
            kw["item_costs"] = eng.predict_costs(model, db, qs, first, planted)
        b = eng.search_batch(db, qs, **kw)
        b.wait()
        launches0 = eng.launches
        ms_runs = []
        for _ in range(max(1, args.batch_reps)):
            ms, _ = timed(lambda: b.run())
            b.wait()
            ms_runs.append(ms)
        ms = float(min(ms_runs))
        res[name] = {"ms": ms, "value": work / (ms / 1e3), "residue_pairs_per_s": pairs / (ms / 1e3),
                     "speedup_vs_plain": plain_ms / ms,
                     "chunk_residues": kw["chunk_residues"], "schedule": SCHED_NAMES[kw["schedule"]],
                     "pack_residues": kw.get("pack_residues", 512),
                     "max_warps": kw.get("max_warps", 0), "plain_unpacked": kw.get("plain_unpacked", 0),
                     "items": b.n_items,
                     "launches_per_run": (eng.launches - launches0) // max(1, args.batch_reps)}
        if b.n_hsps != sum(plain_counts):
            identical = False
        mismatched = [i for i in range(len(qs)) if b.digest(i) != plain_digests[i]]
        res[name]["queries_differing_from_plain"] = len(mismatched)
        if mismatched:
            identical_all = False
        for i in check_q:
            r = b.fetch(i)
            p = plain_check[i]
            if not (np.array_equal(r.counters, p.counters) and np.array_equal(r.hsp_off, p.hsp_off) and
                    np.array_equal(r.hsps_as_array(), p.hsps_as_array())):
                identical = False
        if name == "learned":
            # count error of the model on this workload, per (query, 64Ki-residue
            # chunk) -- the model's unit -- for the checked queries
            first = eng.plan_chunks(db, costmodel.TRAIN_CHUNK_RESIDUES)
            nc = len(first) - 1
            X = eng.batch_features(db, [qs[i] for i in check_q], first, planted)
            pred = model.predict_counts(X)
            true = np.concatenate([costmodel.chunk_sums(plain_check[i].counters, first)[:, [0, 2]]
                                   for i in check_q])
            res[name]["mlp_error"] = {"hits": costmodel.relative_error(pred[:, 0], true[:, 0]),
                                      "extensions": costmodel.relative_error(pred[:, 1], true[:, 1]),
                                      "items": int(len(true)), "queries": len(check_q), "chunks": nc}
        b.close()
    out["batched"] = res
    out["identical_to_plain"] = identical
    out["identical_to_plain_all"] = identical and identical_all
    out["parity_check"] = ("every variant: each of the %d queries' counters, CSR offsets and HSP records equal its "
                           "plain search's (128-bit device digests), total HSP count equal, and queries %s "
                           "compared field by field on the host" % (len(qs), check_q))
    out["hsps"] = int(sum(plain_counts))
    try:
        with open(os.path.join(os.path.dirname(costmodel.MODEL_PATH), "costmodel_b200_report.json")) as f:
            out["mlp_training"] = json.load(f)
    except OSError:
        pass
    for q in qs:
        q.close()
    db.close()
    return out


def run_serving(eng, matrix, args):
    """Poisson arrivals of log-normal queries (median 350, sigma 0.7, 20-4000
    aa) against a resident 5,000,000-subject database, served by one lane of
    queued batches (first come, first served at full width; the dynamic item
    schedule unless --serve-schedule learned); p50/p99 latency and throughput
    at the offered rates and at 80 % of the measured capacity."""
    from blastp_b200 import Server, costmodel, serving, synth
    from blastp_b200._lib import SCHED_COSTS, SCHED_DYNAMIC
    rng = np.random.default_rng(5000)
    lengths = synth.lognormal_lengths(rng, args.serve_subjects, 300, 0.6, 30, 5000)
    off = np.zeros(args.serve_subjects + 1, dtype=np.int64)
    np.cumsum(lengths, out=off[1:])
    res = synth.residues(rng, int(off[-1]))
    nres = int(off[-1])
    # the resident database comes from a database file, streamed into HBM
    # through pinned staging buffers; the direct upload from memory beside it
    import tempfile
    from blastp_b200 import write_database_file
    load = {}
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "serve.bpdb")
        t0 = time.perf_counter()
        write_database_file(path, res, off)
        load["write_s"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        mem_db = eng.database(res, off)
        load["from_memory_s"] = time.perf_counter() - t0
        mem_db.close()
        t0 = time.perf_counter()
        db = eng.open_database(path)
        load["from_file_s"] = time.perf_counter() - t0
    load["gb"] = nres / 1e9
    load["from_file_gbs"] = load["gb"] / load["from_file_s"]
    load["from_memory_gbs"] = load["gb"] / load["from_memory_s"]
    del res
    model = costmodel.CostModel.load(eng)
    lanes, depth, max_batch = args.serve_lanes, args.serve_depth, args.serve_batch
    sched = SCHED_COSTS if args.serve_schedule == "learned" else SCHED_DYNAMIC
    out = {"workload": "serve_vs_5M", "subjects": args.serve_subjects, "residues": nres, "db_load": load,
           "schedule": args.serve_schedule, "lanes": lanes, "lane_depth": depth, "max_batch_queries": max_batch,
           "memory_budget_gb": 16}
    runs = {}
    capacity = None
    # (label, offered rate or None for 80 % of the measured capacity, admission, segments)
    plan = [("offered", args.serve_rate, 0, 1),
            ("sustainable", None, 0, 1),
            ("sustainable_shortest_first", None, 1, 1),
            ("sustainable_preemptive", None, 1, args.serve_segments),
            ("sustainable_preemptive_wait_capped", None, 1, args.serve_segments)]
    if args.serve_rate_high > 0:
        plan.insert(1, ("offered_high", args.serve_rate_high, 0, 1))
    sustained = None        # the sustainable runs share one set of queries and arrival times
    for label, rate, admission, segments in plan:
        n = args.serve_requests if rate is not None else args.serve_sustained_requests
        if segments > 1 and args.serve_segments <= 1:
            continue
        if rate is None:
            if sustained is None:
                sustained = (synth.serving_queries(rng, n), serving.poisson_arrivals(rng, 0.8 * capacity, n),
                             0.8 * capacity)
            qs, arrivals, rate = sustained
        else:
            qs = synth.serving_queries(rng, n)
            arrivals = serving.poisson_arrivals(rng, rate, n)
        # ranges of a preemptive run queue at most one behind the running one
        run_depth = min(depth, 2) if segments > 1 else depth
        srv = Server(eng, db, max_batch_queries=max_batch, lanes=lanes, lane_depth=run_depth, schedule=sched,
                     model=model, chunk_residues=1 << 20, admission=admission, segments=segments,
                     max_wait_ms=args.serve_max_wait_ms if label.endswith("wait_capped") else 0)
        digests = []
        n_check = min(n, args.serve_check)
        t0 = time.perf_counter()
        _, lat, late = serving.drive(srv, qs, arrivals, keep_results=False, digests=digests,
                                     digest_first=n_check)
        wall = time.perf_counter() - t0
        st = srv.stats()
        srv.close()
        # the served results against plain searches of the same queries alone
        same = 0
        alone_ms = []
        for q, dg in zip(qs[:n_check], digests):
            h = eng.query(q)
            r = eng.search(db, h)
            same += int(r.digest() == dg)
            alone_ms.append(eng.last_scan_ms)
            r.close()
            h.close()
        qres = float(sum(len(q) for q in qs))
        runs[label] = {"offered_qps": rate, "requests": n, "admission": ["arrival", "shortest"][admission],
                       "max_wait_ms": args.serve_max_wait_ms if label.endswith("wait_capped") else 0,
                       "segments": segments, "lane_depth": run_depth,
                       "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
                       "max_ms": st["max_ms"], "throughput_qps": st["queries_per_s"],
                       "value": st["queries_per_s"] * nres, "unit": UNIT,
                       "residue_pairs_per_s": st["resq_per_s"], "batches": st["batches"],
                       "mean_batch": st["mean_batch"], "max_in_flight": st["max_in_flight"],
                       "mem_peak_gb": st["mem_peak"] / 1e9, "wall_s": wall,
                       "submit_lateness_ms_max": float(late.max()) if len(late) else 0.0,
                       "submit_lateness_ms_p99": serving.percentile(late, 99) if len(late) else 0.0,
                       "submit_lateness_worst_request": int(np.argmax(late)) if len(late) else -1,
                       "query_residues": qres,
                       "identical_to_plain": same == n_check, "checked_requests": n_check,
                       "alone_scan_ms_median": float(np.median(alone_ms)) if alone_ms else None,
                       "check": "served result digest (counters, offsets, HSP records) == the query's plain "
                                "search alone, first %d requests" % n_check}
        if label.startswith("offered"):   # capacity: the best saturated throughput measured
            capacity = max(capacity or 0.0, st["queries_per_s"])
    out["runs"] = runs
    out["identical_to_plain"] = all(r["identical_to_plain"] for r in runs.values())
    db.close()
    return out


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    sys.path.insert(0, ROOT)
    import oracle
    matrix = oracle.load_fixture_matrix()
    w = load_workload(matrix, 0, args.subjects, args.qlen)
    q = w.queries[0]
    # each step: table build + the reference kernel over a bounded,
    # length-sorted sample of the workload
    n = min(w.db.n_subjects, 50_000)
    res, off = sorted_sample(w, n)
    times = []
    kind, threads = "port", os.cpu_count() or 1
    for i in range(args.warmup + args.steps):
        dt, kind, threads = time_cpu_sample(matrix, q, res, off)
        if i >= args.warmup:
            times.append(dt)
    dt = float(np.sum(times))
    value = int(off[-1]) * len(times) / dt
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded; Robinson-Robinson residues, log-normal lengths, planted homologs)",
            "config": {"workload": w.name, "query_len": len(q), "subjects": w.db.n_subjects,
                       "residues": w.db.n_residues, "sample_subjects": n, "word": 3, "threshold": 11,
                       "window": 40, "x_dropoff": 16, "cutoff": 41},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count() or 1, "threads": threads,
                             "kind": kind,
                             "sample": "first %d subjects (%d residues, sorted by length, as the reference "
                                       "requires) per step: table build + %s" % (
                                           n, int(off[-1]),
                                           "the reference's own kernel (gpu_blastp_kernel.cu host-compiled "
                                           "into oracle/_ref, one POSIX thread per CUDA thread)"
                                           if kind == "reference" else "the oracle port's scan")},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "residue_pairs_per_s": value * len(q)}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local if world > 1 else 0)
    ranks = Ranks("nccl", device="cuda")
    import blastp_b200 as bp
    matrix = bp.blosum62()
    w = load_workload(matrix, rank, args.subjects, args.qlen)
    q = w.queries[0]
    eng = bp.Engine(local if world > 1 else 0)
    db = eng.database(w.db.residues, w.db.offsets)
    qry = eng.query(q)
    stream = torch.cuda.ExternalStream(eng.stream)

    def step():
        r = eng.search(db, qry)
        r.wait()
        ms = eng.last_scan_ms
        r.close()
        return ms

    for _ in range(args.warmup):
        step()
    clk = ClockSampler(local if world > 1 else 0)
    launches0 = eng.launches
    scan_ms, total_ms, _ = timed_steps(step, args.steps, 0, ranks, EventTimer(torch, stream),
                                       sync=torch.cuda.synchronize, during=clk)
    launches = eng.launches - launches0
    units = w.db.n_residues * world                # DB residues x queries (one query per step)
    value = units * args.steps / (total_ms / 1e3)

    # end to end through the C ABI: pinned host buffers in and out every step
    # (--e2e-steps 0 leaves it out, e.g. for profiling runs: the streaming scan
    # it launches waits on copies from another stream)
    n = w.db.n_subjects
    ref_hsps = eng.search(db, qry).fetch()
    e2e = None
    if args.e2e_steps > 0:
        res_pin = torch.empty(len(w.db.residues), dtype=torch.uint8, pin_memory=True)
        res_pin.numpy()[:] = w.db.residues
        off_pin = torch.empty(len(w.db.offsets), dtype=torch.int64, pin_memory=True)
        off_pin.numpy()[:] = w.db.offsets
        cnt_pin = torch.empty((n, 3), dtype=torch.int32, pin_memory=True)
        hoff_pin = torch.empty(n + 1, dtype=torch.int64, pin_memory=True)
        cap = len(ref_hsps.hsps) + 1024
        hsp_pin = torch.empty((cap, 6), dtype=torch.int32, pin_memory=True)
        import ctypes
        from blastp_b200._lib import lib, check
        p = bp.default_params()
        nh = ctypes.c_int64(0)
        qarr = np.ascontiguousarray(q)

        def e2e_step():
            check(lib().bp_blastp_host(eng.h, qarr.ctypes.data, len(q), ctypes.byref(p), res_pin.data_ptr(),
                                       len(w.db.residues), off_pin.data_ptr(), n, cnt_pin.data_ptr(),
                                       hoff_pin.data_ptr(), hsp_pin.data_ptr(), cap, ctypes.byref(nh)), eng.h)

        # (host buffers in and out every step: timed on the host clock between
        # barriers that leave the device idle)
        _, e2e_ms, _ = timed_steps(e2e_step, args.e2e_steps, 1, ranks, WallTimer(), sync=torch.cuda.synchronize)
        e2e_s = e2e_ms / 1e3
        h2d = len(w.db.residues) + 8 * len(w.db.offsets) + len(q)
        # the host link's own rate for the same bytes (pinned, one copy): the floor
        # of the end-to-end step next to the scan kernel's time
        dev_buf = torch.empty(len(w.db.residues), dtype=torch.uint8, device="cuda")
        link = []
        for _ in range(3):
            c0 = torch.cuda.Event(enable_timing=True)
            c1 = torch.cuda.Event(enable_timing=True)
            c0.record()
            dev_buf.copy_(res_pin, non_blocking=True)
            c1.record()
            torch.cuda.synchronize()
            link.append(c0.elapsed_time(c1))
        link_ms = float(min(link))
        del dev_buf
        d2h = 12 * n + 8 * (n + 1) + 24 * int(nh.value)
        e2e = {"value": w.db.n_residues * world * args.e2e_steps / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": 1e3 * e2e_s / args.e2e_steps,
               "upload_overlapped_with_scan": True,
               "link_ms_per_step": link_ms, "link_gbs": len(w.db.residues) / (link_ms / 1e3) / 1e9}

    peak, peak_kind = measured_peak_hbm()
    scan_avg_ms = float(np.mean(scan_ms))
    alg_bytes = w.db.n_residues + 8 * (n + 1) + 12 * n
    achieved = alg_bytes / (scan_avg_ms / 1e3) / 1e9
    tpr = profiled_per_residue("traffic_bytes_per_residue")
    # the bound the scan actually meets: instruction issue.  Warp instructions
    # per residue from the committed ncu capture of the same kernel, against
    # 4 issue slots per SM per cycle at the SM clock sampled under load.
    ipr = profiled_per_residue("warp_instructions_per_residue")
    clocks = clk.summary()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    issue = None
    if ipr and clocks:
        ach = ipr * w.db.n_residues / (scan_avg_ms / 1e3)
        pk = sms * 4 * clocks["sm_mhz"] * 1e6
        issue = {"achieved": ach, "peak": pk, "unit": "warp-instructions/s", "frac": ach / pk,
                 "warp_instructions_per_residue": ipr, "sms": sms, "sm_mhz": clocks["sm_mhz"],
                 "source": "profiles/scan_kernel_q500_vs_1M.md (ncu smsp__inst_executed)"}
    cnt = ref_hsps.counters
    rates = {"word_hits_per_s": float(cnt[:, 0].sum()) / (scan_avg_ms / 1e3),
             "extensions_per_s": float(cnt[:, 2].sum()) / (scan_avg_ms / 1e3),
             "word_hits_per_residue": float(cnt[:, 0].sum()) / w.db.n_residues,
             "extensions_per_residue": float(cnt[:, 2].sum()) / w.db.n_residues}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded; Robinson-Robinson residues, log-normal lengths, planted homologs)",
        "config": {"workload": w.name, "query_len": len(q), "subjects_per_gpu": n,
                   "residues_per_gpu": w.db.n_residues, "word": 3, "threshold": 11, "window": 40,
                   "x_dropoff": 16, "cutoff": 41, "parallelism": "shard%d" % world,
                   "l2": "inputs larger than L2 (%.2f GB database)" % (w.db.n_residues / 1e9)},
        "e2e": e2e,
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": (tpr * w.db.n_residues) if tpr else None,
                     "kernel": "scan_kernel", "kernel_ms": scan_avg_ms,
                     "kernel_ms_min_median_max": [float(np.min(scan_ms)), float(np.median(scan_ms)),
                                                  float(np.max(scan_ms))],
                     "algorithmic_bytes": alg_bytes, "issue": issue},
        "rates": rates,
        "hsps": int(len(ref_hsps.hsps)),
        # the same rate weighted by query length (DB residues x query residues / s)
        "residue_pairs_per_s": value * len(q),
    }
    line["clocks"] = clocks
    if world == 1 and args.config1:
        line["config1"] = run_config1(eng, matrix, args, torch, peak)
    if world == 1 and args.gapped:
        line["gapped"] = run_gapped_stage(eng, db, qry)
    if world == 1 and args.batched:
        line["batched"] = run_batched(eng, matrix, args, torch)
    if world == 1 and args.serve:
        line["serving"] = run_serving(eng, matrix, args)
    if rank == 0:
        sys.path.insert(0, ROOT)
        line["cpu_baseline"] = cpu_baseline(matrix, w, args.cpu_seconds)
        print(json.dumps(line), flush=True)
    qry.close()
    db.close()
    eng.close()
    ranks.close()
    return 0


def main():
    args = parse()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
