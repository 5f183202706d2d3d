"""GPU parity of the batched persistent search (bp_search_batch): every
query's counters and HSP set equal its single-query bp_search result, bit for
bit, under each schedule, chunk size and CTA count, on the first run and on
graph replays.  One query is also checked against the CPU oracle directly."""
import numpy as np
import pytest

from blastp_b200 import BpError, default_params, synth
from blastp_b200._lib import SCHED_COST_ORDER, SCHED_COSTS, SCHED_DYNAMIC, SCHED_STATIC
from helpers import assert_same, oracle_search

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def workload(matrix):
    rng = np.random.default_rng(4242)
    lens = [50, 1, 3, 120, 300, 777, 2000, 4000, 64, 1500]
    qs = [synth.residues(rng, n) for n in lens]
    qs.append(np.full(200, synth.encode("L")[0], dtype=np.uint8))      # one cell holds every offset
    db = synth.make_database(rng, 12_000, qs, 0.01, (40, 150), (0.25, 0.5), matrix)
    return qs, db


@pytest.fixture(scope="module")
def singles(engine, workload):
    qs, db = workload
    d = engine.database(db.residues, db.offsets)
    out = []
    for q in qs:
        h = engine.query(q)
        out.append(engine.search(d, h).fetch())
        h.close()
    d.close()
    return out


def _run(engine, workload, **kw):
    qs, db = workload
    d = engine.database(db.residues, db.offsets)
    hs = [engine.query(q) for q in qs]
    b = engine.search_batch(d, hs, **kw)
    return b, d, hs


def _check(b, singles, what):
    for i, s in enumerate(singles):
        r = b.fetch(i)
        assert_same(r, (s.counters, s.hsp_off, s.hsps_as_array()), "%s query %d" % (what, i))


def test_one_query_vs_oracle(engine, matrix, workload):
    qs, db = workload
    b, d, hs = _run(engine, workload, chunk_residues=1 << 16)
    for i in (0, 4, 10):
        ref = oracle_search(qs[i], db.residues, db.offsets, matrix)
        assert_same(b.fetch(i), ref, "batched query %d vs oracle" % i)
    b.close()


@pytest.mark.parametrize("schedule", [SCHED_DYNAMIC, SCHED_STATIC, SCHED_COSTS, SCHED_COST_ORDER])
@pytest.mark.parametrize("chunk", [1 << 12, 1 << 18, 1 << 30])
def test_schedules_and_chunks(engine, workload, singles, schedule, chunk):
    qs, db = workload
    d = engine.database(db.residues, db.offsets)
    hs = [engine.query(q) for q in qs]
    costs = None
    if schedule in (SCHED_COSTS, SCHED_COST_ORDER):
        n_items = len(qs) * (len(engine.plan_chunks(d, chunk)) - 1)
        costs = np.random.default_rng(chunk).random(n_items).astype(np.float32)
    b = engine.search_batch(d, hs, chunk_residues=chunk, schedule=schedule, item_costs=costs)
    _check(b, singles, "sched %d chunk %d" % (schedule, chunk))
    if schedule == SCHED_COSTS:
        qc = b.queue_costs()
        assert abs(qc.sum() - costs.sum()) < 1e-3 * max(1.0, costs.sum())
    b.close()


@pytest.mark.parametrize("ctas,max_warps", [(1, 0), (7, 4), (0, 1), (300, 0)])
def test_cta_shapes(engine, workload, singles, ctas, max_warps):
    b, d, hs = _run(engine, workload, chunk_residues=1 << 15, ctas=ctas, max_warps=max_warps,
                    schedule=SCHED_STATIC if ctas == 7 else SCHED_DYNAMIC)
    _check(b, singles, "ctas %d warps %d" % (ctas, max_warps))
    b.close()


@pytest.mark.parametrize("use_graph", [True, False])
def test_rerun_and_replay(engine, workload, singles, use_graph):
    b, d, hs = _run(engine, workload, chunk_residues=1 << 17, use_graph=use_graph)
    b.wait()
    n0 = b.n_hsps
    l0 = engine.launches
    for _ in range(3):
        b.run()
    b.wait()
    assert b.n_hsps == n0
    assert engine.launches - l0 >= 3 * 6          # scan + the 5 ordering kernels per run
    _check(b, singles, "re-run graph=%s" % use_graph)
    b.close()


def test_record_overflow_regrows(engine, matrix):
    # repeats of the query in every subject make far more HSPs than the first
    # capacity guess: the batch re-runs with a larger buffer and still matches
    rng = np.random.default_rng(7)
    q = synth.residues(rng, 400)
    parts = [np.concatenate([q, q, q])] * 3000
    res = np.concatenate(parts).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum([len(p) for p in parts])]).astype(np.int64)
    d = engine.database(res, off)
    h = engine.query(q)
    single = engine.search(d, h).fetch()
    b = engine.search_batch(d, [h, h], chunk_residues=1 << 14)
    for i in range(2):
        assert_same(b.fetch(i), (single.counters, single.hsp_off, single.hsps_as_array()), "overflow %d" % i)
    b.close()


def test_empty_batch_and_empty_database(engine):
    rng = np.random.default_rng(3)
    d = engine.database(np.zeros(0, np.uint8), np.zeros(1, np.int64))
    h = engine.query(synth.residues(rng, 100))
    b = engine.search_batch(d, [h, h])
    assert b.wait().n_hsps == 0
    assert b.fetch(1).counters.shape == (0, 3)
    b.close()
    d2 = engine.database(synth.residues(rng, 1000), np.array([0, 500, 1000], np.int64))
    b = engine.search_batch(d2, [])
    assert b.wait().n_hsps == 0
    b.close()


def test_batch_rejects_mixed_windows_and_missing_costs(engine):
    rng = np.random.default_rng(5)
    d = engine.database(synth.residues(rng, 1000), np.array([0, 1000], np.int64))
    a = engine.query(synth.residues(rng, 50))
    c = engine.query(synth.residues(rng, 50), default_params(window=20))
    with pytest.raises(BpError):
        engine.search_batch(d, [a, c])
    with pytest.raises(BpError):
        engine.search_batch(d, [a], schedule=SCHED_COSTS)


@pytest.mark.parametrize("first,count", [(0, 5000), (3333, 4000), (11_999, 1), (12_000, 0), (7000, -1)])
def test_subject_range(engine, workload, first, count):
    qs, db = workload
    d = engine.database(db.residues, db.offsets)
    hs = [engine.query(q) for q in qs[:4]]
    b = engine.search_batch(d, hs, chunk_residues=1 << 16, first=first, count=count)
    for i, h in enumerate(hs):
        s = engine.search(d, h, first, count).fetch()
        assert_same(b.fetch(i), (s.counters, s.hsp_off, s.hsps_as_array()), "range query %d" % i)
    b.close()


def test_bad_subject_range_rejected(engine, workload):
    qs, db = workload
    d = engine.database(db.residues, db.offsets)
    h = engine.query(qs[0])
    for first, count in ((-1, 5), (0, 12_001), (12_001, -1)):
        with pytest.raises(BpError):
            engine.search_batch(d, [h], first=first, count=count)


def test_autotune_picks_a_measured_candidate(engine, workload, singles):
    qs, db = workload
    d = engine.database(db.residues, db.offsets)
    hs = [engine.query(q) for q in qs]
    best, trials = engine.autotune(d, hs, sample_subjects=3000, chunk_sizes=[1 << 14, 1 << 18], warp_caps=[0, 8],
                                   schedules=(SCHED_DYNAMIC, SCHED_STATIC), reps=1)
    assert len(trials) == 9                    # 2 chunks x 3 packings, 1 schedule, 1 warp cap, plain
    assert [t["plain_unpacked"] for t in trials] == [0] * 8 + [1]
    fastest = min(trials, key=lambda t: t["ms"])
    assert (best["chunk_residues"], best["schedule"], best["max_warps"], best["plain_unpacked"]) == (
        fastest["chunk_residues"], fastest["schedule"], fastest["max_warps"], fastest["plain_unpacked"])
    b = engine.search_batch(d, hs, **best)
    _check(b, singles, "autotuned")
    b.close()


@pytest.mark.parametrize("pack", [256, 2048, 8000])
@pytest.mark.parametrize("schedule", [SCHED_DYNAMIC, SCHED_COSTS, SCHED_COST_ORDER])
def test_packed_tables(engine, workload, singles, pack, schedule):
    # short queries share packed tables; every query's result stays its own
    qs, db = workload
    d = engine.database(db.residues, db.offsets)
    hs = [engine.query(q) for q in qs]
    costs = None
    if schedule in (SCHED_COSTS, SCHED_COST_ORDER):
        costs = np.random.default_rng(pack).random(len(qs) * (len(engine.plan_chunks(d, 1 << 16)) - 1))
    b = engine.search_batch(d, hs, chunk_residues=1 << 16, schedule=schedule, item_costs=costs,
                            pack_residues=pack)
    _check(b, singles, "pack %d sched %d" % (pack, schedule))
    b.run()
    _check(b, singles, "pack %d sched %d replay" % (pack, schedule))
    b.close()


def test_many_short_queries_packed(engine, matrix):
    # 70 short queries (more than one full pack of 32), a subject range, and
    # per-query parameters: packed results equal each query searched alone
    rng = np.random.default_rng(31)
    qs = [synth.residues(rng, int(n)) for n in rng.integers(3, 120, size=70)]
    db = synth.make_database(rng, 5000, qs, 0.02, (30, 100), (0.35, 0.6), matrix)
    d = engine.database(db.residues, db.offsets)
    params = [default_params(x_dropoff=12 + (i % 3) * 4, cutoff_score=35 + (i % 4) * 3) for i in range(len(qs))]
    hs = [engine.query(q, p) for q, p in zip(qs, params)]
    b = engine.search_batch(d, hs, chunk_residues=1 << 15, pack_residues=3000, first=100, count=4500)
    for i, h in enumerate(hs):
        s = engine.search(d, h, 100, 4500).fetch()
        assert_same(b.fetch(i), (s.counters, s.hsp_off, s.hsps_as_array()), "short query %d" % i)
    b.close()


def test_digests_match_plain_and_tell_results_apart(engine, workload):
    # The device-side digest of each query's batched result equals the digest
    # of its plain search; the queries' digests all differ (their results do),
    # and a result differing in one HSP field changes the digest.
    qs, db = workload
    d = engine.database(db.residues, db.offsets)
    hs = [engine.query(q) for q in qs]
    plain = []
    for h in hs:
        r = engine.search(d, h)
        plain.append((r.digest(), r.fetch()))
        r.close()
    b = engine.search_batch(d, hs, chunk_residues=1 << 16)
    digests = [b.digest(i) for i in range(len(qs))]
    for i, (pd, res) in enumerate(plain):
        assert digests[i] == pd, "query %d" % i
    distinct = {digests[i] for i in range(len(qs)) if len(plain[i][1].hsps)}
    assert len(distinct) == sum(1 for _, r in plain if len(r.hsps))
    b.close()
    for h in hs:
        h.close()
    d.close()


@pytest.mark.parametrize("pack", [0, 1024])
@pytest.mark.parametrize("use_graph", [False, True])
def test_plain_unpacked(engine, workload, singles, pack, use_graph):
    # the queries that are not packed run as plain single-query scans inside
    # the batch (packed tables, if any, as batched items): every query's
    # result equals its single-query search, on replays too
    qs, db = workload
    d = engine.database(db.residues, db.offsets)
    hs = [engine.query(q) for q in qs]
    b = engine.search_batch(d, hs, chunk_residues=1 << 16, pack_residues=pack, plain_unpacked=1,
                            use_graph=use_graph)
    _check(b, singles, "plain unpacked, pack %d" % pack)
    b.run()
    _check(b, singles, "plain unpacked, replayed")
    b.close()
