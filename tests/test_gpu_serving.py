"""GPU checks of the serving loop (bp_server_*): requests that arrive while
others run are admitted and overlap on the device, and every request's result
is bit-identical to the plain single-query search of the same query alone."""
import numpy as np
import pytest

from blastp_b200 import BpError, Server, costmodel, serving, synth
from blastp_b200._lib import SCHED_COSTS
from helpers import assert_same

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def world(engine, matrix):
    rng = np.random.default_rng(55)
    qs = synth.serving_queries(rng, 24, median=250, hi=1500)
    db = synth.make_database(rng, 15_000, qs[:6], 0.01, (60, 150), (0.3, 0.5), matrix)
    d = engine.database(db.residues, db.offsets)
    alone = []
    for q in qs:
        h = engine.query(q)
        alone.append(engine.search(d, h).fetch())
        h.close()
    return qs, db, d, alone


def _check(results, alone, what):
    for i, (r, a) in enumerate(zip(results, alone)):
        assert_same(r, (a.counters, a.hsp_off, a.hsps_as_array()), "%s request %d" % (what, i))


def test_mix_equals_alone_and_overlaps(engine, world):
    qs, db, d, alone = world
    srv = Server(engine, d, max_batch_queries=4, lanes=2, chunk_residues=1 << 18)
    arr = serving.poisson_arrivals(np.random.default_rng(1), 2000.0, len(qs))
    results, lat, _ = serving.drive(srv, qs, arr)
    _check(results, alone, "mix")
    st = srv.stats()
    assert st["completed"] == len(qs) and st["failed"] == 0
    assert st["batches"] >= len(qs) // 4
    assert st["max_in_flight"] > 4          # a second batch was admitted while the first ran
    assert st["p99_ms"] >= st["p50_ms"] > 0
    assert abs(serving.percentile(lat, 50) - st["p50_ms"]) < 1e-6
    assert st["mem_used"] == 0
    srv.close()


def test_memory_budget_limits_admission(engine, world):
    qs, db, d, alone = world
    per_request = 15_000 * 24 + (19684 * 4) + 40 * 1500 + 4096 + int(3e-4 * 1.5 * 3 * db.n_residues) * 60
    srv = Server(engine, d, max_batch_queries=8, lanes=2, memory_budget=2 * per_request)
    results, _, _ = serving.drive(srv, qs[:10], np.zeros(10))
    _check(results, alone[:10], "budget")
    st = srv.stats()
    assert st["max_in_flight"] <= 4          # without the budget: 16 (two lanes of 8)
    assert st["mem_peak"] <= 2 * per_request
    srv.close()


def test_learned_schedule_in_server(engine, world):
    qs, db, d, alone = world
    model = costmodel.CostModel.load(engine)
    srv = Server(engine, d, max_batch_queries=6, lanes=2, schedule=SCHED_COSTS, model=model, planted_density=0.01)
    results, _, _ = serving.drive(srv, qs[:12], serving.poisson_arrivals(np.random.default_rng(2), 500.0, 12))
    _check(results, alone[:12], "learned")
    srv.close()


def test_results_stay_until_released(engine, world):
    qs, db, d, alone = world
    srv = Server(engine, d, max_batch_queries=2, lanes=1)
    t = [srv.submit(q) for q in qs[:3]]
    for x in t:
        srv.wait(x)
    assert srv.stats()["mem_used"] > 0
    r, _ = srv.result(t[1])
    _check([r], [alone[1]], "held")
    for x in t:
        srv.release(x)
    with pytest.raises(BpError):
        srv.release(t[0])
    assert srv.stats()["mem_used"] == 0
    srv.close()


def test_bad_requests_rejected(engine, world):
    qs, db, d, alone = world
    srv = Server(engine, d)
    with pytest.raises(BpError):
        srv.submit(np.array([1, 0, 3], np.uint8))
    with pytest.raises(BpError):
        srv.submit(np.ones(70_000, np.uint8))
    srv.close()


def test_served_digests_equal_plain(engine, world):
    # the digest of each served request equals its plain search's digest
    qs, db, d, alone = world
    srv = Server(engine, d, max_batch_queries=4, lanes=2, chunk_residues=1 << 18)
    tickets = [srv.submit(q) for q in qs[:8]]
    for i, t in enumerate(tickets):
        srv.wait(t)
        h = engine.query(qs[i])
        r = engine.search(d, h)
        assert srv.digest(t) == r.digest(), "request %d" % i
        r.close()
        h.close()
        srv.release(t)
    srv.close()


def test_lane_depth_runs_batches_back_to_back_in_order(engine, world):
    # one lane holding up to three batches of one query each: requests
    # submitted together complete in submission order (the lane's batches run
    # one after the other on the device), more than one batch is in flight on
    # the lane, and every result equals the query searched alone
    qs, db, d, alone = world
    srv = Server(engine, d, max_batch_queries=1, lanes=1, lane_depth=3, chunk_residues=1 << 18)
    tickets = [srv.submit(q) for q in qs[:12]]
    lat = []
    for i, t in enumerate(tickets):
        srv.wait(t)
        r, ms = srv.result(t)
        a = alone[i]
        assert_same(r, (a.counters, a.hsp_off, a.hsps_as_array()), "depth-3 lane, request %d" % i)
        lat.append(ms)
        srv.release(t)
    st = srv.stats()
    srv.close()
    assert st["completed"] == 12 and st["max_in_flight"] >= 2
    # arrivals were microseconds apart: completion order shows in the latencies
    assert all(lat[i] <= lat[i + 1] + 0.5 for i in range(len(lat) - 1)), lat


def test_shortest_first_admission(engine, matrix):
    # one lane, one query per batch: a long request runs while six more wait,
    # submitted longest first; arrival order completes them longest first,
    # shortest-first admission completes them shortest first. Each result's
    # digest equals its plain search's.
    import time
    from blastp_b200._lib import ADMIT_ARRIVAL, ADMIT_SHORTEST
    rng = np.random.default_rng(77)
    head = synth.residues(rng, 2000)
    waiting = [synth.residues(rng, n) for n in (900, 700, 500, 300, 150, 60)]
    db = synth.make_database(rng, 250_000, [head], 0.001, (60, 150), (0.3, 0.5), matrix)
    d = engine.database(db.residues, db.offsets)
    plain = []
    for q in [head] + waiting:
        h = engine.query(q)
        r = engine.search(d, h)
        plain.append(r.digest())
        r.close()
        h.close()
    for policy in (ADMIT_ARRIVAL, ADMIT_SHORTEST):
        srv = Server(engine, d, max_batch_queries=1, lanes=1, lane_depth=1, admission=policy,
                     chunk_residues=1 << 20, poll_us=50)
        t0 = time.perf_counter()
        first = srv.submit(head)
        while srv.state(first) == 0:            # queued: wait until the head is admitted
            pass
        offs, tickets = [], []
        for q in waiting:
            offs.append((time.perf_counter() - t0) * 1e3)
            tickets.append(srv.submit(q))
        submitted = (time.perf_counter() - t0) * 1e3
        srv.wait(first)
        head_ms = srv.latency(first)
        done = []
        for i, t in enumerate(tickets):
            srv.wait(t)
            assert srv.digest(t) == plain[1 + i], "policy %d request %d" % (policy, i)
            done.append(offs[i] + srv.latency(t))
        srv.close()
        if head_ms <= submitted:
            pytest.skip("the head request finished before the others were submitted")
        order = list(np.argsort(done, kind="stable"))
        # waiting is longest first: arrival order keeps it, shortest-first reverses it
        assert order == (list(range(6)) if policy == ADMIT_ARRIVAL else list(range(5, -1, -1))), (policy, done)
    d.close()


@pytest.mark.parametrize("admission", [0, 1])
def test_segmented_requests_equal_alone(engine, world, admission):
    # each request searched as 4 jobs over consecutive subject ranges, the
    # ranges of different requests interleaved on one lane: every result (read
    # back piece by piece) and every digest equals the plain search alone
    qs, db, d, alone = world
    srv = Server(engine, d, lanes=1, lane_depth=2, segments=4, admission=admission, chunk_residues=1 << 16)
    arr = serving.poisson_arrivals(np.random.default_rng(5), 3000.0, 12)
    digs = []
    results, lat, _ = serving.drive(srv, qs[:12], arr, digests=digs, digest_first=12)
    _check(results, alone[:12], "segmented")
    for i in range(12):
        h = engine.query(qs[i])
        r = engine.search(d, h)
        assert digs[i] == r.digest(), "request %d" % i
        r.close()
        h.close()
    st = srv.stats()
    assert st["completed"] == 12 and st["failed"] == 0
    assert st["batches"] == 12 * 4            # one job per range
    assert st["mem_used"] == 0
    srv.close()


def test_segmented_shortest_first_preempts_a_long_request(engine, matrix):
    # a long request running range by range while six short ones arrive:
    # with the least-work-left policy the short ones go ahead of the long
    # one's remaining ranges and all finish before it; in arrival order the
    # long one finishes first
    import time
    from blastp_b200._lib import ADMIT_ARRIVAL, ADMIT_SHORTEST
    rng = np.random.default_rng(78)
    head = synth.residues(rng, 2000)
    short = [synth.residues(rng, n) for n in (120, 90, 150, 60, 100, 80)]
    db = synth.make_database(rng, 400_000, [head], 0.001, (60, 150), (0.3, 0.5), matrix)
    d = engine.database(db.residues, db.offsets)
    plain = []
    for q in [head] + short:
        h = engine.query(q)
        r = engine.search(d, h)
        plain.append(r.digest())
        r.close()
        h.close()
    # (a wait limit of 1 ms makes the long request overdue at once: it goes first again)
    for policy, max_wait in ((ADMIT_ARRIVAL, 0), (ADMIT_SHORTEST, 0), (ADMIT_SHORTEST, 1)):
        srv = Server(engine, d, lanes=1, lane_depth=1, segments=8, admission=policy, chunk_residues=1 << 20,
                     poll_us=50, max_wait_ms=max_wait)
        t0 = time.perf_counter()
        first = srv.submit(head)
        while srv.state(first) < 2:             # until its first range runs
            pass
        offs, tickets = [], []
        for q in short:
            offs.append((time.perf_counter() - t0) * 1e3)
            tickets.append(srv.submit(q))
        submitted = (time.perf_counter() - t0) * 1e3
        srv.wait(first)
        head_end = srv.latency(first)
        assert srv.digest(first) == plain[0]
        ends = []
        for i, t in enumerate(tickets):
            srv.wait(t)
            assert srv.digest(t) == plain[1 + i], "policy %d request %d" % (policy, i)
            ends.append(offs[i] + srv.latency(t))
        srv.close()
        if head_end <= submitted:
            pytest.skip("the long request finished before the short ones were submitted")
        if policy == ADMIT_SHORTEST and max_wait == 0:
            assert max(ends) < head_end, (ends, head_end)
        else:
            assert min(ends) > head_end, (policy, max_wait, ends, head_end)
    d.close()


def test_shortest_first_leaves_room_for_the_requests_it_overtakes(engine, world):
    # a client that reads its requests in submission order and releases each
    # after reading it: the long request it waits for must be admitted even
    # though later, shorter requests were admitted ahead of it and hold their
    # (unread) results -- shortest-first keeps room for the older request
    qs, db, d, alone = world
    lens = np.array([len(q) for q in qs])
    li = int(np.argmax(lens))
    short = [int(i) for i in np.argsort(lens)[:10]]

    def per(L):   # the server's estimate of a request's device bytes
        return (19684 * 4 + 40 * L + 4096) + (db.n_subjects * 24 + 8) + int(3e-4 * 1.5 * L / 500.0 * db.n_residues) * 60

    budget = per(lens[li]) + 2 * per(max(lens[i] for i in short))
    srv = Server(engine, d, max_batch_queries=1, lanes=1, lane_depth=1, admission=1, memory_budget=budget)
    head = srv.submit(qs[li])
    a = srv.submit(qs[li])
    rest = [srv.submit(qs[i]) for i in short]
    for t, qi in [(head, li), (a, li)] + list(zip(rest, short)):
        srv.wait(t, 60_000)             # raises if the server stalled
        r, _ = srv.result(t)
        _check([r], [alone[qi]], "request %d" % qi)
        srv.release(t)
    st = srv.stats()
    assert st["completed"] == 12 and st["mem_peak"] <= budget and st["mem_used"] == 0
    srv.close()


def test_segmented_two_lanes_under_a_memory_budget(engine, world):
    # ranges of different requests on two lanes at once, shortest first, with a
    # budget of about three requests: every result equals the plain search and
    # the budget is never exceeded
    qs, db, d, alone = world
    per = 19684 * 4 + 40 * 1500 + 4096 + db.n_subjects * 24 + 8 + int(3e-4 * 1.5 * 3 * db.n_residues) * 60
    srv = Server(engine, d, lanes=2, lane_depth=2, segments=3, admission=1, memory_budget=3 * per)
    arr = serving.poisson_arrivals(np.random.default_rng(8), 4000.0, 16)
    results, _, _ = serving.drive(srv, qs[:16], arr)
    _check(results, alone[:16], "two lanes, ranges")
    st = srv.stats()
    assert st["completed"] == 16 and st["batches"] == 16 * 3
    assert st["mem_peak"] <= 3 * per and st["mem_used"] == 0
    srv.close()
