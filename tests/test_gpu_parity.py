"""GPU parity of the plain path (C ABI: bp_query_create / bp_search) against
the CPU oracle: bit-exact counters and HSP sets, in discovery order."""
import numpy as np
import pytest

import oracle
from blastp_b200 import BpError, default_params, synth
from helpers import assert_same, gpu_search, oracle_search

pytestmark = pytest.mark.gpu


def enc(s):
    return synth.encode(s)


@pytest.mark.parametrize("text_or_len", [0, 1, 2, 3, 50, 300, 2000, "LLLLLLLLLLLLLLLLLLLLLLLLLLLLLL",
                                         "BZXUOJ*ACDEFGHIKLMNPQRSTVWY", "WWWWCCCCHHHH"])
def test_device_table_matches_oracle(engine, matrix, text_or_len):
    if isinstance(text_or_len, str):
        q = enc(text_or_len)
    else:
        q = synth.residues(np.random.default_rng(text_or_len), text_or_len)
    for thr in (11, 13):
        start, ent = engine.query(q, default_params(threshold=thr)).table()
        ostart, oent = oracle.build_table(q, matrix, thr)
        assert (start == ostart).all()
        assert (ent == oent).all()


def test_shape1_full(engine, matrix):
    w = synth.shape1(matrix)
    q = w.queries[0]
    assert_same(gpu_search(engine, q, w.db.residues, w.db.offsets),
                oracle_search(q, w.db.residues, w.db.offsets, matrix), "q300 vs 10k")


def test_shape2_reduced(engine, matrix):
    w = synth.shape2(matrix, n_subjects=60_000)
    q = w.queries[0]
    assert_same(gpu_search(engine, q, w.db.residues, w.db.offsets),
                oracle_search(q, w.db.residues, w.db.offsets, matrix), "q500 vs 60k")


@pytest.mark.parametrize("qlen", [50, 1000, 2000, 4000])
def test_query_lengths(engine, matrix, qlen):
    rng = np.random.default_rng(qlen)
    q = synth.residues(rng, qlen)
    db = synth.make_database(rng, 3000, [q], 0.02, (60, 150), (0.25, 0.45), matrix)
    assert_same(gpu_search(engine, q, db.residues, db.offsets),
                oracle_search(q, db.residues, db.offsets, matrix), "qlen %d" % qlen)


def test_long_query_16384(engine, matrix):
    # the reference's QUERY_LENGTH_MAX (gpu_cpu_common.h:25)
    rng = np.random.default_rng(16384)
    q = synth.residues(rng, 16384)
    db = synth.make_database(rng, 300, [q], 0.05, (60, 150), (0.3, 0.5), matrix)
    assert_same(gpu_search(engine, q, db.residues, db.offsets),
                oracle_search(q, db.residues, db.offsets, matrix), "qlen 16384")


def test_edge_subjects(engine, matrix):
    rng = np.random.default_rng(11)
    q = synth.residues(rng, 400)
    parts = [enc(""), enc("W"), enc("WC"), enc("WCW"), q[:3].copy(), q.copy(), enc("")]
    parts.append(synth.residues(rng, 40_000))                     # very long subject
    parts.append(np.concatenate([q[100:250], q[100:250]]))        # repeat: many two-hit pairs
    parts.append(np.array([23, 24, 25, 26, 27, 2, 21] * 20, dtype=np.uint8))   # ambiguity letters
    parts.append(np.full(500, enc("L")[0], dtype=np.uint8))       # low complexity
    res = np.concatenate(parts).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum([len(p) for p in parts])]).astype(np.int64)
    assert_same(gpu_search(engine, q, res, off), oracle_search(q, res, off, matrix), "edge subjects")
    # poly-L query against the same subjects: one cell holds every query offset
    qL = np.full(300, enc("L")[0], dtype=np.uint8)
    assert_same(gpu_search(engine, qL, res, off), oracle_search(qL, res, off, matrix), "poly-L query")


def test_empty_database_and_short_queries(engine, matrix):
    res = np.zeros(0, dtype=np.uint8)
    off = np.zeros(1, dtype=np.int64)
    r = gpu_search(engine, enc("WCWCWC"), res, off)
    assert r.counters.shape == (0, 3) and len(r.hsps) == 0 and r.hsp_off.tolist() == [0]
    rng = np.random.default_rng(2)
    db = synth.make_database(rng, 200, [], 0.0, (1, 1), (0, 0), matrix)
    for qlen in (0, 1, 2):
        q = synth.residues(rng, qlen)
        r = gpu_search(engine, q, db.residues, db.offsets)
        assert (r.counters == 0).all() and len(r.hsps) == 0


def test_identical_sequences(engine, matrix):
    rng = np.random.default_rng(7)
    s = synth.residues(rng, 120)
    off = np.array([0, 120], dtype=np.int64)
    r = gpu_search(engine, s, s, off)
    g = r.hsps_as_array()
    main = g[g[:, 0] == g[:, 1]]
    assert len(main) == 1
    assert tuple(main[0][[0, 1, 4, 5]]) == (0, 0, 120, int(matrix[s, s].astype(int).sum()))


@pytest.mark.parametrize("kw", [dict(window=20), dict(x_dropoff=7), dict(cutoff_score=25), dict(threshold=12),
                                dict(window=1), dict(x_dropoff=0)])
def test_parameters(engine, matrix, kw):
    w = synth.shape1(matrix, n_subjects=2000)
    q = w.queries[0]
    p = default_params(**kw)
    assert_same(gpu_search(engine, q, w.db.residues, w.db.offsets, p),
                oracle_search(q, w.db.residues, w.db.offsets, matrix, p), str(kw))


def test_subject_range_and_repeatability(engine, matrix):
    w = synth.shape1(matrix, n_subjects=5000)
    q = w.queries[0]
    full = oracle_search(q, w.db.residues, w.db.offsets, matrix)
    db = engine.database(w.db.residues, w.db.offsets)
    qq = engine.query(q)
    a = engine.search(db, qq).fetch()
    b = engine.search(db, qq).fetch()
    assert_same(a, full, "run 1")
    assert_same(b, full, "run 2")
    part = engine.search(db, qq, 1000, 2500).fetch()
    counters, hoff, hsps = full
    assert (part.counters == counters[1000:3500]).all()
    ph = part.hsps_as_array()
    assert (ph == hsps[hoff[1000]:hoff[3500]]).all()


def test_end_to_end_host_call_matches(engine, matrix):
    w = synth.shape1(matrix, n_subjects=4000)
    q = w.queries[0]
    r = engine.blastp_host(q, default_params(), w.db.residues, w.db.offsets, hsp_cap=8)   # forces a resize
    assert_same(r, oracle_search(q, w.db.residues, w.db.offsets, matrix), "bp_blastp_host")


def test_invalid_inputs_rejected(engine):
    with pytest.raises(BpError):
        engine.query(enc("WC-W"))                          # gap letter inside a query
    with pytest.raises(BpError):
        engine.query(np.array([1, 2, 40], dtype=np.uint8))   # code >= 28
    with pytest.raises(BpError):
        engine.query(enc("WCW"), default_params(word_length=2))
    with pytest.raises(BpError):
        engine.database(np.array([1, 2, 99], dtype=np.uint8), np.array([0, 3], dtype=np.int64))
    with pytest.raises(BpError):
        engine.database(np.array([1, 2, 3], dtype=np.uint8), np.array([0, 2], dtype=np.int64))
    with pytest.raises(BpError):
        engine.query(np.ones(70000, dtype=np.uint8))


def test_shape2_full_size(engine, matrix):
    """The 1,000,000-subject database of the headline benchmark: bit-exact
    against the oracle, plus size-independent invariants."""
    w = synth.shape2(matrix)
    q = w.queries[0]
    r = gpu_search(engine, q, w.db.residues, w.db.offsets)
    ref = oracle_search(q, w.db.residues, w.db.offsets, matrix)
    assert_same(r, ref, "q500 vs 1M")
    g = r.hsps_as_array()
    assert r.hsp_off[-1] == len(g) == r.counters[:, 1].sum()
    assert (g[:, 5] >= 41).all()
    lens = np.diff(w.db.offsets)
    owner = np.repeat(np.arange(len(lens)), np.diff(r.hsp_off))
    assert (g[:, 1] >= 0).all() and (g[:, 1] + g[:, 4] <= lens[owner]).all()
    assert (g[:, 0] + g[:, 4] <= len(q)).all()
    # every planted homolog long enough to matter is found
    found = set(owner.tolist())
    planted = w.db.plants[w.db.plants[:, 4] >= 100][:, 0]
    assert np.mean([p in found for p in planted]) > 0.9


def test_host_path_overlapped_chunks(engine, matrix):
    # ~144M residues: the host-to-host call uploads three chunks under the
    # scans of the earlier ones; results equal the resident-database search,
    # from pinned and from pageable host memory, and on a repeated call
    import torch
    w = synth.shape2(matrix, n_subjects=400_000)
    q = w.queries[0]
    ref = gpu_search(engine, q, w.db.residues, w.db.offsets)
    got = engine.blastp_host(q, default_params(), w.db.residues, w.db.offsets)
    assert_same(got, (ref.counters, ref.hsp_off, ref.hsps_as_array()), "pageable")
    pin = torch.empty(len(w.db.residues), dtype=torch.uint8, pin_memory=True)
    pin.numpy()[:] = w.db.residues
    got = engine.blastp_host(q, default_params(), pin.numpy(), w.db.offsets)
    assert_same(got, (ref.counters, ref.hsp_off, ref.hsps_as_array()), "pinned")
    got = engine.blastp_host(q, default_params(), pin.numpy(), w.db.offsets)
    assert_same(got, (ref.counters, ref.hsp_off, ref.hsps_as_array()), "pinned, again")
    # pinned outputs: each chunk's counters come back as soon as its scan ends
    cnt = torch.full((w.db.n_subjects, 3), -1, dtype=torch.int32, pin_memory=True)
    hoff = torch.full((w.db.n_subjects + 1,), -1, dtype=torch.int64, pin_memory=True)
    got = engine.blastp_host(q, default_params(), pin.numpy(), w.db.offsets, counters=cnt.numpy(),
                             hsp_off=hoff.numpy())
    assert_same(got, (ref.counters, ref.hsp_off, ref.hsps_as_array()), "pinned in and out")


def test_host_path_pinned_edges(engine, matrix):
    # pinned residues: empty, 1- and 2-letter, identical and very long subjects
    # through the single streaming launch, then a query of 8,200 letters
    # (32-bit diagonal entries), which takes one launch per chunk instead
    import torch
    rng = np.random.default_rng(29)
    q = synth.residues(rng, 400)
    parts = [enc(""), enc("W"), enc("WC"), q.copy(), enc("")]
    parts.append(synth.residues(rng, 40_000))
    parts += [synth.residues(rng, int(n)) for n in rng.integers(0, 600, size=3000)]
    parts.append(np.concatenate([q[50:200], q[50:200]]))
    res = np.concatenate(parts).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum([len(x) for x in parts])]).astype(np.int64)
    pin = torch.empty(len(res), dtype=torch.uint8, pin_memory=True)
    pin.numpy()[:] = res
    for query in (q, synth.residues(rng, 8200)):
        got = engine.blastp_host(query, default_params(), pin.numpy(), off)
        assert_same(got, oracle_search(query, res, off, matrix), "pinned, qlen %d" % len(query))


def test_host_path_rejects_bad_offsets(engine):
    # a decreasing offset inside the first chunk (the chunk boundaries are
    # in order): refused before any scan, the engine stays usable
    rng = np.random.default_rng(3)
    n = 5000
    off = np.concatenate([[0], np.cumsum(rng.integers(50, 400, size=n))]).astype(np.int64)
    res = synth.residues(rng, int(off[-1]))
    bad = off.copy()
    bad[100], bad[101] = off[101], off[100]
    q = synth.residues(rng, 300)
    with pytest.raises(BpError):
        engine.blastp_host(q, default_params(), res, bad)
    got = engine.blastp_host(q, default_params(), res, off)
    ref = gpu_search(engine, q, res, off)
    assert_same(got, (ref.counters, ref.hsp_off, ref.hsps_as_array()), "after a refused call")
    # from pinned memory (the single streaming launch checks the offsets itself)
    import torch
    pin = torch.empty(len(res), dtype=torch.uint8, pin_memory=True)
    pin.numpy()[:] = res
    with pytest.raises(BpError):
        engine.blastp_host(q, default_params(), pin.numpy(), bad)
    got = engine.blastp_host(q, default_params(), pin.numpy(), off)
    assert_same(got, (ref.counters, ref.hsp_off, ref.hsps_as_array()), "pinned, after a refused call")


def test_host_path_rejects_bad_residues(engine):
    import torch
    res = np.ones(1000, dtype=np.uint8)
    res[777] = 50
    with pytest.raises(BpError):
        engine.blastp_host(enc("WCWHEAL"), default_params(), res, np.array([0, 500, 1000], np.int64))
    # pinned: the streaming launch checks residue codes as it reads them
    pin = torch.empty(len(res), dtype=torch.uint8, pin_memory=True)
    pin.numpy()[:] = res
    with pytest.raises(BpError):
        engine.blastp_host(enc("WCWHEAL"), default_params(), pin.numpy(), np.array([0, 500, 1000], np.int64))
    pin.numpy()[777] = 28
    with pytest.raises(BpError):
        engine.blastp_host(enc("WCWHEAL"), default_params(), pin.numpy(), np.array([0, 500, 1000], np.int64))
    pin.numpy()[777] = 27
    engine.blastp_host(enc("WCWHEAL"), default_params(), pin.numpy(), np.array([0, 500, 1000], np.int64))


def test_host_path_stalled_chunk_times_out(engine, matrix):
    # A chunk whose arrival is never announced (its data is copied, its flag
    # is not): the streaming scan's bounded wait runs out after the set limit,
    # the call returns BP_ERR_TIMEOUT within seconds, and the engine then
    # searches correctly with the default limit restored.
    import time

    import torch
    w = synth.shape2(matrix, rep=4, n_subjects=60_000)      # ~21.6M residues: three 8 MiB chunks
    q = w.queries[0]
    pin = torch.empty(len(w.db.residues), dtype=torch.uint8, pin_memory=True)
    pin.numpy()[:] = w.db.residues
    ref = gpu_search(engine, q, w.db.residues, w.db.offsets)
    for chunk in (1, 0):
        engine.set_upload_wait(5)
        engine.drop_chunk_flag(chunk)
        t0 = time.time()
        with pytest.raises(BpError) as ei:
            engine.blastp_host(q, default_params(), pin.numpy(), w.db.offsets)
        assert ei.value.status == 5, str(ei.value)          # BP_ERR_TIMEOUT
        assert time.time() - t0 < 10.0
        engine.set_upload_wait(20_000)
        got = engine.blastp_host(q, default_params(), pin.numpy(), w.db.offsets)
        assert_same(got, (ref.counters, ref.hsp_off, ref.hsps_as_array()), "after a stalled chunk %d" % chunk)
