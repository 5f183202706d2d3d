"""GPU parity of the gapped stage (bp_gapped_run): the device's gapped HSPs
and per-subject counts equal the oracle's (oracle/gapped.c) bit for bit, run
on the same ungapped HSPs, over parameter sweeps, edge cases and the
wide-band path (a band wider than the ring redone by a second launch).  The
oracle restates the published algorithm; parity with NCBI's own gapped code
is unpinned (it is not in the reference tree)."""
import numpy as np
import pytest

import oracle
from blastp_b200 import BpError, default_params, gapped_params, synth
from helpers import gpu_search, oracle_search

pytestmark = pytest.mark.gpu


def run_gapped(engine, query, residues, offsets, ring=0, **kw):
    d = engine.database(residues, offsets)
    q = engine.query(query, default_params())
    r = engine.search(d, q)
    g = r.gapped(gapped_params(**kw), ring_columns=ring)
    u = r.fetch()
    r.close()
    q.close()
    d.close()
    return u, g


def check(engine, matrix, query, residues, offsets, ring=0, **kw):
    u, g = run_gapped(engine, query, residues, offsets, ring=ring, **kw)
    p = gapped_params(**kw)
    want_off, want = oracle.gapped(residues, offsets, query, u.hsp_off, u.hsps_as_array(), matrix, p.gap_open,
                                   p.gap_extend, p.x_dropoff, p.cutoff_score)
    assert (g.counters[:, 0] == np.diff(u.hsp_off)).all()
    assert (g.counters[:, 1] == np.diff(want_off)).all(), "gapped counts differ at %s" % (
        np.nonzero(g.counters[:, 1] != np.diff(want_off))[0][:5])
    assert (g.off == want_off).all()
    got = g.hsps_as_array()
    assert got.shape == want.shape
    rows = np.nonzero((got != want).any(axis=1))[0]
    assert len(rows) == 0, "gapped HSPs differ at %s: gpu %s oracle %s" % (rows[:3], got[rows[:3]].tolist(),
                                                                          want[rows[:3]].tolist())
    return u, g


def test_config1_full(engine, matrix):
    w = synth.shape1(matrix)
    u, g = check(engine, matrix, w.queries[0], w.db.residues, w.db.offsets)
    assert len(g.hsps) > 100 and g.counters[:, 2].sum() >= len(g.hsps)


@pytest.mark.parametrize("go,ge,xd,cut", [(11, 1, 38, 0), (11, 1, 20, 60), (5, 2, 60, 0), (0, 1, 15, 0),
                                          (20, 3, 100, 50)])
def test_parameter_sweep(engine, matrix, go, ge, xd, cut):
    w = synth.shape1(matrix, rep=7, n_subjects=3000)
    check(engine, matrix, w.queries[0], w.db.residues, w.db.offsets, gap_open=go, gap_extend=ge, x_dropoff=xd,
          cutoff_score=cut)


def test_many_hsps_per_subject_and_containment(engine, matrix):
    # several planted copies of query segments per subject, some overlapping:
    # later HSPs inside earlier gapped HSPs are skipped
    rng = np.random.default_rng(17)
    q = synth.residues(rng, 300)
    subs = []
    for i in range(400):
        parts = [synth.residues(rng, int(rng.integers(0, 40)))]
        for _ in range(int(rng.integers(1, 6))):
            a = int(rng.integers(0, 240))
            seg = q[a:a + int(rng.integers(30, 60))].copy()
            if rng.random() < 0.5 and len(seg) > 20:        # an indel inside the copy
                k = int(rng.integers(5, len(seg) - 5))
                seg = np.concatenate([seg[:k], synth.residues(rng, int(rng.integers(1, 4))), seg[k:]])
            parts.append(seg)
            parts.append(synth.residues(rng, int(rng.integers(0, 50))))
        subs.append(np.concatenate(parts).astype(np.uint8))
    res = np.concatenate(subs).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum([len(s) for s in subs])]).astype(np.int64)
    u, g = check(engine, matrix, q, res, off)
    assert (g.counters[:, 2] < g.counters[:, 0]).any()        # some skipped as contained


def test_sequence_ends_and_identical(engine, matrix):
    # HSPs touching both ends of query and subject, the query itself as a
    # subject, empty and 1-letter subjects
    rng = np.random.default_rng(23)
    q = synth.residues(rng, 200)
    parts = [q.copy(), q[:50].copy(), q[-50:].copy(), synth.encode(""), synth.encode("W"),
             np.concatenate([q[150:], synth.residues(rng, 30), q[:40]]).astype(np.uint8)]
    parts += [synth.residues(rng, int(n)) for n in rng.integers(0, 400, size=300)]
    res = np.concatenate(parts).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum([len(x) for x in parts])]).astype(np.int64)
    u, g = check(engine, matrix, q, res, off)
    assert g.hsps[0]["score"] == int(matrix[q, q].astype(int).sum())


def test_wide_band_second_launch(engine, matrix):
    # low-complexity subjects against a low-complexity query give wide bands:
    # with a 64-column ring they are redone by the wide-ring launch, with the
    # same results as the default ring
    rng = np.random.default_rng(31)
    q = np.concatenate([np.full(150, synth.encode("L")[0]), synth.residues(rng, 100)]).astype(np.uint8)
    parts = [np.full(int(n), synth.encode("L")[0], dtype=np.uint8) for n in (60, 200, 400, 900)]
    parts += [synth.residues(rng, int(n)) for n in rng.integers(50, 400, size=200)]
    res = np.concatenate(parts).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum([len(x) for x in parts])]).astype(np.int64)
    for xd in (38, 150):
        check(engine, matrix, q, res, off, ring=64, x_dropoff=xd)
        check(engine, matrix, q, res, off, x_dropoff=xd)


def test_no_hsps(engine, matrix):
    rng = np.random.default_rng(41)
    q = synth.residues(rng, 30)
    res = synth.residues(rng, 2000)
    off = np.array([0, 700, 2000], dtype=np.int64)
    u, g = check(engine, matrix, q, res, off, cutoff_score=10 ** 6)
    assert len(g.hsps) == 0


def test_rejects_bad_parameters(engine, matrix):
    w = synth.shape1(matrix, n_subjects=200)
    with pytest.raises(BpError):
        run_gapped(engine, w.queries[0], w.db.residues, w.db.offsets, gap_extend=0)
    with pytest.raises(BpError):
        run_gapped(engine, w.queries[0], w.db.residues, w.db.offsets, ring=100)
