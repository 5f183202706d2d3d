"""The oracle pinned to the reference's own code (CPU).

oracle/_ref holds the reference's gpu_blastp_kernel.cu (the two-hit kernel and
its three extenders, gpu_blastp_kernel.cu:42-320,341-549) compiled unmodified
for the host and run one POSIX thread per CUDA thread (oracle/ref_driver.cpp).
Every case here runs it and the oracle (oracle.c) on the same inputs and
requires identical per-subject counters and identical records:
  - libref_ring64: the reference kernel with its record ring widened to 64,
    so every record of every subject survives; compared with the oracle's
    complete HSP set, in discovery order;
  - libref_ring2: the kernel exactly as shipped (two ring slots); compared
    with the ring the oracle's set leaves (slot = rank & 1).
The reference kernel scans each subject over its group's padded length (zeros
after the subject), so the oracle is given the same padded subjects; one case
uses groups of equal lengths that are multiples of 64, where the padded and
the true lengths coincide, and compares with the oracle on the unpadded
database directly.

What stays unpinned is NCBI's own code the reference calls but does not ship:
the neighbour-word rule (BlastAaLookupTableNew) and the cutoff / x-drop raw
values (BlastInitialWordParametersNew); both tables come from the oracle here.
"""
import numpy as np
import pytest

import oracle
from oracle import refkernel
from blastp_b200 import synth

pytestmark = pytest.mark.skipif(not (refkernel.available(64) and refkernel.available(2)),
                                reason="oracle/_ref not built (make -C oracle ref needs the reference tree)")

CTX = [(0, 16, 41)]


def enc(s):
    return synth.encode(s)


def check(residues, offsets, query, matrix, contexts=CTX, window=40, blocks=1, threads=64,
          matrix_bytes=28 * 28, table=None, threshold=11):
    table = table if table is not None else oracle.build_table(query, matrix, threshold)
    hits, ring, glen = refkernel.two_hit(residues, offsets, query, table, matrix, contexts, window=window,
                                         blocks=blocks, threads=threads, matrix_bytes=matrix_bytes, slots=64)
    flat, poff = refkernel.padded(residues, offsets, glen)
    dmask = oracle.diag_mask_for(len(query), window)
    counters, hoff, hsps = oracle.scan(flat, poff, query, table, matrix, contexts, window=window,
                                       diag_mask=dmask)
    bad = np.nonzero((hits != counters).any(axis=1))[0]
    assert len(bad) == 0, "counters differ at %s: ref %s oracle %s" % (
        bad[:5], hits[bad[:5]].tolist(), counters[bad[:5]].tolist())
    assert counters[:, 1].max(initial=0) <= 64, "a subject has more records than the widened ring holds"
    full = refkernel.ring_of(counters, hoff, hsps, 64)
    rows = np.nonzero((full != ring).any(axis=(1, 2)))[0]
    assert len(rows) == 0, "records differ at subjects %s" % rows[:5]
    hits2, ring2, _ = refkernel.two_hit(residues, offsets, query, table, matrix, contexts, window=window,
                                        blocks=blocks, threads=threads, matrix_bytes=matrix_bytes, slots=2)
    assert (hits2 == hits).all()
    assert (ring2 == refkernel.ring_of(counters, hoff, hsps, 2)).all()
    return counters, hoff, hsps, glen


def test_config1_full(matrix):
    # one 300-aa query against 10,000 subjects
    w = synth.shape1(matrix)
    c, hoff, hsps, _ = check(w.db.residues, w.db.offsets, w.queries[0], matrix)
    assert c[:, 0].sum() > 10 ** 6 and len(hsps) > 100


def test_config2_sample_50k(matrix):
    # the 500-aa query against 50,000 subjects of the 1M-subject workload's distribution
    w = synth.shape2(matrix, n_subjects=50_000)
    c, hoff, hsps, _ = check(w.db.residues, w.db.offsets, w.queries[0], matrix)
    assert len(hsps) > 500 and c[:, 1].max() >= 2


@pytest.mark.parametrize("blocks,threads", [(1, 16), (1, 32), (3, 16), (2, 128)])
def test_launch_shapes(matrix, blocks, threads):
    # the group size (blocks x threads) changes the interleaving and padding only
    w = synth.shape1(matrix, rep=3, n_subjects=1500)
    check(w.db.residues, w.db.offsets, w.queries[0], matrix, blocks=blocks, threads=threads)


def test_many_records_per_subject(matrix):
    # planted copies of the query: subjects with several records each, all of
    # which survive in the widened ring and in discovery order
    rng = np.random.default_rng(11)
    q = synth.residues(rng, 200)
    subs = []
    for i in range(300):
        parts = [synth.residues(rng, int(rng.integers(5, 60)))]
        for _ in range(int(rng.integers(1, 5))):
            a = int(rng.integers(0, 150))
            parts.append(q[a:a + int(rng.integers(25, 50))])
            parts.append(synth.residues(rng, int(rng.integers(41, 80))))
        subs.append(np.concatenate(parts).astype(np.uint8))
    res = np.concatenate(subs).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum([len(s) for s in subs])]).astype(np.int64)
    c, hoff, hsps, _ = check(res, off, q, matrix)
    assert c[:, 1].max() >= 3


@pytest.mark.parametrize("D", [2, 3, 39, 40, 41])
def test_window_edges(matrix, D):
    q = np.full(D + 3, enc("G")[0], dtype=np.uint8)
    q[0:3] = enc("WCW")
    q[D:D + 3] = enc("WCW")
    subj = np.full(5 + D + 3 + 5, enc("G")[0], dtype=np.uint8)
    subj[5:8] = enc("WCW")
    subj[5 + D:8 + D] = enc("WCW")
    start = np.zeros((1 << 15) + 1, dtype=np.uint32)
    cell = (int(enc("W")[0]) << 10) | (int(enc("C")[0]) << 5) | int(enc("W")[0])
    start[cell + 1:] = 2
    table = (start, np.array([0, D], dtype=np.uint16))
    c, _, _, _ = check(subj, np.array([0, len(subj)], dtype=np.int64), q, matrix, table=table)
    assert c[0, 2] == (1 if 3 <= D < 40 else 0)


def test_identical_sequences(matrix):
    rng = np.random.default_rng(7)
    s = synth.residues(rng, 120)
    c, _, hsps, _ = check(s, np.array([0, len(s)], dtype=np.int64), s, matrix)
    assert (hsps[:, 0] == hsps[:, 1]).sum() == 1


def test_left_walk_fails(matrix):
    q = enc("PPPPPPPPPPWWWAAAA")
    s = enc("GGGGGGGGGGWWWAAAA")
    check(s, np.array([0, len(s)], dtype=np.int64), q, matrix)


def test_short_and_empty_subjects(matrix):
    q = enc("WCWCWCWCWC")
    subj = np.concatenate([enc("WC"), enc(""), enc("WCW"), enc("WCWCWC"), enc("")]).astype(np.uint8)
    off = np.array([0, 2, 2, 5, 11, 11], dtype=np.int64)
    check(subj, off, q, matrix, threads=16)


def test_multi_context(matrix):
    rng = np.random.default_rng(5)
    a = synth.residues(rng, 80)
    b = synth.residues(rng, 80)
    q = np.concatenate([a, [0], b]).astype(np.uint8)
    w = synth.make_database(rng, 400, [a, b], 0.3, (20, 60), (0.3, 0.7), matrix, median=150, lo=0, hi=500)
    for ctx in ([(0, 16, 41), (81, 16, 41)], [(0, 16, 41), (81, 9, 30)], [(0, 16, 41), (81, 16, 10 ** 6)]):
        check(w.residues, w.offsets, q, matrix, contexts=ctx)


def test_parameter_sweep(matrix):
    rng = np.random.default_rng(21)
    q = synth.residues(rng, 250)
    w = synth.make_database(rng, 600, [q], 0.2, (30, 90), (0.25, 0.6), matrix, median=200, lo=0, hi=900)
    for thr, window, xdrop, cutoff in ((11, 40, 16, 41), (13, 40, 16, 41), (11, 20, 10, 30), (11, 60, 24, 50)):
        check(w.residues, w.offsets, q, matrix, contexts=[(0, xdrop, cutoff)], window=window, threshold=thr)


def test_ambiguity_letters(matrix):
    # B, Z, X, U, *, O, J in query and subjects: scored from the full table
    rng = np.random.default_rng(9)
    q = synth.residues(rng, 150)
    q[::17] = rng.integers(1, 28, size=len(q[::17]))
    w = synth.make_database(rng, 300, [q], 0.3, (20, 60), (0.4, 0.8), matrix, median=150, lo=0, hi=500)
    res = w.residues.copy()
    res[::23] = rng.integers(1, 28, size=len(res[::23]))
    check(res, w.offsets, q, matrix)


def test_shipped_matrix_size_on_standard_letters(matrix):
    # the reference ships the first 640 bytes of the table (gpu_cpu_common.h:28);
    # over the 20 standard letters the outcome equals the whole table's
    w = synth.shape1(matrix, rep=5, n_subjects=800)
    check(w.db.residues, w.db.offsets, w.queries[0], matrix, matrix_bytes=640)


def test_true_lengths_when_groups_need_no_padding(matrix):
    # groups of 16 subjects that all have the same length, a multiple of 64:
    # the reference scans exactly the subjects, so the oracle on the unpadded
    # database (the engine's semantics) must give the same answer
    rng = np.random.default_rng(3)
    q = synth.residues(rng, 300)
    lens = np.repeat(rng.integers(1, 12, size=40) * 64, 16)
    res = np.concatenate([synth.residues(rng, int(n)) for n in lens]).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    # plant homologous segments so that records exist
    for s in range(0, len(lens), 3):
        a = int(rng.integers(0, 240))
        seg = q[a:a + 50]
        p = int(off[s]) + int(rng.integers(0, int(lens[s]) - 50))
        res[p:p + 50] = seg
    c, hoff, hsps, glen = check(res, off, q, matrix, threads=16)
    assert (glen == lens).all()
    table = oracle.build_table(q, matrix, 11)
    c2, hoff2, hsps2 = oracle.scan(res, off, q, table, matrix, CTX)
    assert (c2 == c).all() and (hoff2 == hoff).all() and (hsps2 == hsps).all()
    assert len(hsps) > 10
