"""CPU tests of the oracle itself: pinned against the reference's scoring
table (fixture) and hand-computed known answers, and cross-checked against
the independent pure-Python restatement."""
import numpy as np
import pytest

import oracle
from oracle import pyoracle
from blastp_b200 import synth

CTX = [(0, 16, 41)]


def enc(s):
    return synth.encode(s)


def test_fixture_matrix_is_symmetric_and_sentinel(matrix):
    assert matrix.shape == (28, 28)
    assert (matrix == matrix.T).all()
    assert (matrix[0] == -128).all() and (matrix[:, 0] == -128).all()
    # every standard residue's self-score is >= 4, so every exact word of
    # standard residues scores >= 12 >= T=11
    std = synth.STANDARD_CODES
    assert matrix[std, std].min() == 4


def test_table_kat_aaa(matrix):
    # S(A,x) <= 4 with equality only for A, and the next best is 1 (S):
    # 4+4+1 = 9 < 11, so "AAA" has exactly one neighbour: itself.
    start, ent = oracle.build_table(enc("AAA"), matrix, 11)
    assert len(ent) == 1 and ent[0] == 0
    c = pyoracle.code3(*enc("AAA"))
    assert start[c + 1] - start[c] == 1


def test_table_kat_ccc(matrix):
    # S(C,C)=9 and S(C,x) in [-4, 0] otherwise: a word scores >= 11 against
    # CCC iff it has at least two C's: 3*26 + 1 = 79 words over letters 1..27.
    start, ent = oracle.build_table(enc("CCC"), matrix, 11)
    assert len(ent) == 79


def test_table_exact_word_below_threshold(matrix):
    # X scores -1 with itself: "XXX" self-scores -3 < 11, so only the exact
    # word is listed (NCBI adds exact matches scoring below T).
    start, ent = oracle.build_table(enc("XXX"), matrix, 11)
    assert len(ent) == 1
    c = pyoracle.code3(*enc("XXX"))
    assert start[c + 1] - start[c] == 1


def test_extend_kat_identical_alternating(matrix):
    # subject = query = WCWCWCWCWC; second hit at 5 (C W C: 9, 20, 29 -> shift 3),
    # left walk from 7 to 0 is monotone (80 at 8 letters), reaches s_left=3,
    # right walk over W, C adds 20 and runs off the end: s_last = 10.
    s = enc("WCWCWCWCWC")
    out = oracle.extend_two_hit(matrix, s, s, 3, 5, 5, 16)
    assert out == (0, 0, 10, 100, 10, 1)
    M = matrix.astype(int).tolist()
    assert pyoracle.extend_two_hit(M, list(s), list(s), 3, 5, 5, 16) == (0, 0, 10, 100, 10, True)


def test_extend_kat_left_fails(matrix):
    # Second word WWW at s=10 (q=10); before it the subject is G's against
    # the query's P's (S(P,G) = -2): the left walk collects 33 over WWW then
    # drops by 2 per letter; it stops after 8 letters (33-16 = 17), so it
    # never reaches s_left = 1 and no right extension happens.
    q = enc("PPPPPPPPPPWWWAAAA")
    s = enc("GGGGGGGGGGWWWAAAA")
    hq, hs, ln, score, s_last, rext = oracle.extend_two_hit(matrix, s, q, 1, 10, 10, 16)
    assert rext == 0 and score == 33 and ln == 3 and hs == 10 and hq == 10


def _hand_table(entries_by_word):
    start = np.zeros((1 << 15) + 1, dtype=np.uint32)
    cells = {pyoracle.code3(*enc(w)): qs for w, qs in entries_by_word.items()}
    ent = []
    for c in range(1 << 15):
        start[c] = len(ent)
        ent.extend(cells.get(c, []))
    start[1 << 15] = len(ent)
    return start, np.array(ent if ent else [0], dtype=np.uint16)[:len(ent)]


@pytest.mark.parametrize("D,expect_ext", [(2, 0), (3, 1), (39, 1), (40, 0), (41, 0)])
def test_scan_window_edges(matrix, D, expect_ext):
    # Table: WCW -> query offsets {0, D}.  Subject has WCW at s1=5 and s1+D, so
    # hits (q=0, s1) and (q=D, s1+D) share a diagonal at distance D.  Two-hit
    # fires iff 3 <= D < 40 (gpu_blastp_kernel.cu:224-234).
    qlen = D + 3
    q = np.full(qlen, enc("G")[0], dtype=np.uint8)
    q[0:3] = enc("WCW")
    q[D:D + 3] = enc("WCW")
    subj = np.full(5 + D + 3 + 5, enc("G")[0], dtype=np.uint8)
    subj[5:8] = enc("WCW")
    subj[5 + D:8 + D] = enc("WCW")
    table = _hand_table({"WCW": [0, D]})
    off = np.array([0, len(subj)], dtype=np.int64)
    counters, hoff, hsps = oracle.scan(subj, off, q, table, matrix, CTX)
    assert counters[0, 0] == 4          # 2 positions x 2 listed offsets
    assert counters[0, 2] == expect_ext


def test_scan_identical_sequences_one_hsp_per_seed_diagonal(matrix):
    # Query = subject (standard residues score >= 4 with themselves): on the
    # main diagonal the first two-hit pair extends left to 0 and right to the
    # end, so the main diagonal yields exactly one HSP covering everything
    # with the full self-score, and the flag then skips every later hit there.
    rng = np.random.default_rng(7)
    s = synth.residues(rng, 120)
    table = oracle.build_table(s, matrix, 11)
    off = np.array([0, len(s)], dtype=np.int64)
    counters, hoff, hsps = oracle.scan(s, off, s, table, matrix, CTX)
    main = hsps[hsps[:, 0] == hsps[:, 1]]
    self_score = int(matrix[s, s].astype(int).sum())
    assert len(main) == 1
    assert tuple(main[0][[0, 1, 4, 5]]) == (0, 0, 120, self_score)


def test_scan_short_and_empty_subjects(matrix):
    q = enc("WCWCWCWCWC")
    table = oracle.build_table(q, matrix, 11)
    subj = np.concatenate([enc("WC"), enc(""), enc("WCW"), enc("WCWCWC")])
    off = np.array([0, 2, 2, 5, 11], dtype=np.int64)
    counters, hoff, hsps = oracle.scan(subj, off, q, table, matrix, CTX)
    assert counters[0].tolist() == [0, 0, 0]      # shorter than a word
    assert counters[1].tolist() == [0, 0, 0]      # empty
    assert counters[2, 0] > 0 and counters[2, 2] == 0   # one word: hits, no pair
    assert hoff.tolist()[0] == 0


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_c_oracle_matches_python_restatement(matrix, seed):
    rng = np.random.default_rng(100 + seed)
    q = synth.residues(rng, int(rng.integers(20, 200)))
    db = synth.make_database(rng, 150, [q], 0.1, (20, 60), (0.3, 0.6), matrix, median=120, lo=0, hi=400)
    table = oracle.build_table(q, matrix, 11)
    cells = pyoracle.build_table(list(q), matrix.astype(int).tolist(), 11)
    start, ent = table
    for c, qs in cells.items():
        assert ent[start[c]:start[c + 1]].tolist() == qs
    assert int(start[-1]) == sum(len(v) for v in cells.values())
    counters, hoff, hsps = oracle.scan(db.residues, db.offsets, q, table, matrix, CTX, threads=3)
    mask = oracle.diag_mask_for(len(q), 40)
    M = matrix.astype(int).tolist()
    for i in range(db.n_subjects):
        cnt, hl = pyoracle.scan_subject(db.subject(i).tolist(), list(q), cells, M, CTX, 40, mask)
        assert tuple(counters[i]) == cnt
        assert [tuple(x) for x in hsps[hoff[i]:hoff[i + 1]]] == hl


def test_multi_context_selects_cutoff_per_context(matrix):
    # Two contexts concatenated with a gap-letter separator (as NCBI
    # concatenates queries): the second context gets an unreachable cutoff,
    # so only HSPs whose second hit lies in context 0 survive.
    rng = np.random.default_rng(5)
    a = synth.residues(rng, 80)
    b = synth.residues(rng, 80)
    q = np.concatenate([a, [0], b]).astype(np.uint8)
    subj = np.concatenate([a, b]).astype(np.uint8)
    off = np.array([0, len(subj)], dtype=np.int64)
    table = oracle.build_table(q, matrix, 11)
    both = oracle.scan(subj, off, q, table, matrix, [(0, 16, 41), (81, 16, 41)])
    only0 = oracle.scan(subj, off, q, table, matrix, [(0, 16, 41), (81, 16, 10 ** 6)])
    assert len(both[2]) > len(only0[2]) > 0
    assert (only0[2][:, 2] < 81).all()
