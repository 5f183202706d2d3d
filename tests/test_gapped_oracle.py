"""CPU tests of the gapped-stage oracle (oracle/gapped.c): hand-computed
known answers, and agreement with the independent pure-Python restatement
(oracle/pyoracle.py) over parameter sweeps.  Parity with NCBI's own gapped
code is unpinned: it is not in the reference tree."""
import numpy as np
import pytest

import oracle
from oracle import pyoracle
from blastp_b200 import synth


def enc(s):
    return synth.encode(s)


def test_identical_sequences_align_end_to_end(matrix):
    # a sequence against itself: no gap beats the diagonal, both extensions run
    # to the ends, the score is the self-score
    rng = np.random.default_rng(2)
    s = synth.residues(rng, 60)
    best, i, j = oracle.gapped_extend(matrix, s, s)
    assert (best, i, j) == (int(matrix[s, s].astype(int).sum()), 60, 60)


def test_one_inserted_letter_costs_open_plus_extend(matrix):
    # the subject is the query with one letter inserted in the middle: the
    # best alignment takes a one-letter gap (11 + 1) and both halves
    rng = np.random.default_rng(3)
    q = synth.residues(rng, 40)
    s = np.concatenate([q[:20], enc("G"), q[20:]]).astype(np.uint8)
    self_score = int(matrix[q, q].astype(int).sum())
    best, i, j = oracle.gapped_extend(matrix, q, s, xdrop=38)
    assert (best, i, j) == (self_score - 12, 40, 41)
    # the same through a whole subject: one ungapped HSP on each half, the
    # better one seeds the gapped HSP and the other lies inside it
    hsps = np.array([[0, 0, 5, 5, 20, int(matrix[q[:20], q[:20]].astype(int).sum())],
                     [20, 21, 25, 26, 20, int(matrix[q[20:], q[20:]].astype(int).sum())]], dtype=np.int32)
    goff, g = oracle.gapped(s, np.array([0, len(s)]), q, np.array([0, 2]), hsps, matrix)
    assert goff.tolist() == [0, 1]
    assert g[0, 0] == self_score - 12 and g[0, 1:5].tolist() == [0, 40, 0, 41]


def test_xdrop_stops_at_a_bad_stretch(matrix):
    # 32 W's against 10 W's, 12 G's, 10 W's: with a small x-drop the
    # extension stops before the G's; with a large one it crosses them, and
    # the cheapest crossing is a 12-letter gap in the query (11 + 12 = 23),
    # not 12 W/G pairs (12 x -2 = -24): 110 - 23 + 110 over 20 query letters
    # and 32 subject letters
    q = enc("W" * 32)
    s = enc("W" * 10 + "G" * 12 + "W" * 10)
    assert int(matrix[enc("W")[0], enc("G")[0]]) == -2
    assert oracle.gapped_extend(matrix, q, s, xdrop=10) == (110, 10, 10)
    assert oracle.gapped_extend(matrix, q, s, xdrop=60) == (197, 20, 32)


def test_empty_sides():
    m = oracle.load_fixture_matrix()
    assert oracle.gapped_extend(m, enc(""), enc("WWW")) == (0, 0, 0)
    assert oracle.gapped_extend(m, enc("WWW"), enc("")) == (0, 0, 0)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_c_oracle_matches_python_restatement(matrix, seed):
    rng = np.random.default_rng(300 + seed)
    q = synth.residues(rng, int(rng.integers(60, 250)))
    db = synth.make_database(rng, 200, [q], 0.3, (20, 90), (0.25, 0.7), matrix, median=160, lo=0, hi=600)
    table = oracle.build_table(q, matrix, 11)
    _, ho, hs = oracle.scan(db.residues, db.offsets, q, table, matrix, [(0, 16, 41)])
    M = matrix.astype(int).tolist()
    for go, ge, xd, cut in ((11, 1, 38, 0), (11, 1, 20, 45), (5, 2, 50, 0), (0, 1, 15, 0), (20, 3, 80, 60)):
        goff, g = oracle.gapped(db.residues, db.offsets, q, ho, hs, matrix, go, ge, xd, cut, threads=3)
        for i in range(db.n_subjects):
            want = pyoracle.gapped_subject(M, list(q), db.subject(i).tolist(),
                                           [tuple(x) for x in hs[ho[i]:ho[i + 1]]], go, ge, xd, cut)
            assert [tuple(x) for x in g[goff[i]:goff[i + 1]]] == want, (go, ge, xd, cut, i)


def test_low_complexity_wide_band(matrix):
    # poly-L against poly-L: many diagonals stay within x-drop of the best
    q = np.full(120, enc("L")[0], dtype=np.uint8)
    s = np.full(150, enc("L")[0], dtype=np.uint8)
    M = matrix.astype(int).tolist()
    for xd in (38, 120):
        assert oracle.gapped_extend(matrix, q, s, xdrop=xd) == pyoracle.gapped_extend(M, list(q), list(s), xd, 11, 1)
