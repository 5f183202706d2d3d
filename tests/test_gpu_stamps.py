"""GPU parity where the diagonal stamp offset is reset or moved.

The scan keeps one stamp offset per warp; with 16-bit diagonal entries the
offset is moved inside any subject longer than about 16,000 - Q letters and
reset every few dozen subjects, with 32-bit entries (query + window above
8,192) almost never.  These cases put extensions, pending marks and
extension ends across those points: subjects of 40-70K letters made of
mutated and exact query copies, runs of short subjects after them, both
sides of the 16-/32-bit boundary, a short query with a very large window,
and the batched kernel, whose warps share one array between queries of
different lengths.  Everything is checked bit for bit against the oracle or
the single-query path."""
import numpy as np
import pytest

from blastp_b200 import default_params, synth
from helpers import assert_same, gpu_search, oracle_search

pytestmark = pytest.mark.gpu


def _long_subjects(rng, q, matrix, n_letters):
    """Subjects that keep the two-hit state busy for n_letters letters: mutated
    query copies (60-90 % identity) between random spacers, exact copies
    back to back (right walks that run to the query's end), random letters,
    then a run of short subjects."""
    tabs = synth.substitution_tables(matrix)
    parts = []
    # mutated copies with spacers
    acc, pieces = 0, []
    while acc < n_letters:
        ident = rng.uniform(0.6, 0.9)
        lo = int(rng.integers(0, max(1, len(q) - 60)))
        hi = int(min(len(q), lo + rng.integers(60, 400)))
        pieces.append(synth.mutate(rng, q[lo:hi], ident, tabs))
        pieces.append(synth.residues(rng, int(rng.integers(0, 90))))
        acc += len(pieces[-1]) + len(pieces[-2])
    parts.append(np.concatenate(pieces))
    # exact copies back to back
    reps = max(1, n_letters // max(1, len(q)))
    parts.append(np.tile(q, reps))
    # random
    parts.append(synth.residues(rng, n_letters))
    # lengths around one 16-bit offset period
    for n in (16_200, 16_300, 16_384, 16_500):
        seg = synth.residues(rng, n)
        k = min(len(q), 300)
        seg[n - k - 50:n - 50] = q[:k]          # a homolog near the end
        parts.append(seg)
    # many short subjects after the long ones (offset resets at subject starts)
    for _ in range(400):
        n = int(rng.integers(0, 400))
        s = synth.residues(rng, n)
        if n > 80 and rng.random() < 0.3:
            k = min(n - 10, len(q), 70)
            s[5:5 + k] = synth.mutate(rng, q[:k], 0.7, tabs)
        parts.append(s)
    res = np.concatenate(parts).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum([len(p) for p in parts])]).astype(np.int64)
    return res, off


@pytest.mark.parametrize("qlen", [100, 500, 3000, 8100, 8200])
def test_long_subjects(engine, matrix, qlen):
    # 100: extensions at once; 500, 3000: queued; 8100: 16-bit entries with
    # the shortest offset period; 8200: 32-bit entries
    rng = np.random.default_rng(7000 + qlen)
    q = synth.residues(rng, qlen)
    res, off = _long_subjects(rng, q, matrix, 70_000 if qlen < 8000 else 40_000)
    ref = oracle_search(q, res, off, matrix)
    assert ref[0][:, 2].sum() > 1000, "the workload should extend often"
    assert_same(gpu_search(engine, q, res, off), ref, "qlen %d" % qlen)


def test_large_window_short_query(engine, matrix):
    # query + window above 8,192: 32-bit entries for a 100-letter query
    rng = np.random.default_rng(77)
    q = synth.residues(rng, 100)
    res, off = _long_subjects(rng, q, matrix, 30_000)
    p = default_params(window=9000)
    assert_same(gpu_search(engine, q, res, off, p), oracle_search(q, res, off, matrix, p), "window 9000")


@pytest.mark.parametrize("pack", [0, 512])
def test_batched_long_subjects(engine, matrix, pack):
    rng = np.random.default_rng(99)
    lens = [60, 150, 340, 500, 1200, 2500, 45, 90]
    qs = [synth.residues(rng, n) for n in lens]
    res, off = _long_subjects(rng, qs[3], matrix, 50_000)
    d = engine.database(res, off)
    hs = [engine.query(q) for q in qs]
    singles = [engine.search(d, h).fetch() for h in hs]
    b = engine.search_batch(d, hs, chunk_residues=1 << 16, pack_residues=pack)
    for i, s in enumerate(singles):
        assert_same(b.fetch(i), (s.counters, s.hsp_off, s.hsps_as_array()), "pack %d query %d" % (pack, i))
    for i in (0, 3, 5):
        assert_same(singles[i], oracle_search(qs[i], res, off, matrix), "single query %d vs oracle" % i)
    b.close()
    for h in hs:
        h.close()
    d.close()
