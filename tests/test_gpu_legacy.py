"""GPU parity of the reference-compatible entry points (GPU_BLASTP,
GPU_BLASTP_get_data, GPU_BLASTP_free_memory, GPU_BLASTP_check_memory),
driven with NCBI-style inputs: a lookup table as presence vector + thick
backbone + overflow, and the 4-byte-interleaved GPU database volume.

Expected values: the oracle run on the same subjects padded with zeros to
their group length (which is what the reference kernel scans,
gpu_blastp_kernel.cu:138,151), and the two-slot ring the reference kernel
leaves behind (slot = HSP rank & 1, gpu_blastp_kernel.cu:274)."""
import numpy as np
import pytest

import oracle
from blastp_b200 import _lib, synth
from blastp_b200.legacy import LegacyCall, gpu_volume

pytestmark = pytest.mark.gpu


def expected_ring(counters, hoff, hsps):
    n = len(counters)
    ring = np.zeros((n, 2, 6), dtype=np.int32)
    for s in np.nonzero(counters[:, 1])[0]:
        succ = counters[s, 1]
        for k in range(max(0, succ - 2), succ):
            ring[s, k & 1] = hsps[hoff[s] + k]
    return ring


def run_case(matrix, query, contexts, residues, offsets, blocks, threads, sort=False):
    if sort:   # the reference requires volumes sorted by length (functions.cpp:433-438)
        lens = np.diff(offsets)
        order = np.argsort(lens, kind="stable")
        residues = np.concatenate([residues[offsets[i]:offsets[i + 1]] for i in order]).astype(np.uint8)
        offsets = np.concatenate([[0], np.cumsum(lens[order])]).astype(np.int64)
    G = blocks * threads
    table = oracle.build_table(query, matrix, 11)
    vol, glen, flat, poff = gpu_volume(residues, offsets, G)
    n = len(offsets) - 1
    L = 1
    while L < len(query) + 40:
        L <<= 1
    call = LegacyCall(query, contexts, table[0], table[1], 40, L, vol, glen, n, blocks, threads)
    assert call.check_memory()
    call.run()
    hits, ring = call.get_data()
    full_off, full_hsps = call.get_hsps()
    call.free()
    counters, hoff, hsps = oracle.scan(flat, poff, query, table, matrix, contexts, window=40, diag_mask=L - 1)
    # the complete set, not only the two ring slots: every subject's HSPs
    assert (full_off == hoff).all()
    assert full_hsps.shape == hsps.shape and (full_hsps == hsps).all()
    return hits, ring, counters, hoff, hsps


@pytest.mark.parametrize("blocks,threads,sort", [(4, 8, False), (2, 64, True), (1, 1, False)])
def test_gpu_blastp_drop_in(matrix, blocks, threads, sort):
    w = synth.shape1(matrix, n_subjects=1500)
    q = w.queries[0]
    hits, ring, counters, hoff, hsps = run_case(matrix, q, [(0, 16, 41)], w.db.residues, w.db.offsets,
                                                blocks, threads, sort)
    assert (hits == counters).all()
    assert (ring == expected_ring(counters, hoff, hsps)).all()
    assert counters[:, 1].sum() > 0


def test_gpu_blastp_full_hsp_set_beyond_ring(matrix):
    # subjects holding several separated copies of query segments have more
    # HSPs than the two ring slots; GPU_BLASTP_get_hsps returns all of them
    rng = np.random.default_rng(21)
    q = synth.residues(rng, 400)
    parts = []
    for i in range(300):
        if i % 3 == 0:
            segs = [q[a:a + 60] for a in (0, 100, 200, 300)]
            fill = [synth.residues(rng, 50) for _ in segs]
            parts.append(np.concatenate([x for pair in zip(fill, segs) for x in pair]))
        else:
            parts.append(synth.residues(rng, int(rng.integers(50, 400))))
    res = np.concatenate(parts).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum([len(p) for p in parts])]).astype(np.int64)
    hits, ring, counters, hoff, hsps = run_case(matrix, q, [(0, 16, 41)], res, off, 4, 32)
    assert (counters[:, 1] > 2).sum() >= 90
    assert (hits == counters).all()
    assert (ring == expected_ring(counters, hoff, hsps)).all()


def test_gpu_blastp_multi_context(matrix):
    # three queries concatenated with gap-letter separators, one context each
    rng = np.random.default_rng(9)
    qs = [synth.residues(rng, n) for n in (120, 300, 80)]
    parts, ctx, pos = [], [], 0
    for i, q in enumerate(qs):
        ctx.append((pos, 16 - 2 * i, 41 - 5 * i))
        parts.append(q)
        pos += len(q)
        if i + 1 < len(qs):
            parts.append(np.zeros(1, dtype=np.uint8))
            pos += 1
    query = np.concatenate(parts).astype(np.uint8)
    db = synth.make_database(rng, 1200, qs, 0.05, (60, 150), (0.3, 0.5), matrix)
    hits, ring, counters, hoff, hsps = run_case(matrix, query, ctx, db.residues, db.offsets, 8, 16)
    assert (hits == counters).all()
    assert (ring == expected_ring(counters, hoff, hsps)).all()


def test_check_availability_and_memory_gate(matrix):
    L = _lib.lib()
    assert L.GPU_BLAST_check_availability() == 1
    w = synth.shape1(matrix, n_subjects=64)
    q = w.queries[0]
    table = oracle.build_table(q, matrix, 11)
    vol, glen, flat, poff = gpu_volume(w.db.residues, w.db.offsets, 32)
    ok = LegacyCall(q, [(0, 16, 41)], table[0], table[1], 40, 512, vol, glen, 64, 1, 32)
    assert ok.check_memory()
    # the engine sizes its own diagonal array from query + window, whatever
    # the caller's diag table is; a query whose array cannot fit shared
    # memory is refused
    assert LegacyCall(q, [(0, 16, 41)], table[0], table[1], 40, 1 << 20, vol, glen, 64, 1, 32).check_memory()
    qlong = synth.residues(np.random.default_rng(9), 60_000)
    tl = oracle.build_table(qlong, matrix, 11)
    huge = LegacyCall(qlong, [(0, 16, 41)], tl[0], tl[1], 40, 1 << 16, vol, glen, 64, 1, 32)
    assert not huge.check_memory()      # diagonal array beyond shared memory
