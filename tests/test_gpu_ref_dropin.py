"""The drop-in on the GPU against the reference's own kernel, with no oracle in
between: GPU_BLASTP + GPU_BLASTP_get_data on the 4-byte-interleaved volume
give per-subject counters and a two-slot record ring; the reference's
gpu_blastp_kernel.cu, host-compiled unmodified into oracle/_ref, run on the
same volume layout (same blocks x threads group size, groups padded to 64)
with the same table and parameters, must leave identical counters and an
identical ring.  Skipped where oracle/_ref was not built."""
import numpy as np
import pytest

import oracle
from oracle import refkernel
from blastp_b200 import synth
from blastp_b200.legacy import LegacyCall, gpu_volume

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refkernel.available(2), reason="oracle/_ref not built")]


def drop_in(query, contexts, table, residues, offsets, blocks, threads):
    G = blocks * threads
    vol, glen, _, _ = gpu_volume(residues, offsets, G)
    L = 1
    while L < len(query) + 40:
        L <<= 1
    call = LegacyCall(query, contexts, table[0], table[1], 40, L, vol, glen, len(offsets) - 1, blocks, threads)
    call.run()
    hits, ring = call.get_data()
    call.free()
    return hits, ring


@pytest.mark.parametrize("blocks,threads", [(4, 16), (2, 64), (1, 128)])
def test_drop_in_equals_reference_kernel(matrix, blocks, threads):
    w = synth.shape1(matrix, rep=2, n_subjects=3000)
    q = w.queries[0]
    table = oracle.build_table(q, matrix, 11)
    ctx = [(0, 16, 41)]
    hits, ring = drop_in(q, ctx, table, w.db.residues, w.db.offsets, blocks, threads)
    rh, rring, _ = refkernel.two_hit(w.db.residues, w.db.offsets, q, table, matrix, ctx, blocks=blocks,
                                     threads=threads, slots=2)
    assert (hits == rh).all()
    assert (ring == rring).all()
    assert hits[:, 1].sum() > 10


def test_drop_in_multi_context_equals_reference_kernel(matrix):
    rng = np.random.default_rng(19)
    qs = [synth.residues(rng, n) for n in (150, 260, 90)]
    parts, ctx, pos = [], [], 0
    for i, q in enumerate(qs):
        ctx.append((pos, 16 - 3 * i, 41 - 6 * i))
        parts.append(q)
        pos += len(q)
        if i + 1 < len(qs):
            parts.append(np.zeros(1, dtype=np.uint8))
            pos += 1
    query = np.concatenate(parts).astype(np.uint8)
    db = synth.make_database(rng, 2000, qs, 0.05, (60, 150), (0.3, 0.5), matrix)
    table = oracle.build_table(query, matrix, 11)
    hits, ring = drop_in(query, ctx, table, db.residues, db.offsets, 4, 32)
    rh, rring, _ = refkernel.two_hit(db.residues, db.offsets, query, table, matrix, ctx, blocks=4, threads=32,
                                     slots=2)
    assert (hits == rh).all()
    assert (ring == rring).all()
    assert (hits[:, 1] > 2).sum() > 0      # subjects whose ring wrapped
