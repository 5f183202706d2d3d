"""Shared helpers for the GPU parity tests: run the CUDA path through the C
ABI and the CPU oracle on the same inputs, and compare bit for bit."""
import numpy as np

import oracle

CTX_DEFAULT = (16, 41)   # raw x-drop, raw cutoff


def oracle_search(query, residues, offsets, matrix, params=None, threads=0):
    p = params
    xdrop = p.x_dropoff if p else CTX_DEFAULT[0]
    cutoff = p.cutoff_score if p else CTX_DEFAULT[1]
    window = p.window if p else 40
    thr = p.threshold if p else 11
    table = oracle.build_table(query, matrix, thr)
    return oracle.scan(residues, offsets, query, table, matrix, [(0, xdrop, cutoff)], window=window,
                       threads=threads)


def gpu_search(engine, query, residues, offsets, params=None, first=0, count=-1):
    from blastp_b200 import default_params
    p = params or default_params()
    db = engine.database(residues, offsets)
    q = engine.query(query, p)
    r = engine.search(db, q, first, count).fetch()
    q.close()
    db.close()
    return r


def assert_same(gpu, ref, what=""):
    counters, hoff, hsps = ref
    assert gpu.counters.shape == counters.shape, what
    bad = np.nonzero((gpu.counters != counters).any(axis=1))[0]
    assert len(bad) == 0, "%s: counters differ at subjects %s: gpu %s oracle %s" % (
        what, bad[:5], gpu.counters[bad[:5]].tolist(), counters[bad[:5]].tolist())
    assert (gpu.hsp_off == hoff).all(), what
    g = gpu.hsps_as_array()
    assert g.shape == hsps.shape, (what, g.shape, hsps.shape)
    if len(g):
        rows = np.nonzero((g != hsps).any(axis=1))[0]
        assert len(rows) == 0, "%s: HSPs differ at %s: gpu %s oracle %s" % (
            what, rows[:5], g[rows[:5]].tolist(), hsps[rows[:5]].tolist())
