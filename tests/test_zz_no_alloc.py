"""bp_search_noalloc: the plain search for callers that cannot allocate device
memory (a fixed device-memory budget handed out at start-up, a latency path
where cudaMalloc would synchronise the device, or buffers owned by an outside
allocator).  It must give exactly what bp_search gives, call after call, while
using only the caller's buffers plus the library's static scratch array.

This file is named to be collected last, so a run that stops at the first
failure has already run every other test; it also passes on its own in a
fresh process (the first call there performs the per-device set-up)."""
import ctypes

import numpy as np
import pytest
import torch

from blastp_b200 import Engine, default_params, lib, synth
from helpers import assert_same

pytestmark = pytest.mark.gpu


def run_noalloc(query, residues, offsets, params, hsp_cap):
    dev = torch.device("cuda", 0)
    q = torch.from_numpy(np.ascontiguousarray(query, dtype=np.uint8)).to(dev)
    res = torch.from_numpy(np.ascontiguousarray(residues, dtype=np.uint8)).to(dev)
    off = torch.from_numpy(np.ascontiguousarray(offsets, dtype=np.int64)).to(dev)
    n = len(offsets) - 1
    counters = torch.full((n, 3), -7, dtype=torch.int32, device=dev)       # garbage: must be overwritten
    hoff = torch.full((n + 1,), -7, dtype=torch.int64, device=dev)
    hsps = torch.full((max(hsp_cap, 1), 6), -7, dtype=torch.int32, device=dev)
    nh = ctypes.c_int64(-1)
    stream = torch.cuda.current_stream(dev).cuda_stream
    st = lib().bp_search_noalloc(q.data_ptr(), len(query), ctypes.byref(params), res.data_ptr(), len(residues),
                                 off.data_ptr(), n, counters.data_ptr(), hoff.data_ptr(), hsps.data_ptr(), hsp_cap,
                                 ctypes.byref(nh), ctypes.c_void_p(stream))
    return st, nh.value, counters.cpu().numpy(), hoff.cpu().numpy(), hsps.cpu().numpy()[:max(nh.value, 0)]


class _R:
    def __init__(self, counters, hoff, hsps):
        self.counters, self.hsp_off, self._h = counters, hoff, hsps

    def hsps_as_array(self):
        return self._h


def test_noalloc_matches_bp_search_on_two_calls_in_a_row():
    matrix = np.asarray(__import__("blastp_b200").blosum62())
    p = default_params()
    eng = Engine(0)
    try:
        cases = [synth.shape1(matrix, n_subjects=20_000), synth.shape2(matrix, n_subjects=30_000)]
        for w in cases:   # two calls in a row, different inputs: no state may leak from the first
            q = w.queries[0]
            ref = eng.search(eng.database(w.db.residues, w.db.offsets), eng.query(q, p)).fetch()
            st, nh, counters, hoff, hsps = run_noalloc(q, w.db.residues, w.db.offsets, p, hsp_cap=65536)
            assert st == 0, "bp_search_noalloc returned status %d" % st
            assert nh == len(ref.hsps)
            assert_same(_R(counters, hoff, hsps), (ref.counters, ref.hsp_off, ref.hsps_as_array()), w.name)
    finally:
        eng.close()


def test_noalloc_reports_limits():
    matrix = np.asarray(__import__("blastp_b200").blosum62())
    w = synth.shape1(matrix, n_subjects=5_000)
    q = w.queries[0]
    p = default_params()
    # too small an output buffer: status TOO_LARGE, the true count, complete counters
    st, nh, counters, hoff, _ = run_noalloc(q, w.db.residues, w.db.offsets, p, hsp_cap=1)
    assert st == 4 and nh > 1 and hoff[-1] == nh == counters[:, 1].sum()
    # a query longer than the stated maximum
    st, *_ = run_noalloc(synth.residues(np.random.default_rng(0), 5000), w.db.residues, w.db.offsets, p, 1024)
    assert st == 4
    # an invalid residue code in the query
    bad = q.copy()
    bad[3] = 0
    st, *_ = run_noalloc(bad, w.db.residues, w.db.offsets, p, 1024)
    assert st == 1


def test_noalloc_rejects_malformed_offsets():
    # Offsets are checked on the device before any subject is read: a
    # decreasing pair, an end past the residues, a start other than 0 and a
    # subject longer than 2^29 are each refused with BP_ERR_INVALID, and the
    # next call with good offsets still matches bp_search.
    matrix = np.asarray(__import__("blastp_b200").blosum62())
    w = synth.shape1(matrix, n_subjects=4_000)
    q = w.queries[0]
    p = default_params()
    off = w.db.offsets
    bads = []
    b = off.copy()
    b[100], b[101] = off[101], off[100]
    bads.append(b)
    b = off.copy()
    b[2000] = off[-1] + 4096
    bads.append(b)
    b = off.copy()
    b[-1] = off[-1] + 64
    bads.append(b)
    b = off.copy()
    b[0] = 8
    bads.append(b)
    b = off.copy()
    b[1:] = off[-1]
    b[1] = (1 << 29) + 1
    bads.append(b)
    for k, bad in enumerate(bads):
        st, *_ = run_noalloc(q, w.db.residues, bad, p, 1024)
        assert st == 1, "malformed offsets %d: status %d" % (k, st)
    eng = Engine(0)
    try:
        ref = eng.search(eng.database(w.db.residues, off), eng.query(q, p)).fetch()
    finally:
        eng.close()
    st, nh, counters, hoff, hsps = run_noalloc(q, w.db.residues, off, p, hsp_cap=65536)
    assert st == 0 and nh == len(ref.hsps)
    assert_same(_R(counters, hoff, hsps), (ref.counters, ref.hsp_off, ref.hsps_as_array()), "after refusals")
