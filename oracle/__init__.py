"""ctypes bindings for the CPU oracle (oracle.c).  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference legs may import this package, and only as the checker or the timed
CPU baseline; the product path never does.  Parity against the reference's
own kernel is pinned by tests/test_ref_pinned.py (see oracle.h).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NCELL = 1 << 15
_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle not built: run `make -C oracle`")
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        L.or_build_table.restype = ctypes.c_int64
        L.or_build_table.argtypes = [P, ctypes.c_int32, P, ctypes.c_int32, P, P, ctypes.c_int64]
        L.or_scan.restype = ctypes.c_int64
        L.or_scan.argtypes = [P, P, ctypes.c_int32, P, ctypes.c_int32, P, P,
                              ctypes.c_int32, P, P, P, ctypes.c_int32, ctypes.c_int32,
                              P, ctypes.c_int32, P, P, P, ctypes.c_int64]
        L.or_extend_two_hit.restype = None
        L.or_extend_two_hit.argtypes = [P, P, ctypes.c_int32, P, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, P]
        i32 = ctypes.c_int32
        L.or_gapped.restype = ctypes.c_int64
        L.or_gapped.argtypes = [P, P, i32, P, i32, P, P, P, P, i32, P, P, ctypes.c_int64]
        L.or_gapped_extend.restype = i32
        L.or_gapped_extend.argtypes = [P, P, i32, P, i32, i32, i32, i32, i32, P, P, P, P]
        L.or_gapped_seed.restype = None
        L.or_gapped_seed.argtypes = [P, P, P, i32, i32, i32, P, P]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def load_fixture_matrix():
    path = os.path.join(os.path.dirname(HERE), "tests", "golden", "blosum62_ncbistdaa.txt")
    return np.loadtxt(path, dtype=np.int64).astype(np.int8)


def build_table(query, matrix28, threshold=11):
    """Returns (cell_start uint32[NCELL+1], entries uint16[])."""
    q = np.ascontiguousarray(query, dtype=np.uint8)
    m = np.ascontiguousarray(matrix28, dtype=np.int8)
    start = np.zeros(NCELL + 1, dtype=np.uint32)
    cap = max(1, 200 * len(q))
    while True:
        ent = np.zeros(cap, dtype=np.uint16)
        n = lib().or_build_table(_p(q), len(q), _p(m), threshold, _p(start), _p(ent), cap)
        if n >= 0:
            return start, ent[:n].copy()
        cap = int(start[-1])


def diag_mask_for(qlen, window):
    n = 1
    while n < qlen + window:
        n <<= 1
    return n - 1


def scan(residues, offsets, query, table, matrix28, contexts, window=40, diag_mask=None,
         threads=0):
    """contexts: list of (query_offset, xdrop, cutoff).  Returns
    (counters int32[n,3], hsp_off int64[n+1], hsps int32[k,6])."""
    res = np.ascontiguousarray(residues, dtype=np.uint8)
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    q = np.ascontiguousarray(query, dtype=np.uint8)
    start, ent = table
    ent = ent if len(ent) else np.zeros(1, dtype=np.uint16)
    m = np.ascontiguousarray(matrix28, dtype=np.int8)
    n = len(off) - 1
    if diag_mask is None:
        diag_mask = diag_mask_for(len(q), window)
    co = np.array([c[0] for c in contexts], dtype=np.int32)
    cx = np.array([c[1] for c in contexts], dtype=np.int32)
    cc = np.array([c[2] for c in contexts], dtype=np.int32)
    counters = np.zeros((n, 3), dtype=np.int32)
    hoff = np.zeros(n + 1, dtype=np.int64)
    cap = max(1024, n // 4)
    while True:
        hsps = np.zeros((cap, 6), dtype=np.int32)
        total = lib().or_scan(_p(res), _p(off), n, _p(q), len(q), _p(start), _p(ent),
                              len(contexts), _p(co), _p(cx), _p(cc), window, diag_mask,
                              _p(m), threads, _p(counters), _p(hoff), _p(hsps), cap)
        if total <= cap:
            return counters, hoff, hsps[:total].copy()
        cap = int(total)


def extend_two_hit(matrix28, subject, query, s_left, s_right, q_right, xdrop):
    m = np.ascontiguousarray(matrix28, dtype=np.int8)
    s = np.ascontiguousarray(subject, dtype=np.uint8)
    q = np.ascontiguousarray(query, dtype=np.uint8)
    out = np.zeros(6, dtype=np.int32)
    lib().or_extend_two_hit(_p(m), _p(s), len(s), _p(q), len(q), s_left, s_right, q_right, xdrop,
                            _p(out))
    return tuple(int(x) for x in out)


GHSP_FIELDS = ("score", "q_start", "q_end", "s_start", "s_end", "q_seed", "s_seed", "ungapped")


class GappedParams(ctypes.Structure):
    _fields_ = [("gap_open", ctypes.c_int32), ("gap_extend", ctypes.c_int32), ("xdrop", ctypes.c_int32),
                ("cutoff", ctypes.c_int32)]


def gapped(residues, offsets, query, hsp_off, hsps, matrix28, gap_open=11, gap_extend=1, xdrop=38, cutoff=0,
           threads=0):
    """The gapped stage (gapped.h) over the ungapped result (hsp_off, hsps
    int32[k, 6]).  Returns (goff int64[n+1], ghsps int32[g, 8] with the
    fields of GHSP_FIELDS)."""
    res = np.ascontiguousarray(residues, dtype=np.uint8)
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    q = np.ascontiguousarray(query, dtype=np.uint8)
    ho = np.ascontiguousarray(hsp_off, dtype=np.int64)
    h = np.ascontiguousarray(hsps, dtype=np.int32).reshape(-1, 6)
    if len(h) == 0:
        h = np.zeros((1, 6), dtype=np.int32)
    m = np.ascontiguousarray(matrix28, dtype=np.int8)
    n = len(off) - 1
    p = GappedParams(gap_open, gap_extend, xdrop, cutoff)
    goff = np.zeros(n + 1, dtype=np.int64)
    cap = max(1024, int(ho[-1]) if n else 1)
    while True:
        out = np.zeros((cap, 8), dtype=np.int32)
        total = lib().or_gapped(_p(res if len(res) else np.zeros(1, np.uint8)), _p(off), n, _p(q), len(q),
                                _p(ho), _p(h), _p(m), ctypes.byref(p), threads or (os.cpu_count() or 1),
                                _p(goff), _p(out), cap)
        if total <= cap:
            return goff, out[:total].copy()
        cap = int(total)


def gapped_extend(matrix28, A, B, xdrop=38, gap_open=11, gap_extend=1):
    """One forward extension over A and B (gapped.h): (best, i, j)."""
    a = np.ascontiguousarray(A, dtype=np.uint8)
    b = np.ascontiguousarray(B, dtype=np.uint8)
    m = np.ascontiguousarray(matrix28, dtype=np.int8)
    H = np.zeros(len(b) + 1, dtype=np.int32)
    F = np.zeros(len(b) + 1, dtype=np.int32)
    bi = ctypes.c_int32(0)
    bj = ctypes.c_int32(0)
    best = lib().or_gapped_extend(_p(m), _p(a if len(a) else np.zeros(1, np.uint8)), len(a),
                                  _p(b if len(b) else np.zeros(1, np.uint8)), len(b), 1, xdrop, gap_open, gap_extend,
                                  _p(H), _p(F), ctypes.byref(bi), ctypes.byref(bj))
    return int(best), int(bi.value), int(bj.value)
