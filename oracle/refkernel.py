"""ctypes bindings for the reference's own kernel run on the CPU
(oracle/_ref/libref_ring*.so, built by `make -C oracle ref` from the
reference's gpu_blastp_kernel.cu through ref_driver.cpp).  TEST
INFRASTRUCTURE ONLY: it pins the oracle (oracle.c) to the reference's code;
the product path never imports it.

`two_hit` returns what the reference's GPU_BLASTP + GPU_BLASTP_get_data hand
to NCBI (gpu_blastp.cu:224-259): per-subject counters and the record ring,
plus the padded length each subject was scanned over (its group's longest
member rounded up to 64, functions.cpp:428-545).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_libs = {}


def path(slots):
    return os.path.join(REF_DIR, "libref_ring%d.so" % slots)


def available(slots=64):
    return os.path.exists(path(slots))


def _lib(slots):
    if slots not in _libs:
        p = path(slots)
        if not os.path.exists(p):
            raise RuntimeError("reference kernel not built: run `make -C oracle ref`")
        L = ctypes.CDLL(p)
        P = ctypes.c_void_p
        i32 = ctypes.c_int32
        L.ref_ring_slots.restype = i32
        L.ref_ring_slots.argtypes = []
        L.ref_two_hit.restype = i32
        L.ref_two_hit.argtypes = [P, P, i32, P, i32, P, P, P, i32, i32, P, P, P, i32, i32, i32,
                                  i32, i32, P, P, P, P]
        assert L.ref_ring_slots() == slots
        _libs[slots] = L
    return _libs[slots]


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def two_hit(residues, offsets, query, table, matrix28, contexts, window=40,
            diag_array_length=None, diag_offset=None, blocks=1, threads=64,
            matrix_bytes=28 * 28, slots=64, timing=None):
    """contexts: list of (query_offset, xdrop, cutoff).  Returns
    (hits int32[n,3], ring int32[n,slots,6], group_len int32[n]); when
    `timing` is a dict, timing["kernel_s"] receives the kernel's own time."""
    res = np.ascontiguousarray(residues, dtype=np.uint8)
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    q = np.ascontiguousarray(query, dtype=np.uint8)
    start, ent = table
    start = np.ascontiguousarray(start, dtype=np.uint32)
    ent = np.ascontiguousarray(ent if len(ent) else np.zeros(1, dtype=np.uint16), dtype=np.uint16)
    m = np.ascontiguousarray(matrix28, dtype=np.int8)
    n = len(off) - 1
    if diag_array_length is None:
        diag_array_length = 1
        while diag_array_length < len(q) + window:
            diag_array_length <<= 1
    co = np.array([c[0] for c in contexts], dtype=np.int32)
    cx = np.array([c[1] for c in contexts], dtype=np.int32)
    cc = np.array([c[2] for c in contexts], dtype=np.int32)
    hits = np.zeros((max(n, 1), 3), dtype=np.int32)
    ring = np.zeros((max(n, 1), slots, 6), dtype=np.int32)
    glen = np.zeros(max(n, 1), dtype=np.int32)
    kns = ctypes.c_int64(0)
    rc = _lib(slots).ref_two_hit(_p(res if len(res) else np.zeros(1, np.uint8)), _p(off), n, _p(q), len(q),
                                 _p(start), _p(ent), _p(m), matrix_bytes, len(contexts), _p(co), _p(cx),
                                 _p(cc), window, diag_array_length,
                                 window if diag_offset is None else diag_offset, blocks, threads,
                                 _p(hits), _p(ring), _p(glen), ctypes.byref(kns))
    if rc != 0:
        raise ValueError("ref_two_hit rejected its arguments (code %d)" % rc)
    if timing is not None:
        timing["kernel_s"] = kns.value / 1e9
    return hits[:n], ring[:n], glen[:n]


def padded(residues, offsets, group_len):
    """The flat database the reference kernel effectively scans: each subject
    followed by zeros up to its group length."""
    off = np.asarray(offsets, dtype=np.int64)
    n = len(off) - 1
    poff = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.asarray(group_len, dtype=np.int64), out=poff[1:])
    flat = np.zeros(int(poff[-1]), dtype=np.uint8)
    for s in range(n):
        ln = int(off[s + 1] - off[s])
        flat[poff[s]:poff[s] + ln] = residues[off[s]:off[s + 1]]
    return flat, poff


def ring_of(counters, hoff, hsps, slots):
    """The ring a complete HSP set leaves behind when each record goes to slot
    rank mod slots (gpu_blastp_kernel.cu:274): the last `slots` records."""
    n = len(counters)
    ring = np.zeros((n, slots, 6), dtype=np.int32)
    for s in np.nonzero(counters[:, 1])[0]:
        succ = int(counters[s, 1])
        for k in range(max(0, succ - slots), succ):
            ring[s, k % slots] = hsps[hoff[s] + k]
    return ring
