"""Drive the reference-compatible entry points (GPU_BLASTP and family) from
Python, the way NCBI's preliminary search drives them
(ncbi_blast_files/functions.cpp:641-699,1099,1328,1407).

It builds the inputs an NCBI caller would hand over -- the lookup table as a
presence vector + thick backbone of AaLookupSmallboneCell + overflow array,
the diagonal-table parameters, per-context cutoffs, and the GPU-format
database volume (4-byte-interleaved groups, each padded to its longest member
rounded up to 64; ncbi_blast_files/functions.cpp:428-545) -- using the
stand-in structure layouts of include/ncbi_compat.h.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import lib

P = ctypes.c_void_p
Int4 = ctypes.c_int32
Uint2 = ctypes.c_uint16


class BLAST_SequenceBlk(ctypes.Structure):
    _fields_ = [("sequence", P), ("length", Int4)]


class BlastContextInfo(ctypes.Structure):
    _fields_ = [("query_offset", Int4)]


class BlastQueryInfo(ctypes.Structure):
    _fields_ = [("num_queries", Int4), ("contexts", P)]


class _Payload(ctypes.Union):
    _fields_ = [("entries", Uint2 * 3), ("overflow_cursor", Int4)]


class AaLookupSmallboneCell(ctypes.Structure):
    _fields_ = [("num_used", Int4), ("payload", _Payload)]


class BlastAaLookupTable(ctypes.Structure):
    _fields_ = [("mask", Int4), ("charsize", Int4), ("word_length", Int4), ("backbone_size", Int4),
                ("thick_backbone", P), ("overflow", P), ("overflow_size", Int4), ("pv", P)]


class LookupTableWrap(ctypes.Structure):
    _fields_ = [("lut_type", Int4), ("lut", P)]


class BLAST_DiagTable(ctypes.Structure):
    _fields_ = [("diag_array_length", Int4), ("diag_mask", Int4), ("offset", Int4), ("window", Int4)]


class Blast_ExtendWord(ctypes.Structure):
    _fields_ = [("diag_table", P)]


class BlastUngappedCutoffs(ctypes.Structure):
    _fields_ = [("x_dropoff", Int4), ("cutoff_score", Int4)]


class BlastInitialWordParameters(ctypes.Structure):
    _fields_ = [("cutoffs", P)]


class BlastGPUOptions(ctypes.Structure):
    _fields_ = [("use_gpu", ctypes.c_char), ("num_blocksx", ctypes.c_int), ("num_threadsx", ctypes.c_int),
                ("num_sequences_to", ctypes.c_int), ("method", ctypes.c_int), ("cpu_threads", ctypes.c_int)]


def round2multiple(x: int) -> int:
    v = Int4(x)
    lib().Round2Multiple(ctypes.byref(v))
    return v.value


def ncbi_table(cell_start: np.ndarray, entries: np.ndarray):
    """CSR table -> (pv uint32[1024+pad], cells AaLookupSmallboneCell[32768], overflow uint16[])."""
    ncell = 1 << 15
    cells = (AaLookupSmallboneCell * ncell)()
    pv = np.zeros((ncell >> 5) + 64, dtype=np.uint32)
    overflow = []
    for c in np.nonzero(np.diff(cell_start.astype(np.int64)))[0]:
        lo, hi = int(cell_start[c]), int(cell_start[c + 1])
        cells[c].num_used = hi - lo
        pv[c >> 5] |= np.uint32(1 << (c & 31))
        if hi - lo <= 3:
            for k in range(hi - lo):
                cells[c].payload.entries[k] = int(entries[lo + k])
        else:
            cells[c].payload.overflow_cursor = len(overflow)
            overflow.extend(int(x) for x in entries[lo:hi])
    return pv, cells, np.array(overflow if overflow else [0], dtype=np.uint16)


def gpu_volume(residues: np.ndarray, offsets: np.ndarray, group_size: int):
    """The reference's GPU database layout: (volume bytes, group lengths,
    padded flat copy with its offsets).  Member i of group g stores residue k
    at base_g + ((k>>2)*group_size + i)*4 + (k&3); every member is padded with
    zeros to its group's length."""
    n = len(offsets) - 1
    lens = np.diff(offsets)
    n_groups = (n + group_size - 1) // group_size
    glen = np.zeros(n_groups, dtype=np.int32)
    for g in range(n_groups):
        m = int(lens[g * group_size:(g + 1) * group_size].max()) if n else 0
        glen[g] = round2multiple(m) if m else 64
    gbase = np.zeros(n_groups + 1, dtype=np.int64)
    np.cumsum(glen.astype(np.int64) * group_size, out=gbase[1:])
    vol = np.zeros(int(gbase[-1]), dtype=np.uint8)
    seq = np.arange(n)
    g = seq // group_size
    i = seq % group_size
    flat_off = gbase[g] + i * glen[g]
    flat = np.zeros(int(gbase[-1]), dtype=np.uint8)
    for s in range(n):
        k = np.arange(lens[s])
        sub = residues[offsets[s]:offsets[s + 1]]
        vol[gbase[g[s]] + ((k >> 2) * group_size + i[s]) * 4 + (k & 3)] = sub
        flat[flat_off[s]:flat_off[s] + lens[s]] = sub
    padded_off = np.concatenate([flat_off, [flat_off[-1] + glen[g[-1]] if n else 0]]).astype(np.int64)
    return vol, glen, flat, padded_off


class LegacyCall:
    """Holds every object an NCBI caller keeps alive across GPU_BLASTP,
    GPU_BLASTP_get_data and GPU_BLASTP_free_memory."""

    def __init__(self, query, contexts, cell_start, entries, window, diag_array_length,
                 volume, glen, n_subjects, blocks, threads, diag_offset=None):
        self.query = np.ascontiguousarray(query, dtype=np.uint8)
        self.seq = BLAST_SequenceBlk(self.query.ctypes.data, len(self.query))
        self.ctx = (BlastContextInfo * len(contexts))(*[BlastContextInfo(c[0]) for c in contexts])
        self.qinfo = BlastQueryInfo(len(contexts), ctypes.cast(self.ctx, P))
        self.pv, self.cells, self.overflow = ncbi_table(cell_start, entries)
        self.lut = BlastAaLookupTable((1 << 15) - 1, 5, 3, 1 << 15, ctypes.cast(self.cells, P),
                                      self.overflow.ctypes.data, len(self.overflow), self.pv.ctypes.data)
        self.wrap = LookupTableWrap(0, ctypes.cast(ctypes.pointer(self.lut), P))
        self.diag = BLAST_DiagTable(diag_array_length, diag_array_length - 1,
                                    window if diag_offset is None else diag_offset, window)
        self.ewp = Blast_ExtendWord(ctypes.cast(ctypes.pointer(self.diag), P))
        self.cut = (BlastUngappedCutoffs * len(contexts))(*[BlastUngappedCutoffs(c[1], c[2]) for c in contexts])
        self.wp = BlastInitialWordParameters(ctypes.cast(self.cut, P))
        self.opts = BlastGPUOptions(b"\x01", blocks, threads, n_subjects, 1, 1)
        self.glen = np.ascontiguousarray(glen, dtype=np.int32)
        self.volume = np.ascontiguousarray(volume, dtype=np.uint8)
        self.n = n_subjects
        self.hits_bytes = n_subjects * 3 * 4
        self.list_bytes = n_subjects * 2 * 24
        self.slots = [P() for _ in range(9)]   # d_Hits, d_list, d_db, d_matrix, d_lenvec, d_pv, d_bb, d_ovf, d_diag

    def check_memory(self):
        return bool(lib().GPU_BLASTP_check_memory(ctypes.byref(self.wrap), ctypes.byref(self.ewp),
                                                  ctypes.byref(self.opts), len(self.volume), self.hits_bytes,
                                                  self.list_bytes, len(self.glen), self.qinfo.num_queries,
                                                  len(self.query)))

    def run(self):
        s = self.slots
        lib().GPU_BLASTP(ctypes.byref(self.seq), ctypes.byref(self.qinfo), ctypes.byref(self.wrap),
                         ctypes.byref(self.ewp), ctypes.byref(self.wp), ctypes.byref(self.opts),
                         self.glen.ctypes.data, len(self.volume), self.volume.ctypes.data,
                         ctypes.byref(s[0]), self.hits_bytes, ctypes.byref(s[1]), self.list_bytes,
                         ctypes.byref(s[2]), ctypes.byref(s[3]), ctypes.byref(s[4]), ctypes.byref(s[5]),
                         ctypes.byref(s[6]), ctypes.byref(s[7]), ctypes.byref(s[8]))

    def get_data(self):
        hits = np.zeros((self.n, 3), dtype=np.int32)
        ring = np.zeros((self.n, 2, 6), dtype=np.int32)
        lib().GPU_BLASTP_get_data(hits.ctypes.data, self.slots[0], self.hits_bytes, ring.ctypes.data,
                                  self.slots[1], self.list_bytes, self.n)
        return hits, ring

    def get_hsps(self):
        """The complete HSP set (hsp_off [n+1], hsps [k, 6]) after get_data."""
        k = ctypes.c_int64(0)
        assert lib().GPU_BLASTP_get_hsps(self.slots[0], None, None, 0, ctypes.byref(k))
        off = np.zeros(self.n + 1, dtype=np.int64)
        hsps = np.zeros((max(k.value, 1), 6), dtype=np.int32)
        assert lib().GPU_BLASTP_get_hsps(self.slots[0], off.ctypes.data, hsps.ctypes.data, k.value,
                                         ctypes.byref(k))
        return off, hsps[:k.value]

    def free(self):
        lib().GPU_BLASTP_free_memory(*[ctypes.byref(x) for x in self.slots])
