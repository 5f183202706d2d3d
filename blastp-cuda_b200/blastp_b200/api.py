"""Python host layer over the native C ABI: the same operations as the C
entry points, with numpy arrays in and out.  The work runs in
libblastp_b200.so on the GPU; nothing here computes results.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import (COST_FEATURES, BpAutotuneOptions, BpAutotuneTrial, BpBatchOptions, BpGappedParams, BpParams,
                   BpServerMetrics, BpServerOptions, check, lib)

HSP_DTYPE = np.dtype([("hsp_q", "<i4"), ("hsp_s", "<i4"), ("query_offset", "<i4"),
                      ("subject_offset", "<i4"), ("hsp_len", "<i4"), ("score", "<i4")])


GAPPED_DTYPE = np.dtype([("score", "<i4"), ("q_start", "<i4"), ("q_end", "<i4"), ("s_start", "<i4"),
                         ("s_end", "<i4"), ("q_seed", "<i4"), ("s_seed", "<i4"), ("ungapped", "<i4")])


def gapped_params(**kw) -> BpGappedParams:
    p = BpGappedParams()
    lib().bp_gapped_params_default(ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def default_params(**kw) -> BpParams:
    p = BpParams()
    lib().bp_params_default(ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def blosum62() -> np.ndarray:
    out = np.zeros(28 * 28, dtype=np.int8)
    lib().bp_blosum62_ncbistdaa(_p(out))
    return out.reshape(28, 28)


class Result:
    """Per-subject counters (hits, successful extensions, extensions) and the
    HSP set as CSR (offsets into a structured array, discovery order)."""

    def __init__(self, counters, hsp_off, hsps):
        self.counters = counters
        self.hsp_off = hsp_off
        self.hsps = hsps

    def hsps_as_array(self):
        return self.hsps.view(np.int32).reshape(-1, 6)


class Engine:
    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        check(lib().bp_engine_create(device, ctypes.byref(h)))
        self.h = h
        self.device = device

    def close(self):
        if self.h:
            lib().bp_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return lib().bp_engine_stream(self.h) or 0

    @property
    def launches(self) -> int:
        return int(lib().bp_engine_launch_count(self.h))

    @property
    def last_scan_ms(self) -> float:
        return float(lib().bp_engine_last_scan_ms(self.h))

    def synchronize(self):
        check(lib().bp_engine_synchronize(self.h), self.h)

    def set_upload_wait(self, ms: int):
        """How long a streaming blastp_host scan waits for one upload chunk."""
        check(lib().bp_engine_set_upload_wait(self.h, int(ms)), self.h)

    def drop_chunk_flag(self, chunk: int):
        """Fault injection: the next streaming blastp_host call does not
        announce upload chunk `chunk`, so the scan's bounded wait runs out."""
        check(lib().bp_engine_drop_chunk_flag(self.h, int(chunk)), self.h)

    def database(self, residues: np.ndarray, offsets: np.ndarray) -> "Database":
        return Database(self, residues, offsets)

    def open_database(self, path) -> "Database":
        """A database file streamed into HBM (bp_db_open)."""
        return Database(self, path=path)

    def query(self, residues: np.ndarray, params: BpParams | None = None) -> "Query":
        return Query(self, residues, params or default_params())

    def search(self, db: "Database", q: "Query", first: int = 0, count: int = -1) -> "PendingResult":
        h = ctypes.c_void_p()
        check(lib().bp_search(self.h, db.h, q.h, first, count, ctypes.byref(h)), self.h)
        return PendingResult(self, h, keep=(db, q))

    def plan_chunks(self, db: "Database", chunk_residues: int, first: int = 0, count: int = -1) -> np.ndarray:
        """Chunk boundaries of a batched search over subjects [first,
        first+count): chunk c holds subjects [b[c], b[c+1])."""
        n = ctypes.c_int32(0)
        check(lib().bp_batch_plan(db.h, first, count, chunk_residues, None, ctypes.byref(n)), self.h)
        out = np.zeros(n.value + 1, dtype=np.int32)
        check(lib().bp_batch_plan(db.h, first, count, chunk_residues, _p(out), ctypes.byref(n)), self.h)
        return out

    def search_batch(self, db: "Database", queries, chunk_residues: int = 1 << 18, schedule: int = 0,
                     ctas: int = 0, max_warps: int = 0, use_graph: bool = True, item_costs=None,
                     first: int = 0, count: int = -1, pack_residues: int = 512,
                     plain_unpacked: int = 0) -> "Batch":
        """Many queries against db in one persistent launch; each query's
        result equals its single-query search."""
        o = BpBatchOptions()
        lib().bp_batch_options_default(ctypes.byref(o))
        o.chunk_residues = chunk_residues
        o.schedule = schedule
        o.ctas = ctas
        o.max_warps = max_warps
        o.use_graph = int(bool(use_graph))
        o.subject_first = first
        o.subject_count = count
        o.pack_residues = pack_residues
        o.plain_unpacked = plain_unpacked
        costs = None
        if item_costs is not None:
            costs = np.ascontiguousarray(item_costs, dtype=np.float32)
            o.item_costs = costs.ctypes.data
        arr = (ctypes.c_void_p * max(1, len(queries)))(*[q.h.value for q in queries])
        h = ctypes.c_void_p()
        check(lib().bp_search_batch(self.h, db.h, arr, len(queries), ctypes.byref(o), ctypes.byref(h)), self.h)
        b = Batch(self, h, db, list(queries))
        b.n_chunks = len(self.plan_chunks(db, chunk_residues, first, count)) - 1
        b.n_subjects = (db.n_subjects - first) if count < 0 else count
        return b

    def chunk_histograms(self, db: "Database", chunk_first) -> np.ndarray:
        """Residue counts (28 NCBIstdaa bins) of every chunk, on the device."""
        first = np.ascontiguousarray(chunk_first, dtype=np.int32)
        n = len(first) - 1
        out = np.zeros((max(n, 0), 28), dtype=np.uint32)
        check(lib().bp_db_chunk_histograms(self.h, db.h, _p(first), n, _p(out)), self.h)
        return out

    def batch_features(self, db: "Database", queries, chunk_first, planted_density: float = 0.0) -> np.ndarray:
        """Cost-model features of every (query, chunk) item, row q*n_chunks + c."""
        first = np.ascontiguousarray(chunk_first, dtype=np.int32)
        n = len(first) - 1
        X = np.zeros((len(queries) * n, COST_FEATURES), dtype=np.float32)
        arr = (ctypes.c_void_p * max(1, len(queries)))(*[q.h.value for q in queries])
        check(lib().bp_batch_features(self.h, db.h, arr, len(queries), _p(first), n, planted_density, _p(X)),
              self.h)
        return X

    def predict_costs(self, model, db: "Database", queries, chunk_first, planted_density: float = 0.0):
        """Item costs of the cost schedule (bp_batch_predict_costs) from a
        costmodel.CostModel."""
        first = np.ascontiguousarray(chunk_first, dtype=np.int32)
        n = len(first) - 1
        out = np.zeros(len(queries) * n, dtype=np.float32)
        w = np.ascontiguousarray(model.weights, dtype=np.float32)
        arr = (ctypes.c_void_p * max(1, len(queries)))(*[q.h.value for q in queries])
        check(lib().bp_batch_predict_costs(self.h, model.mlp.h, _p(w), db.h, arr, len(queries), _p(first), n,
                                           planted_density, _p(out)), self.h)
        return out

    def autotune(self, db: "Database", queries, model=None, planted_density: float = 0.0, sample_subjects: int = 0,
                 chunk_sizes=None, warp_caps=None, schedules=(0, 1, 2, 3), reps: int = 2, pack_sizes=None):
        """Times candidate batch configurations on a sample of the subjects
        (bp_batch_autotune); returns (best options dict, list of trials)."""
        o = BpAutotuneOptions()
        lib().bp_autotune_options_default(ctypes.byref(o))
        keep = []
        if chunk_sizes is not None:
            cs = np.ascontiguousarray(chunk_sizes, dtype=np.int32)
            keep.append(cs)
            o.chunk_sizes = cs.ctypes.data
            o.n_chunk_sizes = len(cs)
        if warp_caps is not None:
            wc = np.ascontiguousarray(warp_caps, dtype=np.int32)
            keep.append(wc)
            o.warp_caps = wc.ctypes.data
            o.n_warp_caps = len(wc)
        if pack_sizes is not None:
            ps = np.ascontiguousarray(pack_sizes, dtype=np.int32)
            keep.append(ps)
            o.pack_sizes = ps.ctypes.data
            o.n_pack_sizes = len(ps)
        o.schedules_mask = sum(1 << s for s in schedules)
        if model is not None:
            o.model = model.mlp.h.value
            for i in range(3):
                o.cost_weights[i] = float(model.weights[i])
        o.planted_density = planted_density
        o.sample_subjects = sample_subjects
        o.reps = reps
        best = BpBatchOptions()
        trials = (BpAutotuneTrial * 256)()
        nt = ctypes.c_int32(0)
        arr = (ctypes.c_void_p * max(1, len(queries)))(*[q.h.value for q in queries])
        check(lib().bp_batch_autotune(self.h, db.h, arr, len(queries), ctypes.byref(o), ctypes.byref(best), trials,
                                      256, ctypes.byref(nt)), self.h)
        out = [{"chunk_residues": t.chunk_residues, "schedule": t.schedule, "max_warps": t.max_warps,
                "pack_residues": t.pack_residues, "plain_unpacked": t.plain_unpacked, "ms": float(t.ms)}
               for t in trials[:min(nt.value, 256)]]
        return ({"chunk_residues": best.chunk_residues, "schedule": best.schedule, "max_warps": best.max_warps,
                 "pack_residues": best.pack_residues, "plain_unpacked": best.plain_unpacked}, out)

    def blastp_host(self, query, params, residues, offsets, hsp_cap=None, counters=None, hsp_off=None):
        """End-to-end: host buffers in, host buffers out (one C call).
        counters ([n, 3] int32) and hsp_off ([n + 1] int64) may be given, e.g.
        views of pinned memory, into which each chunk's counters are copied
        as soon as its scan ends."""
        q = np.ascontiguousarray(query, dtype=np.uint8)
        res = np.ascontiguousarray(residues, dtype=np.uint8)
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        n = len(off) - 1
        if counters is None:
            counters = np.zeros((n, 3), dtype=np.int32)
        if hsp_off is None:
            hsp_off = np.zeros(n + 1, dtype=np.int64)
        if (counters.shape != (n, 3) or counters.dtype != np.int32 or not counters.flags.c_contiguous or
                hsp_off.shape != (n + 1,) or hsp_off.dtype != np.int64 or not hsp_off.flags.c_contiguous):
            raise ValueError("counters must be [n, 3] int32 and hsp_off [n + 1] int64, both contiguous")
        hoff = hsp_off
        nh = ctypes.c_int64(0)
        cap = hsp_cap if hsp_cap is not None else max(4096, n // 2)
        hsps = np.zeros(cap, dtype=HSP_DTYPE)
        st = lib().bp_blastp_host(self.h, _p(q), len(q), ctypes.byref(params), _p(res), len(res), _p(off), n,
                                  _p(counters), _p(hoff), _p(hsps), cap, ctypes.byref(nh))
        if st == 4 and nh.value > cap:   # too small: retry once with the exact size
            hsps = np.zeros(nh.value, dtype=HSP_DTYPE)
            st = lib().bp_blastp_host(self.h, _p(q), len(q), ctypes.byref(params), _p(res), len(res), _p(off), n,
                                      _p(counters), _p(hoff), _p(hsps), nh.value, ctypes.byref(nh))
        check(st, self.h)
        return Result(counters, hoff, hsps[:nh.value])


def write_database_file(path, residues, offsets, volume_residues: int = 0, sort_by_length: bool = False):
    """Writes the subjects to a database file (bp_dbfile_write); no GPU needed."""
    res = np.ascontiguousarray(residues, dtype=np.uint8)
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    check(lib().bp_dbfile_write(str(path).encode(), _p(res), len(res), _p(off), len(off) - 1, volume_residues,
                                int(bool(sort_by_length))))


def read_database_file(path):
    """(residues, offsets, oids, n_volumes) of a database file, in stored order;
    oids[i] is the original index of stored subject i.  No GPU needed."""
    n = ctypes.c_int32(0)
    r = ctypes.c_int64(0)
    v = ctypes.c_int32(0)
    srt = ctypes.c_int32(0)
    check(lib().bp_dbfile_info(str(path).encode(), ctypes.byref(n), ctypes.byref(r), ctypes.byref(v),
                               ctypes.byref(srt)))
    res = np.zeros(r.value, dtype=np.uint8)
    off = np.zeros(n.value + 1, dtype=np.int64)
    oids = np.zeros(n.value, dtype=np.int32)
    check(lib().bp_dbfile_read_host(str(path).encode(), _p(res), _p(off), _p(oids)))
    return res, off, oids, v.value


class Database:
    def __init__(self, engine: Engine, residues=None, offsets=None, path=None):
        h = ctypes.c_void_p()
        if path is not None:
            check(lib().bp_db_open(engine.h, str(path).encode(), ctypes.byref(h)), engine.h)
            self.n_subjects = int(lib().bp_db_subjects(h))
            self.n_residues = int(lib().bp_db_residues(h))
        else:
            res = np.ascontiguousarray(residues, dtype=np.uint8)
            off = np.ascontiguousarray(offsets, dtype=np.int64)
            check(lib().bp_db_create(engine.h, _p(res), len(res), _p(off), len(off) - 1, ctypes.byref(h)), engine.h)
            self.n_subjects = len(off) - 1
            self.n_residues = len(res)
        self.h = h
        self.engine = engine

    def close(self):
        if self.h:
            lib().bp_db_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Query:
    def __init__(self, engine: Engine, residues, params: BpParams):
        q = np.ascontiguousarray(residues, dtype=np.uint8)
        h = ctypes.c_void_p()
        check(lib().bp_query_create(engine.h, _p(q), len(q), ctypes.byref(params), ctypes.byref(h)), engine.h)
        self.h = h
        self.engine = engine
        self.length = len(q)
        self.params = params

    def table(self):
        start = np.zeros((1 << 15) + 1, dtype=np.uint32)
        n = ctypes.c_int64(0)
        check(lib().bp_query_table(self.h, _p(start), None, 0, ctypes.byref(n)), self.engine.h)
        ent = np.zeros(max(1, n.value), dtype=np.uint16)
        check(lib().bp_query_table(self.h, None, _p(ent), n.value, ctypes.byref(n)), self.engine.h)
        return start, ent[:n.value]

    def close(self):
        if self.h:
            lib().bp_query_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GappedResult:
    """Per-subject counters (ungapped HSPs, gapped HSPs reported, extensions
    run) and the gapped HSPs as CSR, in processing order."""

    def __init__(self, counters, off, hsps, ms):
        self.counters = counters
        self.off = off
        self.hsps = hsps
        self.ms = ms

    def hsps_as_array(self):
        return self.hsps.view(np.int32).reshape(-1, 8)


class PendingResult:
    def __init__(self, engine: Engine, h, keep=()):
        self.engine = engine
        self.h = h
        self._keep = keep      # the database and query must outlive the search

    def wait(self):
        check(lib().bp_result_wait(self.h), self.engine.h)
        return self

    def fetch(self) -> Result:
        self.wait()
        n = lib().bp_result_subjects(self.h)
        k = lib().bp_result_hsps(self.h)
        counters = np.zeros((n, 3), dtype=np.int32)
        hoff = np.zeros(n + 1, dtype=np.int64)
        hsps = np.zeros(max(k, 1), dtype=HSP_DTYPE)
        check(lib().bp_result_copy(self.h, _p(counters), _p(hoff), _p(hsps)), self.engine.h)
        return Result(counters, hoff, hsps[:k])

    def gapped(self, params: BpGappedParams | None = None, ring_columns: int = 0) -> "GappedResult":
        """The gapped stage on this result (bp_gapped_run)."""
        self.wait()
        h = ctypes.c_void_p()
        p = params or gapped_params()
        if ring_columns:
            check(lib().bp_gapped_run_ring(self.h, ctypes.byref(p), int(ring_columns), ctypes.byref(h)),
                  self.engine.h)
        else:
            check(lib().bp_gapped_run(self.h, ctypes.byref(p), ctypes.byref(h)), self.engine.h)
        try:
            n = lib().bp_result_subjects(self.h)
            k = int(lib().bp_gapped_hsps(h))
            counters = np.zeros((n, 3), dtype=np.int32)
            off = np.zeros(n + 1, dtype=np.int64)
            hsps = np.zeros(max(k, 1), dtype=GAPPED_DTYPE)
            check(lib().bp_gapped_copy(h, _p(counters), _p(off), _p(hsps)), self.engine.h)
            return GappedResult(counters, off, hsps[:k], float(lib().bp_gapped_ms(h)))
        finally:
            lib().bp_gapped_destroy(h)

    def digest(self) -> tuple:
        """128-bit device-side digest of the result (bp_result_digest)."""
        out = (ctypes.c_uint64 * 2)()
        check(lib().bp_result_digest(self.h, out), self.engine.h)
        return (int(out[0]), int(out[1]))

    def close(self):
        if self.h:
            lib().bp_result_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """A batched search that can be re-run (a CUDA graph replay by default)."""

    def __init__(self, engine: Engine, h, db, queries):
        self.engine = engine
        self.h = h
        self._keep = (db, queries)     # must outlive the batch
        self.n_subjects = db.n_subjects
        self.n_queries = len(queries)

    def run(self):
        check(lib().bp_batch_run(self.h), self.engine.h)
        return self

    def wait(self):
        check(lib().bp_batch_wait(self.h), self.engine.h)
        return self

    @property
    def n_hsps(self) -> int:
        return int(lib().bp_batch_hsps(self.h))

    @property
    def n_items(self) -> int:
        return int(lib().bp_batch_items(self.h))

    @property
    def last_scan_ms(self) -> float:
        return float(lib().bp_batch_last_scan_ms(self.h))

    def queue_costs(self) -> np.ndarray:
        n = ctypes.c_int32(0)
        check(lib().bp_batch_queue_costs(self.h, None, ctypes.byref(n)), self.engine.h)
        out = np.zeros(n.value, dtype=np.float64)
        check(lib().bp_batch_queue_costs(self.h, _p(out), ctypes.byref(n)), self.engine.h)
        return out

    def item_queues(self) -> np.ndarray:
        n = self.n_queries * self.n_chunks
        out = np.zeros(max(n, 1), dtype=np.int32)
        check(lib().bp_batch_item_queues(self.h, _p(out)), self.engine.h)
        return out[:n]

    def fetch(self, qi: int) -> Result:
        self.wait()
        n = self.n_subjects
        nh = ctypes.c_int64(0)
        check(lib().bp_batch_copy_query(self.h, qi, None, None, None, ctypes.byref(nh)), self.engine.h)
        counters = np.zeros((n, 3), dtype=np.int32)
        hoff = np.zeros(n + 1, dtype=np.int64)
        hsps = np.zeros(max(nh.value, 1), dtype=HSP_DTYPE)
        check(lib().bp_batch_copy_query(self.h, qi, _p(counters), _p(hoff), _p(hsps), ctypes.byref(nh)),
              self.engine.h)
        return Result(counters, hoff, hsps[:nh.value])

    def digest(self, qi: int) -> tuple:
        """Query qi's result digest (bp_batch_digest), equal to its plain search's."""
        out = (ctypes.c_uint64 * 2)()
        check(lib().bp_batch_digest(self.h, qi, out), self.engine.h)
        return (int(out[0]), int(out[1]))

    def close(self):
        if self.h:
            lib().bp_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Mlp:
    """Two-layer MLP (ReLU hidden layer, fp32) trained and evaluated on the
    device by the library's kernels (bp_mlp_*)."""

    def __init__(self, engine: Engine, n_in: int = COST_FEATURES, n_hidden: int = 64, n_out: int = 2,
                 seed: int = 0):
        h = ctypes.c_void_p()
        check(lib().bp_mlp_create(engine.h, n_in, n_hidden, n_out, seed, ctypes.byref(h)), engine.h)
        self.h = h
        self.engine = engine
        self.shape = (n_in, n_hidden, n_out)

    @property
    def n_params(self) -> int:
        return int(lib().bp_mlp_num_params(self.h))

    def get_params(self):
        p = np.zeros(self.n_params, dtype=np.float32)
        norm = np.zeros(2 * self.shape[0] + 2 * self.shape[2], dtype=np.float32)
        check(lib().bp_mlp_get_params(self.h, _p(p), _p(norm)), self.engine.h)
        return p, norm

    def set_params(self, params=None, norm=None):
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float32)
        n = None if norm is None else np.ascontiguousarray(norm, dtype=np.float32)
        check(lib().bp_mlp_set_params(self.h, _p(p), _p(n)), self.engine.h)

    def loss_grad(self, X, T):
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        loss = ctypes.c_float(0)
        g = np.zeros(self.n_params, dtype=np.float32)
        check(lib().bp_mlp_loss_grad(self.h, _p(X), _p(T), len(X), ctypes.byref(loss), _p(g)), self.engine.h)
        return float(loss.value), g

    def fit(self, X, T, epochs=200, batch=1024, lr=3e-3, seed=0):
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        curve = np.zeros(max(epochs, 1), dtype=np.float32)
        check(lib().bp_mlp_fit(self.h, _p(X), _p(T), len(X), epochs, batch, lr, seed, _p(curve)), self.engine.h)
        return curve[:epochs]

    def predict(self, X) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.zeros((len(X), self.shape[2]), dtype=np.float32)
        check(lib().bp_mlp_predict(self.h, _p(X), len(X), _p(Y)), self.engine.h)
        return Y

    def close(self):
        if self.h:
            lib().bp_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching request loop over a resident database
    (bp_server_*): submit() from any thread, results per ticket."""

    def __init__(self, engine: Engine, db: Database, max_batch_queries: int = 32, memory_budget: int = 16 << 30,
                 chunk_residues: int = 1 << 20, schedule: int = 0, lanes: int = 2, model=None,
                 planted_density: float = 0.0, params: BpParams | None = None, poll_us: int = 200,
                 lane_depth: int = 1, admission: int = 0, segments: int = 1, max_wait_ms: int = 0):
        o = BpServerOptions()
        lib().bp_server_options_default(ctypes.byref(o))
        o.max_batch_queries = max_batch_queries
        o.device_memory_budget = memory_budget
        o.chunk_residues = chunk_residues
        o.schedule = schedule
        o.lanes = lanes
        o.lane_depth = lane_depth
        o.admission = admission
        o.segments = segments
        o.max_wait_ms = max_wait_ms
        o.poll_us = poll_us
        if model is not None:
            o.model = model.mlp.h.value
            for i in range(3):
                o.cost_weights[i] = float(model.weights[i])
        o.planted_density = planted_density
        if params is not None:
            o.params = params
        h = ctypes.c_void_p()
        check(lib().bp_server_create(engine.h, db.h, ctypes.byref(o), ctypes.byref(h)), engine.h)
        self.h = h
        self.engine = engine
        self._keep = (db, model)
        self.n_subjects = db.n_subjects

    def submit(self, query) -> int:
        q = np.ascontiguousarray(query, dtype=np.uint8)
        t = ctypes.c_uint64(0)
        check(lib().bp_server_submit(self.h, _p(q), len(q), ctypes.byref(t)))
        return int(t.value)

    def state(self, ticket: int) -> int:
        return int(lib().bp_server_state(self.h, ticket))

    def wait(self, ticket: int, timeout_ms: int = -1):
        check(lib().bp_server_wait(self.h, ticket, timeout_ms))

    def result(self, ticket: int):
        """(Result, latency in ms) of a finished request."""
        nh = ctypes.c_int64(0)
        lat = ctypes.c_double(0)
        check(lib().bp_server_result(self.h, ticket, None, None, None, ctypes.byref(nh), ctypes.byref(lat)))
        n = self.n_subjects
        counters = np.zeros((n, 3), dtype=np.int32)
        hoff = np.zeros(n + 1, dtype=np.int64)
        hsps = np.zeros(max(nh.value, 1), dtype=HSP_DTYPE)
        check(lib().bp_server_result(self.h, ticket, _p(counters), _p(hoff), _p(hsps), ctypes.byref(nh), None))
        return Result(counters, hoff, hsps[:nh.value]), float(lat.value)

    def digest(self, ticket: int) -> tuple:
        """A finished request's result digest (bp_server_digest)."""
        out = (ctypes.c_uint64 * 2)()
        check(lib().bp_server_digest(self.h, ticket, out))
        return (int(out[0]), int(out[1]))

    def latency(self, ticket: int) -> float:
        """Arrival-to-completion time (ms) of a finished request."""
        lat = ctypes.c_double(0)
        check(lib().bp_server_result(self.h, ticket, None, None, None, None, ctypes.byref(lat)))
        return float(lat.value)

    def release(self, ticket: int):
        check(lib().bp_server_release(self.h, ticket))

    def stats(self) -> dict:
        m = BpServerMetrics()
        check(lib().bp_server_stats(self.h, ctypes.byref(m)))
        return {k: getattr(m, k) for k, _ in BpServerMetrics._fields_}

    def close(self):
        if self.h:
            lib().bp_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
