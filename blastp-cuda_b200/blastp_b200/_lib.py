"""ctypes bindings to libblastp_b200.so (include/blastp_b200.h and
include/gpu_cpu_common_b200.h).

The library is the product; this module only declares its signatures.  It
fails loudly when the library is missing: there is no Python or CPU fallback.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "lib", "libblastp_b200.so")

P = ctypes.c_void_p
i32 = ctypes.c_int32
i64 = ctypes.c_int64
u64 = ctypes.c_uint64

BP_OK = 0
STATUS_NAMES = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of device memory",
                4: "input too large", 5: "device wait timed out", 6: "not ready", 7: "no CUDA device"}


class BpParams(ctypes.Structure):
    _fields_ = [("word_length", i32), ("threshold", i32), ("window", i32),
                ("x_dropoff", i32), ("cutoff_score", i32)]


class BpGappedParams(ctypes.Structure):
    _fields_ = [("gap_open", i32), ("gap_extend", i32), ("x_dropoff", i32), ("cutoff_score", i32)]


class BpBatchOptions(ctypes.Structure):
    _fields_ = [("chunk_residues", i32), ("schedule", i32), ("ctas", i32), ("max_warps", i32),
                ("use_graph", i32), ("item_costs", P), ("subject_first", i32), ("subject_count", i32),
                ("pack_residues", i32), ("plain_unpacked", i32)]


class BpAutotuneTrial(ctypes.Structure):
    _fields_ = [("chunk_residues", i32), ("schedule", i32), ("max_warps", i32), ("ms", ctypes.c_float),
                ("pack_residues", i32), ("plain_unpacked", i32)]


class BpAutotuneOptions(ctypes.Structure):
    _fields_ = [("chunk_sizes", P), ("n_chunk_sizes", i32), ("warp_caps", P), ("n_warp_caps", i32),
                ("schedules_mask", i32), ("model", P), ("cost_weights", ctypes.c_float * 3),
                ("planted_density", ctypes.c_float), ("sample_subjects", i32), ("reps", i32),
                ("pack_sizes", P), ("n_pack_sizes", i32)]


class BpServerOptions(ctypes.Structure):
    _fields_ = [("max_batch_queries", i32), ("device_memory_budget", i64), ("chunk_residues", i32),
                ("schedule", i32), ("lanes", i32), ("poll_us", i32), ("model", P),
                ("cost_weights", ctypes.c_float * 3), ("planted_density", ctypes.c_float), ("params", BpParams),
                ("lane_depth", i32), ("admission", i32), ("segments", i32),
                ("max_wait_ms", i32)]


class BpServerMetrics(ctypes.Structure):
    _fields_ = [("completed", i64), ("failed", i64), ("batches", i64), ("pending", i64), ("mean_batch", ctypes.c_double),
                ("max_in_flight", i32), ("mem_used", i64), ("mem_peak", i64), ("p50_ms", ctypes.c_double),
                ("p99_ms", ctypes.c_double), ("max_ms", ctypes.c_double), ("queries_per_s", ctypes.c_double),
                ("resq_per_s", ctypes.c_double)]


REQ_STATES = {-1: "unknown", 0: "queued", 1: "admitted", 2: "running", 3: "done", 4: "failed"}
SCHED_DYNAMIC, SCHED_STATIC, SCHED_COSTS, SCHED_COST_ORDER = 0, 1, 2, 3
ADMIT_ARRIVAL, ADMIT_SHORTEST = 0, 1
SCHED_NAMES = {0: "dynamic", 1: "static", 2: "learned", 3: "learned_order"}
COST_FEATURES = 24


class BpError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__("%s (%d)%s" % (STATUS_NAMES.get(status, "?"), status, (": " + msg) if msg else ""))


# exported symbol -> (restype, argtypes)
SIGNATURES = {
    "bp_params_default": (None, [P]),
    "bp_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "bp_blosum62_ncbistdaa": (None, [P]),
    "bp_engine_create": (ctypes.c_int, [ctypes.c_int, P]),
    "bp_engine_destroy": (None, [P]),
    "bp_last_error": (ctypes.c_char_p, [P]),
    "bp_engine_stream": (P, [P]),
    "bp_engine_launch_count": (u64, [P]),
    "bp_engine_last_scan_ms": (ctypes.c_float, [P]),
    "bp_engine_synchronize": (ctypes.c_int, [P]),
    "bp_result_digest": (ctypes.c_int, [P, P]),
    "bp_batch_digest": (ctypes.c_int, [P, ctypes.c_int32, P]),
    "bp_server_digest": (ctypes.c_int, [P, ctypes.c_uint64, P]),
    "bp_gapped_params_default": (None, [P]),
    "bp_gapped_run": (ctypes.c_int, [P, P, P]),
    "bp_gapped_run_ring": (ctypes.c_int, [P, P, ctypes.c_int32, P]),
    "bp_gapped_hsps": (ctypes.c_int64, [P]),
    "bp_gapped_ms": (ctypes.c_float, [P]),
    "bp_gapped_copy": (ctypes.c_int, [P, P, P, P]),
    "bp_gapped_destroy": (None, [P]),
    "bp_engine_set_upload_wait": (ctypes.c_int, [P, ctypes.c_uint32]),
    "bp_engine_drop_chunk_flag": (ctypes.c_int, [P, ctypes.c_int32]),
    "bp_db_create": (ctypes.c_int, [P, P, i64, P, i32, P]),
    "bp_db_create_device": (ctypes.c_int, [P, P, i64, P, i32, P]),
    "bp_db_destroy": (None, [P]),
    "bp_dbfile_write": (ctypes.c_int, [ctypes.c_char_p, P, i64, P, i32, i64, i32]),
    "bp_dbfile_info": (ctypes.c_int, [ctypes.c_char_p, P, P, P, P]),
    "bp_dbfile_read_host": (ctypes.c_int, [ctypes.c_char_p, P, P, P]),
    "bp_db_open": (ctypes.c_int, [P, ctypes.c_char_p, P]),
    "bp_db_subjects": (i32, [P]),
    "bp_db_residues": (i64, [P]),
    "bp_query_create": (ctypes.c_int, [P, P, i32, P, P]),
    "bp_query_destroy": (None, [P]),
    "bp_query_table": (ctypes.c_int, [P, P, P, i64, P]),
    "bp_search": (ctypes.c_int, [P, P, P, i32, i32, P]),
    "bp_result_wait": (ctypes.c_int, [P]),
    "bp_result_subjects": (i32, [P]),
    "bp_result_hsps": (i64, [P]),
    "bp_result_copy": (ctypes.c_int, [P, P, P, P]),
    "bp_result_destroy": (None, [P]),
    "bp_blastp_host": (ctypes.c_int, [P, P, i32, P, P, i64, P, i32, P, P, P, i64, P]),
    "bp_search_noalloc": (ctypes.c_int, [P, i32, P, P, i64, P, i32, P, P, P, i64, P, P]),
    "bp_batch_options_default": (None, [P]),
    "bp_batch_plan": (ctypes.c_int, [P, i32, i32, i32, P, P]),
    "bp_search_batch": (ctypes.c_int, [P, P, P, i32, P, P]),
    "bp_batch_run": (ctypes.c_int, [P]),
    "bp_batch_wait": (ctypes.c_int, [P]),
    "bp_batch_hsps": (i64, [P]),
    "bp_batch_items": (i32, [P]),
    "bp_batch_last_scan_ms": (ctypes.c_float, [P]),
    "bp_batch_copy_query": (ctypes.c_int, [P, i32, P, P, P, P]),
    "bp_batch_queue_costs": (ctypes.c_int, [P, P, P]),
    "bp_batch_item_queues": (ctypes.c_int, [P, P]),
    "bp_batch_destroy": (None, [P]),
    "bp_db_chunk_histograms": (ctypes.c_int, [P, P, P, i32, P]),
    "bp_batch_features": (ctypes.c_int, [P, P, P, i32, P, i32, ctypes.c_float, P]),
    "bp_mlp_create": (ctypes.c_int, [P, i32, i32, i32, u64, P]),
    "bp_mlp_destroy": (None, [P]),
    "bp_mlp_num_params": (i32, [P]),
    "bp_mlp_get_params": (ctypes.c_int, [P, P, P]),
    "bp_mlp_set_params": (ctypes.c_int, [P, P, P]),
    "bp_mlp_loss_grad": (ctypes.c_int, [P, P, P, i32, P, P]),
    "bp_mlp_fit": (ctypes.c_int, [P, P, P, i32, i32, i32, ctypes.c_float, u64, P]),
    "bp_mlp_predict": (ctypes.c_int, [P, P, i32, P]),
    "bp_batch_predict_costs": (ctypes.c_int, [P, P, P, P, P, i32, P, i32, ctypes.c_float, P]),
    "bp_autotune_options_default": (None, [P]),
    "bp_cosched_split_costs": (i32, [P, i32, ctypes.c_double]),
    "bp_cosched_split": (ctypes.c_int, [P, P, P, P, P, i32, ctypes.c_float, ctypes.c_double, P]),
    "bp_batch_autotune": (ctypes.c_int, [P, P, P, i32, P, P, P, i32, P]),
    "bp_server_options_default": (None, [P]),
    "bp_server_create": (ctypes.c_int, [P, P, P, P]),
    "bp_server_submit": (ctypes.c_int, [P, P, i32, P]),
    "bp_server_state": (i32, [P, u64]),
    "bp_server_wait": (ctypes.c_int, [P, u64, i32]),
    "bp_server_result": (ctypes.c_int, [P, u64, P, P, P, P, P]),
    "bp_server_release": (ctypes.c_int, [P, u64]),
    "bp_server_stats": (ctypes.c_int, [P, P]),
    "bp_server_destroy": (None, [P]),
    # reference-compatible entry points
    "GPU_BLASTP": (None, [P] * 7 + [ctypes.c_int, P, P, i32, P, i32] + [P] * 7),
    "GPU_BLASTP_get_data": (None, [P, P, i32, P, P, i32, i32]),
    "GPU_BLASTP_free_memory": (None, [P] * 9),
    "GPU_BLASTP_check_memory": (ctypes.c_uint8, [P, P, P, ctypes.c_int, i32, i32, i32, i32, i32]),
    "GPU_BLAST_check_availability": (ctypes.c_uint8, []),
    "Round2Multiple": (None, [P]),
    "GPU_BLASTP_get_hsps": (ctypes.c_uint8, [P, P, P, i64, P]),
}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libblastp_b200.so is not built (%s): run `make -C blastp-cuda_b200` "
                               "or __graft_entry__.build()" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status, engine=None):
    if status != BP_OK:
        msg = ""
        if engine:
            msg = (lib().bp_last_error(engine) or b"").decode(errors="replace")
        raise BpError(status, msg)
