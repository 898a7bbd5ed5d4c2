"""ctypes binding of libqsketch.so (the C ABI declared in include/qsketch_c.h).

The shared library is built in-tree by ``python qsketch_b200/build.py``.  There is no
fallback: importing this module without the library raises ImportError.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libqsketch.so")

QS_OK = 0
QS_ERR_INVALID_ARG = 1
QS_ERR_OOM = 2
QS_ERR_CUDA = 3
QS_ERR_POOL_FULL = 4
QS_ERR_TIMEOUT = 5
QS_ERR_NO_DEVICE = 6
QS_ERR_CAPACITY = 7

QS_KIND_MSWS = 0
QS_KIND_PLAIN_CM = 1
QS_KIND_BUCKET = 2
QS_FLAG_COMPAT_V3 = 0x1
QS_FLAG_NO_CHUNK_RAMP = 0x2


class qs_params(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_uint32),
        ("flags", ctypes.c_uint32),
        ("n_low", ctypes.c_uint64),
        ("low_bytes", ctypes.c_uint64),
        ("m_low", ctypes.c_uint32),
        ("m_high", ctypes.c_uint32),
        ("n_high", ctypes.c_uint64),
        ("seed_sz", ctypes.c_uint32),
        ("hash_mask_table_sz", ctypes.c_uint32),
        ("hash_mask_ones", ctypes.c_uint32),
        ("hash_seed", ctypes.c_uint32),
        ("seed_rng", ctypes.c_uint32),
        ("mask_rng", ctypes.c_uint32),
        ("seeds", ctypes.c_void_p),
        ("mask_table", ctypes.c_void_p),
        ("max_batch", ctypes.c_uint64),
        ("device", ctypes.c_int32),
        ("lanes_per_key", ctypes.c_uint32),
        ("aggregate", ctypes.c_uint32),
        ("route", ctypes.c_uint32),
        ("ctas_per_sm", ctypes.c_uint32),
        ("first_chunk", ctypes.c_uint64),
        ("keys_per_tile", ctypes.c_uint32),
    ]


class qs_stats(ctypes.Structure):
    _fields_ = [
        ("status_bits", ctypes.c_uint32),
        ("next_level_id", ctypes.c_uint32),
        ("linked_buckets", ctypes.c_uint64),
        ("dropped_keys", ctypes.c_uint64),
        ("repaired_buckets", ctypes.c_uint64),
        ("repaired_keys", ctypes.c_uint64),
        ("inserted_keys", ctypes.c_uint64),
    ]


class qs_profile(ctypes.Structure):
    _fields_ = [
        ("insert_ms", ctypes.c_double),
        ("repair_ms", ctypes.c_double),
        ("query_ms", ctypes.c_double),
        ("insert_timed", ctypes.c_uint64),
        ("repair_timed", ctypes.c_uint64),
        ("query_timed", ctypes.c_uint64),
        ("insert_launches", ctypes.c_uint64),
        ("repair_launches", ctypes.c_uint64),
        ("query_launches", ctypes.c_uint64),
        ("repairs_active", ctypes.c_uint64),
        ("repair_phase_ms", ctypes.c_double * 12),
    ]


class qs_learned_params(ctypes.Structure):
    _fields_ = [
        ("budget_bytes", ctypes.c_uint64),
        ("table_slots", ctypes.c_uint32),
        ("table_max_fill", ctypes.c_float),
        ("warmup_keys", ctypes.c_uint64),
        ("heavy_fraction", ctypes.c_double),
        ("epochs", ctypes.c_uint32),
        ("batch", ctypes.c_uint32),
        ("lr", ctypes.c_float),
        ("max_pos_weight", ctypes.c_float),
        ("eligible_recall", ctypes.c_float),
        ("hash_seed", ctypes.c_uint32),
        ("seed_rng", ctypes.c_uint32),
        ("mask_rng", ctypes.c_uint32),
        ("init_seed", ctypes.c_uint32),
        ("max_batch", ctypes.c_uint64),
        ("device", ctypes.c_int32),
        ("neg_per_pos", ctypes.c_uint32),
        ("replay_warmup", ctypes.c_uint32),
    ]


class qs_learned_info(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in (
        "budget_bytes", "sketch_bytes", "table_bytes", "mlp_bytes", "n_low", "n_high", "table_slots", "table_fill",
        "warmup_keys", "warmup_seen", "train_examples", "train_positives", "admitted_after_warmup")] + \
        [(n, ctypes.c_uint32) for n in ("threshold", "trained", "epochs", "steps")] + \
        [(n, ctypes.c_float) for n in ("pos_weight", "loss_first", "loss_last", "train_precision", "train_recall",
                                       "logit_threshold")] + \
        [("train_ms", ctypes.c_double), ("warmup_replayed", ctypes.c_uint64),
         ("train_phase_ms", ctypes.c_double * 5)]


class qs_batch_params(ctypes.Structure):
    _fields_ = [
        ("n_streams", ctypes.c_uint32),
        ("n_low", ctypes.c_void_p),
        ("n_high", ctypes.c_void_p),
        ("hash_seeds", ctypes.c_void_p),
        ("seed_rng", ctypes.c_uint32),
        ("mask_rng", ctypes.c_uint32),
        ("hash_mask_table_sz", ctypes.c_uint32),
        ("hash_mask_ones", ctypes.c_uint32),
        ("mask_table", ctypes.c_void_p),
        ("flags", ctypes.c_uint32),
        ("aggregate", ctypes.c_uint32),
        ("route", ctypes.c_uint32),
        ("lanes_per_key", ctypes.c_uint32),
        ("ctas_per_sm", ctypes.c_uint32),
        ("max_batch", ctypes.c_uint64),
        ("first_chunk", ctypes.c_uint64),
        ("device", ctypes.c_int32),
        ("class_lanes_per_key", ctypes.c_void_p),
    ]


class qs_tune_config(ctypes.Structure):
    _fields_ = [("lanes_per_key", ctypes.c_uint32), ("aggregate", ctypes.c_uint32), ("route", ctypes.c_uint32),
                ("ctas_per_sm", ctypes.c_uint32), ("max_batch", ctypes.c_uint64), ("first_chunk", ctypes.c_uint64),
                ("keys_per_tile", ctypes.c_uint32), ("pad", ctypes.c_uint32), ("insert_ms", ctypes.c_double)]


class qs_batch_info(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in (
        "n_streams", "low_buckets", "high_buckets", "table_bytes", "max_batch", "inserts", "queries",
        "graph_launches", "launches")] + [("graph_capture", ctypes.c_uint32), ("streams_pool_full", ctypes.c_uint32)]


QS_MLP_PARAMS = 20865

# Every symbol include/qsketch_c.h declares, with its ctypes signature.
_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64
_SZ = ctypes.c_size_t
_I = ctypes.c_int
SIGNATURES = {
    "qs_abi_version": (_U32, []),
    "qs_status_string": (ctypes.c_char_p, [_I]),
    "qs_last_error_string": (ctypes.c_char_p, []),
    "qs_params_default": (None, [ctypes.POINTER(qs_params)]),
    "qs_find_greatest_prime": (_U64, [_U64]),
    "qs_number_of_buckets": (_U64, [_U64, _U64, ctypes.c_double, _U32]),
    "qs_generate_hashmask": (_I, [_U32, _SZ, _SZ, _SZ, _SZ, _P]),
    "qs_draw_seeds": (_I, [_U32, _SZ, _P]),
    "qs_create": (_I, [ctypes.POINTER(qs_params), ctypes.POINTER(_P)]),
    "qs_destroy": (_I, [_P]),
    "qs_insert": (_I, [_P, _P, _SZ, _P]),
    "qs_remove": (_I, [_P, _P, _SZ, _P]),
    "qs_get_params": (_I, [_P, ctypes.POINTER(qs_params)]),
    "qs_snapshot_bytes": (_I, [_P, ctypes.POINTER(_U64)]),
    "qs_snapshot_save": (_I, [_P, _P, _U64]),
    "qs_snapshot_load": (_I, [_P, _U64, ctypes.c_int32, ctypes.POINTER(_P)]),
    "qs_save": (_I, [_P, ctypes.c_char_p]),
    "qs_load": (_I, [ctypes.c_char_p, ctypes.c_int32, ctypes.POINTER(_P)]),
    "qs_query": (_I, [_P, _P, _SZ, _P, _P]),
    "qs_insert_host": (_I, [_P, _P, _SZ]),
    "qs_query_host": (_I, [_P, _P, _SZ, _P]),
    "qs_clear": (_I, [_P, _P]),
    "qs_sync": (_I, [_P, _P]),
    "qs_get_stats": (_I, [_P, ctypes.POINTER(qs_stats)]),
    "qs_reset_status": (_I, [_P]),
    "qs_set_profiling": (_I, [_P, _I]),
    "qs_get_profile": (_I, [_P, ctypes.POINTER(qs_profile)]),
    "qs_get_info": (_I, [_P, ctypes.POINTER(_U64), ctypes.POINTER(_U64), ctypes.POINTER(_U32), _P, _P]),
    "qs_get_tables": (_I, [_P, _P, _P]),
    "qs_gen_keys": (_I, [_U32, _U64, _U64, ctypes.c_double, _U64, _P, _P, _SZ, _P]),
    "qs_gen_rank_keys": (_I, [_U64, _U64, _P, _SZ, _P]),
    "qs_gen_class_keys": (_I, [_U64, _U32, ctypes.c_double, ctypes.c_double, _U64, _P, _SZ, _P]),
    "qs_rank_histogram": (_I, [_P, _SZ, _P, _U64, _P]),
    "qs_error_metrics": (_I, [_P, _P, _SZ, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), _P]),
    "qs_probe": (_I, [_U32, _U64, _U64, ctypes.POINTER(ctypes.c_double)]),
    "qs_test_fail_allocations": (None, [ctypes.c_int32]),
    "qs_shard_scratch_words": (_SZ, [_SZ, _U32]),
    "qs_shard_partition": (_I, [_P, _SZ, _U32, _U64, _U32, _P, _P, _P, _P, _P]),
    "qs_shard_unpartition": (_I, [_P, _P, _SZ, _P, _P]),
    "qs_msws_insert_noalloc": (_I, [_P, _U64, _P, _U64, _P, _P, _U32, _U32, _U32, _P, _SZ, _P]),
    "qs_autotune": (_I, [ctypes.POINTER(qs_params), _P, _SZ, _U32, ctypes.POINTER(qs_tune_config), _P, _U32,
                         ctypes.POINTER(_U32)]),
    "qs_autotune_lookup": (_I, [_U64, ctypes.POINTER(qs_tune_config)]),
    "qs_autotune_reset": (None, []),
    "qs_batch_params_default": (None, [ctypes.POINTER(qs_batch_params)]),
    "qs_batch_create": (_I, [ctypes.POINTER(qs_batch_params), ctypes.POINTER(_P)]),
    "qs_batch_destroy": (_I, [_P]),
    "qs_batch_insert": (_I, [_P, _P, _P, _U64, _P]),
    "qs_batch_query": (_I, [_P, _P, _P, _U64, _P, _P]),
    "qs_batch_insert_graph": (_I, [_P, _P, _P, _U64, _P]),
    "qs_batch_query_graph": (_I, [_P, _P, _P, _U64, _P, _P]),
    "qs_batch_autotune": (_I, [_P, _P, _P, _U64, _U32, _P]),
    "qs_batch_clear": (_I, [_P, _P]),
    "qs_batch_sync": (_I, [_P, _P]),
    "qs_batch_stream_status": (_I, [_P, _P]),
    "qs_batch_seeds": (_I, [_P, _P]),
    "qs_batch_get_info": (_I, [_P, ctypes.POINTER(qs_batch_info)]),
    "qs_batch_arena": (_P, [_P]),
    "qs_learned_params_default": (None, [ctypes.POINTER(qs_learned_params)]),
    "qs_learned_admit_keys": (_I, [_P, _P, _SZ]),
    "qs_learned_create": (_I, [ctypes.POINTER(qs_learned_params), ctypes.POINTER(_P)]),
    "qs_learned_destroy": (_I, [_P]),
    "qs_learned_insert": (_I, [_P, _P, _SZ, _P]),
    "qs_learned_query": (_I, [_P, _P, _SZ, _P, _P]),
    "qs_learned_get_info": (_I, [_P, ctypes.POINTER(qs_learned_info)]),
    "qs_learned_get_table": (_I, [_P, _P, _P, ctypes.POINTER(_U32)]),
    "qs_mlp_get_params": (_I, [_P, _P]),
    "qs_mlp_set_params": (_I, [_P, _P]),
    "qs_mlp_forward": (_I, [_P, _P, _SZ, _P, _P]),
    "qs_mlp_grads": (_I, [_P, _P, _P, _SZ, ctypes.c_float, _P, ctypes.POINTER(ctypes.c_double)]),
    "qs_mlp_train": (_I, [_P, _P, _P, _SZ, _U32, _U32, ctypes.c_float, ctypes.c_float,
                          ctypes.POINTER(ctypes.c_double)]),
}
QS_NOALLOC_MAX_KEYS = 1 << 18
QS_NOALLOC_MAX_BUCKETS = 1 << 26
QS_MSWS_STATE_BYTES = 256
QS_MSWS_STATE_ALIGN = 16


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python qsketch_b200/build.py` "
            "(there is no CPU fallback for the sketch kernels)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class QsError(RuntimeError):
    """A non-OK qs_status; ``.status`` holds the code."""

    def __init__(self, status, where=""):
        self.status = status
        text = lib.qs_status_string(status).decode()
        detail = lib.qs_last_error_string().decode()
        super().__init__(f"{where}: {text} ({detail})" if where else f"{text} ({detail})")


def check(status, where=""):
    if status != QS_OK:
        raise QsError(status, where)
    return status
