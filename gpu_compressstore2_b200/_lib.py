"""ctypes bindings of the C ABI in include/compressstore.h (libcompressstore.so).

The shared library is the product; this module only declares its signatures. Loading
fails loudly if the library has not been built: there is no Python or CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libcompressstore.so"
CUB_PATH = PKG / "libcs_cubflagged.so"

c_u64 = ctypes.c_uint64
c_u32 = ctypes.c_uint32
c_i32 = ctypes.c_int32
c_int = ctypes.c_int
c_vp = ctypes.c_void_p
c_size = ctypes.c_size_t

# cs_status
PENDING = 1
SUCCESS = 0
ERR_INVALID_VALUE = -1
ERR_MISALIGNED = -2
ERR_WORKSPACE = -3
ERR_CUDA = -4
ERR_TIMEOUT = -5
ERR_NO_DEVICE = -6
ERR_OUT_OF_MEMORY = -7
ERR_NOT_SUPPORTED = -8
ERR_ADMISSION = -9

# cs_algo
ALGO_AUTO = 0
ALGO_1PASS = 1
ALGO_3PASS = 2
ALGO_NAIVE = 3

COUNT_ERROR = 0xFFFFFFFFFFFFFFFF

# cs_serve_mode
SERVE_BATCH = 0
SERVE_PER_CALL = 1


class CsConfig(ctypes.Structure):
    _fields_ = [
        ("algo", c_i32),
        ("chunk_length", c_u32),
        ("grid_dim", c_u32),
        ("skip", c_u32),
        ("timeout_ns", c_u64),
        ("selectivity", ctypes.c_float),
    ]


class CsColumn(ctypes.Structure):
    _fields_ = [
        ("d_in", c_vp),
        ("d_mask", c_vp),
        ("d_out", c_vp),
        ("n", c_u64),
        ("elem_bytes", c_u32),
        ("reserved", c_u32),
        ("d_count", c_vp),
    ]


class CsPredicate(ctypes.Structure):
    _fields_ = [
        ("op", c_i32),
        ("type", c_i32),
        ("a", c_u64),
        ("b", c_u64),
    ]


# cs_pred_op / cs_elem_type
PRED_LT, PRED_LE, PRED_GT, PRED_GE, PRED_EQ, PRED_NE, PRED_BETWEEN = range(7)
TYPE_U8, TYPE_U16, TYPE_U32, TYPE_U64, TYPE_I8, TYPE_I16, TYPE_I32, TYPE_I64, TYPE_F32, TYPE_F64 = range(10)


class CsServerConfig(ctypes.Structure):
    _fields_ = [
        ("out_budget_bytes", c_u64),
        ("max_batch_elems", c_u64),
        ("max_batch", c_u32),
        ("slots", c_u32),
        ("mode", c_i32),
        ("reserved", c_u32),
        ("timeout_ns", c_u64),
    ]


class CsRequest(ctypes.Structure):
    _fields_ = [
        ("d_in", c_vp),
        ("d_mask", c_vp),
        ("n", c_u64),
        ("elem_bytes", c_u32),
        ("reserved", c_u32),
    ]


class CsResult(ctypes.Structure):
    _fields_ = [
        ("d_out", c_vp),
        ("count", c_u64),
        ("latency_ns", c_u64),
        ("queue_ns", c_u64),
        ("status", c_i32),
        ("batch_size", c_u32),
    ]


class CsServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", c_u64),
        ("completed", c_u64),
        ("rejected", c_u64),
        ("batches", c_u64),
        ("batched_requests", c_u64),
        ("arena_bytes", c_u64),
        ("arena_used", c_u64),
        ("arena_peak", c_u64),
        ("kernel_launches", c_u64),
    ]


# name -> (restype, argtypes); every symbol include/compressstore.h declares
SIGNATURES: dict[str, tuple] = {
    "compressstore": (c_int, [c_vp, c_vp, c_vp, c_u64, c_u32, c_vp, c_vp]),
    "compressstore_cfg": (c_int, [c_vp, c_vp, c_vp, c_u64, c_u32, c_vp, ctypes.POINTER(CsConfig), c_vp]),
    "compressstore_noalloc": (c_int, [c_vp, c_vp, c_vp, c_u64, c_u32, c_vp, c_vp]),
    "compressstore_workspace_size": (c_size, [c_u64, c_u32, ctypes.POINTER(CsConfig)]),
    "cs_workspace_init": (c_int, [c_vp, c_size, c_vp]),
    "compressstore_ex": (c_int, [c_vp, c_vp, c_vp, c_u64, c_u32, c_vp, c_vp, c_size, ctypes.POINTER(CsConfig), c_vp]),
    "compressstore_if": (c_int, [c_vp, c_vp, c_u64, ctypes.POINTER(CsPredicate), c_vp, c_vp, c_vp]),
    "compressstore_pattern": (c_int, [c_vp, c_vp, c_u64, c_u32, c_u32, c_u32, c_vp, c_vp]),
    "compressstore_host": (c_int, [c_vp, c_vp, c_vp, c_u64, c_u32, ctypes.POINTER(c_u64), ctypes.POINTER(CsConfig)]),
    "cs_workspace_check": (c_int, [c_vp, c_vp]),
    "compressstore_check": (c_int, [c_vp]),
    "compressstore_release": (c_int, [c_vp]),
    "compressstore_host_release": (c_int, []),
    "cs_popc_chunks": (c_int, [c_vp, c_u64, c_u32, c_vp, c_vp]),
    "cs_scan_workspace_size": (c_size, [c_u64]),
    "cs_chunk_prefix_sum": (c_int, [c_vp, c_u64, c_vp, c_vp, c_vp, c_size, c_vp]),
    "cs_writeout": (c_int, [c_vp, c_vp, c_vp, c_u64, c_u32, c_vp, c_vp, c_u32, c_i32, c_vp]),
    "cs_gen_payload": (c_int, [c_vp, c_u64, c_u32, c_u64, c_i32, c_vp]),
    "cs_gen_mask_bernoulli": (c_int, [c_vp, c_u64, ctypes.c_double, c_u64, c_vp]),
    "cs_gen_mask_runs_workspace_size": (c_size, [c_u64]),
    "cs_gen_mask_runs": (c_int, [c_vp, c_u64, ctypes.c_double, c_u64, c_vp, c_size, c_vp]),
    "cs_gen_mask_dense_prefix": (c_int, [c_vp, c_u64, ctypes.c_float, c_vp]),
    "cs_gen_mask_pattern": (c_int, [c_vp, c_u64, c_u32, c_u32, c_vp]),
    "cs_batch_create": (c_int, [ctypes.POINTER(c_vp), ctypes.POINTER(CsColumn), c_u32, ctypes.POINTER(CsConfig), c_vp]),
    "cs_batch_run": (c_int, [c_vp, c_vp]),
    "cs_batch_graph": (c_int, [c_vp, c_vp]),
    "cs_batch_check": (c_int, [c_vp, c_vp]),
    "cs_batch_device_bytes": (c_u64, [c_vp]),
    "cs_batch_launches": (c_u32, [c_vp]),
    "cs_batch_one_pass_columns": (c_u32, [c_vp]),
    "cs_batch_run_per_call": (c_int, [c_vp, c_vp]),
    "cs_batch_destroy": (c_int, [c_vp]),
    "cs_server_create": (c_int, [ctypes.POINTER(c_vp), ctypes.POINTER(CsServerConfig)]),
    "cs_server_submit": (c_int, [c_vp, ctypes.POINTER(CsRequest), ctypes.POINTER(c_u64)]),
    "cs_server_poll": (c_int, [c_vp, c_u64, ctypes.POINTER(CsResult)]),
    "cs_server_wait": (c_int, [c_vp, c_u64, c_u64, ctypes.POINTER(CsResult)]),
    "cs_server_next": (c_int, [c_vp, c_u64, ctypes.POINTER(c_u64), ctypes.POINTER(CsResult)]),
    "cs_server_release": (c_int, [c_vp, c_u64]),
    "cs_server_stats_get": (c_int, [c_vp, ctypes.POINTER(CsServerStats)]),
    "cs_server_replay": (c_int, [c_vp, ctypes.POINTER(CsRequest), ctypes.POINTER(c_u64), c_u32,
                                 ctypes.POINTER(CsResult)]),
    "cs_server_destroy": (c_int, [c_vp]),
    "cs_tune_set": (c_int, [c_u32, c_i32, c_i32, c_u32]),
    "cs_tune_get": (c_int, [c_u32, c_u64, ctypes.POINTER(c_i32), ctypes.POINTER(c_u32)]),
    "cs_tune_size_bucket": (c_int, [c_u64]),
    "cs_tune_batch_set": (c_int, [c_u32, c_i32, c_i32, c_i32]),
    "cs_tune_batch_get": (c_int, [c_u32, c_u64, ctypes.c_double, ctypes.POINTER(c_i32)]),
    "cs_tune_sel_set": (c_int, [c_u32, c_i32, c_i32, c_i32, c_u32]),
    "cs_tune_sel_get": (c_int, [c_u32, c_u64, ctypes.c_double, ctypes.POINTER(c_i32), ctypes.POINTER(c_u32)]),
    "cs_tune_sel_bucket": (c_int, [ctypes.c_double]),
    "cs_tune_load": (c_int, [ctypes.c_char_p]),
    "cs_tune_save": (c_int, [ctypes.c_char_p]),
    "cs_status_string": (ctypes.c_char_p, [c_int]),
    "cs_launch_count": (c_u64, []),
    "cs_tile_elems": (c_u32, [c_u32]),
    "cs_compact_smem_bytes": (c_u32, [c_u32, c_i32]),
    "cs_version": (c_u32, []),
}

CUB_SIGNATURES: dict[str, tuple] = {
    "cs_cub_flagged_temp_bytes": (c_size, [c_u64, c_u32]),
    "cs_cub_flagged": (c_int, [c_vp, c_vp, c_vp, c_u64, c_u32, c_vp, c_vp, c_size, c_vp]),
}


class CsError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = _lib.cs_status_string(status).decode() if _lib is not None else str(status)
        super().__init__(f"{what}: {msg} ({status})" if what else f"{msg} ({status})")


def _bind(lib: ctypes.CDLL, sigs: dict) -> ctypes.CDLL:
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def _load(path: Path, sigs: dict, what: str) -> ctypes.CDLL:
    if not path.exists():
        raise ImportError(
            f"{what} not built: {path} is missing. Build it with "
            f"`python -m gpu_compressstore2_b200.build` (nvcc, sm_100a)."
        )
    return _bind(ctypes.CDLL(str(path), mode=os.RTLD_NOW | os.RTLD_LOCAL), sigs)


_lib: ctypes.CDLL | None = None
_cub: ctypes.CDLL | None = None


TUNE_TABLE = PKG / "tune_b200.txt"  # autotuner output measured on B200 (cs_tune_save format)


def lib() -> ctypes.CDLL:
    """Load libcompressstore.so; installs the packaged autotuner table unless the
    environment names one (CS_TUNE_TABLE)."""
    global _lib
    if _lib is None:
        loaded = _load(LIB_PATH, SIGNATURES, "libcompressstore.so")
        if not os.environ.get("CS_TUNE_TABLE") and TUNE_TABLE.exists():
            st = loaded.cs_tune_load(str(TUNE_TABLE).encode())
            if st != SUCCESS:
                raise ImportError(f"{TUNE_TABLE}: not a valid tuning table ({st})")
        _lib = loaded
    return _lib


def cub() -> ctypes.CDLL:
    global _cub
    if _cub is None:
        _cub = _load(CUB_PATH, CUB_SIGNATURES, "libcs_cubflagged.so")
    return _cub


def check(status: int, what: str = "") -> None:
    if status != SUCCESS:
        raise CsError(status, what)
