"""ctypes binding of lib/liberq.so (include/erq.h, include/erq_debug.h).

There is no fallback: if the CUDA library is missing or fails to load, every
entry point raises.  Build it with ``make -C extended-rabitq_b200``.
"""
from __future__ import annotations

import ctypes as C
import os

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "lib", "liberq.so")

# erq_status values (include/erq.h)
ERQ_OK = 0
ERQ_ERR_TIMEOUT = 7
STATUS_NAMES = {
    0: "ERQ_OK",
    1: "ERQ_ERR_INVALID_ARGUMENT",
    2: "ERQ_ERR_IO",
    3: "ERQ_ERR_FORMAT",
    4: "ERQ_ERR_UNSUPPORTED",
    5: "ERQ_ERR_CUDA",
    6: "ERQ_ERR_OUT_OF_MEMORY",
    7: "ERQ_ERR_TIMEOUT",
}

# Every symbol include/erq.h and include/erq_debug.h declare.
EXPORTED_SYMBOLS = (
    "erq_version", "erq_status_string", "erq_last_error", "erq_index_load",
    "erq_index_get_info", "erq_index_free", "erq_rotate", "erq_search", "erq_search_raw",
    "erq_search_noalloc", "erq_kmeans", "erq_kmeans_step", "erq_build_index",
    "erq_debug_scan_capacity", "erq_debug_centroid_dists", "erq_debug_probe", "erq_debug_scan",
    "erq_profile_enable", "erq_profile_reset", "erq_profile_read",
    "erq_probe_features", "erq_probe_model_train", "erq_probe_model_save", "erq_probe_model_load",
    "erq_probe_model_free", "erq_probe_model_predict", "erq_search_learned",
    "erq_search_learned_raw",
    "erq_debug_probe_model_grads", "erq_debug_probe_model_params",
    "erq_plan_create", "erq_plan_free", "erq_plan_set_learned", "erq_plan_autotune",
    "erq_plan_set_tuning", "erq_plan_get_tuning", "erq_plan_search", "erq_plan_device_bytes", "erq_plan_set_graphs", "erq_plan_set_pipeline", "erq_plan_search_async", "erq_debug_gemm_bf16", "erq_debug_set_gemm_wait_limit", "erq_debug_probe_fallbacks", "erq_debug_refine_stats",
)


class ErqError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        self.status_name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{self.status_name}: {message}")


class PlanTuning(C.Structure):
    _fields_ = [
        ("queries_per_item", C.c_uint32),
        ("blocks_per_item", C.c_uint32),
        ("warps", C.c_uint32),
        ("refine_warps", C.c_uint32),
    ]

    def as_dict(self):
        return {"queries_per_item": self.queries_per_item, "blocks_per_item": self.blocks_per_item,
                "warps": self.warps, "refine_warps": self.refine_warps}


class IndexInfo(C.Structure):
    _fields_ = [
        ("n", C.c_uint64),
        ("dim", C.c_uint64),
        ("padded_dim", C.c_uint64),
        ("num_clusters", C.c_uint64),
        ("ex_bits", C.c_uint64),
        ("device_bytes", C.c_uint64),
        ("device", C.c_int),
        ("block_factors", C.c_int),
    ]


_lib = None


def load_library(path: str | None = None) -> C.CDLL:
    """Load liberq.so once and declare its signatures."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is not built; run `make -C {PKG_ROOT}` (this package has no CPU fallback)")
    lib = C.CDLL(path)
    vp, u64, f32p, u32p = C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p
    lib.erq_version.restype = C.c_int
    lib.erq_status_string.argtypes = [C.c_int]
    lib.erq_status_string.restype = C.c_char_p
    lib.erq_last_error.restype = C.c_char_p
    lib.erq_index_load.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]
    lib.erq_index_load.restype = C.c_int
    lib.erq_index_get_info.argtypes = [vp, C.POINTER(IndexInfo)]
    lib.erq_index_get_info.restype = C.c_int
    lib.erq_index_free.argtypes = [vp]
    lib.erq_index_free.restype = None
    lib.erq_rotate.argtypes = [vp, f32p, u64, f32p, vp]
    lib.erq_rotate.restype = C.c_int
    lib.erq_search.argtypes = [vp, f32p, u64, u64, u64, u32p, f32p, vp]
    lib.erq_search.restype = C.c_int
    lib.erq_search_raw.argtypes = [vp, f32p, u64, u64, u64, u32p, f32p, vp]
    lib.erq_search_raw.restype = C.c_int
    lib.erq_search_noalloc.argtypes = [vp, f32p, u64, u64, u64, u32p, f32p, vp]
    lib.erq_search_noalloc.restype = C.c_int
    lib.erq_build_index.argtypes = [vp, u64, u64, vp, u64, vp, u64, vp, u64, C.c_char_p, C.c_int]
    lib.erq_build_index.restype = C.c_int
    lib.erq_kmeans.argtypes = [vp, u64, u64, u64, C.c_int, u64, vp, vp, C.c_int]
    lib.erq_kmeans.restype = C.c_int
    lib.erq_kmeans_step.argtypes = [vp, u64, u64, u64, vp, u64, vp, vp, vp, C.c_int]
    lib.erq_kmeans_step.restype = C.c_int
    lib.erq_debug_scan_capacity.argtypes = [vp, u64, u64]
    lib.erq_debug_scan_capacity.restype = u64
    lib.erq_debug_centroid_dists.argtypes = [vp, f32p, u64, f32p]
    lib.erq_debug_centroid_dists.restype = C.c_int
    lib.erq_debug_probe.argtypes = [vp, f32p, u64, u64, u32p, f32p]
    lib.erq_debug_probe.restype = C.c_int
    lib.erq_debug_scan.argtypes = [vp, f32p, u64, u64, u32p, f32p, f32p, f32p, vp, vp, u64]
    lib.erq_debug_scan.restype = C.c_int
    lib.erq_plan_create.argtypes = [vp, vp, u64, u64, u64, C.c_int, C.POINTER(C.c_void_p)]
    lib.erq_plan_create.restype = C.c_int
    lib.erq_plan_free.argtypes = [vp]
    lib.erq_plan_free.restype = None
    lib.erq_plan_set_learned.argtypes = [vp, C.c_float, C.c_float]
    lib.erq_plan_set_learned.restype = C.c_int
    lib.erq_plan_autotune.argtypes = [vp, vp, u64, C.c_int, C.POINTER(PlanTuning),
                                      C.POINTER(C.c_float)]
    lib.erq_plan_autotune.restype = C.c_int
    lib.erq_plan_set_tuning.argtypes = [vp, u64, C.POINTER(PlanTuning)]
    lib.erq_plan_set_tuning.restype = C.c_int
    lib.erq_plan_get_tuning.argtypes = [vp, u64, C.POINTER(PlanTuning)]
    lib.erq_plan_get_tuning.restype = C.c_int
    lib.erq_plan_search.argtypes = [vp, vp, u64, vp, vp, vp, vp]
    lib.erq_plan_search.restype = C.c_int
    lib.erq_plan_device_bytes.argtypes = [vp]
    lib.erq_plan_device_bytes.restype = u64
    lib.erq_debug_gemm_bf16.argtypes = [vp, vp, u64, u64, u64, vp, C.c_int]
    lib.erq_debug_gemm_bf16.restype = C.c_int
    lib.erq_debug_set_gemm_wait_limit.argtypes = [C.c_uint32]
    lib.erq_debug_set_gemm_wait_limit.restype = C.c_int
    lib.erq_debug_probe_fallbacks.argtypes = [C.c_int, C.POINTER(C.c_uint64), C.c_int]
    lib.erq_debug_probe_fallbacks.restype = C.c_int
    lib.erq_debug_refine_stats.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_uint64)]
    lib.erq_debug_refine_stats.restype = C.c_int
    lib.erq_plan_search_async.argtypes = [vp, vp, u64, vp, vp, vp, vp]
    lib.erq_plan_search_async.restype = C.c_int
    lib.erq_plan_set_pipeline.argtypes = [vp, C.c_int]
    lib.erq_plan_set_pipeline.restype = C.c_int
    lib.erq_plan_set_graphs.argtypes = [vp, C.c_int]
    lib.erq_plan_set_graphs.restype = C.c_int
    lib.erq_profile_enable.argtypes = [C.c_int]
    lib.erq_profile_enable.restype = None
    lib.erq_profile_reset.restype = None
    lib.erq_profile_read.argtypes = [C.c_char_p, C.POINTER(C.c_uint64), C.POINTER(C.c_double)]
    lib.erq_profile_read.restype = C.c_int
    lib.erq_probe_features.argtypes = [vp, f32p, u64, f32p, vp]
    lib.erq_probe_features.restype = C.c_int
    lib.erq_probe_model_train.argtypes = [vp, vp, u64, vp, C.c_int, C.c_int, C.c_float, u64,
                                          C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_float)]
    lib.erq_probe_model_train.restype = C.c_int
    lib.erq_probe_model_save.argtypes = [vp, C.c_char_p]
    lib.erq_probe_model_save.restype = C.c_int
    lib.erq_probe_model_load.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]
    lib.erq_probe_model_load.restype = C.c_int
    lib.erq_probe_model_free.argtypes = [vp]
    lib.erq_probe_model_free.restype = None
    lib.erq_probe_model_predict.argtypes = [vp, vp, u64, vp, vp]
    lib.erq_probe_model_predict.restype = C.c_int
    lib.erq_search_learned.argtypes = [vp, vp, f32p, u64, u64, u64, C.c_float, C.c_float, u32p,
                                       f32p, vp, vp]
    lib.erq_search_learned.restype = C.c_int
    lib.erq_search_learned_raw.argtypes = lib.erq_search_learned.argtypes
    lib.erq_search_learned_raw.restype = C.c_int
    lib.erq_debug_probe_model_grads.argtypes = [vp, vp, vp, u64, C.POINTER(C.c_float), vp]
    lib.erq_debug_probe_model_grads.restype = C.c_int
    lib.erq_debug_probe_model_params.argtypes = [vp, vp, vp, vp, vp]
    lib.erq_debug_probe_model_params.restype = C.c_int
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != ERQ_OK:
        msg = load_library().erq_last_error().decode(errors="replace")
        raise ErqError(status, msg)


KERNELS = ("rotate", "centroid_dist", "select_probe", "scan", "refine", "split", "gemm",
           "probe", "order", "mlp")


def profile_enable(on: bool = True) -> None:
    load_library().erq_profile_enable(1 if on else 0)


def profile_reset() -> None:
    load_library().erq_profile_reset()


def probe_fallbacks(device: int = 0, reset: bool = True) -> int:
    """Queries whose probe fell back to all K exact distances since the last reset."""
    n = C.c_uint64()
    check(load_library().erq_debug_probe_fallbacks(device, C.byref(n), 1 if reset else 0))
    return int(n.value)


def refine_stats(device: int = 0, enable: bool = False) -> dict:
    """Refinement counters since the last call (exact candidates, distances
    computed, windows, window blocks); counting is then on for later
    refinement launches when `enable` (graphs captured earlier keep their
    setting)."""
    v = (C.c_uint64 * 4)()
    check(load_library().erq_debug_refine_stats(device, 1 if enable else 0, v))
    return dict(zip(("candidates", "refined", "windows", "blocks"), (int(x) for x in v)))


def profile_read() -> dict:
    """{kernel: (launches, total_ms)} since the last reset (waits for the events)."""
    lib = load_library()
    out = {}
    for k in KERNELS:
        n, ms = C.c_uint64(), C.c_double()
        check(lib.erq_profile_read(k.encode(), C.byref(n), C.byref(ms)))
        out[k] = (int(n.value), float(ms.value))
    return out
