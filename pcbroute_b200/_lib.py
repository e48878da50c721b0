"""ctypes bindings of the pcbg C ABI (include/pcbg.h) in pcbroute_b200/lib/libpcbgpu.so.

The library is built in-tree (python -m pcbroute_b200.build). There is no fallback: if it is missing, load()
raises, and every entry point that needs it fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

from . import build as _build

LIB_PATH = _build.LIB

# the symbols include/pcbg.h declares (C linkage) and include/gpu.h declares (C++ linkage, mangled)
PCBG_SYMBOLS = [
    "pcbg_available", "pcbg_configure", "pcbg_solve", "pcbg_host_acquire", "pcbg_host_release", "pcbg_last_error",
    "pcbg_solve_batch", "pcbg_solve_noalloc", "pcbg_batch_window", "pcbg_batcher_stats", "pcbg_spec_create",
    "pcbg_spec_destroy", "pcbg_spec_set_scheduler", "pcbg_spec_set_observer", "pcbg_spec_iterate", "pcbg_spec_path",
    "pcbg_spec_add_history", "pcbg_spec_window_reads", "pcbg_spec_net", "pcbg_spec_board", "pcbg_spec_costs",
    "pcbg_sched_create", "pcbg_sched_destroy", "pcbg_sched_attach", "pcbg_sched_attach_logger", "pcbg_sched_label",
    "pcbg_sched_log_size", "pcbg_sched_train", "pcbg_sched_counts", "pcbg_sched_nparams", "pcbg_sched_get_params",
    "pcbg_sched_set_params", "pcbg_sched_forward_host", "pcbg_sched_grad_host", "pcbg_last_batch_tile_visits", "pcbg_last_batch_layer_visits", "pcbg_last_batch_rounds",
    "pcbg_last_batch_kernel_ms", "pcbg_last_batch_launches", "pcbg_last_batch_local_iters", "pcbg_synth_search",
    "pcbg_last_batch_deferred", "pcbg_last_batch_dropped", "pcbg_set_round_band", "pcbg_round_band",
    "pcbg_set_max_rounds", "pcbg_last_batch_settled", "pcbg_mirror_class", "pcbg_mirror_spans",
    "pcbg_mirror_history", "pcbg_mirror_download", "pcbg_sched_add_log_host", "pcbg_rsched_mode",
    "pcbg_rsched_begin", "pcbg_rsched_net", "pcbg_rsched_allow", "pcbg_rsched_started", "pcbg_rsched_committed",
    "pcbg_rsched_verdict", "pcbg_rsched_end", "pcbg_rsched_get_stats", "pcbg_autotune", "pcbg_autotune_batch",
    "pcbg_last_batch_blocks_per_sm", "pcbg_last_batch_busy_frac", "pcbg_set_visit_order", "pcbg_visit_order",
    "pcbg_synth_search_host", "pcbg_costs_create", "pcbg_costs_destroy", "pcbg_costs_set_static",
    "pcbg_costs_set_occupancy", "pcbg_costs_set_history", "pcbg_costs_set_ground", "pcbg_costs_rebuild",
    "pcbg_costs_stamp", "pcbg_costs_add_history", "pcbg_costs_download", "pcbg_costs_download_history",
    "pcbg_costs_device_map", "pcbg_costs_time_rebuild",
]
GPU_H_SYMBOLS = [
    "_Z13gpu_availablev",                        # bool gpu_available()
    "_Z13gpu_configureim",                       # void gpu_configure(int, size_t)
    "_Z9gpu_solveRK8GpuQueryR6GpuOutb",          # int gpu_solve(const GpuQuery&, GpuOut&, bool)
    "_ZN6GpuOutD1Ev",                            # GpuOut::~GpuOut()
    "_ZN6GpuOut7reserveEm",                      # void GpuOut::reserve(size_t)
    "_ZNK6GpuOutclEl",                           # float GpuOut::operator()(int64_t) const
]


class TuneEntry(C.Structure):
    _fields_ = [("layers_lo", C.c_int32), ("layers_hi", C.c_int32), ("batch_class", C.c_int32), ("band", C.c_int32),
                ("blocks_per_sm", C.c_int32), ("ms", C.c_float), ("ms_untuned", C.c_float), ("searches", C.c_int32),
                ("rw", C.c_int32), ("rh", C.c_int32), ("nl", C.c_int32)]


class Query(C.Structure):
    """struct pcbg_query (GpuQuery of src/gpu.h:10-36 with flattened vectors)."""
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nl", C.c_int32),
        ("wi0", C.c_int32), ("wj0", C.c_int32), ("ww", C.c_int32), ("wh", C.c_int32),
        ("me", C.c_uint16),
        ("via_cost", C.c_float), ("step", C.c_float),
        ("dirf", (C.c_float * 8) * 8),
        ("lay", C.c_uint8 * 8),
        ("cst", C.c_void_p * 8),
        ("st", C.c_void_p * 8),
        ("vcst", C.c_void_p), ("vst", C.c_void_p), ("tbit", C.c_void_p),
        ("own_cf_idx", C.c_void_p), ("own_cf_val", C.c_void_p), ("n_own_cf", C.c_int64),
        ("own_vcf_idx", C.c_void_p), ("own_vcf_val", C.c_void_p), ("n_own_vcf", C.c_int64),
        ("start_idx", C.c_void_p), ("start_val", C.c_void_p), ("n_starts", C.c_int64),
        ("prior", C.c_void_p),
        ("pi0", C.c_int32), ("pj0", C.c_int32), ("pw", C.c_int32), ("ph", C.c_int32), ("pnl", C.c_int32),
        ("pcol", C.c_void_p), ("prow", C.c_void_p),
        ("play", C.c_int32 * 8),
        ("mlf", C.c_float * 256),
        ("mthr", C.c_uint8), ("corridor", C.c_uint8),
    ]


class Result(C.Structure):
    """struct pcbg_result (GpuOut of src/gpu.h:39-50 plus diagnostics)."""
    _fields_ = [
        ("rx0", C.c_int32), ("ry0", C.c_int32), ("rw", C.c_int32), ("rh", C.c_int32), ("nl", C.c_int32),
        ("ww", C.c_int32), ("wh", C.c_int32),
        ("best", C.c_int64),
        ("d", C.POINTER(C.c_float)), ("cap", C.c_size_t),
        ("rounds", C.c_int32), ("tries", C.c_int32), ("wide", C.c_int32),
        ("tile_visits", C.c_int64),
        ("ub", C.c_double),
    ]


class Search(C.Structure):
    """struct pcbg_search: one device-resident resolved search of a batch."""
    _fields_ = [
        ("rw", C.c_int32), ("rh", C.c_int32), ("nl", C.c_int32), ("pitch", C.c_int32), ("hpad", C.c_int32),
        ("fac", (C.c_float * 8) * 8),
        ("cf", C.c_void_p), ("flags", C.c_void_p), ("vcf", C.c_void_p),
        ("start_idx", C.c_void_p), ("start_d", C.c_void_p), ("n_starts", C.c_int32),
        ("out", C.c_void_p),
        ("path", C.c_void_p), ("path_cap", C.c_int32), ("path_len", C.c_void_p),
        ("best", C.c_int64), ("best_d", C.c_uint64),
        ("status", C.c_int32), ("rounds", C.c_int32),
    ]


class Net(C.Structure):
    """struct pcbg_net: a net of a speculative round (window and pins as board states)."""
    _fields_ = [("x0", C.c_int32), ("y0", C.c_int32), ("x1", C.c_int32), ("y1", C.c_int32),
                ("src", C.c_uint32), ("tgt", C.c_uint32)]


class SpecStats(C.Structure):
    """struct pcbg_spec_stats."""
    _fields_ = [("searches", C.c_int64), ("wasted", C.c_int64), ("batches", C.c_int64), ("commits", C.c_int64),
                ("conflicts", C.c_int64), ("search_ms", C.c_double), ("total_ms", C.c_double),
                ("relax_ms", C.c_double)]


SCHEDULER = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.c_int32,
                        C.POINTER(C.c_int32))
OBSERVER = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32)

_lib = None


def load() -> C.CDLL:
    """Load libpcbgpu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run python -m pcbroute_b200.build")
    lib = C.CDLL(LIB_PATH)
    lib.pcbg_available.restype = C.c_int
    lib.pcbg_configure.argtypes = [C.c_int, C.c_size_t]
    lib.pcbg_solve.argtypes = [C.POINTER(Query), C.POINTER(Result), C.c_int]
    lib.pcbg_solve.restype = C.c_int
    lib.pcbg_host_acquire.argtypes = [C.c_size_t, C.POINTER(C.c_size_t)]
    lib.pcbg_host_acquire.restype = C.POINTER(C.c_float)
    lib.pcbg_host_release.argtypes = [C.POINTER(C.c_float), C.c_size_t]
    lib.pcbg_last_error.restype = C.c_char_p
    lib.pcbg_solve_batch.argtypes = [C.POINTER(Search), C.c_int32, C.c_void_p]
    lib.pcbg_solve_batch.restype = C.c_int
    lib.pcbg_solve_noalloc.argtypes = [C.POINTER(Search), C.c_void_p]
    lib.pcbg_solve_noalloc.restype = C.c_int
    lib.pcbg_last_batch_tile_visits.restype = C.c_int64
    lib.pcbg_last_batch_layer_visits.restype = C.c_int64
    lib.pcbg_last_batch_rounds.restype = C.c_int32
    lib.pcbg_last_batch_kernel_ms.restype = C.c_float
    lib.pcbg_last_batch_launches.restype = C.c_int32
    lib.pcbg_last_batch_local_iters.restype = C.c_int64
    lib.pcbg_last_batch_deferred.restype = C.c_int64
    lib.pcbg_last_batch_dropped.restype = C.c_int64
    lib.pcbg_last_batch_settled.restype = C.c_int64
    lib.pcbg_mirror_class.argtypes = [C.c_int32] * 4 + [C.c_void_p] * 7
    lib.pcbg_mirror_class.restype = C.c_int
    lib.pcbg_mirror_spans.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int32]
    lib.pcbg_mirror_spans.restype = C.c_int
    lib.pcbg_mirror_history.argtypes = [C.c_int32]
    lib.pcbg_mirror_history.restype = C.c_int
    lib.pcbg_mirror_download.argtypes = [C.c_int32] + [C.c_void_p] * 4
    lib.pcbg_mirror_download.restype = C.c_int
    lib.pcbg_sched_add_log_host.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]
    lib.pcbg_sched_add_log_host.restype = C.c_int
    lib.pcbg_autotune.argtypes = [C.c_void_p, C.c_void_p, C.c_int32]
    lib.pcbg_autotune.restype = C.c_int32
    lib.pcbg_autotune_batch.argtypes = [C.POINTER(Search), C.c_int32, C.c_void_p, C.c_void_p]
    lib.pcbg_autotune_batch.restype = C.c_int32
    lib.pcbg_last_batch_blocks_per_sm.restype = C.c_int32
    lib.pcbg_last_batch_busy_frac.restype = C.c_float
    lib.pcbg_set_visit_order.argtypes = [C.c_int32]
    lib.pcbg_set_visit_order.restype = None
    lib.pcbg_visit_order.restype = C.c_int32
    lib.pcbg_set_round_band.argtypes = [C.c_int32]
    lib.pcbg_set_round_band.restype = None
    lib.pcbg_round_band.restype = C.c_int32
    lib.pcbg_set_max_rounds.argtypes = [C.c_int32]
    lib.pcbg_set_max_rounds.restype = None
    lib.pcbg_spec_create.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_float]
    lib.pcbg_spec_create.restype = C.c_void_p
    lib.pcbg_spec_destroy.argtypes = [C.c_void_p]
    lib.pcbg_spec_destroy.restype = None
    lib.pcbg_spec_set_scheduler.argtypes = [C.c_void_p, SCHEDULER, C.c_void_p]
    lib.pcbg_spec_set_scheduler.restype = None
    lib.pcbg_spec_set_observer.argtypes = [C.c_void_p, OBSERVER, C.c_void_p]
    lib.pcbg_spec_set_observer.restype = None
    lib.pcbg_spec_iterate.argtypes = [C.c_void_p, C.c_float, C.c_int32, C.c_int32, C.POINTER(SpecStats)]
    lib.pcbg_spec_iterate.restype = C.c_int
    lib.pcbg_spec_path.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32]
    lib.pcbg_spec_path.restype = C.c_int32
    lib.pcbg_spec_add_history.argtypes = [C.c_void_p, C.c_float]
    lib.pcbg_spec_add_history.restype = C.c_int32
    lib.pcbg_spec_window_reads.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32]
    lib.pcbg_spec_window_reads.restype = C.c_int32
    lib.pcbg_sched_create.argtypes = [C.c_uint64]
    lib.pcbg_sched_create.restype = C.c_void_p
    lib.pcbg_sched_destroy.argtypes = [C.c_void_p]
    lib.pcbg_sched_destroy.restype = None
    lib.pcbg_sched_attach.argtypes = [C.c_void_p, C.c_void_p, C.c_float]
    lib.pcbg_sched_attach.restype = None
    lib.pcbg_sched_attach_logger.argtypes = [C.c_void_p, C.c_void_p]
    lib.pcbg_sched_attach_logger.restype = None
    lib.pcbg_sched_label.argtypes = [C.c_void_p, C.c_void_p]
    lib.pcbg_sched_label.restype = C.c_int64
    lib.pcbg_sched_log_size.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
    lib.pcbg_sched_log_size.restype = C.c_int64
    lib.pcbg_sched_train.argtypes = [C.c_void_p, C.c_int32, C.c_float, C.c_int32, C.c_uint64, C.POINTER(C.c_float)]
    lib.pcbg_sched_train.restype = C.c_int
    lib.pcbg_sched_counts.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    lib.pcbg_sched_counts.restype = None
    lib.pcbg_sched_nparams.argtypes = [C.c_void_p]
    lib.pcbg_sched_nparams.restype = C.c_int64
    lib.pcbg_sched_get_params.argtypes = [C.c_void_p, C.c_void_p]
    lib.pcbg_sched_get_params.restype = C.c_int
    lib.pcbg_sched_set_params.argtypes = [C.c_void_p, C.c_void_p]
    lib.pcbg_sched_set_params.restype = C.c_int
    lib.pcbg_sched_forward_host.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
    lib.pcbg_sched_forward_host.restype = C.c_int
    lib.pcbg_sched_grad_host.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                         C.POINTER(C.c_float)]
    lib.pcbg_sched_grad_host.restype = C.c_int
    lib.pcbg_spec_net.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
    lib.pcbg_spec_net.restype = C.c_int
    lib.pcbg_spec_board.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.pcbg_spec_board.restype = None
    lib.pcbg_spec_costs.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.pcbg_spec_costs.restype = C.c_int
    lib.pcbg_batch_window.argtypes = [C.c_int32]
    lib.pcbg_batch_window.restype = None
    lib.pcbg_batcher_stats.argtypes = [C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    lib.pcbg_batcher_stats.restype = None
    lib.pcbg_synth_search_host.argtypes = [C.c_uint64, C.c_int32, C.c_int32, C.c_int32, C.c_float, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]
    lib.pcbg_synth_search_host.restype = C.c_int
    lib.pcbg_synth_search.argtypes = [C.c_uint64, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.pcbg_synth_search.restype = C.c_int
    V = C.c_void_p
    lib.pcbg_costs_create.argtypes = [C.c_int32] * 4
    lib.pcbg_costs_create.restype = V
    lib.pcbg_costs_destroy.argtypes = [V]
    lib.pcbg_costs_set_static.argtypes = [V, C.c_int32, V, V]
    lib.pcbg_costs_set_occupancy.argtypes = [V, C.c_int32, V, V]
    lib.pcbg_costs_set_history.argtypes = [V, V]
    lib.pcbg_costs_set_ground.argtypes = [V, C.c_int32, V]
    lib.pcbg_costs_rebuild.argtypes = [V, C.c_float, C.c_int32]
    lib.pcbg_costs_stamp.argtypes = [V, C.c_int32, C.c_int32, C.c_int32, V, C.c_int32, C.c_int32]
    lib.pcbg_costs_add_history.argtypes = [V, V, C.c_int32, C.c_float]
    lib.pcbg_costs_download.argtypes = [V, C.c_int32, V, V]
    lib.pcbg_costs_download_history.argtypes = [V, V]
    lib.pcbg_costs_device_map.argtypes = [V, C.c_int32, C.c_int32]
    lib.pcbg_costs_device_map.restype = V
    lib.pcbg_costs_time_rebuild.argtypes = [V, C.c_float, C.c_int32, C.c_int32]
    lib.pcbg_costs_time_rebuild.restype = C.c_float
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    """Dynamic symbols of the library that include/*.h declare and that are missing (empty: all present)."""
    lib = load()
    missing = []
    for s in PCBG_SYMBOLS + GPU_H_SYMBOLS:
        try:
            getattr(lib, s)
        except AttributeError:
            missing.append(s)
    return missing


def last_error() -> str:
    return load().pcbg_last_error().decode()
