"""ctypes view of the C ABI in include/gtpb200.h.

Loading fails loudly when the compiled library is missing: there is no
Python or CPU fallback for the engine.
"""
from __future__ import annotations

import ctypes as C
import os

from .build import LIB

GTP_OK = 0
GTP_GENERAL_ERROR = -1
GTP_EINVAL = -2
GTP_ENOMEM = -3
GTP_ECUDA = -4
GTP_ETIMEOUT = -5
GTP_EOVERFLOW = -6
GTP_ESTATE = -7

STATUS_NAMES = {
    0: "GTP_OK", -1: "GTP_GENERAL_ERROR", -2: "GTP_EINVAL", -3: "GTP_ENOMEM",
    -4: "GTP_ECUDA", -5: "GTP_ETIMEOUT", -6: "GTP_EOVERFLOW", -7: "GTP_ESTATE",
}

GTP_AXIS_NONE, GTP_AXIS_SLEW, GTP_AXIS_CAP = 0, 1, 2
GROUP_NAMES = ["Combinational", "Sequential", "Clock", "Macro", "Pad"]
GTP_N_GROUP = 5


class gtp_table(C.Structure):
    _fields_ = [("order", C.c_int32), ("axis1_var", C.c_int32), ("axis2_var", C.c_int32),
                ("n1", C.c_int32), ("n2", C.c_int32), ("axis1_off", C.c_int64),
                ("axis2_off", C.c_int64), ("value_off", C.c_int64), ("scale", C.c_float),
                ("reserved", C.c_int32)]


class gtp_when(C.Structure):
    _fields_ = [("cube_off", C.c_int32), ("n_cube", C.c_int32)]


class gtp_internal_power(C.Structure):
    _fields_ = [("pin", C.c_int32), ("related_pin", C.c_int32), ("when", gtp_when),
                ("rise_table", C.c_int32), ("fall_table", C.c_int32)]


class gtp_leakage_power(C.Structure):
    _fields_ = [("when", gtp_when), ("power", C.c_float), ("reserved", C.c_int32)]


class gtp_cell_type(C.Structure):
    _fields_ = [("n_pin", C.c_int32), ("n_in", C.c_int32), ("ipwr_off", C.c_int32),
                ("n_ipwr", C.c_int32), ("leak_off", C.c_int32), ("n_leak", C.c_int32),
                ("cell_leakage_power", C.c_float), ("has_cell_leakage_power", C.c_int32)]


_P = C.c_void_p


class gtp_design(C.Structure):
    _fields_ = [("timescale", C.c_double), ("clk_period", C.c_float), ("reserved0", C.c_int32),
                ("time_max", C.c_int64),
                ("n_cell", C.c_int32), ("n_pin", C.c_int32), ("n_net", C.c_int32),
                ("n_type", C.c_int32),
                ("cell_pin_off", _P), ("cell_type", _P), ("cell_group", _P), ("cell_arc_off", _P),
                ("pin_net", _P), ("pin_slew_rise", _P), ("pin_slew_fall", _P),
                ("pin_load_cap", _P), ("pin_voltage", _P), ("pin_default_state", _P),
                ("pin_is_clock", _P),
                ("arc_delay", _P), ("n_arc_delay", C.c_int64),
                ("types", _P), ("internal_powers", _P), ("leakage_powers", _P), ("tables", _P),
                ("lut_pool", _P), ("when_cubes", _P),
                ("n_internal_power", C.c_int32), ("n_leakage_power", C.c_int32),
                ("n_table", C.c_int32), ("n_when_cube", C.c_int32),
                ("lut_pool_len", C.c_int64)]


class gtp_events(C.Structure):
    _fields_ = [("n_event", C.c_int64), ("net_off", _P), ("time", _P), ("value_packed", _P),
                ("net_base", _P), ("t_lo", C.c_int64), ("t_hi", C.c_int64)]


class gtp_config(C.Structure):
    _fields_ = [("cuda_device_id", C.c_int32), ("cycles_per_tile", C.c_int32),
                ("n_thread_per_block", C.c_int32), ("gates_per_block", C.c_int32),
                ("max_n_pin_for_leakage_power", C.c_int32), ("collect_counts", C.c_int32),
                ("max_event_num", C.c_int64), ("sort_by_work", C.c_int32),
                ("clock_runs", C.c_int32), ("split_events", C.c_int32), ("separate_kernels", C.c_int32),
                ("warp_walk", C.c_int32), ("reserved32", C.c_int32), ("reserved", C.c_int64 * 1)]


class gtp_counts(C.Structure):
    _fields_ = [("cell_events", _P), ("cell_glitches", _P), ("cell_half_toggles", _P),
                ("cell_related", _P), ("cycle_events", _P), ("cycle_glitches", _P),
                ("dropped", C.c_int64)]


class gtp_bits_window(C.Structure):
    _fields_ = [("d_net_off", _P), ("d_time", _P), ("c_lo", C.c_int64), ("c_hi", C.c_int64)]


BITS_MAX_WINDOWS = 64


class gtp_proxy_config(C.Structure):
    _fields_ = [("cuda_device_id", C.c_int32), ("n_in", C.c_int32), ("n_hidden", C.c_int32),
                ("n_out", C.c_int32), ("batch", C.c_int32), ("lr", C.c_float),
                ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float),
                ("weight_decay", C.c_float), ("seed", C.c_uint64), ("use_graph", C.c_int32),
                ("reserved32", C.c_int32), ("reserved", C.c_int64 * 4)]


class gtp_batch_config(C.Structure):
    _fields_ = [("use_graph", C.c_int32), ("blocks_per_sm", C.c_int32), ("reserved", C.c_int64 * 4)]


# Every symbol the headers declare (include/gtpb200.h, include/gtpb200_proxy.h).
EXPORTED = sorted([
    "gtp_config_default", "gtp_create", "gtp_destroy", "gtp_last_error", "gtp_n_period",
    "gtp_ticks_per_cycle", "gtp_reset", "gtp_push_events", "gtp_push_events_device",
    "gtp_sync", "gtp_get_stream", "gtp_set_stream", "gtp_finalize", "gtp_fetch",
    "gtp_evaluate_noalloc", "gtp_pack_values",
    "gtp_set_cycle_groups", "gtp_n_cycle_groups", "gtp_fetch_cycle_groups", "gtp_clock_run_nets",
    "gtp_walk_items", "gtp_set_cell_range", "gtp_accumulator_bytes", "gtp_export_accumulators",
    "gtp_import_accumulators", "gtp_push_events_device_ranges", "gtp_write_cell_power",
    "gtp_vcd_create", "gtp_vcd_parse", "gtp_vcd_fetch", "gtp_vcd_stats", "gtp_vcd_last_error", "gtp_vcd_destroy", "gtp_write_per_cycle_waveform",
    "gtp_batch_config_default", "gtp_batch_create", "gtp_batch_destroy", "gtp_batch_last_error",
    "gtp_batch_push_device", "gtp_batch_sync", "gtp_batch_get_stream", "gtp_batch_stats",
    "gtp_proxy_config_default", "gtp_proxy_create", "gtp_proxy_destroy", "gtp_proxy_last_error",
    "gtp_proxy_get_stream", "gtp_proxy_set_stream", "gtp_proxy_n_param",
    "gtp_proxy_set_training_data", "gtp_proxy_get_norm", "gtp_proxy_train",
    "gtp_proxy_compute_grads", "gtp_proxy_adam_step", "gtp_proxy_get_params",
    "gtp_proxy_set_params", "gtp_proxy_get_grads", "gtp_proxy_predict", "gtp_toggle_bits", "gtp_toggle_bits_windows",
    "gtp_net_toggle_stats", "gtp_bf16_gemm", "gtp_bf16_gemm_checked",
])

_lib = None


def lib() -> C.CDLL:
    """Loads libgtpb200.so (building it first if nvcc is available and the
    library is missing or stale). Raises if it cannot be loaded."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        try:
            from .build import build_engine
            build_engine()
        except Exception as e:  # pragma: no cover - depends on toolchain
            raise RuntimeError(f"libgtpb200.so is missing and could not be built: {e}") from e
    L = C.CDLL(LIB)
    L.gtp_config_default.argtypes = [C.POINTER(gtp_config)]
    L.gtp_config_default.restype = None
    L.gtp_create.argtypes = [C.POINTER(gtp_design), C.POINTER(gtp_config), C.POINTER(C.c_void_p)]
    L.gtp_create.restype = C.c_int32
    L.gtp_destroy.argtypes = [C.c_void_p]
    L.gtp_destroy.restype = None
    L.gtp_last_error.argtypes = [C.c_void_p]
    L.gtp_last_error.restype = C.c_char_p
    L.gtp_n_period.argtypes = [C.c_void_p]
    L.gtp_n_period.restype = C.c_int64
    L.gtp_ticks_per_cycle.argtypes = [C.c_void_p]
    L.gtp_ticks_per_cycle.restype = C.c_int64
    L.gtp_reset.argtypes = [C.c_void_p]
    L.gtp_reset.restype = C.c_int32
    L.gtp_push_events.argtypes = [C.c_void_p, C.POINTER(gtp_events)]
    L.gtp_push_events.restype = C.c_int32
    L.gtp_push_events_device.argtypes = [C.c_void_p, C.POINTER(gtp_events)]
    L.gtp_push_events_device.restype = C.c_int32
    L.gtp_sync.argtypes = [C.c_void_p]
    L.gtp_sync.restype = C.c_int32
    L.gtp_get_stream.argtypes = [C.c_void_p]
    L.gtp_get_stream.restype = C.c_void_p
    L.gtp_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    L.gtp_set_stream.restype = C.c_int32
    L.gtp_finalize.argtypes = [C.c_void_p]
    L.gtp_finalize.restype = C.c_int32
    L.gtp_fetch.argtypes = [C.c_void_p, _P, _P, _P, _P, C.POINTER(gtp_counts)]
    L.gtp_fetch.restype = C.c_int32
    L.gtp_evaluate_noalloc.argtypes = [C.c_void_p, C.POINTER(gtp_events), _P, _P, _P]
    L.gtp_evaluate_noalloc.restype = C.c_int32
    L.gtp_pack_values.argtypes = [_P, C.c_int64, _P]
    L.gtp_pack_values.restype = None
    L.gtp_set_cycle_groups.argtypes = [C.c_void_p, _P, C.c_int32]
    L.gtp_set_cycle_groups.restype = C.c_int32
    L.gtp_n_cycle_groups.argtypes = [C.c_void_p]
    L.gtp_n_cycle_groups.restype = C.c_int32
    L.gtp_fetch_cycle_groups.argtypes = [C.c_void_p, _P]
    L.gtp_fetch_cycle_groups.restype = C.c_int32
    L.gtp_clock_run_nets.argtypes = [C.c_void_p, _P, _P]
    L.gtp_clock_run_nets.restype = C.c_int32
    L.gtp_walk_items.argtypes = [C.c_void_p, _P]
    L.gtp_walk_items.restype = C.c_int32
    L.gtp_set_cell_range.argtypes = [C.c_void_p, C.c_int32, C.c_int32]
    L.gtp_set_cell_range.restype = C.c_int32
    L.gtp_accumulator_bytes.argtypes = [C.c_void_p]
    L.gtp_accumulator_bytes.restype = C.c_int64
    L.gtp_export_accumulators.argtypes = [C.c_void_p, _P]
    L.gtp_export_accumulators.restype = C.c_int32
    L.gtp_import_accumulators.argtypes = [C.c_void_p, _P]
    L.gtp_import_accumulators.restype = C.c_int32
    L.gtp_push_events_device_ranges.argtypes = [C.c_void_p, C.POINTER(gtp_events), _P, C.c_int32]
    L.gtp_push_events_device_ranges.restype = C.c_int32
    L.gtp_vcd_create.argtypes = [C.c_char_p, _P, C.c_int32, _P, _P, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]
    L.gtp_vcd_create.restype = C.c_int32
    L.gtp_vcd_parse.argtypes = [C.c_void_p, C.c_char_p, C.c_int64, C.POINTER(gtp_events), C.POINTER(C.c_int64)]
    L.gtp_vcd_parse.restype = C.c_int32
    L.gtp_vcd_fetch.argtypes = [C.c_void_p, _P, _P, _P]
    L.gtp_vcd_fetch.restype = C.c_int32
    L.gtp_vcd_stats.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.gtp_vcd_stats.restype = C.c_int32
    L.gtp_vcd_last_error.argtypes = [C.c_void_p]
    L.gtp_vcd_last_error.restype = C.c_char_p
    L.gtp_vcd_destroy.argtypes = [C.c_void_p]
    L.gtp_vcd_destroy.restype = None
    L.gtp_write_cell_power.argtypes = [C.c_char_p, C.c_int32, _P, _P, _P, _P, C.c_char_p]
    L.gtp_write_cell_power.restype = C.c_int32
    L.gtp_write_per_cycle_waveform.argtypes = [C.c_char_p, C.c_int64, _P, C.c_char_p, C.c_char_p]
    L.gtp_write_per_cycle_waveform.restype = C.c_int32
    _bind_proxy(L)
    _lib = L
    return L


class GtpError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def check(status: int, ctx=None) -> None:
    if status != GTP_OK:
        msg = lib().gtp_last_error(ctx)
        raise GtpError(status, msg.decode() if msg else "")


def _bind_proxy(L: C.CDLL) -> None:
    i32, i64, f = C.c_int32, C.c_int64, C.c_float
    sigs = {
        "gtp_proxy_config_default": ([C.POINTER(gtp_proxy_config)], None),
        "gtp_proxy_create": ([C.POINTER(gtp_proxy_config), C.POINTER(C.c_void_p)], i32),
        "gtp_proxy_destroy": ([_P], None),
        "gtp_proxy_last_error": ([_P], C.c_char_p),
        "gtp_proxy_get_stream": ([_P], _P),
        "gtp_proxy_set_stream": ([_P, _P], i32),
        "gtp_proxy_n_param": ([_P], i64),
        "gtp_proxy_set_training_data": ([_P, _P, _P, i64], i32),
        "gtp_proxy_get_norm": ([_P, _P, _P], i32),
        "gtp_proxy_train": ([_P, i32, _P], i32),
        "gtp_proxy_compute_grads": ([_P, _P, C.POINTER(f)], i32),
        "gtp_proxy_adam_step": ([_P], i32),
        "gtp_proxy_get_params": ([_P, _P], i32),
        "gtp_proxy_set_params": ([_P, _P], i32),
        "gtp_proxy_get_grads": ([_P, _P], i32),
        "gtp_proxy_predict": ([_P, _P, i64, _P], i32),
        "gtp_toggle_bits": ([_P, _P, _P, i32, i64, i64, i64, _P, i64, _P], i32),
        "gtp_toggle_bits_windows": ([C.POINTER(gtp_bits_window), i32, _P, i32, i64, i64, _P, i64, _P], i32),
        "gtp_net_toggle_stats": ([_P, _P, i32, i64, i64, i64, _P, _P, _P, _P], i32),
        "gtp_bf16_gemm": ([_P, i64, _P, i64, i64, i64, i64, _P, i32, _P, i64, _P], i32),
        "gtp_bf16_gemm_checked": ([_P, i64, _P, i64, i64, i64, i64, _P, i32, _P, i64, i64, i32, _P, _P], i32),
    }
    for name, (args, res) in sigs.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
