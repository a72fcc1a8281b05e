"""ctypes binding of the C ABI (include/ballasim_b200.h) and its status-code -> exception mapping.

The library is built in place (ballasim_b200/build.py). It is the only compute path: if it is missing or no
B200 is visible, the calls raise; nothing falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libballasim_b200.so"

BS_OK, BS_EINVAL, BS_ELOGIC, BS_ENOMEM, BS_ECUDA, BS_EREFUSED, BS_EIO, BS_ECANCELLED = 0, 1, 2, 3, 4, 5, 6, 7


class FileInfo(C.Structure):
    """bs_file_info: an event file's size, SHA-256 and its events stream."""
    _fields_ = [("bytes", C.c_uint64), ("sha256", C.c_char * 65), ("count", C.c_int64), ("t_first", C.c_int64),
                ("t_last", C.c_int64)]


class ExportError(ValueError):
    """An export refused its input or options; the message names the reason (the reference's
    ballasim.export.errors.ExportError, raised for the writers' Refused)."""


class Cancelled(Exception):
    """A window stopped by its CancelToken (the reference's _engine.Cancelled, src/engine/cancel.h:28-30)."""


class MemoryBudgetError(MemoryError):
    """A window or call that does not fit the device memory (MemoryBudgetError of the reference)."""


class Params(C.Structure):
    _fields_ = [("photoreceptor", C.c_int32)] + \
               [(n, C.c_double) for n in ("theta_on", "theta_off", "sigma_theta_on", "sigma_theta_off",
                                          "theta_onoff_corr", "theta_floor")] + \
               [("reset_mode", C.c_int32), ("refractory_s", C.c_double), ("eps_ci", C.c_double),
                ("initial_phase", C.c_int32)] + \
               [(n, C.c_double) for n in ("leak_rate_hz", "leak_sigma_log10", "leak_ea_eV", "dark_current_fA",
                                          "dark_sigma_ln", "dark_ea_eV", "temperature_K", "reference_temperature_K",
                                          "illuminance_scale", "label_share_cut", "readout_quantum_s",
                                          "readout_delay_s", "clock_drift_ppm")] + \
               [("clock_offset_ns", C.c_int64), ("hot_fraction", C.c_double), ("noise_shot_rate_hz", C.c_double),
                ("noise_ba_median_hz", C.c_double), ("noise_ba_sigma_ln", C.c_double)] + \
               [(n, C.c_double) for n in ("k", "tau_o", "tau_sf", "eps_L")] + [("noise", C.c_int32)] + \
               [("sigma_o", C.c_double), ("noise_margin_z", C.c_double), ("noise_leaf_level", C.c_int32),
                ("noise_diffusion", C.c_int32), ("initial_state", C.c_int32), ("stationary_probe_pixels", C.c_int32),
                ("stationary_burnin_ns", C.c_int64), ("fingerprint", C.c_uint64)]


class EventColumns(C.Structure):
    _fields_ = [("pixel", C.c_void_p), ("x", C.c_void_p), ("y", C.c_void_p), ("p", C.c_void_p),
                ("t_cross_ns", C.c_void_p), ("t_reported_ns", C.c_void_p), ("label", C.c_void_p),
                ("flags", C.c_void_p), ("ds", C.c_void_p), ("dn", C.c_void_p), ("dl", C.c_void_p),
                ("l_first", C.c_void_p)]


class OutputColumns(C.Structure):
    _fields_ = [("t_reported_ns", C.c_void_p), ("t_cross_ns", C.c_void_p), ("x", C.c_void_p), ("y", C.c_void_p),
                ("flags", C.c_void_p), ("p", C.c_void_p), ("label", C.c_void_p)]


class DeviceRuns(C.Structure):
    _fields_ = [("pixel", C.c_void_p), ("row_start", C.c_void_p), ("row_count", C.c_void_p), ("n", C.c_size_t),
                ("t", C.c_void_p), ("irr", C.c_void_p), ("n_samples", C.c_size_t)]


class DeviceEvents(C.Structure):
    _fields_ = [("data", C.c_void_p), ("count", C.c_size_t)]


class SampleRequest(C.Structure):
    _fields_ = [("cam", C.c_uint16), ("flags", C.c_uint16), ("pixel", C.c_uint32), ("k_begin", C.c_uint32),
                ("k_count", C.c_uint32), ("t_off_ns", C.c_int32), ("pose_slot", C.c_uint32)]


RENDER_FN = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.POINTER(SampleRequest), C.c_size_t, C.POINTER(C.c_uint32),
                        C.POINTER(C.c_float), C.POINTER(C.c_uint64), C.c_uint32)


class WindowRules(C.Structure):
    _fields_ = [("tol", C.c_float), ("dark", C.c_float), ("midpoint", C.c_int32), ("refine_signature", C.c_int32),
                ("max_refine_levels", C.c_int32), ("min_dt_ns", C.c_int64), ("cam", C.c_uint16),
                ("subsamples", C.c_uint32), ("cancel", C.c_void_p)]


class Field(C.Structure):
    _fields_ = [("kind", C.c_int32), ("width", C.c_uint32), ("height", C.c_uint32), ("base", C.c_float),
                ("amp", C.c_float), ("nx", C.c_float), ("ny", C.c_float), ("c", C.c_float), ("speed", C.c_float),
                ("width_px", C.c_float), ("n_blobs", C.c_int32), ("blobs", C.c_void_p)]


class SampleRules(C.Structure):
    _fields_ = [("tol", C.c_float), ("dark", C.c_float), ("midpoint", C.c_int32), ("refine_signature", C.c_int32),
                ("max_refine_levels", C.c_int32), ("min_dt_ns", C.c_int64), ("l_min", C.c_int32),
                ("l_max", C.c_int32)]


# (name, restype, argtypes); every function returns bs_status unless stated.
_P = C.c_void_p
_SIGS = {
    "bs_last_error": (C.c_char_p, []),
    "bs_version": (C.c_char_p, []),
    "bs_cuda_available": (C.c_int32, []),
    "bs_model_create": (C.c_int32, [C.POINTER(Params), C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32, C.c_int32,
                                    C.POINTER(_P)]),
    "bs_model_destroy": (C.c_int32, [_P]),
    "bs_model_init": (C.c_int32, [_P, C.c_int64, _P]),
    "bs_model_init_device": (C.c_int32, [_P, C.c_int64, _P, _P]),
    "bs_model_advance_runs": (C.c_int32, [_P, _P, C.c_size_t, _P, _P, C.c_size_t, _P, _P, C.c_int64,
                                          C.POINTER(C.c_size_t)]),
    "bs_model_advance_device": (C.c_int32, [_P, C.POINTER(DeviceRuns), C.c_int64, _P, C.POINTER(DeviceEvents)]),
    "bs_model_download_events": (C.c_int32, [_P, C.POINTER(DeviceEvents), C.POINTER(EventColumns)]),
    "bs_model_event_count": (C.c_int32, [_P, C.POINTER(C.c_size_t)]),
    "bs_model_take_events": (C.c_int32, [_P, C.POINTER(EventColumns)]),
    "bs_model_maps": (C.c_int32, [_P, _P, _P, _P, _P, _P]),
    "bs_model_stats": (C.c_int32, [_P, _P]),
    "bs_model_noise_maps": (C.c_int32, [_P, _P, _P]),
    "bs_model_output_prepare": (C.c_int32, [_P, C.POINTER(C.c_size_t)]),
    "bs_model_output_take": (C.c_int32, [_P, C.POINTER(OutputColumns)]),
    "bs_model_output_held": (C.c_int32, [_P, C.POINTER(C.c_size_t)]),
    "bs_model_reset_stats": (C.c_int32, [_P]),
    "bs_model_info": (C.c_int32, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_float), C.POINTER(C.c_int32)]),
    "bs_model_set_photometry": (C.c_int32, [_P, C.c_double, _P, C.c_size_t]),
    "bs_raw_writer_create": (C.c_int32, [C.c_char_p, C.c_char_p, C.c_int32, C.c_int32, C.c_int64, C.c_int64,
                                         C.c_char_p, C.c_int32, C.c_int32, C.c_char_p, C.POINTER(C.c_void_p)]),
    "bs_dat_writer_create": (C.c_int32, [C.c_char_p, C.c_int32, C.c_int32, C.c_int64, C.c_int64, C.c_int32,
                                         C.c_int32, C.c_char_p, C.POINTER(C.c_void_p)]),
    "bs_event_writer_append": (C.c_int32, [_P, _P, _P, _P, _P, C.c_size_t]),
    "bs_event_writer_append_device": (C.c_int32, [_P, _P, _P, _P, _P, C.c_size_t, _P]),
    "bs_event_writer_close": (C.c_int32, [_P, _P]),
    "bs_event_writer_stats": (C.c_int32, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_double),
                                          C.POINTER(C.c_uint64), _P]),
    "bs_event_writer_destroy": (C.c_int32, [_P]),
    "bs_sha256_hex": (C.c_int32, [_P, C.c_size_t, C.c_char_p]),
    "bs_model_gain_map": (C.c_int32, [_P, _P]),
    "bs_model_state_bytes": (C.c_int32, [_P, C.POINTER(C.c_size_t)]),
    "bs_model_save_state": (C.c_int32, [_P, _P, C.c_size_t]),
    "bs_model_load_state": (C.c_int32, [_P, _P, C.c_size_t]),
    "bs_model_set_block": (C.c_int32, [_P, C.c_int32]),
    "bs_model_set_long_run": (C.c_int32, [_P, C.c_int32]),
    "bs_model_take_timing": (C.c_int32, [_P, _P]),
    "bs_sampler_create": (C.c_int32, [C.POINTER(Field), C.POINTER(_P)]),
    "bs_sampler_destroy": (C.c_int32, [_P]),
    "bs_sample_window": (C.c_int32, [_P, C.c_int64, _P, _P, C.c_size_t, _P, _P, C.POINTER(SampleRules),
                                     C.POINTER(C.c_size_t)]),
    "bs_sampler_download": (C.c_int32, [_P, _P, _P, _P]),
    "bs_sample_window_static": (C.c_int32, [C.POINTER(Field), C.c_int64, _P, _P, C.c_size_t, _P, _P,
                                            C.POINTER(SampleRules), _P, _P, _P, C.c_size_t, _P, _P, _P,
                                            C.POINTER(C.c_size_t)]),
    "bs_sampler_device_runs": (C.c_int32, [_P, C.POINTER(DeviceRuns)]),
    "bs_window_create": (C.c_int32, [C.c_int32, _P, _P, C.POINTER(_P)]),
    "bs_window_destroy": (C.c_int32, [_P]),
    "bs_window_run": (C.c_int32, [_P, C.c_int64, _P, _P, C.c_size_t, _P, _P, C.POINTER(WindowRules), RENDER_FN, _P,
                                  C.POINTER(C.c_size_t)]),
    "bs_window_runs": (C.c_int32, [_P, _P, _P, _P]),
    "bs_window_stats": (C.c_int32, [_P, _P, _P, C.c_size_t, C.POINTER(C.c_size_t)]),
    "bs_sample_window_device": (C.c_int32, [_P, C.c_int64, _P, _P, C.c_size_t, _P, _P, _P, _P,
                                            C.POINTER(SampleRules), _P, C.POINTER(C.c_size_t)]),
    "bs_field_levels_device": (C.c_int32, [_P, C.c_int64, C.c_int32, C.c_int32, _P, _P]),
    "bs_field_frame_device": (C.c_int32, [_P, C.c_int64, _P, _P]),
    "bs_field_levels": (C.c_int32, [_P, C.c_int64, C.c_int32, C.c_int32, _P]),
    "bs_field_frame": (C.c_int32, [_P, C.c_int64, _P]),
    "bs_midpoint_eta": (C.c_int32, [C.c_float, C.c_float, C.c_int32, _P, _P, _P, _P, _P, C.c_size_t, _P, _P]),
    "bs_level_cap": (C.c_int32, [_P, C.c_size_t, C.c_int64, C.c_int32, C.POINTER(C.c_int32)]),
    "bs_engine_create": (C.c_int32, [_P, C.POINTER(Field), C.c_int32, C.POINTER(SampleRules), C.POINTER(_P)]),
    "bs_engine_destroy": (C.c_int32, [_P]),
    "bs_engine_start": (C.c_int32, [_P, C.c_int64, _P]),
    "bs_engine_start_frames": (C.c_int32, [_P, C.c_int64, _P, _P]),
    "bs_engine_run": (C.c_int32, [_P, C.c_int32, _P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "bs_engine_take_events": (C.c_int32, [_P, _P]),
    "bs_engine_set_launch": (C.c_int32, [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "bs_engine_get_launch": (C.c_int32, [_P, _P]),
    "bs_engine_set_graph": (C.c_int32, [_P, C.c_int32]),
    "bs_engine_autotune": (C.c_int32, [_P, C.c_int32, _P, _P, C.c_size_t, C.POINTER(C.c_size_t)]),
    "bs_engine_last_ms": (C.c_int32, [_P, C.POINTER(C.c_double)]),
    "bs_mlp_create": (C.c_int32, [C.c_uint64, C.POINTER(_P)]),
    "bs_mlp_destroy": (C.c_int32, [_P]),
    "bs_mlp_get_params": (C.c_int32, [_P, _P]),
    "bs_mlp_set_params": (C.c_int32, [_P, _P]),
    "bs_mlp_steps": (C.c_int32, [_P, C.POINTER(C.c_int64)]),
    "bs_mlp_forward": (C.c_int32, [_P, _P, C.c_size_t, _P, _P]),
    "bs_mlp_gradient": (C.c_int32, [_P, _P, _P, C.c_size_t, _P, C.POINTER(C.c_double), _P]),
    "bs_mlp_train": (C.c_int32, [_P, _P, _P, C.c_size_t, C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_uint64, _P,
                                 _P]),
    "bs_trace_pairs": (C.c_int32, [C.POINTER(Field), C.POINTER(SampleRules), C.c_int64, C.c_int32, C.c_uint32,
                                   C.c_float, C.c_uint64, _P, _P, _P, C.c_size_t, C.POINTER(C.c_size_t),
                                   C.POINTER(C.c_size_t), _P]),
    "bs_engine_set_proposal": (C.c_int32, [_P, _P, C.c_float]),
    "bs_engine_set_record": (C.c_int32, [_P, C.c_size_t]),
    "bs_engine_take_record": (C.c_int32, [_P, C.c_int32, C.c_size_t, _P, _P, _P, C.POINTER(C.c_size_t)]),
}

_lib = None


def lib():
    """The loaded library; raises ImportError (no silent fallback) when it is not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"ballasim_b200: the CUDA library is not built ({LIB_PATH}); run "
                              "`python -m ballasim_b200.build` (nvcc, sm_100a)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return list(_SIGS)


def check(status: int) -> None:
    """Raises the reference's exception type for a failed call."""
    if status == BS_OK:
        return
    msg = lib().bs_last_error().decode(errors="replace")
    if status == BS_EINVAL:
        raise ValueError(msg)
    if status == BS_ENOMEM:
        raise MemoryBudgetError(msg)
    if status == BS_EREFUSED:
        raise ExportError(msg)
    if status == BS_EIO:
        raise OSError(msg)
    if status == BS_ECANCELLED:
        raise Cancelled(msg)
    raise RuntimeError(msg)


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


def cuda_available() -> bool:
    """True if the library is built and a B200 (compute capability 10.x) is visible."""
    try:
        return bool(lib().bs_cuda_available())
    except ImportError:
        return False
