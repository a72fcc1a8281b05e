"""The sensor model with the interface of ``ballasim._sensor`` (src/sensor/sensor_module.cpp:446-656).

``SensorModel(params, width, height, seed, light_groups, camera, num_threads=0, precision=None, overrides=None,
device='cuda', roi=None)`` runs BallaSim's pixel model (the instantaneous response, or the cascade photoreceptor
with or without its noise lattice) on the B200 through the C ABI; its events
are the reference's CPU fp32 path's, bit for bit (the reference asserts the same of its own GPU path,
src/sensor/sensor_cuda.h:1-3). This build runs device 'cuda', precision 'fp32', one constant light group and no
region of interest; other values raise ValueError. Errors map as the reference's: ValueError for refused input
(the model unchanged), RuntimeError for a call before init.
"""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np

from . import _lib
from .params import SensorParams, fingerprint, preset_names, resolve  # noqa: F401  (re-exported: the reference's module API)

cuda_available = _lib.cuda_available

EVENT_COLUMNS = (("x", np.uint16), ("y", np.uint16), ("p", np.uint8), ("t_cross_ns", np.int64),
                 ("t_reported_ns", np.int64), ("label", np.uint8), ("flags", np.uint16), ("ds", np.float32),
                 ("dn", np.float32), ("dl", np.float32), ("l_first", np.float32))


def params_struct(p: SensorParams) -> _lib.Params:
    v = p.as_dict()
    s = _lib.Params()
    s.photoreceptor = 1 if v["photoreceptor"] == "instantaneous" else 0
    for name in ("theta_on", "theta_off", "sigma_theta_on", "sigma_theta_off", "theta_onoff_corr", "theta_floor",
                 "refractory_s", "eps_ci", "leak_rate_hz", "leak_sigma_log10", "leak_ea_eV", "dark_current_fA",
                 "dark_sigma_ln", "dark_ea_eV", "temperature_K", "reference_temperature_K", "illuminance_scale",
                 "label_share_cut", "readout_quantum_s", "readout_delay_s", "clock_drift_ppm", "hot_fraction",
                 "noise_shot_rate_hz", "noise_ba_median_hz", "noise_ba_sigma_ln", "k", "tau_o", "tau_sf", "eps_L",
                 "sigma_o", "noise_margin_z"):
        setattr(s, name, float(v[name]))
    s.noise = 1 if v["noise"] else 0
    s.noise_leaf_level = int(v["noise_leaf_level"])
    s.noise_diffusion = 1 if v["noise_diffusion"] == "transient" else 0
    s.initial_state = 1 if v["initial_state"] == "stationary" else 0
    s.stationary_probe_pixels = int(v["stationary_probe_pixels"])
    s.stationary_burnin_ns = int(v["stationary_burnin_ns"])
    s.reset_mode = 1 if v["reset_mode"] == "ideal" else 0
    s.initial_phase = {"uniform": 0, "symmetric": 1, "zero": 2}[v["initial_phase"]]
    s.clock_offset_ns = int(v["clock_offset_ns"])
    s.fingerprint = fingerprint(p)
    return s


def _check_light_groups(light_groups) -> int:
    groups = list(light_groups)
    if not groups:
        raise ValueError("SensorModel: need 1 to 8 light groups")
    for g in groups:
        d = g.get("waveform", g) if isinstance(g, dict) else g
        kind = d.get("type", "") if isinstance(d, dict) else ""
        if kind not in ("constant", "fourier", "pulse"):
            raise ValueError("light group: waveform type must be 'constant', 'fourier' or 'pulse'")
        if kind != "constant":
            raise ValueError("SensorModel: this build runs constant light groups only")
    if len(groups) != 1:
        raise ValueError("SensorModel: this build runs one light group")
    return 1


def new_columns(n: int) -> dict:
    """Fresh host columns for n events; every element is written by the library (so not zero-filled first)."""
    return {name: np.empty(n, dt) for name, dt in EVENT_COLUMNS}


def column_struct(cols: dict, with_pixel: np.ndarray | None = None) -> _lib.EventColumns:
    s = _lib.EventColumns()
    for name, _ in EVENT_COLUMNS:
        setattr(s, name, cols[name].ctypes.data if len(cols[name]) else None)
    s.pixel = with_pixel.ctypes.data if with_pixel is not None and len(with_pixel) else None
    return s


class SensorModel:
    """One camera's sensor on the B200 (the reference's ballasim._sensor.SensorModel)."""

    def __init__(self, params, width: int, height: int, seed: int, light_groups, camera: int, num_threads: int = 0,
                 precision=None, overrides=None, device: str = "cuda", roi=None):
        if device not in ("cpu", "cuda"):
            raise ValueError("device must be 'cpu' or 'cuda'")
        if device != "cuda":
            raise ValueError("SensorModel: this build has no CPU path; use device='cuda'")
        if precision not in (None, "fp32", "fp64"):
            raise ValueError("precision must be 'fp64' or 'fp32'")
        if precision == "fp64":
            raise ValueError("SensorModel: the CUDA device runs fp32 only")
        if roi is not None:
            raise ValueError("SensorModel: this build has no region-of-interest models")
        self._groups = _check_light_groups(light_groups)
        self._params = resolve(params, overrides)
        if self._params.photoreceptor == "cascade" and self._params.noise_on():
            raise ValueError("SensorModel: shot and background-activity noise run with the instantaneous response only")
        self._width, self._height, self._seed, self._camera = int(width), int(height), int(seed), int(camera)
        self._num_threads = int(num_threads)
        self._lock = threading.Lock()
        L = _lib.lib()
        h = C.c_void_p()
        self._ps = params_struct(self._params)
        _lib.check(L.bs_model_create(C.byref(self._ps), self._width, self._height, self._seed, self._camera,
                                     self._groups, C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        self._h = None
        if h:
            try:
                _lib.lib().bs_model_destroy(h)
            except Exception:  # interpreter shutdown: the library (and the process) is going away
                pass

    @property
    def handle(self):
        return self._h

    # ---- properties ----
    width = property(lambda self: self._width)
    height = property(lambda self: self._height)
    groups = property(lambda self: self._groups)
    params = property(lambda self: self._params.copy())
    num_threads = property(lambda self: self._num_threads)
    precision = property(lambda self: "fp32")
    device = property(lambda self: "cuda")
    roi = property(lambda self: None)

    def _info(self):
        t, irr_max, init = C.c_int64(), C.c_float(), C.c_int32()
        _lib.check(_lib.lib().bs_model_info(self._h, C.byref(t), C.byref(irr_max), C.byref(init)))
        return t.value, irr_max.value, bool(init.value)

    @property
    def time_ns(self) -> int:
        return self._info()[0]

    @property
    def irr_max(self) -> float:
        return self._info()[1]

    @property
    def initialized(self) -> bool:
        return self._info()[2]

    # ---- calls ----
    def init(self, t0_ns: int, irradiance0) -> None:
        a = np.ascontiguousarray(irradiance0, np.float32)
        n = self._width * self._height
        if a.ndim != 2 or a.shape != (n, self._groups):
            raise ValueError("init: irradiance0 must have shape (height * width, groups)")
        with self._lock:
            _lib.check(_lib.lib().bs_model_init(self._h, int(t0_ns), a.ctypes.data))

    def advance(self, pixel_ids, t_ns, irradiance, t_end_ns: int, counts=None, offsets=None) -> dict:
        """Advance to t_end_ns (sensor_module.cpp:302-351): rectangular runs t_ns (n, m), irradiance (n, m, groups)
        with optional counts, or ragged runs t_ns (S,), irradiance (S, groups) and offsets (n + 1,). Returns the
        event columns sorted by (t_cross_ns, pixel)."""
        if not isinstance(pixel_ids, np.ndarray) or pixel_ids.dtype != np.uint32 or pixel_ids.ndim != 1:
            raise TypeError("advance: pixel_ids must be a uint32 array (n,)")
        ids = np.ascontiguousarray(pixel_ids)
        n, G = len(ids), self._groups

        def exact(a, dtype, ndim, what):
            if not isinstance(a, np.ndarray) or a.dtype != dtype or a.ndim != ndim:
                raise TypeError(f"advance: {what} has the wrong dtype or number of dimensions")
            return np.ascontiguousarray(a)

        if offsets is None:
            t = exact(t_ns, np.int64, 2, "t_ns (int64, n x m)")
            irr = np.ascontiguousarray(irradiance, np.float32)
            if irr.ndim != 3:
                raise TypeError("advance: irradiance (n x m x groups) has the wrong dtype or number of dimensions")
            m = t.shape[1]
            if t.shape[0] != n or irr.shape != (n, m, G):
                raise ValueError("advance: t_ns must be (n, m) and irradiance (n, m, groups) for n pixel ids")
            if counts is not None:
                cnt = exact(counts, np.int32, 1, "counts (int32)")
                if len(cnt) != n:
                    raise ValueError("advance: counts must have one entry per pixel id")
                if np.any(cnt < 0) or np.any(cnt > m):
                    raise ValueError("SensorModel.advance: count out of range")
            else:
                cnt = np.full(n, m, np.int32)
            start = np.arange(n, dtype=np.int64) * m
            t_flat, irr_flat = t.reshape(-1), irr.reshape(-1)
        else:
            if counts is not None:
                raise ValueError("advance: pass either counts or offsets, not both")
            t_flat = exact(t_ns, np.int64, 1, "t_ns (int64, S)")
            irr_flat = np.ascontiguousarray(irradiance, np.float32)
            if irr_flat.ndim != 2:
                raise TypeError("advance: irradiance (S x groups) has the wrong dtype or number of dimensions")
            off = exact(offsets, np.int64, 1, "offsets (int64, n + 1)")
            S = len(t_flat)
            if irr_flat.shape != (S, G):
                raise ValueError("advance: with offsets, t_ns must be (S,) and irradiance (S, groups)")
            if len(off) != n + 1 or off[0] != 0 or off[n] != S:
                raise ValueError("advance: offsets must be (n + 1,) from 0 to the number of samples")
            d = np.diff(off)
            if np.any(d < 0) or np.any(d > np.iinfo(np.int32).max):
                raise ValueError("advance: offsets must be non-decreasing")
            start, cnt = off[:-1].copy(), d.astype(np.int32)
            irr_flat = irr_flat.reshape(-1)
        return self.advance_runs(ids, t_flat, irr_flat, t_end_ns, start, cnt)

    def advance_runs(self, pixel_ids, t_ns, irradiance, t_end_ns, row_start, row_count) -> dict:
        """SensorModel::advance_runs: ragged runs in one sample array."""
        ids = np.ascontiguousarray(pixel_ids, np.uint32)
        t = np.ascontiguousarray(t_ns, np.int64).reshape(-1)
        irr = np.ascontiguousarray(irradiance, np.float32).reshape(-1)
        rs = np.ascontiguousarray(row_start, np.int64)
        rc = np.ascontiguousarray(row_count, np.int32)
        ne = C.c_size_t()
        with self._lock:
            _lib.check(_lib.lib().bs_model_advance_runs(self._h, _lib.ptr(ids), len(ids), _lib.ptr(t), _lib.ptr(irr),
                                                        len(t), _lib.ptr(rs), _lib.ptr(rc), int(t_end_ns),
                                                        C.byref(ne)))
            return self._take(ne.value)

    def init_device(self, t0_ns: int, irradiance0_ptr: int, stream: int | None = None) -> None:
        """init from a device array of height * width floats (the frame a device renderer wrote), on stream."""
        with self._lock:
            _lib.check(_lib.lib().bs_model_init_device(self._h, int(t0_ns), irradiance0_ptr, stream))

    def advance_device(self, runs: _lib.DeviceRuns, t_end_ns: int, stream: int | None = None) -> _lib.DeviceEvents:
        """SensorModel::advance_device (src/sensor/sensor_model.h:157-167): runs in device memory (DeviceRuns), queued
        on stream; one synchronization reads the call's counters. The events stay on the device (RawEvent records,
        unordered), valid until the model advances again."""
        ev = _lib.DeviceEvents()
        with self._lock:
            _lib.check(_lib.lib().bs_model_advance_device(self._h, C.byref(runs), int(t_end_ns), stream, C.byref(ev)))
        return ev

    def download_events(self, events: _lib.DeviceEvents, with_pixel: bool = False) -> dict:
        """SensorModel::download_events (sensor_model.h:167): a call's device events as host columns sorted by
        (t_cross_ns, pixel)."""
        n = int(events.count)
        cols = new_columns(n)
        px = np.zeros(n, np.uint32) if with_pixel else None
        s = column_struct(cols, px)
        with self._lock:
            _lib.check(_lib.lib().bs_model_download_events(self._h, C.byref(events), C.byref(s)))
        if with_pixel:
            cols["pixel"] = px
        return cols

    def _take(self, n: int, with_pixel: bool = False) -> dict:
        cols = new_columns(n)
        px = np.zeros(n, np.uint32) if with_pixel else None
        s = column_struct(cols, px)
        _lib.check(_lib.lib().bs_model_take_events(self._h, C.byref(s)))
        if with_pixel:
            cols["pixel"] = px
        return cols

    def take_events(self, with_pixel: bool = False) -> dict:
        """The events the model keeps (an engine run's), sorted; the list is cleared."""
        n = C.c_size_t()
        with self._lock:
            _lib.check(_lib.lib().bs_model_event_count(self._h, C.byref(n)))
            return self._take(n.value, with_pixel)

    def take_output(self) -> dict:
        """The engine's output stage (Camera::output, src/engine/engine_impl.h:1761-1847, without crop and ground
        truth): the events not taken with take_events, with those held from earlier calls, in output order
        (t_reported, x, y, t_cross); the ones reported before the model time on the sensor clock are returned
        (columns t_reported_ns, t_cross_ns, x, y, p, label (S1 codes: 0 signal, 2 noise, 3 leak, 4 hot), flags),
        the rest stay held for the next call."""
        n = C.c_size_t()
        with self._lock:
            _lib.check(_lib.lib().bs_model_output_prepare(self._h, C.byref(n)))
            k = n.value
            cols = {"t_reported_ns": np.zeros(k, np.int64), "t_cross_ns": np.zeros(k, np.int64),
                    "x": np.zeros(k, np.uint16), "y": np.zeros(k, np.uint16), "flags": np.zeros(k, np.uint16),
                    "p": np.zeros(k, np.uint8), "label": np.zeros(k, np.uint8)}
            s = _lib.OutputColumns(*(cols[f].ctypes.data for f, _ in _lib.OutputColumns._fields_))
            _lib.check(_lib.lib().bs_model_output_take(self._h, C.byref(s)))
            return cols

    @property
    def output_held(self) -> int:
        """Events the output stage holds for a later call."""
        n = C.c_size_t()
        _lib.check(_lib.lib().bs_model_output_held(self._h, C.byref(n)))
        return n.value

    def sensor_maps(self) -> dict:
        n = self._width * self._height
        a = {k: np.zeros(n) for k in ("theta_on", "theta_off", "leak", "dark_current_fA", "phi0")}
        _lib.check(_lib.lib().bs_model_maps(self._h, *(a[k].ctypes.data for k in a)))
        return {k: v.reshape(self._height, self._width) for k, v in a.items()}

    def set_photometry(self, illuminance_scale: float, gain=None) -> None:
        """Photometry (sensor_module.cpp:477-486): the photocurrent scale (fA per renderer unit on axis) and the
        per-pixel gain map (height * width gains in pixel order, any shape; None: 1 everywhere). irr_max follows the
        largest gain at once; the states take the photometry at the next init: call it before init."""
        g = None
        if gain is not None:
            try:
                g = np.ascontiguousarray(gain, np.float32).reshape(-1)
            except (TypeError, ValueError):
                raise TypeError("set_photometry: gain must be a float array") from None
            if not np.all(np.isfinite(g) & (g > 0)):
                raise ValueError("set_photometry: gains must be finite and > 0")
        p = self._params.copy()
        p.illuminance_scale = float(illuminance_scale)
        p.validate()
        with self._lock:
            _lib.check(_lib.lib().bs_model_set_photometry(self._h, float(illuminance_scale),
                                                          g.ctypes.data if g is not None else None,
                                                          g.size if g is not None else 0))
            self._params = p

    def gain_map(self) -> np.ndarray:
        """The static pixel gains (height, width), float32 (set_photometry; 1 everywhere by default)."""
        g = np.zeros(self._width * self._height, np.float32)
        _lib.check(_lib.lib().bs_model_gain_map(self._h, g.ctypes.data))
        return g.reshape(self._height, self._width)

    def noise_maps(self) -> dict:
        """This build's noise maps (height, width): the background-activity rate and the shot-noise dominating
        rate r sqrt(100 fA / I_dk) of each pixel (Hz)."""
        n = self._width * self._height
        ba, shot = np.zeros(n), np.zeros(n)
        _lib.check(_lib.lib().bs_model_noise_maps(self._h, ba.ctypes.data, shot.ctypes.data))
        return {"ba_rate_hz": ba.reshape(self._height, self._width),
                "shot_max_hz": shot.reshape(self._height, self._width)}

    def stats(self) -> dict:
        out = np.zeros(9, np.uint64)
        _lib.check(_lib.lib().bs_model_stats(self._h, out.ctypes.data))
        return {"substeps": int(out[0]), "pieces": int(out[0]), "leaf_intervals": int(out[1]),
                "input_clamps": int(out[2]), "pixel_samples": int(out[3]), "noise_candidates": int(out[4]),
                "gpu_launches": int(out[5]), "gpu_reruns": int(out[6]), "gpu_launch_ms_total": out[7] / 1000.0,
                "gpu_launch_ms_max": out[8] / 1000.0}

    def reset_stats(self) -> None:
        _lib.check(_lib.lib().bs_model_reset_stats(self._h))

    def state_bytes(self) -> int:
        n = C.c_size_t()
        _lib.check(_lib.lib().bs_model_state_bytes(self._h, C.byref(n)))
        return n.value

    def save_state(self) -> bytes:
        buf = np.zeros(self.state_bytes(), np.uint8)
        with self._lock:
            _lib.check(_lib.lib().bs_model_save_state(self._h, buf.ctypes.data, len(buf)))
        return buf.tobytes()

    def load_state(self, state: bytes) -> None:
        b = np.frombuffer(state, np.uint8)
        with self._lock:
            _lib.check(_lib.lib().bs_model_load_state(self._h, b.ctypes.data, len(b)))

    def take_timing(self) -> dict:
        """The last download of device events, in parts (ms): the sort and column split on the device, the copy to
        pinned host memory, the copies into the returned arrays, and the whole call."""
        out = np.zeros(4)
        _lib.check(_lib.lib().bs_model_take_timing(self._h, out.ctypes.data))
        return dict(zip(("sort_split_ms", "copy_out_ms", "host_copy_ms", "total_ms"), out.tolist()))

    def set_long_run(self, samples: int) -> None:
        """Threads per pixel of the row-major kernel: runs longer than `samples` are walked by a whole warp (32 lanes,
        32 samples at a time), the others one per lane (0: the default, 32; -1: every run by one lane)."""
        _lib.check(_lib.lib().bs_model_set_long_run(self._h, int(samples)))

    def set_block(self, threads: int) -> None:
        """Launch policy of the pixel model on runs: 0, the row-major kernel split in two launches (the default for
        the instantaneous response: runs stopped at a segment that is not clean are finished one thread each by a
        second kernel); 1, the row-major kernel in one launch; 32, 64, 96 or 128, one thread per pixel with that many
        threads per block."""
        _lib.check(_lib.lib().bs_model_set_block(self._h, int(threads)))
