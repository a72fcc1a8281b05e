"""The fused window engine: every window of one or more sensors sampled and sensed on the device, each pixel's
sampler and pixel model on the same thread with the state in registers (the reference's per-window
``Camera::sample_and_sense``, src/engine/engine_impl.h:1253-1357: WindowEngine runs, then
SensorModel::advance_device, without the runs ever leaving the chip).

    eng = Engine([(model, field), ...], tol=0.01, dark=0.01, min_dt_ns=8192, max_refine_levels=10)
    eng.start(0)                       # renders every field at t0 and initializes each model from it
    samples, events = eng.run(windows) # whole windows from the model time; events kept per model
    cols = model.take_events()         # sorted (t_cross, pixel), as SensorModel.advance returns them

The events are bit-identical to running, per window, ``sample_window`` (levels by the field's rule) and then
``SensorModel.advance`` on its runs.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .fields import Field
from .sampling import field_struct
from .sensor import SensorModel


class Engine:
    def __init__(self, sensors, *, tol: float = 0.01, dark: float = 0.01, min_dt_ns: int = 8192,
                 max_refine_levels: int = 10, l_min: int = 1, l_max: int = 10, refine_signature: bool = True):
        self.sensors = [(m, f) for m, f in sensors]
        if not self.sensors:
            raise ValueError("engine: at least one sensor")
        for m, f in self.sensors:
            if not isinstance(m, SensorModel) or not isinstance(f, Field):
                raise TypeError("engine: sensors are (SensorModel, Field) pairs")
        n = len(self.sensors)
        self._fields = (_lib.Field * n)(*[field_struct(f) for _, f in self.sensors])
        self._keep = [field_struct(f) for _, f in self.sensors]  # blob tables alive during create
        for i, s in enumerate(self._keep):
            self._fields[i] = s
        models = (C.c_void_p * n)(*[m.handle.value for m, _ in self.sensors])
        self._rules = _lib.SampleRules(tol, dark, 1, 1 if refine_signature else 0, max_refine_levels, min_dt_ns,
                                       l_min, l_max)
        h = C.c_void_p()
        _lib.check(_lib.lib().bs_engine_create(models, self._fields, n, C.byref(self._rules), C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        self._h = None
        if h:
            try:
                _lib.lib().bs_engine_destroy(h)
            except Exception:  # interpreter shutdown
                pass

    def start(self, t0_ns: int = 0, stream: int | None = None, frames=None) -> None:
        """Initializes every model at t0: from its field rendered on the device, or from host frames (one float32
        array of width * height per sensor; copied to the device)."""
        if frames is None:
            _lib.check(_lib.lib().bs_engine_start(self._h, int(t0_ns), stream))
            return
        arrs = [np.ascontiguousarray(f, np.float32).reshape(-1) for f in frames]
        if len(arrs) != len(self.sensors) or any(a.size != m.width * m.height
                                                 for a, (m, _) in zip(arrs, self.sensors)):
            raise ValueError("engine: one frame of width * height per sensor")
        ptrs = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
        _lib.check(_lib.lib().bs_engine_start_frames(self._h, int(t0_ns), ptrs, stream))

    def run(self, windows: int, stream: int | None = None) -> tuple[int, int]:
        """Samples and senses `windows` whole windows; returns (pixel-samples, events) of the call."""
        s, e = C.c_uint64(), C.c_uint64()
        _lib.check(_lib.lib().bs_engine_run(self._h, int(windows), stream, C.byref(s), C.byref(e)))
        return s.value, e.value

    def take_events(self, with_pixel: bool = False) -> list[dict]:
        """Every sensor's events, as SensorModel.take_events gives them, in the engine's sensor order; the models'
        lists are cleared. The sensors' device sorts and copies are queued together, and each sensor's host copies
        run while the device works on the sensors after it."""
        import contextlib

        from .sensor import column_struct, new_columns

        models = [m for m, _ in self.sensors]
        with contextlib.ExitStack() as stack:
            for m in models:
                stack.enter_context(m._lock)
            out, structs = [], []
            for m in models:
                n = C.c_size_t()
                _lib.check(_lib.lib().bs_model_event_count(m._h, C.byref(n)))
                cols = new_columns(n.value)
                px = np.zeros(n.value, np.uint32) if with_pixel else None
                structs.append(column_struct(cols, px))
                if with_pixel:
                    cols["pixel"] = px
                out.append(cols)
            arr = (_lib.EventColumns * len(structs))(*structs)
            _lib.check(_lib.lib().bs_engine_take_events(self._h, arr))
        return out

    def set_launch(self, warps_per_block: int = 0, blocks_per_sm: int = 0, stage: int = 0,
                   tile_width: int = 0) -> None:
        """Launch shape of the persistent grid, the stage (0 streaming; 16 or 32 staged in shared memory; 64 staged
        with the warp's crossing search; 1 the split engine: per window one launch for every pixel's common path and
        one for the pixels posted at a segment that is not clean) and the tile width (4, 8, 16 or 32 px; the tile is
        32 / width px high)."""
        _lib.check(_lib.lib().bs_engine_set_launch(self._h, int(warps_per_block), int(blocks_per_sm), int(stage),
                                                   int(tile_width)))

    @property
    def launch(self) -> dict:
        out = np.zeros(4, np.int32)
        _lib.check(_lib.lib().bs_engine_get_launch(self._h, out.ctypes.data))
        return {"warps_per_block": int(out[0]), "blocks_per_sm": int(out[1]), "stage": int(out[2]),
                "tile_width": int(out[3])}

    def set_graph(self, on: bool) -> None:
        """Each run as one CUDA graph launch (default) or as separate stream operations."""
        _lib.check(_lib.lib().bs_engine_set_graph(self._h, 1 if on else 0))

    def autotune(self, windows: int = 8, stream: int | None = None) -> list[dict]:
        """Times trial steps of `windows` windows for each candidate launch shape (the models keep their state) and
        keeps the fastest; returns the candidates with their kernel ms."""
        rows = np.zeros((64, 4))
        n = C.c_size_t()
        _lib.check(_lib.lib().bs_engine_autotune(self._h, int(windows), stream, rows.ctypes.data, 64, C.byref(n)))
        return [{"tile_width": int(r[0]), "warps_per_block": int(r[1]), "stage": int(r[2]), "ms": float(r[3])}
                for r in rows[:n.value]]

    @property
    def last_ms(self) -> float:
        ms = C.c_double()
        _lib.check(_lib.lib().bs_engine_last_ms(self._h, C.byref(ms)))
        return ms.value

    def set_proposal(self, mlp=None, margin: float = 0.25) -> None:
        """Samples with the learned step proposal of `mlp` (a learned.StepMLP; None: the plain sampler). Every
        proposed step is judged by the plain midpoint rule, and a rejected one is refined by it. The walk state
        restarts from the current frame, and again at every start()."""
        self._mlp = mlp  # the engine borrows the network: keep it alive
        _lib.check(_lib.lib().bs_engine_set_proposal(self._h, mlp.handle if mlp is not None else None,
                                                     float(margin)))

    def set_record(self, capacity: int) -> None:
        """Records up to `capacity` rows of every sample and every proposed step of each following run (0: off)."""
        _lib.check(_lib.lib().bs_engine_set_record(self._h, int(capacity)))

    def take_record(self, which: str = "samples") -> dict:
        """The last run's record: 'samples' (t_ns, sensor, pixel, irradiance) or 'steps' (t_ns, sensor, pixel,
        log2 step), in recording order. Raises RuntimeError if the record's capacity was exceeded."""
        w = {"samples": 0, "steps": 1}[which]
        n = C.c_size_t()
        _lib.check(_lib.lib().bs_engine_take_record(self._h, w, 0, None, None, None, C.byref(n)))
        k = n.value
        t = np.zeros(k, np.int64)
        px = np.zeros(k, np.uint32)
        v = np.zeros(k, np.float32)
        got = C.c_size_t()
        _lib.check(_lib.lib().bs_engine_take_record(self._h, w, k, t.ctypes.data, px.ctypes.data, v.ctypes.data,
                                                    C.byref(got)))
        if got.value != k:
            raise RuntimeError(f"engine record: {got.value} rows recorded, more than its capacity")
        out = {"t_ns": t, "sensor": (px >> 24).astype(np.int32), "pixel": px & 0xFFFFFF}
        out["irradiance" if w == 0 else "log2_step"] = v if w == 0 else v.astype(np.int32)
        return out
