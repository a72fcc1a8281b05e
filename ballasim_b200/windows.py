"""The reference engine's per-window loop with the runs in HBM (Camera::sample_and_sense,
src/engine/engine_impl.h:1253-1343): per sensor and window, the lattice levels by the field's rule, sample_window on
device-resident inputs into CSR runs in device memory (WindowEngine<Space::kDevice>::run, src/engine/window.h:133-174;
bs_sample_window_device), then SensorModel::advance_device on those runs (src/sensor/sensor_model.h:157-167); the
events stay on the device.

This is the two-kernel form of what the fused engine (engine.Engine) does in one launch: it writes and re-reads the
runs (12 B per pixel-sample each way) and synchronizes twice per sensor and window (the window's sample count with
its input flags, the sensor's counters), as the reference's engine synchronizes per window. The sensors are
independent, so by default each sensor's windows run in order on a stream of its own, driven from a host thread of
its own: one sensor's synchronizations and host work overlap the others' kernels. Device buffers are torch tensors.
"""
from __future__ import annotations

import ctypes as C
from concurrent.futures import ThreadPoolExecutor, wait

import numpy as np

from . import _lib
from .sampling import MidpointTest, rules_struct, sampler_for


def _stream_handle(stream: int | None) -> int:
    """The stream every call of a step goes to: the given handle, else torch's current stream (its legacy default
    stream, handle 0, passed as cudaStreamLegacy: a NULL stream means each library object's own stream, and the
    sampler's runs must be written on the stream that the pixel model then reads them on)."""
    if stream:
        return int(stream)
    import torch

    return int(torch.cuda.current_stream().cuda_stream) or 1  # 1: cudaStreamLegacy


class DeviceWindows:
    """Sensors (SensorModel, Field) sampled and sensed window by window through the C ABI's device boundary, every
    call of a step on one stream."""

    def __init__(self, sensors, *, tol: float = 0.01, dark: float = 0.01, min_dt_ns: int = 8192,
                 max_refine_levels: int = 10, l_min: int = 1, l_max: int = 10):
        import torch

        self.sensors = list(sensors)
        if not self.sensors:
            raise ValueError("DeviceWindows: need at least one sensor")
        self.rules = rules_struct(MidpointTest(tol, dark, [1.0], [1.0]), True, max_refine_levels, min_dt_ns)
        self.l_min, self.l_max = int(l_min), int(l_max)
        dev = torch.device("cuda")
        self._bufs = []
        for m, f in self.sensors:
            if (f.width, f.height) != (m.width, m.height):
                raise ValueError("DeviceWindows: a field's frame must match its sensor")
            n = m.width * m.height
            self._bufs.append({
                "sampler": sampler_for(f),
                "ids": torch.arange(n, dtype=torch.int32, device=dev),
                "level": torch.empty(n, dtype=torch.uint8, device=dev),
                "carried": [torch.empty(n, dtype=torch.float32, device=dev) for _ in range(2)],
                "sig": [torch.zeros(n, dtype=torch.int64, device=dev) for _ in range(2)],
                "cur": 0,
            })
        self.t_ns = 0
        self.launch_ms = 0.0
        self._streams = None  # the sensors' own streams and their host threads, made at the first concurrent run
        self._pool = None

    def start(self, t0_ns: int = 0, stream: int | None = None, frames=None) -> None:
        """Renders every field at t0 on the device (or copies frames[i], sensor i's host frame of height * width
        floats, ideally pinned), initializes each model from it, and carries it as each pixel's first sample."""
        import torch

        if t0_ns % (1 << 23):
            raise ValueError("DeviceWindows.start: t0 must be a window start")
        stream = _stream_handle(stream)
        for i, ((m, _), b) in enumerate(zip(self.sensors, self._bufs)):
            b["cur"] = 0
            b["sig"][0].zero_()
            if frames is not None:
                src = torch.from_numpy(np.ascontiguousarray(frames[i], np.float32).reshape(-1))
                b["carried"][0].copy_(src, non_blocking=True)
            else:
                _lib.check(_lib.lib().bs_field_frame_device(b["sampler"].h, int(t0_ns), b["carried"][0].data_ptr(),
                                                            stream))
            m.init_device(int(t0_ns), b["carried"][0].data_ptr(), stream)
        self.t_ns = int(t0_ns)

    def run(self, windows: int, stream: int | None = None, on_events=None, concurrent: bool = True) -> tuple[int, int]:
        """Samples and senses `windows` windows of every sensor. on_events(i, model, events) sees each call's device
        events (valid until that model advances again), in window order for each sensor. Returns the pixel-samples and
        events of the call; launch_ms accumulates the sensors' kernel times.

        concurrent (with more than one sensor): each sensor's windows on its own stream from its own host thread,
        those streams starting after the work already queued on `stream` and `stream` waiting for them at the end
        (on_events is then called from those threads, each sensor's calls from one). Otherwise window-major on
        `stream` (each window of every sensor, then the next), as the reference's engine runs its cameras."""
        stream = _stream_handle(stream)
        t0 = self.t_ns
        n_sensors = len(self.sensors)
        if concurrent and n_sensors > 1:
            import torch

            dev = torch.cuda.current_device()
            if self._streams is None:
                self._streams = [torch.cuda.Stream(device=dev) for _ in range(n_sensors)]
                self._pool = ThreadPoolExecutor(max_workers=n_sensors, thread_name_prefix="bs-sensor")
            caller = (torch.cuda.current_stream(dev) if stream == 1
                      else torch.cuda.ExternalStream(stream, device=dev))
            ready = torch.cuda.Event()
            ready.record(caller)
            for st in self._streams:
                st.wait_event(ready)

            def one(i):
                torch.cuda.set_device(dev)
                return self._sensor_windows(i, t0, windows, self._streams[i].cuda_stream, on_events)

            futures = [self._pool.submit(one, i) for i in range(n_sensors)]
            wait(futures)  # every sensor's thread done before any error reaches the caller
            parts = [f.result() for f in futures]
            for st in self._streams:
                done = torch.cuda.Event()
                done.record(st)
                caller.wait_event(done)
        else:
            parts = [[0, 0, 0.0] for _ in range(n_sensors)]
            for w in range(int(windows)):
                for i in range(n_sensors):
                    got = self._sensor_windows(i, t0 + w * (1 << 23), 1, stream, on_events)
                    parts[i] = [a + b for a, b in zip(parts[i], got)]
        self.launch_ms += sum(p[2] for p in parts)
        self.t_ns = t0 + int(windows) * (1 << 23)
        return sum(p[0] for p in parts), sum(p[1] for p in parts)

    def _sensor_windows(self, i: int, t_w: int, windows: int, stream: int, on_events) -> list:
        """Sensor i's windows [t_w, t_w + windows * 2^23) on `stream`: [pixel-samples, events, kernel ms]."""
        L = _lib.lib()
        (m, _), b = self.sensors[i], self._bufs[i]
        s, n = b["sampler"], m.width * m.height
        total = C.c_size_t()
        runs = _lib.DeviceRuns()
        samples = events = 0
        ms = 0.0
        for _ in range(int(windows)):
            cur = b["cur"]
            _lib.check(L.bs_field_levels_device(s.h, t_w, self.l_min, self.l_max, b["level"].data_ptr(), stream))
            _lib.check(L.bs_sample_window_device(
                s.h, t_w, b["ids"].data_ptr(), b["level"].data_ptr(), n, b["carried"][cur].data_ptr(),
                b["sig"][cur].data_ptr(), b["carried"][1 - cur].data_ptr(), b["sig"][1 - cur].data_ptr(),
                C.byref(self.rules), stream, C.byref(total)))
            _lib.check(L.bs_sampler_device_runs(s.h, C.byref(runs)))
            ms0 = m.stats()["gpu_launch_ms_total"]
            ev = m.advance_device(runs, t_w + (1 << 23), stream)
            ms += m.stats()["gpu_launch_ms_total"] - ms0
            if on_events is not None:
                on_events(i, m, ev)
            samples += int(total.value)
            events += int(ev.count)
            b["cur"] = 1 - cur
            t_w += 1 << 23
        return [samples, events, ms]


def carried_samples(dw: DeviceWindows, i: int) -> np.ndarray:
    """Sensor i's carried samples (each pixel's last sample) as a host array."""
    b = dw._bufs[i]
    return b["carried"][b["cur"]].cpu().numpy()
