"""Window sampling with the interface of ``ballasim.engine.sampling`` / ``ballasim._engine``
(python/ballasim/engine/sampling.py:19-38, src/engine/bindings/engine_module.cpp:1346-1470).

``sample_window(t_w, pixel_ids, levels, rank, carried_irr, carried_sig, render, *, refine_signature, midpoint,
max_refine_levels, min_dt_ns, ...)`` runs the dyadic lattice, the eta_L midpoint refinement and the run assembly
on the B200. ``render`` is a device field (ballasim_b200.fields.Field): the renderer's stand-in evaluated inside
the sampler kernel. The economy-schedule switches (mid_levels, tau_jump_ns, delta_ref, half_ratio, eps_jump,
jump, counters, carried_class) must keep their Phase 1 defaults on this path.
"""
from __future__ import annotations

import ctypes as C
import threading
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .fields import Field

WINDOW_NS = 1 << 23


Cancelled = _lib.Cancelled


class CancelToken:
    """A cooperative cancel (the reference's _engine.CancelToken, engine_module.cpp:1351-1357): set() from any
    thread; sample_window checks it at each pixel batch and refinement round (the flag the C window reads)."""

    def __init__(self):
        self._ev = threading.Event()
        self._flag = C.c_int32(0)

    def set(self) -> None:
        """Requests the cancel (never cleared)."""
        self._flag.value = 1
        self._ev.set()

    def is_set(self) -> bool:
        return self._ev.is_set()


def _check_cancel(cancel, where: str) -> None:
    if cancel is not None and cancel.is_set():
        raise Cancelled(where + ": cancelled")


def waveform_range(waveform) -> tuple[float, float]:
    """(min, max) over all time of a light group's waveform m(t) (src/engine/window.cpp:15-23)."""
    d = waveform.get("waveform", waveform) if isinstance(waveform, dict) else waveform
    kind = d.get("type", "")
    if kind == "constant":
        return (1.0, 1.0)
    if kind == "fourier":
        s = float(sum(abs(a) for a in d["a"]))
        return (1.0 - s, 1.0 + s)
    if kind == "pulse":
        return (float(d["floor"]), 1.0)
    raise ValueError("light group: waveform type must be 'constant', 'fourier' or 'pulse'")


class MidpointTest:
    """P3 section 6.3's eta_L midpoint test (sampling.h:36-69): tolerance, dark term (renderer units) and each light
    group's waveform range; eta and exceeds evaluated on the device."""

    def __init__(self, tol: float, dark: float, m_min, m_max):
        self.m_min = tuple(float(v) for v in m_min)
        self.m_max = tuple(float(v) for v in m_max)
        if not self.m_min or len(self.m_min) != len(self.m_max) or len(self.m_min) > 8:
            raise ValueError("midpoint test: need 1 to 8 light groups")
        self.tol = float(tol)
        self.dark = float(dark)

    @staticmethod
    def for_groups(tol: float, dark: float, waveforms) -> "MidpointTest":
        r = [waveform_range(w) for w in waveforms]
        return MidpointTest(tol, dark, [a for a, _ in r], [b for _, b in r])

    def _run(self, ea, em, eb):
        G = len(self.m_min)
        a = [np.ascontiguousarray(x, np.float32).reshape(-1, G) for x in (ea, em, eb)]
        n = a[0].shape[0]
        if any(x.shape != (n, G) for x in a):
            raise ValueError("MidpointTest.eta: ea, em and eb need the same shape (n, groups)")
        eta = np.zeros(n, np.float32)
        ex = np.zeros(n, np.uint8)
        mn = np.asarray(self.m_min, np.float32)
        mx = np.asarray(self.m_max, np.float32)
        _lib.check(_lib.lib().bs_midpoint_eta(self.tol, self.dark, G, mn.ctypes.data, mx.ctypes.data,
                                              a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, n,
                                              eta.ctypes.data, ex.ctypes.data))
        return eta, ex

    def eta(self, ea, em, eb) -> np.ndarray:
        return self._run(ea, em, eb)[0]

    def exceeds(self, ea, em, eb) -> np.ndarray:
        return self._run(ea, em, eb)[1].astype(bool)


def level_cap(levels, budget: int, l_min: int):
    """The finest level keeping a window's lattice within budget samples, None when the levels fit
    (src/engine/window.cpp:25-50)."""
    lv = np.ascontiguousarray(levels, np.int64)
    cap = C.c_int32()
    _lib.check(_lib.lib().bs_level_cap(lv.ctypes.data if lv.size else None, lv.size, int(budget), int(l_min),
                                       C.byref(cap)))
    return None if cap.value < 0 else int(cap.value)


@dataclass
class WindowRuns:
    """Sample runs of one window, ready for ``SensorModel.advance(..., offsets=...)``."""

    pixel_ids: np.ndarray
    t_ns: np.ndarray
    irradiance: np.ndarray
    offsets: np.ndarray
    last_irradiance: np.ndarray
    last_signature: np.ndarray
    stats: dict = field(default_factory=dict)


def field_struct(f: Field) -> _lib.Field:
    blobs = np.ascontiguousarray(f.blobs, np.float32)
    s = _lib.Field(f.kind, f.width, f.height, f.base, f.amp, f.nx, f.ny, f.c, f.speed, f.width_px, f.n_blobs,
                   blobs.ctypes.data if blobs.size else None)
    s._keep = blobs
    return s


def rules_struct(midpoint: "MidpointTest | None", refine_signature: bool, max_refine_levels: int, min_dt_ns: int,
                 l_min: int = 1, l_max: int = 10) -> _lib.SampleRules:
    if midpoint is not None and (midpoint.m_min != (1.0,) or midpoint.m_max != (1.0,)):
        raise ValueError("sample_window: this build samples one constant light group (m_min = m_max = [1])")
    return _lib.SampleRules(midpoint.tol if midpoint else 0.0, midpoint.dark if midpoint else 0.0,
                            1 if midpoint is not None else 0, 1 if refine_signature else 0, int(max_refine_levels),
                            int(min_dt_ns), int(l_min), int(l_max))


class _SamplerCache:
    """One device sampler per field object (the field's blob table is uploaded once)."""

    def __init__(self):
        self._by_id = {}

    def get(self, f: Field):
        key = id(f)
        hit = self._by_id.get(key)
        if hit is not None and hit[0] is f:
            return hit[1]
        h = C.c_void_p()
        s = field_struct(f)
        _lib.check(_lib.lib().bs_sampler_create(C.byref(s), C.byref(h)))
        sampler = _Sampler(h)
        self._by_id[key] = (f, sampler)
        return sampler


class _Sampler:
    def __init__(self, h):
        self.h = h

    def __del__(self):
        h = getattr(self, "h", None)
        self.h = None
        if h:
            try:
                _lib.lib().bs_sampler_destroy(h)
            except Exception:  # interpreter shutdown
                pass


_samplers = _SamplerCache()


def sampler_for(f: Field):
    return _samplers.get(f)


def _render_batch(render, pixel: np.ndarray, t: np.ndarray, groups: int):
    """One render call: the callable gets (pixel_ids uint32 (n,), t_ns int64 (n,)) and returns (irradiance (n,
    groups), signature (n,)) (engine_module.cpp:227-262)."""
    res = render(pixel, t)
    e = np.ascontiguousarray(res[0], np.float32)
    s = np.ascontiguousarray(res[1], np.uint64)
    n = len(pixel)
    if e.ndim != 2 or e.shape != (n, groups) or s.shape != (n,):
        raise ValueError("render: the callable must return (irradiance (n, groups), signature (n,))")
    return e, s


def _host_window(t_w: int, ids: np.ndarray, lv: np.ndarray, ci: np.ndarray, cs: np.ndarray, render, midpoint,
                 refine_signature: bool, max_refine_levels: int, min_dt_ns: int, cancel) -> tuple:
    """The window with a Python callable as the renderer, through the C ABI's render-hook window (bs_window_run: the
    reference's host WindowEngine, src/engine/window_impl.h:462-714, breadth-first, one render call per round, the
    midpoint tests on the device). The callable sees each call's requests as (pixel_ids, t_ns); ci / cs take each
    pixel's sample at t_w + 2^23."""
    n, G = len(ids), ci.shape[1]
    errors = []

    def fn(_user, req, m, out_index, irr, sig, _subsamples):
        try:
            words = np.ctypeslib.as_array(C.cast(req, C.POINTER(C.c_uint32)), (m * 6,)).reshape(m, 6)
            idx = np.ctypeslib.as_array(out_index, (m,)).astype(np.int64)
            px = words[:, 1].copy()
            t = int(t_w) + words[:, 4].view(np.int32).astype(np.int64)
            e, s = _render_batch(render, px, t, G)
            rows = int(idx.max()) + 1
            np.ctypeslib.as_array(irr, (rows * G,)).reshape(rows, G)[idx] = e
            np.ctypeslib.as_array(sig, (rows,))[idx] = s
            return 0
        except BaseException as ex:  # the callback cannot raise through C: kept, and raised after the call
            errors.append(ex)
            return 1

    cb = _lib.RENDER_FN(fn)
    mn = np.ascontiguousarray(midpoint.m_min if midpoint is not None else [1.0] * G, np.float32)
    mx = np.ascontiguousarray(midpoint.m_max if midpoint is not None else [1.0] * G, np.float32)
    h = C.c_void_p()
    _lib.check(_lib.lib().bs_window_create(G, mn.ctypes.data, mx.ctypes.data, C.byref(h)))
    try:
        rules = _lib.WindowRules(midpoint.tol if midpoint is not None else 0.0,
                                 midpoint.dark if midpoint is not None else 0.0, 1 if midpoint is not None else 0,
                                 1 if refine_signature else 0, int(max_refine_levels), int(min_dt_ns), 0, 64,
                                 C.addressof(cancel._flag) if cancel is not None else None)
        total = C.c_size_t()
        st = _lib.lib().bs_window_run(h, int(t_w), _lib.ptr(ids), _lib.ptr(lv), n, _lib.ptr(ci), _lib.ptr(cs),
                                      C.byref(rules), cb, None, C.byref(total))
        if errors:
            raise errors[0]
        _lib.check(st)
        S = total.value
        off = np.zeros(n + 1, np.int64)
        t = np.zeros(S, np.int64)
        irr = np.zeros((S, G), np.float32)
        _lib.check(_lib.lib().bs_window_runs(h, off.ctypes.data, t.ctypes.data if S else None,
                                             irr.ctypes.data if S else None))
        counters = np.zeros(4, np.uint64)
        rounds = C.c_size_t()
        by_round = np.zeros(64, np.uint64)
        _lib.check(_lib.lib().bs_window_stats(h, counters.ctypes.data, by_round.ctypes.data, 64, C.byref(rounds)))
    finally:
        _lib.lib().bs_window_destroy(h)
    k = min(rounds.value, 64)
    stats = {"pixels": n, "samples_by_round": [int(v) for v in by_round[:k]],
             "flagged_signature": int(counters[0]), "flagged_midpoint": int(counters[1]),
             "refine_cap_hits": int(counters[2]), "render_calls": int(counters[3]),
             "band_samples_by_round": [0] * k}
    return t, irr, off, stats


def sample_window(t_w: int, pixel_ids, levels, rank, carried_irr, carried_sig, render, *, refine_signature: bool,
                  midpoint, max_refine_levels: int, min_dt_ns: int, mid_levels=None, tau_jump_ns=None,
                  delta_ref: float = 0.0, half_ratio: float = 0.0, eps_jump=None, jump=None, counters: bool = False,
                  carried_class=None, cancel=None) -> WindowRuns:
    """sample_window (engine_module.cpp:311-355). ``render`` is a device field (ballasim_b200.fields.Field), sampled
    inside the sampler kernel, or a Python callable render(pixel_ids, t_ns) -> (irradiance (n, groups), signature
    (n,)) as the reference's host path takes (engine_module.cpp:227-305): that window runs breadth-first on the
    host with the midpoint tests on the device."""
    host = not isinstance(render, Field)
    if host and not callable(render):
        raise TypeError("sample_window: render must be a device field or a callable render(pixel_ids, t_ns)")
    if any(v is not None for v in (mid_levels, tau_jump_ns, eps_jump, jump, carried_class)) or delta_ref != 0.0 \
            or half_ratio != 0.0 or counters:
        raise ValueError("sample_window: the economy-schedule switches are not on this path (Phase 1 rules only)")
    if min_dt_ns < 1 or min_dt_ns > WINDOW_NS or (min_dt_ns & (min_dt_ns - 1)) != 0:
        raise ValueError("min_dt_ns must be a power of two in [1, 2^23]")
    if max_refine_levels < 0:
        raise ValueError("max_refine_levels must be >= 0")
    if not host:
        _check_cancel(cancel, "window: batch")
    ids = np.ascontiguousarray(pixel_ids, np.uint32).reshape(-1)
    n = len(ids)
    lv64 = np.ascontiguousarray(levels, np.int64).reshape(-1)
    max_level = 23 - (int(min_dt_ns).bit_length() - 1)
    if np.any(lv64 < 0) or np.any(lv64 > max_level):
        raise ValueError("levels must lie in [0, 23 - log2(min_dt_ns)]")
    lv = lv64.astype(np.uint8)
    rk = np.ascontiguousarray(rank, np.uint32).reshape(-1)
    ci = np.array(carried_irr, np.float32, copy=True)
    if ci.ndim == 1:
        ci = ci.reshape(-1, 1)
    cs = np.array(carried_sig, np.uint64, copy=True).reshape(-1)
    if len(rk) != n or ci.shape[0] != n or len(cs) != n or len(lv) != n:
        raise ValueError("pixel_ids, levels, rank, carried_irr and carried_sig need one entry per pixel")
    if host:
        G = ci.shape[1]
        if G < 1 or G > 8:
            raise ValueError("need 1 to 8 light groups")
        if midpoint is not None and (len(midpoint.m_min) != G or len(midpoint.m_max) != G):
            raise ValueError("MidpointTest: one waveform range per light group is needed")
        t, irr, off, stats = _host_window(int(t_w), ids, lv, ci, cs, render, midpoint, bool(refine_signature),
                                          int(max_refine_levels), int(min_dt_ns), cancel)
        return WindowRuns(ids.copy(), t, irr, off, ci, cs, stats)
    if ci.shape[1] != 1:
        raise ValueError("sample_window: this build samples one light group")
    rules = rules_struct(midpoint, refine_signature, max_refine_levels, min_dt_ns)
    s = sampler_for(render)
    total = C.c_size_t()
    cflat = np.ascontiguousarray(ci.reshape(-1))
    _lib.check(_lib.lib().bs_sample_window(s.h, int(t_w), _lib.ptr(ids), _lib.ptr(lv), n, _lib.ptr(cflat),
                                           _lib.ptr(cs), C.byref(rules), C.byref(total)))
    S = total.value
    off = np.zeros(n + 1, np.int64)
    t = np.zeros(S, np.int64)
    irr = np.zeros(S, np.float32)
    _lib.check(_lib.lib().bs_sampler_download(s.h, off.ctypes.data, t.ctypes.data if S else None,
                                              irr.ctypes.data if S else None))
    stats = {"pixels": n, "samples": S}
    return WindowRuns(ids.copy(), t, irr.reshape(S, 1), off, cflat.reshape(n, 1), cs, stats)


def fixed_rate_samples(t_w: int, period_ns: int) -> int:
    """Samples of the fixed-rate grid in the window at t_w besides its carried one (src/engine/window.cpp:52-56):
    the multiples of period_ns strictly inside (t_w, t_w + W), plus t_w + W itself."""
    q = t_w // period_ns
    inner = -((-(t_w + WINDOW_NS)) // period_ns) - q - 1
    return max(inner, 0) + 1


def fixed_rate_window(t_w: int, pixel_ids, rank, period_ns: int, carried_irr, carried_sig, render) -> WindowRuns:
    """fixed_rate_window (engine_module.cpp:356-365) with a Python callable render(pixel_ids, t_ns) ->
    (irradiance (n, groups), signature (n,)): every pixel's samples at the absolute multiples of period_ns inside
    (t_w, t_w + W) and at t_w + W (sampling.h:344-350), after its carried one; no refinement. One render call, in
    pixel-major slot order."""
    if period_ns < 1:
        raise ValueError("period_ns must be >= 1")
    ids = np.ascontiguousarray(pixel_ids, np.uint32).reshape(-1)
    n = len(ids)
    rk = np.ascontiguousarray(rank, np.uint32).reshape(-1)
    ci = np.array(carried_irr, np.float32, copy=True)
    if ci.ndim == 1:
        ci = ci.reshape(-1, 1)
    cs = np.array(carried_sig, np.uint64, copy=True).reshape(-1)
    if len(rk) != n or ci.shape[0] != n or len(cs) != n:
        raise ValueError("pixel_ids, levels, rank, carried_irr and carried_sig need one entry per pixel")
    G = ci.shape[1]
    if G < 1 or G > 8:
        raise ValueError("need 1 to 8 light groups")
    m = fixed_rate_samples(int(t_w), int(period_ns))
    stats = {"pixels": n, "samples_by_round": [0], "flagged_signature": 0, "flagged_midpoint": 0,
             "refine_cap_hits": 0, "band_samples_by_round": [0]}
    if n == 0:
        return WindowRuns(ids.copy(), np.zeros(0, np.int64), np.zeros((0, G), np.float32), np.zeros(1, np.int64), ci,
                          cs, stats)
    j = np.arange(m + 1, dtype=np.int64)
    dt = np.where(j == 0, 0, np.where(j >= m, WINDOW_NS, (int(t_w) // int(period_ns) + j) * int(period_ns) - int(t_w)))
    t = np.tile(int(t_w) + dt, n)
    irr = np.zeros((n * (m + 1), G), np.float32)
    first = np.arange(n, dtype=np.int64) * (m + 1)
    irr[first] = ci
    req = np.nonzero(np.tile(j != 0, n))[0]
    e, sig = _render_batch(render, np.repeat(ids, m), t[req], G)
    irr[req] = e
    last = first + m
    ci[:] = irr[last]
    cs[:] = sig.reshape(n, m)[:, -1]
    stats["samples_by_round"] = [len(req)]
    return WindowRuns(ids.copy(), t, irr, np.arange(n + 1, dtype=np.int64) * (m + 1), ci, cs, stats)


def field_levels(f: Field, t_w: int, l_min: int = 1, l_max: int = 10) -> np.ndarray:
    """The field's level rule per pixel at the window start t_w (uint8, pixel order), on the device."""
    s = sampler_for(f)
    out = np.zeros(f.width * f.height, np.uint8)
    _lib.check(_lib.lib().bs_field_levels(s.h, int(t_w), int(l_min), int(l_max), out.ctypes.data))
    return out


def field_frame(f: Field, t_ns: int) -> np.ndarray:
    """The field at t over the frame (float32, pixel order), on the device."""
    s = sampler_for(f)
    out = np.zeros(f.width * f.height, np.float32)
    _lib.check(_lib.lib().bs_field_frame(s.h, int(t_ns), out.ctypes.data))
    return out
