"""ctypes access to the oracle: the C restatement (oracle/port, ``Port``) and the reference's own CPU code
compiled from its sources (oracle/_ref, ``Ref``). TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke()
and bench.py's cpu_baseline leg use it as the checker; the product never imports it.

Both sides take the same inputs: a resolved SensorParams (ballasim_b200.params), a Field (ballasim_b200.fields)
and the sampler rules; events come back as dicts of numpy columns sorted by (t_cross, pixel).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import build as _build

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C")
_u16p = np.ctypeslib.ndpointer(np.uint16, flags="C")


class OrcField(C.Structure):
    _fields_ = [("kind", C.c_int32), ("width", C.c_uint32), ("height", C.c_uint32), ("base", C.c_float),
                ("amp", C.c_float), ("nx", C.c_float), ("ny", C.c_float), ("c", C.c_float), ("speed", C.c_float),
                ("width_px", C.c_float), ("n_blobs", C.c_int32), ("blobs", C.c_void_p)]


class OrcParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("theta_on", "theta_off", "sigma_theta_on", "sigma_theta_off",
                                          "theta_onoff_corr", "theta_floor")] + \
               [("reset_mode", C.c_int32), ("refractory_s", C.c_double), ("eps_ci", C.c_double),
                ("initial_phase", C.c_int32)] + \
               [(n, C.c_double) for n in ("leak_rate_hz", "leak_sigma_log10", "leak_ea_eV", "dark_current_fA",
                                          "dark_sigma_ln", "dark_ea_eV", "temperature_K", "reference_temperature_K",
                                          "illuminance_scale", "label_share_cut", "readout_quantum_s",
                                          "readout_delay_s", "clock_drift_ppm")] + \
               [("clock_offset_ns", C.c_int64), ("noise", C.c_int32), ("shot_rate_hz", C.c_double),
                ("ba_median_hz", C.c_double), ("ba_sigma_ln", C.c_double)]


class OrcRules(C.Structure):
    _fields_ = [("tol", C.c_float), ("dark", C.c_float), ("midpoint", C.c_int32), ("refine_signature", C.c_int32),
                ("max_refine_levels", C.c_int32), ("min_dt_ns", C.c_int64)]


class OrcEvent(C.Structure):
    _fields_ = [("pixel", C.c_uint32), ("polarity", C.c_uint8), ("label", C.c_uint8), ("flags", C.c_uint16),
                ("t_cross", C.c_int64), ("ds", C.c_float), ("dn", C.c_float), ("dl", C.c_float),
                ("l_first", C.c_float)]


EVENT_DTYPE = np.dtype([("pixel", np.uint32), ("polarity", np.uint8), ("label", np.uint8), ("flags", np.uint16),
                        ("t_cross", np.int64), ("ds", np.float32), ("dn", np.float32), ("dl", np.float32),
                        ("l_first", np.float32)])
assert EVENT_DTYPE.itemsize == C.sizeof(OrcEvent) == 32


def field_struct(f):
    """An OrcField of a ballasim_b200.fields.Field (the blob table kept alive on the struct)."""
    blobs = np.ascontiguousarray(f.blobs, np.float32)
    s = OrcField(f.kind, f.width, f.height, f.base, f.amp, f.nx, f.ny, f.c, f.speed, f.width_px, f.n_blobs,
                 blobs.ctypes.data if blobs.size else None)
    s._keep = blobs
    return s


def params_struct(p) -> OrcParams:
    """An OrcParams of a resolved ballasim_b200.params.SensorParams."""
    v = p.as_dict()
    o = OrcParams()
    for name in ("theta_on", "theta_off", "sigma_theta_on", "sigma_theta_off", "theta_onoff_corr", "theta_floor",
                 "refractory_s", "eps_ci", "leak_rate_hz", "leak_sigma_log10", "leak_ea_eV", "dark_current_fA",
                 "dark_sigma_ln", "dark_ea_eV", "temperature_K", "reference_temperature_K", "illuminance_scale",
                 "label_share_cut", "readout_quantum_s", "readout_delay_s", "clock_drift_ppm"):
        setattr(o, name, float(v[name]))
    o.reset_mode = 1 if v["reset_mode"] == "ideal" else 0
    o.initial_phase = {"uniform": 0, "symmetric": 1, "zero": 2}[v["initial_phase"]]
    o.clock_offset_ns = int(v["clock_offset_ns"])
    o.noise = 1 if (v["noise_shot_rate_hz"] > 0 or v["noise_ba_median_hz"] > 0) else 0
    o.shot_rate_hz = float(v["noise_shot_rate_hz"])
    o.ba_median_hz = float(v["noise_ba_median_hz"])
    o.ba_sigma_ln = float(v["noise_ba_sigma_ln"])
    return o


def rules_struct(r) -> OrcRules:
    return OrcRules(r.tol, r.dark, 1, 1, r.max_refine_levels, r.min_dt_ns)


def _events_from_records(rec: np.ndarray, width: int) -> dict:
    return {"pixel": rec["pixel"].copy(), "x": (rec["pixel"] % width).astype(np.uint16),
            "y": (rec["pixel"] // width).astype(np.uint16), "p": rec["polarity"].copy(), "label": rec["label"].copy(),
            "flags": rec["flags"].copy(), "t_cross_ns": rec["t_cross"].copy(), "ds": rec["ds"].copy(),
            "dn": rec["dn"].copy(), "dl": rec["dl"].copy(), "l_first": rec["l_first"].copy()}


class OrcWalk(C.Structure):
    _fields_ = [("hx", C.c_float * 8), ("gaps", C.c_uint64), ("pv", C.c_float), ("valid", C.c_int32)]


class Port:
    """The C restatement (oracle/port/oracle.c)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            L = C.CDLL(str(_build.build_port()))
            L.orc_logf.restype = C.c_float
            L.orc_logf.argtypes = [C.c_float]
            L.orc_log.restype = C.c_double
            L.orc_log.argtypes = [C.c_double]
            L.orc_expf.restype = C.c_float
            L.orc_expf.argtypes = [C.c_float]
            L.orc_draw.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, _u32p]
            L.orc_philox.argtypes = [_u32p, _u32p, _u32p]
            L.orc_field_eval.restype = C.c_float
            L.orc_field_eval.argtypes = [C.POINTER(OrcField), C.c_uint32, C.c_uint32, C.c_int64]
            L.orc_field_level.restype = C.c_int32
            L.orc_field_level.argtypes = [C.POINTER(OrcField), C.c_uint32, C.c_uint32, C.c_int64, C.c_int32,
                                          C.c_int32]
            L.orc_field_frame.argtypes = [C.POINTER(OrcField), C.c_int64, _f32p]
            L.orc_field_samples.argtypes = [C.POINTER(OrcField), _u32p, _i64p, C.c_size_t, _f32p]
            L.orc_field_levels.argtypes = [C.POINTER(OrcField), C.c_int64, C.c_int32, C.c_int32, _u8p]
            L.orc_model_create.restype = C.c_void_p
            L.orc_model_create.argtypes = [C.POINTER(OrcParams), C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32,
                                           C.c_int32]
            L.orc_model_destroy.argtypes = [C.c_void_p]
            L.orc_model_init.argtypes = [C.c_void_p, C.c_int64, _f32p]
            L.orc_model_advance_runs.argtypes = [C.c_void_p, _u32p, C.c_size_t, _i64p, _f32p, C.c_size_t, _i64p,
                                                 _i32p, C.c_int64]
            L.orc_model_event_count.restype = C.c_size_t
            L.orc_model_event_count.argtypes = [C.c_void_p]
            L.orc_model_take_events.argtypes = [C.c_void_p, C.c_void_p]
            L.orc_model_maps.argtypes = [C.c_void_p, _f64p, _f64p, _f64p, _f64p, _f64p]
            L.orc_model_state.argtypes = [C.c_void_p, _i64p, _i64p, _f32p, _f32p, _f32p]
            L.orc_model_noise_maps.argtypes = [C.c_void_p, _f64p]
            L.orc_model_stat.restype = C.c_uint64
            L.orc_model_stat.argtypes = [C.c_void_p, C.c_int32]
            L.orc_last_error.restype = C.c_char_p
            L.orc_sample_window.restype = C.c_int64
            L.orc_sample_window.argtypes = [C.POINTER(OrcField), C.POINTER(OrcRules), C.c_int64, _u32p, _u8p,
                                            C.c_size_t, _f32p, _u64p, _i64p, _i64p, _f32p, C.c_size_t]
            L.orc_midpoint_eta.restype = C.c_float
            L.orc_midpoint_eta.argtypes = [C.c_float, C.c_float, C.c_float, C.c_float, C.c_float]
            L.orc_bf16.restype = C.c_uint16
            L.orc_bf16.argtypes = [C.c_float]
            L.orc_step_features.argtypes = [_f32p, C.c_uint64, C.c_float, _f32p]
            L.orc_walk_reset.argtypes = [C.POINTER(OrcWalk), C.c_float]
            L.orc_walk_window.restype = C.c_int32
            L.orc_walk_window.argtypes = [_i64p, _f32p, C.c_int32, C.c_int64, C.c_int32, C.c_int32, C.c_float,
                                          C.c_uint64, C.c_uint32, C.c_int32, C.POINTER(OrcWalk), _u16p, _f32p,
                                          _u64p, C.c_int32]
            L.orc_learned_window.restype = C.c_int64
            L.orc_learned_window.argtypes = [C.POINTER(OrcField), C.POINTER(OrcRules), C.c_int64, C.c_uint32,
                                             C.c_uint32, C.c_int32, C.c_float, C.POINTER(OrcWalk), _i32p, C.c_int32,
                                             _i64p, _f32p, C.c_size_t]
            cls._lib = L
        return cls._lib

    # ---- scalar helpers ----
    @classmethod
    def draw(cls, seed, purpose, camera, pixel, index) -> np.ndarray:
        out = np.zeros(4, np.uint32)
        cls.lib().orc_draw(seed, purpose, camera, pixel, index, out)
        return out

    @classmethod
    def philox(cls, ctr, key) -> np.ndarray:
        out = np.zeros(4, np.uint32)
        cls.lib().orc_philox(np.asarray(ctr, np.uint32), np.asarray(key, np.uint32), out)
        return out

    @classmethod
    def field_frame(cls, f, t_ns: int) -> np.ndarray:
        s = field_struct(f)
        out = np.zeros(f.width * f.height, np.float32)
        cls.lib().orc_field_frame(C.byref(s), t_ns, out)
        return out

    @classmethod
    def field_samples(cls, f, pixel, t_ns) -> np.ndarray:
        s = field_struct(f)
        px = np.ascontiguousarray(pixel, np.uint32)
        out = np.zeros(len(px), np.float32)
        cls.lib().orc_field_samples(C.byref(s), px, np.ascontiguousarray(t_ns, np.int64), len(px), out)
        return out

    @classmethod
    def levels(cls, f, t_w: int, l_min: int, l_max: int) -> np.ndarray:
        s = field_struct(f)
        out = np.zeros(f.width * f.height, np.uint8)
        cls.lib().orc_field_levels(C.byref(s), t_w, l_min, l_max, out)
        return out

    @classmethod
    def sample_window(cls, f, rules, t_w, pixel, level, carried_irr, carried_sig):
        s, r = field_struct(f), rules_struct(rules)
        n = len(pixel)
        off = np.zeros(n + 1, np.int64)
        cap = max(16, int(np.sum((1 << level.astype(np.int64)) + 1)) * 4)
        while True:
            t = np.zeros(cap, np.int64)
            irr = np.zeros(cap, np.float32)
            ci, cs = carried_irr.copy(), carried_sig.copy()
            k = cls.lib().orc_sample_window(C.byref(s), C.byref(r), t_w, np.ascontiguousarray(pixel, np.uint32),
                                            np.ascontiguousarray(level, np.uint8), n, ci, cs, off, t, irr, cap)
            if k >= 0:
                return t[:k], irr[:k], off, ci, cs
            cap = -k

    # ---- the learned step proposal ----
    @classmethod
    def step_features(cls, hx, gaps: int, x: float) -> np.ndarray:
        out = np.zeros(16, np.float32)
        cls.lib().orc_step_features(np.ascontiguousarray(hx, np.float32), int(gaps), float(x), out)
        return out

    @classmethod
    def walk_pairs(cls, f, rules, windows: int, *, stride: int = 1, eps: float = 1e-4, seed: int = 0,
                   t0: int = 0):
        """The training walk over the oracle sampler's runs: (x uint16 (n, 16), y float32, keys uint64), in
        (pixel, window, step) order."""
        L = cls.lib()
        sh = int(np.log2(rules.min_dt_ns))
        np_ = f.width * f.height
        ids = np.arange(np_, dtype=np.uint32)
        carried = cls.field_frame(f, t0)
        sig = np.zeros(np_, np.uint64)
        walkers = ids[::stride]
        walks = {int(p): OrcWalk() for p in walkers}
        xs, ys, ks = [], [], []
        for w in range(windows):
            t_w = t0 + w * (1 << 23)
            lv = cls.levels(f, t_w, rules.l_min, rules.l_max)
            t, irr, off, carried, sig = cls.sample_window(f, rules, t_w, ids, lv, carried, sig)
            for p in walkers:
                a, b = int(off[p]), int(off[p + 1])
                st = walks[int(p)]
                if w == 0:
                    L.orc_walk_reset(C.byref(st), float(irr[a]))
                cap = 1 << 12
                x = np.zeros((cap, 16), np.uint16)
                y = np.zeros(cap, np.float32)
                k = np.zeros(cap, np.uint64)
                n = L.orc_walk_window(np.ascontiguousarray(t[a:b]), np.ascontiguousarray(irr[a:b]), b - a, t_w,
                                      int(lv[p]), sh, float(eps), int(seed), int(p), w, C.byref(st), x, y, k, cap)
                assert n <= cap
                xs.append(x[:n])
                ys.append(y[:n])
                ks.append(k[:n])
        x, y, k = np.concatenate(xs), np.concatenate(ys), np.concatenate(ks)
        o = np.argsort(k, kind="stable")
        return x[o], y[o], k[o]

    @classmethod
    def learned_replay(cls, f, rules, steps: dict, windows: int, pixels, t0: int = 0):
        """The learned sampler's samples of the given pixels over `windows` windows for the recorded steps
        (steps[pixel] = log2 of every proposed step in time order): {pixel: (t, v)}, slot 0 excluded."""
        L = cls.lib()
        s, r = field_struct(f), rules_struct(rules)
        frame = cls.field_frame(f, t0)
        out = {}
        for p in pixels:
            p = int(p)
            x, y = p % f.width, p // f.width
            w_st = OrcWalk()
            L.orc_walk_reset(C.byref(w_st), float(frame[p]))
            seq = np.ascontiguousarray(steps[p], np.int32)
            k = 0
            ts, vs = [], []
            carried = float(frame[p])
            for w in range(windows):
                t_w = t0 + w * (1 << 23)
                level = int(L.orc_field_level(C.byref(s), x, y, t_w, rules.l_min, rules.l_max))
                # the steps of this window: those that start inside it
                n_w = 0
                cur = 0
                while cur < (1 << 23):
                    if k + n_w >= len(seq):
                        raise AssertionError(f"pixel {p}: recorded steps end inside window {w}")
                    cur += 1 << int(seq[k + n_w])
                    n_w += 1
                cap = 1 << 14
                t = np.zeros(cap, np.int64)
                v = np.zeros(cap, np.float32)
                n = L.orc_learned_window(C.byref(s), C.byref(r), t_w, x, y, level, carried, C.byref(w_st),
                                         np.ascontiguousarray(seq[k:k + n_w]), n_w, t, v, cap)
                if n < 0:
                    raise AssertionError(f"pixel {p} window {w}: invalid recorded steps (code {n})")
                ts.append(t[:n])
                vs.append(v[:n])
                carried = float(v[n - 1])
                k += n_w
            out[p] = (np.concatenate(ts), np.concatenate(vs))
        return out

    # ---- the sensor model ----
    class Model:
        def __init__(self, params, width, height, seed, camera=0):
            self.L = Port.lib()
            self.width, self.height = width, height
            self.p = params_struct(params)
            self.h = self.L.orc_model_create(C.byref(self.p), width, height, seed, camera, 1)
            if not self.h:
                raise ValueError(self.L.orc_last_error().decode())

        def __del__(self):
            if getattr(self, "h", None):
                self.L.orc_model_destroy(self.h)
                self.h = None

        def init(self, t0, irr0):
            if self.L.orc_model_init(self.h, t0, np.ascontiguousarray(irr0, np.float32)) != 0:
                raise ValueError(self.L.orc_last_error().decode())

        def advance_runs(self, ids, t, irr, row_start, row_count, t_end):
            rc = self.L.orc_model_advance_runs(self.h, np.ascontiguousarray(ids, np.uint32), len(ids),
                                               np.ascontiguousarray(t, np.int64),
                                               np.ascontiguousarray(irr, np.float32), len(t),
                                               np.ascontiguousarray(row_start, np.int64),
                                               np.ascontiguousarray(row_count, np.int32), t_end)
            if rc != 0:
                raise ValueError(self.L.orc_last_error().decode())

        def take_events(self) -> dict:
            n = self.L.orc_model_event_count(self.h)
            rec = np.zeros(n, EVENT_DTYPE)
            self.L.orc_model_take_events(self.h, rec.ctypes.data if n else None)
            return _events_from_records(rec, self.width)

        def maps(self) -> dict:
            n = self.width * self.height
            a = [np.zeros(n) for _ in range(5)]
            self.L.orc_model_maps(self.h, *a)
            return dict(zip(("theta_on", "theta_off", "leak", "dark_current_fA", "phi0"), a))

        def ba_rates(self) -> np.ndarray:
            out = np.zeros(self.width * self.height)
            self.L.orc_model_noise_maps(self.h, out)
            return out

        def state(self) -> dict:
            n = self.width * self.height
            t_ref, t_search = np.zeros(n, np.int64), np.zeros(n, np.int64)
            s3, dr, held = np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros(n, np.float32)
            self.L.orc_model_state(self.h, t_ref, t_search, s3, dr, held)
            return {"t_ref": t_ref, "t_search": t_search, "s3_ref": s3, "dr_ref": dr, "held": held}


class Ref:
    """The reference's own CPU code (oracle/_ref/libballa_ref.so, built by oracle/build.py)."""

    _lib = None

    @classmethod
    def available(cls) -> bool:
        try:
            cls.lib()
            return True
        except (OSError, RuntimeError):
            return False

    @classmethod
    def lib(cls):
        if cls._lib is None:
            so = _build.build_ref()
            if so is None or not Path(so).exists():
                raise RuntimeError("the reference harness is not built (no reference tree and no prebuilt library)")
            L = C.CDLL(str(so))
            L.ref_last_error.restype = C.c_char_p
            L.ref_model_create.restype = C.c_void_p
            L.ref_model_create.argtypes = [C.c_char_p, C.POINTER(C.c_char_p), C.POINTER(C.c_double), C.c_int,
                                           C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32, C.c_int]
            L.ref_model_create_prec.restype = C.c_void_p
            L.ref_model_create_prec.argtypes = [C.c_char_p, C.POINTER(C.c_char_p), C.POINTER(C.c_double), C.c_int,
                                                C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32, C.c_int, C.c_int]
            L.ref_model_destroy.argtypes = [C.c_void_p]
            L.ref_fingerprint.restype = C.c_uint64
            L.ref_fingerprint.argtypes = [C.c_char_p, C.POINTER(C.c_char_p), C.POINTER(C.c_double), C.c_int]
            L.ref_model_state_bytes.restype = C.c_size_t
            L.ref_model_state_bytes.argtypes = [C.c_void_p]
            L.ref_model_save_state.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
            L.ref_model_load_state.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
            L.ref_model_init.argtypes = [C.c_void_p, C.c_int64, _f32p]
            L.ref_model_advance_runs.argtypes = [C.c_void_p, _u32p, C.c_size_t, _i64p, _f32p, C.c_size_t, _i64p,
                                                 _i32p, C.c_int64]
            L.ref_model_event_count.restype = C.c_size_t
            L.ref_model_event_count.argtypes = [C.c_void_p]
            L.ref_model_take_events.argtypes = [C.c_void_p, _u32p, _u8p, _u8p, _u16p, _i64p, _f32p, _f32p, _f32p,
                                                _f32p]
            L.ref_model_maps.argtypes = [C.c_void_p, _f64p, _f64p, _f64p, _f64p, _f64p]
            L.ref_model_threads.restype = C.c_int
            L.ref_model_threads.argtypes = [C.c_void_p]
            L.ref_model_irr_max.restype = C.c_float
            L.ref_model_irr_max.argtypes = [C.c_void_p]
            L.ref_model_set_photometry.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_size_t]
            L.ref_sample_window.restype = C.c_int64
            L.ref_sample_window.argtypes = [C.POINTER(OrcField), C.c_float, C.c_float, C.c_int, C.c_int, C.c_int,
                                            C.c_int64, C.c_int64, _u32p, _u8p, C.c_size_t, _f32p, _u64p, _i64p,
                                            _i64p, _f32p, C.c_size_t]
            L.ref_fixed_rate_window_cb.restype = C.c_int64
            L.ref_fixed_rate_window_cb.argtypes = [C.c_int, C.c_int64, C.c_int64, _u32p, C.c_size_t, _f32p, _u64p,
                                                   C.c_void_p, C.c_void_p, _i64p, _i64p, _f32p, C.c_size_t, _u64p]
            L.ref_event_file.restype = C.c_int
            L.ref_event_file.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int32, C.c_int32, C.c_int64, C.c_int64,
                                         C.c_int32, C.c_int32, C.c_char_p, _u16p, _u16p, _u8p, _i64p, _i64p, C.c_int,
                                         _i32p, C.c_char_p, C.c_size_t, _i64p, C.c_char_p]
            L.ref_sample_window_cb.restype = C.c_int64
            L.ref_sample_window_cb.argtypes = [C.c_int, C.c_float, C.c_float, _f64p, _f64p, C.c_int, C.c_int, C.c_int,
                                               C.c_int64, C.c_int64, _u32p, _u8p, C.c_size_t, _f32p, _u64p,
                                               C.c_void_p, C.c_void_p, _i64p, _i64p, _f32p, C.c_size_t, _u64p]
            L.ref_output_order.argtypes = [_i64p, _u16p, _u16p, _i64p, C.c_size_t, C.c_uint32, _u32p]
            L.ref_reported_time.restype = C.c_int64
            L.ref_reported_time.argtypes = [C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_int64]
            L.ref_output_cut.restype = C.c_int64
            L.ref_output_cut.argtypes = [C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_int64]
            L.ref_label_s1.restype = C.c_uint8
            L.ref_label_s1.argtypes = [C.c_uint8]
            L.ref_noise_table.restype = C.c_int64
            L.ref_noise_table.argtypes = [C.c_double] * 4 + [C.c_int, C.c_int, C.c_void_p, C.c_size_t]
            L.ref_special.restype = None
            L.ref_special.argtypes = [C.c_int, C.c_void_p, C.c_size_t, C.c_void_p]
            L.ref_readout_phase.restype = C.c_int64
            L.ref_readout_phase.argtypes = [C.c_uint64, C.c_uint32, C.c_int64]
            L.ref_simulate.restype = C.c_int64
            L.ref_simulate.argtypes = [C.c_void_p, C.POINTER(OrcField), C.c_float, C.c_float, C.c_int, C.c_int64,
                                       C.c_int32, C.c_int32, C.c_int64, C.c_int32, _f64p]
            cls._lib = L
        return cls._lib

    @classmethod
    def output_order(cls, t_cross, x, y, t_reported, height) -> np.ndarray:
        """The reference's output permutation of the event columns (output_order)."""
        n = len(t_cross)
        perm = np.zeros(n, np.uint32)
        cls.lib().ref_output_order(np.ascontiguousarray(t_cross, np.int64), np.ascontiguousarray(x, np.uint16),
                                   np.ascontiguousarray(y, np.uint16), np.ascontiguousarray(t_reported, np.int64), n,
                                   height, perm)
        return perm

    @classmethod
    def sample_window(cls, f, rules, t_w, pixel, level, carried_irr, carried_sig):
        s = field_struct(f)
        n = len(pixel)
        off = np.zeros(n + 1, np.int64)
        cap = max(16, int(np.sum((1 << level.astype(np.int64)) + 1)) * 4)
        while True:
            t = np.zeros(cap, np.int64)
            irr = np.zeros(cap, np.float32)
            ci, cs = carried_irr.copy(), carried_sig.copy()
            k = cls.lib().ref_sample_window(C.byref(s), rules.tol, rules.dark, 1, 1, rules.max_refine_levels,
                                            rules.min_dt_ns, t_w, np.ascontiguousarray(pixel, np.uint32),
                                            np.ascontiguousarray(level, np.uint8), n, ci, cs, off, t, irr, cap)
            if k == np.iinfo(np.int64).min:
                raise ValueError(cls.lib().ref_last_error().decode())
            if k >= 0:
                return t[:k], irr[:k], off, ci, cs
            cap = -k

    @classmethod
    def fixed_rate_window_cb(cls, render, groups, period_ns, t_w, pixel, carried_irr, carried_sig):
        """WindowEngine<kHost> on the fixed-rate grid with the Python callable as its renderer. Returns (t, irr (S,
        groups), offsets, last_irradiance, last_signature, stats)."""
        cb = cls.RENDER_FN(cls._callback(render, groups))
        n = len(pixel)
        cap = max(16, n * (int((1 << 23) // max(1, period_ns)) + 3))
        while True:
            off = np.zeros(n + 1, np.int64)
            t = np.zeros(cap, np.int64)
            irr = np.zeros(cap * groups, np.float32)
            ci = np.array(carried_irr, np.float32).reshape(n, groups).copy()
            cs = np.array(carried_sig, np.uint64).copy()
            st = np.zeros(37, np.uint64)
            k = cls.lib().ref_fixed_rate_window_cb(groups, period_ns, t_w, np.ascontiguousarray(pixel, np.uint32), n,
                                                   ci.reshape(-1), cs, C.cast(cb, C.c_void_p), None, off, t, irr, cap,
                                                   st)
            if k == np.iinfo(np.int64).min:
                raise ValueError(cls.lib().ref_last_error().decode())
            if k >= 0:
                stats = {"flagged_signature": int(st[0]), "flagged_midpoint": int(st[1]),
                         "refine_cap_hits": int(st[2]), "render_calls": int(st[3]),
                         "samples_by_round": [int(v) for v in st[5:5 + int(st[4])]]}
                return t[:k], irr[:k * groups].reshape(k, groups), off, ci, cs, stats
            cap = -k

    FILE_FORMATS = {"evt2": 0, "evt21": 1, "evt3": 2, "dat": 3}

    @classmethod
    def event_file(cls, path, format, width, height, origin_us, epoch_ns, x, y, p, t_ns, bounds=None,
                   evt2_time_high="openeb", t_ns_rem_min=0, t_ns_rem_max=0, version=""):
        """The reference's RawWriter / DatWriter (format "dat") fed the batches [bounds[k], bounds[k + 1]) (None: one
        batch). Returns (info {bytes, sha256, count, t_first, t_last}, per-batch refused flags, last refusal)."""
        n = len(t_ns)
        b = np.asarray([0, n] if bounds is None else bounds, np.int64)
        status = np.zeros(len(b) - 1, np.int32)
        msg = C.create_string_buffer(1024)
        info = np.zeros(4, np.int64)
        sha = C.create_string_buffer(65)
        rc = cls.lib().ref_event_file(str(path).encode(), cls.FILE_FORMATS[format],
                                      1 if evt2_time_high == "change" else 0, width, height, origin_us, epoch_ns,
                                      t_ns_rem_min, t_ns_rem_max, version.encode(),
                                      np.ascontiguousarray(x, np.uint16), np.ascontiguousarray(y, np.uint16),
                                      np.ascontiguousarray(p, np.uint8), np.ascontiguousarray(t_ns, np.int64), b,
                                      len(b) - 1, status, msg, 1024, info, sha)
        if rc != 0:
            raise ValueError(cls.lib().ref_last_error().decode())
        return ({"bytes": int(info[0]), "sha256": sha.value.decode(), "count": int(info[1]),
                 "t_first": int(info[2]), "t_last": int(info[3])}, status.astype(bool), msg.value.decode())

    RENDER_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_int64), C.c_size_t,
                            C.POINTER(C.c_float), C.POINTER(C.c_uint64))

    @staticmethod
    def _callback(render, groups):
        def fn(_user, px, tt, n, irr, sig):
            if n == 0:
                return 0
            e, s = render(np.ctypeslib.as_array(px, (n,)).copy(), np.ctypeslib.as_array(tt, (n,)).copy())
            np.ctypeslib.as_array(irr, (n * groups,))[:] = np.asarray(e, np.float32).reshape(-1)
            np.ctypeslib.as_array(sig, (n,))[:] = np.asarray(s, np.uint64).reshape(-1)
            return 0

        return fn

    @classmethod
    def sample_window_cb(cls, render, groups, midpoint, refine_signature, max_refine_levels, min_dt_ns, t_w, pixel,
                         level, carried_irr, carried_sig):
        """WindowEngine<kHost> with the Python callable render(pixel_ids, t_ns) -> (irradiance (n, groups),
        signature (n,)) as its renderer; midpoint: None or an object with tol, dark, m_min and m_max. Returns
        (t, irr (S, groups), offsets, last_irradiance, last_signature, stats)."""
        cb = cls.RENDER_FN(cls._callback(render, groups))
        n = len(pixel)
        mn = np.asarray(midpoint.m_min if midpoint else [1.0] * groups, np.float64)
        mx = np.asarray(midpoint.m_max if midpoint else [1.0] * groups, np.float64)
        cap = max(16, int(np.sum((1 << np.asarray(level, np.int64)) + 1)) * 4)
        while True:
            off = np.zeros(n + 1, np.int64)
            t = np.zeros(cap, np.int64)
            irr = np.zeros(cap * groups, np.float32)
            ci = np.array(carried_irr, np.float32).reshape(n, groups).copy()
            cs = np.array(carried_sig, np.uint64).copy()
            st = np.zeros(37, np.uint64)
            k = cls.lib().ref_sample_window_cb(groups, midpoint.tol if midpoint else 0.0,
                                               midpoint.dark if midpoint else 0.0, mn, mx, 1 if midpoint else 0,
                                               1 if refine_signature else 0, max_refine_levels, min_dt_ns, t_w,
                                               np.ascontiguousarray(pixel, np.uint32),
                                               np.ascontiguousarray(level, np.uint8), n, ci.reshape(-1), cs,
                                               C.cast(cb, C.c_void_p), None, off, t, irr, cap, st)
            if k == np.iinfo(np.int64).min:
                raise ValueError(cls.lib().ref_last_error().decode())
            if k >= 0:
                stats = {"flagged_signature": int(st[0]), "flagged_midpoint": int(st[1]),
                         "refine_cap_hits": int(st[2]), "render_calls": int(st[3]),
                         "samples_by_round": [int(v) for v in st[5:5 + int(st[4])]]}
                return t[:k], irr[:k * groups].reshape(k, groups), off, ci, cs, stats
            cap = -k

    @classmethod
    def fingerprint(cls, family: str, overrides: dict) -> int:
        """The reference's fingerprint of preset(family) with numeric overrides (harness field names)."""
        keys = list(overrides)
        ck = (C.c_char_p * max(1, len(keys)))(*[k.encode() for k in keys])
        cv = (C.c_double * max(1, len(keys)))(*[float(overrides[k]) for k in keys])
        h = cls.lib().ref_fingerprint(family.encode(), ck, cv, len(keys))
        if h == 0:
            raise ValueError(cls.lib().ref_last_error().decode())
        return int(h)

    class Model:
        # Overrides the harness understands (the SensorParams rows this path reads), from a resolved SensorParams.
        KEYS = ("theta_on", "theta_off", "sigma_theta_on", "sigma_theta_off", "theta_onoff_corr", "theta_floor",
                "refractory_s", "eps_ci", "leak_rate_hz", "leak_sigma_log10", "dark_current_fA", "dark_sigma_ln",
                "illuminance_scale", "label_share_cut", "readout_quantum_s", "readout_delay_s", "k", "tau_o", "tau_sf",
                "eps_L", "sigma_o", "noise_leaf_level", "noise_margin_z", "stationary_burnin_ns",
                "stationary_probe_pixels")

        def __init__(self, params, width, height, seed, camera=0, num_threads=0, fp64=False):
            self.L = Ref.lib()
            self.width, self.height = width, height
            v = params.as_dict()
            keys = list(self.KEYS) + ["reset_mode", "initial_phase", "photoreceptor", "noise", "initial_state",
                                      "noise_diffusion"]
            vals = [float(v[k]) for k in self.KEYS] + [1.0 if v["reset_mode"] == "ideal" else 0.0,
                                                        {"uniform": 0.0, "symmetric": 1.0, "zero": 2.0}[
                                                            v["initial_phase"]],
                                                        0.0 if v["photoreceptor"] == "cascade" else 1.0,
                                                        1.0 if v["noise"] else 0.0,
                                                        1.0 if v["initial_state"] == "stationary" else 0.0,
                                                        1.0 if v["noise_diffusion"] == "transient" else 0.0]
            ck = (C.c_char_p * len(keys))(*[k.encode() for k in keys])
            cv = (C.c_double * len(vals))(*vals)
            self.h = self.L.ref_model_create_prec(v["family"].encode(), ck, cv, len(keys), width, height, seed,
                                                  camera, num_threads, 1 if fp64 else 0)
            if not self.h:
                raise ValueError(self.L.ref_last_error().decode())

        def __del__(self):
            if getattr(self, "h", None):
                self.L.ref_model_destroy(self.h)
                self.h = None

        def save_state(self) -> bytes:
            n = self.L.ref_model_state_bytes(self.h)
            buf = np.zeros(n, np.uint8)
            if self.L.ref_model_save_state(self.h, buf.ctypes.data, n) != 0:
                raise ValueError(self.L.ref_last_error().decode())
            return buf.tobytes()

        def load_state(self, blob: bytes) -> None:
            b = np.frombuffer(blob, np.uint8)
            if self.L.ref_model_load_state(self.h, b.ctypes.data, len(b)) != 0:
                raise ValueError(self.L.ref_last_error().decode())

        @property
        def threads(self) -> int:
            return self.L.ref_model_threads(self.h)

        @property
        def irr_max(self) -> float:
            return self.L.ref_model_irr_max(self.h)

        def set_photometry(self, scale, gain=None):
            g = None if gain is None else np.ascontiguousarray(gain, np.float32).reshape(-1)
            if self.L.ref_model_set_photometry(self.h, float(scale), None if g is None else g.ctypes.data,
                                               0 if g is None else g.size) != 0:
                raise ValueError(self.L.ref_last_error().decode())

        def init(self, t0, irr0):
            if self.L.ref_model_init(self.h, t0, np.ascontiguousarray(irr0, np.float32)) != 0:
                raise ValueError(self.L.ref_last_error().decode())

        def advance_runs(self, ids, t, irr, row_start, row_count, t_end):
            rc = self.L.ref_model_advance_runs(self.h, np.ascontiguousarray(ids, np.uint32), len(ids),
                                               np.ascontiguousarray(t, np.int64),
                                               np.ascontiguousarray(irr, np.float32), len(t),
                                               np.ascontiguousarray(row_start, np.int64),
                                               np.ascontiguousarray(row_count, np.int32), t_end)
            if rc != 0:
                raise ValueError(self.L.ref_last_error().decode())

        def take_events(self) -> dict:
            n = self.L.ref_model_event_count(self.h)
            rec = np.zeros(n, EVENT_DTYPE)
            cols = [np.zeros(n, t) for t in (np.uint32, np.uint8, np.uint8, np.uint16, np.int64, np.float32,
                                             np.float32, np.float32, np.float32)]
            self.L.ref_model_take_events(self.h, *cols)
            for name, col in zip(EVENT_DTYPE.names, cols):
                rec[name] = col
            return _events_from_records(rec, self.width)

        def maps(self) -> dict:
            n = self.width * self.height
            a = [np.zeros(n) for _ in range(5)]
            self.L.ref_model_maps(self.h, *a)
            return dict(zip(("theta_on", "theta_off", "leak", "dark_current_fA", "phi0"), a))

        def simulate(self, f, rules, windows, t0=0):
            """The reference chain end to end (ref_simulate): (events dict, stats dict)."""
            s = field_struct(f)
            st = np.zeros(4)
            n = self.L.ref_simulate(self.h, C.byref(s), rules.tol, rules.dark, rules.max_refine_levels,
                                    rules.min_dt_ns, rules.l_min, rules.l_max, t0, windows, st)
            if n < 0:
                raise ValueError(self.L.ref_last_error().decode())
            return self.take_events(), {"pixel_samples": int(st[0]), "sampler_s": st[1], "sensor_s": st[2],
                                        "windows": int(st[3])}


def simulate_port(spec, rules, windows, t0=0, params=None):
    """The oracle port's chain for one sensor: init from the field, then per window the sampler (levels by the
    field's rule) and the pixel model. Returns (events, stats)."""
    from ballasim_b200.params import resolve

    p = params if params is not None else resolve(spec.preset, spec.overrides)
    f = spec.field
    np_ = spec.width * spec.height
    m = Port.Model(p, spec.width, spec.height, spec.seed, spec.camera)
    frame = Port.field_frame(f, t0)
    m.init(t0, frame)
    ids = np.arange(np_, dtype=np.uint32)
    carried = frame.copy()
    sig = np.zeros(np_, np.uint64)
    samples = 0
    for w in range(windows):
        t_w = t0 + w * (1 << 23)
        lv = Port.levels(f, t_w, rules.l_min, rules.l_max)
        t, irr, off, carried, sig = Port.sample_window(f, rules, t_w, ids, lv, carried, sig)
        m.advance_runs(ids, t, irr, off[:-1], np.diff(off).astype(np.int32), t_w + (1 << 23))
        samples += len(t)
    return m.take_events(), {"pixel_samples": samples}
