"""SensorParams and its presets, with the names, units and rules of ``ballasim._sensor.SensorParams``
(src/sensor/params.h:65-176, src/sensor/param_fields.cpp:40-362 for the rows, :364-512 for the families).

The family priors are configuration data that a drop-in must reproduce value for value (the same preset must
mean the same sensor); they are listed here as data. This path runs the instantaneous log response
(``photoreceptor = "instantaneous"``) with constant light groups, and the cascade photoreceptor with or without its
noise lattice (``photoreceptor = "cascade"``; the lattice with frozen diffusion).

Three rows are this project's own (no reference counterpart, off unless set): ``noise_shot_rate_hz`` (shot-noise
event rate at a photocurrent of 100 fA; the rate scales as 1/sqrt(I)), ``noise_ba_median_hz`` and
``noise_ba_sigma_ln`` (the per-pixel background-activity rate, log-normal).
"""
from __future__ import annotations

import math
import struct

NAN = float("nan")

# Row name -> (default kind, literal default). "family" rows take the family prior.
_ROWS = [
    ("family", "required", ""),
    ("photoreceptor", "family", None),
    ("k", "family", None),
    ("tau_o", "family", None),
    ("tau_sf", "family", None),
    ("sigma_o", "family", None),
    ("noise", "family", None),
    ("illuminance_scale", "required", NAN),
    ("veiling_glare", "literal", 0.0),
    ("dark_current_fA", "family", None),
    ("dark_sigma_ln", "family", None),
    ("dark_ea_eV", "family", None),
    ("temperature_K", "family", None),
    ("reference_temperature_K", "family", None),
    ("theta_on", "family", None),
    ("theta_off", "family", None),
    ("sigma_theta_on", "family", None),
    ("sigma_theta_off", "family", None),
    ("theta_onoff_corr", "family", None),
    ("theta_floor", "family", None),
    ("reset_mode", "family", None),
    ("refractory_s", "family", None),
    ("eps_ci", "family", None),
    ("initial_phase", "family", None),
    ("leak_rate_hz", "family", None),
    ("leak_sigma_log10", "family", None),
    ("leak_ea_eV", "family", None),
    ("tau_hp", "family", None),
    ("tau_hp_sigma_ln", "literal", 0.0),
    ("hot_fraction", "family", None),
    ("hot_rate_law", "family", None),
    ("hot_rate_min_hz", "family", None),
    ("hot_rate_max_hz", "family", None),
    ("hot_rate_median_hz", "family", None),
    ("hot_rate_sigma_ln", "family", None),
    ("hot_leak_fraction", "family", None),
    ("hot_reference_current_fA", "family", None),
    ("readout_quantum_s", "family", None),
    ("readout_delay_s", "family", None),
    ("clock_offset_ns", "literal", 0),
    ("clock_drift_ppm", "family", None),
    ("limiter", "family", None),
    ("limiter_rate0_hz", "family", None),
    ("limiter_rate1_hz", "family", None),
    ("limiter_period_s", "family", None),
    ("limiter_depth", "family", None),
    ("limiter_phase_s", "literal", None),
    ("eps_L", "literal", 0.002),
    ("noise_leaf_level", "literal", 5),
    ("noise_margin_z", "literal", 6.0),
    ("noise_diffusion", "literal", "frozen"),
    ("initial_state", "literal", "phase"),
    ("stationary_burnin_ns", "literal", 0),
    ("stationary_probe_pixels", "literal", 32),
    ("label_share_cut", "literal", 0.5),
    # this project's noise rows (no reference counterpart)
    ("noise_shot_rate_hz", "literal", 0.0),
    ("noise_ba_median_hz", "literal", 0.0),
    ("noise_ba_sigma_ln", "literal", 0.0),
]
ROW_NAMES = [r[0] for r in _ROWS]

_PROPHESEE = {
    "photoreceptor": "cascade", "k": 1.0e16, "tau_o": 25e-6, "tau_sf": 100e-6, "sigma_o": 0.06, "noise": True,
    "dark_current_fA": 0.21, "dark_sigma_ln": 0.3, "dark_ea_eV": 0.78, "temperature_K": 298.15,
    "reference_temperature_K": 298.15, "theta_on": 0.25, "theta_off": 0.25, "sigma_theta_on": 0.03,
    "sigma_theta_off": 0.03, "theta_onoff_corr": 0.0, "theta_floor": 0.01, "reset_mode": "physical",
    "refractory_s": 0.3e-3, "eps_ci": 0.0, "initial_phase": "uniform", "leak_rate_hz": 0.01,
    "leak_sigma_log10": 0.1, "leak_ea_eV": 0.78, "tau_hp": 0.0, "hot_fraction": 0.0, "hot_rate_law": "log_uniform",
    "hot_rate_min_hz": 10.0, "hot_rate_max_hz": 2000.0, "hot_rate_median_hz": 100.0, "hot_rate_sigma_ln": 1.5,
    "hot_leak_fraction": 0.5, "hot_reference_current_fA": 100.0, "readout_quantum_s": 1e-6,
    "readout_delay_s": 300e-6, "clock_drift_ppm": 0.0, "limiter": "off", "limiter_rate0_hz": 6.0e6,
    "limiter_rate1_hz": 6.0e6, "limiter_period_s": 65.6e-3, "limiter_depth": 32,
}
_SAMSUNG = {**_PROPHESEE, "theta_on": 0.20, "theta_off": 0.20, "refractory_s": 196e-6, "readout_delay_s": 100e-6,
            "leak_rate_hz": 0.01, "dark_current_fA": 0.08, "tau_hp": 0.0, "limiter": "off"}
_IDEAL = {**_PROPHESEE, "photoreceptor": "instantaneous", "k": 1.0e18, "tau_o": 1e-6, "tau_sf": 2e-6,
          "noise": False, "dark_current_fA": 0.01, "dark_sigma_ln": 0.0, "theta_on": 0.20, "theta_off": 0.20,
          "sigma_theta_on": 0.0, "sigma_theta_off": 0.0, "reset_mode": "ideal", "refractory_s": 0.0,
          "leak_rate_hz": 0.0, "leak_sigma_log10": 0.0, "tau_hp": 0.0, "hot_fraction": 0.0,
          "readout_quantum_s": 0.0, "readout_delay_s": 0.0, "limiter": "off"}
FAMILIES = {"prophesee_gen3": _PROPHESEE, "samsung_gen3": _SAMSUNG, "ideal": _IDEAL}

ENUMS = {
    "photoreceptor": ("cascade", "instantaneous"),
    "reset_mode": ("physical", "ideal"),
    "initial_phase": ("uniform", "symmetric", "zero"),
    "hot_rate_law": ("log_uniform", "log_normal"),
    "limiter": ("off", "epoch"),
    "noise_diffusion": ("frozen", "transient"),
    "initial_state": ("phase", "stationary"),
}


def preset_names() -> list[str]:
    """Names of the built-in presets (src/sensor/param_fields.cpp:487-514)."""
    return list(FAMILIES)


class SensorParams:
    """Sensor parameters in SI units; one attribute per parameter row. ``SensorParams()`` carries no prior
    (validate() refuses it); ``SensorParams.preset(name)`` fills every row from the family."""

    __slots__ = ("_v",)

    def __init__(self):
        v = {}
        for name, kind, lit in _ROWS:
            v[name] = lit if kind != "family" else NAN
        object.__setattr__(self, "_v", v)

    @staticmethod
    def preset(name: str) -> "SensorParams":
        if name not in FAMILIES:
            raise ValueError(f"unknown sensor preset '{name}' (known: {', '.join(FAMILIES)})")
        p = SensorParams()
        for k, val in FAMILIES[name].items():
            p._v[k] = val
        p._v["family"] = name
        p._v["illuminance_scale"] = 1.0  # the low-level API's neutral scale (src/sensor/params.cpp:126)
        p._v["clock_offset_ns"] = 0
        return p

    def __getattr__(self, name):
        v = object.__getattribute__(self, "_v")
        if name in v:
            return v[name]
        raise AttributeError(f"SensorParams has no field '{name}'")

    def __setattr__(self, name, value):
        if name not in self._v:
            raise AttributeError(f"SensorParams has no field '{name}'")
        if name in ENUMS and value not in ENUMS[name]:
            raise ValueError(f"SensorParams.{name}: one of {', '.join(ENUMS[name])}")
        self._v[name] = value

    def copy(self) -> "SensorParams":
        p = SensorParams()
        p._v.update(self._v)
        return p

    def as_dict(self) -> dict:
        return dict(self._v)

    def validate(self) -> None:
        """The rows' ranges and the cross-key rules (src/sensor/params.cpp:36-98); ValueError naming the field."""
        v = self._v
        if v["family"] not in FAMILIES:
            raise ValueError(f"SensorParams: family = '{v['family']}': one of {', '.join(FAMILIES)}")

        def need(ok, msg):
            if not ok:
                raise ValueError("SensorParams: " + msg)

        for name, kind, _ in _ROWS:
            x = v[name]
            if isinstance(x, float) and name != "limiter_phase_s":
                need(math.isfinite(x), f"{name} must be finite")
        for name in ("k", "tau_o", "tau_sf", "illuminance_scale", "dark_current_fA", "temperature_K",
                     "reference_temperature_K", "theta_on", "theta_off", "theta_floor", "hot_rate_min_hz",
                     "hot_rate_max_hz", "hot_rate_median_hz", "hot_reference_current_fA"):
            need(v[name] > 0, f"{name} must be > 0")
        for name in ("sigma_o", "dark_sigma_ln", "dark_ea_eV", "sigma_theta_on", "sigma_theta_off",
                     "leak_rate_hz", "leak_sigma_log10", "leak_ea_eV", "tau_hp_sigma_ln", "hot_rate_sigma_ln",
                     "noise_shot_rate_hz", "noise_ba_median_hz", "noise_ba_sigma_ln"):
            need(v[name] >= 0, f"{name} must be >= 0")
        need(-1 <= v["theta_onoff_corr"] <= 1, "theta_onoff_corr must lie in [-1, 1]")
        need(0 <= v["refractory_s"] < 10, "refractory_s must lie in [0, 10)")
        need(0 <= v["hot_fraction"] <= 1, "hot_fraction must lie in [0, 1]")
        need(0 <= v["readout_quantum_s"] < 1, "readout_quantum_s must lie in [0, 1)")
        need(0 <= v["readout_delay_s"] < 1, "readout_delay_s must lie in [0, 1)")
        need(0 < v["label_share_cut"] < 1, "label_share_cut must lie in (0, 1)")
        need(0 <= v["veiling_glare"] < 1, "veiling_glare must lie in [0, 1)")
        need(max(v["tau_o"], v["tau_sf"]) >= 1.1 * min(v["tau_o"], v["tau_sf"]),
             "tau_sf and tau_o must differ by at least 10 % (the larger >= 1.1 x the smaller)")
        need(v["theta_on"] > v["theta_floor"], "theta_on must exceed theta_floor")
        need(v["theta_off"] > v["theta_floor"], "theta_off must exceed theta_floor")
        need(abs(v["eps_ci"]) < 0.5 * v["theta_floor"], "|eps_ci| must be < theta_floor / 2")
        need(v["hot_rate_max_hz"] >= v["hot_rate_min_hz"],
             "hot rates must satisfy 0 < hot_rate_min_hz <= hot_rate_max_hz")
        need(v["hot_fraction"] == 0 or v["hot_rate_max_hz"] * v["refractory_s"] < 1.0,
             "hot_rate_max_hz must be < 1 / refractory_s")
        need(v["readout_quantum_s"] == 0 or v["readout_delay_s"] >= v["readout_quantum_s"],
             "readout_delay_s must be >= readout_quantum_s when quantization is on")
        if v["tau_hp"] > 0:
            need(v["photoreceptor"] == "cascade",
                 "tau_hp > 0 needs photoreceptor cascade (the instantaneous response has no filtered reference)")

    def noise_on(self) -> bool:
        """This project's shot / background-activity noise is on (either rate > 0)."""
        return self._v["noise_shot_rate_hz"] > 0 or self._v["noise_ba_median_hz"] > 0

    def __repr__(self) -> str:
        return f"SensorParams(family={self._v['family']!r}, photoreceptor={self._v['photoreceptor']!r})"


# The Value alternative of each row as the reference's row table yields it (config::Value, src/core/config/param.h:44:
# null, bool, int64, double, string, ...): the family and the enums as their choice names, these rows as int64, the
# noise switch as bool, every other row as double (limiter_phase_s: null while unset).
_INT_ROWS = {"clock_offset_ns", "limiter_depth", "noise_leaf_level", "stationary_burnin_ns", "stationary_probe_pixels"}
_STRING_ROWS = {"family", *ENUMS}
_OWN_ROWS = ("noise_shot_rate_hz", "noise_ba_median_hz", "noise_ba_sigma_ln")
_FNV_OFFSET, _FNV_PRIME, _MASK = 0xCBF29CE484222325, 0x100000001B3, (1 << 64) - 1


def _fnv(h: int, data: bytes) -> int:
    for b in data:
        h = ((h ^ b) * _FNV_PRIME) & _MASK
    return h


def fingerprint(p: SensorParams) -> int:
    """The reference's 64-bit fingerprint of the parameters and one constant light group (fingerprint,
    src/sensor/params.cpp:214-263: FNV-1a over every row in row order, each as its Value index (a size_t) and its
    value's bytes, a string as its length and characters; the high-pass filter's rows only while tau_hp > 0, the
    limiter's only while it is on; then the waveform's fields, all zero for a constant group). It goes with saved
    states, which load only into a model of the same fingerprint. This project's own noise rows follow, as doubles,
    only while one of them is not zero, so that a sensor without them has the reference's fingerprint."""
    v = p.as_dict()
    h = _FNV_OFFSET
    for name in ROW_NAMES:
        if name in _OWN_ROWS:
            continue
        if v["tau_hp"] <= 0 and name in ("tau_hp", "tau_hp_sigma_ln"):
            continue
        if v["limiter"] == "off" and name.startswith("limiter"):
            continue
        x = v[name]
        if x is None:
            h = _fnv(h, struct.pack("<Q", 0))
        elif name in _STRING_ROWS:
            b = str(x).encode()
            h = _fnv(h, struct.pack("<QQ", 4, len(b)) + b)
        elif name == "noise":
            h = _fnv(h, struct.pack("<Q?", 1, bool(x)))
        elif name in _INT_ROWS:
            h = _fnv(h, struct.pack("<Qq", 2, int(x)))
        else:
            h = _fnv(h, struct.pack("<Qd", 3, float(x)))
    h = _fnv(h, bytes(4 + 4 + 8 + 2 * 8 * 8 + 6 * 8))  # the constant waveform: type, n_harmonics, f0, a/phi, pulse
    if any(v[name] != 0 for name in _OWN_ROWS):
        for name in _OWN_ROWS:
            h = _fnv(h, struct.pack("<Qd", 3, float(v[name])))
    return h


def resolve(params, overrides: dict | None = None) -> SensorParams:
    """A preset name or SensorParams, with field overrides, validated (sensor_module.cpp:54-68)."""
    p = SensorParams.preset(params) if isinstance(params, str) else params.copy()
    for k, val in (overrides or {}).items():
        setattr(p, k, val)
    p.validate()
    return p
