"""The synthetic workloads of this path's benchmark and parity tests, by their sizes.

Each workload is one or more sensors, each with a seeded analytic field (fields.py), the sensor parameters as
overrides of BallaSim's ``ideal`` preset (the instantaneous log response, src/sensor/param_fields.cpp:487-512),
and the sampler rules. Times are whole windows of W = 2^23 ns from t0 = 0: the sampler samples whole windows
(src/engine/sampling.h:344-350), so a duration D runs ceil(D / W) windows (1.0 s is 120 windows, 1.0066 s).

Sampler rules throughout: tolerance 0.01 as MidpointTest(0.01, dark = I_dk / scale = 0.01, [1], [1]), signature
refinement on (analytic signatures are 0), min_dt_ns = 8192 (10 us rounded down to the power of two the sampler
requires, src/engine/bindings/engine_module.cpp:317-319), lattice levels 1..10 (a level-1 lattice spaces
samples 4.19 ms apart, under the 10 ms maximum step; level 0 cannot refine), max_refine_levels = 10.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

from . import fields as F

WINDOW_NS = 1 << 23


@dataclass
class SensorSpec:
    width: int
    height: int
    seed: int
    camera: int
    overrides: dict  # of the preset below
    field: F.Field
    preset: str = "ideal"


@dataclass
class Rules:
    tol: float = 0.01
    dark: float = 0.01
    min_dt_ns: int = 8192
    max_refine_levels: int = 10
    l_min: int = 1
    l_max: int = 10


@dataclass
class Workload:
    name: str
    sensors: list
    windows: int
    rules: Rules = field(default_factory=Rules)

    @property
    def pixels(self) -> int:
        return sum(s.width * s.height for s in self.sensors)

    def describe(self) -> dict:
        return {"workload": self.name, "sensors": [f"{s.width}x{s.height}" for s in self.sensors],
                "pixels": self.pixels, "windows": self.windows,
                "sim_seconds": round(self.windows * WINDOW_NS * 1e-9, 6)}


def windows_for(seconds: float) -> int:
    return int(math.ceil(seconds * 1e9 / WINDOW_NS - 1e-9))


# Sensor parameters (overrides of preset "ideal").
IDEAL = {}
MISMATCH = {"theta_on": 0.25, "theta_off": 0.2, "sigma_theta_on": 0.03, "sigma_theta_off": 0.03,
            "reset_mode": "physical", "refractory_s": 1e-4}
NOISE = {"leak_rate_hz": 0.1, "leak_sigma_log10": 0.0, "noise_shot_rate_hz": 0.5, "noise_ba_median_hz": 0.05,
         "noise_ba_sigma_ln": 1.0}


def edge_64x48(seconds: float = 1.0, seed: int = 3) -> Workload:
    """64x48 px, a tanh edge, preset ideal (theta 0.2, no mismatch, ideal reset, refractory 0), noise off. The
    default seed is one whose edge crosses the array within the run (most seeds' edges miss a 64 x 48 array)."""
    f = F.tanh_edge(64, 48, seed)
    return Workload("edge_64x48", [SensorSpec(64, 48, seed, 0, dict(IDEAL), f)], windows_for(seconds))


def blobs_346x260(seconds: float = 2.0, seed: int = 2) -> Workload:
    """346x260 px, 16 blobs, theta 0.25/0.2 with mismatch 0.03, physical reset, refractory 100 us, noise off."""
    f = F.blobs(346, 260, seed, 16)
    return Workload("blobs16_346x260", [SensorSpec(346, 260, seed, 0, dict(MISMATCH), f)], windows_for(seconds))


def blobs_346x260_cascade(seconds: float = 2.0, seed: int = 2) -> Workload:
    """blobs_346x260's field and comparator laws (theta 0.25/0.2 with mismatch 0.03, physical reset, refractory
    100 us) with the cascade photoreceptor of preset prophesee_gen3 (k 1e16 A^-1 s^-1, tau_o 25 us, tau_sf 100 us,
    eps_L 0.002, dark current 0.21 fA), its noise lattice off."""
    f = F.blobs(346, 260, seed, 16)
    return Workload("blobs16_346x260_cascade",
                    [SensorSpec(346, 260, seed, 0, {**MISMATCH, "noise": False}, f, "prophesee_gen3")],
                    windows_for(seconds))


def blobs_346x260_lattice(seconds: float = 2.0, seed: int = 2) -> Workload:
    """blobs_346x260_cascade with the cascade's in-path noise lattice on (preset prophesee_gen3's full model: sigma_o
    0.06, leaf level 5, margin z 6, frozen diffusion)."""
    f = F.blobs(346, 260, seed, 16)
    return Workload("blobs16_346x260_lattice",
                    [SensorSpec(346, 260, seed, 0, {**MISMATCH, "noise": True}, f, "prophesee_gen3")],
                    windows_for(seconds))


def blobs_1280x720(seconds: float = 1.0, seed: int = 3) -> Workload:
    """1280x720 px, 256 blobs, the mismatch sensor with leak 0.1 Hz, shot and background-activity noise."""
    f = F.blobs(1280, 720, seed, 256)
    return Workload("blobs256_1280x720_noise", [SensorSpec(1280, 720, seed, 0, {**MISMATCH, **NOISE}, f)],
                    windows_for(seconds))


def six_sensors(seconds: float = 0.5, seed: int = 4) -> Workload:
    """Six sensors (346x260, 640x480 x2, 1280x720 x2, 1920x1080), 128 blobs each, theta_on = theta_off drawn
    U[0.15, 0.3] per sensor, mismatch 0.03, noise as blobs_1280x720."""
    g = F.SplitMix64(seed)
    sizes = [(346, 260), (640, 480), (640, 480), (1280, 720), (1280, 720), (1920, 1080)]
    out = []
    for cam, (w, h) in enumerate(sizes):
        th = float(f"{0.15 + 0.15 * g.uniform():.6f}")
        s = seed * 100 + cam
        ov = {**MISMATCH, **NOISE, "theta_on": th, "theta_off": th}
        out.append(SensorSpec(w, h, s, cam, ov, F.blobs(w, h, s, 128)))
    return Workload("six_sensors_4.6Mpx", out, windows_for(seconds))


def small(kind: str, width: int, height: int, windows: int, seed: int = 7) -> Workload:
    """A reduced case of the same laws for parity tests the CPU oracle finishes in seconds."""
    if kind == "edge":
        return Workload(f"edge_{width}x{height}", [SensorSpec(width, height, seed, 0, dict(IDEAL),
                                                              F.tanh_edge(width, height, seed))], windows)
    n = 16 if kind == "blobs" else 32
    ov = dict(MISMATCH) if kind == "blobs" else {**MISMATCH, **NOISE}
    return Workload(f"{kind}_{width}x{height}", [SensorSpec(width, height, seed, 0, ov,
                                                            F.blobs(width, height, seed, n))], windows)


def blobs_noise(width: int, height: int, seed: int, seconds: float = 1.0) -> Workload:
    """blobs_1280x720's laws (the mismatch sensor, leak, shot and background-activity noise) at another frame size,
    with the same blob density (256 blobs per 1280 x 720 px). The learned step proposal trains on such fields with
    training seeds and is evaluated on a held-out seed."""
    n = max(1, round(256 * width * height / (1280 * 720)))
    f = F.blobs(width, height, seed, n)
    return Workload(f"blobs{n}_{width}x{height}_noise", [SensorSpec(width, height, seed, 0, {**MISMATCH, **NOISE}, f)],
                    windows_for(seconds))


# Seeds of the learned proposal's training fields and its held-out evaluation field.
LEARN_TRAIN_SEEDS = (1001, 1002, 1003, 1004)
LEARN_EVAL_SEED = 2077


@dataclass
class EventStream:
    """A camera's events in output order for the event file sink: x, y (uint16), p (uint8) and t_ns (int64, the
    sub-microsecond part 0), with their sizes."""
    name: str
    width: int
    height: int
    x: object
    y: object
    p: object
    t_ns: object

    def describe(self) -> dict:
        n = len(self.t_ns)
        span_us = int(self.t_ns[-1] - self.t_ns[0]) // 1000 if n else 0
        return {"workload": self.name, "sensor": f"{self.width}x{self.height}", "events": n,
                "span_us": span_us, "column_bytes": 13 * n}


def event_stream(n: int = 32 << 20, width: int = 1280, height: int = 720, rate_hz: float = 50e6,
                 seed: int = 5) -> EventStream:
    """n events of a 1280 x 720 camera at about rate_hz, as edges make them: runs of 1 + Geometric(1/4) neighbouring
    pixels of one row at one microsecond (the runs' times uniform over n / rate_hz), in the output order (t, then
    y, then x); polarities by run."""
    import numpy as np

    rng = np.random.default_rng(seed)
    runs = []
    total = 0
    span_us = max(1, int(n / rate_hz * 1e6))
    while total < n:
        m = (n - total) // 4 + 16
        length = rng.geometric(0.25, m)
        u = rng.integers(0, span_us, m)
        y = rng.integers(0, height, m)
        x0 = rng.integers(0, width, m)
        p = rng.integers(0, 2, m)
        runs.append((length, u, y, x0, p))
        total += int(length.sum())
    length, u, y, x0, p = (np.concatenate(c) for c in zip(*runs))
    rep = np.repeat(np.arange(len(length)), length)
    off = np.arange(len(rep)) - np.repeat(np.cumsum(length) - length, length)
    xs = np.minimum(x0[rep] + off, width - 1)
    # One sort of the packed key (t, y, x, p) gives the output order; the first n are kept.
    key = np.sort((u[rep] << 23) | (y[rep] << 12) | (xs << 1) | p[rep])[:n]
    return EventStream(f"events{n >> 20}M_{width}x{height}", width, height, ((key >> 1) & 2047).astype(np.uint16),
                       ((key >> 12) & 2047).astype(np.uint16), (key & 1).astype(np.uint8),
                       1000 * (key >> 23))
