"""Statistics of the shot and background-activity noise (this build's own law; no reference counterpart).

A static scene (every pixel holds its init irradiance, no leak, physical reset without refractory) fires noise
events only. Pixel p's noise is then a Poisson process of rate Lambda_p = r sqrt(100 fA / I_p) + b_p (shot at its
photocurrent I_p, background activity at its drawn rate b_p), so that:
- the inter-event intervals dt after an event (or the start) at t, mapped through
  (1 - exp(-Lambda_p dt)) / (1 - exp(-Lambda_p (T - t))) (the law of an interval seen to end before T), are
  uniform: KS test, p > 0.01;
- the drawn rates b_p are log-normal (median, sigma): KS test of ln b_p against the normal law, p > 0.01;
- the event count over all pixels matches sum(Lambda_p) T within 4 sigma, and ON / OFF are balanced within 4 sigma.
The CPU test checks the oracle's restatement of the law; the GPU test the CUDA path (which the parity tests
show to be bit-identical to it) at a larger size."""
import math

import numpy as np
import pytest
from scipy import stats

from ballasim_b200.params import resolve

SHOT_R, BA_MEDIAN, BA_SIGMA = 2.0, 20.0, 1.0
OVERRIDES = {"reset_mode": "physical", "refractory_s": 0.0, "noise_shot_rate_hz": SHOT_R,
             "noise_ba_median_hz": BA_MEDIAN, "noise_ba_sigma_ln": BA_SIGMA}


def frame(n: int) -> np.ndarray:
    """Irradiance log-spaced over 1 .. 1000 (renderer units = fA at scale 1)."""
    return np.exp(np.linspace(0.0, math.log(1000.0), n)).astype(np.float32)


def check(events: dict, irr0: np.ndarray, ba: np.ndarray, dark: float, T_ns: int, n: int) -> None:
    assert np.all(events["label"] == 1), "a static scene fires noise events only"
    I = (dark + irr0.astype(np.float32)).astype(np.float64)  # photocurrent dark + scale v, scale 1
    lam = SHOT_R * np.sqrt(100.0 / I) + ba
    px = events["pixel"].astype(np.int64)
    t = events["t_cross_ns"].astype(np.int64)
    order = np.lexsort((t, px))
    px, t = px[order], t[order]
    first = np.r_[True, px[1:] != px[:-1]]
    prev = np.where(first, 0, np.r_[0, t[:-1]])
    dt = (t - prev) * 1e-9
    # An interval is only seen when it ends before T: conditioned on that, F(dt) / F(T - prev) is uniform.
    u = -np.expm1(-lam[px] * dt) / -np.expm1(-lam[px] * (T_ns - prev) * 1e-9)
    assert stats.kstest(u, "uniform").pvalue > 0.01
    total, want = len(t), lam.sum() * T_ns * 1e-9
    assert abs(total - want) < 4.0 * math.sqrt(want), (total, want)
    on = int(np.count_nonzero(events["p"] == 1))
    assert abs(on - total / 2) < 4.0 * math.sqrt(total / 4)
    z = (np.log(ba) - math.log(BA_MEDIAN)) / BA_SIGMA
    assert stats.kstest(z, "norm").pvalue > 0.01
    assert len(np.unique(px)) > 0.9 * n


def test_noise_law_in_the_oracle(oracle_port):
    p = resolve("ideal", OVERRIDES)
    w, h = 24, 16
    n = w * h
    irr0 = frame(n)
    m = oracle_port.Model(p, w, h, 21, 0)
    m.init(0, irr0)
    z = np.zeros(0, np.int64)
    T = 40 << 23
    for k in range(1, 41):
        m.advance_runs(np.zeros(0, np.uint32), z, np.zeros(0, np.float32), z, np.zeros(0, np.int32), k << 23)
    check(m.take_events(), irr0, m.ba_rates(), p.dark_current_fA, T, n)


@pytest.mark.gpu
def test_noise_law_on_the_device(cuda_lib):
    from ballasim_b200.sensor import SensorModel

    p = resolve("ideal", OVERRIDES)
    w, h = 128, 96
    n = w * h
    irr0 = frame(n)
    m = SensorModel(p, w, h, 33, [{"type": "constant"}], 0)
    m.init(0, irr0.reshape(n, 1))
    z = np.zeros(0, np.int64)
    parts = []
    T = 120 << 23
    for k in range(1, 121):
        ev = m.advance(np.zeros(0, np.uint32), z, np.zeros((0, 1), np.float32), k << 23,
                       offsets=np.zeros(1, np.int64))
        ev["pixel"] = ev["y"].astype(np.int64) * w + ev["x"]
        parts.append(ev)
    events = {k: np.concatenate([q[k] for q in parts]) for k in parts[0]}
    check(events, irr0, m.noise_maps()["ba_rate_hz"].reshape(-1), p.dark_current_fA, T, n)
    assert len(events["t_cross_ns"]) > 100_000
