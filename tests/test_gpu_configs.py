"""The CUDA path against the oracle at the benchmark configurations' own sizes, and on several sensors of different
shapes in one launch (a B200, through the C ABI; bit-exact like every parity test here).

- Several sensors in one persistent launch: each sensor's tile range, frame size, seed, thresholds, noise and field
  are its own, and its events and samples equal the oracle chain run on that sensor alone (the reference runs one
  SensorModel per camera and cameras one after another, src/engine/engine.h:1-8), at every engine stage.
- 64 x 48, tanh edge, 1.0 s (120 windows) against the reference's own chain (the committed golden fixture made by
  tests/golden/make_golden.py); 346 x 260, 16 blobs, 2.0 s (239 windows) against the reference compiled here
  (oracle/_ref); 1280 x 720, 256 blobs with noise and leak, its first 8 windows, and the six-sensor 4.6 Mpx
  launch, its first 2 windows, against the oracle port.
- The reference's known answers (tests/sensor/test_pixel.cpp:92-198) through SensorModel on the device.
"""
import math
from pathlib import Path

import numpy as np
import pytest

from ballasim_b200 import fields as F
from ballasim_b200 import workloads as W
from ballasim_b200.params import resolve

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
EVENT_KEYS = ("p", "label", "flags", "t_cross_ns", "ds", "dn", "dl", "l_first")


def same_events(dev: dict, ora: dict, width: int, what: str = "") -> None:
    assert len(dev["t_cross_ns"]) == len(ora["t_cross_ns"]), (what, len(dev["t_cross_ns"]), len(ora["t_cross_ns"]))
    px = dev["y"].astype(np.int64) * width + dev["x"]
    assert np.array_equal(px, np.asarray(ora["pixel"]).astype(np.int64)), what
    for k in EVENT_KEYS:
        a, b = np.asarray(dev[k]), np.asarray(ora[k])
        if a.dtype.kind == "f":
            a, b = a.view(np.uint32), b.view(np.uint32)
        assert np.array_equal(a, b), f"{what}: column {k} differs"


def make_engine(specs, rules, stage=None, tile=None):
    from ballasim_b200.engine import Engine
    from ballasim_b200.sensor import SensorModel

    models = [SensorModel(resolve(s.preset, s.overrides), s.width, s.height, s.seed, [{"type": "constant"}],
                          s.camera) for s in specs]
    eng = Engine([(m, s.field) for m, s in zip(models, specs)], tol=rules.tol, dark=rules.dark,
                 min_dt_ns=rules.min_dt_ns, max_refine_levels=rules.max_refine_levels, l_min=rules.l_min,
                 l_max=rules.l_max)
    if stage is not None:
        eng.set_launch(0, 0, stage, tile)
    return eng, models


def run_engine(eng, models, chunks):
    """Runs the chunks of windows; returns each model's events (concatenated over the calls) and the samples."""
    eng.start(0)
    samples, parts = 0, [[] for _ in models]
    for c in chunks:
        s, _ = eng.run(c)
        samples += s
        for i, m in enumerate(models):
            parts[i].append(m.take_events())
    return [{k: np.concatenate([p[k] for p in ps]) for k in ps[0]} for ps in parts], samples


def mixed_sensors():
    """Three sensors of different shapes and laws: a 64 x 48 blob field with mismatch and refractory, a 96 x 72 blob
    field with noise and leak at its own thresholds, and a 40 x 30 tanh edge on the ideal preset."""
    a = W.SensorSpec(64, 48, 21, 0, dict(W.MISMATCH), F.blobs(64, 48, 21, 12))
    b = W.SensorSpec(96, 72, 22, 1, {**W.MISMATCH, **W.NOISE, "theta_on": 0.18, "theta_off": 0.22,
                                     "noise_shot_rate_hz": 30.0, "noise_ba_median_hz": 20.0, "leak_rate_hz": 2.0},
                     F.blobs(96, 72, 22, 24))
    c = W.SensorSpec(40, 30, 3, 2, dict(W.IDEAL), F.tanh_edge(40, 30, 3))
    return [a, b, c]


@pytest.mark.parametrize("stage,tile", [(0, 8), (16, 8), (64, 8), (0, 4), (64, 16), (32, 32), (1, 8), (1, 16)])
def test_several_sensors_in_one_launch_equal_each_sensor_alone(cuda_lib, stage, tile):
    """A launch over three sensors of different sizes, seeds, thresholds and laws: each sensor's events and the
    total samples equal the oracle chain of each sensor run alone, bit for bit, over two calls."""
    from oracle.oracle import simulate_port

    specs = mixed_sensors()
    rules = W.Rules()
    windows = 24
    want = [simulate_port(s, rules, windows, params=resolve(s.preset, s.overrides)) for s in specs]
    eng, models = make_engine(specs, rules, stage, tile)
    got, samples = run_engine(eng, models, [7, windows - 7])
    assert samples == sum(st["pixel_samples"] for _, st in want)
    for i, (s, (ev, _)) in enumerate(zip(specs, want)):
        same_events(got[i], ev, s.width, f"sensor {i} ({s.width}x{s.height})")
        assert len(ev["t_cross_ns"]) > 50, i
    assert np.count_nonzero(got[1]["label"] == 1) > 5  # sensor 1's noise events are there


def test_engine_take_of_every_sensor_equals_each_model_take(cuda_lib):
    """Engine.take_events (every sensor's sort and copy queued together, the host copies overlapped) gives each
    sensor the columns SensorModel.take_events gives, over two calls, with and without the pixel column."""
    specs = mixed_sensors()
    rules = W.Rules()
    got = []
    for batched in (False, True):
        eng, models = make_engine(specs, rules, 1, 8)
        eng.start(0)
        calls = []
        for chunk, with_pixel in ((5, True), (9, False)):
            eng.run(chunk)
            if batched:
                calls.append(eng.take_events(with_pixel=with_pixel))
            else:
                calls.append([m.take_events(with_pixel=with_pixel) for m in models])
            assert all(m.take_events()["t_cross_ns"].size == 0 for m in models)  # the lists are cleared
        got.append(calls)
    for call_a, call_b in zip(*got):
        for a, b in zip(call_a, call_b):
            assert a.keys() == b.keys()
            for k in a:
                assert np.array_equal(np.asarray(a[k]).view(np.uint8), np.asarray(b[k]).view(np.uint8)), k
    assert sum(len(c["t_cross_ns"]) for c in got[1][0]) > 100


def test_sensor_order_in_the_launch_does_not_matter(cuda_lib):
    """The same three sensors listed in reverse order give each sensor the same events."""
    specs = mixed_sensors()
    rules = W.Rules()
    eng, models = make_engine(specs, rules)
    fwd, s1 = run_engine(eng, models, [12])
    eng2, models2 = make_engine(specs[::-1], rules)
    rev, s2 = run_engine(eng2, models2, [12])
    assert s1 == s2
    for i in range(3):
        a, b = fwd[i], rev[2 - i]
        for k in a:
            assert np.array_equal(a[k], b[k]), (i, k)


def test_edge_64x48_one_second_equals_the_reference_fixture(cuda_lib):
    """64 x 48, tanh edge, 120 windows (1.0 s): the engine's events equal the reference's own sampler + SensorModel
    chain recorded in the golden fixture."""
    g = np.load(GOLDEN / "chain_edge64.npz")
    wl = W.edge_64x48()
    assert wl.windows == int(g["windows"]) == 120
    eng, models = make_engine(wl.sensors, wl.rules)
    got, samples = run_engine(eng, models, [wl.windows])
    assert samples == int(g["pixel_samples"])
    same_events(got[0], {k: g[k] for k in g.files}, 64)
    assert len(g["t_cross_ns"]) > 10_000


def test_blobs_346x260_two_seconds_equals_the_reference(cuda_lib, ref):
    """346 x 260, 16 blobs, 239 windows (2.0 s), mismatch and refractory: the engine (at the launch shape the
    autotuner picks) equals the reference's chain (WindowEngine<kHost>, then its fp32 SensorModel per window)."""
    wl = W.blobs_346x260()
    spec = wl.sensors[0]
    want, st = ref.Model(resolve(spec.preset, spec.overrides), spec.width, spec.height, spec.seed,
                         spec.camera).simulate(spec.field, wl.rules, wl.windows)
    eng, models = make_engine(wl.sensors, wl.rules)
    eng.start(0)
    eng.autotune(4)
    got, samples = run_engine(eng, models, [100, wl.windows - 100])
    assert samples == st["pixel_samples"]
    same_events(got[0], want, spec.width)
    assert len(want["t_cross_ns"]) > 100_000


def test_blobs_1280x720_noise_first_windows_equal_the_oracle(cuda_lib):
    """1280 x 720, 256 blobs, leak, shot and background-activity noise: the first 8 windows at full frame."""
    from oracle.oracle import simulate_port

    wl = W.blobs_1280x720()
    spec = wl.sensors[0]
    windows = 8
    want, st = simulate_port(spec, wl.rules, windows)
    for stage in (0, 64, 1):
        eng, models = make_engine(wl.sensors, wl.rules, stage, 8)
        got, samples = run_engine(eng, models, [windows])
        assert samples == st["pixel_samples"]
        same_events(got[0], want, spec.width, f"stage {stage}")
    assert len(want["t_cross_ns"]) > 10_000
    assert np.count_nonzero(want["label"] == 1) > 100


def test_six_sensors_first_windows_equal_the_oracle(cuda_lib):
    """The six-sensor launch (346x260, 640x480 x2, 1280x720 x2, 1920x1080; 4.6 Mpx, noise and leak, thresholds per
    sensor) at full size: its first 2 windows, each sensor against the oracle chain run alone."""
    from oracle.oracle import simulate_port

    wl = W.six_sensors()
    windows = 2
    want = [simulate_port(s, wl.rules, windows) for s in wl.sensors]
    for stage in (None, 1):
        eng, models = make_engine(wl.sensors, wl.rules, stage, 8 if stage else None)
        got, samples = run_engine(eng, models, [windows])
        assert samples == sum(st["pixel_samples"] for _, st in want)
        for i, (s, (ev, _)) in enumerate(zip(wl.sensors, want)):
            same_events(got[i], ev, s.width, f"stage {stage}, sensor {i} ({s.width}x{s.height})")
    assert sum(len(ev["t_cross_ns"]) for ev, _ in want) > 10_000


# ---- the reference's known answers (tests/sensor/test_pixel.cpp:92-198) on the device ----

def empty_call(t_end):
    z = np.zeros(0, np.int64)
    return (np.zeros(0, np.uint32), z, np.zeros((0, 1), np.float32), t_end, z, np.zeros(0, np.int32))


def device_model(p, w, h, seed, irr0, t0=0):
    from ballasim_b200.sensor import SensorModel

    m = SensorModel(p, w, h, seed, [{"type": "constant"}], 0)
    m.init(t0, np.asarray(irr0, np.float32).reshape(-1, 1))
    return m


def test_static_pixel_never_fires_on_the_device(cuda_lib):
    """A pixel whose irradiance never changes emits nothing over 20 windows (test_pixel.cpp:92-104)."""
    p = resolve("ideal", {})
    irr0 = np.array([1.0 + 300.0 * (i % 7) for i in range(16 * 8)], np.float32)
    m = device_model(p, 16, 8, 3, irr0)
    n = 0
    for w in range(1, 21):
        n += len(m.advance_runs(*empty_call(w * (1 << 23)))["t_cross_ns"])
    assert n == 0


def test_leak_events_follow_the_closed_form_on_the_device(cuda_lib, oracle_port):
    """Leak alone: the first event at t0 + ceil((theta - phi0) / l), then one every T_r + theta / l
    (test_pixel.cpp:106-136), and the device's events equal the oracle's bit for bit."""
    p = resolve("ideal", {"reset_mode": "physical", "refractory_s": 1e-4, "leak_rate_hz": 40.0,
                          "theta_on": 0.25, "theta_off": 0.25})
    t0 = 12345
    m = device_model(p, 8, 4, 11, np.full(32, 500, np.float32), t0)
    ev = m.advance_runs(*empty_call(300_000_000))
    o = oracle_port.Model(p, 8, 4, 11, 0)
    o.init(t0, np.full(32, 500, np.float32))
    o.advance_runs(np.zeros(0, np.uint32), np.zeros(0, np.int64), np.zeros(0, np.float32), np.zeros(0, np.int64),
                   np.zeros(0, np.int32), 300_000_000)
    same_events(ev, o.take_events(), 8)
    maps = m.sensor_maps()
    th, phi, leak = (np.asarray(maps[k], np.float64).reshape(-1) for k in ("theta_on", "phi0", "leak"))
    px_of = ev["y"].astype(np.int64) * 8 + ev["x"]
    checked = 0
    for px in range(32):
        sel = px_of == px
        times = ev["t_cross_ns"][sel]
        assert np.all(ev["p"][sel] == 1) and np.all(ev["label"][sel][1:] == 2)
        expect = t0 + math.ceil((th[px] - phi[px]) / leak[px] * 1e9)
        tol = 1 + math.ceil(4 * 2.0**-23 * th[px] / leak[px] * 1e9)
        for t in times:
            assert abs(int(t) - expect) <= tol
            expect = int(t) + 100_000 + math.ceil(th[px] / leak[px] * 1e9)
            checked += 1
    assert checked > 64


@pytest.mark.parametrize("sigma", [0.0, 0.021])
def test_o13_ramp_event_count_on_the_device(cuda_lib, sigma):
    """A 5-log ramp over 10 ms sampled every 10 us, then held: floor((swing + phi0) / theta_on) ON events per
    pixel, exactly 25 at sigma 0 (test_pixel.cpp:138-198, the instantaneous case)."""
    p = resolve("ideal", {"sigma_theta_on": sigma, "sigma_theta_off": sigma})
    Wd = Hd = 16
    n = Wd * Hd
    I0, T = 1000.0, 10_000_000
    times = np.linspace(10_000, T, 999).astype(np.int64)
    vals = (I0 * np.exp(5.0 * times.astype(np.float64) / T)).astype(np.float32)
    ids = np.arange(n, dtype=np.uint32)
    tt = np.tile(times, n)
    vv = np.tile(vals, n).reshape(-1, 1)
    starts = np.arange(n, dtype=np.int64) * len(times)
    counts = np.full(n, len(times), np.int32)
    m = device_model(p, Wd, Hd, 99, np.full(n, I0, np.float32))
    ev1 = m.advance_runs(ids, tt, vv, T, starts, counts)
    ev2 = m.advance_runs(*empty_call(T + 20_000_000))
    p_all = np.concatenate([ev1["p"], ev2["p"]])
    px = np.concatenate([ev1["y"].astype(np.int64) * Wd + ev1["x"], ev2["y"].astype(np.int64) * Wd + ev2["x"]])
    assert np.all(p_all == 1)
    count = np.bincount(px, minlength=n)
    maps = m.sensor_maps()
    th = np.asarray(maps["theta_on"], np.float64).reshape(-1)
    phi = np.asarray(maps["phi0"], np.float64).reshape(-1)
    d = p.dark_current_fA
    swing = math.log((I0 * math.exp(5.0) + d) / (I0 + d))
    exact = skipped = 0
    for i in range(n):
        levels = (swing + phi[i]) / th[i]
        if abs(levels - round(levels)) < 1e-6:
            skipped += 1
            continue
        exact += count[i] == math.floor(levels)
    assert exact == n - skipped
    if sigma == 0.0:
        assert skipped == 0 and np.all(count == 25)


# ---- the reference engine's per-window loop with the runs in HBM (sample_window on the device, advance_device) ----

@pytest.mark.parametrize("case,concurrent", [("blobs", True), ("noise", True), ("mixed", True), ("mixed", False)])
def test_device_windows_equal_the_oracle(cuda_lib, case, concurrent):
    """Levels, sample_window on device-resident inputs and advance_device on the runs, window by window and sensor by
    sensor (each sensor on its own stream and host thread, or all window-major on one stream): each sensor's events
    (downloaded per call) and the samples equal the oracle chain, bit for bit."""
    from ballasim_b200.sensor import SensorModel
    from ballasim_b200.windows import DeviceWindows
    from oracle.oracle import simulate_port

    if case == "mixed":
        specs = mixed_sensors()
    else:
        wl = W.small(case, 60, 40, 1)
        specs = wl.sensors
    rules, windows = W.Rules(), 16
    want = [simulate_port(s, rules, windows, params=resolve(s.preset, s.overrides)) for s in specs]
    models = [SensorModel(resolve(s.preset, s.overrides), s.width, s.height, s.seed, [{"type": "constant"}], s.camera)
              for s in specs]
    dw = DeviceWindows([(m, s.field) for m, s in zip(models, specs)], tol=rules.tol, dark=rules.dark,
                       min_dt_ns=rules.min_dt_ns, max_refine_levels=rules.max_refine_levels, l_min=rules.l_min,
                       l_max=rules.l_max)
    dw.start(0)
    parts = [[] for _ in specs]
    samples, events = dw.run(windows, on_events=lambda i, m, ev: parts[i].append(m.download_events(ev)),
                             concurrent=concurrent)
    assert samples == sum(st["pixel_samples"] for _, st in want)
    for i, (s, (ev, _)) in enumerate(zip(specs, want)):
        got = {k: np.concatenate([p[k] for p in parts[i]]) for k in parts[i][0]}
        same_events(got, ev, s.width, f"sensor {i}")
    assert events == sum(len(ev["t_cross_ns"]) for ev, _ in want) > 50


def test_device_windows_finish_every_sensor_before_an_error(cuda_lib):
    """With each sensor on its own thread, an error in one sensor's call (here its events callback) reaches the caller
    only after every other sensor has run all its windows."""
    from ballasim_b200.sensor import SensorModel
    from ballasim_b200.windows import DeviceWindows

    specs, rules, windows = mixed_sensors(), W.Rules(), 4
    models = [SensorModel(resolve(s.preset, s.overrides), s.width, s.height, s.seed, [{"type": "constant"}], s.camera)
              for s in specs]
    dw = DeviceWindows([(m, s.field) for m, s in zip(models, specs)], tol=rules.tol, dark=rules.dark,
                       min_dt_ns=rules.min_dt_ns, max_refine_levels=rules.max_refine_levels, l_min=rules.l_min,
                       l_max=rules.l_max)
    dw.start(0)
    calls = [0] * len(specs)

    def on_events(i, m, ev):
        calls[i] += 1
        if i == 1 and calls[i] == 2:
            raise RuntimeError("stop sensor 1")

    with pytest.raises(RuntimeError, match="stop sensor 1"):
        dw.run(windows, on_events=on_events)
    assert calls[1] == 2
    assert all(c == windows for i, c in enumerate(calls) if i != 1)


def test_device_window_refuses_bad_inputs_and_recovers(cuda_lib):
    """bs_sample_window_device checks the device ids and levels before it samples: a level above the finest or an id
    outside the field is refused (ValueError) with nothing written, and the next valid call samples as usual."""
    import ctypes as C

    import torch

    from ballasim_b200 import _lib
    from ballasim_b200.sampling import MidpointTest, field_frame, field_levels, rules_struct, sample_window, sampler_for

    wl = W.small("blobs", 32, 24, 1)
    spec, r = wl.sensors[0], wl.rules
    f, n = spec.field, 32 * 24
    s = sampler_for(f)
    rules = rules_struct(MidpointTest(r.tol, r.dark, [1.0], [1.0]), True, r.max_refine_levels, r.min_dt_ns)
    dev = torch.device("cuda")
    frame = field_frame(f, 0)
    lv = field_levels(f, 0, r.l_min, r.l_max)
    ids = torch.arange(n, dtype=torch.int32, device=dev)
    c_in = torch.from_numpy(frame.copy()).to(dev)
    s_in = torch.zeros(n, dtype=torch.int64, device=dev)
    c_out = torch.zeros(n, dtype=torch.float32, device=dev)
    s_out = torch.zeros(n, dtype=torch.int64, device=dev)
    total = C.c_size_t()

    def call(lv_t, ids_t):
        torch.cuda.synchronize()
        return _lib.lib().bs_sample_window_device(s.h, 0, ids_t.data_ptr(), lv_t.data_ptr(), n, c_in.data_ptr(),
                                                  s_in.data_ptr(), c_out.data_ptr(), s_out.data_ptr(),
                                                  C.byref(rules), None, C.byref(total))

    bad_lv = lv.copy()
    bad_lv[5] = 23 - (r.min_dt_ns.bit_length() - 1) + 1
    with pytest.raises(ValueError, match="levels must lie in"):
        _lib.check(call(torch.from_numpy(bad_lv).to(dev), ids))
    bad_ids = ids.clone()
    bad_ids[n - 1] = n
    with pytest.raises(ValueError, match="pixel id outside the field"):
        _lib.check(call(torch.from_numpy(lv).to(dev), bad_ids))
    _lib.check(call(torch.from_numpy(lv).to(dev), ids))
    torch.cuda.synchronize()
    want = sample_window(0, np.arange(n, dtype=np.uint32), lv, np.arange(n, dtype=np.uint32), frame.reshape(n, 1),
                         np.zeros(n, np.uint64), f, refine_signature=True,
                         midpoint=MidpointTest(r.tol, r.dark, [1.0], [1.0]), max_refine_levels=r.max_refine_levels,
                         min_dt_ns=r.min_dt_ns)
    assert total.value == len(want.t_ns)
    assert np.array_equal(c_out.cpu().numpy().view(np.uint32), want.last_irradiance.reshape(-1).view(np.uint32))


@pytest.mark.parametrize("leak_hz", [8.0, 40.0])
def test_cooperative_search_where_leak_balances_a_falling_signal(cuda_lib, leak_hz):
    """Strong leak against irradiance falling behind receding blobs: Delta lingers just below a level over long pieces,
    where the warp-cooperative search (stage 64) visits many nodes. Its events equal the oracle's and the serial
    stage's, and the run ends without a search bound error."""
    from oracle.oracle import simulate_port

    wl = W.small("blobs", 60, 40, 20)
    spec = W.SensorSpec(60, 40, 9, 0, {**W.MISMATCH, "leak_rate_hz": leak_hz, "leak_sigma_log10": 0.3,
                                      "refractory_s": 0.0}, F.blobs(60, 40, 9, 16))
    want, st = simulate_port(spec, wl.rules, wl.windows, params=resolve(spec.preset, spec.overrides))
    for stage in (64, 0):
        eng, models = make_engine([spec], wl.rules, stage, 8)
        got, samples = run_engine(eng, models, [wl.windows])
        assert samples == st["pixel_samples"]
        same_events(got[0], want, spec.width, f"stage {stage}")
        assert models[0].stats()["leaf_intervals"] > 0
    assert np.count_nonzero(want["label"] == 2) > 100  # leak-labelled events
