"""Parity of the CUDA path with the oracle, through the C ABI on a B200: the pixel model on ragged runs, the
window sampler, the device fields, and the fused engine; bit-exact (integer times, polarities, labels, flags and
the fp32 increments). Cases at sizes the CPU oracle finishes in seconds; full sizes are checked by properties
(test_gpu_scale.py)."""
import numpy as np
import pytest

from ballasim_b200 import workloads as W
from ballasim_b200.params import resolve
from runs import random_calls, wide_calls

pytestmark = pytest.mark.gpu

EVENT_KEYS = ("p", "label", "flags", "t_cross_ns", "ds", "dn", "dl", "l_first")


def same_events(dev: dict, ora: dict, width: int) -> None:
    assert len(dev["t_cross_ns"]) == len(ora["t_cross_ns"]), (len(dev["t_cross_ns"]), len(ora["t_cross_ns"]))
    px = dev["y"].astype(np.int64) * width + dev["x"]
    assert np.array_equal(px, ora["pixel"].astype(np.int64))
    for k in EVENT_KEYS:
        a, b = np.asarray(dev[k]), np.asarray(ora[k])
        if a.dtype.kind == "f":
            a, b = a.view(np.uint32), b.view(np.uint32)
        assert np.array_equal(a, b), f"column {k} differs"


@pytest.mark.parametrize("block", [0, 1, 128])
@pytest.mark.parametrize("overrides", [
    {},
    dict(W.MISMATCH),
    {**W.MISMATCH, "leak_rate_hz": 2.0, "leak_sigma_log10": 0.1},
    {"reset_mode": "physical", "refractory_s": 0.0, "eps_ci": 0.002, "initial_phase": "symmetric"},
    {**W.MISMATCH, **W.NOISE, "noise_shot_rate_hz": 50.0, "noise_ba_median_hz": 20.0},
])
def test_pixel_model_on_random_runs(cuda_lib, oracle_port, overrides, block):
    """The pixel model on random ragged runs (random pixel subsets in random order) against the oracle: the
    row-major kernel split in two launches (block 0) and in one (block 1), and the one-thread-per-pixel kernel
    (block 128)."""
    from ballasim_b200.sensor import SensorModel

    rng = np.random.default_rng(17 + len(overrides))
    Wd, Hd = 24, 20
    n = Wd * Hd
    p = resolve("ideal", overrides)
    dev = SensorModel(p, Wd, Hd, 5, [{"type": "constant"}], 0)
    dev.set_block(block)
    ora = oracle_port.Model(p, Wd, Hd, 5, 0)
    irr0 = rng.uniform(20, 200, n).astype(np.float32)
    dev.init(0, irr0.reshape(n, 1))
    ora.init(0, irr0)
    got = []
    for ids, tt, vv, t_end, starts, cnt in random_calls(rng, n, 0, 6):
        got.append(dev.advance_runs(ids, tt, vv, t_end, starts, cnt))
        ora.advance_runs(ids, tt, vv, starts, cnt, t_end)
    merged = {k: np.concatenate([g[k] for g in got]) for k in got[0]}
    same_events(merged, ora.take_events(), Wd)
    assert len(merged["t_cross_ns"]) > 10
    assert dev.time_ns == t_end


@pytest.mark.parametrize("block", [0, 1])
@pytest.mark.parametrize("long_run", [0, 1, 5, -1])
@pytest.mark.parametrize("layout", ["tiled", "long", "shuffled", "gaps", "sparse"])
def test_row_major_kernel_on_every_run_layout(cuda_lib, oracle_port, layout, long_run, block):
    """The row-major kernel against the oracle on every run layout (runs in pixel order tiling the sample arrays,
    runs of hundreds to thousands of samples, runs whose starts are shuffled or leave gaps, a sparse listing whose
    other pixels advance on their held sample) and split between its two walks: runs longer than long_run walked by
    the whole warp (1: every run of two or more samples; 0: the default 32; -1: none)."""
    from ballasim_b200.sensor import SensorModel

    rng = np.random.default_rng({"tiled": 1, "long": 2, "shuffled": 3, "gaps": 4, "sparse": 5}[layout])
    Wd, Hd = 40, 24
    n = Wd * Hd
    p = resolve("ideal", {**W.MISMATCH, **W.NOISE, "noise_shot_rate_hz": 20.0, "noise_ba_median_hz": 10.0,
                          "leak_rate_hz": 1.0})
    dev = SensorModel(p, Wd, Hd, 6, [{"type": "constant"}], 0)
    dev.set_long_run(long_run)
    dev.set_block(block)
    ora = oracle_port.Model(p, Wd, Hd, 6, 0)
    irr0 = rng.uniform(20, 300, n).astype(np.float32)
    dev.init(0, irr0.reshape(n, 1))
    ora.init(0, irr0)
    got, t = [], 0
    for call in range(4):
        t_end = t + (1 << 23)
        ids = np.arange(n, dtype=np.uint32)
        if layout == "sparse":
            ids = np.sort(rng.permutation(n)[: n // 7]).astype(np.uint32)
        hi = 2000 if layout == "long" else 14
        cnt = rng.integers(0, hi, len(ids)).astype(np.int32)
        cnt[rng.random(len(ids)) < 0.2] = 0
        runs = []
        for k in cnt:
            times = np.unique(rng.integers(t + 1, t_end + 1, int(k)))
            if rng.random() < 0.3 and len(times):
                times[0] = t
                times = np.unique(times)
            runs.append(times.astype(np.int64))
        cnt = np.array([len(r) for r in runs], np.int32)
        vals = [(100 * np.exp(np.cumsum(rng.normal(0, 0.05, len(r))))).astype(np.float32) for r in runs]
        order = np.arange(len(ids))
        if layout == "shuffled":
            order = rng.permutation(len(ids))
        pad = 3 if layout == "gaps" else 0
        starts = np.zeros(len(ids), np.int64)
        tt, vv, pos = [], [], 0
        for i in order:
            starts[i] = pos
            tt.append(runs[i])
            vv.append(vals[i])
            pos += len(runs[i])
            if pad:
                tt.append(np.zeros(pad, np.int64))
                vv.append(np.zeros(pad, np.float32))
                pos += pad
        tt = np.concatenate(tt) if tt else np.zeros(0, np.int64)
        vv = np.concatenate(vv) if vv else np.zeros(0, np.float32)
        got.append(dev.advance_runs(ids, tt, vv, t_end, starts, cnt))
        ora.advance_runs(ids, tt, vv, starts, cnt, t_end)
        t = t_end
    merged = {k: np.concatenate([g[k] for g in got]) for k in got[0]}
    same_events(merged, ora.take_events(), Wd)
    assert len(merged["t_cross_ns"]) > 50


@pytest.mark.parametrize("t_off,v_off", [(0, 0), (1, 1), (0, 2), (1, 3)])
def test_row_major_kernel_reads_device_runs_at_any_alignment(cuda_lib, oracle_port, t_off, v_off):
    """advance_device on CSR arrays that start t_off int64 and v_off float elements past a 16-byte boundary (a
    caller's sub-buffers) against the oracle."""
    import torch

    from ballasim_b200 import _lib
    from ballasim_b200.sensor import SensorModel

    rng = np.random.default_rng(40 + 4 * t_off + v_off)
    Wd, Hd = 36, 20
    n = Wd * Hd
    p = resolve("ideal", {**W.MISMATCH, **W.NOISE, "noise_shot_rate_hz": 20.0, "leak_rate_hz": 1.0})
    dev = SensorModel(p, Wd, Hd, 8, [{"type": "constant"}], 0)
    ora = oracle_port.Model(p, Wd, Hd, 8, 0)
    irr0 = rng.uniform(20, 300, n).astype(np.float32)
    dev.init(0, irr0.reshape(n, 1))
    ora.init(0, irr0)
    got, t = [], 0
    ids = np.arange(n, dtype=np.uint32)
    for call in range(3):
        t_end = t + (1 << 23)
        runs = [np.unique(rng.integers(t + 1, t_end + 1, int(k))).astype(np.int64)
                for k in rng.integers(0, 12, n)]
        cnt = np.array([len(r) for r in runs], np.int32)
        starts = np.concatenate([[0], np.cumsum(cnt)[:-1]]).astype(np.int64)
        tt = np.concatenate(runs)
        vv = np.concatenate([(100 * np.exp(np.cumsum(rng.normal(0, 0.08, len(r))))).astype(np.float32)
                             for r in runs])
        d_t = torch.zeros(len(tt) + 2, dtype=torch.int64, device="cuda")
        d_v = torch.zeros(len(vv) + 4, dtype=torch.float32, device="cuda")
        d_t[t_off:t_off + len(tt)] = torch.from_numpy(tt).cuda()
        d_v[v_off:v_off + len(vv)] = torch.from_numpy(vv).cuda()
        d_ids = torch.from_numpy(ids.astype(np.int32)).cuda()
        d_start = torch.from_numpy(starts).cuda()
        d_cnt = torch.from_numpy(cnt).cuda()
        r = _lib.DeviceRuns(d_ids.data_ptr(), d_start.data_ptr(), d_cnt.data_ptr(), n,
                            d_t.data_ptr() + 8 * t_off, d_v.data_ptr() + 4 * v_off, len(tt))
        torch.cuda.synchronize()
        ev = dev.advance_device(r, t_end, 1)
        got.append(dev.download_events(ev))
        ora.advance_runs(ids, tt, vv, starts, cnt, t_end)
        t = t_end
    merged = {k: np.concatenate([g[k] for g in got]) for k in got[0]}
    same_events(merged, ora.take_events(), Wd)
    assert len(merged["t_cross_ns"]) > 20


def test_advance_rectangular_and_ragged_forms_agree(cuda_lib):
    """Ragged runs give the padded rectangle's events bit for bit (tests/sensor/test_model.cpp:180)."""
    from ballasim_b200.sensor import SensorModel

    rng = np.random.default_rng(3)
    n, m = 64, 6
    t = np.sort(rng.integers(1, 1 << 23, (n, m)), axis=1).astype(np.int64)
    t = np.maximum.accumulate(t + np.arange(m), axis=1)
    irr = rng.uniform(10, 300, (n, m, 1)).astype(np.float32)
    counts = rng.integers(0, m + 1, n).astype(np.int32)
    ids = np.arange(n, dtype=np.uint32)
    a = SensorModel("ideal", 8, 8, 2, [{"type": "constant"}], 0)
    b = SensorModel("ideal", 8, 8, 2, [{"type": "constant"}], 0)
    irr0 = np.full((n, 1), 100, np.float32)
    a.init(0, irr0)
    b.init(0, irr0)
    ea = a.advance(ids, t, irr, 1 << 23, counts=counts)
    off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    tt = np.concatenate([t[i, : counts[i]] for i in range(n)]).astype(np.int64)
    vv = np.concatenate([irr[i, : counts[i]] for i in range(n)]).astype(np.float32)
    eb = b.advance(ids, tt, vv, 1 << 23, offsets=off)
    for k in ea:
        assert np.array_equal(ea[k], eb[k]), k


def test_refused_input_leaves_the_model_unchanged(cuda_lib):
    from ballasim_b200.sensor import SensorModel

    m = SensorModel("ideal", 4, 4, 1, [{"type": "constant"}], 0)
    with pytest.raises(RuntimeError):
        m.advance(np.zeros(0, np.uint32), np.zeros(0, np.int64), np.zeros((0, 1), np.float32), 10,
                  offsets=np.zeros(1, np.int64))  # before init
    m.init(100, np.full((16, 1), 50, np.float32))
    one = lambda ids, t, v, t_end: m.advance(np.array(ids, np.uint32), np.array(t, np.int64),  # noqa: E731
                                             np.array(v, np.float32).reshape(-1, 1), t_end,
                                             offsets=np.arange(len(ids) + 1, dtype=np.int64))
    before = m.save_state()
    for bad in [([1], [900], [60], 800), ([1, 1], [200, 300], [60, 60], 2000), ([99], [300], [60], 2000),
                ([2], [50], [60], 2000), ([3], [300], [np.nan], 2000)]:
        with pytest.raises(ValueError):
            one(*bad)
        assert m.save_state() == before and m.time_ns == 100
    with pytest.raises(ValueError):
        one([1], [200], [60], 50)  # t_end before the model time
    with pytest.raises(TypeError):
        m.advance(np.array([1], np.int64), np.array([200], np.int64), np.array([[60]], np.float32), 300,
                  offsets=np.array([0, 1], np.int64))


def test_event_buffer_overflow_reruns(cuda_lib, oracle_port):
    """More events than the initial device buffer: the call is re-run from its unchanged input state."""
    from ballasim_b200.sensor import SensorModel

    p = resolve("ideal", {"theta_on": 0.011, "theta_off": 0.011, "theta_floor": 0.01})
    Wd, Hd = 128, 64
    n = Wd * Hd
    dev = SensorModel(p, Wd, Hd, 9, [{"type": "constant"}], 0)
    ora = oracle_port.Model(p, Wd, Hd, 9, 0)
    irr0 = np.full(n, 10, np.float32)
    dev.init(0, irr0.reshape(n, 1))
    ora.init(0, irr0)
    ids = np.arange(n, dtype=np.uint32)
    tt = np.tile(np.array([1 << 22, 1 << 23], np.int64), n)
    vv = np.tile(np.array([400, 10], np.float32), n)
    starts = np.arange(n, dtype=np.int64) * 2
    cnt = np.full(n, 2, np.int32)
    ev = dev.advance_runs(ids, tt, vv, 1 << 23, starts, cnt)
    ora.advance_runs(ids, tt, vv, starts, cnt, 1 << 23)
    assert len(ev["t_cross_ns"]) > (1 << 16)
    same_events(ev, ora.take_events(), Wd)
    assert dev.stats()["gpu_reruns"] >= 1


@pytest.mark.parametrize("family,overrides", [("ideal", W.MISMATCH), ("prophesee_gen3", {"noise": False}),
                                              ("prophesee_gen3", {})])
def test_save_and_load_state_resume_bitwise(cuda_lib, family, overrides):
    from ballasim_b200.sensor import SensorModel

    rng = np.random.default_rng(8)
    n = 10 * 10
    calls = random_calls(rng, n, 0, 4)
    full = SensorModel(family, 10, 10, 4, [{"type": "constant"}], 0, overrides=overrides)
    part = SensorModel(family, 10, 10, 4, [{"type": "constant"}], 0, overrides=overrides)
    irr0 = rng.uniform(20, 200, (n, 1)).astype(np.float32)
    full.init(0, irr0)
    part.init(0, irr0)
    ev_full = [full.advance_runs(c[0], c[1], c[2], c[3], c[4], c[5]) for c in calls]
    for c in calls[:2]:
        part.advance_runs(c[0], c[1], c[2], c[3], c[4], c[5])
    blob = part.save_state()
    fresh = SensorModel(family, 10, 10, 4, [{"type": "constant"}], 0, overrides=overrides)
    fresh.load_state(blob)
    rest = [fresh.advance_runs(c[0], c[1], c[2], c[3], c[4], c[5]) for c in calls[2:]]
    for a, b in zip(ev_full[2:], rest):
        for k in a:
            assert np.array_equal(a[k], b[k]), k
    assert sum(len(a["t_cross_ns"]) for a in ev_full[2:]) > 10
    other = SensorModel(family, 10, 10, 5, [{"type": "constant"}], 0, overrides=overrides)
    with pytest.raises(ValueError):
        other.load_state(blob)


STATE_CASES = [
    ("ideal", dict(W.MISMATCH)),
    ("ideal", {**W.MISMATCH, "leak_rate_hz": 2.0, "leak_sigma_log10": 0.1, "reset_mode": "ideal"}),
    ("prophesee_gen3", {"noise": False}),
    ("prophesee_gen3", {"noise": True}),
    ("prophesee_gen3", {"noise": True, "noise_diffusion": "transient", "leak_rate_hz": 2.0}),
]


@pytest.mark.parametrize("family,overrides", STATE_CASES)
def test_states_move_between_the_reference_and_this_model(cuda_lib, ref, family, overrides):
    """save_state / load_state in the reference's format (src/sensor/sensor_model.cpp:1198-1262): a state the reference
    saves after two calls resumes here, and one saved here resumes in the reference, each giving the events of an
    uninterrupted reference run over the last two calls, bit for bit; the headers are equal, and a model of another
    seed refuses either state."""
    from ballasim_b200.sensor import SensorModel

    p = resolve(family, overrides)
    Wd, Hd, seed = 20, 16, 13
    n = Wd * Hd
    rng = np.random.default_rng(21)
    irr0 = rng.uniform(10, 300, n).astype(np.float32)
    calls = random_calls(rng, n, 0, 4)
    full = ref.Model(p, Wd, Hd, seed, 0)
    full.init(0, irr0)
    for c in calls[:2]:
        full.advance_runs(c[0], c[1], c[2], c[4], c[5], c[3])
    full.take_events()
    blob_ref = full.save_state()
    for c in calls[2:]:
        full.advance_runs(c[0], c[1], c[2], c[4], c[5], c[3])
    want = full.take_events()
    assert len(want["t_cross_ns"]) > 20

    # reference -> here
    dev = SensorModel(p, Wd, Hd, seed, [{"type": "constant"}], 0)
    assert dev.state_bytes() == len(blob_ref)
    dev.load_state(blob_ref)
    got = [dev.advance_runs(c[0], c[1], c[2], c[3], c[4], c[5]) for c in calls[2:]]
    same_events({k: np.concatenate([g[k] for g in got]) for k in got[0]}, want, Wd)

    # here -> reference
    mine = SensorModel(p, Wd, Hd, seed, [{"type": "constant"}], 0)
    mine.init(0, irr0.reshape(n, 1))
    for c in calls[:2]:
        mine.advance_runs(c[0], c[1], c[2], c[3], c[4], c[5])
    blob_mine = mine.save_state()
    assert blob_mine[:56] == blob_ref[:56]  # the StateHeader: magic, version, shape, seed, fingerprint, time
    back = ref.Model(p, Wd, Hd, seed, 0)
    back.load_state(blob_mine)
    for c in calls[2:]:
        back.advance_runs(c[0], c[1], c[2], c[4], c[5], c[3])
    same_events(back.take_events(), want, Wd)

    other = SensorModel(p, Wd, Hd, seed + 1, [{"type": "constant"}], 0)
    with pytest.raises(ValueError):
        other.load_state(blob_ref)
    other_ref = ref.Model(p, Wd, Hd, seed + 1, 0)
    with pytest.raises(ValueError):
        other_ref.load_state(blob_mine)


@pytest.mark.parametrize("family,overrides,calls,t0", [
    ("prophesee_gen3", {}, random_calls, 0),
    ("prophesee_gen3", {"leak_rate_hz": 2.0, "leak_sigma_log10": 0.1}, random_calls, 0),
    ("prophesee_gen3", {"reset_mode": "ideal", "refractory_s": 0.0}, random_calls, 0),
    ("prophesee_gen3", {"sigma_theta_on": 0.03, "sigma_theta_off": 0.03, "dark_sigma_ln": 0.5}, wide_calls, 0),
    ("prophesee_gen3", {"leak_rate_hz": 1.0, "refractory_s": 0.0}, wide_calls, -123456789),
    ("prophesee_gen3", {"refractory_s": 1e-3, "eps_L": 0.001}, wide_calls, 0),
    ("samsung_gen3", {}, wide_calls, 0),
    ("prophesee_gen3", {"noise": True}, random_calls, 12345),
    ("prophesee_gen3", {"noise": True, "noise_leaf_level": 3, "leak_rate_hz": 2.0, "leak_sigma_log10": 0.1},
     wide_calls, 0),
    ("prophesee_gen3", {"noise": True, "noise_leaf_level": 7, "reset_mode": "ideal", "refractory_s": 0.0},
     random_calls, -123456789),
    ("samsung_gen3", {"noise": True, "sigma_o": 0.2}, wide_calls, 65536 * 3 + 5),
    ("prophesee_gen3", {"noise": True, "noise_diffusion": "transient"}, wide_calls, 0),
    ("prophesee_gen3", {"noise": True, "noise_diffusion": "transient", "noise_leaf_level": 3, "leak_rate_hz": 2.0,
                        "refractory_s": 0.0}, wide_calls, 12345),
    ("prophesee_gen3", {"noise": True, "initial_state": "stationary"}, random_calls, 0),
    ("prophesee_gen3", {"noise": True, "initial_state": "stationary", "stationary_burnin_ns": 300_000_000,
                        "leak_rate_hz": 2.0, "refractory_s": 0.0}, wide_calls, 12345),
])
def test_cascade_model_equals_the_reference(cuda_lib, ref, family, overrides, calls, t0):
    """The cascade photoreceptor on the device (with its noise lattice where noise is on), through the C ABI, gives
    the reference's fp32 SensorModel events bit for bit on random ragged runs."""
    from ballasim_b200.sensor import SensorModel

    p = resolve(family, {"noise": False, **overrides})
    Wd, Hd, seed = 24, 20, 9 + len(overrides)
    n = Wd * Hd
    rng = np.random.default_rng(seed)
    dev = SensorModel(p, Wd, Hd, seed, [{"type": "constant"}], 0)
    ora = ref.Model(p, Wd, Hd, seed, 0)
    irr0 = rng.uniform(5, 400, n).astype(np.float32)
    dev.init(t0, irr0.reshape(n, 1))
    ora.init(t0, irr0)
    got = []
    for ids, tt, vv, t_end, starts, cnt in calls(rng, n, t0, 6):
        got.append(dev.advance_runs(ids, tt, vv, t_end, starts, cnt))
        ora.advance_runs(ids, tt, vv, starts, cnt, t_end)
    merged = {k: np.concatenate([g[k] for g in got]) for k in got[0]}
    same_events(merged, ora.take_events(), Wd)
    assert len(merged["t_cross_ns"]) > 500
    assert dev.time_ns == t_end


@pytest.mark.parametrize("case", ["edge", "blobs"])
def test_fields_and_levels_equal_the_oracle(cuda_lib, oracle_port, case):
    from ballasim_b200.sampling import field_frame, field_levels

    wl = W.small("edge", 37, 23, 1) if case == "edge" else W.small("blobs", 70, 50, 1)
    f = wl.sensors[0].field
    for t in (0, 3 << 23, (5 << 23) + 12345):
        assert np.array_equal(field_frame(f, t).view(np.uint32), oracle_port.field_frame(f, t).view(np.uint32))
    for w in (0, 7):
        assert np.array_equal(field_levels(f, w << 23), oracle_port.levels(f, w << 23, 1, 10))


@pytest.mark.parametrize("case", ["edge", "blobs", "blobs_listed"])
def test_sample_window_equals_the_oracle(cuda_lib, oracle_port, case):
    from ballasim_b200.sampling import MidpointTest, sample_window

    wl = W.small("edge", 20, 16, 1) if case == "edge" else W.small("blobs", 48, 40, 1)
    spec, r = wl.sensors[0], wl.rules
    f = spec.field
    n = spec.width * spec.height
    rng = np.random.default_rng(1)
    ids = np.arange(n, dtype=np.uint32) if case != "blobs_listed" else rng.permutation(n)[: n // 3].astype(np.uint32)
    mt = MidpointTest(r.tol, r.dark, [1.0], [1.0])
    carried = oracle_port.field_frame(f, 0)[ids]
    sig = np.zeros(len(ids), np.uint64)
    if case == "blobs_listed":
        sig[::7] = 5  # carried signatures that differ from the rendered ones flip the first interval
    c_dev, s_dev = carried.copy(), sig.copy()
    for w in range(3):
        t_w = w << 23
        lv_all = oracle_port.levels(f, t_w, 1, 10)
        lv = lv_all[ids] if case != "edge" else np.minimum(lv_all[ids] + (ids % 3).astype(np.uint8), 10)
        t, irr, off, carried, sig = oracle_port.sample_window(f, r, t_w, ids, lv, carried, sig)
        runs = sample_window(t_w, ids, lv, np.arange(len(ids)), c_dev.reshape(-1, 1), s_dev, f,
                             refine_signature=True, midpoint=mt, max_refine_levels=r.max_refine_levels,
                             min_dt_ns=r.min_dt_ns)
        assert np.array_equal(runs.offsets, off)
        assert np.array_equal(runs.t_ns, t)
        assert np.array_equal(runs.irradiance.reshape(-1).view(np.uint32), irr.view(np.uint32))
        assert np.array_equal(runs.last_irradiance.reshape(-1).view(np.uint32), carried.view(np.uint32))
        c_dev, s_dev = runs.last_irradiance.reshape(-1), runs.last_signature


def test_midpoint_test_matches_numpy_fp32(cuda_lib):
    """eta_L equals NumPy fp32 in sampling.py's operation order (tests/cpp/engine/test_window.cpp:19)."""
    from ballasim_b200.sampling import MidpointTest

    rng = np.random.default_rng(4)
    a, m, b = (rng.uniform(0, 300, (500, 2)).astype(np.float32) for _ in range(3))
    t = MidpointTest(0.01, 0.01, [0.5, 1.0], [1.5, 1.0])
    got = t.eta(a, m, b)
    dev = np.abs((a + b) * np.float32(-0.5) + m)
    low = np.minimum(np.minimum(a, m), b)
    num = np.float32(0) + np.float32(1.5) * dev[:, 0]
    num = num + np.float32(1.0) * dev[:, 1]
    den = np.float32(0.01) + np.float32(0.5) * low[:, 0]
    den = den + np.float32(1.0) * low[:, 1]
    med = np.maximum(np.maximum(np.float32(0), np.where(dev[:, 0] == 0, 0, dev[:, 0] / low[:, 0])),
                     np.where(dev[:, 1] == 0, 0, dev[:, 1] / low[:, 1])).astype(np.float32)
    want = np.minimum(num / den, med)
    assert np.array_equal(got.view(np.uint32), want.astype(np.float32).view(np.uint32))
    assert np.array_equal(t.exceeds(a, m, b), want > np.float32(0.01))


@pytest.mark.parametrize("stage,tile,graph", [(0, 8, True), (16, 8, True), (32, 8, True), (0, 4, True),
                                              (16, 16, True), (0, 32, True), (0, 8, False), (64, 8, True),
                                              (64, 4, True), (64, 16, False), (1, 8, True), (1, 4, False),
                                              (1, 32, True)])
@pytest.mark.parametrize("case", ["edge", "blobs", "noise"])
def test_engine_equals_the_oracle_chain(cuda_lib, case, stage, tile, graph):
    """The fused engine (sampler and pixel model on one thread, all windows in one launch; streamed, or staged in
    shared memory per window, stage 64 with the warp-cooperative crossing search, stage 1 split into two launches per
    window; any tile shape; from a CUDA graph or not) gives the oracle chain's events (sample_window, then advance,
    per window) bit for bit."""
    from ballasim_b200.engine import Engine
    from ballasim_b200.sensor import SensorModel
    from oracle.oracle import simulate_port

    wl = {"edge": lambda: W.small("edge", 30, 20, 24), "blobs": lambda: W.small("blobs", 60, 40, 24),
          "noise": lambda: W.small("noise", 40, 30, 30)}[case]()
    spec = wl.sensors[0]
    p = resolve("ideal", spec.overrides)
    if case == "noise":  # rates high enough for many noise events in a short run
        p = resolve(p, {"noise_shot_rate_hz": 40.0, "noise_ba_median_hz": 30.0, "leak_rate_hz": 3.0})
    ora, st = simulate_port(spec, wl.rules, wl.windows, params=p)
    m = SensorModel(p, spec.width, spec.height, spec.seed, [{"type": "constant"}], spec.camera)
    r = wl.rules
    eng = Engine([(m, spec.field)], tol=r.tol, dark=r.dark, min_dt_ns=r.min_dt_ns,
                 max_refine_levels=r.max_refine_levels, l_min=r.l_min, l_max=r.l_max)
    eng.set_launch(0, 0, stage, tile)
    eng.set_graph(graph)
    eng.start(0)
    samples, parts = 0, []
    for chunk in (5, wl.windows - 5):  # two calls: the state and carried samples cross the call boundary
        s, _ = eng.run(chunk)
        samples += s
        parts.append(m.take_events())  # a call's events, as advance_device's, are valid until the next call
    ev = {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}
    assert samples == st["pixel_samples"]
    same_events(ev, ora, spec.width)
    assert len(ev["t_cross_ns"]) > 20
    if case == "noise":
        assert np.count_nonzero(ev["label"] == 1) > 5


@pytest.mark.parametrize("l_min,windows", [(5, 6), (3, 10)])
def test_split_engine_where_windows_overflow_the_stage(cuda_lib, l_min, windows):
    """The split engine where every window (lattice level 5: 32 slots) or some windows overflow its 16-sample stage:
    those are posted whole and walked again by the rest kernel; the events equal the oracle chain's."""
    from dataclasses import replace

    from ballasim_b200.engine import Engine
    from ballasim_b200.sensor import SensorModel
    from oracle.oracle import simulate_port

    wl = W.small("noise", 40, 30, windows)
    spec = wl.sensors[0]
    r = replace(wl.rules, l_min=l_min, l_max=max(l_min, wl.rules.l_max))
    p = resolve(resolve("ideal", spec.overrides), {"noise_shot_rate_hz": 40.0, "noise_ba_median_hz": 30.0,
                                                   "leak_rate_hz": 3.0})
    ora, st = simulate_port(spec, r, windows, params=p)
    m = SensorModel(p, spec.width, spec.height, spec.seed, [{"type": "constant"}], spec.camera)
    eng = Engine([(m, spec.field)], tol=r.tol, dark=r.dark, min_dt_ns=r.min_dt_ns,
                 max_refine_levels=r.max_refine_levels, l_min=r.l_min, l_max=r.l_max)
    eng.set_launch(0, 0, 1, 8)
    eng.start(0)
    s, _ = eng.run(windows)
    assert s == st["pixel_samples"]
    same_events(m.take_events(), ora, spec.width)
    assert len(ora["t_cross_ns"]) > 20


@pytest.mark.gpu
def test_autotune_keeps_the_state_and_the_events(cuda_lib):
    """The autotuner's trial steps leave the models as they were: the run after it gives the events of a run
    without it, at whatever launch shape it picked."""
    from ballasim_b200.engine import Engine
    from ballasim_b200.sensor import SensorModel

    wl = W.small("noise", 64, 40, 12)
    spec, r = wl.sensors[0], wl.rules
    out = []
    for tune in (False, True):
        m = SensorModel(resolve("ideal", spec.overrides), spec.width, spec.height, spec.seed, [{"type": "constant"}],
                        spec.camera)
        eng = Engine([(m, spec.field)], tol=r.tol, dark=r.dark, min_dt_ns=r.min_dt_ns,
                     max_refine_levels=r.max_refine_levels, l_min=r.l_min, l_max=r.l_max)
        eng.start(0)
        if tune:
            rows = eng.autotune(4)
            assert len(rows) == 24 and all(x["ms"] > 0 for x in rows)  # 3 tile widths x 2 warps x stage 0, 1, 16, 64
            best = min(rows, key=lambda x: x["ms"])
            assert eng.launch["tile_width"] == best["tile_width"] and eng.launch["stage"] == best["stage"]
        s, e = eng.run(wl.windows)
        out.append((s, e, m.take_events(with_pixel=True)))
    assert out[0][0] == out[1][0] and out[0][1] == out[1][1]
    for k in ("pixel", "t_cross_ns", "p", "label"):
        assert np.array_equal(out[0][2][k], out[1][2][k])


@pytest.mark.gpu
def test_output_stage_follows_the_reference_order(cuda_lib, ref):
    """The output stage (records released in (t_reported, x, y, t_cross) order at each call's cut on the sensor clock,
    the rest held) equals the reference's output_order and output_cut applied to the same events."""
    from ballasim_b200.engine import Engine
    from ballasim_b200.sensor import SensorModel

    wl = W.small("noise", 48, 32, 12)
    spec, r = wl.sensors[0], wl.rules
    ov = {**spec.overrides, "noise_shot_rate_hz": 40.0, "noise_ba_median_hz": 30.0, "readout_quantum_s": 1e-6,
          "readout_delay_s": 3e-6, "clock_drift_ppm": 40.0, "clock_offset_ns": 12345}
    p = resolve("ideal", ov)
    outs, evs, held = [], [], 0
    for mode in ("output", "events"):
        m = SensorModel(p, spec.width, spec.height, spec.seed, [{"type": "constant"}], spec.camera)
        eng = Engine([(m, spec.field)], tol=r.tol, dark=r.dark, min_dt_ns=r.min_dt_ns,
                     max_refine_levels=r.max_refine_levels, l_min=r.l_min, l_max=r.l_max)
        eng.start(0)
        for chunk in (3, 4, 5):
            eng.run(chunk)
            if mode == "output":
                outs.append(m.take_output())
            else:
                evs.append(m.take_events())
        if mode == "output":
            held = m.output_held
    got = {k: np.concatenate([o[k] for o in outs]) for k in outs[0]}
    ev = {k: np.concatenate([e[k] for e in evs]) for k in evs[0]}
    L = ref.lib()
    phase = L.ref_readout_phase(spec.seed, spec.camera, 1000)
    want_rep = [L.ref_reported_time(1000, 3000, phase, 12345, 40.0, int(t)) for t in ev["t_cross_ns"]]
    assert np.array_equal(ev["t_reported_ns"], np.array(want_rep, np.int64))
    perm = ref.output_order(ev["t_cross_ns"], ev["x"], ev["y"], ev["t_reported_ns"], spec.height)
    cut = L.ref_output_cut(0, 0, 0, 12345, 40.0, wl.windows << 23)
    order = perm[ev["t_reported_ns"][perm] < cut]
    assert len(got["t_cross_ns"]) == len(order) > 100 and held == len(perm) - len(order)
    for k in ("t_reported_ns", "t_cross_ns", "x", "y", "p", "flags"):
        assert np.array_equal(got[k], ev[k][order]), k
    s1 = np.array([L.ref_label_s1(int(c)) for c in ev["label"][order]], np.uint8)
    assert np.array_equal(got["label"], s1)
    assert len(np.unique(ev["label"])) > 1


@pytest.mark.parametrize("tile", [8, 4, 16])
@pytest.mark.parametrize("case", ["blobs", "leak", "lattice", "lattice_leak", "lattice_staged", "lattice_leak_staged",
                                  "lattice_dense_staged", "lattice_stationary_staged", "lattice_transient_staged",
                                  "lattice_transient"])
def test_cascade_engine_equals_the_reference_chain(cuda_lib, ref, case, tile):
    """The fused engine with the cascade photoreceptor, with and without its noise lattice, gives the reference's own
    chain (WindowEngine<kHost> sampling, then the fp32 SensorModel on the runs, per window) bit for bit, over two
    calls and any tile shape; the staged lattice engine too, also where every window overflows its stage (lattice
    levels from 6: at least 65 samples a window) and is redone streaming."""
    import dataclasses

    from ballasim_b200.engine import Engine
    from ballasim_b200.sensor import SensorModel

    wl = W.small("blobs", 60, 40, 24)
    spec, r = wl.sensors[0], wl.rules
    if "dense" in case:
        r = dataclasses.replace(r, l_min=6)
    over = {**W.MISMATCH, "noise": case.startswith("lattice")}
    if "stationary" in case:
        over.update(initial_state="stationary", stationary_burnin_ns=400_000_000)
    if "transient" in case:
        over.update(noise_diffusion="transient")
    if "leak" in case:
        over.update(leak_rate_hz=2.0, leak_sigma_log10=0.1, refractory_s=0.0)
    p = resolve("prophesee_gen3", over)
    want, st = ref.Model(p, spec.width, spec.height, spec.seed, spec.camera).simulate(spec.field, r, wl.windows)
    m = SensorModel(p, spec.width, spec.height, spec.seed, [{"type": "constant"}], spec.camera)
    eng = Engine([(m, spec.field)], tol=r.tol, dark=r.dark, min_dt_ns=r.min_dt_ns,
                 max_refine_levels=r.max_refine_levels, l_min=r.l_min, l_max=r.l_max)
    eng.set_launch(0, 0, 32 if case.endswith("staged") else 0, tile)
    eng.start(0)
    samples, parts = 0, []
    for chunk in (5, wl.windows - 5):
        s, _ = eng.run(chunk)
        samples += s
        parts.append(m.take_events())
    ev = {k: np.concatenate([x[k] for x in parts]) for k in parts[0]}
    assert samples == st["pixel_samples"]
    same_events(ev, want, spec.width)
    assert len(ev["t_cross_ns"]) > 100


@pytest.mark.gpu
def test_engine_refuses_mixed_photoreceptors_and_cascade_options(cuda_lib):
    from ballasim_b200.engine import Engine
    from ballasim_b200.sensor import SensorModel

    wl = W.small("blobs", 32, 16, 2)
    spec, r = wl.sensors[0], wl.rules
    inst = SensorModel(resolve("ideal", spec.overrides), 32, 16, 1, [{"type": "constant"}], 0)
    casc = SensorModel(resolve("prophesee_gen3", {"noise": False}), 32, 16, 2, [{"type": "constant"}], 1)
    with pytest.raises(ValueError):
        Engine([(inst, spec.field), (casc, spec.field)], tol=r.tol, dark=r.dark, min_dt_ns=r.min_dt_ns)
    eng = Engine([(casc, spec.field)], tol=r.tol, dark=r.dark, min_dt_ns=r.min_dt_ns)
    with pytest.raises(ValueError):
        eng.set_launch(0, 0, 16, 8)


@pytest.mark.parametrize("family,overrides", [
    ("ideal", W.MISMATCH),
    ("prophesee_gen3", {"noise": False}),
    ("prophesee_gen3", {"noise": True, "initial_state": "stationary", "stationary_burnin_ns": 300_000_000}),
])
def test_photometry_gain_map_equals_the_reference(cuda_lib, ref, family, overrides):
    """set_photometry (sensor_module.cpp:477-502): a scale and a per-pixel gain map move irr_max to the largest gain
    and each pixel's photocurrent to scale x gain; the model's events equal the reference's own after the same call,
    bit for bit, and a state saved under one gain map does not load under another."""
    from ballasim_b200.sensor import SensorModel

    p = resolve(family, overrides)
    Wd, Hd, seed = 24, 20, 31
    n = Wd * Hd
    rng = np.random.default_rng(seed)
    gain = rng.uniform(0.4, 1.6, (Hd, Wd)).astype(np.float32)
    dev = SensorModel(p, Wd, Hd, seed, [{"type": "constant"}], 0)
    ora = ref.Model(p, Wd, Hd, seed, 0)
    assert np.array_equal(dev.gain_map(), np.ones((Hd, Wd), np.float32))
    dev.set_photometry(2.5, gain)
    ora.set_photometry(2.5, gain)
    assert np.array_equal(dev.gain_map(), gain)
    assert dev.params.illuminance_scale == 2.5
    assert np.float32(dev.irr_max) == np.float32(ora.irr_max)
    assert dev.irr_max == np.float32(1e9 / (2.5 * float(gain.max())))
    irr0 = rng.uniform(5, 400, n).astype(np.float32)
    dev.init(0, irr0.reshape(n, 1))
    ora.init(0, irr0)
    got = []
    for ids, tt, vv, t_end, starts, cnt in random_calls(rng, n, 0, 4):
        got.append(dev.advance_runs(ids, tt, vv, t_end, starts, cnt))
        ora.advance_runs(ids, tt, vv, starts, cnt, t_end)
    merged = {k: np.concatenate([g[k] for g in got]) for k in got[0]}
    same_events(merged, ora.take_events(), Wd)
    assert len(merged["t_cross_ns"]) > 100
    blob = dev.save_state()
    other = SensorModel(p, Wd, Hd, seed, [{"type": "constant"}], 0)
    other.set_photometry(2.5, np.where(gain > 1, gain, 1).astype(np.float32))
    with pytest.raises(ValueError):
        other.load_state(blob)
    other.set_photometry(2.5, gain)
    other.load_state(blob)
    for bad in (np.ones(n - 1, np.float32), np.full(n, -1.0, np.float32), np.full(n, np.inf, np.float32)):
        with pytest.raises(ValueError):
            other.set_photometry(1.0, bad)
    with pytest.raises(ValueError):
        other.set_photometry(0.0)
    other.set_photometry(1.0)
    assert np.array_equal(other.gain_map(), np.ones((Hd, Wd), np.float32))
    assert other.irr_max == np.float32(1e9)


@pytest.mark.parametrize("family,overrides", [("ideal", W.MISMATCH), ("prophesee_gen3", W.MISMATCH),
                                              ("prophesee_gen3", {**W.MISMATCH, "noise": True})])
def test_engine_with_a_gain_map_equals_the_reference_chain(cuda_lib, ref, family, overrides):
    """The fused engine reads each pixel's scale x gain and the camera's clamp: with a vignetting-like gain map its
    events equal the reference's chain under the same set_photometry."""
    from ballasim_b200.engine import Engine
    from ballasim_b200.sensor import SensorModel

    wl = W.small("blobs", 60, 40, 12)
    spec, r = wl.sensors[0], wl.rules
    p = resolve(family, overrides)
    yy, xx = np.mgrid[0:spec.height, 0:spec.width]
    rr = ((xx - spec.width / 2) ** 2 + (yy - spec.height / 2) ** 2) / (spec.width / 2) ** 2
    gain = (1.0 / (1.0 + 0.5 * rr) ** 2).astype(np.float32)
    o = ref.Model(p, spec.width, spec.height, spec.seed, spec.camera)
    o.set_photometry(0.8, gain)
    want, st = o.simulate(spec.field, r, wl.windows)
    m = SensorModel(p, spec.width, spec.height, spec.seed, [{"type": "constant"}], spec.camera)
    m.set_photometry(0.8, gain)
    eng = Engine([(m, spec.field)], tol=r.tol, dark=r.dark, min_dt_ns=r.min_dt_ns,
                 max_refine_levels=r.max_refine_levels, l_min=r.l_min, l_max=r.l_max)
    eng.start(0)
    s, _ = eng.run(wl.windows)
    ev = m.take_events()
    assert s == st["pixel_samples"]
    same_events(ev, want, spec.width)
    assert len(ev["t_cross_ns"]) > 100
