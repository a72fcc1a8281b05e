"""The learned step proposal (no reference counterpart; the plain sampler is its judge and fallback).

- features and the training walk: the CUDA walk over the plain sampler's device runs gives bit-identical pairs
  (BF16 features, targets, keys) to the oracle's C restatement over the oracle's own runs;
- the MLP on the tensor cores: forward pass and gradients against a CPU FP64 restatement that rounds to BF16 at the
  same points (tolerances below), deterministic Adam training that lowers the loss;
- the learned engine: every proposed step is legal (aligned, not below the plain lattice step, tiling each window),
  the samples are exactly those the oracle's judge and plain-rule fallback give for the recorded steps, and the
  events are bit-identical to the oracle pixel model fed those samples;
- the gain: a network trained on training-seed fields needs at least 2x fewer renders per pixel than the plain
  sampler on a held-out field, with the event count within 1 % and the median |dt| of signal events <= 10 us.
"""
import math

import numpy as np
import pytest

from ballasim_b200 import workloads as W
from ballasim_b200.params import resolve


# ---------------------------------------------------------------------------------------------
# CPU: the oracle's own definitions
# ---------------------------------------------------------------------------------------------
def test_features_definition(oracle_port):
    rng = np.random.default_rng(3)
    hx = rng.normal(3.0, 0.01, 8).astype(np.float32)
    x = np.float32(3.0)
    gaps = 0
    for k, g in enumerate([13, 14, 23, 20, 17, 13, 22, 15]):
        gaps |= g << (8 * k)
    f = oracle_port.step_features(hx, gaps, float(x))
    d = (hx.astype(np.float64) - float(x)) * 1e4
    np.testing.assert_allclose(f[:8], np.arcsinh(d) / 4, rtol=2e-6, atol=2e-6)
    np.testing.assert_allclose(f[8:], (np.array([13, 14, 23, 20, 17, 13, 22, 15]) - 13) / 10, atol=1e-7)
    flat = oracle_port.step_features(np.full(8, 2.5, np.float32), 0x1717171717171717, 2.5)
    assert np.all(flat[:8] == 0) and np.all(flat[8:] == np.float32(1.0))


def _bf16_bits(v: np.ndarray) -> np.ndarray:
    import torch

    return torch.from_numpy(np.asarray(v, np.float32)).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)


def test_walk_targets_by_brute_force(oracle_port):
    """The oracle walk's targets equal a direct evaluation of the rule on the plain runs, and its features are the
    definition's values rounded to BF16."""
    wl = W.small("blobs", 40, 24, 4, seed=5)
    f, r = wl.sensors[0].field, wl.rules
    x, y, keys = oracle_port.walk_pairs(f, r, 4, stride=7, eps=1e-4, seed=9)
    assert len(y) > 0
    assert np.all((y >= 0) & (y <= 10))
    # brute force of the first window of a few walkers
    ids = np.arange(f.width * f.height, dtype=np.uint32)
    lv = oracle_port.levels(f, 0, r.l_min, r.l_max)
    t, irr, off, _, _ = oracle_port.sample_window(f, r, 0, ids, lv, oracle_port.field_frame(f, 0),
                                                  np.zeros(len(ids), np.uint64))
    logf = np.vectorize(lambda v: oracle_port.lib().orc_logf(float(v)), otypes=[np.float32])
    checked = 0
    for p in range(0, len(ids), 7)[:12]:
        ts = (t[off[p]:off[p + 1]]).astype(np.int64)
        vs = irr[off[p]:off[p + 1]]
        mine = keys >> np.uint64(32) == p
        first = (keys & np.uint64((1 << 32) - 1)) >> np.uint64(11) == 0
        yp = y[mine & first]
        # the walk's first point is slot 0: its target by brute force
        s_floor = 23 - int(lv[p])
        best = s_floor
        for s in range(s_floor + 1, 24):
            hi = 1 << s
            j = int(np.searchsorted(ts, hi))
            inside = slice(1, j)
            lin = (vs[0] + (vs[j] - vs[0]) * (ts[inside].astype(np.float32) / np.float32(hi))).astype(np.float32)
            if not np.all(np.abs(logf(vs[inside]) - logf(lin)) <= np.float32(1e-4)):
                break
            best = s
        assert yp[0] == best - 13
        checked += 1
    assert checked == 12
    # features: the definition rounded to BF16 (first pair of the first walker: flat virtual history)
    assert np.all(x[0, 8:] == _bf16_bits(np.ones(8)))


def test_mlp_reference_matches_numpy():
    from oracle import mlp_ref

    rng = np.random.default_rng(1)
    p = (rng.normal(size=5313) * 0.2).astype(np.float32)
    xb = _bf16_bits(rng.normal(size=(7, 16)))
    y, _ = mlp_ref.forward(p, xb)
    bf = lambda a: np.asarray(_bf16_bits(a).astype(np.uint32) << 16).view(np.float32).astype(np.float64)  # noqa
    x = bf(np.asarray(xb.astype(np.uint32) << 16).view(np.float32))
    W1, b1 = bf(p[:1024].reshape(16, 64)), p[1024:1088].astype(np.float64)
    W2, b2 = bf(p[1088:5184].reshape(64, 64)), p[5184:5248].astype(np.float64)
    W3, b3 = bf(p[5248:5312]), float(p[5312])
    h1 = bf(np.maximum(x @ W1 + b1, 0).astype(np.float32))
    h2 = bf(np.maximum(h1 @ W2 + b2, 0).astype(np.float32))
    np.testing.assert_allclose(y.numpy(), h2 @ W3 + b3, rtol=1e-6, atol=1e-6)


# ---------------------------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------------------------
def _rand_features(n, seed):
    import torch

    rng = np.random.default_rng(seed)
    f = np.concatenate([rng.normal(0, 1.0, (n, 8)), rng.uniform(0, 1, (n, 8))], axis=1)
    return torch.from_numpy(_bf16_bits(f).astype(np.uint16)).cuda(), _bf16_bits(f)


@pytest.mark.gpu
def test_forward_matches_fp64(cuda_lib):
    from ballasim_b200.learned import StepMLP
    from oracle import mlp_ref

    net = StepMLP(seed=4)
    x, xb = _rand_features(3001, 0)
    y = net.forward(x).cpu().numpy().astype(np.float64)
    ref, _ = mlp_ref.forward(net.params, xb)
    ref = ref.numpy()
    # FP32 accumulation against FP64 differs by rounding, and an activation whose FP32 and FP64 sums round to
    # different BF16 neighbours moves y by one BF16 step of that activation times its weight.
    err = np.abs(y - ref) / (1.0 + np.abs(ref))
    assert err.max() < 1e-2, err.max()
    assert np.median(err) < 1e-5


@pytest.mark.gpu
def test_gradient_check_against_fp64(cuda_lib):
    import torch

    from ballasim_b200.learned import StepMLP
    from oracle import mlp_ref

    net = StepMLP(seed=8)
    n = 1000  # not a multiple of the 128-row tile: the last tile is masked
    x, xb = _rand_features(n, 1)
    tgt = np.random.default_rng(2).uniform(0, 10, n).astype(np.float32)
    g, loss = net.gradient(x, torch.from_numpy(tgt).cuda())
    g_ref, loss_ref = mlp_ref.gradient(net.params, xb, tgt)
    assert abs(loss - loss_ref) <= 1e-4 * loss_ref
    # The device rounds the backward operands dH2 and dH1 to BF16 (2^-9 relative) before its tensor-core passes.
    rel = np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
    assert rel < 1e-2, rel
    for name, (off, size) in {"W1": (0, 1024), "b1": (1024, 64), "W2": (1088, 4096), "b2": (5184, 64),
                              "W3": (5248, 64), "b3": (5312, 1)}.items():
        a, b = g[off:off + size], g_ref[off:off + size]
        assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b) + 1e-9, name


@pytest.mark.gpu
def test_training_lowers_loss_and_is_deterministic(cuda_lib):
    import torch

    from ballasim_b200.learned import StepMLP

    teacher = StepMLP(seed=100)
    x, _ = _rand_features(60000, 5)
    y = teacher.forward(x)
    a, b = StepMLP(seed=1), StepMLP(seed=1)
    la = a.train(x, y, steps=300, batch=8192, lr=1e-3, seed=3)
    lb = b.train(x, y, steps=300, batch=8192, lr=1e-3, seed=3)
    assert a.steps == 300
    assert np.all(np.isfinite(la))
    assert la[-20:].mean() < 0.1 * la[:5].mean(), (la[:5], la[-20:])
    assert np.array_equal(a.params, b.params) and np.array_equal(la, lb)
    # the graph path (32-step chunks) and the eager path take the same steps
    c = StepMLP(seed=1)
    for _ in range(10):
        c.train(x, y, steps=30, batch=8192, lr=1e-3, seed=3)
    assert np.array_equal(a.params, c.params)
    del torch


@pytest.mark.gpu
@pytest.mark.parametrize("stride", [1, 5])
def test_trace_pairs_match_the_oracle(cuda_lib, oracle_port, stride):
    import torch

    from ballasim_b200.learned import trace_pairs

    wl = W.small("blobs", 64, 48, 6, seed=11)
    f, r = wl.sensors[0].field, wl.rules
    x, y, k = trace_pairs(f, r, 6, stride=stride, eps=1e-4, seed=21, keys=True)
    xo, yo, ko = oracle_port.walk_pairs(f, r, 6, stride=stride, eps=1e-4, seed=21)
    k = k.view(torch.int64).cpu().numpy().view(np.uint64)
    assert np.array_equal(k, ko)  # already in (pixel, window, step) order
    assert np.array_equal(y.cpu().numpy(), yo)
    assert np.array_equal(x.cpu().numpy().view(np.uint16), xo)


def _learned_engine_case(margin, mlp_seed, windows=5, w=48, h=32, seed=13, train=False):
    from ballasim_b200.engine import Engine
    from ballasim_b200.learned import StepMLP, trace_pairs
    from ballasim_b200.sensor import SensorModel

    wl = W.small("noise", w, h, windows, seed=seed)
    spec, r = wl.sensors[0], wl.rules
    net = StepMLP(seed=mlp_seed)
    if train:
        x, y, _ = trace_pairs(spec.field, r, 8, stride=1, seed=2)
        net.train(x, y, steps=200, batch=4096)
    m = SensorModel(resolve("ideal", spec.overrides), w, h, spec.seed, [{"type": "constant"}], spec.camera)
    eng = Engine([(m, spec.field)], tol=r.tol, dark=r.dark, min_dt_ns=r.min_dt_ns,
                 max_refine_levels=r.max_refine_levels, l_min=r.l_min, l_max=r.l_max)
    eng.set_proposal(net, margin=margin)
    eng.set_record(1 << 22)
    eng.start(0)
    samples, _ = eng.run(windows)
    return wl, m, eng, samples, net


@pytest.mark.gpu
@pytest.mark.parametrize("margin,trained", [(0.25, True), (-3.0, False), (6.0, False)])
def test_learned_engine_matches_the_oracle(cuda_lib, oracle_port, margin, trained):
    """Steps from a trained net, from a net pushed to long steps (negative margin: the judge rejects, the plain rule
    refines) and to the plain lattice floor; samples and events exact against the oracle."""
    windows = 5
    wl, m, eng, samples, _ = _learned_engine_case(margin, 7, windows=windows, train=trained)
    spec, r = wl.sensors[0], wl.rules
    f = spec.field
    np_ = f.width * f.height
    rs = eng.take_record("samples")
    rp = eng.take_record("steps")
    assert samples == len(rs["t_ns"]) + windows * np_
    # legal steps: per pixel in time order, aligned and tiling every window
    o = np.lexsort((rp["t_ns"], rp["pixel"]))
    steps = {}
    for p in range(np_):
        sel = o[rp["pixel"][o] == p]
        steps[p] = rp["log2_step"][sel]
        t = rp["t_ns"][sel]
        assert t[0] == 0 and np.all(np.diff(t) == (1 << steps[p][:-1].astype(np.int64)))
        assert t[-1] + (1 << int(steps[p][-1])) == windows << 23
    # the oracle's judge and fallback for the recorded steps give the recorded samples
    replay = oracle_port.learned_replay(f, r, steps, windows, range(np_))
    o = np.lexsort((rs["t_ns"], rs["pixel"]))
    px, t, v = rs["pixel"][o], rs["t_ns"][o], rs["irradiance"][o]
    bounds = np.searchsorted(px, np.arange(np_ + 1))
    for p in range(np_):
        tp, vp = replay[p]
        assert np.array_equal(t[bounds[p]:bounds[p + 1]], tp), p
        assert np.array_equal(v[bounds[p]:bounds[p + 1]], vp), p
    # the oracle pixel model on those samples, window by window (slot 0 = the previous window's last sample)
    om = oracle_port.Model(resolve("ideal", spec.overrides), f.width, f.height, spec.seed, spec.camera)
    frame = oracle_port.field_frame(f, 0)
    om.init(0, frame)
    carried = frame.copy()
    ids = np.arange(np_, dtype=np.uint32)
    for w in range(windows):
        lo, hi = w << 23, (w + 1) << 23
        rows_t, rows_v, cnt = [], [], np.zeros(np_, np.int32)
        for p in range(np_):
            tp, vp = replay[p]
            sel = (tp > lo) & (tp <= hi)
            rows_t.append(np.r_[lo, tp[sel]])
            rows_v.append(np.r_[carried[p], vp[sel]].astype(np.float32))
            cnt[p] = 1 + int(sel.sum())
            carried[p] = vp[sel][-1]
        starts = np.r_[0, np.cumsum(cnt)[:-1]].astype(np.int64)
        om.advance_runs(ids, np.concatenate(rows_t).astype(np.int64), np.concatenate(rows_v), starts, cnt, hi)
    ref = om.take_events()
    got = m.take_events(with_pixel=True)
    assert len(got["t_cross_ns"]) == len(ref["t_cross_ns"]) > 0
    for kg, kr in (("pixel", "pixel"), ("t_cross_ns", "t_cross_ns"), ("p", "p"), ("label", "label")):
        assert np.array_equal(np.asarray(got[kg]).astype(np.int64), np.asarray(ref[kr]).astype(np.int64)), kg


@pytest.mark.gpu
def test_trained_proposal_halves_the_renders(cuda_lib):
    """Train on fields of three training seeds (expectile tau 0.25), calibrate the margin on a fourth (validation,
    median |dt| <= 8 us), evaluate on a held-out seed: C3's laws and blob density at 320 x 180, 1 s with noise. Renders per pixel at least 2x fewer than the
    plain sampler's, event count within 1 %, median |dt| of matched signal events <= 10 us."""
    import torch

    from ballasim_b200.learned import StepMLP, calibrate_margin, compare_events, renders_and_events, trace_pairs

    w, h = 320, 180
    xs, ys = [], []
    for s in (W.LEARN_TRAIN_SEEDS[0], W.LEARN_TRAIN_SEEDS[1], W.LEARN_TRAIN_SEEDS[3]):
        tw = W.blobs_noise(w, h, s)
        x, y, _ = trace_pairs(tw.sensors[0].field, tw.rules, tw.windows, stride=1, seed=s)
        xs.append(x)
        ys.append(y)
    x, y = torch.cat(xs), torch.cat(ys)
    net = StepMLP(seed=0)
    losses = net.train(x, y, steps=9000, batch=8192, lr=1e-3, seed=1, tau=0.25)
    assert losses[-100:].mean() < 0.2 * losses[:10].mean()
    margin, table = calibrate_margin(net, W.blobs_noise(w, h, W.LEARN_TRAIN_SEEDS[2]), target_median_ns=8000.0)
    ev = W.blobs_noise(w, h, W.LEARN_EVAL_SEED)
    plain_r, plain_ev, _ = renders_and_events(ev)
    learned_r, learned_ev, _ = renders_and_events(ev, net, margin)
    cmp = compare_events(plain_ev, learned_ev)
    cmp_all = compare_events(plain_ev, learned_ev, signal_only=False)
    print(f"margin {margin} (validation {table}); renders/px plain {plain_r:.1f} learned {learned_r:.1f} "
          f"({plain_r / learned_r:.2f}x); {cmp}; all {cmp_all}")
    assert plain_r / learned_r >= 2.0
    assert abs(cmp_all["count_diff"]) <= 0.01
    assert cmp["median_abs_dt_ns"] <= 10_000
    assert not math.isnan(cmp["p90_abs_dt_ns"])
