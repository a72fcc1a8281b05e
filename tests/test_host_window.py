"""sample_window with a Python callable as the renderer (engine_module.cpp:227-355): the window runs breadth-first on
the host as the reference's WindowEngine<kHost> does, and its runs, carried samples and round statistics equal the
reference's own engine driven by the same callable through the harness. Signature-only rules need no device (the
CPU cases); the midpoint test's triples go to the device (the gpu cases), which also check that a host callable
evaluating the field gives the device-field sampler's runs bit for bit."""
import numpy as np
import pytest

from ballasim_b200 import fields as F
from ballasim_b200 import workloads as W


def _fast_blobs():
    """Small blobs crossing pixels within a window: midpoint flags at coarse lattice levels."""
    return F.blobs(24, 18, 5, 6, r_lo=1.5, r_hi=4.0, v_sigma=3000.0)


def _field_render(port, f, groups=1, step=None):
    """A renderer callable on the oracle's field: group g is the field at t + g x 1 ms scaled by 1 / (g + 1); the
    signature counts the steps of `step` below group 0 (0 everywhere without a step)."""

    def render(pixel, t):
        cols = [port.field_samples(f, pixel, t + g * 1_000_000) / np.float32(g + 1) for g in range(groups)]
        e = np.stack(cols, 1).astype(np.float32)
        s = np.zeros(len(pixel), np.uint64) if step is None else np.floor(e[:, 0] / step).astype(np.uint64)
        return e, s

    return render


def _same_runs(runs, want):
    t, irr, off, ci, cs, st = want
    assert np.array_equal(runs.offsets, off)
    assert np.array_equal(runs.t_ns, t)
    assert np.array_equal(runs.irradiance.view(np.uint32), irr.view(np.uint32))
    assert np.array_equal(runs.last_irradiance.view(np.uint32), ci.view(np.uint32))
    assert np.array_equal(runs.last_signature, cs)
    for k in ("flagged_signature", "flagged_midpoint", "refine_cap_hits", "samples_by_round"):
        assert runs.stats[k] == st[k], k
    assert runs.stats["band_samples_by_round"] == [0] * len(st["samples_by_round"])


def _window_case(port, ref, f, n_px, groups, step, midpoint, refine_signature, max_refine_levels, min_dt_ns,
                 windows=2, listed=False, seed=3, level_cap=8):
    from ballasim_b200.sampling import sample_window

    rng = np.random.default_rng(seed)
    ids = np.arange(n_px, dtype=np.uint32) if not listed else rng.permutation(n_px)[: n_px // 2].astype(np.uint32)
    render = _field_render(port, f, groups, step)
    carried, sig = render(ids, np.zeros(len(ids), np.int64))
    c_ref, s_ref = carried.copy(), sig.copy()
    max_level = 23 - (min_dt_ns.bit_length() - 1)
    rounds = 0
    for w in range(windows):
        t_w = w << 23
        lv = np.minimum(port.levels(f, t_w, 0, level_cap)[ids] + (ids % 3).astype(np.uint8), max_level)
        lv = lv.astype(np.uint8)
        want = ref.sample_window_cb(render, groups, midpoint, refine_signature, max_refine_levels, min_dt_ns, t_w, ids,
                                    lv, c_ref, s_ref)
        runs = sample_window(t_w, ids, lv, np.arange(len(ids)), carried, sig, render,
                             refine_signature=refine_signature, midpoint=midpoint,
                             max_refine_levels=max_refine_levels, min_dt_ns=min_dt_ns)
        _same_runs(runs, want)
        carried, sig = runs.last_irradiance, runs.last_signature
        c_ref, s_ref = want[3], want[4]
        rounds = max(rounds, len(want[5]["samples_by_round"]))
    return rounds


@pytest.mark.parametrize("groups,max_refine_levels,min_dt_ns,listed,fast", [
    (1, 4, 8192, False, False),
    (1, 0, 8192, False, False),
    (3, 6, 1024, True, False),
    (2, 2, 1 << 16, False, False),
    (1, 10, 2048, False, True),
])
def test_signature_refinement_equals_the_reference_engine(oracle_port, ref, groups, max_refine_levels, min_dt_ns,
                                                          listed, fast):
    f = _fast_blobs() if fast else W.small("blobs", 24, 18, 1).sensors[0].field
    rounds = _window_case(oracle_port, ref, f, 24 * 18, groups, 9.0, None, True, max_refine_levels, min_dt_ns,
                          listed=listed, level_cap=2 if fast else 8)
    assert rounds >= min(max_refine_levels, 1) + 1


def test_no_refinement_and_edge_inputs(oracle_port, ref):
    from ballasim_b200.sampling import sample_window

    f = W.small("edge", 16, 8, 1).sensors[0].field
    # Signatures off: the lattice alone, whatever the callable's signatures.
    _window_case(oracle_port, ref, f, 16 * 8, 1, 5.0, None, False, 5, 8192)
    render = _field_render(oracle_port, f)
    empty = sample_window(0, np.zeros(0, np.uint32), np.zeros(0, np.uint8), np.zeros(0, np.uint32),
                          np.zeros((0, 1), np.float32), np.zeros(0, np.uint64), render, refine_signature=True,
                          midpoint=None, max_refine_levels=3, min_dt_ns=8192)
    assert empty.offsets.tolist() == [0] and len(empty.t_ns) == 0 and empty.stats["samples_by_round"] == [0]
    ids = np.arange(4, dtype=np.uint32)
    one = np.ones((4, 1), np.float32)
    with pytest.raises(ValueError):  # a callable that returns the wrong shape
        sample_window(0, ids, np.zeros(4, np.uint8), ids, one, np.zeros(4, np.uint64),
                      lambda p, t: (np.zeros(len(p), np.float32), np.zeros(len(p), np.uint64)),
                      refine_signature=True, midpoint=None, max_refine_levels=1, min_dt_ns=8192)
    with pytest.raises(ValueError):  # a level finer than min_dt_ns allows
        sample_window(0, ids, np.full(4, 11, np.uint8), ids, one, np.zeros(4, np.uint64), render,
                      refine_signature=True, midpoint=None, max_refine_levels=1, min_dt_ns=8192)
    with pytest.raises(TypeError):
        sample_window(0, ids, np.zeros(4, np.uint8), ids, one, np.zeros(4, np.uint64), object(),
                      refine_signature=True, midpoint=None, max_refine_levels=1, min_dt_ns=8192)


@pytest.mark.gpu
@pytest.mark.parametrize("groups,refine_signature,max_refine_levels,min_dt_ns", [
    (1, True, 8, 2048),
    (1, False, 3, 8192),
    (2, True, 5, 4096),
])
def test_midpoint_refinement_equals_the_reference_engine(cuda_lib, oracle_port, ref, groups, refine_signature,
                                                         max_refine_levels, min_dt_ns):
    from ballasim_b200.sampling import MidpointTest

    r = W.small("blobs", 24, 18, 1).rules
    ranges = [(1.0, 1.0), (0.4, 1.0)][:groups]
    mt = MidpointTest(r.tol, r.dark, [a for a, _ in ranges], [b for _, b in ranges])
    rounds = _window_case(oracle_port, ref, _fast_blobs(), 24 * 18, groups, 12.0 if refine_signature else None, mt,
                          refine_signature, max_refine_levels, min_dt_ns, windows=3, listed=groups == 2, level_cap=2)
    assert rounds >= 3


@pytest.mark.gpu
def test_host_callable_equals_the_device_field_sampler(cuda_lib, oracle_port):
    """The same field sampled by the device kernel and by a host callable that evaluates it: the same runs."""
    from ballasim_b200.sampling import MidpointTest, sample_window

    r = W.small("blobs", 24, 18, 1).rules
    f = _fast_blobs()
    n = f.width * f.height
    ids = np.arange(n, dtype=np.uint32)
    mt = MidpointTest(r.tol, r.dark, [1.0], [1.0])
    render = _field_render(oracle_port, f)
    c0 = oracle_port.field_frame(f, 0).reshape(-1, 1)
    s0 = np.zeros(n, np.uint64)
    c_dev, s_dev, c_host, s_host = c0.copy(), s0.copy(), c0.copy(), s0.copy()
    flagged = 0
    for w in range(3):
        t_w = w << 23
        lv = np.minimum(oracle_port.levels(f, t_w, r.l_min, r.l_max), 3)
        kw = dict(refine_signature=True, midpoint=mt, max_refine_levels=r.max_refine_levels, min_dt_ns=r.min_dt_ns)
        dev = sample_window(t_w, ids, lv, ids, c_dev, s_dev, f, **kw)
        host = sample_window(t_w, ids, lv, ids, c_host, s_host, render, **kw)
        assert np.array_equal(dev.offsets, host.offsets)
        assert np.array_equal(dev.t_ns, host.t_ns)
        assert np.array_equal(dev.irradiance.view(np.uint32), host.irradiance.view(np.uint32))
        assert np.array_equal(dev.last_irradiance.view(np.uint32), host.last_irradiance.view(np.uint32))
        assert host.stats["samples_by_round"][0] + n == int(np.sum((1 << lv.astype(np.int64)) + 1))
        c_dev, s_dev = dev.last_irradiance, dev.last_signature
        c_host, s_host = host.last_irradiance, host.last_signature
        flagged += host.stats["flagged_midpoint"]
    assert flagged > 1000


def test_cancel_token_stops_the_window(oracle_port):
    """A CancelToken (engine_module.cpp:1351-1357) set before the window stops it at its batch, with no render call;
    set by the renderer during round 0 it stops the window at the first refinement round."""
    from ballasim_b200.sampling import CancelToken, Cancelled, sample_window

    f = _fast_blobs()
    n = f.width * f.height
    ids = np.arange(n, dtype=np.uint32)
    lv = np.full(n, 2, np.uint8)
    base = _field_render(oracle_port, f, 1, 9.0)
    calls = []
    tok = CancelToken()

    def render(p, t):
        calls.append(len(p))
        tok.set()
        return base(p, t)

    c, s = base(ids, np.zeros(n, np.int64))
    kw = dict(refine_signature=True, midpoint=None, max_refine_levels=4, min_dt_ns=8192)
    with pytest.raises(Cancelled, match="refinement round: cancelled"):
        sample_window(0, ids, lv, ids, c, s, render, cancel=tok, **kw)
    assert calls == [4 * n]
    with pytest.raises(Cancelled, match="batch: cancelled"):
        sample_window(0, ids, lv, ids, c, s, render, cancel=tok, **kw)
    assert calls == [4 * n]


@pytest.mark.parametrize("period_ns,t_w", [(1_000_000, 0), (333_333, 5 << 23), (1 << 23, 3 << 23), (7, -(1 << 23)),
                                           (10 << 23, 2 << 23), (3_000_001, -12345)])
def test_fixed_rate_window_equals_the_reference_engine(oracle_port, ref, period_ns, t_w):
    """fixed_rate_window (engine_module.cpp:356-365): the grid of absolute multiples of the period inside the window,
    then t_w + W, every pixel after its carried sample; runs, carried samples and statistics as the reference's
    WindowEngine<kHost> gives them for the same callable."""
    from ballasim_b200.sampling import fixed_rate_samples, fixed_rate_window

    f = _fast_blobs()
    ids = np.random.default_rng(4).permutation(f.width * f.height)[:100].astype(np.uint32)
    render = _field_render(oracle_port, f, 2, 9.0)
    carried, sig = render(ids, np.full(len(ids), t_w, np.int64))
    if period_ns == 7:  # about 1.2 M samples per pixel: a few pixels only
        ids, carried, sig = ids[:2], carried[:2], sig[:2]
    want = ref.fixed_rate_window_cb(render, 2, period_ns, t_w, ids, carried, sig)
    runs = fixed_rate_window(t_w, ids, np.arange(len(ids)), period_ns, carried, sig, render)
    _same_runs(runs, want)
    assert runs.stats["samples_by_round"] == [len(ids) * fixed_rate_samples(t_w, period_ns)]


@pytest.mark.parametrize("max_refine_levels,min_dt_ns", [(4, 8192), (10, 2048)])
def test_render_calls_follow_the_reference_order(oracle_port, ref, max_refine_levels, min_dt_ns):
    """The render-hook window makes the reference engine's render calls (WindowEngine<kHost>, window_impl.h:462-714):
    the same number of calls, each with the same requests in the same order (the lattice pixel-major and by time,
    then each round's midpoints in interval order), signature refinement with non-zero signatures."""
    from ballasim_b200.sampling import sample_window

    f = _fast_blobs()
    ids = np.random.default_rng(9).permutation(f.width * f.height)[:150].astype(np.uint32)
    base = _field_render(oracle_port, f, 1, 9.0)
    lv = (1 + ids % 4).astype(np.uint8)
    carried, sig = base(ids, np.zeros(len(ids), np.int64))
    assert np.count_nonzero(sig) > 0
    seen = {"ours": [], "ref": []}

    def recorder(key):
        def render(p, t):
            seen[key].append((p.copy(), t.copy()))
            return base(p, t)
        return render

    want = ref.sample_window_cb(recorder("ref"), 1, None, True, max_refine_levels, min_dt_ns, 3 << 23, ids, lv,
                                carried.copy(), sig.copy())
    runs = sample_window(3 << 23, ids, lv, np.arange(len(ids)), carried, sig, recorder("ours"), refine_signature=True,
                         midpoint=None, max_refine_levels=max_refine_levels, min_dt_ns=min_dt_ns)
    _same_runs(runs, want)
    assert len(seen["ours"]) == len(seen["ref"]) == want[5]["render_calls"] >= 2
    for (pa, ta), (pb, tb) in zip(seen["ours"], seen["ref"]):
        assert np.array_equal(pa, pb) and np.array_equal(ta, tb)


def test_window_requests_through_the_c_abi():
    """bs_window_run's requests as a C renderer sees them: 24-byte rows with the camera, flags 0, the pixel, the
    sub-sample range [0, subsamples), the time offset from the window start and the time slot t_off >> log2(min_dt);
    each row's irradiance and signature written at out_index go into the runs; a failing renderer stops the window."""
    import ctypes as C

    from ballasim_b200 import _lib

    L = _lib.lib()
    rows = []

    def fn(_user, req, n, out_index, irr, sig, subsamples):
        idx = np.ctypeslib.as_array(out_index, (n,))
        m = int(idx.max()) + 1
        e = np.ctypeslib.as_array(irr, (m,))
        s = np.ctypeslib.as_array(sig, (m,))
        for i in range(n):
            r = req[i]
            rows.append((r.cam, r.flags, r.pixel, r.k_begin, r.k_count, r.t_off_ns, r.pose_slot, subsamples))
            e[idx[i]] = float(r.pixel) + r.t_off_ns * 1e-6
            s[idx[i]] = r.pixel * 1000 + r.pose_slot
        return 0

    cb = _lib.RENDER_FN(fn)
    h = C.c_void_p()
    _lib.check(L.bs_window_create(1, None, None, C.byref(h)))
    ids = np.array([7, 3, 12], np.uint32)
    lv = np.array([1, 2, 0], np.uint8)
    ci = np.array([1.5, 2.5, 3.5], np.float32)
    cs = np.array([70, 30, 120], np.uint64)
    rules = _lib.WindowRules(0.0, 0.0, 0, 0, 0, 1 << 16, 5, 16, None)
    n_s = C.c_size_t()
    _lib.check(L.bs_window_run(h, 2 << 23, ids.ctypes.data, lv.ctypes.data, 3, ci.ctypes.data, cs.ctypes.data,
                               C.byref(rules), cb, None, C.byref(n_s)))
    assert n_s.value == 3 + 5 + 2 and len(rows) == 2 + 4 + 1
    for cam, flags, px, k0, kn, t_off, slot, sub in rows:
        assert (cam, flags, k0, kn, sub) == (5, 0, 0, 16, 16) and slot == t_off >> 16
    assert [r[2] for r in rows] == [7, 7, 3, 3, 3, 3, 12]
    assert [r[5] for r in rows] == [1 << 22, 1 << 23, 1 << 21, 2 << 21, 3 << 21, 4 << 21, 1 << 23]
    off = np.zeros(4, np.int64)
    t = np.zeros(10, np.int64)
    irr = np.zeros(10, np.float32)
    _lib.check(L.bs_window_runs(h, off.ctypes.data, t.ctypes.data, irr.ctypes.data))
    assert list(off) == [0, 3, 8, 10]
    assert t[0] == 2 << 23 and irr[0] == np.float32(1.5) and t[2] == (2 << 23) + (1 << 23)
    assert irr[2] == np.float32(7 + 8.388608) and ci[0] == irr[2] and cs[0] == 7000 + (1 << 23 >> 16)

    def failing(*_):
        return 3

    bad = _lib.RENDER_FN(failing)
    with pytest.raises(ValueError, match="render callback failed"):
        _lib.check(L.bs_window_run(h, 0, ids.ctypes.data, lv.ctypes.data, 3, ci.ctypes.data, cs.ctypes.data,
                                   C.byref(rules), bad, None, C.byref(n_s)))
    L.bs_window_destroy(h)
