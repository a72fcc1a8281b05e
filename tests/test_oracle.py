"""The oracle (oracle/port, the CPU restatement) pinned before it is trusted: the reference's own known-answer
vectors for Philox and the purpose tags (tests/cpp/test_philox.cpp:11-70), golden fixtures made by the reference's
own code (tests/golden/make_golden.py), and the reference compiled here from its sources (oracle/_ref) on the
same inputs."""
import numpy as np
import pytest

from ballasim_b200 import workloads as W
from ballasim_b200.params import resolve

GOLDEN = __import__("pathlib").Path(__file__).resolve().parent / "golden"

EVENT_KEYS = ("pixel", "p", "label", "flags", "t_cross_ns", "ds", "dn", "dl", "l_first")


def same_events(a: dict, b: dict) -> None:
    assert len(a["t_cross_ns"]) == len(b["t_cross_ns"]), (len(a["t_cross_ns"]), len(b["t_cross_ns"]))
    for k in EVENT_KEYS:
        x, y = np.asarray(a[k]), np.asarray(b[k])
        if x.dtype.kind == "f":
            x, y = x.view(np.uint32), y.view(np.uint32)
        assert np.array_equal(x, y), f"column {k} differs"


# Random123 known-answer vectors (tests/cpp/test_philox.cpp:11-31).
KATS = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]
# Golden first outputs of the purpose tags this path uses (tests/cpp/test_philox.cpp:46-52).
PINS = [(0x0002, 0xCCE173FF, 0xA3C44C71), (0x0022, 0x1F376E45, 0xE68CD7B4)]


@pytest.mark.parametrize("ctr,key,want", KATS)
def test_philox_known_answers(oracle_port, ctr, key, want):
    assert tuple(int(v) for v in oracle_port.philox(ctr, key)) == want


@pytest.mark.parametrize("purpose,origin,word2", PINS)
def test_purpose_tag_golden_outputs(oracle_port, purpose, origin, word2):
    assert int(oracle_port.draw(0, purpose, 0, 0, 0)[0]) == origin
    assert int(oracle_port.draw(0x0123456789ABCDEF, purpose, 2, 307199, 65536)[2]) == word2


def test_logf_matches_reference_method_on_a_sweep(oracle_port):
    """pmath::log fp32 (explog.h:214-225) is within 3 ulp of the correctly rounded log, and exact at 1."""
    L = oracle_port.lib()
    xs = np.exp(np.linspace(-20, 20, 4001)).astype(np.float32)
    got = np.array([L.orc_logf(float(x)) for x in xs], np.float32)
    want = np.log(xs.astype(np.float64)).astype(np.float32)
    ulp = np.abs(got.view(np.int32).astype(np.int64) - want.view(np.int32).astype(np.int64))
    assert ulp.max() <= 3
    assert L.orc_logf(1.0) == 0.0


@pytest.mark.parametrize("case", ["edge", "blobs"])
def test_sampler_matches_golden(oracle_port, case):
    g = np.load(GOLDEN / f"sampler_{case}.npz")
    wl = W.small("edge", 16, 12, 3) if case == "edge" else W.small("blobs", 40, 30, 3)
    spec, r = wl.sensors[0], wl.rules
    n = spec.width * spec.height
    ids = np.arange(n, dtype=np.uint32)
    carried = oracle_port.field_frame(spec.field, 0)
    sig = np.zeros(n, np.uint64)
    for w in range(3):
        lv = oracle_port.levels(spec.field, w << 23, r.l_min, r.l_max)
        assert np.array_equal(lv, g[f"lv{w}"])
        t, irr, off, carried, sig = oracle_port.sample_window(spec.field, r, w << 23, ids, lv, carried, sig)
        assert np.array_equal(off, g[f"off{w}"])
        assert np.array_equal(t, g[f"t{w}"])
        assert np.array_equal(irr.view(np.uint32), g[f"irr{w}"].view(np.uint32))


@pytest.mark.parametrize("case", ["edge", "blobs", "edge64"])
def test_chain_matches_golden(case):
    from oracle.oracle import simulate_port

    wl = {"edge": lambda: W.small("edge", 16, 12, 30), "blobs": lambda: W.small("blobs", 40, 30, 30),
          "edge64": W.edge_64x48}[case]()
    g = np.load(GOLDEN / f"chain_{case}.npz")
    ev, st = simulate_port(wl.sensors[0], wl.rules, wl.windows)
    assert st["pixel_samples"] == int(g["pixel_samples"])
    same_events(ev, g)
    assert len(ev["t_cross_ns"]) > 50


def test_maps_match_golden(oracle_port):
    wl = W.small("blobs", 40, 30, 1)
    spec = wl.sensors[0]
    m = oracle_port.Model(resolve("ideal", spec.overrides), spec.width, spec.height, spec.seed)
    g = np.load(GOLDEN / "maps_mismatch.npz")
    got = m.maps()
    for k in ("theta_on", "theta_off", "leak", "dark_current_fA", "phi0"):
        assert np.array_equal(got[k], g[k]), k
    assert np.std(got["theta_on"]) > 0.01  # the mismatch draws are live


@pytest.mark.parametrize("overrides", [
    {},                                                           # ideal reset, no refractory
    dict(W.MISMATCH),                                             # physical reset with refractory, mismatch
    {**W.MISMATCH, "leak_rate_hz": 2.0, "leak_sigma_log10": 0.1},  # leak (the non-monotone exclusion branch)
    {"reset_mode": "physical", "refractory_s": 0.0, "eps_ci": 0.002, "initial_phase": "symmetric"},
])
def test_port_equals_reference_on_random_runs(oracle_port, ref, overrides):
    """Ragged random runs (empty, single-sample, sample at the model time, sparse and dense), unlisted pixels,
    over several calls: the port's events equal the reference's bit for bit."""
    rng = np.random.default_rng(len(str(overrides)))
    W_, H_ = 12, 10
    n = W_ * H_
    p = resolve("ideal", overrides)
    a = oracle_port.Model(p, W_, H_, 5, 0)
    b = ref.Model(p, W_, H_, 5, 0)
    irr0 = rng.uniform(20, 200, n).astype(np.float32)
    a.init(0, irr0)
    b.init(0, irr0)
    t = 0
    for call in range(6):
        t_end = t + int(rng.integers(1, 3)) * (1 << 23) + int(rng.integers(0, 5000))
        listed = rng.permutation(n)[: int(rng.integers(0, n))].astype(np.uint32)
        ts, vs, starts, counts = [], [], [], []
        pos = 0
        for px in listed:
            k = int(rng.integers(0, 12))
            times = np.unique(rng.integers(t, t_end + 1, k))
            if rng.random() < 0.3 and len(times):
                times[0] = t  # a sample at the model time replaces the held one
                times = np.unique(times)
            vals = (rng.uniform(5, 400, len(times)) * rng.choice([1, 1, 1, 3], len(times))).astype(np.float32)
            ts.append(times.astype(np.int64))
            vs.append(vals)
            starts.append(pos)
            counts.append(len(times))
            pos += len(times)
        tt = np.concatenate(ts) if ts else np.zeros(0, np.int64)
        vv = np.concatenate(vs) if vs else np.zeros(0, np.float32)
        args = (listed, tt, vv, np.array(starts, np.int64), np.array(counts, np.int32), t_end)
        a.advance_runs(*args)
        b.advance_runs(*args)
        t = t_end
    ea, eb = a.take_events(), b.take_events()
    same_events(ea, eb)
    assert len(ea["t_cross_ns"]) > 0


def test_port_refuses_what_the_reference_refuses(oracle_port, ref):
    p = resolve("ideal", {})
    for M in (oracle_port.Model, ref.Model):
        m = M(p, 4, 4, 1, 0)
        m.init(100, np.full(16, 50, np.float32))
        ok = (np.array([1], np.uint32), np.array([200], np.int64), np.array([60], np.float32),
              np.array([0], np.int64), np.array([1], np.int32), 1000)
        m.advance_runs(*ok)
        bad = [
            (np.array([1], np.uint32), np.array([900], np.int64), np.array([60], np.float32),
             np.array([0], np.int64), np.array([1], np.int32), 800),      # after t_end
            (np.array([1, 1], np.uint32), np.array([1200, 1300], np.int64), np.array([60, 60], np.float32),
             np.array([0, 1], np.int64), np.array([1, 1], np.int32), 2000),  # duplicate id
            (np.array([2], np.uint32), np.array([1300, 1300], np.int64), np.array([60, 60], np.float32),
             np.array([0], np.int64), np.array([2], np.int32), 2000),     # not strictly increasing
            (np.array([99], np.uint32), np.array([1300], np.int64), np.array([60], np.float32),
             np.array([0], np.int64), np.array([1], np.int32), 2000),     # id out of range
        ]
        for b in bad:
            with pytest.raises(ValueError):
                m.advance_runs(*b)


@pytest.mark.parametrize("family,overrides", [
    ("ideal", {}), ("ideal", {"theta_on": 0.25, "sigma_theta_on": 0.03}), ("prophesee_gen3", {}),
    ("samsung_gen3", {}), ("prophesee_gen3", {"noise": 0.0}), ("ideal", {"reset_mode": 0.0, "refractory_s": 1e-4}),
    ("prophesee_gen3", {"noise_diffusion": 1.0, "initial_state": 1.0, "stationary_burnin_ns": 3e8}),
    ("ideal", {"clock_offset_ns": 12345, "initial_phase": 1.0, "leak_rate_hz": 0.1, "leak_sigma_log10": 0.0}),
    ("prophesee_gen3", {"noise_leaf_level": 3, "noise_margin_z": 5.0, "eps_L": 0.001, "hot_fraction": 0.0}),
    ("samsung_gen3", {"photoreceptor": 1.0, "noise": 0.0, "dark_current_fA": 0.5, "temperature_K": 310.0}),
])
def test_parameter_fingerprint_equals_the_reference(ref, family, overrides):
    """params.fingerprint restates the reference's fingerprint (src/sensor/params.cpp:246) bit for bit: saved states
    carry it and a state loads only where it matches."""
    from ballasim_b200.params import fingerprint

    enums = {"reset_mode": ("physical", "ideal"), "initial_phase": ("uniform", "symmetric", "zero"),
             "noise_diffusion": ("frozen", "transient"), "initial_state": ("phase", "stationary"),
             "photoreceptor": ("cascade", "instantaneous")}
    ints = {"clock_offset_ns", "noise_leaf_level", "stationary_burnin_ns"}
    ours = {k: enums[k][int(v)] if k in enums else bool(v) if k == "noise" else int(v) if k in ints else v
            for k, v in overrides.items()}
    assert fingerprint(resolve(family, ours)) == ref.fingerprint(family, overrides)
    # this project's own noise rows change it only when set
    assert fingerprint(resolve(family, {**ours, "noise_shot_rate_hz": 0.5})) != fingerprint(resolve(family, ours))
