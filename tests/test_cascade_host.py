"""The cascade photoreceptor's device code (ballasim_b200/csrc/cascade.cuh, special.cuh, lattice.cuh, noise_build.h)
built for the host with g++ and checked bitwise against the reference's fp32 kernel on the CPU: the special functions
and z_step over wide sweeps, the noise-lattice tables, and the processors on random ragged runs against the
reference's SensorModel (photoreceptor cascade, noise lattice off and on). The same code runs on the device under
nvcc --fmad=false; the gpu tests repeat the model checks there."""
import ctypes as C
import re
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from ballasim_b200.params import resolve
from runs import random_calls, wide_calls

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "ballasim_b200" / "csrc"
EV = np.dtype([("pixel", "u4"), ("p", "u1"), ("label", "u1"), ("flags", "u2"), ("t", "i8"), ("ds", "f4"),
               ("dn", "f4"), ("dl", "f4"), ("l_first", "f4")])


@pytest.fixture(scope="session")
def host(tmp_path_factory):
    so = tmp_path_factory.mktemp("cascade") / "libcascade_host.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-pthread",
                    f"-I{CSRC}", str(ROOT / "tests" / "native" / "cascade_host.cc"), "-o", str(so)], check=True)
    H = C.CDLL(str(so))
    H.hc_create.restype = C.c_void_p
    H.hc_create.argtypes = [C.c_uint32] + [C.c_void_p] * 5 + [C.c_float, C.c_void_p, C.c_int, C.c_int64]
    for f in ("hc_init", "hc_advance", "hc_take", "hc_state", "hc_destroy", "hc_special"):
        getattr(H, f).restype = None
    H.hc_init.argtypes = [C.c_void_p, C.c_int64, C.c_void_p]
    H.hc_advance.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                             C.c_int64]
    H.hc_event_count.restype = C.c_size_t
    H.hc_event_count.argtypes = [C.c_void_p]
    H.hc_take.argtypes = [C.c_void_p, C.c_void_p]
    H.hc_state.argtypes = [C.c_void_p, C.c_void_p]
    H.hc_destroy.argtypes = [C.c_void_p]
    H.hc_special.argtypes = [C.c_int, C.c_void_p, C.c_size_t, C.c_void_p]
    H.hc_noise_table.restype = C.c_int64
    H.hc_noise_table.argtypes = [C.c_double] * 4 + [C.c_int, C.c_int, C.c_void_p, C.c_size_t]
    H.hl_create.restype = C.c_void_p
    H.hl_create.argtypes = [C.c_uint32] + [C.c_void_p] * 5 + [C.c_float, C.c_void_p, C.c_int, C.c_int64, C.c_void_p,
                                                              C.c_int, C.c_uint64, C.c_uint32]
    for f in ("hl_init", "hl_advance", "hl_take", "hl_destroy"):
        getattr(H, f).restype = None
    H.hl_init.argtypes = [C.c_void_p, C.c_int64, C.c_void_p]
    H.hl_advance.argtypes = H.hc_advance.argtypes
    H.hl_event_count.restype = C.c_size_t
    H.hl_event_count.argtypes = [C.c_void_p]
    H.hl_take.argtypes = [C.c_void_p, C.c_void_p]
    H.hl_destroy.argtypes = [C.c_void_p]
    H.hl_stationary.restype = None
    H.hl_stationary.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32]
    return H


def test_special_constants_follow_their_constructions():
    """special.cuh's tables are gen_special.py's output (Weideman, Rybicki, Gauss-Legendre)."""
    sys.path.insert(0, str(CSRC))
    try:
        import gen_special
    finally:
        sys.path.remove(str(CSRC))
    c = gen_special.constants()
    src = (CSRC / "special.cuh").read_text()

    def macro(name):
        body = re.search(rf"#define {name}((?:.*\\\n)*.*)", src).group(1)
        return [float.fromhex(h[:-1]) for h in re.findall(r"-?0x[0-9a-f.]+p[-+]\d+f", body)]

    def const(name):
        return float.fromhex(re.search(rf"constexpr float {name} = (-?0x[0-9a-f.]+p[-+]\d+)f;", src).group(1))

    assert macro("BS_WEIDEMAN_P24") == c["weideman_p24"]
    assert macro("BS_RYBICKI_C") == c["rybicki"]
    assert macro("BS_GL8") == [v for triple in c["gl8"] for v in triple]
    assert const("kWeidemanL24") == c["weideman_L24"]
    assert const("kInvSqrtPi") == c["inv_sqrt_pi"]
    assert const("kHalfSqrtPi") == c["half_sqrt_pi"]


def _special(lib, fn, which, x):
    x = np.ascontiguousarray(x, np.float32)
    n = len(x) if which < 8 else len(x) // 5
    out = np.zeros(n, np.float32)
    fn(which, x.ctypes.data, n, out.ctypes.data)
    return out


def test_special_functions_equal_the_reference(host, ref):
    rng = np.random.default_rng(1)
    L = ref.lib()
    u = np.concatenate([rng.uniform(-2, 2, 40000), rng.uniform(-100, 100, 20000), 10 ** rng.uniform(-12, 2, 20000)])
    y = np.concatenate([rng.uniform(0, 3, 40000), 10 ** rng.uniform(-10, 2, 40000)])
    xs = np.concatenate([rng.uniform(0, 10, 40000), 10 ** rng.uniform(-8, 9, 40000), -rng.uniform(0, 5, 200),
                         [0.0, np.inf, 1e8, 1e9]]).astype(np.float32)
    n = 40000
    z0, I0 = 10 ** rng.uniform(-5, 1, n), 10 ** rng.uniform(-2, 4, n)
    I1 = I0 * np.exp(rng.normal(0, 1, n))
    I1[::3] = I0[::3]
    I1[1::7] = I0[1::7] * (1 + 1e-6)
    zs = np.stack([z0, I0, I1, 10 ** rng.uniform(-9, -1, n), np.full(n, 10.0)], 1).ravel()
    cases = [(0, u)] + [(1 + j, y) for j in range(5)] + [(6, xs), (7, np.concatenate([xs, -xs])), (8, zs)]
    for which, x in cases:
        a = _special(L, L.ref_special, which, x)
        b = _special(host, host.hc_special, which, x)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), which


def cascade_consts(p) -> np.ndarray:
    """cascade_constants<float> and the kernel constants the host build takes (src/sensor/sensor_model.cpp:376-433)."""
    f32 = lambda v: float(np.float32(v))  # noqa: E731
    eps_h = p.eps_L / 8.0
    return np.array([f32(p.k * 1e-15), f32(1.0 / p.tau_o), f32(1.0 / p.tau_sf), f32(p.tau_o), f32(p.tau_sf),
                     f32(eps_h / 1.5), f32(max(eps_h / 1024.0, 32.0 * 2.0 ** -23)), f32(p.eps_L / 8.0), f32(p.eps_ci),
                     f32(p.label_share_cut), f32(1e9 / p.illuminance_scale)], np.float32)


CASES = [
    ("prophesee_gen3", {}, random_calls, 0),
    ("prophesee_gen3", {"leak_rate_hz": 2.0, "leak_sigma_log10": 0.1}, random_calls, 0),
    ("prophesee_gen3", {"reset_mode": "ideal", "refractory_s": 0.0}, random_calls, 0),
    ("prophesee_gen3", {"sigma_theta_on": 0.03, "sigma_theta_off": 0.03, "dark_sigma_ln": 0.5}, wide_calls, 0),
    ("prophesee_gen3", {"leak_rate_hz": 1.0, "refractory_s": 0.0}, wide_calls, -123456789),
    ("prophesee_gen3", {"refractory_s": 1e-3, "eps_L": 0.001}, wide_calls, 0),
    ("samsung_gen3", {}, wide_calls, 0),
]


def _host_vs_reference(host, ref, p, calls, t0, seed, n_calls=6, size=(12, 9)):
    W, Hh = size
    n = W * Hh
    rng = np.random.default_rng(seed)
    model = ref.Model(p, W, Hh, seed)
    irr0 = rng.uniform(5, 400, n).astype(np.float32)
    model.init(t0, irr0)
    mp = model.maps()
    arrs = [np.ascontiguousarray(mp[k], np.float32) for k in ("theta_on", "theta_off", "leak", "dark_current_fA",
                                                               "phi0")]
    cs = cascade_consts(p)
    lattice = bool(p.noise)
    pre = "hl" if lattice else "hc"
    if lattice:
        lat = np.array([p.k * 1.602176634e-19, p.sigma_o, p.noise_margin_z, 1.0 / p.tau_o, 1.0 / p.tau_sf,
                        1.0 if p.noise_diffusion == "transient" else 0.0])
        h = host.hl_create(n, *[a.ctypes.data for a in arrs], float(np.float32(p.illuminance_scale)), cs.ctypes.data,
                           1 if p.reset_mode == "ideal" else 0, int(round(p.refractory_s * 1e9)), lat.ctypes.data,
                           int(p.noise_leaf_level), seed, 0)
    else:
        h = host.hc_create(n, *[a.ctypes.data for a in arrs], float(np.float32(p.illuminance_scale)), cs.ctypes.data,
                           1 if p.reset_mode == "ideal" else 0, int(round(p.refractory_s * 1e9)))
    fn = lambda name: getattr(host, f"{pre}_{name}")  # noqa: E731
    try:
        fn("init")(h, t0, irr0.ctypes.data)
        if lattice and p.initial_state == "stationary":
            maps64 = np.concatenate([mp["theta_on"], mp["theta_off"], mp["leak"]]).astype(np.float64)
            st = np.array([p.k * 1.602176634e-19, 1.0 / p.tau_o, 1.0 / p.tau_sf, p.sigma_o, p.k, p.leak_rate_hz])
            host.hl_stationary(h, t0, irr0.ctypes.data, maps64.ctypes.data, st.ctypes.data,
                               int(p.stationary_burnin_ns), int(p.stationary_probe_pixels))
        want, got = [], []
        for ids, tt, vv, t_end, starts, cnt in calls(rng, n, t0, n_calls):
            model.advance_runs(ids, tt, vv, starts, cnt, t_end)
            fn("advance")(h, ids.ctypes.data, len(ids), np.ascontiguousarray(tt).ctypes.data,
                          np.ascontiguousarray(vv).ctypes.data, np.ascontiguousarray(starts).ctypes.data,
                          np.ascontiguousarray(cnt).ctypes.data, t_end)
            want.append(model.take_events())
            m = np.zeros(fn("event_count")(h), EV)
            fn("take")(h, m.ctypes.data)
            got.append(m[np.lexsort((m["pixel"], m["t"]))])
    finally:
        fn("destroy")(h)
    return W, want, got


@pytest.mark.parametrize("family,overrides,calls,t0", CASES)
def test_cascade_host_equals_the_reference(host, ref, family, overrides, calls, t0):
    p = resolve(family, {"noise": False, **overrides})
    W, want, got = _host_vs_reference(host, ref, p, calls, t0, 5 + len(overrides))
    _same(W, want, got)


def _same(W, want, got):
    e = {k: np.concatenate([x[k] for x in want]) for k in want[0]}
    m = np.concatenate(got)
    assert len(m) == len(e["t_cross_ns"]) > 200
    assert np.array_equal(m["pixel"], e["y"].astype(np.int64) * W + e["x"])
    assert np.array_equal(m["t"], e["t_cross_ns"])
    for k in ("p", "label", "flags"):
        assert np.array_equal(m[k], e[k]), k
    for k in ("ds", "dn", "dl", "l_first"):
        assert np.array_equal(m[k].view(np.uint32), np.asarray(e[k], np.float32).view(np.uint32)), k


def test_noise_tables_equal_the_reference(host, ref):
    """The lattice tables (noise_build.h, long double on the host) are the reference's NoiseTables, bit for bit."""
    L = ref.lib()
    for k, tau_o, tau_sf, sigma_o, levels, split in [(1e16, 25e-6, 100e-6, 0.06, 5, 0), (1e16, 100e-6, 25e-6, 0.06, 3, 0),
                                                     (3e15, 40e-6, 200e-6, 0.02, 7, 0), (1e16, 25e-6, 100e-6, 0.06, 0, 0),
                                                     (1e16, 25e-6, 100e-6, 0.06, 5, 1), (3e15, 40e-6, 200e-6, 0.02, 2, 1)]:
        kq = k * 1.602176634e-19
        cap = 800 * (18 + 47 * levels + 12 + 19 * levels)
        a, b = np.zeros(cap, np.float32), np.zeros(cap, np.float32)
        na = L.ref_noise_table(kq, 1 / tau_o, 1 / tau_sf, sigma_o, levels, split, a.ctypes.data, cap)
        nb = host.hc_noise_table(kq, 1 / tau_o, 1 / tau_sf, sigma_o, levels, split, b.ctypes.data, cap)
        assert na == nb > 0
        assert np.array_equal(a[:na].view(np.uint32), b[:nb].view(np.uint32)), levels


LATTICE_CASES = [
    ("prophesee_gen3", {}, random_calls, 0),
    ("prophesee_gen3", {}, random_calls, 12345),
    ("prophesee_gen3", {"noise_leaf_level": 0}, random_calls, 777),
    ("prophesee_gen3", {"noise_leaf_level": 3, "leak_rate_hz": 2.0, "leak_sigma_log10": 0.1}, wide_calls, 0),
    ("prophesee_gen3", {"noise_leaf_level": 7, "reset_mode": "ideal", "refractory_s": 0.0}, random_calls, -123456789),
    ("prophesee_gen3", {"refractory_s": 0.0, "noise_margin_z": 3.0}, wide_calls, 0),
    ("samsung_gen3", {}, wide_calls, 65536 * 3 + 5),
    ("prophesee_gen3", {"sigma_o": 0.2, "sigma_theta_on": 0.03}, random_calls, 0),
    ("prophesee_gen3", {"noise_diffusion": "transient"}, wide_calls, 0),
    ("prophesee_gen3", {"noise_diffusion": "transient", "noise_leaf_level": 3, "leak_rate_hz": 2.0,
                        "refractory_s": 0.0}, wide_calls, 12345),
    ("samsung_gen3", {"noise_diffusion": "transient", "reset_mode": "ideal", "refractory_s": 0.0}, random_calls,
     -65536 * 5),
]


@pytest.mark.parametrize("family,overrides,calls,t0", LATTICE_CASES)
def test_lattice_host_equals_the_reference(host, ref, family, overrides, calls, t0):
    """The cascade with its noise lattice (frozen diffusion): init mid-cell and on a node, leaf levels 0 to 7, both
    resets, the refractory time, leak, another margin z and sigma_o, negative times."""
    p = resolve(family, {"noise": True, **overrides})
    W, want, got = _host_vs_reference(host, ref, p, calls, t0, 5 + len(overrides) + (t0 & 7))
    _same(W, want, got)


@pytest.mark.parametrize("overrides,t0", [
    ({"stationary_burnin_ns": 500_000_000}, 0),
    ({"stationary_burnin_ns": 300_000_000, "leak_rate_hz": 2.0, "refractory_s": 0.0}, 12345),
    ({"stationary_burnin_ns": 200_000_000, "stationary_probe_pixels": 7, "reset_mode": "ideal"}, -65536 * 9),
])
def test_stationary_start_equals_the_reference(host, ref, overrides, t0):
    """The lattice's stationary initial state (stationary.h: probes, their histories, the transfer) equals the
    reference's (sensor_model.cpp:492-700): the events of the calls after it, bit for bit. The default 60 s history
    is checked on the B200 (test_gpu_parity.py)."""
    p = resolve("prophesee_gen3", {"noise": True, "initial_state": "stationary", **overrides})
    W, want, got = _host_vs_reference(host, ref, p, random_calls, t0, 5 + len(overrides), size=(16, 12))
    _same(W, want, got)
    phase = resolve("prophesee_gen3", {"noise": True, **overrides})
    _, want_phase, _ = _host_vs_reference(host, ref, phase, random_calls, t0, 5 + len(overrides), size=(16, 12))
    n_st, n_ph = (sum(len(x["t_cross_ns"]) for x in w) for w in (want, want_phase))
    first_st = np.concatenate([x["t_cross_ns"] for x in want])[:50]
    first_ph = np.concatenate([x["t_cross_ns"] for x in want_phase])[:50]
    assert n_st != n_ph or not np.array_equal(first_st, first_ph)  # the start does change the events
