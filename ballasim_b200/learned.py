"""The learned step proposal: an MLP 16 -> 64 -> 64 -> 1 (ReLU) with BF16 weights and activations and FP32
accumulation, trained and run on the GPU by this package's own tensor-core kernels (no reference counterpart:
BallaSim samples with the plain lattice + midpoint rule only, src/engine/sampling.h).

    x, y, _ = trace_pairs(field, rules, windows)     # (history, step) pairs from the plain sampler's runs
    net = StepMLP(seed=0)
    losses = net.train(x, y, steps=6000)             # Adam, lr 1e-3, batch 8192
    engine.set_proposal(net, margin=0.25)            # the engine now samples with the proposal

Features of a walk point (x = log irradiance of the last 8 walk points, newest first; gaps their log2 spacing):
asinh((x_k - x) 1e4) / 4 and (log2 gap_k - 13) / 10. Target: log2(step / min_dt) of the longest aligned
power-of-two step whose chord stays within eps of the plain run's log irradiance at every run sample inside it.
Device arrays are torch tensors (x: uint16 BF16 bits, n x 16; y: float32).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import _lib
from .fields import Field
from .sampling import field_struct

N_PARAMS = 5313
# Slices of the FP32 parameter vector: W1 [16 in][64 out], b1, W2 [64 in][64 out], b2, W3 [64], b3.
LAYOUT = {"W1": (0, (16, 64)), "b1": (1024, (64,)), "W2": (1088, (64, 64)), "b2": (5184, (64,)),
          "W3": (5248, (64,)), "b3": (5312, ())}


def unpack(params: np.ndarray) -> dict:
    out = {}
    for k, (off, shape) in LAYOUT.items():
        size = int(np.prod(shape)) if shape else 1
        out[k] = np.asarray(params[off:off + size]).reshape(shape) if shape else float(params[off])
    return out


def pack(d: dict) -> np.ndarray:
    p = np.zeros(N_PARAMS, np.float32)
    for k, (off, shape) in LAYOUT.items():
        size = int(np.prod(shape)) if shape else 1
        p[off:off + size] = np.asarray(d[k], np.float32).reshape(-1)
    return p


def _torch():
    import torch

    return torch


def _ptr(t) -> int | None:
    return None if t is None else int(t.data_ptr())


def _check_pairs(x, y=None):
    torch = _torch()
    if not (isinstance(x, torch.Tensor) and x.is_cuda and x.dtype == torch.uint16 and x.dim() == 2
            and x.shape[1] == 16 and x.is_contiguous()):
        raise TypeError("x must be a contiguous CUDA uint16 tensor of shape (n, 16) (BF16 bits)")
    if y is not None and not (isinstance(y, torch.Tensor) and y.is_cuda and y.dtype == torch.float32
                              and y.shape == (x.shape[0],) and y.is_contiguous()):
        raise TypeError("y must be a contiguous CUDA float32 tensor of shape (n,)")


class StepMLP:
    """The proposal network, its FP32 master parameters, Adam state and BF16 operand copies on the device."""

    def __init__(self, seed: int = 0):
        h = C.c_void_p()
        _lib.check(_lib.lib().bs_mlp_create(int(seed), C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        self._h = None
        if h:
            try:
                _lib.lib().bs_mlp_destroy(h)
            except Exception:  # interpreter shutdown
                pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(N_PARAMS, np.float32)
        _lib.check(_lib.lib().bs_mlp_get_params(self._h, p.ctypes.data))
        return p

    @params.setter
    def params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        if p.shape != (N_PARAMS,):
            raise ValueError(f"params must have shape ({N_PARAMS},)")
        _lib.check(_lib.lib().bs_mlp_set_params(self._h, p.ctypes.data))

    @property
    def steps(self) -> int:
        s = C.c_int64()
        _lib.check(_lib.lib().bs_mlp_steps(self._h, C.byref(s)))
        return s.value

    def forward(self, x):
        """MLP(x) for every row (float32 CUDA tensor)."""
        torch = _torch()
        _check_pairs(x)
        y = torch.empty(x.shape[0], dtype=torch.float32, device=x.device)
        _lib.check(_lib.lib().bs_mlp_forward(self._h, _ptr(x), x.shape[0], _ptr(y),
                                             torch.cuda.current_stream().cuda_stream))
        return y

    def gradient(self, x, y) -> tuple[np.ndarray, float]:
        """(dL/dparams, L) for L = sum (MLP(x) - y)^2 / (2 n), from the training kernels."""
        torch = _torch()
        _check_pairs(x, y)
        g = np.zeros(N_PARAMS, np.float64)
        loss = C.c_double()
        _lib.check(_lib.lib().bs_mlp_gradient(self._h, _ptr(x), _ptr(y), x.shape[0], g.ctypes.data, C.byref(loss),
                                              torch.cuda.current_stream().cuda_stream))
        return g, loss.value

    def train(self, x, y, steps: int, batch: int = 8192, lr: float = 1e-3, seed: int = 0,
              tau: float = 0.5) -> np.ndarray:
        """`steps` Adam steps on batches drawn with replacement, on the expectile loss of weight tau (0.5: mean
        squared error; below 0.5 an over-long prediction costs more than a short one); returns every step's batch
        loss."""
        torch = _torch()
        _check_pairs(x, y)
        losses = np.zeros(int(steps), np.float32)
        _lib.check(_lib.lib().bs_mlp_train(self._h, _ptr(x), _ptr(y), x.shape[0], int(steps), int(batch),
                                           float(lr), float(tau), int(seed), losses.ctypes.data,
                                           torch.cuda.current_stream().cuda_stream))
        return losses

    def save(self, path) -> None:
        np.save(Path(path), self.params)

    @classmethod
    def load(cls, path) -> "StepMLP":
        net = cls()
        net.params = np.load(Path(path))
        return net


def trace_pairs(field: Field, rules, windows: int, *, stride: int = 1, eps: float = 1e-4, seed: int = 0,
                t0_ns: int = 0, capacity: int | None = None, keys: bool = False):
    """(x, y, keys) training pairs from the plain sampler over `windows` windows of `field` (rules: a
    workloads.Rules); every stride-th pixel walks its runs. The pairs come back in (pixel, window, step) order, so
    that a dataset (and training on it) is reproducible. capacity defaults to 3 pairs per walked pixel and window
    and is raised and the walk redone when it is not enough."""
    torch = _torch()
    fs = field_struct(field)
    rs = _lib.SampleRules(rules.tol, rules.dark, 1, 1, rules.max_refine_levels, rules.min_dt_ns, rules.l_min,
                          rules.l_max)
    walkers = (field.width * field.height + stride - 1) // stride
    cap = capacity if capacity is not None else max(1024, 3 * walkers * max(1, windows))
    while True:
        x = torch.empty((cap, 16), dtype=torch.uint16, device="cuda")
        y = torch.empty(cap, dtype=torch.float32, device="cuda")
        k = torch.empty(cap, dtype=torch.uint64, device="cuda")
        n_out, total = C.c_size_t(), C.c_size_t()
        _lib.check(_lib.lib().bs_trace_pairs(C.byref(fs), C.byref(rs), int(t0_ns), int(windows), int(stride),
                                             float(eps), int(seed), _ptr(x), _ptr(y), _ptr(k), cap,
                                             C.byref(n_out), C.byref(total),
                                             torch.cuda.current_stream().cuda_stream))
        if total.value <= cap:
            n = n_out.value
            order = torch.argsort(k[:n].view(torch.int64), stable=True)  # keys < 2^63
            x = x[:n].view(torch.int16).index_select(0, order).view(torch.uint16)
            y = y[:n].index_select(0, order)
            k = k[:n].view(torch.int64).index_select(0, order).view(torch.uint64)
            return x, y, (k if keys else None)
        if capacity is not None:
            raise MemoryError(f"trace_pairs: {total.value} pairs exceed the capacity {cap}")
        cap = total.value


def compare_events(ref: dict, other: dict, *, signal_only: bool = True) -> dict:
    """Event-timestamp agreement of two runs of the same sensor (event dicts of SensorModel.take_events): per
    (pixel, polarity) the events are matched one to one in time order wherever both runs hold the same number
    there. signal_only drops NOISE-labelled events (shot and background activity), whose times do not depend on
    the sampling. Returns the event counts, their relative difference, the share of events in (pixel, polarity)
    groups whose counts differ, and the median / 90th percentile |dt| (ns) of the matched events."""

    def prep(ev):
        sel = ev["label"] != 1 if signal_only else np.ones(len(ev["t_cross_ns"]), bool)
        key = ((ev["y"][sel].astype(np.int64) << 20) | ev["x"][sel].astype(np.int64)) * 2 + ev["p"][sel]
        t = ev["t_cross_ns"][sel].astype(np.int64)
        o = np.lexsort((t, key))
        return key[o], t[o]

    ka, ta = prep(ref)
    kb, tb = prep(other)
    ua, ca = np.unique(ka, return_counts=True)
    ub, cb = np.unique(kb, return_counts=True)
    both, ia, ib = np.intersect1d(ua, ub, return_indices=True)
    same = both[ca[ia] == cb[ib]]
    ma, mb = np.isin(ka, same), np.isin(kb, same)
    dt = np.abs(ta[ma] - tb[mb])
    na, nb = len(ta), len(tb)
    return {"events_ref": na, "events": nb, "count_diff": (nb - na) / max(1, na),
            "unmatched_share": 1.0 - (int(ma.sum()) / max(1, na)),
            "median_abs_dt_ns": float(np.median(dt)) if len(dt) else 0.0,
            "p90_abs_dt_ns": float(np.percentile(dt, 90)) if len(dt) else 0.0}


def renders_and_events(workload, proposal=None, margin: float = 0.25):
    """One run of a one-sensor workload from t0 = 0 through the engine: (renders per pixel, events, kernel ms).
    Renders = field evaluations = pixel-samples minus the carried slot of every pixel and window."""
    from .engine import Engine
    from .params import resolve
    from .sensor import SensorModel

    spec, r = workload.sensors[0], workload.rules
    m = SensorModel(resolve(spec.preset, spec.overrides), spec.width, spec.height, spec.seed, [{"type": "constant"}],
                    spec.camera)
    eng = Engine([(m, spec.field)], tol=r.tol, dark=r.dark, min_dt_ns=r.min_dt_ns,
                 max_refine_levels=r.max_refine_levels, l_min=r.l_min, l_max=r.l_max)
    if proposal is not None:
        eng.set_proposal(proposal, margin=margin)
    eng.start(0)
    samples, _ = eng.run(workload.windows)
    px = spec.width * spec.height
    return (samples - workload.windows * px) / px, m.take_events(), eng.last_ms


MARGINS = tuple(round(0.05 * i, 2) for i in range(21))  # 0.0 .. 1.0


def calibrate_margin(net: StepMLP, validation, *, target_median_ns: float = 8000.0, max_count_diff: float = 0.005,
                     margins=MARGINS) -> tuple[float, list]:
    """The smallest margin (the fewest renders) at which the proposal's events on a validation workload (a seed
    neither trained nor evaluated on) stay within the targets against the plain sampler's: median |dt| of matched
    signal events and relative event-count difference. Returns (margin, the table of tried margins); the last
    margin when none meets them."""
    plain_r, plain_ev, _ = renders_and_events(validation)
    table = []
    for mg in margins:
        lr, lev, _ = renders_and_events(validation, net, mg)
        c = compare_events(plain_ev, lev)
        call = compare_events(plain_ev, lev, signal_only=False)
        row = {"margin": mg, "renders_per_px": lr, "plain_renders_per_px": plain_r,
               "median_abs_dt_ns": c["median_abs_dt_ns"], "count_diff": call["count_diff"]}
        table.append(row)
        if c["median_abs_dt_ns"] <= target_median_ns and abs(call["count_diff"]) <= max_count_diff:
            return mg, table
    return margins[-1], table
