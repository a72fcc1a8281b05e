"""Random ragged calls of sample runs for the pixel-model parity tests: per call a random subset of pixels, each
with 0-13 strictly increasing sample times in (t, t_end] (some at the model time itself), values 5-400 (some x3)."""
import numpy as np


def random_calls(rng, n, t0, calls):
    out, t = [], t0
    for _ in range(calls):
        t_end = t + int(rng.integers(1, 3)) * (1 << 23) + int(rng.integers(0, 5000))
        listed = rng.permutation(n)[: int(rng.integers(0, n + 1))].astype(np.uint32)
        ts, vs, cnt = [], [], []
        for _px in listed:
            k = int(rng.integers(0, 14))
            times = np.unique(rng.integers(t, t_end + 1, k))
            if rng.random() < 0.3 and len(times):
                times[0] = t
                times = np.unique(times)
            vals = (rng.uniform(5, 400, len(times)) * rng.choice([1, 1, 1, 3], len(times))).astype(np.float32)
            ts.append(times.astype(np.int64))
            vs.append(vals)
            cnt.append(len(times))
        tt = np.concatenate(ts) if ts else np.zeros(0, np.int64)
        vv = np.concatenate(vs) if vs else np.zeros(0, np.float32)
        starts = np.concatenate([[0], np.cumsum(cnt)[:-1]]).astype(np.int64) if cnt else np.zeros(0, np.int64)
        out.append((listed, tt, vv, t_end, starts, np.array(cnt, np.int32)))
        t = t_end
    return out


def wide_calls(rng, n, t0, calls):
    """random_calls with a tenth of the values 0, a tenth x1000 and a tenth x0.001."""
    out = []
    for ids, tt, vv, t_end, starts, cnt in random_calls(rng, n, t0, calls):
        vv = vv.copy()
        u = rng.random(len(vv))
        vv[u < 0.1] = 0.0
        vv[(u >= 0.1) & (u < 0.2)] *= 1e3
        vv[(u >= 0.2) & (u < 0.3)] *= 1e-3
        out.append((ids, tt, vv.astype(np.float32), t_end, starts, cnt))
    return out
