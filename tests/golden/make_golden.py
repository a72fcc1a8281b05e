"""Generates the golden fixtures of tests/golden/ from the reference's own CPU code (oracle/_ref, compiled from the
reference sources by oracle/build.py). Run from the repository root: ``python tests/golden/make_golden.py``.

Fixtures (numpy .npz, a few hundred KB in all):
- sampler_<case>.npz: WindowEngine<kHost> runs of three consecutive windows (t, irr, offsets, levels);
- chain_<case>.npz: the events of the sampler -> SensorModel chain over whole windows (fp32 precision);
- maps_mismatch.npz: the frozen maps of a sensor with threshold mismatch (fp64).
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from ballasim_b200 import workloads as W  # noqa: E402
from ballasim_b200.params import resolve  # noqa: E402
from oracle.oracle import Ref  # noqa: E402

OUT = Path(__file__).resolve().parent

CASES = {
    "edge": lambda: W.small("edge", 16, 12, 30),
    "blobs": lambda: W.small("blobs", 40, 30, 30),
    "edge64": lambda: W.edge_64x48(),
}


def sampler_case(name, wl):
    spec, r = wl.sensors[0], wl.rules
    from oracle.oracle import Port

    f = spec.field
    n = spec.width * spec.height
    ids = np.arange(n, dtype=np.uint32)
    carried = Port.field_frame(f, 0)
    sig = np.zeros(n, np.uint64)
    out = {}
    for w in range(3):
        t_w = w << 23
        lv = Port.levels(f, t_w, r.l_min, r.l_max)
        t, irr, off, carried, sig = Ref.sample_window(f, r, t_w, ids, lv, carried, sig)
        out[f"t{w}"], out[f"irr{w}"], out[f"off{w}"], out[f"lv{w}"] = t, irr, off, lv
    np.savez_compressed(OUT / f"sampler_{name}.npz", **out)


def chain_case(name, wl):
    spec = wl.sensors[0]
    p = resolve("ideal", spec.overrides)
    m = Ref.Model(p, spec.width, spec.height, spec.seed, spec.camera)
    ev, st = m.simulate(spec.field, wl.rules, wl.windows)
    np.savez_compressed(OUT / f"chain_{name}.npz", windows=wl.windows, pixel_samples=st["pixel_samples"],
                        **{k: v for k, v in ev.items()})


def main():
    for name in ("edge", "blobs"):
        sampler_case(name, CASES[name]())
    for name in ("edge", "blobs", "edge64"):
        chain_case(name, CASES[name]())
    wl = W.small("blobs", 40, 30, 1)
    spec = wl.sensors[0]
    m = Ref.Model(resolve("ideal", spec.overrides), spec.width, spec.height, spec.seed, spec.camera)
    np.savez_compressed(OUT / "maps_mismatch.npz", **m.maps())
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    main()
