"""Benchmark of the per-pixel event-generation path: pixel-samples/s and events/s on B200s.

One step = one pass of the hot path over the workload: every sensor initialized at t0 from its seeded analytic
field, then every window sampled (dyadic lattice + eta_L refinement) and sensed (the instantaneous pixel model, or
the cascade photoreceptor in workloads blobs_346x260_cascade and, with its noise lattice, blobs_346x260_lattice), in
the fused engine. At N = 1 the workload is the largest one-GPU configuration: six sensors (346x260, 640x480 x2,
1280x720 x2, 1920x1080; 4,621,160 px), 128 blobs each, thresholds per sensor, mismatch, leak, shot and
background-activity noise, 0.5 s (60 windows), in one persistent launch; --workload picks another. With N GPUs
(torchrun, one rank per GPU) each rank runs its own replica of the workload (independent sensors, seeds offset by
rank): weak scaling, no collective on the data path; value = all ranks' pixel-samples / the slowest rank's device
time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

The runs_* workloads take the reference engine's own two-kernel route instead (Camera::sample_and_sense): per
sensor and window, sample_window on the device writes CSR runs to HBM and SensorModel::advance_device reads them
(ballasim_b200.windows); the roofline line is then the pixel model on the runs (advance_rows_kernel, or
advance_runs_kernel with --block).

--impl reference times the reference's own CPU implementation (oracle/_ref: WindowEngine<kHost> and
SensorModel fp32 on every host core) on a bounded sample of the same workload (the first windows of every
sensor), rank 0 only, with its fp64 kernel timed once on the same sample beside it.

The sink_* workloads measure the event file sink instead: one step writes a whole RAW (EVT 2.0, 2.1, 3.0) or DAT
file of a seeded 1280 x 720 stream of 32 Mi events (about 50 Mev/s, runs along rows; workloads.event_stream): the
writer made, the columns appended (device-resident for `value`, pinned host columns for `e2e`), the file closed
and hashed. Metric events/s; the reference arm runs the reference's own RawWriter / DatWriter on one host core.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from ballasim_b200 import workloads as W  # noqa: E402
from ballasim_b200.replicas import reduce_max, reduce_step, replica  # noqa: E402

WORKLOADS = {
    "blobs_346x260": W.blobs_346x260,
    "edge_64x48": W.edge_64x48,
    "blobs_1280x720": W.blobs_1280x720,
    "six_sensors": W.six_sensors,
    "blobs_346x260_cascade": W.blobs_346x260_cascade,
    "blobs_346x260_lattice": W.blobs_346x260_lattice,
}
# The same workloads through the reference engine's two-kernel route (runs in HBM).
RUNS = {"runs_six_sensors": W.six_sensors, "runs_blobs_346x260": W.blobs_346x260,
        "runs_blobs_1280x720": W.blobs_1280x720}
DEFAULT_WORKLOAD = "six_sensors"
# The reference arm's bounded sample: the first windows of every sensor.
CPU_WINDOWS = {"six_sensors": 2, "runs_six_sensors": 2, "blobs_1280x720": 4, "runs_blobs_1280x720": 4}
CPU_WINDOWS_DEFAULT = 40
N_SMS, SCHEDULERS_PER_SM = 148, 4
METRIC = "pixel-samples/s"
SINKS = {"sink_evt3_1280x720": "evt3", "sink_evt21_1280x720": "evt21", "sink_evt2_1280x720": "evt2",
         "sink_dat_1280x720": "dat"}
L2_BYTES = 126 * 1024 * 1024
# Per workload, figures of ncu captures of the dominant kernel of this bench's own command, each kept beside the
# kernel name and launch shape it was taken at: DRAM bytes read + written per launch, warp instructions issued per
# pixel-sample, and ncu's issue-slot activity. A run whose kernel or launch shape matches no capture reports null.
NCU = {
    "blobs16_346x260": [{"kernel": "engine_kernel_coop", "stage": 64, "tile_width": 8,
                         "traffic": 8.74e6 + 4.56e6, "inst_per_sample": None, "issue_active": 0.285}],
    # traffic: one pass on the full 60-window launch; instructions and issue-active: the full set on its first 4
    # windows (74,251,870 pixel-samples).
    "six_sensors_4.6Mpx": [
        # The split engine: one pass over all 120 launches of a step (traffic, instructions: the step's sums);
        # issue-active: the two kernels' full-set figures on one window, weighted by their time (that full set was
        # taken while the posted records were one struct per pixel rather than planes).
        {"kernel": "engine_window_kernel+engine_rest_kernel", "stage": 1, "tile_width": 8,
         "traffic": (32.41e9 + 0.5452e9 + 6.498e9) + (19.34e9 + 0.3281e9 + 3.512e9),
         "inst_per_sample": (3.488e10 + 6.022e8 + 1.819e9) / 1103436116, "issue_active": 0.471},
        {"kernel": "engine_kernel_staged<16>", "stage": 16, "tile_width": 8, "traffic": 690.74e6 + 3.59e9,
         "inst_per_sample": 3.329e9 / 74251870, "issue_active": 0.209},
        {"kernel": "engine_kernel_staged<16>", "stage": 16, "tile_width": 4, "traffic": 694.48e6 + 3.67e9,
         "inst_per_sample": 3.3297e9 / 74251870, "issue_active": 0.210},
    ],
    # The runs path: its six advance_rows_kernel launches of one window (one per sensor), DRAM bytes against the
    # window's algorithmic bytes (836.3 MB read + 325.6 MB written; 833.9 MB).
    "runs:six_sensors_4.6Mpx": [
        {"kernel": "advance_rows_kernel", "dram_per_alg_byte": (836.32e6 + 325.60e6) / 833.92e6,
         "capture": "advance_rows_kernel, the six sensors' first window (6 launches, one pass)"},
        {"kernel": "advance_rows_split_kernel+advance_rows_rest_kernel",
         "dram_per_alg_byte": (2.7952e9 + 1.1218e9) / 2.5016e9,
         "capture": "the split kernels (the split kernel at 64 registers), the six sensors' first 3 windows "
                    "(36 launches, one pass)"},
    ],
}


def ncu_capture(name: str, kernel: str, stage=None, tile_width=None):
    """The capture of NCU[name] taken at this kernel and launch shape (stage and tile width where given), or None."""
    for cap in NCU.get(name, []):
        if cap["kernel"] == kernel and (stage is None or cap.get("stage") == stage) and \
                (tile_width is None or cap.get("tile_width") == tile_width):
            return cap
    return None


FALLBACK_HBM_GBS = 6650.0


def measured_hbm() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class Clocks:
    """nvidia-smi clock and throttle samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        self.file.flush()
        rows = [r.split(",") for r in Path(self.file.name).read_text().splitlines() if r.strip()]
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for name, v in zip(names, r[5:9]):
                    if v.strip().lower() in ("active", "1"):
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def b_sense(pixels: int, windows: int, samples: int, events: int) -> int:
    """Algorithmic bytes of the pixel model over the run, per window call at the reference's DeviceRuns boundary:
    12 B per pixel-sample (i64 t + f32 irr), 12 B per listed run, 2 x 48 B of state and 24 B of map per pixel, and
    16 B per compact event."""
    return samples * 12 + windows * pixels * (12 + 2 * 48 + 24) + events * 16


def compute_fraction(wl_name: str, kernel: str, launch: dict, samples: float, kms: float, sm_mhz) -> dict:
    """The issue-slot side of the roofline: warp instructions issued per launch (ncu's count per pixel-sample at the
    captured launch shape, times this launch's pixel-samples) over the SMs' issue slots in the launch's duration at
    the sampled median SM clock (148 SMs x 4 schedulers x cycles), with ncu's own issue-active beside it."""
    cap = ncu_capture(wl_name, kernel, launch.get("stage"), launch.get("tile_width"))
    same = cap is not None
    out = {"ncu_capture": f"{cap['kernel']} stage {cap['stage']} tile {cap['tile_width']}" if cap else None,
           "same_launch_shape": bool(same), "warp_inst_per_launch": None, "issue_slots_per_launch": None,
           "issue_frac": None, "ncu_issue_active": cap.get("issue_active") if same else None}
    if sm_mhz:
        out["issue_slots_per_launch"] = N_SMS * SCHEDULERS_PER_SM * kms * 1e-3 * sm_mhz * 1e6
    if same and cap.get("inst_per_sample") and sm_mhz:
        out["warp_inst_per_launch"] = cap["inst_per_sample"] * samples
        out["issue_frac"] = out["warp_inst_per_launch"] / out["issue_slots_per_launch"]
    return out


def engine_kernel_name(eng, cascade: bool, lattice: bool) -> str:
    if cascade:
        return "engine_lattice_kernel" if lattice else "engine_cascade_kernel"
    return {64: "engine_kernel_coop", 16: "engine_kernel_staged<16>", 32: "engine_kernel_staged<32>",
            1: "engine_window_kernel+engine_rest_kernel"}.get(eng.launch["stage"], "engine_kernel")


def engine_launches(eng, windows: int) -> int:
    """The engine's kernel launches in one step: one persistent launch, or two per window for the split engine."""
    return 2 * windows if eng.launch["stage"] == 1 else 1


def run_ours(args, rank: int, world: int) -> dict | None:
    import torch
    import torch.distributed as dist

    from ballasim_b200 import _lib
    from ballasim_b200.engine import Engine
    from ballasim_b200.params import resolve
    from ballasim_b200.sampling import field_frame
    from ballasim_b200.sensor import SensorModel

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    if not _lib.cuda_available():
        raise RuntimeError("bench: no B200 visible")
    wl = replica(WORKLOADS[args.workload](), rank)
    if args.windows:
        wl.windows = min(wl.windows, args.windows)
    r = wl.rules
    models = [SensorModel(resolve(s.preset, s.overrides), s.width, s.height, s.seed, [{"type": "constant"}], s.camera)
              for s in wl.sensors]
    p0 = resolve(wl.sensors[0].preset, wl.sensors[0].overrides)
    cascade, lattice = p0.photoreceptor == "cascade", p0.photoreceptor == "cascade" and bool(p0.noise)
    eng = Engine([(m, s.field) for m, s in zip(models, wl.sensors)], tol=r.tol, dark=r.dark, min_dt_ns=r.min_dt_ns,
                 max_refine_levels=r.max_refine_levels, l_min=r.l_min, l_max=r.l_max)
    if args.warps or args.blocks_per_sm or args.stage or args.tile_width:
        eng.set_launch(args.warps, args.blocks_per_sm, args.stage, args.tile_width)
    eng.set_graph(not args.no_graph)
    tuned = None
    if not (args.no_autotune or args.warps or args.stage or args.tile_width):
        eng.start(0, torch.cuda.current_stream().cuda_stream)
        tuned = eng.autotune(wl.windows, torch.cuda.current_stream().cuda_stream)  # trial steps of the full run
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")

    def step():
        eng.start(0, sptr)
        return eng.run(wl.windows, sptr)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    kernel_ms, samples, events = [], 0, 0
    with Clocks(torch.cuda.current_device()) as clk:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()  # L2 flush between steps (a write larger than L2), outside the step's events
            starts[k].record(stream)
            s, e = step()
            ends[k].record(stream)
            kernel_ms.append(eng.last_ms)
            samples += s
            events += e
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    step_ms = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    total_ms = float(sum(step_ms))
    total_ms_all, samples_all, events_all = reduce_step(total_ms, float(samples), float(events), world)
    clocks = {k: v for k, v in clk.summary().items() if k != "samples"}

    # e2e through the public API with host buffers: the initial frames from pinned host memory in, every event out;
    # each phase timed on the host after a synchronize, for the split of the e2e step.
    frames = [torch.from_numpy(field_frame(s.field, 0)).pin_memory().numpy() for s in wl.sensors]
    e2e_times, d2h = [], 0
    split = {"start_ms": 0.0, "run_ms": 0.0, "take_events_ms": 0.0, "take_sort_split_ms": 0.0,
             "take_copy_out_ms": 0.0, "take_host_copy_ms": 0.0, "take_download_ms": 0.0}
    for k in range(0 if args.profile else args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.start(0, sptr, frames=frames)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        eng.run(wl.windows, sptr)
        t2 = time.perf_counter()
        n_ev, parts = 0, np.zeros(4)
        for m, cols in zip(models, eng.take_events()):  # every sensor's take, overlapped
            n_ev += len(cols["t_cross_ns"])
            parts += np.array(list(m.take_timing().values()))
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        if k >= args.warmup:
            e2e_times.append(t3 - t0)
            d2h = n_ev * 32
            for key, v in zip(split, (1e3 * (t1 - t0), 1e3 * (t2 - t1), 1e3 * (t3 - t2), *parts)):
                split[key] += v / args.steps
    e2e_s = reduce_max(sum(e2e_times), world)
    h2d = sum(int(f.nbytes) for f in frames)

    if rank != 0:
        return None
    pixels = wl.pixels
    per_step_samples = samples / args.steps
    per_step_events = events / args.steps
    hbm, hbm_kind = measured_hbm()
    kms = statistics.mean(kernel_ms)
    alg = b_sense(pixels, wl.windows, int(per_step_samples), int(per_step_events))
    achieved = alg / (kms * 1e-3) / 1e9
    kname = engine_kernel_name(eng, cascade, lattice)
    cap = ncu_capture(wl.name, kname, eng.launch["stage"], eng.launch["tile_width"])
    same_shape = cap is not None
    out = {
        "metric": METRIC,
        "value": samples_all / (total_ms_all * 1e-3),
        "unit": "pixel-samples/s",
        "events_per_s": events_all / (total_ms_all * 1e-3),
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms_all / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32",
        "data": "synthetic (seeded analytic irradiance fields evaluated on the device)",
        "config": {**wl.describe(), "pixel_samples_per_step": int(per_step_samples),
                   "events_per_step": int(per_step_events), "l2": "flushed between steps (256 MiB write)",
                   "sampler": {"tol": r.tol, "min_dt_ns": r.min_dt_ns, "max_refine_levels": r.max_refine_levels,
                               "levels": [r.l_min, r.l_max]},
                   "parallelism": f"replicas x{world}", "path": "fused engine (runs kept on chip)",
                   "launch": {**eng.launch, "autotuned": tuned is not None, "cuda_graph": not args.no_graph,
                              "threads_per_pixel": 1}},
        # Per step: the first frame and init of every sensor (field_frame_kernel, init_kernel), then the engine.
        "gpu_launches": (2 * len(wl.sensors) + engine_launches(eng, wl.windows)) * args.steps,
        "clocks": clocks,
        "e2e": {"value": samples_all / e2e_s if e2e_times else None, "unit": "pixel-samples/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "split_ms_per_step": {k: round(v, 3) for k, v in split.items()}},
        "roofline": {"kernel": kname + " (sampler + pixel model fused, runs kept on chip)"
                     + (" (per window: the common path, then the posted pixels' rare paths; avg_launch_ms is the "
                        "step's engine time, all windows)" if eng.launch["stage"] == 1 else ""),
                     "bound": "issue",
                     "bound_note": "SIMT fp32 issue and latency (field exps, one log per sample, each crossing's "
                                   "search and fire), not HBM; achieved/peak/frac are the algorithmic bytes of the "
                                   "pixel model (B_sense) over the measured HBM copy bandwidth",
                     "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_kind": hbm_kind, "traffic": cap["traffic"] if same_shape else None,
                     "algorithmic_bytes_per_launch": alg, "avg_launch_ms": kms,
                     "runs_write_avoided_bytes": int(per_step_samples) * 12,
                     "compute": compute_fraction(wl.name, kname, eng.launch, per_step_samples, kms,
                                                 clocks.get("sm_mhz"))},
    }
    if world == 1 and not (args.no_cpu_baseline or args.profile):
        out["cpu_baseline"] = cpu_baseline(wl, cpu_windows(args))
    if rank == 0 and not (args.no_learned or args.profile):
        out["learned_vs_plain"] = learned_comparison(steps=args.learned_steps)
    return out


def run_runs(args, rank: int, world: int) -> dict | None:
    """The reference engine's route with the runs in HBM (ballasim_b200.windows.DeviceWindows): per sensor and
    window, the levels, sample_window on the device (the walk, the scan, the placement) and advance_device (the split
    row-major kernel); the events stay on the device. The sensors run each on its own stream and host thread (or,
    with --window-major, in turn on one stream). Kernel time of the pixel model from CUDA events around each advance
    launch, in window-major steps."""
    import torch
    import torch.distributed as dist

    from ballasim_b200 import _lib
    from ballasim_b200.params import resolve
    from ballasim_b200.sensor import SensorModel
    from ballasim_b200.windows import DeviceWindows

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    if not _lib.cuda_available():
        raise RuntimeError("bench: no B200 visible")
    wl = replica(RUNS[args.workload](), rank)
    if args.windows:
        wl.windows = min(wl.windows, args.windows)
    r = wl.rules
    models = [SensorModel(resolve(s.preset, s.overrides), s.width, s.height, s.seed, [{"type": "constant"}], s.camera)
              for s in wl.sensors]
    for m in models:
        if args.block:
            m.set_block(args.block)
        if args.long_run:
            m.set_long_run(args.long_run)
    dw = DeviceWindows([(m, s.field) for m, s in zip(models, wl.sensors)], tol=r.tol, dark=r.dark,
                       min_dt_ns=r.min_dt_ns, max_refine_levels=r.max_refine_levels, l_min=r.l_min, l_max=r.l_max)
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")

    def step(concurrent=not args.window_major):
        dw.start(0, sptr)
        return dw.run(wl.windows, sptr, concurrent=concurrent)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    samples = events = 0
    dw.launch_ms = 0.0
    launches0 = sum(m.stats()["gpu_launches"] for m in models)
    with Clocks(torch.cuda.current_device()) as clk:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()
            starts[k].record(stream)
            s_, e_ = step()
            ends[k].record(stream)
            samples += s_
            events += e_
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    advance_launches = sum(m.stats()["gpu_launches"] for m in models) - launches0
    timed_launch_ms = dw.launch_ms
    if not args.window_major:
        # The pixel model's kernel times for the roofline from window-major steps on one stream (the sensors'
        # streams overlap their kernels, so each launch's events would also time the other sensors' work).
        dw.launch_ms = 0.0
        for _ in range(args.steps):
            step(concurrent=False)
        torch.cuda.synchronize()
        timed_launch_ms = dw.launch_ms
    step_ms = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    total_ms = float(sum(step_ms))
    total_ms_all, samples_all, events_all = reduce_step(total_ms, float(samples), float(events), world)
    clocks = {k: v for k, v in clk.summary().items() if k != "samples"}

    # e2e through the public API with host buffers: the initial frames from pinned host memory in, per window and
    # sensor every event downloaded to host columns.
    from ballasim_b200.sampling import field_frame

    frames = [torch.from_numpy(field_frame(s.field, 0)).pin_memory().numpy() for s in wl.sensors]
    e2e_times, d2h = [], 0
    for k in range(0 if args.profile else args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dw.start(0, sptr, frames=frames)
        n_ev = [0] * len(models)  # one count per sensor: each sensor's calls come from one thread

        def take(i, m, ev):
            n_ev[i] += len(m.download_events(ev)["t_cross_ns"])

        dw.run(wl.windows, sptr, on_events=take, concurrent=not args.window_major)
        torch.cuda.synchronize()
        if k >= args.warmup:
            e2e_times.append(time.perf_counter() - t0)
            d2h = sum(n_ev) * 32
    e2e_s = reduce_max(sum(e2e_times), world)
    if rank != 0:
        return None
    per_step_samples = samples / args.steps
    per_step_events = events / args.steps
    hbm, hbm_kind = measured_hbm()
    kms_total = timed_launch_ms / args.steps  # the pixel model's kernels, per step
    n_launch = advance_launches / args.steps
    alg = b_sense(wl.pixels, wl.windows, int(per_step_samples), int(per_step_events))
    achieved = alg / (kms_total * 1e-3) / 1e9
    kname = {0: "advance_rows_split_kernel+advance_rows_rest_kernel", 1: "advance_rows_kernel"}.get(
        args.block, "advance_runs_kernel")
    cap = ncu_capture("runs:" + wl.name, kname)
    calls = wl.windows * len(wl.sensors)
    return {
        "metric": METRIC, "value": samples_all / (total_ms_all * 1e-3), "unit": "pixel-samples/s",
        "events_per_s": events_all / (total_ms_all * 1e-3), "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms_all / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
        "data": "synthetic (seeded analytic irradiance fields evaluated on the device)",
        "config": {**wl.describe(), "pixel_samples_per_step": int(per_step_samples),
                   "events_per_step": int(per_step_events), "l2": "flushed between steps (256 MiB write)",
                   "path": "sample_window (device) -> runs in HBM -> advance_device, per sensor and window",
                   "sensors_run": "window-major on one stream" if args.window_major
                   else "each on its own stream and host thread",
                   "parallelism": f"replicas x{world}", "advance_block": args.block or "row-major",
                   "long_run": args.long_run or 32},
        # Per sensor and window: levels, two sample_window passes (the walk, which also checks the inputs, and the
        # placement), three scan kernels and the pixel model (the split row-major kernel's two launches, --block 1
        # one, --block n > 1 the scatter and one; every pixel is listed, so no advance_unlisted_kernel); per sensor
        # and step the first frame and init.
        "gpu_launches": (6 + (1 if args.block == 1 else 2)) * calls * args.steps + 2 * len(wl.sensors) * args.steps,
        "clocks": clocks,
        "e2e": {"value": samples_all / e2e_s if e2e_times else None, "unit": "pixel-samples/s",
                "h2d_bytes_per_step": sum(int(f.nbytes) for f in frames), "d2h_bytes_per_step": d2h},
        "roofline": {"kernel": kname + " (the pixel model on CSR runs read from HBM)", "bound": "hbm",
                     "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_kind": hbm_kind,
                     # DRAM bytes of an average launch: the capture's DRAM bytes per algorithmic byte (its launches
                     # summed) times this run's algorithmic bytes per launch.
                     "traffic": cap["dram_per_alg_byte"] * alg / n_launch if cap and n_launch else None,
                     "traffic_capture": cap["capture"] if cap else None,
                     "algorithmic_bytes_per_step": alg, "launches_per_step": n_launch,
                     "kernel_ms_per_step": kms_total, "kernel_ms_from": "window-major steps on one stream",
                     "share_of_step": kms_total / (total_ms_all / args.steps)},
    }


def _sink_writer(fmt: str, path: str, es):
    from ballasim_b200.export import DatWriter, RawWriter

    if fmt == "dat":
        return DatWriter(path, es.width, es.height, 0, 0, 0, 0)
    return RawWriter(path, fmt, es.width, es.height, 0, 0, "openeb", 0, 0)


def run_sink(args, rank: int, world: int) -> dict | None:
    """The event file sink: whole files of the workload's event stream, device columns (value) and pinned host
    columns (e2e), each step timed between CUDA events on the writer's stream (the step includes its host part: the
    chunk copies, the file writes and close's SHA-256 of the file read back)."""
    import shutil

    import torch

    from ballasim_b200 import _lib

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    if not _lib.cuda_available():
        raise RuntimeError("bench: no B200 visible")
    fmt = SINKS[args.workload]
    es = W.event_stream(seed=5 + 1000 * rank)
    n = len(es.t_ns)
    cols = (es.x, es.y, es.p, es.t_ns)
    dev = [torch.from_numpy(c.view(np.int16) if c.dtype == np.uint16 else c).cuda() for c in cols]
    host = [torch.from_numpy(c.view(np.int16) if c.dtype == np.uint16 else c).pin_memory().numpy() for c in cols]
    host = [h.view(c.dtype) for h, c in zip(host, cols)]
    stream = torch.cuda.current_stream()
    tmp = tempfile.mkdtemp(prefix="bs_sink_")
    last = {}

    def step(k: int, device: bool) -> None:
        path = os.path.join(tmp, f"r{rank}_{k}.{fmt}")
        w = _sink_writer(fmt, path, es)
        if device:
            w.append_device(*(d.data_ptr() for d in dev), n, stream.cuda_stream)
        else:
            w.append(*host)
        last["info"], last["stats"] = w.close(), w.stats()
        os.remove(path)

    try:
        for k in range(args.warmup):
            step(k, True)
        torch.cuda.synchronize()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        kernel_ms = []
        with Clocks(torch.cuda.current_device()) as clk:
            if world > 1:
                import torch.distributed as dist

                dist.barrier()
            torch.cuda.synchronize()
            for k in range(args.steps):
                starts[k].record(stream)
                step(k, True)
                ends[k].record(stream)
                kernel_ms.append(last["stats"]["last_kernel_ms"])
            torch.cuda.synchronize()
        launches = last["stats"]["gpu_launches"] * args.steps  # each writer's own count, one file per step
        step_ms = [a.elapsed_time(b) for a, b in zip(starts, ends)]
        total_ms, ev_all, _ = reduce_step(float(sum(step_ms)), float(n * args.steps), 0.0, world)
        e2e = []
        for k in range(0 if args.profile else args.warmup + args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            step(k, False)
            if k >= args.warmup:
                e2e.append(time.perf_counter() - t0)
        e2e_s = reduce_max(sum(e2e), world) if e2e else None
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    if rank != 0:
        return None
    words = last["stats"]["last_words_bytes"]
    hbm, hbm_kind = measured_hbm()
    kms = statistics.mean(kernel_ms)
    alg = 13 * n + words
    achieved = alg / (kms * 1e-3) / 1e9
    out = {
        "metric": "events/s", "value": ev_all / (total_ms * 1e-3), "unit": "events/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64/uint16", "data": "synthetic (seeded event stream)",
        "config": {**es.describe(), "format": fmt, "file_bytes": last["info"]["bytes"],
                   "l2": "inputs larger than L2 (436 MiB of columns)", "parallelism": f"replicas x{world}",
                   "step": "writer made, one append of every event, close (file written and hashed)"},
        "gpu_launches": launches,
        "clocks": {k: v for k, v in clk.summary().items() if k != "samples"},
        "e2e": {"value": ev_all / e2e_s if e2e_s else None, "unit": "events/s", "h2d_bytes_per_step": 13 * n,
                "d2h_bytes_per_step": words},
        "roofline": {"kernel": "sink count_kernel + scan + range_kernel + write_kernel (per append)", "bound": "hbm",
                     "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "peak_kind": hbm_kind,
                     "traffic": None, "algorithmic_bytes_per_launch": alg, "avg_launch_ms": kms},
    }
    if world == 1 and not (args.no_cpu_baseline or args.profile):
        out["cpu_baseline"] = sink_reference(fmt, es, 8 << 20)
    return out


def sink_reference(fmt: str, es, n: int) -> dict:
    """The reference's own writer (oracle/_ref) on the first n events of the stream, one host core."""
    from oracle.oracle import Ref

    n = min(n, len(es.t_ns))
    with tempfile.TemporaryDirectory(prefix="bs_sink_ref_") as d:
        path = Path(d) / f"ref.{fmt}"
        t0 = time.perf_counter()
        Ref.event_file(path, fmt, es.width, es.height, 0, 0, es.x[:n], es.y[:n], es.p[:n], es.t_ns[:n],
                       t_ns_rem_min=0, t_ns_rem_max=0)
        dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "events/s", "cores": 1, "kind": "reference",
            "sample": f"first {n} of {len(es.t_ns)} events, one file ({dt:.2f} s with close's SHA-256)"}


def learned_comparison(train_stride: int = 4, steps: int = 9000, tau: float = 0.25) -> dict:
    """The learned step proposal against the plain sampler: the network is trained on the GPU (Adam, lr 1e-3,
    batch 8192, expectile weight tau) on (history, step) pairs of the plain sampler over a training-seed
    1280 x 720 field of blobs_1280x720's laws (every train_stride-th pixel, 1.0 s), its margin calibrated on a
    validation seed at 640 x 360 (median |dt| <= 8 us), and both samplers run the held-out-seed 1280 x 720, 1.0 s
    field with noise."""
    import torch

    from ballasim_b200.learned import StepMLP, calibrate_margin, compare_events, renders_and_events, trace_pairs

    t0 = time.perf_counter()
    tw = W.blobs_noise(1280, 720, W.LEARN_TRAIN_SEEDS[0])
    x, y, _ = trace_pairs(tw.sensors[0].field, tw.rules, tw.windows, stride=train_stride, seed=1)
    torch.cuda.synchronize()
    t_pairs = time.perf_counter() - t0
    net = StepMLP(seed=0)
    t0 = time.perf_counter()
    losses = net.train(x, y, steps=steps, batch=8192, lr=1e-3, seed=1, tau=tau)
    t_train = time.perf_counter() - t0
    n_pairs = int(len(y))
    del x, y
    margin, _ = calibrate_margin(net, W.blobs_noise(640, 360, W.LEARN_TRAIN_SEEDS[2]))
    ev = W.blobs_noise(1280, 720, W.LEARN_EVAL_SEED)
    px, sim_s = ev.pixels, ev.windows * W.WINDOW_NS * 1e-9
    plain_r, plain_ev, plain_ms = renders_and_events(ev)
    learned_r, learned_ev, learned_ms = renders_and_events(ev, net, margin)
    sig = compare_events(plain_ev, learned_ev)
    allc = compare_events(plain_ev, learned_ev, signal_only=False)
    return {
        "config": {"eval": f"{ev.name}, seed {W.LEARN_EVAL_SEED}, {ev.windows} windows ({sim_s:.4f} s)",
                   "train": f"blobs256_1280x720_noise seed {W.LEARN_TRAIN_SEEDS[0]}, every {train_stride}th pixel",
                   "pairs": n_pairs, "adam_steps": steps, "batch": 8192, "lr": 1e-3, "expectile_tau": tau,
                   "margin": margin, "margin_from": f"640x360 validation seed {W.LEARN_TRAIN_SEEDS[2]}"},
        "train_s": round(t_train, 3), "pairs_s": round(t_pairs, 3),
        "loss_first_last": [float(np.mean(losses[:10])), float(np.mean(losses[-200:]))],
        "plain": {"renders_per_px": plain_r, "samples_per_px": plain_r + ev.windows,
                  "events": len(plain_ev["t_cross_ns"]), "kernel_ms": plain_ms,
                  "events_per_s": len(plain_ev["t_cross_ns"]) / (plain_ms * 1e-3)},
        "learned": {"renders_per_px": learned_r, "samples_per_px": learned_r + ev.windows,
                    "events": len(learned_ev["t_cross_ns"]), "kernel_ms": learned_ms,
                    "events_per_s": len(learned_ev["t_cross_ns"]) / (learned_ms * 1e-3)},
        "renders_ratio": plain_r / learned_r,
        "samples_ratio": (plain_r + ev.windows) / (learned_r + ev.windows),
        "count_diff": allc["count_diff"],
        "signal_median_abs_dt_us": sig["median_abs_dt_ns"] / 1e3,
        "signal_p90_abs_dt_us": sig["p90_abs_dt_ns"] / 1e3,
        "signal_unmatched_share": sig["unmatched_share"],
        "pixels": px,
    }


def cpu_windows(args) -> int:
    return args.cpu_windows or CPU_WINDOWS.get(args.workload, CPU_WINDOWS_DEFAULT)


def reference_sample(wl: W.Workload, windows: int, fp64: bool = False) -> dict:
    """The reference's own CPU path (oracle/_ref) on a bounded sample of the workload: every sensor, its first
    `windows` windows from t0 (WindowEngine<kHost>, serial by design, then SensorModel on every host thread).
    The reference has no shot or background-activity noise: those rows are not passed, leak is."""
    from ballasim_b200.params import resolve
    from oracle.oracle import Ref

    w = min(windows, wl.windows)
    samples, wall, sampler_s, sensor_s, threads = 0, 0.0, 0.0, 0.0, 0
    for spec in wl.sensors:
        m = Ref.Model(resolve(spec.preset, spec.overrides), spec.width, spec.height, spec.seed, spec.camera,
                      fp64=fp64)
        t0 = time.perf_counter()
        _, st = m.simulate(spec.field, wl.rules, w)
        wall += time.perf_counter() - t0
        samples += st["pixel_samples"]
        sampler_s += st["sampler_s"]
        sensor_s += st["sensor_s"]
        threads = m.threads
    sizes = ", ".join(f"{s.width}x{s.height}" for s in wl.sensors)
    return {"value": samples / wall, "unit": "pixel-samples/s", "cores": threads, "kind": "reference",
            "precision": "fp64" if fp64 else "fp32", "pixel_samples": samples, "seconds": round(wall, 3),
            "sample": f"every sensor ({sizes}), first {w} of {wl.windows} windows ({samples} pixel-samples, "
                      f"{wall:.2f} s: the sampler, serial by design, {sampler_s:.2f} s; the pixel model on "
                      f"{threads} threads {sensor_s:.2f} s); shot and background-activity noise have no reference "
                      f"counterpart and are off there"}


def cpu_baseline(wl: W.Workload, windows: int) -> dict:
    """The reference CPU path's fp32 figure on the bounded sample, its fp64 kernel (the reference's default CPU
    precision) on the same sample beside it."""
    out = reference_sample(wl, windows)
    f64 = reference_sample(wl, windows, fp64=True)
    out["fp64"] = {"value": f64["value"], "seconds": f64["seconds"]}
    return out


def run_reference(args, rank: int) -> dict | None:
    if rank != 0:
        return None
    if args.workload in SINKS:
        es = W.event_stream()
        vals, cb = [], None
        for k in range(args.warmup + args.steps):
            cb = sink_reference(SINKS[args.workload], es, len(es.t_ns))
            if k >= args.warmup:
                vals.append(cb["value"])
        value = statistics.mean(vals)
        return {"impl": "reference", "metric": "events/s", "value": value, "unit": "events/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * len(es.t_ns) / value,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64/uint16",
                "data": "synthetic (seeded event stream)", "config": {**es.describe(), "format": SINKS[args.workload]},
                "cpu_baseline": {**cb, "value": value},
                "e2e": {"value": value, "unit": "events/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    wl = (RUNS.get(args.workload) or WORKLOADS[args.workload])()
    w = cpu_windows(args)
    secs, last = [], None
    for k in range(args.warmup + args.steps):
        last = reference_sample(wl, w)
        if k >= args.warmup:
            secs.append(last["seconds"])
    total = sum(secs)
    value = last["pixel_samples"] * len(secs) / total
    f64 = reference_sample(wl, w, fp64=True)
    cb = {k: last[k] for k in ("unit", "cores", "kind", "sample", "precision")}
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": "pixel-samples/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(secs),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
            "data": "synthetic (seeded analytic irradiance fields)",
            "config": {**wl.describe(), "bounded_windows_per_sensor": min(w, wl.windows)},
            "cpu_baseline": {**cb, "value": value},
            "fp64": {"value": f64["value"], "unit": "pixel-samples/s", "seconds": f64["seconds"],
                     "note": "the reference's fp64 CPU kernel (its default precision) on the same sample, once"},
            "e2e": {"value": value, "unit": "pixel-samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + sorted(RUNS) + sorted(SINKS),
                    default=DEFAULT_WORKLOAD)
    ap.add_argument("--cpu-windows", type=int, default=0,
                    help="windows of every sensor in the reference's bounded sample (0: the workload's default)")
    ap.add_argument("--block", type=int, default=0,
                    help="runs_* workloads: 0 the split row-major kernel, 1 unsplit, n > 1 advance_runs_kernel's block")
    ap.add_argument("--window-major", action="store_true",
                    help="runs_* workloads: every sensor's windows in turn on one stream (default: each sensor on a "
                         "stream and host thread of its own)")
    ap.add_argument("--long-run", type=int, default=0,
                    help="runs_* workloads: runs longer than this are walked by a whole warp (-1: none)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--warps", type=int, default=0)
    ap.add_argument("--blocks-per-sm", type=int, default=0)
    ap.add_argument("--stage", type=int, default=0, help="engine staging depth: 0, 16 or 32")
    ap.add_argument("--tile-width", type=int, default=0, help="engine tile width: 4, 8, 16 or 32 px")
    ap.add_argument("--no-autotune", action="store_true", help="keep the given (or default) launch shape")
    ap.add_argument("--no-graph", action="store_true", help="launch each step's operations without a CUDA graph")
    ap.add_argument("--windows", type=int, default=0, help="run only the first windows (profiling a reduced case)")
    ap.add_argument("--profile", action="store_true", help="no e2e, CPU or learned legs (fewest launches, for ncu)")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-proposal comparison")
    ap.add_argument("--learned-only", action="store_true",
                    help="run the learned-proposal comparison alone (its training and both samplers) and print it")
    ap.add_argument("--learned-steps", type=int, default=9000, help="Adam steps of the learned proposal's training")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.learned_only:
        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        out = {"learned_vs_plain": learned_comparison(steps=args.learned_steps)} if rank == 0 else None
    elif args.impl == "reference":
        out = run_reference(args, rank)
    else:
        if world > 1:
            import datetime

            import torch.distributed as dist

            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        try:
            if args.workload in SINKS:
                out = run_sink(args, rank, world)
            elif args.workload in RUNS:
                out = run_runs(args, rank, world)
            else:
                out = run_ours(args, rank, world)
        finally:
            if world > 1:
                import torch.distributed as dist

                dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
