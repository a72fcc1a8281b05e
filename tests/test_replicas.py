"""The N-GPU path of the benchmark on CPU: two gloo ranks (127.0.0.1), each with its replica of a workload, reduce
their figures as bench.py does on NCCL (the slowest rank's time, the sum of the work)."""
import json
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    import datetime
    import os

    import torch.distributed as dist

    from ballasim_b200 import workloads as W
    from ballasim_b200.replicas import reduce_max, reduce_step, replica

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        wl = replica(W.six_sensors(), rank)
        step = reduce_step(10.0 + rank, 100.0 * (rank + 1), float(rank), world, device="cpu")
        e2e = reduce_max(5.0 + 3.0 * rank, world, device="cpu")
        out = {"step": step, "e2e": e2e, "seeds": [s.seed for s in wl.sensors],
               "sizes": [[s.width, s.height] for s in wl.sensors], "windows": wl.windows,
               "blobs0": wl.sensors[0].field.blobs[:2].tolist()}
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump(out, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_gloo_ranks_reduce_like_the_bench(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    r = [json.load(open(tmp_path / f"rank{k}.json")) for k in range(world)]
    for k in range(world):
        assert r[k]["step"] == [11.0, 300.0, 1.0]  # max time, summed samples and events
        assert r[k]["e2e"] == 8.0
    assert r[0]["sizes"] == r[1]["sizes"] and r[0]["windows"] == r[1]["windows"]  # weak scaling: same work
    assert all(a != b for a, b in zip(r[0]["seeds"], r[1]["seeds"]))            # independent sensors
    assert r[0]["blobs0"] != r[1]["blobs0"]
