"""The multi-GPU path of bench.py is replicas only: N independent solves, one per
rank, timed by the slowest rank. Its host logic (the max-over-ranks reduction every
rank calls, and the whole-job throughput) runs here as two gloo ranks on the CPU."""
import json
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    import sys
    from datetime import timedelta

    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    dev, e2e = 1.0 + rank, 10.0 - 3.0 * rank  # rank 1 is slower on the device, rank 0 end to end
    dev_max, e2e_max = bench.replica_reduce([dev, e2e], world, "cpu")
    value = bench.replica_throughput(3, world, dev_max)
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump({"dev_max": dev_max, "e2e_max": e2e_max, "value": value}, f)
    dist.destroy_process_group()


def test_replicas_take_the_slowest_rank(tmp_path):
    world = 2
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [json.loads((tmp_path / f"r{r}.json").read_text()) for r in range(world)]
    for r in res:
        assert r["dev_max"] == 2.0 and r["e2e_max"] == 10.0
        assert r["value"] == pytest.approx(2 * 3 / 2.0)


def test_single_rank_is_the_identity():
    import bench
    assert bench.replica_reduce([1.5, 2.5], 1, "cpu") == [1.5, 2.5]
    assert bench.replica_throughput(4, 1, 2.0) == 2.0
