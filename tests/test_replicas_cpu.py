"""Host logic of the multi-GPU bench (N independent replicas, one per rank): two gloo ranks on the
CPU take the slowest rank's time and build differently seeded replicas of the same workload."""
import json
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        slowest = bench.max_over_ranks(1.5 + rank, dist, device="cpu")
        again = bench.max_over_ranks(10.0 - rank, dist, device="cpu")
        s, _ = bench.build_system(bench.WORKLOADS["water3k-classical"], rank)
        np.save(os.path.join(out_dir, f"v{rank}.npy"), s.v)
        with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
            json.dump({"slowest": slowest, "again": again, "natom": s.natom}, f)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time_and_seed_their_own_replica(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r = [json.load(open(tmp_path / f"r{k}.json")) for k in range(2)]
    assert r[0]["slowest"] == r[1]["slowest"] == 2.5
    assert r[0]["again"] == r[1]["again"] == 10.0
    assert r[0]["natom"] == r[1]["natom"] == 3000
    v0, v1 = np.load(tmp_path / "v0.npy"), np.load(tmp_path / "v1.npy")
    assert v0.shape == v1.shape and not np.array_equal(v0, v1)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25) == 3.25
    assert bench.replica_seed(2, 0) == 2 and bench.replica_seed(2, 1) != 2
