"""The multi-GPU path of bench.py: one process per GPU, each running its own tunnel (replicas, no
data-path collective), timed as the slowest rank. The cross-rank steps run here as two gloo
ranks on the CPU."""
import os
import socket
import subprocess
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r took (r + 1) * 10 ms for its steps: every rank reports the slowest
        ms = bench.max_over_ranks(dist, 10.0 * (rank + 1))
        dist.barrier()
        out[rank] = (ms, bench.replica_mlups(world, 4_194_304, 1000, ms))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 20.0
    # two tunnels of 4.19 M cells, 1000 updates each, in 20 ms
    assert res[0][1] == pytest.approx(2 * 4_194_304 * 1000 / 0.020 / 1e6)


def test_single_process_is_its_own_max():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(None, 3.5) == 3.5


def test_reference_arm_non_zero_rank_exits_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_measured_traffic_follows_the_launch_shape():
    # the default block of the vectorised kernel (0, 0) is one row of 128 threads on the bench
    # tunnel, so it reads the 128 x 1 entry of the committed profile; shapes never captured give None
    sys.path.insert(0, ROOT)
    import bench

    assert bench.measured_traffic((4, 2, 0, 0)) == bench.measured_traffic((3, 2, 128, 1)) is not None
    assert bench.measured_traffic((4, 2, 64, 2)) is not None
    assert bench.measured_traffic((0, 4, 32, 4)) is None
    assert bench.measured_traffic((0, 0, 0, 0), closure=True) is not None
