"""Multi-process path of bench.py on the CPU (gloo, world size 2).

The DG update does not shard (replicas only): bench.py --gpus N runs one independent instance per
rank and the only cross-rank operations are a barrier and the max over ranks of the device time.
This test runs those helpers in two gloo ranks and checks the aggregate, and that the reference arm
prints nothing on rank != 0.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    dist, r, ws, local = bench.dist_setup()
    assert (r, ws) == (rank, world)
    bench.barrier(dist)
    ms = [12.5, 17.25][rank]  # rank-local device times
    ms_max = bench.max_over_ranks(dist, ms)
    value = bench.aggregate_value(dofs=1000, steps=4, world=ws, ms_max=ms_max)
    q.put((rank, ms_max, value))
    dist.destroy_process_group()


def test_two_rank_timing_aggregate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms_max, value in res:
        assert ms_max == 17.25
        # 3 stage updates per step, summed over the two replicas, over the slowest rank's time
        assert value == pytest.approx(3 * 1000 * 4 * 2 / 17.25e-3)


def test_reference_arm_silent_on_nonzero_rank():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--workload", "ot64_p2", "--steps", "1", "--warmup", "0"],
                         env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0
    assert out.stdout.strip() == ""


def test_reference_arm_line_shape():
    env = dict(os.environ, RANK="0", WORLD_SIZE="1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--workload", "ot64_p2", "--steps", "2", "--warmup", "1"],
                         env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "DOF-stage/s" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
