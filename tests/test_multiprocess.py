"""The multi-process paths of bench.py on the CPU (gloo, world size 2): the
reference arm launched by torchrun (rank 0 alone prints one JSON line, every
rank exits 0) and the max-over-ranks reduction of the timing that the GPU
arm applies to its replicas."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle as O
from helpers import ROOT


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, values, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out[rank] = bench.max_over_ranks(dist, values[rank], "cpu")
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world, port = 2, _port()
    values = [[3.0, 10.0], [5.0, 7.0]]
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, port, values, out), nprocs=world, start_method="spawn")
        assert out[0] == [5.0, 10.0] and out[1] == [5.0, 10.0]


@pytest.mark.skipif(not O.ref_available(2), reason="the reference build (oracle/_ref) is absent")
def test_reference_arm_under_torchrun():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_port()), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(line) for line in r.stdout.splitlines() if line.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["value"] > 0 and line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["steps"] == 1 and line["iterations"] > 1
