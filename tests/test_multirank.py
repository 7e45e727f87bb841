"""The multi-process paths of bench.py on CPU ranks (gloo), as the GPU bench launches them with
torchrun: every rank works on its own shard (replicas, no data-path collective) and the job's time
is the maximum over ranks; the reference arm runs on rank 0 alone and the other ranks exit 0."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

WORLD = 2


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    from agama_b200 import workloads
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(10.0 + 5 * rank, dist, "cpu")
        shard = workloads.disk_particles(64, lambda R: 0 * R + 1.0, seed=3 + rank)   # the bench's per-rank seed
        np.save(os.path.join(out, "shard%d.npy" % rank), shard)
        with open(os.path.join(out, "max%d.txt" % rank), "w") as f:
            f.write(repr(t))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_disjoint_shards(tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(_rank_main, args=(free_port(), str(tmp_path)), nprocs=WORLD, start_method="spawn")
    for r in range(WORLD):
        assert float(open(tmp_path / ("max%d.txt" % r)).read()) == 10.0 + 5 * (WORLD - 1)
    a, b = (np.load(tmp_path / ("shard%d.npy" % r)) for r in range(WORLD))
    assert a.shape == b.shape == (64, 6) and not np.allclose(a, b)


def test_no_reduction_on_one_rank():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5


def test_reference_arm_under_torchrun():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(WORLD),
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", str(WORLD), "--steps", "1", "--warmup", "1", "--particles", "2000",
           "--no-secondary"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT,
                       env=dict(os.environ, OMP_NUM_THREADS="2"))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1                      # rank 0 alone prints
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == WORLD and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "reference"
