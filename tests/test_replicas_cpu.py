"""Replicas across GPUs, on the CPU: two gloo ranks run the host logic `bench.py --gpus 2` uses.

Each rank transports its own pixels with disjoint stream keys (no collective on the data path); the job's
time is the slowest rank's (MAX all-reduce), and the whole-job rate counts every rank's primaries.  The
reference arm runs on rank 0 only.
"""
import os
import socket
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from cudamonsel_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        keys = replicas.pixel_keys(rank, 256)
        gathered = [torch.zeros(256, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(gathered, torch.from_numpy(keys.astype(np.int64)))
        ms = replicas.max_over_ranks(10.0 * (rank + 1))  # rank r "took" 10 (r + 1) ms
        rate = replicas.job_rate(512000, world, ms)
        if rank == 0:
            np.save(out, np.concatenate([np.concatenate([g.numpy() for g in gathered]), [int(ms), int(rate)]]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_disjoint_keys_and_slowest_rank_time(tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "r.npy")
    mp.spawn(_rank, args=(2, _free_port(), out), nprocs=2, join=True)
    r = np.load(out)
    keys, ms, rate = r[:-2], r[-2], r[-1]
    assert len(np.unique(keys)) == 512  # no pixel stream is shared between the replicas
    assert ms == 20  # the slower rank's time
    assert rate == 2 * 512000 * 1000 // 20


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    from cudamonsel_b200 import replicas
    assert replicas.max_over_ranks(3.5) == 3.5
    assert (replicas.pixel_keys(0, 4) == np.arange(4, dtype=np.uint64) + np.uint64(replicas.KEY_STRIDE)).all()


def test_reference_arm_runs_on_rank_0_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
