"""The N > 1 host path of bench.py on CPU: two gloo ranks.

Limbs and polynomials are independent, so ranks share no data; the only
cross-rank steps are the barrier and the max-over-ranks reduction of the
timed region, and rank 0 alone prints.  The reference arm under torchrun
runs on rank 0 only and the other ranks exit 0 without work.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.join(os.path.dirname(__file__), "..")


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        v = bench.max_over_ranks(10.0 + 5.0 * rank, device="cpu")
        out[rank] = v
    finally:
        dist.destroy_process_group()


def _rank_setup_worker(rank, world, port, out):
    """The GPU arm's rank set-up (bench.init_ranks) on a gloo rank: the
    environment a torchrun launch gives, then the max-over-ranks timing."""
    import argparse
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    got = bench.init_ranks(argparse.Namespace(gpus=world), backend="gloo")
    try:
        out[rank] = (got, bench.max_over_ranks(1.0 + rank, device="cpu"))
    finally:
        dist.destroy_process_group()


def test_gpu_arm_rank_setup_gloo():
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_rank_setup_worker, args=(world, free_port(), out), nprocs=world, join=True)
    assert dict(out) == {0: ((2, 0, 0), 2.0), 1: ((2, 1, 1), 2.0)}


def test_world_size_must_match_gpus(monkeypatch):
    import argparse
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("WORLD_SIZE", "2")
    with pytest.raises(SystemExit):
        bench.init_ranks(argparse.Namespace(gpus=4), backend="gloo")


def test_gpus_flag_starts_the_ranks_itself():
    """`python bench.py --gpus 2` (no torchrun) re-launches itself as two
    ranks: one JSON line, from rank 0, with n_gpus 2."""
    from oracle import oracle as O
    if O.ref_lib() is None:
        pytest.skip("compiled reference harness not built")
    env = {k: v for k, v in os.environ.items()
           if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    assert json.loads(lines[0])["n_gpus"] == 2


def test_max_over_ranks_gloo():
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_worker, args=(world, free_port(), out), nprocs=world, join=True)
    assert dict(out) == {0: 15.0, 1: 15.0}


def test_max_over_ranks_single_process():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, device="cpu") == 3.5


def test_reference_arm_two_ranks():
    from oracle import oracle as O
    if O.ref_lib() is None:
        pytest.skip("compiled reference harness not built")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1  # rank 0 only
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference"
