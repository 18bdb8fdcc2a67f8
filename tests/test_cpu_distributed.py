"""The bench's multi-process path (one process per GPU, launched by
torch.distributed.run) exercised on the CPU with the gloo backend and two
ranks: the max-over-ranks timing, the barrier, and the reference arm's
rank-0-only line."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, q) -> None:
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench

    class A:
        gpus = world
    w, r, local, dist = bench.dist_setup(A())
    try:
        got = bench.max_over_ranks(1.5 + r, dist, "cpu")
        dist.barrier()
        q.put((r, w, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert [(r, w) for r, w, _ in res] == [(0, 2), (1, 2)]
    assert all(got == 2.5 for _, _, got in res)  # every rank reports the slowest rank's time


def test_reference_arm_under_torchrun_two_ranks(tmp_path):
    """`bench.py --impl reference --gpus 2` launched by torchrun with two
    ranks: rank 0 prints one line, rank 1 exits 0 without work (here on the
    CPU, gloo)."""
    if not (ROOT / "cudagravitydemo_b200" / "libbh_b200.so").exists():
        pytest.skip("library not built")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), str(ROOT / "bench.py"), "--impl", "reference", "--gpus",
           "2", "--steps", "1", "--warmup", "0", "--bodies", "4096"]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=tmp_path, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
