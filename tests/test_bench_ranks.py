"""bench.py's multi-rank plumbing on CPU: two gloo ranks (127.0.0.1).

The path does not shard (replicas only), so the ranks exchange nothing but
the timing: every device time is reported as the slowest rank's, and the
CPU reference arm runs on rank 0 alone."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r, w, loc = bench.dist_env()
        value = bench.max_over_ranks(10.0 + 5.0 * rank, w, device="cpu")
        out.put((r, w, loc, value))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    assert [g[0] for g in got] == [0, 1]
    assert all(g[1] == world and g[2] == g[0] for g in got)
    assert all(g[3] == 15.0 for g in got)        # the slowest rank's time everywhere


def test_max_over_ranks_single():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5


@pytest.mark.parametrize("rank,prints", [(0, True), (1, False)])
def test_reference_arm_runs_on_rank_zero_only(rank, prints):
    """--impl reference under torchrun: rank 0 times the oracle and prints
    one JSON line; the other ranks exit 0 without work (small sample)."""
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank),
               MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "0", "--n", "24"],
                       capture_output=True, text=True, env=env, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    if prints:
        assert len(lines) == 1
        line = json.loads(lines[0])
        assert line["impl"] == "reference" and line["n_gpus"] == 2
        assert line["cpu_baseline"]["kind"] == "port" and line["value"] > 0
        assert line["e2e"]["h2d_bytes_per_step"] == 0
    else:
        assert lines == []
