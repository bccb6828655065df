"""The N > 1 host logic of bench.py on the CPU, as two gloo ranks: the path
runs as independent replicas (no data-path collective), so what the ranks
share is the timing reduction (the slowest rank's device time), per-rank
seeds, and the host reference arm running on rank 0 alone."""
import json
import os
import subprocess
import sys

import pytest

torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r reports 10 + r ms: every rank must see the largest
        got = bench.rank_max(10.0 + rank, dist)
        q.put((rank, got, bench.replica_seed(rank)))
    finally:
        dist.destroy_process_group()


def _free_port():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_rank_max_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [11.0, 11.0]
    # replicas start from distinct seeded fields
    assert res[0][2] != res[1][2]


def test_rank_max_without_process_group_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.rank_max(3.5, None) == 3.5


def test_reference_arm_under_torchrun_prints_once():
    """`bench.py --impl reference` under torchrun with two gloo ranks: rank 0
    times the host port of the reference's step and prints one JSON line,
    rank 1 exits 0 without work (a 16x16x12 grid keeps it to seconds)."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--grid", "16", "16", "12", "--steps", "2", "--warmup", "1"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2
    assert rec["value"] > 0 and rec["cpu_baseline"]["kind"] == "port"
    assert rec["e2e"]["h2d_bytes_per_step"] == 0
