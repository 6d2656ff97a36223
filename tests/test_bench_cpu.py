"""Host-side checks of bench.py: the reference arm's JSON line, its rank handling, and the max-over-ranks
timing of the replica path over two gloo processes (no GPU)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _ref_built():
    import oracle

    return oracle.ref_available("threaded") or oracle.ref_available("serial")


def test_reference_arm_prints_one_line():
    if not _ref_built():
        pytest.skip("reference CPU build absent")
    env = dict(os.environ, RANK="0")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "16",
                          "--steps", "1"], capture_output=True, text=True, timeout=600, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "particle-steps/s" and d["value"] > 0
    # subcell-centre rule on 32 subcells per axis: centres (i + 1/2)/32 inside [0,0.4] x [0,0.6] x [0,1]
    assert d["config"]["particles"] == 13 * 19 * 32
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "16",
                          "--steps", "1"], capture_output=True, text=True, timeout=300, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    assert not [l for l in out.stdout.splitlines() if l.startswith("{")]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, "cpu")  # rank 1 is the slow one
        value = bench.replica_throughput(world, 1000, 20, ms / 1e3)
        q.put((rank, ms, value))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]          # both ranks report the slowest rank's time
    assert res[0][2] == pytest.approx(2 * 1000 * 20 / 0.015)  # whole-job throughput of 2 replicas


def test_single_process_max_over_ranks_is_identity():
    import bench

    assert bench.max_over_ranks(3.5, "cpu") == 3.5
