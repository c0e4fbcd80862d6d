"""Multi-rank host logic of bench.py on CPU (gloo, world size 2).

A multi-GPU run of bench.py is one process per GPU with no data-path
collective: every rank factors its own seeded matrices or serves its own
seeded request stream, and the only collectives are the two reductions that
turn per-rank numbers into the reported line (the slowest rank's time, the
total work).  These tests run those reductions over gloo with two CPU ranks,
check that the ranks draw different streams, and that the reference arm
prints from rank 0 only.
"""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    for p in (str(ROOT), str(ROOT / "delayed-pivoting_b200")):
        if p not in sys.path:
            sys.path.insert(0, p)
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    import bench
    from delayed_pivoting import serving as sv

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        dev = torch.device("cpu")
        slowest = bench._max_over_ranks(torch, dist, dev, 100.0 + 7.0 * rank)
        total = bench._sum_over_ranks(torch, dist, dev, 3.0 + rank)
        # the serve workload seeds each rank's stream with seed + rank
        reqs = sv.make_stream(24, 16384 + rank)
        mine = [(q.n, q.kappa, len(q.solves)) for q in reqs]
        streams = [None] * world
        dist.all_gather_object(streams, mine)
    finally:
        dist.destroy_process_group()
    out.put((rank, slowest, total, streams))


def test_two_ranks_reduce_time_and_work_and_draw_their_own_streams():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    for rank, slowest, total, streams in results:
        assert slowest == 107.0  # max over ranks: the slowest rank's time
        assert total == 7.0      # sum over ranks: all ranks' work
        assert streams[0] != streams[1]  # independent units, one stream per rank
    assert results[0][3] == results[1][3]  # every rank saw the same gathered streams


@pytest.mark.parametrize("rank,prints", [(0, True), (1, False)])
def test_reference_arm_prints_on_rank_zero_only(rank, prints):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank))
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                        "--workload", "ir", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if prints:
        assert len(lines) == 1
        line = json.loads(lines[0])
        assert line["impl"] == "reference" and "unavailable" in line
    else:
        assert lines == []



@pytest.mark.parametrize("rank,prints", [(0, True), (1, False)])
def test_sytrf_reference_arm_prints_on_rank_zero_only(rank, prints):
    """The LDL^T reference arm (the reference's delayed_sytrf_blocked, or its
    restatement) runs and prints on rank 0 alone; other ranks exit 0."""
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank))
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                        "--workload", "sytrf", "--gpus", "2", "--cpu-n", "256", "--steps", "1",
                        "--warmup", "0"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if prints:
        assert len(lines) == 1
        line = json.loads(lines[0])
        assert line["impl"] == "reference" and line["value"] > 0
        assert line["cpu_baseline"]["kind"] in ("reference", "port")
        assert line["e2e"]["h2d_bytes_per_step"] == 0
    else:
        assert lines == []
