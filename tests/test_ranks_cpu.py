"""Multi-rank plumbing of bench.py on the CPU (gloo, world size 2): the max-over-ranks
timing reduction, the barrier, and the reference arm under torchrun printing one line from
rank 0 only. The data path has no collective (replicas only)."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    ws, r, local, pg = bench.dist_setup()
    assert ws == 2 and r == rank
    m = bench.max_over_ranks(10.0 + 5.0 * rank, pg)
    bench.barrier(pg)
    out.put((rank, m, pg.get_backend()))
    pg.destroy_process_group()


def test_max_over_ranks_and_barrier_on_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [m for _, m, _ in res] == [15.0, 15.0]
    assert {b for _, _, b in res} == {"gloo"}


def test_reference_arm_under_torchrun_prints_once():
    import torch
    if torch.cuda.is_available():
        pytest.skip("exercises the CPU (gloo) path")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1", "--cpu-n", "15", "--cpu-iters", "2"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0


def test_replica_runs_skip_the_time_to_tolerance_blocks():
    """The minutes-long time-to-tolerance and 20-inclusion blocks run on the one-GPU line;
    under torchrun with several ranks they are skipped unless a grid is asked for."""
    import argparse

    sys.path.insert(0, ROOT)
    import bench

    def ns(**kw):
        base = dict(ttt_n=None, ttt_n2=None, incl_default_n=None)
        base.update(kw)
        return argparse.Namespace(**base)

    one = bench.resolve_block_defaults(ns(), 1)
    assert (one.ttt_n, one.ttt_n2, one.incl_default_n) == (511, 255, 255)
    many = bench.resolve_block_defaults(ns(), 4)
    assert (many.ttt_n, many.ttt_n2, many.incl_default_n) == (0, 0, 0)
    asked = bench.resolve_block_defaults(ns(ttt_n=255, ttt_n2=0), 2)
    assert (asked.ttt_n, asked.ttt_n2, asked.incl_default_n) == (255, 0, 0)
