"""bench.py's multi-rank plumbing on the CPU (world size 2, gloo, 127.0.0.1): the
barrier and the max / sum over ranks that make a multi-GPU line's timing the
slowest rank's and its value the whole job's, and the reference arm's rule that
only rank 0 works and prints.  Replicas exchange no simulation data, so this is
all the multi-rank path has to get right besides each rank's own run."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    w, r, local = bench.dist_env()
    g = bench.Group(w)
    g.barrier()
    got = (g.reduce(10.0 * (r + 1), "max"), g.reduce(float(r + 1), "sum"))
    g.barrier()
    g.close()
    out.put((r, w, local, got))


def test_group_max_and_sum_over_two_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[:3] for r in results] == [(0, 2, 0), (1, 2, 1)]
    for r in results:
        assert r[3] == (20.0, 3.0)  # the slowest rank's time, the whole job's count


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1",
               MASTER_PORT=str(_free_port()))
    res = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--gpus", "2"], env=env, capture_output=True, text=True, timeout=300,
                         cwd=ROOT)
    assert res.returncode == 0, res.stderr[-2000:]
    assert res.stdout.strip() == ""


if __name__ == "__main__":
    sys.exit(pytest.main([__file__, "-q"]))
