"""The multi-GPU form of the benchmark is replicas: one solver per rank, no collective on the data
path, the job's time the slowest rank's. These tests run its rank logic as two CPU processes over
gloo (rendezvous, max over ranks, the whole-job rate) and check that the reference arm's other
ranks leave at once."""
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank), PSFEA_DIST_BACKEND="gloo")
    import bench
    r, w, local, pg = bench.dist_setup(world)
    # rank r "took" 1.5 (r + 1) s for its solves: the job time is the slowest rank's
    t = bench.reduce_max(pg, 1.5 * (r + 1))
    out.put((r, w, t, bench.job_rate(w, 12_830_211, 5, t)))
    pg.barrier()
    pg.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r for r, *_ in res] == [0, 1]
    for r, w, t, rate in res:
        assert w == 2 and t == 3.0
        assert abs(rate - 2 * 12_830_211 * 5 / 3.0 / 1e6) < 1e-9


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"], env=env,
                       capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""
