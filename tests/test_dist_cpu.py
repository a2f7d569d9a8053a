"""Multi-rank plumbing of bench.py on CPU (gloo, two ranks): the job time is
the slowest rank's device time, every rank gets the same value, and the
reference arm under torchrun prints one line from rank 0 only."""
import json
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _rank(rank, world, port, q):
    import torch.distributed as D
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    D.init_process_group("gloo", rank=rank, world_size=world)
    try:
        q.put((rank, bench.job_time_ms(10.0 + 7.0 * rank, True)))
    finally:
        D.destroy_process_group()


def test_job_time_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == {0: 17.0, 1: 17.0}


def test_reference_arm_under_torchrun_prints_one_line():
    port = 29600 + os.getpid() % 1000
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--particles", "3000",
           "--ref-targets", "32"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"


def _share_rank(rank, world, port, q):
    import torch.distributed as D
    sys.path.insert(0, ROOT)
    from vortex_b200 import multibody as MB
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    D.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = MB.share(10, rank, world)
        rec = {"requests": len(mine), "steps_requested": 100 * len(mine), "failed": 0, "body_steps": 7,
               "body_steps_per_s": 50.0 + rank, "particle_steps_per_s": 1e6, "ticks": 3, "wall_s": 1.0 + rank,
               "step_ms_p50": 2.0, "step_ms_p99": 4.0 + rank, "ttc_s_p50": 1.0, "ttc_s_p99": 2.0,
               "mean_resident": 4.0}
        parts = [None] * world
        D.all_gather_object(parts, (mine, rec))
        q.put((rank, parts))
    finally:
        D.destroy_process_group()


def test_multibody_partition_over_two_gloo_ranks():
    """Body-partitioned runs: the two ranks' shares cover the population once,
    and the gathered records combine (throughputs add, latencies take the
    slowest rank) to the same record on every rank."""
    sys.path.insert(0, ROOT)
    from vortex_b200 import multibody as MB
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + os.getpid() % 1000
    procs = [ctx.Process(target=_share_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[0] == got[1]
    shares = [m for m, _ in got[0]]
    assert sorted(shares[0] + shares[1]) == list(range(10)) and not set(shares[0]) & set(shares[1])
    c = MB.combine_serve([r for _, r in got[0]])
    assert c["requests"] == 10 and c["body_steps_per_s"] == 101.0 and c["step_ms_p99"] == 5.0
    assert c["wall_s"] == 2.0 and c["ranks"] == 2
    with pytest.raises(ValueError):
        MB.share(4, 2, 2)
