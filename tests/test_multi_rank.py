"""Replica (N > 1) plumbing of bench.py on CPU with two gloo ranks: the
max-over-ranks time and the whole-job rate every rank agrees on, and the
reference arm under torchrun (rank 0 alone prints one line; the other rank
exits 0 without work)."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = [12.5, 40.0][rank]  # the slower rank decides the job's time
    got = bench.max_over_ranks(ms, dist, "cpu")
    rate = bench.replica_rate(1000, 10, got, world)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, got, rate))


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [40.0, 40.0]
    assert out[0][2] == out[1][2] == pytest.approx(2 * 1000 * 10 / 0.040)


def test_single_process_max_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.replica_rate(100, 2, 1.0, 1) == pytest.approx(2.0e5)


def test_reference_arm_under_torchrun():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl",
           "reference", "--gpus", "2", "--steps", "2", "--warmup", "1", "--nel", "6"]
    res = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600,
                         env={**os.environ, "OMP_NUM_THREADS": "2"})
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [l for l in res.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["steps"] == 2 and d["warmup"] == 1
    assert d["n_gpus"] == 2 and d["value"] > 0


def test_both_arms_print_the_same_config_at_one_gpu():
    """The reference arm's `config` equals the GPU arm's at N = 1 (the same
    64^3 workload, one replica), so the two lines compare like for like."""
    sys.path.insert(0, ROOT)
    import bench
    sys_argv = sys.argv
    try:
        sys.argv = ["bench.py"]
        args = bench.parse()
    finally:
        sys.argv = sys_argv
    ours, ref = bench.arm_config(args, 1), bench.arm_config(args)
    assert ours == ref
    assert ref["elements"] == 64 ** 3 and ref["parallelism"] == "replicas x1"

