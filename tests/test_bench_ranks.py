"""Multi-process host logic of bench.py on the CPU: two gloo ranks (the replica
aggregation: the job time is the slowest rank's, the value counts every
rank's work) and the reference arm's rank handling (rank 0 alone works)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        my_ms = [120.0, 150.0][rank]
        total = bench.max_over_ranks(my_ms, dist, "cpu")
        q.put((rank, total, bench.whole_job_rate(world, 10 ** 9, 4, total)))
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [150.0, 150.0]
    # 2 ranks x 1e9 interactions x 4 steps in 150 ms
    assert out[0][2] == pytest.approx(2 * 1e9 * 4 / 0.150 / 1e9)


def test_single_process_needs_no_group():
    assert bench.max_over_ranks(7.0, None, "cpu") == 7.0


def test_reference_arm_runs_on_rank_zero_only(capsys):
    args = bench.main.__globals__["argparse"].Namespace(steps=1, warmup=1, gpus=2, small=False)
    assert bench.run_reference_arm(args, rank=1, world=2) == 0
    assert capsys.readouterr().out == ""


def test_kappa_option_rejects_uneven_column_split():
    """--kappa splits the 64 RHS evenly into wave chunks of a multiple of 16
    columns (1, 2 or 4 wavenumbers); other counts stop before any work."""
    with pytest.raises(SystemExit):
        bench.main(["--kappa", "3,5,7"])
    assert list(bench.KAPPA) == [2.0, 4.0, 8.0, 16.0] and bench.WCS == 16
