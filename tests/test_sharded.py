"""Host logic of the row-sharded apply (baemm_b200.sharded) on CPU ranks: the
row partition, and two / three gloo ranks whose shards (a dense stand-in for
the device shard, P_k = alpha W[:, rows_k] K[rows_k, :] V B + rank-0 terms)
are summed by the all-reduce into the full apply on every rank, with the mass
term and beta C counted once."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from baemm_b200.sharded import ShardedBoundaryApply, row_ranges


@pytest.mark.parametrize("n,world", [(153600, 8), (1000, 3), (100, 4), (129, 2), (0, 2), (5000, 1)])
def test_row_ranges_partition(n, world):
    rr = row_ranges(n, world)
    assert len(rr) == world
    assert rr[0][0] == 0 and rr[-1][1] == n
    for (a0, a1), (b0, b1) in zip(rr, rr[1:]):
        assert a1 == b0 and a0 <= a1
    for r0, r1 in rr:
        assert r0 % 128 == 0 and (r1 % 128 == 0 or r1 == n)
    sizes = [r1 - r0 for r0, r1 in rr]
    if n >= 128 * world:
        assert max(sizes) - min(sizes) <= 128


def _problem(nv, nt, wc, seed=0):
    rng = np.random.default_rng(seed)
    c = lambda *s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    return {"W": c(nv, nt), "K": c(nt, nt), "V": c(nt, nv), "M": c(nv, nv), "c0": 0.5 - 0.25j,
            "B": c(nv, wc + 2), "C": c(nv, wc + 1)}


def _partial_for(p, wc):
    def partial(alpha, B, beta, P, r0, r1, with_mass):
        Bn = B.numpy()[:, :wc]
        out = alpha * p["W"][:, r0:r1] @ (p["K"][r0:r1, :] @ (p["V"] @ Bn))
        if with_mass:
            out = out + alpha * p["c0"] * (p["M"] @ Bn)
        if complex(beta) != 0:
            out = out + beta * P.numpy()
        P.copy_(torch.from_numpy(out))
    return partial


def _worker(rank, world, port, q, nv, nt, wc):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        p = _problem(nv, nt, wc)
        S = ShardedBoundaryApply(n_rows=nt, wave_count=wc, partial=_partial_for(p, wc))
        B = torch.from_numpy(p["B"])
        C = torch.from_numpy(p["C"].copy())
        alpha, beta = 0.75 + 0.5j, -0.25 + 1j
        S(alpha, B, beta, C)
        first = C.numpy().copy()
        S(alpha, B, 0.0, C)          # a second call reuses the buffer; beta = 0 overwrites
        q.put((rank, (S.r0, S.r1), first, C.numpy()))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.mark.parametrize("world,nt", [(2, 300), (3, 700)])
def test_shards_sum_to_the_apply_on_every_rank(world, nt):
    nv, wc = 40, 6
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, nv, nt, wc)) for r in range(world)]
    for pr in procs:
        pr.start()
    out = sorted((q.get(timeout=120) for _ in range(world)), key=lambda t: t[0])
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    p = _problem(nv, nt, wc)
    A = p["W"] @ p["K"] @ p["V"] + p["c0"] * p["M"]
    Bn = p["B"][:, :wc]
    alpha, beta = 0.75 + 0.5j, -0.25 + 1j
    C1 = alpha * A @ Bn + beta * p["C"][:, :wc]
    C2 = alpha * A @ Bn                      # second call, beta = 0
    assert [o[1] for o in out] == row_ranges(nt, world)
    for _, _, first, second in out:
        assert np.allclose(first[:, :wc], C1, rtol=1e-12, atol=1e-9)
        assert np.allclose(second[:, :wc], C2, rtol=1e-12, atol=1e-9)
        assert np.array_equal(second[:, wc:], p["C"][:, wc:])   # columns beyond wave_count untouched


def test_single_process_runs_without_a_group():
    nv, nt, wc = 20, 200, 4
    p = _problem(nv, nt, wc, seed=1)
    S = ShardedBoundaryApply(n_rows=nt, wave_count=wc, partial=_partial_for(p, wc))
    assert (S.rank, S.world, S.r0, S.r1) == (0, 1, 0, nt)
    C = torch.from_numpy(p["C"].copy())
    S(2.0, torch.from_numpy(p["B"]), 0.5, C)
    A = p["W"] @ p["K"] @ p["V"] + p["c0"] * p["M"]
    assert np.allclose(C.numpy()[:, :wc], 2.0 * A @ p["B"][:, :wc] + 0.5 * p["C"][:, :wc])
