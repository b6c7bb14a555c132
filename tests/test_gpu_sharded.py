"""GPU check of the row shards of the boundary apply (the unit of the
multi-GPU apply, baemm_b200.sharded), through the C ABI on one GPU: the shards
of a partition of the triangles, with the mass term and beta C on one shard,
sum to the full apply.  Ranges that are not multiples of the 128-triangle block
and empty ranges included; every arithmetic form; coefficients with the
adjoint double layer (the target normals of a shard).

Tolerances: FP64 within 1e-12 of the full FP64 apply (only the summation order
of AvOp^T across shards differs); FP32 and tensor-core within 1e-6 of the full
apply of the same form and 1e-5 of the FP64 oracle.
"""
import numpy as np
import pytest

from baemm_b200 import APPLY_FP32, APPLY_FP64, APPLY_TC, Helmholtz_CUDA, _capi, meshes
from baemm_b200.sharded import ShardedBoundaryApply, row_ranges
from oracle import oracle as O
from tests.helpers import crandn, relerr

pytestmark = pytest.mark.gpu

KAP = [2.0, 5.0, 9.0, 13.0]
COEFF = {
    "all": np.array([[0.25 + 1j, 1 + 0.5j, 1 - 2j, 0.3j]] * 4, np.complex128),
    "bie": np.array([[0.5, -1j * k, 1, 0] for k in KAP], np.complex128),
}


@pytest.fixture(scope="module")
def env():
    coords, tris = meshes.icosphere(3)
    H = Helmholtz_CUDA(coords, tris, np.eye(3))
    o64 = O.Oracle(coords, tris, np.eye(3), precision=64)
    yield coords, tris, H, o64
    H.close()


def _shard_sum(H, B, C0, alpha, beta, ranges, dtype):
    import torch
    total = None
    for k, (r0, r1) in enumerate(ranges):
        P = C0.clone() if k == 0 else torch.full_like(C0, float("nan"))   # beta = 0 must overwrite
        H.ApplyBoundaryOperatorsRows(alpha, B, beta if k == 0 else 0.0, P, r0, r1, with_mass=(k == 0))
        total = P if total is None else total + P
    torch.cuda.synchronize()
    return total.cpu().numpy().astype(np.complex128)


@pytest.mark.parametrize("mode", [APPLY_FP32, APPLY_TC, APPLY_FP64])
@pytest.mark.parametrize("cname", ["all", "bie"])
@pytest.mark.parametrize("split", ["ragged", "blocks", "with_empty"])
def test_row_shards_sum_to_the_apply(env, mode, cname, split):
    import torch
    coords, tris, H, o64 = env
    nt = tris.shape[0]
    ranges = {"ragged": [(0, 500), (500, 777), (777, nt)],
              "blocks": row_ranges(nt, 3),
              "with_empty": [(0, 0), (0, 1), (1, nt - 1), (nt - 1, nt), (nt, nt)]}[split]
    coeff = COEFF[cname]
    wc = 64
    dt = torch.complex128 if mode == APPLY_FP64 else torch.complex64
    rng = np.random.default_rng(7)
    Bh = crandn(rng, coords.shape[0], wc)
    Ch = crandn(rng, coords.shape[0], wc)
    B = torch.from_numpy(Bh).to(dt).cuda()
    C0 = torch.from_numpy(Ch).to(dt).cuda()
    alpha, beta = 0.5 - 1j, 0.25 + 0.5j
    H.LoadBoundaryOperators_PL(KAP, coeff, wc, 16)
    H.SetApplyMode(mode)
    try:
        full = C0.clone()
        H.ApplyBoundaryOperators_PL(alpha, B, beta, full)
        full = full.cpu().numpy().astype(np.complex128)
        shards = _shard_sum(H, B, C0, alpha, beta, ranges, dt)
    finally:
        H.SetApplyMode(APPLY_FP32)
        H.UnloadBoundaryOperators_PL()
    ref = Ch.copy()
    o64.ApplyBoundaryOperators_PL(alpha, Bh, beta, ref, KAP, coeff, wc, 16)
    if mode == APPLY_FP64:
        assert relerr(shards, full) < 1e-12
    else:
        assert relerr(shards, full) < 1e-6
        assert relerr(shards, ref) < 1e-5


@pytest.mark.parametrize("variant", [0, 2])
def test_row_shards_of_the_packed_and_scalar_kernels(env, variant):
    """The FP32 dense variants read the adjoint-double-layer target normals of a
    shard at the shard's offset."""
    import torch
    coords, tris, H, o64 = env
    wc = 32
    B = torch.from_numpy(crandn(np.random.default_rng(3), coords.shape[0], wc).astype(np.complex64)).cuda()
    C0 = torch.zeros_like(B)
    H.LoadBoundaryOperators_PL(KAP[:2], COEFF["all"][:2], wc, 16)
    H.SetTuning(_capi.TUNE_DENSE_VARIANT, variant)
    try:
        full = C0.clone()
        H.ApplyBoundaryOperators_PL(1.0, B, 0.0, full)
        shards = _shard_sum(H, B, C0, 1.0, 0.0, [(0, 300), (300, 1001), (1001, tris.shape[0])], torch.complex64)
    finally:
        H.SetTuning(_capi.TUNE_DENSE_VARIANT, 0)
        H.UnloadBoundaryOperators_PL()
    assert relerr(shards, full.cpu().numpy()) < 1e-6


def test_sharded_apply_without_a_group_is_the_apply(env):
    """ShardedBoundaryApply in a single process (no process group): the apply."""
    import torch
    coords, tris, H, o64 = env
    wc = 64
    B = torch.from_numpy(crandn(np.random.default_rng(4), coords.shape[0], wc)).cuda()
    C = torch.from_numpy(crandn(np.random.default_rng(5), coords.shape[0], wc + 3)).cuda()
    C_full = C.clone()
    H.LoadBoundaryOperators_PL(KAP, COEFF["bie"], wc, 16)
    try:
        H.ApplyBoundaryOperators_PL(1.5, B, -0.5, C_full)
        ShardedBoundaryApply(H)(1.5, B, -0.5, C)
        torch.cuda.synchronize()
    finally:
        H.UnloadBoundaryOperators_PL()
    assert relerr(C.cpu().numpy(), C_full.cpu().numpy()) < 1e-12


def test_row_range_is_checked(env):
    import torch
    coords, tris, H, o64 = env
    B = torch.zeros((coords.shape[0], 16), dtype=torch.complex128, device="cuda")
    H.LoadBoundaryOperators_PL([2.0], COEFF["all"][:1], 16, 16)
    try:
        with pytest.raises(Exception):
            H.ApplyBoundaryOperatorsRows(1.0, B, 0.0, B.clone(), 10, tris.shape[0] + 1)
        with pytest.raises(Exception):
            H.ApplyBoundaryOperatorsRows(1.0, B, 0.0, B.clone(), 20, 10)
    finally:
        H.UnloadBoundaryOperators_PL()
