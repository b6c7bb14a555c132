"""Row-sharded boundary-operator apply over several GPUs, one process per GPU.

The apply C = alpha A B + beta C with A = AvOp^T (K + diag) AvOp + c0 M splits
by target triangles: rank k owns the contiguous rows [r0_k, r1_k) (whole
128-triangle blocks, balanced) and computes, against every source,

    P_k = alpha AvOp^T|rows_k (K[rows_k, :] + diag) AvOp B   (+ alpha c0 M B + beta C on rank 0),

with baemm_apply_boundary_operators_rows_dev_*; one all-reduce (sum) of the
vertex block over the process group gives every rank C = sum_k P_k.  Each rank
holds the whole mesh and B (the right-hand sides are small next to the
O(N^2) work).  The exchange is nv x wave_count complex values per apply
(39 MB for the 153600-triangle torus with 64 right-hand sides: tens of
microseconds over NVLink against ~150 ms of kernel time), so it is a plain
NCCL all-reduce after the kernel rather than fused into it.
"""
from __future__ import annotations

import math

__all__ = ["row_ranges", "ShardedBoundaryApply"]


def row_ranges(n_rows: int, world: int, align: int = 128):
    """Contiguous, balanced ranges [r0, r1) covering [0, n_rows), cut at
    multiples of `align` (the tensor-core target block) where possible."""
    if world < 1:
        raise ValueError("world must be >= 1")
    blocks = math.ceil(n_rows / align) if n_rows > 0 else 0
    out = []
    for k in range(world):
        b0 = (k * blocks) // world
        b1 = ((k + 1) * blocks) // world
        out.append((min(n_rows, b0 * align), min(n_rows, b1 * align)))
    return out


class ShardedBoundaryApply:
    """C = alpha A B + beta C of the loaded operators of `H`, this rank's rows
    computed here and the shards summed by an all-reduce over `group`.

    Call with torch tensors on this rank's device: B (vertex_count x >= wc) and
    C (vertex_count x >= wc); every rank passes the same B, alpha and beta and
    receives the full result in C.  `partial` replaces the device computation
    of a shard (tests of the orchestration on CPU ranks); it is called as
    partial(alpha, B, beta, P, r0, r1, with_mass) and must write P.
    Without an initialised process group the apply runs on this process alone.
    """

    def __init__(self, H=None, n_rows: int | None = None, wave_count: int | None = None, group=None, partial=None):
        import torch.distributed as dist
        self.group = group
        if dist.is_available() and dist.is_initialized():
            self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        else:
            self.rank, self.world = 0, 1
        n_rows = H.SimplexCount() if n_rows is None else n_rows
        self.wc = H.GetWaveCount() if wave_count is None else wave_count
        self.r0, self.r1 = row_ranges(n_rows, self.world)[self.rank]
        if partial is None:
            def partial(alpha, B, beta, P, r0, r1, with_mass):
                H.ApplyBoundaryOperatorsRows(alpha, B, beta, P, r0, r1, with_mass)
        self._partial = partial
        self._buf = None

    def __call__(self, alpha, B, beta, C):
        import torch
        import torch.distributed as dist
        wc = self.wc
        if self._buf is None or self._buf.shape != (C.shape[0], wc) or self._buf.dtype != C.dtype \
                or self._buf.device != C.device:
            self._buf = torch.empty((C.shape[0], wc), dtype=C.dtype, device=C.device)
        P = self._buf
        first = self.rank == 0
        if first and complex(beta) != 0:
            P.copy_(C[:, :wc])
        self._partial(alpha, B, beta if first else 0.0, P, self.r0, self.r1, first)
        if self.world > 1:
            dist.all_reduce(torch.view_as_real(P), op=dist.ReduceOp.SUM, group=self.group)
        C[:, :wc].copy_(P)
        return C
