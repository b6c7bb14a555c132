"""GPU test of the allocation-free boundary apply (collected last on purpose).

baemm_apply_boundary_operators_noalloc_dev_c serves callers that cannot
allocate device memory while they run (a host framework that owns all device
memory, a server that must not grow its footprint, a loop that cannot afford
cudaMalloc's implicit synchronisation): its intermediate blocks live in a fixed
32 MiB device array of the library.  Called through the C ABI on a fresh
context, it must leave the free device memory unchanged from its second call
on, give the same result as the allocating device-pointer apply on two calls in
a row (the array keeps the previous call's contents), and reject problems
larger than its array.
"""
import ctypes as C

import numpy as np
import pytest

from baemm_b200 import Helmholtz_CUDA, _capi, meshes
from tests.helpers import relerr

pytestmark = pytest.mark.gpu

TOL = 1e-6   # same kernels as the allocating path: agreement is expected to be exact


def _call(fn, H, B, Cd):
    one = np.array([1.0, 0.0], np.float32)
    zero = np.array([0.0, 0.0], np.float32)
    st = fn(H._h, one.ctypes.data_as(_capi.fp), C.c_void_p(B.data_ptr()), B.stride(0),
            zero.ctypes.data_as(_capi.fp), C.c_void_p(Cd.data_ptr()), Cd.stride(0))
    return st


def test_noalloc_apply_matches_allocating_apply_twice():
    import torch
    L = _capi.lib()
    coords, tris = meshes.icosphere(3)
    meas = meshes.fibonacci_sphere(16)
    kappa = np.array([2.0, 7.0])
    coeff = np.array([[0.5, -1j * k, 1.0, 0.25j] for k in kappa])
    with Helmholtz_CUDA(coords, tris, meas) as H:
        H.LoadBoundaryOperators_PL(kappa, coeff, 32, 16)
        rng = np.random.default_rng(99)
        B = torch.from_numpy((rng.standard_normal((coords.shape[0], 32)) +
                              1j * rng.standard_normal((coords.shape[0], 32))).astype(np.complex64)).cuda()
        # every torch block exists before the first no-alloc call, so torch allocates nothing in between
        outs = [torch.full_like(B, complex(np.nan, np.nan)) for _ in range(2)]
        C_ref = torch.zeros_like(B)
        torch.cuda.synchronize()
        free = []
        for C_na in outs:   # the first call on this context (array lookup, kernel loading), then a second
            st = _call(L.baemm_apply_boundary_operators_noalloc_dev_c, H, B, C_na)
            assert st == 0, L.baemm_last_error(H._h)
            H.Synchronize()
            free.append(torch.cuda.mem_get_info()[0])
        assert free[1] == free[0], "the second no-alloc call changed the free device memory"
        assert _call(L.baemm_apply_boundary_operators_dev_c, H, B, C_ref) == 0
        H.Synchronize()
        ref = C_ref.cpu().numpy()
        assert np.isfinite(ref).all() and np.abs(ref).max() > 0
        for C_na in outs:
            assert relerr(C_na.cpu().numpy(), ref) < TOL
        H.UnloadBoundaryOperators_PL()


def test_noalloc_apply_rejects_oversize_problem():
    import torch
    L = _capi.lib()
    coords, tris = meshes.icosphere(5)          # 20480 triangles x 128 RHS needs 40 MiB > 32 MiB
    with Helmholtz_CUDA(coords, tris, meshes.fibonacci_sphere(4)) as H:
        wc = 128
        H.LoadBoundaryOperators_PL(np.ones(8), np.array([[0, 1, 0, 0]] * 8), wc, 16)
        B = torch.zeros((coords.shape[0], wc), dtype=torch.complex64, device="cuda")
        Cd = torch.zeros_like(B)
        st = _call(L.baemm_apply_boundary_operators_noalloc_dev_c, H, B, Cd)
        assert st == 6   # BAEMM_ERR_SIZE
        assert b"no-alloc scratch" in L.baemm_last_error(H._h)
        H.UnloadBoundaryOperators_PL()
