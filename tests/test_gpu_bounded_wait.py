"""GPU test of the tensor-core kernel's bounded pipeline waits: a wait on an
mbarrier that nothing arrives on gives up after its bound, reports its error
code, and the device keeps working (no fault, trap or hang is involved)."""
import ctypes as C

import numpy as np
import pytest

from baemm_b200 import APPLY_TC, Helmholtz_CUDA, _capi, meshes
from tests.helpers import crandn, relerr

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_reports_and_device_stays_usable():
    L = _capi.lib()
    ms, code = C.c_double(0.0), C.c_int32(0)
    assert L.baemm_selftest_bounded_wait(0, C.byref(ms), C.byref(code)) == 0
    assert code.value == 99                  # the code the waiting stage was given
    assert 190.0 <= ms.value <= 2000.0, ms.value   # the 200 ms bound, checked every 64 tests
    # the next tensor-core apply runs and agrees with the FP64 oracle
    from oracle import oracle as O
    c, t = meshes.icosphere(2)
    rng = np.random.default_rng(2)
    B = crandn(rng, c.shape[0], 16)
    kap, coeff = np.array([3.0]), np.array([[0.5, -3j, 1.0, 0.0]])
    Cg, Co = np.zeros_like(B), np.zeros_like(B)
    with Helmholtz_CUDA(c, t, np.eye(3)) as H:
        H.SetApplyMode(APPLY_TC)
        H.ApplyBoundaryOperators_PL(1.0, B, 0.0, Cg, kap, coeff, 16, 16)
    O.Oracle(c, t, np.eye(3), precision=64).ApplyBoundaryOperators_PL(1.0, B, 0.0, Co, kap, coeff, 16, 16)
    assert relerr(Cg, Co) < 1e-5


def test_bounded_wait_rejects_a_bad_device():
    L = _capi.lib()
    ms, code = C.c_double(0.0), C.c_int32(0)
    assert L.baemm_selftest_bounded_wait(-1, C.byref(ms), C.byref(code)) == 1   # BAEMM_ERR_ARG
