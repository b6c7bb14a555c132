"""CPU tests of the C ABI: the library loads without a GPU, exports every
symbol include/baemm.h declares, and rejects bad input on the host before any
device call."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from baemm_b200 import _capi, meshes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "baemm.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(baemm_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _capi.lib()
    syms = header_symbols()
    assert len(syms) >= 50
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    # the ctypes binding covers exactly the declared entry points
    assert sorted(_capi.SIGNATURES) == syms


def test_class_name_without_gpu():
    assert _capi.lib().baemm_class_name() == b"Helmholtz_CUDA"


def test_create_rejects_bad_mesh_on_host():
    L = _capi.lib()
    coords, tris = meshes.icosphere(0)
    tris = tris.copy()
    tris[3, 1] = coords.shape[0]          # out of range
    h = C.c_void_p()
    st = L.baemm_create(coords.ctypes.data_as(_capi.dp), coords.shape[0], tris.ctypes.data_as(_capi.i64p),
                        tris.shape[0], None, 0, 0, 1, C.byref(h))
    assert st == 1 and not h.value
    assert b"out of range" in L.baemm_last_error(None)
    st = L.baemm_create(None, 0, None, 0, None, 0, 0, 1, C.byref(h))
    assert st == 1


def test_create_refuses_meshes_beyond_the_int32_sparse_limit():
    """More than 2^28 triangles or vertices: BAEMM_ERR_SIZE from both index
    widths, before any triangle index is read (the arrays here are tiny)."""
    L = _capi.lib()
    coords, tris = meshes.icosphere(0)
    t32 = tris.astype(np.int32)
    big = (1 << 28) + 1
    for nv, nt in ((coords.shape[0], big), (big, tris.shape[0])):
        h = C.c_void_p()
        st = L.baemm_create(coords.ctypes.data_as(_capi.dp), nv, tris.ctypes.data_as(_capi.i64p), nt, None, 0, 0,
                            1, C.byref(h))
        assert st == 6 and not h.value and b"too large" in L.baemm_last_error(None)
        st = L.baemm_create_i32(coords.ctypes.data_as(_capi.dp), nv, t32.ctypes.data_as(_capi.i32p), nt, None, 0,
                                0, 1, C.byref(h))
        assert st == 6 and not h.value


def test_null_context_is_rejected():
    L = _capi.lib()
    assert L.baemm_synchronize(None) == 1
    assert L.baemm_vertex_count(None) == -1
    assert L.baemm_autotune(None, 1, 1, None) == 1
    L.baemm_destroy(None)   # no-op


def test_device_block_check_refuses_host_tensors_and_bad_shapes():
    """The torch-block check of the Python mirror runs before any device call:
    host tensors are refused, and (through a stand-in with a CUDA device) too
    few rows or columns, a column stride and another dtype are refused."""
    import torch
    from baemm_b200.helmholtz import _check_dev
    with pytest.raises(TypeError):
        _check_dev(torch.zeros((4, 2), dtype=torch.complex64), torch.complex64, 4, 2, 0, "B")

    class Fake(torch.Tensor):
        """A CPU tensor that reports itself as living on cuda:0 (host logic only)."""
        @property
        def is_cuda(self):
            return True

        @property
        def device(self):
            return torch.device("cuda", 0)

    def fake(t):
        return t.as_subclass(Fake)

    ok = fake(torch.zeros((10, 8), dtype=torch.complex64))
    _check_dev(ok, torch.complex64, 10, 8, 0, "B")
    _check_dev(fake(torch.zeros((10, 12), dtype=torch.complex64)[:, :8]), torch.complex64, 10, 8, 0, "B")
    with pytest.raises(ValueError, match="hold"):
        _check_dev(ok, torch.complex64, 11, 8, 0, "B")
    with pytest.raises(ValueError, match="hold"):
        _check_dev(ok, torch.complex64, 10, 9, 0, "B")
    with pytest.raises(ValueError, match="unit column stride"):
        _check_dev(fake(torch.zeros((8, 10), dtype=torch.complex64).t()), torch.complex64, 10, 8, 0, "B")
    with pytest.raises(TypeError, match="must be"):
        _check_dev(ok, torch.complex128, 10, 8, 0, "B")
    with pytest.raises(ValueError, match="context on cuda:1"):
        _check_dev(ok, torch.complex64, 10, 8, 1, "B")
