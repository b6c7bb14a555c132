"""Host logic of the Python mirror without a GPU: which C entry point each
call form of the reference's overloaded wave builders reaches, with which
wave type, and which malformed calls are refused before any call.  The
library is replaced by a recorder; nothing runs on a device."""
import numpy as np
import pytest

from baemm_b200 import helmholtz
from baemm_b200.helmholtz import Helmholtz_CUDA, WaveType


class _Recorder:
    def __init__(self):
        self.calls = []

    def __getattr__(self, name):
        def entry(*args):
            self.calls.append((name, args))
            return 0
        return entry


def _mirror(nv=4, wcs=2, nm=3):
    H = Helmholtz_CUDA.__new__(Helmholtz_CUDA)
    H._lib, H._h, H._user_stream, H._device = _Recorder(), None, None, 0
    H.VertexCount = lambda: nv
    H.GetWaveChunkSize = lambda: wcs
    H.GetMeasCount = lambda: nm
    return H


def _last(H):
    name, args = H._lib.calls[-1]
    return name, args


def test_incident_wave_call_forms():
    H = _mirror()
    dirs = np.eye(3)[:2]
    C = np.zeros((4, 4), complex)
    H.CreateIncidentWave_PL(1.0, dirs, 0.0, C, [2.0, 3.0], [[0, 1, 0, 0]] * 2, 4, 2)
    name, args = _last(H)
    assert name == "baemm_create_incident_wave_z" and args[-1] == int(WaveType.Plane)
    H.CreateIncidentWave_PL(1.0, dirs, 0.0, C, [2.0, 3.0], [[0, 1, 0, 0]] * 2, 4, 2, WaveType.Radial)
    assert _last(H)[0] == "baemm_create_incident_wave_z" and _last(H)[1][-1] == int(WaveType.Radial)
    H.CreateIncidentWave_PL(1.0, dirs, 0.0, C)
    name, args = _last(H)
    assert name == "baemm_create_incident_wave_loaded_z" and args[-1] == int(WaveType.Plane)
    H.CreateIncidentWave_PL(1.0, dirs, 0.0, C, WaveType.Radial)
    assert _last(H)[1][-1] == int(WaveType.Radial)
    H.CreateIncidentWave_PL(1.0, dirs, 0.0, C, wave_type=WaveType.Radial)
    assert _last(H)[1][-1] == int(WaveType.Radial)
    n = len(H._lib.calls)
    with pytest.raises(ValueError, match="wave_chunk_size incident directions"):
        H.CreateIncidentWave_PL(1.0, dirs[:1], 0.0, C)
    with pytest.raises(TypeError):
        H.CreateIncidentWave_PL(1.0, dirs, 0.0, C, [2.0], [[0, 1, 0, 0]])
    with pytest.raises(ValueError, match="vertex_count rows"):
        H.CreateIncidentWave_PL(1.0, dirs, 0.0, np.zeros((3, 4), complex))
    assert len(H._lib.calls) == n   # refused before any call


def test_herglotz_wave_call_forms():
    H = _mirror()
    g = np.ones((3, 4), complex)
    C = np.zeros((4, 4), complex)
    H.CreateHerglotzWave_PL(1.0, g, 0.0, C, [2.0, 3.0], [[0, 1, 0, 0]] * 2, 4, 2)
    assert _last(H)[0] == "baemm_create_herglotz_wave_z"
    H.CreateHerglotzWave_PL(1.0, g, 0.0, C)
    assert _last(H)[0] == "baemm_create_herglotz_wave_loaded_z"
    n = len(H._lib.calls)
    with pytest.raises(ValueError, match="meas_count rows"):
        H.CreateHerglotzWave_PL(1.0, g[:2], 0.0, C)
    with pytest.raises(TypeError):
        H.CreateHerglotzWave_PL(1.0, g, 0.0, C, [2.0])
    with pytest.raises(TypeError):
        H.CreateHerglotzWave_PL(1.0, g, 0.0, C.astype(np.complex64))
    assert len(H._lib.calls) == n


def test_wave_type_values_match_the_c_header():
    assert int(WaveType.Plane) == helmholtz._capi.WAVE_PLANE
    assert int(WaveType.Radial) == helmholtz._capi.WAVE_RADIAL


def test_apply_call_forms():
    """ApplyBoundaryOperators_PL / ApplyFarFieldOperators_PL /
    ApplyNearFieldOperators_PL on host blocks: the overload with parameters
    loads (and for the boundary apply unloads) around the loaded form."""
    H = _mirror()
    B = np.ones((4, 4), complex)
    C = np.zeros((4, 4), complex)
    kap, coeff = [2.0, 3.0], [[0, 1, 0, 0]] * 2
    H.ApplyBoundaryOperators_PL(1.0, B, 0.0, C)
    assert _last(H)[0] == "baemm_apply_boundary_operators_z"
    H._lib.calls.clear()
    H.ApplyBoundaryOperators_PL(1.0, B, 0.0, C, kap, coeff, 4, 2)
    assert [c[0] for c in H._lib.calls] == ["baemm_load_boundary_operators", "baemm_apply_boundary_operators_z",
                                            "baemm_unload_boundary_operators"]
    H.ApplyBoundaryOperators_PL(1.0, B.astype(np.complex64), 0.0, C.astype(np.complex64))
    assert _last(H)[0] == "baemm_apply_boundary_operators_c"
    F = np.zeros((3, 4), complex)
    H.ApplyFarFieldOperators_PL(1.0, B, 0.0, F)
    assert _last(H)[0] == "baemm_apply_far_field_operators_loaded_z"
    H.ApplyFarFieldOperators_PL(1.0, B, 0.0, F, kap, coeff, 4, 2)
    assert _last(H)[0] == "baemm_apply_far_field_operators_z"
    P = np.zeros((5, 4), complex)
    pts = np.zeros((5, 3))
    H.ApplyNearFieldOperators_PL(1.0, B, 0.0, P, pts)
    assert _last(H)[0] == "baemm_apply_near_field_operators_z" and _last(H)[1][-1] == 5
    H.ApplyNearFieldOperators_PL(1.0, B, 0.0, P, kap, coeff, 4, 2, pts)
    assert _last(H)[0] == "baemm_apply_near_field_operators_full_z"
    with pytest.raises(TypeError):
        H.ApplyNearFieldOperators_PL(1.0, B, 0.0, P, kap, pts)


def test_host_blocks_are_checked_before_any_call():
    """Blocks the library reads or writes through plain pointers must hold the
    rows and columns it will touch: too few rows, another dtype, a strided
    output, or (where the entry point has no leading dimension) another column
    count is refused before any call; the shapes the reference uses pass."""
    nv, nm = 4, 3
    H = _mirror(nv=nv, nm=nm)
    kap, inc = np.array([2.0, 3.0]), np.eye(3)[:2]          # wave_count 2 x 2 = 4
    ok = [
        lambda: H.ApplyMassInverse(np.ones((nv, 2), complex), np.zeros((nv, 2), complex), 1e-10),
        lambda: H.ApplyMassInverse(np.ones((nv, 3)), np.zeros((nv, 3)), 1e-10),
        lambda: H.ApplyMassInverse(np.ones(nv), np.zeros(nv), 1e-10),
        lambda: H.ApplyLumpedMassInverse(np.ones((nv, 3)), np.zeros((nv, 3))),
        lambda: H.MassDot(1.0, np.ones((nv, 3)), 0.0, np.zeros((nv, 3))),
        lambda: H.FarField(kap, inc, np.zeros((nm, 4), complex)),
        lambda: H.BoundaryPotential(kap, np.zeros((2, 4), complex), np.ones((nv, 4), complex),
                                    np.zeros((nv, 4), complex), 2, 1e-10, 1e-10),
        lambda: H.DirichletToNeumann(kap, np.ones((nv, 4), complex), np.zeros((nv, 4), complex), 2, 1e-10, 1e-10),
        lambda: H.Derivative_FF_Helper(kap, inc, np.zeros((nv, 4), complex)),
        lambda: H.Derivative_FF(kap, inc, np.ones((nv, 3)), np.zeros((nm, 4), complex), np.zeros((nv, 4), complex)),
        lambda: H.AdjointDerivative_FF(kap, inc, np.ones((nm, 4), complex), np.zeros((nv, 3)),
                                       np.zeros((nv, 4), complex)),
        lambda: H.GaussNewtonSolve(kap, inc, None, None, 1.0, np.ones((nv, 3)), 0.0, np.zeros((nv, 3)),
                                   np.zeros((nv, 4), complex)),
    ]
    for f in ok:
        n = len(H._lib.calls)
        f()
        assert len(H._lib.calls) > n
    bad = [
        lambda: H.ApplyMassInverse(np.ones((nv, 2), complex), np.zeros((nv - 1, 2), complex), 1e-10),
        lambda: H.ApplyMassInverse(np.ones((nv - 1, 2), complex), np.zeros((nv, 2), complex), 1e-10),
        lambda: H.ApplyMassInverse(np.ones((nv, 3)), np.zeros((nv, 3), np.float32), 1e-10),
        lambda: H.ApplyMassInverse(np.ones((nv, 3)), np.zeros((nv, 6))[:, ::2], 1e-10),
        lambda: H.ApplyLumpedMassInverse(np.ones((nv, 3)), np.zeros((nv, 2))),
        lambda: H.MassDot(1.0, np.ones((nv, 3)), 0.0, np.zeros((nv - 1, 3))),
        lambda: H.FarField(kap, inc, np.zeros((nm, 5), complex)),
        lambda: H.FarField(kap, inc, np.zeros((nm - 1, 4), complex)),
        lambda: H.BoundaryPotential(kap, np.zeros((2, 4), complex), np.ones((nv, 4), complex),
                                    np.zeros((nv, 3), complex), 2, 1e-10, 1e-10),
        lambda: H.BoundaryPotential(kap, np.zeros((1, 4), complex), np.ones((nv, 4), complex),
                                    np.zeros((nv, 4), complex), 2, 1e-10, 1e-10),
        lambda: H.DirichletToNeumann(kap, np.ones((nv - 1, 4), complex), np.zeros((nv, 4), complex), 2, 1e-10,
                                     1e-10),
        lambda: H.Derivative_FF_Helper(kap, inc, np.zeros((nv, 3), complex)),
        lambda: H.Derivative_FF(kap, inc, np.ones((nv - 1, 3)), np.zeros((nm, 4), complex)),
        lambda: H.AdjointDerivative_FF(kap, inc, np.ones((nm, 4), complex), np.zeros((nv, 3), np.float32)),
        lambda: H.GaussNewtonSolve(kap, inc, None, None, 1.0, np.ones((nv, 3)), 0.0, np.zeros((nv, 2)), None),
        lambda: H.ApplyBoundaryOperators_PL(1.0, np.ones((nv - 1, 4), complex), 0.0, np.zeros((nv, 4), complex)),
        lambda: H.ApplyFarFieldOperators_PL(1.0, np.ones((nv, 4), complex), 0.0, np.zeros((nm - 1, 4), complex)),
        lambda: H.ApplyNearFieldOperators_PL(1.0, np.ones((nv, 4), complex), 0.0, np.zeros((2, 4), complex),
                                             np.zeros((3, 3))),
    ]
    for f in bad:
        n = len(H._lib.calls)
        with pytest.raises((TypeError, ValueError)):
            f()
        assert len(H._lib.calls) == n
