"""GPU parity of the near-field potential (ApplyNearFieldOperators_PL) against
the oracle, through the C ABI.  The oracle's near-field kernel is pinned to the
reference's own NearFieldOperatorKernel.cl (tests/test_oracle.py).

Tolerances (relative, Frobenius): the FP32 path within 1e-5 of the FP32 oracle;
FP32 and tensor-core paths within 1e-5 of the FP64 oracle;
the FP64 path within 1e-11 of the FP64 oracle.
"""
import numpy as np
import pytest

from baemm_b200 import APPLY_FP32, APPLY_FP64, APPLY_TC, Helmholtz_CUDA, _capi, meshes
from oracle import oracle as O
from tests.helpers import crandn, relerr

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-5
FP32_VS64_TOL = 1e-5
FP64_TOL = 1e-11

COEFFS = {
    "sl": [0, 1, 0, 0],
    "dl": [0, 0, 1, 0],
    "bie": None,                              # (0.5, -i kappa, 1, 0), the mixed BIE tuple
    "all": [0.25 + 1j, 1 + 0.5j, 1 - 2j, 0.3j],
}
WAVES = {  # name: (wave_count, wave_chunk_size, kappa list)
    "w16": (16, 16, [2.0]),
    "w32": (32, 16, [4.0, 8.0]),
    "w8x4": (8, 4, [1.0, 3.0]),
    "w64": (64, 16, [2.0, 4.0, 8.0, 16.0]),
    "w64x32": (64, 32, [3.0, 6.0]),
    "w64x64": (64, 64, [3.0]),
}


def _coeff(name, kap):
    return np.array([COEFFS[name] if name != "bie" else [0.5, -1j * k, 1, 0] for k in kap], np.complex128)


def _points(rng, m):
    """Points inside and outside the unit sphere, at least 0.05 from it."""
    d = rng.standard_normal((m, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.concatenate([rng.uniform(0.1, 0.95, m // 2), rng.uniform(1.05, 3.0, m - m // 2)])
    return d * r[:, None]


@pytest.fixture(scope="module")
def env():
    coords, tris = meshes.icosphere(3)
    meas = meshes.fibonacci_sphere(16)
    H = Helmholtz_CUDA(coords, tris, meas)
    o32 = O.Oracle(coords, tris, meas, precision=32)
    o64 = O.Oracle(coords, tris, meas, precision=64)
    pts = _points(np.random.default_rng(99), 300)
    yield coords, tris, H, o32, o64, pts
    H.close()


def _run(H, mode, *args):
    H.SetApplyMode(mode)
    try:
        return H.ApplyNearFieldOperators_PL(*args)
    finally:
        H.SetApplyMode(APPLY_FP32)


@pytest.mark.parametrize("cname", list(COEFFS))
@pytest.mark.parametrize("wname", ["w16", "w32", "w8x4"])
def test_nearfield_fp32(env, cname, wname):
    coords, tris, H, o32, o64, pts = env
    wc, wcs, kap = WAVES[wname]
    coeff = _coeff(cname, kap)
    rng = np.random.default_rng(hash((cname, wname)) % 2**32)
    B = crandn(rng, coords.shape[0], wc + 3)          # ld > wave_count
    C0 = crandn(rng, pts.shape[0], wc + 1)
    alpha, beta = 0.7 - 0.2j, 0.3 + 0.1j
    Cg = C0.copy()
    _run(H, APPLY_FP32, alpha, B, beta, Cg, kap, coeff, wc, wcs, pts)
    C32, C64 = C0.copy(), C0.copy()
    o32.ApplyNearFieldOperators_PL(alpha, B, beta, C32, kap, coeff, wc, wcs, pts)
    o64.ApplyNearFieldOperators_PL(alpha, B, beta, C64, kap, coeff, wc, wcs, pts)
    assert relerr(Cg[:, :wc], C32[:, :wc]) < FP32_TOL
    assert relerr(Cg[:, :wc], C64[:, :wc]) < FP32_VS64_TOL
    assert np.array_equal(Cg[:, wc:], C0[:, wc:])   # columns beyond wave_count untouched


@pytest.mark.parametrize("cname", ["sl", "dl", "all"])
@pytest.mark.parametrize("wname", ["w16", "w64", "w64x32", "w8x4"])
def test_nearfield_fp64(env, cname, wname):
    coords, tris, H, o32, o64, pts = env
    wc, wcs, kap = WAVES[wname]
    coeff = _coeff(cname, kap)
    B = crandn(np.random.default_rng(17), coords.shape[0], wc)
    Cg = np.zeros((pts.shape[0], wc), np.complex128)
    _run(H, APPLY_FP64, 1.0, B, 0.0, Cg, kap, coeff, wc, wcs, pts)
    C64 = np.zeros_like(Cg)
    o64.ApplyNearFieldOperators_PL(1.0, B, 0.0, C64, kap, coeff, wc, wcs, pts)
    assert relerr(Cg, C64) < FP64_TOL


@pytest.mark.parametrize("cname", list(COEFFS))
@pytest.mark.parametrize("wname", ["w16", "w32", "w64", "w64x32", "w64x64"])
def test_nearfield_tensor_core(env, cname, wname):
    """Compensated tensor-core form at arbitrary targets (no pair excluded);
    with the BIE tuple, w64x32 and w64x64 evaluate each kernel entry once for
    2 and 4 column groups of one wavenumber."""
    coords, tris, H, o32, o64, pts = env
    wc, wcs, kap = WAVES[wname]
    coeff = _coeff(cname, kap)
    rng = np.random.default_rng(41)
    B = crandn(rng, coords.shape[0], wc + 2)
    C0 = crandn(rng, pts.shape[0], wc)
    Cg = C0.copy()
    _run(H, APPLY_TC, 0.5 - 1j, B, 0.25, Cg, kap, coeff, wc, wcs, pts)
    C64 = C0.copy()
    o64.ApplyNearFieldOperators_PL(0.5 - 1j, B, 0.25, C64, kap, coeff, wc, wcs, pts)
    assert relerr(Cg, C64) < FP32_VS64_TOL


@pytest.mark.parametrize("m", [1, 127, 128, 129, 1000])
@pytest.mark.parametrize("mode", [APPLY_FP32, APPLY_TC, APPLY_FP64])
def test_nearfield_ragged_point_counts(env, m, mode):
    """Point counts that are not multiples of the 128-target block."""
    coords, tris, H, o32, o64, _ = env
    wc, wcs, kap = WAVES["w32"]
    coeff = _coeff("all", kap)
    rng = np.random.default_rng(m)
    pts = _points(rng, m) if m > 1 else np.array([[0.2, -0.1, 0.3]])
    B = crandn(rng, coords.shape[0], wc)
    Cg = np.zeros((m, wc), np.complex128)
    _run(H, mode, 1.0, B, 0.0, Cg, kap, coeff, wc, wcs, pts)
    C64 = np.zeros_like(Cg)
    o64.ApplyNearFieldOperators_PL(1.0, B, 0.0, C64, kap, coeff, wc, wcs, pts)
    assert relerr(Cg, C64) < (FP64_TOL if mode == APPLY_FP64 else FP32_VS64_TOL)


@pytest.mark.parametrize("ctas", [1, 7, 148, 5000])
def test_nearfield_tc_persistent_grid(env, ctas):
    """Target blocks of points split between CTAs (stream-K tail and fix-up);
    repeated calls are bitwise identical at a fixed grid size."""
    coords, tris, H, o32, o64, pts = env
    wc, wcs, kap = WAVES["w64"]
    coeff = _coeff("bie", kap)
    B = crandn(np.random.default_rng(5), coords.shape[0], wc)
    C64 = np.zeros((pts.shape[0], wc), np.complex128)
    o64.ApplyNearFieldOperators_PL(1.0, B, 0.0, C64, kap, coeff, wc, wcs, pts)
    H.SetTuning(_capi.TUNE_TC_CTAS, ctas)
    try:
        C1, C2 = np.zeros_like(C64), np.zeros_like(C64)
        _run(H, APPLY_TC, 1.0, B, 0.0, C1, kap, coeff, wc, wcs, pts)
        _run(H, APPLY_TC, 1.0, B, 0.0, C2, kap, coeff, wc, wcs, pts)
    finally:
        H.SetTuning(_capi.TUNE_TC_CTAS, 0)
    assert relerr(C1, C64) < FP32_VS64_TOL
    assert np.array_equal(C1, C2)


@pytest.mark.parametrize("variant", [0, 1, 2])
def test_nearfield_dense_variants(env, variant):
    """Every plain FP32 dense-kernel variant (scalar, packed x1, packed x2)."""
    coords, tris, H, o32, o64, pts = env
    wc, wcs, kap = WAVES["w64x32"]
    coeff = _coeff("all", kap)
    B = crandn(np.random.default_rng(31), coords.shape[0], wc)
    C32 = np.zeros((pts.shape[0], wc), np.complex128)
    o32.ApplyNearFieldOperators_PL(1.0, B, 0.0, C32, kap, coeff, wc, wcs, pts)
    old = H.GetTuning(_capi.TUNE_DENSE_VARIANT)
    H.SetTuning(_capi.TUNE_DENSE_VARIANT, variant)
    try:
        Cg = np.zeros_like(C32)
        _run(H, APPLY_FP32, 1.0, B, 0.0, Cg, kap, coeff, wc, wcs, pts)
    finally:
        H.SetTuning(_capi.TUNE_DENSE_VARIANT, old)
    assert relerr(Cg, C32) < FP32_TOL


def test_nearfield_leaves_output_alone_without_layers(env):
    """Only mass and adjoint double layer, or no points: C_out untouched (the
    reference returns before its kernel); beta = 0 overwrites NaNs."""
    coords, tris, H, o32, o64, pts = env
    rng = np.random.default_rng(8)
    B = crandn(rng, coords.shape[0], 16)
    C0 = crandn(rng, pts.shape[0], 16)
    C = C0.copy()
    H.ApplyNearFieldOperators_PL(1.0, B, 0.0, C, [2.0], np.array([[1.0, 0, 0, 1.0]]), 16, 16, pts)
    assert np.array_equal(C, C0)
    Cz = np.zeros((0, 16), np.complex128)
    H.ApplyNearFieldOperators_PL(1.0, B, 0.0, Cz, [2.0], np.array([[0, 1.0, 0, 0]]), 16, 16, np.zeros((0, 3)))
    Cn = np.full((pts.shape[0], 16), np.nan, np.complex128)
    H.ApplyNearFieldOperators_PL(1.0, B, 0.0, Cn, [2.0], np.array([[0, 1.0, 0, 0]]), 16, 16, pts)
    assert np.isfinite(Cn).all()


def test_nearfield_mass_and_adjoint_coefficients_ignored(env):
    coords, tris, H, o32, o64, pts = env
    B = crandn(np.random.default_rng(9), coords.shape[0], 16)
    a = np.zeros((pts.shape[0], 16), np.complex128)
    b = np.zeros_like(a)
    H.ApplyNearFieldOperators_PL(1.0, B, 0.0, a, [2.0], np.array([[0, 1.0, 2.0, 0]]), 16, 16, pts)
    H.ApplyNearFieldOperators_PL(1.0, B, 0.0, b, [2.0], np.array([[5.0, 1.0, 2.0, 7.0]]), 16, 16, pts)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("mode", [APPLY_FP32, APPLY_TC])
def test_nearfield_point_on_a_midpoint_is_nonfinite_in_its_row(env, mode):
    """r = 0 at a triangle midpoint: the reference's kernel divides by zero
    there (NearFieldOperatorKernel.cl:94-96), and so does this one; the other
    rows are unaffected.  (The point is the FP32 midpoint, which the FP32 and
    tensor-core paths use; the FP64 path's midpoint differs by rounding.)"""
    coords, tris, H, o32, o64, pts = env
    mid = H.TriangleMidpoints()[:, :3]
    P = np.concatenate([pts[:5], mid[7:8], pts[5:10]])
    wc, wcs, kap = WAVES["w16"]
    coeff = _coeff("all", kap)
    B = crandn(np.random.default_rng(10), coords.shape[0], wc)
    Cg = np.zeros((P.shape[0], wc), np.complex128)
    _run(H, mode, 1.0, B, 0.0, Cg, kap, coeff, wc, wcs, P)
    assert not np.isfinite(Cg[5]).any()
    keep = np.r_[0:5, 6:11]
    C64 = np.zeros((10, wc), np.complex128)
    o64.ApplyNearFieldOperators_PL(1.0, B, 0.0, C64, kap, coeff, wc, wcs, P[keep])
    assert relerr(Cg[keep], C64) < FP32_VS64_TOL


@pytest.mark.parametrize("mode", [APPLY_FP32, APPLY_TC, APPLY_FP64])
def test_nearfield_gauss_law(mode):
    """Double-layer potential of density 1 at kappa = 0 on a closed surface:
    -1 inside, 0 outside (solid angle), to the midpoint rule's O(h^2)."""
    coords, tris = meshes.icosphere(4)
    H = Helmholtz_CUDA(coords, tris, np.eye(3))
    try:
        rng = np.random.default_rng(6)
        d = rng.standard_normal((40, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        pts = np.concatenate([d * 0.5, d * 2.0])
        ones = np.ones((coords.shape[0], 16), np.complex128)
        C = np.zeros((80, 16), np.complex128)
        _run(H, mode, 1.0, ones, 0.0, C, [0.0], np.array([[0, 0, 1.0, 0]]), 16, 16, pts)
    finally:
        H.close()
    assert np.max(np.abs(C[:40] + 1.0)) < 2e-3
    assert np.max(np.abs(C[40:])) < 2e-3


def test_nearfield_complex64_and_device_paths(env):
    import torch
    coords, tris, H, o32, o64, pts = env
    wc, wcs, kap = WAVES["w32"]
    coeff = _coeff("all", kap)
    B = crandn(np.random.default_rng(12), coords.shape[0], wc)
    ref = np.zeros((pts.shape[0], wc), np.complex128)
    o32.ApplyNearFieldOperators_PL(1.0, B, 0.0, ref, kap, coeff, wc, wcs, pts)
    # complex64 host blocks and float points
    Ch = np.zeros(ref.shape, np.complex64)
    H.ApplyNearFieldOperators_PL(1.0, B.astype(np.complex64), 0.0, Ch, kap, coeff, wc, wcs, pts.astype(np.float32))
    assert relerr(Ch, ref) < FP32_TOL
    # loaded parameters (the reference's second overload) on torch tensors
    H.LoadParameters(kap, coeff, wc, wcs)
    for dt in (torch.complex128, torch.complex64):
        Bd = torch.from_numpy(B).to(dt).cuda()
        Cd = torch.zeros((pts.shape[0], wc), dtype=dt, device="cuda")
        H.ApplyNearFieldOperators_PL(1.0, Bd, 0.0, Cd, torch.from_numpy(pts).cuda())
        torch.cuda.synchronize()
        assert relerr(Cd.cpu().numpy(), ref) < FP32_TOL
    Cl = np.zeros_like(ref)
    H.ApplyNearFieldOperators_PL(1.0, B, 0.0, Cl, pts)     # host, loaded parameters
    assert relerr(Cl, ref) < FP32_TOL


def test_nearfield_full_size_torus():
    """The bench's near-field workload at a quarter of its points (torus
    153600 T, 64 RHS, 38400 points at least 0.05 from the surface): the
    tensor-core and FP32 forms within 1e-5 of the FP64 path, which matches the
    FP64 oracle to 1e-11 on the small cases."""
    import torch
    coords, tris = meshes.torus(1.0, 0.4, 160, 480)
    H = Helmholtz_CUDA(coords, tris, np.eye(3))
    try:
        rng = np.random.default_rng(0)
        pts = meshes.points_off_torus(38400, seed=0)
        kap = [2.0, 4.0, 8.0, 16.0]
        coeff = _coeff("bie", kap)
        H.LoadParameters(kap, coeff, 64, 16)
        B = torch.from_numpy(crandn(rng, coords.shape[0], 64)).cuda()
        P = torch.from_numpy(pts).cuda()
        out = {}
        for mode in (APPLY_FP64, APPLY_FP32, APPLY_TC):
            H.SetApplyMode(mode)
            C = torch.zeros((pts.shape[0], 64), dtype=torch.complex128, device="cuda")
            H.ApplyNearFieldOperators_PL(1.0, B, 0.0, C, P)
            torch.cuda.synchronize()
            out[mode] = C.cpu().numpy()
        H.SetApplyMode(APPLY_FP32)
    finally:
        H.close()
    assert np.isfinite(out[APPLY_FP64]).all()
    assert relerr(out[APPLY_FP32], out[APPLY_FP64]) < FP32_VS64_TOL
    assert relerr(out[APPLY_TC], out[APPLY_FP64]) < FP32_VS64_TOL
