"""GPU parity of the solver compositions of FarField.hpp against the oracle,
plus mathematical known-answer tests (Mie series, reciprocity)."""
import numpy as np
import pytest
from scipy.special import eval_legendre, spherical_jn, spherical_yn

from baemm_b200 import APPLY_FP32, APPLY_FP64, APPLY_TC, Helmholtz_CUDA, WaveType, meshes
from oracle import oracle as O
from tests.helpers import crandn, relerr

pytestmark = pytest.mark.gpu


def mie_far_field(kappa, radius, cos_theta, nmax=40):
    """Far field of the sound-soft sphere for the plane wave e^{i k x.d}:
    u_inf(x) = (i/k) sum_n (2n+1) j_n(k a)/h_n(k a) P_n(x.d)."""
    out = 0
    for n in range(nmax):
        jn = spherical_jn(n, kappa * radius)
        hn = jn + 1j * spherical_yn(n, kappa * radius)
        out = out + (2 * n + 1) * (jn / hn) * eval_legendre(n, cos_theta)
    return 1j / kappa * out


@pytest.fixture(scope="module")
def env():
    coords, tris = meshes.icosphere(3)
    meas = meshes.fibonacci_sphere(64)
    inc = meshes.fibonacci_sphere(16)
    H = Helmholtz_CUDA(coords, tris, meas)
    o32 = O.Oracle(coords, tris, meas, precision=32)
    o64 = O.Oracle(coords, tris, meas, precision=64)
    yield coords, tris, meas, inc, H, o32, o64
    H.close()


def test_far_field_fp32_matches_oracle(env):
    coords, tris, meas, inc, H, o32, o64 = env
    kap = np.array([2.0, 5.0])
    Fg = np.zeros((meas.shape[0], 32), complex)
    Fo = np.zeros_like(Fg)
    H.FarField(kap, inc, Fg, WaveType.Plane, 1e-10, 1e-10)
    o32.FarField(kap, inc, Fo, WaveType.Plane, 1e-10, 1e-10)
    st = H.LastSolveStats()
    assert st["gmres_converged"] == 1 and st["gmres_relative_residual"] < 1e-10
    assert relerr(Fg, Fo) < 1e-5


def test_far_field_fp64_matches_oracle(env):
    coords, tris, meas, inc, H, o32, o64 = env
    kap = np.array([3.0])
    Fg = np.zeros((meas.shape[0], 16), complex)
    Fo = np.zeros_like(Fg)
    H.SetApplyMode(APPLY_FP64)
    try:
        H.FarField(kap, inc, Fg, WaveType.Plane, 1e-12, 1e-12)
    finally:
        H.SetApplyMode(APPLY_FP32)
    o64.FarField(kap, inc, Fo, WaveType.Plane, 1e-12, 1e-12)
    assert relerr(Fg, Fo) < 1e-9


@pytest.mark.parametrize("mode", [APPLY_FP32, APPLY_TC])
def test_far_field_refined_fp32_reaches_fp64(env, mode):
    """FP32 (plain or compensated tensor-core) apply inside FP64 iterative
    refinement reaches the FP64 solution."""
    coords, tris, meas, inc, H, o32, o64 = env
    kap = np.array([3.0])
    Fg = np.zeros((meas.shape[0], 16), complex)
    Fo = np.zeros_like(Fg)
    H.SetRefinement(6, 1e-5)
    H.SetApplyMode(mode)
    try:
        H.FarField(kap, inc, Fg, WaveType.Plane, 1e-12, 1e-11)
        st = H.LastSolveStats()
    finally:
        H.SetRefinement(0)
        H.SetApplyMode(APPLY_FP32)
    o64.FarField(kap, inc, Fo, WaveType.Plane, 1e-12, 1e-12)
    assert st["refinement_steps"] >= 1 and st["gmres_converged"] == 1
    assert relerr(Fg, Fo) < 1e-8


def test_far_field_mie_series():
    coords, tris = meshes.icosphere(4)
    meas = meshes.fibonacci_sphere(64)
    inc = meshes.fibonacci_sphere(16)
    with Helmholtz_CUDA(coords, tris, meas) as H:
        F = np.zeros((64, 16), complex)
        H.FarField([2.0], inc, F, WaveType.Plane, 1e-10, 1e-10)
    ref = mie_far_field(2.0, 1.0, meas @ inc.T)
    # midpoint-rule P1 BEM on the 5120-triangle icosphere: ~0.8% discretisation error
    assert relerr(F, ref) < 1.5e-2


def test_far_field_reciprocity():
    """u_inf(x, d) = u_inf(-d, -x) for directions closed under negation."""
    coords, tris = meshes.icosphere(3)
    half = meshes.fibonacci_sphere(8)
    dirs = np.vstack([half, -half])           # 16 directions, dirs[i + 8] = -dirs[i]
    with Helmholtz_CUDA(coords, tris, dirs) as H:
        F = np.zeros((16, 16), complex)
        H.FarField([2.5], dirs, F, WaveType.Plane, 1e-10, 1e-10)
    neg = np.r_[np.arange(8, 16), np.arange(0, 8)]
    Frec = F[np.ix_(neg, neg)].T               # u_inf(-d_j, -x_i)
    assert relerr(F, Frec) < 2e-2


def test_boundary_potential_and_dtn_match_oracle(env):
    coords, tris, meas, inc, H, o32, o64 = env
    rng = np.random.default_rng(21)
    kap = np.array([4.0])
    wave = crandn(rng, coords.shape[0], 16)
    coeff = np.zeros((1, 4), complex)
    phi_g, phi_o = np.zeros_like(wave), np.zeros_like(wave)
    H.BoundaryPotential(kap, coeff, wave, phi_g, 16, 1e-10, 1e-10)
    o32.BoundaryPotential(kap, wave, phi_o, 16, 1e-10, 1e-10)
    assert np.allclose(coeff, [[0.5, -4j, 1, 0]])
    assert relerr(phi_g, phi_o) < 1e-5
    dn_g, dn_o = np.zeros_like(wave), np.zeros_like(wave)
    H.DirichletToNeumann(kap, wave, dn_g, 16, 1e-10, 1e-10)
    o32.DirichletToNeumann(kap, wave, dn_o, 16, 1e-10, 1e-10)
    assert relerr(dn_g, dn_o) < 1e-5


@pytest.mark.parametrize("nk", [1, 3, 5])
def test_boundary_potential_fp64_column_counts(env, nk):
    """FP64 GMRES on 16 nk columns (16, 48, 80): the column sums of the Krylov
    reductions are finished by one warp per column, so counts that are not
    multiples of 32 (and more columns than a warp loop covers once) are
    checked against the FP64 oracle."""
    coords, tris, meas, inc, H, o32, o64 = env
    rng = np.random.default_rng(30 + nk)
    kap = np.linspace(2.0, 6.0, nk)
    wave = crandn(rng, coords.shape[0], 16 * nk)
    coeff = np.zeros((nk, 4), complex)
    phi_g, phi_o = np.zeros_like(wave), np.zeros_like(wave)
    H.SetApplyMode(APPLY_FP64)
    try:
        H.BoundaryPotential(kap, coeff, wave, phi_g, 16, 1e-12, 1e-12)
    finally:
        H.SetApplyMode(APPLY_FP32)
    o64.BoundaryPotential(kap, wave, phi_o, 16, 1e-12, 1e-12)
    assert relerr(phi_g, phi_o) < 1e-9


def test_derivative_and_adjoint_match_oracle(env):
    coords, tris, meas, inc, H, o32, o64 = env
    kap = np.array([2.0])
    wc = 16
    nv, nm = coords.shape[0], meas.shape[0]
    rng = np.random.default_rng(8)
    h = rng.standard_normal((nv, 3))
    # library-allocated du_dn (calloc path), then reused
    DFg = np.zeros((nm, wc), complex)
    DFg, du_dn = H.Derivative_FF(kap, inc, h, DFg, None, WaveType.Plane, 1e-10, 1e-10)
    du_o = np.zeros((nv, wc), complex)
    o32.Derivative_FF_Helper(kap, inc, du_o, WaveType.Plane, 1e-10, 1e-10)
    assert relerr(du_dn, du_o) < 1e-5
    DFo = np.zeros_like(DFg)
    o32.Derivative_FF(kap, inc, h, DFo, du_o, False, WaveType.Plane, 1e-10, 1e-10)
    assert relerr(DFg, DFo) < 1e-5
    g = crandn(rng, nm, wc)
    Yg, Yo = np.zeros((nv, 3)), np.zeros((nv, 3))
    H.AdjointDerivative_FF(kap, inc, g, Yg, du_dn, WaveType.Plane, 1e-10, 1e-10)
    o32.AdjointDerivative_FF(kap, inc, g, Yo, du_o, False, WaveType.Plane, 1e-10, 1e-10)
    assert relerr(Yg, Yo) < 1e-5


def test_gauss_newton_matches_oracle():
    coords, tris = meshes.icosphere(2)
    meas = meshes.fibonacci_sphere(32)
    inc = meshes.fibonacci_sphere(16)
    kap = np.array([2.0])
    nv = coords.shape[0]
    regpar = 1e-1   # (M + DF*DF) with regpar 1e-2 needs > 90 GMRES iterations on this mesh
    rng = np.random.default_rng(12)
    B = rng.standard_normal((nv, 3))
    o = O.Oracle(coords, tris, meas, precision=32)
    du_o = np.zeros((nv, 16), complex)
    o.Derivative_FF_Helper(kap, inc, du_o, WaveType.Plane, 1e-10, 1e-10)
    Xo = np.zeros((nv, 3))
    ok_o = o.GaussNewtonSolve(kap, inc, regpar, 1.0, B, 0.0, Xo, du_o, WaveType.Plane, 1e-10, 1e-8, 1e-6)
    with Helmholtz_CUDA(coords, tris, meas) as H:
        Xg = np.zeros((nv, 3))
        L = 1.0 / o.lumped_inverse_diag()

        def Mop(x, y):
            H.MassDot(regpar, x, 0.0, y)

        def Pop(x, y):
            y[:] = x / (L[:, None] * regpar)

        ok_g = H.GaussNewtonSolve(kap, inc, Mop, Pop, 1.0, B, 0.0, Xg, du_o.copy(), WaveType.Plane, 1e-10, 1e-8,
                                  1e-6, solver=0)
        Xc = np.zeros((nv, 3))
        ok_c = H.GaussNewtonSolve(kap, inc, Mop, Pop, 1.0, B, 0.0, Xc, du_o.copy(), WaveType.Plane, 1e-10, 1e-8,
                                  1e-6, solver=1)
    assert ok_o and ok_g and ok_c
    assert relerr(Xg, Xo) < 1e-5
    assert relerr(Xc, Xo) < 1e-5


def test_profile_krylov_reports_positive_rates(env):
    """The Krylov-vector measurement hook: every kernel timed, bytes as stated."""
    coords, tris, meas, inc, H, o32, o64 = env
    prof = H.ProfileKrylov(columns=16, iterations=3, basis=4)
    n = coords.shape[0]
    for name, v in prof.items():
        assert v["ms"] > 0 and v["algorithmic_bytes"] > 0 and v["GB_s"] > 0, name
    assert prof["cg_pupdate"]["algorithmic_bytes"] == 3 * n * 32 * 8
    assert prof["gs_update"]["algorithmic_bytes"] == (4 + 2) * n * 16 * 16
