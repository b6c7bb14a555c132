"""CPU tests of the oracle: pinned against the reference's own kernels (the
golden fixtures from oracle/_ref, and the live shim build when present) and
against closed-form properties of the geometry, mass matrix and solvers."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import crandn, relerr, tiny_meshes


def _oracle_for(golden, precision):
    return O.Oracle(golden["coords"], golden["tris"], golden["meas"], precision=precision)


def test_oracle_geometry_matches_fixture(golden):
    o = _oracle_for(golden, 32)
    mid, nrm, area, diag = o.geometry()
    assert np.array_equal(mid.astype(np.float32), golden["mid4"])
    assert np.array_equal(nrm.astype(np.float32), golden["nrm4"])
    assert np.array_equal(area.astype(np.float32), golden["area"])


@pytest.mark.parametrize("name", ["sl", "dl", "adl", "bie_dl", "mix_2k", "wcs4"])
def test_oracle_boundary_kernel_pinned_to_reference(golden, name):
    B, Cref = golden[f"bnd_{name}_B"], golden[f"bnd_{name}_C"]
    coeff, kappa, wcs = golden[f"bnd_{name}_coeff"], golden[f"bnd_{name}_kappa"], int(golden[f"bnd_{name}_wcs"])
    wc = B.shape[1]
    c32 = _oracle_for(golden, 32).boundary_kernel_tri(B, kappa, coeff, wc, wcs)
    c64 = _oracle_for(golden, 64).boundary_kernel_tri(B, kappa, coeff, wc, wcs)
    # FP32 restatement vs the reference's FP32 kernel: rounding only
    assert relerr(c32, Cref) < 2e-6
    # the reference's FP32 kernel vs the FP64 twin: the FP32 path's own error
    assert relerr(Cref, c64) < 2e-5


@pytest.mark.parametrize("name", ["ff_sl", "ff_mix"])
def test_oracle_farfield_kernel_pinned_to_reference(golden, name):
    B, Cref = golden[f"{name}_B"], golden[f"{name}_C"]
    coeff, kappa, wcs = golden[f"{name}_coeff"], golden[f"{name}_kappa"], int(golden[f"{name}_wcs"])
    wc = B.shape[1]
    f32 = _oracle_for(golden, 32).farfield_kernel_tri(B, kappa, coeff, wc, wcs)
    f64 = _oracle_for(golden, 64).farfield_kernel_tri(B, kappa, coeff, wc, wcs)
    assert relerr(f32, Cref) < 2e-6
    assert relerr(Cref, f64) < 2e-5


def test_oracle_herglotz_kernel_pinned_to_reference(golden):
    G, Cref = golden["hw_G"], golden["hw_C"]
    coeff, kappa, wcs = golden["hw_coeff"], golden["hw_kappa"], int(golden["hw_wcs"])
    h32 = _oracle_for(golden, 32).herglotz_kernel_tri(G, kappa, coeff, G.shape[1], wcs)
    h64 = _oracle_for(golden, 64).herglotz_kernel_tri(G, kappa, coeff, G.shape[1], wcs)
    assert relerr(h32, Cref) < 2e-6
    assert relerr(Cref, h64) < 2e-5


@pytest.mark.parametrize("name", ["nf_sl", "nf_dl", "nf_mix", "nf_wcs4"])
def test_oracle_nearfield_kernel_pinned_to_reference(golden, name):
    B, Cref, pts = golden[f"{name}_B"], golden[f"{name}_C"], golden["nf_points"]
    coeff, kappa, wcs = golden[f"{name}_coeff"], golden[f"{name}_kappa"], int(golden[f"{name}_wcs"])
    wc = B.shape[1]
    p32 = _oracle_for(golden, 32).nearfield_kernel_tri(B, kappa, coeff, wc, wcs, pts)
    p64 = _oracle_for(golden, 64).nearfield_kernel_tri(B, kappa, coeff, wc, wcs, pts)
    assert relerr(p32, Cref) < 2e-6
    assert relerr(Cref, p64) < 2e-5


def test_oracle_nearfield_apply_is_kernel_of_avop(golden):
    """ApplyNearFieldOperators_PL = alpha * kernel(AvOp B) + beta * C, written with ldC."""
    o = _oracle_for(golden, 64)
    rng = np.random.default_rng(3)
    nv = golden["coords"].shape[0]
    pts = golden["nf_points"]
    coeff = np.array([[0.5, 1 - 1j, 0.25 + 2j, 3.0]] * 2)
    kappa = np.array([2.0, 5.0])
    B = crandn(rng, nv, 32)
    C0 = crandn(rng, pts.shape[0], 40)
    C = C0.copy()
    alpha, beta = 0.5 - 2j, 1.5 + 0.25j
    o.ApplyNearFieldOperators_PL(alpha, B, beta, C, kappa, coeff, 32, 16, pts)
    # the same through the raw kernel on the triangle values (AvOp = area / 3 per vertex)
    mid, nrm, area, _ = o.geometry()
    tris = golden["tris"]
    Btri = (area / 3.0)[:, None] * B[tris].sum(axis=1)
    P = o.nearfield_kernel_tri(Btri, kappa, coeff, 32, 16, pts)
    assert relerr(C[:, :32], alpha * P + beta * C0[:, :32]) < 1e-13
    assert np.array_equal(C[:, 32:], C0[:, 32:])     # columns past wave_count untouched
    # beta == 0 overwrites (NaNs in C do not survive)
    Cn = np.full((pts.shape[0], 32), np.nan, np.complex128)
    o.ApplyNearFieldOperators_PL(alpha, B, 0.0, Cn, kappa, coeff, 32, 16, pts)
    assert relerr(Cn, alpha * P) < 1e-13


def test_oracle_nearfield_ignores_mass_and_adjoint_layer(golden):
    o = _oracle_for(golden, 64)
    rng = np.random.default_rng(4)
    nv = golden["coords"].shape[0]
    pts = golden["nf_points"]
    B = crandn(rng, nv, 16)
    C = crandn(rng, pts.shape[0], 16)
    C0 = C.copy()
    # only mass and adjoint double layer: the reference leaves C_out untouched
    o.ApplyNearFieldOperators_PL(1.0, B, 0.0, C, [2.0], np.array([[1.0, 0, 0, 1.0]]), 16, 16, pts)
    assert np.array_equal(C, C0)
    a = o.ApplyNearFieldOperators_PL(1.0, B, 0.0, np.zeros_like(C), [2.0], np.array([[0, 1.0, 2.0, 0]]), 16, 16, pts)
    b = o.ApplyNearFieldOperators_PL(1.0, B, 0.0, np.zeros_like(C), [2.0], np.array([[5.0, 1.0, 2.0, 7.0]]), 16, 16,
                                     pts)
    assert np.array_equal(a, b)


def test_oracle_nearfield_potential_known_answers(sphere3):
    """Closed forms on the unit sphere (kappa = 0, density 1): the double-layer
    potential is -1 inside and 0 outside (Gauss: the solid angle of the
    surface, with z = y - x and outward normals), the single-layer potential is
    R = 1 inside and R^2 / |x| outside.  Midpoint rule on level 3 (1280 T)."""
    coords, tris = sphere3
    o = O.Oracle(coords, tris, np.eye(3), precision=64)
    nv = coords.shape[0]
    rng = np.random.default_rng(5)
    d = rng.standard_normal((12, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r_in, r_out = 0.4, 2.5
    pts = np.concatenate([d * r_in, d * r_out])
    ones = np.ones((nv, 1), np.complex128)
    dl = o.ApplyNearFieldOperators_PL(1.0, ones, 0.0, np.zeros((24, 1), np.complex128), [0.0],
                                      np.array([[0, 0, 1.0, 0]]), 1, 1, pts)[:, 0]
    sl = o.ApplyNearFieldOperators_PL(1.0, ones, 0.0, np.zeros((24, 1), np.complex128), [0.0],
                                      np.array([[0, 1.0, 0, 0]]), 1, 1, pts)[:, 0]
    # midpoint-rule error O(h^2): 2.9e-3 inside at level 3
    assert np.max(np.abs(dl[:12] + 1.0)) < 5e-3
    assert np.max(np.abs(dl[12:])) < 5e-3
    # the flat triangles lie inside the sphere: area 0.9959 of 4 pi at level 3
    assert np.max(np.abs(sl[:12] - 1.0)) < 1e-2
    assert np.max(np.abs(sl[12:] - 1.0 / r_out)) < 1e-2


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built here")
def test_oracle_nearfield_vs_live_reference_kernel(sphere3):
    coords, tris = sphere3
    rng = np.random.default_rng(8)
    o = O.Oracle(coords, tris, np.eye(3), precision=32)
    mid, nrm, _, _ = o.geometry()
    B = crandn(rng, tris.shape[0], 32, dtype=np.complex64)
    pts = rng.uniform(-2.0, 2.0, (200, 3))
    kappa = np.array([6.0, 11.0])
    coeff = np.array([[0, 0.3 - 1j, 2.0 + 0.5j, -1.0j]] * 2)
    Cref = O.ref_nearfield(mid, nrm, B, pts, kappa, O.scaled_coefficients(coeff), 16)
    assert relerr(o.nearfield_kernel_tri(B, kappa, coeff, 32, 16, pts), Cref) < 3e-6


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built here")
def test_oracle_vs_live_reference_kernel(sphere3):
    coords, tris = sphere3
    rng = np.random.default_rng(7)
    o = O.Oracle(coords, tris, np.eye(3), precision=32)
    mid, nrm, _, _ = o.geometry()
    B = crandn(rng, tris.shape[0], 32, dtype=np.complex64)
    kappa = np.array([6.0, 11.0])
    coeff = np.array([[0, 0.3 - 1j, 2.0 + 0.5j, -1.0j]] * 2)
    Cref = O.ref_boundary(mid, nrm, B, kappa, O.scaled_coefficients(coeff), 16)
    assert relerr(o.boundary_kernel_tri(B, kappa, coeff, 32, 16), Cref) < 3e-6


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built here")
@pytest.mark.parametrize("name", ["tri1", "quad2", "tetra", "strip17"])
def test_oracle_vs_live_reference_kernel_on_tiny_meshes(name):
    """Meshes of 1, 2, 4 and 17 triangles (the GPU edge-case meshes): the FP32
    restatement equals the reference's own kernel, and the FP64 twin agrees
    to FP32 rounding, so the GPU tests on these meshes check against a pinned
    oracle."""
    coords, tris = tiny_meshes()[name]
    rng = np.random.default_rng(13)
    o32 = O.Oracle(coords, tris, np.eye(3), precision=32)
    o64 = O.Oracle(coords, tris, np.eye(3), precision=64)
    mid, nrm, _, _ = o32.geometry()
    B = crandn(rng, tris.shape[0], 16, dtype=np.complex64)
    kappa = np.array([3.0])
    coeff = np.array([[0.25 + 1j, 1 + 0.5j, 1 - 2j, 0.3j]])
    Cref = O.ref_boundary(mid, nrm, B, kappa, O.scaled_coefficients(coeff), 16)
    assert relerr(o32.boundary_kernel_tri(B, kappa, coeff, 16, 16), Cref) < 3e-6
    assert relerr(o64.boundary_kernel_tri(B.astype(np.complex128), kappa, coeff, 16, 16), Cref) < 1e-5


def _self_integral_quadrature(p0, p1, p2, nq=4000):
    """Integral of 1/|y - c| over the triangle (c = centroid) by splitting at c
    into three sub-triangles and integrating R(theta) in polar coordinates."""
    c = (p0 + p1 + p2) / 3.0
    total = 0.0
    for a, b in ((p0, p1), (p1, p2), (p2, p0)):
        u, v = a - c, b - c
        e1 = u / np.linalg.norm(u)
        nrm = np.cross(u, v)
        e2 = np.cross(nrm, e1); e2 /= np.linalg.norm(e2)
        ang = np.arctan2(v @ e2, v @ e1)
        t = (np.arange(nq) + 0.5) / nq * ang
        dirs = np.outer(np.cos(t), e1) + np.outer(np.sin(t), e2)
        # ray-segment intersection distance R(t) from c to edge a-b
        d = b - a
        R = []
        for w in dirs:
            M = np.stack([w, -d], axis=1)
            sol, *_ = np.linalg.lstsq(M, a - c, rcond=None)
            R.append(sol[0])
        total += np.sum(R) * ang / nq
    return total


def test_single_layer_diagonal_matches_quadrature():
    rng = np.random.default_rng(3)
    coords = np.array([[0.0, 0.0, 0.0], [1.0, 0.1, 0.0], [0.3, 0.8, 0.2]]) + rng.standard_normal(3) * 0.01
    tris = np.array([[0, 1, 2]])
    o = O.Oracle(coords, tris, np.eye(3), precision=64)
    _, _, area, diag = o.geometry()
    q = _self_integral_quadrature(coords[0], coords[1], coords[2])
    assert abs(diag[0] * area[0] - q) / q < 1e-5


def test_mass_matrix_properties(sphere2):
    coords, tris = sphere2
    o = O.Oracle(coords, tris, np.eye(3), precision=64)
    outer, inner, val = o.mass_matrix()
    _, _, area, _ = o.geometry()
    n = coords.shape[0]
    M = np.zeros((n, n))
    for v in range(n):
        M[v, inner[outer[v]:outer[v + 1]]] = val[outer[v]:outer[v + 1]]
    assert np.allclose(M, M.T)
    assert abs(M.sum() - area.sum()) < 1e-12 * area.sum()
    # 1^T M 1 = total area; lumped inverse is 1/(sum a/9) (Initialize.hpp:339-353)
    L = o.lumped_inverse_diag()
    assert np.allclose(1.0 / L, M.sum(axis=1) / 3.0)  # row sum = sum a/3, lumped = sum a/9
    assert np.all(np.linalg.eigvalsh(M) > 0)


def test_gmres_restatement_solves_dense_system():
    rng = np.random.default_rng(11)
    n, k = 60, 3
    A = np.eye(n) * 4 + crandn(rng, n, n) / np.sqrt(n)
    b = crandn(rng, n, k)
    x, ok, its = O.gmres_dense(A, b, restart=30, cycles=4, tol=1e-12)
    assert ok
    assert relerr(x, np.linalg.solve(A, b)) < 1e-10


def test_mass_inverse_restatement(sphere2):
    coords, tris = sphere2
    o = O.Oracle(coords, tris, np.eye(3), precision=64)
    outer, inner, val = o.mass_matrix()
    n = coords.shape[0]
    M = np.zeros((n, n))
    for v in range(n):
        M[v, inner[outer[v]:outer[v + 1]]] = val[outer[v]:outer[v + 1]]
    rng = np.random.default_rng(5)
    X = crandn(rng, n, 4)
    Y = np.zeros_like(X)
    # 20 CG iterations (ApplyMassInverse.hpp:48) reach ~1e-9 on this mesh
    assert o.ApplyMassInverse(X, Y, 1e-8)
    assert relerr(M @ Y, X) < 1e-8


@pytest.mark.parametrize("precision,tol", [(64, 1e-12), (32, 2e-5)])
def test_oracle_curl_operator_known_answer(sphere2, precision, tol):
    """CurlOp (Initialize.hpp:146-211) applied to the vertex values of a linear
    field f(x) = g . x gives, per triangle, area * nu x g (P1 interpolation of a
    linear field is exact, and nu x grad_tan f = nu x g); rows of a triangle
    hold its three vertices in ascending order."""
    coords, tris = sphere2
    o = O.Oracle(coords, tris, np.eye(3), precision=precision)
    outer, inner, val = o.curl_operator()
    nt = tris.shape[0]
    assert np.array_equal(outer, 3 * np.arange(3 * nt + 1))
    assert np.array_equal(inner.reshape(nt, 3, 3), np.repeat(np.sort(tris, axis=1)[:, None, :], 3, axis=1))
    _, nrm, area, _ = o.geometry()
    g = np.array([0.3, -1.2, 0.7])
    f = coords @ g
    rows = np.add.reduceat(val * f[inner], outer[:-1])
    want = area[:, None] * np.cross(nrm[:, :3], g)
    assert np.max(np.abs(rows.reshape(nt, 3) - want)) < tol * np.max(np.abs(want))


def test_apply_at_vertices_composition_matches_full_oracle_apply():
    """The sampled-vertex composition used by the full-size torus GPU test
    (tests/helpers.oracle_apply_at_vertices) equals the oracle's own full apply."""
    from baemm_b200 import meshes
    from tests.helpers import oracle_apply_at_vertices
    coords, tris = meshes.icosphere(2)
    kap = np.array([2.0, 5.0])
    coeff = np.array([[0.0, -1j * k, 1.0, 0.0] for k in kap])
    rng = np.random.default_rng(4)
    B = rng.standard_normal((coords.shape[0], 32)) + 1j * rng.standard_normal((coords.shape[0], 32))
    verts = np.array([0, 7, 33, 161])
    for prec in (64, 32):
        orc = O.Oracle(coords, tris, np.eye(3), precision=prec)
        full = np.zeros_like(B)
        orc.ApplyBoundaryOperators_PL(1.0, B, 0.0, full, kap, coeff, 32, 16)
        part = oracle_apply_at_vertices(orc, tris, B, kap, coeff, 32, 16, verts)
        assert np.linalg.norm(part - full[verts]) <= (1e-12 if prec == 64 else 1e-6) * np.linalg.norm(full[verts])
