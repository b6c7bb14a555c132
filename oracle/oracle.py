"""ORACLE TEST INFRASTRUCTURE -- not part of the product.

ctypes front end for
  * oracle/_build/liboracle.so    -- the CPU restatement (baemm_oracle.cpp),
                                     FP32 reference arithmetic or FP64 twin;
  * oracle/_ref/libbaemm_refcl.so -- the reference's own OpenCL kernels
                                     compiled as C++ (build_ref.sh).

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg import
this module, and only as the checker.  Method names follow the reference's
Helmholtz_OpenCL API so tests read like the reference's own call sequences.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libbaemm_refcl.so")
REF_FAST_SO = os.path.join(HERE, "_ref", "libbaemm_refcl_fast.so")   # -ffast-math: the timed CPU baseline only

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)


def build(reference_root: str | None = None) -> None:
    """Compile the restatement, and the reference kernels when the reference
    tree exists (build_ref.sh finds it from the argument, BAEMM_REFERENCE or
    its own default, and skips cleanly without one)."""
    subprocess.check_call([os.path.join(HERE, "build_oracle.sh")])
    ref = reference_root or os.environ.get("BAEMM_REFERENCE")
    subprocess.check_call([os.path.join(HERE, "build_ref.sh")] + ([ref] if ref else []))


def reference_root() -> str | None:
    """The reference tree: BAEMM_REFERENCE, else the root build_ref.sh last
    built from (oracle/_ref/REFERENCE_ROOT); None when neither exists."""
    env = os.environ.get("BAEMM_REFERENCE")
    if env:
        return env if os.path.isdir(env) else None
    rec = os.path.join(HERE, "_ref", "REFERENCE_ROOT")
    if os.path.exists(rec):
        root = open(rec).read().strip()
        return root if os.path.isdir(root) else None
    return None


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError(f"oracle library missing: {ORACLE_SO} (run oracle/build_oracle.sh)")
        L = C.CDLL(ORACLE_SO)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [_dp, C.c_int64, _i32p, C.c_int64, _dp, C.c_int64, C.c_int, C.c_int]
        V, I, I64, D, i = C.c_void_p, C.c_int, C.c_int64, C.c_double, C.c_int
        sig = {
            "orc_destroy": [V],
            "orc_use_diagonal": [V, I],
            "orc_set_gmres": [V, I, I],
            "orc_last_stats": [V, C.POINTER(C.c_int), _dp, C.POINTER(C.c_int)],
            "orc_geometry": [V, _dp, _dp, _dp, _dp],
            "orc_mass_nnz": [V],
            "orc_mass_csr": [V, _i64p, _i32p, _dp],
            "orc_lumped_inv": [V, _dp],
            "orc_curl_csr": [V, _i64p, _i32p, _dp],
            "orc_load_parameters": [V, _dp, _dp, I, I, D],
            "orc_apply_boundary": [V, _dp, _dp, I64, _dp, _dp, I64],
            "orc_boundary_kernel_tri": [V, _dp, _dp],
            "orc_farfield_kernel_tri": [V, _dp, _dp],
            "orc_herglotz_kernel_tri": [V, _dp, _dp],
            "orc_apply_farfield": [V, _dp, _dp, I64, _dp, _dp, I64],
            "orc_apply_nearfield": [V, _dp, _dp, I64, _dp, _dp, I64, _dp, I64],
            "orc_nearfield_kernel_tri": [V, _dp, _dp, I64, _dp],
            "orc_create_herglotz": [V, _dp, _dp, I64, _dp, _dp, I64],
            "orc_create_incident": [V, _dp, _dp, _dp, _dp, I64, I],
            "orc_mass_dot": [V, _dp, _dp, I64, _dp, _dp, I64, I],
            "orc_mass_inverse_c": [V, _dp, I64, _dp, I64, I, D],
            "orc_mass_inverse_r": [V, _dp, I64, _dp, I64, I, D],
            "orc_lumped_inverse_c": [V, _dp, I64, _dp, I64, I],
            "orc_farfield": [V, _dp, I, _dp, I, _dp, I, _dp, D, D],
            "orc_boundary_potential": [V, _dp, _dp, _dp, _dp, I, I, D, D],
            "orc_dirichlet_to_neumann": [V, _dp, _dp, _dp, I, I, D, D],
            "orc_derivative_helper": [V, _dp, I, _dp, I, _dp, I, D, D],
            "orc_derivative": [V, _dp, I, _dp, I, _dp, _dp, _dp, I, I, D, D],
            "orc_adjoint_derivative": [V, _dp, I, _dp, I, _dp, _dp, _dp, I, I, D, D],
            "orc_gauss_newton": [V, _dp, I, _dp, I, D, D, _dp, I64, D, _dp, I64, _dp, I, D, D, D],
            "orc_dot_with_normals": [V, _dp, _dp, D],
            "orc_multiply_with_normals": [V, _dp, _dp, D, D],
            "orc_gmres_dense": [I64, I, _dp, _dp, _dp, I, I, D, C.POINTER(C.c_int)],
            "orc_boundary_kernel_tri_rows": [V, _dp, _dp, I64, I64],
            "orc_boundary_kernel_tri_index": [V, _dp, _dp, _i64p, I64],
            "orc_set_geometry": [V, _dp, _dp],
        }
        for name, args in sig.items():
            getattr(L, name).argtypes = args
        L.orc_mass_nnz.restype = C.c_int64
        L.orc_gauss_newton.restype = C.c_int
        _lib = L
    return _lib


def ref_available(fast: bool = False) -> bool:
    return os.path.exists(REF_FAST_SO if fast else REF_SO)


def reflib(fast: bool = False):
    """The reference kernels compiled as C++: strict IEEE (the parity checker),
    or fast=True, the -ffast-math build (the timed CPU baseline only)."""
    global _ref
    if _ref is None:
        _ref = {}
    path = REF_FAST_SO if fast else REF_SO
    if path not in _ref:
        if not os.path.exists(path):
            raise RuntimeError(f"reference kernel library missing: {path} (run oracle/build_ref.sh)")
        L = C.CDLL(path)
        L.refcl_max_threads.restype = C.c_int
        F, I = _fp, C.c_int
        L.refcl_boundary.argtypes = [F, F, F, F, F, F, I, I, I, I, I, I]
        L.refcl_farfield.argtypes = [F, F, F, F, F, F, F, I, I, I, I, I, I, I]
        L.refcl_herglotz.argtypes = [F, F, F, F, F, F, F, I, I, I, I, I, I, I]
        L.refcl_nearfield.argtypes = [F, F, F, F, F, F, F, I, I, I, I, I, I, I]
        _ref[path] = L
    return _ref[path]


def _c128(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Oracle:
    """CPU twin of Helmholtz_OpenCL (Helmholtz_OpenCL.hpp:109-159).

    precision=32: the reference's FP32-inside arithmetic; precision=64: FP64 twin.
    """

    PLANE = 201
    RADIAL = 202

    def __init__(self, coords, tris, meas, precision: int = 32, threads: int = 0):
        self.coords = _f64(coords)
        self.tris = np.ascontiguousarray(tris, dtype=np.int32)
        self.meas = _f64(meas).reshape(-1, 3)
        self.nv, self.nt, self.nm = self.coords.shape[0], self.tris.shape[0], self.meas.shape[0]
        self.precision = precision
        L = lib()
        self._h = C.c_void_p(L.orc_create(_p(self.coords), self.nv, _p(self.tris, _i32p), self.nt,
                                          _p(self.meas), self.nm, precision, threads))
        self.wave_count = 0
        self.wave_chunk_size = 16

    def __del__(self):
        try:
            lib().orc_destroy(self._h)
        except Exception:
            pass

    # --- getters -----------------------------------------------------------
    def geometry(self):
        mid = np.zeros((self.nt, 4)); nrm = np.zeros((self.nt, 4))
        area = np.zeros(self.nt); diag = np.zeros(self.nt)
        lib().orc_geometry(self._h, _p(mid), _p(nrm), _p(area), _p(diag))
        return mid, nrm, area, diag

    def mass_matrix(self):
        L = lib()
        nnz = L.orc_mass_nnz(self._h)
        outer = np.zeros(self.nv + 1, np.int64); inner = np.zeros(nnz, np.int32); val = np.zeros(nnz)
        L.orc_mass_csr(self._h, _p(outer, _i64p), _p(inner, _i32p), _p(val))
        return outer, inner, val

    def curl_operator(self):
        """CurlOp CSR (Initialize.hpp:146-211): (outer, inner, values)."""
        outer = np.zeros(3 * self.nt + 1, np.int64)
        inner = np.zeros(9 * self.nt, np.int32)
        val = np.zeros(9 * self.nt, np.float64)
        lib().orc_curl_csr(self._h, outer.ctypes.data_as(_i64p), inner.ctypes.data_as(_i32p), _p(val))
        return outer, inner, val

    def lumped_inverse_diag(self):
        out = np.zeros(self.nv)
        lib().orc_lumped_inv(self._h, _p(out))
        return out

    def UseDiagonal(self, on: bool):
        lib().orc_use_diagonal(self._h, int(bool(on)))

    def set_gmres(self, max_iter=30, max_restarts=3):
        lib().orc_set_gmres(self._h, int(max_iter), int(max_restarts))

    def last_stats(self):
        it = C.c_int(); rr = C.c_double(); cg = C.c_int()
        lib().orc_last_stats(self._h, C.byref(it), C.byref(rr), C.byref(cg))
        return {"gmres_iterations": it.value, "gmres_relres": rr.value, "cg_iterations": cg.value}

    # --- operators -----------------------------------------------------------
    def LoadParameters(self, kappa, coeff, wave_count, wave_chunk_size, factor=1.0):
        kappa = _f64(kappa); coeff = _c128(coeff)
        self.wave_count, self.wave_chunk_size = int(wave_count), int(wave_chunk_size)
        lib().orc_load_parameters(self._h, _p(kappa), _p(coeff.view(np.float64)), int(wave_count),
                                  int(wave_chunk_size), C.c_double(factor))

    def ApplyBoundaryOperators_PL(self, alpha, B, beta, Cout, kappa, coeff, wave_count, wave_chunk_size):
        self.LoadParameters(kappa, coeff, wave_count, wave_chunk_size)
        B = _c128(B)
        assert Cout.dtype == np.complex128 and Cout.flags.c_contiguous
        a = np.array([complex(alpha)], np.complex128); b = np.array([complex(beta)], np.complex128)
        lib().orc_apply_boundary(self._h, _p(a.view(np.float64)), _p(B.view(np.float64)), B.shape[1],
                                 _p(b.view(np.float64)), _p(Cout.view(np.float64)), Cout.shape[1])
        return Cout

    def boundary_kernel_tri(self, Btri, kappa, coeff, wave_count, wave_chunk_size):
        self.LoadParameters(kappa, coeff, wave_count, wave_chunk_size)
        Btri = _c128(Btri)
        Ct = np.zeros_like(Btri)
        lib().orc_boundary_kernel_tri(self._h, _p(Btri.view(np.float64)), _p(Ct.view(np.float64)))
        return Ct

    def boundary_kernel_tri_rows(self, Btri, kappa, coeff, wave_count, wave_chunk_size, row_begin, row_end):
        """boundary_kernel_tri for target rows [row_begin, row_end) only ((row_end - row_begin) x wc)."""
        self.LoadParameters(kappa, coeff, wave_count, wave_chunk_size)
        Btri = _c128(Btri)
        Ct = np.zeros((row_end - row_begin, wave_count), np.complex128)
        lib().orc_boundary_kernel_tri_rows(self._h, _p(Btri.view(np.float64)), _p(Ct.view(np.float64)),
                                           int(row_begin), int(row_end))
        return Ct

    def boundary_kernel_tri_index(self, Btri, kappa, coeff, wave_count, wave_chunk_size, rows):
        """boundary_kernel_tri for the target rows `rows` (any order): len(rows) x wc."""
        self.LoadParameters(kappa, coeff, wave_count, wave_chunk_size)
        Btri = _c128(Btri)
        idx = np.ascontiguousarray(rows, np.int64)
        Ct = np.zeros((idx.shape[0], wave_count), np.complex128)
        lib().orc_boundary_kernel_tri_index(self._h, _p(Btri.view(np.float64)), _p(Ct.view(np.float64)),
                                            _p(idx, _i64p), int(idx.shape[0]))
        return Ct

    def set_geometry(self, mid4, nrm4):
        """Replace the midpoints and normals the kernels use (n x 4 each), e.g.
        by another implementation's FP32 geometry, so that kernel arithmetic
        compares on identical inputs."""
        m, n = _f64(mid4).reshape(self.nt, 4), _f64(nrm4).reshape(self.nt, 4)
        lib().orc_set_geometry(self._h, _p(m), _p(n))

    def farfield_kernel_tri(self, Btri, kappa, coeff, wave_count, wave_chunk_size):
        self.LoadParameters(kappa, coeff, wave_count, wave_chunk_size)
        Btri = _c128(Btri)
        F = np.zeros((self.nm, wave_count), np.complex128)
        lib().orc_farfield_kernel_tri(self._h, _p(Btri.view(np.float64)), _p(F.view(np.float64)))
        return F

    def herglotz_kernel_tri(self, g, kappa, coeff, wave_count, wave_chunk_size):
        self.LoadParameters(kappa, coeff, wave_count, wave_chunk_size, 4.0 * np.pi / self.nm)
        g = _c128(g)
        Ct = np.zeros((self.nt, wave_count), np.complex128)
        lib().orc_herglotz_kernel_tri(self._h, _p(g.view(np.float64)), _p(Ct.view(np.float64)))
        return Ct

    def ApplyFarFieldOperators_PL(self, alpha, B, beta, Cout, kappa, coeff, wave_count, wave_chunk_size):
        self.LoadParameters(kappa, coeff, wave_count, wave_chunk_size)
        B = _c128(B)
        a = np.array([complex(alpha)], np.complex128); b = np.array([complex(beta)], np.complex128)
        lib().orc_apply_farfield(self._h, _p(a.view(np.float64)), _p(B.view(np.float64)), B.shape[1],
                                 _p(b.view(np.float64)), _p(Cout.view(np.float64)), Cout.shape[1])
        return Cout

    def ApplyNearFieldOperators_PL(self, alpha, B, beta, Cout, kappa, coeff, wave_count, wave_chunk_size,
                                   evaluation_points):
        """ApplyNearFieldOperators.hpp:27-122: Cout (m x wc) = alpha K(points) AvOp B + beta Cout."""
        self.LoadParameters(kappa, coeff, wave_count, wave_chunk_size)
        B = _c128(B); pts = _f64(evaluation_points).reshape(-1, 3)
        assert Cout.dtype == np.complex128 and Cout.flags.c_contiguous
        a = np.array([complex(alpha)], np.complex128); b = np.array([complex(beta)], np.complex128)
        lib().orc_apply_nearfield(self._h, _p(a.view(np.float64)), _p(B.view(np.float64)), B.shape[1],
                                  _p(b.view(np.float64)), _p(Cout.view(np.float64)), Cout.shape[1], _p(pts),
                                  pts.shape[0])
        return Cout

    def nearfield_kernel_tri(self, Btri, kappa, coeff, wave_count, wave_chunk_size, evaluation_points):
        self.LoadParameters(kappa, coeff, wave_count, wave_chunk_size)
        Btri = _c128(Btri); pts = _f64(evaluation_points).reshape(-1, 3)
        P = np.zeros((pts.shape[0], wave_count), np.complex128)
        lib().orc_nearfield_kernel_tri(self._h, _p(Btri.view(np.float64)), _p(pts), pts.shape[0],
                                       _p(P.view(np.float64)))
        return P

    def CreateHerglotzWave_PL(self, alpha, g, beta, Cout, kappa, coeff, wave_count, wave_chunk_size):
        self.LoadParameters(kappa, coeff, wave_count, wave_chunk_size, 4.0 * np.pi / self.nm)
        g = _c128(g)
        a = np.array([complex(alpha)], np.complex128); b = np.array([complex(beta)], np.complex128)
        lib().orc_create_herglotz(self._h, _p(a.view(np.float64)), _p(g.view(np.float64)), g.shape[1],
                                  _p(b.view(np.float64)), _p(Cout.view(np.float64)), Cout.shape[1])
        return Cout

    def CreateIncidentWave_PL(self, alpha, dirs, beta, Cout, kappa, coeff, wave_count, wave_chunk_size,
                              wave_type=PLANE):
        self.LoadParameters(kappa, coeff, wave_count, wave_chunk_size, 4.0 * np.pi)
        dirs = _f64(dirs)
        a = np.array([complex(alpha)], np.complex128); b = np.array([complex(beta)], np.complex128)
        lib().orc_create_incident(self._h, _p(a.view(np.float64)), _p(dirs), _p(b.view(np.float64)),
                                  _p(Cout.view(np.float64)), Cout.shape[1], int(wave_type))
        return Cout

    def MassDot(self, factor, X, addTo, Y, ncols=None):
        X = _c128(X)
        ncols = X.shape[1] if ncols is None else ncols
        f = np.array([complex(factor)]); t = np.array([complex(addTo)])
        lib().orc_mass_dot(self._h, _p(f.view(np.float64)), _p(X.view(np.float64)), X.shape[1],
                           _p(t.view(np.float64)), _p(Y.view(np.float64)), Y.shape[1], int(ncols))
        return Y

    def ApplyMassInverse(self, X, Y, cg_tol):
        if np.iscomplexobj(X):
            X = _c128(X)
            ok = lib().orc_mass_inverse_c(self._h, _p(X.view(np.float64)), X.shape[1], _p(Y.view(np.float64)),
                                          Y.shape[1], X.shape[1], C.c_double(cg_tol))
        else:
            X = _f64(X)
            ok = lib().orc_mass_inverse_r(self._h, _p(X), X.shape[1], _p(Y), Y.shape[1], X.shape[1],
                                          C.c_double(cg_tol))
        return bool(ok)

    def ApplyLumpedMassInverse(self, X, Y):
        X = _c128(X)
        lib().orc_lumped_inverse_c(self._h, _p(X.view(np.float64)), X.shape[1], _p(Y.view(np.float64)),
                                   Y.shape[1], X.shape[1])
        return Y

    # --- solvers ---------------------------------------------------------------
    def FarField(self, kappa, inc, Y, wave_type=PLANE, cg_tol=1e-5, gmres_tol=1e-4, eta=None):
        kappa = _f64(kappa); inc = _f64(inc)
        eta_p = _p(_f64(eta)) if eta is not None else None
        lib().orc_farfield(self._h, _p(kappa), kappa.size, _p(inc), inc.shape[0], _p(Y.view(np.float64)),
                           int(wave_type), eta_p, C.c_double(cg_tol), C.c_double(gmres_tol))
        return Y

    def BoundaryPotential(self, kappa, wave, phi, wave_chunk_size, cg_tol, gmres_tol, eta=None):
        kappa = _f64(kappa); wave = _c128(wave)
        eta_p = _p(_f64(eta)) if eta is not None else None
        lib().orc_boundary_potential(self._h, _p(kappa), _p(wave.view(np.float64)), _p(phi.view(np.float64)),
                                     eta_p, kappa.size, int(wave_chunk_size), C.c_double(cg_tol),
                                     C.c_double(gmres_tol))
        return phi

    def DirichletToNeumann(self, kappa, wave, out, wave_chunk_size, cg_tol, gmres_tol):
        kappa = _f64(kappa); wave = _c128(wave)
        lib().orc_dirichlet_to_neumann(self._h, _p(kappa), _p(wave.view(np.float64)), _p(out.view(np.float64)),
                                       kappa.size, int(wave_chunk_size), C.c_double(cg_tol), C.c_double(gmres_tol))
        return out

    def Derivative_FF_Helper(self, kappa, inc, du_dn, wave_type=PLANE, cg_tol=1e-5, gmres_tol=1e-4):
        kappa = _f64(kappa); inc = _f64(inc)
        lib().orc_derivative_helper(self._h, _p(kappa), kappa.size, _p(inc), inc.shape[0],
                                    _p(du_dn.view(np.float64)), int(wave_type), C.c_double(cg_tol),
                                    C.c_double(gmres_tol))
        return du_dn

    def Derivative_FF(self, kappa, inc, X, Y, du_dn, compute_du_dn=False, wave_type=PLANE, cg_tol=1e-5,
                      gmres_tol=1e-4):
        kappa = _f64(kappa); inc = _f64(inc); X = _f64(X)
        lib().orc_derivative(self._h, _p(kappa), kappa.size, _p(inc), inc.shape[0], _p(X), _p(Y.view(np.float64)),
                             _p(du_dn.view(np.float64)), int(compute_du_dn), int(wave_type), C.c_double(cg_tol),
                             C.c_double(gmres_tol))
        return Y

    def AdjointDerivative_FF(self, kappa, inc, g, Y, du_dn, compute_du_dn=False, wave_type=PLANE, cg_tol=1e-5,
                             gmres_tol=1e-4):
        kappa = _f64(kappa); inc = _f64(inc); g = _c128(g)
        lib().orc_adjoint_derivative(self._h, _p(kappa), kappa.size, _p(inc), inc.shape[0], _p(g.view(np.float64)),
                                     _p(Y), _p(du_dn.view(np.float64)), int(compute_du_dn), int(wave_type),
                                     C.c_double(cg_tol), C.c_double(gmres_tol))
        return Y

    def GaussNewtonSolve(self, kappa, inc, regpar, alpha, B, beta, X, du_dn, wave_type=PLANE, cg_tol=1e-5,
                         gmres_tol_inner=5e-3, gmres_tol_outer=1e-2):
        kappa = _f64(kappa); inc = _f64(inc); B = _f64(B)
        ok = lib().orc_gauss_newton(self._h, _p(kappa), kappa.size, _p(inc), inc.shape[0], C.c_double(regpar),
                                    C.c_double(alpha), _p(B), B.shape[1], C.c_double(beta), _p(X), X.shape[1],
                                    _p(du_dn.view(np.float64)), int(wave_type), C.c_double(cg_tol),
                                    C.c_double(gmres_tol_inner), C.c_double(gmres_tol_outer))
        return bool(ok)

    def DotWithNormals(self, X, Y, cg_tol):
        X = _f64(X)
        lib().orc_dot_with_normals(self._h, _p(X), _p(Y), C.c_double(cg_tol))
        return Y

    def MultiplyWithNormals(self, X, Y, factor, cg_tol):
        X = _c128(X)
        lib().orc_multiply_with_normals(self._h, _p(X.view(np.float64)), _p(Y), C.c_double(factor),
                                        C.c_double(cg_tol))
        return Y


def gmres_dense(A, b, restart=30, cycles=3, tol=1e-10):
    A = _c128(A); b = _c128(b)
    n, nrhs = b.shape
    x = np.zeros_like(b)
    it = C.c_int()
    ok = lib().orc_gmres_dense(C.c_int64(n), nrhs, _p(A.view(np.float64)), _p(b.view(np.float64)),
                               _p(x.view(np.float64)), restart, cycles, C.c_double(tol), C.byref(it))
    return x, bool(ok), it.value


# ---------------------------------------------------------------------------
# The reference's own kernels (shim-compiled).  Inputs use the reference's
# float4 / float2 layouts; coefficients already scaled as LoadParameters does.
# ---------------------------------------------------------------------------
def scaled_coefficients(coeff, factor=1.0):
    """LoadParameters.hpp:65-79 in float32: c0 as is, c1..c3 * (1/4pi) * factor."""
    c = np.asarray(coeff, np.complex128).reshape(-1, 4).astype(np.complex64)
    oofp = np.float32(1.0) / (np.float32(2.0) * (np.float32(2.0) * np.float32(np.pi)))
    out = c.copy()
    out[:, 1:] = (c[:, 1:] * oofp) * np.float32(factor)
    return out.astype(np.complex64)


def ref_boundary(mid4, nrm4, Btri, kappa, coeff_scaled, wave_chunk_size, row_begin=0, row_end=None, threads=0,
                 fast=False):
    mid4 = np.ascontiguousarray(mid4, np.float32); nrm4 = np.ascontiguousarray(nrm4, np.float32)
    Btri = np.ascontiguousarray(Btri, np.complex64)
    n, wc = Btri.shape
    Cout = np.zeros_like(Btri)
    kap = np.ascontiguousarray(kappa, np.float32); co = np.ascontiguousarray(coeff_scaled, np.complex64)
    row_end = n if row_end is None else row_end
    rc = reflib(fast).refcl_boundary(_p(mid4, _fp), _p(nrm4, _fp), _p(Btri.view(np.float32), _fp),
                                 _p(Cout.view(np.float32), _fp), _p(kap, _fp), _p(co.view(np.float32), _fp),
                                 n, wc, int(wave_chunk_size), int(row_begin), int(row_end), int(threads))
    if rc != 0:
        raise ValueError("refcl_boundary: unsupported wave_chunk_size")
    return Cout


def ref_farfield(mid4, nrm4, meas4, Btri, kappa, coeff_scaled, wave_chunk_size, threads=0):
    mid4 = np.ascontiguousarray(mid4, np.float32); nrm4 = np.ascontiguousarray(nrm4, np.float32)
    meas4 = np.ascontiguousarray(meas4, np.float32)
    Btri = np.ascontiguousarray(Btri, np.complex64)
    n, wc = Btri.shape
    m = meas4.shape[0]
    Cout = np.zeros((m, wc), np.complex64)
    kap = np.ascontiguousarray(kappa, np.float32); co = np.ascontiguousarray(coeff_scaled, np.complex64)
    rc = reflib().refcl_farfield(_p(mid4, _fp), _p(nrm4, _fp), _p(meas4, _fp), _p(Btri.view(np.float32), _fp),
                                 _p(Cout.view(np.float32), _fp), _p(kap, _fp), _p(co.view(np.float32), _fp),
                                 n, m, wc, int(wave_chunk_size), 0, m, int(threads))
    if rc != 0:
        raise ValueError("refcl_farfield: unsupported wave_chunk_size")
    return Cout


def ref_herglotz(mid4, nrm4, meas4, G, kappa, coeff_scaled, wave_chunk_size, threads=0):
    mid4 = np.ascontiguousarray(mid4, np.float32); nrm4 = np.ascontiguousarray(nrm4, np.float32)
    meas4 = np.ascontiguousarray(meas4, np.float32)
    G = np.ascontiguousarray(G, np.complex64)
    m, wc = G.shape
    n = mid4.shape[0]
    Cout = np.zeros((n, wc), np.complex64)
    kap = np.ascontiguousarray(kappa, np.float32); co = np.ascontiguousarray(coeff_scaled, np.complex64)
    rc = reflib().refcl_herglotz(_p(mid4, _fp), _p(nrm4, _fp), _p(meas4, _fp), _p(G.view(np.float32), _fp),
                                 _p(Cout.view(np.float32), _fp), _p(kap, _fp), _p(co.view(np.float32), _fp),
                                 n, m, wc, int(wave_chunk_size), 0, n, int(threads))
    if rc != 0:
        raise ValueError("refcl_herglotz: unsupported wave_chunk_size")
    return Cout


def ref_nearfield(mid4, nrm4, Btri, points, kappa, coeff_scaled, wave_chunk_size, row_begin=0, row_end=None,
                  threads=0, fast=False):
    """The reference's NearFieldOperatorKernel.cl on triangle data: P (m x wc) at points (m x 3)."""
    mid4 = np.ascontiguousarray(mid4, np.float32); nrm4 = np.ascontiguousarray(nrm4, np.float32)
    Btri = np.ascontiguousarray(Btri, np.complex64)
    pts = np.asarray(points, np.float64).reshape(-1, 3)
    pts4 = np.zeros((pts.shape[0], 4), np.float32)
    pts4[:, :3] = pts.astype(np.float32)   # ApplyNearFieldOperators.hpp:98-107
    n, wc = Btri.shape
    m = pts4.shape[0]
    Cout = np.zeros((m, wc), np.complex64)
    kap = np.ascontiguousarray(kappa, np.float32); co = np.ascontiguousarray(coeff_scaled, np.complex64)
    row_end = m if row_end is None else row_end
    rc = reflib(fast).refcl_nearfield(_p(mid4, _fp), _p(nrm4, _fp), _p(Btri.view(np.float32), _fp), _p(pts4, _fp),
                                  _p(Cout.view(np.float32), _fp), _p(kap, _fp), _p(co.view(np.float32), _fp),
                                  n, m, wc, int(wave_chunk_size), int(row_begin), int(row_end), int(threads))
    if rc != 0:
        raise ValueError("refcl_nearfield: unsupported wave_chunk_size")
    return Cout
