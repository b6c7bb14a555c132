// ORACLE TEST INFRASTRUCTURE -- not part of the product.
//
// CPU restatement of BAEMM's boundary-operator path (HenrikSchumacher/BAEMM),
// used only by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
// as the checker.  The product (baemm_b200/) never links or calls this file.
//
// Two arithmetic variants share one template:
//   Real = float  : the reference's own precision split -- geometry, the dense
//                   kernels, AvOp output and the SL diagonal in FP32
//                   (src/Helmholtz_Common/Definitions.hpp:3-6), everything in
//                   the caller's precision (double) afterwards.
//   Real = double : an FP64 twin of every step (no reference counterpart), with
//                   blocked (two-level) summation in the dense kernels.  This is
//                   the 1e-11 oracle.
//
// Solvers: GMRES and CG live in the unvendored Tensors library, so their exact
// iteration is unpinned.  They are restated here as documented standard
// algorithms (left-preconditioned restarted GMRES with CGS2 Arnoldi and complex
// Givens rotations; preconditioned CG per real column, zero initial guess) and
// the CUDA product implements the same definitions.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <numeric>
#include <vector>
#include <omp.h>

namespace orc
{
using cd = std::complex<double>;

template <class S> static inline double sq_abs(const S &x) { return std::norm(x); }
static inline double sq_abs(const double &x) { return x * x; }
template <class S> static inline S conj_(const S &x) { return std::conj(x); }
static inline double conj_(const double &x) { return x; }

// ---------------------------------------------------------------------------
// Restarted, left-preconditioned GMRES, one independent Krylov space per
// column of an n x nrhs row-major block (ld = nrhs).  Zero initial guess.
// Convergence per column: ||P(b - A x)|| <= tol * ||P b|| (2-norm), estimated
// from the Givens-rotated right-hand side.  `restart` = inner iterations per
// cycle (gmres_max_iter), `cycles` = number of cycles (gmres_max_restarts).
// Output: x_out = alpha * x + beta * x_out.
// Replaces Tensors::GMRES<WC,Scal,Size_T,Side::Left> as called at
// FarField.hpp:538-539, 706-708, 764-768, 828-830, 870-874.
// ---------------------------------------------------------------------------
template <class S>
struct GmresStats { bool converged = false; int iterations = 0; double max_rel_res = 0; };

template <class S>
static GmresStats<S> gmres(int64_t n, int nrhs, int restart, int cycles,
                           const std::function<void(const S *, S *)> &A,
                           const std::function<void(const S *, S *)> &P,
                           S alpha, const S *b, int64_t ldb,
                           S beta, S *x_out, int64_t ldx, double tol)
{
    const int64_t N = n * nrhs;
    const int m = restart;
    std::vector<S> x(N, S(0)), r(N), w(N), tmp(N), bb(N);
    for (int64_t i = 0; i < n; ++i)
        for (int k = 0; k < nrhs; ++k) bb[i * nrhs + k] = b[i * ldb + k];

    std::vector<S> V((int64_t)(m + 1) * N);
    std::vector<S> H((int64_t)(m + 1) * m * nrhs);   // H[(i*m + j)*nrhs + k]
    std::vector<S> g((m + 1) * nrhs), sn(m * nrhs);
    std::vector<double> cs(m * nrhs), bnorm(nrhs, 0), res(nrhs, 0);
    auto colnorm = [&](const S *v, std::vector<double> &out) {
        std::fill(out.begin(), out.end(), 0.0);
        for (int64_t i = 0; i < n; ++i)
            for (int k = 0; k < nrhs; ++k) out[k] += sq_abs(v[i * nrhs + k]);
        for (auto &o : out) o = std::sqrt(o);
    };

    GmresStats<S> st;
    P(bb.data(), tmp.data());
    colnorm(tmp.data(), bnorm);
    auto all_conv = [&](const std::vector<double> &rr) {
        for (int k = 0; k < nrhs; ++k)
            if (!(rr[k] <= tol * bnorm[k])) return false;
        return true;
    };

    for (int cyc = 0; cyc < cycles; ++cyc)
    {
        // z = P (b - A x)
        if (cyc == 0) { r = bb; }
        else
        {
            A(x.data(), tmp.data());
            for (int64_t e = 0; e < N; ++e) r[e] = bb[e] - tmp[e];
        }
        P(r.data(), w.data());
        std::vector<double> beta0(nrhs);
        colnorm(w.data(), beta0);
        if (all_conv(beta0)) { res = beta0; st.converged = true; break; }
        for (int64_t i = 0; i < n; ++i)
            for (int k = 0; k < nrhs; ++k)
                V[i * nrhs + k] = beta0[k] > 0 ? w[i * nrhs + k] / beta0[k] : S(0);
        std::fill(g.begin(), g.end(), S(0));
        std::fill(H.begin(), H.end(), S(0));
        for (int k = 0; k < nrhs; ++k) g[k] = beta0[k];

        int jend = 0;
        for (int j = 0; j < m; ++j)
        {
            S *Vj = &V[(int64_t)j * N];
            A(Vj, tmp.data());
            P(tmp.data(), w.data());
            // CGS2: two passes of classical Gram-Schmidt.
            for (int pass = 0; pass < 2; ++pass)
            {
                std::vector<S> h((j + 1) * nrhs, S(0));
                for (int i = 0; i <= j; ++i)
                {
                    const S *Vi = &V[(int64_t)i * N];
                    for (int64_t q = 0; q < n; ++q)
                        for (int k = 0; k < nrhs; ++k)
                            h[i * nrhs + k] += conj_(Vi[q * nrhs + k]) * w[q * nrhs + k];
                }
                for (int i = 0; i <= j; ++i)
                {
                    const S *Vi = &V[(int64_t)i * N];
                    for (int64_t q = 0; q < n; ++q)
                        for (int k = 0; k < nrhs; ++k)
                            w[q * nrhs + k] -= h[i * nrhs + k] * Vi[q * nrhs + k];
                    for (int k = 0; k < nrhs; ++k) H[((int64_t)i * m + j) * nrhs + k] += h[i * nrhs + k];
                }
            }
            std::vector<double> hn(nrhs);
            colnorm(w.data(), hn);
            S *Vn = &V[(int64_t)(j + 1) * N];
            for (int64_t q = 0; q < n; ++q)
                for (int k = 0; k < nrhs; ++k)
                    Vn[q * nrhs + k] = hn[k] > 0 ? w[q * nrhs + k] / hn[k] : S(0);
            for (int k = 0; k < nrhs; ++k)
            {
                H[((int64_t)(j + 1) * m + j) * nrhs + k] = hn[k];
                // previous rotations
                for (int i = 0; i < j; ++i)
                {
                    S &h0 = H[((int64_t)i * m + j) * nrhs + k];
                    S &h1 = H[((int64_t)(i + 1) * m + j) * nrhs + k];
                    const double c = cs[i * nrhs + k];
                    const S s = sn[i * nrhs + k];
                    const S t0 = c * h0 + s * h1;
                    const S t1 = -conj_(s) * h0 + c * h1;
                    h0 = t0; h1 = t1;
                }
                S &a = H[((int64_t)j * m + j) * nrhs + k];
                S &bq = H[((int64_t)(j + 1) * m + j) * nrhs + k];
                const double aa = std::sqrt(sq_abs(a)), bbv = std::sqrt(sq_abs(bq));
                double c; S s;
                if (aa == 0.0) { c = 0.0; s = S(1); a = bq; }
                else
                {
                    const double t = std::sqrt(aa * aa + bbv * bbv);
                    c = aa / t;
                    s = (a / aa) * conj_(bq) / t;
                    a = (a / aa) * t;
                }
                bq = S(0);
                cs[j * nrhs + k] = c; sn[j * nrhs + k] = s;
                const S gj = g[j * nrhs + k];
                g[j * nrhs + k] = c * gj;
                g[(j + 1) * nrhs + k] = -conj_(s) * gj;
                res[k] = std::sqrt(sq_abs(g[(j + 1) * nrhs + k]));
            }
            st.iterations++;
            jend = j + 1;
            if (all_conv(res)) break;
        }
        // back substitution and update
        for (int k = 0; k < nrhs; ++k)
        {
            std::vector<S> y(jend);
            for (int i = jend - 1; i >= 0; --i)
            {
                S s = g[i * nrhs + k];
                for (int l = i + 1; l < jend; ++l) s -= H[((int64_t)i * m + l) * nrhs + k] * y[l];
                const S d = H[((int64_t)i * m + i) * nrhs + k];
                y[i] = (d == S(0)) ? S(0) : s / d;
            }
            for (int i = 0; i < jend; ++i)
            {
                const S *Vi = &V[(int64_t)i * N];
                for (int64_t q = 0; q < n; ++q) x[q * nrhs + k] += y[i] * Vi[q * nrhs + k];
            }
        }
        if (all_conv(res)) { st.converged = true; break; }
    }
    st.max_rel_res = 0;
    for (int k = 0; k < nrhs; ++k)
        if (bnorm[k] > 0) st.max_rel_res = std::max(st.max_rel_res, res[k] / bnorm[k]);
    for (int64_t i = 0; i < n; ++i)
        for (int k = 0; k < nrhs; ++k)
        {
            S &o = x_out[i * ldx + k];
            o = (beta == S(0)) ? alpha * x[i * nrhs + k] : alpha * x[i * nrhs + k] + beta * o;
        }
    return st;
}

// ---------------------------------------------------------------------------
// Preconditioned CG per real column on an n x ncols row-major block.
// Zero initial guess, at most max_iter iterations, stop when every column has
// ||r|| <= tol * ||b||.  Replaces Tensors::ConjugateGradient as called at
// ApplyMassInverse.hpp:67-105, 120-147 (complex data is viewed as 2*nrhs real
// columns, ApplyMassInverse.hpp:71-98).
// ---------------------------------------------------------------------------
static bool cg_real(int64_t n, int ncols, int max_iter,
                    const std::function<void(const double *, double *)> &A,
                    const std::function<void(const double *, double *)> &P,
                    const double *b, double *x, double tol, int *iters_out)
{
    const int64_t N = n * ncols;
    std::vector<double> r(b, b + N), z(N), p(N), q(N), rz(ncols), bn(ncols, 0), rn(ncols);
    std::fill(x, x + N, 0.0);
    for (int64_t i = 0; i < n; ++i)
        for (int k = 0; k < ncols; ++k) bn[k] += b[i * ncols + k] * b[i * ncols + k];
    for (auto &v : bn) v = std::sqrt(v);
    P(r.data(), z.data());
    p = z;
    std::fill(rz.begin(), rz.end(), 0.0);
    for (int64_t e = 0; e < N; ++e) rz[e % ncols] += r[e] * z[e];
    auto conv = [&]() {
        std::fill(rn.begin(), rn.end(), 0.0);
        for (int64_t e = 0; e < N; ++e) rn[e % ncols] += r[e] * r[e];
        for (int k = 0; k < ncols; ++k)
            if (!(std::sqrt(rn[k]) <= tol * bn[k])) return false;
        return true;
    };
    int it = 0;
    bool ok = conv();
    while (!ok && it < max_iter)
    {
        A(p.data(), q.data());
        std::vector<double> pq(ncols, 0.0), rz2(ncols, 0.0), al(ncols), be(ncols);
        for (int64_t e = 0; e < N; ++e) pq[e % ncols] += p[e] * q[e];
        for (int k = 0; k < ncols; ++k) al[k] = pq[k] != 0 ? rz[k] / pq[k] : 0.0;
        for (int64_t e = 0; e < N; ++e) { x[e] += al[e % ncols] * p[e]; r[e] -= al[e % ncols] * q[e]; }
        P(r.data(), z.data());
        for (int64_t e = 0; e < N; ++e) rz2[e % ncols] += r[e] * z[e];
        for (int k = 0; k < ncols; ++k) { be[k] = rz[k] != 0 ? rz2[k] / rz[k] : 0.0; rz[k] = rz2[k]; }
        for (int64_t e = 0; e < N; ++e) p[e] = z[e] + be[e % ncols] * p[e];
        ++it;
        ok = conv();
    }
    if (iters_out) *iters_out = it;
    return ok;
}

struct CSR
{
    int64_t rows = 0, cols = 0;
    std::vector<int64_t> outer;
    std::vector<int32_t> inner;
    std::vector<double> val_d;   // values as stored (Real), widened for use
};

// ---------------------------------------------------------------------------
// The oracle context.  Mirrors the state of Helmholtz_OpenCL
// (MemberVariables.hpp:36-98) minus the OpenCL objects.
// ---------------------------------------------------------------------------
struct Base
{
    virtual ~Base() {}
    int64_t nv = 0, nt = 0, nm = 0;
    int threads = 1;
    bool use_diagonal = true;
    int wave_count = 0, wave_chunk_size = 16, wave_chunk_count = 0;
    int gmres_max_iter = 30, gmres_max_restarts = 3;
    int last_gmres_iterations = 0;
    double last_gmres_relres = 0;
    int last_cg_iterations = 0;
    bool Re_mass = false, Im_mass = false, Re_sl = false, Im_sl = false;
    bool Re_dl = false, Im_dl = false, Re_adl = false, Im_adl = false;
    CSR AvOp, AvOpT, Mass;
    std::vector<double> lumped_inv;
    std::vector<double> meas_d;         // nm x 3 (as given)
    std::vector<double> coords_d;       // nv x 3 (as given)
    std::vector<int32_t> tris_i;        // nt x 3 (as given)

    bool any_layer() const { return Re_sl || Im_sl || Re_dl || Im_dl || Re_adl || Im_adl; }
    bool any_sl_dl() const { return Re_sl || Im_sl || Re_dl || Im_dl; }

    virtual void load_parameters(const double *kappa, const cd *coeff, int wc, int wcs, double factor) = 0;
    virtual void avop(const cd *B, int64_t ldB, int ncols) = 0;               // -> internal B_tri
    virtual void boundary_kernel() = 0;                                        // B_tri -> C_tri
    virtual void boundary_kernel_rows(int64_t r0, int64_t r1) = 0;             // target rows [r0, r1) only
    virtual void boundary_kernel_index(const int64_t *idx, int64_t m, double *out) = 0;   // rows idx -> out (m x wc)
    virtual void set_geometry(const double *mid4, const double *nrm4) = 0;      // replace midpoints and normals
    virtual void sl_diagonal() = 0;                                            // C_tri += diag term
    virtual void avopT_out(cd alpha, cd beta, cd *C, int64_t ldC, int ncols) = 0; // C = alpha AvOpT C_tri + beta C
    virtual void farfield_kernel() = 0;                                        // B_tri -> F (nm x wc)
    virtual void farfield_out(cd alpha, cd beta, cd *C, int64_t ldC) = 0;
    virtual void herglotz_kernel(const cd *g, int64_t ldg) = 0;                // g -> C_tri
    virtual void nearfield_kernel(const double *pts, int64_t m) = 0;           // B_tri -> P (m x wc)
    virtual void nearfield_out(cd alpha, cd beta, cd *C, int64_t ldC, int64_t m) = 0;
    virtual void incident_kernel(const double *dirs, int type) = 0;            // -> C_tri
    virtual void get_geometry(double *mid, double *nrm, double *areas, double *diag) = 0;
    // real-typed PL->PC / PC->PL helpers used by the normal-field helpers
    virtual void dot_with_normals_weak(const double *X, double *Yweak) = 0;    // FarField.hpp:980-1012
    virtual void mult_with_normals_weak(const cd *X, double factor, double *Yweak) = 0; // FarField.hpp:914-942

    // y = factor * M x + addTo * y on `ncols` complex columns (ext precision)
    void mass_dot_c(cd factor, const cd *X, int64_t ldX, cd addTo, cd *Y, int64_t ldY, int ncols) const
    {
        #pragma omp parallel for num_threads(threads)
        for (int64_t v = 0; v < nv; ++v)
        {
            for (int k = 0; k < ncols; ++k)
            {
                cd s = 0;
                for (int64_t e = Mass.outer[v]; e < Mass.outer[v + 1]; ++e)
                    s += Mass.val_d[e] * X[(int64_t)Mass.inner[e] * ldX + k];
                cd &o = Y[v * ldY + k];
                o = (addTo == cd(0)) ? factor * s : factor * s + addTo * o;
            }
        }
    }
    void mass_dot_r(double factor, const double *X, int64_t ldX, double addTo, double *Y, int64_t ldY, int ncols) const
    {
        #pragma omp parallel for num_threads(threads)
        for (int64_t v = 0; v < nv; ++v)
            for (int k = 0; k < ncols; ++k)
            {
                double s = 0;
                for (int64_t e = Mass.outer[v]; e < Mass.outer[v + 1]; ++e)
                    s += Mass.val_d[e] * X[(int64_t)Mass.inner[e] * ldX + k];
                double &o = Y[v * ldY + k];
                o = (addTo == 0.0) ? factor * s : factor * s + addTo * o;
            }
    }

    // ApplyLumpedMassInverse.hpp:162-197 on real columns.
    void lumped_inverse_r(const double *X, int64_t ldX, double *Y, int64_t ldY, int ncols) const
    {
        for (int64_t v = 0; v < nv; ++v)
            for (int k = 0; k < ncols; ++k) Y[v * ldY + k] = lumped_inv[v] * X[v * ldX + k];
    }

    // ApplyMassInverse.hpp:7-156 on real columns: CG on M, lumped preconditioner.
    bool mass_inverse_r(const double *X, int64_t ldX, double *Y, int64_t ldY, int ncols, double tol)
    {
        std::vector<double> b(nv * ncols), x(nv * ncols);
        for (int64_t v = 0; v < nv; ++v)
            for (int k = 0; k < ncols; ++k) b[v * ncols + k] = X[v * ldX + k];
        auto A = [&](const double *p, double *q) { mass_dot_r(1.0, p, ncols, 0.0, q, ncols, ncols); };
        auto P = [&](const double *p, double *q) { lumped_inverse_r(p, ncols, q, ncols, ncols); };
        int it = 0;
        bool ok = cg_real(nv, ncols, 20, A, P, b.data(), x.data(), tol, &it);
        last_cg_iterations = it;
        for (int64_t v = 0; v < nv; ++v)
            for (int k = 0; k < ncols; ++k) Y[v * ldY + k] = x[v * ncols + k];
        return ok;
    }
    bool mass_inverse_c(const cd *X, int64_t ldX, cd *Y, int64_t ldY, int ncols, double tol)
    {
        // complex columns as interleaved real columns (ApplyMassInverse.hpp:71-98)
        return mass_inverse_r(reinterpret_cast<const double *>(X), 2 * ldX,
                              reinterpret_cast<double *>(Y), 2 * ldY, 2 * ncols, tol);
    }

    // ApplyBoundaryOperators.hpp:289-391
    void apply_boundary(cd alpha, const cd *B, int64_t ldB, cd beta, cd *C, int64_t ldC)
    {
        if (wave_chunk_count < 1) return;
        cd addTo = 0;
        if (any_layer())
        {
            avop(B, ldB, wave_count);
            boundary_kernel();
            sl_diagonal();
            avopT_out(alpha, beta, C, ldC, wave_count);
            addTo = 1;
        }
        else addTo = beta;
        if (Re_mass || Im_mass) apply_mass_part(alpha, B, ldB, addTo, C, ldC);
    }
    virtual void apply_mass_part(cd alpha, const cd *B, int64_t ldB, cd addTo, cd *C, int64_t ldC) = 0;

    // ApplyFarFieldOperators.hpp:356-412
    void apply_farfield(cd alpha, const cd *B, int64_t ldB, cd beta, cd *C, int64_t ldC)
    {
        if (wave_chunk_count < 1) return;
        if (any_sl_dl())
        {
            avop(B, ldB, wave_count);
            farfield_kernel();
            farfield_out(alpha, beta, C, ldC);
        }
    }
    // ApplyNearFieldOperators.hpp:56-122 (output written with ldC; the
    // reference uses wave_count, the same when ldC == wave_count)
    void apply_nearfield(cd alpha, const cd *B, int64_t ldB, cd beta, cd *C, int64_t ldC, const double *pts,
                         int64_t m)
    {
        if (wave_chunk_count < 1) return;
        if (any_sl_dl())
        {
            avop(B, ldB, wave_count);
            nearfield_kernel(pts, m);
            nearfield_out(alpha, beta, C, ldC, m);
        }
    }
    // CreateHerglotzWave.hpp:50-95
    void create_herglotz(cd alpha, const cd *g, int64_t ldg, cd beta, cd *C, int64_t ldC)
    {
        if (wave_chunk_count < 1) return;
        if (any_sl_dl())
        {
            herglotz_kernel(g, ldg);
            avopT_out(alpha, beta, C, ldC, wave_count);
        }
    }
    // CreateIncidentWave.hpp:54-127
    void create_incident(cd alpha, const double *dirs, cd beta, cd *C, int64_t ldC, int type)
    {
        if (wave_chunk_count < 1) return;
        if (any_sl_dl())
        {
            incident_kernel(dirs, type);
            avopT_out(alpha, beta, C, ldC, wave_count);
        }
    }

    // BoundaryPotential_parameters (FarField.hpp:678-771) and
    // DirichletToNeumann (FarField.hpp:790-879): GMRES on (coeff) with P = M^-1.
    void bie_solve(const double *kappa, const cd *coeff4, const cd *rhs, cd *sol,
                   int wcc, int wcs, double cg_tol, double gmres_tol)
    {
        const int wc = wcc * wcs;
        load_parameters(kappa, coeff4, wc, wcs, 1.0);
        std::function<void(const cd *, cd *)> A = [&](const cd *x, cd *y) {
            apply_boundary(1.0, x, wc, 0.0, y, wc);
        };
        std::function<void(const cd *, cd *)> P = [&](const cd *x, cd *y) {
            mass_inverse_c(x, wc, y, wc, wc, cg_tol);
        };
        auto st = gmres<cd>(nv, wc, gmres_max_iter, gmres_max_restarts, A, P, cd(1), rhs, wc, cd(0), sol, wc, gmres_tol);
        last_gmres_iterations = st.iterations;
        last_gmres_relres = st.max_rel_res;
    }
    void boundary_potential(const double *kappa, cd *coeff, const cd *wave, cd *phi, const double *eta,
                            int wcc, int wcs, double cg_tol, double gmres_tol)
    {
        for (int i = 0; i < wcc; ++i)
        {
            coeff[4 * i + 0] = cd(0.5, 0.0);
            coeff[4 * i + 1] = cd(0.0, -eta[i]);
            coeff[4 * i + 2] = cd(1.0);
            coeff[4 * i + 3] = cd(0.0);
        }
        bie_solve(kappa, coeff, wave, phi, wcc, wcs, cg_tol, gmres_tol);
    }
    void dirichlet_to_neumann(const double *kappa, const cd *wave, cd *du_dn, int wcc, int wcs,
                              double cg_tol, double gmres_tol)
    {
        std::vector<cd> c(4 * wcc);
        for (int i = 0; i < wcc; ++i)
        {
            c[4 * i + 0] = cd(0.5, 0.0);
            c[4 * i + 1] = cd(0.0, -kappa[i]);
            c[4 * i + 2] = cd(0.0);
            c[4 * i + 3] = cd(1.0);
        }
        bie_solve(kappa, c.data(), wave, du_dn, wcc, wcs, cg_tol, gmres_tol);
    }
    // FarField_parameters (FarField.hpp:90-144)
    void farfield_parameters(const double *kappa, int wcc, const double *inc, int wcs, cd *Y,
                             int type, const double *eta, double cg_tol, double gmres_tol)
    {
        const int wc = wcc * wcs;
        std::vector<cd> inc_coeff(4 * wcc), coeff(4 * wcc), wave(nv * wc), phi(nv * wc);
        for (int i = 0; i < wcc; ++i)
        {
            inc_coeff[4 * i + 0] = 0.0; inc_coeff[4 * i + 1] = -1.0;
            inc_coeff[4 * i + 2] = 0.0; inc_coeff[4 * i + 3] = 0.0;
        }
        load_parameters(kappa, inc_coeff.data(), wc, wcs, 4.0 * M_PI);
        create_incident(1.0, inc, 0.0, wave.data(), wc, type);
        boundary_potential(kappa, coeff.data(), wave.data(), phi.data(), eta, wcc, wcs, cg_tol, gmres_tol);
        load_parameters(kappa, coeff.data(), wc, wcs, 1.0);
        apply_farfield(1.0, phi.data(), wc, 0.0, Y, wc);
    }
    // Derivative_FF_Helper (FarField.hpp:148-207)
    void derivative_helper(const double *kappa, int wcc, const double *inc, int wcs, cd *du_dn,
                           int type, double cg_tol, double gmres_tol)
    {
        const int wc = wcc * wcs;
        std::vector<cd> inc_coeff(4 * wcc), inc_wave(nv * wc);
        for (int i = 0; i < wcc; ++i)
        {
            inc_coeff[4 * i + 0] = 0.0; inc_coeff[4 * i + 1] = cd(0.0, -kappa[i]);
            inc_coeff[4 * i + 2] = 1.0; inc_coeff[4 * i + 3] = 0.0;
        }
        load_parameters(kappa, inc_coeff.data(), wc, wcs, 4.0 * M_PI);
        create_incident(1.0, inc, 0.0, inc_wave.data(), wc, type);
        dirichlet_to_neumann(kappa, inc_wave.data(), du_dn, wcc, wcs, cg_tol, gmres_tol);
    }
    // DotWithNormals_PL (FarField.hpp:956-1022)
    void dot_with_normals(const double *X, double *Y, double cg_tol)
    {
        std::vector<double> Yw(nv);
        dot_with_normals_weak(X, Yw.data());
        mass_inverse_r(Yw.data(), 1, Y, 1, 1, cg_tol);
    }
    // MultiplyWithNormals_PL (FarField.hpp:886-952)
    void multiply_with_normals(const cd *X, double *Y, double factor, double cg_tol)
    {
        std::vector<double> Yw(nv * 3);
        mult_with_normals_weak(X, factor, Yw.data());
        mass_inverse_r(Yw.data(), 3, Y, 3, 3, cg_tol);
    }
    // Derivative_FF (FarField.hpp:227-321); du_dn must be provided (n x wc).
    void derivative(const double *kappa, int wcc, const double *inc, int wcs, const double *X, cd *Y,
                    cd *du_dn, int type, double cg_tol, double gmres_tol, bool compute_du_dn)
    {
        const int wc = wcc * wcs;
        if (compute_du_dn) derivative_helper(kappa, wcc, inc, wcs, du_dn, type, cg_tol, gmres_tol);
        std::vector<cd> coeff(4 * wcc), bc(nv * wc), bcw(nv * wc), phi(nv * wc);
        std::vector<double> xn(nv);
        dot_with_normals(X, xn.data(), cg_tol);
        for (int64_t i = 0; i < nv; ++i)
            for (int k = 0; k < wc; ++k) bc[i * wc + k] = -xn[i] * du_dn[i * wc + k];
        mass_dot_c(1.0, bc.data(), wc, 0.0, bcw.data(), wc, wc);
        boundary_potential(kappa, coeff.data(), bcw.data(), phi.data(), kappa, wcc, wcs, cg_tol, gmres_tol);
        load_parameters(kappa, coeff.data(), wc, wcs, 1.0);
        apply_farfield(1.0, phi.data(), wc, 0.0, Y, wc);
    }
    // AdjointDerivative_FF (FarField.hpp:342-428)
    void adjoint_derivative(const double *kappa, int wcc, const double *inc, int wcs, const cd *g, double *Y,
                            cd *du_dn, int type, double cg_tol, double gmres_tol, bool compute_du_dn)
    {
        const int wc = wcc * wcs;
        if (compute_du_dn) derivative_helper(kappa, wcc, inc, wcs, du_dn, type, cg_tol, gmres_tol);
        std::vector<cd> hw(nv * wc), dv(nv * wc), prod(nv), inc_coeff(4 * wcc);
        for (int i = 0; i < wcc; ++i)
        {
            inc_coeff[4 * i + 0] = 0.0; inc_coeff[4 * i + 1] = cd(0.0, -kappa[i]);
            inc_coeff[4 * i + 2] = 1.0; inc_coeff[4 * i + 3] = 0.0;
        }
        load_parameters(kappa, inc_coeff.data(), wc, wcs, 4.0 * M_PI / (double)nm);
        create_herglotz(1.0, g, wc, 0.0, hw.data(), wc);
        dirichlet_to_neumann(kappa, hw.data(), dv.data(), wcc, wcs, cg_tol, gmres_tol);
        // HadamardProduct.hpp:18-25 with dot_buffers taken as the plain (non-conjugating) sum
        for (int64_t i = 0; i < nv; ++i)
        {
            cd s = 0;
            for (int k = 0; k < wc; ++k) s += du_dn[i * wc + k] * dv[i * wc + k];
            prod[i] = s;
        }
        multiply_with_normals(prod.data(), Y, -1.0 / wc, cg_tol);
    }
};

template <class Real>
struct Ctx : Base
{
    using C = std::complex<Real>;
    std::vector<Real> mid, nrm, area, diag, meas4;   // float4-padded mid/nrm/meas
    std::vector<Real> kappa;
    std::vector<C> c;                                // wcc x 4
    std::vector<C> Btri, Ctri, F;                    // nt x wc, nt x wc, nm x wc
    std::vector<C> P;                                // near field: m x wc
    static constexpr bool fp32 = std::is_same<Real, float>::value;

    void init(const double *coords, int64_t nv_, const int32_t *tris, int64_t nt_,
              const double *meas, int64_t nm_, int threads_)
    {
        nv = nv_; nt = nt_; nm = nm_; threads = threads_ > 0 ? threads_ : omp_get_max_threads();
        mid.assign(4 * nt, 0); nrm.assign(4 * nt, 0); area.assign(nt, 0); diag.assign(nt, 0);
        meas4.assign(4 * nm, 0); meas_d.assign(meas, meas + 3 * nm);
        coords_d.assign(coords, coords + 3 * nv); tris_i.assign(tris, tris + 3 * nt);
        // InitializeBuffers.hpp:415-424
        for (int64_t i = 0; i < nm; ++i)
            for (int d = 0; d < 3; ++d) meas4[4 * i + d] = (Real)meas[3 * i + d];
        const Real third = Real(1) / Real(3);
        const Real half = Real(1) / Real(2);
        const Real sixth = half * third, twelveth = half * sixth;
        std::vector<int64_t> i_list(9 * nt), j_list(9 * nt);
        std::vector<Real> a_list(9 * nt);
        // Initialize.hpp:57-305 (CurlOp omitted: built but unused by the reference)
        #pragma omp parallel for num_threads(threads)
        for (int64_t i = 0; i < nt; ++i)
        {
            const int32_t v[3] = {tris[3 * i], tris[3 * i + 1], tris[3 * i + 2]};
            Real x[3][3];
            for (int a = 0; a < 3; ++a)
                for (int d = 0; d < 3; ++d) x[a][d] = (Real)coords[3 * (int64_t)v[a] + d];
            Real cc[3], u[3][3], df0[3], df1[3], anu[3];
            for (int d = 0; d < 3; ++d) cc[d] = third * (x[0][d] + x[1][d] + x[2][d]);
            for (int a = 0; a < 3; ++a)
                for (int d = 0; d < 3; ++d) u[a][d] = x[a][d] - cc[d];
            for (int d = 0; d < 3; ++d) { mid[4 * i + d] = cc[d]; df0[d] = x[1][d] - x[0][d]; df1[d] = x[2][d] - x[0][d]; }
            anu[0] = half * (df0[1] * df1[2] - df0[2] * df1[1]);
            anu[1] = half * (df0[2] * df1[0] - df0[0] * df1[2]);
            anu[2] = half * (df0[0] * df1[1] - df0[1] * df1[0]);
            const Real a = std::sqrt(anu[0] * anu[0] + anu[1] * anu[1] + anu[2] * anu[2]);
            area[i] = a;
            const Real ainv = Real(1) / a;
            for (int d = 0; d < 3; ++d) nrm[4 * i + d] = ainv * anu[d];
            for (int p = 0; p < 3; ++p)
                for (int q = 0; q < 3; ++q)
                {
                    i_list[9 * i + 3 * p + q] = v[p];
                    j_list[9 * i + 3 * p + q] = v[q];
                    a_list[9 * i + 3 * p + q] = (p == q) ? a * sixth : a * twelveth;
                }
            // Initialize.hpp:251-302: analytic self-integral of 1/r over the triangle
            auto dot = [](const Real *p, const Real *q) { return p[0] * q[0] + p[1] * q[1] + p[2] * q[2]; };
            const Real u00 = dot(u[0], u[0]), u11 = dot(u[1], u[1]), u22 = dot(u[2], u[2]);
            const Real u01 = dot(u[0], u[1]), u12 = dot(u[1], u[2]), u20 = dot(u[2], u[0]);
            const Real L[3] = {std::sqrt(u00), std::sqrt(u11), std::sqrt(u22)};
            const Real Li[3] = {Real(1) / L[0], Real(1) / L[1], Real(1) / L[2]};
            Real sum = 0;
            auto edge = [&](Real aa, Real bb, Real La, Real Lai, Real Lbi) {
                const Real vni = Real(1) / std::sqrt(std::abs(aa + bb));
                const Real sa = Lai * vni * aa, sb = Lbi * vni * bb;
                return La * std::sqrt(Real(1) - sa * sa) * (std::atanh(sa) + std::atanh(sb));
            };
            sum += edge(u11 - u12, u22 - u12, L[1], Li[1], Li[2]);
            sum += edge(u22 - u20, u00 - u20, L[2], Li[2], Li[0]);
            sum += edge(u00 - u01, u11 - u01, L[0], Li[0], Li[1]);
            diag[i] = sum / area[i];
        }
        // AvOp (Initialize.hpp:133-143, 307-315): rows = triangles, sorted columns, value a/3
        AvOp.rows = nt; AvOp.cols = nv;
        AvOp.outer.resize(nt + 1); AvOp.inner.resize(3 * nt); AvOp.val_d.resize(3 * nt);
        for (int64_t i = 0; i <= nt; ++i) AvOp.outer[i] = 3 * i;
        for (int64_t i = 0; i < nt; ++i)
        {
            int32_t v[3] = {tris[3 * i], tris[3 * i + 1], tris[3 * i + 2]};
            std::sort(v, v + 3);
            const Real a3 = area[i] * third;
            for (int q = 0; q < 3; ++q) { AvOp.inner[3 * i + q] = v[q]; AvOp.val_d[3 * i + q] = (double)a3; }
        }
        // AvOp^T
        AvOpT.rows = nv; AvOpT.cols = nt;
        AvOpT.outer.assign(nv + 1, 0);
        for (int64_t e = 0; e < 3 * nt; ++e) AvOpT.outer[AvOp.inner[e] + 1]++;
        for (int64_t v = 0; v < nv; ++v) AvOpT.outer[v + 1] += AvOpT.outer[v];
        AvOpT.inner.resize(3 * nt); AvOpT.val_d.resize(3 * nt);
        {
            std::vector<int64_t> pos(AvOpT.outer.begin(), AvOpT.outer.end() - 1);
            for (int64_t i = 0; i < nt; ++i)
                for (int q = 0; q < 3; ++q)
                {
                    const int64_t e = 3 * i + q;
                    const int64_t p = pos[AvOp.inner[e]]++;
                    AvOpT.inner[p] = (int32_t)i; AvOpT.val_d[p] = AvOp.val_d[e];
                }
        }
        // MassOp from summed triplets (Initialize.hpp:214-247, 329-334), values summed in Real
        {
            std::vector<int64_t> order(9 * nt);
            std::iota(order.begin(), order.end(), 0);
            std::stable_sort(order.begin(), order.end(), [&](int64_t p, int64_t q) {
                return i_list[p] != i_list[q] ? i_list[p] < i_list[q] : j_list[p] < j_list[q];
            });
            Mass.rows = nv; Mass.cols = nv;
            Mass.outer.assign(nv + 1, 0);
            Mass.inner.clear(); Mass.val_d.clear();
            int64_t e = 0;
            while (e < (int64_t)order.size())
            {
                const int64_t r = i_list[order[e]], cc = j_list[order[e]];
                Real s = 0;
                while (e < (int64_t)order.size() && i_list[order[e]] == r && j_list[order[e]] == cc)
                    s += a_list[order[e++]];
                Mass.inner.push_back((int32_t)cc);
                Mass.val_d.push_back((double)s);
                Mass.outer[r + 1]++;
            }
            for (int64_t v = 0; v < nv; ++v) Mass.outer[v + 1] += Mass.outer[v];
        }
        // areas_lumped_inv (Initialize.hpp:339-353): 1 / (AvOp^T . (1/3)) in Real
        lumped_inv.assign(nv, 0);
        for (int64_t v = 0; v < nv; ++v)
        {
            Real s = 0;
            for (int64_t e = AvOpT.outer[v]; e < AvOpT.outer[v + 1]; ++e) s += (Real)AvOpT.val_d[e] * third;
            lumped_inv[v] = (double)(Real(1) / s);
        }
    }

    // LoadParameters.hpp:20-81
    void load_parameters(const double *kappa_list, const cd *coeff_list, int wc, int wcs, double factor) override
    {
        wave_count = wc; wave_chunk_size = wcs;
        wave_chunk_count = (wc + wcs - 1) / wcs;
        kappa.assign(wave_chunk_count, 0); c.assign(4 * wave_chunk_count, C(0));
        Re_mass = Im_mass = Re_sl = Im_sl = Re_dl = Im_dl = Re_adl = Im_adl = false;
        const Real oofp = Real(1) / (Real(2) * (Real(2) * Real(M_PI)));
        for (int k = 0; k < wave_chunk_count; ++k)
        {
            kappa[k] = (Real)kappa_list[k];
            C z = c[4 * k + 0] = C(coeff_list[4 * k + 0]);
            Re_mass |= z.real() != 0; Im_mass |= z.imag() != 0;
            z = c[4 * k + 1] = C(coeff_list[4 * k + 1]) * oofp * (Real)factor;
            Re_sl |= z.real() != 0; Im_sl |= z.imag() != 0;
            z = c[4 * k + 2] = C(coeff_list[4 * k + 2]) * oofp * (Real)factor;
            Re_dl |= z.real() != 0; Im_dl |= z.imag() != 0;
            z = c[4 * k + 3] = C(coeff_list[4 * k + 3]) * oofp * (Real)factor;
            Re_adl |= z.real() != 0; Im_adl |= z.imag() != 0;
        }
    }

    // AvOp.Dot: ext complex in, Real complex out (ApplyBoundaryOperators.hpp:333-337)
    void avop(const cd *B, int64_t ldB, int ncols) override
    {
        Btri.assign(nt * wave_count, C(0));
        #pragma omp parallel for num_threads(threads)
        for (int64_t i = 0; i < nt; ++i)
            for (int k = 0; k < ncols; ++k)
            {
                cd s = 0;
                for (int64_t e = AvOp.outer[i]; e < AvOp.outer[i + 1]; ++e)
                    s += AvOp.val_d[e] * B[(int64_t)AvOp.inner[e] * ldB + k];
                Btri[i * wave_count + k] = C(s);
            }
    }

    // Sum over sources j of T(i,j) * X[j], sequential in j for FP32 (the
    // reference's order), blocked two-level for FP64.
    // Rows [r0, rows) when r0 is given (the rows below are left untouched).
    template <class Gen>
    void dense_rows(int64_t rows, int64_t srcs, const C *X, C *Y, int chunk, Gen &&gen, int64_t r0 = 0)
    {
        const int wcs = wave_chunk_size, ld = wave_count;
        #pragma omp parallel for schedule(dynamic, 8) num_threads(threads)
        for (int64_t i = r0; i < rows; ++i)
        {
            std::vector<C> acc(wcs, C(0)), blk(wcs, C(0));
            const int64_t BLK = fp32 ? srcs : 256;
            for (int64_t j0 = 0; j0 < srcs; j0 += BLK)
            {
                std::fill(blk.begin(), blk.end(), C(0));
                const int64_t j1 = std::min(srcs, j0 + BLK);
                for (int64_t j = j0; j < j1; ++j)
                {
                    const C A = gen(i, j);
                    if (A == C(0)) continue;
                    const C *x = &X[j * ld + chunk * wcs];
                    for (int k = 0; k < wcs; ++k) blk[k] += A * x[k];
                }
                for (int k = 0; k < wcs; ++k) acc[k] += blk[k];
            }
            for (int k = 0; k < wcs; ++k) Y[i * ld + chunk * wcs + k] = acc[k];
        }
    }

    // BoundaryOperatorKernel.cl:100-224 (formula; the Re/Im flags only prune zero terms):
    // the entry A_ij of wave chunk ch.
    C boundary_entry(int64_t i, int64_t j, int ch, bool dl, bool adl) const
    {
        if (i == j) return C(0);
        const Real kap = kappa[ch];
        const C c1 = c[4 * ch + 1], c2 = c[4 * ch + 2], c3 = c[4 * ch + 3];
        const Real zx = mid[4 * j] - mid[4 * i], zy = mid[4 * j + 1] - mid[4 * i + 1], zz = mid[4 * j + 2] - mid[4 * i + 2];
        const Real r = std::sqrt(zx * zx + zy * zy + zz * zz);
        const Real rinv = Real(1) / r;
        const Real kr = kap * r;
        const Real sn = std::sin(kr), cs = std::cos(kr);
        C A = c1 * C(cs * rinv, sn * rinv);
        if (dl || adl)
        {
            const Real r3 = rinv * rinv * rinv;
            const C g(-(kr * sn + cs) * r3, (kr * cs - sn) * r3);
            C f(0);
            if (dl) f += c2 * (zx * nrm[4 * j] + zy * nrm[4 * j + 1] + zz * nrm[4 * j + 2]);
            if (adl) f -= c3 * (zx * nrm[4 * i] + zy * nrm[4 * i + 1] + zz * nrm[4 * i + 2]);
            A += f * g;
        }
        return A;
    }

    void boundary_kernel() override { boundary_kernel_rows(0, nt); }

    // The same for target rows [r0, r1) against all sources (the other rows of C_tri are zero).
    void boundary_kernel_rows(int64_t r0, int64_t r1) override
    {
        Ctri.assign(nt * wave_count, C(0));
        const int kcc = wave_count / wave_chunk_size;   // truncating, BoundaryOperatorKernel.cl:17
        const bool dl = Re_dl || Im_dl, adl = Re_adl || Im_adl;
        for (int ch = 0; ch < kcc; ++ch)
            dense_rows(r1, nt, Btri.data(), Ctri.data(), ch,
                       [&](int64_t i, int64_t j) -> C { return boundary_entry(i, j, ch, dl, adl); }, r0);
    }

    // Target rows idx[0 .. m) (any order, repeats allowed) against all sources,
    // into out (m x wave_count interleaved complex), the same arithmetic.
    void boundary_kernel_index(const int64_t *idx, int64_t m, double *out) override
    {
        const int kcc = wave_count / wave_chunk_size;
        const int wcs = wave_chunk_size, ld = wave_count;
        const bool dl = Re_dl || Im_dl, adl = Re_adl || Im_adl;
        #pragma omp parallel for schedule(dynamic, 4) num_threads(threads)
        for (int64_t r = 0; r < m; ++r)
        {
            const int64_t i = idx[r];
            std::vector<C> acc(wcs), blk(wcs);
            for (int ch = 0; ch < kcc; ++ch)
            {
                std::fill(acc.begin(), acc.end(), C(0));
                const int64_t BLK = fp32 ? nt : 256;
                for (int64_t j0 = 0; j0 < nt; j0 += BLK)
                {
                    std::fill(blk.begin(), blk.end(), C(0));
                    const int64_t j1 = std::min(nt, j0 + BLK);
                    for (int64_t j = j0; j < j1; ++j)
                    {
                        const C A = boundary_entry(i, j, ch, dl, adl);
                        if (A == C(0)) continue;
                        const C *x = &Btri[j * ld + ch * wcs];
                        for (int k = 0; k < wcs; ++k) blk[k] += A * x[k];
                    }
                    for (int k = 0; k < wcs; ++k) acc[k] += blk[k];
                }
                for (int k = 0; k < wcs; ++k)
                {
                    out[2 * (r * ld + ch * wcs + k)] = (double)acc[k].real();
                    out[2 * (r * ld + ch * wcs + k) + 1] = (double)acc[k].imag();
                }
            }
        }
    }

    // Replace the midpoints and normals (4 per triangle) used by the kernels,
    // e.g. by the FP32 geometry of another implementation: the kernels'
    // arithmetic then compares on identical inputs.
    void set_geometry(const double *mid4, const double *nrm4) override
    {
        for (int64_t e = 0; e < 4 * nt; ++e)
        {
            mid[e] = (Real)mid4[e];
            nrm[e] = (Real)nrm4[e];
        }
    }

    // ApplySingleLayerDiagonal.hpp:397-454
    void sl_diagonal() override
    {
        if (!(use_diagonal && (Re_sl || Im_sl) && wave_chunk_count >= 1)) return;
        const int wcs = wave_chunk_size, ld = wave_count;
        #pragma omp parallel for num_threads(threads)
        for (int64_t i = 0; i < nt; ++i)
            for (int ch = 0; ch < wave_chunk_count; ++ch)
            {
                const int cols = std::min(wcs, wave_count - wcs * ch);
                const C factor = c[4 * ch + 1] * (C(diag[i]) + C(0, kappa[ch]));
                for (int k = 0; k < cols; ++k)
                    Ctri[i * ld + ch * wcs + k] += factor * Btri[i * ld + ch * wcs + k];
            }
    }

    // AvOpTransp.Dot: Real complex in, ext out, C = alpha * AvOp^T C_tri + beta * C
    void avopT_out(cd alpha, cd beta, cd *Cout, int64_t ldC, int ncols) override
    {
        #pragma omp parallel for num_threads(threads)
        for (int64_t v = 0; v < nv; ++v)
            for (int k = 0; k < ncols; ++k)
            {
                cd s = 0;
                for (int64_t e = AvOpT.outer[v]; e < AvOpT.outer[v + 1]; ++e)
                    s += AvOpT.val_d[e] * cd(Ctri[(int64_t)AvOpT.inner[e] * wave_count + k]);
                cd &o = Cout[v * ldC + k];
                o = (beta == cd(0)) ? alpha * s : alpha * s + beta * o;
            }
    }

    // ApplyBoundaryOperators.hpp:363-387: mass per chunk in ext precision
    void apply_mass_part(cd alpha, const cd *B, int64_t ldB, cd addTo, cd *Cout, int64_t ldC) override
    {
        for (int ch = 0; ch < wave_chunk_count; ++ch)
        {
            const cd factor = alpha * cd(c[4 * ch + 0]);
            const int cols = (ch < wave_chunk_count - 1) ? wave_chunk_size : wave_count - wave_chunk_size * ch;
            mass_dot_c(factor, B + wave_chunk_size * ch, ldB, addTo, Cout + wave_chunk_size * ch, ldC, cols);
        }
    }

    // FarFieldOperatorKernel.cl:85-165 with zero-padded sources
    void farfield_kernel() override
    {
        F.assign(nm * wave_count, C(0));
        const int kcc = wave_count / wave_chunk_size;
        for (int ch = 0; ch < kcc; ++ch)
        {
            const Real kap = kappa[ch];
            const C c1 = c[4 * ch + 1], c2 = c[4 * ch + 2];
            dense_rows(nm, nt, Btri.data(), F.data(), ch, [&](int64_t i, int64_t j) -> C {
                const Real *x = &meas4[4 * i];
                const Real th = kap * (mid[4 * j] * x[0] + mid[4 * j + 1] * x[1] + mid[4 * j + 2] * x[2]);
                const C e(std::cos(th), -std::sin(th));
                const Real dk = kap * (nrm[4 * j] * x[0] + nrm[4 * j + 1] * x[1] + nrm[4 * j + 2] * x[2]);
                return (c1 + c2 * C(0, -dk)) * e;
            });
        }
    }
    void farfield_out(cd alpha, cd beta, cd *Cout, int64_t ldC) override
    {
        const cd al = cd(C(alpha));   // combine_matrices takes alpha as internal Complex
        for (int64_t i = 0; i < nm; ++i)
            for (int k = 0; k < wave_count; ++k)
            {
                cd &o = Cout[i * ldC + k];
                o = (beta == cd(0)) ? al * cd(F[i * wave_count + k]) : al * cd(F[i * wave_count + k]) + beta * o;
            }
    }

    // HerglotzWaveKernel.cl:85-160 (conj(g) applied), zero-padded sources
    void herglotz_kernel(const cd *g, int64_t ldg) override
    {
        std::vector<C> G(nm * wave_count);
        for (int64_t j = 0; j < nm; ++j)
            for (int k = 0; k < wave_count; ++k) G[j * wave_count + k] = std::conj(C(g[j * ldg + k]));
        Ctri.assign(nt * wave_count, C(0));
        Btri.assign(nt * wave_count, C(0));
        const int kcc = wave_count / wave_chunk_size;
        for (int ch = 0; ch < kcc; ++ch)
        {
            const Real kap = kappa[ch];
            const C c1 = c[4 * ch + 1], c2 = c[4 * ch + 2];
            dense_rows(nt, nm, G.data(), Ctri.data(), ch, [&](int64_t i, int64_t j) -> C {
                const Real *d = &meas4[4 * j];
                const Real th = kap * (d[0] * mid[4 * i] + d[1] * mid[4 * i + 1] + d[2] * mid[4 * i + 2]);
                const C e(std::cos(th), -std::sin(th));
                const Real dk = kap * (nrm[4 * i] * d[0] + nrm[4 * i + 1] * d[1] + nrm[4 * i + 2] * d[2]);
                return (c1 + c2 * C(0, -dk)) * e;
            });
        }
    }

    // NearFieldOperatorKernel.cl:86-149: z = y_j - x_i at the evaluation points
    // (converted to Real, ApplyNearFieldOperators.hpp:98-107), no pair excluded,
    // A = c1 e^{ikr}/r + c2 (z.mu_j) (ikr - 1) e^{ikr}/r^3.
    void nearfield_kernel(const double *pts, int64_t m) override
    {
        P.assign(m * wave_count, C(0));
        std::vector<Real> x4(4 * m, Real(0));
        for (int64_t i = 0; i < m; ++i)
            for (int d = 0; d < 3; ++d) x4[4 * i + d] = (Real)pts[3 * i + d];
        const int kcc = wave_count / wave_chunk_size;
        const bool sl = Re_sl || Im_sl, dl = Re_dl || Im_dl;
        for (int ch = 0; ch < kcc; ++ch)
        {
            const Real kap = kappa[ch];
            const C c1 = c[4 * ch + 1], c2 = c[4 * ch + 2];
            dense_rows(m, nt, Btri.data(), P.data(), ch, [&](int64_t i, int64_t j) -> C {
                const Real *x = &x4[4 * i];
                const Real zx = mid[4 * j] - x[0], zy = mid[4 * j + 1] - x[1], zz = mid[4 * j + 2] - x[2];
                const Real r = std::sqrt(zx * zx + zy * zy + zz * zz);
                const Real rinv = Real(1) / r;
                const Real kr = kap * r;
                const Real sn = std::sin(kr), cs = std::cos(kr);
                C A(0);
                if (sl) A = c1 * C(cs * rinv, sn * rinv);
                if (dl)
                {
                    const Real r3 = rinv * rinv * rinv;
                    const C g(-(kr * sn + cs) * r3, (kr * cs - sn) * r3);
                    A += c2 * (zx * nrm[4 * j] + zy * nrm[4 * j + 1] + zz * nrm[4 * j + 2]) * g;
                }
                return A;
            });
        }
    }
    // combine_matrices(alpha, C_ptr, ..., beta, C_out, ...) with the external
    // alpha (ApplyNearFieldOperators.hpp:112-116); beta == 0 overwrites.
    void nearfield_out(cd alpha, cd beta, cd *Cout, int64_t ldC, int64_t m) override
    {
        for (int64_t i = 0; i < m; ++i)
            for (int k = 0; k < wave_count; ++k)
            {
                cd &o = Cout[i * ldC + k];
                const cd v = alpha * cd(P[i * wave_count + k]);
                o = (beta == cd(0)) ? v : v + beta * o;
            }
    }

    // IncidentWaveKernel_Plane.hpp:189-233 (type 201), IncidentWaveKernel_Radial.hpp:5-57 (type 202)
    void incident_kernel(const double *dirs, int type) override
    {
        const int wcs = wave_chunk_size;
        Ctri.assign(nt * wave_count, C(0));
        Btri.assign(nt * wave_count, C(0));
        std::vector<Real> w(3 * wcs);
        for (int q = 0; q < 3 * wcs; ++q) w[q] = (Real)dirs[q];
        const Real oofp = Real(1) / (Real(2) * (Real(2) * Real(M_PI)));
        #pragma omp parallel for num_threads(threads)
        for (int64_t i = 0; i < nt; ++i)
            for (int ch = 0; ch < wave_chunk_count; ++ch)
            {
                const Real K = kappa[ch];
                const C c1 = c[4 * ch + 1], c2 = c[4 * ch + 2];
                for (int j = 0; j < wcs; ++j)
                {
                    const Real *d = &w[3 * j];
                    C val;
                    if (type == 202)
                    {
                        const Real dl[3] = {mid[4 * i] - d[0], mid[4 * i + 1] - d[1], mid[4 * i + 2] - d[2]};
                        const Real R2 = dl[0] * dl[0] + dl[1] * dl[1] + dl[2] * dl[2];
                        const Real R = std::sqrt(R2), oR = 1 / R, oR2 = 1 / R2;
                        const Real dn = nrm[4 * i] * dl[0] + nrm[4 * i + 1] * dl[1] + nrm[4 * i + 2] * dl[2];
                        const C Aa(oofp * oR);
                        const C Bb(-dn * oR2, dn * K * oR);
                        val = (c1 * Aa + c2 * Aa * Bb) * std::exp(C(0, K * R));
                    }
                    else
                    {
                        const Real dm = mid[4 * i] * d[0] + mid[4 * i + 1] * d[1] + mid[4 * i + 2] * d[2];
                        const Real dn = nrm[4 * i] * d[0] + nrm[4 * i + 1] * d[1] + nrm[4 * i + 2] * d[2];
                        val = (c1 + c2 * C(0, K * dn)) * std::exp(C(0, K * dm));
                    }
                    Ctri[i * wave_count + ch * wcs + j] = val;
                }
            }
    }

    void get_geometry(double *m_, double *n_, double *a_, double *d_) override
    {
        for (int64_t i = 0; i < nt; ++i)
        {
            for (int d = 0; d < 4; ++d) { if (m_) m_[4 * i + d] = mid[4 * i + d]; if (n_) n_[4 * i + d] = nrm[4 * i + d]; }
            if (a_) a_[i] = area[i];
            if (d_) d_[i] = diag[i];
        }
    }

    // FarField.hpp:980-1012 (Real precision inside)
    void dot_with_normals_weak(const double *X, double *Yw) override
    {
        std::vector<Real> Xt(3 * nt), Y(nt);
        for (int64_t i = 0; i < nt; ++i)
            for (int d = 0; d < 3; ++d)
            {
                double s = 0;
                for (int64_t e = AvOp.outer[i]; e < AvOp.outer[i + 1]; ++e) s += AvOp.val_d[e] * X[3 * (int64_t)AvOp.inner[e] + d];
                Xt[3 * i + d] = (Real)s;
            }
        for (int64_t i = 0; i < nt; ++i)
        {
            const Real f = Real(1) / area[i];
            Real s = 0;
            for (int d = 0; d < 3; ++d) s += nrm[4 * i + d] * Xt[3 * i + d] * f;
            Y[i] = s;
        }
        for (int64_t v = 0; v < nv; ++v)
        {
            Real s = 0;
            for (int64_t e = AvOpT.outer[v]; e < AvOpT.outer[v + 1]; ++e) s += (Real)AvOpT.val_d[e] * Y[AvOpT.inner[e]];
            Yw[v] = (double)s;
        }
    }
    // FarField.hpp:914-942
    void mult_with_normals_weak(const cd *X, double factor, double *Yw) override
    {
        std::vector<Real> Y(3 * nt);
        for (int64_t i = 0; i < nt; ++i)
        {
            cd s = 0;
            for (int64_t e = AvOp.outer[i]; e < AvOp.outer[i + 1]; ++e) s += AvOp.val_d[e] * X[AvOp.inner[e]];
            const Real mul = C(s).real() / area[i];
            for (int d = 0; d < 3; ++d) Y[3 * i + d] = mul * nrm[4 * i + d];
        }
        for (int64_t v = 0; v < nv; ++v)
            for (int d = 0; d < 3; ++d)
            {
                Real s = 0;
                for (int64_t e = AvOpT.outer[v]; e < AvOpT.outer[v + 1]; ++e) s += (Real)AvOpT.val_d[e] * Y[3 * (int64_t)AvOpT.inner[e] + d];
                Yw[3 * v + d] = (double)((Real)factor * s);
            }
    }
};

} // namespace orc

using namespace orc;

// CurlOp (Initialize.hpp:146-211) restated in the precision of the context:
// rows 3 t + d, columns the triangle's vertices ascending (SortInner,
// Initialize.hpp:317-323), values (a_nu x grad_f)[d] with a_nu the half cross
// product of the edges and grad_f the P1 gradient operator from the
// pseudo-inverse g^-1 df^T of the edge frame.
template <class Real>
static void curl_csr(const std::vector<double> &coords, const std::vector<int32_t> &tris, int64_t nt, int64_t *outer,
                     int32_t *inner, double *val)
{
    for (int64_t r = 0; r <= 3 * nt; ++r) outer[r] = 3 * r;
    for (int64_t i = 0; i < nt; ++i)
    {
        int32_t v[3];
        Real x[3][3];
        for (int a = 0; a < 3; ++a)
        {
            v[a] = tris[3 * i + a];
            for (int d = 0; d < 3; ++d) x[a][d] = (Real)coords[3 * (int64_t)v[a] + d];
        }
        Real df0[3], df1[3], anu[3];
        for (int d = 0; d < 3; ++d) { df0[d] = x[1][d] - x[0][d]; df1[d] = x[2][d] - x[0][d]; }
        const Real half = Real(1) / Real(2);
        anu[0] = half * (df0[1] * df1[2] - df0[2] * df1[1]);
        anu[1] = half * (df0[2] * df1[0] - df0[0] * df1[2]);
        anu[2] = half * (df0[0] * df1[1] - df0[1] * df1[0]);
        Real g00 = 0, g01 = 0, g11 = 0;
        for (int d = 0; d < 3; ++d) { g00 += df0[d] * df0[d]; g01 += df0[d] * df1[d]; g11 += df1[d] * df1[d]; }
        const Real det_inv = Real(1) / (g00 * g11 - g01 * g01);
        const Real i00 = g11 * det_inv, i01 = -g01 * det_inv, i11 = g00 * det_inv;
        Real grad[3][3];
        for (int k = 0; k < 3; ++k)
        {
            const Real p0 = i00 * df0[k] + i01 * df1[k], p1 = i01 * df0[k] + i11 * df1[k];
            grad[k][0] = -p0 - p1; grad[k][1] = p0; grad[k][2] = p1;
        }
        Real curl[3][3];
        for (int a = 0; a < 3; ++a)
        {
            curl[0][a] = anu[1] * grad[2][a] - anu[2] * grad[1][a];
            curl[1][a] = anu[2] * grad[0][a] - anu[0] * grad[2][a];
            curl[2][a] = anu[0] * grad[1][a] - anu[1] * grad[0][a];
        }
        int p[3] = {0, 1, 2};
        std::sort(p, p + 3, [&](int a, int b) { return v[a] < v[b]; });
        for (int d = 0; d < 3; ++d)
            for (int k = 0; k < 3; ++k)
            {
                inner[9 * i + 3 * d + k] = v[p[k]];
                val[9 * i + 3 * d + k] = (double)curl[d][p[k]];
            }
    }
}

extern "C" {

// precision: 32 -> reference arithmetic (FP32 inside), 64 -> FP64 twin.
void *orc_create(const double *coords, int64_t nv, const int32_t *tris, int64_t nt,
                 const double *meas, int64_t nm, int precision, int threads)
{
    if (precision == 64) { auto *c = new Ctx<double>(); c->init(coords, nv, tris, nt, meas, nm, threads); return c; }
    auto *c = new Ctx<float>(); c->init(coords, nv, tris, nt, meas, nm, threads); return c;
}
void orc_destroy(void *h) { delete static_cast<Base *>(h); }
void orc_use_diagonal(void *h, int on) { static_cast<Base *>(h)->use_diagonal = on != 0; }
void orc_set_gmres(void *h, int max_iter, int max_restarts)
{
    auto *b = static_cast<Base *>(h); b->gmres_max_iter = max_iter; b->gmres_max_restarts = max_restarts;
}
void orc_last_stats(void *h, int *gmres_iters, double *gmres_relres, int *cg_iters)
{
    auto *b = static_cast<Base *>(h);
    *gmres_iters = b->last_gmres_iterations; *gmres_relres = b->last_gmres_relres; *cg_iters = b->last_cg_iterations;
}
void orc_geometry(void *h, double *mid4, double *nrm4, double *areas, double *diag)
{
    static_cast<Base *>(h)->get_geometry(mid4, nrm4, areas, diag);
}
int64_t orc_mass_nnz(void *h) { return (int64_t)static_cast<Base *>(h)->Mass.inner.size(); }
void orc_mass_csr(void *h, int64_t *outer, int32_t *inner, double *val)
{
    auto &M = static_cast<Base *>(h)->Mass;
    std::copy(M.outer.begin(), M.outer.end(), outer);
    std::copy(M.inner.begin(), M.inner.end(), inner);
    std::copy(M.val_d.begin(), M.val_d.end(), val);
}
void orc_curl_csr(void *h, int64_t *outer, int32_t *inner, double *val)
{
    auto *b = static_cast<Base *>(h);
    if (dynamic_cast<Ctx<float> *>(b)) curl_csr<float>(b->coords_d, b->tris_i, b->nt, outer, inner, val);
    else curl_csr<double>(b->coords_d, b->tris_i, b->nt, outer, inner, val);
}
void orc_lumped_inv(void *h, double *out)
{
    auto &v = static_cast<Base *>(h)->lumped_inv; std::copy(v.begin(), v.end(), out);
}
void orc_load_parameters(void *h, const double *kappa, const double *coeff, int wc, int wcs, double factor)
{
    static_cast<Base *>(h)->load_parameters(kappa, reinterpret_cast<const cd *>(coeff), wc, wcs, factor);
}
void orc_apply_boundary(void *h, const double *alpha, const double *B, int64_t ldB,
                        const double *beta, double *C, int64_t ldC)
{
    static_cast<Base *>(h)->apply_boundary(cd(alpha[0], alpha[1]), reinterpret_cast<const cd *>(B), ldB,
                                           cd(beta[0], beta[1]), reinterpret_cast<cd *>(C), ldC);
}
// Raw dense boundary kernel on triangle data (B_tri -> C_tri), no AvOp / diagonal.
void orc_boundary_kernel_tri(void *h, const double *Btri, double *Ctri)
{
    auto *b = static_cast<Base *>(h);
    if (auto *c = dynamic_cast<Ctx<float> *>(b))
    {
        const int64_t N = c->nt * c->wave_count;
        c->Btri.resize(N);
        for (int64_t e = 0; e < N; ++e) c->Btri[e] = std::complex<float>((float)Btri[2 * e], (float)Btri[2 * e + 1]);
        c->boundary_kernel();
        for (int64_t e = 0; e < N; ++e) { Ctri[2 * e] = c->Ctri[e].real(); Ctri[2 * e + 1] = c->Ctri[e].imag(); }
    }
    else
    {
        auto *d = static_cast<Ctx<double> *>(b);
        const int64_t N = d->nt * d->wave_count;
        d->Btri.resize(N);
        for (int64_t e = 0; e < N; ++e) d->Btri[e] = cd(Btri[2 * e], Btri[2 * e + 1]);
        d->boundary_kernel();
        for (int64_t e = 0; e < N; ++e) { Ctri[2 * e] = d->Ctri[e].real(); Ctri[2 * e + 1] = d->Ctri[e].imag(); }
    }
}
// The same for target rows [r0, r1): Ctri holds (r1 - r0) x wave_count (parity
// of sampled rows of meshes too large for the full O(N^2) oracle).
void orc_boundary_kernel_tri_rows(void *h, const double *Btri, double *Ctri, int64_t r0, int64_t r1)
{
    auto run = [&](auto *c) {
        using Cx = typename std::remove_reference<decltype(c->Btri[0])>::type;
        const int64_t N = c->nt * c->wave_count;
        c->Btri.resize(N);
        for (int64_t e = 0; e < N; ++e) c->Btri[e] = Cx(Btri[2 * e], Btri[2 * e + 1]);
        c->boundary_kernel_rows(r0, r1);
        const int64_t off = r0 * c->wave_count, M = (r1 - r0) * c->wave_count;
        for (int64_t e = 0; e < M; ++e)
        {
            Ctri[2 * e] = c->Ctri[off + e].real();
            Ctri[2 * e + 1] = c->Ctri[off + e].imag();
        }
    };
    auto *b = static_cast<Base *>(h);
    if (auto *c = dynamic_cast<Ctx<float> *>(b)) run(c);
    else run(static_cast<Ctx<double> *>(b));
}
// Target rows idx[0 .. m) of the raw dense boundary kernel: Ctri holds m x wave_count.
void orc_boundary_kernel_tri_index(void *h, const double *Btri, double *Ctri, const int64_t *idx, int64_t m)
{
    auto run = [&](auto *c) {
        using Cx = typename std::remove_reference<decltype(c->Btri[0])>::type;
        const int64_t N = c->nt * c->wave_count;
        c->Btri.resize(N);
        for (int64_t e = 0; e < N; ++e) c->Btri[e] = Cx(Btri[2 * e], Btri[2 * e + 1]);
        c->boundary_kernel_index(idx, m, Ctri);
    };
    auto *b = static_cast<Base *>(h);
    if (auto *c = dynamic_cast<Ctx<float> *>(b)) run(c);
    else run(static_cast<Ctx<double> *>(b));
}
void orc_set_geometry(void *h, const double *mid4, const double *nrm4)
{
    static_cast<Base *>(h)->set_geometry(mid4, nrm4);
}
// Raw far-field kernel on triangle data (B_tri -> F, nm x wc), no AvOp / combine.
void orc_farfield_kernel_tri(void *h, const double *Btri, double *F)
{
    auto run = [&](auto *c) {
        using Cx = typename std::remove_reference<decltype(c->Btri[0])>::type;
        const int64_t N = c->nt * c->wave_count;
        c->Btri.resize(N);
        for (int64_t e = 0; e < N; ++e) c->Btri[e] = Cx(Btri[2 * e], Btri[2 * e + 1]);
        c->farfield_kernel();
        for (int64_t e = 0; e < c->nm * c->wave_count; ++e) { F[2 * e] = c->F[e].real(); F[2 * e + 1] = c->F[e].imag(); }
    };
    auto *b = static_cast<Base *>(h);
    if (auto *c = dynamic_cast<Ctx<float> *>(b)) run(c); else run(static_cast<Ctx<double> *>(b));
}
// Raw Herglotz kernel (g: nm x wc -> C_tri: nt x wc), no AvOp^T.
void orc_herglotz_kernel_tri(void *h, const double *g, double *Ctri)
{
    auto run = [&](auto *c) {
        c->herglotz_kernel(reinterpret_cast<const cd *>(g), c->wave_count);
        for (int64_t e = 0; e < c->nt * c->wave_count; ++e) { Ctri[2 * e] = c->Ctri[e].real(); Ctri[2 * e + 1] = c->Ctri[e].imag(); }
    };
    auto *b = static_cast<Base *>(h);
    if (auto *c = dynamic_cast<Ctx<float> *>(b)) run(c); else run(static_cast<Ctx<double> *>(b));
}
void orc_apply_farfield(void *h, const double *alpha, const double *B, int64_t ldB,
                        const double *beta, double *C, int64_t ldC)
{
    static_cast<Base *>(h)->apply_farfield(cd(alpha[0], alpha[1]), reinterpret_cast<const cd *>(B), ldB,
                                           cd(beta[0], beta[1]), reinterpret_cast<cd *>(C), ldC);
}
void orc_apply_nearfield(void *h, const double *alpha, const double *B, int64_t ldB, const double *beta, double *C,
                         int64_t ldC, const double *pts, int64_t m)
{
    static_cast<Base *>(h)->apply_nearfield(cd(alpha[0], alpha[1]), reinterpret_cast<const cd *>(B), ldB,
                                            cd(beta[0], beta[1]), reinterpret_cast<cd *>(C), ldC, pts, m);
}
// Raw near-field kernel on triangle data (B_tri: nt x wc -> P: m x wc), no AvOp / combine.
void orc_nearfield_kernel_tri(void *h, const double *Btri, const double *pts, int64_t m, double *P)
{
    auto run = [&](auto *c) {
        using Cx = typename std::remove_reference<decltype(c->Btri[0])>::type;
        const int64_t N = c->nt * c->wave_count;
        c->Btri.resize(N);
        for (int64_t e = 0; e < N; ++e) c->Btri[e] = Cx(Btri[2 * e], Btri[2 * e + 1]);
        c->nearfield_kernel(pts, m);
        for (int64_t e = 0; e < m * c->wave_count; ++e) { P[2 * e] = c->P[e].real(); P[2 * e + 1] = c->P[e].imag(); }
    };
    auto *b = static_cast<Base *>(h);
    if (auto *c = dynamic_cast<Ctx<float> *>(b)) run(c); else run(static_cast<Ctx<double> *>(b));
}
void orc_create_herglotz(void *h, const double *alpha, const double *g, int64_t ldg,
                         const double *beta, double *C, int64_t ldC)
{
    static_cast<Base *>(h)->create_herglotz(cd(alpha[0], alpha[1]), reinterpret_cast<const cd *>(g), ldg,
                                            cd(beta[0], beta[1]), reinterpret_cast<cd *>(C), ldC);
}
void orc_create_incident(void *h, const double *alpha, const double *dirs, const double *beta,
                         double *C, int64_t ldC, int type)
{
    static_cast<Base *>(h)->create_incident(cd(alpha[0], alpha[1]), dirs, cd(beta[0], beta[1]),
                                            reinterpret_cast<cd *>(C), ldC, type);
}
void orc_mass_dot(void *h, const double *factor, const double *X, int64_t ldX, const double *addTo,
                  double *Y, int64_t ldY, int ncols)
{
    static_cast<Base *>(h)->mass_dot_c(cd(factor[0], factor[1]), reinterpret_cast<const cd *>(X), ldX,
                                       cd(addTo[0], addTo[1]), reinterpret_cast<cd *>(Y), ldY, ncols);
}
int orc_mass_inverse_c(void *h, const double *X, int64_t ldX, double *Y, int64_t ldY, int ncols, double tol)
{
    return static_cast<Base *>(h)->mass_inverse_c(reinterpret_cast<const cd *>(X), ldX, reinterpret_cast<cd *>(Y), ldY, ncols, tol);
}
int orc_mass_inverse_r(void *h, const double *X, int64_t ldX, double *Y, int64_t ldY, int ncols, double tol)
{
    return static_cast<Base *>(h)->mass_inverse_r(X, ldX, Y, ldY, ncols, tol);
}
void orc_lumped_inverse_c(void *h, const double *X, int64_t ldX, double *Y, int64_t ldY, int ncols)
{
    static_cast<Base *>(h)->lumped_inverse_r(X, 2 * ldX, Y, 2 * ldY, 2 * ncols);
}
void orc_farfield(void *h, const double *kappa, int wcc, const double *inc, int wcs, double *Y, int type,
                  const double *eta, double cg_tol, double gmres_tol)
{
    static_cast<Base *>(h)->farfield_parameters(kappa, wcc, inc, wcs, reinterpret_cast<cd *>(Y), type,
                                                eta ? eta : kappa, cg_tol, gmres_tol);
}
void orc_boundary_potential(void *h, const double *kappa, const double *wave, double *phi, const double *eta,
                            int wcc, int wcs, double cg_tol, double gmres_tol)
{
    std::vector<cd> coeff(4 * wcc);
    static_cast<Base *>(h)->boundary_potential(kappa, coeff.data(), reinterpret_cast<const cd *>(wave),
                                               reinterpret_cast<cd *>(phi), eta ? eta : kappa, wcc, wcs, cg_tol, gmres_tol);
}
void orc_dirichlet_to_neumann(void *h, const double *kappa, const double *wave, double *out, int wcc, int wcs,
                              double cg_tol, double gmres_tol)
{
    static_cast<Base *>(h)->dirichlet_to_neumann(kappa, reinterpret_cast<const cd *>(wave), reinterpret_cast<cd *>(out),
                                                 wcc, wcs, cg_tol, gmres_tol);
}
void orc_derivative_helper(void *h, const double *kappa, int wcc, const double *inc, int wcs, double *du_dn,
                           int type, double cg_tol, double gmres_tol)
{
    static_cast<Base *>(h)->derivative_helper(kappa, wcc, inc, wcs, reinterpret_cast<cd *>(du_dn), type, cg_tol, gmres_tol);
}
void orc_derivative(void *h, const double *kappa, int wcc, const double *inc, int wcs, const double *X, double *Y,
                    double *du_dn, int compute_du_dn, int type, double cg_tol, double gmres_tol)
{
    static_cast<Base *>(h)->derivative(kappa, wcc, inc, wcs, X, reinterpret_cast<cd *>(Y), reinterpret_cast<cd *>(du_dn),
                                       type, cg_tol, gmres_tol, compute_du_dn != 0);
}
void orc_adjoint_derivative(void *h, const double *kappa, int wcc, const double *inc, int wcs, const double *g, double *Y,
                            double *du_dn, int compute_du_dn, int type, double cg_tol, double gmres_tol)
{
    static_cast<Base *>(h)->adjoint_derivative(kappa, wcc, inc, wcs, reinterpret_cast<const cd *>(g), Y,
                                               reinterpret_cast<cd *>(du_dn), type, cg_tol, gmres_tol, compute_du_dn != 0);
}
// GaussNewtonSolve (FarField.hpp:457-604) with the metric M = regpar * Mass and
// preconditioner P = (1/regpar) * lumped inverse (the reference's metric is a
// user callable; this pair is the stand-in used by the tests).
int orc_gauss_newton(void *h, const double *kappa, int wcc, const double *inc, int wcs,
                     double regpar, double alpha, const double *B, int64_t ldB, double beta, double *X, int64_t ldX,
                     double *du_dn, int type, double cg_tol, double gmres_tol_inner, double gmres_tol_outer)
{
    auto *b = static_cast<Base *>(h);
    const int64_t n = b->nv;
    const int wc = wcc * wcs;
    std::vector<cd> DF(b->nm * wc);
    std::vector<double> ys(n * 3), Bl(n * 3), Xl(n * 3);
    for (int64_t i = 0; i < n; ++i) for (int d = 0; d < 3; ++d) Bl[3 * i + d] = B[i * ldB + d];
    std::function<void(const double *, double *)> A = [&](const double *x, double *y) {
        b->mass_dot_r(regpar, x, 3, 0.0, y, 3, 3);
        b->derivative(kappa, wcc, inc, wcs, x, DF.data(), reinterpret_cast<cd *>(du_dn), type, cg_tol, gmres_tol_inner, false);
        b->adjoint_derivative(kappa, wcc, inc, wcs, DF.data(), ys.data(), reinterpret_cast<cd *>(du_dn), type, cg_tol, gmres_tol_inner, false);
        b->mass_dot_r(1.0, ys.data(), 3, 1.0, y, 3, 3);
    };
    std::function<void(const double *, double *)> P = [&](const double *x, double *y) {
        for (int64_t i = 0; i < n; ++i) for (int d = 0; d < 3; ++d) y[3 * i + d] = b->lumped_inv[i] * x[3 * i + d] / regpar;
    };
    // outer GMRES<1> on 3n reals (FarField.hpp:538-539, 575-579)
    auto st = gmres<double>(3 * n, 1, b->gmres_max_iter, b->gmres_max_restarts, A, P, 1.0, Bl.data(), 1, 0.0, Xl.data(), 1, gmres_tol_outer);
    b->last_gmres_iterations = st.iterations; b->last_gmres_relres = st.max_rel_res;
    // FarField.hpp:575-599: with ldX == 3 the solution is written directly (alpha, beta unused)
    for (int64_t i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d)
        {
            double &o = X[i * ldX + d];
            o = (ldX == 3) ? Xl[3 * i + d] : alpha * Xl[3 * i + d] + beta * o;
        }
    return st.converged ? 1 : 0;
}
void orc_dot_with_normals(void *h, const double *X, double *Y, double cg_tol)
{
    static_cast<Base *>(h)->dot_with_normals(X, Y, cg_tol);
}
void orc_multiply_with_normals(void *h, const double *X, double *Y, double factor, double cg_tol)
{
    static_cast<Base *>(h)->multiply_with_normals(reinterpret_cast<const cd *>(X), Y, factor, cg_tol);
}
// Generic GMRES on a user dense complex matrix (test of the solver restatement).
int orc_gmres_dense(int64_t n, int nrhs, const double *Amat, const double *b, double *x, int restart, int cycles,
                    double tol, int *iters)
{
    const cd *A = reinterpret_cast<const cd *>(Amat);
    std::function<void(const cd *, cd *)> Aop = [&](const cd *p, cd *q) {
        for (int64_t i = 0; i < n; ++i)
            for (int k = 0; k < nrhs; ++k)
            {
                cd s = 0;
                for (int64_t j = 0; j < n; ++j) s += A[i * n + j] * p[j * nrhs + k];
                q[i * nrhs + k] = s;
            }
    };
    std::function<void(const cd *, cd *)> Pop = [&](const cd *p, cd *q) { std::copy(p, p + n * nrhs, q); };
    auto st = gmres<cd>(n, nrhs, restart, cycles, Aop, Pop, cd(1), reinterpret_cast<const cd *>(b), nrhs, cd(0),
                        reinterpret_cast<cd *>(x), nrhs, tol);
    if (iters) *iters = st.iterations;
    return st.converged ? 1 : 0;
}

} // extern "C"
