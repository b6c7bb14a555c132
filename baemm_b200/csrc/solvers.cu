// Solver compositions of FarField.hpp on device blocks: the mixed indirect
// boundary-integral solves, the far field, its shape derivative and adjoint.
#include "ctx.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>

namespace baemm
{

static const double2 kOne = make_double2(1.0, 0.0);
static const double2 kZero = make_double2(0.0, 0.0);

// GMRES on the operator given by (kappa, coeff4) with P = M^-1.
// Without refinement this is the reference's solve (FarField.hpp:706-768,
// 828-874).  With refinement (ir_max_steps > 0) GMRES in the context's apply
// mode is the inner solve of an FP64 iterative refinement: r = b - A64 x,
// A d = r to ir_inner_tol, x += d, until ||P r_k|| <= gmres_tol ||P b_k||.
void Ctx::bie_solve(const double *kappa, const zc *coeff4, const double2 *rhs, double2 *sol, int wcc, int wcs,
                    double cg_tol, double gmres_tol)
{
    const auto t0 = std::chrono::steady_clock::now();
    const int wc = wcc * wcs;
    const int64_t nv = mesh.nv;
    load_parameters(kappa, coeff4, wc, wcs, 1.0);
    operators_loaded = true;
    stats = baemm_solve_stats{};
    stats.cg_converged = 1;
    // With a packer the dense stage joins the packer's launches, which cannot
    // be captured in this context's graph: the apply then runs ungraphed.
    PackerSession session(packer);
    GmresSolver<double2>::Op A = [&](const double2 *x, double2 *y) {
        if (packer) apply_boundary<double2>(kOne, x, wc, kZero, y, wc);
        else
            run_graphed(GraphKey{1, x, y, wc, wc, apply_mode, wave_count},
                        [&] { apply_boundary<double2>(kOne, x, wc, kZero, y, wc); });
    };
    GmresSolver<double2>::Op P = [&](const double2 *x, double2 *y) {
        mass_inverse_complex(x, wc, y, wc, wc, cg_tol);
    };
    if (ir_max_steps <= 0)
    {
        auto st = gmres_c.solve(nv, wc, gmres_max_iter, gmres_max_restarts, A, P, kOne, rhs, wc, kZero, sol, wc,
                                gmres_tol, stream);
        stats.gmres_iterations = st.iterations;
        stats.gmres_converged = st.converged;
        stats.gmres_relative_residual = st.max_rel_res;
    }
    else
    {
        const int64_t N = nv * wc;
        double2 *r = sv_res.reserve(N), *d = sv_d.reserve(N), *pr = sv_tmp.reserve(N);
        std::vector<double> pb(wc), prn(wc);
        P(rhs, pr);
        device_colnorms(pr, nv, wc, pb.data(), reduce_scratch, stream);
        BAEMM_CUDA(cudaMemsetAsync(sol, 0, N * sizeof(double2), stream));
        BAEMM_CUDA(cudaMemcpyAsync(r, rhs, N * sizeof(double2), cudaMemcpyDeviceToDevice, stream));
        const int mode = apply_mode;
        bool conv = false;
        double rel = 1.0;
        for (int step = 0; step < ir_max_steps && !conv; ++step)
        {
            auto st = gmres_c.solve(nv, wc, gmres_max_iter, gmres_max_restarts, A, P, kOne, r, wc, kZero, d, wc,
                                    ir_inner_tol, stream);
            stats.gmres_iterations += st.iterations;
            launch_axpby<double2>(nv, wc, kOne, d, wc, kOne, sol, wc, stream);
            // r = b - A64 x
            BAEMM_CUDA(cudaMemcpyAsync(r, rhs, N * sizeof(double2), cudaMemcpyDeviceToDevice, stream));
            apply_mode = BAEMM_APPLY_FP64;
            apply_boundary<double2>(make_double2(-1.0, 0.0), sol, wc, kOne, r, wc);
            apply_mode = mode;
            P(r, pr);
            device_colnorms(pr, nv, wc, prn.data(), reduce_scratch, stream);
            rel = 0.0;
            conv = true;
            for (int k = 0; k < wc; ++k)
            {
                if (pb[k] > 0) rel = std::max(rel, prn[k] / pb[k]);
                if (!(prn[k] <= gmres_tol * pb[k])) conv = false;
            }
            stats.refinement_steps = step + 1;
        }
        stats.gmres_converged = conv;
        stats.gmres_relative_residual = rel;
    }
    operators_loaded = false;
    sync();
    stats.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// BoundaryPotential_parameters (FarField.hpp:678-771): (1/2 M - i eta SL + DL) phi = wave
void Ctx::boundary_potential(const double *kappa, zc *coeff, const double2 *wave, double2 *phi, const double *eta,
                             int wcc, int wcs, double cg_tol, double gmres_tol)
{
    for (int i = 0; i < wcc; ++i)
    {
        coeff[4 * i + 0] = zc(0.5, 0.0);
        coeff[4 * i + 1] = zc(0.0, -eta[i]);
        coeff[4 * i + 2] = zc(1.0, 0.0);
        coeff[4 * i + 3] = zc(0.0, 0.0);
    }
    bie_solve(kappa, coeff, wave, phi, wcc, wcs, cg_tol, gmres_tol);
}

// DirichletToNeumann (FarField.hpp:790-879): (1/2 M - i kappa SL + DL') du_dn = wave
void Ctx::dirichlet_to_neumann(const double *kappa, const double2 *wave, double2 *du_dn, int wcc, int wcs,
                               double cg_tol, double gmres_tol)
{
    std::vector<zc> c(4 * wcc);
    for (int i = 0; i < wcc; ++i)
    {
        c[4 * i + 0] = zc(0.5, 0.0);
        c[4 * i + 1] = zc(0.0, -kappa[i]);
        c[4 * i + 2] = zc(0.0, 0.0);
        c[4 * i + 3] = zc(1.0, 0.0);
    }
    bie_solve(kappa, c.data(), wave, du_dn, wcc, wcs, cg_tol, gmres_tol);
}

// FarField_parameters (FarField.hpp:90-144)
void Ctx::farfield_parameters(const double *kappa, int wcc, const double *inc, int wcs, double2 *Y, int type,
                              const double *eta, double cg_tol, double gmres_tol)
{
    const int wc = wcc * wcs;
    const int64_t N = mesh.nv * wc;
    std::vector<zc> inc_coeff(4 * wcc), coeff(4 * wcc);
    for (int i = 0; i < wcc; ++i)
    {
        inc_coeff[4 * i + 0] = 0.0; inc_coeff[4 * i + 1] = -1.0;
        inc_coeff[4 * i + 2] = 0.0; inc_coeff[4 * i + 3] = 0.0;
    }
    double2 *wave = sv_wave.reserve(N), *phi = sv_phi.reserve(N);
    load_parameters(kappa, inc_coeff.data(), wc, wcs, 4.0 * M_PI);
    incident(1.0, inc, 0.0, wave, wc, type);
    boundary_potential(kappa, coeff.data(), wave, phi, eta, wcc, wcs, cg_tol, gmres_tol);
    load_parameters(kappa, coeff.data(), wc, wcs, 1.0);
    apply_farfield(1.0, phi, wc, 0.0, Y, wc);
}

// Derivative_FF_Helper (FarField.hpp:148-207)
void Ctx::derivative_helper(const double *kappa, int wcc, const double *inc, int wcs, double2 *du_dn, int type,
                            double cg_tol, double gmres_tol)
{
    const int wc = wcc * wcs;
    std::vector<zc> inc_coeff(4 * wcc);
    for (int i = 0; i < wcc; ++i)
    {
        inc_coeff[4 * i + 0] = 0.0; inc_coeff[4 * i + 1] = zc(0.0, -kappa[i]);
        inc_coeff[4 * i + 2] = 1.0; inc_coeff[4 * i + 3] = 0.0;
    }
    double2 *wave = sv_wave.reserve(mesh.nv * wc);
    load_parameters(kappa, inc_coeff.data(), wc, wcs, 4.0 * M_PI);
    incident(1.0, inc, 0.0, wave, wc, type);
    dirichlet_to_neumann(kappa, wave, du_dn, wcc, wcs, cg_tol, gmres_tol);
}

// DotWithNormals_PL (FarField.hpp:956-1022): Y = M^-1 AvOp^T (n . AvOp X / a)
void Ctx::dot_with_normals(const double *X, double *Y, double cg_tol)
{
    double *ytri = sv_ytri.reserve(std::max<int64_t>(3 * mesh.nt, 1));
    double *yw = sv_yw.reserve(std::max<int64_t>(3 * mesh.nv, 1));
    launch_dot_with_normals_weak(mesh, aux_fp64(), X, ytri, yw, stream);
    mass_inverse_real(yw, 1, Y, 1, 1, cg_tol);
}

// MultiplyWithNormals_PL (FarField.hpp:886-952): Y = M^-1 AvOp^T (factor Re(AvOp X)/a n)
void Ctx::multiply_with_normals(const double2 *X, double *Y, double factor, double cg_tol)
{
    double *ytri = sv_ytri.reserve(std::max<int64_t>(3 * mesh.nt, 1));
    double *yw = sv_yw.reserve(std::max<int64_t>(3 * mesh.nv, 1));
    launch_mult_with_normals_weak(mesh, aux_fp64(), X, factor, ytri, yw, stream);
    mass_inverse_real(yw, 3, Y, 3, 3, cg_tol);
}

// Derivative_FF (FarField.hpp:284-318) with du_dn given (device, nv x wc)
void Ctx::derivative(const double *kappa, int wcc, const double *inc, int wcs, const double *X, double2 *Y,
                     const double2 *du_dn, double cg_tol, double gmres_tol)
{
    (void)inc;
    const int wc = wcc * wcs;
    const int64_t nv = mesh.nv, N = nv * wc;
    std::vector<zc> coeff(4 * wcc);
    double *xn = sv_xn.reserve(nv);
    double2 *bc = sv_bc.reserve(N), *bcw = sv_bcw.reserve(N), *phi = sv_phi.reserve(N);
    dot_with_normals(X, xn, cg_tol);
    launch_scale_rows_neg(nv, wc, xn, du_dn, bc, stream);
    // MassOp.Dot<WC> in external precision (FarField.hpp:303-307)
    launch_mass_dot_real(mesh, mass_values_fp64(), 1.0, reinterpret_cast<const double *>(bc), 2 * wc, 0.0,
                         reinterpret_cast<double *>(bcw), 2 * wc, 2 * wc, stream);
    boundary_potential(kappa, coeff.data(), bcw, phi, kappa, wcc, wcs, cg_tol, gmres_tol);
    load_parameters(kappa, coeff.data(), wc, wcs, 1.0);
    apply_farfield(1.0, phi, wc, 0.0, Y, wc);
}

// AdjointDerivative_FF (FarField.hpp:394-425) with du_dn given
void Ctx::adjoint_derivative(const double *kappa, int wcc, const double *inc, int wcs, const double2 *g, double *Y,
                             const double2 *du_dn, double cg_tol, double gmres_tol)
{
    (void)inc;
    const int wc = wcc * wcs;
    const int64_t nv = mesh.nv, N = nv * wc;
    std::vector<zc> inc_coeff(4 * wcc);
    for (int i = 0; i < wcc; ++i)
    {
        inc_coeff[4 * i + 0] = 0.0; inc_coeff[4 * i + 1] = zc(0.0, -kappa[i]);
        inc_coeff[4 * i + 2] = 1.0; inc_coeff[4 * i + 3] = 0.0;
    }
    double2 *hw = sv_hw.reserve(N), *dv = sv_dv.reserve(N), *prod = sv_prod.reserve(nv);
    // CreateHerglotzWave_PL scales by 4 pi / meas_count (CreateHerglotzWave.hpp:40)
    load_parameters(kappa, inc_coeff.data(), wc, wcs, 4.0 * M_PI / (double)mesh.nm);
    herglotz(1.0, g, wc, 0.0, hw, wc);
    dirichlet_to_neumann(kappa, hw, dv, wcc, wcs, cg_tol, gmres_tol);
    launch_row_dot(nv, wc, du_dn, dv, prod, stream);
    multiply_with_normals(prod, Y, -1.0 / wc, cg_tol);
}

} // namespace baemm
