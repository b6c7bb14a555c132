// Helmholtz_CUDA.hpp -- header-only C++ drop-in for BAEMM::Helmholtz_OpenCL
// (HenrikSchumacher/BAEMM, Helmholtz_OpenCL.hpp) over the C ABI of
// libbaemm_cuda.so (baemm.h).  User code swaps the class name:
//
//     using Helmholtz_T = BAEMM::Helmholtz_CUDA;   // was BAEMM::Helmholtz_OpenCL
//
// Signatures follow the reference: templates on the external real, complex
// and integer types (R_ext, C_ext, I_ext) and the compile-time wave count WC
// (0 = run time).  External data may be double or float precision; the
// library computes internally in FP32 (the reference's Real) or FP64 (see
// SetApplyMode).  Errors are printed to std::cerr and the call returns, as the
// reference's eprint does; GaussNewtonSolve returns the reference's bool.
// Link with -lbaemm_cuda (and -Wl,-rpath to its directory).
#pragma once

#include <complex>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <string>
#include <type_traits>
#include <vector>

#include "baemm.h"

namespace BAEMM
{

// BAEMM_Common.hpp:7-11
enum class WaveType : unsigned char
{
    Plane = 201,
    Radial = 202
};

class Helmholtz_CUDA
{
public:
    // Definitions.hpp:3-9
    using Int = int32_t;
    using LInt = std::size_t;
    using Real = float;
    using Complex = std::complex<float>;

    struct MassMatrix_T   // CSR view of the P1 mass matrix (Sparse_T in the reference)
    {
        std::vector<int64_t> outer;
        std::vector<int32_t> inner;
        std::vector<float> values;
        int64_t rows = 0, cols = 0;

        // Y = alpha M X + beta Y on nrhs columns (MatrixCSR::Dot)
        template <int NRHS = 0, typename T>
        void Dot(T alpha, const T *X, Int ldX, T beta, T *Y, Int ldY, Int nrhs = NRHS) const
        {
            for (int64_t i = 0; i < rows; ++i)
                for (Int k = 0; k < nrhs; ++k)
                {
                    T s = T(0);
                    for (int64_t e = outer[i]; e < outer[i + 1]; ++e) s += T(values[e]) * X[inner[e] * ldX + k];
                    Y[i * ldY + k] = (beta == T(0)) ? alpha * s : alpha * s + beta * Y[i * ldY + k];
                }
        }
    };

    // MemberVariables.hpp:97-98 (public in the reference)
    Int gmres_max_iter = 30;
    Int gmres_max_restarts = 3;

    // Helmholtz_OpenCL.hpp:109-159
    template <typename ExtReal, typename ExtInt>
    Helmholtz_CUDA(const ExtReal *vertex_coords_, ExtInt vertex_count_, const ExtInt *triangles_,
                   ExtInt simplex_count_, const ExtReal *meas_directions_, ExtInt meas_count_,
                   ExtInt CPU_thread_count_)
    {
        init(vertex_coords_, vertex_count_, triangles_, simplex_count_, meas_directions_, meas_count_, 0,
             CPU_thread_count_);
    }

    // Helmholtz_OpenCL.hpp:175-249
    template <typename ExtReal, typename ExtInt>
    Helmholtz_CUDA(const ExtReal *vertex_coords_, ExtInt vertex_count_, const ExtInt *triangles_,
                   ExtInt simplex_count_, const ExtReal *meas_directions_, ExtInt meas_count_, ExtInt device_num,
                   ExtInt CPU_thread_count_)
    {
        init(vertex_coords_, vertex_count_, triangles_, simplex_count_, meas_directions_, meas_count_,
             (int)device_num, CPU_thread_count_);
    }

    ~Helmholtz_CUDA() { baemm_destroy(ctx_); }

    Helmholtz_CUDA(const Helmholtz_CUDA &) = delete;
    Helmholtz_CUDA &operator=(const Helmholtz_CUDA &) = delete;

    // ---- getters / setters (GetSetters.hpp) -------------------------------------------
    std::string ClassName() const { return std::string(baemm_class_name()); }
    std::string DeviceInfo()
    {
        std::vector<char> buf(4096, 0);
        check(baemm_device_info(ctx_, buf.data(), buf.size()), "DeviceInfo");
        return std::string(buf.data());
    }
    Int VertexCount() const { return (Int)baemm_vertex_count(ctx_); }
    Int SimplexCount() const { return (Int)baemm_simplex_count(ctx_); }
    Int GetMeasCount() const { return (Int)baemm_meas_count(ctx_); }
    Int GetWaveCount() const { return baemm_get_wave_count(ctx_); }
    Int GetWaveChunkSize() const { return baemm_get_wave_chunk_size(ctx_); }
    void SetWaveChunkSize(Int wcs) { check(baemm_set_wave_chunk_size(ctx_, wcs), "SetWaveChunkSize"); }
    Int GetWaveChunkCount(Int wave_count_) const
    {
        const Int wcs = GetWaveChunkSize();
        return (wave_count_ + wcs - 1) / wcs;
    }
    Int GetBlockSize() const { return baemm_get_block_size(ctx_); }
    void SetBlockSize(Int bs) { check(baemm_set_block_size(ctx_, bs), "SetBlockSize"); }
    void UseDiagonal(bool use_it) { check(baemm_use_diagonal(ctx_, use_it ? 1 : 0), "UseDiagonal"); }
    void SetApplyMode(int mode) { check(baemm_set_apply_mode(ctx_, mode), "SetApplyMode"); }
    void SetRefinement(int steps, double inner_tol) { check(baemm_set_refinement(ctx_, steps, inner_tol), "SetRefinement"); }
    // Additions without reference counterpart (see include/baemm.h).
    void SetTuning(int key, int value) { check(baemm_set_tuning(ctx_, key, value), "SetTuning"); }
    int GetTuning(int key) const { return baemm_get_tuning(ctx_, key); }
    // 16-column groups per shared kernel-entry evaluation of the tensor-core apply (1, 2 or 4)
    int TcEntrySharing() const
    {
        const int r = baemm_tc_entry_sharing(ctx_);
        if (r < 0) check(r, "TcEntrySharing");
        return r;
    }
    baemm_tune_result Autotune(int mode, int repeats = 2)
    {
        baemm_tune_result r{};
        check(baemm_autotune(ctx_, mode, repeats, &r), "Autotune");
        return r;
    }
    void SetGraphs(bool on) { check(baemm_set_graphs(ctx_, on ? 1 : 0), "SetGraphs"); }
    template <typename ExtReal, typename ExtInt>
    void SetMesh(const ExtReal *coords, ExtInt nv, const ExtInt *tris, ExtInt nt)
    {
        auto c = to_d(coords, 3 * (size_t)nv);
        std::vector<int64_t> t(3 * (size_t)nt);
        for (size_t e = 0; e < t.size(); ++e) t[e] = (int64_t)tris[e];
        if (check(baemm_set_mesh(ctx_, c.data(), (int64_t)nv, t.data(), (int64_t)nt), "SetMesh"))
        {
            areas_.clear(); normals_.clear(); midpoints_.clear(); diag_.clear();
            mass_ = MassMatrix_T{};
            curl_ = MassMatrix_T{};
        }
    }

    const Real *Areas() { return tri_field(areas_, baemm_get_areas, 1); }
    const Real *TriangleAreas() { return Areas(); }
    const Real *TriangleNormals() { return tri_field(normals_, baemm_get_triangle_normals, 4); }
    const Real *TriangleMidpoints() { return tri_field(midpoints_, baemm_get_triangle_midpoints, 4); }
    const Real *SingleLayerDiagonal() { return tri_field(diag_, baemm_get_single_layer_diagonal, 1); }

    const MassMatrix_T &MassMatrix()
    {
        if (mass_.rows == 0)
        {
            int64_t nnz = 0;
            check(baemm_get_mass_matrix(ctx_, nullptr, nullptr, nullptr, &nnz), "MassMatrix");
            mass_.rows = mass_.cols = VertexCount();
            mass_.outer.resize(mass_.rows + 1);
            mass_.inner.resize(nnz);
            mass_.values.resize(nnz);
            check(baemm_get_mass_matrix(ctx_, mass_.outer.data(), mass_.inner.data(), mass_.values.data(), &nnz),
                  "MassMatrix");
        }
        return mass_;
    }

    // CurlOp (Initialize.hpp:146-211; a member of the reference class that no
    // method uses): 3 SimplexCount() x VertexCount() CSR in FP32.
    const MassMatrix_T &CurlOperator()
    {
        if (curl_.rows == 0)
        {
            int64_t nnz = 0;
            check(baemm_get_curl_operator(ctx_, nullptr, nullptr, nullptr, &nnz), "CurlOperator");
            curl_.rows = 3 * (int64_t)SimplexCount();
            curl_.cols = VertexCount();
            curl_.outer.resize(curl_.rows + 1);
            curl_.inner.resize(nnz);
            curl_.values.resize(nnz);
            check(baemm_get_curl_operator(ctx_, curl_.outer.data(), curl_.inner.data(), curl_.values.data(), &nnz),
                  "CurlOperator");
        }
        return curl_;
    }

    baemm_solve_stats LastSolveStats() const
    {
        baemm_solve_stats s{};
        baemm_last_solve_stats(ctx_, &s);
        return s;
    }

    baemm_ctx *native_handle() { return ctx_; }

    // ---- parameters (LoadParameters.hpp:2-81) -------------------------------------------
    template <typename R_ext, typename C_ext, typename I_ext>
    void LoadParameters(const R_ext *kappa_list, const C_ext *coeff_list, I_ext wave_count_, I_ext wave_chunk_size_,
                        R_ext factor = R_ext(1))
    {
        auto k = to_d(kappa_list, chunks(wave_count_, wave_chunk_size_));
        auto c = to_z(coeff_list, 4 * chunks(wave_count_, wave_chunk_size_));
        check(baemm_load_parameters(ctx_, k.data(), dd(c.data()), (int)wave_count_, (int)wave_chunk_size_,
                                    (double)factor), "LoadParameters");
    }

    // ---- boundary operators (ApplyBoundaryOperators.hpp) ----------------------------------
    template <Int WC = 0, typename R_ext, typename C_ext, typename I_ext>
    void ApplyBoundaryOperators_PL(const C_ext alpha, const C_ext *B_in, const I_ext ldB_in, const C_ext beta,
                                   C_ext *C_out, const I_ext ldC_out, const R_ext *kappa_list, const C_ext *coeff_list,
                                   const I_ext wave_count_, const I_ext wave_chunk_size_)
    {
        LoadBoundaryOperators_PL(kappa_list, coeff_list, wave_count_, wave_chunk_size_);
        ApplyBoundaryOperators_PL<WC>(alpha, B_in, ldB_in, beta, C_out, ldC_out);
        UnloadBoundaryOperators_PL();
    }

    template <typename R_ext, typename C_ext, typename I_ext>
    void LoadBoundaryOperators_PL(const R_ext *kappa_list, const C_ext *coeff_list, const I_ext wave_count_,
                                  const I_ext wave_chunk_size_)
    {
        auto k = to_d(kappa_list, chunks(wave_count_, wave_chunk_size_));
        auto c = to_z(coeff_list, 4 * chunks(wave_count_, wave_chunk_size_));
        check(baemm_load_boundary_operators(ctx_, k.data(), dd(c.data()), (int)wave_count_, (int)wave_chunk_size_),
              "LoadBoundaryOperators_PL");
    }

    void UnloadBoundaryOperators_PL() { check(baemm_unload_boundary_operators(ctx_), "UnloadBoundaryOperators_PL"); }

    template <Int WC = 0, typename C_ext, typename I_ext>
    void ApplyBoundaryOperators_PL(const C_ext alpha, const C_ext *B_in, const I_ext ldB_in, const C_ext beta,
                                   C_ext *C_out, const I_ext ldC_out)
    {
        if (WC > 0 && WC != GetWaveCount())
        {
            std::cerr << ClassName() << "::ApplyBoundaryOperators_PL: WC != wave_count. Doing nothing.\n";
            return;
        }
        if constexpr (std::is_same<C_ext, std::complex<double>>::value)
        {
            const double a[2] = {alpha.real(), alpha.imag()}, b[2] = {beta.real(), beta.imag()};
            check(baemm_apply_boundary_operators_z(ctx_, a, reinterpret_cast<const double *>(B_in), (int64_t)ldB_in,
                                                   b, reinterpret_cast<double *>(C_out), (int64_t)ldC_out),
                  "ApplyBoundaryOperators_PL");
        }
        else
        {
            static_assert(std::is_same<C_ext, std::complex<float>>::value, "C_ext must be std::complex<double|float>");
            const float a[2] = {alpha.real(), alpha.imag()}, b[2] = {beta.real(), beta.imag()};
            check(baemm_apply_boundary_operators_c(ctx_, a, reinterpret_cast<const float *>(B_in), (int64_t)ldB_in, b,
                                                   reinterpret_cast<float *>(C_out), (int64_t)ldC_out),
                  "ApplyBoundaryOperators_PL");
        }
    }

    // ---- far field (ApplyFarFieldOperators.hpp) -------------------------------------------
    template <Int WC = 0, typename R_ext, typename C_ext, typename I_ext>
    void ApplyFarFieldOperators_PL(const C_ext alpha, const C_ext *B_in, const I_ext ldB_in, const C_ext beta,
                                   C_ext *C_out, const I_ext ldC_out, const R_ext *kappa_list,
                                   const C_ext *coeff_list, const I_ext wave_count_, const I_ext wave_chunk_size_)
    {
        LoadParameters(kappa_list, coeff_list, wave_count_, wave_chunk_size_);
        ApplyFarFieldOperators_PL<WC>(alpha, B_in, ldB_in, beta, C_out, ldC_out);
    }

    template <Int WC = 0, typename C_ext, typename I_ext>
    void ApplyFarFieldOperators_PL(const C_ext alpha, const C_ext *B_in, const I_ext ldB_in, const C_ext beta,
                                   C_ext *C_out, const I_ext ldC_out)
    {
        const Int wc = GetWaveCount();
        auto B = to_z_block(B_in, VertexCount(), wc, ldB_in);
        std::vector<std::complex<double>> C((size_t)GetMeasCount() * wc);
        copy_block(C_out, ldC_out, C.data(), wc, GetMeasCount(), wc);
        const double a[2] = {(double)alpha.real(), (double)alpha.imag()};
        const double b[2] = {(double)beta.real(), (double)beta.imag()};
        if (check(baemm_apply_far_field_operators_loaded_z(ctx_, a, dd(B.data()), wc, b, dd(C.data()), wc),
                  "ApplyFarFieldOperators_PL"))
            copy_block(C.data(), wc, C_out, ldC_out, GetMeasCount(), wc);
    }

    // ---- near field (ApplyNearFieldOperators.hpp) ------------------------------------------
    template <typename R_ext, typename C_ext, typename I_ext>
    void ApplyNearFieldOperators_PL(const C_ext alpha, const C_ext *B_in, const I_ext ldB_in, const C_ext beta,
                                    C_ext *C_out, const I_ext ldC_out, const R_ext *kappa_list,
                                    const C_ext *coeff_list, const I_ext wave_count_, const I_ext wave_chunk_size_,
                                    const R_ext *evaluation_points, const I_ext evaluation_count)
    {
        LoadParameters(kappa_list, coeff_list, wave_count_, wave_chunk_size_);
        ApplyNearFieldOperators_PL(alpha, B_in, ldB_in, beta, C_out, ldC_out, evaluation_points, evaluation_count);
    }

    // C_out (evaluation_count x wave_count, ld ldC_out) = alpha (c1 SL + c2 DL)(points) B_in + beta C_out
    template <typename R_ext, typename C_ext, typename I_ext>
    void ApplyNearFieldOperators_PL(const C_ext alpha, const C_ext *B_in, const I_ext ldB_in, const C_ext beta,
                                    C_ext *C_out, const I_ext ldC_out, const R_ext *evaluation_points,
                                    const I_ext evaluation_count)
    {
        const Int wc = GetWaveCount();
        const Int m = (Int)evaluation_count;
        auto B = to_z_block(B_in, VertexCount(), wc, ldB_in);
        std::vector<std::complex<double>> C((size_t)m * wc);
        copy_block(C_out, ldC_out, C.data(), wc, m, wc);
        auto P = to_d(evaluation_points, 3 * (size_t)m);
        const double a[2] = {(double)alpha.real(), (double)alpha.imag()};
        const double b[2] = {(double)beta.real(), (double)beta.imag()};
        if (check(baemm_apply_near_field_operators_z(ctx_, a, dd(B.data()), wc, b, dd(C.data()), wc, P.data(),
                                                     (int64_t)m),
                  "ApplyNearFieldOperators_PL"))
            copy_block(C.data(), wc, C_out, ldC_out, m, wc);
    }

    // ---- waves (CreateIncidentWave.hpp, CreateHerglotzWave.hpp) ---------------------------
    template <typename R_ext, typename C_ext, typename I_ext>
    void CreateIncidentWave_PL(const C_ext alpha, const R_ext *incident_directions, const I_ext inc_count,
                               const C_ext beta, C_ext *C_out, const I_ext ldC_out, const R_ext *kappa_list,
                               const C_ext *coeff_list, const I_ext wave_count_, const I_ext wave_chunk_size_,
                               WaveType type = WaveType::Plane)
    {
        const Int wcc = chunks(wave_count_, wave_chunk_size_);
        auto k = to_d(kappa_list, wcc);
        auto c = to_z(coeff_list, 4 * wcc);
        auto d = to_d(incident_directions, 3 * (size_t)inc_count);
        if ((Int)inc_count > (Int)wave_chunk_size_)
            std::cerr << ClassName() << "::CreateIncidentWave_PL : Number of incident waves has to match the size "
                      << "of the wave chunks. Excess incident directions will be ignored\n";
        std::vector<std::complex<double>> C((size_t)VertexCount() * wave_count_);
        copy_block(C_out, ldC_out, C.data(), (Int)wave_count_, VertexCount(), (Int)wave_count_);
        const double a[2] = {(double)alpha.real(), (double)alpha.imag()};
        const double b[2] = {(double)beta.real(), (double)beta.imag()};
        if (check(baemm_create_incident_wave_z(ctx_, a, d.data(), (int)inc_count, b, dd(C.data()), (int)wave_count_,
                                               k.data(), dd(c.data()), (int)wave_count_, (int)wave_chunk_size_, (int)type),
                  "CreateIncidentWave_PL"))
            copy_block(C.data(), (Int)wave_count_, C_out, ldC_out, VertexCount(), (Int)wave_count_);
    }

    // The overload with the loaded parameters (CreateIncidentWave.hpp:55-124): the
    // parameters of the last LoadParameters call, wave_chunk_size directions.
    template <typename R_ext, typename C_ext, typename I_ext>
    void CreateIncidentWave_PL(const C_ext alpha, const R_ext *incident_directions, const C_ext beta, C_ext *C_out,
                               const I_ext ldC_out, WaveType type)
    {
        const Int wc = GetWaveCount(), wcs = GetWaveChunkSize();
        if (wc < 1) return;   // nothing loaded: C_out untouched, as in the reference
        auto d = to_d(incident_directions, 3 * (size_t)wcs);
        std::vector<std::complex<double>> C((size_t)VertexCount() * wc);
        copy_block(C_out, ldC_out, C.data(), wc, VertexCount(), wc);
        const double a[2] = {(double)alpha.real(), (double)alpha.imag()};
        const double b[2] = {(double)beta.real(), (double)beta.imag()};
        if (check(baemm_create_incident_wave_loaded_z(ctx_, a, d.data(), b, dd(C.data()), wc, (int)type),
                  "CreateIncidentWave_PL"))
            copy_block(C.data(), wc, C_out, ldC_out, VertexCount(), wc);
    }

    template <typename R_ext, typename C_ext, typename I_ext>
    void CreateHerglotzWave_PL(const C_ext alpha, const C_ext *B_in, const I_ext ldB_in, const C_ext beta,
                               C_ext *C_out, const I_ext ldC_out, const R_ext *kappa_list, const C_ext *coeff_list,
                               const I_ext wave_count_, const I_ext wave_chunk_size_)
    {
        const Int wcc = chunks(wave_count_, wave_chunk_size_);
        auto k = to_d(kappa_list, wcc);
        auto c = to_z(coeff_list, 4 * wcc);
        auto g = to_z_block(B_in, GetMeasCount(), (Int)wave_count_, ldB_in);
        std::vector<std::complex<double>> C((size_t)VertexCount() * wave_count_);
        copy_block(C_out, ldC_out, C.data(), (Int)wave_count_, VertexCount(), (Int)wave_count_);
        const double a[2] = {(double)alpha.real(), (double)alpha.imag()};
        const double b[2] = {(double)beta.real(), (double)beta.imag()};
        if (check(baemm_create_herglotz_wave_z(ctx_, a, dd(g.data()), (int)wave_count_, b, dd(C.data()),
                                               (int)wave_count_, k.data(), dd(c.data()), (int)wave_count_,
                                               (int)wave_chunk_size_),
                  "CreateHerglotzWave_PL"))
            copy_block(C.data(), (Int)wave_count_, C_out, ldC_out, VertexCount(), (Int)wave_count_);
    }

    // The overload with the loaded parameters (CreateHerglotzWave.hpp:51-95).
    template <typename C_ext, typename I_ext>
    void CreateHerglotzWave_PL(const C_ext alpha, const C_ext *B_in, const I_ext ldB_in, const C_ext beta,
                               C_ext *C_out, const I_ext ldC_out)
    {
        const Int wc = GetWaveCount();
        if (wc < 1) return;   // nothing loaded: C_out untouched, as in the reference
        auto g = to_z_block(B_in, GetMeasCount(), wc, ldB_in);
        std::vector<std::complex<double>> C((size_t)VertexCount() * wc);
        copy_block(C_out, ldC_out, C.data(), wc, VertexCount(), wc);
        const double a[2] = {(double)alpha.real(), (double)alpha.imag()};
        const double b[2] = {(double)beta.real(), (double)beta.imag()};
        if (check(baemm_create_herglotz_wave_loaded_z(ctx_, a, dd(g.data()), wc, b, dd(C.data()), wc),
                  "CreateHerglotzWave_PL"))
            copy_block(C.data(), wc, C_out, ldC_out, VertexCount(), wc);
    }

    // ---- mass inverse (ApplyMassInverse.hpp) --------------------------------------------
    template <Int NRHS = 0, typename X_T, typename Y_T, typename R_ext>
    void ApplyMassInverse(const X_T *X, const Int ldX, Y_T *Y, const Int ldY, const R_ext cg_tol,
                          const Int nrhs = NRHS)
    {
        if (nrhs > ldX || nrhs > ldY) { std::cerr << "nrhs > ld\n"; return; }
        mass_op(X, ldX, Y, ldY, nrhs, (double)cg_tol, false);
    }

    template <Int NRHS = 0, typename X_T, typename Y_T>
    void ApplyLumpedMassInverse(const X_T *X, const Int ldX, Y_T *Y, const Int ldY, const Int nrhs = NRHS)
    {
        mass_op(X, ldX, Y, ldY, nrhs, 0.0, true);
    }

    // ---- solvers (FarField.hpp) ------------------------------------------------------
    template <Int WC, typename I_ext, typename R_ext, typename C_ext>
    void FarField(const R_ext *kappa_, const I_ext wave_chunk_count_, R_ext *inc_directions,
                  const I_ext wave_chunk_size_, C_ext *Y_out, const WaveType type, const R_ext cg_tol,
                  const R_ext gmres_tol)
    {
        FarField_parameters<WC>(kappa_, wave_chunk_count_, inc_directions, wave_chunk_size_, Y_out, type, kappa_,
                                cg_tol, gmres_tol);
    }

    template <Int WC = 0, typename I_ext, typename R_ext, typename C_ext>
    void FarField_parameters(const R_ext *kappa_, const I_ext wave_chunk_count_, R_ext *inc_directions,
                             const I_ext wave_chunk_size_, C_ext *Y_out, const WaveType type, const R_ext *eta,
                             const R_ext cg_tol, const R_ext gmres_tol)
    {
        push_gmres();
        const Int wcc = (Int)wave_chunk_count_, wcs = (Int)wave_chunk_size_, wc = wcc * wcs;
        auto k = to_d(kappa_, wcc), e = to_d(eta, wcc), d = to_d(inc_directions, 3 * (size_t)wcs);
        std::vector<std::complex<double>> Y((size_t)GetMeasCount() * wc);
        if (check(baemm_far_field_parameters(ctx_, k.data(), wcc, d.data(), wcs, dd(Y.data()), (int)type, e.data(),
                                             (double)cg_tol, (double)gmres_tol),
                  "FarField_parameters"))
            copy_out(Y, Y_out);
    }

    template <Int WC = 0, typename I_ext, typename R_ext, typename C_ext>
    void Derivative_FF_Helper(const R_ext *kappa_, const I_ext wave_chunk_count_, const R_ext *inc_directions,
                              const I_ext wave_chunk_size_, C_ext *du_dn, const WaveType type, const R_ext cg_tol,
                              const R_ext gmres_tol)
    {
        push_gmres();
        const Int wcc = (Int)wave_chunk_count_, wcs = (Int)wave_chunk_size_, wc = wcc * wcs;
        auto k = to_d(kappa_, wcc), d = to_d(inc_directions, 3 * (size_t)wcs);
        std::vector<std::complex<double>> D((size_t)VertexCount() * wc);
        if (check(baemm_derivative_ff_helper(ctx_, k.data(), wcc, d.data(), wcs, dd(D.data()), (int)type,
                                             (double)cg_tol, (double)gmres_tol),
                  "Derivative_FF_Helper"))
            copy_out(D, du_dn);
    }

    // du_dn == nullptr: allocated with calloc and filled (the caller frees it), FarField.hpp:273-283
    template <Int WC = 0, typename I_ext, typename R_ext, typename C_ext>
    void Derivative_FF(const R_ext *kappa_, const I_ext wave_chunk_count_, const R_ext *inc_directions,
                       const I_ext wave_chunk_size_, const R_ext *X_in, C_ext *Y_out, C_ext *&du_dn,
                       const WaveType type, const R_ext cg_tol, const R_ext gmres_tol)
    {
        push_gmres();
        const Int wcc = (Int)wave_chunk_count_, wcs = (Int)wave_chunk_size_, wc = wcc * wcs;
        if (du_dn == nullptr)
        {
            du_dn = static_cast<C_ext *>(std::calloc((size_t)VertexCount() * wc, sizeof(C_ext)));
            Derivative_FF_Helper<WC>(kappa_, wave_chunk_count_, inc_directions, wave_chunk_size_, du_dn, type, cg_tol,
                                     gmres_tol);
        }
        auto k = to_d(kappa_, wcc), d = to_d(inc_directions, 3 * (size_t)wcs);
        auto X = to_d(X_in, 3 * (size_t)VertexCount());
        auto D = to_z(du_dn, (size_t)VertexCount() * wc);
        double *Dp = dd(D.data());
        std::vector<std::complex<double>> Y((size_t)GetMeasCount() * wc);
        if (check(baemm_derivative_ff(ctx_, k.data(), wcc, d.data(), wcs, X.data(), dd(Y.data()), &Dp, (int)type,
                                      (double)cg_tol, (double)gmres_tol),
                  "Derivative_FF"))
            copy_out(Y, Y_out);
    }

    template <Int WC, typename I_ext, typename R_ext, typename C_ext>
    void AdjointDerivative_FF(const R_ext *kappa_, const I_ext wave_chunk_count_, const R_ext *inc_directions,
                              const I_ext wave_chunk_size_, const C_ext *g, R_ext *Y_out, C_ext *&du_dn,
                              const WaveType type, const R_ext cg_tol, const R_ext gmres_tol)
    {
        push_gmres();
        const Int wcc = (Int)wave_chunk_count_, wcs = (Int)wave_chunk_size_, wc = wcc * wcs;
        if (du_dn == nullptr)
        {
            du_dn = static_cast<C_ext *>(std::calloc((size_t)VertexCount() * wc, sizeof(C_ext)));
            Derivative_FF_Helper<WC>(kappa_, wave_chunk_count_, inc_directions, wave_chunk_size_, du_dn, type, cg_tol,
                                     gmres_tol);
        }
        auto k = to_d(kappa_, wcc), d = to_d(inc_directions, 3 * (size_t)wcs);
        auto G = to_z(g, (size_t)GetMeasCount() * wc);
        auto D = to_z(du_dn, (size_t)VertexCount() * wc);
        double *Dp = dd(D.data());
        std::vector<double> Y(3 * (size_t)VertexCount());
        if (check(baemm_adjoint_derivative_ff(ctx_, k.data(), wcc, d.data(), wcs, dd(G.data()), Y.data(), &Dp,
                                              (int)type, (double)cg_tol, (double)gmres_tol),
                  "AdjointDerivative_FF"))
            for (size_t q = 0; q < Y.size(); ++q) Y_out[q] = (R_ext)Y[q];
    }

    // FarField.hpp:457-604: M and P are callables void(const R_ext *, R_ext *) on n x 3 arrays.
    template <Int WC, typename I_ext, typename R_ext, typename C_ext, typename M_T, typename P_T>
    bool GaussNewtonSolve(const R_ext *kappa_, const I_ext wave_chunk_count_, const R_ext *inc_directions,
                          const I_ext wave_chunk_size_, M_T &M, P_T &P, const R_ext alpha, const R_ext *B_in,
                          const I_ext ldB, const R_ext beta, R_ext *X_out, const I_ext ldX, C_ext *&du_dn,
                          const WaveType type, const R_ext cg_tol, const R_ext gmres_tol_inner,
                          const R_ext gmres_tol_outer)
    {
        static_assert(std::is_same<R_ext, double>::value, "GaussNewtonSolve: R_ext = double");
        push_gmres();
        const Int wcc = (Int)wave_chunk_count_, wcs = (Int)wave_chunk_size_, wc = wcc * wcs;
        if (du_dn == nullptr)
        {
            du_dn = static_cast<C_ext *>(std::calloc((size_t)VertexCount() * wc, sizeof(C_ext)));
            Derivative_FF_Helper<WC>(kappa_, wave_chunk_count_, inc_directions, wave_chunk_size_, du_dn, type, cg_tol,
                                     gmres_tol_inner);
        }
        auto k = to_d(kappa_, wcc), d = to_d(inc_directions, 3 * (size_t)wcs);
        auto D = to_z(du_dn, (size_t)VertexCount() * wc);
        double *Dp = dd(D.data());
        auto mcb = [](const double *x, double *y, void *u) { (*static_cast<M_T *>(u))(x, y); };
        auto pcb = [](const double *x, double *y, void *u) { (*static_cast<P_T *>(u))(x, y); };
        int ok = 0;
        check(baemm_gauss_newton_solve(ctx_, k.data(), wcc, d.data(), wcs, mcb, &M, pcb, &P, alpha, B_in,
                                       (int64_t)ldB, beta, X_out, (int64_t)ldX, &Dp, (int)type, (double)cg_tol,
                                       (double)gmres_tol_inner, (double)gmres_tol_outer, 0, &ok),
              "GaussNewtonSolve");
        return ok != 0;
    }

    template <Int WC = 0, typename I_ext, typename R_ext, typename C_ext>
    void BoundaryPotential(const R_ext *kappa_, C_ext *coeff, C_ext *wave, C_ext *phi, const I_ext wave_chunk_count_,
                           const I_ext wave_chunk_size_, const R_ext cg_tol, const R_ext gmres_tol)
    {
        push_gmres();
        const Int wcc = (Int)wave_chunk_count_, wcs = (Int)wave_chunk_size_, wc = wcc * wcs;
        auto k = to_d(kappa_, wcc);
        auto W = to_z(wave, (size_t)VertexCount() * wc);
        std::vector<std::complex<double>> c(4 * (size_t)wcc), ph((size_t)VertexCount() * wc);
        if (check(baemm_boundary_potential(ctx_, k.data(), dd(c.data()), dd(W.data()), dd(ph.data()), wcc, wcs,
                                           (double)cg_tol, (double)gmres_tol),
                  "BoundaryPotential"))
        {
            copy_out(c, coeff);
            copy_out(ph, phi);
        }
    }

    template <Int WC = 0, typename I_ext, typename R_ext, typename C_ext>
    void DirichletToNeumann(const R_ext *kappa_, C_ext *wave, C_ext *neumann_trace, const I_ext wave_chunk_count_,
                            const I_ext wave_chunk_size_, const R_ext cg_tol, const R_ext gmres_tol)
    {
        push_gmres();
        const Int wcc = (Int)wave_chunk_count_, wcs = (Int)wave_chunk_size_, wc = wcc * wcs;
        auto k = to_d(kappa_, wcc);
        auto W = to_z(wave, (size_t)VertexCount() * wc);
        std::vector<std::complex<double>> out((size_t)VertexCount() * wc);
        if (check(baemm_dirichlet_to_neumann(ctx_, k.data(), dd(W.data()), dd(out.data()), wcc, wcs, (double)cg_tol,
                                             (double)gmres_tol),
                  "DirichletToNeumann"))
            copy_out(out, neumann_trace);
    }

private:
    baemm_ctx *ctx_ = nullptr;
    std::vector<Real> areas_, normals_, midpoints_, diag_;
    MassMatrix_T mass_;
    MassMatrix_T curl_;

    template <typename ExtReal, typename ExtInt>
    void init(const ExtReal *coords, ExtInt nv, const ExtInt *tris, ExtInt nt, const ExtReal *meas, ExtInt nm,
              int device, ExtInt threads)
    {
        auto c = to_d(coords, 3 * (size_t)nv);
        auto m = to_d(meas, 3 * (size_t)nm);
        std::vector<int64_t> t(3 * (size_t)nt);
        for (size_t e = 0; e < t.size(); ++e) t[e] = (int64_t)tris[e];
        const int st = baemm_create(c.data(), (int64_t)nv, t.data(), (int64_t)nt, m.data(), (int64_t)nm, device,
                                    (int)threads, &ctx_);
        if (st != BAEMM_OK)
            std::cerr << "Helmholtz_CUDA: construction failed: " << baemm_last_error(nullptr) << "\n";
    }

    bool check(int st, const char *what) const
    {
        if (st == BAEMM_OK) return true;
        std::cerr << "Helmholtz_CUDA::" << what << ": " << baemm_last_error(ctx_) << " (status " << st << ")\n";
        return false;
    }

    void push_gmres() { check(baemm_set_gmres_params(ctx_, gmres_max_iter, gmres_max_restarts), "gmres_params"); }

    template <typename I>
    static Int chunks(I wc, I wcs) { return (Int)((wc + wcs - 1) / wcs); }

    template <typename T>
    static std::vector<double> to_d(const T *p, size_t n)
    {
        std::vector<double> v(n);
        for (size_t q = 0; q < n; ++q) v[q] = (double)p[q];
        return v;
    }
    template <typename C>
    static std::vector<std::complex<double>> to_z(const C *p, size_t n)
    {
        std::vector<std::complex<double>> v(n);
        for (size_t q = 0; q < n; ++q) v[q] = std::complex<double>((double)p[q].real(), (double)p[q].imag());
        return v;
    }
    template <typename C, typename I>
    static std::vector<std::complex<double>> to_z_block(const C *p, Int rows, Int cols, I ld)
    {
        std::vector<std::complex<double>> v((size_t)rows * cols);
        for (Int i = 0; i < rows; ++i)
            for (Int k = 0; k < cols; ++k)
                v[(size_t)i * cols + k] = std::complex<double>((double)p[(size_t)i * ld + k].real(),
                                                               (double)p[(size_t)i * ld + k].imag());
        return v;
    }
    template <typename A, typename B, typename I1, typename I2>
    static void copy_block(const A *src, I1 lds, B *dst, I2 ldd, Int rows, Int cols)
    {
        for (Int i = 0; i < rows; ++i)
            for (Int k = 0; k < cols; ++k)
                dst[(size_t)i * ldd + k] = B(src[(size_t)i * lds + k].real(), src[(size_t)i * lds + k].imag());
    }
    template <typename C>
    static void copy_out(const std::vector<std::complex<double>> &v, C *out)
    {
        for (size_t q = 0; q < v.size(); ++q) out[q] = C(v[q].real(), v[q].imag());
    }
    static double *dd(std::complex<double> *p) { return reinterpret_cast<double *>(p); }
    static const double *dd(const std::complex<double> *p) { return reinterpret_cast<const double *>(p); }

    template <typename Fn>
    const Real *tri_field(std::vector<Real> &v, Fn fn, int width)
    {
        v.assign((size_t)SimplexCount() * width, 0.f);
        check(fn(ctx_, v.data()), "triangle data");
        return v.data();
    }

    template <typename X_T, typename Y_T>
    void mass_op(const X_T *X, Int ldX, Y_T *Y, Int ldY, Int nrhs, double tol, bool lumped)
    {
        const Int n = VertexCount();
        constexpr bool cplx = !std::is_arithmetic<X_T>::value;
        const Int w = cplx ? 2 : 1;
        std::vector<double> x((size_t)n * nrhs * w), y((size_t)n * nrhs * w);
        for (Int i = 0; i < n; ++i)
            for (Int k = 0; k < nrhs; ++k)
            {
                if constexpr (cplx)
                {
                    x[((size_t)i * nrhs + k) * 2] = (double)X[(size_t)i * ldX + k].real();
                    x[((size_t)i * nrhs + k) * 2 + 1] = (double)X[(size_t)i * ldX + k].imag();
                }
                else
                    x[(size_t)i * nrhs + k] = (double)X[(size_t)i * ldX + k];
            }
        int st;
        if (cplx)
            st = lumped ? baemm_apply_lumped_mass_inverse_z(ctx_, x.data(), nrhs, y.data(), nrhs, nrhs)
                        : baemm_apply_mass_inverse_z(ctx_, x.data(), nrhs, y.data(), nrhs, nrhs, tol);
        else
            st = lumped ? baemm_apply_lumped_mass_inverse_d(ctx_, x.data(), nrhs, y.data(), nrhs, nrhs)
                        : baemm_apply_mass_inverse_d(ctx_, x.data(), nrhs, y.data(), nrhs, nrhs, tol);
        if (!check(st, "ApplyMassInverse")) return;
        for (Int i = 0; i < n; ++i)
            for (Int k = 0; k < nrhs; ++k)
            {
                if constexpr (cplx)
                    Y[(size_t)i * ldY + k] = Y_T(y[((size_t)i * nrhs + k) * 2], y[((size_t)i * nrhs + k) * 2 + 1]);
                else
                    Y[(size_t)i * ldY + k] = (Y_T)y[(size_t)i * nrhs + k];
            }
    }
};

} // namespace BAEMM
