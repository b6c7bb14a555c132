// Compile-and-link check of the C++ drop-in class: the call sequence of the
// reference's Example_OpenCL/main.cpp:86-233 with Helmholtz_OpenCL replaced by
// Helmholtz_CUDA.  Run on a GPU box it computes a small far field and its
// derivative; without a device every call reports an error and returns.
#include "Helmholtz_CUDA.hpp"
#include "BAEMM_Meshes.hpp"

#include <cmath>
#include <complex>
#include <cstdio>
#include <vector>

int main()
{
    using namespace BAEMM;
    using Real = double;
    using Complex = std::complex<Real>;
    using Int = long;
    // one octahedron: 6 vertices, 8 triangles, outward
    std::vector<Real> coords = {1, 0, 0, -1, 0, 0, 0, 1, 0, 0, -1, 0, 0, 0, 1, 0, 0, -1};
    std::vector<Int> tris = {0, 2, 4, 2, 1, 4, 1, 3, 4, 3, 0, 4, 2, 0, 5, 1, 2, 5, 3, 1, 5, 0, 3, 5};
    std::vector<Real> meas = {0, 0, 1, 0, 0, -1};
    Helmholtz_CUDA H(coords.data(), Int(6), tris.data(), Int(8), meas.data(), Int(2), Int(0), Int(1));
    constexpr Int wave_count = 4, wave_chunk_size = 4, wave_chunk_count = 1;
    std::vector<Real> kappa = {2.0};
    std::vector<Real> inc = {1, 0, 0, 0, 1, 0, 0, 0, 1, -1, 0, 0};
    std::vector<Complex> F(2 * wave_count), DF(2 * wave_count);
    H.UseDiagonal(true);
    H.FarField<wave_count>(kappa.data(), wave_chunk_count, inc.data(), wave_chunk_size, F.data(), WaveType::Plane,
                           Real(1e-5), Real(1e-4));
    std::vector<Real> h(coords);
    Complex *du_dn = nullptr;
    H.Derivative_FF<wave_count>(kappa.data(), wave_chunk_count, inc.data(), wave_chunk_size, h.data(), DF.data(),
                                du_dn, WaveType::Plane, Real(1e-5), Real(1e-4));
    std::vector<Real> w(18);
    H.AdjointDerivative_FF<wave_count>(kappa.data(), wave_chunk_count, inc.data(), wave_chunk_size, DF.data(),
                                       w.data(), du_dn, WaveType::Plane, Real(1e-5), Real(1e-4));
    std::printf("%s |F| = %g\n", H.ClassName().c_str(), std::abs(F[0]));
    std::free(du_dn);
    // additions: re-mesh the context in place, graphs, tuning
    H.SetMesh(coords.data(), Int(6), tris.data(), Int(8));
    H.SetGraphs(true);
    H.SetTuning(BAEMM_TUNE_TC_SEGMENT, 8);
    H.SetTuning(BAEMM_TUNE_TC_SHARE, 4);
    H.SetApplyMode(BAEMM_APPLY_TC);
    H.FarField<wave_count>(kappa.data(), wave_chunk_count, inc.data(), wave_chunk_size, F.data(), WaveType::Plane,
                           Real(1e-5), Real(1e-4));
    // the near-field potential of a density at two points, CurlOp, the mesh readers
    std::vector<Complex> B(6 * wave_count, Complex(1.0, 0.0)), P(2 * wave_count);
    std::vector<Real> pts = {0.1, 0.0, 0.0, 3.0, 0.0, 0.0};
    std::vector<Complex> coeff = {Complex(0), Complex(1), Complex(1), Complex(0)};
    H.ApplyNearFieldOperators_PL(Complex(1), B.data(), wave_count, Complex(0), P.data(), wave_count, kappa.data(),
                                 coeff.data(), wave_count, wave_chunk_size, pts.data(), Int(2));
    // the waves, both overloads of each (the second form uses the loaded parameters)
    std::vector<Complex> W(6 * wave_count), G(2 * wave_count, Complex(1.0, 0.0));
    H.CreateIncidentWave_PL(Complex(1), inc.data(), wave_chunk_size, Complex(0), W.data(), wave_count, kappa.data(),
                            coeff.data(), wave_count, wave_chunk_size, WaveType::Plane);
    H.LoadParameters(kappa.data(), coeff.data(), wave_count, wave_chunk_size, Real(4 * M_PI));
    H.CreateIncidentWave_PL(Complex(1), inc.data(), Complex(0), W.data(), wave_count, WaveType::Plane);
    H.CreateHerglotzWave_PL(Complex(1), G.data(), wave_count, Complex(0), W.data(), wave_count, kappa.data(),
                            coeff.data(), wave_count, wave_chunk_size);
    H.CreateHerglotzWave_PL(Complex(1), G.data(), wave_count, Complex(0), W.data(), wave_count);
    const auto &curl = H.CurlOperator();
    std::printf("near field %g, CurlOp rows %lld\n", std::abs(P[0]), (long long)curl.rows);
    std::vector<double> mesh_coords;
    std::vector<int64_t> mesh_tris;
    if (BAEMM::ReadMeshFromFile("Sphere_00001280T.txt", mesh_coords, mesh_tris))
        std::printf("read %zu triangles\n", mesh_tris.size() / 3);
    return 0;
}
