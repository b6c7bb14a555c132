// The reference's example call sequence (Example_OpenCL/main.cpp:86-233) run
// through the C++ drop-in class with Helmholtz_OpenCL replaced by
// Helmholtz_CUDA: FarField, Derivative_FF (du_dn allocated by the library)
// and AdjointDerivative_FF applied to the derivative, on 16 plane waves of one
// wavenumber.  Inputs and outputs are text files so that a test can compare
// them with the CPU oracle:
//
//   dropin_farfield MESH.txt DIRS.txt MEAS.txt KAPPA CG_TOL GMRES_TOL OUT_PREFIX
//
// MESH.txt is the reference's mesh format (read with BAEMM::ReadMeshFromFile);
// DIRS.txt holds 16 incident directions and MEAS.txt the measurement
// directions, three numbers per line.  Writes OUT_PREFIX{F,DF,DFT}.txt:
// F and DF as meas_count x 16 complex (re im pairs per line), DFT as
// vertex_count x 3 reals.  As in the example, h = the vertex coordinates.
#include "BAEMM_Meshes.hpp"
#include "Helmholtz_CUDA.hpp"

#include <complex>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

namespace
{
std::vector<double> read_rows3(const char *path)
{
    std::vector<double> v;
    std::ifstream s(path);
    double x;
    while (s >> x) v.push_back(x);
    return v;
}

template <class T>
bool write_block(const std::string &path, const T *data, long rows, long cols)
{
    std::FILE *f = std::fopen(path.c_str(), "w");
    if (!f) return false;
    for (long i = 0; i < rows; ++i)
    {
        for (long k = 0; k < cols; ++k)
        {
            if constexpr (std::is_same<T, std::complex<double>>::value)
                std::fprintf(f, "%.17g %.17g ", data[i * cols + k].real(), data[i * cols + k].imag());
            else
                std::fprintf(f, "%.17g ", data[i * cols + k]);
        }
        std::fprintf(f, "\n");
    }
    return std::fclose(f) == 0;
}
} // namespace

int main(int argc, char **argv)
{
    using namespace BAEMM;
    using Real = double;
    using Complex = std::complex<Real>;
    using Int = int64_t;
    if (argc != 8)
    {
        std::fprintf(stderr, "usage: %s MESH DIRS MEAS KAPPA CG_TOL GMRES_TOL OUT_PREFIX\n", argv[0]);
        return 2;
    }
    std::vector<double> coords;
    std::vector<int64_t> tris;
    if (!ReadMeshFromFile(argv[1], coords, tris)) return 3;
    std::vector<double> inc = read_rows3(argv[2]), meas = read_rows3(argv[3]);   // non-const: FarField.hpp takes R_ext *
    const Int vertex_count = (Int)coords.size() / 3, simplex_count = (Int)tris.size() / 3;
    const Int meas_count = (Int)meas.size() / 3;
    constexpr Int wave_count = 16, wave_chunk_size = 16, wave_chunk_count = wave_count / wave_chunk_size;
    if ((Int)inc.size() != 3 * wave_chunk_size || meas_count < 1) return 4;
    const Real kappa[wave_chunk_count] = {std::atof(argv[4])};
    Real cg_tol = std::atof(argv[5]), gmres_tol = std::atof(argv[6]);
    const std::string out = argv[7];

    Helmholtz_CUDA H(coords.data(), vertex_count, tris.data(), simplex_count, meas.data(), meas_count, Int(0),
                     Int(1));
    H.UseDiagonal(true);
    std::vector<Complex> F(meas_count * wave_count), DFh(meas_count * wave_count);
    H.FarField<wave_count>(kappa, wave_chunk_count, inc.data(), wave_chunk_size, F.data(), WaveType::Plane, cg_tol,
                           gmres_tol);
    std::vector<Real> h(coords), w(vertex_count * 3);
    Complex *du_dn = nullptr;   // allocated by the library (FarField.hpp:273-283), freed below
    H.Derivative_FF<wave_count>(kappa, wave_chunk_count, inc.data(), wave_chunk_size, h.data(), DFh.data(), du_dn,
                                WaveType::Plane, cg_tol, gmres_tol);
    H.AdjointDerivative_FF<wave_count>(kappa, wave_chunk_count, inc.data(), wave_chunk_size, DFh.data(), w.data(),
                                       du_dn, WaveType::Plane, cg_tol, gmres_tol);
    if (du_dn == nullptr) return 5;
    std::free(du_dn);
    const bool ok = write_block(out + "F.txt", F.data(), meas_count, wave_count) &&
                    write_block(out + "DF.txt", DFh.data(), meas_count, wave_count) &&
                    write_block(out + "DFT.txt", w.data(), vertex_count, 3);
    return ok ? 0 : 6;
}
