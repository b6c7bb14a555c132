// ORACLE TEST INFRASTRUCTURE -- not part of the product.
//
// Host driver for the shim-compiled reference kernels (see cl_shim.h).  It is
// appended after the kernel sources by build_ref.sh, so the namespaces
// refcl_k<K>::{bok,ffk,hwk,nfk} (K = k_chunk_size) are visible here.
//
// Each entry point runs the reference kernel once per target row in
// [row_begin, row_end) on an OpenMP team: the same NDRange the reference
// launches (BoundaryOperatorKernel.hpp:16-18, FarFieldOperatorKernel.hpp:287-289,
// HerglotzWaveKernel.hpp, NearFieldOperatorKernel.hpp:98-101), with
// block_size == 1.  Coefficients must already be
// scaled as LoadParameters.hpp:65-79 does (c1..c3 times factor/(4 pi)).
// Not reentrant: the specialisation flags are process globals.
#include <omp.h>

thread_local int cl_shim_global_id = 0;
int Re_single_layer = 0, Im_single_layer = 0;
int Re_double_layer = 0, Im_double_layer = 0;
int Re_adjdbl_layer = 0, Im_adjdbl_layer = 0;

namespace refcl_driver
{
    // LoadParameters.hpp:47-80: a flag is set when any chunk has a non-zero part.
    static void set_flags(const float2 *coeff, int chunk_count)
    {
        Re_single_layer = Im_single_layer = 0;
        Re_double_layer = Im_double_layer = 0;
        Re_adjdbl_layer = Im_adjdbl_layer = 0;
        for (int k = 0; k < chunk_count; ++k)
        {
            Re_single_layer |= (coeff[4 * k + 1].x != 0.f);
            Im_single_layer |= (coeff[4 * k + 1].y != 0.f);
            Re_double_layer |= (coeff[4 * k + 2].x != 0.f);
            Im_double_layer |= (coeff[4 * k + 2].y != 0.f);
            Re_adjdbl_layer |= (coeff[4 * k + 3].x != 0.f);
            Im_adjdbl_layer |= (coeff[4 * k + 3].y != 0.f);
        }
    }

    template <class F>
    static void run_rows(int row_begin, int row_end, int nthreads, F &&f)
    {
        if (nthreads <= 0) nthreads = omp_get_max_threads();
        #pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
        for (int i = row_begin; i < row_end; ++i)
        {
            cl_shim_global_id = i;
            f();
        }
    }
}

#define REFCL_DISPATCH(K, CALL)                               \
    switch (K)                                                \
    {                                                         \
        case 1:  { namespace ns = refcl_k1;  CALL; break; }   \
        case 2:  { namespace ns = refcl_k2;  CALL; break; }   \
        case 4:  { namespace ns = refcl_k4;  CALL; break; }   \
        case 8:  { namespace ns = refcl_k8;  CALL; break; }   \
        case 16: { namespace ns = refcl_k16; CALL; break; }   \
        case 32: { namespace ns = refcl_k32; CALL; break; }   \
        case 64: { namespace ns = refcl_k64; CALL; break; }   \
        default: return 1;                                    \
    }

extern "C" {

// BoundaryOperatorKernel.cl:5-239.  B, C: n x wave_count complex64 rows.
int refcl_boundary(const float4 *mid, const float4 *nrm, const float2 *B, float2 *C,
                   const float *kappa, const float2 *coeff,
                   int n, int wave_count, int wave_chunk_size,
                   int row_begin, int row_end, int nthreads)
{
    const int chunk_count = wave_count / wave_chunk_size;
    refcl_driver::set_flags(coeff, chunk_count);
    REFCL_DISPATCH(wave_chunk_size,
        refcl_driver::run_rows(row_begin, row_end, nthreads, [&] {
            ns::bok::BoundaryOperatorKernel(mid, nrm, B, C, kappa, coeff, &n, &wave_count);
        }))
    return 0;
}

// FarFieldOperatorKernel.cl:5-178.  B: n x wave_count, C: m x wave_count.
int refcl_farfield(const float4 *mid, const float4 *nrm, const float4 *meas,
                   const float2 *B, float2 *C,
                   const float *kappa, const float2 *coeff,
                   int n, int m, int wave_count, int wave_chunk_size,
                   int row_begin, int row_end, int nthreads)
{
    const int chunk_count = wave_count / wave_chunk_size;
    refcl_driver::set_flags(coeff, chunk_count);
    REFCL_DISPATCH(wave_chunk_size,
        refcl_driver::run_rows(row_begin, row_end, nthreads, [&] {
            ns::ffk::FarFieldOperatorKernel(mid, nrm, meas, B, C, kappa, coeff, &n, &m, &wave_count);
        }))
    return 0;
}

// HerglotzWaveKernel.cl:5-176.  B (the kernel g): m x wave_count, C: n x wave_count.
int refcl_herglotz(const float4 *mid, const float4 *nrm, const float4 *meas,
                   const float2 *B, float2 *C,
                   const float *kappa, const float2 *coeff,
                   int n, int m, int wave_count, int wave_chunk_size,
                   int row_begin, int row_end, int nthreads)
{
    const int chunk_count = wave_count / wave_chunk_size;
    refcl_driver::set_flags(coeff, chunk_count);
    REFCL_DISPATCH(wave_chunk_size,
        refcl_driver::run_rows(row_begin, row_end, nthreads, [&] {
            ns::hwk::HerglotzWaveKernel(mid, nrm, meas, B, C, kappa, coeff, &n, &m, &wave_count);
        }))
    return 0;
}

// NearFieldOperatorKernel.cl:5-194.  B: n x wave_count (triangle values),
// points: m evaluation points (xyz, w = 0), C: m x wave_count.
int refcl_nearfield(const float4 *mid, const float4 *nrm, const float2 *B, const float4 *points, float2 *C,
                    const float *kappa, const float2 *coeff,
                    int n, int m, int wave_count, int wave_chunk_size,
                    int row_begin, int row_end, int nthreads)
{
    const int chunk_count = wave_count / wave_chunk_size;
    refcl_driver::set_flags(coeff, chunk_count);
    REFCL_DISPATCH(wave_chunk_size,
        refcl_driver::run_rows(row_begin, row_end, nthreads, [&] {
            ns::nfk::NearFieldOperatorKernel(mid, nrm, B, points, C, kappa, coeff, &n, &wave_count, &m);
        }))
    return 0;
}

int refcl_max_threads(void) { return omp_get_max_threads(); }

} // extern "C"
