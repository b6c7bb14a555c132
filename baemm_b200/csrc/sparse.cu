// Sparse vertex <-> triangle operators and small row/column kernels.
//   AvOp     (PL -> PC)  Initialize.hpp:133-143, used ApplyBoundaryOperators.hpp:333-337
//   AvOp^T   (PC -> PL)  ApplyBoundaryOperators.hpp:349-353, fused here with the
//                        SL diagonal (ApplySingleLayerDiagonal.hpp:397-454) and the
//                        mass term (ApplyBoundaryOperators.hpp:363-387)
//   Mass     CSR SpMM on real columns (ApplyMassInverse.hpp:82-89)
// All are HBM-bound gathers: one thread per (row, column), consecutive
// threads walk consecutive columns of a row so every gathered row is read as
// one contiguous segment.
#include "ops.cuh"

namespace baemm
{
namespace
{

template <class T> __device__ __forceinline__ double2 ld2(const T *p);
template <> __device__ __forceinline__ double2 ld2<float2>(const float2 *p) { float2 v = __ldg(p); return make_double2(v.x, v.y); }
template <> __device__ __forceinline__ double2 ld2<double2>(const double2 *p) { return __ldg(p); }
template <class T> __device__ __forceinline__ T st2(double2 v);
template <> __device__ __forceinline__ float2 st2<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }
template <> __device__ __forceinline__ double2 st2<double2>(double2 v) { return v; }

__device__ __forceinline__ double2 dmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }

// 2-D grid: threadIdx.x / blockIdx.y run over the columns (a warp reads 32
// consecutive columns of a row), threadIdx.y / blockIdx.x over the rows.
constexpr int kRowsPerBlock = 8;

template <class Text, class R>
__global__ void __launch_bounds__(32 * kRowsPerBlock)
avop_kernel(int64_t nt, int wc, const int32_t *__restrict__ tri_sorted, const R *__restrict__ a3,
            const Text *__restrict__ Bin, int64_t ldB, cplx<R> *__restrict__ Btri)
{
    const int64_t t = (int64_t)blockIdx.x * kRowsPerBlock + threadIdx.y;
    const int k = blockIdx.y * 32 + threadIdx.x;
    if (t >= nt || k >= wc) return;
    const int64_t idx = t * wc + k;
    const double a = (double)a3[t];
    double2 s = make_double2(0.0, 0.0);
    #pragma unroll
    for (int q = 0; q < 3; ++q)
    {
        const double2 b = ld2<Text>(&Bin[(int64_t)tri_sorted[3 * t + q] * ldB + k]);
        s.x += a * b.x;
        s.y += a * b.y;
    }
    cplx<R> o;
    o.x = (R)s.x;
    o.y = (R)s.y;
    Btri[idx] = o;
}

template <class R> struct PrmOf;
template <> struct PrmOf<float> { using type = ChunkParamsF; };
template <> struct PrmOf<double> { using type = ChunkParamsD; };

template <class Text, class R>
__global__ void __launch_bounds__(32 * kRowsPerBlock)
epilogue_kernel(int64_t nv, int wc, int wcs, bool layers, bool sl_diag, bool mass,
                                const int32_t *__restrict__ avt_outer, const int32_t *__restrict__ avt_inner,
                                const R *__restrict__ a3, const R *__restrict__ diag,
                                const cplx<R> *__restrict__ Ctri, const cplx<R> *__restrict__ Btri,
                                const typename PrmOf<R>::type *__restrict__ prm,
                                const int32_t *__restrict__ m_outer, const int32_t *__restrict__ m_inner,
                                const R *__restrict__ m_val,
                                const Text *__restrict__ Bin, int64_t ldB, double2 alpha, double2 beta,
                                Text *__restrict__ Cout, int64_t ldC, int64_t t_begin, int64_t t_end)
{
    const int64_t v = (int64_t)blockIdx.x * kRowsPerBlock + threadIdx.y;
    const int k = blockIdx.y * 32 + threadIdx.x;
    if (v >= nv || k >= wc) return;
    const int ch = k / wcs;
    double2 out = make_double2(0.0, 0.0);
    if (layers)
    {
        cplx<R> c1, ik;
        if (sl_diag)
        {
            c1 = prm[ch].c[1];
            ik.x = R(0);
            ik.y = prm[ch].kappa;
        }
        double2 s = make_double2(0.0, 0.0);
        for (int32_t e = avt_outer[v]; e < avt_outer[v + 1]; ++e)
        {
            const int64_t t = avt_inner[e];
            if (t < t_begin || t >= t_end) continue;   // a row shard: triangles of other shards
            cplx<R> ct = Ctri[t * wc + k];
            if (sl_diag)
            {
                // C[i,k] += c1 (diag_i + i kappa) B[i,k]   (ApplySingleLayerDiagonal.hpp:427-433)
                cplx<R> f = ik;
                f.x += diag[t];
                f = cmul(c1, f);
                cfma(ct, f, Btri[t * wc + k]);
            }
            const double a = (double)a3[t];
            s.x += a * (double)ct.x;
            s.y += a * (double)ct.y;
        }
        out = dmul(alpha, s);
    }
    if (mass)
    {
        // factor = alpha * c0 (c0 stored in the internal precision, ApplyBoundaryOperators.hpp:367-368)
        const cplx<R> c0 = prm[ch].c[0];
        const double2 f = dmul(alpha, make_double2((double)c0.x, (double)c0.y));
        double2 s = make_double2(0.0, 0.0);
        for (int32_t e = m_outer[v]; e < m_outer[v + 1]; ++e)
        {
            const double mv = (double)m_val[e];
            const double2 b = ld2<Text>(&Bin[(int64_t)m_inner[e] * ldB + k]);
            s.x += mv * b.x;
            s.y += mv * b.y;
        }
        const double2 t = dmul(f, s);
        out.x += t.x;
        out.y += t.y;
    }
    Text *o = &Cout[v * ldC + k];
    if (beta.x != 0.0 || beta.y != 0.0)
    {
        const double2 b = dmul(beta, ld2<Text>(o));
        out.x += b.x;
        out.y += b.y;
    }
    *o = st2<Text>(out);
}

// DotWithNormals_PL (FarField.hpp:980-1005), per triangle, in precision R.
template <class R>
__global__ void dot_normals_tri_kernel(int64_t nt, const int32_t *__restrict__ tri_sorted, const R *__restrict__ a3,
                                       const R *__restrict__ area, const R *__restrict__ nrm4,
                                       const double *__restrict__ X, R *__restrict__ Ytri)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const double a = (double)a3[t];
    const R f = R(1) / area[t];
    R s = R(0);
    for (int d = 0; d < 3; ++d)
    {
        double x = 0.0;
        for (int q = 0; q < 3; ++q) x += a * X[3 * (int64_t)tri_sorted[3 * t + q] + d];
        s += nrm4[4 * t + d] * (R)x * f;
    }
    Ytri[t] = s;
}

// MultiplyWithNormals_PL (FarField.hpp:914-935), per triangle.
template <class R>
__global__ void mult_normals_tri_kernel(int64_t nt, const int32_t *__restrict__ tri_sorted, const R *__restrict__ a3,
                                        const R *__restrict__ area, const R *__restrict__ nrm4,
                                        const double2 *__restrict__ X, R *__restrict__ Ytri)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const double a = (double)a3[t];
    double re = 0.0;
    for (int q = 0; q < 3; ++q) re += a * X[tri_sorted[3 * t + q]].x;
    const R mul = (R)re / area[t];
    for (int d = 0; d < 3; ++d) Ytri[3 * t + d] = mul * nrm4[4 * t + d];
}

// AvOp^T on `cols` real columns in precision R: Yw[v,d] = factor * sum a3_t Ytri[t,d].
template <class R>
__global__ void avopT_real_kernel(int64_t nv, int cols, const int32_t *__restrict__ avt_outer,
                                  const int32_t *__restrict__ avt_inner, const R *__restrict__ a3,
                                  const R *__restrict__ Ytri, R factor, double *__restrict__ Yw)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nv * cols) return;
    const int64_t v = idx / cols;
    const int d = (int)(idx - v * cols);
    R s = R(0);
    for (int32_t e = avt_outer[v]; e < avt_outer[v + 1]; ++e)
    {
        const int64_t t = avt_inner[e];
        s += a3[t] * Ytri[t * cols + d];
    }
    Yw[idx] = (double)(factor * s);
}

__global__ void scale_rows_neg_kernel(int64_t nv, int wc, const double *__restrict__ s, const double2 *__restrict__ du,
                                      double2 *__restrict__ out)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nv * wc) return;
    const double f = -s[idx / wc];
    const double2 d = du[idx];
    out[idx] = make_double2(f * d.x, f * d.y);
}

__global__ void row_dot_kernel(int64_t nv, int wc, const double2 *__restrict__ a, const double2 *__restrict__ b,
                               double2 *__restrict__ out)
{
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    double2 s = make_double2(0.0, 0.0);
    for (int k = 0; k < wc; ++k)
    {
        const double2 x = a[v * wc + k], y = b[v * wc + k];
        s.x += x.x * y.x - x.y * y.y;
        s.y += x.x * y.y + x.y * y.x;
    }
    out[v] = s;
}

template <class RV>
__global__ void mass_dot_real_kernel(int64_t nv, int cols, const int32_t *__restrict__ m_outer,
                                     const int32_t *__restrict__ m_inner, const RV *__restrict__ m_val, double alpha,
                                     const double *__restrict__ X, int64_t ldX, double beta, double *__restrict__ Y,
                                     int64_t ldY)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nv * cols) return;
    const int64_t v = idx / cols;
    const int k = (int)(idx - v * cols);
    double s = 0.0;
    for (int32_t e = m_outer[v]; e < m_outer[v + 1]; ++e) s += (double)m_val[e] * X[(int64_t)m_inner[e] * ldX + k];
    double *o = &Y[v * ldY + k];
    *o = (beta == 0.0) ? alpha * s : alpha * s + beta * (*o);
}

template <class RV>
__global__ void lumped_real_kernel(int64_t nv, int cols, const RV *__restrict__ L, const double *__restrict__ X,
                                   int64_t ldX, double *__restrict__ Y, int64_t ldY)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nv * cols) return;
    const int64_t v = idx / cols;
    const int k = (int)(idx - v * cols);
    Y[v * ldY + k] = (double)L[v] * X[v * ldX + k];
}

template <class Tsrc, class Tdst> __device__ __forceinline__ Tdst conv(Tsrc v);
template <> __device__ __forceinline__ double2 conv<double2, double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 conv<double2, float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }
template <> __device__ __forceinline__ double2 conv<float2, double2>(float2 v) { return make_double2(v.x, v.y); }
template <> __device__ __forceinline__ float2 conv<float2, float2>(float2 v) { return v; }
template <> __device__ __forceinline__ double conv<double, double>(double v) { return v; }
template <> __device__ __forceinline__ float conv<float, float>(float v) { return v; }

template <class Tsrc, class Tdst>
__global__ void copy_block_kernel(int64_t rows, int cols, const Tsrc *__restrict__ src, int64_t lds,
                                  Tdst *__restrict__ dst, int64_t ldd)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= rows * cols) return;
    const int64_t r = idx / cols;
    const int c = (int)(idx - r * cols);
    dst[r * ldd + c] = conv<Tsrc, Tdst>(src[r * lds + c]);
}

__device__ __forceinline__ double mulT(double a, double b) { return a * b; }
__device__ __forceinline__ double2 mulT(double2 a, double2 b) { return dmul(a, b); }
__device__ __forceinline__ double addT(double a, double b) { return a + b; }
__device__ __forceinline__ double2 addT(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ bool isZero(double a) { return a == 0.0; }
__device__ __forceinline__ bool isZero(double2 a) { return a.x == 0.0 && a.y == 0.0; }

template <class T>
__global__ void axpby_kernel(int64_t rows, int cols, T a, const T *__restrict__ x, int64_t ldx, T b, T *__restrict__ y,
                             int64_t ldy)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= rows * cols) return;
    const int64_t r = idx / cols;
    const int c = (int)(idx - r * cols);
    T *o = &y[r * ldy + c];
    const T ax = mulT(a, x[r * ldx + c]);
    *o = isZero(b) ? ax : addT(ax, mulT(b, *o));
}

// Cout = alpha Cin + beta Cout (keep = false: beta == 0, overwrite, so stale
// NaNs do not survive), in double, Cin packed with ld wc.
template <class Text, class R>
__global__ void combine_kernel(int64_t rows, int wc, double2 alpha, const cplx<R> *__restrict__ Cin, double2 beta,
                               Text *__restrict__ Cout, int64_t ldC, bool keep)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= rows * wc) return;
    const int64_t r = idx / wc;
    const int c = (int)(idx - r * wc);
    const cplx<R> x = Cin[idx];
    double2 v = dmul(alpha, make_double2((double)x.x, (double)x.y));
    Text *o = &Cout[r * ldC + c];
    if (keep)
    {
        const Text yo = *o;   // read and written by this thread only
        const double2 y = dmul(beta, make_double2((double)yo.x, (double)yo.y));
        v.x += y.x;
        v.y += y.y;
    }
    *o = st2<Text>(v);
}

constexpr int kT = 256;
inline int grid_for(int64_t n) { return ceil_div(n, kT); }

} // namespace

template <class Text, class R>
void launch_avop(const MeshDev &m, const Text *Bin, int64_t ldB, int wc, cplx<R> *Btri, cudaStream_t st)
{
    const int64_t n = m.nt * wc;
    if (n == 0) return;
    const R *a3;
    if constexpr (std::is_same<R, float>::value) a3 = m.a3_f; else a3 = m.a3_d;
    const dim3 grid(ceil_div(m.nt, kRowsPerBlock), ceil_div(wc, 32)), block(32, kRowsPerBlock);
    avop_kernel<Text, R><<<grid, block, 0, st>>>(m.nt, wc, m.tri_sorted, a3, Bin, ldB, Btri);
    BAEMM_LAUNCH_CHECK();
}

template <class Text, class R>
void launch_epilogue(const MeshDev &m, const EpilogueArgs &a, const cplx<R> *Ctri, const cplx<R> *Btri,
                     const void *chunk_params, const Text *Bin, int64_t ldB, Text alpha, Text beta, Text *Cout,
                     int64_t ldC, cudaStream_t st)
{
    const int64_t n = m.nv * a.wc;
    if (n == 0) return;
    const R *a3, *diag, *mv;
    if constexpr (std::is_same<R, float>::value) { a3 = m.a3_f; diag = m.diag_f; mv = m.mass_f; }
    else { a3 = m.a3_d; diag = m.diag_d; mv = m.mass_d; }
    const double2 al = make_double2((double)alpha.x, (double)alpha.y);
    const double2 be = make_double2((double)beta.x, (double)beta.y);
    const dim3 grid(ceil_div(m.nv, kRowsPerBlock), ceil_div(a.wc, 32)), block(32, kRowsPerBlock);
    epilogue_kernel<Text, R><<<grid, block, 0, st>>>(
        m.nv, a.wc, a.wcs, a.layers, a.sl_diag, a.mass, m.avt_outer, m.avt_inner, a3, diag, Ctri, Btri,
        static_cast<const typename PrmOf<R>::type *>(chunk_params), m.mass_outer, m.mass_inner, mv, Bin, ldB, al, be,
        Cout, ldC, a.t_begin, a.t_end);
    BAEMM_LAUNCH_CHECK();
}

void launch_dot_with_normals_weak(const MeshDev &m, bool fp64, const double *X, double *Ytri, double *Yw,
                                  cudaStream_t st)
{
    if (fp64)
    {
        dot_normals_tri_kernel<double><<<grid_for(m.nt), kT, 0, st>>>(m.nt, m.tri_sorted, m.a3_d, m.area_d, m.nrm_d, X,
                                                                       Ytri);
        avopT_real_kernel<double><<<grid_for(m.nv), kT, 0, st>>>(m.nv, 1, m.avt_outer, m.avt_inner, m.a3_d, Ytri, 1.0,
                                                                  Yw);
    }
    else
    {
        float *Yt = reinterpret_cast<float *>(Ytri);
        dot_normals_tri_kernel<float><<<grid_for(m.nt), kT, 0, st>>>(m.nt, m.tri_sorted, m.a3_f, m.area_f, m.nrm_f, X,
                                                                      Yt);
        avopT_real_kernel<float><<<grid_for(m.nv), kT, 0, st>>>(m.nv, 1, m.avt_outer, m.avt_inner, m.a3_f, Yt, 1.f,
                                                                 Yw);
    }
    BAEMM_LAUNCH_CHECK();
}

void launch_mult_with_normals_weak(const MeshDev &m, bool fp64, const double2 *X, double factor, double *Ytri,
                                   double *Yw, cudaStream_t st)
{
    if (fp64)
    {
        mult_normals_tri_kernel<double><<<grid_for(m.nt), kT, 0, st>>>(m.nt, m.tri_sorted, m.a3_d, m.area_d, m.nrm_d,
                                                                        X, Ytri);
        avopT_real_kernel<double><<<grid_for(m.nv * 3), kT, 0, st>>>(m.nv, 3, m.avt_outer, m.avt_inner, m.a3_d, Ytri,
                                                                      factor, Yw);
    }
    else
    {
        float *Yt = reinterpret_cast<float *>(Ytri);
        mult_normals_tri_kernel<float><<<grid_for(m.nt), kT, 0, st>>>(m.nt, m.tri_sorted, m.a3_f, m.area_f, m.nrm_f,
                                                                       X, Yt);
        avopT_real_kernel<float><<<grid_for(m.nv * 3), kT, 0, st>>>(m.nv, 3, m.avt_outer, m.avt_inner, m.a3_f, Yt,
                                                                     (float)factor, Yw);
    }
    BAEMM_LAUNCH_CHECK();
}

void launch_scale_rows_neg(int64_t nv, int wc, const double *s, const double2 *du, double2 *out, cudaStream_t st)
{
    if (nv * wc == 0) return;
    scale_rows_neg_kernel<<<grid_for(nv * wc), kT, 0, st>>>(nv, wc, s, du, out);
    BAEMM_LAUNCH_CHECK();
}

void launch_row_dot(int64_t nv, int wc, const double2 *du, const double2 *dv, double2 *out, cudaStream_t st)
{
    if (nv == 0) return;
    row_dot_kernel<<<grid_for(nv), kT, 0, st>>>(nv, wc, du, dv, out);
    BAEMM_LAUNCH_CHECK();
}

void launch_mass_dot_real(const MeshDev &m, bool fp64_values, double alpha, const double *X, int64_t ldX, double beta,
                          double *Y, int64_t ldY, int ncols, cudaStream_t st)
{
    const int64_t n = m.nv * ncols;
    if (n == 0) return;
    if (fp64_values)
        mass_dot_real_kernel<double><<<grid_for(n), kT, 0, st>>>(m.nv, ncols, m.mass_outer, m.mass_inner, m.mass_d,
                                                                  alpha, X, ldX, beta, Y, ldY);
    else
        mass_dot_real_kernel<float><<<grid_for(n), kT, 0, st>>>(m.nv, ncols, m.mass_outer, m.mass_inner, m.mass_f,
                                                                 alpha, X, ldX, beta, Y, ldY);
    BAEMM_LAUNCH_CHECK();
}

void launch_lumped_real(const MeshDev &m, bool fp64_values, const double *X, int64_t ldX, double *Y, int64_t ldY,
                        int ncols, cudaStream_t st)
{
    const int64_t n = m.nv * ncols;
    if (n == 0) return;
    if (fp64_values)
        lumped_real_kernel<double><<<grid_for(n), kT, 0, st>>>(m.nv, ncols, m.lumped_d, X, ldX, Y, ldY);
    else
        lumped_real_kernel<float><<<grid_for(n), kT, 0, st>>>(m.nv, ncols, m.lumped_f, X, ldX, Y, ldY);
    BAEMM_LAUNCH_CHECK();
}

template <class Text, class R>
void launch_combine(int64_t rows, int wc, double2 alpha, const cplx<R> *Cin, double2 beta, Text *Cout, int64_t ldC,
                    cudaStream_t st)
{
    if (rows * wc == 0) return;
    const bool keep = !(beta.x == 0.0 && beta.y == 0.0);
    combine_kernel<Text, R><<<grid_for(rows * wc), kT, 0, st>>>(rows, wc, alpha, Cin, beta, Cout, ldC, keep);
    BAEMM_LAUNCH_CHECK();
}

template <class Tsrc, class Tdst>
void launch_copy_block(int64_t rows, int cols, const Tsrc *src, int64_t lds, Tdst *dst, int64_t ldd, cudaStream_t st)
{
    if (rows * cols == 0) return;
    copy_block_kernel<Tsrc, Tdst><<<grid_for(rows * cols), kT, 0, st>>>(rows, cols, src, lds, dst, ldd);
    BAEMM_LAUNCH_CHECK();
}

template <class T>
void launch_axpby(int64_t rows, int cols, T a, const T *x, int64_t ldx, T b, T *y, int64_t ldy, cudaStream_t st)
{
    if (rows * cols == 0) return;
    axpby_kernel<T><<<grid_for(rows * cols), kT, 0, st>>>(rows, cols, a, x, ldx, b, y, ldy);
    BAEMM_LAUNCH_CHECK();
}

// explicit instantiations
template void launch_avop<double2, float>(const MeshDev &, const double2 *, int64_t, int, float2 *, cudaStream_t);
template void launch_avop<float2, float>(const MeshDev &, const float2 *, int64_t, int, float2 *, cudaStream_t);
template void launch_avop<double2, double>(const MeshDev &, const double2 *, int64_t, int, double2 *, cudaStream_t);
template void launch_avop<float2, double>(const MeshDev &, const float2 *, int64_t, int, double2 *, cudaStream_t);
template void launch_epilogue<double2, float>(const MeshDev &, const EpilogueArgs &, const float2 *, const float2 *,
                                              const void *, const double2 *, int64_t, double2, double2, double2 *,
                                              int64_t, cudaStream_t);
template void launch_epilogue<float2, float>(const MeshDev &, const EpilogueArgs &, const float2 *, const float2 *,
                                             const void *, const float2 *, int64_t, float2, float2, float2 *, int64_t,
                                             cudaStream_t);
template void launch_epilogue<double2, double>(const MeshDev &, const EpilogueArgs &, const double2 *, const double2 *,
                                               const void *, const double2 *, int64_t, double2, double2, double2 *,
                                               int64_t, cudaStream_t);
template void launch_epilogue<float2, double>(const MeshDev &, const EpilogueArgs &, const double2 *, const double2 *,
                                              const void *, const float2 *, int64_t, float2, float2, float2 *,
                                              int64_t, cudaStream_t);
template void launch_combine<double2, float>(int64_t, int, double2, const float2 *, double2, double2 *, int64_t,
                                            cudaStream_t);
template void launch_combine<double2, double>(int64_t, int, double2, const double2 *, double2, double2 *, int64_t,
                                             cudaStream_t);
template void launch_combine<float2, float>(int64_t, int, double2, const float2 *, double2, float2 *, int64_t,
                                           cudaStream_t);
template void launch_combine<float2, double>(int64_t, int, double2, const double2 *, double2, float2 *, int64_t,
                                            cudaStream_t);
template void launch_copy_block<double2, double2>(int64_t, int, const double2 *, int64_t, double2 *, int64_t,
                                                  cudaStream_t);
template void launch_copy_block<double2, float2>(int64_t, int, const double2 *, int64_t, float2 *, int64_t,
                                                 cudaStream_t);
template void launch_copy_block<float2, double2>(int64_t, int, const float2 *, int64_t, double2 *, int64_t,
                                                 cudaStream_t);
template void launch_copy_block<float2, float2>(int64_t, int, const float2 *, int64_t, float2 *, int64_t,
                                                cudaStream_t);
template void launch_copy_block<double, double>(int64_t, int, const double *, int64_t, double *, int64_t,
                                                cudaStream_t);
template void launch_axpby<double>(int64_t, int, double, const double *, int64_t, double, double *, int64_t,
                                   cudaStream_t);
template void launch_axpby<double2>(int64_t, int, double2, const double2 *, int64_t, double2, double2 *, int64_t,
                                    cudaStream_t);

} // namespace baemm
