// Per-triangle geometry, mass-matrix values and the lumped-mass inverse.
// Restates Initialize.hpp:57-353 of the reference on the device, in float
// (the reference's Real) and, as a separate copy, in double.
#include "ops.cuh"

namespace baemm
{
namespace
{

template <class R> __device__ __forceinline__ R dsqrt(R x);
template <> __device__ __forceinline__ float dsqrt<float>(float x) { return sqrtf(x); }
template <> __device__ __forceinline__ double dsqrt<double>(double x) { return sqrt(x); }
template <class R> __device__ __forceinline__ R datanh(R x);
template <> __device__ __forceinline__ float datanh<float>(float x) { return atanhf(x); }
template <> __device__ __forceinline__ double datanh<double>(double x) { return atanh(x); }

// Initialize.hpp:78-302: midpoint, area-weighted normal, area, AvOp value a/3
// and the analytic self-integral of 1/r over the triangle divided by its area.
template <class R>
__global__ void geometry_kernel(const double *__restrict__ coords, const int32_t *__restrict__ tris, int64_t nt,
                                R *__restrict__ mid4, R *__restrict__ nrm4, R *__restrict__ area,
                                R *__restrict__ a3, R *__restrict__ diag)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt) return;
    const R third = R(1) / R(3);
    const R half = R(1) / R(2);
    R x[3][3];
    #pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        const int64_t v = tris[3 * i + a];
        #pragma unroll
        for (int d = 0; d < 3; ++d) x[a][d] = (R)coords[3 * v + d];
    }
    R c[3], u[3][3], df0[3], df1[3], anu[3];
    #pragma unroll
    for (int d = 0; d < 3; ++d)
    {
        c[d] = third * (x[0][d] + x[1][d] + x[2][d]);
        df0[d] = x[1][d] - x[0][d];
        df1[d] = x[2][d] - x[0][d];
    }
    #pragma unroll
    for (int a = 0; a < 3; ++a)
        #pragma unroll
        for (int d = 0; d < 3; ++d) u[a][d] = x[a][d] - c[d];
    anu[0] = half * (df0[1] * df1[2] - df0[2] * df1[1]);
    anu[1] = half * (df0[2] * df1[0] - df0[0] * df1[2]);
    anu[2] = half * (df0[0] * df1[1] - df0[1] * df1[0]);
    const R a = dsqrt<R>(anu[0] * anu[0] + anu[1] * anu[1] + anu[2] * anu[2]);
    const R ainv = R(1) / a;
    mid4[4 * i + 0] = c[0]; mid4[4 * i + 1] = c[1]; mid4[4 * i + 2] = c[2]; mid4[4 * i + 3] = R(0);
    nrm4[4 * i + 0] = ainv * anu[0]; nrm4[4 * i + 1] = ainv * anu[1]; nrm4[4 * i + 2] = ainv * anu[2];
    nrm4[4 * i + 3] = R(0);
    area[i] = a;
    a3[i] = a * third;

    auto dot = [](const R *p, const R *q) { return p[0] * q[0] + p[1] * q[1] + p[2] * q[2]; };
    const R u00 = dot(u[0], u[0]), u11 = dot(u[1], u[1]), u22 = dot(u[2], u[2]);
    const R u01 = dot(u[0], u[1]), u12 = dot(u[1], u[2]), u20 = dot(u[2], u[0]);
    const R L0 = dsqrt<R>(u00), L1 = dsqrt<R>(u11), L2 = dsqrt<R>(u22);
    const R L0i = R(1) / L0, L1i = R(1) / L1, L2i = R(1) / L2;
    // One term per triangle edge (Initialize.hpp:269-300).
    auto edge = [](R aa, R bb, R La, R Lai, R Lbi) {
        const R vni = R(1) / dsqrt<R>(fabs(aa + bb));
        const R sa = Lai * vni * aa, sb = Lbi * vni * bb;
        return La * dsqrt<R>(R(1) - sa * sa) * (datanh<R>(sa) + datanh<R>(sb));
    };
    R sum = R(0);
    sum += edge(u11 - u12, u22 - u12, L1, L1i, L2i);
    sum += edge(u22 - u20, u00 - u20, L2, L2i, L0i);
    sum += edge(u00 - u01, u11 - u01, L0, L0i, L1i);
    diag[i] = sum / a;
}

// Row v of the P1 mass matrix: for every incident triangle t, a_t/6 on the
// diagonal and a_t/12 for the two other vertices (the summed triplets of
// Initialize.hpp:214-247), accumulated in R in ascending triangle order.
template <class R>
__global__ void mass_values_kernel(int64_t nv, const int32_t *__restrict__ tris, const int32_t *__restrict__ avt_outer,
                                   const int32_t *__restrict__ avt_inner, const R *__restrict__ area,
                                   const int32_t *__restrict__ m_outer, const int32_t *__restrict__ m_inner,
                                   R *__restrict__ m_val, R *__restrict__ lumped)
{
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    const R third = R(1) / R(3);
    const R half = R(1) / R(2);
    const R sixth = half * third, twelveth = half * sixth;
    const int32_t e0 = m_outer[v], e1 = m_outer[v + 1];
    for (int32_t e = e0; e < e1; ++e) m_val[e] = R(0);
    R lump = R(0);
    for (int32_t q = avt_outer[v]; q < avt_outer[v + 1]; ++q)
    {
        const int32_t t = avt_inner[q];
        const R a = area[t];
        lump += (a * third) * third;  // AvOp^T . (1/3), Initialize.hpp:339-345
        for (int s = 0; s < 3; ++s)
        {
            const int32_t w = tris[3 * (int64_t)t + s];
            const R val = (w == v) ? a * sixth : a * twelveth;
            for (int32_t e = e0; e < e1; ++e)
                if (m_inner[e] == w) { m_val[e] += val; break; }
        }
    }
    lumped[v] = R(1) / lump;
}

// CurlOp (Initialize.hpp:146-211): per triangle three rows (x, y, z) of
// area-weighted nu x grad of the three P1 basis functions, in FP32 (the
// reference's Real).  grad comes from the pseudo-inverse of the edge frame
// (df0, df1): df^+ = g^-1 df^T with g the 2 x 2 Gram matrix.  The row's three
// entries are written with their vertex columns in ascending order (the
// reference sorts each row, Initialize.hpp:317-323).
__global__ void curl_kernel(const double *__restrict__ coords, const int32_t *__restrict__ tris, int64_t nt,
                            int32_t *__restrict__ inner, float *__restrict__ vals)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt) return;
    int32_t v[3];
    float x[3][3];
    #pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        v[a] = tris[3 * i + a];
        #pragma unroll
        for (int d = 0; d < 3; ++d) x[a][d] = (float)coords[3 * (int64_t)v[a] + d];
    }
    float df0[3], df1[3], anu[3];
    #pragma unroll
    for (int d = 0; d < 3; ++d)
    {
        df0[d] = x[1][d] - x[0][d];
        df1[d] = x[2][d] - x[0][d];
    }
    anu[0] = 0.5f * (df0[1] * df1[2] - df0[2] * df1[1]);
    anu[1] = 0.5f * (df0[2] * df1[0] - df0[0] * df1[2]);
    anu[2] = 0.5f * (df0[0] * df1[1] - df0[1] * df1[0]);
    const float g00 = df0[0] * df0[0] + df0[1] * df0[1] + df0[2] * df0[2];
    const float g01 = df0[0] * df1[0] + df0[1] * df1[1] + df0[2] * df1[2];
    const float g11 = df1[0] * df1[0] + df1[1] * df1[1] + df1[2] * df1[2];
    const float dinv = 1.0f / (g00 * g11 - g01 * g01);
    const float i00 = g11 * dinv, i01 = -g01 * dinv, i11 = g00 * dinv;
    float grad[3][3];   // grad[component][corner]
    #pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        const float p0 = i00 * df0[k] + i01 * df1[k];
        const float p1 = i01 * df0[k] + i11 * df1[k];
        grad[k][0] = -p0 - p1;
        grad[k][1] = p0;
        grad[k][2] = p1;
    }
    float curl[3][3];   // curl[row][corner] = (anu x grad)[row]
    #pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        curl[0][a] = anu[1] * grad[2][a] - anu[2] * grad[1][a];
        curl[1][a] = anu[2] * grad[0][a] - anu[0] * grad[2][a];
        curl[2][a] = anu[0] * grad[1][a] - anu[1] * grad[0][a];
    }
    // corners in ascending vertex order
    int p[3] = {0, 1, 2};
    if (v[p[1]] < v[p[0]]) { const int t = p[0]; p[0] = p[1]; p[1] = t; }
    if (v[p[2]] < v[p[1]]) { const int t = p[1]; p[1] = p[2]; p[2] = t; }
    if (v[p[1]] < v[p[0]]) { const int t = p[0]; p[0] = p[1]; p[1] = t; }
    #pragma unroll
    for (int d = 0; d < 3; ++d)
        #pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            inner[9 * i + 3 * d + k] = v[p[k]];
            vals[9 * i + 3 * d + k] = curl[d][p[k]];
        }
}

} // namespace

void launch_curl(const MeshDev &m, int32_t *inner, float *vals, cudaStream_t st)
{
    if (m.nt == 0) return;
    curl_kernel<<<ceil_div(m.nt, 128), 128, 0, st>>>(m.coords, m.tris, m.nt, inner, vals);
    BAEMM_LAUNCH_CHECK();
}

void launch_geometry(const MeshDev &m, bool fp64, cudaStream_t st)
{
    if (m.nt == 0) return;
    const int T = 128;
    if (fp64)
        geometry_kernel<double><<<ceil_div(m.nt, T), T, 0, st>>>(m.coords, m.tris, m.nt, m.mid_d, m.nrm_d, m.area_d,
                                                                 m.a3_d, m.diag_d);
    else
        geometry_kernel<float><<<ceil_div(m.nt, T), T, 0, st>>>(m.coords, m.tris, m.nt, m.mid_f, m.nrm_f, m.area_f,
                                                                m.a3_f, m.diag_f);
    BAEMM_LAUNCH_CHECK();
}

void launch_mass_values(const MeshDev &m, bool fp64, cudaStream_t st)
{
    if (m.nv == 0) return;
    const int T = 128;
    if (fp64)
        mass_values_kernel<double><<<ceil_div(m.nv, T), T, 0, st>>>(m.nv, m.tris, m.avt_outer, m.avt_inner, m.area_d,
                                                                    m.mass_outer, m.mass_inner, m.mass_d,
                                                                    m.lumped_d);
    else
        mass_values_kernel<float><<<ceil_div(m.nv, T), T, 0, st>>>(m.nv, m.tris, m.avt_outer, m.avt_inner, m.area_f,
                                                                   m.mass_outer, m.mass_inner, m.mass_f,
                                                                   m.lumped_f);
    BAEMM_LAUNCH_CHECK();
}

} // namespace baemm
