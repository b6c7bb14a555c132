// Dense, matrix-free Helmholtz kernels on the triangle midpoints.
//
//   boundary  C_i = sum_{j != i} A_ij(kappa) B_j     BoundaryOperatorKernel.cl:5-239
//             A_ij = c1 e^{i k r}/r + (c2 (z.mu_j) - c3 (z.nu_i)) (i k r - 1) e^{i k r}/r^3,
//             z = y_j - x_i, r = |z|; c1..c3 already carry 1/(4 pi).
//   near field  the same sum with c3 = 0 at arbitrary points x_i, no pair
//             excluded                               NearFieldOperatorKernel.cl:5-194
//   far field F_i = sum_j (c1 - i k c2 (x_i.mu_j)) e^{-i k x_i.y_j} B_j     FarFieldOperatorKernel.cl:85-133
//   Herglotz  C_i = sum_j (c1 - i k c2 (nu_i.d_j)) e^{-i k x_i.d_j} conj(g_j) HerglotzWaveKernel.cl:85-160
//   incident  plane / radial waves at the midpoints                          IncidentWaveKernel_*.hpp
//
// Plain form (this file): one thread owns one target and a group of COLS
// (<= 16) right-hand-side columns of one wave chunk, accumulating COLS complex
// sums in registers; a CTA of 128 targets streams the sources through shared
// memory in tiles of 64 (midpoint, normal and the tile's RHS rows), so every
// generated kernel entry is reused for COLS complex FMAs.  Padded sources are
// zero (no reading of padded rows, unlike the reference's far-field and
// Herglotz kernels whose mask is always 1, FarFieldOperatorKernel.cl:89).
#include "ops.cuh"

namespace baemm
{

namespace
{

template <class R> struct Prm;
template <> struct Prm<float> { using type = ChunkParamsF; };
template <> struct Prm<double> { using type = ChunkParamsD; };

__device__ __forceinline__ void dsincos(float x, float *s, float *c) { __sincosf(x, s, c); }
__device__ __forceinline__ void dsincos(double x, double *s, double *c) { sincos(x, s, c); }
__device__ __forceinline__ void acc_sincos(float x, float *s, float *c) { sincosf(x, s, c); }
__device__ __forceinline__ void acc_sincos(double x, double *s, double *c) { sincos(x, s, c); }
__device__ __forceinline__ float drsqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ double drsqrt(double x) { return rsqrt(x); }

constexpr int kTargets = 128;   // threads per CTA (one target per thread per pass)
constexpr int kTile = 64;       // sources per shared-memory tile

template <class R, int COLS>
struct Tile
{
    R y[kTile][4];
    R mu[kTile][4];
    cplx<R> B[kTile][COLS];
};

// Stage sources [j0, j0 + kTile) of (pos4, aux4) and COLS columns of rows of
// X (ld) starting at column col0.  Out-of-range sources are zero.
template <class R, int COLS, bool AUX, bool CONJ, class Tx>
__device__ __forceinline__ void stage_tile(Tile<R, COLS> &t, const R *__restrict__ pos4, const R *__restrict__ aux4,
                                           const Tx *__restrict__ X, int64_t ldx, int col0, int j0, int nsrc)
{
    const int tid = threadIdx.x;
    if (tid < kTile)
    {
        const int j = j0 + tid;
        #pragma unroll
        for (int d = 0; d < 4; ++d) t.y[tid][d] = (j < nsrc) ? pos4[4 * (int64_t)j + d] : R(0);
    }
    else if (AUX && tid < 2 * kTile)
    {
        const int s = tid - kTile, j = j0 + s;
        #pragma unroll
        for (int d = 0; d < 4; ++d) t.mu[s][d] = (j < nsrc) ? aux4[4 * (int64_t)j + d] : R(0);
    }
    for (int idx = tid; idx < kTile * COLS; idx += kTargets)
    {
        const int s = idx / COLS, k = idx - s * COLS, j = j0 + s;
        cplx<R> v;
        v.x = R(0);
        v.y = R(0);
        if (j < nsrc)
        {
            const Tx b = X[(int64_t)j * ldx + col0 + k];
            v.x = (R)b.x;
            v.y = CONJ ? -(R)b.y : (R)b.y;
        }
        t.B[s][k] = v;
    }
}

// FP64: 4 CTAs of 128 threads per SM (<= 128 registers; a few bytes spill)
// keep more warps in flight for the FP64 pipe than the 3 CTAs that the 134
// registers of an unbounded build allow: 916 vs 946 ms on the 153,600-triangle
// torus with 64 right-hand sides, identical results.
template <class R, int COLS, bool SL, bool DL, bool ADL>
__global__ void __launch_bounds__(kTargets, std::is_same<R, double>::value ? 4 : 1)
boundary_dense_kernel(DenseTargets<R> tg, const R *__restrict__ mid4, const R *__restrict__ nrm4,
                      const cplx<R> *__restrict__ B, cplx<R> *__restrict__ C,
                      const typename Prm<R>::type *__restrict__ prm, int n, int wc, int wcs)
{
    __shared__ Tile<R, COLS> tile;
    const int i = blockIdx.x * kTargets + threadIdx.x;
    const int iself = tg.self ? tg.off + i : -1;   // the source index excluded for this target (none: -1)
    const int col0 = blockIdx.y * COLS;
    const int ch = col0 / wcs;
    const R kap = prm[ch].kappa;
    const cplx<R> c1 = prm[ch].c[1], c2 = prm[ch].c[2], c3 = prm[ch].c[3];
    R x0 = R(0), x1 = R(0), x2 = R(0), n0 = R(0), n1 = R(0), n2 = R(0);
    if (i < tg.m)
    {
        const R *x = tg.pts4;
        x0 = x[4 * (int64_t)i]; x1 = x[4 * (int64_t)i + 1]; x2 = x[4 * (int64_t)i + 2];
        if (ADL)
        {
            const int64_t gi = (int64_t)tg.off + i;   // the target's triangle (ADL: targets are midpoints)
            n0 = nrm4[4 * gi]; n1 = nrm4[4 * gi + 1]; n2 = nrm4[4 * gi + 2];
        }
    }
    // FP32: two-level sum -- each 64-source tile into fresh accumulators, then
    // into the running total (the error of one long FP32 chain over ~1e5
    // sources would be ~5x larger); FP64: one accumulator.
    constexpr bool kTwoLevel = std::is_same<R, float>::value;
    cplx<R> acc[COLS], tacc[COLS];
    #pragma unroll
    for (int k = 0; k < COLS; ++k) { acc[k].x = R(0); acc[k].y = R(0); }

    for (int j0 = 0; j0 < n; j0 += kTile)
    {
        __syncthreads();
        stage_tile<R, COLS, DL, false>(tile, mid4, nrm4, B, wc, col0, j0, n);
        __syncthreads();
        const int smax = min(kTile, n - j0);
        #pragma unroll
        for (int k = 0; k < COLS; ++k)
        {
            tacc[k].x = R(0);
            tacc[k].y = R(0);
        }
        cplx<R>(&sum)[COLS] = kTwoLevel ? tacc : acc;
        #pragma unroll 2
        for (int s = 0; s < smax; ++s)
        {
            const R zx = tile.y[s][0] - x0, zy = tile.y[s][1] - x1, zz = tile.y[s][2] - x2;
            const R r2 = zx * zx + zy * zy + zz * zz;
            const R rinv = (j0 + s == iself) ? R(0) : drsqrt(r2);
            const R r = r2 * rinv;
            const R kr = kap * r;
            R sn, cs;
            dsincos(kr, &sn, &cs);
            cplx<R> A;
            A.x = R(0);
            A.y = R(0);
            if (SL)
            {
                const R er = cs * rinv, ei = sn * rinv;
                A.x = c1.x * er - c1.y * ei;
                A.y = c1.x * ei + c1.y * er;
            }
            if (DL || ADL)
            {
                const R r3 = rinv * rinv * rinv;
                const R g0 = -(kr * sn + cs) * r3;
                const R g1 = (kr * cs - sn) * r3;
                R fx = R(0), fy = R(0);
                if (DL)
                {
                    const R dm = zx * tile.mu[s][0] + zy * tile.mu[s][1] + zz * tile.mu[s][2];
                    fx += c2.x * dm;
                    fy += c2.y * dm;
                }
                if (ADL)
                {
                    const R dn = zx * n0 + zy * n1 + zz * n2;
                    fx -= c3.x * dn;
                    fy -= c3.y * dn;
                }
                A.x += fx * g0 - fy * g1;
                A.y += fx * g1 + fy * g0;
            }
            #pragma unroll
            for (int k = 0; k < COLS; ++k) cfma(sum[k], A, tile.B[s][k]);
        }
        if (kTwoLevel)
        {
            #pragma unroll
            for (int k = 0; k < COLS; ++k)
            {
                acc[k].x += tacc[k].x;
                acc[k].y += tacc[k].y;
            }
        }
    }
    if (i < tg.m)
    {
        cplx<R> *out = &C[(int64_t)i * wc + col0];
        #pragma unroll
        for (int k = 0; k < COLS; ++k) out[k] = acc[k];
    }
}

// Plain FP32 form with packed FP32x2 arithmetic (sm_100 FFMA2).  Each thread
// owns TT targets (i, i + 128, ...) and the 16 columns of one wave chunk.  A
// complex MAC  c += a b  is two packed FMAs:
//     c += (a.re, a.re) * (b.re, b.im)
//     c += (a.im, a.im) * (-b.im, b.re)
// so the tile stages every RHS row twice, as b and as the swapped, negated
// (-b.im, b.re).  Half the issue slots of the scalar form for the same FMA-pipe
// work; TT > 1 shares every staged RHS row between TT targets.
constexpr int kPackedCols = 16;

struct PackedTile
{
    float4 y[kTile];
    float4 mu[kTile];
    float2 B[kTile][kPackedCols];
    float2 Bw[kTile][kPackedCols];
};

template <int TT, bool SL, bool DL, bool ADL>
__global__ void __launch_bounds__(kTargets, TT == 1 ? 4 : 3)
boundary_packed_kernel(DenseTargets<float> tg, const float *__restrict__ mid4, const float *__restrict__ nrm4,
                       const float2 *__restrict__ B, float2 *__restrict__ C, const ChunkParamsF *__restrict__ prm,
                       int n, int wc, int wcs)
{
    __shared__ PackedTile tile;
    const int col0 = blockIdx.y * kPackedCols;
    const int ch = col0 / wcs;
    const float kap = prm[ch].kappa;
    const float2 c1 = prm[ch].c[1], c2 = prm[ch].c[2], c3 = prm[ch].c[3];
    int ti[TT], tself[TT];
    float3 x[TT], nu[TT];
    #pragma unroll
    for (int t = 0; t < TT; ++t)
    {
        ti[t] = blockIdx.x * (kTargets * TT) + t * kTargets + threadIdx.x;
        tself[t] = tg.self ? tg.off + ti[t] : -1;
        x[t] = make_float3(0.f, 0.f, 0.f);
        nu[t] = make_float3(0.f, 0.f, 0.f);
        if (ti[t] < tg.m)
        {
            const float4 m = reinterpret_cast<const float4 *>(tg.pts4)[ti[t]];
            x[t] = make_float3(m.x, m.y, m.z);
            if (ADL)
            {
                const float4 q = reinterpret_cast<const float4 *>(nrm4)[tg.off + ti[t]];
                nu[t] = make_float3(q.x, q.y, q.z);
            }
        }
    }
    float2 acc[TT][kPackedCols], tacc[TT][kPackedCols];   // running total, this tile's sum (two-level sum)
    #pragma unroll
    for (int t = 0; t < TT; ++t)
        #pragma unroll
        for (int k = 0; k < kPackedCols; ++k) acc[t][k] = make_float2(0.f, 0.f);

    for (int j0 = 0; j0 < n; j0 += kTile)
    {
        __syncthreads();
        {
            const int tid = threadIdx.x;
            if (tid < kTile)
            {
                const int j = j0 + tid;
                tile.y[tid] = (j < n) ? reinterpret_cast<const float4 *>(mid4)[j] : make_float4(0.f, 0.f, 0.f, 0.f);
            }
            else if (DL && tid < 2 * kTile)
            {
                const int sidx = tid - kTile, j = j0 + sidx;
                tile.mu[sidx] = (j < n) ? reinterpret_cast<const float4 *>(nrm4)[j] : make_float4(0.f, 0.f, 0.f, 0.f);
            }
            for (int idx = tid; idx < kTile * kPackedCols; idx += kTargets)
            {
                const int sidx = idx / kPackedCols, k = idx % kPackedCols, j = j0 + sidx;
                const float2 b = (j < n) ? B[(int64_t)j * wc + col0 + k] : make_float2(0.f, 0.f);
                tile.B[sidx][k] = b;
                tile.Bw[sidx][k] = make_float2(-b.y, b.x);
            }
        }
        __syncthreads();
        const int smax = min(kTile, n - j0);
        #pragma unroll
        for (int t = 0; t < TT; ++t)
            #pragma unroll
            for (int k = 0; k < kPackedCols; ++k) tacc[t][k] = make_float2(0.f, 0.f);
        for (int s = 0; s < smax; ++s)
        {
            const float4 yv = tile.y[s];
            float4 mv = make_float4(0.f, 0.f, 0.f, 0.f);
            if (DL) mv = tile.mu[s];
            float2 Ar[TT], Ai[TT];
            #pragma unroll
            for (int t = 0; t < TT; ++t)
            {
                const float zx = yv.x - x[t].x, zy = yv.y - x[t].y, zz = yv.z - x[t].z;
                const float r2 = zx * zx + zy * zy + zz * zz;
                const float rinv = (j0 + s == tself[t]) ? 0.f : rsqrtf(r2);
                const float r = r2 * rinv;
                const float kr = kap * r;
                float sn, cs;
                __sincosf(kr, &sn, &cs);
                float ax = 0.f, ay = 0.f;
                if (SL)
                {
                    const float er = cs * rinv, ei = sn * rinv;
                    ax = c1.x * er - c1.y * ei;
                    ay = c1.x * ei + c1.y * er;
                }
                if (DL || ADL)
                {
                    const float r3 = rinv * rinv * rinv;
                    const float g0 = -(kr * sn + cs) * r3;
                    const float g1 = (kr * cs - sn) * r3;
                    float fx = 0.f, fy = 0.f;
                    if (DL)
                    {
                        const float dm = zx * mv.x + zy * mv.y + zz * mv.z;
                        fx += c2.x * dm;
                        fy += c2.y * dm;
                    }
                    if (ADL)
                    {
                        const float dn = zx * nu[t].x + zy * nu[t].y + zz * nu[t].z;
                        fx -= c3.x * dn;
                        fy -= c3.y * dn;
                    }
                    ax += fx * g0 - fy * g1;
                    ay += fx * g1 + fy * g0;
                }
                Ar[t] = make_float2(ax, ax);
                Ai[t] = make_float2(ay, ay);
            }
            #pragma unroll
            for (int k = 0; k < kPackedCols; ++k)
            {
                const float2 b = tile.B[s][k], bw = tile.Bw[s][k];
                #pragma unroll
                for (int t = 0; t < TT; ++t)
                {
                    tacc[t][k] = __ffma2_rn(Ar[t], b, tacc[t][k]);
                    tacc[t][k] = __ffma2_rn(Ai[t], bw, tacc[t][k]);
                }
            }
        }
        #pragma unroll
        for (int t = 0; t < TT; ++t)
            #pragma unroll
            for (int k = 0; k < kPackedCols; ++k) acc[t][k] = __fadd2_rn(acc[t][k], tacc[t][k]);
    }
    #pragma unroll
    for (int t = 0; t < TT; ++t)
        if (ti[t] < tg.m)
        {
            float4 *out = reinterpret_cast<float4 *>(&C[(int64_t)ti[t] * wc + col0]);
            #pragma unroll
            for (int k = 0; k < kPackedCols; k += 2)
                out[k / 2] = make_float4(acc[t][k].x, acc[t][k].y, acc[t][k + 1].x, acc[t][k + 1].y);
        }
}

template <class R, int COLS, bool SL, bool DL>
__global__ void __launch_bounds__(kTargets)
farfield_partial_kernel(const R *__restrict__ meas4, const R *__restrict__ mid4, const R *__restrict__ nrm4,
                        const cplx<R> *__restrict__ B, const typename Prm<R>::type *__restrict__ prm, int m, int n,
                        int wc, int wcs, int per_split, cplx<R> *__restrict__ partial)
{
    __shared__ Tile<R, COLS> tile;
    const int i = blockIdx.x * kTargets + threadIdx.x;
    const int col0 = blockIdx.y * COLS;
    const int split = blockIdx.z;
    const int ch = col0 / wcs;
    const R kap = prm[ch].kappa;
    const cplx<R> c1 = prm[ch].c[1], c2 = prm[ch].c[2];
    R x0 = R(0), x1 = R(0), x2 = R(0);
    if (i < m) { x0 = meas4[4 * (int64_t)i]; x1 = meas4[4 * (int64_t)i + 1]; x2 = meas4[4 * (int64_t)i + 2]; }
    cplx<R> acc[COLS];
    #pragma unroll
    for (int k = 0; k < COLS; ++k) { acc[k].x = R(0); acc[k].y = R(0); }
    const int jb = split * per_split, je = min(n, jb + per_split);
    for (int j0 = jb; j0 < je; j0 += kTile)
    {
        __syncthreads();
        stage_tile<R, COLS, DL, false>(tile, mid4, nrm4, B, wc, col0, j0, je);
        __syncthreads();
        const int smax = min(kTile, je - j0);
        for (int s = 0; s < smax; ++s)
        {
            const R th = kap * (tile.y[s][0] * x0 + tile.y[s][1] * x1 + tile.y[s][2] * x2);
            R sn, cs;
            dsincos(th, &sn, &cs);
            // e = exp(-i th); A = (c1 + c2 (-i k mu.x)) e
            cplx<R> f;
            f.x = SL ? c1.x : R(0);
            f.y = SL ? c1.y : R(0);
            if (DL)
            {
                const R dk = kap * (tile.mu[s][0] * x0 + tile.mu[s][1] * x1 + tile.mu[s][2] * x2);
                f.x += c2.y * dk;
                f.y -= c2.x * dk;
            }
            cplx<R> A;
            A.x = f.x * cs + f.y * sn;
            A.y = f.y * cs - f.x * sn;
            #pragma unroll
            for (int k = 0; k < COLS; ++k) cfma(acc[k], A, tile.B[s][k]);
        }
    }
    if (i < m)
    {
        cplx<R> *out = &partial[((int64_t)split * m + i) * wc + col0];
        #pragma unroll
        for (int k = 0; k < COLS; ++k) out[k] = acc[k];
    }
}

template <class R>
__global__ void farfield_reduce_kernel(const cplx<R> *__restrict__ partial, int splits, int m, int wc, double2 alpha,
                                       double2 beta, double2 *__restrict__ Cout, int64_t ldC)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)m * wc) return;
    const int64_t i = idx / wc;
    const int k = (int)(idx - i * wc);
    double sx = 0.0, sy = 0.0;
    for (int s = 0; s < splits; ++s)
    {
        const cplx<R> p = partial[((int64_t)s * m + i) * wc + k];
        sx += (double)p.x;
        sy += (double)p.y;
    }
    double2 o = make_double2(alpha.x * sx - alpha.y * sy, alpha.x * sy + alpha.y * sx);
    double2 *c = &Cout[i * ldC + k];
    if (beta.x != 0.0 || beta.y != 0.0)
    {
        const double2 b = *c;
        o.x += beta.x * b.x - beta.y * b.y;
        o.y += beta.x * b.y + beta.y * b.x;
    }
    *c = o;
}

template <class R, int COLS, bool SL, bool DL>
__global__ void __launch_bounds__(kTargets)
herglotz_kernel(const R *__restrict__ mid4, const R *__restrict__ nrm4, const R *__restrict__ meas4,
                const double2 *__restrict__ g, int64_t ldg, const typename Prm<R>::type *__restrict__ prm, int n, int m,
                int wc, int wcs, cplx<R> *__restrict__ C)
{
    __shared__ Tile<R, COLS> tile;
    const int i = blockIdx.x * kTargets + threadIdx.x;
    const int col0 = blockIdx.y * COLS;
    const int ch = col0 / wcs;
    const R kap = prm[ch].kappa;
    const cplx<R> c1 = prm[ch].c[1], c2 = prm[ch].c[2];
    R x0 = R(0), x1 = R(0), x2 = R(0), n0 = R(0), n1 = R(0), n2 = R(0);
    if (i < n)
    {
        x0 = mid4[4 * (int64_t)i]; x1 = mid4[4 * (int64_t)i + 1]; x2 = mid4[4 * (int64_t)i + 2];
        n0 = nrm4[4 * (int64_t)i]; n1 = nrm4[4 * (int64_t)i + 1]; n2 = nrm4[4 * (int64_t)i + 2];
    }
    cplx<R> acc[COLS];
    #pragma unroll
    for (int k = 0; k < COLS; ++k) { acc[k].x = R(0); acc[k].y = R(0); }
    for (int j0 = 0; j0 < m; j0 += kTile)
    {
        __syncthreads();
        stage_tile<R, COLS, false, true>(tile, meas4, nullptr, g, ldg, col0, j0, m);
        __syncthreads();
        const int smax = min(kTile, m - j0);
        for (int s = 0; s < smax; ++s)
        {
            const R th = kap * (tile.y[s][0] * x0 + tile.y[s][1] * x1 + tile.y[s][2] * x2);
            R sn, cs;
            dsincos(th, &sn, &cs);
            cplx<R> f;
            f.x = SL ? c1.x : R(0);
            f.y = SL ? c1.y : R(0);
            if (DL)
            {
                const R dk = kap * (n0 * tile.y[s][0] + n1 * tile.y[s][1] + n2 * tile.y[s][2]);
                f.x += c2.y * dk;
                f.y -= c2.x * dk;
            }
            cplx<R> A;
            A.x = f.x * cs + f.y * sn;
            A.y = f.y * cs - f.x * sn;
            #pragma unroll
            for (int k = 0; k < COLS; ++k) cfma(acc[k], A, tile.B[s][k]);
        }
    }
    if (i < n)
    {
        cplx<R> *out = &C[(int64_t)i * wc + col0];
        #pragma unroll
        for (int k = 0; k < COLS; ++k) out[k] = acc[k];
    }
}

template <class R>
__global__ void incident_kernel(int64_t nt, const R *__restrict__ mid4, const R *__restrict__ nrm4,
                                const typename Prm<R>::type *__restrict__ prm, int wc, int wcs,
                                const R *__restrict__ dirs, int type, cplx<R> *__restrict__ C)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nt * wc) return;
    const int64_t i = idx / wc;
    const int k = (int)(idx - i * wc);
    const int ch = k / wcs, j = k - ch * wcs;
    const R K = prm[ch].kappa;
    const cplx<R> c1 = prm[ch].c[1], c2 = prm[ch].c[2];
    const R m0 = mid4[4 * i], m1 = mid4[4 * i + 1], m2 = mid4[4 * i + 2];
    const R q0 = nrm4[4 * i], q1 = nrm4[4 * i + 1], q2 = nrm4[4 * i + 2];
    const R d0 = dirs[3 * j], d1 = dirs[3 * j + 1], d2 = dirs[3 * j + 2];
    cplx<R> f, e;
    if (type == BAEMM_WAVE_RADIAL)
    {
        // IncidentWaveKernel_Radial.hpp:28-51
        const R oofp = R(1) / (R(2) * (R(2) * R(3.14159265358979323846)));
        const R dl0 = m0 - d0, dl1 = m1 - d1, dl2 = m2 - d2;
        const R R2 = dl0 * dl0 + dl1 * dl1 + dl2 * dl2;
        const R Rr = sqrt(R2), oR = R(1) / Rr, oR2 = R(1) / R2;
        const R dn = q0 * dl0 + q1 * dl1 + q2 * dl2;
        const R A = oofp * oR;
        cplx<R> Bc;
        Bc.x = -dn * oR2;
        Bc.y = dn * K * oR;
        // factor = c1 A + c2 A B
        f.x = c1.x * A + A * (c2.x * Bc.x - c2.y * Bc.y);
        f.y = c1.y * A + A * (c2.x * Bc.y + c2.y * Bc.x);
        R s, c;
        acc_sincos(K * Rr, &s, &c);
        e.x = c;
        e.y = s;
    }
    else
    {
        // IncidentWaveKernel_Plane.hpp:208-227: (c1 + c2 i k <d,n>) e^{i k <d,x>}
        const R dm = m0 * d0 + m1 * d1 + m2 * d2;
        const R dn = q0 * d0 + q1 * d1 + q2 * d2;
        f.x = c1.x - c2.y * (K * dn);
        f.y = c1.y + c2.x * (K * dn);
        R s, c;
        acc_sincos(K * dm, &s, &c);
        e.x = c;
        e.y = s;
    }
    C[idx] = cmul(f, e);
}

// Evaluation points (m x 3 doubles) as m x 4 reals, w = 0
// (ApplyNearFieldOperators.hpp:96-107 pads them the same way).
template <class R>
__global__ void pack_points_kernel(int64_t m, const double *__restrict__ pts3, R *__restrict__ pts4)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    pts4[4 * i + 0] = (R)pts3[3 * i + 0];
    pts4[4 * i + 1] = (R)pts3[3 * i + 1];
    pts4[4 * i + 2] = (R)pts3[3 * i + 2];
    pts4[4 * i + 3] = R(0);
}

// ---- dispatch helpers -----------------------------------------------------------
template <class R, int COLS>
void boundary_cols(const OpFlags &f, dim3 grid, cudaStream_t st, DenseTargets<R> tg, const R *mid, const R *nrm,
                   const cplx<R> *B, cplx<R> *C, const typename Prm<R>::type *p, int n, int wc, int wcs)
{
    const int code = (f.sl() ? 1 : 0) | (f.dl() ? 2 : 0) | (f.adl() ? 4 : 0);
#define BAEMM_BK(SL, DL, ADL) boundary_dense_kernel<R, COLS, SL, DL, ADL><<<grid, kTargets, 0, st>>>(tg, mid, nrm, B, C, p, n, wc, wcs)
    switch (code)
    {
        case 1: BAEMM_BK(true, false, false); break;
        case 2: BAEMM_BK(false, true, false); break;
        case 3: BAEMM_BK(true, true, false); break;
        case 4: BAEMM_BK(false, false, true); break;
        case 5: BAEMM_BK(true, false, true); break;
        case 6: BAEMM_BK(false, true, true); break;
        case 7: BAEMM_BK(true, true, true); break;
        default: break;
    }
#undef BAEMM_BK
}

template <class R, int COLS>
void farfield_cols(const OpFlags &f, dim3 grid, cudaStream_t st, const R *meas, const R *mid, const R *nrm,
                   const cplx<R> *B, const typename Prm<R>::type *p, int m, int n, int wc, int wcs, int per_split,
                   cplx<R> *partial)
{
    if (f.sl() && f.dl())
        farfield_partial_kernel<R, COLS, true, true><<<grid, kTargets, 0, st>>>(meas, mid, nrm, B, p, m, n, wc, wcs, per_split, partial);
    else if (f.sl())
        farfield_partial_kernel<R, COLS, true, false><<<grid, kTargets, 0, st>>>(meas, mid, nrm, B, p, m, n, wc, wcs, per_split, partial);
    else
        farfield_partial_kernel<R, COLS, false, true><<<grid, kTargets, 0, st>>>(meas, mid, nrm, B, p, m, n, wc, wcs, per_split, partial);
}

template <class R, int COLS>
void herglotz_cols(const OpFlags &f, dim3 grid, cudaStream_t st, const R *mid, const R *nrm, const R *meas,
                   const double2 *g, int64_t ldg, const typename Prm<R>::type *p, int n, int m, int wc, int wcs,
                   cplx<R> *C)
{
    if (f.sl() && f.dl())
        herglotz_kernel<R, COLS, true, true><<<grid, kTargets, 0, st>>>(mid, nrm, meas, g, ldg, p, n, m, wc, wcs, C);
    else if (f.sl())
        herglotz_kernel<R, COLS, true, false><<<grid, kTargets, 0, st>>>(mid, nrm, meas, g, ldg, p, n, m, wc, wcs, C);
    else
        herglotz_kernel<R, COLS, false, true><<<grid, kTargets, 0, st>>>(mid, nrm, meas, g, ldg, p, n, m, wc, wcs, C);
}

template <class R> const R *geo_mid(const MeshDev &m);
template <> const float *geo_mid<float>(const MeshDev &m) { return m.mid_f; }
template <> const double *geo_mid<double>(const MeshDev &m) { return m.mid_d; }
template <class R> const R *geo_nrm(const MeshDev &m);
template <> const float *geo_nrm<float>(const MeshDev &m) { return m.nrm_f; }
template <> const double *geo_nrm<double>(const MeshDev &m) { return m.nrm_d; }
template <class R> const R *geo_meas(const MeshDev &m);
template <> const float *geo_meas<float>(const MeshDev &m) { return m.meas_f; }
template <> const double *geo_meas<double>(const MeshDev &m) { return m.meas_d; }

inline int cols_for(int wcs) { return wcs < 16 ? wcs : 16; }

template <int TT>
void packed_dispatch(int code, DenseTargets<float> tg, int n, int wc, int wcs, const float *mid, const float *nrm,
                     const float2 *B, float2 *C, const ChunkParamsF *p, cudaStream_t st)
{
    dim3 grid(ceil_div(tg.m, kTargets * TT), wc / kPackedCols);
#define BAEMM_PK(SL, DL, ADL) boundary_packed_kernel<TT, SL, DL, ADL><<<grid, kTargets, 0, st>>>(tg, mid, nrm, B, C, p, n, wc, wcs)
    switch (code)
    {
        case 1: BAEMM_PK(true, false, false); break;
        case 2: BAEMM_PK(false, true, false); break;
        case 3: BAEMM_PK(true, true, false); break;
        case 4: BAEMM_PK(false, false, true); break;
        case 5: BAEMM_PK(true, false, true); break;
        case 6: BAEMM_PK(false, true, true); break;
        case 7: BAEMM_PK(true, true, true); break;
        default: break;
    }
#undef BAEMM_PK
}

// Ctri (tg.m x wc) = K Btri over all nt sources for the targets tg.
template <class R>
void dense_dispatch(const MeshDev &m, const OpFlags &f, const void *chunk_params, int wc, int wcs,
                    DenseTargets<R> tg, const cplx<R> *Btri, cplx<R> *Ctri, cudaStream_t st, int variant)
{
    if (!f.any_layer() || m.nt == 0 || tg.m == 0) return;
    const int n = (int)m.nt;
    const int cols = cols_for(wcs);
    dim3 grid(ceil_div(tg.m, kTargets), wc / cols);
    const auto *p = static_cast<const typename Prm<R>::type *>(chunk_params);
    const R *mid = geo_mid<R>(m), *nrm = geo_nrm<R>(m);
    if constexpr (std::is_same<R, float>::value)
    {
        if (cols == kPackedCols && variant > 0)
        {
            const int code = (f.sl() ? 1 : 0) | (f.dl() ? 2 : 0) | (f.adl() ? 4 : 0);
            if (variant == 2) packed_dispatch<2>(code, tg, n, wc, wcs, mid, nrm, Btri, Ctri, p, st);
            else packed_dispatch<1>(code, tg, n, wc, wcs, mid, nrm, Btri, Ctri, p, st);
            BAEMM_LAUNCH_CHECK();
            return;
        }
    }
    switch (cols)
    {
        case 1: boundary_cols<R, 1>(f, grid, st, tg, mid, nrm, Btri, Ctri, p, n, wc, wcs); break;
        case 2: boundary_cols<R, 2>(f, grid, st, tg, mid, nrm, Btri, Ctri, p, n, wc, wcs); break;
        case 4: boundary_cols<R, 4>(f, grid, st, tg, mid, nrm, Btri, Ctri, p, n, wc, wcs); break;
        case 8: boundary_cols<R, 8>(f, grid, st, tg, mid, nrm, Btri, Ctri, p, n, wc, wcs); break;
        case 16: boundary_cols<R, 16>(f, grid, st, tg, mid, nrm, Btri, Ctri, p, n, wc, wcs); break;
        default: throw Error(BAEMM_ERR_SIZE, "wave_chunk_size must be a power of two <= 64");
    }
    BAEMM_LAUNCH_CHECK();
}

} // namespace

template <class R>
void launch_boundary_dense(const MeshDev &m, const OpFlags &f, const void *chunk_params, int wc, int wcs,
                           const cplx<R> *Btri, cplx<R> *Ctri, cudaStream_t st, int variant, int64_t row_begin,
                           int64_t row_end)
{
    const int64_t r0 = std::max<int64_t>(0, row_begin), r1 = row_end < 0 ? m.nt : std::min<int64_t>(row_end, m.nt);
    if (r1 <= r0) return;
    dense_dispatch<R>(m, f, chunk_params, wc, wcs, DenseTargets<R>{geo_mid<R>(m) + 4 * r0, (int)(r1 - r0), 1, (int)r0},
                      Btri, Ctri + r0 * wc, st, variant);
}

template <class R>
void launch_nearfield_dense(const MeshDev &m, const OpFlags &f, const void *chunk_params, int wc, int wcs,
                            const R *pts4, int64_t npts, const cplx<R> *Btri, cplx<R> *Cpts, cudaStream_t st,
                            int variant)
{
    BAEMM_REQUIRE(!f.adl() && !f.mass(), BAEMM_ERR_ARG, "near field: single and double layer only");
    BAEMM_REQUIRE(npts <= INT32_MAX, BAEMM_ERR_SIZE, "too many evaluation points");
    dense_dispatch<R>(m, f, chunk_params, wc, wcs, DenseTargets<R>{pts4, (int)npts, 0, 0}, Btri, Cpts, st, variant);
}

template <class R>
void launch_pack_points(int64_t m, const double *pts3, R *pts4, cudaStream_t st)
{
    if (m == 0) return;
    pack_points_kernel<R><<<ceil_div(m, 256), 256, 0, st>>>(m, pts3, pts4);
    BAEMM_LAUNCH_CHECK();
}

static int farfield_splits(const MeshDev &m, int wc, int wcs)
{
    const int cols = cols_for(wcs);
    const int ctas = ceil_div(m.nm, kTargets) * (wc / cols);
    int splits = ceil_div(4 * 148, ctas);
    const int max_splits = ceil_div(m.nt, kTile);
    if (splits > max_splits) splits = max_splits;
    if (splits < 1) splits = 1;
    return splits;
}

size_t farfield_partial_elems(const MeshDev &m, int wc, int wcs)
{
    return (size_t)farfield_splits(m, wc, wcs) * (size_t)m.nm * (size_t)wc;
}

template <class R>
void launch_farfield(const MeshDev &m, const OpFlags &f, const void *chunk_params, int wc, int wcs,
                     const cplx<R> *Btri, cplx<R> *partial, size_t partial_cap, double2 alpha, double2 beta,
                     double2 *Cout, int64_t ldC, cudaStream_t st)
{
    if (!(f.sl() || f.dl()) || m.nm == 0) return;
    const int splits = farfield_splits(m, wc, wcs);
    BAEMM_REQUIRE((size_t)splits * m.nm * wc <= partial_cap, BAEMM_ERR_SIZE, "far-field partial buffer too small");
    const int per_split = ceil_div(ceil_div(m.nt, splits), kTile) * kTile;
    const int cols = cols_for(wcs);
    dim3 grid(ceil_div(m.nm, kTargets), wc / cols, splits);
    const auto *p = static_cast<const typename Prm<R>::type *>(chunk_params);
    const R *mid = geo_mid<R>(m), *nrm = geo_nrm<R>(m), *meas = geo_meas<R>(m);
    const int mm = (int)m.nm, n = (int)m.nt;
    switch (cols)
    {
        case 1: farfield_cols<R, 1>(f, grid, st, meas, mid, nrm, Btri, p, mm, n, wc, wcs, per_split, partial); break;
        case 2: farfield_cols<R, 2>(f, grid, st, meas, mid, nrm, Btri, p, mm, n, wc, wcs, per_split, partial); break;
        case 4: farfield_cols<R, 4>(f, grid, st, meas, mid, nrm, Btri, p, mm, n, wc, wcs, per_split, partial); break;
        case 8: farfield_cols<R, 8>(f, grid, st, meas, mid, nrm, Btri, p, mm, n, wc, wcs, per_split, partial); break;
        case 16: farfield_cols<R, 16>(f, grid, st, meas, mid, nrm, Btri, p, mm, n, wc, wcs, per_split, partial); break;
        default: throw Error(BAEMM_ERR_SIZE, "wave_chunk_size must be a power of two <= 64");
    }
    BAEMM_LAUNCH_CHECK();
    farfield_reduce_kernel<R><<<ceil_div((int64_t)mm * wc, 256), 256, 0, st>>>(partial, splits, mm, wc, alpha, beta,
                                                                               Cout, ldC);
    BAEMM_LAUNCH_CHECK();
}

template <class R>
void launch_herglotz(const MeshDev &m, const OpFlags &f, const void *chunk_params, int wc, int wcs, const double2 *g,
                     int64_t ldg, cplx<R> *Ctri, cudaStream_t st)
{
    if (!(f.sl() || f.dl()) || m.nt == 0) return;
    const int cols = cols_for(wcs);
    dim3 grid(ceil_div(m.nt, kTargets), wc / cols);
    const auto *p = static_cast<const typename Prm<R>::type *>(chunk_params);
    const R *mid = geo_mid<R>(m), *nrm = geo_nrm<R>(m), *meas = geo_meas<R>(m);
    const int n = (int)m.nt, mm = (int)m.nm;
    switch (cols)
    {
        case 1: herglotz_cols<R, 1>(f, grid, st, mid, nrm, meas, g, ldg, p, n, mm, wc, wcs, Ctri); break;
        case 2: herglotz_cols<R, 2>(f, grid, st, mid, nrm, meas, g, ldg, p, n, mm, wc, wcs, Ctri); break;
        case 4: herglotz_cols<R, 4>(f, grid, st, mid, nrm, meas, g, ldg, p, n, mm, wc, wcs, Ctri); break;
        case 8: herglotz_cols<R, 8>(f, grid, st, mid, nrm, meas, g, ldg, p, n, mm, wc, wcs, Ctri); break;
        case 16: herglotz_cols<R, 16>(f, grid, st, mid, nrm, meas, g, ldg, p, n, mm, wc, wcs, Ctri); break;
        default: throw Error(BAEMM_ERR_SIZE, "wave_chunk_size must be a power of two <= 64");
    }
    BAEMM_LAUNCH_CHECK();
}

template <class R>
void launch_incident(const MeshDev &m, const void *chunk_params, int wc, int wcs, const R *dirs, int type,
                     cplx<R> *Ctri, cudaStream_t st)
{
    const int64_t n = m.nt * wc;
    if (n == 0) return;
    incident_kernel<R><<<ceil_div(n, 256), 256, 0, st>>>(m.nt, geo_mid<R>(m), geo_nrm<R>(m),
                                                         static_cast<const typename Prm<R>::type *>(chunk_params), wc,
                                                         wcs, dirs, type, Ctri);
    BAEMM_LAUNCH_CHECK();
}

template void launch_boundary_dense<float>(const MeshDev &, const OpFlags &, const void *, int, int, const float2 *,
                                           float2 *, cudaStream_t, int, int64_t, int64_t);
template void launch_pack_points<float>(int64_t, const double *, float *, cudaStream_t);
template void launch_pack_points<double>(int64_t, const double *, double *, cudaStream_t);
template void launch_nearfield_dense<float>(const MeshDev &, const OpFlags &, const void *, int, int, const float *,
                                            int64_t, const float2 *, float2 *, cudaStream_t, int);
template void launch_nearfield_dense<double>(const MeshDev &, const OpFlags &, const void *, int, int, const double *,
                                             int64_t, const double2 *, double2 *, cudaStream_t, int);
template void launch_boundary_dense<double>(const MeshDev &, const OpFlags &, const void *, int, int, const double2 *,
                                            double2 *, cudaStream_t, int, int64_t, int64_t);
template void launch_farfield<float>(const MeshDev &, const OpFlags &, const void *, int, int, const float2 *, float2 *,
                                     size_t, double2, double2, double2 *, int64_t, cudaStream_t);
template void launch_farfield<double>(const MeshDev &, const OpFlags &, const void *, int, int, const double2 *,
                                      double2 *, size_t, double2, double2, double2 *, int64_t, cudaStream_t);
template void launch_herglotz<float>(const MeshDev &, const OpFlags &, const void *, int, int, const double2 *, int64_t,
                                     float2 *, cudaStream_t);
template void launch_herglotz<double>(const MeshDev &, const OpFlags &, const void *, int, int, const double2 *,
                                      int64_t, double2 *, cudaStream_t);
template void launch_incident<float>(const MeshDev &, const void *, int, int, const float *, int, float2 *,
                                     cudaStream_t);
template void launch_incident<double>(const MeshDev &, const void *, int, int, const double *, int, double2 *,
                                      cudaStream_t);

} // namespace baemm
