// Device CG (mass inverse) and batched GMRES.  See krylov.cuh for the
// algorithm definitions.  Column reductions are two-level and deterministic:
// each block reduces its row range in shared memory and writes one partial
// per column; a single-block finalize kernel sums the partials in block
// order.
#include "krylov.cuh"

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

namespace baemm
{
namespace
{

constexpr int RT = 256;          // threads per reduction block
constexpr int kTargetBlocks = 592;   // reduction blocks over the rows (4 per SM: the Gram-Schmidt dots ran 117 -> 72 us at level 6 with twice 296)

struct Layout
{
    int cp = 1, rp = 1, nchunk = 1, nblk = 1;
    int64_t rows_per_block = 1;
};

Layout make_layout(int64_t n, int c)
{
    Layout L;
    L.cp = std::min(c, RT);
    L.rp = RT / L.cp;
    L.nchunk = ceil_div(c, L.cp);
    int64_t rpb = std::max<int64_t>(L.rp, (n + kTargetBlocks - 1) / kTargetBlocks);
    rpb = ((rpb + L.rp - 1) / L.rp) * L.rp;
    L.rows_per_block = rpb;
    L.nblk = std::max(1, ceil_div(n, rpb));
    return L;
}

// ---- scalar helpers for S = double / double2 ---------------------------------
__device__ __forceinline__ double re(double a) { return a; }
__device__ __forceinline__ double re(double2 a) { return a.x; }
__device__ __forceinline__ double im(double) { return 0.0; }
__device__ __forceinline__ double im(double2 a) { return a.y; }
template <class S> __device__ __forceinline__ S mkS(double x, double y);
template <> __device__ __forceinline__ double mkS<double>(double x, double) { return x; }
template <> __device__ __forceinline__ double2 mkS<double2>(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ double Sabs2(double a) { return a * a; }
__device__ __forceinline__ double Sabs2(double2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ double Smul(double a, double b) { return a * b; }
__device__ __forceinline__ double2 Smul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double Sconj(double a) { return a; }
__device__ __forceinline__ double2 Sconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double Sadd(double a, double b) { return a + b; }
__device__ __forceinline__ double2 Sadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double Ssub(double a, double b) { return a - b; }
__device__ __forceinline__ double2 Ssub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double Sscale(double a, double s) { return a * s; }
__device__ __forceinline__ double2 Sscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double Sdiv(double a, double b) { return a / b; }
__device__ __forceinline__ double2 Sdiv(double2 a, double2 b)
{
    const double d = b.x * b.x + b.y * b.y;
    return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
template <class S> constexpr int kWords = sizeof(S) / sizeof(double);

// Block reduction of one value per (row-lane, column) into partial[out_index].
__device__ __forceinline__ void block_reduce_store(double v, double *sm, int tr, int tc, int cp, int rp, bool active,
                                                   double *dst)
{
    sm[threadIdx.x] = active ? v : 0.0;
    __syncthreads();
    if (tr == 0 && active)
    {
        double s = 0.0;
        for (int q = 0; q < rp; ++q) s += sm[q * cp + tc];
        *dst = s;
    }
    __syncthreads();
}

// ============================== CG =============================================
// col_ layout: [0,c) rz  [c,2c) bn  [2c,3c) alpha  [3c,4c) beta ; flags_: [0] done [1] iters [2..) conv



// Sum of one column of the per-block partial sums, partial[q * ld + off] over
// q < nblk, by one warp: lane l takes q = l, l + 32, ... into four running
// sums (q / 32 mod 4), so four loads per lane are in flight instead of one
// dependent chain of round trips; the four are added in a fixed order and a
// shuffle tree adds the lanes in a fixed order, every lane returning lane 0's
// total (so the result does not depend on timing).  The finalize kernels
// below give each column its own warp, instead of one thread summing all
// nblk values in turn.
__device__ __forceinline__ double warp_sum_partials(const double *__restrict__ partial, int64_t ld, int64_t off,
                                                    int nblk)
{
    const int lane = threadIdx.x & 31;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int q = lane;
    for (; q + 96 < nblk; q += 128)
    {
        const double v0 = partial[(int64_t)q * ld + off], v1 = partial[(int64_t)(q + 32) * ld + off];
        const double v2 = partial[(int64_t)(q + 64) * ld + off], v3 = partial[(int64_t)(q + 96) * ld + off];
        s0 += v0; s1 += v1; s2 += v2; s3 += v3;
    }
    if (q < nblk) s0 += partial[(int64_t)q * ld + off];
    if (q + 32 < nblk) s1 += partial[(int64_t)(q + 32) * ld + off];
    if (q + 64 < nblk) s2 += partial[(int64_t)(q + 64) * ld + off];
    double s = (s0 + s1) + (s2 + s3);
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    return __shfl_sync(0xffffffffu, s, 0);
}

// Two-level column totals of per-block partial sums, run inside the kernel
// that produced them (the "last block" reduction: no launch of its own).
constexpr int kSumGroup = 16;   // blocks per first-level group
__host__ __device__ constexpr int cg_groups(int nblk) { return (nblk + kSumGroup - 1) / kSumGroup; }

// dst[m] = sum of src[q * S + m] over q < nrows, for m < S, by all threads of
// the block: thread t takes m = t, t + blockDim.x, ...; eight loads in flight
// into eight running sums (q mod 8), added in a fixed order.  The rows were
// written by other blocks of the running kernel: loads bypass L1.
__device__ void block_sum_rows(const double *src, int S, int nrows, double *dst)
{
    for (int m = threadIdx.x; m < S; m += blockDim.x)
    {
        double a[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        int q = 0;
        for (; q + 8 <= nrows; q += 8)
        {
            double v[8];
            #pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = __ldcg(src + (int64_t)(q + j) * S + m);
            #pragma unroll
            for (int j = 0; j < 8; ++j) a[j] += v[j];
        }
        #pragma unroll
        for (int j = 0; j < 7; ++j)
            if (q + j < nrows) a[j] += __ldcg(src + (int64_t)(q + j) * S + m);
        dst[m] = ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
    }
}

// Called by every thread of every block after the block has written its part
// of row blockIdx.x of the S partial sums (partial[blockIdx.x * S ...]).  The
// last block of each group of kSumGroup rows sums the group's rows into its
// group row, and the last group to finish sums the group rows into the totals;
// true (in all threads) in that one block, with *tot = the S totals.  Layout
// of `partial`: gridDim.x rows, then cg_groups(gridDim.x) group rows, then the
// totals.  counter[0] counts finished groups, counter[1 + g] the blocks of
// group g; both are back at zero when the kernel ends.  Fixed summation orders
// throughout, so the totals do not depend on timing.  (One block summing all
// rows directly took 58 us of an 85 us CG update on 40962 x 64 values.)
__device__ bool cg_column_totals(double *partial, int S, unsigned int *counter, const double **tot)
{
    __shared__ bool last;
    const int nblk = gridDim.x, ng = cg_groups(nblk);
    const int g = blockIdx.x / kSumGroup, g0 = g * kSumGroup, g1 = min(nblk, g0 + kSumGroup);
    double *gpart = partial + (int64_t)nblk * S;
    double *tt = gpart + (int64_t)ng * S;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
    {
        const unsigned int members = (unsigned int)(g1 - g0) * gridDim.y;
        last = atomicAdd(counter + 1 + g, 1u) == members - 1;
        if (last) counter[1 + g] = 0u;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    block_sum_rows(partial + (int64_t)g0 * S, S, g1 - g0, gpart + (int64_t)g * S);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
    {
        last = atomicAdd(counter, 1u) == (unsigned int)ng - 1;
        if (last) counter[0] = 0u;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    block_sum_rows(gpart, S, ng, tt);
    __syncthreads();
    *tot = tt;
    return true;
}

// Column steps of the CG phases over the column totals tot (one thread per
// column; ApplyMassInverse.hpp:67-147):
//   init:  rz = <r, z>, bn = ||b||, convergence of zero columns    tot = [rz | bb]
//   alpha: alpha = rz / <p, q>                                       tot = [pq]
//   beta:  beta = rz_new / rz, rz = rz_new, convergence ||r|| <= tol ||b||   tot = [rz_new | rr]
// col layout: [0,c) rz  [c,2c) bn  [2c,3c) alpha  [3c,4c) beta ; flags: [0] done [1] iters [2..) conv
__device__ void cg_fin_init(int c, const double *tot, double *col, int *flags, double tol)
{
    int all = 1;
    for (int k = threadIdx.x; k < c; k += blockDim.x)
    {
        const double rz = __ldcg(tot + k), bb = __ldcg(tot + c + k);
        const double bn = sqrt(bb);
        col[k] = rz;
        col[c + k] = bn;
        col[2 * c + k] = 0.0;
        col[3 * c + k] = 0.0;
        const int cv = (bn <= tol * bn) ? 1 : 0;
        flags[2 + k] = cv;
        all &= cv;
    }
    all = __syncthreads_and(all);
    if (threadIdx.x == 0) { flags[0] = all; flags[1] = 0; }
}

__device__ void cg_fin_alpha(int c, const double *tot, double *col, const int *flags)
{
    for (int k = threadIdx.x; k < c; k += blockDim.x)
    {
        const double pq = __ldcg(tot + k);
        col[2 * c + k] = (flags[2 + k] || pq == 0.0) ? 0.0 : col[k] / pq;
    }
}

__device__ void cg_fin_beta(int c, const double *tot, double *col, int *flags, double tol)
{
    int all = 1;
    for (int k = threadIdx.x; k < c; k += blockDim.x)
    {
        const double rzn = __ldcg(tot + k), rr = __ldcg(tot + c + k);
        const int was = flags[2 + k];
        col[3 * c + k] = (was || col[k] == 0.0) ? 0.0 : rzn / col[k];
        col[k] = rzn;
        const int cv = was || (sqrt(rr) <= tol * col[c + k]);
        flags[2 + k] = cv;
        all &= cv;
    }
    all = __syncthreads_and(all);
    if (threadIdx.x == 0) { flags[0] = all; flags[1] += 1; }
}


template <class RV>
__global__ void cg_init_kernel(int64_t n, int c, int cp, int rp, int64_t rpb, const double *__restrict__ b,
                               int64_t ldb, const RV *__restrict__ L, double *__restrict__ x, double *__restrict__ r,
                               double *__restrict__ z, double *__restrict__ p, double *partial,
                               unsigned int *counter, double *col, int *flags, double tol)
{
    __shared__ double sm[RT];
    const int tr = threadIdx.x / cp, tc = threadIdx.x % cp;
    const int k = blockIdx.y * cp + tc;
    const bool active = tr < rp && k < c;
    double rz = 0.0, bb = 0.0;
    if (active)
    {
        const int64_t r0 = blockIdx.x * rpb, r1 = min(n, r0 + rpb);
        for (int64_t row = r0 + tr; row < r1; row += rp)
        {
            const double bv = b[row * ldb + k];
            const double zv = (double)L[row] * bv;
            const int64_t e = row * c + k;
            x[e] = 0.0; r[e] = bv; z[e] = zv; p[e] = zv;
            rz += bv * zv;
            bb += bv * bv;
        }
    }
    double *out = partial + (int64_t)blockIdx.x * 2 * c;
    block_reduce_store(rz, sm, tr, tc, cp, rp, active, out + k);
    block_reduce_store(bb, sm, tr, tc, cp, rp, active, out + c + k);
    const double *tot;
    if (cg_column_totals(partial, 2 * c, counter, &tot)) cg_fin_init(c, tot, col, flags, tol);
}

template <class RV>
__global__ void cg_matvec_kernel(int64_t n, int c, int cp, int rp, int64_t rpb, const int32_t *__restrict__ mo,
                                 const int32_t *__restrict__ mi, const RV *__restrict__ mv, const double *__restrict__ p,
                                 double *__restrict__ q, double *partial, unsigned int *counter, double *col,
                                 const int *flags)
{
    if (flags[0]) return;
    __shared__ double sm[RT];
    const int tr = threadIdx.x / cp, tc = threadIdx.x % cp;
    const int k = blockIdx.y * cp + tc;
    const bool active = tr < rp && k < c;
    double pq = 0.0;
    if (active)
    {
        const int64_t r0 = blockIdx.x * rpb, r1 = min(n, r0 + rpb);
        for (int64_t row = r0 + tr; row < r1; row += rp)
        {
            // the row's first kPf entries (a P1 mass row has 1 + the vertex
            // degree, ~7) are loaded before any gather, so their gathers are in
            // flight together instead of one dependent chain per entry; the sum
            // runs in entry order as before
            constexpr int kPf = 8;
            const int32_t e0 = mo[row], e1 = mo[row + 1];
            int32_t ci[kPf];
            double cv[kPf], pv[kPf];
            #pragma unroll
            for (int j = 0; j < kPf; ++j)
            {
                const bool in = e0 + j < e1;
                ci[j] = in ? mi[e0 + j] : 0;
                cv[j] = in ? (double)mv[e0 + j] : 0.0;
            }
            #pragma unroll
            for (int j = 0; j < kPf; ++j) pv[j] = e0 + j < e1 ? p[(int64_t)ci[j] * c + k] : 0.0;
            double s = 0.0;
            #pragma unroll
            for (int j = 0; j < kPf; ++j)
                if (e0 + j < e1) s += cv[j] * pv[j];
            for (int32_t e = e0 + kPf; e < e1; ++e) s += (double)mv[e] * p[(int64_t)mi[e] * c + k];
            q[row * c + k] = s;
            pq += p[row * c + k] * s;
        }
    }
    block_reduce_store(pq, sm, tr, tc, cp, rp, active, partial + (int64_t)blockIdx.x * c + k);
    const double *tot;
    if (cg_column_totals(partial, c, counter, &tot)) cg_fin_alpha(c, tot, col, flags);
}


template <class RV>
__global__ void cg_update_kernel(int64_t n, int c, int cp, int rp, int64_t rpb, const RV *__restrict__ L,
                                 double *col, double *__restrict__ x, double *__restrict__ r,
                                 double *__restrict__ z, const double *__restrict__ p, const double *__restrict__ q,
                                 double *partial, unsigned int *counter, int *flags, double tol)
{
    if (flags[0]) return;
    __shared__ double sm[RT];
    const int tr = threadIdx.x / cp, tc = threadIdx.x % cp;
    const int k = blockIdx.y * cp + tc;
    const bool active = tr < rp && k < c;
    double rz = 0.0, rr = 0.0;
    if (active)
    {
        const double a = col[2 * c + k];
        const int64_t r0 = blockIdx.x * rpb, r1 = min(n, r0 + rpb);
        // four rows' operands are loaded before any of them is used (four
        // times the loads in flight per thread); the dots accumulate in row
        // order as in the one-row loop below
        int64_t row = r0 + tr;
        for (; row + 3 * rp < r1; row += 4 * rp)
        {
            double pv[4], xv[4], rv[4], qv[4], lv[4];
            #pragma unroll
            for (int u = 0; u < 4; ++u)
            {
                const int64_t e = (row + u * rp) * c + k;
                pv[u] = p[e]; xv[u] = x[e]; rv[u] = r[e]; qv[u] = q[e];
                lv[u] = (double)L[row + u * rp];
            }
            #pragma unroll
            for (int u = 0; u < 4; ++u)
            {
                const int64_t e = (row + u * rp) * c + k;
                x[e] = xv[u] + a * pv[u];
                const double rn = rv[u] - a * qv[u];
                r[e] = rn;
                const double zv = lv[u] * rn;
                z[e] = zv;
                rz += rn * zv;
                rr += rn * rn;
            }
        }
        for (; row < r1; row += rp)
        {
            const int64_t e = row * c + k;
            x[e] += a * p[e];
            const double rn = r[e] - a * q[e];
            r[e] = rn;
            const double zv = (double)L[row] * rn;
            z[e] = zv;
            rz += rn * zv;
            rr += rn * rn;
        }
    }
    double *out = partial + (int64_t)blockIdx.x * 2 * c;
    block_reduce_store(rz, sm, tr, tc, cp, rp, active, out + k);
    block_reduce_store(rr, sm, tr, tc, cp, rp, active, out + c + k);
    const double *tot;
    if (cg_column_totals(partial, 2 * c, counter, &tot)) cg_fin_beta(c, tot, col, flags, tol);
}


__global__ void cg_pupdate_kernel(int64_t total, int c, const double *__restrict__ col, const double *__restrict__ z,
                                  double *__restrict__ p, const int *__restrict__ flags)
{
    if (flags[0]) return;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const int k = (int)(e % c);
    p[e] = z[e] + col[3 * c + k] * p[e];
}

// CG mass inverse on meshes of up to kCgBlockMaxRows vertices: one block per
// column, every iteration in one launch.  The CG's columns are independent
// (each has its own dot products and step lengths), so a block that owns a
// column needs no other block: the phases of an iteration are separated by
// __syncthreads only, and the 3 launches and 3 cross-block column sums of
// an iteration of the multi-block kernels become block sums.  The block's
// vectors are column-major in global memory (column k at x + k n),
// L2-resident at these sizes, except the search direction p, which lives in
// the block's shared memory (n doubles, at most 128 KB): the matvec's gathers
// of p read shared memory instead of L2.  Same steps and stopping rule as the
// multi-block kernels (ApplyMassInverse.hpp:48-156): x = 0, r = b, z = L r,
// p = z; per iteration q = M p, alpha = <r,z> / <p,q>, x += alpha p,
// r -= alpha q, z = L r, beta = <r,z>_new / <r,z>, converged once
// ||r|| <= tol ||b|| (a column of zeros at once), p = z + beta p.  Block sums
// add the threads' row-ordered partials by a fixed shuffle and shared-memory
// tree, so runs are reproducible.  flags: [0] columns not converged, [1] the
// largest iteration count (both zeroed before the launch), [2 + k] column k
// converged.
constexpr int kCgBlockThreads = 1024;
// Up to this many rows one block per column is faster: on the icosphere of
// level 5 (10242 vertices, 128 real columns) one iteration takes 26.5 us
// against 60.3 us for the three multi-block kernels; on level 6 (40962
// vertices, 64 columns) 130 us against 92 us, too few blocks for the rows.
// The bound also keeps p (n doubles) within a block's shared memory.
constexpr int64_t kCgBlockMaxRows = 16384;

// totals of a and b over the block, in every thread (red: 2 x 33 doubles)
__device__ __forceinline__ void block_sum2(double &a, double &b, double *red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    __syncthreads();   // red is free (its previous totals have been read)
    if (lane == 0) { red[warp] = a; red[33 + warp] = b; }
    __syncthreads();
    if (warp == 0)
    {
        double ta = lane < nw ? red[lane] : 0.0, tb = lane < nw ? red[33 + lane] : 0.0;
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1)
        {
            ta += __shfl_down_sync(0xffffffffu, ta, o);
            tb += __shfl_down_sync(0xffffffffu, tb, o);
        }
        if (lane == 0) { red[32] = ta; red[65] = tb; }
    }
    __syncthreads();
    a = red[32];
    b = red[65];
}

template <class RV>
__global__ void __launch_bounds__(kCgBlockThreads, 1)
cg_block_kernel(int64_t n, int c, const double *__restrict__ b, int64_t ldb, const int32_t *__restrict__ mo,
                const int32_t *__restrict__ mi, const RV *__restrict__ mv, const RV *__restrict__ L, double *xs,
                double *rs, double *zs, double *qs, double *__restrict__ y, int64_t ldy, int *flags,
                double tol, int max_iter)
{
    __shared__ double red[66];
    extern __shared__ double p[];   // the column's search direction, n doubles
    const int k = blockIdx.x;
    const int64_t off = (int64_t)k * n;
    // the column's vectors are separate buffers: no aliasing, so the loads of a
    // thread's next row can be issued before the stores of its current one
    double *__restrict__ x = xs + off;
    double *__restrict__ r = rs + off;
    double *__restrict__ z = zs + off;
    double *__restrict__ q = qs + off;
    double rz = 0.0, bb = 0.0;
    for (int64_t row = threadIdx.x; row < n; row += blockDim.x)
    {
        const double bv = b[row * ldb + k];
        const double zv = (double)L[row] * bv;
        x[row] = 0.0; r[row] = bv; z[row] = zv; p[row] = zv;
        rz += bv * zv;
        bb += bv * bv;
    }
    block_sum2(rz, bb, red);   // ends with a barrier: p is complete
    const double bn = sqrt(bb);
    bool conv = bn <= tol * bn;
    int it = 0;
    for (; it < max_iter && !conv; ++it)   // conv and it are block-uniform
    {
        double pq = 0.0, unused = 0.0;
        for (int64_t row = threadIdx.x; row < n; row += blockDim.x)
        {
            // the row's first 8 entries (1 + the vertex degree, ~7) loaded before their gathers
            constexpr int kPf = 8;
            const int32_t e0 = mo[row], e1 = mo[row + 1];
            int32_t ci[kPf];
            double cv[kPf], pv[kPf];
            #pragma unroll
            for (int j = 0; j < kPf; ++j)
            {
                const bool in = e0 + j < e1;
                ci[j] = in ? mi[e0 + j] : 0;
                cv[j] = in ? (double)mv[e0 + j] : 0.0;
            }
            #pragma unroll
            for (int j = 0; j < kPf; ++j) pv[j] = e0 + j < e1 ? p[ci[j]] : 0.0;
            double sacc = 0.0;
            #pragma unroll
            for (int j = 0; j < kPf; ++j)
                if (e0 + j < e1) sacc += cv[j] * pv[j];
            for (int32_t e = e0 + kPf; e < e1; ++e) sacc += (double)mv[e] * p[mi[e]];
            q[row] = sacc;
            pq += p[row] * sacc;
        }
        block_sum2(pq, unused, red);
        const double alpha = pq == 0.0 ? 0.0 : rz / pq;
        double rzn = 0.0, rr = 0.0;
        #pragma unroll 2
        for (int64_t row = threadIdx.x; row < n; row += blockDim.x)
        {
            x[row] += alpha * p[row];
            const double rv = r[row] - alpha * q[row];
            r[row] = rv;
            const double zv = (double)L[row] * rv;
            z[row] = zv;
            rzn += rv * zv;
            rr += rv * rv;
        }
        block_sum2(rzn, rr, red);
        const double beta = rz == 0.0 ? 0.0 : rzn / rz;
        rz = rzn;
        conv = sqrt(rr) <= tol * bn;
        #pragma unroll 4
        for (int64_t row = threadIdx.x; row < n; row += blockDim.x) p[row] = z[row] + beta * p[row];
        __syncthreads();   // p complete before the next iteration's gathers
    }
    for (int64_t row = threadIdx.x; row < n; row += blockDim.x) y[row * ldy + k] = x[row];
    if (threadIdx.x == 0)
    {
        flags[2 + k] = conv ? 1 : 0;
        if (!conv) atomicAdd(&flags[0], 1);
        atomicMax(&flags[1], it);
    }
}

// One block per column with p (n doubles) in dynamic shared memory; the limit
// above 48 KB is a per-device attribute of each instantiation, set once.
template <class RV>
void launch_cg_block(cudaStream_t st, int64_t n, int c, const double *b, int64_t ldb, const int32_t *mo,
                     const int32_t *mi, const RV *mv, const RV *L, double *x, double *r, double *z, double *q,
                     double *y, int64_t ldy, int *flags, double tol, int max_iter)
{
    constexpr int kMaxBytes = (int)(kCgBlockMaxRows * sizeof(double));
    int dev = 0;
    BAEMM_CUDA(cudaGetDevice(&dev));
    static std::mutex mu;
    static bool done[64] = {};
    {
        std::lock_guard<std::mutex> lock(mu);
        if (dev < 0 || dev >= 64 || !done[dev])
        {
            BAEMM_CUDA(cudaFuncSetAttribute(cg_block_kernel<RV>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxBytes));
            if (dev >= 0 && dev < 64) done[dev] = true;
        }
    }
    cg_block_kernel<<<c, kCgBlockThreads, (size_t)n * sizeof(double), st>>>(n, c, b, ldb, mo, mi, mv, L, x, r, z, q,
                                                                              y, ldy, flags, tol, max_iter);
}

__global__ void cg_output_kernel(int64_t n, int c, const double *__restrict__ x, double *__restrict__ y, int64_t ldy)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * c) return;
    const int64_t row = e / c;
    const int k = (int)(e - row * c);
    y[row * ldy + k] = x[e];
}

// ============================== GMRES ==========================================

// partial[blk][i*c + k] (S words) = sum_rows conj(V_i[r,k]) w[r,k], i < nvec.
// The vectors are taken in groups of kGroup so the accumulators stay in
// registers; w is re-read per group (it is L2-resident).
constexpr int kGroup = 8;
template <class S>
__global__ void gs_dot_kernel(int64_t n, int c, int cp, int rp, int64_t rpb, const S *__restrict__ V, int nvec,
                              const S *__restrict__ w, double *__restrict__ partial)
{
    __shared__ double sm[RT];
    const int tr = threadIdx.x / cp, tc = threadIdx.x % cp;
    const int k = blockIdx.y * cp + tc;
    const bool active = tr < rp && k < c;
    const int64_t stride = n * c;
    constexpr int W = kWords<S>;
    double *out = partial + (int64_t)blockIdx.x * nvec * c * W;
    const int64_t r0 = blockIdx.x * rpb, r1 = min(n, r0 + rpb);
    for (int g0 = 0; g0 < nvec; g0 += kGroup)
    {
        double ax[kGroup], ay[kGroup];
        #pragma unroll
        for (int i = 0; i < kGroup; ++i) { ax[i] = 0.0; ay[i] = 0.0; }
        if (active)
        {
            for (int64_t row = r0 + tr; row < r1; row += rp)
            {
                const S wv = w[row * c + k];
                #pragma unroll
                for (int i = 0; i < kGroup; ++i)
                {
                    if (g0 + i < nvec)
                    {
                        const S v = V[(g0 + i) * stride + row * c + k];
                        ax[i] += re(v) * re(wv) + im(v) * im(wv);
                        ay[i] += re(v) * im(wv) - im(v) * re(wv);
                    }
                }
            }
        }
        #pragma unroll
        for (int i = 0; i < kGroup; ++i)
        {
            if (g0 + i < nvec)
            {
                double *dst = out + ((int64_t)(g0 + i) * c + k) * W;
                block_reduce_store(ax[i], sm, tr, tc, cp, rp, active, dst);
                if (W == 2) block_reduce_store(ay[i], sm, tr, tc, cp, rp, active, dst + 1);
            }
        }
    }
}

// h[i*c+k] = sum_blk partial; H[(i*m + j)*c + k] (+)= h
template <class S>
__global__ void gs_finalize_kernel(int c, int nblk, int nvec, const double *__restrict__ partial, S *__restrict__ h,
                                   S *__restrict__ H, int m, int j, int accumulate)
{
    // one warp per item (a basis vector's dot product with one column)
    const int item = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (item >= nvec * c) return;   // warp-uniform
    constexpr int W = kWords<S>;
    const int64_t ld = (int64_t)nvec * c * W;
    const double sx = warp_sum_partials(partial, ld, (int64_t)item * W, nblk);
    const double sy = W == 2 ? warp_sum_partials(partial, ld, (int64_t)item * W + 1, nblk) : 0.0;
    if ((threadIdx.x & 31) != 0) return;
    const S v = mkS<S>(sx, sy);
    h[item] = v;
    const int i = item / c, k = item - i * c;
    S &dst = H[((int64_t)i * m + j) * c + k];
    dst = accumulate ? Sadd(dst, v) : v;
}

template <class S>
__global__ void gs_update_kernel(int64_t n, int c, const S *__restrict__ V, int nvec, const S *__restrict__ h,
                                 S *__restrict__ w)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * c) return;
    const int k = (int)(e % c);
    const int64_t stride = n * c;
    S acc = w[e];
    for (int i = 0; i < nvec; ++i) acc = Ssub(acc, Smul(h[i * c + k], V[i * stride + e]));
    w[e] = acc;
}

template <class S>
__global__ void norm_partial_kernel(int64_t n, int c, int cp, int rp, int64_t rpb, const S *__restrict__ w,
                                    double *__restrict__ partial)
{
    __shared__ double sm[RT];
    const int tr = threadIdx.x / cp, tc = threadIdx.x % cp;
    const int k = blockIdx.y * cp + tc;
    const bool active = tr < rp && k < c;
    double s = 0.0;
    if (active)
    {
        const int64_t r0 = blockIdx.x * rpb, r1 = min(n, r0 + rpb);
        for (int64_t row = r0 + tr; row < r1; row += rp) s += Sabs2(w[row * c + k]);
    }
    block_reduce_store(s, sm, tr, tc, cp, rp, active, partial + (int64_t)blockIdx.x * c + k);
}

// hn[k] = ||w_k||; mode 0: H[(j+1)m + j] = hn ; mode 1: start of a cycle (res, g, bnorm)
template <class S>
__global__ void norm_finalize_kernel(int c, int nblk, const double *__restrict__ partial, double *__restrict__ hn,
                                     S *__restrict__ H, int m, int j, int mode, double *__restrict__ res,
                                     S *__restrict__ g, double *__restrict__ bnorm, int *__restrict__ flags, double tol)
{
    int all = 1;
    const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5, lane = threadIdx.x & 31;
    for (int k = warp; k < c; k += nwarps)
    {
        const double nv = sqrt(warp_sum_partials(partial, c, k, nblk));
        if (mode != 0)
            for (int i = lane; i <= m; i += 32) g[(int64_t)i * c + k] = mkS<S>(i == 0 ? nv : 0.0, 0.0);
        if (lane != 0) continue;
        hn[k] = nv;
        if (mode == 0)
            H[((int64_t)(j + 1) * m + j) * c + k] = mkS<S>(nv, 0.0);
        else
        {
            if (mode == 2) bnorm[k] = nv;   // first cycle: ||P b||
            res[k] = nv;
            all &= (nv <= tol * bnorm[k]) ? 1 : 0;
        }
    }
    if (mode != 0)
    {
        all = __syncthreads_and(all);
        if (threadIdx.x == 0) flags[0] = all;
    }
}

template <class S>
__global__ void normalize_kernel(int64_t n, int c, const S *__restrict__ w, const double *__restrict__ hn,
                                 S *__restrict__ v)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * c) return;
    const double d = hn[e % c];
    v[e] = d > 0.0 ? Sscale(w[e], 1.0 / d) : mkS<S>(0.0, 0.0);
}

template <class S>
__global__ void givens_kernel(int c, int m, int j, S *__restrict__ H, double *__restrict__ cs, S *__restrict__ sn,
                              S *__restrict__ g, double *__restrict__ res, const double *__restrict__ bnorm,
                              int *__restrict__ flags, double tol)
{
    int all = 1;
    for (int k = threadIdx.x; k < c; k += blockDim.x)
    {
        for (int i = 0; i < j; ++i)
        {
            S &h0 = H[((int64_t)i * m + j) * c + k];
            S &h1 = H[((int64_t)(i + 1) * m + j) * c + k];
            const double cc = cs[i * c + k];
            const S s = sn[i * c + k];
            const S t0 = Sadd(Sscale(h0, cc), Smul(s, h1));
            const S t1 = Sadd(Sscale(Smul(Sconj(s), h0), -1.0), Sscale(h1, cc));
            h0 = t0;
            h1 = t1;
        }
        S &a = H[((int64_t)j * m + j) * c + k];
        S &b = H[((int64_t)(j + 1) * m + j) * c + k];
        const double aa = sqrt(Sabs2(a)), bb = sqrt(Sabs2(b));
        double cc;
        S s;
        if (aa == 0.0)
        {
            cc = 0.0;
            s = mkS<S>(1.0, 0.0);
            a = b;
        }
        else
        {
            const double t = sqrt(aa * aa + bb * bb);
            cc = aa / t;
            const S ua = Sscale(a, 1.0 / aa);
            s = Sscale(Smul(ua, Sconj(b)), 1.0 / t);
            a = Sscale(ua, t);
        }
        b = mkS<S>(0.0, 0.0);
        cs[j * c + k] = cc;
        sn[j * c + k] = s;
        const S gj = g[(int64_t)j * c + k];
        g[(int64_t)j * c + k] = Sscale(gj, cc);
        const S gn = Sscale(Smul(Sconj(s), gj), -1.0);
        g[(int64_t)(j + 1) * c + k] = gn;
        const double rn = sqrt(Sabs2(gn));
        res[k] = rn;
        all &= (rn <= tol * bnorm[k]) ? 1 : 0;
    }
    all = __syncthreads_and(all);
    if (threadIdx.x == 0) flags[0] = all;
}

template <class S>
__global__ void backsolve_kernel(int c, int m, int jend, const S *__restrict__ H, const S *__restrict__ g,
                                 S *__restrict__ y)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= c) return;
    for (int i = jend - 1; i >= 0; --i)
    {
        S s = g[(int64_t)i * c + k];
        for (int l = i + 1; l < jend; ++l) s = Ssub(s, Smul(H[((int64_t)i * m + l) * c + k], y[(int64_t)l * c + k]));
        const S d = H[((int64_t)i * m + i) * c + k];
        y[(int64_t)i * c + k] = (Sabs2(d) == 0.0) ? mkS<S>(0.0, 0.0) : Sdiv(s, d);
    }
}

template <class S>
__global__ void update_x_kernel(int64_t n, int c, int jend, const S *__restrict__ V, const S *__restrict__ y,
                                S *__restrict__ x)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * c) return;
    const int k = (int)(e % c);
    const int64_t stride = n * c;
    S acc = x[e];
    for (int i = 0; i < jend; ++i) acc = Sadd(acc, Smul(y[(int64_t)i * c + k], V[i * stride + e]));
    x[e] = acc;
}

// r = b - Ax; r may be Ax (the restart computes it in place), so those two
// are not restrict-qualified.
template <class S>
__global__ void residual_kernel(int64_t total, const S *__restrict__ b, const S *Ax, S *r)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    r[e] = Ssub(b[e], Ax[e]);
}

template <class S>
__global__ void gather_kernel(int64_t n, int c, const S *__restrict__ src, int64_t lds, S *__restrict__ dst)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * c) return;
    const int64_t row = e / c;
    dst[e] = src[row * lds + (e - row * c)];
}

template <class S>
__global__ void output_kernel(int64_t n, int c, S alpha, const S *__restrict__ x, S beta, S *__restrict__ out,
                              int64_t ldo)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * c) return;
    const int64_t row = e / c;
    S *o = &out[row * ldo + (e - row * c)];
    const S ax = Smul(alpha, x[e]);
    *o = (Sabs2(beta) == 0.0) ? ax : Sadd(ax, Smul(beta, *o));
}

inline int eg(int64_t n) { return ceil_div(n, 256); }

} // namespace

// =================================== CG host ======================================
CgSolver::~CgSolver()
{
    if (host_flags_) cudaFreeHost(host_flags_);
}

bool CgSolver::solve_mass(const MeshDev &m, bool fp64_values, const double *b, int64_t ldb, double *y, int64_t ldy,
                          int c, double tol, int max_iter, cudaStream_t st, int *iterations)
{
    enqueue_mass(m, fp64_values, b, ldb, y, ldy, c, tol, max_iter, st);
    return finish(st, iterations);
}

bool CgSolver::finish(cudaStream_t st, int *iterations)
{
    BAEMM_CUDA(cudaStreamSynchronize(st));
    if (iterations) *iterations = host_flags_[1];
    // flags[0]: all converged (multi-block kernels) or columns not converged (cg_block_kernel)
    return block_path_ ? host_flags_[0] == 0 : host_flags_[0] != 0;
}

void CgSolver::reserve_totals(int nblk, int S, cudaStream_t st)
{
    const int ng = cg_groups(nblk);
    partial_.reserve((size_t)(nblk + ng + 1) * S);
    const size_t nc = 1 + (size_t)ng;
    if (counter_.n < nc)
    {
        counter_.reserve(nc);
        BAEMM_CUDA(cudaMemsetAsync(counter_.p, 0, counter_.n * sizeof(unsigned int), st));
    }
}

void CgSolver::enqueue_mass(const MeshDev &m, bool fp64_values, const double *b, int64_t ldb, double *y,
                            int64_t ldy, int c, double tol, int max_iter, cudaStream_t st)
{
    const int64_t n = m.nv;
    BAEMM_REQUIRE(c >= 1 && c <= kMaxKrylovColumns, BAEMM_ERR_SIZE, "CG column count out of range");
    const int64_t N = n * c;
    x_.reserve(N); r_.reserve(N); z_.reserve(N); p_.reserve(N); q_.reserve(N);
    col_.reserve(4 * (size_t)c);
    flags_.reserve(2 + (size_t)c);
    if (!host_flags_) BAEMM_CUDA(cudaMallocHost(&host_flags_, 2 * sizeof(int)));
    block_path_ = n <= kCgBlockMaxRows;
    if (block_path_)
    {
        // one block per column, all iterations in one launch
        BAEMM_CUDA(cudaMemsetAsync(flags_.p, 0, 2 * sizeof(int), st));
        auto runb = [&](auto Lv, auto Mv) {
            launch_cg_block(st, n, c, b, ldb, m.mass_outer, m.mass_inner, Mv, Lv, x_.p, r_.p, z_.p, q_.p, y, ldy,
                            flags_.p, tol, max_iter);
        };
        if (fp64_values) runb(m.lumped_d.p, m.mass_d.p);
        else runb(m.lumped_f.p, m.mass_f.p);
        BAEMM_LAUNCH_CHECK();
        BAEMM_CUDA(cudaMemcpyAsync(host_flags_, flags_.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
        return;
    }
    const Layout L = make_layout(n, c);
    reserve_totals(L.nblk, 2 * c, st);
    dim3 grid(L.nblk, L.nchunk);
    auto run = [&](auto Lv, auto Mv) {
        // three launches per iteration: each column-sum step runs in the last
        // block of the kernel that produced the partial sums
        cg_init_kernel<<<grid, RT, 0, st>>>(n, c, L.cp, L.rp, L.rows_per_block, b, ldb, Lv, x_.p, r_.p, z_.p, p_.p,
                                            partial_.p, counter_.p, col_.p, flags_.p, tol);
        for (int it = 0; it < max_iter; ++it)
        {
            cg_matvec_kernel<<<grid, RT, 0, st>>>(n, c, L.cp, L.rp, L.rows_per_block, m.mass_outer, m.mass_inner, Mv,
                                                  p_.p, q_.p, partial_.p, counter_.p, col_.p, flags_.p);
            cg_update_kernel<<<grid, RT, 0, st>>>(n, c, L.cp, L.rp, L.rows_per_block, Lv, col_.p, x_.p, r_.p, z_.p,
                                                  p_.p, q_.p, partial_.p, counter_.p, flags_.p, tol);
            cg_pupdate_kernel<<<eg(N), 256, 0, st>>>(N, c, col_.p, z_.p, p_.p, flags_.p);
        }
    };
    if (fp64_values) run(m.lumped_d.p, m.mass_d.p);
    else run(m.lumped_f.p, m.mass_f.p);
    BAEMM_LAUNCH_CHECK();
    cg_output_kernel<<<eg(N), 256, 0, st>>>(n, c, x_.p, y, ldy);
    BAEMM_LAUNCH_CHECK();
    BAEMM_CUDA(cudaMemcpyAsync(host_flags_, flags_.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
}

double CgSolver::profile_block(const MeshDev &m, bool fp64_values, int c, int iterations, cudaStream_t st)
{
    const int64_t n = m.nv;
    BAEMM_REQUIRE(c >= 1 && c <= kMaxKrylovColumns, BAEMM_ERR_SIZE, "CG column count out of range");
    BAEMM_REQUIRE(iterations >= 1, BAEMM_ERR_ARG, "at least one iteration");
    if (n > kCgBlockMaxRows) return 0.0;
    const int64_t N = n * c;
    DevBuf<double> b, y;
    b.reserve(N);
    y.reserve(N);
    std::vector<double> ones((size_t)N, 1.0);
    BAEMM_CUDA(cudaMemcpyAsync(b.p, ones.data(), N * sizeof(double), cudaMemcpyHostToDevice, st));
    x_.reserve(N); r_.reserve(N); z_.reserve(N); p_.reserve(N); q_.reserve(N);
    flags_.reserve(2 + (size_t)c);
    cudaEvent_t e0, e1;
    BAEMM_CUDA(cudaEventCreate(&e0));
    BAEMM_CUDA(cudaEventCreate(&e1));
    float ms = 0.f;
    auto runb = [&](auto Lv, auto Mv) {
        // tol < 0: no column converges, every iteration does its work; a first launch warms up
        for (int rep = 0; rep < 2; ++rep)
        {
            BAEMM_CUDA(cudaMemsetAsync(flags_.p, 0, 2 * sizeof(int), st));
            BAEMM_CUDA(cudaEventRecord(e0, st));
            launch_cg_block(st, n, c, b.p, c, m.mass_outer, m.mass_inner, Mv, Lv, x_.p, r_.p, z_.p, q_.p, y.p, c,
                            flags_.p, -1.0, iterations);
            BAEMM_CUDA(cudaEventRecord(e1, st));
        }
    };
    if (fp64_values) runb(m.lumped_d.p, m.mass_d.p);
    else runb(m.lumped_f.p, m.mass_f.p);
    BAEMM_LAUNCH_CHECK();
    BAEMM_CUDA(cudaEventSynchronize(e1));
    BAEMM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return (double)ms / iterations;
}

void CgSolver::profile(const MeshDev &m, bool fp64_values, int c, int iterations, cudaStream_t st, double ms_out[3])
{
    const int64_t n = m.nv;
    BAEMM_REQUIRE(c >= 1 && c <= kMaxKrylovColumns, BAEMM_ERR_SIZE, "CG column count out of range");
    BAEMM_REQUIRE(iterations >= 1, BAEMM_ERR_ARG, "at least one iteration");
    const int64_t N = n * c;
    DevBuf<double> b;
    b.reserve(N);
    std::vector<double> ones((size_t)N, 1.0);
    BAEMM_CUDA(cudaMemcpyAsync(b.p, ones.data(), N * sizeof(double), cudaMemcpyHostToDevice, st));
    x_.reserve(N); r_.reserve(N); z_.reserve(N); p_.reserve(N); q_.reserve(N);
    col_.reserve(4 * (size_t)c);
    flags_.reserve(2 + (size_t)c);
    const Layout L = make_layout(n, c);
    reserve_totals(L.nblk, 2 * c, st);
    dim3 grid(L.nblk, L.nchunk);
    cudaEvent_t ev[4];
    for (auto &e : ev) BAEMM_CUDA(cudaEventCreate(&e));
    double acc[3] = {0.0, 0.0, 0.0};
    auto run = [&](auto Lv, auto Mv) {
        // tol < 0: no column converges, every launch does its work
        cg_init_kernel<<<grid, RT, 0, st>>>(n, c, L.cp, L.rp, L.rows_per_block, b.p, c, Lv, x_.p, r_.p, z_.p, p_.p,
                                            partial_.p, counter_.p, col_.p, flags_.p, -1.0);
        for (int it = 0; it < iterations; ++it)
        {
            BAEMM_CUDA(cudaEventRecord(ev[0], st));
            cg_matvec_kernel<<<grid, RT, 0, st>>>(n, c, L.cp, L.rp, L.rows_per_block, m.mass_outer, m.mass_inner, Mv,
                                                  p_.p, q_.p, partial_.p, counter_.p, col_.p, flags_.p);
            BAEMM_CUDA(cudaEventRecord(ev[1], st));
            cg_update_kernel<<<grid, RT, 0, st>>>(n, c, L.cp, L.rp, L.rows_per_block, Lv, col_.p, x_.p, r_.p, z_.p,
                                                  p_.p, q_.p, partial_.p, counter_.p, flags_.p, -1.0);
            BAEMM_CUDA(cudaEventRecord(ev[2], st));
            cg_pupdate_kernel<<<eg(N), 256, 0, st>>>(N, c, col_.p, z_.p, p_.p, flags_.p);
            BAEMM_CUDA(cudaEventRecord(ev[3], st));
            BAEMM_CUDA(cudaEventSynchronize(ev[3]));
            for (int q = 0; q < 3; ++q)
            {
                float ms = 0.f;
                BAEMM_CUDA(cudaEventElapsedTime(&ms, ev[q], ev[q + 1]));
                acc[q] += ms;
            }
        }
    };
    try
    {
        if (fp64_values) run(m.lumped_d.p, m.mass_d.p);
        else run(m.lumped_f.p, m.mass_f.p);
        BAEMM_LAUNCH_CHECK();
    }
    catch (...)
    {
        for (auto &e : ev) cudaEventDestroy(e);
        throw;
    }
    for (auto &e : ev) BAEMM_CUDA(cudaEventDestroy(e));
    for (int q = 0; q < 3; ++q) ms_out[q] = acc[q] / iterations;
}

void profile_gram_schmidt(int64_t n, int c, int nvec, int reps, cudaStream_t st, double ms_out[2])
{
    BAEMM_REQUIRE(c >= 1 && c <= kMaxKrylovColumns && nvec >= 1 && nvec <= kMaxRestart + 1 && reps >= 1,
                  BAEMM_ERR_ARG, "Gram-Schmidt profile: sizes out of range");
    const int64_t N = n * c;
    DevBuf<double2> V, w, h;
    V.reserve((size_t)nvec * N);
    w.reserve(N);
    h.reserve((size_t)nvec * c);
    const Layout L = make_layout(n, c);
    DevBuf<double> partial;
    partial.reserve((size_t)L.nblk * nvec * c * 2);
    // constant blocks (the timing does not depend on the values); h small so w stays finite
    BAEMM_CUDA(cudaMemsetAsync(V.p, 0, (size_t)nvec * N * sizeof(double2), st));
    BAEMM_CUDA(cudaMemsetAsync(w.p, 0, N * sizeof(double2), st));
    BAEMM_CUDA(cudaMemsetAsync(h.p, 0, (size_t)nvec * c * sizeof(double2), st));
    dim3 grid(L.nblk, L.nchunk);
    cudaEvent_t ev[3];
    for (auto &e : ev) BAEMM_CUDA(cudaEventCreate(&e));
    double acc[2] = {0.0, 0.0};
    try
    {
        for (int r = 0; r <= reps; ++r)   // the first round is a warm-up
        {
            BAEMM_CUDA(cudaEventRecord(ev[0], st));
            gs_dot_kernel<double2><<<grid, RT, 0, st>>>(n, c, L.cp, L.rp, L.rows_per_block, V.p, nvec, w.p,
                                                        partial.p);
            BAEMM_CUDA(cudaEventRecord(ev[1], st));
            gs_update_kernel<double2><<<eg(N), 256, 0, st>>>(n, c, V.p, nvec, h.p, w.p);
            BAEMM_CUDA(cudaEventRecord(ev[2], st));
            BAEMM_CUDA(cudaEventSynchronize(ev[2]));
            BAEMM_LAUNCH_CHECK();
            if (r == 0) continue;
            for (int q = 0; q < 2; ++q)
            {
                float ms = 0.f;
                BAEMM_CUDA(cudaEventElapsedTime(&ms, ev[q], ev[q + 1]));
                acc[q] += ms;
            }
        }
    }
    catch (...)
    {
        for (auto &e : ev) cudaEventDestroy(e);
        throw;
    }
    for (auto &e : ev) BAEMM_CUDA(cudaEventDestroy(e));
    ms_out[0] = acc[0] / reps;
    ms_out[1] = acc[1] / reps;
}

// =================================== GMRES host ===================================
template <class S>
GmresSolver<S>::~GmresSolver()
{
    if (host_flags_) cudaFreeHost(host_flags_);
    if (host_res_) cudaFreeHost(host_res_);
}

template <class S>
size_t GmresSolver<S>::device_bytes() const
{
    return (V_.n + H_.n + sn_.n + g_.n + h_.n + y_.n + w_.n + tmp_.n + x_.n + b_.n) * sizeof(S) +
           (cs_.n + res_.n + bnorm_.n + hn_.n + partial_.n) * sizeof(double);
}

template <class S>
typename GmresSolver<S>::Stats GmresSolver<S>::solve(int64_t n, int c, int restart, int cycles, const Op &A,
                                                     const Op &P, S alpha, const S *b, int64_t ldb, S beta, S *x_out,
                                                     int64_t ldx, double tol, cudaStream_t st)
{
    BAEMM_REQUIRE(c >= 1 && c <= kMaxKrylovColumns, BAEMM_ERR_SIZE, "GMRES column count out of range");
    BAEMM_REQUIRE(restart >= 1 && restart <= kMaxRestart, BAEMM_ERR_SIZE, "GMRES restart length out of range");
    BAEMM_REQUIRE(cycles >= 1, BAEMM_ERR_ARG, "GMRES needs at least one cycle");
    const int m = restart;
    const int64_t N = n * c;
    V_.reserve((size_t)(m + 1) * N);
    H_.reserve((size_t)(m + 1) * m * c);
    sn_.reserve((size_t)m * c); cs_.reserve((size_t)m * c);
    g_.reserve((size_t)(m + 1) * c);
    h_.reserve((size_t)(m + 1) * c);
    y_.reserve((size_t)m * c);
    w_.reserve(N); tmp_.reserve(N); x_.reserve(N); b_.reserve(N);
    res_.reserve(c); bnorm_.reserve(c); hn_.reserve(c);
    flags_.reserve(4);
    const Layout L = make_layout(n, c);
    constexpr int W = kWords<S>;
    partial_.reserve((size_t)L.nblk * (m + 1) * c * W);
    if (!host_flags_) BAEMM_CUDA(cudaMallocHost(&host_flags_, 4 * sizeof(int)));
    if (host_cap_ < c)
    {
        if (host_res_) cudaFreeHost(host_res_);
        BAEMM_CUDA(cudaMallocHost(&host_res_, 2 * (size_t)c * sizeof(double)));
        host_cap_ = c;
    }
    dim3 grid(L.nblk, L.nchunk);
    const int fin = std::min(1024, ((c + 31) / 32) * 32);   // givens: one thread per column
    const int fin_w = std::min(1024, 32 * c);                // norm finalize: one warp per column

    auto read_flag = [&]() {
        BAEMM_CUDA(cudaMemcpyAsync(host_flags_, flags_.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        BAEMM_CUDA(cudaStreamSynchronize(st));
        return host_flags_[0] != 0;
    };
    // hn = ||w|| columnwise, with `mode` as in norm_finalize_kernel
    auto norms = [&](const S *w, int j, int mode) {
        norm_partial_kernel<S><<<grid, RT, 0, st>>>(n, c, L.cp, L.rp, L.rows_per_block, w, partial_.p);
        norm_finalize_kernel<S><<<1, fin_w, 0, st>>>(c, L.nblk, partial_.p, hn_.p, H_.p, m, j, mode, res_.p, g_.p,
                                                   bnorm_.p, flags_.p, tol);
        BAEMM_LAUNCH_CHECK();
    };

    Stats stats;
    gather_kernel<S><<<eg(N), 256, 0, st>>>(n, c, b, ldb, b_.p);
    BAEMM_CUDA(cudaMemsetAsync(x_.p, 0, N * sizeof(S), st));
    BAEMM_LAUNCH_CHECK();
    bool conv = false;
    for (int cyc = 0; cyc < cycles; ++cyc)
    {
        if (cyc == 0)
        {
            P(b_.p, w_.p);
            norms(w_.p, 0, 2);
        }
        else
        {
            A(x_.p, tmp_.p);
            residual_kernel<S><<<eg(N), 256, 0, st>>>(N, b_.p, tmp_.p, tmp_.p);
            P(tmp_.p, w_.p);
            norms(w_.p, 0, 1);
        }
        if (read_flag()) { conv = true; break; }
        normalize_kernel<S><<<eg(N), 256, 0, st>>>(n, c, w_.p, hn_.p, V_.p);
        BAEMM_CUDA(cudaMemsetAsync(H_.p, 0, (size_t)(m + 1) * m * c * sizeof(S), st));
        int jend = 0;
        for (int j = 0; j < m; ++j)
        {
            S *Vj = V_.p + (int64_t)j * N;
            A(Vj, tmp_.p);
            P(tmp_.p, w_.p);
            const int nvec = j + 1;
            const int fg = ceil_div((int64_t)nvec * c * 32, 256);   // one warp per item
            for (int pass = 0; pass < 2; ++pass)
            {
                gs_dot_kernel<S><<<grid, RT, 0, st>>>(n, c, L.cp, L.rp, L.rows_per_block, V_.p, nvec, w_.p,
                                                      partial_.p);
                gs_finalize_kernel<S><<<fg, 256, 0, st>>>(c, L.nblk, nvec, partial_.p, h_.p, H_.p, m, j, pass);
                gs_update_kernel<S><<<eg(N), 256, 0, st>>>(n, c, V_.p, nvec, h_.p, w_.p);
            }
            norms(w_.p, j, 0);
            normalize_kernel<S><<<eg(N), 256, 0, st>>>(n, c, w_.p, hn_.p, V_.p + (int64_t)(j + 1) * N);
            givens_kernel<S><<<1, fin, 0, st>>>(c, m, j, H_.p, cs_.p, sn_.p, g_.p, res_.p, bnorm_.p, flags_.p, tol);
            BAEMM_LAUNCH_CHECK();
            stats.iterations++;
            jend = j + 1;
            if (read_flag()) { conv = true; break; }
        }
        backsolve_kernel<S><<<ceil_div(c, 128), 128, 0, st>>>(c, m, jend, H_.p, g_.p, y_.p);
        update_x_kernel<S><<<eg(N), 256, 0, st>>>(n, c, jend, V_.p, y_.p, x_.p);
        BAEMM_LAUNCH_CHECK();
        if (conv) break;
    }
    output_kernel<S><<<eg(N), 256, 0, st>>>(n, c, alpha, x_.p, beta, x_out, ldx);
    BAEMM_LAUNCH_CHECK();
    BAEMM_CUDA(cudaMemcpyAsync(host_res_, res_.p, c * sizeof(double), cudaMemcpyDeviceToHost, st));
    BAEMM_CUDA(cudaMemcpyAsync(host_res_ + c, bnorm_.p, c * sizeof(double), cudaMemcpyDeviceToHost, st));
    BAEMM_CUDA(cudaStreamSynchronize(st));
    stats.converged = conv;
    stats.max_rel_res = 0.0;
    for (int k = 0; k < c; ++k)
        if (host_res_[c + k] > 0) stats.max_rel_res = std::max(stats.max_rel_res, host_res_[k] / host_res_[c + k]);
    return stats;
}

namespace
{
__global__ void dot_partial_kernel(const double *__restrict__ a, const double *__restrict__ b, int64_t n,
                                   double *__restrict__ partial)
{
    __shared__ double sm[RT];
    double s = 0.0;
    for (int64_t e = (int64_t)blockIdx.x * RT + threadIdx.x; e < n; e += (int64_t)gridDim.x * RT) s += a[e] * b[e];
    sm[threadIdx.x] = s;
    __syncthreads();
    for (int w = RT / 2; w > 0; w >>= 1)
    {
        if (threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sm[0];
}
} // namespace

double device_dot(const double *a, const double *b, int64_t n, DevBuf<double> &partial, cudaStream_t st)
{
    constexpr int nb = 256;
    std::vector<double> h(nb);
    dot_partial_kernel<<<nb, RT, 0, st>>>(a, b, n, partial.reserve(nb));
    BAEMM_LAUNCH_CHECK();
    BAEMM_CUDA(cudaMemcpyAsync(h.data(), partial.p, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
    BAEMM_CUDA(cudaStreamSynchronize(st));
    double s = 0.0;
    for (double v : h) s += v;
    return s;
}

void device_colnorms(const double2 *w, int64_t n, int c, double *out_host, DevBuf<double> &partial,
                     cudaStream_t st)
{
    const Layout L = make_layout(n, c);
    partial.reserve((size_t)L.nblk * c);
    norm_partial_kernel<double2><<<dim3(L.nblk, L.nchunk), RT, 0, st>>>(n, c, L.cp, L.rp, L.rows_per_block, w,
                                                                        partial.p);
    BAEMM_LAUNCH_CHECK();
    std::vector<double> h((size_t)L.nblk * c);
    BAEMM_CUDA(cudaMemcpyAsync(h.data(), partial.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    BAEMM_CUDA(cudaStreamSynchronize(st));
    for (int k = 0; k < c; ++k)
    {
        double s = 0.0;
        for (int q = 0; q < L.nblk; ++q) s += h[(size_t)q * c + k];
        out_host[k] = std::sqrt(s);
    }
}

template class GmresSolver<double>;
template class GmresSolver<double2>;

} // namespace baemm
