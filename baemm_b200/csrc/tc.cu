// Compensated tensor-core form of the dense boundary kernel (sm_100a, tcgen05).
//
// The apply C_i = sum_j A_ij(kappa) B_j of BoundaryOperatorKernel.cl:5-239 as
// a real GEMM per wave chunk (16 right-hand sides):
//     [C_re | C_im]  (128 x 32)  =  A  (128 x 2S)  x  Bimg^T  (2S x 32)
// with A[i][2s] = Re A_is, A[i][2s+1] = Im A_is and, for each source s,
//     Bimg[q][2s] = Re b_sq,  Bimg[q][2s+1] = -Im b_sq,
//     Bimg[16+q][2s] = Im b_sq, Bimg[16+q][2s+1] = Re b_sq   (q < 16).
// Operands are split into TF32 hi + lo parts and the product is compensated:
//     A B ~= Ahi Bhi + Alo Bhi + Ahi Blo       (FP32 accumulation in TMEM),
// which keeps ~21 bits per product (TF32 hi+lo), well inside 1e-5 relative.
//
// Work unit = (group of up to 4 chunks, block of 128 targets, 16-source tile).
// The grid is persistent (one CTA per SM, it holds all 512 TMEM columns) and
// splits the linear range of units evenly ("stream-K"): a CTA walks its range
// as pieces (runs of tiles of one target block).  A piece covering a whole
// block writes C_tri; a partial piece (at most the first and the last of a
// CTA) writes its partial sums to a workspace slot, and tc_fixup_kernel adds
// the slots of each split block in CTA order (deterministic).
// Warp roles (384 threads):
//   warps 0-7   generators: thread (lane quarter q = warp % 4, half g = warp / 4)
//               owns target row 32 q + lane and sources 8 g .. 8 g + 7 of each
//               16-source K tile; it evaluates the kernel entries in registers
//               (geometry shared by all chunks), splits them into hi / lo and
//               writes them straight into TMEM (tcgen05.st), so the A operand
//               never touches shared memory;
//   warps 8-9   expanders: expand the tile's 16 B_tri rows into hi / lo K-major
//               SWIZZLE_128B images in shared memory;
//   warp 10     bulk-copy producer: cp.async.bulk of the raw tile (B_tri rows,
//               midpoints, normals) into shared memory;
//   warp 11     MMA issuer: 12 tcgen05.mma (kind::tf32, A from TMEM, B from
//               shared memory, M 128, N 32, K 8) per chunk and tile.
// Pipelines use mbarriers (A stages in TMEM, B stages in shared memory).
// Every wait is bounded: on time-out the CTA raises a shared abort flag, writes
// an error code for the host, waits (bounded) for its issued MMAs and frees
// its TMEM before returning.
#include "ops.cuh"

#include <algorithm>
#include <mutex>

namespace baemm
{
namespace
{

constexpr int TC_M = 128;          // targets per CTA (TMEM lanes)
constexpr int TC_SRC = 16;         // sources per K tile
constexpr int TC_N = 32;           // MMA N: 16 columns as (re | im)
constexpr int TC_CHMAX = 4;        // chunks per work unit
constexpr int TC_MAXCHUNKS = 32;   // wave_count <= 512 with wave_chunk_size 16
constexpr int TC_GEN_THREADS = 256;
constexpr int TC_EXP_THREADS = 64;
constexpr int TC_THREADS = TC_GEN_THREADS + TC_EXP_THREADS + 64;   // + TMA producer warp + MMA warp
constexpr int TC_ASTAGES = 4;      // A stages in TMEM (one chunk of one tile each)
constexpr int TC_BSTAGES = 3;      // expanded B image stages in shared memory
constexpr int TC_RSTAGES = 6;      // raw tile stages filled by bulk copies
constexpr uint32_t TC_TMEM_COLS = 512;
constexpr uint32_t TC_ACC_COLS = TC_CHMAX * TC_N;    // one accumulator buffer (128 columns)
constexpr uint32_t TC_ACOL = 2 * TC_ACC_COLS;        // A stages after two accumulator buffers
constexpr int TC_IMG = TC_N * 128;                   // one K-major SW128 image: 32 rows x 128 B
constexpr uint64_t kWaitNs = 200ull * 1000 * 1000;   // 200 ms per wait (a pipeline stage takes microseconds)

// Raw tile: the 16 source rows of B_tri (this CTA's columns) plus their
// midpoints and normals, filled by cp.async.bulk.
struct TcRaw
{
    float2 b[TC_SRC][TC_CHMAX * 16];   // 8 KB
    float4 y[TC_SRC];
    float4 mu[TC_SRC];
};

struct __align__(1024) TcSmem
{
    uint8_t img[TC_BSTAGES][TC_CHMAX][2][TC_IMG];   // [stage][chunk][hi, lo]
    TcRaw raw[TC_RSTAGES];
    uint64_t a_full[TC_ASTAGES], a_empty[TC_ASTAGES];
    uint64_t b_full[TC_BSTAGES], b_empty[TC_BSTAGES];
    uint64_t r_full[TC_RSTAGES], r_empty[TC_RSTAGES];
    uint64_t seg_full[2], seg_empty[2];
    uint32_t tmem_base;
    int abort_flag;
    float4 prm[TC_MAXCHUNKS][2];   // (kappa, c1.x, c1.y, c2.x), (c2.y, c3.x, c3.y, 0)
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// try_wait with a suspend-time hint: the thread sleeps in hardware until the
// phase completes (or the hint runs out) instead of spinning.
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity), "r"(20000u)
                 : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait (at most kWaitNs of wall time).  Returns false when the CTA is
// aborting: the shared flag was raised by another thread, another CTA has
// already reported an error, or this wait ran out (then it raises the flag and
// writes `code` to the error word).
__device__ __forceinline__ bool wait_bar(uint64_t *bar, uint32_t parity, volatile int *abort_flag, int *err,
                                         int code, bool honour_abort = true)
{
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 1;; ++it)
    {
        if (mbar_try_wait(bar, parity)) return true;
        if (honour_abort && *abort_flag) return false;
        if ((it & 63u) == 0)
        {
            if (honour_abort && *(volatile int *)err) return false;
            if (global_ns() - t0 > kWaitNs) break;
        }
    }
    *abort_flag = 1;
    atomicExch(err, code);
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Round an FP32 value to TF32 (10 stored mantissa bits), to nearest with ties
// away from zero, as an integer add on the bit pattern: adding half a TF32 ulp
// to the magnitude and clearing the 13 low bits.  A mantissa carry moves into
// the exponent, which is the correct rounding.  Only used on finite values of
// moderate size (kernel entries and right-hand sides), so Inf/NaN and overflow
// past FLT_MAX need no handling.
__device__ __forceinline__ uint32_t to_tf32(float x) { return (__float_as_uint(x) + 0x1000u) & 0xffffe000u; }

// hi = tf32(x) (round to nearest), lo = x - hi exactly in FP32.  The tensor
// core reads the top 19 bits of lo; |lo| <= 2^-11 |x|, so the bits it drops
// are below 2^-21 |x|.
__device__ __forceinline__ void split_tf32(float x, uint32_t &hi, uint32_t &lo)
{
    hi = to_tf32(x);
    lo = __float_as_uint(x - __uint_as_float(hi));
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&v)[16])
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                 "%13, %14, %15, %16};" ::"r"(taddr),
                 "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]),
                 "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
                 : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&v)[8])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr)
                 : "memory");
}

// Shared-memory matrix descriptor: K-major, SWIZZLE_128B, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t sw128_desc(const void *p)
{
    const uint32_t a = smem_u32(p);
    uint64_t d = 0;
    d |= (uint64_t)((a >> 4) & 0x3FFF);          // start address
    d |= (uint64_t)1 << 16;                      // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;            // stride byte offset
    d |= (uint64_t)1 << 46;                      // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;                      // SWIZZLE_128B
    return d;
}

// Instruction descriptor: D F32, A/B TF32, both K-major, N = 32, M = 128.
constexpr uint32_t kIdescTf32 = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                                ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
                 "r"(a_tmem), "l"(b_desc), "r"(kIdescTf32), "r"(accumulate)
                 : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Untiled bulk copy global -> shared (no multicast); 16-byte aligned, size multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Byte offset of the 16-byte group of sources (2 sp, 2 sp + 1), i.e. K
// elements 4 sp .. 4 sp + 3, of row `row` in a K-major SWIZZLE_128B image.
__device__ __forceinline__ uint32_t img_off16(int row, int sp) { return (uint32_t)(row * 128 + ((sp ^ (row & 7)) << 4)); }

// The partition of the unit range over the persistent grid.
struct TcPlan
{
    int n, wc, nblk, ntiles, ncg, seg_tiles;
    int64_t units;   // ncg * nblk * ntiles
    int ctas;        // grid size (<= units)
};

__host__ __device__ __forceinline__ int64_t tc_start(const TcPlan &p, int k) { return (int64_t)k * p.units / p.ctas; }
// The CTA whose range holds unit x.
__host__ __device__ __forceinline__ int tc_cta_of(const TcPlan &p, int64_t x)
{
    return (int)(((x + 1) * p.ctas - 1) / p.units);
}

// Walks a CTA's unit range as pieces (cg, blk, tiles [tb, te)).
struct PieceIter
{
    int64_t u, u1;
    int per_cg;
    __device__ PieceIter(const TcPlan &p, int k) : u(tc_start(p, k)), u1(tc_start(p, k + 1)), per_cg(p.nblk * p.ntiles) {}
    __device__ bool next(const TcPlan &p, int &cg, int &blk, int &tb, int &te)
    {
        if (u >= u1) return false;
        cg = (int)(u / per_cg);
        const int rem = (int)(u - (int64_t)cg * per_cg);
        blk = rem / p.ntiles;
        tb = rem - blk * p.ntiles;
        te = (int)min((int64_t)p.ntiles, (int64_t)tb + (u1 - u));
        u += te - tb;
        return true;
    }
};

template <int CH, bool SL, bool DL, bool ADL>
__global__ void __launch_bounds__(TC_THREADS, 1)
boundary_tc_kernel(const float *__restrict__ mid4, const float *__restrict__ nrm4, const float2 *__restrict__ Btri,
                   float2 *__restrict__ Ctri, float2 *__restrict__ ws, const ChunkParamsF *__restrict__ prm,
                   const TcPlan plan, int *err)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // Align inside the shared window by pointer arithmetic on the shared array,
    // so every access below compiles to a shared-memory instruction.
    TcSmem &sm = *reinterpret_cast<TcSmem *>(smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u));
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int n = plan.n, wc = plan.wc, ntiles = plan.ntiles;
    const int S = plan.seg_tiles;   // tiles per TMEM partial sum
    const int k_cta = blockIdx.x;
    volatile int *abort_flag = &sm.abort_flag;
    // An earlier CTA gave up: do nothing.  Read once and shared, so the exit is
    // CTA-uniform and happens before any barrier init or TMEM allocation.
    if (tid == 0) sm.abort_flag = *(volatile int *)err;
    __syncthreads();
    if (sm.abort_flag != 0) return;
    __syncthreads();

    if (tid == 0)
    {
        for (int k = 0; k < TC_ASTAGES; ++k) { mbar_init(&sm.a_full[k], TC_GEN_THREADS); mbar_init(&sm.a_empty[k], 1); }
        for (int k = 0; k < TC_BSTAGES; ++k) { mbar_init(&sm.b_full[k], TC_EXP_THREADS); mbar_init(&sm.b_empty[k], 1); }
        for (int k = 0; k < TC_RSTAGES; ++k)
        {
            mbar_init(&sm.r_full[k], 1);
            mbar_init(&sm.r_empty[k], TC_GEN_THREADS + TC_EXP_THREADS);
        }
        for (int k = 0; k < 2; ++k) { mbar_init(&sm.seg_full[k], 1); mbar_init(&sm.seg_empty[k], TC_GEN_THREADS); }
        sm.abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int c = tid; c < wc / 16; c += blockDim.x)
    {
        const ChunkParamsF p = prm[c];
        sm.prm[c][0] = make_float4(p.kappa, p.c[1].x, p.c[1].y, p.c[2].x);
        sm.prm[c][1] = make_float4(p.c[2].y, p.c[3].x, p.c[3].y, 0.f);
    }
    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem_base)),
                     "r"(TC_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = sm.tmem_base;

    if (tid < TC_GEN_THREADS)
    {
        // ------------------------------ generators ------------------------------
        const int q = warp & 3, g = warp >> 2;
        const uint32_t lane_addr = tbase + ((uint32_t)(q * 32) << 16);
        float2 racc[CH][8];
        bool ok = true;
        int pending = -1;   // A stage written but not yet published
        int T = 0, SG = 0;  // tiles and TMEM segments handled so far by this CTA
        auto publish = [&]() {
            if (pending >= 0)
            {
                asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
                tc_fence_before();
                mbar_arrive(&sm.a_full[pending]);
                pending = -1;
            }
        };
        // add the finished TMEM partial sum of segment `sg` to the registers
        auto drain = [&](int sg) {
            const int buf = sg & 1;
            const bool got = wait_bar(&sm.seg_full[buf], (uint32_t)(sg >> 1) & 1u, abort_flag, err, 2);
            if (!__all_sync(0xffffffffu, got)) return false;
            tc_fence_after();
            #pragma unroll
            for (int c = 0; c < CH; ++c)
            {
                uint32_t re[8], im[8];
                const uint32_t col = (uint32_t)buf * TC_ACC_COLS + (uint32_t)(c * TC_N + g * 8);
                tmem_ld8(lane_addr + col, re);
                tmem_ld8(lane_addr + col + 16u, im);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                #pragma unroll
                for (int k = 0; k < 8; ++k)
                {
                    racc[c][k].x += __uint_as_float(re[k]);
                    racc[c][k].y += __uint_as_float(im[k]);
                }
            }
            tc_fence_before();
            mbar_arrive(&sm.seg_empty[buf]);
            return true;
        };
        PieceIter it(plan, k_cta);
        int cg, blk, tb, te;
        bool first_piece = true;
        while (ok && it.next(plan, cg, blk, tb, te))
        {
            const int i = blk * TC_M + q * 32 + lane;
            float x0 = 0.f, x1 = 0.f, x2 = 0.f, n0 = 0.f, n1 = 0.f, n2 = 0.f;
            if (i < n)
            {
                const float4 m = reinterpret_cast<const float4 *>(mid4)[i];
                x0 = m.x; x1 = m.y; x2 = m.z;
                if (ADL)
                {
                    const float4 v = reinterpret_cast<const float4 *>(nrm4)[i];
                    n0 = v.x; n1 = v.y; n2 = v.z;
                }
            }
            #pragma unroll
            for (int c = 0; c < CH; ++c)
                #pragma unroll
                for (int k = 0; k < 8; ++k) racc[c][k] = make_float2(0.f, 0.f);
            for (int t = tb; t < te; ++t, ++T)
            {
                const int rs = T % TC_RSTAGES;
                {
                    const bool got = wait_bar(&sm.r_full[rs], (uint32_t)(T / TC_RSTAGES) & 1u, abort_flag, err, 1);
                    if (!__all_sync(0xffffffffu, got)) { ok = false; break; }
                }
                // per source: 1/r, r, (z.mu_j)/r^2, (z.nu_i)/r^2; shared by every chunk
                float rinv[8], r[8], dmu[8], dnu[8];
                #pragma unroll
                for (int s8 = 0; s8 < 8; ++s8)
                {
                    const int sl = g * 8 + s8, j = t * TC_SRC + sl;
                    // rows past the end were not copied: never read them
                    const bool inside = j < n;
                    const float4 y = inside ? sm.raw[rs].y[sl] : make_float4(x0, x1, x2, 0.f);
                    const float zx = y.x - x0, zy = y.y - x1, zz = y.z - x2;
                    const bool valid = inside && (j != i);
                    const float r2 = zx * zx + zy * zy + zz * zz;
                    rinv[s8] = valid ? rsqrtf(r2) : 0.f;
                    r[s8] = r2 * rinv[s8];
                    const float rinv2 = rinv[s8] * rinv[s8];
                    if (DL)
                    {
                        const float4 mu = inside ? sm.raw[rs].mu[sl] : make_float4(0.f, 0.f, 0.f, 0.f);
                        dmu[s8] = (zx * mu.x + zy * mu.y + zz * mu.z) * rinv2;
                    }
                    if (ADL) dnu[s8] = (zx * n0 + zy * n1 + zz * n2) * rinv2;
                }
                mbar_arrive(&sm.r_empty[rs]);
                for (int c = 0; c < CH; ++c)
                {
                    const float4 p0 = sm.prm[cg * CH + c][0], p1 = sm.prm[cg * CH + c][1];
                    const float kap = p0.x;
                    const float c1x = p0.y, c1y = p0.z, c2x = p0.w, c2y = p1.x, c3x = p1.y, c3y = p1.z;
                    uint32_t hi[16], lo[16];
                    #pragma unroll
                    for (int s8 = 0; s8 < 8; ++s8)
                    {
                        // A = e^{i k r} g / r,  g = c1 + w (i k r - 1),  w = (c2 (z.mu_j) - c3 (z.nu_i)) / r^2
                        const float kr = kap * r[s8];
                        float sn, cs;
                        __sincosf(kr, &sn, &cs);
                        float gx = SL ? c1x : 0.f, gy = SL ? c1y : 0.f;
                        if (DL || ADL)
                        {
                            float wx = 0.f, wy = 0.f;
                            if (DL) { wx = c2x * dmu[s8]; wy = c2y * dmu[s8]; }
                            if (ADL) { wx -= c3x * dnu[s8]; wy -= c3y * dnu[s8]; }
                            gx = gx - wx - kr * wy;
                            gy = gy - wy + kr * wx;
                        }
                        const float tx = gx * rinv[s8], ty = gy * rinv[s8];
                        const float ax = cs * tx - sn * ty;
                        const float ay = sn * tx + cs * ty;
                        split_tf32(ax, hi[2 * s8], lo[2 * s8]);
                        split_tf32(ay, hi[2 * s8 + 1], lo[2 * s8 + 1]);
                    }
                    // publish the previous stage now that its stores had this chunk's math to land
                    publish();
                    const int u = T * CH + c;
                    const int stage = u % TC_ASTAGES;
                    bool got = true;
                    if (u >= TC_ASTAGES)
                        got = wait_bar(&sm.a_empty[stage], (uint32_t)((u / TC_ASTAGES) - 1) & 1u, abort_flag, err, 3);
                    // the tcgen05 stores below are warp-collective: the warp agrees on the outcome
                    if (!__all_sync(0xffffffffu, got)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t acol = TC_ACOL + (uint32_t)stage * 64u + (uint32_t)g * 16u;
                    tmem_st16(lane_addr + acol, hi);
                    tmem_st16(lane_addr + acol + 32u, lo);
                    pending = stage;
                }
                if (!ok) break;
                const int lt = t - tb;
                if (lt % S == S - 1 || t == te - 1)
                {
                    // segment SG finished generating: drain the previous one of this piece
                    publish();
                    if (lt >= S && !drain(SG - 1)) { ok = false; break; }
                    if (t == te - 1 && !drain(SG)) { ok = false; break; }
                    ++SG;
                }
            }
            if (!ok) break;
            // ------------------------------ piece epilogue ------------------------------
            const int cw = CH * 16;
            if (tb == 0 && te == ntiles)
            {
                if (i < n)
                {
                    #pragma unroll
                    for (int c = 0; c < CH; ++c)
                    {
                        float4 *out = reinterpret_cast<float4 *>(&Ctri[(int64_t)i * wc + cg * cw + c * 16 + g * 8]);
                        #pragma unroll
                        for (int k = 0; k < 8; k += 2)
                            out[k / 2] = make_float4(racc[c][k].x, racc[c][k].y, racc[c][k + 1].x, racc[c][k + 1].y);
                    }
                }
            }
            else
            {
                const int slot = first_piece ? 0 : 1;
                const int row = q * 32 + lane;
                #pragma unroll
                for (int c = 0; c < CH; ++c)
                {
                    float4 *out = reinterpret_cast<float4 *>(
                        &ws[((int64_t)(k_cta * 2 + slot) * TC_M + row) * (TC_CHMAX * 16) + c * 16 + g * 8]);
                    #pragma unroll
                    for (int k = 0; k < 8; k += 2)
                        out[k / 2] = make_float4(racc[c][k].x, racc[c][k].y, racc[c][k + 1].x, racc[c][k + 1].y);
                }
            }
            first_piece = false;
        }
        if (!ok) publish();
    }
    else if (tid < TC_GEN_THREADS + TC_EXP_THREADS)
    {
        // ------------------------------ expanders ------------------------------
        // item = (16-byte group of sources sp, chunk c, row pair qq / qq + 16);
        // 8 lanes of a quarter-warp write 8 different rows' swizzled 16-byte
        // groups, which cover all 32 banks.
        const int lt = tid - TC_GEN_THREADS;
        constexpr int items = (TC_SRC / 2) * CH * 16;
        PieceIter it(plan, k_cta);
        int cg, blk, tb, te, T = 0;
        bool ok = true;
        while (ok && it.next(plan, cg, blk, tb, te))
        {
            for (int t = tb; t < te; ++t, ++T)
            {
                const int rs = T % TC_RSTAGES, b = T % TC_BSTAGES;
                if (!wait_bar(&sm.r_full[rs], (uint32_t)(T / TC_RSTAGES) & 1u, abort_flag, err, 4)) { ok = false; break; }
                if (T >= TC_BSTAGES &&
                    !wait_bar(&sm.b_empty[b], (uint32_t)((T / TC_BSTAGES) - 1) & 1u, abort_flag, err, 5))
                {
                    ok = false;
                    break;
                }
                const int nsrc = n - t * TC_SRC;   // valid rows in this tile (may exceed 16)
                #pragma unroll 2
                for (int e = lt; e < items; e += TC_EXP_THREADS)
                {
                    const int qq = e & 15, sp = (e >> 4) & 7, c = e >> 7;
                    const int s0 = 2 * sp, s1 = s0 + 1;
                    const float2 v0 = (s0 < nsrc) ? sm.raw[rs].b[s0][c * 16 + qq] : make_float2(0.f, 0.f);
                    const float2 v1 = (s1 < nsrc) ? sm.raw[rs].b[s1][c * 16 + qq] : make_float2(0.f, 0.f);
                    uint32_t hr0, lr0, hi0, li0, hr1, lr1, hi1, li1;
                    split_tf32(v0.x, hr0, lr0);
                    split_tf32(v0.y, hi0, li0);
                    split_tf32(v1.x, hr1, lr1);
                    split_tf32(v1.y, hi1, li1);
                    constexpr uint32_t sgn = 0x80000000u;
                    uint8_t *hi_img = sm.img[b][c][0];
                    uint8_t *lo_img = sm.img[b][c][1];
                    // row qq: (re, -im) per source; row qq + 16: (im, re)
                    *reinterpret_cast<uint4 *>(hi_img + img_off16(qq, sp)) = make_uint4(hr0, hi0 ^ sgn, hr1, hi1 ^ sgn);
                    *reinterpret_cast<uint4 *>(lo_img + img_off16(qq, sp)) = make_uint4(lr0, li0 ^ sgn, lr1, li1 ^ sgn);
                    *reinterpret_cast<uint4 *>(hi_img + img_off16(qq + 16, sp)) = make_uint4(hi0, hr0, hi1, hr1);
                    *reinterpret_cast<uint4 *>(lo_img + img_off16(qq + 16, sp)) = make_uint4(li0, lr0, li1, lr1);
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                mbar_arrive(&sm.r_empty[rs]);
                mbar_arrive(&sm.b_full[b]);
            }
        }
    }
    else if (warp == (TC_GEN_THREADS + TC_EXP_THREADS) / 32)
    {
        // ------------------------------ bulk-copy producer ------------------------------
        if (lane == 0)
        {
            const int cw = CH * 16;
            const uint32_t row_bytes = (uint32_t)(cw * sizeof(float2));
            PieceIter it(plan, k_cta);
            int cg, blk, tb, te, T = 0;
            bool ok = true;
            while (ok && it.next(plan, cg, blk, tb, te))
            {
                for (int t = tb; t < te; ++t, ++T)
                {
                    const int rs = T % TC_RSTAGES;
                    if (T >= TC_RSTAGES &&
                        !wait_bar(&sm.r_empty[rs], (uint32_t)((T / TC_RSTAGES) - 1) & 1u, abort_flag, err, 6))
                    {
                        ok = false;
                        break;
                    }
                    const int j0 = t * TC_SRC;
                    const int rows = min(TC_SRC, n - j0);
                    mbar_expect_tx(&sm.r_full[rs], (uint32_t)rows * (row_bytes + 32u));
                    bulk_g2s(sm.raw[rs].y, mid4 + 4 * (int64_t)j0, (uint32_t)rows * 16u, &sm.r_full[rs]);
                    bulk_g2s(sm.raw[rs].mu, nrm4 + 4 * (int64_t)j0, (uint32_t)rows * 16u, &sm.r_full[rs]);
                    // one contiguous block when the tile's rows are whole B_tri rows of
                    // exactly the raw row width; otherwise one copy per row
                    if (CH == TC_CHMAX && cw == wc)
                        bulk_g2s(sm.raw[rs].b, Btri + (int64_t)j0 * wc, (uint32_t)rows * row_bytes, &sm.r_full[rs]);
                    else
                        for (int sl = 0; sl < rows; ++sl)
                            bulk_g2s(sm.raw[rs].b[sl], Btri + (int64_t)(j0 + sl) * wc + cg * cw, row_bytes,
                                     &sm.r_full[rs]);
                }
            }
        }
    }
    else if (lane == 0)
    {
        // ------------------------------ MMA issuer ------------------------------
        bool ok = true;
        int T = 0, SG = 0;
        PieceIter it(plan, k_cta);
        int cg, blk, tb, te;
        while (ok && it.next(plan, cg, blk, tb, te))
        {
            for (int t = tb; t < te; ++t, ++T)
            {
                const int b = T % TC_BSTAGES;
                const int lt = t - tb;
                const int buf = SG & 1;
                const bool first = (lt % S) == 0;
                if (!wait_bar(&sm.b_full[b], (uint32_t)(T / TC_BSTAGES) & 1u, abort_flag, err, 7)) { ok = false; break; }
                if (first && SG >= 2 &&
                    !wait_bar(&sm.seg_empty[buf], (uint32_t)((SG >> 1) - 1) & 1u, abort_flag, err, 8))
                {
                    ok = false;
                    break;
                }
                for (int c = 0; c < CH; ++c)
                {
                    const int u = T * CH + c;
                    const int stage = u % TC_ASTAGES;
                    if (!wait_bar(&sm.a_full[stage], (uint32_t)(u / TC_ASTAGES) & 1u, abort_flag, err, 9))
                    {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t d = tbase + (uint32_t)buf * TC_ACC_COLS + (uint32_t)(c * TC_N);
                    const uint32_t a_hi = tbase + TC_ACOL + (uint32_t)stage * 64u;
                    const uint32_t a_lo = a_hi + 32u;
                    const uint64_t b_hi = sw128_desc(sm.img[b][c][0]);
                    const uint64_t b_lo = sw128_desc(sm.img[b][c][1]);
                    #pragma unroll
                    for (int ks = 0; ks < 4; ++ks)
                    {
                        const uint64_t koff = (uint64_t)(ks * 32 >> 4);
                        mma_tf32(d, a_lo + 8u * ks, b_hi + koff, (!first || ks > 0) ? 1u : 0u);
                        mma_tf32(d, a_hi + 8u * ks, b_lo + koff, 1u);
                        mma_tf32(d, a_hi + 8u * ks, b_hi + koff, 1u);
                    }
                    mma_commit(&sm.a_empty[stage]);
                }
                if (!ok) break;
                mma_commit(&sm.b_empty[b]);
                if (lt % S == S - 1 || t == te - 1)
                {
                    mma_commit(&sm.seg_full[buf]);
                    ++SG;
                }
            }
        }
        if (!ok)
        {
            // wait (bounded) for the MMAs already issued before the TMEM is freed
            const int buf = SG & 1;
            mma_commit(&sm.seg_full[buf]);
            wait_bar(&sm.seg_full[buf], (uint32_t)((SG >> 1) & 1), abort_flag, err, 10, false);
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 0)
    {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TC_TMEM_COLS) : "memory");
    }
}

// Adds the workspace slots of every target block that was split between CTAs,
// in CTA order, and writes the block's rows of C_tri.
__global__ void tc_fixup_kernel(const float2 *__restrict__ ws, float2 *__restrict__ Ctri, const TcPlan plan, int cw)
{
    const int cg = blockIdx.x / plan.nblk, blk = blockIdx.x - cg * plan.nblk;
    const int64_t lo = ((int64_t)cg * plan.nblk + blk) * plan.ntiles, hi = lo + plan.ntiles;
    const int k_first = tc_cta_of(plan, lo), k_last = tc_cta_of(plan, hi - 1);
    if (k_first == k_last) return;   // written directly by its CTA
    for (int e = threadIdx.x; e < TC_M * cw; e += blockDim.x)
    {
        const int row = e / cw, col = e - row * cw;
        const int i = blk * TC_M + row;
        if (i >= plan.n) continue;
        float2 acc = make_float2(0.f, 0.f);
        for (int k = k_first; k <= k_last; ++k)
        {
            const int slot = (tc_start(plan, k) >= lo) ? 0 : 1;   // the CTA's first piece, or its last
            const float2 v = ws[((int64_t)(k * 2 + slot) * TC_M + row) * (TC_CHMAX * 16) + col];
            acc.x += v.x;
            acc.y += v.y;
        }
        Ctri[(int64_t)i * plan.wc + cg * cw + col] = acc;
    }
}

template <int CH, bool SL, bool DL, bool ADL>
void tc_launch(cudaStream_t st, const float *mid, const float *nrm, const float2 *B, float2 *C, float2 *ws,
               const ChunkParamsF *p, const TcPlan &plan, int *err)
{
    // More than half of the SM's shared memory, so one CTA per SM: the CTA
    // allocates all 512 TMEM columns and a second resident CTA would only wait.
    const size_t bytes = std::max(sizeof(TcSmem) + 1024, (size_t)(116 * 1024));
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [&] {
        attr = cudaFuncSetAttribute(boundary_tc_kernel<CH, SL, DL, ADL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)bytes);
    });
    BAEMM_CUDA(attr);
    boundary_tc_kernel<CH, SL, DL, ADL><<<plan.ctas, TC_THREADS, bytes, st>>>(mid, nrm, B, C, ws, p, plan, err);
}

template <int CH>
void tc_flags(int code, cudaStream_t st, const float *mid, const float *nrm, const float2 *B, float2 *C, float2 *ws,
              const ChunkParamsF *p, const TcPlan &plan, int *err)
{
    switch (code)
    {
        case 1: tc_launch<CH, true, false, false>(st, mid, nrm, B, C, ws, p, plan, err); break;
        case 2: tc_launch<CH, false, true, false>(st, mid, nrm, B, C, ws, p, plan, err); break;
        case 3: tc_launch<CH, true, true, false>(st, mid, nrm, B, C, ws, p, plan, err); break;
        case 4: tc_launch<CH, false, false, true>(st, mid, nrm, B, C, ws, p, plan, err); break;
        case 5: tc_launch<CH, true, false, true>(st, mid, nrm, B, C, ws, p, plan, err); break;
        case 6: tc_launch<CH, false, true, true>(st, mid, nrm, B, C, ws, p, plan, err); break;
        case 7: tc_launch<CH, true, true, true>(st, mid, nrm, B, C, ws, p, plan, err); break;
        default: break;
    }
}

int device_sm_count()
{
    int dev = 0;
    BAEMM_CUDA(cudaGetDevice(&dev));
    static std::mutex mu;
    static int cached[64] = {};
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 0 || dev >= 64) return 148;
    if (cached[dev] == 0) BAEMM_CUDA(cudaDeviceGetAttribute(&cached[dev], cudaDevAttrMultiProcessorCount, dev));
    return cached[dev];
}

} // namespace

bool tc_supported(int wc, int wcs) { return wcs == 16 && wc % 16 == 0 && wc <= 16 * TC_MAXCHUNKS; }

size_t tc_workspace_elems(int ctas)
{
    if (ctas <= 0) ctas = device_sm_count();
    return (size_t)ctas * 2 * TC_M * TC_CHMAX * 16;
}

void launch_boundary_tc(const MeshDev &m, const OpFlags &f, const void *chunk_params, int wc, int wcs,
                        const float2 *Btri, float2 *Ctri, float2 *ws, size_t ws_elems, int *err, cudaStream_t st,
                        int seg_tiles, int ctas)
{
    BAEMM_REQUIRE(tc_supported(wc, wcs), BAEMM_ERR_SIZE,
                  "tensor-core apply needs wave_chunk_size 16 and wave_count <= 512");
    if (!f.any_layer() || m.nt == 0) return;
    TcPlan plan;
    plan.n = (int)m.nt;
    plan.wc = wc;
    const int CH = (wc % 64 == 0) ? 4 : (wc % 32 == 0) ? 2 : 1;
    plan.ncg = wc / (16 * CH);
    plan.nblk = ceil_div(plan.n, TC_M);
    plan.ntiles = ceil_div(plan.n, TC_SRC);
    plan.seg_tiles = std::max(1, seg_tiles);
    plan.units = (int64_t)plan.ncg * plan.nblk * plan.ntiles;
    if (ctas <= 0) ctas = device_sm_count();
    plan.ctas = (int)std::min<int64_t>(ctas, plan.units);
    BAEMM_REQUIRE(ws && ws_elems >= tc_workspace_elems(plan.ctas), BAEMM_ERR_ARG, "tensor-core workspace too small");
    const int code = (f.sl() ? 1 : 0) | (f.dl() ? 2 : 0) | (f.adl() ? 4 : 0);
    const auto *p = static_cast<const ChunkParamsF *>(chunk_params);
    const float *mid = m.mid_f, *nrm = m.nrm_f;
    if (CH == 4) tc_flags<4>(code, st, mid, nrm, Btri, Ctri, ws, p, plan, err);
    else if (CH == 2) tc_flags<2>(code, st, mid, nrm, Btri, Ctri, ws, p, plan, err);
    else tc_flags<1>(code, st, mid, nrm, Btri, Ctri, ws, p, plan, err);
    BAEMM_LAUNCH_CHECK();
    tc_fixup_kernel<<<plan.ncg * plan.nblk, 256, 0, st>>>(ws, Ctri, plan, CH * 16);
    BAEMM_LAUNCH_CHECK();
}

} // namespace baemm
