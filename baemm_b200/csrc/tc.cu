// Compensated tensor-core form of the dense boundary kernel (sm_100a, tcgen05).
//
// The apply C_i = sum_j A_ij(kappa) B_j of BoundaryOperatorKernel.cl:5-239 as
// a real GEMM per wave chunk (16 right-hand sides):
//     [C_re | C_im]  (128 x 32)  =  A  (128 x 2S)  x  Bimg^T  (2S x 32)
// with the K index ordered by source pairs (s0, s1) = (2p, 2p + 1):
//     A[i][4p .. 4p+3]      = (Re A_is0, Re A_is1, Im A_is0, Im A_is1),
//     Bimg[q][4p .. 4p+3]   = (Re b_s0q, Re b_s1q, -Im b_s0q, -Im b_s1q),
//     Bimg[16+q][4p .. 4p+3] = (Im b_s0q, Im b_s1q, Re b_s0q, Re b_s1q)   (q < 16),
// so that the generators evaluate two sources per packed FP32x2 instruction
// and each packed result is already in the register order of the TMEM store.
// Operands are split into TF32 hi + lo parts and the product is compensated:
//     A B ~= Ahi Bhi + Alo Bhi + Ahi Blo       (FP32 accumulation in TMEM),
// issued as two MMAs per K step: Ahi [Bhi | Blo] (N = 64, into a main and a
// correction half of the chunk's accumulator) and Alo Bhi (N = 32, into the
// correction half); a tcgen05.mma costs about the same for N = 32 and 64.
// which keeps ~21 bits per product (TF32 hi+lo), well inside 1e-5 relative.
//
// Work unit = (group of up to 4 chunks, block of 128 targets, 16-source tile).
// The grid is persistent (one CTA per SM, it holds all 512 TMEM columns).
// Whole target blocks are dealt out in waves (all CTAs sweep the source tiles
// in step, so the tiles in use stay cached); the blocks left over after the
// last full wave are split evenly by tiles ("stream-K").  A piece covering a
// whole block writes C_tri; a partial piece (at most the first and the last
// tail piece of a CTA) writes its partial sums to a workspace slot, and
// tc_fixup_kernel adds the slots of each split block in CTA order
// (deterministic).
// Warp roles (GW generator warps + 1 + 2 = 19 or 11 warps):
//   warps 0 .. GW-1  generators: thread (lane quarter q = warp % 4, group
//               g = warp / 4) owns target row 32 q + lane and 16 / (GW / 4)
//               sources of each 16-source K tile; it evaluates the kernel
//               entries in registers, two sources per FP32x2 instruction
//               (geometry shared by all chunks), splits them into hi / lo and
//               writes them straight into TMEM (tcgen05.st), so the A operand
//               never touches shared memory;
//   warp GW     bulk-copy producer: cp.async.bulk (no multicast) of the tile's
//               geometry and of its B images, expanded once per apply by
//               tc_expand_kernel, into shared memory;
//   warps GW+1, GW+2  MMA issuers, every other entry set each (a chunk, or
//               R chunks of one wavenumber sharing their entries; one issuer
//               when a tile has a single set): 8 tcgen05.mma (kind::tf32, A
//               from TMEM, B from shared memory, M 128, K 8) per set and tile.
// Pipelines use mbarriers (A stages in TMEM, B and geometry stages in shared
// memory).  All roles wait with mbarrier.try_wait, which suspends the warp in
// hardware.
// Every wait is bounded: on time-out the CTA raises a shared abort flag, writes
// an error code for the host, waits (bounded) for its issued MMAs and frees
// its TMEM before returning.
#include "ops.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <utility>
#include <vector>
#include <cstddef>
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
// Generator warps GW = 16 (4 per SM sub-partition, 4 sources per thread and
// tile) or 8 (8 sources per thread); the autotuner picks one per problem
// shape.  16 hide the latency of the entry evaluation better on large blocks.
template <int GW>
struct TcShape
{
    static_assert(GW == 8 || GW == 16, "8 or 16 generator warps");
    static constexpr int GEN_THREADS = 32 * GW;
    static constexpr int GROUPS = GW / 4;        // source groups of a tile (4 warps cover the 128 rows)
    static constexpr int SPT = 16 / GROUPS;      // sources per generator thread and tile
    static constexpr int PPT = SPT / 2;          // their pairs
    static constexpr int KPT = 2 * SPT;          // their K columns of an A stage
    static constexpr int CPG = 16 / GROUPS;      // right-hand sides per thread in the drain
};
// MMA-issuing warps of a block: two (each takes every other chunk), so that
// the issue work of a tile is split between two SM sub-partitions.  The
// register file is split between the sub-partitions, so a block's register
// cap is set by the sub-partition with the most warps: 16 generator warps +
// the bulk-copy warp + 2 issuers are 19 warps (5 on a sub-partition, 96
// registers); one issuer per chunk would make 21 (6, 80 registers: the
// generators spill).  With 8 generator warps, 4 issuers measured slower than
// 2 (128 instead of 168 registers for the generators).
// With R > 1 the R groups of an entry set share one A stage and one issuer,
// so the issuers split the CH / R entry sets of a tile.
template <int GW, int CH, int R>
constexpr int tc_mma_warps() { return CH / R >= 2 ? 2 : 1; }
// generators + the bulk-copy warp + the MMA issuers
template <int GW, int CH, int R>
constexpr int tc_threads() { return 32 * GW + 32 + 32 * tc_mma_warps<GW, CH, R>(); }
constexpr int TC_BSTAGES = 4;      // B image stages in shared memory (bulk copies of the expanded images)
constexpr int TC_RSTAGES = 6;      // tile geometry stages (bulk copies)
constexpr uint32_t TC_TMEM_COLS = 512;
// per chunk: main (Ahi Bhi) and correction (Ahi Blo + Alo Bhi) accumulators;
// an entry set of R chunks holds its R main parts, then its R corrections
constexpr uint32_t TC_DCOLS = 2 * TC_N;
// A stages in TMEM (one chunk of one tile each, 64 columns) take the columns
// after the accumulator of a CH-chunk work unit: 4 stages for 4 chunks, 6 for
// 2, 7 for 1.  Within a stage, K step ks (8 K columns) has its hi part at
// columns 16 ks .. 16 ks + 7 and its lo part right after, so a generator
// thread writes the hi and lo parts of its K step with one 16-column store
// (1.3 % faster than separate hi and lo halves of the stage).
template <int CH>
constexpr int tc_astages() { return (int)(TC_TMEM_COLS / TC_DCOLS) - CH; }
constexpr int TC_ASTAGES_MAX = (int)(TC_TMEM_COLS / TC_DCOLS) - 1;
constexpr int TC_IMG = TC_N * 128;                   // one K-major SW128 image: 32 rows x 128 B
constexpr uint64_t kWaitNs = 200ull * 1000 * 1000;   // 200 ms per wait (a pipeline stage takes microseconds)

// Source geometry of one 16-source tile, structure of arrays (built once per
// mesh by tc_tile_geometry_kernel; padding sources past the end are zero).
struct TcTileGeo
{
    float x[TC_SRC], y[TC_SRC], z[TC_SRC];      // midpoints
    float mx[TC_SRC], my[TC_SRC], mz[TC_SRC];   // unit normals
};
static_assert(sizeof(TcTileGeo) % 16 == 0, "bulk copies move multiples of 16 bytes");

// The right-hand sides of one 16-source tile and one 16-column group as the
// MMA's B operand: the hi and the lo image (32 rows each, 8 KB; ordered within
// an entry set as tc_expand_kernel describes), expanded once per apply into
// global memory and bulk-copied into a B stage as they are.
constexpr int TC_GROUP_BYTES = 2 * TC_IMG;

struct __align__(1024) TcSmem
{
    uint8_t img[TC_BSTAGES][TC_CHMAX][2][TC_IMG];   // per stage the unit's images as tc_expand_kernel lays them out
    TcTileGeo geo[TC_RSTAGES];
    uint64_t a_full[TC_ASTAGES_MAX], a_empty[TC_ASTAGES_MAX];
    uint64_t b_full[TC_BSTAGES], b_empty[TC_BSTAGES];
    uint64_t r_full[TC_RSTAGES], r_empty[TC_RSTAGES];
    uint64_t seg_full, seg_empty;   // TMEM accumulator: segment summed / drained
    uint64_t mma_done[TC_CHMAX];    // an issuer's MMAs in flight completed (abort path only)
    uint32_t tmem_base;
    int abort_flag;
    // per chunk, broadcast pairs (v, v): kappa, -kappa, c1.x, c1.y, -c2.x, -c2.y, c3.x, c3.y
    alignas(16) float2 prm[TC_MAXCHUNKS][8];
    // FP32 sums of the TMEM partial sums, one padded row per target (the
    // 16-byte pad spreads the rows of a quarter-warp over all banks)
    alignas(16) float2 acc[TC_M][TC_CHMAX * 16 + 2];   // accessed as float4
};

static_assert(sizeof(TcSmem) + 1024 <= 227 * 1024, "shared memory per CTA");
static_assert(offsetof(TcSmem, acc) % 16 == 0 && (sizeof(float2) * (TC_CHMAX * 16 + 2)) % 16 == 0,
              "accumulator rows are read and written as float4");
static_assert(offsetof(TcSmem, geo) % 16 == 0 && offsetof(TcSmem, img) % 1024 == 0 && TC_GROUP_BYTES % 1024 == 0,
              "bulk-copy destinations are 16-byte aligned; images keep the 1024-byte swizzle alignment");

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// try_wait without a suspend-time hint: the thread is suspended in hardware
// until the phase completes or a system-dependent time limit passes.  (With
// an explicit hint the wait measured 3.5 % slower on the torus apply: it
// became a polling loop with sleeps, whose instructions took issue slots from
// the generator warps.)
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

// Non-blocking test of a phase: the result is not needed until it is used, so
// a test issued ahead of other work hides the latency of the barrier access.
__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
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

// The slow path of a wait, out of line so that the hot loops stay small: the
// fast path is one suspending try_wait.
__device__ __noinline__ bool wait_bar_slow(uint64_t *bar, uint32_t parity, volatile int *abort_flag, int *err,
                                           int code)
{
    return wait_bar(bar, parity, abort_flag, err, code);
}

// Warp-uniform bounded wait: true on every lane when the phase completed for
// the whole warp (the warp-collective tcgen05 instructions that follow need
// the warp to agree).
__device__ __forceinline__ bool warp_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag, int *err, int code)
{
    if (__all_sync(0xffffffffu, mbar_try_wait(bar, parity))) return true;
    return __all_sync(0xffffffffu, wait_bar_slow(bar, parity, abort_flag, err, code));
}

// One lane of a converged warp (the lowest), for the single-thread
// instructions (bulk copies, tcgen05.mma, tcgen05.commit).  Warp-wide loops
// with an elected issuer keep the loop state warp-uniform, so the compiler can
// hold the MMA operands in uniform registers.
__device__ __forceinline__ bool elect_one()
{
    uint32_t p = 0;
    asm volatile("{\n\t.reg .pred P;\n\t"
                 "elect.sync _|P, 0xffffffff;\n\t"
                 "selp.u32 %0, 1, 0, P;\n\t}"
                 : "=r"(p));
    return p != 0;
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
// are below 2^-21 |x|.  Used for the right-hand sides (expanded once per tile).
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

__device__ __forceinline__ void tmem_ld4(uint32_t taddr, uint32_t (&v)[4])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
                 : "r"(taddr)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&v)[8])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr)
                 : "memory");
}

template <int N>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, uint32_t (&v)[N])
{
    if constexpr (N == 8) tmem_ld8(taddr, v);
    else tmem_ld4(taddr, v);
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

// Instruction descriptor: D F32, A/B TF32, both K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_tf32(int n)
{
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t accumulate,
                                         uint32_t idesc)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
                 "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate)
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

// The schedule over the persistent grid of `ctas` CTAs.  Blocks (cg, blk) are
// numbered b = cg * nblk + blk.  The first full_waves * ctas blocks are whole
// pieces, CTA k taking blocks k, k + ctas, ...: in each wave every CTA sweeps
// the source tiles from the first, in step with the others, so the tiles being
// read at any time stay few and cached.  The remaining blocks ("tail") are
// split evenly by 16-source tiles ("stream-K"): CTA k takes the tail units
// [tail_start(k), tail_start(k + 1)), where a unit is one tile of one block.
// One problem of a packed launch (device memory; the fields of a single
// launch's plan and arguments, per problem).  prm: the broadcast parameter
// pairs of the problem's chunk groups, 8 per group (kappa, -kappa, c1.x, c1.y,
// -c2.x, -c2.y, c3.x, c3.y, each as (v, v)); err: the problem's error word.
struct TcProblem
{
    const float *mid4, *nrm4;
    const TcTileGeo *tgeo;
    const uint8_t *img;   // the expanded B images (tc_expand_kernel)
    float2 *Ctri;
    const float2 *prm;
    int *err;
    int n, m, wc, nblk, ntiles, self, off;
    float ki_s;
};

struct TcPlan
{
    int n, wc, nblk, ntiles, ncg, seg_tiles;
    int m;             // targets (rows of C): n for the boundary operators, the point count for the near field
    int self;          // 1: target i is source off + i and the pair is excluded (boundary); 0: no pair excluded
    int off;           // with self: the triangle of target 0 (a row shard of the boundary apply)
    int ctas;          // grid size
    int full_waves;    // whole blocks per CTA before the tail
    int tail_blocks;   // ncg * nblk - full_waves * ctas
    int64_t tail_units;   // tail_blocks * ntiles
    int stagger;       // whole-block sweeps of CTA k start at tile (k % 8) * stagger; -1: k * ntiles / ctas
    float ki_s;        // KI form: the common ratio s = c1.y / kappa (scaled coefficients)
    // packed launch: CTA k runs the whole blocks pieces[cta_begin[k] .. cta_begin[k + 1]),
    // each (problem, block of that problem); the scalar fields above are unused
    const TcProblem *probs;
    const int *cta_begin;
    const int2 *pieces;
};

__host__ __device__ __forceinline__ int64_t tc_tail_start(const TcPlan &p, int k)
{
    return (int64_t)k * p.tail_units / p.ctas;
}
// The CTA whose tail range holds tail unit x (a CTA with an empty range holds none).
__host__ __device__ __forceinline__ int tc_cta_of(const TcPlan &p, int64_t x)
{
    return (int)(((x + 1) * p.ctas - 1) / p.tail_units);
}

// Walks a CTA's work as pieces (cg, blk, tiles [tb, te)); `slot` is the
// workspace slot of a partial tail piece (0: the CTA's first tail piece,
// 1: its last); `rot` rotates the tile order of a whole-block piece (source
// tile = (t + rot) mod ntiles), 0 for tail pieces.
struct PieceIter
{
    int k, w;
    int64_t u, u0, u1;
    __device__ PieceIter(const TcPlan &p, int k_)
        : k(k_), w(0), u(tc_tail_start(p, k_)), u0(tc_tail_start(p, k_)), u1(tc_tail_start(p, k_ + 1)) {}
    __device__ bool next(const TcPlan &p, int &cg, int &blk, int &tb, int &te, int &slot, int &rot)
    {
        int b;
        rot = 0;
        if (w < p.full_waves)
        {
            b = w * p.ctas + k;
            ++w;
            tb = 0;
            te = p.ntiles;
            slot = 0;
            rot = p.stagger < 0 ? (int)((int64_t)k * p.ntiles / p.ctas) : (int)(((int64_t)(k % 8) * p.stagger) % p.ntiles);
        }
        else
        {
            if (u >= u1) return false;
            const int j = (int)(u / p.ntiles);
            b = p.full_waves * p.ctas + j;
            tb = (int)(u - (int64_t)j * p.ntiles);
            te = (int)min((int64_t)p.ntiles, (int64_t)tb + (u1 - u));
            slot = (u == u0) ? 0 : 1;
            u += te - tb;
        }
        cg = b / p.nblk;
        blk = b - cg * p.nblk;
        return true;
    }
};

// The pieces of a packed launch: whole blocks, every sweep from the first
// tile, so a problem's sums do not depend on what it is packed with.
struct PackIter
{
    int e, e1;
    __device__ PackIter() : e(0), e1(0) {}
    __device__ PackIter(const TcPlan &p, int k) : e(p.cta_begin[k]), e1(p.cta_begin[k + 1]) {}
    __device__ bool next(const TcPlan &p, int &prob, int &cg, int &blk, int &tb, int &te, int &slot, int &rot)
    {
        if (e >= e1) return false;
        const int2 q = p.pieces[e++];
        prob = q.x;
        const int nblk = p.probs[prob].nblk;
        cg = q.y / nblk;
        blk = q.y - cg * nblk;
        tb = 0;
        te = p.probs[prob].ntiles;
        slot = 0;
        rot = 0;
        return true;
    }
};

// The problem a piece belongs to, as the roles read it.
struct TcView
{
    const float *mid4, *nrm4;
    const TcTileGeo *tgeo;
    const uint8_t *img;
    float2 *Ctri;
    const float2 *prm;   // chunk group 0's 8 broadcast pairs (shared memory in a single launch)
    int n, m, wc, ntiles, self, off;
    float ki_s;
};

__device__ __forceinline__ TcView view_of(const TcProblem &q)
{
    return TcView{q.mid4, q.nrm4, q.tgeo, q.img, q.Ctri, q.prm, q.n, q.m, q.wc, q.ntiles, q.self, q.off, q.ki_s};
}

// Both piece walks behind one interface for the roles.
template <bool PACK>
struct Pieces
{
    PieceIter solo;
    PackIter pack;
    TcView single;
    __device__ Pieces(const TcPlan &p, int k, const TcView &v)
        : solo(p, PACK ? 0 : k), pack(PACK ? PackIter(p, k) : PackIter()), single(v) {}
    __device__ bool next(const TcPlan &p, TcView &v, int &cg, int &blk, int &tb, int &te, int &slot, int &rot)
    {
        if (PACK)
        {
            int prob;
            if (!pack.next(p, prob, cg, blk, tb, te, slot, rot)) return false;
            v = view_of(p.probs[prob]);
            return true;
        }
        v = single;
        return solo.next(p, cg, blk, tb, te, slot, rot);
    }
};

// The kernel entries of one wave chunk for this thread's PPT source pairs,
// in the A operand's K order (Re A_s0, Re A_s1, Im A_s0, Im A_s1) per pair,
// split into hi (the FP32 bits; the tensor core reads their top 19 as TF32)
// and lo = x - trunc_tf32(x).  P: the chunk's broadcast pairs kappa, -kappa,
// c1.x, c1.y, -c2.x, -c2.y, c3.x, c3.y.  Per pair: rinv = 1/r, r, dmu =
// (z.mu_j)/r^3, dnu = (z.nu_i)/r^3 (zero rinv masks a pair).
//   A = e^{i k r} h,  h = c1 / r + u + i k r (-u),  u = -(c2 dmu - c3 dnu):
//   hx = c1x / r + ux + k r uy,   hy = c1y / r + uy - k r ux.
// RI: every chunk's single-layer coefficient is imaginary and its double- and
// adjoint-double-layer coefficients are real (the mixed BIE and DtN tuples of
// FarField.hpp), so u is real: hx = ux, hy = c1y / r - k r ux.  The sincos is
// taken of -k r there, which gives -sin(k r) and saves the negation of the
// rotation's real part.
template <int PPT, bool SL, bool DL, bool ADL, bool RI>
__device__ __forceinline__ void tc_entries(const float2 *__restrict__ P, const float2 (&rinv)[PPT],
                                           const float2 (&r)[PPT], const float2 (&dmu)[PPT],
                                           const float2 (&dnu)[PPT], uint32_t (&hi)[4 * PPT],
                                           uint32_t (&lo)[4 * PPT])
{
    const float2 m1 = make_float2(-1.f, -1.f);
    #pragma unroll
    for (int p = 0; p < PPT; ++p)
    {
        float2 ax, ay;
        if (RI)
        {
            const float2 nkr = __fmul2_rn(P[1], r[p]);   // -k r
            float sn0, cs0, sn1, cs1;
            __sincosf(nkr.x, &sn0, &cs0);
            __sincosf(nkr.y, &sn1, &cs1);
            const float2 cs = make_float2(cs0, cs1), nsn = make_float2(sn0, sn1);   // cos(k r), -sin(k r)
            float2 ux = make_float2(0.f, 0.f);
            if (DL) ux = __fmul2_rn(P[4], dmu[p]);
            if (ADL) ux = DL ? __ffma2_rn(P[6], dnu[p], ux) : __fmul2_rn(P[6], dnu[p]);
            float2 hy;
            if (DL || ADL) hy = SL ? __ffma2_rn(nkr, ux, __fmul2_rn(P[3], rinv[p])) : __fmul2_rn(nkr, ux);
            else hy = __fmul2_rn(P[3], rinv[p]);
            // (ax, ay) = (ux cs - hy sn, ux sn + hy cs)
            ax = __ffma2_rn(hy, nsn, __fmul2_rn(ux, cs));
            ay = __ffma2_rn(hy, cs, __fmul2_rn(ux, __fmul2_rn(m1, nsn)));
            if (!(DL || ADL)) ax = __fmul2_rn(hy, nsn);
        }
        else
        {
            const float2 kr = __fmul2_rn(P[0], r[p]);
            float sn0, cs0, sn1, cs1;
            __sincosf(kr.x, &sn0, &cs0);
            __sincosf(kr.y, &sn1, &cs1);
            const float2 cs = make_float2(cs0, cs1), sn = make_float2(sn0, sn1);
            float2 hx = make_float2(0.f, 0.f), hy = make_float2(0.f, 0.f);
            if (SL)
            {
                hx = __fmul2_rn(P[2], rinv[p]);
                hy = __fmul2_rn(P[3], rinv[p]);
            }
            if (DL || ADL)
            {
                float2 ux = make_float2(0.f, 0.f), uy = make_float2(0.f, 0.f);
                if (DL) { ux = __fmul2_rn(P[4], dmu[p]); uy = __fmul2_rn(P[5], dmu[p]); }
                if (ADL) { ux = __ffma2_rn(P[6], dnu[p], ux); uy = __ffma2_rn(P[7], dnu[p], uy); }
                const float2 nkr = __fmul2_rn(P[1], r[p]);
                hx = __ffma2_rn(kr, uy, __fadd2_rn(hx, ux));
                hy = __ffma2_rn(nkr, ux, __fadd2_rn(hy, uy));
            }
            // (ax, ay) = (hx cs - hy sn, hx sn + hy cs)
            ax = __ffma2_rn(hy, __fmul2_rn(m1, sn), __fmul2_rn(hx, cs));
            ay = __ffma2_rn(hy, cs, __fmul2_rn(hx, sn));
        }
        const float2 tx = make_float2(__uint_as_float(__float_as_uint(ax.x) & 0xffffe000u),
                                      __uint_as_float(__float_as_uint(ax.y) & 0xffffe000u));
        const float2 ty = make_float2(__uint_as_float(__float_as_uint(ay.x) & 0xffffe000u),
                                      __uint_as_float(__float_as_uint(ay.y) & 0xffffe000u));
        const float2 lx = __ffma2_rn(tx, m1, ax), ly = __ffma2_rn(ty, m1, ay);
        hi[4 * p + 0] = __float_as_uint(ax.x);
        hi[4 * p + 1] = __float_as_uint(ax.y);
        hi[4 * p + 2] = __float_as_uint(ay.x);
        hi[4 * p + 3] = __float_as_uint(ay.y);
        lo[4 * p + 0] = __float_as_uint(lx.x);
        lo[4 * p + 1] = __float_as_uint(lx.y);
        lo[4 * p + 2] = __float_as_uint(ly.x);
        lo[4 * p + 3] = __float_as_uint(ly.y);
    }
}

// KI: RI with the structure of the BIE and DtN tuples over all chunks:
// c1 = i s kappa with s common, c2 and c3 real and common.  Then
//   hy = c1y / r - k r ux = kappa v,   v = s / r - r ux,
// and ux, -ux and v are per source pair, shared by every chunk (computed with
// the pair geometry): a chunk costs the phase, its sincos, hy, the rotation
// and the split.
template <int PPT>
__device__ __forceinline__ void tc_entries_ki(const float2 *__restrict__ P, const float2 (&r)[PPT],
                                              const float2 (&ux)[PPT], const float2 (&nux)[PPT],
                                              const float2 (&v)[PPT], uint32_t (&hi)[4 * PPT],
                                              uint32_t (&lo)[4 * PPT])
{
    const float2 m1 = make_float2(-1.f, -1.f);
    #pragma unroll
    for (int p = 0; p < PPT; ++p)
    {
        const float2 nkr = __fmul2_rn(P[1], r[p]);   // -k r
        float sn0, cs0, sn1, cs1;
        __sincosf(nkr.x, &sn0, &cs0);
        __sincosf(nkr.y, &sn1, &cs1);
        const float2 cs = make_float2(cs0, cs1), nsn = make_float2(sn0, sn1);   // cos(k r), -sin(k r)
        const float2 hy = __fmul2_rn(P[0], v[p]);
        // (ax, ay) = (ux cs - hy sn, ux sn + hy cs)
        const float2 ax = __ffma2_rn(hy, nsn, __fmul2_rn(ux[p], cs));
        const float2 ay = __ffma2_rn(hy, cs, __fmul2_rn(nux[p], nsn));
        const float2 tx = make_float2(__uint_as_float(__float_as_uint(ax.x) & 0xffffe000u),
                                      __uint_as_float(__float_as_uint(ax.y) & 0xffffe000u));
        const float2 ty = make_float2(__uint_as_float(__float_as_uint(ay.x) & 0xffffe000u),
                                      __uint_as_float(__float_as_uint(ay.y) & 0xffffe000u));
        const float2 lx = __ffma2_rn(tx, m1, ax), ly = __ffma2_rn(ty, m1, ay);
        hi[4 * p + 0] = __float_as_uint(ax.x);
        hi[4 * p + 1] = __float_as_uint(ax.y);
        hi[4 * p + 2] = __float_as_uint(ay.x);
        hi[4 * p + 3] = __float_as_uint(ay.y);
        lo[4 * p + 0] = __float_as_uint(lx.x);
        lo[4 * p + 1] = __float_as_uint(lx.y);
        lo[4 * p + 2] = __float_as_uint(ly.x);
        lo[4 * p + 3] = __float_as_uint(ly.y);
    }
}

// RI, KI: see tc_entries and tc_entries_ki.  GW: generator warps (TcShape).
// PACK: a packed launch over plan.probs (the pointer arguments are unused).
// R: groups of 16 columns that share one evaluation of the kernel entries (the
// KI form, whose entries depend on a group only through its wavenumber, with
// equal wavenumbers in every aligned block of R groups).  The CH groups of a
// work unit are CH / R entry sets; per tile the generators evaluate each set
// once into one A stage, and its issuer multiplies it with the R groups' B
// images: per K step one MMA of N = 64 R, Ahi [Bhi | Blo] (the set's R hi
// images are followed by its R lo images, tc_expand_kernel), into the set's
// main parts and corrections (consecutive in TMEM), and one of N = 32 R,
// Alo Bhi, into the corrections.
template <int GW, int CH, int R, bool SL, bool DL, bool ADL, bool RI, bool KI, bool PACK>
__global__ void __launch_bounds__(tc_threads<GW, CH, R>(), 1)
boundary_tc_kernel(const float *__restrict__ mid4, const float *__restrict__ nrm4, const TcTileGeo *__restrict__ tgeo,
                   const uint8_t *__restrict__ img, float2 *__restrict__ Ctri, float2 *__restrict__ ws,
                   const ChunkParamsF *__restrict__ prm, const TcPlan plan, int *err)
{
    constexpr int TC_GEN_THREADS = TcShape<GW>::GEN_THREADS;
    constexpr int TC_SPT = TcShape<GW>::SPT, TC_PPT = TcShape<GW>::PPT, TC_KPT = TcShape<GW>::KPT;
    constexpr int TC_CPG = TcShape<GW>::CPG;
    static_assert(R == 1 || (KI && !PACK && CH % R == 0), "shared entry sets need the KI form and R | CH");
    constexpr int E = CH / R;   // entry sets per tile
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // Align inside the shared window by pointer arithmetic on the shared array,
    // so every access below compiles to a shared-memory instruction.
    TcSmem &sm = *reinterpret_cast<TcSmem *>(smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u));
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
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
        for (int k = 0; k < tc_astages<CH>(); ++k) { mbar_init(&sm.a_full[k], TC_GEN_THREADS); mbar_init(&sm.a_empty[k], 1); }
        for (int k = 0; k < TC_BSTAGES; ++k) { mbar_init(&sm.b_full[k], 1); mbar_init(&sm.b_empty[k], tc_mma_warps<GW, CH, R>()); }
        for (int k = 0; k < TC_RSTAGES; ++k)
        {
            mbar_init(&sm.r_full[k], 1);
            mbar_init(&sm.r_empty[k], TC_GEN_THREADS);
        }
        mbar_init(&sm.seg_full, tc_mma_warps<GW, CH, R>());
        mbar_init(&sm.seg_empty, TC_GEN_THREADS);
        for (int k = 0; k < TC_CHMAX; ++k) mbar_init(&sm.mma_done[k], 1);
        sm.abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // the single problem's broadcast parameter pairs (a packed launch reads each problem's from global memory)
    for (int c = tid; c < (PACK ? 0 : plan.wc / 16); c += blockDim.x)
    {
        const ChunkParamsF p = prm[c];
        const float v[8] = {p.kappa, -p.kappa, p.c[1].x, p.c[1].y, -p.c[2].x, -p.c[2].y, p.c[3].x, p.c[3].y};
        #pragma unroll
        for (int k = 0; k < 8; ++k) sm.prm[c][k] = make_float2(v[k], v[k]);
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
    const TcView V0{mid4, nrm4, tgeo, img, Ctri, &sm.prm[0][0], plan.n, plan.m, plan.wc, plan.ntiles, plan.self,
                    plan.off, plan.ki_s};

    if (tid < TC_GEN_THREADS)
    {
        // ------------------------------ generators ------------------------------
        // Per tile: the pair geometry (shared by every chunk), then per entry
        // set (unrolled; a set is R chunks): its entries, the wait for its A
        // stage, one 16-column TMEM store per K step the thread covers
        // (hi | lo) and the stage's publication (with 8 warps deferred until
        // the next set's entries are computed, so the stores land meanwhile).
        // The ring index of set e of tile T is (T E + e) mod AS.
        const int q = warp & 3, g = warp >> 2;
        const int row = q * 32 + lane;
        const uint32_t lane_addr = tbase + ((uint32_t)(q * 32) << 16);
        constexpr int AS = tc_astages<CH>();
        const uint32_t a_addr = lane_addr + (uint32_t)(CH * TC_DCOLS + g * 2 * TC_KPT);
        float2 *acc_row = &sm.acc[row][g * TC_CPG];
        bool ok = true;
        bool pend = false;          // an A stage is written and not yet published
        uint32_t pend_stage = 0;
        int T = 0, SG = 0;          // tiles and TMEM segments handled so far by this CTA
        auto publish = [&]() {
            if (pend)
            {
                asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
                tc_fence_before();
                mbar_arrive(&sm.a_full[pend_stage]);
                pend = false;
            }
        };
        // add (or, first in a piece, store) the finished TMEM partial sum of
        // segment `sg` (main + correction) into this thread's accumulator row
        auto drain = [&](int sg, bool first) {
            if (!warp_wait(&sm.seg_full, (uint32_t)sg & 1u, abort_flag, err, 2)) return false;
            tc_fence_after();
            #pragma unroll
            for (int c = 0; c < CH; ++c)
            {
                uint32_t re[TC_CPG], im[TC_CPG], cre[TC_CPG], cim[TC_CPG];
                // the accumulator of an entry set: the main parts of its R chunks, then their corrections
                const uint32_t col = (uint32_t)((c - c % R) * TC_DCOLS + (c % R) * TC_N + g * TC_CPG);
                tmem_ld<TC_CPG>(lane_addr + col, re);
                tmem_ld<TC_CPG>(lane_addr + col + 16u, im);
                tmem_ld<TC_CPG>(lane_addr + col + (uint32_t)(R * TC_N), cre);
                tmem_ld<TC_CPG>(lane_addr + col + (uint32_t)(R * TC_N) + 16u, cim);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                float4 *a4 = reinterpret_cast<float4 *>(acc_row + c * 16);
                #pragma unroll
                for (int k = 0; k < TC_CPG / 2; ++k)
                {
                    float4 v = first ? make_float4(0.f, 0.f, 0.f, 0.f) : a4[k];
                    v.x += __uint_as_float(re[2 * k]) + __uint_as_float(cre[2 * k]);
                    v.y += __uint_as_float(im[2 * k]) + __uint_as_float(cim[2 * k]);
                    v.z += __uint_as_float(re[2 * k + 1]) + __uint_as_float(cre[2 * k + 1]);
                    v.w += __uint_as_float(im[2 * k + 1]) + __uint_as_float(cim[2 * k + 1]);
                    a4[k] = v;
                }
            }
            tc_fence_before();
            mbar_arrive(&sm.seg_empty);
            return true;
        };
        Pieces<PACK> it(plan, k_cta, V0);
        TcView V;
        int cg, blk, tb, te, slot, rot;
        while (ok && it.next(plan, V, cg, blk, tb, te, slot, rot))
        {
            const int n = V.n, mt = V.m, wc = V.wc, ntiles = V.ntiles;
            const int i = blk * TC_M + row;
            const int iself = V.self ? V.off + i : -1;   // the source excluded for this target (none: -1)
            // -x_i and nu_i as broadcast pairs
            float2 nx0 = make_float2(0.f, 0.f), nx1 = nx0, nx2 = nx0, tn0 = nx0, tn1 = nx0, tn2 = nx0;
            if (i < mt)
            {
                const float4 m = reinterpret_cast<const float4 *>(V.mid4)[i];
                nx0 = make_float2(-m.x, -m.x); nx1 = make_float2(-m.y, -m.y); nx2 = make_float2(-m.z, -m.z);
                if (ADL)
                {
                    const float4 v = reinterpret_cast<const float4 *>(V.nrm4)[i];
                    tn0 = make_float2(v.x, v.x); tn1 = make_float2(v.y, v.y); tn2 = make_float2(v.z, v.z);
                }
            }
            const float2 *Pg = V.prm + cg * CH * 8;
            // the source tiles that hold the target block's own triangles (masked)
            const int self_lo = V.self ? (V.off + blk * TC_M) / TC_SRC : ntiles;
            const int self_hi = V.self ? (V.off + blk * TC_M + TC_M - 1) / TC_SRC : -1;
            bool first_drain = true;
            // A finished segment is drained right after the next segment's first
            // chunk is stored, so the tensor core has work waiting when it resumes.
            int drain_due = -1;
            int sp = 0;   // tiles of the current segment done (a counter: S is a runtime value)
            for (int t = tb; t < te; ++t, ++T)
            {
                const int rs = T % TC_RSTAGES;
                const int ts = t + rot < ntiles ? t + rot : t + rot - ntiles;   // source tile (rot < ntiles)
                if (!warp_wait(&sm.r_full[rs], (uint32_t)(T / TC_RSTAGES) & 1u, abort_flag, err, 1))
                {
                    ok = false;
                    break;
                }
                // per source pair: 1/r, r, (z.mu_j)/r^3, (z.nu_i)/r^3; shared by every chunk
                float2 rinv[TC_PPT], r[TC_PPT], dmu[TC_PPT], dnu[TC_PPT];
                {
                    const TcTileGeo &G = sm.geo[rs];
                    const int s0 = g * TC_SPT;
                    // tiles that hold the target itself or padding past the end need masks
                    const bool special = (ts == ntiles - 1) || (ts >= self_lo && ts <= self_hi);
                    #pragma unroll
                    for (int p = 0; p < TC_PPT; ++p)
                    {
                        const int sl = s0 + 2 * p;
                        const float2 zx = __fadd2_rn(*reinterpret_cast<const float2 *>(&G.x[sl]), nx0);
                        const float2 zy = __fadd2_rn(*reinterpret_cast<const float2 *>(&G.y[sl]), nx1);
                        const float2 zz = __fadd2_rn(*reinterpret_cast<const float2 *>(&G.z[sl]), nx2);
                        const float2 r2 = __ffma2_rn(zz, zz, __ffma2_rn(zy, zy, __fmul2_rn(zx, zx)));
                        float ri0 = rsqrtf(r2.x), ri1 = rsqrtf(r2.y);
                        if (special)
                        {
                            const int j = ts * TC_SRC + sl;
                            if (!(j < n && j != iself)) ri0 = 0.f;
                            if (!(j + 1 < n && j + 1 != iself)) ri1 = 0.f;
                        }
                        rinv[p] = make_float2(ri0, ri1);
                        r[p] = __fmul2_rn(r2, rinv[p]);
                        const float2 ri3 = __fmul2_rn(__fmul2_rn(rinv[p], rinv[p]), rinv[p]);
                        if (DL)
                        {
                            const float2 mx = *reinterpret_cast<const float2 *>(&G.mx[sl]);
                            const float2 my = *reinterpret_cast<const float2 *>(&G.my[sl]);
                            const float2 mz = *reinterpret_cast<const float2 *>(&G.mz[sl]);
                            dmu[p] = __fmul2_rn(__ffma2_rn(zz, mz, __ffma2_rn(zy, my, __fmul2_rn(zx, mx))), ri3);
                        }
                        if (ADL) dnu[p] = __fmul2_rn(__ffma2_rn(zz, tn2, __ffma2_rn(zy, tn1, __fmul2_rn(zx, tn0))), ri3);
                    }
                }
                mbar_arrive(&sm.r_empty[rs]);
                // KI: ux = -(c2 dmu - c3 dnu), -ux and v = s / r - r ux per pair (every chunk's c2, c3 and s)
                float2 kux[TC_PPT], knux[TC_PPT], kv[TC_PPT];
                if (KI)
                {
                    const float2 s2 = make_float2(V.ki_s, V.ki_s);
                    #pragma unroll
                    for (int p = 0; p < TC_PPT; ++p)
                    {
                        float2 ux = make_float2(0.f, 0.f);
                        if (DL) ux = __fmul2_rn(Pg[4], dmu[p]);
                        if (ADL) ux = DL ? __ffma2_rn(Pg[6], dnu[p], ux) : __fmul2_rn(Pg[6], dnu[p]);
                        kux[p] = ux;
                        knux[p] = make_float2(-ux.x, -ux.y);
                        kv[p] = __ffma2_rn(r[p], knux[p], __fmul2_rn(s2, rinv[p]));
                    }
                }
                #pragma unroll
                for (int e = 0; e < E; ++e)
                {
                    uint32_t hi[TC_KPT], lo[TC_KPT];
                    if (KI) tc_entries_ki<TC_PPT>(Pg + 8 * (e * R), r, kux, knux, kv, hi, lo);
                    else tc_entries<TC_PPT, SL, DL, ADL, RI>(Pg + 8 * e, rinv, r, dmu, dnu, hi, lo);
                    const uint32_t u = (uint32_t)T * E + e;
                    const uint32_t stage = u % AS;
                    // (8 warps) publish the previous set's stage now that its stores had this math to land
                    publish();
                    // the stage is free once the MMAs that read it AS sets ago completed
                    if (!warp_wait(&sm.a_empty[stage], ((u / AS) & 1u) ^ 1u, abort_flag, err, 3))
                    {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    #pragma unroll
                    for (int h = 0; h < TC_KPT / 8; ++h)
                    {
                        uint32_t v[16];
                        #pragma unroll
                        for (int k = 0; k < 8; ++k) { v[k] = hi[8 * h + k]; v[8 + k] = lo[8 * h + k]; }
                        tmem_st16(a_addr + stage * 64u + 16u * h, v);
                    }
                    pend = true;
                    pend_stage = stage;
                    // 16 warps: publish at once, the issuers wait for it; the other three
                    // generator warps of the sub-partition cover the wait for the stores
                    if (GW == 16) publish();
                    if (e == 0 && drain_due >= 0)
                    {
                        publish();
                        if (!drain(drain_due, first_drain)) { ok = false; break; }
                        first_drain = false;
                        drain_due = -1;
                    }
                }
                if (!ok) break;
                if (++sp == S || t == te - 1)
                {
                    sp = 0;
                    // segment SG finished generating
                    if (t == te - 1)
                    {
                        publish();
                        if (!drain(SG, first_drain)) { ok = false; break; }
                        first_drain = false;
                    }
                    else
                        drain_due = SG;
                    ++SG;
                }
            }
            if (!ok) break;
            // ------------------------------ piece epilogue ------------------------------
            const int cw = CH * 16;
            float2 *dst = nullptr;
            if (tb == 0 && te == ntiles)
            {
                if (i < mt) dst = &V.Ctri[(int64_t)i * wc + cg * cw];
            }
            else
                dst = &ws[((int64_t)(k_cta * 2 + slot) * TC_M + row) * (TC_CHMAX * 16)];
            if (dst)
            {
                #pragma unroll
                for (int c = 0; c < CH; ++c)
                {
                    const float4 *a4 = reinterpret_cast<const float4 *>(acc_row + c * 16);
                    float4 *out = reinterpret_cast<float4 *>(dst + c * 16 + g * TC_CPG);
                    #pragma unroll
                    for (int k = 0; k < TC_CPG / 2; ++k) out[k] = a4[k];
                }
            }
        }
        if (!ok) publish();
    }
    else if (warp == TC_GEN_THREADS / 32)
    {
        // ------------------------------ bulk-copy producer ------------------------------
        // Per tile: its geometry into a geometry stage (for the generators) and
        // its expanded B images of this piece's chunk group into a B stage (for
        // the MMAs), each stage reused once its consumers released it.
        const uint32_t img_bytes = (uint32_t)(CH * TC_GROUP_BYTES);
        Pieces<PACK> it(plan, k_cta, V0);
        TcView V;
        int cg, blk, tb, te, slot, rot, T = 0;
        bool ok = true;
        while (ok && it.next(plan, V, cg, blk, tb, te, slot, rot))
        {
            const int ntiles = V.ntiles, groups = V.wc / 16;
            for (int t = tb; t < te; ++t, ++T)
            {
                const int rs = T % TC_RSTAGES, b = T % TC_BSTAGES;
                if (!warp_wait(&sm.r_empty[rs], ((uint32_t)(T / TC_RSTAGES) & 1u) ^ 1u, abort_flag, err, 6) ||
                    !warp_wait(&sm.b_empty[b], ((uint32_t)(T / TC_BSTAGES) & 1u) ^ 1u, abort_flag, err, 5))
                {
                    ok = false;
                    break;
                }
                const int ts = t + rot < ntiles ? t + rot : t + rot - ntiles;   // source tile (rot < ntiles)
                if (elect_one())
                {
                    mbar_expect_tx(&sm.r_full[rs], (uint32_t)sizeof(TcTileGeo));
                    bulk_g2s(&sm.geo[rs], V.tgeo + ts, (uint32_t)sizeof(TcTileGeo), &sm.r_full[rs]);
                    mbar_expect_tx(&sm.b_full[b], img_bytes);
                    bulk_g2s(sm.img[b], V.img + ((size_t)ts * groups + (size_t)cg * CH) * TC_GROUP_BYTES, img_bytes,
                             &sm.b_full[b]);
                }
                __syncwarp();
            }
        }
    }
    else
    {
        // ------------------------------ MMA issuers ------------------------------
        // MW warps; warp w issues the MMAs of entry sets w, w + MW, ... of
        // every tile (their own accumulator columns and A stages), so the
        // issue work is spread over SM sub-partitions instead of queueing
        // behind the generator warps of one.  Each warp runs its loop
        // warp-wide and waits; one elected lane issues.  B stages and the
        // segment's end are released by a commit of every issuer (barrier
        // counts MW).
        constexpr int MW = tc_mma_warps<GW, CH, R>();
        constexpr int AS = tc_astages<CH>();
        const int w = warp - (TC_GEN_THREADS / 32 + 1);
        bool ok = true;
        int T = 0, SG = 0;
        uint32_t pre = 0;   // the next tile's B stage (bit 0) / first A stage (bit 1) found complete by an early test
        // descriptors and TMEM addresses from bases fixed for the whole kernel: a
        // (stage, chunk) image is a constant byte offset from img[0][0][0], and
        // the descriptor's start-address field is that address >> 4
        const uint64_t desc0 = sw128_desc(&sm.img[0][0][0][0]);
        Pieces<PACK> it(plan, k_cta, V0);
        TcView V;
        int cg, blk, tb, te, slot, rot;
        while (ok && it.next(plan, V, cg, blk, tb, te, slot, rot))
        {
            int sp = 0;   // tiles of the current segment done (a counter: S is a runtime value)
            for (int t = tb; t < te; ++t, ++T)
            {
                const int b = T % TC_BSTAGES;
                const bool first = sp == 0;
                {
                    bool got = (pre & 1u) || warp_wait(&sm.b_full[b], (uint32_t)(T / TC_BSTAGES) & 1u, abort_flag, err, 7);
                    // a new segment overwrites the accumulator: the previous one must be drained
                    if (got && first && SG >= 1)
                        got = warp_wait(&sm.seg_empty, (uint32_t)(SG - 1) & 1u, abort_flag, err, 8);
                    if (!got) { ok = false; break; }
                }
                const bool seg_end = sp + 1 == S || t == te - 1;
                #pragma unroll
                for (int k = 0; k < E / MW; ++k)
                {
                    const int e = w + k * MW, c0 = e * R;   // entry set e: chunks c0 .. c0 + R - 1
                    const uint32_t u = (uint32_t)T * E + e;
                    const uint32_t stage = u % AS;
                    if (!(k == 0 && (pre & 2u)) && !warp_wait(&sm.a_full[stage], (u / AS) & 1u, abort_flag, err, 9))
                    {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t d = tbase + (uint32_t)(c0 * TC_DCOLS);
                    const uint32_t a_hi = tbase + (uint32_t)(CH * TC_DCOLS) + stage * 64u;
                    const uint32_t a_lo = a_hi + 8u;
                    // the set's R hi images (32 rows each) are followed by its R lo
                    // images (same 1024-byte group stride): one N = 64 R operand
                    // [Bhi | Blo] whose first 32 R rows are the N = 32 R operand Bhi
                    const uint64_t b_hilo = desc0 + (uint64_t)(((b * TC_CHMAX + c0) * TC_GROUP_BYTES) >> 4);
                    // Before the tile's last MMAs (whose issue waits for the tensor
                    // core), test the next tile's B stage and this warp's first A
                    // stage of it; the results are read after the MMAs are issued.
                    const bool last = k == E / MW - 1;
                    bool nb = false, na = false;
                    if (last)
                    {
                        const uint32_t un = (uint32_t)(T + 1) * E + w;
                        nb = mbar_test(&sm.b_full[(T + 1) % TC_BSTAGES], (uint32_t)((T + 1) / TC_BSTAGES) & 1u);
                        na = mbar_test(&sm.a_full[un % AS], (un / AS) & 1u);
                    }
                    if (elect_one())
                    {
                        #pragma unroll
                        for (int ks = 0; ks < 4; ++ks)
                        {
                            const uint64_t koff = (uint64_t)(ks * 32 >> 4);
                            // [main | corr] (+)= Ahi [Bhi | Blo];  corr += Alo Bhi (each over the set's chunks)
                            mma_tf32(d, a_hi + 16u * ks, b_hilo + koff, (!first || ks > 0) ? 1u : 0u,
                                     idesc_tf32(2 * TC_N * R));
                            mma_tf32(d + (uint32_t)(TC_N * R), a_lo + 16u * ks, b_hilo + koff, 1u, idesc_tf32(TC_N * R));
                        }
                        mma_commit(&sm.a_empty[stage]);
                        if (last)
                        {
                            mma_commit(&sm.b_empty[b]);
                            if (seg_end) mma_commit(&sm.seg_full);
                        }
                    }
                    __syncwarp();
                    if (last) pre = (__all_sync(0xffffffffu, nb) ? 1u : 0u) | (__all_sync(0xffffffffu, na) ? 2u : 0u);
                }
                if (!ok) break;
                sp = seg_end ? 0 : sp + 1;
                if (seg_end) ++SG;
            }
        }
        if (!ok)
        {
            // wait (bounded) for this warp's MMAs already issued before the TMEM is freed
            if (elect_one()) mma_commit(&sm.mma_done[w]);
            __syncwarp();
            wait_bar(&sm.mma_done[w], 0u, abort_flag, err, 10, false);
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

// The MMA's B operand for every 16-source tile t and 16-column group G, as the
// bytes a B stage holds: a hi and a lo image, each 32 K-major SWIZZLE_128B
// rows of 128 bytes.  The groups of tile t take TC_GROUP_BYTES each from
// t * groups * TC_GROUP_BYTES; within each aligned block of `share` groups
// (the groups that share one evaluation of the kernel entries) the hi images
// come first, then the lo images, so that one MMA reads [Bhi | Blo] of the
// whole block and another its Bhi (share = 1: hi, lo per group).  Row
// q < 16 (real part of column q's result) holds per source pair
// sp = (s0, s1) = (2 sp, 2 sp + 1) the 16-byte group (Re b_s0, Re b_s1,
// -Im b_s0, -Im b_s1); row 16 + q holds (Im b_s0, Im b_s1, Re b_s0, Re b_s1);
// group sp of row r sits at ((sp ^ (r & 7)) * 16) (img_off16).  hi = tf32(x)
// rounded to nearest, lo = x - hi (split_tf32).  Sources past n are zero.
// Thread (t, G, q, sp), sp fastest: 8 threads fill one row's 128 bytes.
__global__ void tc_expand_kernel(const float2 *__restrict__ Btri, int n, int wc, int64_t total, int share,
                                 uint8_t *__restrict__ img)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const int groups = wc / 16;
    const int sp = (int)(e & 7), q = (int)((e >> 3) & 15);
    const int64_t tg = e >> 7;                       // t * groups + G
    const int64_t t = tg / groups;
    const int G = (int)(tg - t * groups);
    const int64_t j0 = t * TC_SRC + 2 * sp;
    const int col = G * 16 + q;
    const float2 v0 = j0 < n ? Btri[j0 * wc + col] : make_float2(0.f, 0.f);
    const float2 v1 = j0 + 1 < n ? Btri[(j0 + 1) * wc + col] : make_float2(0.f, 0.f);
    uint32_t hr0, lr0, hi0, li0, hr1, lr1, hi1, li1;
    split_tf32(v0.x, hr0, lr0);
    split_tf32(v0.y, hi0, li0);
    split_tf32(v1.x, hr1, lr1);
    split_tf32(v1.y, hi1, li1);
    constexpr uint32_t sgn = 0x80000000u;
    const int r = G % share;   // place in the block of groups sharing the entries
    uint8_t *blk = img + (tg - r) * TC_GROUP_BYTES;
    uint8_t *hi_img = blk + r * TC_IMG, *lo_img = blk + (share + r) * TC_IMG;
    *reinterpret_cast<uint4 *>(hi_img + img_off16(q, sp)) = make_uint4(hr0, hr1, hi0 ^ sgn, hi1 ^ sgn);
    *reinterpret_cast<uint4 *>(lo_img + img_off16(q, sp)) = make_uint4(lr0, lr1, li0 ^ sgn, li1 ^ sgn);
    *reinterpret_cast<uint4 *>(hi_img + img_off16(q + 16, sp)) = make_uint4(hi0, hi1, hr0, hr1);
    *reinterpret_cast<uint4 *>(lo_img + img_off16(q + 16, sp)) = make_uint4(li0, li1, lr0, lr1);
}

// Midpoints and normals of each 16-source tile as structure of arrays (zeros
// past the last triangle).
__global__ void tc_tile_geometry_kernel(const float *__restrict__ mid4, const float *__restrict__ nrm4,
                                        TcTileGeo *__restrict__ out, int n, int ntiles)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ntiles * TC_SRC) return;
    const int t = e / TC_SRC, s = e - t * TC_SRC;
    float4 m = make_float4(0.f, 0.f, 0.f, 0.f), v = m;
    if (e < n)
    {
        m = reinterpret_cast<const float4 *>(mid4)[e];
        v = reinterpret_cast<const float4 *>(nrm4)[e];
    }
    TcTileGeo &G = out[t];
    G.x[s] = m.x; G.y[s] = m.y; G.z[s] = m.z;
    G.mx[s] = v.x; G.my[s] = v.y; G.mz[s] = v.z;
}

} // namespace

const uint8_t *launch_tc_expand(const float2 *Btri, int64_t n, int wc, DevBuf<uint8_t> &img, cudaStream_t st,
                                int share)
{
    const int64_t ntiles = ceil_div(n, TC_SRC), groups = wc / 16;
    const size_t bytes = (size_t)(ntiles * groups) * TC_GROUP_BYTES;
    uint8_t *out = img.reserve(bytes);
    const int64_t total = ntiles * groups * 128;
    if (total > 0)
    {
        tc_expand_kernel<<<ceil_div(total, 256), 256, 0, st>>>(Btri, (int)n, wc, total, share, out);
        BAEMM_LAUNCH_CHECK();
    }
    return out;
}

namespace
{
// Adds the workspace slots of every target block that was split between CTAs,
// in CTA order, and writes the block's rows of C_tri.
__global__ void tc_fixup_kernel(const float2 *__restrict__ ws, float2 *__restrict__ Ctri, const TcPlan plan, int cw)
{
    const int j = blockIdx.x;   // tail block
    const int b = plan.full_waves * plan.ctas + j;
    const int cg = b / plan.nblk, blk = b - cg * plan.nblk;
    const int64_t lo = (int64_t)j * plan.ntiles, hi = lo + plan.ntiles;
    const int k_first = tc_cta_of(plan, lo), k_last = tc_cta_of(plan, hi - 1);
    if (k_first == k_last) return;   // written directly by its CTA
    for (int e = threadIdx.x; e < TC_M * cw; e += blockDim.x)
    {
        const int row = e / cw, col = e - row * cw;
        const int i = blk * TC_M + row;
        if (i >= plan.m) continue;
        float2 acc = make_float2(0.f, 0.f);
        for (int k = k_first; k <= k_last; ++k)
        {
            const int64_t s0 = tc_tail_start(plan, k);
            if (tc_tail_start(plan, k + 1) == s0) continue;   // no tail units: wrote nothing
            const int slot = (s0 >= lo) ? 0 : 1;             // the CTA's first tail piece, or its last
            const float2 v = ws[((int64_t)(k * 2 + slot) * TC_M + row) * (TC_CHMAX * 16) + col];
            acc.x += v.x;
            acc.y += v.y;
        }
        Ctri[(int64_t)i * plan.wc + cg * cw + col] = acc;
    }
}

template <int GW, int CH, int R, bool SL, bool DL, bool ADL, bool RI, bool KI, bool PACK = false>
void tc_launch(cudaStream_t st, const float *mid, const float *nrm, const TcTileGeo *tg, const uint8_t *B, float2 *C,
               float2 *ws, const ChunkParamsF *p, const TcPlan &plan, int *err)
{
    // More than half of the SM's shared memory, so one CTA per SM: the CTA
    // allocates all 512 TMEM columns and a second resident CTA would only wait.
    const size_t bytes = std::max(sizeof(TcSmem) + 1024, (size_t)(116 * 1024));
    // The shared-memory limit is a per-device attribute of the function: set
    // it once on every device this instantiation is launched on.
    int dev = 0;
    BAEMM_CUDA(cudaGetDevice(&dev));
    static std::mutex mu;
    static bool done[64] = {};
    {
        std::lock_guard<std::mutex> lock(mu);
        if (dev < 0 || dev >= 64 || !done[dev])
        {
            BAEMM_CUDA(cudaFuncSetAttribute(boundary_tc_kernel<GW, CH, R, SL, DL, ADL, RI, KI, PACK>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
            if (dev >= 0 && dev < 64) done[dev] = true;
        }
    }
    boundary_tc_kernel<GW, CH, R, SL, DL, ADL, RI, KI, PACK><<<plan.ctas, tc_threads<GW, CH, R>(), bytes, st>>>(
        mid, nrm, tg, B, C, ws, p, plan, err);
}

template <int GW, int CH, bool RI>
void tc_flags(int code, cudaStream_t st, const float *mid, const float *nrm, const TcTileGeo *tg, const uint8_t *B,
              float2 *C, float2 *ws, const ChunkParamsF *p, const TcPlan &plan, int *err)
{
    switch (code)
    {
        case 1: tc_launch<GW, CH, 1, true, false, false, RI, false>(st, mid, nrm, tg, B, C, ws, p, plan, err); break;
        case 2: tc_launch<GW, CH, 1, false, true, false, RI, false>(st, mid, nrm, tg, B, C, ws, p, plan, err); break;
        case 3: tc_launch<GW, CH, 1, true, true, false, RI, false>(st, mid, nrm, tg, B, C, ws, p, plan, err); break;
        case 4: tc_launch<GW, CH, 1, false, false, true, RI, false>(st, mid, nrm, tg, B, C, ws, p, plan, err); break;
        case 5: tc_launch<GW, CH, 1, true, false, true, RI, false>(st, mid, nrm, tg, B, C, ws, p, plan, err); break;
        case 6: tc_launch<GW, CH, 1, false, true, true, RI, false>(st, mid, nrm, tg, B, C, ws, p, plan, err); break;
        case 7: tc_launch<GW, CH, 1, true, true, true, RI, false>(st, mid, nrm, tg, B, C, ws, p, plan, err); break;
        default: break;
    }
}

// The KI form for the operator combinations of the solves: the mixed BIE
// (SL + DL), the DtN operator (SL + ADL) and all three layers.
template <int GW, int CH, int R>
bool tc_flags_ki(int code, cudaStream_t st, const float *mid, const float *nrm, const TcTileGeo *tg, const uint8_t *B,
                 float2 *C, float2 *ws, const ChunkParamsF *p, const TcPlan &plan, int *err)
{
    switch (code)
    {
        case 3: tc_launch<GW, CH, R, true, true, false, true, true>(st, mid, nrm, tg, B, C, ws, p, plan, err); return true;
        case 5: tc_launch<GW, CH, R, true, false, true, true, true>(st, mid, nrm, tg, B, C, ws, p, plan, err); return true;
        case 7: tc_launch<GW, CH, R, true, true, true, true, true>(st, mid, nrm, tg, B, C, ws, p, plan, err); return true;
        default: return false;
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

TcCoeffForm tc_coeff_form(const ChunkParamsF *h, int groups)
{
    TcCoeffForm out;
    if (groups < 1 || h[0].kappa == 0.f) return out;
    const float s = h[0].c[1].y / h[0].kappa;
    for (int i = 0; i < groups; ++i)
    {
        const ChunkParamsF &q = h[i];
        if (q.kappa == 0.f || q.c[1].x != 0.f || q.c[2].y != 0.f || q.c[3].y != 0.f) return out;
        if (q.c[2].x != h[0].c[2].x || q.c[3].x != h[0].c[3].x) return out;
        // c1.y = s kappa up to the rounding of the scaled coefficients (a few ulps)
        if (std::fabs(q.c[1].y - s * q.kappa) > 1e-6f * std::fabs(q.c[1].y)) return out;
    }
    out.ki = true;
    out.s = s;
    // In this form a group's entries depend on the group only through kappa:
    // the most groups of an aligned block (4, 2, 1) with one wavenumber.
    for (out.share = 4; out.share > 1; out.share /= 2)
    {
        bool same = true;
        for (int i = 0; i < groups && same; ++i) same = h[i].kappa == h[i - i % out.share].kappa;
        if (same) break;
    }
    return out;
}

int tc_entry_sharing(const OpFlags &f, const TcCoeffForm &form, int wc, const TcTuning &tune)
{
    const bool ri = !f.re_sl && !f.im_dl && !f.im_adl && (f.dl() || f.adl());
    const int code = (f.sl() ? 1 : 0) | (f.dl() ? 2 : 0) | (f.adl() ? 4 : 0);
    if (!ri || !form.ki || !(code == 3 || code == 5 || code == 7)) return 1;
    return std::min({form.share, std::max(1, tune.share), tc_chunks_per_unit(wc, tune.chunks)});
}

int tc_chunks_per_unit(int wc, int chunks)
{
    const int groups = wc / 16;
    int ch = (groups % 4 == 0) ? 4 : (groups % 2 == 0) ? 2 : 1;   // the most the wave shape allows
    if (chunks == 1 || chunks == 2 || chunks == 4)
        while (ch > chunks) ch /= 2;
    return ch;
}

// Groups of 16 columns share a wavenumber: wave_chunk_size a multiple of 16.
bool tc_supported(int wc, int wcs) { return wcs % 16 == 0 && wcs > 0 && wc % wcs == 0 && wc <= 16 * TC_MAXCHUNKS; }

size_t tc_workspace_elems(int ctas)
{
    if (ctas <= 0) ctas = device_sm_count();
    return (size_t)ctas * 2 * TC_M * TC_CHMAX * 16;
}

size_t tc_tile_geometry_floats(int64_t nt) { return (size_t)ceil_div(nt, TC_SRC) * (sizeof(TcTileGeo) / sizeof(float)); }

void launch_tc_tile_geometry(const MeshDev &m, float *tgeo, cudaStream_t st)
{
    if (m.nt == 0) return;
    const int n = (int)m.nt, ntiles = ceil_div(n, TC_SRC);
    tc_tile_geometry_kernel<<<ceil_div((int64_t)ntiles * TC_SRC, 256), 256, 0, st>>>(
        m.mid_f, m.nrm_f, reinterpret_cast<TcTileGeo *>(tgeo), n, ntiles);
    BAEMM_LAUNCH_CHECK();
}

namespace
{
template <int GW>
void tc_dispatch(int CH, int R, bool ri, bool ki, int code, cudaStream_t st, const float *pts4, const float *nrm,
                 const TcTileGeo *tg, const uint8_t *Btri, float2 *Ctri, float2 *ws, const ChunkParamsF *p,
                 const TcPlan &plan, int *err)
{
    bool done = false;
    if (ri && ki)
    {
        if (CH == 4 && R == 4) done = tc_flags_ki<GW, 4, 4>(code, st, pts4, nrm, tg, Btri, Ctri, ws, p, plan, err);
        else if (CH == 4 && R == 2) done = tc_flags_ki<GW, 4, 2>(code, st, pts4, nrm, tg, Btri, Ctri, ws, p, plan, err);
        else if (CH == 4) done = tc_flags_ki<GW, 4, 1>(code, st, pts4, nrm, tg, Btri, Ctri, ws, p, plan, err);
        else if (CH == 2 && R == 2) done = tc_flags_ki<GW, 2, 2>(code, st, pts4, nrm, tg, Btri, Ctri, ws, p, plan, err);
        else if (CH == 2) done = tc_flags_ki<GW, 2, 1>(code, st, pts4, nrm, tg, Btri, Ctri, ws, p, plan, err);
        else done = tc_flags_ki<GW, 1, 1>(code, st, pts4, nrm, tg, Btri, Ctri, ws, p, plan, err);
    }
    if (done) return;
    if (ri)
    {
        if (CH == 4) tc_flags<GW, 4, true>(code, st, pts4, nrm, tg, Btri, Ctri, ws, p, plan, err);
        else if (CH == 2) tc_flags<GW, 2, true>(code, st, pts4, nrm, tg, Btri, Ctri, ws, p, plan, err);
        else tc_flags<GW, 1, true>(code, st, pts4, nrm, tg, Btri, Ctri, ws, p, plan, err);
    }
    else
    {
        if (CH == 4) tc_flags<GW, 4, false>(code, st, pts4, nrm, tg, Btri, Ctri, ws, p, plan, err);
        else if (CH == 2) tc_flags<GW, 2, false>(code, st, pts4, nrm, tg, Btri, Ctri, ws, p, plan, err);
        else tc_flags<GW, 1, false>(code, st, pts4, nrm, tg, Btri, Ctri, ws, p, plan, err);
    }
}

// One launch of the tensor-core form over the targets (pts4, m_targets) and all
// nt sources of the mesh; self = 1: the targets are the midpoints of triangles
// off .. off + m_targets - 1 and the pair i == j is excluded.
void tc_run(const MeshDev &m, const OpFlags &f, const void *chunk_params, const TcCoeffForm &form, int wc, int wcs,
            const float *tgeo, const float *pts4, int64_t m_targets, int self, int64_t off, const float2 *Btri,
            float2 *Ctri, float2 *ws, size_t ws_elems, DevBuf<uint8_t> &img, int *err, cudaStream_t st,
            const TcTuning &tune)
{
    BAEMM_REQUIRE(tc_supported(wc, wcs), BAEMM_ERR_SIZE,
                  "tensor-core apply needs wave_chunk_size a multiple of 16 and wave_count <= 512");
    BAEMM_REQUIRE(m_targets <= INT32_MAX - TC_M, BAEMM_ERR_SIZE, "too many targets");
    BAEMM_REQUIRE(tune.gen_warps == 8 || tune.gen_warps == 16, BAEMM_ERR_ARG, "generator warps: 8 or 16");
    if (!f.any_layer() || m.nt == 0 || m_targets == 0) return;
    TcPlan plan;
    plan.n = (int)m.nt;
    plan.m = (int)m_targets;
    plan.self = self;
    plan.off = (int)off;
    plan.wc = wc;
    const int CH = tc_chunks_per_unit(wc, tune.chunks);
    plan.ncg = wc / (16 * CH);
    plan.nblk = ceil_div(plan.m, TC_M);
    plan.ntiles = ceil_div(plan.n, TC_SRC);
    plan.seg_tiles = std::max(1, tune.seg_tiles);
    const int blocks = plan.ncg * plan.nblk;
    const int ctas = tune.ctas > 0 ? tune.ctas : device_sm_count();
    plan.ctas = (int)std::min<int64_t>(ctas, (int64_t)blocks * plan.ntiles);
    plan.full_waves = blocks / plan.ctas;
    plan.tail_blocks = blocks - plan.full_waves * plan.ctas;
    plan.tail_units = (int64_t)plan.tail_blocks * plan.ntiles;
    plan.stagger = tune.stagger;
    plan.ki_s = form.s;
    BAEMM_REQUIRE(ws && ws_elems >= tc_workspace_elems(plan.ctas), BAEMM_ERR_ARG, "tensor-core workspace too small");
    const int code = (f.sl() ? 1 : 0) | (f.dl() ? 2 : 0) | (f.adl() ? 4 : 0);
    const auto *p = static_cast<const ChunkParamsF *>(chunk_params);
    const float *nrm = m.nrm_f + 4 * off;   // target normals: read only with the adjoint double layer (targets = midpoints)
    const auto *tg = reinterpret_cast<const TcTileGeo *>(tgeo);
    BAEMM_REQUIRE(tg, BAEMM_ERR_ARG, "tensor-core tile geometry missing");
    // the real / imaginary coefficient structure of the BIE solves (see boundary_tc_kernel)
    const bool ri = !f.re_sl && !f.im_dl && !f.im_adl && (f.dl() || f.adl());
    const int R = tc_entry_sharing(f, form, wc, tune);
    const uint8_t *im = launch_tc_expand(Btri, m.nt, wc, img, st, R);
    if (tune.gen_warps == 8) tc_dispatch<8>(CH, R, ri, form.ki, code, st, pts4, nrm, tg, im, Ctri, ws, p, plan, err);
    else tc_dispatch<16>(CH, R, ri, form.ki, code, st, pts4, nrm, tg, im, Ctri, ws, p, plan, err);
    BAEMM_LAUNCH_CHECK();
    if (plan.tail_blocks > 0)
    {
        tc_fixup_kernel<<<plan.tail_blocks, 256, 0, st>>>(ws, Ctri, plan, CH * 16);
        BAEMM_LAUNCH_CHECK();
    }
}
} // namespace

namespace
{
// After a packed launch: a time-out the launch reported goes to every packed
// problem's own error word (read by its context like a single launch's), and
// the packer's word is cleared for the next launch.
__global__ void tc_pack_err_kernel(int *err, const TcProblem *probs, int count)
{
    const int e = *(volatile int *)err;
    if (e == 0) return;
    for (int q = threadIdx.x; q < count; q += blockDim.x) atomicExch(probs[q].err, e);
    __syncthreads();
    if (threadIdx.x == 0) *err = 0;
}

// The KI-form operators the packed launch serves (the solves' mixed BIE and
// DtN operators and all three layers); false for any other structure.
template <int GW, int CH>
bool tc_pack_flags(int code, cudaStream_t st, const TcPlan &plan, int *err)
{
    switch (code)
    {
        case 3: tc_launch<GW, CH, 1, true, true, false, true, true, true>(st, 0, 0, 0, 0, 0, 0, 0, plan, err); return true;
        case 5: tc_launch<GW, CH, 1, true, false, true, true, true, true>(st, 0, 0, 0, 0, 0, 0, 0, plan, err); return true;
        case 7: tc_launch<GW, CH, 1, true, true, true, true, true, true>(st, 0, 0, 0, 0, 0, 0, 0, plan, err); return true;
        default: return false;
    }
}

// One warp waits, through the kernel's own bounded waits, on an mbarrier that
// nothing arrives on: the wait gives up after kWaitNs and writes `code` to
// the error word, as a pipeline wait of the tensor-core kernel does.
__global__ void bounded_wait_probe_kernel(int *err, unsigned long long *ns, int code)
{
    __shared__ uint64_t bar;
    __shared__ int abort_flag;
    if (threadIdx.x == 0)
    {
        mbar_init(&bar, 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const uint64_t t0 = global_ns();
    const bool got = warp_wait(&bar, 0u, &abort_flag, err, code);
    if (threadIdx.x == 0) ns[0] = got ? 0ull : global_ns() - t0;
}
} // namespace

void tc_bounded_wait_probe(int code, double *elapsed_ms, int *code_out)
{
    DevBuf<int> err;
    DevBuf<unsigned long long> ns;
    err.reserve(1);
    ns.reserve(1);
    BAEMM_CUDA(cudaMemset(err.p, 0, sizeof(int)));
    BAEMM_CUDA(cudaMemset(ns.p, 0, sizeof(unsigned long long)));
    bounded_wait_probe_kernel<<<1, 32>>>(err.p, ns.p, code);
    BAEMM_LAUNCH_CHECK();
    BAEMM_CUDA(cudaDeviceSynchronize());
    int e = 0;
    unsigned long long t = 0;
    BAEMM_CUDA(cudaMemcpy(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost));
    BAEMM_CUDA(cudaMemcpy(&t, ns.p, sizeof(t), cudaMemcpyDeviceToHost));
    *code_out = e;
    *elapsed_ms = (double)t * 1e-6;
}

TcPackScratch::~TcPackScratch()
{
    if (uploaded) cudaEventDestroy(uploaded);
    if (host) cudaFreeHost(host);
}

void TcPackScratch::reserve(size_t bytes)
{
    dev.reserve(bytes);
    if (bytes > host_cap)
    {
        if (uploaded) BAEMM_CUDA(cudaEventSynchronize(uploaded));
        if (host) cudaFreeHost(host);
        host = nullptr;
        host_cap = 0;
        BAEMM_CUDA(cudaMallocHost(&host, bytes));
        host_cap = bytes;
    }
    if (!uploaded) BAEMM_CUDA(cudaEventCreateWithFlags(&uploaded, cudaEventDisableTiming));
}

uint8_t *TcPackScratch::stage(const void *src, size_t bytes, cudaStream_t st)
{
    BAEMM_CUDA(cudaEventSynchronize(uploaded));   // the previous upload has read the pinned copy
    std::memcpy(host, src, bytes);
    BAEMM_CUDA(cudaMemcpyAsync(dev.p, host, bytes, cudaMemcpyHostToDevice, st));
    BAEMM_CUDA(cudaEventRecord(uploaded, st));
    return dev.p;
}

void tc_broadcast_params(const ChunkParamsF *h, int groups, std::vector<float2> &out)
{
    out.resize((size_t)groups * 8);
    for (int g = 0; g < groups; ++g)
    {
        const ChunkParamsF &p = h[g];
        const float v[8] = {p.kappa, -p.kappa, p.c[1].x, p.c[1].y, -p.c[2].x, -p.c[2].y, p.c[3].x, p.c[3].y};
        for (int k = 0; k < 8; ++k) out[(size_t)g * 8 + k] = make_float2(v[k], v[k]);
    }
}

int tc_sm_count() { return device_sm_count(); }

bool tc_packable(const OpFlags &f, const TcCoeffForm &form, int wc, int wcs)
{
    const bool ri = !f.re_sl && !f.im_dl && !f.im_adl && (f.dl() || f.adl());
    const int code = (f.sl() ? 1 : 0) | (f.dl() ? 2 : 0) | (f.adl() ? 4 : 0);
    return tc_supported(wc, wcs) && ri && form.ki && (code == 3 || code == 5 || code == 7);
}

int tc_pack_class(const OpFlags &f, int wc, const TcTuning &tune)
{
    const int code = (f.sl() ? 1 : 0) | (f.dl() ? 2 : 0) | (f.adl() ? 4 : 0);
    // operator structure, chunk groups, warps and segment length: a packed launch runs one of each
    return ((code * 8 + tc_chunks_per_unit(wc, tune.chunks)) * 2 + (tune.gen_warps == 8 ? 1 : 0)) * 4096 +
           std::min(std::max(tune.seg_tiles, 1), 4095);
}

void launch_boundary_tc_packed(const TcPackItem *items, int count, const OpFlags &f, const TcTuning &tune,
                               TcPackScratch &scr, int *err, cudaStream_t st)
{
    BAEMM_REQUIRE(count >= 1, BAEMM_ERR_ARG, "packed launch without problems");
    const int code = (f.sl() ? 1 : 0) | (f.dl() ? 2 : 0) | (f.adl() ? 4 : 0);
    // every problem's chunk groups per unit under its own tuning (the packing
    // class holds it; tune is the first problem's, so it does not decide this)
    const int CH = items[0].ch;
    // the problem table and the blocks (problem, block), costed by their source tiles
    std::vector<TcProblem> probs((size_t)count);
    std::vector<std::pair<int, int2>> blocks;   // (tiles, (problem, block))
    for (int q = 0; q < count; ++q)
    {
        const TcPackItem &it = items[q];
        BAEMM_REQUIRE(it.ch == CH && (CH == 1 || CH == 2 || CH == 4) && it.wc % (16 * CH) == 0, BAEMM_ERR_ARG,
                      "packed problems need the same chunk groups per unit");
        TcProblem &P = probs[(size_t)q];
        P.mid4 = it.mid4;
        P.nrm4 = it.nrm4;
        P.tgeo = reinterpret_cast<const TcTileGeo *>(it.tgeo);
        P.img = it.img;
        P.Ctri = it.Ctri;
        P.prm = it.prm_bcast;
        P.err = it.err;
        P.n = (int)it.nt;
        P.m = (int)it.nt;
        P.wc = it.wc;
        P.nblk = ceil_div(it.nt, TC_M);
        P.ntiles = ceil_div(it.nt, TC_SRC);
        P.self = 1;
        P.off = 0;
        P.ki_s = it.ki_s;
        const int nb = (it.wc / (16 * CH)) * P.nblk;
        for (int b = 0; b < nb; ++b) blocks.push_back({P.ntiles, make_int2(q, b)});
    }
    // longest first onto the least loaded CTA (deterministic: ties by index)
    std::stable_sort(blocks.begin(), blocks.end(),
                     [](const std::pair<int, int2> &a, const std::pair<int, int2> &b) { return a.first > b.first; });
    const int ctas = (int)std::min<size_t>((size_t)(tune.ctas > 0 ? tune.ctas : device_sm_count()), blocks.size());
    std::vector<int64_t> load((size_t)ctas, 0);
    std::vector<std::vector<int2>> per((size_t)ctas);
    for (const auto &b : blocks)
    {
        const size_t k = (size_t)(std::min_element(load.begin(), load.end()) - load.begin());
        load[k] += b.first;
        per[k].push_back(b.second);
    }
    // one staging block: problems, then cta_begin, then the pieces
    const size_t nprob_b = sizeof(TcProblem) * (size_t)count;
    const size_t nbeg_b = sizeof(int) * (size_t)(ctas + 1);
    const size_t npiece_b = sizeof(int2) * blocks.size();
    const size_t off_beg = (nprob_b + 15) / 16 * 16, off_piece = (off_beg + nbeg_b + 15) / 16 * 16;
    const size_t total = off_piece + npiece_b;
    scr.reserve(total);
    std::vector<uint8_t> host(total);
    std::memcpy(host.data(), probs.data(), nprob_b);
    int *beg = reinterpret_cast<int *>(host.data() + off_beg);
    int2 *pcs = reinterpret_cast<int2 *>(host.data() + off_piece);
    int e = 0;
    for (int k = 0; k < ctas; ++k)
    {
        beg[k] = e;
        for (const int2 &q : per[(size_t)k]) pcs[e++] = q;
    }
    beg[ctas] = e;
    uint8_t *dev = scr.stage(host.data(), total, st);
    TcPlan plan{};
    plan.ctas = ctas;
    plan.seg_tiles = std::max(1, tune.seg_tiles);
    plan.probs = reinterpret_cast<const TcProblem *>(dev);
    plan.cta_begin = reinterpret_cast<const int *>(dev + off_beg);
    plan.pieces = reinterpret_cast<const int2 *>(dev + off_piece);
    bool ok;
    if (tune.gen_warps == 8)
        ok = (CH == 4) ? tc_pack_flags<8, 4>(code, st, plan, err)
             : (CH == 2) ? tc_pack_flags<8, 2>(code, st, plan, err) : tc_pack_flags<8, 1>(code, st, plan, err);
    else
        ok = (CH == 4) ? tc_pack_flags<16, 4>(code, st, plan, err)
             : (CH == 2) ? tc_pack_flags<16, 2>(code, st, plan, err) : tc_pack_flags<16, 1>(code, st, plan, err);
    BAEMM_REQUIRE(ok, BAEMM_ERR_ARG, "packed launch: operator structure not packable");
    BAEMM_LAUNCH_CHECK();
    tc_pack_err_kernel<<<1, 32, 0, st>>>(err, plan.probs, count);
    BAEMM_LAUNCH_CHECK();
}

void launch_boundary_tc(const MeshDev &m, const OpFlags &f, const void *chunk_params, const TcCoeffForm &form, int wc,
                        int wcs, const float *tgeo, const float2 *Btri, float2 *Ctri, float2 *ws, size_t ws_elems,
                        DevBuf<uint8_t> &img, int *err, cudaStream_t st, const TcTuning &tune, int64_t row_begin,
                        int64_t row_end)
{
    const int64_t r0 = std::max<int64_t>(0, row_begin), r1 = row_end < 0 ? m.nt : std::min<int64_t>(row_end, m.nt);
    if (r1 <= r0) return;
    tc_run(m, f, chunk_params, form, wc, wcs, tgeo, m.mid_f + 4 * r0, r1 - r0, 1, r0, Btri, Ctri + r0 * wc, ws, ws_elems,
           img, err, st, tune);
}

void launch_nearfield_tc(const MeshDev &m, const OpFlags &f, const void *chunk_params, const TcCoeffForm &form,
                         int wc, int wcs, const float *tgeo, const float *pts4, int64_t npts, const float2 *Btri,
                         float2 *Cpts, float2 *ws, size_t ws_elems, DevBuf<uint8_t> &img, int *err, cudaStream_t st,
                         const TcTuning &tune)
{
    BAEMM_REQUIRE(!f.adl() && !f.mass(), BAEMM_ERR_ARG, "near field: single and double layer only");
    tc_run(m, f, chunk_params, form, wc, wcs, tgeo, pts4, npts, 0, 0, Btri, Cpts, ws, ws_elems, img, err, st, tune);
}

} // namespace baemm
