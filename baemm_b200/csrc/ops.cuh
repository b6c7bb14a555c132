// Host-side launchers of the device kernels (all asynchronous on `st`).
// Layouts (row-major, complex interleaved):
//   mid4 / nrm4      nt x 4 reals (xyz, w = 0)      float and double copies
//   area, a3, diag   nt reals (a3 = area/3, the AvOp value)
//   Btri / Ctri      nt x wc complex (internal precision R)
//   vertex blocks    nv x ld complex (external precision)
//   AvOp             per triangle its 3 vertex ids sorted ascending (tri_sorted)
//   AvOp^T           CSR over vertices: avt_outer (nv+1), avt_inner (3 nt) = triangle ids ascending
//   Mass             CSR over vertices: mass_outer, mass_inner (sorted), values float and double
#pragma once
#include <vector>
#include "common.cuh"

namespace baemm
{

struct MeshDev
{
    int64_t nv = 0, nt = 0, nm = 0;
    DevBuf<double> coords;       // nv x 3
    DevBuf<int32_t> tris;        // nt x 3 (as given)
    DevBuf<int32_t> tri_sorted;  // nt x 3 (AvOp columns, sorted)
    DevBuf<int32_t> avt_outer, avt_inner;
    DevBuf<int32_t> mass_outer, mass_inner;
    DevBuf<float> mid_f, nrm_f, area_f, a3_f, diag_f, mass_f, lumped_f, meas_f;
    DevBuf<float> tgeo_f;        // tensor-core form: source geometry per 16-source tile (lazily built)
    DevBuf<double> mid_d, nrm_d, area_d, a3_d, diag_d, mass_d, lumped_d, meas_d;
};

// Target points of a dense launch: the triangle midpoints with the pair i == j
// excluded (self = 1, boundary operators) or arbitrary points with no pair
// excluded (self = 0, near field).  pts4: m x 4 reals (xyz, w unused).  With
// self = 1 the targets may be a row range of the midpoints: target i is
// triangle off + i (pts4 = midpoints + 4 off).
template <class R>
struct DenseTargets
{
    const R *pts4;
    int m;
    int self;
    int off;
};

// ---- mesh.cu -------------------------------------------------------------------
// Initialize.hpp:57-302 (geometry and single-layer diagonal) in precision R.
void launch_geometry(const MeshDev &m, bool fp64, cudaStream_t st);
// MassOp values (Initialize.hpp:214-247, 329-334) and areas_lumped_inv
// (Initialize.hpp:339-353), after launch_geometry.
void launch_mass_values(const MeshDev &m, bool fp64, cudaStream_t st);

// CurlOp values (Initialize.hpp:146-211, FP32): rows 3 t + d of triangle t,
// 9 entries per triangle, columns ascending within each row.
void launch_curl(const MeshDev &m, int32_t *inner, float *vals, cudaStream_t st);

// ---- sparse.cu -----------------------------------------------------------------
// AvOp (PL -> PC): Btri[t,k] = a3_t * sum_q Bin[v_q, k]; Text = float2/double2, R = internal.
template <class Text, class R>
void launch_avop(const MeshDev &m, const Text *Bin, int64_t ldB, int wc, cplx<R> *Btri, cudaStream_t st);

struct EpilogueArgs
{
    bool layers = false;      // add alpha * AvOp^T (Ctri [+ SL diagonal])
    bool sl_diag = false;     // SL diagonal (ApplySingleLayerDiagonal.hpp:397-454)
    bool mass = false;        // add alpha * c0 * M Bin (ApplyBoundaryOperators.hpp:363-387)
    int wc = 0, wcs = 1;
    // AvOp^T over the triangles [t_begin, t_end) only (a row shard of the
    // apply); the other rows of Ctri are not read
    int64_t t_begin = 0, t_end = INT64_MAX;
};
// C_out[v,k] = [layers] alpha * sum_{t ∋ v} a3_t (Ctri[t,k] + diag-term) + [mass] alpha c0 (M Bin)[v,k]
//              + beta * C_out[v,k]   (beta == 0 overwrites)
template <class Text, class R>
void launch_epilogue(const MeshDev &m, const EpilogueArgs &a, const cplx<R> *Ctri, const cplx<R> *Btri,
                     const void *chunk_params, const Text *Bin, int64_t ldB, Text alpha, Text beta,
                     Text *Cout, int64_t ldC, cudaStream_t st);

// Real-column helpers of FarField.hpp:886-1022.
// Yw[v] = sum_t a3_t * (n_t . (AvOp X)_t / a_t)       (DotWithNormals_PL, FarField.hpp:980-1012)
void launch_dot_with_normals_weak(const MeshDev &m, bool fp64, const double *X, double *Ytri, double *Yw,
                                  cudaStream_t st);
// Yw[v,d] = factor * sum_t a3_t * Re((AvOp X)_t) / a_t * n_t[d]   (FarField.hpp:914-942)
void launch_mult_with_normals_weak(const MeshDev &m, bool fp64, const double2 *X, double factor, double *Ytri,
                                   double *Yw, cudaStream_t st);
// bdr[v,k] = -s[v] * du[v,k]   (FarField.hpp:288-300)
void launch_scale_rows_neg(int64_t nv, int wc, const double *s, const double2 *du, double2 *out, cudaStream_t st);
// prod[v] = sum_k du[v,k] * dv[v,k]   (HadamardProduct.hpp:18-25, no conjugation)
void launch_row_dot(int64_t nv, int wc, const double2 *du, const double2 *dv, double2 *out, cudaStream_t st);

// Mass SpMM on real columns: Y = alpha M X + beta Y (values in fp64 or fp32-widened).
void launch_mass_dot_real(const MeshDev &m, bool fp64_values, double alpha, const double *X, int64_t ldX,
                          double beta, double *Y, int64_t ldY, int ncols, cudaStream_t st);
// Lumped inverse on real columns: Y = L X.
void launch_lumped_real(const MeshDev &m, bool fp64_values, const double *X, int64_t ldX, double *Y, int64_t ldY,
                        int ncols, cudaStream_t st);
// Cout[r, k] = alpha Cin[r, k] + beta Cout[r, k] over rows x wc, Cin packed
// (ld wc, internal precision R), arithmetic in double; beta == 0 overwrites
// (combine_matrices as called at ApplyNearFieldOperators.hpp:112-116).
template <class Text, class R>
void launch_combine(int64_t rows, int wc, double2 alpha, const cplx<R> *Cin, double2 beta, Text *Cout, int64_t ldC,
                    cudaStream_t st);
// Strided copies / conversions of external blocks.
template <class Tsrc, class Tdst>
void launch_copy_block(int64_t rows, int cols, const Tsrc *src, int64_t lds, Tdst *dst, int64_t ldd, cudaStream_t st);
// y = a * x + b * y over rows x cols (double or double2 element types)
template <class T>
void launch_axpby(int64_t rows, int cols, T a, const T *x, int64_t ldx, T b, T *y, int64_t ldy, cudaStream_t st);

// ---- dense.cu ------------------------------------------------------------------
// Dense boundary kernel (BoundaryOperatorKernel.cl:5-239): Ctri = K(kappa) Btri
// chunk by chunk, the self pair excluded.  R = float (plain FP32) or double.
// variant (FP32, 16-column groups): 0 scalar FMA kernel, 1 / 2 packed FP32x2
// kernel with 1 / 2 targets per thread.  [row_begin, row_end) restricts the
// targets to those triangles (rows of Ctri outside are not written; row_end
// < 0: all).
constexpr int kDenseVariants = 3;
template <class R>
void launch_boundary_dense(const MeshDev &m, const OpFlags &f, const void *chunk_params, int wc, int wcs,
                           const cplx<R> *Btri, cplx<R> *Ctri, cudaStream_t st, int variant = 2,
                           int64_t row_begin = 0, int64_t row_end = -1);
// Near-field kernel (NearFieldOperatorKernel.cl:5-194): Cpts (npts x wc) =
// K(kappa) Btri at the points pts4 (npts x 4 reals), single and double layer
// (c1, c2) only, no pair excluded.  Same kernels and variants as the boundary form.
template <class R>
void launch_nearfield_dense(const MeshDev &m, const OpFlags &f, const void *chunk_params, int wc, int wcs,
                            const R *pts4, int64_t npts, const cplx<R> *Btri, cplx<R> *Cpts, cudaStream_t st,
                            int variant = 2);
// Evaluation points (m x 3 doubles, device) -> m x 4 reals, w = 0.
template <class R>
void launch_pack_points(int64_t m, const double *pts3, R *pts4, cudaStream_t st);
// Compensated tensor-core dense kernel (tc.cu): TF32 hi/lo split, three
// tcgen05 MMAs per K step, FP32 accumulation in TMEM.  wave_chunk_size 16.
// `err` (device int) receives a non-zero code when a bounded wait gave up.
bool tc_supported(int wc, int wcs);
// The coefficient structure of the loaded chunks the tensor-core form
// specialises on (host side, once per LoadParameters): ki = every chunk has
// c1 = i s kappa with one common s, and c2, c3 real and common to all chunks
// (the mixed BIE and DtN tuples of FarField.hpp).
struct TcCoeffForm
{
    bool ki = false;
    float s = 0.f;
    int share = 1;   // KI form: groups per aligned block with one wavenumber (1, 2 or 4)
};
TcCoeffForm tc_coeff_form(const ChunkParamsF *host_params, int groups);
// Settings of the tensor-core form (the autotuner's search space):
//   seg_tiles  16-source tiles accumulated in TMEM before the partial sum is
//              added to FP32 registers (bounds the tensor-core accumulation chain);
//   ctas       persistent grid size (0: one CTA per SM);
//   stagger    sweep offset between CTAs (tiles; -1: spread evenly);
//   gen_warps  generator warps, 8 or 16;
//   chunks     16-column groups per work unit, 1, 2 or 4 (0: the most the wave shape allows).
struct TcTuning
{
    int seg_tiles = 16;
    int ctas = 0;
    int stagger = 0;
    int gen_warps = 16;
    int chunks = 0;
    int share = 4;   // most groups of 16 columns sharing one evaluation of the kernel entries (1, 2 or 4)
};
// The chunk groups per work unit a launch uses for wave_count wc and the setting `chunks`.
int tc_chunks_per_unit(int wc, int chunks);
// The groups per entry set a launch uses: groups with one wavenumber share the
// kernel entries in the KI form of the mixed BIE / DtN operators, up to the
// setting `share` and the chunk groups per work unit (packed launches use 1).
int tc_entry_sharing(const OpFlags &f, const TcCoeffForm &form, int wc, const TcTuning &tune);
void launch_boundary_tc(const MeshDev &m, const OpFlags &f, const void *chunk_params, const TcCoeffForm &form, int wc,
                        int wcs, const float *tgeo, const float2 *Btri, float2 *Ctri, float2 *ws, size_t ws_elems,
                        DevBuf<uint8_t> &img, int *err, cudaStream_t st, const TcTuning &tune,
                        int64_t row_begin = 0, int64_t row_end = -1);
// The tensor-core form of the near field: targets pts4 (npts x 4 floats), no
// pair excluded, flags without the adjoint double layer.
void launch_nearfield_tc(const MeshDev &m, const OpFlags &f, const void *chunk_params, const TcCoeffForm &form,
                         int wc, int wcs, const float *tgeo, const float *pts4, int64_t npts, const float2 *Btri,
                         float2 *Cpts, float2 *ws, size_t ws_elems, DevBuf<uint8_t> &img, int *err, cudaStream_t st,
                         const TcTuning &tune);
// The tensor-core form's B operand: every 16-source tile's hi / lo images of
// B_tri (n x wc) per 16-column group, as the kernel's B stages hold them
// (8 KB each); returns img's device block (grown as needed).
// Self-test of the bounded pipeline waits: one warp waits on an mbarrier that
// nothing arrives on; returns the error code the wait wrote and its duration.
void tc_bounded_wait_probe(int code, double *elapsed_ms, int *code_out);
// share: groups per aligned block that share the kernel entries (tc_entry_sharing; 1 for packed launches)
const uint8_t *launch_tc_expand(const float2 *Btri, int64_t n, int wc, DevBuf<uint8_t> &img, cudaStream_t st,
                                int share = 1);
// ---- packed tensor-core launches (several problems in one persistent launch) ----
// One problem as the host describes it: the boundary operator of one mesh
// (targets = sources = its nt triangles) on its device blocks.
struct TcPackItem
{
    const float *mid4, *nrm4;       // triangle midpoints and normals (float4)
    const float *tgeo;              // tile geometry (launch_tc_tile_geometry)
    const uint8_t *img;             // the expanded B operand (launch_tc_expand)
    float2 *Ctri;
    const float2 *prm_bcast;        // tc_broadcast_params on the device
    int *err;                       // the problem's error word (a time-out lands here)
    int64_t nt;
    int wc;
    float ki_s;
    int ch;                         // chunk groups per work unit under the problem's own tuning
                                    // (tc_chunks_per_unit; set by Packer::apply)
};
// Tables of packed launches: a grow-only device block and a pinned host copy
// it is uploaded from (on the launch's stream; reused once the last upload
// has completed).
struct TcPackScratch
{
    DevBuf<uint8_t> dev;
    uint8_t *host = nullptr;
    size_t host_cap = 0;
    cudaEvent_t uploaded = nullptr;
    TcPackScratch() = default;
    TcPackScratch(const TcPackScratch &) = delete;
    TcPackScratch &operator=(const TcPackScratch &) = delete;
    ~TcPackScratch();
    void reserve(size_t bytes);
    uint8_t *stage(const void *src, size_t bytes, cudaStream_t st);
};
// 8 broadcast pairs per 16-column group (kappa, -kappa, c1.x, c1.y, -c2.x, -c2.y, c3.x, c3.y).
void tc_broadcast_params(const ChunkParamsF *host_params, int groups, std::vector<float2> &out);
// SMs of the current device (cached).
int tc_sm_count();
// Whether the loaded operators can join a packed launch (the KI-form solve operators).
bool tc_packable(const OpFlags &f, const TcCoeffForm &form, int wc, int wcs);
// Problems with equal classes can share a packed launch (operator structure, chunk groups, warps, segment).
int tc_pack_class(const OpFlags &f, int wc, const TcTuning &tune);
// One launch over `count` problems of one class: whole target blocks, assigned
// longest first to the least loaded CTA, so each problem's result is the same
// whatever it is packed with.
void launch_boundary_tc_packed(const TcPackItem *items, int count, const OpFlags &f, const TcTuning &tune,
                               TcPackScratch &scratch, int *err, cudaStream_t st);
// Source geometry of the tensor-core form, per 16-source tile (built once per mesh).
size_t tc_tile_geometry_floats(int64_t nt);
void launch_tc_tile_geometry(const MeshDev &m, float *tgeo, cudaStream_t st);
// float2 elements of the tensor-core workspace for a persistent grid of `ctas`
// CTAs (0: one per SM of the current device).
size_t tc_workspace_elems(int ctas = 0);
// Far-field kernel (FarFieldOperatorKernel.cl:5-178) with source splitting and
// a deterministic second-pass reduction; Cout = alpha F + beta Cout.
template <class R>
void launch_farfield(const MeshDev &m, const OpFlags &f, const void *chunk_params, int wc, int wcs,
                     const cplx<R> *Btri, cplx<R> *partial, size_t partial_cap, double2 alpha, double2 beta,
                     double2 *Cout, int64_t ldC, cudaStream_t st);
size_t farfield_partial_elems(const MeshDev &m, int wc, int wcs);
// Herglotz kernel (HerglotzWaveKernel.cl:5-176) applied to conj(g).
template <class R>
void launch_herglotz(const MeshDev &m, const OpFlags &f, const void *chunk_params, int wc, int wcs,
                     const double2 *g, int64_t ldg, cplx<R> *Ctri, cudaStream_t st);
// Incident waves at the midpoints (IncidentWaveKernel_Plane.hpp:189-233, _Radial.hpp:5-57).
template <class R>
void launch_incident(const MeshDev &m, const void *chunk_params, int wc, int wcs, const R *dirs, int type,
                     cplx<R> *Ctri, cudaStream_t st);

} // namespace baemm
