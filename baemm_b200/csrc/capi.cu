// extern "C" entry points of libbaemm_cuda.so (declared in include/baemm.h).
// Each call validates its arguments, runs on the context's stream and
// converts exceptions into a baemm_status plus a message for baemm_last_error.
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>

#include "ctx.cuh"

using baemm::Ctx;
using baemm::DevBuf;
using baemm::DeviceScope;
using baemm::Error;
using baemm::zc;

namespace
{

thread_local std::string g_create_error;

template <class F>
int guarded(baemm_ctx *ctx, F &&f)
{
    if (!ctx || !ctx->impl) return BAEMM_ERR_ARG;
    try
    {
        DeviceScope scope(ctx->impl->device);
        f(*ctx->impl);
        ctx->impl->last_error.clear();
        return BAEMM_OK;
    }
    catch (const Error &e)
    {
        ctx->impl->last_error = e.what();
        return e.code;
    }
    catch (const std::bad_alloc &)
    {
        ctx->impl->last_error = "host allocation failed";
        return BAEMM_ERR_ALLOC;
    }
    catch (const std::exception &e)
    {
        ctx->impl->last_error = e.what();
        return BAEMM_ERR_ARG;
    }
}

inline double2 z2(const double *p) { return p ? make_double2(p[0], p[1]) : make_double2(0.0, 0.0); }
inline float2 c2(const float *p) { return p ? make_float2(p[0], p[1]) : make_float2(0.f, 0.f); }
inline zc zz(const double *p) { return p ? zc(p[0], p[1]) : zc(0.0, 0.0); }

// Copy an nrows x ncols host block (ld) into a contiguous device buffer (ld = ncols).
template <class T>
void h2d_block(Ctx &c, T *dst, const T *src, int64_t rows, int cols, int64_t ld)
{
    if (rows * cols == 0) return;
    BAEMM_CUDA(cudaMemcpy2DAsync(dst, cols * sizeof(T), src, ld * sizeof(T), cols * sizeof(T), rows,
                                 cudaMemcpyHostToDevice, c.stream));
}
template <class T>
void d2h_block(Ctx &c, T *dst, int64_t ld, const T *src, int64_t rows, int cols)
{
    if (rows * cols == 0) return;
    BAEMM_CUDA(cudaMemcpy2DAsync(dst, ld * sizeof(T), src, cols * sizeof(T), cols * sizeof(T), rows,
                                 cudaMemcpyDeviceToHost, c.stream));
}

bool is_zero(const double *b) { return !b || (b[0] == 0.0 && b[1] == 0.0); }
bool is_zero(const float *b) { return !b || (b[0] == 0.f && b[1] == 0.f); }

int create_impl(const double *coords, int64_t nv, const int32_t *tris, int64_t nt, const double *meas, int64_t nm,
                int device, int threads, baemm_ctx **out)
{
    if (!out) return BAEMM_ERR_ARG;
    *out = nullptr;
    if (!coords || !tris || nv <= 0 || nt <= 0 || nm < 0 || (nm > 0 && !meas))
    {
        g_create_error = "invalid mesh arguments";
        return BAEMM_ERR_ARG;
    }
    if (nt > baemm::kMaxMeshSize || nv > baemm::kMaxMeshSize || nm > baemm::kMaxMeshSize)
    {
        g_create_error = "mesh too large (at most 2^28 triangles, vertices and measurement directions)";
        return BAEMM_ERR_SIZE;
    }
    for (int64_t e = 0; e < 3 * nt; ++e)
        if (tris[e] < 0 || tris[e] >= nv)
        {
            g_create_error = "triangle index out of range at entry " + std::to_string(e);
            return BAEMM_ERR_ARG;
        }
    try
    {
        DeviceScope keep(-1);   // the constructor selects its device; the caller's is restored
        std::unique_ptr<baemm_ctx> c(new baemm_ctx());
        c->impl = new Ctx(coords, nv, tris, nt, meas, nm, device, threads);
        *out = c.release();
        g_create_error.clear();
        return BAEMM_OK;
    }
    catch (const Error &e)
    {
        g_create_error = e.what();
        return e.code;
    }
    catch (const std::bad_alloc &)
    {
        g_create_error = "host allocation failed";
        return BAEMM_ERR_ALLOC;
    }
    catch (const std::exception &e)
    {
        g_create_error = e.what();
        return BAEMM_ERR_ARG;
    }
}

} // namespace

static int copy_tri_field(baemm_ctx *ctx, float *out, const float *src, int64_t count)
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(out, BAEMM_ERR_ARG, "null output");
        BAEMM_CUDA(cudaMemcpyAsync(out, src, count * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
    });
}

template <class T, class S>
static void apply_host(Ctx &c, const S *alpha, const S *B, int64_t ldB, const S *beta, S *C, int64_t ldC)
{
    c.require_loaded();
    BAEMM_REQUIRE(B && C, BAEMM_ERR_ARG, "null block");
    const int wc = c.wave_count;
    BAEMM_REQUIRE(ldB >= wc && ldC >= wc, BAEMM_ERR_ARG, "leading dimension smaller than wave_count");
    const int64_t nv = c.mesh.nv, N = nv * wc;
    static_assert(sizeof(T) == 2 * sizeof(S), "complex layout");
    T *dB = reinterpret_cast<T *>(c.io_a.reserve((N * sizeof(T) + 15) / 16));
    T *dC = reinterpret_cast<T *>(c.io_b.reserve((N * sizeof(T) + 15) / 16));
    h2d_block<T>(c, dB, reinterpret_cast<const T *>(B), nv, wc, ldB);
    if (!is_zero(beta)) h2d_block<T>(c, dC, reinterpret_cast<const T *>(C), nv, wc, ldC);
    T al, be;
    al.x = alpha ? alpha[0] : 0; al.y = alpha ? alpha[1] : 0;
    be.x = beta ? beta[0] : 0; be.y = beta ? beta[1] : 0;
    const bool touches = c.flags.any_layer() || c.flags.mass();
    c.apply_boundary<T>(al, dB, wc, be, dC, wc);
    if (touches) d2h_block<T>(c, reinterpret_cast<T *>(C), ldC, dC, nv, wc);
    c.sync();
}

static void farfield_host(Ctx &c, const double *alpha, const double *B, int64_t ldB, const double *beta, double *C,
                          int64_t ldC)
{
    BAEMM_REQUIRE(B && C, BAEMM_ERR_ARG, "null block");
    const int wc = c.wave_count;
    if (c.wave_chunk_count < 1 || !(c.flags.sl() || c.flags.dl())) return;
    BAEMM_REQUIRE(ldB >= wc && ldC >= wc, BAEMM_ERR_ARG, "leading dimension smaller than wave_count");
    const int64_t nv = c.mesh.nv, nm = c.mesh.nm;
    double2 *dB = c.io_a.reserve(nv * wc), *dC = c.io_b.reserve(std::max<int64_t>(nm * wc, 1));
    h2d_block<double2>(c, dB, reinterpret_cast<const double2 *>(B), nv, wc, ldB);
    if (!is_zero(beta)) h2d_block<double2>(c, dC, reinterpret_cast<const double2 *>(C), nm, wc, ldC);
    c.apply_farfield(zz(alpha), dB, wc, zz(beta), dC, wc);
    d2h_block<double2>(c, reinterpret_cast<double2 *>(C), ldC, dC, nm, wc);
    c.sync();
}

// ApplyNearFieldOperators.hpp:56-122 with host blocks: B (nv x wc, ld ldB) in,
// C (npts x wc, ld ldC) in/out, points npts x 3 (real type S).
template <class T, class S>
static void nearfield_host(Ctx &c, const S *alpha, const S *B, int64_t ldB, const S *beta, S *C, int64_t ldC,
                           const S *points, int64_t npts)
{
    BAEMM_REQUIRE(B && C, BAEMM_ERR_ARG, "null block");
    const int wc = c.wave_count;
    if (c.wave_chunk_count < 1 || !(c.flags.sl() || c.flags.dl())) return;
    BAEMM_REQUIRE(ldB >= wc && ldC >= wc, BAEMM_ERR_ARG, "leading dimension smaller than wave_count");
    BAEMM_REQUIRE(npts >= 0, BAEMM_ERR_ARG, "negative evaluation point count");
    BAEMM_REQUIRE(npts <= baemm::kMaxMeshSize, BAEMM_ERR_SIZE, "at most 2^28 evaluation points per call");
    if (npts == 0) return;
    BAEMM_REQUIRE(points, BAEMM_ERR_ARG, "null evaluation points");
    static_assert(sizeof(T) == 2 * sizeof(S), "complex layout");
    const int64_t nv = c.mesh.nv;
    T *dB = reinterpret_cast<T *>(c.io_a.reserve((nv * wc * sizeof(T) + 15) / 16));
    T *dC = reinterpret_cast<T *>(c.io_b.reserve((npts * wc * sizeof(T) + 15) / 16));
    double *dP = c.io_r1.reserve(3 * npts);
    std::vector<double> pts(points, points + 3 * npts);   // widened; the kernels take their own precision
    BAEMM_CUDA(cudaMemcpyAsync(dP, pts.data(), 3 * npts * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    h2d_block<T>(c, dB, reinterpret_cast<const T *>(B), nv, wc, ldB);
    if (!is_zero(beta)) h2d_block<T>(c, dC, reinterpret_cast<const T *>(C), npts, wc, ldC);
    T al, be;
    al.x = alpha ? alpha[0] : 0; al.y = alpha ? alpha[1] : 0;
    be.x = beta ? beta[0] : 0; be.y = beta ? beta[1] : 0;
    c.apply_nearfield<T>(al, dB, wc, be, dC, wc, dP, npts);
    d2h_block<T>(c, reinterpret_cast<T *>(C), ldC, dC, npts, wc);
    c.sync();   // pts is a host temporary
}

static void mass_inverse_host(Ctx &c, const double *X, int64_t ldX, double *Y, int64_t ldY, int cols, double tol,
                              bool lumped)
{
    BAEMM_REQUIRE(X && Y && cols >= 1, BAEMM_ERR_ARG, "invalid arguments");
    BAEMM_REQUIRE(cols <= ldX && cols <= ldY, BAEMM_ERR_ARG, "nrhs > ld");   // ApplyMassInverse.hpp:34-44
    const int64_t nv = c.mesh.nv;
    double *dX = c.io_r1.reserve(nv * cols), *dY = c.io_r2.reserve(nv * cols);
    h2d_block<double>(c, dX, X, nv, cols, ldX);
    c.stats.cg_converged = 1;
    c.stats.cg_iterations = 0;
    if (lumped) baemm::launch_lumped_real(c.mesh, c.mass_values_fp64(), dX, cols, dY, cols, cols, c.stream);
    else c.mass_inverse_real(dX, cols, dY, cols, cols, tol);
    d2h_block<double>(c, Y, ldY, dY, nv, cols);
    c.sync();
}

static void check_solver_args(Ctx &c, const double *kappa, int wcc, const double *inc, int wcs)
{
    BAEMM_REQUIRE(kappa && inc, BAEMM_ERR_ARG, "null kappa or incident directions");
    BAEMM_REQUIRE(wcc >= 1 && wcs >= 1, BAEMM_ERR_ARG, "wave_chunk_count and wave_chunk_size must be positive");
    BAEMM_REQUIRE(c.mesh.nm > 0, BAEMM_ERR_SIZE, "no measurement directions");
}

// Uploads *du_dn, or allocates (calloc) and computes it when *du_dn == NULL
// (FarField.hpp:273-283, 381-391).  Leaves the device copy in `dd`.
static void ensure_du_dn(Ctx &c, const double *kappa, int wcc, const double *inc, int wcs, double **du_dn, int type,
                         double cg_tol, double gmres_tol, double2 *dd)
{
    BAEMM_REQUIRE(du_dn, BAEMM_ERR_ARG, "du_dn must be a valid pointer to a pointer");
    const int64_t N = c.mesh.nv * wcc * wcs;
    if (*du_dn == nullptr)
    {
        void *p = std::calloc((size_t)N, sizeof(double2));
        BAEMM_REQUIRE(p, BAEMM_ERR_ALLOC, "calloc of du_dn failed");
        c.derivative_helper(kappa, wcc, inc, wcs, dd, type, cg_tol, gmres_tol);
        BAEMM_CUDA(cudaMemcpyAsync(p, dd, N * sizeof(double2), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        *du_dn = static_cast<double *>(p);
    }
    else
    {
        BAEMM_CUDA(cudaMemcpyAsync(dd, *du_dn, N * sizeof(double2), cudaMemcpyHostToDevice, c.stream));
    }
}

namespace
{
// The weak incident wave with the loaded parameters (CreateIncidentWave.hpp:55-124):
// wave_chunk_size directions; C untouched without loaded chunks or without a
// single- or double-layer coefficient, as in the reference.
void incident_host(Ctx &c, const double alpha[2], const double *dirs, const double beta[2], double *C, int64_t ldC,
                   int type)
{
    if (c.wave_chunk_count < 1) return;
    const int wc = c.wave_count;
    BAEMM_REQUIRE(ldC >= wc, BAEMM_ERR_ARG, "leading dimension smaller than wave_count");
    if (!(c.flags.sl() || c.flags.dl())) return;
    const int64_t nv = c.mesh.nv;
    double2 *dC = c.io_b.reserve(nv * wc);
    if (!is_zero(beta)) h2d_block<double2>(c, dC, reinterpret_cast<const double2 *>(C), nv, wc, ldC);
    c.incident(zz(alpha), dirs, zz(beta), dC, wc, type);
    d2h_block<double2>(c, reinterpret_cast<double2 *>(C), ldC, dC, nv, wc);
    c.sync();
}

// The weak Herglotz wave of g (meas_count x wave_count) with the loaded
// parameters (CreateHerglotzWave.hpp:51-95).
void herglotz_host(Ctx &c, const double alpha[2], const double *g, int64_t ldg, const double beta[2], double *C,
                   int64_t ldC)
{
    if (c.wave_chunk_count < 1) return;
    BAEMM_REQUIRE(c.mesh.nm > 0, BAEMM_ERR_SIZE, "no measurement directions");
    const int wc = c.wave_count;
    BAEMM_REQUIRE(ldg >= wc && ldC >= wc, BAEMM_ERR_ARG, "leading dimension smaller than wave_count");
    if (!(c.flags.sl() || c.flags.dl())) return;
    const int64_t nv = c.mesh.nv, nm = c.mesh.nm;
    double2 *dg = c.io_a.reserve(nm * wc), *dC = c.io_b.reserve(nv * wc);
    h2d_block<double2>(c, dg, reinterpret_cast<const double2 *>(g), nm, wc, ldg);
    if (!is_zero(beta)) h2d_block<double2>(c, dC, reinterpret_cast<const double2 *>(C), nv, wc, ldC);
    c.herglotz(zz(alpha), dg, wc, zz(beta), dC, wc);
    d2h_block<double2>(c, reinterpret_cast<double2 *>(C), ldC, dC, nv, wc);
    c.sync();
}
} // namespace

extern "C" {

int baemm_create_i32(const double *coords, int64_t nv, const int32_t *tris, int64_t nt, const double *meas,
                     int64_t nm, int device, int cpu_threads, baemm_ctx **out)
{
    return create_impl(coords, nv, tris, nt, meas, nm, device, cpu_threads, out);
}

int baemm_create(const double *coords, int64_t nv, const int64_t *tris, int64_t nt, const double *meas, int64_t nm,
                 int device, int cpu_threads, baemm_ctx **out)
{
    if (!tris || nt <= 0) return create_impl(coords, nv, nullptr, nt, meas, nm, device, cpu_threads, out);
    if (nt > baemm::kMaxMeshSize || nv > baemm::kMaxMeshSize)   // before any index is read
    {
        g_create_error = "mesh too large (at most 2^28 triangles and vertices)";
        if (out) *out = nullptr;
        return BAEMM_ERR_SIZE;
    }
    std::vector<int32_t> t(3 * nt);
    for (int64_t e = 0; e < 3 * nt; ++e)
    {
        if (tris[e] < 0 || tris[e] >= nv)
        {
            g_create_error = "triangle index out of range at entry " + std::to_string(e);
            if (out) *out = nullptr;
            return BAEMM_ERR_ARG;
        }
        t[e] = (int32_t)tris[e];
    }
    return create_impl(coords, nv, t.data(), nt, meas, nm, device, cpu_threads, out);
}

int baemm_set_mesh(baemm_ctx *ctx, const double *coords, int64_t nv, const int64_t *tris, int64_t nt)
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(coords && tris && nv > 0 && nt > 0, BAEMM_ERR_ARG, "invalid mesh arguments");
        BAEMM_REQUIRE(nt <= baemm::kMaxMeshSize && nv <= baemm::kMaxMeshSize, BAEMM_ERR_SIZE,
                      "mesh too large (at most 2^28 triangles and vertices)");
        std::vector<int32_t> t(3 * nt);
        for (int64_t e = 0; e < 3 * nt; ++e)
        {
            BAEMM_REQUIRE(tris[e] >= 0 && tris[e] < nv, BAEMM_ERR_ARG,
                          "triangle index out of range at entry " + std::to_string(e));
            t[e] = (int32_t)tris[e];
        }
        c.set_mesh(coords, nv, t.data(), nt);
    });
}

void baemm_destroy(baemm_ctx *ctx)
{
    if (!ctx) return;
    try
    {
        if (ctx->impl)
        {
            DeviceScope scope(ctx->impl->device);
            delete ctx->impl;
        }
    }
    catch (...) {}
    delete ctx;
}

const char *baemm_last_error(const baemm_ctx *ctx)
{
    if (!ctx || !ctx->impl) return g_create_error.c_str();
    return ctx->impl->last_error.c_str();
}

int baemm_device_info(baemm_ctx *ctx, char *buf, size_t len)
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(buf && len > 0, BAEMM_ERR_ARG, "null buffer");
        const std::string s = c.device_info();
        std::strncpy(buf, s.c_str(), len - 1);
        buf[len - 1] = 0;
    });
}

const char *baemm_class_name(void) { return "Helmholtz_CUDA"; }

void *baemm_stream(baemm_ctx *ctx) { return (ctx && ctx->impl) ? (void *)ctx->impl->stream : nullptr; }

int baemm_set_stream(baemm_ctx *ctx, void *stream)
{
    return guarded(ctx, [&](Ctx &c) { c.switch_stream((cudaStream_t)stream); });
}

int baemm_synchronize(baemm_ctx *ctx)
{
    return guarded(ctx, [&](Ctx &c) { c.sync(); });
}

// ---- getters / setters --------------------------------------------------------
int64_t baemm_vertex_count(const baemm_ctx *ctx) { return (ctx && ctx->impl) ? ctx->impl->mesh.nv : -1; }
int64_t baemm_simplex_count(const baemm_ctx *ctx) { return (ctx && ctx->impl) ? ctx->impl->mesh.nt : -1; }
int64_t baemm_meas_count(const baemm_ctx *ctx) { return (ctx && ctx->impl) ? ctx->impl->mesh.nm : -1; }
int baemm_get_wave_count(const baemm_ctx *ctx) { return (ctx && ctx->impl) ? ctx->impl->wave_count : -1; }
int baemm_get_wave_chunk_size(const baemm_ctx *ctx) { return (ctx && ctx->impl) ? ctx->impl->wave_chunk_size : -1; }
int baemm_set_wave_chunk_size(baemm_ctx *ctx, int wcs)
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(wcs >= 1 && wcs <= 64 && (wcs & (wcs - 1)) == 0, BAEMM_ERR_SIZE,
                      "wave_chunk_size must be a power of two <= 64");
        c.wave_chunk_size = wcs;
    });
}
int baemm_get_block_size(const baemm_ctx *ctx) { return (ctx && ctx->impl) ? ctx->impl->block_size : -1; }
int baemm_set_block_size(baemm_ctx *ctx, int bs)
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(bs >= 1, BAEMM_ERR_ARG, "block size must be positive");
        c.block_size = bs;
    });
}
int baemm_use_diagonal(baemm_ctx *ctx, int use_it)
{
    return guarded(ctx, [&](Ctx &c) {
        c.use_diagonal = use_it != 0;
        ++c.graph_state;
    });
}
int baemm_set_gmres_params(baemm_ctx *ctx, int max_iter, int max_restarts)
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(max_iter >= 1 && max_iter <= baemm::kMaxRestart && max_restarts >= 1, BAEMM_ERR_ARG,
                      "gmres_max_iter must be in [1, 64] and gmres_max_restarts >= 1");
        c.gmres_max_iter = max_iter;
        c.gmres_max_restarts = max_restarts;
    });
}
int baemm_get_gmres_params(const baemm_ctx *ctx, int *max_iter, int *max_restarts)
{
    if (!ctx || !ctx->impl) return BAEMM_ERR_ARG;
    if (max_iter) *max_iter = ctx->impl->gmres_max_iter;
    if (max_restarts) *max_restarts = ctx->impl->gmres_max_restarts;
    return BAEMM_OK;
}
int baemm_set_apply_mode(baemm_ctx *ctx, int mode)
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(mode == BAEMM_APPLY_FP32 || mode == BAEMM_APPLY_TC || mode == BAEMM_APPLY_FP64,
                      BAEMM_ERR_ARG, "unsupported apply mode");
        c.apply_mode = mode;
        ++c.graph_state;
    });
}
int baemm_set_graphs(baemm_ctx *ctx, int on)
{
    return guarded(ctx, [&](Ctx &c) {
        c.use_graphs = on != 0;
        if (!c.use_graphs) c.clear_graphs();
    });
}
int baemm_graph_stats(const baemm_ctx *ctx, int64_t *captures, int64_t *replays)
{
    if (!ctx || !ctx->impl) return BAEMM_ERR_ARG;
    if (captures) *captures = ctx->impl->graph_captures;
    if (replays) *replays = ctx->impl->graph_replays;
    return BAEMM_OK;
}
int baemm_set_tuning(baemm_ctx *ctx, int key, int value)
{
    return guarded(ctx, [&](Ctx &c) {
        ++c.graph_state;
        switch (key)
        {
            case BAEMM_TUNE_DENSE_VARIANT:
                BAEMM_REQUIRE(value >= 0 && value < baemm::kDenseVariants, BAEMM_ERR_ARG, "unknown kernel variant");
                c.dense_variant = value;
                break;
            case BAEMM_TUNE_TC_SEGMENT:
                BAEMM_REQUIRE(value >= 1, BAEMM_ERR_ARG, "segment length must be >= 1");
                c.tc_tune.seg_tiles = value;
                break;
            case BAEMM_TUNE_TC_STAGGER:
                BAEMM_REQUIRE(value >= -1 && value <= 1 << 20, BAEMM_ERR_ARG, "stagger must be -1 or >= 0");
                c.tc_tune.stagger = value;
                break;
            case BAEMM_TUNE_TC_CTAS:
                BAEMM_REQUIRE(value >= 0 && value <= 65535, BAEMM_ERR_ARG, "grid size must be in [0, 65535]");
                c.tc_tune.ctas = value;
                break;
            case BAEMM_TUNE_TC_GEN_WARPS:
                BAEMM_REQUIRE(value == 8 || value == 16, BAEMM_ERR_ARG, "generator warps must be 8 or 16");
                c.tc_tune.gen_warps = value;
                break;
            case BAEMM_TUNE_TC_CHUNKS:
                BAEMM_REQUIRE(value == 0 || value == 1 || value == 2 || value == 4, BAEMM_ERR_ARG,
                              "chunks per unit must be 0, 1, 2 or 4");
                c.tc_tune.chunks = value;
                break;
            case BAEMM_TUNE_TC_SHARE:
                BAEMM_REQUIRE(value == 1 || value == 2 || value == 4, BAEMM_ERR_ARG,
                              "groups per shared entry set must be 1, 2 or 4");
                c.tc_tune.share = value;
                break;
            default: throw Error(BAEMM_ERR_ARG, "unknown tuning key");
        }
    });
}
int baemm_get_tuning(const baemm_ctx *ctx, int key)
{
    if (!ctx || !ctx->impl) return -1;
    if (key == BAEMM_TUNE_DENSE_VARIANT) return ctx->impl->dense_variant;
    if (key == BAEMM_TUNE_TC_SEGMENT) return ctx->impl->tc_tune.seg_tiles;
    if (key == BAEMM_TUNE_TC_CTAS) return ctx->impl->tc_tune.ctas;
    if (key == BAEMM_TUNE_TC_STAGGER) return ctx->impl->tc_tune.stagger;
    if (key == BAEMM_TUNE_TC_GEN_WARPS) return ctx->impl->tc_tune.gen_warps;
    if (key == BAEMM_TUNE_TC_CHUNKS) return ctx->impl->tc_tune.chunks;
    if (key == BAEMM_TUNE_TC_SHARE) return ctx->impl->tc_tune.share;
    return -1;
}
int baemm_tc_entry_sharing(const baemm_ctx *ctx)
{
    if (!ctx || !ctx->impl) return BAEMM_ERR_ARG;
    const baemm::Ctx &c = *ctx->impl;
    if (!c.operators_loaded) return BAEMM_ERR_NOT_LOADED;
    return baemm::tc_entry_sharing(c.flags, c.tc_form, c.wave_count, c.tc_tune);
}
int baemm_get_apply_mode(const baemm_ctx *ctx) { return (ctx && ctx->impl) ? ctx->impl->apply_mode : -1; }
int baemm_set_refinement(baemm_ctx *ctx, int max_steps, double inner_tol)
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(max_steps >= 0 && inner_tol > 0.0, BAEMM_ERR_ARG, "invalid refinement parameters");
        c.ir_max_steps = max_steps;
        c.ir_inner_tol = inner_tol;
    });
}


int baemm_get_areas(baemm_ctx *ctx, float *out)
{
    return (ctx && ctx->impl) ? copy_tri_field(ctx, out, ctx->impl->mesh.area_f, ctx->impl->mesh.nt) : BAEMM_ERR_ARG;
}
int baemm_get_triangle_normals(baemm_ctx *ctx, float *out4)
{
    return (ctx && ctx->impl) ? copy_tri_field(ctx, out4, ctx->impl->mesh.nrm_f, 4 * ctx->impl->mesh.nt) : BAEMM_ERR_ARG;
}
int baemm_get_triangle_midpoints(baemm_ctx *ctx, float *out4)
{
    return (ctx && ctx->impl) ? copy_tri_field(ctx, out4, ctx->impl->mesh.mid_f, 4 * ctx->impl->mesh.nt) : BAEMM_ERR_ARG;
}
int baemm_get_single_layer_diagonal(baemm_ctx *ctx, float *out)
{
    return (ctx && ctx->impl) ? copy_tri_field(ctx, out, ctx->impl->mesh.diag_f, ctx->impl->mesh.nt) : BAEMM_ERR_ARG;
}
int baemm_get_mass_matrix(baemm_ctx *ctx, int64_t *outer, int32_t *inner, float *values, int64_t *nnz)
{
    return guarded(ctx, [&](Ctx &c) {
        const int64_t z = (int64_t)c.mass_inner_h.size();
        if (nnz) *nnz = z;
        if (!outer) return;
        for (int64_t v = 0; v <= c.mesh.nv; ++v) outer[v] = c.mass_outer_h[v];
        if (inner) std::memcpy(inner, c.mass_inner_h.data(), z * sizeof(int32_t));
        if (values)
        {
            BAEMM_CUDA(cudaMemcpyAsync(values, c.mesh.mass_f.p, z * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
            c.sync();
        }
    });
}
int baemm_get_curl_operator(baemm_ctx *ctx, int64_t *outer, int32_t *inner, float *values, int64_t *nnz)
{
    return guarded(ctx, [&](Ctx &c) {
        const int64_t nt = c.mesh.nt, z = 9 * nt;
        if (nnz) *nnz = z;
        if (!outer) return;
        for (int64_t r = 0; r <= 3 * nt; ++r) outer[r] = 3 * r;
        if (!inner && !values) return;
        DevBuf<int32_t> di;
        DevBuf<float> dv;
        launch_curl(c.mesh, di.reserve(z), dv.reserve(z), c.stream);
        if (inner) BAEMM_CUDA(cudaMemcpyAsync(inner, di.p, z * sizeof(int32_t), cudaMemcpyDeviceToHost, c.stream));
        if (values) BAEMM_CUDA(cudaMemcpyAsync(values, dv.p, z * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
    });
}
int baemm_last_solve_stats(const baemm_ctx *ctx, baemm_solve_stats *out)
{
    if (!ctx || !ctx->impl || !out) return BAEMM_ERR_ARG;
    *out = ctx->impl->stats;
    return BAEMM_OK;
}

// ---- parameters and operators ----------------------------------------------------
int baemm_load_parameters(baemm_ctx *ctx, const double *kappa, const double *coeff, int wc, int wcs, double factor)
{
    return guarded(ctx, [&](Ctx &c) {
        c.load_parameters(kappa, reinterpret_cast<const zc *>(coeff), wc, wcs, factor);
    });
}
int baemm_load_boundary_operators(baemm_ctx *ctx, const double *kappa, const double *coeff, int wc, int wcs)
{
    return guarded(ctx, [&](Ctx &c) {
        c.load_parameters(kappa, reinterpret_cast<const zc *>(coeff), wc, wcs, 1.0);
        c.operators_loaded = true;
    });
}
int baemm_unload_boundary_operators(baemm_ctx *ctx)
{
    return guarded(ctx, [&](Ctx &c) {
        c.sync();
        c.operators_loaded = false;
    });
}

int baemm_apply_boundary_operators_dev_z(baemm_ctx *ctx, const double alpha[2], const double *B, int64_t ldB,
                                         const double beta[2], double *C, int64_t ldC)
{
    return guarded(ctx, [&](Ctx &c) {
        c.require_loaded();
        BAEMM_REQUIRE(B && C, BAEMM_ERR_ARG, "null block");
        c.apply_boundary<double2>(z2(alpha), reinterpret_cast<const double2 *>(B), ldB, z2(beta),
                                  reinterpret_cast<double2 *>(C), ldC);
    });
}
int baemm_apply_boundary_operators_dev_c(baemm_ctx *ctx, const float alpha[2], const float *B, int64_t ldB,
                                         const float beta[2], float *C, int64_t ldC)
{
    return guarded(ctx, [&](Ctx &c) {
        c.require_loaded();
        BAEMM_REQUIRE(B && C, BAEMM_ERR_ARG, "null block");
        c.apply_boundary<float2>(c2(alpha), reinterpret_cast<const float2 *>(B), ldB, c2(beta),
                                 reinterpret_cast<float2 *>(C), ldC);
    });
}



int baemm_apply_boundary_operators_rows_dev_z(baemm_ctx *ctx, const double alpha[2], const double *B, int64_t ldB,
                                              const double beta[2], double *C, int64_t ldC, int64_t row_begin,
                                              int64_t row_end, int with_mass)
{
    return guarded(ctx, [&](Ctx &c) {
        c.require_loaded();
        BAEMM_REQUIRE(B && C, BAEMM_ERR_ARG, "null block");
        c.apply_boundary_rows<double2>(z2(alpha), reinterpret_cast<const double2 *>(B), ldB, z2(beta),
                                       reinterpret_cast<double2 *>(C), ldC, row_begin, row_end, with_mass != 0);
    });
}
int baemm_apply_boundary_operators_rows_dev_c(baemm_ctx *ctx, const float alpha[2], const float *B, int64_t ldB,
                                              const float beta[2], float *C, int64_t ldC, int64_t row_begin,
                                              int64_t row_end, int with_mass)
{
    return guarded(ctx, [&](Ctx &c) {
        c.require_loaded();
        BAEMM_REQUIRE(B && C, BAEMM_ERR_ARG, "null block");
        c.apply_boundary_rows<float2>(c2(alpha), reinterpret_cast<const float2 *>(B), ldB, c2(beta),
                                      reinterpret_cast<float2 *>(C), ldC, row_begin, row_end, with_mass != 0);
    });
}

struct baemm_packer
{
    baemm::Packer *impl = nullptr;
};

baemm_packer *baemm_packer_create(int device, int max_wait_us)
{
    try
    {
        int n = 0;
        BAEMM_CUDA(cudaGetDeviceCount(&n));
        BAEMM_REQUIRE(device >= 0 && device < n, BAEMM_ERR_ARG, "no such device");
        auto *p = new baemm_packer;
        try
        {
            p->impl = new baemm::Packer(device, max_wait_us);
        }
        catch (...)
        {
            delete p;
            throw;
        }
        g_create_error.clear();
        return p;
    }
    catch (const std::exception &e)
    {
        g_create_error = e.what();
        return nullptr;
    }
}

void baemm_packer_destroy(baemm_packer *p)
{
    if (!p) return;
    delete p->impl;
    delete p;
}

int baemm_set_packer(baemm_ctx *ctx, baemm_packer *p)
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(!p || (p->impl && p->impl->device() == c.device), BAEMM_ERR_ARG,
                      "the packer belongs to another device");
        c.packer = p ? p->impl : nullptr;
    });
}

int baemm_packer_stats(const baemm_packer *p, int64_t *launches, int64_t *problems)
{
    if (!p || !p->impl) return BAEMM_ERR_ARG;
    if (launches) *launches = p->impl->launches();
    if (problems) *problems = p->impl->problems();
    return BAEMM_OK;
}

int baemm_selftest_bounded_wait(int device, double *elapsed_ms, int *code)
{
    try
    {
        BAEMM_REQUIRE(elapsed_ms && code, BAEMM_ERR_ARG, "null output");
        int n = 0;
        BAEMM_CUDA(cudaGetDeviceCount(&n));
        BAEMM_REQUIRE(device >= 0 && device < n, BAEMM_ERR_ARG, "no such device");
        DeviceScope scope(device);
        baemm::tc_bounded_wait_probe(99, elapsed_ms, code);
        g_create_error.clear();
        return BAEMM_OK;
    }
    catch (const Error &e)
    {
        g_create_error = e.what();
        return e.code;
    }
    catch (const std::exception &e)
    {
        g_create_error = e.what();
        return BAEMM_ERR_ARG;
    }
}

int baemm_profile_krylov(baemm_ctx *ctx, int columns, int iterations, int basis, double out[10])
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(out, BAEMM_ERR_ARG, "null output");
        BAEMM_REQUIRE(columns >= 1 && 2 * columns <= baemm::kMaxKrylovColumns && iterations >= 1 && basis >= 1 &&
                          basis <= baemm::kMaxRestart + 1,
                      BAEMM_ERR_ARG, "profile_krylov: sizes out of range");
        const bool v64 = c.mass_values_fp64();
        const int rc = 2 * columns;   // complex columns as interleaved real columns (ApplyMassInverse.hpp:71-98)
        double cg_ms[3], gs_ms[2];
        baemm::CgSolver cg;
        cg.profile(c.mesh, v64, rc, iterations, c.stream, cg_ms);
        baemm::profile_gram_schmidt(c.mesh.nv, columns, basis, iterations, c.stream, gs_ms);
        const double n = (double)c.mesh.nv, nnz = (double)c.mass_inner_h.size(), vs = v64 ? 8.0 : 4.0;
        const double vec = n * rc * 8.0, cvec = n * columns * 16.0;
        out[0] = cg_ms[0]; out[1] = cg_ms[1]; out[2] = cg_ms[2]; out[3] = gs_ms[0]; out[4] = gs_ms[1];
        out[5] = (n + 1) * 4 + nnz * (4 + vs) + 2 * vec;   // CSR, p gathered once, q written
        out[6] = n * vs + 7 * vec;                          // L; x, p, r, q read; x, r, z written
        out[7] = 3 * vec;                                   // z, p read; p written
        out[8] = (basis + 1) * cvec;                        // w and the basis vectors read
        out[9] = (basis + 2) * cvec;                        // w and the basis read, w written
    });
}

int baemm_profile_cg(baemm_ctx *ctx, int columns, int iterations, double out[3])
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(out, BAEMM_ERR_ARG, "null output");
        BAEMM_REQUIRE(columns >= 1 && 2 * columns <= baemm::kMaxKrylovColumns && iterations >= 1, BAEMM_ERR_ARG,
                      "profile_cg: sizes out of range");
        const bool v64 = c.mass_values_fp64();
        const int rc = 2 * columns;   // complex columns as interleaved real columns (ApplyMassInverse.hpp:71-98)
        baemm::CgSolver cg;
        const double n = (double)c.mesh.nv, nnz = (double)c.mass_inner_h.size(), vs = v64 ? 8.0 : 4.0;
        const double vec = n * rc * 8.0;
        // algorithmic bytes of one iteration: the matvec (CSR, p gathered once, q written), the update
        // (L; x, p, r, q read; x, r, z written) and the p update (z, p read; p written)
        out[1] = (n + 1) * 4 + nnz * (4 + vs) + 2 * vec + n * vs + 7 * vec + 3 * vec;
        const double blk = cg.profile_block(c.mesh, v64, rc, iterations, c.stream);
        if (blk > 0.0)
        {
            out[0] = blk;
            out[2] = 1.0;
        }
        else
        {
            double ms[3];
            cg.profile(c.mesh, v64, rc, iterations, c.stream, ms);
            out[0] = ms[0] + ms[1] + ms[2];
            out[2] = 0.0;
        }
    });
}

int baemm_boundary_operator_kernel_dev_c(baemm_ctx *ctx, const float *B_tri, float *C_tri, int64_t row_begin,
                                         int64_t row_end)
{
    return guarded(ctx, [&](Ctx &c) {
        c.require_loaded();
        BAEMM_REQUIRE(B_tri && C_tri, BAEMM_ERR_ARG, "null block");
        BAEMM_REQUIRE(c.apply_mode != BAEMM_APPLY_FP64, BAEMM_ERR_ARG,
                      "the FP64 apply mode takes complex128 blocks (baemm_boundary_operator_kernel_dev_z)");
        BAEMM_REQUIRE(row_begin >= 0 && row_begin <= row_end && row_end <= c.mesh.nt, BAEMM_ERR_ARG,
                      "row range outside [0, simplex_count]");
        if (row_end > row_begin && c.flags.any_layer())
            c.boundary_kernel_rows<float>(reinterpret_cast<const float2 *>(B_tri), reinterpret_cast<float2 *>(C_tri), row_begin,
                                 row_end);
    });
}
int baemm_boundary_operator_kernel_dev_z(baemm_ctx *ctx, const double *B_tri, double *C_tri, int64_t row_begin,
                                         int64_t row_end)
{
    return guarded(ctx, [&](Ctx &c) {
        c.require_loaded();
        BAEMM_REQUIRE(B_tri && C_tri, BAEMM_ERR_ARG, "null block");
        BAEMM_REQUIRE(c.apply_mode == BAEMM_APPLY_FP64, BAEMM_ERR_ARG,
                      "complex128 blocks need the FP64 apply mode (BAEMM_APPLY_FP64)");
        BAEMM_REQUIRE(row_begin >= 0 && row_begin <= row_end && row_end <= c.mesh.nt, BAEMM_ERR_ARG,
                      "row range outside [0, simplex_count]");
        if (row_end > row_begin && c.flags.any_layer())
            c.boundary_kernel_rows<double>(reinterpret_cast<const double2 *>(B_tri), reinterpret_cast<double2 *>(C_tri),
                                  row_begin, row_end);
    });
}

int baemm_apply_boundary_operators_z(baemm_ctx *ctx, const double alpha[2], const double *B, int64_t ldB,
                                     const double beta[2], double *C, int64_t ldC)
{
    return guarded(ctx, [&](Ctx &c) { apply_host<double2, double>(c, alpha, B, ldB, beta, C, ldC); });
}
int baemm_apply_boundary_operators_c(baemm_ctx *ctx, const float alpha[2], const float *B, int64_t ldB,
                                     const float beta[2], float *C, int64_t ldC)
{
    return guarded(ctx, [&](Ctx &c) { apply_host<float2, float>(c, alpha, B, ldB, beta, C, ldC); });
}
int baemm_apply_boundary_operators_full_z(baemm_ctx *ctx, const double alpha[2], const double *B, int64_t ldB,
                                          const double beta[2], double *C, int64_t ldC, const double *kappa,
                                          const double *coeff, int wc, int wcs)
{
    return guarded(ctx, [&](Ctx &c) {
        c.load_parameters(kappa, reinterpret_cast<const zc *>(coeff), wc, wcs, 1.0);
        c.operators_loaded = true;
        apply_host<double2, double>(c, alpha, B, ldB, beta, C, ldC);
        c.operators_loaded = false;
    });
}



int baemm_apply_far_field_operators_z(baemm_ctx *ctx, const double alpha[2], const double *B, int64_t ldB,
                                      const double beta[2], double *C, int64_t ldC, const double *kappa,
                                      const double *coeff, int wc, int wcs)
{
    return guarded(ctx, [&](Ctx &c) {
        c.load_parameters(kappa, reinterpret_cast<const zc *>(coeff), wc, wcs, 1.0);
        farfield_host(c, alpha, B, ldB, beta, C, ldC);
    });
}
int baemm_apply_far_field_operators_loaded_z(baemm_ctx *ctx, const double alpha[2], const double *B, int64_t ldB,
                                             const double beta[2], double *C, int64_t ldC)
{
    return guarded(ctx, [&](Ctx &c) { farfield_host(c, alpha, B, ldB, beta, C, ldC); });
}
int baemm_apply_far_field_operators_dev_z(baemm_ctx *ctx, const double alpha[2], const double *B, int64_t ldB,
                                          const double beta[2], double *C, int64_t ldC)
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(B && C, BAEMM_ERR_ARG, "null block");
        c.apply_farfield(zz(alpha), reinterpret_cast<const double2 *>(B), ldB, zz(beta),
                         reinterpret_cast<double2 *>(C), ldC);
    });
}

int baemm_apply_near_field_operators_z(baemm_ctx *ctx, const double alpha[2], const double *B, int64_t ldB,
                                       const double beta[2], double *C, int64_t ldC, const double *points,
                                       int64_t npts)
{
    return guarded(ctx, [&](Ctx &c) { nearfield_host<double2, double>(c, alpha, B, ldB, beta, C, ldC, points, npts); });
}
int baemm_apply_near_field_operators_c(baemm_ctx *ctx, const float alpha[2], const float *B, int64_t ldB,
                                       const float beta[2], float *C, int64_t ldC, const float *points, int64_t npts)
{
    return guarded(ctx, [&](Ctx &c) { nearfield_host<float2, float>(c, alpha, B, ldB, beta, C, ldC, points, npts); });
}
int baemm_apply_near_field_operators_full_z(baemm_ctx *ctx, const double alpha[2], const double *B, int64_t ldB,
                                            const double beta[2], double *C, int64_t ldC, const double *kappa,
                                            const double *coeff, int wc, int wcs, const double *points, int64_t npts)
{
    return guarded(ctx, [&](Ctx &c) {
        c.load_parameters(kappa, reinterpret_cast<const zc *>(coeff), wc, wcs, 1.0);
        nearfield_host<double2, double>(c, alpha, B, ldB, beta, C, ldC, points, npts);
    });
}
int baemm_apply_near_field_operators_dev_z(baemm_ctx *ctx, const double alpha[2], const double *B, int64_t ldB,
                                           const double beta[2], double *C, int64_t ldC, const double *points,
                                           int64_t npts)
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(B && C, BAEMM_ERR_ARG, "null block");
        c.apply_nearfield<double2>(z2(alpha), reinterpret_cast<const double2 *>(B), ldB, z2(beta),
                                   reinterpret_cast<double2 *>(C), ldC, points, npts);
    });
}
int baemm_apply_near_field_operators_dev_c(baemm_ctx *ctx, const float alpha[2], const float *B, int64_t ldB,
                                           const float beta[2], float *C, int64_t ldC, const double *points,
                                           int64_t npts)
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(B && C, BAEMM_ERR_ARG, "null block");
        c.apply_nearfield<float2>(c2(alpha), reinterpret_cast<const float2 *>(B), ldB, c2(beta),
                                  reinterpret_cast<float2 *>(C), ldC, points, npts);
    });
}

int baemm_create_incident_wave_z(baemm_ctx *ctx, const double alpha[2], const double *dirs, int inc_count,
                                 const double beta[2], double *C, int64_t ldC, const double *kappa,
                                 const double *coeff, int wc, int wcs, int type)
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(dirs && C, BAEMM_ERR_ARG, "null argument");
        // CreateIncidentWave.hpp:35-45: inc_count must equal wave_chunk_size (excess is ignored)
        BAEMM_REQUIRE(inc_count >= wcs, BAEMM_ERR_ARG,
                      "number of incident waves has to match the size of the wave chunks");
        c.load_parameters(kappa, reinterpret_cast<const zc *>(coeff), wc, wcs, 4.0 * M_PI);
        incident_host(c, alpha, dirs, beta, C, ldC, type);
    });
}

int baemm_create_incident_wave_loaded_z(baemm_ctx *ctx, const double alpha[2], const double *dirs,
                                        const double beta[2], double *C, int64_t ldC, int type)
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(dirs && C, BAEMM_ERR_ARG, "null argument");
        incident_host(c, alpha, dirs, beta, C, ldC, type);
    });
}

int baemm_create_herglotz_wave_z(baemm_ctx *ctx, const double alpha[2], const double *g, int64_t ldg,
                                 const double beta[2], double *C, int64_t ldC, const double *kappa,
                                 const double *coeff, int wc, int wcs)
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(g && C, BAEMM_ERR_ARG, "null argument");
        BAEMM_REQUIRE(c.mesh.nm > 0, BAEMM_ERR_SIZE, "no measurement directions");
        c.load_parameters(kappa, reinterpret_cast<const zc *>(coeff), wc, wcs, 4.0 * M_PI / (double)c.mesh.nm);
        herglotz_host(c, alpha, g, ldg, beta, C, ldC);
    });
}

int baemm_create_herglotz_wave_loaded_z(baemm_ctx *ctx, const double alpha[2], const double *g, int64_t ldg,
                                        const double beta[2], double *C, int64_t ldC)
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(g && C, BAEMM_ERR_ARG, "null argument");
        herglotz_host(c, alpha, g, ldg, beta, C, ldC);
    });
}



int baemm_apply_mass_inverse_d(baemm_ctx *ctx, const double *X, int64_t ldX, double *Y, int64_t ldY, int nrhs,
                               double tol)
{
    return guarded(ctx, [&](Ctx &c) { mass_inverse_host(c, X, ldX, Y, ldY, nrhs, tol, false); });
}
int baemm_apply_mass_inverse_z(baemm_ctx *ctx, const double *X, int64_t ldX, double *Y, int64_t ldY, int nrhs,
                               double tol)
{
    return guarded(ctx, [&](Ctx &c) { mass_inverse_host(c, X, 2 * ldX, Y, 2 * ldY, 2 * nrhs, tol, false); });
}
int baemm_apply_lumped_mass_inverse_d(baemm_ctx *ctx, const double *X, int64_t ldX, double *Y, int64_t ldY, int nrhs)
{
    return guarded(ctx, [&](Ctx &c) { mass_inverse_host(c, X, ldX, Y, ldY, nrhs, 0.0, true); });
}
int baemm_apply_lumped_mass_inverse_z(baemm_ctx *ctx, const double *X, int64_t ldX, double *Y, int64_t ldY, int nrhs)
{
    return guarded(ctx, [&](Ctx &c) { mass_inverse_host(c, X, 2 * ldX, Y, 2 * ldY, 2 * nrhs, 0.0, true); });
}
int baemm_mass_dot_d(baemm_ctx *ctx, double alpha, const double *X, int64_t ldX, double beta, double *Y, int64_t ldY,
                     int nrhs)
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(X && Y && nrhs >= 1 && nrhs <= ldX && nrhs <= ldY, BAEMM_ERR_ARG, "invalid arguments");
        const int64_t nv = c.mesh.nv;
        double *dX = c.io_r1.reserve(nv * nrhs), *dY = c.io_r2.reserve(nv * nrhs);
        h2d_block<double>(c, dX, X, nv, nrhs, ldX);
        if (beta != 0.0) h2d_block<double>(c, dY, Y, nv, nrhs, ldY);
        baemm::launch_mass_dot_real(c.mesh, c.mass_values_fp64(), alpha, dX, nrhs, beta, dY, nrhs, nrhs, c.stream);
        d2h_block<double>(c, Y, ldY, dY, nv, nrhs);
        c.sync();
    });
}

// ---- solvers -----------------------------------------------------------------------


int baemm_far_field_parameters(baemm_ctx *ctx, const double *kappa, int wcc, const double *inc, int wcs, double *Y,
                               int type, const double *eta, double cg_tol, double gmres_tol)
{
    return guarded(ctx, [&](Ctx &c) {
        check_solver_args(c, kappa, wcc, inc, wcs);
        BAEMM_REQUIRE(Y, BAEMM_ERR_ARG, "null output");
        const int wc = wcc * wcs;
        double2 *dY = c.io_c.reserve(c.mesh.nm * wc);
        c.farfield_parameters(kappa, wcc, inc, wcs, dY, type, eta ? eta : kappa, cg_tol, gmres_tol);
        BAEMM_CUDA(cudaMemcpyAsync(Y, dY, c.mesh.nm * wc * sizeof(double2), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
    });
}
int baemm_far_field(baemm_ctx *ctx, const double *kappa, int wcc, const double *inc, int wcs, double *Y, int type,
                    double cg_tol, double gmres_tol)
{
    return baemm_far_field_parameters(ctx, kappa, wcc, inc, wcs, Y, type, kappa, cg_tol, gmres_tol);
}

int baemm_boundary_potential(baemm_ctx *ctx, const double *kappa, double *coeff, const double *wave, double *phi,
                             int wcc, int wcs, double cg_tol, double gmres_tol)
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(kappa && coeff && wave && phi && wcc >= 1 && wcs >= 1, BAEMM_ERR_ARG, "invalid arguments");
        const int wc = wcc * wcs;
        const int64_t N = c.mesh.nv * wc;
        double2 *dw = c.io_a.reserve(N), *dp = c.io_b.reserve(N);
        BAEMM_CUDA(cudaMemcpyAsync(dw, wave, N * sizeof(double2), cudaMemcpyHostToDevice, c.stream));
        c.boundary_potential(kappa, reinterpret_cast<zc *>(coeff), dw, dp, kappa, wcc, wcs, cg_tol, gmres_tol);
        BAEMM_CUDA(cudaMemcpyAsync(phi, dp, N * sizeof(double2), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
    });
}

int baemm_dirichlet_to_neumann(baemm_ctx *ctx, const double *kappa, const double *wave, double *out, int wcc, int wcs,
                               double cg_tol, double gmres_tol)
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(kappa && wave && out && wcc >= 1 && wcs >= 1, BAEMM_ERR_ARG, "invalid arguments");
        const int wc = wcc * wcs;
        const int64_t N = c.mesh.nv * wc;
        double2 *dw = c.io_a.reserve(N), *dp = c.io_b.reserve(N);
        BAEMM_CUDA(cudaMemcpyAsync(dw, wave, N * sizeof(double2), cudaMemcpyHostToDevice, c.stream));
        c.dirichlet_to_neumann(kappa, dw, dp, wcc, wcs, cg_tol, gmres_tol);
        BAEMM_CUDA(cudaMemcpyAsync(out, dp, N * sizeof(double2), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
    });
}

int baemm_derivative_ff_helper(baemm_ctx *ctx, const double *kappa, int wcc, const double *inc, int wcs,
                               double *du_dn, int type, double cg_tol, double gmres_tol)
{
    return guarded(ctx, [&](Ctx &c) {
        check_solver_args(c, kappa, wcc, inc, wcs);
        BAEMM_REQUIRE(du_dn, BAEMM_ERR_ARG, "null du_dn");
        const int64_t N = c.mesh.nv * wcc * wcs;
        double2 *dd = c.io_c.reserve(N);
        c.derivative_helper(kappa, wcc, inc, wcs, dd, type, cg_tol, gmres_tol);
        BAEMM_CUDA(cudaMemcpyAsync(du_dn, dd, N * sizeof(double2), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
    });
}



int baemm_derivative_ff(baemm_ctx *ctx, const double *kappa, int wcc, const double *inc, int wcs, const double *X_in,
                        double *Y_out, double **du_dn, int type, double cg_tol, double gmres_tol)
{
    return guarded(ctx, [&](Ctx &c) {
        check_solver_args(c, kappa, wcc, inc, wcs);
        BAEMM_REQUIRE(X_in && Y_out, BAEMM_ERR_ARG, "null argument");
        const int wc = wcc * wcs;
        const int64_t nv = c.mesh.nv, nm = c.mesh.nm;
        double2 *dd = c.io_c.reserve(nv * wc), *dY = c.io_b.reserve(nm * wc);
        double *dX = c.io_r1.reserve(3 * nv);
        ensure_du_dn(c, kappa, wcc, inc, wcs, du_dn, type, cg_tol, gmres_tol, dd);
        BAEMM_CUDA(cudaMemcpyAsync(dX, X_in, 3 * nv * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        c.derivative(kappa, wcc, inc, wcs, dX, dY, dd, cg_tol, gmres_tol);
        BAEMM_CUDA(cudaMemcpyAsync(Y_out, dY, nm * wc * sizeof(double2), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
    });
}

int baemm_adjoint_derivative_ff(baemm_ctx *ctx, const double *kappa, int wcc, const double *inc, int wcs,
                                const double *g, double *Y_out, double **du_dn, int type, double cg_tol,
                                double gmres_tol)
{
    return guarded(ctx, [&](Ctx &c) {
        check_solver_args(c, kappa, wcc, inc, wcs);
        BAEMM_REQUIRE(g && Y_out, BAEMM_ERR_ARG, "null argument");
        const int wc = wcc * wcs;
        const int64_t nv = c.mesh.nv, nm = c.mesh.nm;
        double2 *dd = c.io_c.reserve(nv * wc), *dg = c.io_a.reserve(nm * wc);
        double *dY = c.io_r2.reserve(3 * nv);
        ensure_du_dn(c, kappa, wcc, inc, wcs, du_dn, type, cg_tol, gmres_tol, dd);
        BAEMM_CUDA(cudaMemcpyAsync(dg, g, nm * wc * sizeof(double2), cudaMemcpyHostToDevice, c.stream));
        c.adjoint_derivative(kappa, wcc, inc, wcs, dg, dY, dd, cg_tol, gmres_tol);
        BAEMM_CUDA(cudaMemcpyAsync(Y_out, dY, 3 * nv * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
    });
}

int baemm_gauss_newton_solve(baemm_ctx *ctx, const double *kappa, int wcc, const double *inc, int wcs,
                             baemm_real_op M, void *M_user, baemm_real_op P, void *P_user, double alpha,
                             const double *B_in, int64_t ldB, double beta, double *X_out, int64_t ldX, double **du_dn,
                             int type, double cg_tol, double gmres_tol_inner, double gmres_tol_outer, int solver,
                             int *succeeded)
{
    return guarded(ctx, [&](Ctx &c) {
        check_solver_args(c, kappa, wcc, inc, wcs);
        BAEMM_REQUIRE(M && P && B_in && X_out && ldB >= 3 && ldX >= 3, BAEMM_ERR_ARG, "invalid arguments");
        BAEMM_REQUIRE(solver == 0 || solver == 1, BAEMM_ERR_ARG, "solver must be 0 (GMRES) or 1 (CG)");
        const int wc = wcc * wcs;
        const int64_t nv = c.mesh.nv, nm = c.mesh.nm, n3 = 3 * nv;
        DevBuf<double2> dd, dDF;
        DevBuf<double> dB, dX, dys, dxin, dyout;
        dd.reserve(nv * wc); dDF.reserve(nm * wc);
        dB.reserve(n3); dX.reserve(n3); dys.reserve(n3); dxin.reserve(n3); dyout.reserve(n3);
        ensure_du_dn(c, kappa, wcc, inc, wcs, du_dn, type, cg_tol, gmres_tol_inner, dd.p);
        h2d_block<double>(c, dB.p, B_in, nv, 3, ldB);
        std::vector<double> xh(n3), yh(n3);
        // A x = M x + Mass . DF* DF x   (FarField.hpp:551-572)
        auto Aop = [&](const double *x, double *y) {
            BAEMM_CUDA(cudaMemcpyAsync(xh.data(), x, n3 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
            c.sync();
            M(xh.data(), yh.data(), M_user);
            BAEMM_CUDA(cudaMemcpyAsync(y, yh.data(), n3 * sizeof(double), cudaMemcpyHostToDevice, c.stream));
            c.derivative(kappa, wcc, inc, wcs, x, dDF.p, dd.p, cg_tol, gmres_tol_inner);
            c.adjoint_derivative(kappa, wcc, inc, wcs, dDF.p, dys.p, dd.p, cg_tol, gmres_tol_inner);
            baemm::launch_mass_dot_real(c.mesh, c.mass_values_fp64(), 1.0, dys.p, 3, 1.0, y, 3, 3, c.stream);
            c.sync();
        };
        auto Pop = [&](const double *x, double *y) {
            BAEMM_CUDA(cudaMemcpyAsync(xh.data(), x, n3 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
            c.sync();
            P(xh.data(), yh.data(), P_user);
            BAEMM_CUDA(cudaMemcpyAsync(y, yh.data(), n3 * sizeof(double), cudaMemcpyHostToDevice, c.stream));
            c.sync();
        };
        bool ok = false;
        int iters = 0;
        double relres = 0.0;
        if (solver == 0)
        {
            // outer GMRES<1> on 3n reals (FarField.hpp:538-539, 575-579)
            auto st = c.gmres_r.solve(n3, 1, c.gmres_max_iter, c.gmres_max_restarts, Aop, Pop, 1.0, dB.p, 1, 0.0,
                                      dX.p, 1, gmres_tol_outer, c.stream);
            ok = st.converged;
            iters = st.iterations;
            relres = st.max_rel_res;
        }
        else
        {
            // preconditioned CG on the symmetric positive (semi)definite M + DF* DF
            DevBuf<double> r, z, p, q;
            r.reserve(n3); z.reserve(n3); p.reserve(n3); q.reserve(n3);
            BAEMM_CUDA(cudaMemsetAsync(dX.p, 0, n3 * sizeof(double), c.stream));
            BAEMM_CUDA(cudaMemcpyAsync(r.p, dB.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
            Pop(r.p, z.p);
            BAEMM_CUDA(cudaMemcpyAsync(p.p, z.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
            double rz = baemm::device_dot(r.p, z.p, n3, c.reduce_scratch, c.stream);
            const double bn = std::sqrt(baemm::device_dot(dB.p, dB.p, n3, c.reduce_scratch, c.stream));
            double rn = bn;
            const int max_it = c.gmres_max_iter * c.gmres_max_restarts;
            while (!(rn <= gmres_tol_outer * bn) && iters < max_it)
            {
                Aop(p.p, q.p);
                const double pq = baemm::device_dot(p.p, q.p, n3, c.reduce_scratch, c.stream);
                if (pq == 0.0) break;
                const double a = rz / pq;
                baemm::launch_axpby<double>(n3, 1, a, p.p, 1, 1.0, dX.p, 1, c.stream);
                baemm::launch_axpby<double>(n3, 1, -a, q.p, 1, 1.0, r.p, 1, c.stream);
                Pop(r.p, z.p);
                const double rzn = baemm::device_dot(r.p, z.p, n3, c.reduce_scratch, c.stream);
                rn = std::sqrt(baemm::device_dot(r.p, r.p, n3, c.reduce_scratch, c.stream));
                baemm::launch_axpby<double>(n3, 1, 1.0, z.p, 1, rz != 0.0 ? rzn / rz : 0.0, p.p, 1, c.stream);
                rz = rzn;
                ++iters;
            }
            ok = rn <= gmres_tol_outer * bn;
            relres = bn > 0 ? rn / bn : 0.0;
        }
        // FarField.hpp:575-599: with ldX == 3 the solution is written directly (alpha, beta unused)
        if (ldX == 3)
            d2h_block<double>(c, X_out, 3, dX.p, nv, 3);
        else
        {
            DevBuf<double> dXo;
            dXo.reserve(n3);
            h2d_block<double>(c, dXo.p, X_out, nv, 3, ldX);
            baemm::launch_axpby<double>(nv, 3, alpha, dX.p, 3, beta, dXo.p, 3, c.stream);
            d2h_block<double>(c, X_out, ldX, dXo.p, nv, 3);
            c.sync();
        }
        c.sync();
        c.stats.gmres_iterations = iters;
        c.stats.gmres_converged = ok;
        c.stats.gmres_relative_residual = relres;
        if (succeeded) *succeeded = ok ? 1 : 0;
    });
}

int baemm_set_profiling(baemm_ctx *ctx, int on)
{
    return guarded(ctx, [&](Ctx &c) {
        c.profiling = on != 0;
        c.prof_valid = false;
    });
}

int baemm_last_apply_times(baemm_ctx *ctx, float *ms3)
{
    return guarded(ctx, [&](Ctx &c) {
        BAEMM_REQUIRE(ms3, BAEMM_ERR_ARG, "null output");
        BAEMM_REQUIRE(c.prof_valid, BAEMM_ERR_ARG, "no profiled apply (enable baemm_set_profiling first)");
        BAEMM_CUDA(cudaEventSynchronize(c.prof_ev[3]));
        for (int q = 0; q < 3; ++q) BAEMM_CUDA(cudaEventElapsedTime(&ms3[q], c.prof_ev[q], c.prof_ev[q + 1]));
    });
}

int64_t baemm_kernel_launch_count(void) { return (int64_t)baemm::g_kernel_launches.load(); }

void baemm_free(void *p) { std::free(p); }

} // extern "C"
