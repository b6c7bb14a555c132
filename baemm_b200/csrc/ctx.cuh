// The context behind baemm_ctx: the device-resident mesh, the loaded operator
// parameters, work buffers and the solvers.  Mirrors the state of the
// reference class Helmholtz_OpenCL (MemberVariables.hpp:36-98) with the
// OpenCL objects replaced by device buffers on one CUDA stream.
#pragma once
#include <complex>
#include <functional>
#include <map>
#include <string>
#include <vector>

#include "krylov.cuh"
#include "ops.cuh"
#include "pack.cuh"

namespace baemm
{

using zc = std::complex<double>;

class Ctx
{
public:
    Ctx(const double *coords, int64_t nv, const int32_t *tris, int64_t nt, const double *meas, int64_t nm, int device,
        int cpu_threads);
    ~Ctx();

    // ---- state ----------------------------------------------------------------
    int device = 0;
    int cpu_threads = 1;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    MeshDev mesh;
    std::vector<double> meas_h;                     // nm x 3 (as given)
    std::vector<int32_t> mass_outer_h, mass_inner_h;

    int wave_count = 0, wave_chunk_size = 16, wave_chunk_count = 0;
    std::vector<double> kappa_h;
    std::vector<zc> coeff_h;                        // unscaled, wcc x 4
    double factor_h = 1.0;
    OpFlags flags;
    std::vector<ChunkParamsF> prm_f_h;
    std::vector<ChunkParamsD> prm_d_h;
    DevBuf<ChunkParamsF> prm_f;
    std::vector<ChunkParamsF> prm16_f_h;   // per 16-column group (tensor-core form)
    std::vector<float2> prm_bc_h;
    DevBuf<ChunkParamsF> prm16_f;
    TcCoeffForm tc_form;                    // coefficient structure the tensor-core form specialises on
    DevBuf<float2> prm_bc;                  // broadcast parameter pairs of the 16-column groups (packed launches)
    DevBuf<uint8_t> tc_img;                 // the tensor-core form's expanded B operand (launch_tc_expand)
    Packer *packer = nullptr;               // shared packer of concurrent solves' applies (not owned)
    DevBuf<ChunkParamsD> prm_d;
    bool operators_loaded = false;

    bool use_diagonal = true;
    int block_size = 64;
    int gmres_max_iter = 30, gmres_max_restarts = 3;
    int apply_mode = BAEMM_APPLY_FP32;
    int dense_variant = 0;            // plain FP32 dense kernel variant (launch_boundary_dense)
    TcTuning tc_tune;                 // tensor-core form settings (TcTuning in ops.cuh)
    DevBuf<float2> tc_ws;             // tensor-core form: partial sums of target blocks split between CTAs
    bool tc_geo_ready = false;        // mesh.tgeo_f built
    int ir_max_steps = 0;
    double ir_inner_tol = 1e-4;
    baemm_solve_stats stats{};
    DevBuf<int> tc_err;               // error word of the tensor-core kernel's bounded waits
    DevBuf<double> reduce_scratch;    // per-block partial sums of device_dot / device_colnorms
    int *tc_err_host = nullptr;
    bool tc_pending = false;          // a tensor-core launch since the last error check
    bool profiling = false;
    cudaEvent_t prof_ev[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t handoff_ev = nullptr;   // orders a newly set stream after the previous one
    bool prof_valid = false;
    std::string last_error;

    // work buffers
    DevBuf<float2> Btri_f, Ctri_f, ff_partial_f;
    DevBuf<double2> Btri_d, Ctri_d, ff_partial_d;
    DevBuf<float> dirs_f;
    DevBuf<double> dirs_d;
    DevBuf<float> pts_f;                // near field: evaluation points, npts x 4
    DevBuf<double> pts_d;
    DevBuf<float2> Cpts_f;              // near field: values at the points, npts x wc
    DevBuf<double2> Cpts_d;
    DevBuf<double2> io_a, io_b, io_c;   // host-API staging
    DevBuf<double> io_r1, io_r2, tri_r;
    // solver scratch (one buffer per role; the compositions nest)
    DevBuf<double2> sv_wave, sv_phi, sv_bc, sv_bcw, sv_hw, sv_dv, sv_prod, sv_res, sv_d, sv_tmp;
    DevBuf<double> sv_xn, sv_yw, sv_ytri, sv_ys;
    CgSolver cg;
    GmresSolver<double2> gmres_c;
    GmresSolver<double> gmres_r;

    // ---- parameters -------------------------------------------------------------
    // LoadParameters.hpp:20-81
    void load_parameters(const double *kappa, const zc *coeff, int wc, int wcs, double factor);
    void require_loaded() const;

    // ---- operators on device blocks (async on `stream`) --------------------------
    template <class Text>
    void apply_boundary(Text alpha, const Text *B, int64_t ldB, Text beta, Text *C, int64_t ldC);
    // One row shard of the apply: C = alpha AvOp^T|[r0,r1) (K[r0,r1) + diag) AvOp B
    // [+ alpha c0 M B if with_mass] + beta C.  The shards of a partition of the
    // triangles, with the mass term and beta on one of them, sum to the apply.
    template <class Text>
    void apply_boundary_rows(Text alpha, const Text *B, int64_t ldB, Text beta, Text *C, int64_t ldC, int64_t r0,
                             int64_t r1, bool with_mass);
    // The dense stage alone on device triangle blocks (BoundaryOperatorKernel.hpp:5-28):
    // Ctri rows [r0, r1) = K[r0, r1) Btri in the current arithmetic (R = float: plain or
    // tensor-core form; R = double: FP64).
    template <class R>
    void boundary_kernel_rows(const cplx<R> *Btri, cplx<R> *Ctri, int64_t r0, int64_t r1)
    {
        dense_apply<R>(Btri, Ctri, r0, r1);
    }
    // Far field: C (nm x wc) = alpha FF B + beta C   (ApplyFarFieldOperators.hpp:356-412)
    void apply_farfield(zc alpha, const double2 *B, int64_t ldB, zc beta, double2 *C, int64_t ldC);
    // ApplyNearFieldOperators.hpp:56-122 on device blocks: C (npts x wc) =
    // alpha K(points) AvOp B + beta C at the points pts3 (npts x 3 doubles,
    // device), in the apply arithmetic (FP32, tensor-core or FP64).
    template <class Text>
    void apply_nearfield(Text alpha, const Text *B, int64_t ldB, Text beta, Text *C, int64_t ldC, const double *pts3,
                         int64_t npts);
    // Incident wave: C = alpha wave + beta C (CreateIncidentWave.hpp:54-127), dirs on host (wcs x 3)
    void incident(zc alpha, const double *dirs, zc beta, double2 *C, int64_t ldC, int type);
    // Herglotz wave of g (device, nm x ld): C = alpha HW + beta C (CreateHerglotzWave.hpp:50-95)
    void herglotz(zc alpha, const double2 *g, int64_t ldg, zc beta, double2 *C, int64_t ldC);
    // The O(N wc) and O(m N wc) steps around the dense apply (incident and
    // Herglotz waves, far field, mass values, normal-field helpers) run in FP64
    // when the apply is FP64 or when FP64 iterative refinement is on.
    bool aux_fp64() const { return apply_mode == BAEMM_APPLY_FP64 || ir_max_steps > 0; }
    bool mass_values_fp64() const { return aux_fp64(); }
    // CG mass inverse on real columns (device); returns convergence
    bool mass_inverse_real(const double *X, int64_t ldX, double *Y, int64_t ldY, int ncols, double tol);
    bool mass_inverse_complex(const double2 *X, int64_t ldX, double2 *Y, int64_t ldY, int ncols, double tol);

    // ---- solvers (device blocks, nv x wc) -------------------------------------------
    // GMRES on the loaded boundary operators with P = M^-1 (BoundaryPotential_parameters /
    // DirichletToNeumann core, FarField.hpp:706-768, 828-874), optional FP64 refinement.
    void bie_solve(const double *kappa, const zc *coeff4, const double2 *rhs, double2 *sol, int wcc, int wcs,
                   double cg_tol, double gmres_tol);
    void boundary_potential(const double *kappa, zc *coeff, const double2 *wave, double2 *phi, const double *eta,
                            int wcc, int wcs, double cg_tol, double gmres_tol);
    void dirichlet_to_neumann(const double *kappa, const double2 *wave, double2 *du_dn, int wcc, int wcs,
                              double cg_tol, double gmres_tol);
    void farfield_parameters(const double *kappa, int wcc, const double *inc, int wcs, double2 *Y, int type,
                             const double *eta, double cg_tol, double gmres_tol);
    void derivative_helper(const double *kappa, int wcc, const double *inc, int wcs, double2 *du_dn, int type,
                           double cg_tol, double gmres_tol);
    void dot_with_normals(const double *X, double *Y, double cg_tol);
    void multiply_with_normals(const double2 *X, double *Y, double factor, double cg_tol);
    void derivative(const double *kappa, int wcc, const double *inc, int wcs, const double *X, double2 *Y,
                    const double2 *du_dn, double cg_tol, double gmres_tol);
    void adjoint_derivative(const double *kappa, int wcc, const double *inc, int wcs, const double2 *g, double *Y,
                            const double2 *du_dn, double cg_tol, double gmres_tol);

    void sync();
    void check_tc_error();
    // Continue on stream `s` (null: the own stream), ordered after the work
    // already queued on the current one, without a host synchronisation.
    void switch_stream(cudaStream_t s);
    std::string device_info() const;
    // Times the dense-kernel settings of `mode` on the loaded operators and
    // keeps the fastest (tune.cu).
    void autotune(int mode, int repeats, baemm_tune_result *out);
    // ---- CUDA graphs of the solver's inner operators (baemm_set_graphs) --------
    // The GMRES operator apply and the CG mass inverse are fixed launch
    // sequences; with use_graphs on, the second call with the same operands is
    // captured and later calls replay the graph.  Any device-buffer
    // reallocation in the library (g_devbuf_epoch) or a change of the loaded
    // operators, mesh, mode or tuning (graph_state) drops the graphs.
    struct GraphKey
    {
        int kind;
        const void *x;
        const void *y;
        int64_t ldx, ldy;
        long long a, b;   // kind-specific (columns, tolerance bits, mode, ...)
        bool operator<(const GraphKey &o) const
        {
            if (kind != o.kind) return kind < o.kind;
            if (x != o.x) return x < o.x;
            if (y != o.y) return y < o.y;
            if (ldx != o.ldx) return ldx < o.ldx;
            if (ldy != o.ldy) return ldy < o.ldy;
            if (a != o.a) return a < o.a;
            return b < o.b;
        }
    };
    struct GraphEntry
    {
        cudaGraphExec_t exec = nullptr;
        int eager_runs = 0;
        bool broken = false;
    };
    bool use_graphs = false;
    long long graph_state = 0;           // bumped when captured work would change
    long long graphs_epoch = -1, graphs_state = -1;
    long long graph_captures = 0, graph_replays = 0;
    std::map<GraphKey, GraphEntry> graph_cache;
    void clear_graphs();
    // Runs `enqueue` (which only enqueues work on `stream`) through the cache.
    void run_graphed(const GraphKey &key, const std::function<void()> &enqueue);

    // Replace the mesh (same measurement directions); unloads the operators.
    void set_mesh(const double *coords, int64_t nv, const int32_t *tris, int64_t nt);
    long long mesh_generation = 0;   // bumped by every mesh set-up

private:
    void init_mesh(const double *coords, int64_t nv, const int32_t *tris, int64_t nt);
    void build_topology(const int32_t *tris);
    template <class R>
    void dense_apply(const cplx<R> *Btri, cplx<R> *Ctri, int64_t r0 = 0, int64_t r1 = -1);
};

} // namespace baemm

// The opaque handle of the C ABI (include/baemm.h).
struct baemm_ctx
{
    baemm::Ctx *impl = nullptr;
};
