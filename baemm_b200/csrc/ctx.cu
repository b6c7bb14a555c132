// Context set-up, parameter loading and the operator applies.
#include "ctx.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <sstream>

namespace baemm
{

std::atomic<long long> g_kernel_launches{0};
std::atomic<long long> g_devbuf_epoch{0};

Ctx::Ctx(const double *coords, int64_t nv, const int32_t *tris, int64_t nt, const double *meas, int64_t nm, int dev,
         int threads)
    : device(dev), cpu_threads(threads)
{
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
    {
        (void)cudaGetLastError();
        throw Error(BAEMM_ERR_CUDA, std::string("no CUDA device available: ") + cudaGetErrorString(e));
    }
    // Helmholtz_OpenCL.hpp:217-224: an out-of-range device number falls back to device 0.
    if (device < 0 || device >= count) device = 0;
    BAEMM_CUDA(cudaSetDevice(device));
    BAEMM_CUDA(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
    stream = own_stream;

    mesh.nm = nm;
    meas_h.assign(meas, meas + 3 * nm);
    init_mesh(coords, nv, tris, nt);

    // Measurement directions padded to 4 (InitializeBuffers.hpp:415-424).
    std::vector<float> mf(4 * std::max<int64_t>(nm, 1), 0.f);
    std::vector<double> md(4 * std::max<int64_t>(nm, 1), 0.0);
    for (int64_t i = 0; i < nm; ++i)
        for (int d = 0; d < 3; ++d)
        {
            mf[4 * i + d] = (float)meas[3 * i + d];
            md[4 * i + d] = meas[3 * i + d];
        }
    BAEMM_CUDA(cudaMemcpyAsync(mesh.meas_f.reserve(mf.size()), mf.data(), mf.size() * sizeof(float),
                               cudaMemcpyHostToDevice, stream));
    BAEMM_CUDA(cudaMemcpyAsync(mesh.meas_d.reserve(md.size()), md.data(), md.size() * sizeof(double),
                               cudaMemcpyHostToDevice, stream));
    BAEMM_CUDA(cudaMemsetAsync(tc_err.reserve(1), 0, sizeof(int), stream));
    BAEMM_CUDA(cudaMallocHost(&tc_err_host, sizeof(int)));
    sync();
}

// Mesh-dependent state (Initialize.hpp:57-353): coordinates and triangles on
// the device, the integer topology, geometry, mass values.  Device buffers
// only grow, so a context re-meshed with a mesh no larger than one it held
// before allocates nothing.
void Ctx::init_mesh(const double *coords, int64_t nv, const int32_t *tris, int64_t nt)
{
    mesh.nv = nv;
    mesh.nt = nt;
    BAEMM_CUDA(cudaMemcpyAsync(mesh.coords.reserve(3 * nv), coords, 3 * nv * sizeof(double), cudaMemcpyHostToDevice,
                               stream));
    BAEMM_CUDA(cudaMemcpyAsync(mesh.tris.reserve(3 * nt), tris, 3 * nt * sizeof(int32_t), cudaMemcpyHostToDevice,
                               stream));
    build_topology(tris);   // ends with a stream synchronisation: the host arrays are free afterwards

    mesh.mid_f.reserve(4 * nt); mesh.nrm_f.reserve(4 * nt);
    mesh.area_f.reserve(nt); mesh.a3_f.reserve(nt); mesh.diag_f.reserve(nt);
    mesh.mid_d.reserve(4 * nt); mesh.nrm_d.reserve(4 * nt);
    mesh.area_d.reserve(nt); mesh.a3_d.reserve(nt); mesh.diag_d.reserve(nt);
    mesh.mass_f.reserve(mass_inner_h.size()); mesh.mass_d.reserve(mass_inner_h.size());
    mesh.lumped_f.reserve(nv); mesh.lumped_d.reserve(nv);
    launch_geometry(mesh, false, stream);
    launch_geometry(mesh, true, stream);
    launch_mass_values(mesh, false, stream);
    launch_mass_values(mesh, true, stream);
    tc_geo_ready = false;
    operators_loaded = false;
    ++mesh_generation;
    ++graph_state;
}

// Replaces the mesh of a live context (no reference counterpart: the
// reference builds a new Helmholtz_OpenCL per mesh).
void Ctx::set_mesh(const double *coords, int64_t nv, const int32_t *tris, int64_t nt)
{
    BAEMM_CUDA(cudaSetDevice(device));
    sync();
    init_mesh(coords, nv, tris, nt);
    sync();
}

void Ctx::clear_graphs()
{
    for (auto &kv : graph_cache)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    graph_cache.clear();
}

void Ctx::run_graphed(const GraphKey &key, const std::function<void()> &enqueue)
{
    // Capture needs a stream of our own kind (not the legacy default stream)
    // and nothing host-side inside the work (profiling reads events back).
    if (!use_graphs || profiling || stream == nullptr || stream == cudaStreamLegacy)
    {
        enqueue();
        return;
    }
    const long long epoch = g_devbuf_epoch.load(std::memory_order_relaxed);
    if (epoch != graphs_epoch || graph_state != graphs_state)
    {
        clear_graphs();
        graphs_epoch = epoch;
        graphs_state = graph_state;
    }
    GraphEntry &e = graph_cache[key];
    if (e.broken || (!e.exec && e.eager_runs == 0))
    {
        // first use of these operands (it may allocate), or not capturable
        ++e.eager_runs;
        enqueue();
        return;
    }
    if (!e.exec)
    {
        BAEMM_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        bool failed = false;
        try
        {
            enqueue();
        }
        catch (const Error &)
        {
            failed = true;
        }
        cudaGraph_t g = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(stream, &g);
        if (failed || ec != cudaSuccess || !g ||
            g_devbuf_epoch.load(std::memory_order_relaxed) != graphs_epoch ||
            cudaGraphInstantiate(&e.exec, g, 0) != cudaSuccess)
        {
            (void)cudaGetLastError();
            if (e.exec) cudaGraphExecDestroy(e.exec);
            e.exec = nullptr;
            e.broken = true;
            if (g) cudaGraphDestroy(g);
            enqueue();   // run it uncaptured
            return;
        }
        cudaGraphDestroy(g);
        ++graph_captures;
    }
    BAEMM_CUDA(cudaGraphLaunch(e.exec, stream));
    ++graph_replays;
    if (apply_mode == BAEMM_APPLY_TC) tc_pending = true;   // the graph may hold the tensor-core kernel
}

Ctx::~Ctx()
{
    clear_graphs();
    if (tc_err_host) cudaFreeHost(tc_err_host);
    for (auto &e : prof_ev)
        if (e) cudaEventDestroy(e);
    if (handoff_ev) cudaEventDestroy(handoff_ev);
    if (own_stream)
    {
        cudaStreamSynchronize(own_stream);
        cudaStreamDestroy(own_stream);
    }
}

void Ctx::switch_stream(cudaStream_t s)
{
    if (!s) s = own_stream;
    if (s == stream) return;
    if (!handoff_ev) BAEMM_CUDA(cudaEventCreateWithFlags(&handoff_ev, cudaEventDisableTiming));
    BAEMM_CUDA(cudaEventRecord(handoff_ev, stream));
    BAEMM_CUDA(cudaStreamWaitEvent(s, handoff_ev, 0));
    stream = s;
}

void Ctx::sync()
{
    BAEMM_CUDA(cudaStreamSynchronize(stream));
    if (tc_pending) check_tc_error();
}

// The tensor-core kernel reports a bounded wait that gave up through tc_err.
void Ctx::check_tc_error()
{
    tc_pending = false;
    BAEMM_CUDA(cudaMemcpyAsync(tc_err_host, tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    BAEMM_CUDA(cudaStreamSynchronize(stream));
    if (*tc_err_host != 0)
    {
        const int code = *tc_err_host;
        BAEMM_CUDA(cudaMemsetAsync(tc_err.p, 0, sizeof(int), stream));
        BAEMM_CUDA(cudaStreamSynchronize(stream));
        throw Error(BAEMM_ERR_TIMEOUT, "tensor-core apply: a bounded device wait gave up (code " +
                                           std::to_string(code) + ")");
    }
}

// Integer topology (host): AvOp columns sorted per triangle (Initialize.hpp:307-313),
// AvOp^T as a vertex -> triangle CSR in ascending triangle order (Initialize.hpp:315),
// and the sparsity pattern of the P1 mass matrix (Initialize.hpp:329-334).
void Ctx::build_topology(const int32_t *tris)
{
    const int64_t nv = mesh.nv, nt = mesh.nt;
    std::vector<int32_t> ts(3 * nt);
    for (int64_t i = 0; i < nt; ++i)
    {
        int32_t v[3] = {tris[3 * i], tris[3 * i + 1], tris[3 * i + 2]};
        std::sort(v, v + 3);
        ts[3 * i] = v[0]; ts[3 * i + 1] = v[1]; ts[3 * i + 2] = v[2];
    }
    std::vector<int32_t> ao(nv + 1, 0), ai(3 * nt);
    for (int64_t e = 0; e < 3 * nt; ++e) ao[ts[e] + 1]++;
    for (int64_t v = 0; v < nv; ++v) ao[v + 1] += ao[v];
    {
        std::vector<int32_t> pos(ao.begin(), ao.end() - 1);
        for (int64_t i = 0; i < nt; ++i)
            for (int q = 0; q < 3; ++q) ai[pos[ts[3 * i + q]]++] = (int32_t)i;
    }
    // mass pattern: unique neighbours (incl. self) per vertex, sorted
    std::vector<int64_t> keys;
    keys.reserve(9 * nt);
    for (int64_t i = 0; i < nt; ++i)
        for (int p = 0; p < 3; ++p)
            for (int q = 0; q < 3; ++q) keys.push_back((int64_t)tris[3 * i + p] * nv + tris[3 * i + q]);
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    mass_outer_h.assign(nv + 1, 0);
    mass_inner_h.resize(keys.size());
    for (size_t e = 0; e < keys.size(); ++e)
    {
        mass_outer_h[keys[e] / nv + 1]++;
        mass_inner_h[e] = (int32_t)(keys[e] % nv);
    }
    for (int64_t v = 0; v < nv; ++v) mass_outer_h[v + 1] += mass_outer_h[v];

    auto up = [&](DevBuf<int32_t> &d, const std::vector<int32_t> &h) {
        BAEMM_CUDA(cudaMemcpyAsync(d.reserve(std::max<size_t>(h.size(), 1)), h.data(), h.size() * sizeof(int32_t),
                                   cudaMemcpyHostToDevice, stream));
    };
    up(mesh.tri_sorted, ts);
    up(mesh.avt_outer, ao);
    up(mesh.avt_inner, ai);
    up(mesh.mass_outer, mass_outer_h);
    up(mesh.mass_inner, mass_inner_h);
    // The host vectors must outlive the asynchronous copies.
    sync();
}

void Ctx::load_parameters(const double *kappa, const zc *coeff, int wc, int wcs, double factor)
{
    BAEMM_REQUIRE(wcs >= 1 && wcs <= 64 && (wcs & (wcs - 1)) == 0, BAEMM_ERR_SIZE,
                  "wave_chunk_size must be a power of two <= 64");
    BAEMM_REQUIRE(wc >= 1 && wc <= kMaxWaveCount / 2, BAEMM_ERR_SIZE, "wave_count must be in [1, 512]");
    BAEMM_REQUIRE(wc % wcs == 0, BAEMM_ERR_SIZE, "wave_count must be a multiple of wave_chunk_size");
    BAEMM_REQUIRE(kappa && coeff, BAEMM_ERR_ARG, "kappa and coeff must not be null");
    wave_count = wc;
    wave_chunk_size = wcs;
    wave_chunk_count = wc / wcs;
    const int wcc = wave_chunk_count;
    ++graph_state;
    kappa_h.assign(kappa, kappa + wcc);
    coeff_h.assign(coeff, coeff + 4 * wcc);
    factor_h = factor;
    prm_f_h.assign(wcc, ChunkParamsF{});
    prm_d_h.assign(wcc, ChunkParamsD{});
    flags = OpFlags{};
    // LoadParameters.hpp:56-80: c0 as is, c1..c3 * one_over_four_pi * factor, in float
    const float oofp = 1.0f / (2.0f * (2.0f * 3.14159265358979323846f));
    const double oofp_d = 1.0 / (4.0 * M_PI);
    for (int k = 0; k < wcc; ++k)
    {
        ChunkParamsF &pf = prm_f_h[k];
        ChunkParamsD &pd = prm_d_h[k];
        pf.kappa = (float)kappa[k];
        pd.kappa = kappa[k];
        for (int q = 0; q < 4; ++q)
        {
            std::complex<float> z((float)coeff[4 * k + q].real(), (float)coeff[4 * k + q].imag());
            zc zd = coeff[4 * k + q];
            if (q > 0)
            {
                z = z * oofp * (float)factor;
                zd = zd * oofp_d * factor;
            }
            pf.c[q] = make_float2(z.real(), z.imag());
            pd.c[q] = make_double2(zd.real(), zd.imag());
            const bool re = z.real() != 0.f, im = z.imag() != 0.f;
            switch (q)
            {
                case 0: flags.re_mass |= re; flags.im_mass |= im; break;
                case 1: flags.re_sl |= re; flags.im_sl |= im; break;
                case 2: flags.re_dl |= re; flags.im_dl |= im; break;
                default: flags.re_adl |= re; flags.im_adl |= im; break;
            }
        }
    }
    BAEMM_CUDA(cudaMemcpyAsync(prm_f.reserve(wcc), prm_f_h.data(), wcc * sizeof(ChunkParamsF), cudaMemcpyHostToDevice,
                               stream));
    BAEMM_CUDA(cudaMemcpyAsync(prm_d.reserve(wcc), prm_d_h.data(), wcc * sizeof(ChunkParamsD), cudaMemcpyHostToDevice,
                               stream));
    // The tensor-core form works on groups of 16 columns: one parameter set per
    // group (a chunk of wave_chunk_size = 16 m columns repeats its set m times).
    if (wcs % 16 == 0)
    {
        const int groups = wc / 16, rep = wcs / 16;
        prm16_f_h.resize(groups);
        for (int gi = 0; gi < groups; ++gi) prm16_f_h[gi] = prm_f_h[gi / rep];
        BAEMM_CUDA(cudaMemcpyAsync(prm16_f.reserve(groups), prm16_f_h.data(), groups * sizeof(ChunkParamsF),
                                   cudaMemcpyHostToDevice, stream));
        tc_form = tc_coeff_form(prm16_f_h.data(), groups);
        tc_broadcast_params(prm16_f_h.data(), groups, prm_bc_h);
        BAEMM_CUDA(cudaMemcpyAsync(prm_bc.reserve(prm_bc_h.size()), prm_bc_h.data(), prm_bc_h.size() * sizeof(float2),
                                   cudaMemcpyHostToDevice, stream));
    }
    else
        tc_form = TcCoeffForm();
}

void Ctx::require_loaded() const
{
    BAEMM_REQUIRE(operators_loaded && wave_chunk_count >= 1, BAEMM_ERR_NOT_LOADED,
                  "boundary operators are not loaded (call baemm_load_boundary_operators first)");
}

template <class R>
void Ctx::dense_apply(const cplx<R> *Btri, cplx<R> *Ctri, int64_t r0, int64_t r1)
{
    if constexpr (std::is_same<R, double>::value)
        launch_boundary_dense<double>(mesh, flags, prm_d.p, wave_count, wave_chunk_size, Btri, Ctri, stream, 2, r0,
                                      r1);
    else if (apply_mode == BAEMM_APPLY_TC && tc_supported(wave_count, wave_chunk_size))
    {
        if (!tc_geo_ready)
        {
            launch_tc_tile_geometry(mesh, mesh.tgeo_f.reserve(tc_tile_geometry_floats(mesh.nt)), stream);
            tc_geo_ready = true;
        }
        // Only problems whose own launch cannot fill the GPU (at most two target blocks per SM) are packed;
        // a large one would hold its packed partners back until its own sweep ends.
        const int64_t blocks = (int64_t)(wave_count / (16 * tc_chunks_per_unit(wave_count, tc_tune.chunks))) *
                               ceil_div(mesh.nt, 128);
        if (packer && r0 == 0 && (r1 < 0 || r1 == mesh.nt) && blocks <= 2 * (int64_t)tc_sm_count() &&
            tc_packable(flags, tc_form, wave_count, wave_chunk_size))
        {
            // one problem of the packer's next launch (the stream waits for that launch)
            const uint8_t *img = launch_tc_expand(Btri, mesh.nt, wave_count, tc_img, stream);
            const TcPackItem item{mesh.mid_f, mesh.nrm_f, mesh.tgeo_f.p, img, Ctri, prm_bc.p, tc_err.p, mesh.nt,
                                  wave_count, tc_form.s};
            packer->apply(item, flags, tc_tune, stream);
            tc_pending = true;
            return;
        }
        const size_t ws_elems = tc_workspace_elems(tc_tune.ctas);
        launch_boundary_tc(mesh, flags, prm16_f.p, tc_form, wave_count, wave_chunk_size, mesh.tgeo_f.p, Btri, Ctri,
                           tc_ws.reserve(ws_elems), ws_elems, tc_img, tc_err.p, stream, tc_tune, r0,
                           r1);
        tc_pending = true;
    }
    else
        launch_boundary_dense<float>(mesh, flags, prm_f.p, wave_count, wave_chunk_size, Btri, Ctri, stream,
                                     dense_variant, r0, r1);
}

// ApplyBoundaryOperators.hpp:289-391 on device blocks.
template <class Text>
void Ctx::apply_boundary(Text alpha, const Text *B, int64_t ldB, Text beta, Text *C, int64_t ldC)
{
    apply_boundary_rows<Text>(alpha, B, ldB, beta, C, ldC, 0, mesh.nt, true);
}

template <class Text>
void Ctx::apply_boundary_rows(Text alpha, const Text *B, int64_t ldB, Text beta, Text *C, int64_t ldC, int64_t r0,
                              int64_t r1, bool with_mass)
{
    if (wave_chunk_count < 1) return;
    BAEMM_REQUIRE(r0 >= 0 && r0 <= r1 && r1 <= mesh.nt, BAEMM_ERR_ARG, "row range outside [0, simplex_count]");
    BAEMM_REQUIRE(ldB >= wave_count && ldC >= wave_count, BAEMM_ERR_ARG, "leading dimension smaller than wave_count");
    const bool layers = flags.any_layer();
    if (!layers && !flags.mass()) return;   // the reference leaves C_out untouched
    EpilogueArgs ea;
    ea.layers = layers;
    ea.sl_diag = layers && use_diagonal && flags.sl();
    ea.mass = flags.mass() && with_mass;
    ea.wc = wave_count;
    ea.wcs = wave_chunk_size;
    ea.t_begin = r0;
    ea.t_end = r1;
    const bool rows = r1 > r0;
    const int64_t tri_elems = mesh.nt * wave_count;
    if (profiling)
    {
        for (auto &e : prof_ev)
            if (!e) BAEMM_CUDA(cudaEventCreate(&e));
        BAEMM_CUDA(cudaEventRecord(prof_ev[0], stream));
    }
    auto mark = [&](int q) {
        if (profiling) BAEMM_CUDA(cudaEventRecord(prof_ev[q], stream));
    };
    if (apply_mode == BAEMM_APPLY_FP64)
    {
        double2 *Bt = Btri_d.reserve(tri_elems), *Ct = Ctri_d.reserve(tri_elems);
        if (layers) launch_avop<Text, double>(mesh, B, ldB, wave_count, Bt, stream);
        mark(1);
        if (layers && rows) dense_apply<double>(Bt, Ct, r0, r1);
        mark(2);
        launch_epilogue<Text, double>(mesh, ea, Ct, Bt, prm_d.p, B, ldB, alpha, beta, C, ldC, stream);
    }
    else
    {
        float2 *Bt = Btri_f.reserve(tri_elems), *Ct = Ctri_f.reserve(tri_elems);
        if (layers) launch_avop<Text, float>(mesh, B, ldB, wave_count, Bt, stream);
        mark(1);
        if (layers && rows) dense_apply<float>(Bt, Ct, r0, r1);
        mark(2);
        launch_epilogue<Text, float>(mesh, ea, Ct, Bt, prm_f.p, B, ldB, alpha, beta, C, ldC, stream);
    }
    mark(3);
    prof_valid = profiling;
}

template <class Text>
void Ctx::apply_nearfield(Text alpha, const Text *B, int64_t ldB, Text beta, Text *C, int64_t ldC, const double *pts3,
                          int64_t npts)
{
    if (wave_chunk_count < 1) return;
    // the near-field kernel reads the single- and double-layer coefficients only
    // (NearFieldOperatorKernel.cl:105-149); without either C is left untouched
    OpFlags nf;
    nf.re_sl = flags.re_sl;
    nf.im_sl = flags.im_sl;
    nf.re_dl = flags.re_dl;
    nf.im_dl = flags.im_dl;
    if (!nf.any_layer()) return;
    BAEMM_REQUIRE(ldB >= wave_count && ldC >= wave_count, BAEMM_ERR_ARG, "leading dimension smaller than wave_count");
    BAEMM_REQUIRE(npts >= 0, BAEMM_ERR_ARG, "negative evaluation point count");
    BAEMM_REQUIRE(npts <= kMaxMeshSize, BAEMM_ERR_SIZE, "at most 2^28 evaluation points per call");
    if (npts == 0) return;
    BAEMM_REQUIRE(pts3, BAEMM_ERR_ARG, "null evaluation points");
    const int64_t tri_elems = mesh.nt * wave_count, pt_elems = npts * wave_count;
    if (profiling)
    {
        for (auto &e : prof_ev)
            if (!e) BAEMM_CUDA(cudaEventCreate(&e));
        BAEMM_CUDA(cudaEventRecord(prof_ev[0], stream));
    }
    auto mark = [&](int q) {
        if (profiling) BAEMM_CUDA(cudaEventRecord(prof_ev[q], stream));
    };
    const double2 al = make_double2((double)alpha.x, (double)alpha.y), be = make_double2((double)beta.x, (double)beta.y);
    if (apply_mode == BAEMM_APPLY_FP64)
    {
        double2 *Bt = Btri_d.reserve(tri_elems), *Cp = Cpts_d.reserve(pt_elems);
        double *p4 = pts_d.reserve(4 * npts);
        launch_avop<Text, double>(mesh, B, ldB, wave_count, Bt, stream);
        launch_pack_points<double>(npts, pts3, p4, stream);
        mark(1);
        launch_nearfield_dense<double>(mesh, nf, prm_d.p, wave_count, wave_chunk_size, p4, npts, Bt, Cp, stream);
        mark(2);
        launch_combine<Text, double>(npts, wave_count, al, Cp, be, C, ldC, stream);
    }
    else
    {
        float2 *Bt = Btri_f.reserve(tri_elems), *Cp = Cpts_f.reserve(pt_elems);
        float *p4 = pts_f.reserve(4 * npts);
        launch_avop<Text, float>(mesh, B, ldB, wave_count, Bt, stream);
        launch_pack_points<float>(npts, pts3, p4, stream);
        mark(1);
        if (apply_mode == BAEMM_APPLY_TC && tc_supported(wave_count, wave_chunk_size))
        {
            if (!tc_geo_ready)
            {
                launch_tc_tile_geometry(mesh, mesh.tgeo_f.reserve(tc_tile_geometry_floats(mesh.nt)), stream);
                tc_geo_ready = true;
            }
            const size_t ws_elems = tc_workspace_elems(tc_tune.ctas);
            launch_nearfield_tc(mesh, nf, prm16_f.p, tc_form, wave_count, wave_chunk_size, mesh.tgeo_f.p, p4, npts, Bt, Cp,
                                tc_ws.reserve(ws_elems), ws_elems, tc_img, tc_err.p, stream, tc_tune);
            tc_pending = true;
        }
        else
            launch_nearfield_dense<float>(mesh, nf, prm_f.p, wave_count, wave_chunk_size, p4, npts, Bt, Cp, stream,
                                          dense_variant);
        mark(2);
        launch_combine<Text, float>(npts, wave_count, al, Cp, be, C, ldC, stream);
    }
    mark(3);
    prof_valid = profiling;
}

template void Ctx::apply_nearfield<double2>(double2, const double2 *, int64_t, double2, double2 *, int64_t,
                                            const double *, int64_t);
template void Ctx::apply_nearfield<float2>(float2, const float2 *, int64_t, float2, float2 *, int64_t, const double *,
                                           int64_t);
template void Ctx::dense_apply<float>(const float2 *, float2 *, int64_t, int64_t);
template void Ctx::dense_apply<double>(const double2 *, double2 *, int64_t, int64_t);
template void Ctx::apply_boundary_rows<double2>(double2, const double2 *, int64_t, double2, double2 *, int64_t,
                                                int64_t, int64_t, bool);
template void Ctx::apply_boundary_rows<float2>(float2, const float2 *, int64_t, float2, float2 *, int64_t, int64_t,
                                               int64_t, bool);
template void Ctx::apply_boundary<double2>(double2, const double2 *, int64_t, double2, double2 *, int64_t);
template void Ctx::apply_boundary<float2>(float2, const float2 *, int64_t, float2, float2 *, int64_t);

void Ctx::apply_farfield(zc alpha, const double2 *B, int64_t ldB, zc beta, double2 *C, int64_t ldC)
{
    if (wave_chunk_count < 1) return;
    if (!(flags.sl() || flags.dl())) return;
    BAEMM_REQUIRE(mesh.nm > 0, BAEMM_ERR_SIZE, "no measurement directions");
    BAEMM_REQUIRE(ldB >= wave_count && ldC >= wave_count, BAEMM_ERR_ARG, "leading dimension smaller than wave_count");
    const int64_t tri_elems = mesh.nt * wave_count;
    const size_t pe = farfield_partial_elems(mesh, wave_count, wave_chunk_size);
    const double2 be = make_double2(beta.real(), beta.imag());
    if (aux_fp64())
    {
        double2 *Bt = Btri_d.reserve(tri_elems);
        launch_avop<double2, double>(mesh, B, ldB, wave_count, Bt, stream);
        launch_farfield<double>(mesh, flags, prm_d.p, wave_count, wave_chunk_size, Bt, ff_partial_d.reserve(pe), pe,
                                make_double2(alpha.real(), alpha.imag()), be, C, ldC, stream);
    }
    else
    {
        float2 *Bt = Btri_f.reserve(tri_elems);
        launch_avop<double2, float>(mesh, B, ldB, wave_count, Bt, stream);
        // combine_matrices takes alpha as the internal Complex (ApplyFarFieldOperators.hpp:405-409)
        const double2 al = make_double2((double)(float)alpha.real(), (double)(float)alpha.imag());
        launch_farfield<float>(mesh, flags, prm_f.p, wave_count, wave_chunk_size, Bt, ff_partial_f.reserve(pe), pe,
                               al, be, C, ldC, stream);
    }
}

void Ctx::incident(zc alpha, const double *dirs, zc beta, double2 *C, int64_t ldC, int type)
{
    if (wave_chunk_count < 1) return;
    if (!(flags.sl() || flags.dl())) return;
    BAEMM_REQUIRE(type == BAEMM_WAVE_PLANE || type == BAEMM_WAVE_RADIAL, BAEMM_ERR_ARG, "unknown wave type");
    const int wcs = wave_chunk_size;
    const int64_t tri_elems = mesh.nt * wave_count;
    EpilogueArgs ea;
    ea.layers = true;
    ea.wc = wave_count;
    ea.wcs = wcs;
    const double2 al = make_double2(alpha.real(), alpha.imag()), be = make_double2(beta.real(), beta.imag());
    if (aux_fp64())
    {
        BAEMM_CUDA(cudaMemcpyAsync(dirs_d.reserve(3 * wcs), dirs, 3 * wcs * sizeof(double), cudaMemcpyHostToDevice,
                                   stream));
        double2 *Ct = Ctri_d.reserve(tri_elems);
        launch_incident<double>(mesh, prm_d.p, wave_count, wcs, dirs_d.p, type, Ct, stream);
        launch_epilogue<double2, double>(mesh, ea, Ct, Ct, prm_d.p, nullptr, 0, al, be, C, ldC, stream);
    }
    else
    {
        std::vector<float> df(3 * wcs);
        for (int q = 0; q < 3 * wcs; ++q) df[q] = (float)dirs[q];
        BAEMM_CUDA(cudaMemcpyAsync(dirs_f.reserve(3 * wcs), df.data(), 3 * wcs * sizeof(float),
                                   cudaMemcpyHostToDevice, stream));
        float2 *Ct = Ctri_f.reserve(tri_elems);
        launch_incident<float>(mesh, prm_f.p, wave_count, wcs, dirs_f.p, type, Ct, stream);
        launch_epilogue<double2, float>(mesh, ea, Ct, Ct, prm_f.p, nullptr, 0, al, be, C, ldC, stream);
        sync();   // df is a host temporary
    }
}

void Ctx::herglotz(zc alpha, const double2 *g, int64_t ldg, zc beta, double2 *C, int64_t ldC)
{
    if (wave_chunk_count < 1) return;
    if (!(flags.sl() || flags.dl())) return;
    BAEMM_REQUIRE(mesh.nm > 0, BAEMM_ERR_SIZE, "no measurement directions");
    const int64_t tri_elems = mesh.nt * wave_count;
    EpilogueArgs ea;
    ea.layers = true;
    ea.wc = wave_count;
    ea.wcs = wave_chunk_size;
    const double2 al = make_double2(alpha.real(), alpha.imag()), be = make_double2(beta.real(), beta.imag());
    if (aux_fp64())
    {
        double2 *Ct = Ctri_d.reserve(tri_elems);
        launch_herglotz<double>(mesh, flags, prm_d.p, wave_count, wave_chunk_size, g, ldg, Ct, stream);
        launch_epilogue<double2, double>(mesh, ea, Ct, Ct, prm_d.p, nullptr, 0, al, be, C, ldC, stream);
    }
    else
    {
        float2 *Ct = Ctri_f.reserve(tri_elems);
        launch_herglotz<float>(mesh, flags, prm_f.p, wave_count, wave_chunk_size, g, ldg, Ct, stream);
        launch_epilogue<double2, float>(mesh, ea, Ct, Ct, prm_f.p, nullptr, 0, al, be, C, ldC, stream);
    }
}

bool Ctx::mass_inverse_real(const double *X, int64_t ldX, double *Y, int64_t ldY, int ncols, double tol)
{
    int it = 0;
    // ApplyMassInverse.hpp:48: max_iter = 20
    const bool v64 = mass_values_fp64();
    bool ok;
    if (use_graphs)
    {
        long long tb = 0;
        std::memcpy(&tb, &tol, sizeof(tb));
        run_graphed(GraphKey{2, X, Y, ldX, ldY, 2LL * ncols + (v64 ? 1 : 0), tb},
                    [&] { cg.enqueue_mass(mesh, v64, X, ldX, Y, ldY, ncols, tol, 20, stream); });
        ok = cg.finish(stream, &it);
    }
    else
        ok = cg.solve_mass(mesh, v64, X, ldX, Y, ldY, ncols, tol, 20, stream, &it);
    stats.cg_iterations = std::max(stats.cg_iterations, it);
    stats.cg_converged = stats.cg_converged && ok;
    return ok;
}

bool Ctx::mass_inverse_complex(const double2 *X, int64_t ldX, double2 *Y, int64_t ldY, int ncols, double tol)
{
    // complex columns as interleaved real columns (ApplyMassInverse.hpp:71-98)
    return mass_inverse_real(reinterpret_cast<const double *>(X), 2 * ldX, reinterpret_cast<double *>(Y), 2 * ldY,
                             2 * ncols, tol);
}

std::string Ctx::device_info() const
{
    cudaDeviceProp p;
    std::ostringstream s;
    if (cudaGetDeviceProperties(&p, device) != cudaSuccess)
    {
        (void)cudaGetLastError();
        return "Helmholtz_CUDA::DeviceInfo: unavailable";
    }
    int rt = 0, drv = 0;
    cudaRuntimeGetVersion(&rt);
    cudaDriverGetVersion(&drv);
    s << "Helmholtz_CUDA::DeviceInfo\n"
      << "DEVICE_NAME                        = " << p.name << "\n"
      << "DEVICE_INDEX                       = " << device << "\n"
      << "COMPUTE_CAPABILITY                 = " << p.major << "." << p.minor << "\n"
      << "MULTIPROCESSOR_COUNT               = " << p.multiProcessorCount << "\n"
      << "GLOBAL_MEM_SIZE                    = " << p.totalGlobalMem << "\n"
      << "SHARED_MEM_PER_BLOCK_OPTIN         = " << p.sharedMemPerBlockOptin << "\n"
      << "L2_CACHE_SIZE                      = " << p.l2CacheSize << "\n"
      << "RUNTIME_VERSION                    = " << rt << "\n"
      << "DRIVER_VERSION                     = " << drv << "\n";
    return s.str();
}

} // namespace baemm
