// An allocation-free variant of the device-pointer boundary-operator apply
// (baemm_apply_boundary_operators_noalloc_dev_c in include/baemm.h).
//
// Who needs it: callers that cannot call cudaMalloc while they run -- host
// frameworks that own all device memory through their own pool or a fixed
// budget and forbid allocations behind their back, long-running servers that
// must not grow their device footprint after start-up, and latency-critical
// loops for which cudaMalloc's and cudaFree's implicit device synchronisation
// is unacceptable.  The regular apply keeps its triangle-level intermediate
// blocks (B_tri = AvOp B and C_tri = K B_tri, 2 * simplex_count * wave_count
// complex64) in grow-only cudaMalloc'ed buffers of the context; this variant
// places them in one file-scope __device__ array of fixed size instead, so the
// call itself allocates nothing and frees nothing.
//
// Costs and rules:
//   * The array (kNoAllocScratchBytes = 32 MiB) is reserved on every GPU that
//     loads this library, for the life of the process.
//   * Problems larger than the array are rejected with BAEMM_ERR_SIZE:
//     2 * simplex_count * wave_count * 8 bytes must fit in 32 MiB.
//   * The device address of the array is looked up (cudaGetSymbolAddress) the
//     first time the entry point runs on a device, with that device current;
//     make that first call before any stream capture begins.  The address is
//     cached per device ordinal for the life of the process, so
//     cudaDeviceReset is not supported while the library is loaded.
//   * All calls share the one array and it keeps the last call's contents.
//     Both halves are fully overwritten by every call before they are read, so
//     nothing needs clearing; but calls whose work overlaps on the GPU (two
//     streams, two contexts on one device) race on the array and must be
//     serialised by the caller.
//   * Only the plain FP32 apply mode is offered; the operators must have been
//     loaded with baemm_load_boundary_operators beforehand.  The call records
//     no phase timings (baemm_last_apply_times reports none after it).
#include <mutex>
#include <new>

#include "ctx.cuh"

namespace baemm
{
namespace
{

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
constexpr size_t kNoAllocElems = kNoAllocScratchBytes / sizeof(float2);
constexpr int kMaxDevices = 64;

static __device__ __align__(256) float2 g_noalloc_scratch[kNoAllocElems];

std::mutex g_scratch_mutex;
float2 *g_scratch_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on `device` (which must be current);
// looked up once per device.  The host-side symbol itself is only a handle.
float2 *scratch_for(int device)
{
    BAEMM_REQUIRE(device >= 0 && device < kMaxDevices, BAEMM_ERR_ARG, "device index out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[device])
    {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr)
        {
            (void)cudaGetLastError();
            throw Error(BAEMM_ERR_CUDA, std::string("cudaGetSymbolAddress of the no-alloc scratch failed: ") +
                                            cudaGetErrorString(e));
        }
        g_scratch_ptr[device] = static_cast<float2 *>(p);
    }
    return g_scratch_ptr[device];
}

} // namespace
} // namespace baemm

extern "C" int baemm_apply_boundary_operators_noalloc_dev_c(baemm_ctx *ctx, const float alpha[2], const float *B_in,
                                                            int64_t ldB, const float beta[2], float *C_out,
                                                            int64_t ldC)
{
    using namespace baemm;
    if (!ctx || !ctx->impl) return BAEMM_ERR_ARG;
    Ctx &c = *ctx->impl;
    c.prof_valid = false;   // no phase timings for this call
    try
    {
        c.require_loaded();
        BAEMM_REQUIRE(B_in && C_out, BAEMM_ERR_ARG, "null block");
        BAEMM_REQUIRE(c.apply_mode == BAEMM_APPLY_FP32, BAEMM_ERR_ARG,
                      "the no-alloc apply runs the plain FP32 apply mode only");
        const int wc = c.wave_count;
        BAEMM_REQUIRE(ldB >= wc && ldC >= wc, BAEMM_ERR_ARG, "leading dimension smaller than wave_count");
        const size_t tri_elems = (size_t)c.mesh.nt * (size_t)wc;
        BAEMM_REQUIRE(2 * tri_elems <= kNoAllocElems, BAEMM_ERR_SIZE,
                      "problem too large for the no-alloc scratch: 2 * simplex_count * wave_count * 8 bytes = " +
                          std::to_string(2 * tri_elems * sizeof(float2)) + " > " +
                          std::to_string(kNoAllocScratchBytes) + " bytes (use the allocating apply)");
        DeviceScope scope(c.device);   // restores the caller's device on return
        float2 *Bt = scratch_for(c.device);
        float2 *Ct = Bt + tri_elems;
        const bool layers = c.flags.any_layer();
        if (layers || c.flags.mass())
        {
            EpilogueArgs ea;
            ea.layers = layers;
            ea.sl_diag = layers && c.use_diagonal && c.flags.sl();
            ea.mass = c.flags.mass();
            ea.wc = wc;
            ea.wcs = c.wave_chunk_size;
            const float2 *B = reinterpret_cast<const float2 *>(B_in);
            float2 *C = reinterpret_cast<float2 *>(C_out);
            const float2 al = make_float2(alpha ? alpha[0] : 0.f, alpha ? alpha[1] : 0.f);
            const float2 be = make_float2(beta ? beta[0] : 0.f, beta ? beta[1] : 0.f);
            if (layers)
            {
                launch_avop<float2, float>(c.mesh, B, ldB, wc, Bt, c.stream);
                launch_boundary_dense<float>(c.mesh, c.flags, c.prm_f.p, wc, c.wave_chunk_size, Bt, Ct, c.stream,
                                             c.dense_variant);
            }
            launch_epilogue<float2, float>(c.mesh, ea, Ct, Bt, c.prm_f.p, B, ldB, al, be, C, ldC, c.stream);
        }
        c.last_error.clear();
        return BAEMM_OK;
    }
    catch (const Error &e)
    {
        c.last_error = e.what();
        return e.code;
    }
    catch (const std::bad_alloc &)
    {
        c.last_error = "host allocation failed";
        return BAEMM_ERR_ALLOC;
    }
    catch (const std::exception &e)   // e.g. std::system_error from the mutex
    {
        c.last_error = e.what();
        return BAEMM_ERR_ARG;
    }
}
