// Autotuner of the dense boundary kernel (baemm_autotune in include/baemm.h).
//
// The kernel shapes that matter depend on the mesh size and the wave block:
// the plain FP32 form has three variants (scalar FMA with 16 columns per
// thread, packed FP32x2 with one or two targets per thread), the tensor-core
// form the length of its TMEM accumulation segment.  The tuner runs each
// candidate on the loaded operators with the context's mesh and wave counts
// (a constant right-hand-side block; the kernels' cost does not depend on the
// values), times it with CUDA events on the context's stream, keeps the
// fastest and reports it.
#include <algorithm>
#include <vector>

#include "ctx.cuh"

namespace baemm
{

void Ctx::autotune(int mode, int repeats, baemm_tune_result *out)
{
    require_loaded();
    BAEMM_REQUIRE(out, BAEMM_ERR_ARG, "null result");
    BAEMM_REQUIRE(mode == BAEMM_APPLY_FP32 || mode == BAEMM_APPLY_TC, BAEMM_ERR_ARG,
                  "autotune: mode must be BAEMM_APPLY_FP32 or BAEMM_APPLY_TC");
    BAEMM_REQUIRE(flags.any_layer(), BAEMM_ERR_ARG, "autotune: the loaded operators have no layer term");
    repeats = std::max(1, repeats);
    BAEMM_CUDA(cudaSetDevice(device));
    if (mode == BAEMM_APPLY_TC && !tc_supported(wave_count, wave_chunk_size)) mode = BAEMM_APPLY_FP32;

    const size_t elems = (size_t)mesh.nt * (size_t)wave_count;
    float2 *Bt = Btri_f.reserve(elems), *Ct = Ctri_f.reserve(elems);
    BAEMM_CUDA(cudaMemsetAsync(Bt, 0x3c, elems * sizeof(float2), stream));   // every float 0.0115

    cudaEvent_t e0 = nullptr, e1 = nullptr;
    BAEMM_CUDA(cudaEventCreate(&e0));
    BAEMM_CUDA(cudaEventCreate(&e1));
    const int saved_mode = apply_mode, saved_variant = dense_variant, saved_seg = tc_seg_tiles;
    auto time_current = [&]() {
        dense_apply<float>(Bt, Ct);   // warm-up (and first-use set-up)
        float best = 1e30f;
        for (int r = 0; r < repeats; ++r)
        {
            BAEMM_CUDA(cudaEventRecord(e0, stream));
            dense_apply<float>(Bt, Ct);
            BAEMM_CUDA(cudaEventRecord(e1, stream));
            BAEMM_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            BAEMM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            best = std::min(best, ms);
        }
        if (tc_pending) check_tc_error();
        return (double)best;
    };
    try
    {
        apply_mode = mode;
        const double before = time_current();
        std::vector<int> cands;
        if (mode == BAEMM_APPLY_TC)
            cands = {4, 8, 16, 32};
        else
            for (int v = 0; v < kDenseVariants; ++v) cands.push_back(v);
        double best = 1e300;
        int best_c = mode == BAEMM_APPLY_TC ? saved_seg : saved_variant;
        for (int c : cands)
        {
            if (mode == BAEMM_APPLY_TC) tc_seg_tiles = c;
            else dense_variant = c;
            const double ms = time_current();
            if (ms < best)
            {
                best = ms;
                best_c = c;
            }
        }
        if (mode == BAEMM_APPLY_TC)
        {
            tc_seg_tiles = best_c;
            dense_variant = saved_variant;
        }
        else
        {
            dense_variant = best_c;
            tc_seg_tiles = saved_seg;
        }
        apply_mode = saved_mode;
        out->apply_mode = mode;
        out->dense_variant = dense_variant;
        out->tc_segment = tc_seg_tiles;
        out->tc_ctas = tc_ctas;
        out->tc_stagger = tc_stagger;
        out->candidates = (int32_t)cands.size();
        out->best_ms = best;
        out->before_ms = before;
    }
    catch (...)
    {
        apply_mode = saved_mode;
        dense_variant = saved_variant;
        tc_seg_tiles = saved_seg;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

} // namespace baemm

extern "C" int baemm_autotune(baemm_ctx *ctx, int mode, int repeats, baemm_tune_result *out)
{
    if (!ctx || !ctx->impl) return BAEMM_ERR_ARG;
    baemm::Ctx &c = *ctx->impl;
    try
    {
        c.autotune(mode, repeats, out);
        c.last_error.clear();
        return BAEMM_OK;
    }
    catch (const baemm::Error &e)
    {
        c.last_error = e.what();
        return e.code;
    }
}
