// Autotuner of the dense boundary kernel (baemm_autotune in include/baemm.h).
//
// The kernel shapes that matter depend on the mesh size and the wave block:
// the plain FP32 form has three variants (scalar FMA with 16 columns per
// thread, packed FP32x2 with one or two targets per thread); the tensor-core
// form has its generator-warp count (8 or 16), the 16-column groups per work
// unit (1, 2 or 4: fewer give small meshes more units to spread over the SMs
// at the cost of re-evaluating the pair geometry per group) and the length of
// its TMEM accumulation segment.  The tuner runs each candidate on the loaded
// operators with the context's mesh and wave counts (a constant
// right-hand-side block; the kernels' cost does not depend on the values),
// times it with CUDA events on the context's stream and keeps the fastest.
// The tensor-core search is two-staged: warps x chunks at the default
// segment, then the segment lengths around the winner.
//
// Choices are cached for the process per (device, mesh size, wave shape,
// arithmetic form, operator structure): a second context with the same key,
// or the same context after a re-mesh of equal size, takes the cached choice
// without timing anything.  One context at a time times a key; a concurrent
// caller with the same key waits and takes that choice, so every context of
// the process runs a key with the same settings.
#include <algorithm>
#include <condition_variable>
#include <map>
#include <mutex>
#include <set>
#include <tuple>
#include <vector>

#include "ctx.cuh"

namespace baemm
{
namespace
{

using TuneKey = std::tuple<int, int64_t, int64_t, int, int, int, int, int>;

struct TuneChoice
{
    int dense_variant = 0;
    TcTuning tc;
    double best_ms = 0.0;
    int candidates = 0;
};

std::mutex g_tune_mutex;
std::condition_variable g_tune_cv;
std::map<TuneKey, TuneChoice> g_tune_cache;
std::set<TuneKey> g_tuning;   // keys being timed now: a second caller waits for the first one's choice

} // namespace

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
    *out = baemm_tune_result{};
    out->apply_mode = mode;

    const int code = (flags.sl() ? 1 : 0) | (flags.dl() ? 2 : 0) | (flags.adl() ? 4 : 0);
    const bool ri = !flags.re_sl && !flags.im_dl && !flags.im_adl && (flags.dl() || flags.adl());
    const int form = (ri ? 1 : 0) | (tc_form.ki ? 2 : 0) | (tc_entry_sharing(flags, tc_form, wave_count, TcTuning{}) << 2) |
                     (tc_tune.share << 5);
    const TuneKey key{device, mesh.nt, mesh.nv, wave_count, wave_chunk_size, mode, code, form};
    auto report = [&](const TuneChoice &ch, double before, int cached) {
        out->dense_variant = dense_variant;
        out->tc_segment = tc_tune.seg_tiles;
        out->tc_ctas = tc_tune.ctas;
        out->tc_stagger = tc_tune.stagger;
        out->candidates = ch.candidates;
        out->best_ms = ch.best_ms;
        out->before_ms = before;
        out->tc_gen_warps = tc_tune.gen_warps;
        out->tc_chunks = tc_chunks_per_unit(wave_count, tc_tune.chunks);
        out->cached = cached;
    };
    {
        std::unique_lock<std::mutex> lock(g_tune_mutex);
        g_tune_cv.wait(lock, [&] { return g_tuning.count(key) == 0; });
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end())
        {
            ++graph_state;
            if (mode == BAEMM_APPLY_TC) tc_tune = it->second.tc;   // the key holds the share setting
            else dense_variant = it->second.dense_variant;
            report(it->second, -1.0, 1);
            return;
        }
        g_tuning.insert(key);   // one context times a key; the others take its choice
    }
    auto release = [&](const TuneChoice *ch) {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        if (ch) g_tune_cache[key] = *ch;
        g_tuning.erase(key);
        g_tune_cv.notify_all();
    };

    // from here on every exit releases the key (the set-up below can throw too)
    float2 *Bt = nullptr, *Ct = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    try
    {
        const size_t elems = (size_t)mesh.nt * (size_t)wave_count;
        Bt = Btri_f.reserve(elems);
        Ct = Ctri_f.reserve(elems);
        BAEMM_CUDA(cudaMemsetAsync(Bt, 0x3c, elems * sizeof(float2), stream));   // every float 0.0115
        BAEMM_CUDA(cudaEventCreate(&e0));
        BAEMM_CUDA(cudaEventCreate(&e1));
    }
    catch (...)
    {
        if (e0) cudaEventDestroy(e0);
        release(nullptr);
        throw;
    }
    const int saved_mode = apply_mode, saved_variant = dense_variant;
    const TcTuning saved_tc = tc_tune;
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
    TuneChoice choice;
    try
    {
        apply_mode = mode;
        const double before = time_current();
        choice.best_ms = 1e300;
        auto consider = [&](double ms) {
            ++choice.candidates;
            if (ms < choice.best_ms)
            {
                choice.best_ms = ms;
                choice.tc = tc_tune;
                choice.dense_variant = dense_variant;
            }
        };
        if (mode == BAEMM_APPLY_TC)
        {
            const int most = tc_chunks_per_unit(wave_count, 0);
            std::vector<int> chunk_opts;
            for (int ch = most; ch >= 1; ch /= 2) chunk_opts.push_back(ch);
            for (int gw : {16, 8})
                for (int ch : chunk_opts)
                {
                    tc_tune = saved_tc;
                    tc_tune.gen_warps = gw;
                    tc_tune.chunks = ch;
                    tc_tune.seg_tiles = 16;
                    consider(time_current());
                }
            const TcTuning stage1 = choice.tc;
            for (int seg : {8, 32})
            {
                tc_tune = stage1;
                tc_tune.seg_tiles = seg;
                consider(time_current());
            }
            tc_tune = choice.tc;
            dense_variant = saved_variant;
        }
        else
        {
            for (int v = 0; v < kDenseVariants; ++v)
            {
                dense_variant = v;
                consider(time_current());
            }
            dense_variant = choice.dense_variant;
            tc_tune = saved_tc;
        }
        apply_mode = saved_mode;
        ++graph_state;
        report(choice, before, 0);
    }
    catch (...)
    {
        apply_mode = saved_mode;
        dense_variant = saved_variant;
        tc_tune = saved_tc;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        release(nullptr);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    release(&choice);
}

void autotune_forget()
{
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache.clear();
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
    catch (const std::bad_alloc &)
    {
        c.last_error = "host allocation failed";
        return BAEMM_ERR_ALLOC;
    }
    catch (const std::exception &e)
    {
        c.last_error = e.what();
        return BAEMM_ERR_ARG;
    }
}

extern "C" void baemm_autotune_forget(void) { baemm::autotune_forget(); }
