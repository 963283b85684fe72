// guiding_api.cu -- C-ABI entry points of the path-guiding model (include/spt.h).
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "guiding_host.h"
#include "wavefront.h"

using namespace spt;
using namespace spt::guide;

namespace {

spt_status upload_records(spt_context* ctx, const spt_guide_record* recs, uint32_t n, float4** out) {
    void* d;
    spt_status st = scratch(ctx, 3, static_cast<size_t>(n) * sizeof(spt_guide_record), &d);
    if (st != SPT_OK) return st;
    SPT_CUDA(ctx, cudaMemcpyAsync(d, recs, static_cast<size_t>(n) * sizeof(spt_guide_record), cudaMemcpyHostToDevice,
                                  ctx->stream));
    *out = static_cast<float4*>(d);
    return SPT_OK;
}

}  // namespace

extern "C" {

spt_status spt_guide_create(spt_context* ctx, const spt_guide_config* cfg, spt_guide** out) {
    if (!ctx || !cfg || !out) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    if (!(cfg->lr > 0.0f) || cfg->batch == 0 || !(cfg->mix >= 0.0f && cfg->mix <= 1.0f))
        return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "guide config: lr > 0, batch > 0, mix in [0, 1]");
    if ((cfg->cache_res != 0 && (cfg->cache_res < 4 || cfg->cache_res > 128)) ||
        (cfg->train_path != SPT_GUIDE_TRAIN_TCGEN05 && cfg->train_path != SPT_GUIDE_TRAIN_MMA_SYNC) ||
        cfg->reserved != 0)
        return fail(ctx, SPT_ERR_INVALID_ARGUMENT,
                    "guide config: cache_res 0 or 4..128, train_path 0 or 1, reserved 0");
    SPT_CUDA(ctx, cudaSetDevice(ctx->device));
    auto g = std::unique_ptr<spt_guide>(new (std::nothrow) spt_guide());
    if (!g) return SPT_ERR_OUT_OF_MEMORY;
    spt_status st = g->g.alloc(ctx, *cfg);
    if (st != SPT_OK) return st;
    SPT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *out = g.release();
    return SPT_OK;
}

spt_status spt_guide_destroy(spt_guide* guide) {
    if (!guide) return SPT_ERR_INVALID_ARGUMENT;
    cudaSetDevice(guide->g.ctx->device);
    cudaStreamSynchronize(guide->g.ctx->stream);
    delete guide;
    return SPT_OK;
}

spt_status spt_guide_get_params(spt_guide* guide, float* grid, float* mlp) {
    if (!guide) return SPT_ERR_INVALID_ARGUMENT;
    Guide& G = guide->g;
    spt_context* ctx = G.ctx;
    SPT_CUDA(ctx, cudaSetDevice(ctx->device));
    if (grid) SPT_CUDA(ctx, cudaMemcpyAsync(grid, G.grid_master, kGridParams * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (mlp) SPT_CUDA(ctx, cudaMemcpyAsync(mlp, G.mlp_master, kMlpParams * 4, cudaMemcpyDeviceToHost, ctx->stream));
    SPT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return SPT_OK;
}

spt_status spt_guide_set_params(spt_guide* guide, const float* grid, const float* mlp) {
    if (!guide) return SPT_ERR_INVALID_ARGUMENT;
    Guide& G = guide->g;
    spt_context* ctx = G.ctx;
    SPT_CUDA(ctx, cudaSetDevice(ctx->device));
    if (grid) SPT_CUDA(ctx, cudaMemcpyAsync(G.grid_master, grid, kGridParams * 4, cudaMemcpyHostToDevice, ctx->stream));
    if (mlp) SPT_CUDA(ctx, cudaMemcpyAsync(G.mlp_master, mlp, kMlpParams * 4, cudaMemcpyHostToDevice, ctx->stream));
    spt_status st = G.refresh();
    if (st != SPT_OK) return st;
    SPT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return SPT_OK;
}

spt_status spt_guide_eval(spt_context* ctx, spt_guide* guide, const float* in, uint32_t n, float* out) {
    if (!ctx || !guide || (n && (!in || !out))) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n == 0) return SPT_OK;
    SPT_CUDA(ctx, cudaSetDevice(ctx->device));
    void *d_in, *d_out;
    spt_status st;
    if ((st = scratch(ctx, 0, static_cast<size_t>(n) * 48, &d_in)) != SPT_OK) return st;
    if ((st = scratch(ctx, 1, static_cast<size_t>(n) * kOutUsed * 4, &d_out)) != SPT_OK) return st;
    SPT_CUDA(ctx, cudaMemcpyAsync(d_in, in, static_cast<size_t>(n) * 48, cudaMemcpyHostToDevice, ctx->stream));
    if ((st = guide->g.infer(static_cast<float4*>(d_in), n, static_cast<float*>(d_out), ctx->stream)) != SPT_OK)
        return st;
    SPT_CUDA(ctx, cudaMemcpyAsync(out, d_out, static_cast<size_t>(n) * kOutUsed * 4, cudaMemcpyDeviceToHost, ctx->stream));
    return check_status(ctx);
}

spt_status spt_guide_gradients(spt_context* ctx, spt_guide* guide, const spt_guide_record* recs, uint32_t n,
                               float* grid_grad, float* mlp_grad, float* loss) {
    if (!ctx || !guide || !recs || n == 0) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    SPT_CUDA(ctx, cudaSetDevice(ctx->device));
    Guide& G = guide->g;
    float4* d;
    spt_status st = upload_records(ctx, recs, n, &d);
    if (st != SPT_OK) return st;
    SPT_CUDA(ctx, cudaMemsetAsync(G.grid_grad, 0, kGridParams * 4, ctx->stream));
    if ((st = G.gradients(d, n)) != SPT_OK) return st;
    if (grid_grad) SPT_CUDA(ctx, cudaMemcpyAsync(grid_grad, G.grid_grad, kGridParams * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (mlp_grad) SPT_CUDA(ctx, cudaMemcpyAsync(mlp_grad, G.mlp_grad, kMlpParams * 4, cudaMemcpyDeviceToHost, ctx->stream));
    float h[2];
    SPT_CUDA(ctx, cudaMemcpyAsync(h, G.scalars, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    st = check_status(ctx);
    if (st != SPT_OK) return st;
    SPT_CUDA(ctx, cudaMemsetAsync(G.grid_grad, 0, kGridParams * 4, ctx->stream));
    if (loss) *loss = h[1] / static_cast<float>(n);
    return SPT_OK;
}

spt_status spt_guide_train(spt_context* ctx, spt_guide* guide, const spt_guide_record* recs, uint32_t n, float* loss) {
    if (!ctx || !guide || !recs || n == 0) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    SPT_CUDA(ctx, cudaSetDevice(ctx->device));
    float4* d;
    spt_status st = upload_records(ctx, recs, n, &d);
    if (st != SPT_OK) return st;
    if ((st = guide->g.step(d, n, loss)) != SPT_OK) return st;
    return check_status(ctx);
}

spt_status spt_guide_train_device(spt_context* ctx, spt_guide* guide, const spt_guide_record* d_recs, uint32_t n,
                                  float* gpu_ms) {
    if (!ctx || !guide || !d_recs || n == 0) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    if (guide->g.ctx != ctx) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "the guide belongs to another context");
    SPT_CUDA(ctx, cudaSetDevice(ctx->device));
    SPT_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    spt_status st = guide->g.step(reinterpret_cast<const float4*>(d_recs), n, nullptr);
    if (st != SPT_OK) return st;
    SPT_CUDA(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    if ((st = check_status(ctx)) != SPT_OK) return st;   // synchronises the stream
    if (gpu_ms) SPT_CUDA(ctx, cudaEventElapsedTime(gpu_ms, ctx->ev0, ctx->ev1));
    return SPT_OK;
}

spt_status spt_guide_steps(spt_guide* guide, uint64_t* steps) {
    if (!guide || !steps) return SPT_ERR_INVALID_ARGUMENT;
    *steps = guide->g.steps;
    return SPT_OK;
}

spt_status spt_guided_pathtrace_device(spt_context* ctx, const spt_scene* sc, const spt_camera* cam,
                                       const spt_pt_params* p, spt_guide* guide, float* d_out_rgb,
                                       spt_render_stats* stats) {
    if (!ctx || !guide) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    if (guide->g.ctx != ctx) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "the guide belongs to another context");
    std::vector<PtJob> jobs(1);
    spt_status st = make_job(ctx, sc, cam, p, d_out_rgb, jobs[0]);
    if (st != SPT_OK) return st;
    // Progressive passes: the first passes are small so the guide learns from early paths and the
    // later, larger passes sample a trained guide; once the step budget is spent the rest of the
    // samples go in one pass with the guide frozen.  Every pass is unbiased, so the image (the
    // mean of all samples) is too.
    const PtJob whole = jobs[0];
    const uint32_t spp = whole.spp, npix = std::max(1u, whole.npix);
    // Training is paid for out of the render's own time, so its step budget grows with the render:
    // one optimiser step per 5 batches' worth of camera paths (about a fifth of a plain render's
    // time at 2^18 records per step), at least one and at most max_steps.  On the 64-scene batch set
    // this measured 1.70 / 3.17 (raw / debiased equal-time ratio) against 1.67 / 2.90 for one step
    // per 10 batches.
    const uint64_t per_step = 5ull * std::max(1u, guide->g.cfg.batch);
    const uint32_t budget = static_cast<uint32_t>(
        std::min<uint64_t>(guide->g.cfg.max_steps, std::max<uint64_t>(1, whole.total / per_step)));
    uint32_t pass = std::max(1u, (guide->g.cfg.batch + npix - 1) / npix);
    uint64_t segs = 0, paths = 0;
    double ms = 0.0;
    uint32_t trained = 0;
    for (uint32_t s0 = 0; s0 < spp;) {
        const bool learning = trained < budget;
        const uint32_t s1 = learning ? std::min<uint64_t>(spp, static_cast<uint64_t>(s0) + pass) : spp;
        jobs[0] = whole;
        set_sample_range(jobs[0], s0, s1);
        uint64_t pass_segs = 0;
        float pass_ms = 0.0f;
        uint32_t pass_steps = 0;
        st = render_jobs(ctx, jobs, default_tune(), &pass_segs, &pass_ms, &guide->g, budget - trained, &pass_steps);
        if (st != SPT_OK) return st;
        segs += pass_segs;
        ms += pass_ms;
        paths += jobs[0].total;
        trained += pass_steps;
        s0 = s1;
        if (pass < (1u << 30)) pass *= 2;
    }
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->paths = paths;
        stats->segments = segs;
        stats->gpu_ms = ms;
    }
    return SPT_OK;
}

}  // extern "C"
