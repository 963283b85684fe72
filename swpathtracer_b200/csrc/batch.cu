// batch.cu -- batched rendering of many scenes in one wavefront, and the autotuner that picks the
// wavefront's pool size, kernel shapes and traversal for a batch.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "wavefront.h"

using namespace spt;

namespace {

spt_status build_jobs(spt_context* ctx, const spt_batch_job* jobs, uint32_t n, float* const* d_images,
                      std::vector<PtJob>& out) {
    if (!jobs || n == 0 || !d_images) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "empty batch");
    out.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        spt_status st = make_job(ctx, jobs[i].scene, &jobs[i].camera, &jobs[i].params, d_images[i], out[i]);
        if (st != SPT_OK) return fail(ctx, st, "job " + std::to_string(i) + ": " + ctx->err);
    }
    return SPT_OK;
}

// Key of the tuning cache: the device and the batch's shape (primitive counts, image sizes, spp).
std::string tune_key(spt_context* ctx, const spt_batch_job* jobs, uint32_t n) {
    cudaDeviceProp prop;
    std::memset(&prop, 0, sizeof(prop));
    cudaGetDeviceProperties(&prop, ctx->device);
    uint64_t h = 1469598103934665603ull;  // FNV-1a over the shape
    auto mix = [&h](uint64_t v) {
        for (int k = 0; k < 8; ++k) {
            h ^= (v >> (8 * k)) & 0xFFu;
            h *= 1099511628211ull;
        }
    };
    mix(n);
    for (uint32_t i = 0; i < n; ++i) {
        mix(jobs[i].scene ? jobs[i].scene->dev.n_prims : 0);
        mix(jobs[i].camera.vp_width);
        mix(jobs[i].camera.vp_height);
        mix(jobs[i].params.spp);
        mix(jobs[i].params.termination);
    }
    std::string name(prop.name);
    std::replace(name.begin(), name.end(), ' ', '_');
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%016llx", static_cast<unsigned long long>(h));
    return "v2:" + name + ":" + buf;   // v2: entries carry the stack depth
}

bool cache_lookup(const char* path, const std::string& key, spt_tune& t) {
    if (!path) return false;
    std::ifstream f(path);
    std::string line;
    bool found = false;
    while (std::getline(f, line)) {
        std::istringstream is(line);
        std::string k;
        spt_tune c = default_tune();
        double ms;
        if (is >> k >> c.capacity >> c.extend_block >> c.shade_block >> c.traversal >> c.check_every >> c.sort_shading >>
                c.stack >> ms &&
            k == key) {
            t = c;
            found = true;  // the last entry for a key wins
        }
    }
    return found;
}

void cache_store(const char* path, const std::string& key, const spt_tune& t, double ms) {
    if (!path) return;
    std::ofstream f(path, std::ios::app);
    f << key << " " << t.capacity << " " << t.extend_block << " " << t.shade_block << " " << t.traversal << " "
      << t.check_every << " " << t.sort_shading << " " << t.stack << " " << ms << "\n";
}

}  // namespace

extern "C" {

spt_status spt_tune_default(spt_tune* out) {
    if (!out) return SPT_ERR_INVALID_ARGUMENT;
    *out = default_tune();
    return SPT_OK;
}

spt_status spt_batch_pathtrace(spt_context* ctx, const spt_batch_job* jobs, uint32_t n_jobs, float* const* d_images,
                               const spt_tune* tune, spt_render_stats* stats) {
    if (!ctx) return SPT_ERR_INVALID_ARGUMENT;
    std::vector<PtJob> pj;
    spt_status st = build_jobs(ctx, jobs, n_jobs, d_images, pj);
    if (st != SPT_OK) return st;
    uint64_t segs = 0;
    float ms = 0.0f;
    st = render_jobs(ctx, pj, tune ? *tune : default_tune(), &segs, &ms);
    if (st != SPT_OK) return st;
    if (stats)
        for (uint32_t i = 0; i < n_jobs; ++i) {
            std::memset(&stats[i], 0, sizeof(spt_render_stats));
            stats[i].paths = pj[i].total;
            stats[i].segments = segs;
            stats[i].gpu_ms = ms;
        }
    return SPT_OK;
}

// Coordinate descent over the wavefront settings (traversal, pool capacity, shade block, traversal
// stack depth, grouped shading), each trial a render of the whole batch at 4 samples per pixel into
// scratch images (the caller's images are not touched).
spt_status spt_autotune(spt_context* ctx, const spt_batch_job* jobs, uint32_t n_jobs, const char* cache_path,
                        spt_tune* out) {
    if (!ctx || !jobs || !out || n_jobs == 0) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    const std::string key = tune_key(ctx, jobs, n_jobs);
    spt_tune best = default_tune();
    if (cache_lookup(cache_path, key, best)) {
        *out = best;
        return SPT_OK;
    }
    SPT_CUDA(ctx, cudaSetDevice(ctx->device));
    // scratch images for the trials
    size_t total_px = 0;
    for (uint32_t i = 0; i < n_jobs; ++i) total_px += 3ull * jobs[i].camera.width * jobs[i].camera.height;
    void* mem;
    spt_status st = scratch(ctx, 7, total_px * sizeof(float), &mem);
    if (st != SPT_OK) return st;
    std::vector<float*> imgs(n_jobs);
    size_t off = 0;
    std::vector<spt_batch_job> trial(jobs, jobs + n_jobs);
    for (uint32_t i = 0; i < n_jobs; ++i) {
        imgs[i] = static_cast<float*>(mem) + off;
        off += 3ull * jobs[i].camera.width * jobs[i].camera.height;
        trial[i].params.spp = std::min<uint32_t>(trial[i].params.spp, 4);
    }
    std::vector<PtJob> pj;
    if ((st = build_jobs(ctx, trial.data(), n_jobs, imgs.data(), pj)) != SPT_OK) return st;
    auto time_of = [&](const spt_tune& t, double& ms_out) -> spt_status {
        uint64_t segs = 0;
        float ms = 0.0f;
        std::vector<PtJob> copy = pj;
        spt_status s = render_jobs(ctx, copy, t, &segs, &ms);
        ms_out = ms;
        return s;
    };
    double best_ms = 0.0;
    // warm-up (first-launch costs) and the baseline
    if ((st = time_of(best, best_ms)) != SPT_OK) return st;
    if ((st = time_of(best, best_ms)) != SPT_OK) return st;
    const int32_t travs[] = {2, 1, 0};
    const uint32_t caps[] = {1u << 20, 1u << 21, 1u << 22};
    const uint32_t shades[] = {64, 128, 256};
    // stack depths that hold every scene's 8-wide tree (a shallower stack could overflow)
    uint32_t bound = 0;
    for (uint32_t i = 0; i < n_jobs; ++i) bound = std::max(bound, jobs[i].scene ? jobs[i].scene->wide_stack_bound : 0u);
    const uint32_t stacks[] = {16, 24, 32};
    for (int dim = 0; dim < 5; ++dim) {
        const int n_opt = dim == 4 ? 2 : 3;
        spt_tune round_best = best;
        for (int k = 0; k < n_opt; ++k) {
            spt_tune c = best;
            if (dim == 0) c.traversal = travs[k];
            if (dim == 1) c.capacity = caps[k];
            if (dim == 2) c.shade_block = shades[k];
            if (dim == 3) {
                if (stacks[k] < bound) continue;
                c.stack = stacks[k];
            }
            if (dim == 4) c.sort_shading = static_cast<uint32_t>(k + 1);   // always / never
            if (std::memcmp(&c, &best, sizeof(c)) == 0) continue;
            double ms = 0.0;
            if ((st = time_of(c, ms)) != SPT_OK) return st;
            if (ms < best_ms) {
                best_ms = ms;
                round_best = c;
            }
        }
        best = round_best;
    }
    cache_store(cache_path, key, best, best_ms);
    *out = best;
    return SPT_OK;
}

}  // extern "C"
