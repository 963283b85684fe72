// wavefront.h -- the batched path-tracing wavefront shared by the single-scene entry points, the
// batch entry point and the autotuner.
#pragma once

#include <vector>

#include "spt_internal.h"

namespace spt {

// One scene of a batch as the kernels see it.
struct PtJob {
    DevScene S;
    DevCamera cam;
    uint64_t seed;
    uint64_t first;        // global index of the job's first camera path
    uint64_t total;        // camera paths of the job
    uint32_t spp, nsub;    // samples per pixel (after the square rounding), strata per axis
    float sw;              // stratum width
    int sampler, rr, path_length, cap;
    uint32_t npix;         // viewport pixels
    uint32_t spp_offset;
    uint32_t layered;      // the scene has layered materials (grouped shading pays off)
    uint32_t stack_bound;  // traversal stack entries the scene's 8-wide tree can need (2 (levels - 1))
    uint32_t s_begin, s_end;  // the samples [s_begin, s_end) of the spp this render traces; the image is
                              // cleared when s_begin == 0 and turned into means when s_end == spp
    float* image;          // W*H*3 radiance sums, then means
};

spt_status make_job(spt_context* ctx, const spt_scene* sc, const spt_camera* cam, const spt_pt_params* p,
                    float* d_image, PtJob& out);
spt_tune default_tune();
// Renders all jobs in one wavefront on ctx->stream.  segments: rays traced; gpu_ms: device time.
namespace guide {
struct Guide;
}
// guide: when not null, guidable vertices sample the guide (one-sample MIS) and the guide trains on
// the render's paths for up to train_budget optimiser steps (the number taken goes to train_steps).
spt_status render_jobs(spt_context* ctx, std::vector<PtJob>& jobs, const spt_tune& tune, uint64_t* segments,
                       float* gpu_ms, guide::Guide* guide = nullptr, uint32_t train_budget = 0,
                       uint32_t* train_steps = nullptr);
// Sets the job's sample range to [s_begin, s_end) (clamped to its spp) and its path count to match.
void set_sample_range(PtJob& J, uint32_t s_begin, uint32_t s_end);

}  // namespace spt
