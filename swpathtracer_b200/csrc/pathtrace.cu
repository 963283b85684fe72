// pathtrace.cu -- wavefront path tracer (placeholder until the kernels land).
#include "spt_internal.h"

using namespace spt;

extern "C" {

spt_status spt_pathtrace(spt_context* ctx, const spt_scene*, const spt_camera*, const spt_pt_params*, float*,
                         spt_render_stats*) {
    return fail(ctx, SPT_ERR_UNSUPPORTED, "path tracer not built yet");
}

spt_status spt_pathtrace_device(spt_context* ctx, const spt_scene*, const spt_camera*, const spt_pt_params*, float*,
                                spt_render_stats*) {
    return fail(ctx, SPT_ERR_UNSUPPORTED, "path tracer not built yet");
}

}  // extern "C"
