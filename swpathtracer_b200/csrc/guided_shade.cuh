// guided_shade.cuh -- one-sample MIS between the learned guiding mixture and BSDF sampling.
//
// Guiding applies to materials with one opaque, non-delta layer (Lambertian, Cook-Torrance): there the
// reference's layered walk reduces to one BSDF sample (materials/layered_bsdf.cpp:20-63 with one layer),
// and the BSDF's sampling density is known in closed form.  A direction is drawn from the guide with
// probability mix and from the BSDF sampler otherwise, and weighted by f cos / (mix q + (1 - mix) p_bsdf),
// so the estimator stays unbiased whatever the guide has learned.  Delta and layered materials keep
// the reference's own sampling.
#pragma once

#include "guiding.cuh"
#include "shade.cuh"

namespace spt {

__device__ __forceinline__ bool guidable(const DevScene& S, const DevMaterial& m) {
    if (m.layer_count != 1) return false;
    const int t = S.bsdf[S.layer_ids[m.layer_begin]].type;
    return t == SPT_BSDF_LAMBERTIAN || t == SPT_BSDF_COOK_TORRANCE;
}

// Density of the reference's BSDF sampler at wi (local frame, y = normal):
// cosine (bsdf_samplers/cosine_bsdf_sampler.cpp), uniform (uniform_bsdf_sampler.cpp) and the
// Beckmann microfacet sampler (cook_torrance_bsdf_sampler.cpp:7-20: D(m) cos(theta_m) over m,
// times the reflection Jacobian 1 / (4 |wi.m|)).
__device__ __forceinline__ float sampler_density(const DevBsdf& b, V3 wo, V3 wi) {
    if (!(wi.y > 0.0f)) return 0.0f;
    if (b.sampler == SPT_SAMPLER_UNIFORM) return 1.0f / (2.0f * kPi);
    if (b.type == SPT_BSDF_LAMBERTIAN) return wi.y / kPi;
    const V3 hs = wo + wi;
    const float hl = sqrtf(dot(hs, hs));
    if (!(hl > 0.0f)) return 0.0f;
    const V3 h = hs * (1.0f / hl);
    const float nh = h.y;
    if (!(nh > 0.0f)) return 0.0f;
    const float m2 = b.scalar * b.scalar, nh2 = nh * nh;
    const float d = expf((nh2 - 1.0f) / (m2 * nh2)) / (kPi * m2 * nh2 * nh2);
    const float om = fabsf(dot(wi, h));
    return om > 0.0f ? d * nh / (4.0f * om) : 0.0f;
}

struct GuidedSample {
    V3 wi_local, wi_world;
    V3 f, refl;
    float p;        // mixture density of the sampled direction
};

// frame: columns u, v (= normal), w.  entry: a lobe-cache entry (guiding.cuh, kCacheEntry floats).
__device__ __forceinline__ GuidedSample guided_sample(const DevScene& S, const DevMaterial& m, const float* frame,
                                                      V3 wo, const float* entry, float mix, Stream& s) {
    const DevBsdf b = S.bsdf[S.layer_ids[m.layer_begin]];
    GuidedSample g;
    if (s.next() < mix) {
        const float u0 = s.next(), u1 = s.next(), u2 = s.next();
        g.wi_world = guide::cached_mixture_sample(entry, u0, u1, u2);
        g.wi_local = mat_tmul(frame, g.wi_world);
    } else {
        const BSample bs = bsdf_sample(b, wo, s);
        g.wi_local = bs.wi;
        g.wi_world = mat_mul(frame, bs.wi);
    }
    const V3 wi = g.wi_local;
    g.f = wi.y > 0.0f ? bsdf_f(b, wo, wi) : v3(0.0f, 0.0f, 0.0f);
    g.refl = wi.y > 0.0f ? bsdf_refl(b, wo, wi) : v3(0.0f, 0.0f, 0.0f);
    g.p = mix * guide::cached_mixture_pdf(entry, g.wi_world) + (1.0f - mix) * sampler_density(b, wo, wi);
    return g;
}

}  // namespace spt
