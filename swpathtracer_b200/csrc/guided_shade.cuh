// guided_shade.cuh -- one-sample MIS between the learned guiding mixture and BSDF sampling.
//
// Guiding applies to materials with one opaque, non-delta layer (Lambertian, Cook-Torrance): there the
// reference's layered walk reduces to one BSDF sample (materials/layered_bsdf.cpp:20-63 with one layer),
// and the BSDF's sampling density is known in closed form.  A direction is drawn from the guide with
// probability mix and from the BSDF sampler otherwise, and weighted by f cos / (mix q + (1 - mix) p_bsdf),
// so the estimator stays unbiased whatever the guide has learned.  A smooth dielectric over a
// Cook-Torrance layer is guided through the part of its walk that has a density (coated_sample).
// Other stacks and the delta materials keep the reference's own sampling.
#pragma once

#include "guiding.cuh"
#include "shade.cuh"

namespace spt {

// A smooth dielectric over a Cook-Torrance layer (the reference's 2-layer coating, e.g. a varnished
// metal): guided through the walk's single-internal-bounce component (layered_t1 below).
__device__ __forceinline__ bool coated(const DevScene& S, const DevMaterial& m) {
    if (m.layer_count != 2) return false;
    return S.bsdf[S.layer_ids[m.layer_begin]].type == SPT_BSDF_SMOOTH_DIELECTRIC &&
           S.bsdf[S.layer_ids[m.layer_begin + 1]].type == SPT_BSDF_COOK_TORRANCE;
}

__device__ __forceinline__ bool guidable(const DevScene& S, const DevMaterial& m) {
    if (coated(S, m)) return true;
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
    // where the Beckmann exponential underflows the density is 0 (the 1 / nh^4 factor alone would
    // overflow and turn the product into NaN)
    const float e = expf((nh2 - 1.0f) / (m2 * nh2));
    if (!(e > 0.0f)) return 0.0f;
    const float d = e / (kPi * m2 * nh2 * nh2);
    const float om = fabsf(dot(wi, h));
    return om > 0.0f ? d * nh / (4.0f * om) : 0.0f;
}

// A BSDF value at a direction the guide chose.  Far outside a narrow Cook-Torrance lobe the reference's
// f (bsdf_f, kept bit for bit) meets 0 * infinity; its limit there is 0.
__device__ __forceinline__ V3 finite_or_zero(V3 f) {
    return (isfinite(f.x) && isfinite(f.y) && isfinite(f.z)) ? f : v3(0.0f, 0.0f, 0.0f);
}

struct GuidedSample {
    V3 wi_local, wi_world;
    V3 f, refl;
    float p;        // mixture density of the sampled direction
};

// The coated stack's single-internal-bounce component, evaluated at an exit direction w (local,
// w.y > 0) for the outgoing direction wo (w.y > 0).  The reference's walk (materials/layered_bsdf.cpp:
// 10-74) reaches w this way: at the top it refracts with probability 1 - F(wo) (smooth_dielectric.cpp:
// 30-51; Schlick IOR form, fresnel_schlick.cpp:20-39), the Cook-Torrance layer samples wi' (its own
// sampler's density p_ct), and the top refracts it out along w with probability 1 - F(-wi').  The
// refraction maps (refraction_bsdf_sampler.cpp:5-24) give wi' = (w.x / eta, sqrt(1 - (1 - w.y^2) / eta^2),
// w.z / eta), and the solid angles relate by eta^2 wi'.y dw' = w.y dw.  So the exit direction
// has the density p = T p_ct(wo', wi') w.y / (eta^2 wi'.y), T the two transmission probabilities, and
// the walk's weight f cos / pdf is f_ct(wo', wi') wi'.y / p_ct (layered_bsdf.cpp: the interior layer
// contributes f wi.y, each dielectric crossing f = 1 / wi.y against the path tracer's cos).  Their
// product, the component's integrand g(w) = T f_ct w.y / eta^2, needs no sampler density.  Returned:
// f with f * w.y = g, the density p, the reflectance the walk reports (the Cook-Torrance layer's).
struct CoatT1 {
    V3 f, refl;
    float p;
};
__device__ __forceinline__ CoatT1 coat_t1(const DevBsdf& top, const DevBsdf& bot, V3 wo, V3 w) {
    CoatT1 r;
    r.f = v3(0.0f, 0.0f, 0.0f);
    r.refl = v3(0.0f, 0.0f, 0.0f);
    r.p = 0.0f;
    const float eta = top.scalar, inv = 1.0f / eta;
    const float a0 = 1.0f - inv * inv * (1.0f - wo.y * wo.y), a1 = 1.0f - inv * inv * (1.0f - w.y * w.y);
    if (!(wo.y > 0.0f) || !(w.y > 0.0f) || !(a0 > 0.0f) || !(a1 > 0.0f)) return r;
    const V3 wop = v3(wo.x * inv, sqrtf(a0), wo.z * inv);   // the camera side, inside the coat
    const V3 wip = v3(w.x * inv, sqrtf(a1), w.z * inv);     // the direction that leaves along w
    // the walk's exit test from inside (TIR) is the reference dielectric's, on -wi'
    if (eta * eta * (1.0f - wip.y * wip.y) > 1.0f) return r;
    const float t = (1.0f - fresnel_ior(eta, wo.y)) * (1.0f - fresnel_ior(eta, -wip.y));
    const float pct = sampler_density(bot, wop, wip);
    if (!(pct > 0.0f)) return r;
    const float k = t / (eta * eta);
    r.f = finite_or_zero(bsdf_f(bot, wop, wip)) * k;
    r.p = k * pct * w.y / wip.y;
    r.refl = bsdf_refl(bot, wop, wip);
    return r;
}

// One-sample MIS for the coated stack, with the guide and the reference's own walk as techniques for
// the single-internal-bounce component and the walk alone for the rest (the specular reflection at
// the top, the paths with internal reflections): with probability mix a direction from the guide,
// weighted g / (mix q + (1 - mix) p) (coated_guide_sample); otherwise the walk, whose single-bounce
// outcomes take that same weight and whose other outcomes take f cos / (pdf (1 - mix))
// (coated_walk_weight).  The expectation is the walk's.  The shade kernel makes the technique choice
// and runs the walk itself, so that one copy of the walk serves guided and plain vertices.
__device__ __forceinline__ GuidedSample coated_guide_sample(const DevScene& S, const DevMaterial& m, const float* frame,
                                                            V3 wo, const float* entry, float mix, Stream& s) {
    const DevBsdf top = S.bsdf[S.layer_ids[m.layer_begin]];
    const DevBsdf bot = S.bsdf[S.layer_ids[m.layer_begin + 1]];
    GuidedSample g;
    const float u0 = s.next(), u1 = s.next(), u2 = s.next();
    g.wi_world = guide::cached_mixture_sample(entry, u0, u1, u2);
    g.wi_local = mat_tmul(frame, g.wi_world);
    const CoatT1 c = coat_t1(top, bot, wo, g.wi_local);
    g.f = c.f;
    g.refl = c.refl;
    g.p = mix * guide::cached_mixture_pdf(entry, g.wi_world) + (1.0f - mix) * c.p;
    return g;
}

// The walk's outcome e (eval_layered) as the second technique: f and the density to divide by.
__device__ __forceinline__ void coated_walk_weight(const DevScene& S, const DevMaterial& m, V3 wo, V3 wi_world,
                                                   const LayerEval& e, const float* entry, float mix, V3& f,
                                                   float& pdf) {
    if (e.bounces == 3 && e.out_top && e.pdf > 0.0f && (e.f.x != 0.0f || e.f.y != 0.0f || e.f.z != 0.0f)) {
        const CoatT1 c = coat_t1(S.bsdf[S.layer_ids[m.layer_begin]], S.bsdf[S.layer_ids[m.layer_begin + 1]], wo, e.wi);
        f = c.f;
        pdf = mix * guide::cached_mixture_pdf(entry, wi_world) + (1.0f - mix) * c.p;
    } else {
        f = e.f;
        pdf = e.pdf * (1.0f - mix);
    }
}

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
    g.f = wi.y > 0.0f ? finite_or_zero(bsdf_f(b, wo, wi)) : v3(0.0f, 0.0f, 0.0f);
    g.refl = wi.y > 0.0f ? bsdf_refl(b, wo, wi) : v3(0.0f, 0.0f, 0.0f);
    g.p = mix * guide::cached_mixture_pdf(entry, g.wi_world) + (1.0f - mix) * sampler_density(b, wo, wi);
    return g;
}

}  // namespace spt
