// shade.cuh -- BSDF sampling/evaluation and the layered random walk on the device.
//
// Each function restates the reference's code with its float operation order; the draws come
// from the path's Philox stream (spt_device.cuh) in the order the reference draws from its
// mt19937: sampler draws per layer event, the dielectric's reflect/refract choice, then the
// russian-roulette draw.
#pragma once

#include "spt_device.cuh"

namespace spt {

// FresnelSchlick::getReflectance, normal-incidence form (materials/fresnel_schlick.cpp:14-18)
__device__ __forceinline__ V3 fresnel_f0(const DevBsdf& b, float c) {
    float c5 = 1.0f - c;
    c5 = c5 * c5 * c5 * c5 * c5;
    return v3(b.r + (1.0f - b.r) * c5, b.g + (1.0f - b.g) * c5, b.b + (1.0f - b.b) * c5);
}

// FresnelSchlick::getReflectance, IOR form with ior_i = 1 (materials/fresnel_schlick.cpp:20-38)
__device__ __forceinline__ float fresnel_ior(float ior, float c) {
    float ior_i = 1.0f, ior_t = ior;
    if (c < 0.0f) {
        ior_i = ior;
        ior_t = 1.0f;
        float eta = ior_i / ior_t;
        float a = 1 - eta * eta * (1.0f - c * c);
        c = sqrtf(a);
    }
    float r0 = (ior_i - ior_t) / (ior_i + ior_t);
    r0 = r0 * r0;
    float c5 = 1.0f - c;
    c5 = c5 * c5 * c5 * c5 * c5;
    return r0 + (1.0f - r0) * c5;
}

struct BSample {
    V3 wi;
    float pdf;
};

// bsdf_samplers/cosine_bsdf_sampler.cpp:5-17
__device__ __forceinline__ BSample cosine_sample(Stream& s) {
    float r1 = s.next(), r2 = s.next();
    float phi = 2.0f * kPi * r2;
    float ct = sqrtf(r1);
    float st = sqrtf(1.0f - ct * ct);
    return BSample{v3(cosf(phi) * st, ct, sinf(phi) * st), ct / kPi};
}
// bsdf_samplers/uniform_bsdf_sampler.cpp:5-14
__device__ __forceinline__ BSample uniform_sample(Stream& s) {
    float r1 = s.next(), r2 = s.next();
    float phi = 2.0f * kPi * r2;
    float st = sqrtf(1.0f - r1 * r1);
    return BSample{v3(cosf(phi) * st, r1, sinf(phi) * st), 1.0f / (2.0f * kPi)};
}
// bsdf_samplers/smooth_specular_bsdf_sampler.cpp:5-7
__device__ __forceinline__ BSample mirror_sample(V3 wo) { return BSample{v3(-wo.x, wo.y, -wo.z), 1.0f}; }
// bsdf_samplers/refraction_bsdf_sampler.cpp:5-24 (ior_i = 1)
__device__ __forceinline__ BSample refraction_sample(V3 wo, float ior) {
    float ior_i = 1.0f, ior_t = ior, signal = 1.0f;
    if (wo.y < 0.0f) {
        ior_i = ior;
        ior_t = 1.0f;
        signal = -1.0f;
    }
    float a = 1.0f - ((ior_i * ior_i) / (ior_t * ior_t)) * (1.0f - wo.y * wo.y);
    V3 n = v3(0.0f, 1.0f, 0.0f);
    V3 wi = normalize((ior_i / ior_t) * (n * wo.y - wo) - (signal * n) * sqrtf(a));
    return BSample{wi, 1.0f};
}
// bsdf_samplers/cook_torrance_bsdf_sampler.cpp:22-42
__device__ __forceinline__ float ct_pdf(float m, V3 wo, V3 wi) {
    if (wi.y <= 0.0f) return 1.0f;
    V3 h = normalize(wo + wi);
    float nh = fmaxf(0.0f, h.y);
    if (nh == 0.0f) return 1e-5f;
    float nh2 = nh * nh;
    float m2 = m * m;
    float d1 = 1.0f / (kPi * m2 * nh * nh * nh * nh);
    float d2 = (nh2 - 1.0f) / (m2 * nh2);
    float om = dot(wi, h);
    if (om <= 0.0f) return 1e+5f;
    return (d1 * expf(d2) * nh) / (4.0f * om);
}
// bsdf_samplers/cook_torrance_bsdf_sampler.cpp:7-20
__device__ __forceinline__ BSample ct_sample(float m, V3 wo, Stream& s) {
    float r1 = s.next(), r2 = s.next();
    float phi = 2.0f * kPi * r2;
    float theta = atanf(sqrtf(-(m * m) * logf(1.0f - r1)));
    float st = sinf(theta);
    V3 mv = v3(cosf(phi) * st, cosf(theta), sinf(phi) * st);
    V3 wi = (2.0f * mv) * dot(mv, wo) - wo;
    return BSample{wi, ct_pdf(m, wo, wi)};
}

__device__ __forceinline__ BSample bsdf_sample(const DevBsdf& b, V3 wo, Stream& s) {
    switch (b.type) {
        case SPT_BSDF_LAMBERTIAN:
            return b.sampler == SPT_SAMPLER_UNIFORM ? uniform_sample(s) : cosine_sample(s);
        case SPT_BSDF_SMOOTH_CONDUCTOR:
            return b.sampler == SPT_SAMPLER_UNIFORM ? uniform_sample(s) : mirror_sample(wo);
        case SPT_BSDF_SMOOTH_DIELECTRIC: {  // materials/smooth_dielectric.cpp:30-51
            float ior_i = 1.0f, ior_t = b.scalar;
            if (wo.y < 0.0f) {
                ior_i = b.scalar;
                ior_t = 1.0f;
            }
            float a = ((ior_i * ior_i) / (ior_t * ior_t)) * (1.0f - wo.y * wo.y);
            if (a > 1.0f) return mirror_sample(wo);
            float f = fresnel_ior(b.scalar, wo.y);
            if (s.next() < f) return mirror_sample(wo);
            return refraction_sample(wo, b.scalar);
        }
        default:
            return b.sampler == SPT_SAMPLER_UNIFORM ? uniform_sample(s) : ct_sample(b.scalar, wo, s);
    }
}

// BSDF::f (lambertian.cpp:9-16, smooth_conductor.cpp:6-14, smooth_dielectric.cpp:15-21, cook_torrance.cpp:9-44)
__device__ __forceinline__ V3 bsdf_f(const DevBsdf& b, V3 wo, V3 wi) {
    switch (b.type) {
        case SPT_BSDF_LAMBERTIAN:
            return wi.y > 0.0f ? v3(b.br, b.bg, b.bb) : v3(0.0f, 0.0f, 0.0f);
        case SPT_BSDF_SMOOTH_CONDUCTOR:
            return wi.y > 0.0f ? fresnel_f0(b, wi.y) / wi.y : v3(0.0f, 0.0f, 0.0f);
        case SPT_BSDF_SMOOTH_DIELECTRIC: {
            if (wi.y == 0.0f) return v3(0.0f, 0.0f, 0.0f);
            float q = 1.0f / wi.y;
            return v3(q, q, q);
        }
        default: {
            if (wi.y <= 0.0f) return v3(0.0f, 0.0f, 0.0f);
            V3 h = normalize(wo + wi);
            float nv = fmaxf(0.0f, wo.y), nl = fmaxf(0.0f, wi.y);
            float vh = fmaxf(0.0f, dot(wo, h)), nh = fmaxf(0.0f, h.y);
            float m = b.scalar;
            if ((nv == 0.0f) || (nl == 0.0f) || (vh == 0.0f) || (nh == 0.0f) || (m == 0.0f))
                return v3(0.0f, 0.0f, 0.0f);
            float lh = fmaxf(0.0f, dot(wi, h));
            float nh2 = nh * nh, m2 = m * m;
            float d1 = 1.0f / (kPi * m2 * nh2 * nh2);
            float d2 = (nh2 - 1.0f) / (m2 * nh2);
            float d = d1 * expf(d2);
            float g1 = 2.0f * nh / vh;
            float g = fminf(1.0f, fminf(g1 * nv, g1 * nl));
            V3 f = fresnel_f0(b, lh);
            return (f * d * g) / (4.0f * nv * nl);
        }
    }
}

// BSDF::getReflectance (lambertian.cpp:18-22, smooth_conductor.cpp:16-20, smooth_dielectric.cpp:23-28,
// cook_torrance.cpp:46-51)
__device__ __forceinline__ V3 bsdf_refl(const DevBsdf& b, V3 wo, V3 wi) {
    switch (b.type) {
        case SPT_BSDF_LAMBERTIAN:
            return v3(b.r, b.g, b.b);
        case SPT_BSDF_SMOOTH_CONDUCTOR:
            return fresnel_f0(b, wi.y);
        case SPT_BSDF_SMOOTH_DIELECTRIC:
            return v3(1.0f, 1.0f, 1.0f);
        default: {
            V3 h = normalize(wo + wi);
            float lh = fmaxf(0.0f, dot(wi, h));
            return fresnel_f0(b, lh);
        }
    }
}

struct LayerEval {
    V3 f, refl, wi;
    float pdf;
    int bounces;    // layer events of the walk
    bool out_top;   // the walk left through the top of the stack
};

// LayeredBSDF::evalBSDF (materials/layered_bsdf.cpp:10-74): random walk through the layer stack,
// bounded at 500 layer events like the reference.
__device__ __forceinline__ LayerEval eval_layered(const DevScene& S, const DevMaterial& m, V3 wo, Stream& s) {
    const int n = m.layer_count;
    V3 fb = v3(1.0f, 1.0f, 1.0f), fr = v3(1.0f, 1.0f, 1.0f);
    float fp = 1.0f;
    V3 nwo = wo, wi = v3(0.0f, 0.0f, 0.0f);
    bool inf = false;
    int bounce = 0;
    int id = (nwo.y > 0.0f) ? 0 : n - 1;
    const float INF = __int_as_float(0x7f800000);
    while ((id > -1) && (id < n) && (fp > 0.0f) && !inf && (bounce < 500)) {
        const DevBsdf b = S.bsdf[S.layer_ids[m.layer_begin + id]];
        BSample smp = bsdf_sample(b, nwo, s);
        wi = smp.wi;
        fp *= smp.pdf;
        if (!(fp < INF)) inf = true;
        if (wi.y > 0.0f) {
            V3 f = bsdf_f(b, nwo, wi);
            fb = fb * (id == 0 ? f : f * wi.y);
            fr = fr * bsdf_refl(b, nwo, wi);
            --id;
        } else if ((wi.y < 0.0f) && (b.type == SPT_BSDF_SMOOTH_DIELECTRIC)) {
            V3 f = bsdf_f(b, nwo, wi);
            fb = fb * (id == n - 1 ? f : f * wi.y);
            fr = fr * bsdf_refl(b, nwo, wi);
            ++id;
        } else {
            fp = 0.0f;
        }
        if (!((fb.x < INF) && (fb.y < INF) && (fb.z < INF))) inf = true;
        nwo = -wi;
        ++bounce;
    }
    LayerEval r;
    r.wi = wi;
    r.bounces = bounce;
    r.out_top = id == -1;
    if ((bounce < 500) && !inf && (fp > 0.0f)) {
        r.pdf = fp;
        r.f = fb;
        r.refl = fr;
    } else {
        r.pdf = 1.0f;
        r.f = v3(0.0f, 0.0f, 0.0f);
        r.refl = v3(0.0f, 0.0f, 0.0f);
    }
    return r;
}

// ONB from a normal (core/onb.cpp:3-16): columns u, v = n, w; local y is the normal.
__device__ __forceinline__ void onb_from_normal(V3 v, float m[9]) {
    V3 w = (fabsf(v.x) > fabsf(v.y)) ? normalize(v3(v.z, 0.0f, -v.x)) : normalize(v3(0.0f, -v.z, v.y));
    V3 u = cross(v, w);
    m[0] = u.x; m[1] = u.y; m[2] = u.z;
    m[3] = v.x; m[4] = v.y; m[5] = v.z;
    m[6] = w.x; m[7] = w.y; m[8] = w.z;
}

}  // namespace spt
