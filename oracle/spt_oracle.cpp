// spt_oracle.cpp -- TEST INFRASTRUCTURE ONLY (see spt_oracle.h): the project's CPU
// restatement of the reference renderer's hot path, the checker for the CUDA backend.
//
// Compiled with -ffp-contract=off (no FMA contraction) so every float operation rounds
// like the reference's ISO C++14 / SSE build.  Each function names the reference code it
// restates (file:line, paths within the reference project).
#include "spt_oracle.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <vector>

#include <omp.h>

namespace {

const float kPi = 3.141592653589793238462643383279502884f;  // core/core.h:4
const float kInf = std::numeric_limits<float>::infinity();

// ---- vector arithmetic with glm's operation order (see oracle/shim/glm/shim_core.hpp) ----
struct V3 {
    float x, y, z;
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
inline V3 mk(float x, float y, float z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator*(V3 a, V3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
inline V3 operator*(V3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
inline V3 operator*(float s, V3 a) { return mk(s * a.x, s * a.y, s * a.z); }
inline V3 operator/(V3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
inline V3 operator-(V3 a) { return mk(-a.x, -a.y, -a.z); }
inline V3 operator-(V3 a, float s) { return mk(a.x - s, a.y - s, a.z - s); }
inline V3 operator+(V3 a, float s) { return mk(a.x + s, a.y + s, a.z + s); }
inline float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return mk(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y); }
inline V3 normalize(V3 v) { return v * (1.0f / std::sqrt(dot(v, v))); }
inline float fmin_g(float x, float y) { return (y < x) ? y : x; }  // glm::min
inline float fmax_g(float x, float y) { return (x < y) ? y : x; }  // glm::max
inline V3 vmin(V3 a, V3 b) { return mk(fmin_g(a.x, b.x), fmin_g(a.y, b.y), fmin_g(a.z, b.z)); }
inline V3 vmax(V3 a, V3 b) { return mk(fmax_g(a.x, b.x), fmax_g(a.y, b.y), fmax_g(a.z, b.z)); }
inline V3 ld3(const float* p) { return mk(p[0], p[1], p[2]); }

// Column-major 3x3 (columns c0 c1 c2); mul() sums the columns left to right like glm.
struct M3 {
    V3 c0, c1, c2;
};
inline V3 mul(const M3& m, V3 v) {
    return mk(m.c0.x * v.x + m.c1.x * v.y + m.c2.x * v.z, m.c0.y * v.x + m.c1.y * v.y + m.c2.y * v.z,
              m.c0.z * v.x + m.c1.z * v.y + m.c2.z * v.z);
}
inline M3 transpose(const M3& m) {
    return M3{mk(m.c0.x, m.c1.x, m.c2.x), mk(m.c0.y, m.c1.y, m.c2.y), mk(m.c0.z, m.c1.z, m.c2.z)};
}

// ---- AABB (acceleration/aabb.cpp) ---------------------------------------------------------
struct Box {
    V3 mn, mx;
};
inline Box box_union(const Box& a, const Box& b) { return Box{vmin(a.mn, b.mn), vmax(a.mx, b.mx)}; }  // aabb.h:30-32
inline float box_area(const Box& b) {                                                             // aabb.cpp:11-16
    float l = b.mx.x - b.mn.x, m = b.mx.y - b.mn.y, n = b.mx.z - b.mn.z;
    return 2.0f * (l * (m + n) + m * n);
}
// Williams et al. slab test exactly as aabb.cpp:31-99 (1/d per axis, sign-selected planes,
// no tmax >= 0 test, NaN comparisons fall through).
inline bool box_hit(const Box& b, V3 o, V3 d) {
    float tmin, tmax, tymin, tymax, tzmin, tzmax;
    float divx = 1.0f / d.x;
    if (divx >= 0.0f) { tmin = (b.mn.x - o.x) * divx; tmax = (b.mx.x - o.x) * divx; }
    else { tmin = (b.mx.x - o.x) * divx; tmax = (b.mn.x - o.x) * divx; }
    float divy = 1.0f / d.y;
    if (divy >= 0.0f) { tymin = (b.mn.y - o.y) * divy; tymax = (b.mx.y - o.y) * divy; }
    else { tymin = (b.mx.y - o.y) * divy; tymax = (b.mn.y - o.y) * divy; }
    if ((tmin > tymax) || (tymin > tmax)) return false;
    if (tymin > tmin) tmin = tymin;
    if (tymax < tmax) tmax = tymax;
    float divz = 1.0f / d.z;
    if (divz >= 0.0f) { tzmin = (b.mn.z - o.z) * divz; tzmax = (b.mx.z - o.z) * divz; }
    else { tzmin = (b.mx.z - o.z) * divz; tzmax = (b.mn.z - o.z) * divz; }
    if ((tmin > tzmax) || (tzmin > tmax)) return false;
    return true;
}
// aabb.cpp:101-105, epsilon 1e-3 (aabb.cpp:3)
inline bool box_inside(const Box& b, V3 p) {
    const float e = 1e-3f;
    return (p.x >= (b.mn.x - e)) && (p.x <= (b.mx.x + e)) && (p.y >= (b.mn.y - e)) && (p.y <= (b.mx.y + e)) &&
           (p.z >= (b.mn.z - e)) && (p.z <= (b.mx.z + e));
}

// ---- primitives -------------------------------------------------------------------------------
struct Prim {
    int type;
    V3 v0, v1, v2;     // triangle vertices; sphere: v0 = centre
    float radius;
    V3 n0, n1, n2;     // smooth-triangle vertex normals
    V3 face_normal;    // triangle.cpp:6: normalize(cross(v1 - v0, v2 - v0))
    uint32_t material;
};

struct Rec {
    float t;
    V3 pos, normal;
    uint32_t material, prim;
};

// Moller-Trumbore, non-culling branch (primitives/triangle.cpp:12-74), epsilon 1e-6 (:3).
inline bool tri_hit(const Prim& p, V3 o, V3 d, Rec& r) {
    V3 e1 = p.v1 - p.v0;
    V3 e2 = p.v2 - p.v0;
    V3 pvec = cross(d, e2);
    float det = dot(e1, pvec);
    if ((det > -1e-6f) && (det < 1e-6f)) return false;
    float inv_det = 1.0f / det;
    V3 tvec = o - p.v0;
    float u = dot(tvec, pvec) * inv_det;
    if ((u < 0.0f) || (u > 1.0f)) return false;
    V3 qvec = cross(tvec, e1);
    float v = dot(d, qvec) * inv_det;
    if ((v < 0.0f) || ((u + v) > 1.0f)) return false;
    float t = dot(e2, qvec) * inv_det;
    r.t = t;
    r.pos = o + d * t;
    if (p.type == SPT_PRIM_SMOOTH_TRIANGLE)  // smooth_triangle.h:11-13
        r.normal = normalize(p.n0 * ((1.0f - u) - v) + p.n1 * u + p.n2 * v);
    else
        r.normal = p.face_normal;
    r.material = p.material;
    return true;
}

// Hultquist ray-sphere (primitives/sphere.cpp:6-38), epsilon 1e-5 (sphere.h:22).
inline bool sphere_hit(const Prim& p, V3 o, V3 d, Rec& r) {
    V3 eo = p.v0 - o;
    float v = dot(eo, d);
    float disc = (p.radius * p.radius) - (dot(eo, eo) - (v * v));
    if (disc < 0.0f) return false;
    float dd = std::sqrt(disc);
    float t1 = v - dd, t2 = v + dd;
    r.t = (t1 > 1e-5f) ? t1 : t2;
    r.pos = o + r.t * d;
    r.normal = normalize(r.pos - p.v0);
    r.material = p.material;
    return true;
}

inline bool prim_hit(const Prim& p, V3 o, V3 d, Rec& r) {
    return p.type == SPT_PRIM_SPHERE ? sphere_hit(p, o, d, r) : tri_hit(p, o, d, r);
}

inline Box prim_box(const Prim& p) {
    if (p.type == SPT_PRIM_SPHERE) return Box{p.v0 - p.radius, p.v0 + p.radius};  // sphere.cpp:48-56
    return Box{vmin(vmin(p.v0, p.v1), p.v2), vmax(vmax(p.v0, p.v1), p.v2)};        // triangle.cpp:76-83
}
inline V3 prim_centroid(const Prim& p) {
    if (p.type == SPT_PRIM_SPHERE) return p.v0;        // sphere.cpp:58-60
    return ((p.v0 + p.v1) + p.v2) * (1.0f / 3.0f);       // triangle.cpp:85-87
}

// ---- materials (materials/*.cpp, bsdf_samplers/*.cpp) -------------------------------------------
struct Bsdf {
    int type, sampler;
    V3 rgb;
    float scalar;
    V3 brdf;  // lambertian.cpp:6, reflectance / PI
};

struct Scene;

// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as easy as 1, 2, 3", SC'11).
void philox(const uint32_t c_in[4], const uint32_t k_in[2], uint32_t out[4]) {
    uint32_t c0 = c_in[0], c1 = c_in[1], c2 = c_in[2], c3 = c_in[3];
    uint32_t k0 = k_in[0], k1 = k_in[1];
    for (int r = 0; r < 10; ++r) {
        if (r > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c0;
        uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c2;
        uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
        uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// One sample stream: counter (path lo, path hi, stream id, block), 4 uniforms per block.
struct Stream {
    uint32_t key[2];
    uint32_t ctr[4];
    uint32_t buf[4];
    int pos;
    Stream(uint64_t seed, uint64_t path, uint32_t stream_id) {
        key[0] = static_cast<uint32_t>(seed);
        key[1] = static_cast<uint32_t>(seed >> 32);
        ctr[0] = static_cast<uint32_t>(path);
        ctr[1] = static_cast<uint32_t>(path >> 32);
        ctr[2] = stream_id;
        ctr[3] = 0;
        pos = 4;
    }
    float next() {
        if (pos == 4) {
            philox(ctr, key, buf);
            ++ctr[3];
            pos = 0;
        }
        return static_cast<float>(buf[pos++] >> 8) * (1.0f / 16777216.0f);
    }
};

// FresnelSchlick::getReflectance (materials/fresnel_schlick.cpp:11-39).
V3 fresnel_f0(V3 f0, float c) {
    float c5 = 1.0f - c;
    c5 = c5 * c5 * c5 * c5 * c5;
    return f0 + mk(1.0f - f0.x, 1.0f - f0.y, 1.0f - f0.z) * c5;
}
V3 fresnel_ior(float ior_i_, float ior_t_, float c) {
    float ior_i = ior_i_, ior_t = ior_t_;
    if (c < 0.0f) {
        ior_i = ior_t_;
        ior_t = ior_i_;
        float eta = ior_i / ior_t;
        float a = 1 - eta * eta * (1.0f - c * c);
        c = std::sqrt(a);
    }
    float r0 = (ior_i - ior_t) / (ior_i + ior_t);
    r0 = r0 * r0;
    float c5 = 1.0f - c;
    c5 = c5 * c5 * c5 * c5 * c5;
    float f = r0 + (1.0f - r0) * c5;
    return mk(f, f, f);
}

struct Sample {
    V3 wi;
    float pdf;
};

// bsdf_samplers/cosine_bsdf_sampler.cpp:5-17
Sample cosine_sample(Stream& s) {
    float r1 = s.next(), r2 = s.next();
    float phi = 2.0f * kPi * r2;
    float ct = std::sqrt(r1);
    float st = std::sqrt(1.0f - ct * ct);
    return Sample{mk(std::cos(phi) * st, ct, std::sin(phi) * st), ct / kPi};
}
// bsdf_samplers/uniform_bsdf_sampler.cpp:5-14
Sample uniform_sample(Stream& s) {
    float r1 = s.next(), r2 = s.next();
    float phi = 2.0f * kPi * r2;
    float st = std::sqrt(1.0f - r1 * r1);
    return Sample{mk(std::cos(phi) * st, r1, std::sin(phi) * st), 1.0f / (2.0f * kPi)};
}
// bsdf_samplers/smooth_specular_bsdf_sampler.cpp:5-7
Sample mirror_sample(V3 wo) { return Sample{mk(-wo.x, wo.y, -wo.z), 1.0f}; }
// bsdf_samplers/refraction_bsdf_sampler.cpp:5-24 (ior_i = 1)
Sample refraction_sample(V3 wo, float ior_) {
    float ior_i = 1.0f, ior_t = ior_, signal = 1.0f;
    if (wo.y < 0.0f) { ior_i = ior_; ior_t = 1.0f; signal = -1.0f; }
    float a = 1.0f - ((ior_i * ior_i) / (ior_t * ior_t)) * (1.0f - wo.y * wo.y);
    V3 n = mk(0.0f, 1.0f, 0.0f);
    V3 wi = normalize((ior_i / ior_t) * (n * wo.y - wo) - (signal * n) * std::sqrt(a));
    return Sample{wi, 1.0f};
}
// bsdf_samplers/cook_torrance_bsdf_sampler.cpp:22-42
float ct_pdf(float m, V3 wo, V3 wi) {
    if (wi.y <= 0.0f) return 1.0f;
    V3 h = normalize(wo + wi);
    float nh = std::max(0.0f, h.y);
    if (nh == 0.0f) return 1e-5f;
    float nh2 = nh * nh;
    float m2 = m * m;
    float d1 = 1.0f / (kPi * m2 * nh * nh * nh * nh);
    float d2 = (nh2 - 1.0f) / (m2 * nh2);
    float om = dot(wi, h);
    if (om <= 0.0f) return 1e+5f;
    return (d1 * std::exp(d2) * nh) / (4.0f * om);
}
// bsdf_samplers/cook_torrance_bsdf_sampler.cpp:7-20
Sample ct_sample(float m, V3 wo, Stream& s) {
    float r1 = s.next(), r2 = s.next();
    float phi = 2.0f * kPi * r2;
    float theta = std::atan(std::sqrt(-(m * m) * std::log(1.0f - r1)));
    V3 mv = mk(std::cos(phi) * std::sin(theta), std::cos(theta), std::sin(phi) * std::sin(theta));
    V3 wi = (2.0f * mv) * dot(mv, wo) - wo;
    return Sample{wi, ct_pdf(m, wo, wi)};
}

Sample bsdf_sample(const Bsdf& b, V3 wo, Stream& s) {
    switch (b.type) {
        case SPT_BSDF_LAMBERTIAN:
            return b.sampler == SPT_SAMPLER_UNIFORM ? uniform_sample(s) : cosine_sample(s);
        case SPT_BSDF_SMOOTH_CONDUCTOR:
            return b.sampler == SPT_SAMPLER_UNIFORM ? uniform_sample(s) : mirror_sample(wo);
        case SPT_BSDF_SMOOTH_DIELECTRIC: {  // materials/smooth_dielectric.cpp:30-51
            float ior_i = 1.0f, ior_t = b.scalar;
            if (wo.y < 0.0f) { ior_i = b.scalar; ior_t = 1.0f; }
            float a = ((ior_i * ior_i) / (ior_t * ior_t)) * (1.0f - wo.y * wo.y);
            if (a > 1.0f) return mirror_sample(wo);
            V3 f = fresnel_ior(1.0f, b.scalar, wo.y);
            float mr = std::max(std::max(f.x, f.y), f.z);
            if (s.next() < mr) return mirror_sample(wo);
            return refraction_sample(wo, b.scalar);
        }
        default:
            return b.sampler == SPT_SAMPLER_UNIFORM ? uniform_sample(s) : ct_sample(b.scalar, wo, s);
    }
}

// BSDF::f (lambertian.cpp:9-16, smooth_conductor.cpp:6-14, smooth_dielectric.cpp:15-21, cook_torrance.cpp:9-44)
V3 bsdf_f(const Bsdf& b, V3 wo, V3 wi) {
    switch (b.type) {
        case SPT_BSDF_LAMBERTIAN:
            return wi.y > 0.0f ? b.brdf : mk(0.0f, 0.0f, 0.0f);
        case SPT_BSDF_SMOOTH_CONDUCTOR:
            return wi.y > 0.0f ? fresnel_f0(b.rgb, wi.y) / wi.y : mk(0.0f, 0.0f, 0.0f);
        case SPT_BSDF_SMOOTH_DIELECTRIC:
            if (wi.y == 0.0) return mk(0.0f, 0.0f, 0.0f);
            return mk(1.0f / wi.y, 1.0f / wi.y, 1.0f / wi.y);
        default: {
            if (wi.y <= 0.0f) return mk(0.0f, 0.0f, 0.0f);
            V3 h = normalize(wo + wi);
            float nv = std::max(0.0f, wo.y), nl = std::max(0.0f, wi.y);
            float vh = std::max(0.0f, dot(wo, h)), nh = std::max(0.0f, h.y);
            float m = b.scalar;
            if ((nv == 0.0f) || (nl == 0.0f) || (vh == 0.0f) || (nh == 0.0f) || (m == 0.0f)) return mk(0.0f, 0.0f, 0.0f);
            float lh = std::max(0.0f, dot(wi, h));
            float nh2 = nh * nh, m2 = m * m;
            float d1 = 1.0f / (kPi * m2 * nh2 * nh2);
            float d2 = (nh2 - 1.0f) / (m2 * nh2);
            float d = d1 * std::exp(d2);
            float g1 = 2.0f * nh / vh;
            float g = std::min(1.0f, std::min(g1 * nv, g1 * nl));
            V3 f = fresnel_f0(b.rgb, lh);
            return (f * d * g) / (4.0f * nv * nl);
        }
    }
}

// BSDF::getReflectance (lambertian.cpp:18-22, smooth_conductor.cpp:16-20, smooth_dielectric.cpp:23-28,
// cook_torrance.cpp:46-51)
V3 bsdf_refl(const Bsdf& b, V3 wo, V3 wi) {
    switch (b.type) {
        case SPT_BSDF_LAMBERTIAN: return b.rgb;
        case SPT_BSDF_SMOOTH_CONDUCTOR: return fresnel_f0(b.rgb, wi.y);
        case SPT_BSDF_SMOOTH_DIELECTRIC: return mk(1.0f, 1.0f, 1.0f);
        default: {
            V3 h = normalize(wo + wi);
            float lh = std::max(0.0f, dot(wi, h));
            return fresnel_f0(b.rgb, lh);
        }
    }
}

struct Material {
    std::vector<int> layers;
    V3 emission;
};

// LayeredBSDF::evalBSDF (materials/layered_bsdf.cpp:10-74).
void eval_layered(const std::vector<Bsdf>& bsdfs, const Material& m, V3 wo, Stream& s, V3& f_out, V3& refl_out,
                  float& pdf_out, V3& wi_out) {
    const int n = static_cast<int>(m.layers.size());
    V3 fb = mk(1.0f, 1.0f, 1.0f), fr = mk(1.0f, 1.0f, 1.0f);
    float fp = 1.0f;
    V3 nwo = wo, wi = mk(0.0f, 0.0f, 0.0f);
    bool inf = false;
    int bounce = 0;
    int id = (nwo.y > 0.0f) ? 0 : n - 1;
    while ((id > -1) && (id < n) && (fp > 0.0f) && !inf && (bounce < 500)) {
        const Bsdf& b = bsdfs[m.layers[id]];
        Sample smp = bsdf_sample(b, nwo, s);
        wi = smp.wi;
        fp *= smp.pdf;
        if (!(fp < kInf)) inf = true;
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
        if (!((fb.x < kInf) && (fb.y < kInf) && (fb.z < kInf))) inf = true;
        nwo = -wi;
        ++bounce;
    }
    wi_out = wi;
    if ((bounce < 500) && !inf && (fp > 0.0f)) {
        pdf_out = fp;
        f_out = fb;
        refl_out = fr;
    } else {
        pdf_out = 1.0f;
        f_out = mk(0.0f, 0.0f, 0.0f);
        refl_out = mk(0.0f, 0.0f, 0.0f);
    }
}

// ONB from a normal (core/onb.cpp:3-16, 29-35): v = n, local y is the normal.
M3 onb_from_normal(V3 v) {
    V3 w = (std::fabs(v.x) > std::fabs(v.y)) ? normalize(mk(v.z, 0.0f, -v.x)) : normalize(mk(0.0f, -v.z, v.y));
    V3 u = cross(v, w);
    return M3{u, v, w};
}

// ---- scene + tree ---------------------------------------------------------------------------
struct Node {
    Box box;
    uint32_t right, first, count;
    bool leaf;
};

struct Scene {
    std::vector<Prim> prims;
    std::vector<Bsdf> bsdfs;
    std::vector<Material> materials;
    V3 background;
    int accel;
    std::vector<Node> nodes;
    std::vector<uint32_t> refs;
    spt_bvh_stats stats;
    bool built = false;
};

struct Ref {
    long id;
    Box box;
    V3 c;
};

// SBVH::splitNode, object-split half (acceleration/sbvh.cpp:58-121, 306-421): for each axis,
// std::sort by centroid (unstable; sbvh_node.h:26-38), prefix/suffix box sweeps and the SAH
// cost 2*1.2 + (A_L/A)*N_L + (A_R/A)*N_R against the leaf cost 1.0*N.  The builder keeps the
// first best split found (axis 0..2, events from N-2 down to 0, strict <).
void split(Scene& sc, std::vector<Ref>& refs, const Box& box, uint32_t depth) {
    const std::size_t n = refs.size();
    uint32_t me = static_cast<uint32_t>(sc.nodes.size());
    sc.nodes.push_back(Node{box, 0, 0, 0, false});
    float best_cost = 1.0f * static_cast<float>(n);
    int best_axis = -1;
    long best_event = -1;
    std::vector<float> left_area(n > 1 ? n - 1 : 0);
    const float node_area = box_area(box);
    for (int axis = 0; axis < 3; ++axis) {
        std::sort(refs.begin(), refs.end(), [axis](const Ref& a, const Ref& b) { return a.c[axis] < b.c[axis]; });
        Box acc{};
        for (std::size_t i = 0; i + 1 < n; ++i) {
            acc = (i == 0) ? refs[0].box : box_union(acc, refs[i].box);
            left_area[i] = box_area(acc);
        }
        Box racc{};
        for (long i = static_cast<long>(n) - 2; i >= 0; --i) {
            racc = (i == static_cast<long>(n) - 2) ? refs[i + 1].box : box_union(racc, refs[i + 1].box);
            float ra = box_area(racc);
            // SBVH::SAH (sbvh.cpp:47-56), with its float evaluation order.
            float cost = 2.0f * 1.2f + ((left_area[i] / node_area) * static_cast<float>(i + 1) * 1.0f) +
                         ((ra / node_area) * static_cast<float>(n - 1 - i) * 1.0f);
            if (cost < best_cost) {
                best_cost = cost;
                best_event = i;
                best_axis = axis;
            }
        }
    }
    if (best_axis == -1) {
        Node& nd = sc.nodes[me];
        nd.leaf = true;
        nd.first = static_cast<uint32_t>(sc.refs.size());
        nd.count = static_cast<uint32_t>(n);
        for (const Ref& r : refs) sc.refs.push_back(static_cast<uint32_t>(r.id));
        return;
    }
    std::sort(refs.begin(), refs.end(), [best_axis](const Ref& a, const Ref& b) { return a.c[best_axis] < b.c[best_axis]; });
    std::vector<Ref> lr(refs.begin(), refs.begin() + best_event + 1);
    std::vector<Ref> rr(refs.begin() + best_event + 1, refs.end());
    refs.clear();
    refs.shrink_to_fit();
    Box lb = lr[0].box, rb = rr[0].box;
    for (std::size_t i = 1; i < lr.size(); ++i) lb = box_union(lb, lr[i].box);
    for (std::size_t i = 1; i < rr.size(); ++i) rb = box_union(rb, rr[i].box);
    lb = Box{lb.mn - 1e-3f, lb.mx + 1e-3f};  // sbvh.cpp:409-412
    rb = Box{rb.mn - 1e-3f, rb.mx + 1e-3f};
    split(sc, lr, lb, depth + 1);
    sc.nodes[me].right = static_cast<uint32_t>(sc.nodes.size());
    split(sc, rr, rb, depth + 1);
}

// SBVH::collectTreeStatistics (sbvh.cpp:517-575), by a level-order walk.
void collect_stats(Scene& sc) {
    spt_bvh_stats& s = sc.stats;
    std::memset(&s, 0, sizeof(s));
    s.min_prims_leaf = std::numeric_limits<uint64_t>::max();
    std::vector<uint32_t> seen(sc.prims.size(), 0);
    std::vector<uint32_t> level{0}, next;
    uint64_t levels = 0;
    while (!level.empty()) {
        ++levels;
        next.clear();
        for (uint32_t i : level) {
            const Node& nd = sc.nodes[i];
            ++s.num_nodes;
            if (nd.leaf) {
                ++s.num_leaf_nodes;
                s.num_references += nd.count;
                s.min_prims_leaf = std::min<uint64_t>(s.min_prims_leaf, nd.count);
                s.max_prims_leaf = std::max<uint64_t>(s.max_prims_leaf, nd.count);
                for (uint32_t k = 0; k < nd.count; ++k) ++seen[sc.refs[nd.first + k]];
            } else {
                ++s.num_inner_nodes;
                next.push_back(i + 1);
                next.push_back(nd.right);
            }
        }
        level.swap(next);
    }
    s.tree_height = levels ? levels - 1 : 0;
    for (uint32_t c : seen)
        if (!c) ++s.num_unreferenced;
}

// SBVH::intersect / traverse (sbvh.cpp:39-45, 478-510), the default (!NO_LEAF_TRI_BOX) branch:
// depth-first, left before right, no ordering or pruning; counts every box and primitive test.
bool trace_ref(const Scene& sc, V3 o, V3 d, Rec& best, uint32_t& tests, uint32_t& hits) {
    best.t = kInf;
    tests = hits = 0;
    bool found = false;
    if (sc.accel == SPT_ACCEL_NONE) {  // no_accel_structure.cpp:9-30
        for (std::size_t i = 0; i < sc.prims.size(); ++i) {
            ++tests;
            Rec tmp;
            if (prim_hit(sc.prims[i], o, d, tmp)) {
                ++hits;
                if ((tmp.t < best.t) && (tmp.t > 0.0f)) {
                    tmp.prim = static_cast<uint32_t>(i);
                    best = tmp;
                    found = true;
                }
            }
        }
        return found;
    }
    if (sc.nodes.empty()) return false;
    uint32_t stack[1024];  // tree height is checked against this at build time
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
        const Node& nd = sc.nodes[stack[--sp]];
        ++tests;
        if (!box_hit(nd.box, o, d)) continue;
        ++hits;
        if (nd.leaf) {
            for (uint32_t k = 0; k < nd.count; ++k) {
                ++tests;
                uint32_t pid = sc.refs[nd.first + k];
                Rec tmp;
                if (prim_hit(sc.prims[pid], o, d, tmp)) {
                    ++hits;
                    if ((tmp.t > 0.0f) && (tmp.t < best.t) && box_inside(nd.box, tmp.pos)) {
                        tmp.prim = pid;
                        best = tmp;
                        found = true;
                    }
                }
            }
        } else {
            uint32_t self = static_cast<uint32_t>(&nd - sc.nodes.data());
            stack[sp++] = nd.right;  // visited after the whole left subtree
            stack[sp++] = self + 1;
        }
    }
    return found;
}

// ---- cameras (cameras/*.cpp) -------------------------------------------------------------------
struct Cam {
    int type;
    V3 pos;
    M3 l2w;
    V3 luc;           // local upper-left corner
    float pdx, pdy;   // orthographic pixel deltas
    V3 ortho_dir;
};

Cam make_cam(const spt_camera* c) {
    Cam k;
    k.type = c->type;
    k.pos = ld3(c->position);
    V3 dir = normalize(ld3(c->look_at) - k.pos);                 // camera.cpp:9
    V3 u = normalize(cross(ld3(c->up), -dir));                   // camera.cpp:10
    V3 w = -dir;
    V3 v = cross(w, u);                                          // onb.cpp:18-27
    k.l2w = M3{u, v, w};
    if (c->type == SPT_CAMERA_PINHOLE) {                         // pinhole_camera.cpp:3-12
        float a = c->width * 0.5f;
        double b = c->height * 0.5;
        float ang = c->fov_deg * 0.5f * kPi / 180.0f;            // DEG_TO_RAD expands unparenthesised
        float vpd = static_cast<float>(b / std::tan(static_cast<double>(ang)));
        k.luc = mk(-a, static_cast<float>(b), -vpd);
    } else {                                                     // orthographic_camera.cpp:5-19
        float ww = c->max_x - c->min_x, wh = c->max_y - c->min_y;
        k.luc = mk(c->min_x, c->max_y, 0.0f);
        k.pdx = ww / c->width;
        k.pdy = wh / c->height;
        k.ortho_dir = mul(k.l2w, mk(0.0f, 0.0f, -1.0f));
    }
    return k;
}

inline void cam_ray(const Cam& k, float x, float y, V3& o, V3& d) {
    if (k.type == SPT_CAMERA_PINHOLE) {                          // pinhole_camera.cpp:14-18
        V3 ld = normalize(k.luc + mk(x, -y, 0.0f));
        d = mul(k.l2w, ld);
        o = k.pos;
    } else {                                                     // orthographic_camera.cpp:21-25
        V3 lo = k.luc + mk(x * k.pdx, y * -k.pdy, 0.0f);
        o = mul(k.l2w, lo) + k.pos;
        d = k.ortho_dir;
    }
}

}  // namespace

extern "C" {

void spto_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) { philox(ctr, key, out); }

void* spto_scene_create(const spt_scene_desc* d) {
    auto sc = std::make_unique<Scene>();
    sc->prims.resize(d->n_prims);
    for (uint32_t i = 0; i < d->n_prims; ++i) {
        Prim& p = sc->prims[i];
        const float* q = d->prim_data + 9ull * i;
        p.type = d->prim_type[i];
        p.material = d->prim_material[i];
        p.v0 = ld3(q);
        p.v1 = ld3(q + 3);
        p.v2 = ld3(q + 6);
        p.radius = q[3];
        if (p.type == SPT_PRIM_SMOOTH_TRIANGLE) {
            const float* nq = d->prim_normals + 9ull * i;
            p.n0 = ld3(nq);
            p.n1 = ld3(nq + 3);
            p.n2 = ld3(nq + 6);
        }
        if (p.type != SPT_PRIM_SPHERE) p.face_normal = normalize(cross(p.v1 - p.v0, p.v2 - p.v0));
    }
    for (uint32_t i = 0; i < d->n_bsdfs; ++i) {
        const spt_bsdf& b = d->bsdfs[i];
        Bsdf o;
        o.type = b.type;
        o.sampler = b.sampler;
        o.rgb = ld3(b.rgb);
        o.scalar = b.scalar;
        o.brdf = o.rgb / kPi;
        sc->bsdfs.push_back(o);
    }
    for (uint32_t i = 0; i < d->n_materials; ++i) {
        Material m;
        uint32_t l = d->materials[i].layered_bsdf;
        for (uint32_t k = d->layered_offsets[l]; k < d->layered_offsets[l + 1]; ++k)
            m.layers.push_back(static_cast<int>(d->layered_bsdf_ids[k]));
        m.emission = ld3(d->materials[i].emission);
        sc->materials.push_back(m);
    }
    sc->background = ld3(d->background);
    sc->accel = d->accel;
    return sc.release();
}

void spto_scene_destroy(void* s) { delete static_cast<Scene*>(s); }

int spto_bvh_build(void* s) {
    Scene& sc = *static_cast<Scene*>(s);
    sc.nodes.clear();
    sc.refs.clear();
    if (sc.prims.empty() || sc.accel == SPT_ACCEL_NONE) return 0;
    auto t0 = std::chrono::steady_clock::now();
    std::vector<Ref> refs;
    refs.reserve(sc.prims.size());
    Box root{};
    for (std::size_t i = 0; i < sc.prims.size(); ++i) {  // sbvh.cpp:17-24
        Ref r{static_cast<long>(i), prim_box(sc.prims[i]), prim_centroid(sc.prims[i])};
        root = (i == 0) ? r.box : box_union(root, r.box);
        refs.push_back(r);
    }
    split(sc, refs, root, 0);
    collect_stats(sc);
    if (sc.stats.tree_height >= 1000) return 2;
    sc.stats.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    sc.built = true;
    return 0;
}

int spto_tree_stats(void* s, spt_bvh_stats* out) {
    Scene& sc = *static_cast<Scene*>(s);
    if (!sc.built) return 1;
    *out = sc.stats;
    return 0;
}

int spto_tree_export(void* s, spt_bvh2_node* nodes, uint64_t* n_nodes, uint32_t* refs, uint64_t* n_refs) {
    Scene& sc = *static_cast<Scene*>(s);
    *n_nodes = sc.nodes.size();
    *n_refs = sc.refs.size();
    if (nodes)
        for (std::size_t i = 0; i < sc.nodes.size(); ++i) {
            const Node& nd = sc.nodes[i];
            spt_bvh2_node& o = nodes[i];
            o.min[0] = nd.box.mn.x; o.min[1] = nd.box.mn.y; o.min[2] = nd.box.mn.z;
            o.max[0] = nd.box.mx.x; o.max[1] = nd.box.mx.y; o.max[2] = nd.box.mx.z;
            o.right = nd.leaf ? nd.first : nd.right;
            o.count = nd.leaf ? nd.count : 0;
        }
    if (refs) std::memcpy(refs, sc.refs.data(), sc.refs.size() * sizeof(uint32_t));
    return 0;
}

int spto_intersect(void* s, const float* rays, uint64_t n, spt_hit* hits, float* normals, uint32_t* tests,
                   uint32_t* nhits, int n_threads) {
    const Scene& sc = *static_cast<Scene*>(s);
    int nt = n_threads > 0 ? n_threads : omp_get_num_procs();
#pragma omp parallel for schedule(dynamic, 1024) num_threads(nt)
    for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
        const float* r = rays + 8 * i;
        Rec rec;
        uint32_t t_, h_;
        bool hit = trace_ref(sc, ld3(r), ld3(r + 4), rec, t_, h_);
        if (hits) {
            hits[i].t = hit ? rec.t : kInf;
            hits[i].prim_id = hit ? rec.prim : SPT_MISS;
            hits[i].u = hits[i].v = 0.0f;
        }
        if (normals) {
            normals[3 * i] = hit ? rec.normal.x : 0.0f;
            normals[3 * i + 1] = hit ? rec.normal.y : 0.0f;
            normals[3 * i + 2] = hit ? rec.normal.z : 0.0f;
        }
        if (tests) tests[i] = t_;
        if (nhits) nhits[i] = h_;
    }
    return 0;
}

int spto_camera_rays(const spt_camera* c, float* rays) {
    Cam k = make_cam(c);
    for (uint32_t y = 0; y < c->height; ++y)
        for (uint32_t x = 0; x < c->width; ++x) {
            V3 o, d;
            cam_ray(k, x + 0.5f, y + 0.5f, o, d);
            float* q = rays + 8ull * (static_cast<uint64_t>(y) * c->width + x);
            q[0] = o.x; q[1] = o.y; q[2] = o.z; q[3] = 0.0f;
            q[4] = d.x; q[5] = d.y; q[6] = d.z; q[7] = 0.0f;
        }
    return 0;
}

int spto_raycast(void* s, const spt_camera* c, int32_t mode, void* out, spt_render_stats* stats, int n_threads) {
    const Scene& sc = *static_cast<Scene*>(s);
    Cam k = make_cam(c);
    const uint32_t W = c->width, H = c->height;
    std::vector<uint32_t> tests(static_cast<std::size_t>(W) * H), nh(tests.size());
    int nt = n_threads > 0 ? n_threads : omp_get_num_procs();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int64_t y = 0; y < H; ++y)
        for (uint32_t x = 0; x < W; ++x) {
            V3 o, d;
            cam_ray(k, x + 0.5f, static_cast<uint32_t>(y) + 0.5f, o, d);
            Rec rec;
            uint32_t t_, h_;
            bool hit = trace_ref(sc, o, d, rec, t_, h_);
            std::size_t idx = static_cast<std::size_t>(y) * W + x;
            tests[idx] = t_;
            nh[idx] = h_;
            if (mode == SPT_RAYCAST_NORMAL) {  // normal_raycaster.cpp:19-31
                float* q = static_cast<float*>(out) + 3 * idx;
                q[0] = hit ? rec.normal.x : 0.0f;
                q[1] = hit ? rec.normal.y : 0.0f;
                q[2] = hit ? rec.normal.z : 0.0f;
            } else if (mode == SPT_RAYCAST_DEPTH) {  // depth_raycaster.cpp:36-48
                static_cast<float*>(out)[idx] = hit ? rec.t : -1.0f;
            } else {  // int_test_count_raycaster.cpp:75-85
                static_cast<int64_t*>(out)[idx] = t_;
            }
        }
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->min_tests_pp = stats->min_hits_pp = std::numeric_limits<uint64_t>::max();
        for (std::size_t i = 0; i < tests.size(); ++i) {
            stats->int_tests += tests[i];
            stats->int_hits += nh[i];
            stats->min_tests_pp = std::min<uint64_t>(stats->min_tests_pp, tests[i]);
            stats->max_tests_pp = std::max<uint64_t>(stats->max_tests_pp, tests[i]);
            stats->min_hits_pp = std::min<uint64_t>(stats->min_hits_pp, nh[i]);
            stats->max_hits_pp = std::max<uint64_t>(stats->max_hits_pp, nh[i]);
        }
        stats->paths = tests.size();
        stats->segments = tests.size();
    }
    return 0;
}

// Path tracer: the recursion of PathTracer::traceRay (integrators/pathtracer.cpp:12-57) as a loop
// with a path throughput, drawing from Philox streams keyed by (seed) with counter (path index,
// stream, block): stream 0 = the pixel sample, stream depth+1 = the BSDF walk and roulette at
// that depth.  Path index = (spp_offset + s) * viewport_pixels + viewport pixel index.
int spto_pathtrace(void* s, const spt_camera* c, const spt_pt_params* p, float* out, int n_threads, double* seconds,
                   uint64_t* segments) {
    const Scene& sc = *static_cast<Scene*>(s);
    Cam k = make_cam(c);
    const uint32_t W = c->width, H = c->height;
    std::memset(out, 0, sizeof(float) * 3ull * W * H);
    // pixel samplers: regular/jittered round spp up to a square (regular_pixel_sampler.cpp:4-7)
    uint32_t spp = p->spp, nsub = 1;
    float sw = 1.0f;
    if (p->pixel_sampler != SPT_PIXEL_UNIFORM) {
        nsub = static_cast<uint32_t>(std::ceil(std::sqrt(static_cast<double>(p->spp))));
        spp = nsub * nsub;
        sw = 1.0f / nsub;
    }
    const uint64_t npix = static_cast<uint64_t>(c->vp_width) * c->vp_height;
    const int cap = p->max_depth > 0 ? p->max_depth - 1 : 1000;
    const bool rr = p->termination == SPT_TERMINATE_RUSSIAN_ROULETTE;
    int nt = n_threads > 0 ? n_threads : omp_get_num_procs();
    uint64_t seg_total = 0;
    auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt) reduction(+ : seg_total)
    for (int64_t yy = 0; yy < static_cast<int64_t>(c->vp_height); ++yy)
        for (uint32_t xx = 0; xx < c->vp_width; ++xx) {
            const uint32_t x = c->vp_left + xx, y = c->vp_top + static_cast<uint32_t>(yy);
            const uint64_t pix = static_cast<uint64_t>(yy) * c->vp_width + xx;
            V3 acc = mk(0.0f, 0.0f, 0.0f);
            for (uint32_t si = 0; si < spp; ++si) {
                const uint64_t path = static_cast<uint64_t>(p->spp_offset + si) * npix + pix;
                Stream cs(p->seed, path, 0);
                float sx, sy;
                if (p->pixel_sampler == SPT_PIXEL_UNIFORM) {  // uniform_pixel_sampler.cpp:7-10
                    sx = cs.next();
                    sy = cs.next();
                } else {
                    const uint32_t i = si / nsub, j = si % nsub;
                    if (p->pixel_sampler == SPT_PIXEL_REGULAR) {  // regular_pixel_sampler.cpp:10-13
                        float off = sw * 0.5f;
                        sx = sw * i + off;
                        sy = sw * j + off;
                    } else {  // jittered_pixel_sampler.cpp:11-20
                        float u0 = cs.next(), u1 = cs.next();
                        sx = sw * i + sw * u0;
                        sy = sw * j + sw * u1;
                    }
                }
                V3 o, d;
                cam_ray(k, x + sx, y + sy, o, d);
                V3 L = mk(0.0f, 0.0f, 0.0f), beta = mk(1.0f, 1.0f, 1.0f);
                for (int depth = 0;; ++depth) {
                    if (!rr && depth >= p->path_length) break;  // pathtracer.cpp:18-19
                    Rec rec;
                    uint32_t t_, h_;
                    ++seg_total;
                    if (!trace_ref(sc, o, d, rec, t_, h_)) {     // pathtracer.cpp:21-26
                        if (depth == 0) L = L + beta * sc.background;
                        break;
                    }
                    const Material& m = sc.materials[rec.material];
                    M3 frame = onb_from_normal(rec.normal);    // pathtracer.cpp:28-30
                    V3 wo = normalize(mul(transpose(frame), -d));
                    Stream bs(p->seed, path, static_cast<uint32_t>(depth) + 1u);
                    V3 f, refl, wi;
                    float pdf;
                    eval_layered(sc.bsdfs, m, wo, bs, f, refl, pdf, wi);
                    V3 wwi = mul(frame, wi);                     // pathtracer.cpp:37-38
                    V3 no = rec.pos + wwi * 1e-3f;
                    L = L + beta * m.emission;
                    float kk = std::max(std::max(refl.x, refl.y), refl.z);
                    if (rr && depth >= p->path_length) {           // pathtracer.cpp:43-49
                        if ((bs.next() < kk) && (depth < cap)) f = f / kk;
                        else break;
                    } else if (rr && depth >= cap) {
                        break;
                    }
                    beta = ((beta * f) * wi.y) / pdf;              // pathtracer.cpp:52-54
                    if (beta.x == 0.0f && beta.y == 0.0f && beta.z == 0.0f) break;
                    o = no;
                    d = wwi;
                }
                acc = acc + L;
            }
            float* q = out + 3ull * (static_cast<uint64_t>(y) * W + x);
            V3 mean = acc / static_cast<float>(spp);                 // pathtracer.cpp:120-121
            q[0] = mean.x; q[1] = mean.y; q[2] = mean.z;
        }
    if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (segments) *segments = seg_total;
    return 0;
}

int spto_eval_material(void* s, uint32_t material, const float* wo, uint64_t n, float* out, uint64_t seed,
                       uint64_t path_index0, uint32_t depth) {
    const Scene& sc = *static_cast<Scene*>(s);
    const Material& m = sc.materials[material];
    for (uint64_t i = 0; i < n; ++i) {
        Stream bs(seed, path_index0 + i, depth + 1u);
        V3 f, refl, wi;
        float pdf;
        eval_layered(sc.bsdfs, m, ld3(wo + 3 * i), bs, f, refl, pdf, wi);
        float* q = out + 10 * i;
        q[0] = f.x; q[1] = f.y; q[2] = f.z;
        q[3] = refl.x; q[4] = refl.y; q[5] = refl.z;
        q[6] = pdf;
        q[7] = wi.x; q[8] = wi.y; q[9] = wi.z;
    }
    return 0;
}

// DepthRayCaster::saveImageToFile (integrators/depth_raycaster.cpp:9-34); min_d / max_d = -1 means
// "take it from the image" as the reference's prescribed_*_depth_ does.
int spto_depth_to_rgb(const float* depth, uint32_t w, uint32_t h, float min_d, float max_d, float* rgb) {
    float mn = kInf, mx = -kInf;
    const std::size_t n = static_cast<std::size_t>(w) * h;
    for (std::size_t i = 0; i < n; ++i) {
        mx = (mx < depth[i]) ? depth[i] : mx;
        mn = ((depth[i] > 0.0f) && (mn > depth[i])) ? depth[i] : mn;
    }
    mn = (min_d != -1.0f) ? min_d : mn;
    mx = (max_d != -1.0f) ? max_d : mx;
    float range = mx - mn;
    for (std::size_t i = 0; i < n; ++i) {
        float v;
        if (depth[i] != -1.0f) v = range != 0.0f ? (depth[i] - mn) / range : 1.0f;
        else v = 0.0f;
        rgb[3 * i] = rgb[3 * i + 1] = rgb[3 * i + 2] = v;
    }
    return 0;
}

static float hue2rgb(float v1, float v2, float hh) {  // int_test_count_raycaster.cpp:10-18
    if (hh < 0.0f) hh += 1.0f;
    if (hh > 1.0f) hh -= 1.0f;
    if ((6.0f * hh) < 1.0f) return v1 + (v2 - v1) * 6.0f * hh;
    if ((2.0f * hh) < 1.0f) return v2;
    if ((3.0f * hh) < 2.0f) return v1 + (v2 - v1) * ((2.0f / 3.0f) - hh) * 6.0f;
    return v1;
}

// IntTestCountRayCaster::saveImageToFile (int_test_count_raycaster.cpp:20-73).
int spto_count_to_rgb(const int64_t* count, uint32_t w, uint32_t h, int64_t min_c, int64_t max_c, uint64_t min_pp,
                      uint64_t max_pp, float* rgb) {
    std::size_t mnpp = (min_c != -1) ? static_cast<std::size_t>(min_c) : min_pp;
    std::size_t mxpp = (max_c != -1) ? static_cast<std::size_t>(max_c) : max_pp;
    unsigned int range = static_cast<unsigned int>(mxpp - mnpp);
    const std::size_t n = static_cast<std::size_t>(w) * h;
    for (std::size_t i = 0; i < n; ++i) {
        float t;
        if (range > 0) t = (static_cast<std::size_t>(count[i]) - mnpp) / static_cast<float>(range);
        else if (mxpp > 0) t = 1.0f;
        else t = 0.0f;
        float hsl0 = 0.65f - (t * 0.65f), hsl1 = 1.0f, hsl2 = t * 0.5f;
        float v2 = (hsl2 < 0.5f) ? hsl2 * (1.0f + hsl1) : (hsl2 + hsl1) - (hsl1 * hsl2);
        float v1 = 2.0f * hsl2 - v2;
        rgb[3 * i] = hue2rgb(v1, v2, hsl0 + (1.0f / 3.0f));
        rgb[3 * i + 1] = hue2rgb(v1, v2, hsl0);
        rgb[3 * i + 2] = hue2rgb(v1, v2, hsl0 - (1.0f / 3.0f));
    }
    return 0;
}

}  // extern "C"
