// spt_device.cuh -- device-side scene layout and the per-ray / per-sample math of the backend.
//
// The whole library is compiled with --fmad=false, IEEE division and square root and no
// flush-to-zero, so every expression below rounds exactly like the reference's FMA-free
// single-precision C++ (glm operation order: dot sums left to right, normalize = v * (1/sqrt(dot)),
// column-major mat3 * v sums the columns left to right).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/spt.h"

namespace spt {

// ---------------------------------------------------------------------------------------------
// Device scene layout (all arrays in HBM, built by scene.cu)
//
//   tri[3*slot .. 3*slot+2]   one 48-byte record per leaf reference, in depth-first leaf order
//                             (the reference's traversal order, used to break equal-t ties):
//                               triangle: {v0, prim id} {e1 = v1 - v0, leaf id} {e2 = v2 - v0, type}
//                               sphere:   {centre, prim id} {radius, 0, 0, leaf id} {0, 0, 0, type}
//   pair[4*i .. 4*i+3]        one 64-byte record per inner node i (pre-order ordinal): both
//                             children's boxes + child refs (>= 0 inner ordinal, < 0 ~leaf id)
//   leaf[l]                   {first slot, count} of leaf l; leaf_box[l] its box (inside test)
//   node2[]                   the flattened binary tree (spt_bvh2_node), for the exhaustive
//                             reference-order traversal that counts tests
// ---------------------------------------------------------------------------------------------
struct DevBsdf {
    int type, sampler;
    float r, g, b;        // kd or F0
    float scalar;         // ior or roughness
    float br, bg, bb;     // Lambertian kd / PI (lambertian.cpp:6)
    float pad;
};

struct DevMaterial {
    int layer_begin, layer_count;
    float er, eg, eb;
    float pad;
};

struct DevScene {
    const float4* tri;
    const float4* pair;
    const int2* leaf;
    const float* leaf_box;      // 6 floats per leaf
    const spt_bvh2_node* node2;
    const float4* face_normal;  // per primitive (flat triangles)
    const float4* smooth_normal;  // 3 per primitive, or null
    const uint32_t* prim_mat;
    const uint8_t* prim_type;
    const DevBsdf* bsdf;
    const DevMaterial* mat;
    const int* layer_ids;
    const uint4* wnode;         // 8-wide quantized nodes, 5 x uint4 each (wide_build.h)
    const float4* wtri;         // 3 float4 per triangle in wide-node order: {v0, rank}{e1, type}{e2, leaf}
    float root_min[3], root_max[3];
    float bg[3];
    uint32_t n_prims, n_inner, n_leaves, n_nodes2, n_wnodes;
    int root_is_leaf;           // the whole scene is one leaf (or no acceleration structure)
    int no_accel;               // NoAccelStructure semantics (no_accel_structure.cpp:9-30)
    int has_spheres;
    int empty;
    int traversal;              // 0: binary pair nodes, 1: 8-wide quantized nodes, 2: 1 + dynamic fetch
};

// Camera constants computed on the host exactly as the reference constructors do.
struct DevCamera {
    int type;
    float pos[3];
    float l2w[9];        // column-major: columns u, v, w
    float luc[3];        // local upper-left corner
    float pdx, pdy;      // orthographic pixel size
    float odir[3];       // orthographic world direction
    uint32_t width, height;
    uint32_t vp_top, vp_left, vp_width, vp_height;
};

const float kPi = 3.141592653589793238462643383279502884f;

struct V3 {
    float x, y, z;
};
__host__ __device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__host__ __device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__host__ __device__ __forceinline__ V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ V3 operator*(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
__host__ __device__ __forceinline__ V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
__host__ __device__ __forceinline__ V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
__host__ __device__ __forceinline__ float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__host__ __device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
__host__ __device__ __forceinline__ V3 normalize(V3 v) { return v * (1.0f / sqrtf(dot(v, v))); }
__host__ __device__ __forceinline__ V3 mat_mul(const float* m, V3 v) {  // column-major, glm order
    return v3(m[0] * v.x + m[3] * v.y + m[6] * v.z, m[1] * v.x + m[4] * v.y + m[7] * v.z,
              m[2] * v.x + m[5] * v.y + m[8] * v.z);
}
__host__ __device__ __forceinline__ V3 mat_tmul(const float* m, V3 v) {  // transpose(m) * v
    return v3(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
              m[6] * v.x + m[7] * v.y + m[8] * v.z);
}
__device__ __forceinline__ V3 f3v(float4 a) { return v3(a.x, a.y, a.z); }

// ---- ray / box: the reference's Williams slab test (acceleration/aabb.cpp:31-99) -------------
// The per-axis branch on the sign of 1/d is taken once per ray (near/far plane selection is the
// same choice the reference makes per box).  Returns the reference's pass/fail; tmin/tmax, the
// fully combined interval, are used only to order and prune the traversal.
struct RayInv {
    V3 o, inv;
    bool sx, sy, sz;
};
__device__ __forceinline__ RayInv ray_inv(V3 o, V3 d) {
    RayInv r;
    r.o = o;
    r.inv = v3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    r.sx = r.inv.x >= 0.0f;
    r.sy = r.inv.y >= 0.0f;
    r.sz = r.inv.z >= 0.0f;
    return r;
}
__device__ __forceinline__ bool slab(const RayInv& r, float nx, float ny, float nz, float xx, float xy, float xz,
                                     float& tmin_out, float& tmax_out) {
    float tmin = ((r.sx ? nx : xx) - r.o.x) * r.inv.x;
    float tmax = ((r.sx ? xx : nx) - r.o.x) * r.inv.x;
    float tymin = ((r.sy ? ny : xy) - r.o.y) * r.inv.y;
    float tymax = ((r.sy ? xy : ny) - r.o.y) * r.inv.y;
    if ((tmin > tymax) || (tymin > tmax)) return false;
    if (tymin > tmin) tmin = tymin;
    if (tymax < tmax) tmax = tymax;
    float tzmin = ((r.sz ? nz : xz) - r.o.z) * r.inv.z;
    float tzmax = ((r.sz ? xz : nz) - r.o.z) * r.inv.z;
    if ((tmin > tzmax) || (tzmin > tmax)) return false;
    if (tzmin > tmin) tmin = tzmin;
    if (tzmax < tmax) tmax = tzmax;
    tmin_out = tmin;
    tmax_out = tmax;
    return true;
}
// AABB::isPointInside, epsilon 1e-3 (aabb.cpp:3, 101-105)
__device__ __forceinline__ bool inside(const float* b, V3 p) {
    const float e = 1e-3f;
    return (p.x >= (b[0] - e)) && (p.x <= (b[3] + e)) && (p.y >= (b[1] - e)) && (p.y <= (b[4] + e)) &&
           (p.z >= (b[2] - e)) && (p.z <= (b[5] + e));
}

// ---- primitives ------------------------------------------------------------------------------
// Moller-Trumbore, non-culling (primitives/triangle.cpp:12-74); e1, e2 precomputed on the host
// with the same subtraction the reference does per test.
__device__ __forceinline__ bool tri_test(V3 v0, V3 e1, V3 e2, V3 o, V3 d, float& t, float& u, float& v) {
    V3 pvec = cross(d, e2);
    float det = dot(e1, pvec);
    if ((det > -1e-6f) && (det < 1e-6f)) return false;
    float inv_det = 1.0f / det;
    V3 tvec = o - v0;
    u = dot(tvec, pvec) * inv_det;
    if ((u < 0.0f) || (u > 1.0f)) return false;
    V3 qvec = cross(tvec, e1);
    v = dot(d, qvec) * inv_det;
    if ((v < 0.0f) || ((u + v) > 1.0f)) return false;
    t = dot(e2, qvec) * inv_det;
    return true;
}
// Hultquist ray-sphere (primitives/sphere.cpp:6-38)
__device__ __forceinline__ bool sphere_test(V3 c, float radius, V3 o, V3 d, float& t) {
    V3 eo = c - o;
    float v = dot(eo, d);
    float disc = (radius * radius) - (dot(eo, eo) - (v * v));
    if (disc < 0.0f) return false;
    float dd = sqrtf(disc);
    float t1 = v - dd, t2 = v + dd;
    t = (t1 > 1e-5f) ? t1 : t2;
    return true;
}
// Hit position as each primitive's intersect writes it (triangle.cpp:69, sphere.cpp:33).
__device__ __forceinline__ V3 hit_pos(bool sphere, V3 o, V3 d, float t) { return sphere ? o + t * d : o + d * t; }

// Shading normal at a hit (triangle.h:17-21, smooth_triangle.h:11-13, sphere.cpp:34).
__device__ __forceinline__ V3 hit_normal(const DevScene& S, uint32_t prim, float u, float v, V3 pos) {
    const uint8_t ty = S.prim_type[prim];
    if (ty == SPT_PRIM_SPHERE) {
        // centre is stored in the face-normal slot for spheres
        float4 c = S.face_normal[prim];
        return normalize(pos - f3v(c));
    }
    if (ty == SPT_PRIM_SMOOTH_TRIANGLE) {
        V3 n0 = f3v(S.smooth_normal[3 * prim]), n1 = f3v(S.smooth_normal[3 * prim + 1]);
        V3 n2 = f3v(S.smooth_normal[3 * prim + 2]);
        return normalize(n0 * ((1.0f - u) - v) + n1 * u + n2 * v);
    }
    return f3v(S.face_normal[prim]);
}

// ---- cameras (cameras/pinhole_camera.cpp:14-18, orthographic_camera.cpp:21-25) -----------------
__device__ __forceinline__ void camera_ray(const DevCamera& c, float x, float y, V3& o, V3& d) {
    if (c.type == SPT_CAMERA_PINHOLE) {
        V3 ld = normalize(v3(c.luc[0] + x, c.luc[1] + (-y), c.luc[2] + 0.0f));
        d = mat_mul(c.l2w, ld);
        o = v3(c.pos[0], c.pos[1], c.pos[2]);
    } else {
        V3 lo = v3(c.luc[0] + x * c.pdx, c.luc[1] + y * -c.pdy, c.luc[2] + 0.0f);
        o = mat_mul(c.l2w, lo) + v3(c.pos[0], c.pos[1], c.pos[2]);
        d = v3(c.odir[0], c.odir[1], c.odir[2]);
    }
}

// ---- Philox-4x32-10 (Salmon et al., SC'11) ------------------------------------------------------
__device__ __forceinline__ uint4 philox(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
    }
    return c;
}

// One sample stream: counter (path index lo, hi, stream id, block); 4 uniforms per block.
struct Stream {
    uint4 ctr;
    uint32_t k0, k1;
    uint4 buf;
    int pos;
    __device__ __forceinline__ Stream(uint64_t seed, uint64_t path, uint32_t sid)
        : ctr(make_uint4(static_cast<uint32_t>(path), static_cast<uint32_t>(path >> 32), sid, 0u)),
          k0(static_cast<uint32_t>(seed)),
          k1(static_cast<uint32_t>(seed >> 32)),
          pos(4) {}
    __device__ __forceinline__ float next() {
        if (pos == 4) {
            buf = philox(ctr, k0, k1);
            ++ctr.w;
            pos = 0;
        }
        uint32_t x = pos == 0 ? buf.x : (pos == 1 ? buf.y : (pos == 2 ? buf.z : buf.w));
        ++pos;
        return static_cast<float>(x >> 8) * (1.0f / 16777216.0f);
    }
};

}  // namespace spt
