// guiding.cuh -- the neural path-guiding model on the device (no reference counterpart).
//
// A multiresolution hash grid encodes the shading position; a 4-hidden-layer ReLU MLP (width 64,
// no biases) maps [grid features, normal, outgoing direction] to a mixture of 8 von Mises-Fisher
// lobes over world directions.  The MLP runs on the tensor cores: mma.sync m16n8k16 with bf16
// operands and fp32 accumulation, one warp per tile of 32 samples, and the output fragments of one
// layer become the A fragments of the next without leaving registers (two adjacent n8 output tiles
// hold exactly the rows/columns of one k16 input step).
#pragma once

#include <cuda_bf16.h>

#include "spt_device.cuh"

namespace spt {
namespace guide {

constexpr int kLevels = 16, kFeat = 2, kLog2T = 19;
constexpr uint32_t kT = 1u << kLog2T;
constexpr int kNMin = 16, kNMax = 1024;
constexpr int kIn = 48, kHid = 64, kOut = 48, kLobes = 8, kOutUsed = 40;
constexpr float kKappaLo = -2.3f, kKappaHi = 7.0f;
// layer l: out x in
__host__ __device__ constexpr int layer_in(int l) { return l == 0 ? kIn : kHid; }
__host__ __device__ constexpr int layer_out(int l) { return l == 4 ? kOut : kHid; }
constexpr int kLayers = 5;
// offsets of each layer's weights in the packed [out][in] parameter vector
__host__ __device__ constexpr int w_offset(int l) {
    return l == 0 ? 0 : w_offset(l - 1) + layer_out(l - 1) * layer_in(l - 1);
}
constexpr int kMlpParams = w_offset(kLayers);  // 18432
constexpr uint64_t kGridParams = static_cast<uint64_t>(kLevels) * kT * kFeat;

// smem row strides (bf16 elements): +8 keeps fragment loads free of bank conflicts
__host__ __device__ constexpr int pad(int k) { return k + 8; }
// packed smem image: every layer's W [out][pad(in)] first (all that inference stages), then every
// layer's W^T [in][pad(out)] (the backward pass)
__host__ __device__ constexpr int sw_offset(int l) {
    return l == 0 ? 0 : sw_offset(l - 1) + layer_out(l - 1) * pad(layer_in(l - 1));
}
constexpr int kFwdWeights = sw_offset(kLayers);  // bf16 elements of the forward half
__host__ __device__ constexpr int swt_rel(int l) {
    return l == 0 ? 0 : swt_rel(l - 1) + layer_in(l - 1) * pad(layer_out(l - 1));
}
__host__ __device__ constexpr int swt_offset(int l) { return kFwdWeights + swt_rel(l); }
constexpr int kSmemWeights = kFwdWeights + swt_rel(kLayers);  // bf16 elements

struct GridLevel {
    uint32_t res;    // cells per axis
    uint32_t dense;  // 1: index = x + y*(res+1) + z*(res+1)^2, 0: spatial hash
};

struct Model {
    const __nv_bfloat16* grid;   // [L][T][F] bf16 (inference / forward copy)
    const __nv_bfloat16* smem_image;  // kSmemWeights bf16, the layout staged into shared memory
    float lo[3], inv_ext[3];     // scene box used to normalise positions
    GridLevel level[kLevels];
};

__device__ __forceinline__ uint32_t grid_index(const GridLevel& lv, uint32_t x, uint32_t y, uint32_t z) {
    if (lv.dense) {
        const uint32_t n = lv.res + 1;
        return x + y * n + z * n * n;
    }
    return (x * 1u ^ y * 2654435761u ^ z * 805459861u) & (kT - 1u);
}

__device__ __forceinline__ V3 normalised_pos(const Model& M, V3 p) {
    V3 q = v3((p.x - M.lo[0]) * M.inv_ext[0], (p.y - M.lo[1]) * M.inv_ext[1], (p.z - M.lo[2]) * M.inv_ext[2]);
    // [0, 1): a corner index never passes the last grid point of a dense level
    const float hi = 0.99999994f;
    q.x = fminf(fmaxf(q.x, 0.0f), hi);
    q.y = fminf(fmaxf(q.y, 0.0f), hi);
    q.z = fminf(fmaxf(q.z, 0.0f), hi);
    return q;
}

// Corner c of level l: index and trilinear weight.
struct Corner {
    uint32_t idx;
    float w;
};
__device__ __forceinline__ Corner grid_corner(const GridLevel& lv, V3 q, int c) {
    const float px = q.x * lv.res, py = q.y * lv.res, pz = q.z * lv.res;
    const float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
    const float rx = px - fx, ry = py - fy, rz = pz - fz;
    const uint32_t ix = static_cast<uint32_t>(fx) + (c & 1), iy = static_cast<uint32_t>(fy) + ((c >> 1) & 1),
                   iz = static_cast<uint32_t>(fz) + ((c >> 2) & 1);
    Corner k;
    k.idx = grid_index(lv, ix, iy, iz);
    k.w = ((c & 1) ? rx : 1.0f - rx) * ((c & 2) ? ry : 1.0f - ry) * ((c & 4) ? rz : 1.0f - rz);
    return k;
}

// The two features of level l at the normalised position q (trilinear over the 8 cell corners).
__device__ __forceinline__ __nv_bfloat162 encode_level(const Model& M, const GridLevel& lv, V3 q, int l) {
    float a = 0.0f, b = 0.0f;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const Corner k = grid_corner(lv, q, c);
        const __nv_bfloat162 f =
            *reinterpret_cast<const __nv_bfloat162*>(M.grid + (static_cast<uint64_t>(l) * kT + k.idx) * kFeat);
        a = __fmaf_rn(k.w, __bfloat162float(f.x), a);
        b = __fmaf_rn(k.w, __bfloat162float(f.y), b);
    }
    return __floats2bfloat162_rn(a, b);
}

// The 16 network inputs after the grid features: normal, wo, zeros.
__device__ __forceinline__ void direction_inputs(V3 nrm, V3 wo, __nv_bfloat162* row) {
    row[16] = __floats2bfloat162_rn(nrm.x, nrm.y);
    row[17] = __floats2bfloat162_rn(nrm.z, wo.x);
    row[18] = __floats2bfloat162_rn(wo.y, wo.z);
    for (int i = 19; i < kIn / 2; ++i) row[i] = __floats2bfloat162_rn(0.0f, 0.0f);
}

// The 48 network inputs of one sample, as bf16 pairs: 32 grid features, normal, wo, zeros.
__device__ __forceinline__ void encode_inputs(const Model& M, V3 pos, V3 nrm, V3 wo, __nv_bfloat162* row) {
    const V3 q = normalised_pos(M, pos);
#pragma unroll 2
    for (int l = 0; l < kLevels; ++l) row[l] = encode_level(M, M.level[l], q, l);
    direction_inputs(nrm, wo, row);
}

// ---- warp-level MMA --------------------------------------------------------------------------
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

// A fragments of a [16 rows][K] bf16 tile stored row-major in shared memory (row stride ld).
template <int KSTEPS>
__device__ __forceinline__ void load_a(const __nv_bfloat16* tile, int ld, uint32_t (&a)[KSTEPS][4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int s = 0; s < KSTEPS; ++s) {
        const __nv_bfloat16* r0 = tile + g * ld + 16 * s + 2 * t;
        const __nv_bfloat16* r1 = r0 + 8 * ld;
        a[s][0] = *reinterpret_cast<const uint32_t*>(r0);
        a[s][1] = *reinterpret_cast<const uint32_t*>(r1);
        a[s][2] = *reinterpret_cast<const uint32_t*>(r0 + 8);
        a[s][3] = *reinterpret_cast<const uint32_t*>(r1 + 8);
    }
}

// One layer for a 16-row tile: out[n-tile][4] = A * B where B comes from a [N][pad(K)] smem matrix
// (the B column n of k16 step s is row n of that matrix, elements 16s..16s+15).
template <int KSTEPS, int NTILES>
__device__ __forceinline__ void layer_mma(const uint32_t (&a)[KSTEPS][4], const __nv_bfloat16* w, int ldw,
                                          float (&out)[NTILES][4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int j = 0; j < NTILES; ++j) {
        out[j][0] = out[j][1] = out[j][2] = out[j][3] = 0.0f;
        const __nv_bfloat16* row = w + (8 * j + g) * ldw + 2 * t;
#pragma unroll
        for (int s = 0; s < KSTEPS; ++s) {
            const uint32_t b0 = *reinterpret_cast<const uint32_t*>(row + 16 * s);
            const uint32_t b1 = *reinterpret_cast<const uint32_t*>(row + 16 * s + 8);
            mma_bf16(out[j], a[s], b0, b1);
        }
    }
}

// Output tiles of a layer -> A fragments of the next layer (optionally through ReLU).
template <int NTILES>
__device__ __forceinline__ void chain(const float (&d)[NTILES][4], uint32_t (&a)[NTILES / 2][4], bool relu) {
#pragma unroll
    for (int s = 0; s < NTILES / 2; ++s) {
        float v[8];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            v[k] = d[2 * s][k];
            v[4 + k] = d[2 * s + 1][k];
        }
        if (relu)
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = fmaxf(v[k], 0.0f);
        a[s][0] = pack_bf16(v[0], v[1]);
        a[s][1] = pack_bf16(v[2], v[3]);
        a[s][2] = pack_bf16(v[4], v[5]);
        a[s][3] = pack_bf16(v[6], v[7]);
    }
}

// Store output tiles (fp32) of a 16-row tile to a row-major smem tile.
template <int NTILES>
__device__ __forceinline__ void store_tile(const float (&d)[NTILES][4], float* tile, int ld) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int j = 0; j < NTILES; ++j) {
        tile[g * ld + 8 * j + 2 * t] = d[j][0];
        tile[g * ld + 8 * j + 2 * t + 1] = d[j][1];
        tile[(g + 8) * ld + 8 * j + 2 * t] = d[j][2];
        tile[(g + 8) * ld + 8 * j + 2 * t + 1] = d[j][3];
    }
}

// Forward pass of 16 rows whose inputs sit in a bf16 smem tile [16][pad(kIn)]; the 48 outputs land
// in `y` (fp32 smem tile [16][kOut + 4]).  sw: the staged weight image.
__device__ __forceinline__ void forward16(const __nv_bfloat16* sw, const __nv_bfloat16* xin, float* y) {
    uint32_t a0[3][4];
    load_a<3>(xin, pad(kIn), a0);
    float d[8][4];
    layer_mma<3, 8>(a0, sw + sw_offset(0), pad(kIn), d);
    uint32_t a[4][4];
    chain<8>(d, a, true);
    layer_mma<4, 8>(a, sw + sw_offset(1), pad(kHid), d);
    chain<8>(d, a, true);
    layer_mma<4, 8>(a, sw + sw_offset(2), pad(kHid), d);
    chain<8>(d, a, true);
    layer_mma<4, 8>(a, sw + sw_offset(3), pad(kHid), d);
    chain<8>(d, a, true);
    float o[6][4];
    layer_mma<4, 6>(a, sw + sw_offset(4), pad(kHid), o);
    store_tile<6>(o, y, kOut + 4);
}

// ---- the vMF mixture ---------------------------------------------------------------------------
struct Lobe {
    V3 mu;
    float kappa, w;
};

// y: the 40 used outputs of one sample -> 8 lobes (normalised weights).
__device__ __forceinline__ void decode(const float* y, Lobe (&lb)[kLobes]) {
    float mx = -3.0e38f;
    for (int k = 0; k < kLobes; ++k) mx = fmaxf(mx, y[5 * k + 4]);
    float sum = 0.0f;
    for (int k = 0; k < kLobes; ++k) {
        V3 m = v3(y[5 * k], y[5 * k + 1], y[5 * k + 2]);
        const float n = sqrtf(dot(m, m));
        lb[k].mu = n > 1e-12f ? m * (1.0f / n) : v3(0.0f, 1.0f, 0.0f);
        lb[k].kappa = expf(fminf(fmaxf(y[5 * k + 3], kKappaLo), kKappaHi));
        lb[k].w = expf(y[5 * k + 4] - mx);
        sum += lb[k].w;
    }
    for (int k = 0; k < kLobes; ++k) lb[k].w /= sum;
}

__device__ __forceinline__ float vmf_pdf(const Lobe& l, V3 w) {
    const float c = dot(l.mu, w);
    return l.kappa / (2.0f * kPi * (1.0f - expf(-2.0f * l.kappa))) * expf(l.kappa * (c - 1.0f));
}

__device__ __forceinline__ float mixture_pdf(const Lobe (&lb)[kLobes], V3 w) {
    float q = 0.0f;
    for (int k = 0; k < kLobes; ++k) q += lb[k].w * vmf_pdf(lb[k], w);
    return q;
}

// Sample a direction from the mixture with three uniforms (lobe choice, then the vMF sampling of
// W. Jakob, "Numerically stable sampling of the von Mises Fisher distribution on S^2", 2012).
__device__ __forceinline__ V3 mixture_sample(const Lobe (&lb)[kLobes], float u0, float u1, float u2) {
    int k = 0;
    float acc = lb[0].w;
    while (k < kLobes - 1 && u0 >= acc) acc += lb[++k].w;
    const Lobe& l = lb[k];
    // u1 = 0 with e^{-2 kappa} underflowing gives log(0): the cosine's limit there is -1
    const float w = fmaxf(1.0f + logf(u1 + (1.0f - u1) * expf(-2.0f * l.kappa)) / l.kappa, -1.0f);
    const float s = sqrtf(fmaxf(0.0f, 1.0f - w * w));
    const float phi = 2.0f * kPi * u2;
    // frame around mu
    const V3 n = l.mu;
    const V3 a = fabsf(n.x) > 0.9f ? v3(0.0f, 1.0f, 0.0f) : v3(1.0f, 0.0f, 0.0f);
    const V3 t = normalize(cross(a, n));
    const V3 b = cross(n, t);
    return normalize(t * (s * cosf(phi)) + b * (s * sinf(phi)) + n * w);
}

// ---- the lobe cache that guided rendering samples (Guide::refresh_cache) -----------------------
// An entry holds six fields of the 8 lobes, field-major: mu.x[8], mu.y[8], mu.z[8], kappa[8], w[8],
// wc[8] with wc = w * C(kappa) and C(kappa) = kappa / (2 pi (1 - e^{-2 kappa})) the vMF
// normalisation, so the density of a direction costs one exp per lobe.  Field-major, the density
// streams one float4 of each field per four lobes, and sampling reads the weights and then only the
// chosen lobe: guided shading never holds the whole entry in registers.  The mixture is a sampling
// density, not part of the reference's exact ray arithmetic, so it uses the fast exp/log/sincos
// intrinsics and fused multiply-adds; sampling and density use the same ones, so they agree.
constexpr int kCacheLobe = 6;                      // fields per lobe
constexpr int kCacheEntry = kLobes * kCacheLobe;   // 48 floats
enum CacheField { kMuX = 0, kMuY = 1, kMuZ = 2, kKappa = 3, kWeight = 4, kWeightC = 5 };

__device__ __forceinline__ float cached_mixture_pdf(const float* entry, V3 w) {
    const float4* e = reinterpret_cast<const float4*>(entry);
    float q = 0.0f;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const float4 mx = __ldg(e + 2 * kMuX + h), my = __ldg(e + 2 * kMuY + h), mz = __ldg(e + 2 * kMuZ + h);
        const float4 ka = __ldg(e + 2 * kKappa + h), wc = __ldg(e + 2 * kWeightC + h);
        const float c0 = __fmaf_rn(mx.x, w.x, __fmaf_rn(my.x, w.y, __fmul_rn(mz.x, w.z)));
        const float c1 = __fmaf_rn(mx.y, w.x, __fmaf_rn(my.y, w.y, __fmul_rn(mz.y, w.z)));
        const float c2 = __fmaf_rn(mx.z, w.x, __fmaf_rn(my.z, w.y, __fmul_rn(mz.z, w.z)));
        const float c3 = __fmaf_rn(mx.w, w.x, __fmaf_rn(my.w, w.y, __fmul_rn(mz.w, w.z)));
        q = __fmaf_rn(wc.x, __expf(__fmul_rn(ka.x, c0 - 1.0f)), q);
        q = __fmaf_rn(wc.y, __expf(__fmul_rn(ka.y, c1 - 1.0f)), q);
        q = __fmaf_rn(wc.z, __expf(__fmul_rn(ka.z, c2 - 1.0f)), q);
        q = __fmaf_rn(wc.w, __expf(__fmul_rn(ka.w, c3 - 1.0f)), q);
    }
    return q;
}

// A direction from the cached mixture: the first lobe whose cumulative weight exceeds u0 (the last
// one if rounding leaves u0 above the sum), then Jakob's vMF sampler around its mean, in the
// orthonormal basis of Duff et al., "Building an Orthonormal Basis, Revisited" (JCGT 2017).
__device__ __forceinline__ V3 cached_mixture_sample(const float* entry, float u0, float u1, float u2) {
    const float4* e4 = reinterpret_cast<const float4*>(entry);
    const float4 wa = __ldg(e4 + 2 * kWeight), wb = __ldg(e4 + 2 * kWeight + 1);
    const float w8[kLobes] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
    uint32_t k = kLobes - 1;
    float acc = 0.0f;
    bool found = false;
#pragma unroll
    for (int j = 0; j < kLobes - 1; ++j) {
        acc += w8[j];
        const bool take = !found && u0 < acc;
        k = take ? static_cast<uint32_t>(j) : k;
        found = found || take;
    }
    const float mx = __ldg(entry + kLobes * kMuX + k), my = __ldg(entry + kLobes * kMuY + k);
    const float mz = __ldg(entry + kLobes * kMuZ + k), kappa = __ldg(entry + kLobes * kKappa + k);
    // The uniforms include 0: with u1 = 0 and e^{-2 kappa} underflowing (kappa above about 44) the
    // logarithm is -inf, and the cosine takes its limit -1 instead of turning the direction into NaN.
    const float w =
        fmaxf(__fmaf_rn(__logf(__fmaf_rn(1.0f - u1, __expf(-2.0f * kappa), u1)), __frcp_rn(kappa), 1.0f), -1.0f);
    const float s = sqrtf(fmaxf(0.0f, __fmaf_rn(-w, w, 1.0f)));
    float sn, cs;
    __sincosf(2.0f * kPi * u2, &sn, &cs);
    const float sg = copysignf(1.0f, mz);
    const float a = -__frcp_rn(sg + mz), b = mx * my * a;
    const V3 t = v3(__fmaf_rn(sg * mx * mx, a, 1.0f), sg * b, -sg * mx);
    const V3 bt = v3(b, __fmaf_rn(my * my, a, sg), -my);
    const float ts = s * cs, bs = s * sn;
    const V3 r = v3(__fmaf_rn(t.x, ts, __fmaf_rn(bt.x, bs, mx * w)), __fmaf_rn(t.y, ts, __fmaf_rn(bt.y, bs, my * w)),
                    __fmaf_rn(t.z, ts, __fmaf_rn(bt.z, bs, mz * w)));
    return r * rsqrtf(__fmaf_rn(r.x, r.x, __fmaf_rn(r.y, r.y, r.z * r.z)));
}

}  // namespace guide
}  // namespace spt
