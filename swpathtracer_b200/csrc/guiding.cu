// guiding.cu -- training and inference of the path-guiding model (guiding.cuh).
//
//   k_stage        fp32 master weights -> the bf16 shared-memory image (W and W^T of every layer)
//   k_infer        encode + forward + decode for a list of samples (one warp per 32 samples)
//   k_train        encode + forward + vMF-mixture loss + backward through the MLP on the tensor
//                  cores; writes every layer's input X_l and output gradient dZ_l (bf16, transposed:
//                  feature-major, sample-minor) and scatters the hash-grid gradient
//   k_wgrad        dW_l = dZ_l^T X_l on the tensor cores, split over sample chunks (partials)
//   k_reduce       sums the partials in a fixed order (deterministic)
//   k_adam         Adam update of a parameter vector (+ its bf16 copy), clears the gradient
#include <cstring>
#include <memory>
#include <vector>

#include <algorithm>
#include <cmath>

#include "guiding_host.h"

namespace spt {
namespace guide {
namespace {

constexpr int kWarps = 4;            // warps per block in k_train
constexpr int kInferWarps = 16;      // warps per block in k_infer (one block per SM: 200 KB of smem)
constexpr int kTileRows = 32;        // samples per warp tile
constexpr int kYld = kOut + 4;       // fp32 output tile row stride

__global__ void k_stage(const float* __restrict__ w, __nv_bfloat16* __restrict__ img) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kMlpParams) return;
    int l = 0;
    while (l + 1 < kLayers && i >= w_offset(l + 1)) ++l;
    const int r = i - w_offset(l), in = layer_in(l), out = layer_out(l);
    const int o = r / in, k = r % in;
    const __nv_bfloat16 v = __float2bfloat16_rn(w[i]);
    img[sw_offset(l) + o * pad(in) + k] = v;
    img[swt_offset(l) + k * pad(out) + o] = v;
}

// The first `count` bf16 elements of the weight image (a multiple of 8).
__device__ __forceinline__ void stage_weights(const Model& M, __nv_bfloat16* sw, int count) {
    const uint4* src = reinterpret_cast<const uint4*>(M.smem_image);
    uint4* dst = reinterpret_cast<uint4*>(sw);
    for (int i = threadIdx.x; i < count / 8; i += blockDim.x) dst[i] = __ldg(src + i);
    __syncthreads();
}

// ---- inference --------------------------------------------------------------------------------
// k_encode: the hash-grid features of n samples, one thread per (sample, level) so that every SM
// keeps many gathers in flight; feats[16 i + l] = level l's two bf16 features of sample i.
__global__ void __launch_bounds__(256) k_encode(const __grid_constant__ Model M, const float4* __restrict__ in,
                                                uint32_t n_host, const uint32_t* __restrict__ n_dev,
                                                uint32_t* __restrict__ feats) {
    const uint32_t n = n_dev ? *n_dev : n_host;
    const uint64_t total = static_cast<uint64_t>(n) * kLevels;
    for (uint64_t t = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t i = static_cast<uint32_t>(t / kLevels), l = static_cast<uint32_t>(t % kLevels);
        const V3 q = normalised_pos(M, f3v(__ldg(in + 3 * i)));
        const __nv_bfloat162 f = encode_level(M, M.level[l], q, static_cast<int>(l));
        feats[t] = *reinterpret_cast<const uint32_t*>(&f);
    }
}

// in: n samples, 3 float4 each (position, normal, outgoing direction); out: 40 floats per sample
// (8 lobes x {mu.xyz, kappa, weight}), already decoded.
// The network inputs of the guide cache: entry ((iz * R + iy) * R + ix) * 6 + bin is the centre of
// cell (ix, iy, iz) of an R^3 grid over the box, with the normal +x, -x, +y, -y, +z, -z for bin 0..5
// (wo = the normal).
// Network inputs of cache entries first .. first + n - 1 of the list (of the whole cache when list is
// NULL): the cell centre and the axis normal, which also stands in for the view direction.
__global__ void k_cache_inputs(Model M, uint32_t R, const uint32_t* __restrict__ list, uint32_t first, uint32_t n,
                               float4* __restrict__ in) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint32_t e = list ? list[first + j] : first + j;
        const uint32_t bin = e % 6, cell = e / 6;
        const uint32_t ix = cell % R, iy = (cell / R) % R, iz = cell / (R * R);
        const float x = M.lo[0] + (ix + 0.5f) / (R * M.inv_ext[0]);
        const float y = M.lo[1] + (iy + 0.5f) / (R * M.inv_ext[1]);
        const float z = M.lo[2] + (iz + 0.5f) / (R * M.inv_ext[2]);
        const float sgn = (bin & 1u) ? -1.0f : 1.0f;
        const float4 nrm = make_float4(bin < 2 ? sgn : 0.0f, (bin >> 1) == 1 ? sgn : 0.0f, bin >= 4 ? sgn : 0.0f, 0.0f);
        in[3 * j] = make_float4(x, y, z, 0.0f);
        in[3 * j + 1] = nrm;
        in[3 * j + 2] = nrm;
    }
}

// Decoded lobes {mu.xyz, kappa, w} of n listed entries -> their field-major cache entries of mu.xyz,
// kappa, w, w * C(kappa) (guiding.cuh).
__global__ void k_cache_pack(const float* __restrict__ raw, uint32_t n, const uint32_t* __restrict__ list,
                             uint32_t first, float* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n * kLobes; i += gridDim.x * blockDim.x) {
        const float* l = raw + 5ull * i;
        const uint32_t lobe = i % kLobes, j = i / kLobes;
        const uint32_t e = list ? list[first + j] : first + j;
        float* o = out + static_cast<uint64_t>(kCacheEntry) * e + lobe;
        const float kappa = l[3];
        o[kLobes * kMuX] = l[0];
        o[kLobes * kMuY] = l[1];
        o[kLobes * kMuZ] = l[2];
        o[kLobes * kKappa] = kappa;
        o[kLobes * kWeight] = l[4];
        o[kLobes * kWeightC] = l[4] * (kappa / (2.0f * kPi * (1.0f - expf(-2.0f * kappa))));
    }
}

// The touched entries, in any order (each entry's refresh is independent of the others), and their
// count at list[n]; warp-aggregated so one atomic serves a warp's hits.
__global__ void k_cache_select(const uint8_t* __restrict__ touched, uint32_t n, uint32_t* __restrict__ list) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint32_t e = base + threadIdx.x;
        const bool hit = e < n && touched[e] != 0;
        const unsigned mask = __ballot_sync(0xFFFFFFFFu, hit);
        uint32_t first = 0;
        if (lane == 0 && mask) first = atomicAdd(list + n, static_cast<uint32_t>(__popc(mask)));
        first = __shfl_sync(0xFFFFFFFFu, first, 0);
        if (hit) list[first + __popc(mask & ((1u << lane) - 1u))] = e;
    }
}

// feats: the k_encode output for the same samples.
__global__ void __launch_bounds__(kInferWarps * 32) k_infer(Model M, const float4* __restrict__ in, uint32_t n_host,
                                                            const uint32_t* __restrict__ n_dev,
                                                            const uint32_t* __restrict__ feats, float* __restrict__ out) {
    const uint32_t n = n_dev ? *n_dev : n_host;
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* sw = reinterpret_cast<__nv_bfloat16*>(smem);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __nv_bfloat16* xin = sw + kFwdWeights + warp * kTileRows * pad(kIn);
    float* y = reinterpret_cast<float*>(sw + kFwdWeights + kInferWarps * kTileRows * pad(kIn)) + warp * kTileRows * kYld;
    stage_weights(M, sw, kFwdWeights);
    const uint32_t tiles = (n + kTileRows - 1) / kTileRows;
    for (uint32_t tile = blockIdx.x * kInferWarps + warp; tile < tiles; tile += gridDim.x * kInferWarps) {
        const uint32_t i = tile * kTileRows + lane;
        __nv_bfloat162* row = reinterpret_cast<__nv_bfloat162*>(xin + lane * pad(kIn));
        if (i < n) {
            const uint4* f = reinterpret_cast<const uint4*>(feats + 16ull * i);
            uint4* r4 = reinterpret_cast<uint4*>(row);
            for (int k = 0; k < 4; ++k) r4[k] = __ldg(f + k);
            direction_inputs(f3v(in[3 * i + 1]), f3v(in[3 * i + 2]), row);
        } else {
            for (int k = 0; k < kIn / 2; ++k) row[k] = __floats2bfloat162_rn(0.0f, 0.0f);
        }
        __syncwarp();
        forward16(sw, xin, y);
        forward16(sw, xin + 16 * pad(kIn), y + 16 * kYld);
        __syncwarp();
        if (i < n) {
            Lobe lb[kLobes];
            decode(y + lane * kYld, lb);
            float* o = out + static_cast<uint64_t>(i) * kOutUsed;
            for (int k = 0; k < kLobes; ++k) {
                o[5 * k] = lb[k].mu.x;
                o[5 * k + 1] = lb[k].mu.y;
                o[5 * k + 2] = lb[k].mu.z;
                o[5 * k + 3] = lb[k].kappa;
                o[5 * k + 4] = lb[k].w;
            }
        }
        __syncwarp();
    }
}

// ---- training ---------------------------------------------------------------------------------
// d loss / d outputs of one sample for loss = -c log q(wi); y: 48 outputs, g: 48 gradients.
__device__ __forceinline__ float loss_grad(const float* y, V3 wi, float c, float* g) {
    Lobe lb[kLobes];
    decode(y, lb);
    float f[kLobes], q = 0.0f;
    for (int k = 0; k < kLobes; ++k) {
        f[k] = vmf_pdf(lb[k], wi);
        q += lb[k].w * f[k];
    }
    q = fmaxf(q, 1e-30f);
    for (int k = 0; k < kLobes; ++k) {
        const float r = lb[k].w * f[k] / q;
        const float kap = lb[k].kappa;
        const float cs = dot(lb[k].mu, wi);
        const float e2 = expf(-2.0f * kap);
        const float dlnC = 1.0f / kap - 2.0f * e2 / (1.0f - e2);
        const float raw3 = y[5 * k + 3];
        const bool in_range = raw3 > kKappaLo && raw3 < kKappaHi;
        g[5 * k + 4] = -c * (r - lb[k].w);
        g[5 * k + 3] = in_range ? -c * r * (dlnC + (cs - 1.0f)) * kap : 0.0f;
        // through the normalisation of mu
        const V3 m = v3(y[5 * k], y[5 * k + 1], y[5 * k + 2]);
        const float mn = fmaxf(sqrtf(dot(m, m)), 1e-12f);
        const V3 gmu = wi * (-c * r * kap);
        const V3 gm = (gmu - lb[k].mu * dot(gmu, lb[k].mu)) * (1.0f / mn);
        g[5 * k] = gm.x;
        g[5 * k + 1] = gm.y;
        g[5 * k + 2] = gm.z;
    }
    for (int k = kOutUsed; k < kOut; ++k) g[k] = 0.0f;
    return -c * logf(q);
}

// A fragments of a 16-row tile -> transposed global store (feature-major, sample-minor), bf16.
template <int KSTEPS>
__device__ __forceinline__ void store_frag_t(const uint32_t (&a)[KSTEPS][4], __nv_bfloat16* dst, uint32_t n_total,
                                             uint32_t row0) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int s = 0; s < KSTEPS; ++s) {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const uint32_t row = row0 + g + ((r & 1) ? 8 : 0);
            const uint32_t col = 16 * s + 2 * t + ((r & 2) ? 8 : 0);
            const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162*>(&a[s][r]);
            dst[static_cast<uint64_t>(col) * n_total + row] = v.x;
            dst[static_cast<uint64_t>(col + 1) * n_total + row] = v.y;
        }
    }
}

// dX (fp32 tiles of 16 rows) masked by the ReLU of the layer input X (bf16 smem tile, row stride ld)
template <int NTILES>
__device__ __forceinline__ void relu_mask(float (&d)[NTILES][4], const __nv_bfloat16* x, int ld) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int j = 0; j < NTILES; ++j) {
        const int c = 8 * j + 2 * t;
        if (!(__bfloat162float(x[g * ld + c]) > 0.0f)) d[j][0] = 0.0f;
        if (!(__bfloat162float(x[g * ld + c + 1]) > 0.0f)) d[j][1] = 0.0f;
        if (!(__bfloat162float(x[(g + 8) * ld + c]) > 0.0f)) d[j][2] = 0.0f;
        if (!(__bfloat162float(x[(g + 8) * ld + c + 1]) > 0.0f)) d[j][3] = 0.0f;
    }
}

template <int KSTEPS>
__device__ __forceinline__ void store_a_rowmajor(const uint32_t (&a)[KSTEPS][4], __nv_bfloat16* tile, int ld) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int s = 0; s < KSTEPS; ++s) {
        *reinterpret_cast<uint32_t*>(tile + g * ld + 16 * s + 2 * t) = a[s][0];
        *reinterpret_cast<uint32_t*>(tile + (g + 8) * ld + 16 * s + 2 * t) = a[s][1];
        *reinterpret_cast<uint32_t*>(tile + g * ld + 16 * s + 8 + 2 * t) = a[s][2];
        *reinterpret_cast<uint32_t*>(tile + (g + 8) * ld + 16 * s + 8 + 2 * t) = a[s][3];
    }
}

struct TrainIO {
    const float4* rec;         // 4 float4 per record: pos+w, normal, wo, wi
    uint32_t n;                // records
    uint32_t n_pad;            // n rounded up to the 32-row tile: stride of the transposed buffers
    const float* mean_w;       // device: mean record weight (loss normalisation)
    __nv_bfloat16* xt[kLayers];   // [in_l][n]
    __nv_bfloat16* dzt[kLayers];  // [out_l][n]
    float* grid_grad;          // [L][T][F]
    float* loss_sum;           // device accumulator
};

// 16 rows of the backward/forward for one m-tile.  xin: input tile (bf16, 16 rows), xs[l]: smem tiles
// of the hidden-layer inputs for the ReLU masks, y/g: fp32 output & gradient tiles.
__global__ void __launch_bounds__(kWarps * 32) k_train(Model M, TrainIO io) {
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* sw = reinterpret_cast<__nv_bfloat16*>(smem);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // per-warp scratch: input tile, 4 hidden-input tiles, output tile (fp32), gradient tile (bf16)
    __nv_bfloat16* wbase = sw + kSmemWeights + warp * (kTileRows * pad(kIn) + 4 * kTileRows * pad(kHid) +
                                                       kTileRows * pad(kOut));
    __nv_bfloat16* xin = wbase;
    __nv_bfloat16* xh = xin + kTileRows * pad(kIn);          // 4 tiles [32][pad(64)]
    __nv_bfloat16* gy = xh + 4 * kTileRows * pad(kHid);      // [32][pad(48)]
    float* y = reinterpret_cast<float*>(sw + kSmemWeights + kWarps * (kTileRows * pad(kIn) + 4 * kTileRows * pad(kHid) +
                                                                    kTileRows * pad(kOut))) + warp * kTileRows * kYld;
    stage_weights(M, sw, kSmemWeights);
    const float inv_mean = 1.0f / fmaxf(*io.mean_w, 1e-30f);
    const uint32_t tiles = (io.n + kTileRows - 1) / kTileRows;
    float loss_acc = 0.0f;
    for (uint32_t tile = blockIdx.x * kWarps + warp; tile < tiles; tile += gridDim.x * kWarps) {
        const uint32_t i = tile * kTileRows + lane;
        const bool valid = i < io.n;
        __nv_bfloat162* row = reinterpret_cast<__nv_bfloat162*>(xin + lane * pad(kIn));
        float4 r0 = make_float4(0, 0, 0, 0), r1 = r0, r2 = r0, r3 = r0;
        if (valid) {
            r0 = io.rec[4 * i];
            r1 = io.rec[4 * i + 1];
            r2 = io.rec[4 * i + 2];
            r3 = io.rec[4 * i + 3];
            encode_inputs(M, f3v(r0), f3v(r1), f3v(r2), row);
        } else {
            for (int k = 0; k < kIn / 2; ++k) row[k] = __floats2bfloat162_rn(0.0f, 0.0f);
        }
        __syncwarp();
        // forward, two m-tiles; keep every layer's input for the masks and the weight gradients
        for (int m = 0; m < 2; ++m) {
            const uint32_t row0 = tile * kTileRows + 16 * m;
            uint32_t a0[3][4];
            load_a<3>(xin + 16 * m * pad(kIn), pad(kIn), a0);
            store_frag_t<3>(a0, io.xt[0], io.n_pad, row0);
            float d[8][4];
            layer_mma<3, 8>(a0, sw + sw_offset(0), pad(kIn), d);
            uint32_t a[4][4];
            for (int l = 1; l < kLayers; ++l) {
                chain<8>(d, a, true);
                store_a_rowmajor<4>(a, xh + (l - 1) * kTileRows * pad(kHid) + 16 * m * pad(kHid), pad(kHid));
                store_frag_t<4>(a, io.xt[l], io.n_pad, row0);
                if (l < kLayers - 1) {
                    layer_mma<4, 8>(a, sw + sw_offset(l), pad(kHid), d);
                } else {
                    float o[6][4];
                    layer_mma<4, 6>(a, sw + sw_offset(4), pad(kHid), o);
                    store_tile<6>(o, y + 16 * m * kYld, kYld);
                }
            }
        }
        __syncwarp();
        // loss and d loss / d y for this lane's sample (mean over the batch: 1/n)
        {
            float g[kOut];
            if (valid) {
                const float c = r0.w * inv_mean;
                loss_acc += loss_grad(y + lane * kYld, f3v(r3), c, g);
                for (int k = 0; k < kOut; ++k) g[k] *= 1.0f / static_cast<float>(io.n);
            } else {
                for (int k = 0; k < kOut; ++k) g[k] = 0.0f;
            }
            __nv_bfloat162* gr = reinterpret_cast<__nv_bfloat162*>(gy + lane * pad(kOut));
            for (int k = 0; k < kOut / 2; ++k) gr[k] = __floats2bfloat162_rn(g[2 * k], g[2 * k + 1]);
        }
        __syncwarp();
        // backward, two m-tiles
        for (int m = 0; m < 2; ++m) {
            const uint32_t row0 = tile * kTileRows + 16 * m;
            uint32_t ag[3][4];
            load_a<3>(gy + 16 * m * pad(kOut), pad(kOut), ag);
            store_frag_t<3>(ag, io.dzt[4], io.n_pad, row0);
            float d[8][4];
            layer_mma<3, 8>(ag, sw + swt_offset(4), pad(kOut), d);   // dX_4 = dZ_4 W_4
            uint32_t a[4][4];
            for (int l = 3; l >= 0; --l) {
                relu_mask<8>(d, xh + l * kTileRows * pad(kHid) + 16 * m * pad(kHid), pad(kHid));  // dZ_l
                chain<8>(d, a, false);
                store_frag_t<4>(a, io.dzt[l], io.n_pad, row0);
                if (l > 0) {
                    layer_mma<4, 8>(a, sw + swt_offset(l), pad(kHid), d);
                } else {
                    float dx[6][4];
                    layer_mma<4, 6>(a, sw + swt_offset(0), pad(kHid), dx);  // d loss / d inputs
                    store_tile<6>(dx, y + 16 * m * kYld, kYld);
                }
            }
        }
        __syncwarp();
        // hash-grid gradient of this lane's sample
        if (valid) {
            const V3 q = normalised_pos(M, f3v(r0));
            const float* gx = y + lane * kYld;
            for (int l = 0; l < kLevels; ++l) {
                const GridLevel lv = M.level[l];
                const float g0 = gx[2 * l], g1 = gx[2 * l + 1];
                if (g0 == 0.0f && g1 == 0.0f) continue;
                for (int c = 0; c < 8; ++c) {
                    const Corner k = grid_corner(lv, q, c);
                    float* p = io.grid_grad + (static_cast<uint64_t>(l) * kT + k.idx) * kFeat;
                    atomicAdd(reinterpret_cast<float2*>(p), make_float2(k.w * g0, k.w * g1));
                }
            }
        }
        __syncwarp();
    }
    for (int o = 16; o > 0; o >>= 1) loss_acc += __shfl_xor_sync(0xFFFFFFFFu, loss_acc, o);
    if (lane == 0) atomicAdd(io.loss_sum, loss_acc);
}

constexpr int kChunk = 256;   // samples per k_wgrad block (256 blocks for 2^16 samples)

// partial[chunk][out][in] = sum over the chunk of dZ^T[out][s] X^T[in][s] (one layer per launch)
template <int IN, int OUT>
__global__ void __launch_bounds__(128) k_wgrad(const __nv_bfloat16* __restrict__ dzt, const __nv_bfloat16* __restrict__ xt,
                                               uint32_t n, float* __restrict__ partial) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const uint32_t s0 = blockIdx.x * kChunk;
    const uint32_t s1 = min(n, s0 + kChunk);
    constexpr int MT = OUT / 16, NT = IN / 8;
    for (int mt = warp; mt < MT; mt += 4) {
        float acc[NT][4];
        for (int j = 0; j < NT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
        for (uint32_t s = s0; s + 16 <= s1; s += 16) {
            uint32_t a[1][4];
            const __nv_bfloat16* r0 = dzt + static_cast<uint64_t>(16 * mt + g) * n + s + 2 * t;
            const __nv_bfloat16* r1 = r0 + 8ull * n;
            a[0][0] = *reinterpret_cast<const uint32_t*>(r0);
            a[0][1] = *reinterpret_cast<const uint32_t*>(r1);
            a[0][2] = *reinterpret_cast<const uint32_t*>(r0 + 8);
            a[0][3] = *reinterpret_cast<const uint32_t*>(r1 + 8);
#pragma unroll
            for (int j = 0; j < NT; ++j) {
                const __nv_bfloat16* b = xt + static_cast<uint64_t>(8 * j + g) * n + s + 2 * t;
                mma_bf16(acc[j], a[0], *reinterpret_cast<const uint32_t*>(b), *reinterpret_cast<const uint32_t*>(b + 8));
            }
        }
        float* p = partial + static_cast<uint64_t>(blockIdx.x) * OUT * IN;
        for (int j = 0; j < NT; ++j) {
            p[(16 * mt + g) * IN + 8 * j + 2 * t] = acc[j][0];
            p[(16 * mt + g) * IN + 8 * j + 2 * t + 1] = acc[j][1];
            p[(16 * mt + g + 8) * IN + 8 * j + 2 * t] = acc[j][2];
            p[(16 * mt + g + 8) * IN + 8 * j + 2 * t + 1] = acc[j][3];
        }
    }
}

__global__ void k_reduce(const float* __restrict__ partial, uint32_t chunks, uint32_t count, float* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    float s = 0.0f;
    for (uint32_t c = 0; c < chunks; ++c) s += partial[static_cast<uint64_t>(c) * count + i];
    out[i] = s;
}

__global__ void k_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v, float* __restrict__ g,
                       __nv_bfloat16* __restrict__ copy, uint64_t n, float lr, float c1, float c2) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        const float mi = 0.9f * m[i] + 0.1f * gi;
        const float vi = 0.99f * v[i] + 0.01f * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + 1e-15f);
        p[i] = pi;
        g[i] = 0.0f;
        if (copy) copy[i] = __float2bfloat16_rn(pi);
    }
}

// Lazy Adam for the hash grid: an entry the batch did not touch (gradient exactly 0) keeps its
// parameter and moments, so a step reads 4 bytes per untouched entry instead of updating all
// 16.8M (the full update moved 571 MB per step).  Touched entries get the same update as k_adam.
__global__ void k_adam_sparse(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                              float* __restrict__ g, __nv_bfloat16* __restrict__ copy, uint64_t n, float lr, float c1,
                              float c2) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        if (gi == 0.0f) continue;
        const float mi = 0.9f * m[i] + 0.1f * gi;
        const float vi = 0.99f * v[i] + 0.01f * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + 1e-15f);
        p[i] = pi;
        g[i] = 0.0f;
        copy[i] = __float2bfloat16_rn(pi);
    }
}

__global__ void k_to_bf16(const float* __restrict__ p, __nv_bfloat16* __restrict__ q, uint64_t n) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        q[i] = __float2bfloat16_rn(p[i]);
}

__global__ void k_mean_weight(const float4* __restrict__ rec, uint32_t n, float* __restrict__ out) {
    float s = 0.0f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += rec[4 * i].w;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, s / static_cast<float>(n));
}

// deterministic initialisation: grid U(-1e-4, 1e-4), weights N(0, 2/fan_in) (Box-Muller on Philox)
__global__ void k_init(float* __restrict__ p, uint64_t n, uint64_t seed, int kind) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint4 r = philox(make_uint4(static_cast<uint32_t>(i), static_cast<uint32_t>(i >> 32), 0x6775u, kind),
                               static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
        const float u0 = ((r.x >> 8) + 0.5f) * (1.0f / 16777216.0f), u1 = (r.y >> 8) * (1.0f / 16777216.0f);
        if (kind == 0) {
            p[i] = (u0 * 2.0f - 1.0f) * 1e-4f;
        } else {
            int l = 0;
            while (l + 1 < kLayers && static_cast<int>(i) >= w_offset(l + 1)) ++l;
            const float sd = sqrtf(2.0f / layer_in(l)) * (l == kLayers - 1 ? 0.25f : 1.0f);
            p[i] = sd * sqrtf(-2.0f * logf(u0)) * cosf(2.0f * kPi * u1);
        }
    }
}

}  // namespace

size_t infer_smem_bytes() {
    return kFwdWeights * sizeof(__nv_bfloat16) + kInferWarps * kTileRows * pad(kIn) * sizeof(__nv_bfloat16) +
           kInferWarps * kTileRows * kYld * sizeof(float);
}

void k_mean_weight_launch(const float4* d_rec, uint32_t n, float* out, cudaStream_t s) {
    k_mean_weight<<<256, 256, 0, s>>>(d_rec, n, out);
}

void k_reduce_launch(const float* partial, uint32_t chunks, uint32_t count, float* out, cudaStream_t s) {
    k_reduce<<<(count + 255) / 256, 256, 0, s>>>(partial, chunks, count, out);
}

size_t train_smem_bytes() {
    return kSmemWeights * sizeof(__nv_bfloat16) +
           kWarps * (kTileRows * pad(kIn) + 4 * kTileRows * pad(kHid) + kTileRows * pad(kOut)) * sizeof(__nv_bfloat16) +
           kWarps * kTileRows * kYld * sizeof(float);
}

spt_status Guide::alloc(spt_context* c, const spt_guide_config& cfg_) {
    ctx = c;
    cfg = cfg_;
    auto dal = [&](void** p, size_t bytes) -> spt_status {
        SPT_CUDA(ctx, cudaMalloc(p, bytes));
        allocations.push_back(*p);
        SPT_CUDA(ctx, cudaMemsetAsync(*p, 0, bytes, ctx->stream));
        return SPT_OK;
    };
    spt_status st;
    if ((st = dal(reinterpret_cast<void**>(&grid_master), kGridParams * 4)) != SPT_OK) return st;
    if ((st = dal(reinterpret_cast<void**>(&grid_m), kGridParams * 4)) != SPT_OK) return st;
    if ((st = dal(reinterpret_cast<void**>(&grid_v), kGridParams * 4)) != SPT_OK) return st;
    if ((st = dal(reinterpret_cast<void**>(&grid_grad), kGridParams * 4)) != SPT_OK) return st;
    if ((st = dal(reinterpret_cast<void**>(&grid_bf16), kGridParams * 2)) != SPT_OK) return st;
    if ((st = dal(reinterpret_cast<void**>(&mlp_master), kMlpParams * 4)) != SPT_OK) return st;
    if ((st = dal(reinterpret_cast<void**>(&mlp_m), kMlpParams * 4)) != SPT_OK) return st;
    if ((st = dal(reinterpret_cast<void**>(&mlp_v), kMlpParams * 4)) != SPT_OK) return st;
    if ((st = dal(reinterpret_cast<void**>(&mlp_grad), kMlpParams * 4)) != SPT_OK) return st;
    if ((st = dal(reinterpret_cast<void**>(&smem_image), kSmemWeights * 2)) != SPT_OK) return st;
    if ((st = dal(reinterpret_cast<void**>(&scalars), 64)) != SPT_OK) return st;
    k_init<<<1024, 256, 0, ctx->stream>>>(grid_master, kGridParams, cfg.seed, 0);
    k_init<<<72, 256, 0, ctx->stream>>>(mlp_master, kMlpParams, cfg.seed, 1);
    SPT_CUDA(ctx, cudaGetLastError());
    SPT_CUDA(ctx, cudaFuncSetAttribute(k_infer, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(infer_smem_bytes())));
    SPT_CUDA(ctx, cudaFuncSetAttribute(k_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(train_smem_bytes())));
    for (int k = 0; k < 3; ++k) {
        model.lo[k] = cfg.box_min[k];
        const float ext = cfg.box_max[k] - cfg.box_min[k];
        model.inv_ext[k] = ext > 0.0f ? 1.0f / ext : 1.0f;
    }
    const double b = std::exp(std::log(static_cast<double>(kNMax) / kNMin) / (kLevels - 1));
    for (int l = 0; l < kLevels; ++l) {
        const uint32_t res = static_cast<uint32_t>(std::floor(kNMin * std::pow(b, l) + 1e-6));
        model.level[l].res = res;
        model.level[l].dense = static_cast<uint64_t>(res + 1) * (res + 1) * (res + 1) <= kT ? 1u : 0u;
    }
    model.grid = grid_bf16;
    model.smem_image = smem_image;
    // everything a guided render needs is allocated here, so renders and training steps allocate
    // nothing: the training buffers of one batch, the lobe cache and its inference scratch
    if ((st = ensure_train_buffers(cfg.batch)) != SPT_OK) return st;
    cache_res = cfg.cache_res ? cfg.cache_res : kCacheRes;
    n_cache = cache_res * cache_res * cache_res * 6;
    const uint32_t chunk = std::min(n_cache, kCacheChunk);
    if ((st = ensure_features(chunk)) != SPT_OK) return st;
    SPT_CUDA(ctx, cudaMalloc(&cache, static_cast<size_t>(n_cache) * kCacheEntry * sizeof(float)));
    SPT_CUDA(ctx, cudaMalloc(&cache_raw, static_cast<size_t>(chunk) * kOutUsed * sizeof(float)));
    SPT_CUDA(ctx, cudaMalloc(&cache_in, static_cast<size_t>(chunk) * 3 * sizeof(float4)));
    SPT_CUDA(ctx, cudaMalloc(&touched, n_cache));
    SPT_CUDA(ctx, cudaMemsetAsync(touched, 0, n_cache, ctx->stream));
    SPT_CUDA(ctx, cudaMalloc(&cache_list, (static_cast<size_t>(n_cache) + 1) * sizeof(uint32_t)));
    if ((st = refresh()) != SPT_OK) return st;
    return refresh_cache();
}

// bf16 copies of the current master parameters (which have changed: a new parameter version)
spt_status Guide::refresh() {
    ++version;
    k_stage<<<(kMlpParams + 255) / 256, 256, 0, ctx->stream>>>(mlp_master, smem_image);
    k_to_bf16<<<4096, 256, 0, ctx->stream>>>(grid_master, grid_bf16, kGridParams);
    SPT_CUDA(ctx, cudaGetLastError());
    return SPT_OK;
}

spt_status Guide::ensure_features(uint32_t n) {
    if (n <= feats_cap) return SPT_OK;
    if (feats) SPT_CUDA(ctx, cudaFree(feats));
    feats = nullptr;
    feats_cap = 0;
    SPT_CUDA(ctx, cudaMalloc(&feats, static_cast<size_t>(n) * kLevels * sizeof(uint32_t)));
    feats_cap = n;
    return SPT_OK;
}

spt_status Guide::refresh_cache() {
    if (cache_version == version) return SPT_OK;
    uint32_t n = n_cache;
    const uint32_t* list = nullptr;
    if (touched_any) {
        // only the entries guided renders have read; the count comes back to the host to size the passes
        SPT_CUDA(ctx, cudaMemsetAsync(cache_list + n_cache, 0, sizeof(uint32_t), ctx->stream));
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
        const unsigned g = static_cast<unsigned>(std::min<uint64_t>((n_cache + 255) / 256, 8ull * sms));
        k_cache_select<<<g, 256, 0, ctx->stream>>>(touched, n_cache, cache_list);
        SPT_CUDA(ctx, cudaGetLastError());
        SPT_CUDA(ctx, cudaMemcpyAsync(&n, cache_list + n_cache, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
        SPT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        list = cache_list;
    }
    for (uint32_t first = 0; first < n; first += kCacheChunk) {
        const uint32_t c = std::min(kCacheChunk, n - first);
        k_cache_inputs<<<256, 256, 0, ctx->stream>>>(model, cache_res, list, first, c, cache_in);
        SPT_CUDA(ctx, cudaGetLastError());
        spt_status st = infer(cache_in, c, cache_raw, ctx->stream);
        if (st != SPT_OK) return st;
        k_cache_pack<<<256, 256, 0, ctx->stream>>>(cache_raw, c, list, first, cache);
        SPT_CUDA(ctx, cudaGetLastError());
    }
    cache_version = version;
    return SPT_OK;
}

spt_status Guide::infer(const float4* d_in, uint32_t n, float* d_out, cudaStream_t s) {
    if (n == 0) return SPT_OK;
    spt_status st = ensure_features(n);
    if (st != SPT_OK) return st;
    return infer_list(d_in, nullptr, n, d_out, s);
}

spt_status Guide::infer_list(const float4* d_in, const uint32_t* d_n, uint32_t max_n, float* d_out, cudaStream_t s) {
    if (max_n > feats_cap) return fail(ctx, SPT_ERR_INTERNAL, "guide feature buffer smaller than the sample list");
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    const uint32_t tiles = (max_n + kTileRows - 1) / kTileRows;
    const uint64_t pairs = static_cast<uint64_t>(max_n) * kLevels;
    const unsigned g_enc = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>((pairs + 255) / 256, 16ull * sms)));
    const unsigned grid =
        static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>((tiles + kInferWarps - 1) / kInferWarps, sms)));
    const uint32_t n_host = d_n ? 0u : max_n;
    k_encode<<<g_enc, 256, 0, s>>>(model, d_in, n_host, d_n, feats);
    k_infer<<<grid, kInferWarps * 32, infer_smem_bytes(), s>>>(model, d_in, n_host, d_n, feats, d_out);
    SPT_CUDA(ctx, cudaGetLastError());
    return SPT_OK;
}

spt_status Guide::ensure_train_buffers(uint32_t n) {
    n = (n + 31u) & ~31u;
    if (n <= train_cap) return SPT_OK;
    for (void* p : train_allocs) cudaFree(p);
    train_allocs.clear();
    train_cap = 0;
    for (int l = 0; l < kLayers; ++l) {
        SPT_CUDA(ctx, cudaMalloc(&xt[l], static_cast<size_t>(layer_in(l)) * n * 2));
        train_allocs.push_back(xt[l]);
        SPT_CUDA(ctx, cudaMalloc(&dzt[l], static_cast<size_t>(layer_out(l)) * n * 2));
        train_allocs.push_back(dzt[l]);
    }
    const uint32_t chunks = (n + kChunk - 1) / kChunk;
    SPT_CUDA(ctx, cudaMalloc(&partial, static_cast<size_t>(chunks) * kHid * kHid * 4));
    train_allocs.push_back(partial);
    train_cap = n;
    return SPT_OK;
}

// Gradients of the batch loss (into grid_grad / mlp_grad, which must be zero) and the loss sum: on the
// tensor-memory kernels (guiding_tc.cu) unless the config asks for the warp-level mma.sync kernels.
spt_status Guide::gradients(const float4* d_rec, uint32_t n) {
    if (cfg.train_path == SPT_GUIDE_TRAIN_TCGEN05) return gradients_tc(d_rec, n);
    spt_status st = ensure_train_buffers(n);
    if (st != SPT_OK) return st;
    cudaStream_t s = ctx->stream;
    // pad n to a multiple of 16 for the tensor-core tiles (padding rows carry zero gradients)
    SPT_CUDA(ctx, cudaMemsetAsync(scalars, 0, 64, s));
    k_mean_weight<<<256, 256, 0, s>>>(d_rec, n, scalars);
    TrainIO io;
    io.rec = d_rec;
    io.n = n;
    io.n_pad = (n + 31u) & ~31u;
    io.mean_w = scalars;
    for (int l = 0; l < kLayers; ++l) {
        io.xt[l] = xt[l];
        io.dzt[l] = dzt[l];
    }
    io.grid_grad = grid_grad;
    io.loss_sum = scalars + 1;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    const uint32_t tiles = (n + kTileRows - 1) / kTileRows;
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>((tiles + kWarps - 1) / kWarps, 2ull * sms));
    k_train<<<grid, kWarps * 32, train_smem_bytes(), s>>>(model, io);
    SPT_CUDA(ctx, cudaGetLastError());
    const uint32_t chunks = (io.n_pad + kChunk - 1) / kChunk;
    for (int l = 0; l < kLayers; ++l) {
        const int in = layer_in(l), out = layer_out(l);
        if (l == 0) k_wgrad<kIn, kHid><<<chunks, 128, 0, s>>>(dzt[l], xt[l], io.n_pad, partial);
        else if (l == kLayers - 1) k_wgrad<kHid, kOut><<<chunks, 128, 0, s>>>(dzt[l], xt[l], io.n_pad, partial);
        else k_wgrad<kHid, kHid><<<chunks, 128, 0, s>>>(dzt[l], xt[l], io.n_pad, partial);
        k_reduce<<<(in * out + 255) / 256, 256, 0, s>>>(partial, chunks, in * out, mlp_grad + w_offset(l));
    }
    SPT_CUDA(ctx, cudaGetLastError());
    return SPT_OK;
}

spt_status Guide::step(const float4* d_rec, uint32_t n, float* loss) {
    spt_status st = gradients(d_rec, n);
    if (st != SPT_OK) return st;
    ++steps;
    ++version;
    const float c1 = 1.0f - std::pow(0.9f, static_cast<float>(steps));
    const float c2 = 1.0f - std::pow(0.99f, static_cast<float>(steps));
    k_adam_sparse<<<4096, 256, 0, ctx->stream>>>(grid_master, grid_m, grid_v, grid_grad, grid_bf16, kGridParams, cfg.lr,
                                                 c1, c2);
    k_adam<<<72, 256, 0, ctx->stream>>>(mlp_master, mlp_m, mlp_v, mlp_grad, nullptr, kMlpParams, cfg.lr, c1, c2);
    k_stage<<<(kMlpParams + 255) / 256, 256, 0, ctx->stream>>>(mlp_master, smem_image);
    SPT_CUDA(ctx, cudaGetLastError());
    if (tc_image && (st = stage_tc()) != SPT_OK) return st;
    if (loss) {
        float h[2];
        SPT_CUDA(ctx, cudaMemcpyAsync(h, scalars, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
        SPT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        *loss = h[1] / static_cast<float>(n);
    }
    return SPT_OK;
}

}  // namespace guide
}  // namespace spt
