// guiding_tc.cu -- one optimiser step's gradients of the path-guiding model with the MLP on the
// 5th-generation tensor cores (tcgen05, tensor memory), in tiles of 128 training records.
//
//   k_stage_tc     fp32 master weights -> bf16 W_l and W_l^T in the core-matrix layout (tc_sm100.cuh)
//   k_train_inputs the hash-grid features of every record, one thread per (record, level)
//   k_train_tc     per 128-record tile: forward through the five layers, the vMF-mixture loss and its
//                  gradient, the backward pass, and dW_l = dZ_l^T X_l accumulated in tensor memory over
//                  every tile of the CTA; writes the gradient of the 32 grid features per record and
//                  one dW partial per CTA
//   k_grid_scatter the grid gradient: d loss / d feature spread over the 8 cell corners of each level
//
// k_train_tc is persistent (one CTA per SM, 128 threads; thread t owns record t of the tile and tensor
// memory lane t).  Thread 0 issues every MMA and commits them to one mbarrier; the other threads wait
// on it (bounded) and move the accumulator through registers: ReLU and bf16 for the next layer's input,
// the ReLU mask on the way back.  Tensor memory (512 columns): columns 0-63 hold the M = 128
// accumulator of the current layer; dW_0..dW_3 (M = 64: out x in) and dW_4^T (in x out) sit at
// dw_col(l) and keep accumulating until the CTA has no tile left.  In the M = 64 accumulators row r
// lives in lane 32 * (r / 16) + r % 16.
#include <cuda_bf16.h>

#include <algorithm>

#include "guiding_host.h"
#include "tc_sm100.cuh"

namespace spt {
namespace guide {
namespace {

constexpr int kTcRows = 128;         // records per tile = threads per CTA = tensor-memory lanes
constexpr uint32_t kTmemCols = 512;
// first tensor-memory column of dW_l: 48 + 64 + 64 + 64 + 48 columns after the 64 of the layer accumulator
__host__ __device__ constexpr uint32_t dw_col(int l) {
    return l == 0 ? 64u : l == 1 ? 112u : l == 2 ? 176u : l == 3 ? 240u : 304u;
}
constexpr long long kWaitCycles = 2000000000ll;                   // about a second

// Byte offsets of the layers' W (rows = out, K = in) and W^T (rows = in, K = out) in the image.
__host__ __device__ constexpr uint32_t wf_off(int l) {
    return l == 0 ? 0u : wf_off(l - 1) + 2u * layer_in(l - 1) * layer_out(l - 1);
}
constexpr uint32_t kWHalf = wf_off(kLayers);   // 36,864 bytes
__host__ __device__ constexpr uint32_t wb_off(int l) { return kWHalf + wf_off(l); }
constexpr uint32_t kImageBytes = 2 * kWHalf;

// Shared memory: the weight image, the five layer inputs X_0..X_4 (record-major, core layout), one
// output-gradient tile, the mbarrier and the tensor-memory address.
__host__ __device__ constexpr uint32_t x_off(int l) {
    return kImageBytes + (l == 0 ? 0u : 2u * kTcRows * kIn + 2u * kTcRows * kHid * (l - 1));
}
constexpr uint32_t kDzOff = x_off(kLayers);
constexpr uint32_t kBarOff = kDzOff + 2u * kTcRows * kHid;
constexpr uint32_t kSmemTc = kBarOff + 64;
static_assert(kSmemTc <= 227u * 1024u, "shared memory of k_train_tc");
static_assert(dw_col(kLayers - 1) + kOut <= kTmemCols, "tensor-memory columns");

__global__ void k_stage_tc(const float* __restrict__ w, unsigned char* __restrict__ img) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kMlpParams) return;
    int l = 0;
    while (l + 1 < kLayers && i >= w_offset(l + 1)) ++l;
    const int r = i - w_offset(l), in = layer_in(l), out = layer_out(l);
    const int o = r / in, k = r % in;
    const __nv_bfloat16 v = __float2bfloat16_rn(w[i]);
    *reinterpret_cast<__nv_bfloat16*>(img + wf_off(l) + tc::core_offset(o, k, in)) = v;
    *reinterpret_cast<__nv_bfloat16*>(img + wb_off(l) + tc::core_offset(k, o, out)) = v;
}

// feats[16 i + l]: level l's two bf16 features of record i (records: 4 float4, position first).
__global__ void __launch_bounds__(256) k_train_inputs(const __grid_constant__ Model M, const float4* __restrict__ rec,
                                                      uint32_t n, uint32_t* __restrict__ feats) {
    const uint64_t total = static_cast<uint64_t>(n) * kLevels;
    for (uint64_t t = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t i = static_cast<uint32_t>(t / kLevels), l = static_cast<uint32_t>(t % kLevels);
        const V3 q = normalised_pos(M, f3v(__ldg(rec + 4ull * i)));
        const __nv_bfloat162 f = encode_level(M, M.level[l], q, static_cast<int>(l));
        feats[t] = *reinterpret_cast<const uint32_t*>(&f);
    }
}

// d loss / d outputs of one record (loss = -c log q(wi)), on registers: y[48] in, g[48] out.
__device__ __forceinline__ float loss_grad_regs(const float (&y)[kOut], V3 wi, float c, float (&g)[kOut]) {
    float mx = -3.0e38f;
#pragma unroll
    for (int k = 0; k < kLobes; ++k) mx = fmaxf(mx, y[5 * k + 4]);
    float wsum = 0.0f, w[kLobes], kap[kLobes], f[kLobes], cs[kLobes], mn[kLobes];
    V3 mu[kLobes];
#pragma unroll
    for (int k = 0; k < kLobes; ++k) {
        const V3 a = v3(y[5 * k], y[5 * k + 1], y[5 * k + 2]);
        const float nrm = sqrtf(dot(a, a));
        mn[k] = fmaxf(nrm, 1e-12f);
        mu[k] = nrm > 1e-12f ? a * (1.0f / nrm) : v3(0.0f, 1.0f, 0.0f);
        kap[k] = expf(fminf(fmaxf(y[5 * k + 3], kKappaLo), kKappaHi));
        w[k] = expf(y[5 * k + 4] - mx);
        wsum += w[k];
    }
    float q = 0.0f;
#pragma unroll
    for (int k = 0; k < kLobes; ++k) {
        w[k] /= wsum;
        cs[k] = dot(mu[k], wi);
        f[k] = kap[k] / (2.0f * kPi * (1.0f - expf(-2.0f * kap[k]))) * expf(kap[k] * (cs[k] - 1.0f));
        q += w[k] * f[k];
    }
    q = fmaxf(q, 1e-30f);
#pragma unroll
    for (int k = 0; k < kLobes; ++k) {
        const float r = w[k] * f[k] / q;
        const float e2 = expf(-2.0f * kap[k]);
        const float dlnC = 1.0f / kap[k] - 2.0f * e2 / (1.0f - e2);
        const float raw3 = y[5 * k + 3];
        const bool in_range = raw3 > kKappaLo && raw3 < kKappaHi;
        g[5 * k + 4] = -c * (r - w[k]);
        g[5 * k + 3] = in_range ? -c * r * (dlnC + (cs[k] - 1.0f)) * kap[k] : 0.0f;
        const V3 gmu = wi * (-c * r * kap[k]);
        const V3 gm = (gmu - mu[k] * dot(gmu, mu[k])) * (1.0f / mn[k]);
        g[5 * k] = gm.x;
        g[5 * k + 1] = gm.y;
        g[5 * k + 2] = gm.z;
    }
#pragma unroll
    for (int k = kOutUsed; k < kOut; ++k) g[k] = 0.0f;
    return -c * logf(q);
}

struct TcIO {
    const unsigned char* image;    // k_stage_tc output (kImageBytes)
    const float4* rec;             // 4 float4 per record: pos + weight, normal, wo, wi
    const uint32_t* feats;         // k_train_inputs output
    uint32_t n;
    const float* mean_w;           // mean record weight (loss normalisation)
    float* dx0;                    // [n][32]: d loss / d grid feature
    float* partial;                // [gridDim.x][kMlpParams]: this CTA's dW, in mlp parameter order
    float* loss_sum;
    uint32_t* status;              // bit 2: a bounded wait ran out
};

// 16 bytes of a bf16 row into the core layout of a [128][K] tile: elements k0..k0+7 of row r.
__device__ __forceinline__ void put16(unsigned char* tile, uint32_t r, uint32_t k0, uint32_t K, uint4 v) {
    *reinterpret_cast<uint4*>(tile + tc::core_offset(r, k0, K)) = v;
}
__device__ __forceinline__ uint4 get16(const unsigned char* tile, uint32_t r, uint32_t k0, uint32_t K) {
    return *reinterpret_cast<const uint4*>(tile + tc::core_offset(r, k0, K));
}
__device__ __forceinline__ uint32_t pack2(float a, float b) {
    __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&v);
}

// NCOL columns (a multiple of 16) of this thread's lane, from column col.
template <int NCOL>
__device__ __forceinline__ void ld_row(uint32_t tmem, uint32_t col, float (&v)[NCOL]) {
    const uint32_t lane_base = (threadIdx.x & ~31u) << 16;
#pragma unroll
    for (int c = 0; c < NCOL / 16; ++c) {
        float t[16];
        tc::ld16(tmem + lane_base + col + 16u * c, t);
#pragma unroll
        for (int j = 0; j < 16; ++j) v[16 * c + j] = t[j];
    }
    tc::wait_ld();
}

// D (columns 0..N-1) = A [128 x K] * B^T with B [N x K], both K-major core-layout tiles.
template <int N, int K>
__device__ __forceinline__ void mma_tile(uint32_t tmem, uint32_t a_addr, uint32_t b_addr) {
    constexpr uint32_t idesc = tc::idesc_bf16(128, N, false, false);
#pragma unroll
    for (int s = 0; s < K / 16; ++s)
        tc::mma_bf16(tmem, tc::smem_desc(a_addr + 256u * s, 128u, (K / 8) * 128u),
                     tc::smem_desc(b_addr + 256u * s, 128u, (K / 8) * 128u), idesc, s > 0);
}

// D [64 x N] (+)= A^T B over the 128 records of the tile: A is a [128][64] tile, B a [128][N] tile,
// both record-major, read MN-major (records = K).
template <int N, int KA>
__device__ __forceinline__ void mma_dw(uint32_t tmem, uint32_t a_addr, uint32_t b_addr, bool accumulate) {
    constexpr uint32_t idesc = tc::idesc_bf16(64, N, true, true);
#pragma unroll
    for (int s = 0; s < kTcRows / 16; ++s)
        tc::mma_bf16(tmem, tc::smem_desc(a_addr + 2u * (KA / 8) * 128u * s, (KA / 8) * 128u, 128u),
                     tc::smem_desc(b_addr + 2u * (N / 8) * 128u * s, (N / 8) * 128u, 128u), idesc,
                     accumulate || s > 0);
}

__global__ void __launch_bounds__(kTcRows, 1) k_train_tc(TcIO io) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const uint32_t bar = tc::smem_addr(smem + kBarOff);
    const uint32_t slot = tc::smem_addr(smem + kBarOff + 16);
    // weights into shared memory
    {
        const uint4* src = reinterpret_cast<const uint4*>(io.image);
        uint4* dst = reinterpret_cast<uint4*>(smem);
        for (uint32_t i = tid; i < kImageBytes / 16; i += kTcRows) dst[i] = __ldg(src + i);
    }
    if (warp == 0) tc::tmem_alloc(slot, kTmemCols);
    if (tid == 0) tc::mbar_init(bar, 1);
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(smem + kBarOff + 16);
    const uint32_t sbase = tc::smem_addr(smem);
    const float inv_mean = 1.0f / fmaxf(*io.mean_w, 1e-30f);
    const float inv_n = 1.0f / static_cast<float>(io.n);
    const uint32_t tiles = (io.n + kTcRows - 1) / kTcRows;
    uint32_t phase = 0;
    bool ok = true, any = false;
    float loss_acc = 0.0f;
    auto issue = [&](auto&& body) {
        if (tid == 0) {
            tc::fence_after_sync();
            body();
            tc::commit(bar);
        }
    };
    // wait for the committed MMAs; every thread learns whether any wait ran out
    auto wait_all = [&]() -> bool {
        const bool mine = tc::mbar_wait(bar, phase, kWaitCycles);
        phase ^= 1u;
        tc::fence_after_sync();
        return __syncthreads_and(mine) != 0;
    };
    for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const uint32_t row = tile * kTcRows + tid;
        const bool valid = row < io.n;
        // X_0: 32 grid features, normal, wo, zeros
        float4 r1 = make_float4(0.f, 0.f, 0.f, 0.f), r2 = r1, r3 = r1;
        float weight = 0.0f;
        {
            unsigned char* x0 = smem + x_off(0);
            uint4 f[4] = {make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0)};
            if (valid) {
                const uint4* src = reinterpret_cast<const uint4*>(io.feats + 16ull * row);
#pragma unroll
                for (int c = 0; c < 4; ++c) f[c] = __ldg(src + c);
                weight = __ldg(io.rec + 4ull * row).w;
                r1 = __ldg(io.rec + 4ull * row + 1);
                r2 = __ldg(io.rec + 4ull * row + 2);
                r3 = __ldg(io.rec + 4ull * row + 3);
            }
#pragma unroll
            for (int c = 0; c < 4; ++c) put16(x0, tid, 8u * c, kIn, f[c]);
            const uint4 d = valid ? make_uint4(pack2(r1.x, r1.y), pack2(r1.z, r2.x), pack2(r2.y, r2.z), 0u)
                                  : make_uint4(0, 0, 0, 0);
            put16(x0, tid, 32, kIn, d);
            put16(x0, tid, 40, kIn, make_uint4(0, 0, 0, 0));
        }
        tc::fence_proxy_async();
        tc::fence_before_sync();
        __syncthreads();
        // ---- forward ----
        float y[kOut];
#pragma unroll
        for (int l = 0; l < kLayers; ++l) {
            issue([&] {
                if (l == 0) mma_tile<kHid, kIn>(tmem, sbase + x_off(0), sbase + wf_off(0));
                else if (l < kLayers - 1) mma_tile<kHid, kHid>(tmem, sbase + x_off(l), sbase + wf_off(l));
                else mma_tile<kOut, kHid>(tmem, sbase + x_off(l), sbase + wf_off(l));
            });
            if (!(ok = wait_all())) break;
            if (l < kLayers - 1) {
                float v[kHid];
                ld_row<kHid>(tmem, 0, v);
                unsigned char* xn = smem + x_off(l + 1);
#pragma unroll
                for (int c = 0; c < kHid / 8; ++c) {
                    const uint4 p = make_uint4(pack2(fmaxf(v[8 * c], 0.f), fmaxf(v[8 * c + 1], 0.f)),
                                               pack2(fmaxf(v[8 * c + 2], 0.f), fmaxf(v[8 * c + 3], 0.f)),
                                               pack2(fmaxf(v[8 * c + 4], 0.f), fmaxf(v[8 * c + 5], 0.f)),
                                               pack2(fmaxf(v[8 * c + 6], 0.f), fmaxf(v[8 * c + 7], 0.f)));
                    put16(xn, tid, 8u * c, kHid, p);
                }
            } else {
                ld_row<kOut>(tmem, 0, y);
            }
            tc::fence_proxy_async();
            tc::fence_before_sync();
            __syncthreads();
        }
        if (!ok) break;
        // ---- loss and its gradient (mean over the batch) -> dZ_4 ----
        {
            float g[kOut];
            if (valid) {
                loss_acc += loss_grad_regs(y, f3v(r3), weight * inv_mean, g);
#pragma unroll
                for (int k = 0; k < kOut; ++k) g[k] *= inv_n;
            } else {
#pragma unroll
                for (int k = 0; k < kOut; ++k) g[k] = 0.0f;
            }
            unsigned char* dz = smem + kDzOff;
#pragma unroll
            for (int c = 0; c < kOut / 8; ++c)
                put16(dz, tid, 8u * c, kOut,
                      make_uint4(pack2(g[8 * c], g[8 * c + 1]), pack2(g[8 * c + 2], g[8 * c + 3]),
                                 pack2(g[8 * c + 4], g[8 * c + 5]), pack2(g[8 * c + 6], g[8 * c + 7])));
        }
        tc::fence_proxy_async();
        tc::fence_before_sync();
        __syncthreads();
        // ---- backward: dX_l = dZ_l W_l (into columns 0..), dW_l += dZ_l^T X_l ----
        const bool acc = any;
#pragma unroll
        for (int l = kLayers - 1; l >= 0; --l) {
            issue([&] {
                const uint32_t dz = sbase + kDzOff;
                if (l == kLayers - 1) {
                    mma_tile<kHid, kOut>(tmem, dz, sbase + wb_off(l));
                    // dW_4^T [in x out] = X_4^T dZ_4
                    mma_dw<kOut, kHid>(tmem + dw_col(l), sbase + x_off(l), dz, acc);
                } else if (l > 0) {
                    mma_tile<kHid, kHid>(tmem, dz, sbase + wb_off(l));
                    mma_dw<kHid, kHid>(tmem + dw_col(l), dz, sbase + x_off(l), acc);
                } else {
                    mma_tile<kIn, kHid>(tmem, dz, sbase + wb_off(0));
                    mma_dw<kIn, kHid>(tmem + dw_col(0), dz, sbase + x_off(0), acc);
                }
            });
            if (!(ok = wait_all())) break;
            if (l > 0) {
                // dZ_{l-1} = dX_l masked by the ReLU of X_l (this thread's row of the X_l tile)
                float v[kHid];
                ld_row<kHid>(tmem, 0, v);
                const unsigned char* xl = smem + x_off(l);
                unsigned char* dz = smem + kDzOff;
#pragma unroll
                for (int c = 0; c < kHid / 8; ++c) {
                    const uint4 xm = get16(xl, tid, 8u * c, kHid);
                    const uint32_t xw[4] = {xm.x, xm.y, xm.z, xm.w};
                    uint32_t o[4];
#pragma unroll
                    for (int h = 0; h < 4; ++h) {
                        // a bf16 is > 0 when its sign bit is clear and it is not zero
                        const uint32_t lo = xw[h] & 0xFFFFu, hi = xw[h] >> 16;
                        const float a = (lo != 0u && !(lo & 0x8000u)) ? v[8 * c + 2 * h] : 0.0f;
                        const float b = (hi != 0u && !(hi & 0x8000u)) ? v[8 * c + 2 * h + 1] : 0.0f;
                        o[h] = pack2(a, b);
                    }
                    put16(dz, tid, 8u * c, kHid, make_uint4(o[0], o[1], o[2], o[3]));
                }
            } else {
                float v[kIn];
                ld_row<kIn>(tmem, 0, v);   // every lane of the warp takes part in the load
                if (valid) {
                    float4* dst = reinterpret_cast<float4*>(io.dx0 + 32ull * row);
#pragma unroll
                    for (int c = 0; c < 8; ++c) dst[c] = make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
                }
            }
            tc::fence_proxy_async();
            tc::fence_before_sync();
            __syncthreads();
        }
        any = true;
    }
    // this CTA's dW (zeros if it had no tile) in parameter order; M = 64 rows live in lanes
    // 32 * (r / 16) + r % 16, so the lanes 0..15 of each warp hold rows 16 * warp + 0..15
    float* part = io.partial + static_cast<uint64_t>(blockIdx.x) * kMlpParams;
    const uint32_t lane = tid & 31u;
    if (ok) {
#pragma unroll
        for (int l = 0; l < kLayers; ++l) {
            const int in = layer_in(l), out = layer_out(l);
            const int ncol = l == kLayers - 1 ? kOut : in;   // columns of the accumulator
            float v[kHid];
            if (any) {
                if (ncol == kHid) ld_row<kHid>(tmem, dw_col(l), v);
                else {
                    float t[kIn];
                    ld_row<kIn>(tmem, dw_col(l), t);
#pragma unroll
                    for (int j = 0; j < kIn; ++j) v[j] = t[j];
                }
            }
            if (lane < 16) {
                const int r = 16 * static_cast<int>(warp) + static_cast<int>(lane);   // accumulator row
#pragma unroll
                for (int j = 0; j < ncol; ++j) {
                    const float x = any ? v[j] : 0.0f;
                    // layers 0-3: row = out, column = in; layer 4 holds the transpose
                    const int idx = l == kLayers - 1 ? j * in + r : r * in + j;
                    part[w_offset(l) + idx] = x;
                }
            }
            (void)out;
        }
    } else if (tid == 0) {
        atomicOr(io.status, 4u);
        // a wait ran out: give the MMAs in flight one more bounded wait before the columns are freed
        tc::mbar_wait(bar, phase, kWaitCycles);
    }
    for (int o = 16; o > 0; o >>= 1) loss_acc += __shfl_xor_sync(0xFFFFFFFFu, loss_acc, o);
    if (lane == 0) atomicAdd(io.loss_sum, loss_acc);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, kTmemCols);
}

// d loss / d grid parameters: each (record, level) spreads its two feature gradients over the cell's
// 8 corners with their trilinear weights.
__global__ void __launch_bounds__(256) k_grid_scatter(const __grid_constant__ Model M, const float4* __restrict__ rec,
                                                      uint32_t n, const float* __restrict__ dx0,
                                                      float* __restrict__ grid_grad) {
    const uint64_t total = static_cast<uint64_t>(n) * kLevels;
    for (uint64_t t = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t i = static_cast<uint32_t>(t / kLevels), l = static_cast<uint32_t>(t % kLevels);
        const float2 g = __ldg(reinterpret_cast<const float2*>(dx0 + 32ull * i) + l);
        if (g.x == 0.0f && g.y == 0.0f) continue;
        const V3 q = normalised_pos(M, f3v(__ldg(rec + 4ull * i)));
        const GridLevel lv = M.level[l];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const Corner k = grid_corner(lv, q, c);
            float* p = grid_grad + (static_cast<uint64_t>(l) * kT + k.idx) * kFeat;
            atomicAdd(reinterpret_cast<float2*>(p), make_float2(k.w * g.x, k.w * g.y));
        }
    }
}

}  // namespace

size_t train_tc_smem_bytes() { return kSmemTc; }
size_t train_tc_image_bytes() { return kImageBytes; }

spt_status Guide::stage_tc() {
    k_stage_tc<<<(kMlpParams + 255) / 256, 256, 0, ctx->stream>>>(mlp_master, tc_image);
    SPT_CUDA(ctx, cudaGetLastError());
    return SPT_OK;
}

// The batch's gradients through the tensor-memory kernels (grid_grad and mlp_grad start at zero).
spt_status Guide::gradients_tc(const float4* d_rec, uint32_t n) {
    spt_status st = ensure_tc_buffers(n);
    if (st != SPT_OK) return st;
    cudaStream_t s = ctx->stream;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    SPT_CUDA(ctx, cudaMemsetAsync(scalars, 0, 64, s));
    k_mean_weight_launch(d_rec, n, scalars, s);
    const uint64_t pairs = static_cast<uint64_t>(n) * kLevels;
    const unsigned g_enc = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>((pairs + 255) / 256, 16ull * sms)));
    k_train_inputs<<<g_enc, 256, 0, s>>>(model, d_rec, n, tc_feats);
    TcIO io;
    io.image = tc_image;
    io.rec = d_rec;
    io.feats = tc_feats;
    io.n = n;
    io.mean_w = scalars;
    io.dx0 = tc_dx0;
    io.partial = tc_partial;
    io.loss_sum = scalars + 1;
    io.status = ctx->d_status;
    const uint32_t tiles = (n + kTcRows - 1) / kTcRows;
    const unsigned grid = static_cast<unsigned>(std::max<uint32_t>(1, std::min<uint32_t>(tiles, static_cast<uint32_t>(sms))));
    k_train_tc<<<grid, kTcRows, kSmemTc, s>>>(io);
    k_grid_scatter<<<g_enc, 256, 0, s>>>(model, d_rec, n, tc_dx0, grid_grad);
    SPT_CUDA(ctx, cudaGetLastError());
    k_reduce_launch(tc_partial, grid, kMlpParams, mlp_grad, s);
    SPT_CUDA(ctx, cudaGetLastError());
    return SPT_OK;
}

spt_status Guide::ensure_tc_buffers(uint32_t n) {
    if (!tc_image) {
        SPT_CUDA(ctx, cudaMalloc(&tc_image, kImageBytes));
        allocations.push_back(tc_image);
        SPT_CUDA(ctx, cudaFuncSetAttribute(k_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(kSmemTc)));
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
        SPT_CUDA(ctx, cudaMalloc(&tc_partial, static_cast<size_t>(sms) * kMlpParams * sizeof(float)));
        allocations.push_back(tc_partial);
        spt_status st = stage_tc();
        if (st != SPT_OK) return st;
    }
    if (n <= tc_cap) return SPT_OK;
    if (tc_feats) cudaFree(tc_feats);
    if (tc_dx0) cudaFree(tc_dx0);
    tc_feats = nullptr;
    tc_dx0 = nullptr;
    tc_cap = 0;
    SPT_CUDA(ctx, cudaMalloc(&tc_feats, static_cast<size_t>(n) * kLevels * sizeof(uint32_t)));
    SPT_CUDA(ctx, cudaMalloc(&tc_dx0, static_cast<size_t>(n) * 32 * sizeof(float)));
    tc_cap = n;
    return SPT_OK;
}

}  // namespace guide
}  // namespace spt
