// postprocess.cu -- the ray casters' image post-processing and the PPM quantization on the device.
//
//   k_depth_range / k_depth_rgb    DepthRayCaster::saveImageToFile (integrators/depth_raycaster.cpp:9-34):
//                                  min over hit depths (> 0), max over all pixels, then a grey ramp
//                                  (v - min) / range, 1 when the range is 0, black for background (-1)
//   k_count_range / k_count_rgb    IntTestCountRayCaster::saveImageToFile (int_test_count_raycaster.cpp:20-73):
//                                  counts normalised by the per-pixel min / max, then the HSL heat map
//   k_normal_rgb                   NormalRayCaster::saveImageToFile (normal_raycaster.cpp:6-17): n * 0.5 + 0.5
//   k_to_bytes                     ImageBuffer::convertTosRGB + saveToFile (core/image_buffer.cpp:22-47):
//                                  clamp, optional pow(c, 1/2.2), int(c * 255 + 0.5)
// All arithmetic is the reference's single-precision sequence (the library is built without FMA
// contraction), so the images match the host post-processing bit for bit; the sRGB curve goes through
// double-precision pow as the reference's does, where CUDA's and the host's results can differ in the
// last bit, which moves a byte by at most one.
#include <fstream>

#include "spt_internal.h"

namespace spt {
namespace {

// Order-preserving map of a float onto an unsigned key (for atomicMin / atomicMax).
__device__ __forceinline__ uint32_t float_key(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

// range[0]: key of the min over depths > 0 (starts at +inf), range[1]: key of the max (starts at -inf).
__global__ void k_depth_range(const float* __restrict__ depth, uint64_t n, uint32_t* range) {
    uint32_t mn = float_key(__int_as_float(0x7f800000)), mx = float_key(__int_as_float(static_cast<int>(0xff800000u)));
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const float v = depth[i];
        const uint32_t k = float_key(v);
        mx = k > mx ? k : mx;
        if (v > 0.0f) mn = k < mn ? k : mn;
    }
    for (int o = 16; o > 0; o >>= 1) {
        mn = min(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, o));
        mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(range, mn);
        atomicMax(range + 1, mx);
    }
}

__global__ void k_depth_rgb(const float* __restrict__ depth, uint64_t n, const uint32_t* range, float pmin, float pmax,
                            float* __restrict__ rgb) {
    const float mn = pmin != -1.0f ? pmin : key_float(range[0]);
    const float mx = pmax != -1.0f ? pmax : key_float(range[1]);
    const float r = mx - mn;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const float v = depth[i];
        const float g = v != -1.0f ? (r != 0.0f ? (v - mn) / r : 1.0f) : 0.0f;
        rgb[3 * i] = g;
        rgb[3 * i + 1] = g;
        rgb[3 * i + 2] = g;
    }
}

// range[0] / range[1]: min / max count over all pixels (unsigned, as the reference's size_t counters).
__global__ void k_count_range(const int64_t* __restrict__ count, uint64_t n, unsigned long long* range) {
    unsigned long long mn = ~0ull, mx = 0ull;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const unsigned long long v = static_cast<unsigned long long>(count[i]);
        mn = v < mn ? v : mn;
        mx = v > mx ? v : mx;
    }
    for (int o = 16; o > 0; o >>= 1) {
        mn = min(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, o));
        mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(range, mn);
        atomicMax(range + 1, mx);
    }
}

__device__ __forceinline__ float hue_to_rgb(float v1, float v2, float h) {  // int_test_count_raycaster.cpp:10-18
    if (h < 0.0f) h += 1.0f;
    if (h > 1.0f) h -= 1.0f;
    if ((6.0f * h) < 1.0f) return v1 + (v2 - v1) * 6.0f * h;
    if ((2.0f * h) < 1.0f) return v2;
    if ((3.0f * h) < 2.0f) return v1 + (v2 - v1) * ((2.0f / 3.0f) - h) * 6.0f;
    return v1;
}

__global__ void k_count_rgb(const int64_t* __restrict__ count, uint64_t n, const unsigned long long* range,
                            long long pmin, long long pmax, float* __restrict__ rgb) {
    // the reference's mix of size_t / long / unsigned int arithmetic, kept as is
    const unsigned long long mn = pmin != -1 ? static_cast<unsigned long long>(pmin) : range[0];
    const unsigned long long mx = pmax != -1 ? static_cast<unsigned long long>(pmax) : range[1];
    const uint32_t span = static_cast<uint32_t>(mx - mn);
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        float t;
        if (span > 0)
            t = static_cast<float>(static_cast<unsigned long long>(count[i]) - mn) / static_cast<float>(span);
        else if (mx > 0)
            t = 1.0f;
        else
            t = 0.0f;
        const float hh = 0.65f - (t * 0.65f), s = 1.0f, l = t * 0.5f;
        const float v2 = (l < 0.5f) ? l * (1.0f + s) : (l + s) - (s * l);
        const float v1 = 2.0f * l - v2;
        rgb[3 * i] = hue_to_rgb(v1, v2, hh + (1.0f / 3.0f));
        rgb[3 * i + 1] = hue_to_rgb(v1, v2, hh);
        rgb[3 * i + 2] = hue_to_rgb(v1, v2, hh - (1.0f / 3.0f));
    }
}

// NormalRayCaster::saveImageToFile (integrators/normal_raycaster.cpp:6-17): n * 0.5 + 0.5 where the pixel
// is not background (all-zero), in place.
__global__ void k_normal_rgb(float* __restrict__ rgb, uint64_t n) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const float x = rgb[3 * i], y = rgb[3 * i + 1], z = rgb[3 * i + 2];
        if (x != 0.0f || y != 0.0f || z != 0.0f) {
            rgb[3 * i] = x * 0.5f + 0.5f;
            rgb[3 * i + 1] = y * 0.5f + 0.5f;
            rgb[3 * i + 2] = z * 0.5f + 0.5f;
        }
    }
}

__device__ __forceinline__ float clamp01(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }

__global__ void k_to_bytes(const float* __restrict__ rgb, uint64_t n, int srgb, uint8_t* __restrict__ out) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        float c = rgb[i];
        // the reference's unqualified pow on these floats is the double-precision one
        if (srgb) c = static_cast<float>(pow(static_cast<double>(clamp01(c)), static_cast<double>(1.0f / 2.2f)));
        out[i] = static_cast<uint8_t>(static_cast<int>(clamp01(c) * 255.0f + 0.5f));
    }
}

unsigned grid_for(spt_context* ctx, uint64_t n) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    return static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 8ull * sms)));
}

}  // namespace
}  // namespace spt

using namespace spt;

extern "C" {

spt_status spt_depth_to_rgb_device(spt_context* ctx, const float* d_depth, uint32_t width, uint32_t height,
                                   float min_depth, float max_depth, float* d_rgb, void* stream) {
    if (!ctx || !d_depth || !d_rgb) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    const uint64_t n = static_cast<uint64_t>(width) * height;
    if (n == 0) return SPT_OK;
    SPT_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    void* r;
    spt_status st = scratch(ctx, 8, 64, &r);
    if (st != SPT_OK) return st;
    uint32_t* range = static_cast<uint32_t*>(r);
    const uint32_t init[2] = {0xFF800000u, 0x007FFFFFu};  // keys of +inf and -inf
    SPT_CUDA(ctx, cudaMemcpyAsync(range, init, sizeof(init), cudaMemcpyHostToDevice, s));
    k_depth_range<<<grid_for(ctx, n), 256, 0, s>>>(d_depth, n, range);
    k_depth_rgb<<<grid_for(ctx, n), 256, 0, s>>>(d_depth, n, range, min_depth, max_depth, d_rgb);
    SPT_CUDA(ctx, cudaGetLastError());
    return SPT_OK;
}

spt_status spt_count_to_rgb_device(spt_context* ctx, const int64_t* d_count, uint32_t width, uint32_t height,
                                   int64_t min_count, int64_t max_count, float* d_rgb, void* stream) {
    if (!ctx || !d_count || !d_rgb) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    const uint64_t n = static_cast<uint64_t>(width) * height;
    if (n == 0) return SPT_OK;
    SPT_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    void* r;
    spt_status st = scratch(ctx, 8, 64, &r);
    if (st != SPT_OK) return st;
    unsigned long long* range = static_cast<unsigned long long*>(r);
    const unsigned long long init[2] = {~0ull, 0ull};
    SPT_CUDA(ctx, cudaMemcpyAsync(range, init, sizeof(init), cudaMemcpyHostToDevice, s));
    k_count_range<<<grid_for(ctx, n), 256, 0, s>>>(d_count, n, range);
    k_count_rgb<<<grid_for(ctx, n), 256, 0, s>>>(d_count, n, range, min_count, max_count, d_rgb);
    SPT_CUDA(ctx, cudaGetLastError());
    return SPT_OK;
}

spt_status spt_normal_to_rgb_device(spt_context* ctx, float* d_rgb, uint32_t width, uint32_t height, void* stream) {
    if (!ctx || !d_rgb) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    const uint64_t n = static_cast<uint64_t>(width) * height;
    if (n == 0) return SPT_OK;
    SPT_CUDA(ctx, cudaSetDevice(ctx->device));
    k_normal_rgb<<<grid_for(ctx, n), 256, 0, static_cast<cudaStream_t>(stream)>>>(d_rgb, n);
    SPT_CUDA(ctx, cudaGetLastError());
    return SPT_OK;
}

spt_status spt_rgb_to_bytes_device(spt_context* ctx, const float* d_rgb, uint64_t n_values, int32_t to_srgb,
                                   uint8_t* d_bytes, void* stream) {
    if (!ctx || (n_values && (!d_rgb || !d_bytes))) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n_values == 0) return SPT_OK;
    SPT_CUDA(ctx, cudaSetDevice(ctx->device));
    k_to_bytes<<<grid_for(ctx, n_values), 256, 0, static_cast<cudaStream_t>(stream)>>>(d_rgb, n_values, to_srgb,
                                                                                        d_bytes);
    SPT_CUDA(ctx, cudaGetLastError());
    return SPT_OK;
}

spt_status spt_write_ppm_bytes(const char* path, const uint8_t* rgb8, uint32_t width, uint32_t height) {
    if (!path || (!rgb8 && width && height)) return SPT_ERR_INVALID_ARGUMENT;
    std::ofstream f(path);
    if (!f) return SPT_ERR_INVALID_ARGUMENT;
    f << "P3" << std::endl << width << " " << height << std::endl << 255 << std::endl;
    const uint64_t n = 3ull * width * height;
    for (uint64_t i = 0; i < n; ++i) f << static_cast<int>(rgb8[i]) << " ";
    return f ? SPT_OK : SPT_ERR_INTERNAL;
}

}  // extern "C"
