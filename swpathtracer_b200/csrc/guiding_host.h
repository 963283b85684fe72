// guiding_host.h -- host-side state of the path-guiding model (guiding.cu).
#pragma once

#include <vector>

#include "guiding.cuh"
#include "spt_internal.h"

namespace spt {
namespace guide {

size_t infer_smem_bytes();
size_t train_smem_bytes();
size_t train_tc_smem_bytes();
size_t train_tc_image_bytes();
// launchers of guiding.cu's helper kernels, for the tensor-memory training path (guiding_tc.cu)
void k_mean_weight_launch(const float4* d_rec, uint32_t n, float* out, cudaStream_t s);
void k_reduce_launch(const float* partial, uint32_t chunks, uint32_t count, float* out, cudaStream_t s);

struct Guide {
    spt_context* ctx = nullptr;
    spt_guide_config cfg{};
    Model model{};
    float *grid_master = nullptr, *grid_m = nullptr, *grid_v = nullptr, *grid_grad = nullptr;
    __nv_bfloat16* grid_bf16 = nullptr;
    float *mlp_master = nullptr, *mlp_m = nullptr, *mlp_v = nullptr, *mlp_grad = nullptr;
    __nv_bfloat16* smem_image = nullptr;
    float* scalars = nullptr;  // [0] mean weight, [1] loss sum
    uint32_t steps = 0;
    std::vector<void*> allocations;
    // training scratch
    __nv_bfloat16* xt[kLayers] = {};
    __nv_bfloat16* dzt[kLayers] = {};
    float* partial = nullptr;
    uint32_t train_cap = 0;
    std::vector<void*> train_allocs;
    // training on the tensor-memory kernels (guiding_tc.cu): the bf16 weight image in the core-matrix
    // layout, the records' grid features, the feature gradients and one dW partial per CTA
    unsigned char* tc_image = nullptr;
    float* tc_partial = nullptr;
    uint32_t* tc_feats = nullptr;
    float* tc_dx0 = nullptr;
    uint32_t tc_cap = 0;
    // inference scratch: the hash-grid features of up to feats_cap samples (k_encode -> k_infer)
    uint32_t* feats = nullptr;
    uint32_t feats_cap = 0;
    // the mixture cached per (cell of a cache_res^3 grid over the box, normal axis): what guided
    // rendering samples.  Filled whole when the guide is created; after that a refresh re-evaluates
    // only the entries guided renders have looked up (touched), kCacheChunk entries per network pass.
    // An entry not refreshed keeps an earlier mixture of the guide, which sampling and density read
    // alike, so the estimator stays unbiased; a refresh is skipped while the parameters are unchanged.
    static constexpr uint32_t kCacheRes = 128;           // cells per axis unless the config names another
    static constexpr uint32_t kCacheChunk = 1u << 20;    // entries per network pass of a refresh
    uint32_t cache_res = kCacheRes;
    uint32_t n_cache = 0;          // cache_res^3 * 6
    float* cache = nullptr;        // n_cache entries of kCacheEntry floats
    float* cache_raw = nullptr;    // one chunk of entries as decoded lobes (40 floats), before packing
    float4* cache_in = nullptr;    // the network inputs of one chunk
    uint8_t* touched = nullptr;    // n_cache flags set by guided shading at every entry it reads
    uint32_t* cache_list = nullptr;   // the touched entries of a refresh, then their count at [n_cache]
    bool touched_any = false;      // a guided render has run with this guide (touched is meaningful)
    uint64_t version = 0;          // bumped by every change of the parameters
    uint64_t cache_version = ~0ull;   // the parameter version the cache was last refreshed at

    spt_status alloc(spt_context* c, const spt_guide_config& cfg);
    spt_status refresh();
    spt_status infer(const float4* d_in, uint32_t n, float* d_out, cudaStream_t s);
    // inference for a device-side count of samples (at most max_n); usable inside a CUDA graph
    // (ensure_features(max_n) first, outside any stream capture)
    spt_status infer_list(const float4* d_in, const uint32_t* d_n, uint32_t max_n, float* d_out, cudaStream_t s);
    spt_status ensure_features(uint32_t n);
    spt_status refresh_cache();
    spt_status ensure_train_buffers(uint32_t n);
    spt_status gradients(const float4* d_rec, uint32_t n);
    spt_status gradients_tc(const float4* d_rec, uint32_t n);
    spt_status ensure_tc_buffers(uint32_t n);
    spt_status stage_tc();
    spt_status step(const float4* d_rec, uint32_t n, float* loss);
    ~Guide() {
        if (tc_feats) cudaFree(tc_feats);
        if (tc_dx0) cudaFree(tc_dx0);
        if (feats) cudaFree(feats);
        if (cache) cudaFree(cache);
        if (cache_raw) cudaFree(cache_raw);
        if (cache_in) cudaFree(cache_in);
        if (touched) cudaFree(touched);
        if (cache_list) cudaFree(cache_list);
        for (void* p : train_allocs) cudaFree(p);
        for (void* p : allocations) cudaFree(p);
    }
};

}  // namespace guide
}  // namespace spt

struct spt_guide {
    spt::guide::Guide g;
};
