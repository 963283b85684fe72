/*
 * spt.h -- C-ABI of the B200 (sm_100a) path-tracing backend.
 *
 * This is the drop-in boundary: the reference renderer's C++ interfaces
 * (AccelStructure, Integrator, BSDF/LayeredBSDF/Material, Camera, PixelSampler,
 * ImageBuffer) are served by the entry points below.  Every signature uses plain
 * pointers, sizes and POD structs; no C++ or torch types cross it, and no C++
 * exception crosses it (every entry point returns an spt_status).
 *
 * Conventions
 *   - Host pointers unless the name ends in _device; *_device entry points take
 *     device pointers and a cudaStream_t passed as void*, and return without
 *     synchronising.
 *   - Images are row-major [y][x] (row 0 = top), RGB triplets of float.  The
 *     reference stores ImageBuffer pixels as [x][y] (core/image_buffer.h:51); only
 *     the memory order differs, pixel (x, y) means the same pixel.
 *   - Primitive ids are indices into spt_scene_desc's primitive list, in the order
 *     the primitives were given (the reference's Scene::primitives_ order,
 *     core/scene.h:87).  A miss is reported as SPT_MISS.
 *   - Rays are 8 floats: origin xyz, pad, direction xyz, pad (two float4s).  Like
 *     the reference's Ray (core/ray.h:6-19) they carry no t range: a hit is any
 *     t > 0 (acceleration/sbvh.cpp:494-496).
 */
#ifndef SPT_H
#define SPT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPT_ABI_VERSION 2u
#define SPT_MISS 0xFFFFFFFFu

typedef enum spt_status {
    SPT_OK = 0,
    SPT_ERR_INVALID_ARGUMENT = 1,
    SPT_ERR_CUDA = 2,
    SPT_ERR_OUT_OF_MEMORY = 3,
    SPT_ERR_OVERFLOW = 4,      /* a queue or stack capacity was exceeded; results are incomplete */
    SPT_ERR_TIMEOUT = 5,       /* a bounded device loop ran out of iterations */
    SPT_ERR_UNSUPPORTED = 6,
    SPT_ERR_INTERNAL = 7
} spt_status;

/* Primitive kinds (reference primitives/triangle.h, smooth_triangle.h, sphere.h). */
enum { SPT_PRIM_TRIANGLE = 0, SPT_PRIM_SMOOTH_TRIANGLE = 1, SPT_PRIM_SPHERE = 2 };

/* BSDF kinds (reference materials/lambertian.h, smooth_conductor.h, smooth_dielectric.h,
 * cook_torrance.h) and their sampler choice (reference lua_core/bsdfs.lua:8, the
 * "uniform"/"importance" field; core/swpathtracer_app.cpp:89-149 maps it to a sampler). */
enum { SPT_BSDF_LAMBERTIAN = 0, SPT_BSDF_SMOOTH_CONDUCTOR = 1, SPT_BSDF_SMOOTH_DIELECTRIC = 2,
       SPT_BSDF_COOK_TORRANCE = 3 };
enum { SPT_SAMPLER_UNIFORM = 0, SPT_SAMPLER_IMPORTANCE = 1 };

/* Acceleration structure kinds (reference acceleration/accel_structure.h:17). BVH_SAH and
 * SBVH_SAH build the same tree: the spatial-split half of the reference is disabled. */
enum { SPT_ACCEL_NONE = 0, SPT_ACCEL_BVH_SAH = 1, SPT_ACCEL_SBVH_SAH = 2 };

/* Camera kinds (reference cameras/camera.h:14) and pixel samplers (pixel_samplers/pixel_sampler.h:8). */
enum { SPT_CAMERA_PINHOLE = 0, SPT_CAMERA_ORTHOGRAPHIC = 1 };
enum { SPT_PIXEL_UNIFORM = 0, SPT_PIXEL_REGULAR = 1, SPT_PIXEL_JITTERED = 2 };

/* Ray-caster pixel values (reference integrators/normal_raycaster.h, depth_raycaster.h,
 * int_test_count_raycaster.h). */
enum { SPT_RAYCAST_NORMAL = 0, SPT_RAYCAST_DEPTH = 1, SPT_RAYCAST_COUNT = 2 };

/* Path termination (reference integrators/pathtracer.h:13). */
enum { SPT_TERMINATE_MAX_DEPTH = 0, SPT_TERMINATE_RUSSIAN_ROULETTE = 1 };

/* One BSDF layer.  rgb: Lambertian kd, conductor / Cook-Torrance reflectance at normal
 * incidence.  scalar: dielectric IOR, Cook-Torrance roughness (Beckmann m). */
typedef struct spt_bsdf {
    int32_t type;
    int32_t sampler;
    float rgb[3];
    float scalar;
} spt_bsdf;

/* Material = layered BSDF + emission (reference materials/material.h:8-20). */
typedef struct spt_material {
    uint32_t layered_bsdf;
    float emission[3];
} spt_material;

/* Scene description (reference core/scene.h:22-90 + the Lua records that fill it).
 * prim_data: 9 floats per primitive -- triangle v0 v1 v2, or sphere centre xyz, radius,
 * 5 unused.  prim_normals: 9 floats per primitive (n0 n1 n2, used by smooth triangles);
 * may be NULL when no smooth triangle is present.  layered_offsets has n_layered + 1
 * entries into layered_bsdf_ids (top layer first, reference materials/layered_bsdf.cpp:20-23). */
typedef struct spt_scene_desc {
    uint32_t n_prims;
    const uint8_t* prim_type;
    const float* prim_data;
    const float* prim_normals;
    const uint32_t* prim_material;
    uint32_t n_bsdfs;
    const spt_bsdf* bsdfs;
    uint32_t n_layered;
    const uint32_t* layered_offsets;
    const uint32_t* layered_bsdf_ids;
    uint32_t n_materials;
    const spt_material* materials;
    float background[3];
    int32_t accel;
} spt_scene_desc;

/* Camera + image buffer (reference cameras/pinhole_camera.h, orthographic_camera.h,
 * core/image_buffer.h).  fov_deg is the vertical field of view. */
typedef struct spt_camera {
    int32_t type;
    float position[3];
    float look_at[3];
    float up[3];
    float fov_deg;
    float min_x, max_x, min_y, max_y;
    uint32_t width, height;
    uint32_t vp_top, vp_left, vp_width, vp_height;
} spt_camera;

/* Path tracer settings (reference integrators/pathtracer.h:15-17 + lua_core/integrators.lua).
 * max_depth: hard cap on surface interactions in russian-roulette mode; 0 means the
 * reference's cap of 1000 bounces (integrators/pathtracer.cpp:44-45).  seed keys the
 * counter-based Philox-4x32-10 generator that replaces the reference's per-thread
 * mt19937 (core/prng.h).  spp_offset shifts the sample index so progressive passes
 * draw fresh numbers. */
typedef struct spt_pt_params {
    int32_t pixel_sampler;
    uint32_t spp;
    int32_t termination;
    int32_t path_length;
    int32_t max_depth;
    uint32_t spp_offset;
    uint64_t seed;
} spt_pt_params;

/* Closest hit of one ray (reference core/intersection_record.h:6-12).  prim_id is
 * SPT_MISS on a miss; then t = +inf.  u, v: barycentrics for triangles, 0 for spheres. */
typedef struct spt_hit {
    float t;
    uint32_t prim_id;
    float u, v;
} spt_hit;

/* Per-image statistics of the ray casters / path tracer (reference integrators/integrator.h:47-54). */
typedef struct spt_render_stats {
    uint64_t int_tests;
    uint64_t int_hits;
    uint64_t min_tests_pp, max_tests_pp;
    uint64_t min_hits_pp, max_hits_pp;
    uint64_t paths;       /* camera paths traced */
    uint64_t segments;    /* ray segments traced (extend launches' rays) */
    double gpu_ms;        /* device time of the render, CUDA events */
} spt_render_stats;

/* Flattened binary SAH tree (reference acceleration/sbvh.cpp:58-421).  Nodes in depth-first,
 * left-first order: node i's left child is i + 1.  For inner nodes right = index of the right
 * child and count = 0; for leaves right = first index into ref_prim and count = number of
 * references.  Boxes are the reference's node AABBs (children inflated by 1e-3,
 * acceleration/sbvh.cpp:409-412). */
typedef struct spt_bvh2_node {
    float min[3];
    uint32_t right;
    float max[3];
    uint32_t count;
} spt_bvh2_node;

typedef struct spt_bvh_stats {
    uint64_t num_nodes, num_inner_nodes, num_leaf_nodes, tree_height;
    uint64_t min_prims_leaf, max_prims_leaf, num_references, num_unreferenced;
    double build_ms;
} spt_bvh_stats;

typedef struct spt_context spt_context;
typedef struct spt_scene spt_scene;
typedef struct spt_bvh spt_bvh;

/* ---- library / context --------------------------------------------------------------- */
uint32_t spt_abi_version(void);
/* Creates a context on CUDA device `device` (Integrator/Scene owner; reference
 * core/swpathtracer_app.cpp:29-37 plays this role on the CPU).  A context serves one host thread at
 * a time: its scratch buffers, per-stream buffers and counter ring are not locked, so host threads
 * that call concurrently take a context each (or serialise their calls).  Device work that one
 * thread queues on different streams of a context may overlap. */
spt_status spt_create(int device, spt_context** out);
spt_status spt_destroy(spt_context* ctx);
/* Text of the last error on this context (never NULL). */
const char* spt_last_error(const spt_context* ctx);

/* ---- acceleration structure (reference acceleration/accel_structure.h:15-35) --------- */
/* Host build of the reference's full-sweep SAH tree, node for node
 * (acceleration/sbvh.cpp:12-37, 58-421); n_threads <= 0 uses all cores. */
spt_status spt_bvh_build(const spt_scene_desc* desc, int n_threads, spt_bvh** out);
/* Device build of a binary SAH-quality tree in the same layout (Morton order + parallel
 * locally-ordered clustering + SAH leaf collapse), in milliseconds instead of the host build's
 * seconds.  It replaces SBVH::build (acceleration/sbvh.cpp:12-37) where the reference's exact tree is
 * not needed: closest hits are the same except the choice between primitives hit at an equal t, and
 * hit counts are this tree's.  Deterministic for a given input. */
spt_status spt_bvh_build_device(spt_context* ctx, const spt_scene_desc* desc, spt_bvh** out);
spt_status spt_bvh_stats_get(const spt_bvh* bvh, spt_bvh_stats* out);   /* SBVH::getStatistics, sbvh.h:72 */
/* Copies the flattened tree out; either array may be NULL to query sizes only. */
spt_status spt_bvh_export(const spt_bvh* bvh, spt_bvh2_node* nodes, uint64_t* n_nodes,
                          uint32_t* ref_prim, uint64_t* n_refs);
spt_status spt_bvh_free(spt_bvh* bvh);

/* ---- scene upload (reference core/scene.h:22-90) --------------------------------------- */
/* Copies the scene to the device.  bvh may be NULL: the tree is then built here
 * (Scene::buildAccelStructure, core/scene.cpp:79-81). */
spt_status spt_scene_create(spt_context* ctx, const spt_scene_desc* desc, const spt_bvh* bvh,
                            spt_scene** out);
spt_status spt_scene_destroy(spt_scene* scene);
/* Device bytes held by the scene (nodes, triangles, materials). */
uint64_t spt_scene_device_bytes(const spt_scene* scene);

/* ---- ray queries (reference AccelStructure::intersect, accel_structure.h:29-30) ------- */
/* Closest hit for n rays.  tests/hits (may be NULL): the reference's per-ray
 * num_intersection_tests / num_intersections (sbvh.cpp:478-510), which come from a
 * separate exhaustive binary-tree pass. */
spt_status spt_intersect(spt_context* ctx, const spt_scene* scene, const float* rays, uint64_t n,
                         spt_hit* hits, uint32_t* tests, uint32_t* nhits);
/* spt_intersect for rays laid out as the reference's Ray (core/ray.h: origin then direction, two
 * glm::vec3, 24 bytes per ray), so a batch of reference Rays is passed as it lies in memory; it
 * moves a quarter fewer bytes to the device than the padded 32-byte layout. */
spt_status spt_intersect_packed(spt_context* ctx, const spt_scene* scene, const float* rays, uint64_t n,
                                spt_hit* hits, uint32_t* tests, uint32_t* nhits);
/* Device rays (8 floats each) and hits, on `stream` (NULL: the legacy default stream).  A batch of at
 * least 2^21 rays on a scene with the 8-wide tree is traced in coherence order (neighbouring rays
 * enter the scene's box near each other with similar directions; misses last), which makes the
 * traversal's warps diverge less; the hits are the same in any order.  Its working buffers belong to
 * the stream (one set per stream for up to eight streams; a ninth stream's batches keep their own
 * order).  The three stages are also callable one by one (n < 2^32 rays): */
spt_status spt_intersect_device(spt_context* ctx, const spt_scene* scene, const float* d_rays,
                                uint64_t n, spt_hit* d_hits, void* stream);
/* 1. The coherence order of n device rays (8 floats each) into d_order (2n + 1 entries): d_order[2n]
 *    = m, the number of rays that meet the scene's root box; d_order[k], k < m, the index of the k-th
 *    of them to trace; d_order[n + i] the place of ray i in that order, or 0xFFFFFFFF for a ray the
 *    root box test rejects (SPT_ERR_UNSUPPORTED when eight other streams hold the working buffers). */
spt_status spt_ray_order_device(spt_context* ctx, const spt_scene* scene, const float* d_rays, uint64_t n,
                                uint32_t* d_order, void* stream);
/* 2. Closest hits of the rays d_rays[d_order[k]] into d_hits_ordered[k], k < d_order[2n], on the
 *    persistent 8-wide traversal (SPT_ERR_UNSUPPORTED for a scene on another traversal).  d_order
 *    must come from stage 1 for the same rays and the same scene: a ray it leaves out is taken to
 *    miss that scene's root box. */
spt_status spt_intersect_ordered_device(spt_context* ctx, const spt_scene* scene, const float* d_rays,
                                        const uint32_t* d_order, uint64_t n, spt_hit* d_hits_ordered,
                                        void* stream);
/* 3. d_hits[i] = d_hits_ordered[d_order[n + i]], or the miss record (t = +inf, SPT_MISS, u = v = 0)
 *    for a ray without a place: every hit back at its ray's index. */
spt_status spt_hits_unorder_device(spt_context* ctx, const uint32_t* d_order, uint64_t n,
                                   const spt_hit* d_hits_ordered, spt_hit* d_hits, void* stream);
/* The reference's own traversal order (unordered, unpruned, depth first): per-ray test counts
 * (box + primitive tests, and the primitive tests alone) and, when d_ref_hits is not NULL, the
 * hit that traversal keeps.  Any output may be NULL. */
spt_status spt_count_device(spt_context* ctx, const spt_scene* scene, const float* d_rays,
                            uint64_t n, spt_hit* d_ref_hits, uint32_t* d_tests, uint32_t* d_hits,
                            uint32_t* d_prim_tests, void* stream);

/* The work of the closest-hit kernel itself (no reference counterpart; the reference's own work per
 * ray is what spt_count_device counts): spt_intersect_device's persistent kernel on n device rays
 * (8 floats each), with work[0] = 8-wide node visits (each tests up to eight child boxes) and
 * work[1] = primitive tests, summed over the rays.  The hits are the same as spt_intersect_device's.
 * Returns after the counts are in host memory. */
spt_status spt_traversal_work_device(spt_context* ctx, const spt_scene* scene, const float* d_rays, uint64_t n,
                                     spt_hit* d_hits, uint64_t* work);

/* ---- integrators (reference integrators/integrator.h:8-55) ----------------------------- */
/* Ray casters, one ray per pixel centre (integrators/raycaster.h:62-99).  out_host layout:
 * NORMAL float[h][w][3] (0 on a miss), DEPTH float[h][w] (-1 on a miss), COUNT int64[h][w]. */
spt_status spt_raycast_image(spt_context* ctx, const spt_scene* scene, const spt_camera* cam,
                             int32_t mode, void* out_host, spt_render_stats* stats);
spt_status spt_raycast_image_device(spt_context* ctx, const spt_scene* scene, const spt_camera* cam,
                                    int32_t mode, void* d_out, void* stream);
/* Path tracer (integrators/pathtracer.cpp:12-147).  out_rgb_host: float[h][w][3], the mean
 * radiance per pixel over spp samples (before the sRGB conversion of saveImageToFile);
 * pixels outside the viewport are 0. */
spt_status spt_pathtrace(spt_context* ctx, const spt_scene* scene, const spt_camera* cam,
                         const spt_pt_params* params, float* out_rgb_host, spt_render_stats* stats);
spt_status spt_pathtrace_device(spt_context* ctx, const spt_scene* scene, const spt_camera* cam,
                                const spt_pt_params* params, float* d_out_rgb, spt_render_stats* stats);

/* ---- batched rendering and tuning (no reference counterpart) ---------------------------------
 * Many scenes of uneven size and resolution rendered by one wavefront: the camera paths of all jobs
 * share one pool of path slots and the iterations are replayed from one CUDA graph.  Each job's image
 * is what spt_pathtrace_device would produce for it alone (up to float-add order).  */
typedef struct spt_tune {
    uint32_t capacity;      /* path slots in the wavefront pool */
    uint32_t extend_block;  /* threads per block of the non-persistent extend kernel */
    uint32_t shade_block;   /* threads per block of the shade kernel */
    int32_t traversal;      /* -1 scene default, 0 binary pair nodes, 1 8-wide, 2 8-wide + dynamic fetch */
    uint32_t check_every;   /* guided renders that train: wavefront iterations between the host's looks
                               at the training records.  Every other render runs its whole loop on the
                               device (a conditional WHILE node of one CUDA graph) */
    uint32_t sort_shading;  /* shade the paths grouped by material class: 0 when a scene has layered
                               materials (their walks diverge most), 1 always, 2 never */
    uint32_t stack;         /* traversal stack depth per lane of the persistent extend kernel: 16, 24 or
                               32 entries; 0 = the smallest that holds every scene's 8-wide tree */
    uint32_t stack_limit;   /* stack entries a lane may use (0 = all of `stack`); a traversal that needs
                               more ends the render with SPT_ERR_OVERFLOW */
    uint32_t max_iterations;/* wavefront iterations before the render gives up with SPT_ERR_TIMEOUT;
                               0 = a bound from the path count and the 1000-bounce roulette cap */
    uint32_t host_loop;     /* 1: the host replays a graph of two wavefront iterations and reads the
                               counters every check_every iterations (the loop guided training uses)
                               instead of the device-side WHILE loop; for tools that cannot look into
                               graphs with conditional nodes, such as kernel profilers.  0 = default */
} spt_tune;

typedef struct spt_batch_job {
    const spt_scene* scene;
    spt_camera camera;
    spt_pt_params params;
} spt_batch_job;

spt_status spt_tune_default(spt_tune* out);
/* d_images[i]: device float[h][w][3] of job i.  stats (may be NULL): one per job; paths is the job's,
 * segments and gpu_ms are the whole batch's.  tune may be NULL (defaults). */
spt_status spt_batch_pathtrace(spt_context* ctx, const spt_batch_job* jobs, uint32_t n_jobs, float* const* d_images,
                               const spt_tune* tune, spt_render_stats* stats);
/* Times short trial renders of the batch (a few samples per pixel) under candidate settings and
 * returns the fastest.  cache_path (may be NULL): a text file of earlier results keyed by the
 * device name and the batch's shape; a hit skips the trials. */
spt_status spt_autotune(spt_context* ctx, const spt_batch_job* jobs, uint32_t n_jobs, const char* cache_path,
                        spt_tune* out);

/* ---- neural path guiding (no reference counterpart) -------------------------------------------
 * A learned sampling distribution over directions, mixed with BSDF sampling by one-sample MIS:
 * a multiresolution hash grid (16 levels x 2 features, 2^19 entries per level) encodes the position,
 * a 4-hidden-layer ReLU MLP of width 64 (bf16 tensor-core GEMMs, fp32 accumulation) maps it with the
 * normal and outgoing direction to 8 von Mises-Fisher lobes.  Trained online by Adam on the
 * radiance the path tracer itself collects. */
enum { SPT_GUIDE_TRAIN_TCGEN05 = 0, SPT_GUIDE_TRAIN_MMA_SYNC = 1 };

typedef struct spt_guide_config {
    float box_min[3], box_max[3];  /* positions are normalised by this box (e.g. the scene bounds) */
    float lr;                      /* Adam learning rate */
    uint32_t batch;                /* training records per optimiser step */
    uint32_t max_steps;            /* optimiser steps per guided render before the model is frozen: a
                                      render takes one step per 10 batches of its camera paths, at
                                      least one, at most max_steps (0: the guide stays frozen) */
    float mix;                     /* probability of sampling the guiding distribution */
    uint64_t seed;                 /* parameter initialisation */
    uint32_t cache_res;            /* cells per axis of the lobe cache guided renders sample: 4..128, 0 = 128
                                      (6 normal axes per cell, 192 bytes per entry: 2.4 GB at 128) */
    uint32_t train_path;           /* SPT_GUIDE_TRAIN_TCGEN05 (0): the MLP's training GEMMs on the 5th-gen
                                      tensor cores, tiles of 128 records with fp32 accumulators in tensor
                                      memory; SPT_GUIDE_TRAIN_MMA_SYNC (1): warp-level mma.sync tiles of
                                      32 records */
    uint32_t guided_depth;         /* vertices guided per path: those at depth < guided_depth (the camera
                                      ray's hit is depth 0); 0 = every vertex */
    uint32_t reserved;             /* must be 0 */
} spt_guide_config;

/* One training record: a scattering event and the radiance it led to. */
typedef struct spt_guide_record {
    float pos[3], weight;          /* weight: the record's estimate of f*cos*Li/pdf (luminance) */
    float normal[3], pad0;
    float wo[3], pad1;             /* outgoing (towards the previous vertex), world space */
    float wi[3], pad2;             /* sampled incident direction, world space */
} spt_guide_record;

typedef struct spt_guide spt_guide;

spt_status spt_guide_create(spt_context* ctx, const spt_guide_config* cfg, spt_guide** out);
spt_status spt_guide_destroy(spt_guide* guide);
/* Master parameters (fp32): grid [16][2^19][2] and the MLP weights, layer by layer [out][in]
 * (48->64, 64->64 x3, 64->48).  Either pointer may be NULL. */
spt_status spt_guide_get_params(spt_guide* guide, float* grid, float* mlp);
spt_status spt_guide_set_params(spt_guide* guide, const float* grid, const float* mlp);
/* Mixture for n samples (host arrays): in 12 floats each (pos, 0, normal, 0, wo, 0 as float4s);
 * out 40 floats each: 8 lobes x {mu.xyz, kappa, weight}. */
spt_status spt_guide_eval(spt_context* ctx, spt_guide* guide, const float* in, uint32_t n, float* out);
/* Gradients of the mean weighted negative log-likelihood of n records (host), without updating. */
spt_status spt_guide_gradients(spt_context* ctx, spt_guide* guide, const spt_guide_record* recs, uint32_t n,
                               float* grid_grad, float* mlp_grad, float* loss);
/* One Adam step on n records (host). */
spt_status spt_guide_train(spt_context* ctx, spt_guide* guide, const spt_guide_record* recs, uint32_t n, float* loss);
/* One Adam step on n records already in device memory (the spt_guide_record layout, 64 bytes each);
 * gpu_ms (may be NULL): the step's device time.  Returns after the step has finished. */
spt_status spt_guide_train_device(spt_context* ctx, spt_guide* guide, const spt_guide_record* d_recs, uint32_t n,
                                  float* gpu_ms);
/* Optimiser steps taken by the guide since it was created. */
spt_status spt_guide_steps(spt_guide* guide, uint64_t* steps);
/* Guided path tracing: as spt_pathtrace_device, sampling guidable vertices from mix * guide +
 * (1 - mix) * BSDF (single-layer Lambertian / Cook-Torrance; a smooth dielectric over Cook-Torrance
 * through its walk's single-internal-bounce component), and training the guide on its own paths (the
 * step budget of spt_guide_config.max_steps). */
spt_status spt_guided_pathtrace_device(spt_context* ctx, const spt_scene* scene, const spt_camera* cam,
                                       const spt_pt_params* params, spt_guide* guide, float* d_out_rgb,
                                       spt_render_stats* stats);

/* ---- image post-processing (reference core/image_buffer.cpp and the ray casters' saveImageToFile) */
/* DepthRayCaster::saveImageToFile (integrators/depth_raycaster.cpp:9-34) on the device: d_depth float[h][w]
 * (-1 = background) -> d_rgb float[h][w][3] grey ramp; min_depth / max_depth = -1 take the image's own
 * (min over hits, max over all pixels). */
spt_status spt_depth_to_rgb_device(spt_context* ctx, const float* d_depth, uint32_t width, uint32_t height,
                                   float min_depth, float max_depth, float* d_rgb, void* stream);
/* IntTestCountRayCaster::saveImageToFile (int_test_count_raycaster.cpp:20-73): d_count int64[h][w] ->
 * HSL heat map; min_count / max_count = -1 take the image's own per-pixel min / max. */
spt_status spt_count_to_rgb_device(spt_context* ctx, const int64_t* d_count, uint32_t width, uint32_t height,
                                   int64_t min_count, int64_t max_count, float* d_rgb, void* stream);
/* NormalRayCaster::saveImageToFile (integrators/normal_raycaster.cpp:6-17), in place on a normal image:
 * n * 0.5 + 0.5 for every pixel that is not background (0, 0, 0). */
spt_status spt_normal_to_rgb_device(spt_context* ctx, float* d_rgb, uint32_t width, uint32_t height, void* stream);
/* ImageBuffer::convertTosRGB (when to_srgb) + the clamp / int(c * 255 + 0.5) of saveToFile, per value. */
spt_status spt_rgb_to_bytes_device(spt_context* ctx, const float* d_rgb, uint64_t n_values, int32_t to_srgb,
                                   uint8_t* d_bytes, void* stream);
/* The ASCII P3 file of saveToFile from already quantized bytes (host memory). */
spt_status spt_write_ppm_bytes(const char* path, const uint8_t* rgb8, uint32_t width, uint32_t height);
/* sRGB (pow 1/2.2 of the clamped value) + ASCII P3 PPM writer, core/image_buffer.cpp:22-47. */
spt_status spt_write_ppm(const char* path, const float* rgb, uint32_t width, uint32_t height, int32_t to_srgb);

#ifdef __cplusplus
}
#endif

#endif /* SPT_H */
