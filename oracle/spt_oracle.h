/*
 * spt_oracle.h -- TEST INFRASTRUCTURE ONLY: the project's CPU restatement of the reference
 * renderer's hot path, used as the checker for the CUDA backend.  Nothing in the product
 * links, loads or calls this library; only tests/, the smoke check and the benchmark's
 * CPU-baseline leg do.
 *
 * Parity status: the geometric path (SAH tree, slab test, Moller-Trumbore, sphere,
 * traversal order and counts, camera rays) is pinned against the reference's own sources
 * compiled by `make -C oracle ref` (oracle/_ref) and against the committed fixtures in
 * tests/golden.  The path tracer uses the project's Philox-4x32-10 streams (the same ones
 * the CUDA kernels draw), so it is pinned to the reference statistically (converged
 * images), not sample by sample.
 */
#ifndef SPT_ORACLE_H
#define SPT_ORACLE_H

#include "../include/spt.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Philox-4x32-10 block (Salmon et al., SC'11): out[4] = philox(ctr[4], key[2]). */
void spto_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

void* spto_scene_create(const spt_scene_desc* desc);
void spto_scene_destroy(void* scene);
/* Reference full-sweep SAH build (acceleration/sbvh.cpp:12-37, 58-421). */
int spto_bvh_build(void* scene);
int spto_tree_stats(void* scene, spt_bvh_stats* out);
int spto_tree_export(void* scene, spt_bvh2_node* nodes, uint64_t* n_nodes, uint32_t* refs, uint64_t* n_refs);
/* Scene::intersect in the reference's traversal order (sbvh.cpp:478-510 or
 * no_accel_structure.cpp:9-30).  Any output may be NULL. */
int spto_intersect(void* scene, const float* rays, uint64_t n, spt_hit* hits, float* normals, uint32_t* tests,
                   uint32_t* nhits, int n_threads);
/* Camera::getRay at every pixel centre, row-major [y][x]. */
int spto_camera_rays(const spt_camera* cam, float* rays);
/* RayCaster<T>::render for one mode (integrators/raycaster.h:62-99), out as spt_raycast_image. */
int spto_raycast(void* scene, const spt_camera* cam, int32_t mode, void* out, spt_render_stats* stats, int n_threads);
/* Path tracer with the project's Philox sample streams; out = mean radiance float[h][w][3]. */
int spto_pathtrace(void* scene, const spt_camera* cam, const spt_pt_params* p, float* out, int n_threads,
                   double* seconds, uint64_t* segments);
/* Material::evalBSDF (materials/material.cpp:6-9) for n outgoing directions, drawing from the
 * stream of (path_index, depth).  out per direction: f rgb, reflectance rgb, pdf, wi xyz. */
int spto_eval_material(void* scene, uint32_t material, const float* wo, uint64_t n, float* out, uint64_t seed,
                       uint64_t path_index0, uint32_t depth);
/* Depth-mode and count-mode image normalisation of saveImageToFile
 * (integrators/depth_raycaster.cpp:9-34, int_test_count_raycaster.cpp:20-73); rgb out float[h][w][3]. */
int spto_depth_to_rgb(const float* depth, uint32_t w, uint32_t h, float min_d, float max_d, float* rgb);
int spto_count_to_rgb(const int64_t* count, uint32_t w, uint32_t h, int64_t min_c, int64_t max_c, uint64_t min_pp,
                      uint64_t max_pp, float* rgb);

#ifdef __cplusplus
}
#endif

#endif /* SPT_ORACLE_H */
