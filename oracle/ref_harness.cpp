// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY (oracle).  Never linked into the product.
//
// A C-callable driver around the reference renderer's OWN, unmodified C++ sources
// (acceleration/, primitives/, materials/, bsdf_samplers/, cameras/, pixel_samplers/,
// integrators/, core/{ray,onb,image_buffer,scene}.cpp), compiled by oracle/Makefile
// into oracle/_ref/libswref.so.  Lua and Assimp are absent here, so scenes are built
// directly from an spt_scene_desc instead of a Lua script (the object graph is the one
// core/swpathtracer_app.cpp:67-259 builds), and glm is replaced by the project-written
// subset in oracle/shim/glm.
//
// Additions that do not change the reference's arithmetic:
//  * Id* primitive subclasses override the virtual Primitive::intersect
//    (primitives/primitive.h:15), call the reference implementation and record the
//    primitive's index in IntersectionRecord::primitive_id_, which the reference
//    declares (core/intersection_record.h:11) but never writes.
//  * SBVH's private tree is read through an access macro to export it node for node;
//    the build calls the reference's own splitNode/collectTreeStatistics exactly as
//    SBVH::build does (acceleration/sbvh.cpp:12-37) but skips its 100-MB text dump
//    unless a dump path is given (then the reference's dumpTree writes it).
//  * The PRNG engines are re-seeded deterministically (core/prng.h:22-25 seeds them
//    from std::random_device, which makes runs unrepeatable).

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <limits>
#include <memory>
#include <queue>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>
#include <omp.h>

#include "glm/glm.hpp"

#define private public
#define protected public
#include "sbvh.h"
#include "raycaster.h"
#undef private
#undef protected

#include "cook_torrance.h"
#include "cook_torrance_bsdf_sampler.h"
#include "cosine_bsdf_sampler.h"
#include "depth_raycaster.h"
#include "fresnel_schlick.h"
#include "int_test_count_raycaster.h"
#include "jittered_pixel_sampler.h"
#include "lambertian.h"
#include "layered_bsdf.h"
#include "material.h"
#include "no_accel_structure.h"
#include "normal_raycaster.h"
#include "orthographic_camera.h"
#include "pathtracer.h"
#include "pinhole_camera.h"
#include "refraction_bsdf_sampler.h"
#include "regular_pixel_sampler.h"
#include "scene.h"
#include "smooth_conductor.h"
#include "smooth_dielectric.h"
#include "smooth_specular_bsdf_sampler.h"
#include "smooth_triangle.h"
#include "sphere.h"
#include "triangle.h"
#include "uniform_bsdf_sampler.h"
#include "uniform_pixel_sampler.h"

#include "../include/spt.h"

namespace {

typedef PRNG<std::uniform_real_distribution, float, std::mt19937> RefPRNG;

thread_local std::uint64_t tl_tri_tests = 0;

class IdTriangle : public Triangle {
   public:
    IdTriangle(const glm::vec3& a, const glm::vec3& b, const glm::vec3& c, unsigned long m, std::size_t id)
        : Triangle(a, b, c, m), id_(id) {}
    bool intersect(const Ray& ray, IntersectionRecord& rec) override {
        ++tl_tri_tests;
        bool r = Triangle::intersect(ray, rec);
        if (r) rec.primitive_id_ = id_;
        return r;
    }
    std::size_t id_;
};

class IdSmoothTriangle : public SmoothTriangle {
   public:
    IdSmoothTriangle(const glm::vec3& a, const glm::vec3& b, const glm::vec3& c, const glm::vec3& na,
                     const glm::vec3& nb, const glm::vec3& nc, unsigned long m, std::size_t id)
        : SmoothTriangle(a, b, c, na, nb, nc, m), id_(id) {}
    bool intersect(const Ray& ray, IntersectionRecord& rec) override {
        ++tl_tri_tests;
        bool r = SmoothTriangle::intersect(ray, rec);
        if (r) rec.primitive_id_ = id_;
        return r;
    }
    std::size_t id_;
};

class IdSphere : public Sphere {
   public:
    IdSphere(const glm::vec3& c, float r, unsigned long m, std::size_t id) : Sphere(c, r, m), id_(id) {}
    bool intersect(const Ray& ray, IntersectionRecord& rec) override {
        ++tl_tri_tests;
        bool r = Sphere::intersect(ray, rec);
        if (r) rec.primitive_id_ = id_;
        return r;
    }
    std::size_t id_;
};

struct NullBuf : std::streambuf {
    int overflow(int c) override { return c; }
};

struct Silence {
    NullBuf nb;
    std::streambuf* o;
    std::streambuf* l;
    Silence() : o(std::cout.rdbuf(&nb)), l(std::clog.rdbuf(&nb)) {}
    ~Silence() {
        std::cout.rdbuf(o);
        std::clog.rdbuf(l);
    }
};

struct RefScene {
    std::unique_ptr<RefPRNG> prng;
    std::unique_ptr<Scene> scene;
    SBVH* sbvh = nullptr;  // owned by scene when accel != NONE
    int max_threads = 1;
    std::string error;
};

glm::vec3 v3(const float* p) { return glm::vec3(p[0], p[1], p[2]); }

void reseed(RefPRNG& prng, std::uint64_t seed) {
    for (std::size_t i = 0; i < prng.engines_.size(); ++i)
        prng.engines_[i].seed(static_cast<std::mt19937::result_type>(seed * 7919u + i * 104729u + 1u));
}

std::unique_ptr<Camera> make_camera(const spt_camera* c) {
    auto ib = std::make_unique<ImageBuffer>(c->width, c->height, c->vp_top, c->vp_left, c->vp_width, c->vp_height,
                                            std::string("/dev/null"));
    if (c->type == SPT_CAMERA_ORTHOGRAPHIC)
        return std::make_unique<OrthographicCamera>(v3(c->position), v3(c->look_at), v3(c->up), c->min_x, c->max_x,
                                                    c->min_y, c->max_y, std::move(ib));
    return std::make_unique<PinholeCamera>(v3(c->position), v3(c->look_at), v3(c->up), c->fov_deg, std::move(ib));
}

// Walks the reference tree depth-first, left first, flattening it in the node order the
// spt_bvh2_node format defines.
void flatten(const SBVHNode* n, std::vector<spt_bvh2_node>& nodes, std::vector<std::uint32_t>& refs) {
    std::size_t me = nodes.size();
    nodes.push_back(spt_bvh2_node{});
    const glm::vec3& mn = n->aabb_.getMin();
    const glm::vec3& mx = n->aabb_.getMax();
    nodes[me].min[0] = mn.x; nodes[me].min[1] = mn.y; nodes[me].min[2] = mn.z;
    nodes[me].max[0] = mx.x; nodes[me].max[1] = mx.y; nodes[me].max[2] = mx.z;
    if (!n->left_node_ && !n->right_node_) {
        nodes[me].right = static_cast<std::uint32_t>(refs.size());
        nodes[me].count = static_cast<std::uint32_t>(n->getNumReferences());
        for (std::size_t i = 0; i < n->getNumReferences(); ++i)
            refs.push_back(static_cast<std::uint32_t>(n->getActualPrimitiveId(i)));
        return;
    }
    flatten(n->left_node_.get(), nodes, refs);
    nodes[me].right = static_cast<std::uint32_t>(nodes.size());
    nodes[me].count = 0;
    flatten(n->right_node_.get(), nodes, refs);
}

}  // namespace

extern "C" {

// Builds the reference Scene for `d`.  dump_path: when non-NULL, the reference's own
// SBVH::dumpTree BFS text dump is written there (acceleration/sbvh.cpp:577-620).
void* swref_scene_create(const spt_scene_desc* d, const char* dump_path, int n_threads) {
    auto rs = std::make_unique<RefScene>();
    rs->max_threads = n_threads > 0 ? n_threads : omp_get_num_procs();
    omp_set_num_threads(rs->max_threads);
    rs->prng = std::make_unique<RefPRNG>(0.0f, 1.0f);
    reseed(*rs->prng, 1);
    RefPRNG& prng = *rs->prng;

    std::unique_ptr<AccelStructure> accel;
    if (d->accel == SPT_ACCEL_NONE)
        accel = std::make_unique<NoAccelStructure>();
    else {
        auto s = std::make_unique<SBVH>(std::numeric_limits<float>::infinity());
        rs->sbvh = s.get();
        accel = std::move(s);
    }
    rs->scene = std::make_unique<Scene>(std::move(accel), v3(d->background));
    Scene& sc = *rs->scene;

    // BSDFs (core/swpathtracer_app.cpp:89-149).
    for (std::uint32_t i = 0; i < d->n_bsdfs; ++i) {
        const spt_bsdf& b = d->bsdfs[i];
        std::unique_ptr<BSDF> bsdf;
        if (b.type == SPT_BSDF_LAMBERTIAN) {
            std::unique_ptr<BSDFSampler> smp;
            if (b.sampler == SPT_SAMPLER_UNIFORM) smp = std::make_unique<UniformBSDFSampler>(prng);
            else smp = std::make_unique<CosineBSDFSampler>(prng);
            bsdf = std::make_unique<Lambertian>(v3(b.rgb), std::move(smp));
        } else if (b.type == SPT_BSDF_SMOOTH_CONDUCTOR) {
            std::unique_ptr<BSDFSampler> smp;
            if (b.sampler == SPT_SAMPLER_UNIFORM) smp = std::make_unique<UniformBSDFSampler>(prng);
            else smp = std::make_unique<SmoothSpecularBSDFSampler>();
            bsdf = std::make_unique<SmoothConductor>(std::make_unique<FresnelSchlick>(v3(b.rgb)), std::move(smp));
        } else if (b.type == SPT_BSDF_SMOOTH_DIELECTRIC) {
            bsdf = std::make_unique<SmoothDielectric>(
                1.0f, b.scalar, std::make_unique<FresnelSchlick>(1.0f, b.scalar),
                std::make_unique<SmoothSpecularBSDFSampler>(), std::make_unique<RefractionBSDFSampler>(1.0f, b.scalar),
                prng);
        } else {
            std::unique_ptr<BSDFSampler> smp;
            if (b.sampler == SPT_SAMPLER_UNIFORM) smp = std::make_unique<UniformBSDFSampler>(prng);
            else smp = std::make_unique<CookTorranceBSDFSampler>(b.scalar, prng);
            bsdf = std::make_unique<CookTorrance>(b.scalar, std::make_unique<FresnelSchlick>(v3(b.rgb)), std::move(smp));
        }
        sc.addBSDF(std::move(bsdf));
    }
    // Layered BSDFs, emissions (one per material, in order), materials (swpathtracer_app.cpp:151-179).
    for (std::uint32_t i = 0; i < d->n_layered; ++i) {
        LayeredBSDF l;
        for (std::uint32_t k = d->layered_offsets[i]; k < d->layered_offsets[i + 1]; ++k)
            l.addBSDF(sc.getBSDFPtr(d->layered_bsdf_ids[k]));
        sc.addLayeredBSDF(l);
    }
    for (std::uint32_t i = 0; i < d->n_materials; ++i) sc.addEmission(v3(d->materials[i].emission));
    for (std::uint32_t i = 0; i < d->n_materials; ++i)
        sc.addMaterial(Material(sc.getLayeredBSDF(d->materials[i].layered_bsdf), sc.getEmission(i)));
    // Primitives (swpathtracer_app.cpp:181-219).
    for (std::uint32_t i = 0; i < d->n_prims; ++i) {
        const float* p = d->prim_data + 9ull * i;
        unsigned long m = d->prim_material[i];
        if (d->prim_type[i] == SPT_PRIM_TRIANGLE)
            sc.addPrimitive(std::make_unique<IdTriangle>(v3(p), v3(p + 3), v3(p + 6), m, i));
        else if (d->prim_type[i] == SPT_PRIM_SMOOTH_TRIANGLE) {
            const float* q = d->prim_normals + 9ull * i;
            sc.addPrimitive(std::make_unique<IdSmoothTriangle>(v3(p), v3(p + 3), v3(p + 6), v3(q), v3(q + 3),
                                                               v3(q + 6), m, i));
        } else
            sc.addPrimitive(std::make_unique<IdSphere>(v3(p), p[3], m, i));
    }
    // SBVH::build (acceleration/sbvh.cpp:12-37) without the unconditional dump.
    if (rs->sbvh) {
        Silence quiet;
        SBVH& s = *rs->sbvh;
        const auto& prims = *s.primitives_;
        if (!prims.empty()) {
            s.root_node_ = std::make_unique<SBVHNode>();
            s.root_node_->primitive_ref_list_ = std::make_unique<std::vector<PrimitiveRef>>();
            for (unsigned long i = 0; i < prims.size(); ++i) {
                s.root_node_->primitive_ref_list_->emplace_back(i, prims[i]->getAABB(), prims[i]->getCentroid());
                if (!i)
                    s.root_node_->aabb_ = (*s.root_node_->primitive_ref_list_)[i].aabb_;
                else
                    s.root_node_->aabb_ = s.root_node_->aabb_ + (*s.root_node_->primitive_ref_list_)[i].aabb_;
            }
            Timer timer;
            timer.start();
            s.splitNode(s.root_node_, s.root_node_->aabb_.getArea(), "", "none", "root");
            timer.finish();
            s.statistics_.build_time_ = timer.getElapsedTime();
            if (dump_path) s.dumpTree(dump_path);
            s.collectTreeStatistics();
        }
    }
    return rs.release();
}

void swref_scene_destroy(void* h) { delete static_cast<RefScene*>(h); }

int swref_tree_stats(void* h, spt_bvh_stats* out) {
    RefScene* rs = static_cast<RefScene*>(h);
    if (!rs->sbvh) return 1;
    const StatsSBVH& s = rs->sbvh->getStatistics();
    out->num_nodes = s.num_nodes_;
    out->num_inner_nodes = s.num_inner_nodes_;
    out->num_leaf_nodes = s.num_leaf_nodes_;
    out->tree_height = s.tree_height_;
    out->min_prims_leaf = s.min_num_primitives_leaf_;
    out->max_prims_leaf = s.max_num_primitives_leaf_;
    out->num_references = s.num_references_;
    out->num_unreferenced = s.num_unreferenced_primitives_;
    out->build_ms = s.build_time_ / 1000.0;
    return 0;
}

// Flattened tree; pass NULL arrays to query the sizes.
int swref_tree_export(void* h, spt_bvh2_node* nodes, std::uint64_t* n_nodes, std::uint32_t* refs,
                      std::uint64_t* n_refs) {
    RefScene* rs = static_cast<RefScene*>(h);
    if (!rs->sbvh || !rs->sbvh->root_node_) return 1;
    std::vector<spt_bvh2_node> nv;
    std::vector<std::uint32_t> rv;
    flatten(rs->sbvh->root_node_.get(), nv, rv);
    if (nodes) std::memcpy(nodes, nv.data(), nv.size() * sizeof(spt_bvh2_node));
    if (refs) std::memcpy(refs, rv.data(), rv.size() * sizeof(std::uint32_t));
    *n_nodes = nv.size();
    *n_refs = rv.size();
    return 0;
}

// Scene::intersect for each ray (core/scene.cpp:83-86 -> SBVH::intersect or
// NoAccelStructure::intersect), OpenMP-parallel over rays.  Any output may be NULL.
// normals: 3 floats per ray (IntersectionRecord::normal_); tri_tests: primitive tests only.
int swref_intersect(void* h, const float* rays, std::uint64_t n, spt_hit* hits, float* normals,
                    std::uint32_t* tests, std::uint32_t* nhits, std::uint32_t* prim_tests, int n_threads,
                    double* seconds) {
    RefScene* rs = static_cast<RefScene*>(h);
    const Scene& sc = *rs->scene;
    int nt = n_threads > 0 ? n_threads : rs->max_threads;
    auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 4096) num_threads(nt)
    for (std::int64_t i = 0; i < static_cast<std::int64_t>(n); ++i) {
        const float* r = rays + 8 * i;
        Ray ray(glm::vec3(r[0], r[1], r[2]), glm::vec3(r[4], r[5], r[6]));
        IntersectionRecord rec;
        rec.primitive_id_ = SPT_MISS;
        std::size_t nt_, nh_;
        tl_tri_tests = 0;
        bool hit = sc.intersect(ray, rec, nt_, nh_);
        if (hits) {
            hits[i].t = hit ? rec.t_ : std::numeric_limits<float>::infinity();
            hits[i].prim_id = hit ? static_cast<std::uint32_t>(rec.primitive_id_) : SPT_MISS;
            hits[i].u = 0.0f;
            hits[i].v = 0.0f;
        }
        if (normals) {
            normals[3 * i] = hit ? rec.normal_.x : 0.0f;
            normals[3 * i + 1] = hit ? rec.normal_.y : 0.0f;
            normals[3 * i + 2] = hit ? rec.normal_.z : 0.0f;
        }
        if (tests) tests[i] = static_cast<std::uint32_t>(nt_);
        if (nhits) nhits[i] = static_cast<std::uint32_t>(nh_);
        if (prim_tests) prim_tests[i] = static_cast<std::uint32_t>(tl_tri_tests);
    }
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    return 0;
}

// Camera::getRay for every pixel centre (integrators/raycaster.h:81-84): 8 floats per ray,
// row-major [y][x].
int swref_camera_rays(const spt_camera* c, float* rays) {
    std::unique_ptr<Camera> cam = make_camera(c);
    RegularPixelSampler ps(1);
    for (std::uint32_t y = 0; y < c->height; ++y)
        for (std::uint32_t x = 0; x < c->width; ++x) {
            float xs = x + ps.getSample(0).x;
            float ys = y + ps.getSample(0).y;
            Ray r = cam->getRay(xs, ys);
            float* o = rays + 8ull * (static_cast<std::uint64_t>(y) * c->width + x);
            o[0] = r.getOrigin().x; o[1] = r.getOrigin().y; o[2] = r.getOrigin().z; o[3] = 0.0f;
            o[4] = r.getDirection().x; o[5] = r.getDirection().y; o[6] = r.getDirection().z; o[7] = 0.0f;
        }
    return 0;
}

// RayCaster<T>::render (integrators/raycaster.h:62-99) for one mode; out layout as
// spt_raycast_image.  stats may be NULL.
int swref_raycast(void* h, const spt_camera* c, int mode, void* out, spt_render_stats* stats, int n_threads,
                  double* seconds) {
    RefScene* rs = static_cast<RefScene*>(h);
    omp_set_num_threads(n_threads > 0 ? n_threads : rs->max_threads);
    std::unique_ptr<Camera> cam = make_camera(c);
    const std::uint32_t W = c->width, H = c->height;
    Silence quiet;
    auto t0 = std::chrono::steady_clock::now();
    std::unique_ptr<Integrator> integ;
    if (mode == SPT_RAYCAST_NORMAL) {
        auto r = std::make_unique<NormalRayCaster>(*cam, *rs->scene);
        r->render();
        float* o = static_cast<float*>(out);
        for (std::uint32_t y = 0; y < H; ++y)
            for (std::uint32_t x = 0; x < W; ++x)
                for (int k = 0; k < 3; ++k) o[(static_cast<std::uint64_t>(y) * W + x) * 3 + k] = r->buffer_[x][y][k];
        integ = std::move(r);
    } else if (mode == SPT_RAYCAST_DEPTH) {
        auto r = std::make_unique<DepthRayCaster>(*cam, *rs->scene, -1.0f, -1.0f);
        r->render();
        float* o = static_cast<float*>(out);
        for (std::uint32_t y = 0; y < H; ++y)
            for (std::uint32_t x = 0; x < W; ++x) o[static_cast<std::uint64_t>(y) * W + x] = r->buffer_[x][y];
        integ = std::move(r);
    } else {
        auto r = std::make_unique<IntTestCountRayCaster>(*cam, *rs->scene, -1, -1);
        r->render();
        std::int64_t* o = static_cast<std::int64_t*>(out);
        for (std::uint32_t y = 0; y < H; ++y)
            for (std::uint32_t x = 0; x < W; ++x) o[static_cast<std::uint64_t>(y) * W + x] = r->buffer_[x][y];
        integ = std::move(r);
    }
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->int_tests = integ->getNumIntersectionTests();
        stats->int_hits = integ->getNumIntersections();
        stats->min_tests_pp = integ->getMinIntersectionTestsPerPixel();
        stats->max_tests_pp = integ->getMaxIntersectionTestsPerPixel();
        stats->min_hits_pp = integ->getMinIntersectionsPerPixel();
        stats->max_hits_pp = integ->getMaxIntersectionsPerPixel();
        stats->paths = static_cast<std::uint64_t>(W) * H;
    }
    return 0;
}

// PathTracer::render (integrators/pathtracer.cpp:59-147).  out: float[h][w][3] mean radiance.
// The reference has either max-length or russian-roulette termination; params->max_depth is
// not supported by it and must be 0.
int swref_pathtrace(void* h, const spt_camera* c, const spt_pt_params* p, float* out, int n_threads,
                    double* seconds) {
    RefScene* rs = static_cast<RefScene*>(h);
    if (p->max_depth != 0) return 2;
    int nt = n_threads > 0 ? n_threads : rs->max_threads;
    if (nt > static_cast<int>(rs->prng->engines_.size())) return 3;
    omp_set_num_threads(nt);
    reseed(*rs->prng, p->seed);
    std::unique_ptr<Camera> cam = make_camera(c);
    std::unique_ptr<PixelSampler> ps;
    if (p->pixel_sampler == SPT_PIXEL_UNIFORM) ps = std::make_unique<UniformPixelSampler>(p->spp, *rs->prng);
    else if (p->pixel_sampler == SPT_PIXEL_REGULAR) ps = std::make_unique<RegularPixelSampler>(p->spp);
    else ps = std::make_unique<JitteredPixelSampler>(p->spp, *rs->prng);
    PathTracer::PathTerminationCriterion crit = p->termination == SPT_TERMINATE_MAX_DEPTH
                                                    ? PathTracer::PathTerminationCriterion::MAX_DEPTH
                                                    : PathTracer::PathTerminationCriterion::RUSSIAN_ROULETTE;
    PathTracer pt(*cam, *rs->scene, crit, p->path_length, std::move(ps), *rs->prng);
    Silence quiet;
    auto t0 = std::chrono::steady_clock::now();
    pt.render();
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    const ImageBuffer& ib = cam->getImageBuffer();
    for (std::uint32_t y = 0; y < c->height; ++y)
        for (std::uint32_t x = 0; x < c->width; ++x) {
            const glm::vec3& v = ib.getPixelValue(x, y);
            float* o = out + (static_cast<std::uint64_t>(y) * c->width + x) * 3;
            o[0] = v.x; o[1] = v.y; o[2] = v.z;
        }
    return 0;
}

// The reference's BSDF objects evaluated directly, for per-BSDF checks:
// Material::evalBSDF (materials/material.cpp:6-9) for `n` outgoing directions of material
// `mat`.  out per direction: bsdf rgb, reflectance rgb, pdf, wi xyz (10 floats).
int swref_eval_material(void* h, std::uint32_t mat, const float* wo, std::uint64_t n, float* out, std::uint64_t seed) {
    RefScene* rs = static_cast<RefScene*>(h);
    omp_set_num_threads(1);
    reseed(*rs->prng, seed);
    const Material& m = rs->scene->getMaterial(mat);
    for (std::uint64_t i = 0; i < n; ++i) {
        glm::vec3 w(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
        glm::vec3 f, refl, wi;
        float pdf;
        m.evalBSDF(w, f, refl, pdf, wi);
        float* o = out + 10 * i;
        o[0] = f.x; o[1] = f.y; o[2] = f.z;
        o[3] = refl.x; o[4] = refl.y; o[5] = refl.z;
        o[6] = pdf;
        o[7] = wi.x; o[8] = wi.y; o[9] = wi.z;
    }
    omp_set_num_threads(rs->max_threads);
    return 0;
}

// BSDF::f and BSDF::getReflectance of BSDF `b` for given (wo, wi) pairs: 6 floats out each.
int swref_bsdf_f(void* h, std::uint32_t b, const float* wo, const float* wi, std::uint64_t n, float* out) {
    RefScene* rs = static_cast<RefScene*>(h);
    const BSDF* bsdf = rs->scene->getBSDFPtr(b);
    for (std::uint64_t i = 0; i < n; ++i) {
        glm::vec3 a(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
        glm::vec3 c(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
        glm::vec3 f = bsdf->f(a, c);
        glm::vec3 r = bsdf->getReflectance(a, c);
        float* o = out + 6 * i;
        o[0] = f.x; o[1] = f.y; o[2] = f.z; o[3] = r.x; o[4] = r.y; o[5] = r.z;
    }
    return 0;
}

}  // extern "C"
