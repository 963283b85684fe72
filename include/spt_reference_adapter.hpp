// spt_reference_adapter.hpp -- the B200 backend behind the reference renderer's own C++ interfaces.
//
// This header belongs on the reference's side of the boundary: a maintainer adds it to the reference
// project (next to integrators/), links libspt_cuda.so, and includes it where SwpathtracerApp builds
// its integrators (core/swpathtracer_app.cpp:221-259).  It needs the reference's headers
// (integrators/, cameras/, core/, pixel_samplers/) and spt.h on the include path, and uses nothing
// of the backend but the C-ABI.
//
//   GpuSceneDesc            the scene as the plain arrays of spt_scene_desc; SwpathtracerApp::loadScene
//                           (core/swpathtracer_app.cpp:67-219) fills it next to its Scene::add* calls
//   GpuBackend              one device context plus the uploaded scene (spt_create, spt_scene_create)
//   GpuPathTracer           an Integrator (integrators/integrator.h:8-55) whose render() runs
//                           spt_pathtrace and writes the camera's ImageBuffer the way
//                           PathTracer::render does (integrators/pathtracer.cpp:59-147)
//   GpuRayCaster<RC>        the reference's own ray caster RC (NormalRayCaster, DepthRayCaster,
//                           IntTestCountRayCaster) with render() replaced by spt_raycast_image: it
//                           fills RC's per-pixel buffer_ and the statistics (raycaster.h:62-99), and
//                           RC's own saveImageToFile post-processes and writes the image unchanged
//
// Errors become std::runtime_error, which the reference's main catches (core/main.cpp:6-11).
#ifndef SPT_REFERENCE_ADAPTER_HPP
#define SPT_REFERENCE_ADAPTER_HPP

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "depth_raycaster.h"
#include "int_test_count_raycaster.h"
#include "integrator.h"
#include "normal_raycaster.h"
#include "orthographic_camera.h"
#include "pinhole_camera.h"
#include "spt.h"

namespace spt_ref {

inline void check(spt_context* ctx, spt_status st, const char* what) {
    if (st != SPT_OK)
        throw std::runtime_error(std::string(what) + ": " + (ctx ? spt_last_error(ctx) : "status " + std::to_string(st)));
}

// The scene as spt_scene_desc's arrays, filled in the order SwpathtracerApp::loadScene adds BSDFs,
// layered BSDFs, materials and primitives (the primitive order decides the SAH tree).
struct GpuSceneDesc {
    std::vector<uint8_t> type;
    std::vector<float> data, normals;
    std::vector<uint32_t> material;
    std::vector<spt_bsdf> bsdfs;
    std::vector<uint32_t> layered_offsets{0}, layered_ids;
    std::vector<spt_material> materials;
    float background[3] = {0.0f, 0.0f, 0.0f};
    int32_t accel = SPT_ACCEL_SBVH_SAH;
    bool smooth = false;

    uint32_t add_bsdf(int32_t bsdf_type, int32_t sampler, const glm::vec3& rgb, float scalar) {
        spt_bsdf b{};
        b.type = bsdf_type;
        b.sampler = sampler;
        b.rgb[0] = rgb.x;
        b.rgb[1] = rgb.y;
        b.rgb[2] = rgb.z;
        b.scalar = scalar;
        bsdfs.push_back(b);
        return static_cast<uint32_t>(bsdfs.size() - 1);
    }
    uint32_t add_layered(const std::vector<uint32_t>& bsdf_ids_top_first) {
        layered_ids.insert(layered_ids.end(), bsdf_ids_top_first.begin(), bsdf_ids_top_first.end());
        layered_offsets.push_back(static_cast<uint32_t>(layered_ids.size()));
        return static_cast<uint32_t>(layered_offsets.size() - 2);
    }
    uint32_t add_material(uint32_t layered, const glm::vec3& emission) {
        spt_material m{};
        m.layered_bsdf = layered;
        m.emission[0] = emission.x;
        m.emission[1] = emission.y;
        m.emission[2] = emission.z;
        materials.push_back(m);
        return static_cast<uint32_t>(materials.size() - 1);
    }
    void add_triangle(const glm::vec3& a, const glm::vec3& b, const glm::vec3& c, uint32_t mat) {
        push(SPT_PRIM_TRIANGLE, {a, b, c}, {glm::vec3(0.0f), glm::vec3(0.0f), glm::vec3(0.0f)}, mat);
    }
    void add_smooth_triangle(const glm::vec3& a, const glm::vec3& b, const glm::vec3& c, const glm::vec3& na,
                             const glm::vec3& nb, const glm::vec3& nc, uint32_t mat) {
        push(SPT_PRIM_SMOOTH_TRIANGLE, {a, b, c}, {na, nb, nc}, mat);
        smooth = true;
    }
    void add_sphere(const glm::vec3& centre, float radius, uint32_t mat) {
        push(SPT_PRIM_SPHERE, {centre, glm::vec3(radius, 0.0f, 0.0f), glm::vec3(0.0f)},
             {glm::vec3(0.0f), glm::vec3(0.0f), glm::vec3(0.0f)}, mat);
    }
    spt_scene_desc view() const {
        spt_scene_desc d{};
        d.n_prims = static_cast<uint32_t>(type.size());
        d.prim_type = type.data();
        d.prim_data = data.data();
        d.prim_normals = smooth ? normals.data() : nullptr;
        d.prim_material = material.data();
        d.n_bsdfs = static_cast<uint32_t>(bsdfs.size());
        d.bsdfs = bsdfs.data();
        d.n_layered = static_cast<uint32_t>(layered_offsets.size() - 1);
        d.layered_offsets = layered_offsets.data();
        d.layered_bsdf_ids = layered_ids.data();
        d.n_materials = static_cast<uint32_t>(materials.size());
        d.materials = materials.data();
        for (int k = 0; k < 3; ++k) d.background[k] = background[k];
        d.accel = accel;
        return d;
    }

   private:
    void push(uint8_t t, std::initializer_list<glm::vec3> p, std::initializer_list<glm::vec3> n, uint32_t mat) {
        type.push_back(t);
        for (const glm::vec3& v : p) data.insert(data.end(), {v.x, v.y, v.z});
        for (const glm::vec3& v : n) normals.insert(normals.end(), {v.x, v.y, v.z});
        material.push_back(mat);
    }
};

// One device context and the scene on it, shared by the integrators of a render.
class GpuBackend {
   public:
    explicit GpuBackend(const GpuSceneDesc& desc, int device = 0) {
        check(nullptr, spt_create(device, &ctx_), "spt_create");
        const spt_scene_desc d = desc.view();
        const spt_status st = spt_scene_create(ctx_, &d, nullptr, &scene_);
        if (st != SPT_OK) {
            const std::string msg = spt_last_error(ctx_);
            spt_destroy(ctx_);
            throw std::runtime_error("spt_scene_create: " + msg);
        }
    }
    ~GpuBackend() {
        spt_scene_destroy(scene_);
        spt_destroy(ctx_);
    }
    GpuBackend(const GpuBackend&) = delete;
    GpuBackend& operator=(const GpuBackend&) = delete;
    spt_context* ctx() const { return ctx_; }
    spt_scene* scene() const { return scene_; }

   private:
    spt_context* ctx_ = nullptr;
    spt_scene* scene_ = nullptr;
};

// The reference camera (cameras/pinhole_camera.h, orthographic_camera.h) and its ImageBuffer's size
// and viewport as an spt_camera.
inline spt_camera camera_of(const Camera& cam) {
    spt_camera c{};
    const glm::vec3 p = cam.getPosition(), l = cam.getLookAt(), u = cam.getUp();
    for (int k = 0; k < 3; ++k) {
        c.position[k] = p[k];
        c.look_at[k] = l[k];
        c.up[k] = u[k];
    }
    if (cam.getType() == Camera::Type::ORTHOGRAPHIC) {
        const auto& o = static_cast<const OrthographicCamera&>(cam);
        c.type = SPT_CAMERA_ORTHOGRAPHIC;
        c.min_x = o.getMinX();
        c.max_x = o.getMaxX();
        c.min_y = o.getMinY();
        c.max_y = o.getMaxY();
    } else {
        c.type = SPT_CAMERA_PINHOLE;
        c.fov_deg = static_cast<const PinholeCamera&>(cam).getVFov();
    }
    const ImageBuffer& ib = cam.getImageBuffer();
    c.width = ib.getImageWidth();
    c.height = ib.getImageHeight();
    c.vp_top = ib.getViewportTop();
    c.vp_left = ib.getViewportLeft();
    c.vp_width = ib.getViewportWidth();
    c.vp_height = ib.getViewportHeight();
    return c;
}

inline int32_t pixel_sampler_of(const PixelSampler& s) {
    switch (s.getType()) {
        case PixelSampler::Type::UNIFORM: return SPT_PIXEL_UNIFORM;
        case PixelSampler::Type::REGULAR: return SPT_PIXEL_REGULAR;
        default: return SPT_PIXEL_JITTERED;
    }
}

// PathTracer's interface and output on the GPU (integrators/pathtracer.h:11-41).  The pixel sampler
// is the reference's own object; its type and spp set the backend's sampler.  `seed` keys the
// backend's Philox streams (the reference's mt19937 streams are not reproducible).
class GpuPathTracer : public Integrator {
   public:
    enum class PathTerminationCriterion { MAX_DEPTH, RUSSIAN_ROULETTE };

    GpuPathTracer(Camera& camera, const Scene& scene, GpuBackend& gpu, PathTerminationCriterion criterion,
                  int path_length, std::unique_ptr<PixelSampler> pixel_sampler, uint64_t seed = 1)
        : Integrator(camera, scene, Integrator::Type::PATHTRACER, std::move(pixel_sampler)), gpu_(gpu) {
        params_.pixel_sampler = pixel_sampler_of(getPixelSampler());
        params_.spp = static_cast<uint32_t>(getPixelSampler().getSPP());
        params_.termination = criterion == PathTerminationCriterion::MAX_DEPTH ? SPT_TERMINATE_MAX_DEPTH
                                                                             : SPT_TERMINATE_RUSSIAN_ROULETTE;
        params_.path_length = path_length;
        params_.seed = seed;
    }
    void render() override {
        const spt_camera c = camera_of(camera_);
        std::vector<float> rgb(3ull * c.width * c.height);
        spt_render_stats st{};
        check(gpu_.ctx(), spt_pathtrace(gpu_.ctx(), gpu_.scene(), &c, &params_, rgb.data(), &st), "spt_pathtrace");
        // PathTracer::render writes the mean radiance of the viewport's pixels into the camera's
        // ImageBuffer; the backend's image is row-major [y][x]
        ImageBuffer& ib = camera_.getImageBuffer();
        for (uint32_t y = c.vp_top; y < c.vp_top + c.vp_height; ++y)
            for (uint32_t x = c.vp_left; x < c.vp_left + c.vp_width; ++x) {
                const float* p = &rgb[3ull * (static_cast<uint64_t>(y) * c.width + x)];
                ib.setPixelValue(x, y, glm::vec3(p[0], p[1], p[2]));
            }
        paths_ = st.paths;
        segments_ = st.segments;
        gpu_ms_ = static_cast<float>(st.gpu_ms);
        int_tests_count_ = int_count_ = 0;
        min_int_tests_count_pp_ = max_int_tests_count_pp_ = min_int_count_pp_ = max_int_count_pp_ = 0;
    }
    // PathTracer::saveImageToFile (integrators/pathtracer.cpp:155-158)
    void saveImageToFile() override {
        camera_.getImageBuffer().convertTosRGB();
        camera_.getImageBuffer().saveToFile();
    }
    uint64_t paths() const { return paths_; }
    uint64_t segments() const { return segments_; }
    float gpu_ms() const { return gpu_ms_; }

   private:
    GpuBackend& gpu_;
    spt_pt_params params_{};
    uint64_t paths_ = 0, segments_ = 0;
    float gpu_ms_ = 0.0f;
};

// The mode of each reference ray caster and how one backend pixel becomes its buffer_ element.
template <class RC>
struct RayCasterMode;
template <>
struct RayCasterMode<NormalRayCaster> {
    static constexpr int32_t mode = SPT_RAYCAST_NORMAL;
    typedef float Pixel[3];
    static glm::vec3 value(const Pixel& p) { return glm::vec3(p[0], p[1], p[2]); }
};
template <>
struct RayCasterMode<DepthRayCaster> {
    static constexpr int32_t mode = SPT_RAYCAST_DEPTH;
    typedef float Pixel;
    static float value(const Pixel& p) { return p; }
};
template <>
struct RayCasterMode<IntTestCountRayCaster> {
    static constexpr int32_t mode = SPT_RAYCAST_COUNT;
    typedef int64_t Pixel;
    static long int value(const Pixel& p) { return static_cast<long int>(p); }
};

// The reference ray caster RC with its render() on the GPU.  Constructor arguments are RC's.
template <class RC>
class GpuRayCaster : public RC {
   public:
    template <typename... Args>
    GpuRayCaster(GpuBackend& gpu, Camera& camera, const Scene& scene, Args&&... args)
        : RC(camera, scene, std::forward<Args>(args)...), gpu_(gpu) {}

    // RayCaster<T>::render (integrators/raycaster.h:62-99): one ray per pixel centre, the buffer
    // element of each pixel and the image statistics.
    void render() override {
        typedef RayCasterMode<RC> M;
        const spt_camera c = camera_of(this->camera_);
        std::vector<typename M::Pixel> out(static_cast<size_t>(c.width) * c.height);
        spt_render_stats st{};
        check(gpu_.ctx(), spt_raycast_image(gpu_.ctx(), gpu_.scene(), &c, M::mode, out.data(), &st),
              "spt_raycast_image");
        for (uint32_t y = 0; y < c.height; ++y)
            for (uint32_t x = 0; x < c.width; ++x) this->buffer_[x][y] = M::value(out[static_cast<size_t>(y) * c.width + x]);
        this->int_tests_count_ = st.int_tests;
        this->int_count_ = st.int_hits;
        this->min_int_tests_count_pp_ = st.min_tests_pp;
        this->max_int_tests_count_pp_ = st.max_tests_pp;
        this->min_int_count_pp_ = st.min_hits_pp;
        this->max_int_count_pp_ = st.max_hits_pp;
        gpu_ms_ = static_cast<float>(st.gpu_ms);
    }
    float gpu_ms() const { return gpu_ms_; }

   private:
    GpuBackend& gpu_;
    float gpu_ms_ = 0.0f;
};

}  // namespace spt_ref

#endif  // SPT_REFERENCE_ADAPTER_HPP
