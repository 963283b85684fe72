// adapter_check.cpp -- TEST INFRASTRUCTURE ONLY.  Builds include/spt_reference_adapter.hpp against the
// reference renderer's own headers and sources (compiled by oracle/Makefile into oracle/_ref) and runs
// the GPU integrators it defines beside the reference's CPU integrators on the same scene:
//
//   * GpuRayCaster<DepthRayCaster / NormalRayCaster / IntTestCountRayCaster> must leave the same
//     per-pixel buffer_ (bit for bit) and the same image statistics as the reference ray casters'
//     render(), and their saveImageToFile (the reference's own post-processing) the same PPM bytes;
//   * GpuPathTracer must write an image into the camera's ImageBuffer whose mean matches the
//     reference PathTracer's within the statistical tolerance of the sample counts.
//
// The scene is built once through each side's own interface (the reference's Scene::add* calls and
// the adapter's GpuSceneDesc), the way SwpathtracerApp::loadScene would fill both.  Exit status 0 and
// "adapter ok" on success; 1 with a message on a mismatch; 2 when no GPU can be used.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <iterator>
#include <limits>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "cosine_bsdf_sampler.h"
#include "jittered_pixel_sampler.h"
#include "lambertian.h"
#include "layered_bsdf.h"
#include "material.h"
#include "pathtracer.h"
#include "sbvh.h"
#include "scene.h"
#include "sphere.h"
#include "triangle.h"

#include "spt_reference_adapter.hpp"

namespace {

typedef PRNG<std::uniform_real_distribution, float, std::mt19937> RefPRNG;

// The protected per-pixel buffer of a ray caster (the reference's or the adapter's).
template <class RC>
struct Peek : RC {
    using RC::RC;
    const auto& buffer() const { return this->buffer_; }
};

std::string slurp(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    return std::string(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
}

int fail(const std::string& msg) {
    std::cerr << "adapter check failed: " << msg << "\n";
    return 1;
}

// An open box of Lambertian walls lit by a ceiling quad, with a Lambertian sphere inside: added to the
// reference Scene and to the adapter's description in the same order.
void build_scene(Scene& sc, spt_ref::GpuSceneDesc& g, RefPRNG& prng) {
    const glm::vec3 grey(0.75f), red(0.63f, 0.06f, 0.05f), green(0.14f, 0.45f, 0.09f), ball(0.4f, 0.5f, 0.7f);
    const glm::vec3 cols[4] = {grey, red, green, ball};
    for (int i = 0; i < 4; ++i) {
        sc.addBSDF(std::make_unique<Lambertian>(cols[i], std::make_unique<CosineBSDFSampler>(prng)));
        g.add_bsdf(SPT_BSDF_LAMBERTIAN, SPT_SAMPLER_IMPORTANCE, cols[i], 0.0f);
    }
    for (uint32_t i = 0; i < 4; ++i) {
        LayeredBSDF l;
        l.addBSDF(sc.getBSDFPtr(i));
        sc.addLayeredBSDF(l);
        g.add_layered({i});
    }
    const glm::vec3 em[5] = {glm::vec3(0.0f), glm::vec3(0.0f), glm::vec3(0.0f), glm::vec3(0.0f), glm::vec3(12.0f)};
    const uint32_t lay[5] = {0, 1, 2, 3, 0};
    for (int i = 0; i < 5; ++i) sc.addEmission(em[i]);
    for (int i = 0; i < 5; ++i) {
        sc.addMaterial(Material(sc.getLayeredBSDF(lay[i]), sc.getEmission(i)));
        g.add_material(lay[i], em[i]);
    }
    auto tri = [&](glm::vec3 a, glm::vec3 b, glm::vec3 c, unsigned long m) {
        sc.addPrimitive(std::make_unique<Triangle>(a, b, c, m));
        g.add_triangle(a, b, c, static_cast<uint32_t>(m));
    };
    auto quad = [&](glm::vec3 a, glm::vec3 b, glm::vec3 c, glm::vec3 d, unsigned long m) {
        tri(a, b, c, m);
        tri(a, c, d, m);
    };
    const float s = 1.0f;
    quad({0, 0, 0}, {s, 0, 0}, {s, 0, -s}, {0, 0, -s}, 0);          // floor
    quad({0, s, 0}, {0, s, -s}, {s, s, -s}, {s, s, 0}, 0);          // ceiling
    quad({0, 0, -s}, {s, 0, -s}, {s, s, -s}, {0, s, -s}, 0);        // back
    quad({0, 0, 0}, {0, 0, -s}, {0, s, -s}, {0, s, 0}, 1);          // left
    quad({s, 0, 0}, {s, s, 0}, {s, s, -s}, {s, 0, -s}, 2);          // right
    const float a = 0.375f, b = 0.625f, h = s - 1e-3f;
    quad({a, h, -a}, {a, h, -b}, {b, h, -b}, {b, h, -a}, 4);        // light
    sc.addPrimitive(std::make_unique<Sphere>(glm::vec3(0.5f, 0.3f, -0.55f), 0.25f, 3));
    g.add_sphere(glm::vec3(0.5f, 0.3f, -0.55f), 0.25f, 3);
}

std::unique_ptr<Camera> make_camera(unsigned w, unsigned h, const std::string& file) {
    return std::make_unique<PinholeCamera>(glm::vec3(0.5f, 0.5f, 1.4f), glm::vec3(0.5f, 0.5f, -0.5f),
                                           glm::vec3(0.0f, 1.0f, 0.0f), 45.0f,
                                           std::make_unique<ImageBuffer>(w, h, 0, 0, w, h, file));
}

template <class RC, typename... Args>
int check_raycaster(const char* name, Scene& sc, spt_ref::GpuBackend& gpu, const std::string& dir, Args... args) {
    const unsigned w = 96, h = 72;
    auto cam_ref = make_camera(w, h, dir + "/ref_" + name + ".ppm");
    auto cam_gpu = make_camera(w, h, dir + "/gpu_" + name + ".ppm");
    Peek<RC> ref(*cam_ref, sc, args...);
    Peek<spt_ref::GpuRayCaster<RC>> gpu_rc(gpu, *cam_gpu, sc, args...);
    {
        std::streambuf* o = std::cout.rdbuf(nullptr);   // the reference prints its timings
        ref.render();
        std::cout.rdbuf(o);
    }
    gpu_rc.render();
    const auto& a = ref.buffer();
    const auto& b = gpu_rc.buffer();
    for (unsigned x = 0; x < w; ++x)
        for (unsigned y = 0; y < h; ++y)
            if (std::memcmp(&a[x][y], &b[x][y], sizeof(a[x][y])) != 0)
                return fail(std::string(name) + ": buffer differs at pixel (" + std::to_string(x) + ", " +
                            std::to_string(y) + ")");
    if (ref.getNumIntersectionTests() != gpu_rc.getNumIntersectionTests() ||
        ref.getNumIntersections() != gpu_rc.getNumIntersections() ||
        ref.getMinIntersectionTestsPerPixel() != gpu_rc.getMinIntersectionTestsPerPixel() ||
        ref.getMaxIntersectionTestsPerPixel() != gpu_rc.getMaxIntersectionTestsPerPixel() ||
        ref.getMinIntersectionsPerPixel() != gpu_rc.getMinIntersectionsPerPixel() ||
        ref.getMaxIntersectionsPerPixel() != gpu_rc.getMaxIntersectionsPerPixel())
        return fail(std::string(name) + ": image statistics differ");
    ref.saveImageToFile();
    gpu_rc.saveImageToFile();
    const std::string pa = slurp(dir + "/ref_" + std::string(name) + ".ppm");
    const std::string pb = slurp(dir + "/gpu_" + std::string(name) + ".ppm");
    if (pa.empty() || pa != pb) return fail(std::string(name) + ": saved images differ");
    std::cout << name << ": buffer, statistics and saved image equal (" << ref.getNumIntersectionTests()
              << " tests)\n";
    return 0;
}

double image_mean(const Camera& cam) {
    const ImageBuffer& ib = cam.getImageBuffer();
    double s = 0.0;
    for (unsigned x = 0; x < ib.getImageWidth(); ++x)
        for (unsigned y = 0; y < ib.getImageHeight(); ++y) {
            const glm::vec3& p = ib.getPixelValue(x, y);
            s += static_cast<double>(p.x) + p.y + p.z;
        }
    return s / (3.0 * ib.getImageWidth() * ib.getImageHeight());
}

}  // namespace

int main(int argc, char** argv) {
    const std::string dir = argc > 1 ? argv[1] : ".";
    RefPRNG prng(0.0f, 1.0f);
    auto accel = std::make_unique<SBVH>(std::numeric_limits<float>::infinity());
    Scene sc(std::move(accel), glm::vec3(0.0f));
    spt_ref::GpuSceneDesc desc;
    build_scene(sc, desc, prng);
    {
        std::streambuf* o = std::cout.rdbuf(nullptr);
        sc.buildAccelStructure();
        std::cout.rdbuf(o);
    }
    desc.accel = SPT_ACCEL_SBVH_SAH;
    std::unique_ptr<spt_ref::GpuBackend> gpu;
    try {
        gpu = std::make_unique<spt_ref::GpuBackend>(desc, 0);
    } catch (const std::exception& e) {
        std::cerr << "no GPU backend: " << e.what() << "\n";
        return 2;
    }
    if (int r = check_raycaster<DepthRayCaster>("depth", sc, *gpu, dir, -1.0f, -1.0f)) return r;
    if (int r = check_raycaster<NormalRayCaster>("normal", sc, *gpu, dir)) return r;
    if (int r = check_raycaster<IntTestCountRayCaster>("count", sc, *gpu, dir, -1L, -1L)) return r;

    // path tracer: the reference's PathTracer and the adapter's GpuPathTracer, max length 4
    const unsigned w = 48, h = 36;
    const int spp_ref = 256, spp_gpu = 4096;
    auto cam_ref = make_camera(w, h, dir + "/ref_pt.ppm");
    auto cam_gpu = make_camera(w, h, dir + "/gpu_pt.ppm");
    PathTracer ref(*cam_ref, sc, PathTracer::PathTerminationCriterion::MAX_DEPTH, 4,
                   std::make_unique<JitteredPixelSampler>(spp_ref, prng), prng);
    spt_ref::GpuPathTracer gpt(*cam_gpu, sc, *gpu, spt_ref::GpuPathTracer::PathTerminationCriterion::MAX_DEPTH, 4,
                               std::make_unique<JitteredPixelSampler>(spp_gpu, prng), 7);
    {
        std::streambuf* o = std::cout.rdbuf(nullptr);
        ref.render();
        std::cout.rdbuf(o);
    }
    gpt.render();
    const double mr = image_mean(*cam_ref), mg = image_mean(*cam_gpu);
    if (gpt.paths() != static_cast<uint64_t>(w) * h * spp_gpu) return fail("path tracer: wrong path count");
    // 110k reference paths: the image mean's standard error is well under 2 %
    if (!(std::fabs(mr - mg) < 0.04 * mr)) return fail("path tracer: image means " + std::to_string(mr) + " vs " +
                                                       std::to_string(mg));
    gpt.saveImageToFile();
    if (slurp(dir + "/gpu_pt.ppm").substr(0, 2) != "P3") return fail("path tracer: no PPM written");
    std::cout << "path tracer: image mean " << mg << " (reference " << mr << ")\n";
    std::cout << "adapter ok\n";
    return 0;
}
