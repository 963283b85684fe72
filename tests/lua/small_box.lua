-- Test scene: an open box (grey back, floor and ceiling, red left and green right walls) with a
-- light quad under the ceiling and a Cook-Torrance sphere.  INTEGRATOR selects the integrator.
require "scene_dsl"

local w, h = 48, 40
Camera{ type = "pinhole", position = {0.5, 0.5, 2.35}, look_at = {0.5, 0.5, 0}, up = {0, 1, 0}, fov = 40 }
PixelSampler{ type = "jittered", spp = 16 }
ImageBuffer{ width = w, height = h, file_name = "small_box.ppm",
             viewport_top = 0, viewport_left = 0, viewport_width = w, viewport_height = h }
GlobalSettings{ background_color = {0, 0, 0}, acceleration_structure = "bvh-sah" }
if INTEGRATOR == "depth" or INTEGRATOR == "normal" or INTEGRATOR == "intersection-test-count" then
    Integrator{ type = "ray-caster", pixel_value = INTEGRATOR, minimum_depth = -1, maximum_depth = -1,
                minimum_count = -1, maximum_count = -1 }
else
    Integrator{ type = "path-tracer", path_termination = "max-length", path_length = 5 }
end

local function matte(r, g, b)
    return Material{ bsdf = LayeredBSDF{ Lambertian{ kd = {r, g, b} } }, emission = Emission{0, 0, 0} }
end
local grey, red, green = matte(0.75, 0.75, 0.75), matte(0.63, 0.06, 0.05), matte(0.14, 0.45, 0.09)
local light = Material{ bsdf = LayeredBSDF{ Lambertian{ kd = {0, 0, 0} } }, emission = Emission{15, 15, 15} }
local metal = Material{ bsdf = LayeredBSDF{ CookTorrance{ roughness = 0.3,
                                                          reflectance_at_normal_incidence = {0.95, 0.64, 0.54} } },
                        emission = Emission{0, 0, 0} }

local function quad(a, b, c, d, m)
    Triangle{ v1 = a, v2 = b, v3 = c, material = m }
    Triangle{ v1 = a, v2 = c, v3 = d, material = m }
end
quad({0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, grey)      -- back
quad({0, 0, 1}, {1, 0, 1}, {1, 0, 0}, {0, 0, 0}, grey)      -- floor
quad({0, 1, 0}, {1, 1, 0}, {1, 1, 1}, {0, 1, 1}, grey)      -- ceiling
quad({0, 0, 1}, {0, 0, 0}, {0, 1, 0}, {0, 1, 1}, red)       -- left
quad({1, 0, 0}, {1, 0, 1}, {1, 1, 1}, {1, 1, 0}, green)     -- right
local y, lo, hi = 0.999, 0.375, 0.625
quad({lo, y, lo}, {lo, y, hi}, {hi, y, hi}, {hi, y, lo}, light)
Sphere{ center = {0.5, 0.3, 0.5}, radius = 0.3, material = metal }
for i = 1, 3 do
    Sphere{ center = {0.2 * i, 0.08, 0.85}, radius = 0.07, material = matte(0.2 * i, 0.5, 1 - 0.2 * i) }
end
