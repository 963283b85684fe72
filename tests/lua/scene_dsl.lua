-- A minimal stand-in for the renderer's scene-description functions, used by the tests where the
-- reference's own lua_core modules are not installed.  It records every element in the global table
-- __RENDERER_ELEMENTS__ with the layout the renderer's Lua binding reads: lists indexed from 1 and
-- their counts; Camera, PixelSampler, ImageBuffer, GlobalSettings and Integrator as single tables.
-- No validation or defaults beyond what the test scenes need.
local E = {}
_G["__RENDERER_ELEMENTS__"] = E
for _, list in ipairs({"OBJECT", "BSDF", "LAYERED_BSDF", "EMISSION", "MATERIAL"}) do
    E["__" .. list .. "S__"] = {}
    E["__" .. list .. "_COUNT__"] = 0
end

local function add(list, item)
    local key = "__" .. list .. "_COUNT__"
    E[key] = E[key] + 1
    E["__" .. list .. "S__"][E[key]] = item
    return E[key]
end

local function bsdf(kind)
    return function(t)
        t.type = kind
        t.bsdf_sampler = t.bsdf_sampler or "importance"
        return add("BSDF", t)
    end
end
Lambertian = bsdf("lambertian")
SmoothConductor = bsdf("smooth_conductor")
SmoothDielectric = bsdf("smooth_dielectric")
CookTorrance = bsdf("cook_torrance")

function LayeredBSDF(t) return add("LAYERED_BSDF", t) end
function Emission(t) return add("EMISSION", t) end
function Material(t) return add("MATERIAL", t) end

local function object(kind)
    return function(t)
        t.type = kind
        add("OBJECT", t)
    end
end
Triangle = object("triangle")
SmoothTriangle = object("smooth_triangle")
Sphere = object("sphere")
Mesh = object("mesh")

function Camera(t) E["__CAMERA__"] = t end
function PixelSampler(t) E["__PIXEL_SAMPLER__"] = t end
function ImageBuffer(t) E["__IMAGE_BUFFER__"] = t end
function GlobalSettings(t) E["__GLOBAL_SETTINGS__"] = t end
function Integrator(t) E["__INTEGRATOR__"] = t end
