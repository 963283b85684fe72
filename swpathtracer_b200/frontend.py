"""The reference renderer's Lua scene scripts, rendered by the B200 backend.

A scene script (the reference's samples/*.lua) `require`s the reference's lua_core modules, which
define Camera{...}, Material{...}, Triangle{...}, ... and collect everything in the global table
__RENDERER_ELEMENTS__.  `load_lua` runs the script with this package's Lua-subset interpreter
(swpathtracer_b200/lua.py) and turns that table into the backend's objects the way the reference's
SwpathtracerApp does (core/swpathtracer_app.cpp:67-259, lua_bind/lua_bind.cpp):

  BSDFs         lambertian / smooth_conductor / smooth_dielectric / cook_torrance, their "bsdf_sampler"
  LayeredBSDF   lists of BSDF ids (1-based in Lua, 0-based here)
  Emission      RGB triplets;  Material: {bsdf = layered id, emission = emission id}
  objects       triangle (v1..v3), smooth_triangle (+ n1..n3), sphere (center, radius), mesh (an OBJ file,
                swpathtracer_b200/obj.py), each with a material id
  Camera        pinhole (fov) / orthographic (min_x..max_y) with the ImageBuffer's size and viewport
  PixelSampler  uniform / regular / jittered and spp;  GlobalSettings: background, acceleration structure
  Integrator    path-tracer (path_termination, path_length) or ray-caster (normal / depth /
                intersection-test-count, with the prescribed ranges of the last two)

`render` runs the integrator on a device and `save` writes the image file the reference would write
(post-processing and 8-bit quantization on the device).  Command line:

    python -m swpathtracer_b200.frontend scene.lua [--lua-path DIR ...] [--out image.ppm] [--seed N]

The lua_core modules are the reference's; --lua-path adds directories to search for them (relative
`package.path` entries of the script are also tried against the script's own directory and its parent).
"""
import argparse
import os
import sys

import numpy as np

from . import abi, lua, scenes

class LuaScene:
    """A scene script, evaluated: the backend's scene description plus the render settings."""

    def __init__(self):
        self.builder = None
        self.packed = None
        self.camera = None
        self.integrator = "path-tracer"   # or "ray-caster"
        self.pt_params = None
        self.raycast_mode = None
        self.prescribed = (-1, -1)        # ray caster: min / max depth or count
        self.file_name = "image.ppm"
        self.output = []                  # the script's print() lines


def _vec3(t, what):
    if not isinstance(t, lua.LuaTable):
        raise ValueError("%s: a table of three numbers expected" % what)
    v = [t[1], t[2], t[3]]
    if any(not isinstance(x, (int, float)) or isinstance(x, bool) for x in v):
        raise ValueError("%s: a table of three numbers expected" % what)
    return tuple(float(x) for x in v)


def _num(t, key, default=None):
    v = t[key]
    if v is None:
        if default is None:
            raise ValueError("missing number field %r" % key)
        return default
    return v


def _id(v, count, what):
    """A 1-based Lua id checked against its table's size, as 0-based."""
    if not isinstance(v, (int, float)) or isinstance(v, bool) or not float(v).is_integer() or not 1 <= v <= count:
        raise ValueError("%s: id %r out of range 1..%d" % (what, v, count))
    return int(v) - 1


def elements_to_scene(E, base_dir="."):
    """The __RENDERER_ELEMENTS__ table -> LuaScene (the SwpathtracerApp::load* sequence)."""
    s = LuaScene()
    gs = E["__GLOBAL_SETTINGS__"] or lua.LuaTable()
    bg = _vec3(gs["background_color"], "background_color") if gs["background_color"] is not None else (0.0, 0.0, 0.0)
    accel = gs["acceleration_structure"] or "bvh-sah"
    if accel not in ("none", "bvh-sah", "sbvh-sah"):
        raise ValueError("unknown acceleration structure %r" % accel)
    sb = scenes.SceneBuilder(background=bg, acceleration_structure=accel)
    # BSDFs (swpathtracer_app.cpp:89-149)
    n_bsdf = int(E["__BSDF_COUNT__"] or 0)
    for i in range(1, n_bsdf + 1):
        b = E["__BSDFS__"][i]
        kind, sampler = b["type"], b["bsdf_sampler"] or "importance"
        if kind == "lambertian":
            sb.lambertian(kd=_vec3(b["kd"], "kd"), bsdf_sampler=sampler)
        elif kind == "smooth_conductor":
            sb.smooth_conductor(_vec3(b["reflectance_at_normal_incidence"], "reflectance_at_normal_incidence"),
                                bsdf_sampler=sampler)
        elif kind == "smooth_dielectric":
            sb.smooth_dielectric(ior=float(_num(b, "ior")), bsdf_sampler=sampler)
        elif kind == "cook_torrance":
            sb.cook_torrance(roughness=float(_num(b, "roughness")),
                             reflectance_at_normal_incidence=_vec3(b["reflectance_at_normal_incidence"],
                                                                   "reflectance_at_normal_incidence"),
                             bsdf_sampler=sampler)
        else:
            raise ValueError("unknown BSDF type %r" % kind)
    # layered BSDFs, emissions, materials (swpathtracer_app.cpp:151-180)
    n_lay = int(E["__LAYERED_BSDF_COUNT__"] or 0)
    for i in range(1, n_lay + 1):
        t = E["__LAYERED_BSDFS__"][i]
        sb.layered_bsdf(*[_id(x, n_bsdf, "layered BSDF layer") for x in t.array()])
    n_em = int(E["__EMISSION_COUNT__"] or 0)
    emissions = [_vec3(E["__EMISSIONS__"][i], "emission") for i in range(1, n_em + 1)]
    n_mat = int(E["__MATERIAL_COUNT__"] or 0)
    for i in range(1, n_mat + 1):
        m = E["__MATERIALS__"][i]
        sb.material(_id(m["bsdf"], n_lay, "material bsdf"), emission=emissions[_id(m["emission"], n_em, "emission")])
    # objects in script order (swpathtracer_app.cpp:182-219); runs of triangles go in one call
    n_obj = int(E["__OBJECT_COUNT__"] or 0)
    if n_obj == 0:
        raise ValueError("no object (primitive) defined")
    tris, mats, norms = [], [], []

    def flush():
        if tris:
            sb.triangles(np.array(tris, np.float32), np.array(mats, np.uint32),
                         normals=np.array(norms, np.float32) if norms and len(norms) == len(tris) else None)
            tris.clear()
            mats.clear()
            norms.clear()

    for i in range(1, n_obj + 1):
        o = E["__OBJECTS__"][i]
        kind = o["type"]
        mat = _id(o["material"], n_mat, "object material")
        if kind == "triangle":
            if norms:
                flush()
            tris.append([_vec3(o["v1"], "v1"), _vec3(o["v2"], "v2"), _vec3(o["v3"], "v3")])
            mats.append(mat)
        elif kind == "smooth_triangle":
            if tris and not norms:
                flush()
            tris.append([_vec3(o["v1"], "v1"), _vec3(o["v2"], "v2"), _vec3(o["v3"], "v3")])
            norms.append([_vec3(o["n1"], "n1"), _vec3(o["n2"], "n2"), _vec3(o["n3"], "n3")])
            mats.append(mat)
        elif kind == "sphere":
            flush()
            sb.sphere(_vec3(o["center"], "center"), float(_num(o, "radius", 1.0)), mat)
        elif kind == "mesh":
            flush()
            from . import obj
            fname = o["filename"]
            path = fname if os.path.isabs(fname) else os.path.join(base_dir, fname)
            submeshes = {}
            sm = o["sub_meshes"]
            if isinstance(sm, lua.LuaTable):
                for _, entry in sm.d.items():
                    submeshes[entry["name"]] = _id(entry["material"], n_mat, "sub-mesh material")
            obj.add_mesh(sb, path, mat, (o["render_submeshes"] or "all") == "all", submeshes)
        else:
            raise ValueError("unknown object type %r" % kind)
    flush()
    s.builder = sb
    s.packed = sb.build()
    # image buffer + camera (lua_bind.cpp getCamera / getImageBuffer)
    ib = E["__IMAGE_BUFFER__"]
    w, h = int(_num(ib, "width", 512)), int(_num(ib, "height", 512))
    vp = (int(_num(ib, "viewport_top", 0)), int(_num(ib, "viewport_left", 0)),
          int(_num(ib, "viewport_width", w)), int(_num(ib, "viewport_height", h)))
    s.file_name = ib["file_name"] or "image.ppm"
    c = E["__CAMERA__"]
    kind = c["type"] or "pinhole"
    common = dict(position=_vec3(c["position"], "position"), look_at=_vec3(c["look_at"], "look_at"),
                  up=_vec3(c["up"], "up"), width=w, height=h, viewport=vp)
    if kind == "pinhole":
        s.camera = scenes.camera("pinhole", fov=float(_num(c, "fov", 55)), **common)
    else:
        s.camera = scenes.camera("orthographic", window=(float(_num(c, "min_x")), float(_num(c, "max_x")),
                                                         float(_num(c, "min_y")), float(_num(c, "max_y"))), **common)
    # integrator + pixel sampler (swpathtracer_app.cpp:221-259)
    it = E["__INTEGRATOR__"]
    s.integrator = it["type"] or "ray-caster"
    if s.integrator == "path-tracer":
        ps = E["__PIXEL_SAMPLER__"]
        s.pt_params = scenes.pt_params(spp=int(_num(ps, "spp", 16)), sampler=ps["type"] or "jittered",
                                       termination=it["path_termination"] or "russian-roulette",
                                       path_length=int(_num(it, "path_length", 5)))
    elif s.integrator == "ray-caster":
        pv = it["pixel_value"] or "normal"
        s.raycast_mode = {"normal": abi.RAYCAST_NORMAL, "depth": abi.RAYCAST_DEPTH,
                          "intersection-test-count": abi.RAYCAST_COUNT}[pv]
        if pv == "depth":
            s.prescribed = (float(_num(it, "minimum_depth", -1)), float(_num(it, "maximum_depth", -1)))
        elif pv == "intersection-test-count":
            s.prescribed = (int(_num(it, "minimum_count", -1)), int(_num(it, "maximum_count", -1)))
    else:
        raise ValueError("unknown integrator %r" % s.integrator)
    return s


def load_lua(path, lua_path=(), seed=None, globals=None):
    """Runs a scene script and returns its LuaScene.  lua_path: extra directories for `require`;
    globals: values (numbers, strings, booleans) set as Lua globals before the script runs."""
    path = os.path.abspath(path)
    here = os.path.dirname(path)
    dirs = [here, os.path.dirname(here)] + [os.path.abspath(d) for d in lua_path]
    interp = lua.Interpreter(search_dirs=dirs, seed=seed)
    for k, v in (globals or {}).items():
        interp.G[k] = v
    for d in lua_path:   # modules directly in the given directories
        interp.G["package"]["path"] = interp.G["package"]["path"] + ";" + os.path.join(os.path.abspath(d), "?.lua")
    try:
        interp.run_file(path)
    except lua.LuaExit as e:
        raise RuntimeError("the scene script exited (os.exit): %s" % "; ".join(interp.output[-3:])) from e
    E = interp.G["__RENDERER_ELEMENTS__"]
    if not isinstance(E, lua.LuaTable):
        raise RuntimeError("the script defined no __RENDERER_ELEMENTS__ (did it require the lua_core modules?)")
    s = elements_to_scene(E, base_dir=here)
    s.output = interp.output
    return s


def render(s, device):
    """Renders on the device.  Returns (image on the host, stats): float[h][w][3] for the path tracer
    and the normal caster, float[h][w] depth or int64[h][w] counts for the other casters."""
    from .api import GpuScene
    gs = GpuScene(device, s.packed)
    try:
        if s.integrator == "path-tracer":
            return gs.pathtrace(s.camera, s.pt_params)
        return gs.raycast(s.camera, s.raycast_mode, stats=True)
    finally:
        gs.close()


def save(s, device, image, path=None):
    """Writes the image file the reference's saveImageToFile writes for this integrator."""
    import torch
    from .api import (count_to_rgb_device, depth_to_rgb_device, normal_to_rgb_device, rgb_to_bytes_device,
                      write_ppm_bytes)
    h, w = image.shape[:2]
    src = torch.from_numpy(np.ascontiguousarray(image)).cuda()
    rgb = torch.empty((h, w, 3), dtype=torch.float32, device="cuda")
    srgb = False
    if s.integrator == "path-tracer":
        rgb = src
        srgb = True          # PathTracer::saveImageToFile converts to sRGB first
    elif s.raycast_mode == abi.RAYCAST_NORMAL:
        rgb = src
        normal_to_rgb_device(device, rgb.data_ptr(), w, h)
    elif s.raycast_mode == abi.RAYCAST_DEPTH:
        depth_to_rgb_device(device, src.data_ptr(), w, h, rgb.data_ptr(), *s.prescribed)
    else:
        count_to_rgb_device(device, src.data_ptr(), w, h, rgb.data_ptr(), *s.prescribed)
    out = torch.empty(3 * w * h, dtype=torch.uint8, device="cuda")
    rgb_to_bytes_device(device, rgb.data_ptr(), 3 * w * h, out.data_ptr(), srgb=srgb)
    torch.cuda.synchronize()
    write_ppm_bytes(path or s.file_name, out.cpu().numpy().reshape(h, w, 3))


def main(argv=None):
    ap = argparse.ArgumentParser(description="Render a swpathtracer Lua scene on the GPU.")
    ap.add_argument("script")
    ap.add_argument("--lua-path", action="append", default=[], help="directory holding the lua_core modules")
    ap.add_argument("--out", default=None, help="image file (default: the script's ImageBuffer file_name)")
    ap.add_argument("--seed", type=int, default=1, help="Philox seed of the path tracer")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    from .api import Device
    s = load_lua(a.script, a.lua_path)
    if s.pt_params is not None:
        s.pt_params.seed = a.seed
    dev = Device(a.device)
    img, st = render(s, dev)
    save(s, dev, img, a.out)
    print("%s: %d primitives, %s, %.1f ms on the GPU -> %s" % (
        os.path.basename(a.script), s.packed.n_prims, s.integrator, st.gpu_ms if hasattr(st, "gpu_ms") else 0.0,
        a.out or s.file_name))
    dev.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
