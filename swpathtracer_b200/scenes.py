"""Scene descriptions and the synthetic workloads this backend is measured on.

SceneBuilder mirrors the reference's Lua scene DSL (lua_core/bsdfs.lua, layered_bsdfs.lua,
materials.lua, objects.lua): BSDFs, layered BSDFs and materials are numbered in creation
order and primitives keep their insertion order, which is the order the reference's
SBVH builder receives them in (core/scene.cpp:41-45).

The workloads are generated, not loaded: there is no dataset.  Every generator uses only
+, -, *, / and sqrt in float64 before the final cast to float32, so the same arguments
give the same bytes on any IEEE machine.
"""
import ctypes as C

import numpy as np

from . import abi

# ----------------------------------------------------------------------------------------
# scene builder
# ----------------------------------------------------------------------------------------

_ACCEL = {"none": abi.ACCEL_NONE, "bvh-sah": abi.ACCEL_BVH_SAH, "sbvh-sah": abi.ACCEL_SBVH_SAH}
_SAMPLER = {"uniform": abi.SAMPLER_UNIFORM, "importance": abi.SAMPLER_IMPORTANCE}


class SceneBuilder:
    """Collects a scene in the reference's object model and packs it as an spt_scene_desc."""

    def __init__(self, background=(0.0, 0.0, 0.0), acceleration_structure="bvh-sah"):
        self.background = tuple(float(c) for c in background)
        self.accel = _ACCEL[acceleration_structure]
        self.bsdfs = []          # (type, sampler, rgb, scalar)
        self.layered = []        # list of bsdf ids, top layer first
        self.materials = []      # (layered id, emission)
        self._chunks = []        # (types uint8[n], data f32[n,9], normals f32[n,9] | None, mat u32[n])

    # BSDFs (lua_core/bsdfs.lua) ---------------------------------------------------------
    def lambertian(self, kd=(0.75, 0.75, 0.75), bsdf_sampler="importance"):
        self.bsdfs.append((abi.BSDF_LAMBERTIAN, _SAMPLER[bsdf_sampler], tuple(kd), 0.0))
        return len(self.bsdfs) - 1

    def smooth_conductor(self, reflectance_at_normal_incidence=(0.99, 0.99, 0.99), bsdf_sampler="importance"):
        self.bsdfs.append((abi.BSDF_SMOOTH_CONDUCTOR, _SAMPLER[bsdf_sampler],
                           tuple(reflectance_at_normal_incidence), 0.0))
        return len(self.bsdfs) - 1

    def smooth_dielectric(self, ior=1.5, bsdf_sampler="importance"):
        self.bsdfs.append((abi.BSDF_SMOOTH_DIELECTRIC, _SAMPLER[bsdf_sampler], (0.0, 0.0, 0.0), float(ior)))
        return len(self.bsdfs) - 1

    def cook_torrance(self, roughness=0.2, reflectance_at_normal_incidence=(0.99, 0.99, 0.99),
                      bsdf_sampler="importance"):
        self.bsdfs.append((abi.BSDF_COOK_TORRANCE, _SAMPLER[bsdf_sampler],
                           tuple(reflectance_at_normal_incidence), float(roughness)))
        return len(self.bsdfs) - 1

    # LayeredBSDF / Material (lua_core/layered_bsdfs.lua, materials.lua) ---------------------
    def layered_bsdf(self, *bsdf_ids):
        self.layered.append([int(b) for b in bsdf_ids])
        return len(self.layered) - 1

    def material(self, bsdf, emission=(0.0, 0.0, 0.0)):
        self.materials.append((int(bsdf), tuple(float(e) for e in emission)))
        return len(self.materials) - 1

    # primitives (lua_core/objects.lua) ------------------------------------------------------
    def triangles(self, tris, material, normals=None):
        tris = np.ascontiguousarray(np.asarray(tris, dtype=np.float32).reshape(-1, 9))
        n = tris.shape[0]
        if normals is None:
            types = np.full(n, abi.PRIM_TRIANGLE, np.uint8)
        else:
            normals = np.ascontiguousarray(np.asarray(normals, dtype=np.float32).reshape(-1, 9))
            types = np.full(n, abi.PRIM_SMOOTH_TRIANGLE, np.uint8)
        mats = np.full(n, material, np.uint32) if np.isscalar(material) else np.asarray(material, np.uint32)
        self._chunks.append((types, tris, normals, mats))

    def triangle(self, v1, v2, v3, material):
        self.triangles(np.array([v1, v2, v3], np.float32), material)

    def smooth_triangle(self, v1, v2, v3, n1, n2, n3, material):
        self.triangles(np.array([v1, v2, v3], np.float32), material, normals=np.array([n1, n2, n3], np.float32))

    def sphere(self, center, radius, material):
        d = np.zeros((1, 9), np.float32)
        d[0, :3] = center
        d[0, 3] = radius
        self._chunks.append((np.array([abi.PRIM_SPHERE], np.uint8), d, None, np.array([material], np.uint32)))

    # packing ------------------------------------------------------------------------------
    def arrays(self):
        """Concatenated primitive arrays: (types, data[n,9], normals[n,9] | None, material)."""
        types = np.concatenate([c[0] for c in self._chunks]) if self._chunks else np.zeros(0, np.uint8)
        data = np.concatenate([c[1] for c in self._chunks]) if self._chunks else np.zeros((0, 9), np.float32)
        mats = np.concatenate([c[3] for c in self._chunks]) if self._chunks else np.zeros(0, np.uint32)
        if any(c[2] is not None for c in self._chunks):
            normals = np.concatenate([c[2] if c[2] is not None else np.zeros_like(c[1]) for c in self._chunks])
        else:
            normals = None
        return types, data, normals, mats

    def build(self):
        return PackedScene(self)


class PackedScene:
    """An spt_scene_desc plus the numpy arrays it points into (kept alive here)."""

    def __init__(self, sb):
        self.types, self.data, self.normals, self.mats = sb.arrays()
        self.data = np.ascontiguousarray(self.data, np.float32)
        self.bsdfs = (abi.Bsdf * max(1, len(sb.bsdfs)))()
        for i, (t, s, rgb, sc) in enumerate(sb.bsdfs):
            self.bsdfs[i].type, self.bsdfs[i].sampler, self.bsdfs[i].scalar = t, s, sc
            for k in range(3):
                self.bsdfs[i].rgb[k] = rgb[k]
        offs = [0]
        ids = []
        for lay in sb.layered:
            ids.extend(lay)
            offs.append(len(ids))
        self.layered_offsets = np.array(offs, np.uint32)
        self.layered_ids = np.array(ids if ids else [0], np.uint32)
        self.materials = (abi.Material * max(1, len(sb.materials)))()
        for i, (lay, em) in enumerate(sb.materials):
            self.materials[i].layered_bsdf = lay
            for k in range(3):
                self.materials[i].emission[k] = em[k]
        d = abi.SceneDesc()
        d.n_prims = len(self.types)
        d.prim_type = abi.ptr(self.types, C.c_uint8)
        d.prim_data = abi.ptr(self.data, C.c_float)
        d.prim_normals = abi.ptr(self.normals, C.c_float)
        d.prim_material = abi.ptr(self.mats, C.c_uint32)
        d.n_bsdfs = len(sb.bsdfs)
        d.bsdfs = C.cast(self.bsdfs, C.POINTER(abi.Bsdf))
        d.n_layered = len(sb.layered)
        d.layered_offsets = abi.ptr(self.layered_offsets, C.c_uint32)
        d.layered_bsdf_ids = abi.ptr(self.layered_ids, C.c_uint32)
        d.n_materials = len(sb.materials)
        d.materials = C.cast(self.materials, C.POINTER(abi.Material))
        for k in range(3):
            d.background[k] = sb.background[k]
        d.accel = sb.accel
        self.desc = d
        self.n_prims = d.n_prims
        self.n_materials = d.n_materials

    def ref(self):
        return C.byref(self.desc)


# ----------------------------------------------------------------------------------------
# geometry generators
# ----------------------------------------------------------------------------------------

def _lowbias32(h):
    """32-bit integer finaliser (xorshift-multiply avalanche) on a uint64 array holding uint32 values."""
    m = np.uint64(0xFFFFFFFF)
    h = h & m
    h ^= h >> np.uint64(16)
    h = (h * np.uint64(0x7FEB352D)) & m
    h ^= h >> np.uint64(15)
    h = (h * np.uint64(0x846CA68B)) & m
    h ^= h >> np.uint64(16)
    return h


def _lattice(ix, iy, iz, seed):
    m = np.uint64(0xFFFFFFFF)
    u = lambda a: a.astype(np.int64).astype(np.uint64) & m
    h = (u(ix) * np.uint64(0x8DA6B343)) ^ (u(iy) * np.uint64(0xD8163841)) ^ (u(iz) * np.uint64(0xCB1AB31F))
    h = (h ^ (np.uint64(seed) * np.uint64(0x165667B1))) & m
    return _lowbias32(h).astype(np.float64) * (2.0 / 4294967296.0) - 1.0


def value_noise(p, seed):
    """Trilinear value noise with smoothstep weights; p: float64 [n,3]; returns [-1, 1]."""
    f = np.floor(p)
    i = f.astype(np.int64)
    t = p - f
    w = t * t * (3.0 - 2.0 * t)
    out = np.zeros(p.shape[0])
    for dx in (0, 1):
        wx = w[:, 0] if dx else 1.0 - w[:, 0]
        for dy in (0, 1):
            wy = w[:, 1] if dy else 1.0 - w[:, 1]
            for dz in (0, 1):
                wz = w[:, 2] if dz else 1.0 - w[:, 2]
                out += wx * wy * wz * _lattice(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz, seed)
    return out


def fbm(p, octaves=8, seed=1, base_frequency=3.0):
    """Fractal sum of `octaves` value-noise octaves (lacunarity 2, gain 0.5), normalised to [-1, 1]."""
    total = np.zeros(p.shape[0])
    amp, norm, freq = 1.0, 0.0, base_frequency
    for o in range(octaves):
        total += amp * value_noise(p * freq, seed + 1013 * o)
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return total / norm


def icosphere(subdivisions):
    """Unit icosphere: (vertices float64 [v,3], faces int64 [f,3]) with outward counter-clockwise faces."""
    phi = (1.0 + np.sqrt(5.0)) / 2.0
    v = np.array([[-1, phi, 0], [1, phi, 0], [-1, -phi, 0], [1, -phi, 0],
                  [0, -1, phi], [0, 1, phi], [0, -1, -phi], [0, 1, -phi],
                  [phi, 0, -1], [phi, 0, 1], [-phi, 0, -1], [-phi, 0, 1]], np.float64)
    v /= np.sqrt((v * v).sum(1))[:, None]
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
                  [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
                  [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
                  [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    for _ in range(subdivisions):
        nv = v.shape[0]
        edges = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        lo, hi = edges.min(1), edges.max(1)
        keys, inv = np.unique(lo * nv + hi, return_inverse=True)
        a, b = keys // nv, keys % nv
        mid = v[a] + v[b]
        mid /= np.sqrt((mid * mid).sum(1))[:, None]
        v = np.concatenate([v, mid])
        nf = f.shape[0]
        m01, m12, m20 = (inv[:nf] + nv, inv[nf:2 * nf] + nv, inv[2 * nf:] + nv)
        f = np.concatenate([
            np.stack([f[:, 0], m01, m20], 1),
            np.stack([f[:, 1], m12, m01], 1),
            np.stack([f[:, 2], m20, m12], 1),
            np.stack([m01, m12, m20], 1)])
    # orient every face outward
    tri = v[f]
    n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    flip = (n * tri.sum(1)).sum(1) < 0
    f[flip] = f[flip][:, [0, 2, 1]]
    return v, f


def displaced_icosphere(subdivisions, radius=1.0, center=(0.0, 0.0, 0.0), amplitude=0.05, octaves=8, seed=1):
    """Icosphere with radial value-noise displacement r * (1 + amplitude * fbm(p)); float32 [n,3,3]."""
    v, f = icosphere(subdivisions)
    if amplitude != 0.0:
        v = v * (1.0 + amplitude * fbm(v, octaves=octaves, seed=seed))[:, None]
    v = v * radius + np.asarray(center, np.float64)[None, :]
    return v.astype(np.float32)[f]


def open_box(size=1.0, light_size=0.25):
    """Open unit cube (no front wall, z = size side) scaled by `size`.

    Returns (walls [10,3,3] float32 with inward-facing winding, wall colour index per triangle
    (0 grey back/floor/ceiling, 1 red left, 2 green right), light quad [2,3,3] facing down)."""
    s = float(size)
    P = lambda x, y, z: (x * s, y * s, z * s)
    quads = [
        (P(0, 0, 0), P(1, 0, 0), P(1, 1, 0), P(0, 1, 0), 0),   # back  z=0, normal +z
        (P(0, 0, 1), P(1, 0, 1), P(1, 0, 0), P(0, 0, 0), 0),   # floor y=0, normal +y
        (P(0, 1, 0), P(1, 1, 0), P(1, 1, 1), P(0, 1, 1), 0),   # ceiling y=1, normal -y
        (P(0, 0, 1), P(0, 0, 0), P(0, 1, 0), P(0, 1, 1), 1),   # left  x=0, normal +x
        (P(1, 0, 0), P(1, 0, 1), P(1, 1, 1), P(1, 1, 0), 2),   # right x=1, normal -x
    ]
    tris, cols = [], []
    for a, b, c, d, col in quads:
        tris += [(a, b, c), (a, c, d)]
        cols += [col, col]
    tris = np.array(tris, np.float32)
    # fix winding so that every wall normal points into the box
    n = np.cross(tris[:, 1] - tris[:, 0], tris[:, 2] - tris[:, 0])
    inward = np.array([0.5 * s, 0.5 * s, 0.5 * s], np.float32) - tris.mean(1)
    flip = (n * inward).sum(1) < 0
    tris[flip] = tris[flip][:, [0, 2, 1]]
    h = 0.5 * light_size * s
    y = s * (1.0 - 1e-3)
    c0 = 0.5 * s
    light = np.array([[(c0 - h, y, c0 - h), (c0 + h, y, c0 + h), (c0 + h, y, c0 - h)],
                      [(c0 - h, y, c0 - h), (c0 - h, y, c0 + h), (c0 + h, y, c0 + h)]], np.float32)
    n = np.cross(light[:, 1] - light[:, 0], light[:, 2] - light[:, 0])
    flip = n[:, 1] > 0
    light[flip] = light[flip][:, [0, 2, 1]]
    return tris, np.array(cols, np.int32), light


def camera(kind="pinhole", position=(0, 0, 1), look_at=(0, 0, 0), up=(0, 1, 0), fov=55.0, width=256, height=256,
           window=(-1.0, 1.0, -1.0, 1.0), viewport=None):
    """spt_camera for a pinhole (vertical fov in degrees) or orthographic camera."""
    c = abi.Camera()
    c.type = abi.CAMERA_PINHOLE if kind == "pinhole" else abi.CAMERA_ORTHOGRAPHIC
    for k in range(3):
        c.position[k], c.look_at[k], c.up[k] = position[k], look_at[k], up[k]
    c.fov_deg = fov
    c.min_x, c.max_x, c.min_y, c.max_y = window
    c.width, c.height = width, height
    vp = viewport if viewport is not None else (0, 0, width, height)
    c.vp_top, c.vp_left, c.vp_width, c.vp_height = vp
    return c


def pt_params(spp=16, sampler="jittered", termination="max-length", path_length=5, max_depth=0, seed=1,
              spp_offset=0):
    p = abi.PtParams()
    p.pixel_sampler = {"uniform": abi.PIXEL_UNIFORM, "regular": abi.PIXEL_REGULAR,
                       "jittered": abi.PIXEL_JITTERED}[sampler]
    p.spp = spp
    p.termination = abi.TERMINATE_MAX_DEPTH if termination == "max-length" else abi.TERMINATE_RUSSIAN_ROULETTE
    p.path_length = path_length
    p.max_depth = max_depth
    p.seed = seed
    p.spp_offset = spp_offset
    return p


# ----------------------------------------------------------------------------------------
# the measured workloads
# ----------------------------------------------------------------------------------------

WALL_COLOURS = [(0.75, 0.75, 0.75), (0.63, 0.06, 0.05), (0.14, 0.45, 0.09)]
CONDUCTOR_F0 = (0.95, 0.64, 0.54)


def _box_into(sb, size, light_size=0.25, emission=15.0):
    walls, cols, light = open_box(size, light_size)
    wall_mats = [sb.material(sb.layered_bsdf(sb.lambertian(kd=c))) for c in WALL_COLOURS]
    light_mat = sb.material(sb.layered_bsdf(sb.lambertian(kd=(0.0, 0.0, 0.0))), emission=(emission,) * 3)
    sb.triangles(walls, np.array([wall_mats[c] for c in cols], np.uint32))
    sb.triangles(light, light_mat)


def box_scene(subdivisions=5, radius=0.3, roughness=0.3):
    """Path tracer, CPU-runnable size: open unit box (10 wall tris + 2 emissive ceiling tris,
    radiance 15) around an icosphere of 20*4^subdivisions tris (20,480 at 5 subdivisions),
    radius 0.3, Cook-Torrance alpha 0.3, Schlick F0 (0.95, 0.64, 0.54)."""
    sb = SceneBuilder(background=(0.0, 0.0, 0.0))
    _box_into(sb, 1.0)
    m = sb.material(sb.layered_bsdf(sb.cook_torrance(roughness=roughness, reflectance_at_normal_incidence=CONDUCTOR_F0)))
    sb.triangles(displaced_icosphere(subdivisions, radius=radius, center=(0.5, radius, 0.5), amplitude=0.0), m)
    return sb


def box_camera(width=256, height=256, scale=1.0, fov=40.0):
    s = scale
    return camera("pinhole", position=(0.5 * s, 0.5 * s, 2.35 * s), look_at=(0.5 * s, 0.5 * s, 0.0), fov=fov,
                  width=width, height=height)


def displaced_mesh_scene(subdivisions=8, seed=1):
    """Ray-cast workload: icosphere with 20*4^subdivisions tris (1,310,720 at 8), radius 1 at the
    origin, radial value-noise displacement (amplitude 0.05, 8 octaves, seeded)."""
    sb = SceneBuilder(background=(0.0, 0.0, 0.0))
    m = sb.material(sb.layered_bsdf(sb.lambertian()))
    sb.triangles(displaced_icosphere(subdivisions, seed=seed), m)
    return sb


def displaced_mesh_camera(width=1920, height=1080):
    return camera("pinhole", position=(0.35, 0.4, 3.0), look_at=(0.0, 0.0, 0.0), fov=40.0, width=width, height=height)


def incoherent_rays(n, seed=1, half_extent=1.5):
    """n rays with origins uniform in a cube of side 2*half_extent at the origin and directions
    uniform on the sphere (z = 1 - 2u, phi = 2 pi v); float32 [n, 8] (origin, 0, dir, 0)."""
    g = np.random.Generator(np.random.Philox(seed))
    o = g.uniform(-half_extent, half_extent, size=(n, 3))
    z = 1.0 - 2.0 * g.random(n)
    ph = 2.0 * np.pi * g.random(n)
    s = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = o
    r[:, 4] = s * np.cos(ph)
    r[:, 5] = s * np.sin(ph)
    r[:, 6] = z
    return r


def small_light_box_scene(subdivisions=4, light_size=0.06):
    """Path guiding workload: the open unit box lit by a small ceiling light of the same power as the
    box scene's (radiance 15 * (0.25 / light_size)^2), around a Lambertian and a Cook-Torrance
    sphere.  The path tracer has no light sampling, so a path finds the light only by sampling its
    direction -- the case a learned directional distribution improves most."""
    sb = SceneBuilder(background=(0.0, 0.0, 0.0))
    _box_into(sb, 1.0, light_size=light_size, emission=15.0 * (0.25 / light_size) ** 2)
    diffuse = sb.material(sb.layered_bsdf(sb.lambertian(kd=(0.8, 0.8, 0.8))))
    metal = sb.material(sb.layered_bsdf(sb.cook_torrance(roughness=0.3, reflectance_at_normal_incidence=CONDUCTOR_F0)))
    sb.triangles(displaced_icosphere(subdivisions, radius=0.2, center=(0.3, 0.2, 0.45), amplitude=0.0), diffuse)
    sb.triangles(displaced_icosphere(subdivisions, radius=0.17, center=(0.72, 0.17, 0.6), amplitude=0.0), metal)
    return sb


def window_room_scene(window=0.1, subdivisions=4):
    """Path guiding workload: a room lit only through a square window.  The open unit box of the box
    scene, its right wall (x = 1) pierced by a window of side `window` centred at (y, z) = (0.6, 0.5),
    and outside it a 2 x 2 emitter of radiance 20 at x = 1.6 facing the room, plus a Lambertian
    sphere.  A path reaches the light only through the window, a small solid angle from most of the
    room: the directional case where a learned sampling distribution pays."""
    sb = SceneBuilder(background=(0.0, 0.0, 0.0))
    grey = sb.material(sb.layered_bsdf(sb.lambertian(kd=WALL_COLOURS[0])))
    red = sb.material(sb.layered_bsdf(sb.lambertian(kd=WALL_COLOURS[1])))
    light = sb.material(sb.layered_bsdf(sb.lambertian(kd=(0.0, 0.0, 0.0))), emission=(20.0, 20.0, 20.0))
    tris, mats = [], []

    def quad(a, b, c, d, m):
        tris.extend([[a, b, c], [a, c, d]])
        mats.extend([m, m])
    quad([0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], grey)          # back
    quad([0, 0, 1], [1, 0, 1], [1, 0, 0], [0, 0, 0], grey)          # floor
    quad([0, 1, 0], [1, 1, 0], [1, 1, 1], [0, 1, 1], grey)          # ceiling
    quad([0, 0, 1], [0, 0, 0], [0, 1, 0], [0, 1, 1], red)           # left
    zlo, zhi, ylo, yhi = 0.5 - window / 2, 0.5 + window / 2, 0.6 - window / 2, 0.6 + window / 2
    quad([1, 0, 0], [1, 0, 1], [1, ylo, 1], [1, ylo, 0], grey)      # right wall around the window
    quad([1, yhi, 0], [1, yhi, 1], [1, 1, 1], [1, 1, 0], grey)
    quad([1, ylo, 0], [1, ylo, zlo], [1, yhi, zlo], [1, yhi, 0], grey)
    quad([1, ylo, zhi], [1, ylo, 1], [1, yhi, 1], [1, yhi, zhi], grey)
    quad([1.6, -0.5, -0.5], [1.6, 1.5, -0.5], [1.6, 1.5, 1.5], [1.6, -0.5, 1.5], light)
    sb.triangles(np.array(tris, np.float32), np.array(mats, np.uint32))
    diffuse = sb.material(sb.layered_bsdf(sb.lambertian(kd=(0.8, 0.8, 0.8))))
    sb.triangles(displaced_icosphere(subdivisions, radius=0.2, center=(0.4, 0.2, 0.5), amplitude=0.0), diffuse)
    return sb


def layered_box_scene(subdivisions=8, seed=1):
    """Full path tracing at 1.3M tris: the displaced mesh (radius 1) inside the open box scaled x3,
    mesh material = LayeredBSDF{SmoothDielectric{ior 1.5}, CookTorrance{roughness 0.2}}."""
    sb = SceneBuilder(background=(0.0, 0.0, 0.0))
    _box_into(sb, 3.0)
    lay = sb.layered_bsdf(sb.smooth_dielectric(ior=1.5),
                          sb.cook_torrance(roughness=0.2, reflectance_at_normal_incidence=CONDUCTOR_F0))
    m = sb.material(lay)
    sb.triangles(displaced_icosphere(subdivisions, radius=1.0, center=(1.5, 1.06, 1.5), seed=seed), m)
    return sb


def layered_box_camera(width=800, height=600):
    return box_camera(width, height, scale=3.0)


def smooth_mesh_scene(subdivisions=4, seed=3):
    """Displaced icosphere as SmoothTriangle primitives (per-vertex normals = normalised vertex
    positions of the undisplaced sphere) plus one sphere, inside the open unit box: covers smooth
    normals, spheres and triangles in one tree."""
    sb = SceneBuilder(background=(0.2, 0.3, 0.4))
    _box_into(sb, 1.0)
    m = sb.material(sb.layered_bsdf(sb.cook_torrance(roughness=0.4, reflectance_at_normal_incidence=CONDUCTOR_F0)))
    v, f = icosphere(subdivisions)
    n = v.astype(np.float32)[f]
    pos = (v * (1.0 + 0.05 * fbm(v, seed=seed))[:, None] * 0.25 + np.array([0.35, 0.3, 0.5]))
    sb.triangles(pos.astype(np.float32)[f], m, normals=n)
    glass = sb.material(sb.layered_bsdf(sb.smooth_dielectric(ior=1.5)))
    sb.sphere((0.72, 0.18, 0.45), 0.17, glass)
    return sb


def furnace_scene(material="lambertian", reflectance=0.999):
    """White furnace (reference samples/furnace_test.lua): emissive sphere r=10, Le 0.5, around a unit
    sphere of the given material with reflectance 0.999."""
    sb = SceneBuilder(background=(0.0, 0.0, 0.0))
    light = sb.material(sb.layered_bsdf(sb.lambertian(kd=(0.0, 0.0, 0.0))), emission=(0.5, 0.5, 0.5))
    r = (reflectance,) * 3
    if material == "lambertian":
        lay = sb.layered_bsdf(sb.lambertian(kd=r))
    elif material == "smooth_conductor":
        lay = sb.layered_bsdf(sb.smooth_conductor(reflectance_at_normal_incidence=r))
    elif material == "smooth_dielectric":
        lay = sb.layered_bsdf(sb.smooth_dielectric(ior=1.49))
    elif material == "cook_torrance":
        lay = sb.layered_bsdf(sb.cook_torrance(roughness=0.2, reflectance_at_normal_incidence=r))
    elif material == "plastic":
        lay = sb.layered_bsdf(sb.smooth_dielectric(ior=1.49), sb.lambertian(kd=r))
    elif material == "coating":
        lay = sb.layered_bsdf(sb.smooth_dielectric(ior=1.49),
                              sb.cook_torrance(roughness=0.2, reflectance_at_normal_incidence=r))
    else:
        raise ValueError(material)
    m = sb.material(lay)
    sb.sphere((0.0, 0.0, 0.0), 10.0, light)
    sb.sphere((0.0, 0.0, 0.0), 1.0, m)
    return sb


def furnace_camera(width=64, height=64):
    return camera("orthographic", position=(0, 0, 6), look_at=(0, 0, 0), width=width, height=height,
                  window=(-1.25, 1.25, -1.25, 1.25))


def uv_sphere(n_tris, radius=1.0, center=(0.0, 0.0, 0.0), amplitude=0.05, octaves=8, seed=1):
    """Latitude-longitude sphere with about n_tris triangles (outward winding), radially displaced like
    displaced_icosphere; float32 [n, 3, 3]."""
    n_lon = max(3, int(round(np.sqrt(n_tris / 2.0))))
    n_lat = max(3, int(round(n_tris / (2.0 * n_lon))) + 1)
    th = np.arange(n_lat + 1) * (np.pi / n_lat)
    ph = np.arange(n_lon) * (2.0 * np.pi / n_lon)
    st, ct = np.sin(th), np.cos(th)
    v = np.stack([np.outer(st, np.cos(ph)), np.repeat(ct[:, None], n_lon, 1), np.outer(st, np.sin(ph))], -1)
    v = v.reshape(-1, 3)
    if amplitude != 0.0:
        v = v * (1.0 + amplitude * fbm(v, octaves=octaves, seed=seed))[:, None]
    v = v * radius + np.asarray(center, np.float64)[None, :]
    idx = lambda i, j: i * n_lon + (j % n_lon)
    faces = []
    for i in range(n_lat):
        j = np.arange(n_lon)
        a, b, c, d = idx(i, j), idx(i, j + 1), idx(i + 1, j), idx(i + 1, j + 1)
        if i > 0:
            faces.append(np.stack([a, b, c], 1))
        if i < n_lat - 1:
            faces.append(np.stack([b, d, c], 1))
    f = np.concatenate(faces)
    tri = v.astype(np.float32)[f]
    n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    cen = tri.mean(1) - np.asarray(center, np.float32)
    flip = (n * cen).sum(1) < 0
    tri[flip] = tri[flip][:, [0, 2, 1]]
    return tri


def batched_scenes(n=64, seed=2024, min_tris=1000, max_tris=500000, min_res=128, max_res=1024, spp=64,
                   max_tris_cap=None):
    """Uneven batch: n seeded scenes, each a displaced sphere of log-uniform [min_tris, max_tris]
    triangles (radius 0.3) in the open unit box, with a material drawn uniformly from {Lambertian,
    rough conductor alpha in [0.05, 0.6], smooth dielectric IOR in [1.3, 1.8], layered dielectric over
    rough conductor}, rendered at a log-uniform square resolution in [min_res, max_res] with `spp`
    jittered samples, max path length 5.  Returns [(SceneBuilder, camera, pt_params, description)]."""
    g = np.random.Generator(np.random.Philox(seed))
    out = []
    for i in range(n):
        n_tris = int(round(np.exp(g.uniform(np.log(min_tris), np.log(max_tris)))))
        if max_tris_cap:
            n_tris = min(n_tris, max_tris_cap)
        res = int(round(np.exp(g.uniform(np.log(min_res), np.log(max_res)))))
        kind = int(g.integers(0, 4))
        sb = SceneBuilder(background=(0.0, 0.0, 0.0))
        _box_into(sb, 1.0)
        if kind == 0:
            kd = tuple(float(x) for x in g.uniform(0.2, 0.9, 3))
            m = sb.material(sb.layered_bsdf(sb.lambertian(kd=kd)))
            desc = "lambertian"
        elif kind == 1:
            a = float(g.uniform(0.05, 0.6))
            m = sb.material(sb.layered_bsdf(sb.cook_torrance(roughness=a, reflectance_at_normal_incidence=CONDUCTOR_F0)))
            desc = "conductor a=%.2f" % a
        elif kind == 2:
            ior = float(g.uniform(1.3, 1.8))
            m = sb.material(sb.layered_bsdf(sb.smooth_dielectric(ior=ior)))
            desc = "dielectric ior=%.2f" % ior
        else:
            a = float(g.uniform(0.05, 0.6))
            m = sb.material(sb.layered_bsdf(sb.smooth_dielectric(ior=1.5),
                                            sb.cook_torrance(roughness=a, reflectance_at_normal_incidence=CONDUCTOR_F0)))
            desc = "layered a=%.2f" % a
        sb.triangles(uv_sphere(n_tris, radius=0.3, center=(0.5, 0.32, 0.5), seed=seed + i), m)
        params = pt_params(spp=spp, sampler="jittered", termination="max-length", path_length=5, seed=seed * 131 + i)
        out.append((sb, box_camera(res, res), params, "%d tris, %dx%d, %s" % (sb.arrays()[0].shape[0], res, res, desc)))
    return out
