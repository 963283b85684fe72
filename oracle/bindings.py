"""ctypes bindings of the CPU checkers -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.

* RefHarness wraps oracle/_ref/libswref.so: the reference renderer's own sources compiled by
  `make -C oracle ref` (present only where the reference sources were available at build time).
* Oracle wraps oracle/libspt_oracle.so: the project's CPU restatement of the reference
  algorithms (oracle/spt_oracle.cpp), built by `make -C oracle`.
"""
import ctypes as C
import os

import numpy as np

from swpathtracer_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libswref.so")
ORACLE_LIB = os.path.join(HERE, "libspt_oracle.so")

vp, u64, u32, i32, f32p = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int, C.POINTER(C.c_float)


def _nullable(a):
    return None if a is None else a.ctypes.data


class RefHarness:
    """The reference renderer's own code (oracle/ref_harness.cpp)."""

    def __init__(self, path=REF_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = self.lib = C.CDLL(path)
        L.swref_scene_create.restype = vp
        L.swref_scene_create.argtypes = [vp, C.c_char_p, i32]
        L.swref_scene_destroy.argtypes = [vp]
        L.swref_tree_stats.argtypes = [vp, vp]
        L.swref_tree_export.argtypes = [vp, vp, vp, vp, vp]
        L.swref_intersect.argtypes = [vp, vp, u64, vp, vp, vp, vp, vp, i32, vp]
        L.swref_camera_rays.argtypes = [vp, vp]
        L.swref_raycast.argtypes = [vp, vp, i32, vp, vp, i32, vp]
        L.swref_pathtrace.argtypes = [vp, vp, vp, vp, i32, vp]
        L.swref_eval_material.argtypes = [vp, u32, vp, u64, vp, u64]
        L.swref_bsdf_f.argtypes = [vp, u32, vp, vp, u64, vp]

    def scene(self, packed, dump_path=None, n_threads=0):
        h = self.lib.swref_scene_create(C.addressof(packed.desc), dump_path.encode() if dump_path else None, n_threads)
        return RefScene(self, h, packed)


class RefScene:
    def __init__(self, harness, handle, packed):
        self.h, self.lib, self.packed = handle, harness.lib, packed

    def close(self):
        if self.h:
            self.lib.swref_scene_destroy(self.h)
            self.h = None

    __del__ = close

    def tree_stats(self):
        s = abi.BvhStats()
        if self.lib.swref_tree_stats(self.h, C.addressof(s)) != 0:
            return None
        return s

    def tree(self):
        nn, nr = C.c_uint64(), C.c_uint64()
        self.lib.swref_tree_export(self.h, None, C.addressof(nn), None, C.addressof(nr))
        nodes = np.zeros(nn.value, abi.BVH2_NODE_DTYPE)
        refs = np.zeros(nr.value, np.uint32)
        self.lib.swref_tree_export(self.h, nodes.ctypes.data, C.addressof(nn), refs.ctypes.data, C.addressof(nr))
        return nodes, refs

    def intersect(self, rays, n_threads=0, want_normals=True):
        n = rays.shape[0]
        rays = np.ascontiguousarray(rays, np.float32)
        hits = np.zeros(n, abi.HIT_DTYPE)
        normals = np.zeros((n, 3), np.float32) if want_normals else None
        tests = np.zeros(n, np.uint32)
        nhits = np.zeros(n, np.uint32)
        ptests = np.zeros(n, np.uint32)
        sec = C.c_double()
        self.lib.swref_intersect(self.h, rays.ctypes.data, n, hits.ctypes.data, _nullable(normals), tests.ctypes.data,
                                 nhits.ctypes.data, ptests.ctypes.data, n_threads, C.addressof(sec))
        return dict(hits=hits, normals=normals, tests=tests, nhits=nhits, prim_tests=ptests, seconds=sec.value)

    def raycast(self, cam, mode, n_threads=0):
        shape = {abi.RAYCAST_NORMAL: ((cam.height, cam.width, 3), np.float32),
                 abi.RAYCAST_DEPTH: ((cam.height, cam.width), np.float32),
                 abi.RAYCAST_COUNT: ((cam.height, cam.width), np.int64)}[mode]
        out = np.zeros(*shape)
        st = abi.RenderStats()
        sec = C.c_double()
        self.lib.swref_raycast(self.h, C.addressof(cam), mode, out.ctypes.data, C.addressof(st), n_threads,
                               C.addressof(sec))
        return out, st, sec.value

    def pathtrace(self, cam, params, n_threads=0):
        out = np.zeros((cam.height, cam.width, 3), np.float32)
        sec = C.c_double()
        rc = self.lib.swref_pathtrace(self.h, C.addressof(cam), C.addressof(params), out.ctypes.data, n_threads,
                                      C.addressof(sec))
        if rc != 0:
            raise RuntimeError("swref_pathtrace failed with %d" % rc)
        return out, sec.value

    def eval_material(self, mat, wo, seed=1):
        wo = np.ascontiguousarray(wo, np.float32)
        out = np.zeros((wo.shape[0], 10), np.float32)
        self.lib.swref_eval_material(self.h, mat, wo.ctypes.data, wo.shape[0], out.ctypes.data, seed)
        return out

    def bsdf_f(self, bsdf, wo, wi):
        wo = np.ascontiguousarray(wo, np.float32)
        wi = np.ascontiguousarray(wi, np.float32)
        out = np.zeros((wo.shape[0], 6), np.float32)
        self.lib.swref_bsdf_f(self.h, bsdf, wo.ctypes.data, wi.ctypes.data, wo.shape[0], out.ctypes.data)
        return out


def camera_rays(cam, harness):
    """The reference's Camera::getRay at every pixel centre (row-major [y][x], 8 floats per ray)."""
    rays = np.zeros((cam.height * cam.width, 8), np.float32)
    harness.lib.swref_camera_rays(C.addressof(cam), rays.ctypes.data)
    return rays


class Oracle:
    """The project's CPU restatement (oracle/spt_oracle.cpp)."""

    def __init__(self, path=ORACLE_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = self.lib = C.CDLL(path)
        L.spto_philox4x32_10.argtypes = [vp, vp, vp]
        L.spto_scene_create.restype = vp
        L.spto_scene_create.argtypes = [vp]
        L.spto_scene_destroy.argtypes = [vp]
        L.spto_bvh_build.argtypes = [vp]
        L.spto_tree_stats.argtypes = [vp, vp]
        L.spto_tree_export.argtypes = [vp, vp, vp, vp, vp]
        L.spto_intersect.argtypes = [vp, vp, u64, vp, vp, vp, vp, i32]
        L.spto_camera_rays.argtypes = [vp, vp]
        L.spto_raycast.argtypes = [vp, vp, i32, vp, vp, i32]
        L.spto_pathtrace.argtypes = [vp, vp, vp, vp, i32, vp, vp]
        L.spto_eval_material.argtypes = [vp, u32, vp, u64, vp, u64, u64, u32]
        L.spto_depth_to_rgb.argtypes = [vp, u32, u32, C.c_float, C.c_float, vp]
        L.spto_count_to_rgb.argtypes = [vp, u32, u32, C.c_int64, C.c_int64, u64, u64, vp]

    def philox(self, ctr, key):
        c = np.asarray(ctr, np.uint32)
        k = np.asarray(key, np.uint32)
        out = np.zeros(4, np.uint32)
        self.lib.spto_philox4x32_10(c.ctypes.data, k.ctypes.data, out.ctypes.data)
        return out

    def scene(self, packed, build=True):
        h = self.lib.spto_scene_create(C.addressof(packed.desc))
        s = OracleScene(self, h, packed)
        if build:
            rc = self.lib.spto_bvh_build(h)
            if rc != 0:
                raise RuntimeError("oracle build failed: %d" % rc)
        return s

    def camera_rays(self, cam):
        rays = np.zeros((cam.height * cam.width, 8), np.float32)
        self.lib.spto_camera_rays(C.addressof(cam), rays.ctypes.data)
        return rays

    def depth_to_rgb(self, depth, min_d=-1.0, max_d=-1.0):
        h, w = depth.shape
        rgb = np.zeros((h, w, 3), np.float32)
        self.lib.spto_depth_to_rgb(np.ascontiguousarray(depth, np.float32).ctypes.data, w, h, min_d, max_d,
                                   rgb.ctypes.data)
        return rgb

    def count_to_rgb(self, count, min_pp, max_pp, min_c=-1, max_c=-1):
        h, w = count.shape
        rgb = np.zeros((h, w, 3), np.float32)
        self.lib.spto_count_to_rgb(np.ascontiguousarray(count, np.int64).ctypes.data, w, h, min_c, max_c, min_pp,
                                   max_pp, rgb.ctypes.data)
        return rgb


class OracleScene:
    def __init__(self, oracle, handle, packed):
        self.h, self.lib, self.packed = handle, oracle.lib, packed

    def close(self):
        if self.h:
            self.lib.spto_scene_destroy(self.h)
            self.h = None

    __del__ = close

    def tree_stats(self):
        s = abi.BvhStats()
        if self.lib.spto_tree_stats(self.h, C.addressof(s)) != 0:
            return None
        return s

    def tree(self):
        nn, nr = C.c_uint64(), C.c_uint64()
        self.lib.spto_tree_export(self.h, None, C.addressof(nn), None, C.addressof(nr))
        nodes = np.zeros(nn.value, abi.BVH2_NODE_DTYPE)
        refs = np.zeros(nr.value, np.uint32)
        self.lib.spto_tree_export(self.h, nodes.ctypes.data, C.addressof(nn), refs.ctypes.data, C.addressof(nr))
        return nodes, refs

    def intersect(self, rays, n_threads=0, want_normals=True):
        n = rays.shape[0]
        rays = np.ascontiguousarray(rays, np.float32)
        hits = np.zeros(n, abi.HIT_DTYPE)
        normals = np.zeros((n, 3), np.float32) if want_normals else None
        tests = np.zeros(n, np.uint32)
        nhits = np.zeros(n, np.uint32)
        self.lib.spto_intersect(self.h, rays.ctypes.data, n, hits.ctypes.data, _nullable(normals), tests.ctypes.data,
                                nhits.ctypes.data, n_threads)
        return dict(hits=hits, normals=normals, tests=tests, nhits=nhits)

    def raycast(self, cam, mode, n_threads=0):
        shape = {abi.RAYCAST_NORMAL: ((cam.height, cam.width, 3), np.float32),
                 abi.RAYCAST_DEPTH: ((cam.height, cam.width), np.float32),
                 abi.RAYCAST_COUNT: ((cam.height, cam.width), np.int64)}[mode]
        out = np.zeros(*shape)
        st = abi.RenderStats()
        self.lib.spto_raycast(self.h, C.addressof(cam), mode, out.ctypes.data, C.addressof(st), n_threads)
        return out, st

    def pathtrace(self, cam, params, n_threads=0):
        out = np.zeros((cam.height, cam.width, 3), np.float32)
        sec = C.c_double()
        seg = C.c_uint64()
        self.lib.spto_pathtrace(self.h, C.addressof(cam), C.addressof(params), out.ctypes.data, n_threads,
                                C.addressof(sec), C.addressof(seg))
        return out, sec.value, seg.value

    def eval_material(self, mat, wo, seed=1, path0=0, depth=0):
        wo = np.ascontiguousarray(wo, np.float32)
        out = np.zeros((wo.shape[0], 10), np.float32)
        self.lib.spto_eval_material(self.h, mat, wo.ctypes.data, wo.shape[0], out.ctypes.data, seed, path0, depth)
        return out
