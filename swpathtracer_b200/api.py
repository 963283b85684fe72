"""Python face of the backend: thin objects over the C-ABI handles.

Device            spt_context on one CUDA device
Bvh               spt_bvh, the host-built reference SAH tree (SBVH::build / getStatistics)
GpuScene          spt_scene: a scene resident in HBM, answering ray queries and rendering
"""
import atexit
import ctypes as C
import weakref

import numpy as np

from . import abi, native


class _Owned:
    """A handle that lives on a context, with the call that frees it; released at most once."""
    __slots__ = ("h", "free")

    def __init__(self, h, free):
        self.h, self.free = h, free

    def release(self):
        h, self.h = self.h, None
        if h:
            self.free(h)


_live_devices = weakref.WeakSet()


@atexit.register
def _close_live_devices():
    # before interpreter teardown, while the CUDA runtime is intact: free every handle, then contexts
    for d in list(_live_devices):
        d.close()


class Device:
    """A context on one CUDA device (its stream, events and scratch buffers)."""

    def __init__(self, device=0):
        self.lib = native.lib()
        h = C.c_void_p()
        native.check(self.lib.spt_create(device, C.byref(h)), None, "spt_create(%d)" % device)
        self.h = h
        self.device = device
        self._owned = []    # handles of scenes and guides on this context, freed before it
        _live_devices.add(self)

    def adopt(self, h, free):
        """Registers a handle that must be released before the context; returns its _Owned."""
        self._owned = [o for o in self._owned if o.h]
        o = _Owned(h, free)
        self._owned.append(o)
        return o

    def close(self):
        if getattr(self, "h", None):
            for o in reversed(self._owned):
                o.release()
            self._owned = []
            self.lib.spt_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, status, what=""):
        native.check(status, self.h, what)


class Bvh:
    """A binary BVH for a packed scene.  By default the reference's own SAH tree, built on the host
    (acceleration/sbvh.cpp:12-37).  With `device`, a tree of similar quality built on that device in
    milliseconds (spt_bvh_build_device): the same closest hits except between primitives hit at an
    equal t, and this tree's hit counts."""

    def __init__(self, packed, n_threads=0, device=None):
        self.lib = native.lib()
        h = C.c_void_p()
        if device is None:
            native.check(self.lib.spt_bvh_build(packed.ref(), n_threads, C.byref(h)), None, "spt_bvh_build")
        else:
            device.check(self.lib.spt_bvh_build_device(device.h, packed.ref(), C.byref(h)), "spt_bvh_build_device")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.spt_bvh_free(self.h)
            self.h = None

    __del__ = close

    def statistics(self):
        s = abi.BvhStats()
        native.check(self.lib.spt_bvh_stats_get(self.h, C.byref(s)))
        return s

    def export(self):
        nn, nr = C.c_uint64(), C.c_uint64()
        self.lib.spt_bvh_export(self.h, None, C.byref(nn), None, C.byref(nr))
        nodes = np.zeros(nn.value, abi.BVH2_NODE_DTYPE)
        refs = np.zeros(nr.value, np.uint32)
        native.check(self.lib.spt_bvh_export(self.h, nodes.ctypes.data, C.byref(nn), refs.ctypes.data, C.byref(nr)))
        return nodes, refs


_MODE_OUT = {abi.RAYCAST_NORMAL: (np.float32, 3), abi.RAYCAST_DEPTH: (np.float32, 1), abi.RAYCAST_COUNT: (np.int64, 1)}


def ray_array(rays, widths):
    """rays as a contiguous float32 [n, w] array with w in `widths`: 8 = origin, 0, direction, 0 (the
    padded layout of spt_intersect); 6 = origin, direction (the reference's Ray, spt_intersect_packed).
    Anything else raises ValueError: the C-ABI reads n * w floats from the pointer it is given."""
    rays = np.ascontiguousarray(rays, np.float32)
    if rays.ndim != 2 or rays.shape[1] not in widths:
        raise ValueError("rays must be float32 [n, w] with w in %s, got shape %s" % (tuple(widths), rays.shape))
    return rays


class GpuScene:
    """A scene uploaded to the device (Scene + its acceleration structure)."""

    def __init__(self, device, packed, bvh=None):
        self.dev = device
        self.lib = device.lib
        self.packed = packed
        h = C.c_void_p()
        device.check(self.lib.spt_scene_create(device.h, packed.ref(), bvh.h if bvh else None, C.byref(h)),
                     "spt_scene_create")
        self.h = h
        self._own = device.adopt(h, self.lib.spt_scene_destroy)

    def close(self):
        own = getattr(self, "_own", None)
        if own is not None:
            own.release()
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def device_bytes(self):
        return self.lib.spt_scene_device_bytes(self.h)

    # ---- ray queries -------------------------------------------------------------------------
    def intersect(self, rays, counts=False, out=None, out_counts=None):
        """Closest hit per ray (rays: float32 [n, 8] = origin, 0, direction, 0; or [n, 6] = the reference's
        Ray layout, origin then direction, through spt_intersect_packed); counts adds the reference's
        per-ray test counts.
        out: optional preallocated (e.g. pinned) array of abi.HIT_DTYPE for the hits; out_counts:
        optional (tests, nhits) uint32 arrays for the counts.  With every buffer page-locked, large
        batches run as a pipeline of chunks whose copies overlap the queries."""
        rays = ray_array(rays, (8, 6))
        n = rays.shape[0]
        hits = out if out is not None else np.zeros(n, abi.HIT_DTYPE)
        if hits.dtype != abi.HIT_DTYPE or hits.shape != (n,) or not hits.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be a contiguous array of %d HIT_DTYPE records" % n)
        if out_counts is not None:
            tests, nh = out_counts
            if not all(a.dtype == np.uint32 and a.shape == (n,) and a.flags["C_CONTIGUOUS"] for a in (tests, nh)):
                raise ValueError("out_counts must be two contiguous uint32 arrays of length %d" % n)
        else:
            tests = np.zeros(n, np.uint32) if counts else None
            nh = np.zeros(n, np.uint32) if counts else None
        fn = self.lib.spt_intersect_packed if rays.shape[1] == 6 else self.lib.spt_intersect
        self.dev.check(fn(self.dev.h, self.h, rays.ctypes.data, n, hits.ctypes.data,
                          None if tests is None else tests.ctypes.data, None if nh is None else nh.ctypes.data),
                       "spt_intersect")
        return dict(hits=hits, tests=tests, nhits=nh)

    def intersect_noalloc(self, rays, counts=False):
        """intersect() through spt_intersect_noalloc (include/spt_noalloc.h): no device allocation in
        the call, at most 65536 rays, calls on one device must not overlap."""
        rays = ray_array(rays, (8,))
        n = rays.shape[0]
        hits = np.zeros(n, abi.HIT_DTYPE)
        tests = np.zeros(n, np.uint32) if counts else None
        nh = np.zeros(n, np.uint32) if counts else None
        self.dev.check(self.lib.spt_intersect_noalloc(self.dev.h, self.h, rays.ctypes.data, n, hits.ctypes.data,
                                                      None if tests is None else tests.ctypes.data,
                                                      None if nh is None else nh.ctypes.data),
                       "spt_intersect_noalloc")
        return dict(hits=hits, tests=tests, nhits=nh)

    def intersect_device(self, d_rays, n, d_hits, stream=0):
        """Closest hits of n device rays (8 floats each); a batch of at least 2^21 rays is traced in
        coherence order (the same hits)."""
        self.dev.check(self.lib.spt_intersect_device(self.dev.h, self.h, d_rays, n, d_hits, stream),
                       "spt_intersect_device")

    def ray_order_device(self, d_rays, n, d_order, stream=0):
        """Stage 1 of intersect_device: the coherence order of n device rays into d_order (2n + 1
        uint32: the rays that meet the scene's box in order, then each ray's place in it or
        0xFFFFFFFF, then the number of those rays)."""
        self.dev.check(self.lib.spt_ray_order_device(self.dev.h, self.h, d_rays, n, d_order, stream),
                       "spt_ray_order_device")

    def intersect_ordered_device(self, d_rays, d_order, n, d_hits_ordered, stream=0):
        """Stage 2: closest hits of the rays d_rays[d_order[k]] into d_hits_ordered[k]."""
        self.dev.check(self.lib.spt_intersect_ordered_device(self.dev.h, self.h, d_rays, d_order, n, d_hits_ordered,
                                                             stream), "spt_intersect_ordered_device")

    def hits_unorder_device(self, d_order, n, d_hits_ordered, d_hits, stream=0):
        """Stage 3: d_hits[i] = d_hits_ordered[d_order[n + i]]."""
        self.dev.check(self.lib.spt_hits_unorder_device(self.dev.h, d_order, n, d_hits_ordered, d_hits, stream),
                       "spt_hits_unorder_device")

    def traversal_work_device(self, d_rays, n, d_hits):
        """The closest-hit kernel's own work on n device rays: (8-wide node visits, primitive tests)."""
        w = (C.c_uint64 * 2)()
        self.dev.check(self.lib.spt_traversal_work_device(self.dev.h, self.h, d_rays, n, d_hits, w),
                       "spt_traversal_work_device")
        return int(w[0]), int(w[1])

    def count_device(self, d_rays, n, d_ref_hits, d_tests, d_hits, d_prim_tests=None, stream=0):
        """The reference-order traversal: its hit (d_ref_hits) and per-ray test counts; any may be None."""
        self.dev.check(self.lib.spt_count_device(self.dev.h, self.h, d_rays, n, d_ref_hits, d_tests, d_hits,
                                                 d_prim_tests, stream), "spt_count_device")

    # ---- integrators -------------------------------------------------------------------------
    def raycast(self, cam, mode, stats=False):
        dt, ch = _MODE_OUT[mode]
        shape = (cam.height, cam.width, 3) if ch == 3 else (cam.height, cam.width)
        out = np.zeros(shape, dt)
        st = abi.RenderStats() if stats else None
        self.dev.check(self.lib.spt_raycast_image(self.dev.h, self.h, C.byref(cam), mode, out.ctypes.data,
                                                  C.byref(st) if st is not None else None), "spt_raycast_image")
        return (out, st) if stats else out

    def raycast_device(self, cam, mode, d_out, stream=0):
        self.dev.check(self.lib.spt_raycast_image_device(self.dev.h, self.h, C.byref(cam), mode, d_out, stream),
                       "spt_raycast_image_device")

    def pathtrace(self, cam, params):
        out = np.zeros((cam.height, cam.width, 3), np.float32)
        st = abi.RenderStats()
        self.dev.check(self.lib.spt_pathtrace(self.dev.h, self.h, C.byref(cam), C.byref(params), out.ctypes.data,
                                              C.byref(st)), "spt_pathtrace")
        return out, st

    def pathtrace_device(self, cam, params, d_out):
        st = abi.RenderStats()
        self.dev.check(self.lib.spt_pathtrace_device(self.dev.h, self.h, C.byref(cam), C.byref(params), d_out,
                                                     C.byref(st)), "spt_pathtrace_device")
        return st

    def pathtrace_guided_device(self, cam, params, guide, d_out):
        """Guided path tracing into the device buffer d_out (float[h][w][3]); the guide trains on the
        render's own paths for up to its config's max_steps optimiser steps."""
        st = abi.RenderStats()
        self.dev.check(self.lib.spt_guided_pathtrace_device(self.dev.h, self.h, C.byref(cam), C.byref(params),
                                                            guide.h, d_out, C.byref(st)),
                       "spt_guided_pathtrace_device")
        return st


def default_tune():
    t = abi.Tune()
    native.check(native.lib().spt_tune_default(C.byref(t)))
    return t


def _batch_jobs(jobs):
    arr = (abi.BatchJob * len(jobs))()
    for i, (scene, cam, params) in enumerate(jobs):
        arr[i].scene = scene.h.value if hasattr(scene.h, "value") else scene.h
        arr[i].camera = cam
        arr[i].params = params
    return arr


def render_batch(device, jobs, d_images, tune=None):
    """Renders jobs = [(GpuScene, camera, pt_params), ...] in one wavefront into the device buffers
    d_images (device pointers, float[h][w][3] each).  Returns per-job RenderStats."""
    arr = _batch_jobs(jobs)
    ptrs = (C.c_void_p * len(jobs))(*d_images)
    stats = (abi.RenderStats * len(jobs))()
    device.check(device.lib.spt_batch_pathtrace(device.h, arr, len(jobs), ptrs, C.byref(tune) if tune else None,
                                                stats), "spt_batch_pathtrace")
    return list(stats)


def autotune(device, jobs, cache_path=None):
    """Wavefront settings for this batch, from short timed trials (or the cache file)."""
    arr = _batch_jobs(jobs)
    t = abi.Tune()
    device.check(device.lib.spt_autotune(device.h, arr, len(jobs), cache_path.encode() if cache_path else None,
                                         C.byref(t)), "spt_autotune")
    return t


def guide_config(box_min=(0, 0, 0), box_max=(1, 1, 1), lr=1e-2, batch=1 << 18, max_steps=256, mix=0.5, seed=1,
                 cache_res=0, train_path=abi.GUIDE_TRAIN_TCGEN05, guided_depth=0):
    """train_path: abi.GUIDE_TRAIN_TCGEN05 (the training GEMMs on tcgen05 with tensor-memory
    accumulators, tiles of 128 records) or abi.GUIDE_TRAIN_MMA_SYNC (warp-level mma.sync).
    guided_depth: guide the path vertices at depth < guided_depth only (0: all)."""
    c = abi.GuideConfig()
    for k in range(3):
        c.box_min[k], c.box_max[k] = box_min[k], box_max[k]
    c.lr, c.batch, c.max_steps, c.mix, c.seed, c.cache_res = lr, batch, max_steps, mix, seed, cache_res
    c.train_path, c.guided_depth = train_path, guided_depth
    return c


class Guide:
    """The neural path-guiding model (hash grid + MLP -> 8 vMF lobes) on one device."""

    def __init__(self, device, config=None):
        self.dev = device
        self.lib = device.lib
        h = C.c_void_p()
        device.check(self.lib.spt_guide_create(device.h, C.byref(config or guide_config()), C.byref(h)),
                     "spt_guide_create")
        self.h = h
        self._own = device.adopt(h, self.lib.spt_guide_destroy)

    def close(self):
        own = getattr(self, "_own", None)
        if own is not None:
            own.release()
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def steps(self):
        """Optimiser steps taken since creation."""
        n = C.c_uint64()
        native.check(self.lib.spt_guide_steps(self.h, C.byref(n)))
        return n.value

    def get_params(self):
        grid = np.zeros(abi.GUIDE_GRID_PARAMS, np.float32)
        mlp = np.zeros(abi.GUIDE_MLP_PARAMS, np.float32)
        native.check(self.lib.spt_guide_get_params(self.h, grid.ctypes.data, mlp.ctypes.data))
        return grid, mlp

    def set_params(self, grid=None, mlp=None):
        g = None if grid is None else np.ascontiguousarray(grid, np.float32)
        m = None if mlp is None else np.ascontiguousarray(mlp, np.float32)
        native.check(self.lib.spt_guide_set_params(self.h, None if g is None else g.ctypes.data,
                                                   None if m is None else m.ctypes.data))

    def eval(self, pos, normal, wo):
        n = len(pos)
        x = np.zeros((n, 12), np.float32)
        x[:, 0:3], x[:, 4:7], x[:, 8:11] = pos, normal, wo
        out = np.zeros((n, 40), np.float32)
        self.dev.check(self.lib.spt_guide_eval(self.dev.h, self.h, x.ctypes.data, n, out.ctypes.data), "spt_guide_eval")
        return out.reshape(n, 8, 5)

    def gradients(self, recs):
        recs = np.ascontiguousarray(recs, abi.GUIDE_RECORD_DTYPE)
        grid = np.zeros(abi.GUIDE_GRID_PARAMS, np.float32)
        mlp = np.zeros(abi.GUIDE_MLP_PARAMS, np.float32)
        loss = C.c_float()
        self.dev.check(self.lib.spt_guide_gradients(self.dev.h, self.h, recs.ctypes.data, len(recs), grid.ctypes.data,
                                                    mlp.ctypes.data, C.byref(loss)), "spt_guide_gradients")
        return grid, mlp, loss.value

    def train_device(self, d_recs, n):
        """One Adam step on n records already on the device (d_recs: device pointer to n
        GUIDE_RECORD_DTYPE records); returns the step's device time in ms."""
        ms = C.c_float()
        self.dev.check(self.lib.spt_guide_train_device(self.dev.h, self.h, d_recs, n, C.byref(ms)),
                       "spt_guide_train_device")
        return ms.value

    def train(self, recs):
        recs = np.ascontiguousarray(recs, abi.GUIDE_RECORD_DTYPE)
        loss = C.c_float()
        self.dev.check(self.lib.spt_guide_train(self.dev.h, self.h, recs.ctypes.data, len(recs), C.byref(loss)),
                       "spt_guide_train")
        return loss.value


def depth_to_rgb_device(device, d_depth, width, height, d_rgb, min_depth=-1.0, max_depth=-1.0, stream=0):
    """DepthRayCaster::saveImageToFile's grey ramp on the device (float[h][w] -> float[h][w][3])."""
    device.check(device.lib.spt_depth_to_rgb_device(device.h, d_depth, width, height, min_depth, max_depth, d_rgb,
                                                    stream), "spt_depth_to_rgb_device")


def count_to_rgb_device(device, d_count, width, height, d_rgb, min_count=-1, max_count=-1, stream=0):
    """IntTestCountRayCaster::saveImageToFile's heat map on the device (int64[h][w] -> float[h][w][3])."""
    device.check(device.lib.spt_count_to_rgb_device(device.h, d_count, width, height, min_count, max_count, d_rgb,
                                                    stream), "spt_count_to_rgb_device")


def normal_to_rgb_device(device, d_rgb, width, height, stream=0):
    """NormalRayCaster::saveImageToFile's n * 0.5 + 0.5 encoding, in place on the device."""
    device.check(device.lib.spt_normal_to_rgb_device(device.h, d_rgb, width, height, stream),
                 "spt_normal_to_rgb_device")


def rgb_to_bytes_device(device, d_rgb, n_values, d_bytes, srgb=True, stream=0):
    """convertTosRGB (when srgb) and the 8-bit quantization of ImageBuffer::saveToFile on the device."""
    device.check(device.lib.spt_rgb_to_bytes_device(device.h, d_rgb, n_values, 1 if srgb else 0, d_bytes, stream),
                 "spt_rgb_to_bytes_device")


def write_ppm_bytes(path, rgb8):
    """The P3 file of ImageBuffer::saveToFile from quantized bytes (uint8 [h, w, 3], host)."""
    rgb8 = np.ascontiguousarray(rgb8, np.uint8)
    h, w = rgb8.shape[:2]
    native.check(native.lib().spt_write_ppm_bytes(path.encode(), rgb8.ctypes.data, w, h), None, "spt_write_ppm_bytes")


def write_ppm(path, rgb, srgb=True):
    """ImageBuffer::saveToFile (core/image_buffer.cpp:32-47), with convertTosRGB first when srgb."""
    rgb = np.ascontiguousarray(rgb, np.float32)
    h, w = rgb.shape[:2]
    native.check(native.lib().spt_write_ppm(path.encode(), rgb.ctypes.data, w, h, 1 if srgb else 0), None,
                 "spt_write_ppm")
