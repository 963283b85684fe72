"""The C-ABI library loads, exports every entry point include/spt.h declares, and rejects bad input
without a GPU (no compute calls here)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from swpathtracer_b200 import abi, native, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"^\s*(?:spt_status|uint32_t|uint64_t|const char\s*\*)\s+(spt_\w+)\s*\(", src, re.M)
    return names


def test_library_loads_and_exports_every_declared_symbol():
    L = native.lib()
    names = declared_functions()
    assert "spt_intersect" in names and "spt_pathtrace" in names
    for n in names:
        assert hasattr(L, n), n
        assert n in native.PROTOTYPES, "no ctypes prototype for " + n


def test_abi_version():
    assert native.lib().spt_abi_version() == abi.SPT_ABI_VERSION


def test_struct_sizes_match_header():
    # sizes as laid out by the C compiler for include/spt.h (x86-64)
    assert C.sizeof(abi.Bsdf) == 24
    assert C.sizeof(abi.Material) == 16
    assert C.sizeof(abi.Hit) == 16 and abi.HIT_DTYPE.itemsize == 16
    assert C.sizeof(abi.Bvh2Node) == 32 and abi.BVH2_NODE_DTYPE.itemsize == 32
    assert C.sizeof(abi.PtParams) == 32
    assert C.sizeof(abi.Camera) == 84
    assert C.sizeof(abi.GuideConfig) == 64


def test_bvh_build_rejects_bad_descriptions():
    L = native.lib()
    sb = scenes.box_scene(1)
    packed = sb.build()
    h = C.c_void_p()
    bad = abi.SceneDesc.from_buffer_copy(packed.desc)
    bad.n_materials = 0
    assert L.spt_bvh_build(C.byref(bad), 1, C.byref(h)) == abi.SPT_ERR_INVALID_ARGUMENT
    assert L.spt_bvh_build(None, 1, C.byref(h)) == abi.SPT_ERR_INVALID_ARGUMENT
    assert L.spt_bvh_build(packed.ref(), 1, None) == abi.SPT_ERR_INVALID_ARGUMENT
    assert L.spt_bvh_build(packed.ref(), 1, C.byref(h)) == abi.SPT_OK
    L.spt_bvh_free(h)


def test_null_handles_are_rejected():
    L = native.lib()
    assert L.spt_destroy(None) == abi.SPT_ERR_INVALID_ARGUMENT
    assert L.spt_scene_destroy(None) == abi.SPT_ERR_INVALID_ARGUMENT
    assert L.spt_intersect(None, None, None, 0, None, None, None) == abi.SPT_ERR_INVALID_ARGUMENT
    assert L.spt_last_error(None) is not None


def test_ppm_writer_format(tmp_path):
    """ImageBuffer::saveToFile (core/image_buffer.cpp:32-47) with convertTosRGB (:22-30)."""
    from swpathtracer_b200 import write_ppm
    rgb = np.array([[[0.0, 0.5, 1.0], [2.0, -1.0, 0.25]]], np.float32)
    p = tmp_path / "a.ppm"
    write_ppm(str(p), rgb, srgb=True)
    txt = p.read_text().split()
    assert txt[:4] == ["P3", "2", "1", "255"]
    vals = [int(v) for v in txt[4:]]
    exp = [int(min(max(float(np.float32(np.power(np.float64(min(max(c, 0.0), 1.0)), np.float64(np.float32(1 / 2.2))))),
                       0.0), 1.0) * np.float32(255.0) + np.float32(0.5)) for c in rgb.reshape(-1)]
    assert vals == exp
    write_ppm(str(p), rgb, srgb=False)
    vals = [int(v) for v in p.read_text().split()[4:]]
    assert vals == [0, 128, 255, 255, 0, 64]


def test_handles_are_freed_once_and_before_their_context():
    """Scenes and guides release their handles before the context, whichever is closed first."""
    from swpathtracer_b200 import api
    calls = []

    class FakeLib:
        def spt_destroy(self, h):
            calls.append(("ctx", h))

    d = object.__new__(api.Device)
    d.lib, d.h, d.device, d._owned = FakeLib(), 1, 0, []
    a = d.adopt(10, lambda h: calls.append(("scene", h)))
    b = d.adopt(20, lambda h: calls.append(("guide", h)))
    a.release()                      # the scene closed by its owner first
    d.close()                        # then the context: the guide goes before it
    b.release()                      # a late close of the guide is a no-op
    d.close()
    assert calls == [("scene", 10), ("guide", 20), ("ctx", 1)]


def _corrupt(packed, **arrays):
    """A copy of packed's description with some arrays replaced (kept alive on the returned object)."""
    d = abi.SceneDesc.from_buffer_copy(packed.desc)

    class Keep:
        pass
    k = Keep()
    k.desc = d
    for name, a in arrays.items():
        setattr(k, name, a)
        if name == "mats":
            d.prim_material = abi.ptr(a, C.c_uint32)
        elif name == "types":
            d.prim_type = abi.ptr(a, C.c_uint8)
        elif name == "layered_ids":
            d.layered_bsdf_ids = abi.ptr(a, C.c_uint32)
        elif name == "layered_offsets":
            d.layered_offsets = abi.ptr(a, C.c_uint32)
    return k


def test_corrupt_scene_tables_are_rejected():
    """Tables that point outside themselves are caught by the scene validation before any build or
    upload (spt_bvh_build runs it on the host, spt_scene_create and spt_bvh_build_device the same)."""
    L = native.lib()
    packed = scenes.box_scene(1).build()
    h = C.c_void_p()
    bad_mat = packed.mats.copy()
    bad_mat[3] = packed.n_materials                       # material index out of range
    bad_type = packed.types.copy()
    bad_type[0] = 7                                       # unknown primitive type
    bad_ids = packed.layered_ids.copy()
    bad_ids[0] = 1000                                     # layered stack names a missing BSDF
    bad_offs = packed.layered_offsets.copy()
    bad_offs[1] = bad_offs[0]                             # a layered stack with no layer
    for k in (_corrupt(packed, mats=bad_mat), _corrupt(packed, types=bad_type),
              _corrupt(packed, layered_ids=bad_ids), _corrupt(packed, layered_offsets=bad_offs)):
        assert L.spt_bvh_build(C.byref(k.desc), 1, C.byref(h)) == abi.SPT_ERR_INVALID_ARGUMENT
    orig = packed.bsdfs[0].type
    packed.bsdfs[0].type = 99                             # unknown BSDF type
    try:
        assert L.spt_bvh_build(packed.ref(), 1, C.byref(h)) == abi.SPT_ERR_INVALID_ARGUMENT
    finally:
        packed.bsdfs[0].type = orig
    assert L.spt_bvh_build(packed.ref(), 1, C.byref(h)) == abi.SPT_OK
    L.spt_bvh_free(h)


def test_ray_arrays_of_the_wrong_shape_are_rejected():
    from swpathtracer_b200.api import ray_array
    r = scenes.incoherent_rays(10, seed=1)
    assert ray_array(r, (8,)).shape == (10, 8)
    assert ray_array(r[:, :6], (8, 6)).shape == (10, 6)
    for bad, widths in ((r[:, :6], (8,)), (r[:, :7], (8, 6)), (r[:, 0], (8, 6))):
        with pytest.raises(ValueError):
            ray_array(bad, widths)
