"""ctypes mirrors of the C-ABI structs and constants declared in include/spt.h.

Field order and types follow include/spt.h exactly; the header documents which
reference interface each one replaces.
"""
import ctypes as C

SPT_ABI_VERSION = 2
GUIDE_TRAIN_TCGEN05, GUIDE_TRAIN_MMA_SYNC = 0, 1
SPT_MISS = 0xFFFFFFFF

(SPT_OK, SPT_ERR_INVALID_ARGUMENT, SPT_ERR_CUDA, SPT_ERR_OUT_OF_MEMORY, SPT_ERR_OVERFLOW,
 SPT_ERR_TIMEOUT, SPT_ERR_UNSUPPORTED, SPT_ERR_INTERNAL) = range(8)
STATUS_NAMES = {0: "SPT_OK", 1: "SPT_ERR_INVALID_ARGUMENT", 2: "SPT_ERR_CUDA", 3: "SPT_ERR_OUT_OF_MEMORY",
                4: "SPT_ERR_OVERFLOW", 5: "SPT_ERR_TIMEOUT", 6: "SPT_ERR_UNSUPPORTED", 7: "SPT_ERR_INTERNAL"}

PRIM_TRIANGLE, PRIM_SMOOTH_TRIANGLE, PRIM_SPHERE = 0, 1, 2
BSDF_LAMBERTIAN, BSDF_SMOOTH_CONDUCTOR, BSDF_SMOOTH_DIELECTRIC, BSDF_COOK_TORRANCE = 0, 1, 2, 3
SAMPLER_UNIFORM, SAMPLER_IMPORTANCE = 0, 1
ACCEL_NONE, ACCEL_BVH_SAH, ACCEL_SBVH_SAH = 0, 1, 2
CAMERA_PINHOLE, CAMERA_ORTHOGRAPHIC = 0, 1
PIXEL_UNIFORM, PIXEL_REGULAR, PIXEL_JITTERED = 0, 1, 2
RAYCAST_NORMAL, RAYCAST_DEPTH, RAYCAST_COUNT = 0, 1, 2
TERMINATE_MAX_DEPTH, TERMINATE_RUSSIAN_ROULETTE = 0, 1

F3 = C.c_float * 3


class Bsdf(C.Structure):
    _fields_ = [("type", C.c_int32), ("sampler", C.c_int32), ("rgb", F3), ("scalar", C.c_float)]


class Material(C.Structure):
    _fields_ = [("layered_bsdf", C.c_uint32), ("emission", F3)]


class SceneDesc(C.Structure):
    _fields_ = [
        ("n_prims", C.c_uint32),
        ("prim_type", C.POINTER(C.c_uint8)),
        ("prim_data", C.POINTER(C.c_float)),
        ("prim_normals", C.POINTER(C.c_float)),
        ("prim_material", C.POINTER(C.c_uint32)),
        ("n_bsdfs", C.c_uint32),
        ("bsdfs", C.POINTER(Bsdf)),
        ("n_layered", C.c_uint32),
        ("layered_offsets", C.POINTER(C.c_uint32)),
        ("layered_bsdf_ids", C.POINTER(C.c_uint32)),
        ("n_materials", C.c_uint32),
        ("materials", C.POINTER(Material)),
        ("background", F3),
        ("accel", C.c_int32),
    ]


class Camera(C.Structure):
    _fields_ = [
        ("type", C.c_int32), ("position", F3), ("look_at", F3), ("up", F3), ("fov_deg", C.c_float),
        ("min_x", C.c_float), ("max_x", C.c_float), ("min_y", C.c_float), ("max_y", C.c_float),
        ("width", C.c_uint32), ("height", C.c_uint32),
        ("vp_top", C.c_uint32), ("vp_left", C.c_uint32), ("vp_width", C.c_uint32), ("vp_height", C.c_uint32),
    ]


class PtParams(C.Structure):
    _fields_ = [
        ("pixel_sampler", C.c_int32), ("spp", C.c_uint32), ("termination", C.c_int32),
        ("path_length", C.c_int32), ("max_depth", C.c_int32), ("spp_offset", C.c_uint32),
        ("seed", C.c_uint64),
    ]


class Hit(C.Structure):
    _fields_ = [("t", C.c_float), ("prim_id", C.c_uint32), ("u", C.c_float), ("v", C.c_float)]


class RenderStats(C.Structure):
    _fields_ = [
        ("int_tests", C.c_uint64), ("int_hits", C.c_uint64),
        ("min_tests_pp", C.c_uint64), ("max_tests_pp", C.c_uint64),
        ("min_hits_pp", C.c_uint64), ("max_hits_pp", C.c_uint64),
        ("paths", C.c_uint64), ("segments", C.c_uint64), ("gpu_ms", C.c_double),
    ]


class Bvh2Node(C.Structure):
    _fields_ = [("min", F3), ("right", C.c_uint32), ("max", F3), ("count", C.c_uint32)]


class BvhStats(C.Structure):
    _fields_ = [
        ("num_nodes", C.c_uint64), ("num_inner_nodes", C.c_uint64), ("num_leaf_nodes", C.c_uint64),
        ("tree_height", C.c_uint64), ("min_prims_leaf", C.c_uint64), ("max_prims_leaf", C.c_uint64),
        ("num_references", C.c_uint64), ("num_unreferenced", C.c_uint64), ("build_ms", C.c_double),
    ]


class Tune(C.Structure):
    _fields_ = [("capacity", C.c_uint32), ("extend_block", C.c_uint32), ("shade_block", C.c_uint32),
                ("traversal", C.c_int32), ("check_every", C.c_uint32), ("sort_shading", C.c_uint32),
                ("stack", C.c_uint32), ("stack_limit", C.c_uint32), ("max_iterations", C.c_uint32),
                ("host_loop", C.c_uint32)]


class BatchJob(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("camera", Camera), ("params", PtParams)]


class GuideConfig(C.Structure):
    _fields_ = [("box_min", F3), ("box_max", F3), ("lr", C.c_float), ("batch", C.c_uint32),
                ("max_steps", C.c_uint32), ("mix", C.c_float), ("seed", C.c_uint64),
                ("cache_res", C.c_uint32), ("train_path", C.c_uint32), ("guided_depth", C.c_uint32),
                ("reserved", C.c_uint32)]


GUIDE_LEVELS, GUIDE_FEATS, GUIDE_T = 16, 2, 1 << 19
GUIDE_GRID_PARAMS = GUIDE_LEVELS * GUIDE_T * GUIDE_FEATS
GUIDE_MLP_SHAPES = [(64, 48), (64, 64), (64, 64), (64, 64), (48, 64)]
GUIDE_MLP_PARAMS = sum(a * b for a, b in GUIDE_MLP_SHAPES)


# numpy dtypes with the same layout, for bulk arrays crossing the ABI.
def _np_dtypes():
    import numpy as np
    hit = np.dtype([("t", "<f4"), ("prim_id", "<u4"), ("u", "<f4"), ("v", "<f4")])
    node = np.dtype([("min", "<f4", 3), ("right", "<u4"), ("max", "<f4", 3), ("count", "<u4")])
    rec = np.dtype([("pos", "<f4", 3), ("weight", "<f4"), ("normal", "<f4", 3), ("pad0", "<f4"),
                    ("wo", "<f4", 3), ("pad1", "<f4"), ("wi", "<f4", 3), ("pad2", "<f4")])
    return hit, node, rec


HIT_DTYPE, BVH2_NODE_DTYPE, GUIDE_RECORD_DTYPE = _np_dtypes()


def ptr(arr, ctype):
    """ctypes pointer to a contiguous numpy array's data (None for None)."""
    if arr is None:
        return None
    assert arr.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return arr.ctypes.data_as(C.POINTER(ctype))
