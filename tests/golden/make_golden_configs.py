"""Golden fixtures at the benchmark configurations themselves, from the REFERENCE's own code.

Run here, where the reference sources exist:
    make -C oracle ref && python tests/golden/make_golden_configs.py [c1] [c0]
It drives oracle/_ref/libswref.so (the reference renderer's unmodified sources) and writes:

  c1_mesh.npz / configs.json["c1"] -- the 1,310,720-triangle displaced icosphere
    (scenes.displaced_mesh_scene(8)):
      * SHA-256 and StatsSBVH of the tree SBVH::build makes (acceleration/sbvh.cpp:12-37);
      * for a seeded sample of 2^16 of the 2^24 headline rays (scenes.incoherent_rays(2^24, seed=1)):
        the ray index, primitive id, t bits and the test / pass counts of SBVH::intersect
        (acceleration/sbvh.cpp:478-510);
      * the three 1920x1080 ray-cast images (integrators/raycaster.h:62-99): the SHA-256 of each
        whole image and every 8th row of each, plus the image statistics.
  c0_box_pt.npz / configs.json["c0"] -- the 20,492-triangle box scene (scenes.box_scene(5)) at
    256x256, jittered sampler, max length 5: the mean of two independent 4,096-spp renders of
    PathTracer::render (integrators/pathtracer.cpp:59-147, reseeded mt19937 engines), and the relMSE
    between the two renders (the noise floor of a comparison).
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from swpathtracer_b200 import abi, scenes  # noqa: E402

C1_SAMPLE = 1 << 16
C1_ROW_STEP = 8
C0_SPP = 4096


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def c1_sample_indices(n_total=1 << 24, n=C1_SAMPLE, seed=2026):
    g = np.random.Generator(np.random.Philox(seed))
    return np.sort(g.choice(n_total, size=n, replace=False)).astype(np.uint32)


def make_c1(H, threads):
    packed = scenes.displaced_mesh_scene(8).build()
    t0 = time.perf_counter()
    rs = H.scene(packed, n_threads=threads)
    build_s = time.perf_counter() - t0
    nodes, refs = rs.tree()
    st = rs.tree_stats()
    idx = c1_sample_indices()
    rays = scenes.incoherent_rays(1 << 24, seed=1)[idx]
    r = rs.intersect(rays, n_threads=threads, want_normals=False)
    cam = scenes.displaced_mesh_camera(1920, 1080)
    arrays = dict(index=idx, prim=r["hits"]["prim_id"], t=r["hits"]["t"], tests=r["tests"], nhits=r["nhits"])
    meta = {"n_prims": int(packed.n_prims), "build_s_reference": round(build_s, 2),
            "tree_sha256": sha(nodes, refs),
            "tree_stats": {f: getattr(st, f) for f, _ in abi.BvhStats._fields_ if f != "build_ms"},
            "sample_seed": 2026, "sample_size": C1_SAMPLE, "row_step": C1_ROW_STEP, "images": {}}
    for name, mode in (("normal", abi.RAYCAST_NORMAL), ("depth", abi.RAYCAST_DEPTH), ("count", abi.RAYCAST_COUNT)):
        img, ist, secs = rs.raycast(cam, mode, n_threads=threads)
        arrays["rows_" + name] = img[::C1_ROW_STEP].copy()
        meta["images"][name] = {"sha256": sha(img), "seconds": round(secs, 2),
                                "stats": {f: getattr(ist, f) for f, _ in abi.RenderStats._fields_
                                          if f not in ("gpu_ms", "segments", "paths")}}
        print("c1", name, secs, flush=True)
    rs.close()
    np.savez_compressed(os.path.join(HERE, "c1_mesh.npz"), **arrays)
    return meta


def make_c0(H, threads):
    packed = scenes.box_scene(5).build()
    cam = scenes.box_camera(256, 256)
    rs = H.scene(packed, n_threads=threads)
    imgs, secs = [], 0.0
    for seed in (11, 1011):
        p = scenes.pt_params(spp=C0_SPP, sampler="jittered", termination="max-length", path_length=5, seed=seed)
        img, s = rs.pathtrace(cam, p, n_threads=threads)
        imgs.append(img)
        secs += s
        print("c0 render", seed, s, flush=True)
    rs.close()
    a, b = imgs
    floor = float(np.mean((a - b) ** 2 / (a ** 2 + 1e-2)))
    mean = (0.5 * (a.astype(np.float64) + b)).astype(np.float32)
    np.savez_compressed(os.path.join(HERE, "c0_box_pt.npz"), image=mean)
    return {"n_prims": int(packed.n_prims), "width": 256, "height": 256, "spp_per_render": C0_SPP, "renders": 2,
            "termination": "max-length", "path_length": 5, "sampler": "jittered",
            "relmse_between_renders": floor, "mean": float(mean.mean()), "seconds": round(secs, 1)}


def main():
    from oracle.bindings import RefHarness
    H = RefHarness()
    threads = os.cpu_count() or 1
    which = set(sys.argv[1:]) or {"c1", "c0"}
    path = os.path.join(HERE, "configs.json")
    meta = json.load(open(path)) if os.path.exists(path) else {}
    if "c1" in which:
        meta["c1"] = make_c1(H, threads)
    if "c0" in which:
        meta["c0"] = make_c0(H, threads)
    with open(path, "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
