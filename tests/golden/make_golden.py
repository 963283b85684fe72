"""Generates the golden fixtures in tests/golden from the REFERENCE's own code.

Run here, where the reference sources exist:  make -C oracle ref && python tests/golden/make_golden.py
It drives oracle/_ref/libswref.so (the reference renderer's unmodified sources, compiled by
oracle/Makefile) on the project's seeded synthetic scenes and stores its outputs:
  * tree statistics and a SHA-256 of the exported SAH tree (node boxes, child links, leaf refs);
  * closest hits (primitive id, t bits), normals and the per-ray test / pass counts of
    SBVH::intersect for a seeded ray batch (the rays themselves are stored too);
  * the three ray-cast images for a small camera;
  * a converged path-traced image (many samples, reseeded mt19937 engines).
The Philox-4x32-10 known-answer vectors are the published ones (Salmon et al., SC'11, Random123).
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from swpathtracer_b200 import abi, scenes  # noqa: E402

PHILOX_KAT = [
    {"ctr": [0, 0, 0, 0], "key": [0, 0], "out": [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]},
    {"ctr": [0xFFFFFFFF] * 4, "key": [0xFFFFFFFF] * 2, "out": [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]},
    {"ctr": [0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], "key": [0xA4093822, 0x299F31D0],
     "out": [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]},
]

# name -> (scene builder, ray half extent, camera)
SCENES = {
    "box_icosphere": (lambda: scenes.box_scene(3), 1.0, lambda: scenes.box_camera(64, 48)),
    "displaced_mesh": (lambda: scenes.displaced_mesh_scene(5), 1.5, lambda: scenes.displaced_mesh_camera(80, 45)),
    "furnace_spheres": (lambda: scenes.furnace_scene("coating"), 11.0, lambda: scenes.furnace_camera(48, 48)),
    "smooth_mesh": (lambda: scenes.smooth_mesh_scene(3), 1.0, lambda: scenes.box_camera(64, 48)),
}


def scene_hash(packed):
    h = hashlib.sha256()
    h.update(packed.types.tobytes())
    h.update(packed.data.tobytes())
    if packed.normals is not None:
        h.update(packed.normals.tobytes())
    h.update(packed.mats.tobytes())
    return h.hexdigest()


def tree_hash(nodes, refs):
    h = hashlib.sha256()
    h.update(nodes.tobytes())
    h.update(refs.tobytes())
    return h.hexdigest()


def main():
    from oracle.bindings import RefHarness
    H = RefHarness()
    meta = {"philox_kat": PHILOX_KAT, "scenes": {}}
    for name, (mk, ext, mkcam) in SCENES.items():
        packed = mk().build()
        rs = H.scene(packed, n_threads=8)
        nodes, refs = rs.tree()
        st = rs.tree_stats()
        rays = scenes.incoherent_rays(2048, seed=11, half_extent=ext)
        r = rs.intersect(rays, n_threads=8)
        cam = mkcam()
        normal, nst, _ = rs.raycast(cam, abi.RAYCAST_NORMAL, n_threads=8)
        depth, _, _ = rs.raycast(cam, abi.RAYCAST_DEPTH, n_threads=8)
        count, _, _ = rs.raycast(cam, abi.RAYCAST_COUNT, n_threads=8)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), rays=rays, prim=r["hits"]["prim_id"],
                            t=r["hits"]["t"], normals=r["normals"], tests=r["tests"], nhits=r["nhits"],
                            img_normal=normal, img_depth=depth, img_count=count.astype(np.int32))
        meta["scenes"][name] = {
            "scene_sha256": scene_hash(packed), "n_prims": int(packed.n_prims),
            "tree_sha256": tree_hash(nodes, refs),
            "tree_stats": {f: getattr(st, f) for f, _ in abi.BvhStats._fields_ if f != "build_ms"},
            "raycast_stats": {f: getattr(nst, f) for f, _ in abi.RenderStats._fields_
                              if f not in ("gpu_ms", "segments", "paths")},
            "camera": {"width": cam.width, "height": cam.height},
        }
        print(name, packed.n_prims, st.num_nodes, flush=True)
    # converged path-traced images from the reference (statistical pins for the path tracer)
    pt = {}
    for name, mk, cam, params in [
        ("box_icosphere_pt", lambda: scenes.box_scene(3), scenes.box_camera(48, 48),
         scenes.pt_params(spp=4096, sampler="jittered", termination="max-length", path_length=5, seed=5)),
        ("layered_box_pt", lambda: scenes.layered_box_scene(3), scenes.layered_box_camera(48, 36),
         scenes.pt_params(spp=4096, sampler="jittered", termination="russian-roulette", path_length=3, seed=6)),
    ]:
        packed = mk().build()
        rs = H.scene(packed, n_threads=8)
        img, secs = rs.pathtrace(cam, params, n_threads=8)
        # a second, independent render measures the noise floor of the comparison
        params.seed += 1000
        img2, _ = rs.pathtrace(cam, params, n_threads=8)
        params.seed -= 1000
        floor = float(np.mean((img2 - img) ** 2 / (img ** 2 + 1e-2)))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), image=img)
        pt[name] = {"scene_sha256": scene_hash(packed), "spp": params.spp, "seconds": round(secs, 2),
                    "termination": params.termination, "path_length": params.path_length,
                    "width": cam.width, "height": cam.height, "relmse_two_reference_renders": floor,
                    "mean": float(img.mean())}
        print(name, secs, flush=True)
    meta["pathtrace"] = pt
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
