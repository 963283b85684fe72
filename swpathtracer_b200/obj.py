"""Wavefront OBJ meshes for the scene front end (the reference's Scene::loadMesh, core/scene.cpp:32-68).

The reference reads meshes through Assimp (aiProcess_FindDegenerates | aiProcess_Triangulate,
core/scene.cpp:34-35; Assimp is a system package there, its version not pinned by CMakeLists.txt:30)
and turns every three consecutive entries of a sub-mesh's vertex array into a SmoothTriangle with the
normals at the same entries (core/scene.cpp:50-63).  Assimp's OBJ importer gives every face corner its
own vertex, so for triangle faces those triples are the faces.  Assimp is not available here; this
reader restates that model:

  * one sub-mesh per (object or group name, usemtl) run, in order of first appearance; the name is the
    current `o` / `g` name ("defaultobject" before any);
  * polygons are split into fans (0, i, i+1), as Assimp's triangulation of a convex polygon;
  * corners take their `vn` normal.  The reference reads mNormals for every vertex without a check
    (core/scene.cpp:59-62), and Assimp leaves mNormals unset for a file without normals, so such a
    face has no defined result there: it is rejected here with ValueError;
  * degenerate faces are kept.  aiProcess_FindDegenerates, in Assimp's default configuration
    (AI_CONFIG_PP_FD_REMOVE off), only shortens the index list of a face whose corners repeat a
    position (turning it into a line or a point); it leaves the vertex array alone, and the
    reference reads the vertex array, not the faces.  A face with repeated or collinear corners
    therefore still becomes a triangle of zero area there, which the Moller-Trumbore test never hits
    (|det| < 1e-6, primitives/triangle.cpp:20-21); the same happens here;
  * indices may be negative (relative to the end of the list so far), `v/vt/vn`, `v//vn`; a corner
    without a normal index (`v/vt`, `v`) is a face without normals.
Parity with Assimp itself is unpinned: it is not present to compare with.
"""
import numpy as np


class SubMesh:
    def __init__(self, name):
        self.name = name
        self.tris = []     # [[v0, v1, v2]] positions
        self.norms = []    # [[n0, n1, n2]]


def _index(tok, n):
    i = int(tok)
    return i - 1 if i > 0 else n + i


def read_obj(path):
    """The sub-meshes of an OBJ file, in file order."""
    verts, normals = [], []
    meshes, current = {}, None
    obj_name, mtl = "defaultobject", None
    order = []
    with open(path) as f:
        for raw in f:
            line = raw.split("#", 1)[0].strip()
            if not line:
                continue
            parts = line.split()
            tag = parts[0]
            if tag == "v":
                verts.append([float(x) for x in parts[1:4]])
            elif tag == "vn":
                normals.append([float(x) for x in parts[1:4]])
            elif tag in ("o", "g"):
                obj_name = " ".join(parts[1:]) if len(parts) > 1 else "defaultobject"
                current = None
            elif tag == "usemtl":
                mtl = " ".join(parts[1:])
                current = None
            elif tag == "f":
                if current is None:
                    key = (obj_name, mtl)
                    if key not in meshes:
                        meshes[key] = SubMesh(obj_name)
                        order.append(key)
                    current = meshes[key]
                corners = []
                for c in parts[1:]:
                    fields = c.split("/")
                    vi = _index(fields[0], len(verts))
                    ni = _index(fields[2], len(normals)) if len(fields) > 2 and fields[2] else None
                    corners.append((vi, ni))
                if any(nidx is None for _, nidx in corners):
                    raise ValueError("%s: face %r has no vertex normals; the reference reads a normal for "
                                     "every vertex (core/scene.cpp:59-62)" % (path, line))
                for k in range(1, len(corners) - 1):
                    tri = [corners[0], corners[k], corners[k + 1]]
                    current.tris.append([verts[v] for v, _ in tri])
                    current.norms.append([normals[nidx] for _, nidx in tri])
    return [meshes[k] for k in order]


def add_mesh(builder, path, material, render_all_submeshes=True, submeshes=None):
    """Adds an OBJ file's triangles to a SceneBuilder as smooth triangles (Scene::loadMesh).
    submeshes: {sub-mesh name: material id}.  Returns the number of triangles added."""
    submeshes = submeshes or {}
    added = 0
    for m in read_obj(path):
        if m.name not in submeshes and not render_all_submeshes:
            continue
        if not m.tris:
            continue
        mat = submeshes.get(m.name, material)
        builder.triangles(np.array(m.tris, np.float32), mat, normals=np.array(m.norms, np.float32))
        added += len(m.tris)
    return added
