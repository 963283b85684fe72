"""Wavefront OBJ meshes for the scene front end (the reference's Scene::loadMesh, core/scene.cpp:32-68).

The reference reads meshes through Assimp (aiProcess_Triangulate | aiProcess_FindDegenerates) and adds
every triangle of every sub-mesh as a SmoothTriangle with per-corner positions and normals; a sub-mesh
named in the script's sub_meshes list gets that material, the others get the mesh's material, or are
skipped when render_submeshes is not "all".  Assimp is not available here; this reader follows the
same model:

  * one sub-mesh per (object or group name, usemtl) run, in order of first appearance; the name is the
    current `o` / `g` name ("defaultobject" before any);
  * polygons are split into fans (0, i, i+1);
  * corners take their `vn` normal; a face without normals gets its geometric normal at every corner;
  * indices may be negative (relative to the end of the list so far), `v/vt/vn`, `v//vn`, `v/vt`, `v`.
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
                for k in range(1, len(corners) - 1):
                    tri = [corners[0], corners[k], corners[k + 1]]
                    p = [verts[v] for v, _ in tri]
                    if all(nidx is not None for _, nidx in tri):
                        nrm = [normals[nidx] for _, nidx in tri]
                    else:
                        a, b, c3 = (np.array(x, np.float64) for x in p)
                        g = np.cross(b - a, c3 - a)
                        ln = np.linalg.norm(g)
                        g = g / ln if ln > 0 else np.array([0.0, 0.0, 1.0])
                        nrm = [list(g)] * 3
                    current.tris.append(p)
                    current.norms.append(nrm)
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
