"""The Lua-subset interpreter (swpathtracer_b200/lua.py), the scene front end and the OBJ reader, on CPU.

The reference's own scene scripts (samples/*.lua with lua_core/*.lua) run where the reference sources
are present; elsewhere those cases skip and tests/lua/scene_dsl.lua stands in for lua_core."""
import os

import numpy as np
import pytest

from swpathtracer_b200 import abi, frontend, lua, obj

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("SPT_REFERENCE_DIR", "/root/reference")


def run(src, **globals_):
    it = lua.Interpreter()
    for k, v in globals_.items():
        it.G[k] = v
    it.run_string(src)
    return it


def test_arithmetic_follows_lua_5_3():
    it = run("a = 7 // 2; b = 7 / 2; c = -7 % 3; d = 7.5 // 2; e = 2^10; f = 3 % -2; g = 1e2; h = 0x10;"
             "i = 5 // 0.0; j = -7 // 2; k = 10 - 2 * 3; l = 2^3^2; m = -2^2")
    G = it.G
    assert (G["a"], G["b"], G["c"], G["d"], G["e"], G["f"], G["g"], G["h"]) == (3, 3.5, 2, 3.0, 1024.0, -1, 100.0, 16)
    assert isinstance(G["a"], int) and isinstance(G["b"], float) and isinstance(G["d"], float)
    assert G["i"] == float("inf") and G["j"] == -4 and G["k"] == 4 and G["l"] == 512.0 and G["m"] == -4.0


def test_strings_tables_and_functions():
    it = run('''
        local t = {10, 20, 30, n = "x", [5] = 50}
        len = #t
        s = "a" .. 1 .. "-" .. 2.5 .. tostring(nil) .. tostring(true)
        local sum = 0
        for i, v in ipairs(t) do sum = sum + v end
        isum = sum
        local keys = 0
        for k, v in pairs(t) do keys = keys + 1 end
        nkeys = keys
        function counter()
            local c = 0
            return function() c = c + 1; return c end
        end
        local f = counter(); f(); f()
        cval = f()
        local function va(...) return select("#", ...), ... end
        vn, v1, v2 = va(7, 8)
        obj = {v = 1}
        function obj:add(x) self.v = self.v + x; return self end
        obj:add(2):add(3)
        fmt = string.format("%03d|%.2f|%s|%5s", 7, 3.14159, "ok", "r")
        sub = ("hello"):sub(2, -2)
        up = string.upper("abc")
        local tt = {}
        table.insert(tt, "a"); table.insert(tt, 1, "b"); table.insert(tt, "c")
        joined = table.concat(tt, ",")
        removed = table.remove(tt, 1)
    ''')
    G = it.G
    assert G["len"] == 3 and G["s"] == "a1-2.5niltrue" and G["isum"] == 60 and G["nkeys"] == 5
    assert G["cval"] == 3 and (G["vn"], G["v1"], G["v2"]) == (2, 7, 8) and G["obj"]["v"] == 6
    assert G["fmt"] == "007|3.14|ok|    r" and G["sub"] == "ell" and G["up"] == "ABC"
    assert G["joined"] == "b,a,c" and G["removed"] == "b"


def test_control_flow():
    it = run('''
        local n = 0
        for i = 10, 1, -3 do n = n + i end          -- 10 + 7 + 4 + 1
        down = n
        local x = 0
        for i = 0, 1, 0.25 do x = x + 1 end
        steps = x
        local k = 0
        while true do k = k + 1; if k >= 4 then break end end
        wk = k
        local r = 0
        repeat local y = r; r = r + 1 until y >= 2
        rr = r
        if false then z = 1 elseif nil then z = 2 else z = 3 end
        a = nil and 1 or 2
        b = false or "dflt"
        c = not nil
    ''')
    G = it.G
    assert (G["down"], G["steps"], G["wk"], G["rr"], G["z"], G["a"], G["b"], G["c"]) == (22, 5, 4, 3, 3, 2, "dflt", True)


def test_errors_carry_lines_and_exit_is_reported():
    with pytest.raises(lua.LuaError) as e:
        run("local a = 1\nlocal b = nil + a")
    assert "line 2" in str(e.value)
    with pytest.raises(lua.LuaError):
        run("x = = 1")
    with pytest.raises(lua.LuaExit):
        run("print('bye') os.exit()")
    it = lua.Interpreter()
    with pytest.raises(lua.LuaError):
        it.run_string('error("boom")')


def test_require_searches_package_path(tmp_path):
    (tmp_path / "mods").mkdir()
    (tmp_path / "mods" / "m1.lua").write_text('require "m2"\nM1 = M2 + 1\nreturn {name = "m1"}')
    (tmp_path / "mods" / "m2.lua").write_text("M2 = 41\ncount = (count or 0) + 1")
    (tmp_path / "main.lua").write_text('package.path = package.path .. ";./mods/?.lua"\n'
                                       'local m = require "m1"\nrequire "m2"\nNAME = m.name')
    it = lua.run(str(tmp_path / "main.lua"))
    assert it.G["M1"] == 42 and it.G["NAME"] == "m1" and it.G["count"] == 1
    with pytest.raises(lua.LuaError):
        lua.Interpreter().run_string('require "no_such_module"')


def test_front_end_builds_the_test_scene():
    s = frontend.load_lua(os.path.join(HERE, "lua", "small_box.lua"))
    assert s.integrator == "path-tracer" and s.pt_params.spp == 16 and s.pt_params.path_length == 5
    assert s.pt_params.termination == abi.TERMINATE_MAX_DEPTH
    assert s.packed.n_prims == 12 + 4
    assert (s.camera.width, s.camera.height) == (48, 40) and s.camera.fov_deg == 40
    assert s.file_name == "small_box.ppm"
    s = frontend.load_lua(os.path.join(HERE, "lua", "small_box.lua"), globals={"INTEGRATOR": "depth"})
    assert s.integrator == "ray-caster" and s.raycast_mode == abi.RAYCAST_DEPTH and s.prescribed == (-1.0, -1.0)


def test_obj_reader(tmp_path):
    p = tmp_path / "m.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvn 0 0 1\nvn 0 1 0\n"
                 "o first\nf 1//1 2//1 3//1 4//1\n"          # a quad with normals -> 2 triangles
                 "g second\nusemtl red\nf -4//-1 -3//-1 -2//-2\n"   # relative indices
                 "usemtl blue\nf 1/1/1 3/1/2 4/1/1\n")
    meshes = obj.read_obj(str(p))
    assert [m.name for m in meshes] == ["first", "second", "second"]
    assert [len(m.tris) for m in meshes] == [2, 1, 1]
    np.testing.assert_allclose(meshes[0].tris[1], [[0, 0, 0], [1, 1, 0], [0, 1, 0]])
    np.testing.assert_allclose(meshes[1].norms[0], [[0, 1, 0], [0, 1, 0], [0, 0, 1]])
    from swpathtracer_b200 import scenes
    sb = scenes.SceneBuilder()
    m0 = sb.material(sb.layered_bsdf(sb.lambertian()))
    m1 = sb.material(sb.layered_bsdf(sb.lambertian()))
    assert obj.add_mesh(sb, str(p), m0, True, {"second": m1}) == 4
    assert obj.add_mesh(sb, str(p), m0, False, {"second": m1}) == 2
    packed = sb.build()
    assert packed.n_prims == 6


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "lua_core")), reason="reference Lua sources not present")
@pytest.mark.parametrize("name,prims,integrator", [("procedural.lua", 102, "path-tracer"),
                                                    ("furnace_test.lua", 2, "path-tracer"),
                                                    ("materials_test.lua", 10, "path-tracer"),
                                                    ("monkey_in_a_box.lua", 12 + 968, "path-tracer")])
def test_reference_samples_load(name, prims, integrator):
    s = frontend.load_lua(os.path.join(REF, "samples", name))
    assert s.packed.n_prims == prims
    assert s.integrator == integrator
    assert s.camera.width > 0 and s.pt_params.spp > 0


def test_obj_without_normals_is_rejected(tmp_path):
    """The reference reads mNormals for every vertex (core/scene.cpp:59-62); a file without normals
    has no defined result there, so the reader refuses it instead of inventing normals."""
    p = tmp_path / "n.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    with pytest.raises(ValueError):
        obj.read_obj(str(p))
    p.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nvn 0 0 1\nf 1//1 2//1 3\n")   # one corner without
    with pytest.raises(ValueError):
        obj.read_obj(str(p))


def test_obj_degenerate_faces_are_kept_and_never_hit(tmp_path, oracle):
    """aiProcess_FindDegenerates (default configuration) leaves the vertex array the reference reads
    untouched, so faces with a repeated corner or collinear corners still become triangles; their
    zero area makes the Moller-Trumbore test reject every ray (primitives/triangle.cpp:20-21)."""
    from swpathtracer_b200 import scenes
    p = tmp_path / "d.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nv 2 0 0\nvn 0 0 1\n"
                 "f 1//1 2//1 3//1\n"        # a proper triangle
                 "f 1//1 2//1 2//1\n"        # a repeated corner
                 "f 1//1 2//1 4//1\n")       # three collinear corners
    meshes = obj.read_obj(str(p))
    assert [len(m.tris) for m in meshes] == [3]
    sb = scenes.SceneBuilder()
    m = sb.material(sb.layered_bsdf(sb.lambertian()))
    assert obj.add_mesh(sb, str(p), m) == 3
    packed = sb.build()
    rays = np.zeros((3, 8), np.float32)
    rays[:, 0:3] = [[0.2, 0.2, 1.0], [0.5, 0.0, 1.0], [1.5, 0.0, 1.0]]   # onto the proper triangle and
    rays[:, 4:7] = [0.0, 0.0, -1.0]                                      # onto the two degenerate ones
    r = oracle.scene(packed).intersect(rays)
    assert list(r["hits"]["prim_id"][:1]) == [0]
    assert r["hits"]["prim_id"][2] == abi.SPT_MISS      # only the collinear face spans x = 1.5
    assert r["hits"]["prim_id"][1] in (0, abi.SPT_MISS)  # x = 0.5, y = 0 lies on the proper triangle's edge
