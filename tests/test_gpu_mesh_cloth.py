"""Cloth from a triangle mesh (ClothPatch::Init(mesh), Physics/ClothPatch.cpp:42-133)
through the C ABI: the library's topology and rest data equal the reference
build's, and its steps equal the oracle's in check mode."""
import ctypes as C

import numpy as np
import pytest

from solidcloth_b200 import scenes

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _reference(v, idx, uv, col, prm):
    from oracle.bridge import RefCloth, available
    if not available("ref"):
        pytest.skip("reference build absent")
    RefCloth.set_threads(1)
    r = RefCloth()
    pa = prm.as_array()
    r._fn("set_params")(r.h, pa.ctypes.data_as(C.POINTER(C.c_float)), pa.size)
    r.init_mesh(v, idx, uv, col, (0, 0, 0), True)
    return r


@pytest.mark.parametrize("fem", [True, False])
def test_mesh_cloth_topology_and_check_mode(fem):
    from solidcloth_b200 import api
    from oracle.bridge import PortCloth
    v, idx, uv, col, prm = scenes.mesh_cloth()
    prm.fem = fem
    w = api.CollisionWorld()
    p = api.ClothPatch(w)
    p.model.set_params(prm)
    p.set_num_steps(prm.substeps)
    p.init_mesh(v, idx, uv, col, (0, 0, 0), True)
    r = _reference(v, idx, uv, col, prm)
    # particles (merge, pins), triangles with rest data, bends, links, edges
    pos, prev, vel, inv = r.state()
    assert np.array_equal(_bits(p.model.positions()), _bits(pos))
    assert np.array_equal(p.model.inv_masses(), inv)
    ti, tr = r.tris()
    assert np.array_equal(p.model.tris().astype(np.uint32), ti)
    assert np.array_equal(_bits(p.model.tri_rest()), _bits(tr))
    assert np.array_equal(p.model.bends(), r.bends())
    li, lr = r.links()
    gi, gr = p.model.links()
    assert np.array_equal(gi, li) and np.array_equal(_bits(gr), _bits(lr))
    assert np.array_equal(p.model.edges(), r.edges())
    # check mode: the oracle with this topology, in the GPU's constraint orders
    PortCloth.set_portable_math(True)
    o = PortCloth()
    pa = prm.as_array()
    o._fn("set_params")(o.h, pa.ctypes.data_as(C.POINTER(C.c_float)), pa.size)
    o.load_topology(pos, inv, ti, tr, r.bends(), li, lr)
    o.set_tri_order(p.model.constraint_order(0)[0])
    o.set_bend_order(p.model.constraint_order(1)[0])
    if not fem:
        o.set_link_order(p.model.constraint_order(2)[0])
    dt = 1.0 / 60
    for f in range(6):
        p.step(dt)
        o.step(dt)
        g = p.model.positions()
        assert np.array_equal(_bits(g), _bits(o.positions())), (f, float(np.abs(g - o.positions()).max()))
    assert p.status() == 0
    assert p.particle_map().max() == pos.shape[0] - 1
    p.free()
    w.free()


def test_obj_cloth_equals_array_cloth(tmp_path):
    """A cloth read from an OBJ file (v, vt, quads fanned into triangles) equals
    the same triangle soup given as arrays: same particles, triangles, rest data."""
    from solidcloth_b200 import api
    n, side = 6, 0.3
    xs = np.linspace(-side / 2, side / 2, n).astype(np.float32)
    lines = []
    for j in range(n):
        for i in range(n):
            lines.append(f"v {xs[i]:.6f} 0.2 {xs[j]:.6f}")
            lines.append(f"vt {xs[i]:.6f} {xs[j]:.6f}")
    for j in range(n - 1):
        for i in range(n - 1):
            a, b, c, d = j * n + i + 1, j * n + i + 2, (j + 1) * n + i + 2, (j + 1) * n + i + 1
            lines.append(f"f {a}/{a} {b}/{b} {c}/{c} {d}/{d}")
    path = tmp_path / "sheet.obj"
    path.write_text("\n".join(lines) + "\n")
    w = api.CollisionWorld()
    p1 = api.ClothPatch(w)
    p1.model.set_params(scenes.Params(flags=0))
    assert p1.init_obj(path)
    # the same soup by hand: quads fanned (a b c), (a c d), one vertex per corner
    verts = np.array([[float(t) for t in l.split()[1:]] for l in lines if l.startswith("v ")], np.float32)
    uvs = np.array([[float(t) for t in l.split()[1:]] for l in lines if l.startswith("vt ")], np.float32)
    soup_v, soup_uv = [], []
    for l in lines:
        if not l.startswith("f "):
            continue
        q = [int(t.split("/")[0]) - 1 for t in l.split()[1:]]
        for tri in ((q[0], q[1], q[2]), (q[0], q[2], q[3])):
            for k in tri:
                soup_v.append(verts[k])
                soup_uv.append(uvs[k])
    p2 = api.ClothPatch(w)
    p2.model.set_params(scenes.Params(flags=0))
    p2.init_mesh(np.array(soup_v), np.arange(len(soup_v)), np.array(soup_uv))
    assert np.array_equal(p1.model.positions(), p2.model.positions())
    assert np.array_equal(p1.model.tris(), p2.model.tris())
    assert np.array_equal(_bits(p1.model.tri_rest()), _bits(p2.model.tri_rest()))
    assert p1.model.positions().shape[0] == n * n
    p1.free()
    p2.free()
    w.free()
