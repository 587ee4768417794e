"""ctypes driver for the two CPU oracles (TEST INFRASTRUCTURE ONLY).

  RefCloth  -> oracle/_ref/libscref.so   the reference's own sources + harness
  PortCloth -> oracle/_build/liboracle.so this project's restatement

Both expose the same methods so tests drive them interchangeably. Only tests/,
__graft_entry__.smoke() and bench.py's CPU legs may import this module.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libscref.so"
# the same reference sources built without -fopenmp: single-threaded, as the
# reference's C-ABI library (ClothLib, CMakeLists.txt:42) is
REF_SERIAL_LIB = HERE / "_ref" / "libscref_serial.so"
PORT_LIB = HERE / "_build" / "liboracle.so"

_f = C.POINTER(C.c_float)
_i = C.POINTER(C.c_int)
_u = C.POINTER(C.c_uint)


def _fp(a):
    return None if a is None else a.ctypes.data_as(_f)


def _ip(a):
    return None if a is None else a.ctypes.data_as(_i)


def _up(a):
    return None if a is None else a.ctypes.data_as(_u)


_LIBS = {}


def _load(path: Path, prefix: str):
    key = str(path)
    if key in _LIBS:
        return _LIBS[key]
    if not path.exists():
        raise FileNotFoundError(f"{path} is not built (make -C oracle)")
    lib = C.CDLL(str(path))
    P = prefix
    sig = {
        "create": ([], C.c_void_p), "destroy": ([C.c_void_p], None),
        "add_walls": ([C.c_void_p, _f], None),
        "add_sphere": ([C.c_void_p, C.c_float, C.c_float, C.c_float, C.c_float], None),
        "add_sdf": ([C.c_void_p, C.c_int, C.c_int, C.c_int, _f, _f], None),
        "add_mesh": ([C.c_void_p, C.c_int, _f, C.c_int, _u], None),
        "init_grid": ([C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int, C.c_int], None),
        "set_params": ([C.c_void_p, _f, C.c_int], None),
        "set_ccd": ([C.c_void_p, C.c_int], None),
        "set_solver": ([C.c_void_p, C.c_int], None),
        "num_particles": ([C.c_void_p], C.c_int), "num_tris": ([C.c_void_p], C.c_int),
        "num_bends": ([C.c_void_p], C.c_int), "num_edges": ([C.c_void_p], C.c_int),
        "set_positions": ([C.c_void_p, _f], None),
        "set_state": ([C.c_void_p, _f, _f, _f], None),
        "set_masses": ([C.c_void_p, _f], None),
        "get_state": ([C.c_void_p, _f, _f, _f, _f], None),
        "get_tris": ([C.c_void_p, _u, _f], None),
        "get_bends": ([C.c_void_p, _u], None),
        "get_edges": ([C.c_void_p, _i], None),
        "num_links": ([C.c_void_p], C.c_int),
        "get_links": ([C.c_void_p, _u, _f], None),
        "step": ([C.c_void_p, C.c_float], None),
        "update_mesh": ([C.c_void_p], None),
        "predict_detect": ([C.c_void_p, C.c_float, C.c_int], None),
        "num_contacts": ([C.c_void_p, C.c_int], C.c_int),
        "get_vertex_contacts": ([C.c_void_p, _i, _f], None),
        "get_tri_contacts": ([C.c_void_p, _i, _f], None),
        "get_edge_contacts": ([C.c_void_p, _i, _f], None),
        "get_self_contacts": ([C.c_void_p, C.c_int, _i, _f], None),
        "get_mesh_normals": ([C.c_void_p, C.c_int, _f], None),
        "get_mesh_tri_normals": ([C.c_void_p, C.c_int, _f], None),
        "ccd_narrow_on": ([C.c_void_p, C.c_int, _i, C.c_int, _i], None),
        "swept_boxes": ([C.c_void_p, C.c_int, C.c_float, _f], None),
    }
    if prefix == "ref_":
        sig.update({"set_threads": ([C.c_int], None), "max_threads": ([], C.c_int),
                    "ccd_midphase": ([C.c_void_p], None),
                    "ccd_num_candidates": ([C.c_void_p, C.c_int], C.c_int),
                    "ccd_get_candidates": ([C.c_void_p, C.c_int, _i], None),
                    "solver_iterations": ([C.c_void_p], C.c_int),
                    "init_mesh": ([C.c_void_p, C.c_int, _f, C.c_int, _u, _f, _f, C.c_float, C.c_float, C.c_float, C.c_int], None),
                    "sdf_from_mesh": ([C.c_int, _f, C.c_int, _u, C.c_int, C.c_int, C.c_int, _f, _f], None),
                    "sdf_write": ([C.c_int, C.c_int, C.c_int, _f, _f, C.c_char_p], None),
                    "sdf_read": ([C.c_char_p, _i, _f, _f, C.c_int], C.c_int)})
    else:
        sig.update({"set_tri_order": ([C.c_void_p, _i, C.c_int], None),
                    "set_bend_order": ([C.c_void_p, _i, C.c_int], None),
                    "set_contact_order": ([C.c_void_p, C.c_int], None),
                    "set_static_colours": ([C.c_void_p, _i, C.c_int, C.c_int, _i, C.c_int, C.c_int], None),
                    "set_portable_math": ([C.c_int], None),
                    "portable_acos": ([C.c_float], C.c_float),
                    "self_contact_colours": ([C.c_void_p, C.c_int, _i], None),
                    "ccd_broadphase": ([C.c_void_p, C.c_float, C.c_int, _i, C.c_int], C.c_int),
                    "set_bruteforce_broadphase": ([C.c_void_p, C.c_int], None),
                    "residual": ([C.c_void_p], C.c_float),
                    "set_link_order": ([C.c_void_p, _i, C.c_int], None),
                    "load_topology": ([C.c_void_p, C.c_int, _f, _f, C.c_int, _u, _f, C.c_int, _u, C.c_int, _u, _f], None),
                    })
    for name, (args, res) in sig.items():
        fn = getattr(lib, P + name)
        fn.argtypes = args
        fn.restype = res
    _LIBS[key] = lib
    return lib


class CpuCloth:
    """One cloth patch + collision world in a CPU oracle library."""

    def __init__(self, path: Path, prefix: str):
        self.lib = _load(path, prefix)
        self.p = prefix
        self.h = self._fn("create")()

    def _fn(self, name):
        return getattr(self.lib, self.p + name)

    def close(self):
        if self.h:
            self._fn("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- building ----
    @classmethod
    def from_scene(cls, scene, **kw):
        obj = cls(**kw)
        obj.load_scene(scene)
        return obj

    def load_scene(self, s):
        if s.walls is not None:
            self._fn("add_walls")(self.h, _fp(np.ascontiguousarray(s.walls, np.float32)))
        for (c, r) in s.spheres:
            self._fn("add_sphere")(self.h, float(c[0]), float(c[1]), float(c[2]), float(r))
        for g in s.sdfs:
            self._fn("add_sdf")(self.h, g.cells[0], g.cells[1], g.cells[2],
                                _fp(np.ascontiguousarray(g.box, np.float32)),
                                _fp(np.ascontiguousarray(g.values, np.float32)))
        for m in s.meshes:
            v = np.ascontiguousarray(m.vertices, np.float32)
            idx = np.ascontiguousarray(m.indices, np.uint32)
            self._fn("add_mesh")(self.h, v.shape[0], _fp(v), idx.size // 3, _up(idx))
        pa = s.params.as_array()
        self._fn("set_params")(self.h, _fp(pa), pa.size)
        self._fn("set_solver")(self.h, int(getattr(s.params, "solver", 1)))
        off = s.offset
        self._fn("init_grid")(self.h, s.n, s.n, float(s.inc), float(off[0]), float(off[1]), float(off[2]), 1,
                              int(s.attached))
        self._fn("set_masses")(self.h, _fp(np.ascontiguousarray(s.masses, np.float32)))
        self._fn("set_positions")(self.h, _fp(np.ascontiguousarray(s.positions, np.float32)))
        self._fn("set_ccd")(self.h, int(s.ccd))
        self.scene = s

    # ---- queries ----
    @property
    def n(self):
        return self._fn("num_particles")(self.h)

    def state(self):
        n = self.n
        pos = np.zeros((n, 3), np.float32)
        prev = np.zeros((n, 3), np.float32)
        vel = np.zeros((n, 3), np.float32)
        w = np.zeros(n, np.float32)
        self._fn("get_state")(self.h, _fp(pos), _fp(prev), _fp(vel), _fp(w))
        return pos, prev, vel, w

    def positions(self):
        return self.state()[0]

    def set_state(self, pos, prev, vel):
        self._fn("set_state")(self.h, _fp(np.ascontiguousarray(pos, np.float32)),
                              _fp(np.ascontiguousarray(prev, np.float32)),
                              _fp(np.ascontiguousarray(vel, np.float32)))

    def tris(self):
        t = self._fn("num_tris")(self.h)
        idx = np.zeros((t, 3), np.uint32)
        rest = np.zeros((t, 10), np.float32)
        self._fn("get_tris")(self.h, _up(idx), _fp(rest))
        return idx, rest

    def bends(self):
        b = self._fn("num_bends")(self.h)
        idx = np.zeros((b, 4), np.uint32)
        self._fn("get_bends")(self.h, _up(idx))
        return idx

    def edges(self):
        e = self._fn("num_edges")(self.h)
        out = np.zeros((e, 4), np.int32)
        self._fn("get_edges")(self.h, _ip(out))
        return out

    def links(self):
        """(n, 2) indices and (n, 2) rest length / stiffness, in creation order"""
        n = self._fn("num_links")(self.h)
        idx = np.zeros((n, 2), np.uint32)
        ls = np.zeros((n, 2), np.float32)
        self._fn("get_links")(self.h, _up(idx), _fp(ls))
        return idx, ls

    def step(self, dt):
        self._fn("step")(self.h, float(dt))

    def update_mesh(self):
        self._fn("update_mesh")(self.h)

    def predict_detect(self, h, ccd=False):
        self._fn("predict_detect")(self.h, float(h), int(ccd))

    def contacts(self, kind):
        """kind 0 vertex, 1 tri, 2 edge, 3 self VT, 4 self EE"""
        n = self._fn("num_contacts")(self.h, kind)
        if kind == 0:
            a = np.zeros((n, 2), np.int32); f = np.zeros((n, 7), np.float32)
            self._fn("get_vertex_contacts")(self.h, _ip(a), _fp(f))
        elif kind == 1:
            a = np.zeros((n, 4), np.int32); f = np.zeros((n, 9), np.float32)
            self._fn("get_tri_contacts")(self.h, _ip(a), _fp(f))
        elif kind == 2:
            a = np.zeros((n, 3), np.int32); f = np.zeros((n, 8), np.float32)
            self._fn("get_edge_contacts")(self.h, _ip(a), _fp(f))
        else:
            a = np.zeros((n, 4), np.int32); f = np.zeros((n, 7), np.float32)
            self._fn("get_self_contacts")(self.h, kind, _ip(a), _fp(f))
        return a, f

    def mesh_normals(self, prev=False):
        n = np.zeros((self.n, 3), np.float32)
        self._fn("get_mesh_normals")(self.h, int(prev), _fp(n))
        return n

    def swept_boxes(self, kind, tol):
        count = {0: self._fn("num_tris")(self.h), 1: self.n, 2: self._fn("num_edges")(self.h)}[kind]
        out = np.zeros((count, 6), np.float32)
        self._fn("swept_boxes")(self.h, kind, float(tol), _fp(out))
        return out

    def ccd_narrow_on(self, vt, ee):
        vt = np.ascontiguousarray(vt, np.int32).reshape(-1, 2)
        ee = np.ascontiguousarray(ee, np.int32).reshape(-1, 2)
        self._fn("ccd_narrow_on")(self.h, vt.shape[0], _ip(vt), ee.shape[0], _ip(ee))


class RefCloth(CpuCloth):
    """The SolidCloth reference compiled from its own sources (oracle/_ref);
    serial=True loads the build without OpenMP."""

    def __init__(self, serial: bool = False):
        super().__init__(REF_SERIAL_LIB if serial else REF_LIB, "ref_")

    def init_mesh(self, vertices, indices, uvs=None, colors=None, offset=(0, 0, 0), attached=False):
        """ClothPatch::Init(mesh, offset, attached) in the reference build"""
        v = np.ascontiguousarray(vertices, np.float32)
        idx = np.ascontiguousarray(indices, np.uint32)
        u = None if uvs is None else np.ascontiguousarray(uvs, np.float32)
        c = None if colors is None else np.ascontiguousarray(colors, np.float32)
        self._fn("init_mesh")(self.h, v.shape[0], _fp(v), idx.size, _up(idx), None if u is None else _fp(u),
                              None if c is None else _fp(c), float(offset[0]), float(offset[1]), float(offset[2]),
                              int(attached))

    @staticmethod
    def set_threads(n: int):
        _load(REF_LIB, "ref_").ref_set_threads(int(n))

    def iterations(self):
        return self._fn("solver_iterations")(self.h)

    def ccd_midphase(self):
        self._fn("ccd_midphase")(self.h)
        out = []
        for kind in (0, 1):
            n = self._fn("ccd_num_candidates")(self.h, kind)
            a = np.zeros((n, 2), np.int32)
            self._fn("ccd_get_candidates")(self.h, kind, _ip(a))
            out.append(a)
        return out


class PortCloth(CpuCloth):
    """This project's CPU restatement of the step (oracle/cloth_oracle.cpp)."""

    def __init__(self):
        super().__init__(PORT_LIB, "orc_")

    @staticmethod
    def set_portable_math(on: bool):
        """True: bends and normal weights use the library's portable arc cosine
        (check mode against the GPU); False: libm acosf (as the reference)."""
        _load(PORT_LIB, "orc_").orc_set_portable_math(int(on))

    @staticmethod
    def portable_acos(x: float) -> float:
        return _load(PORT_LIB, "orc_").orc_portable_acos(float(x))

    def set_tri_order(self, order):
        if order is None:
            self._fn("set_tri_order")(self.h, None, 0)
        else:
            o = np.ascontiguousarray(order, np.int32)
            self._fn("set_tri_order")(self.h, _ip(o), o.size)

    def set_bend_order(self, order):
        if order is None:
            self._fn("set_bend_order")(self.h, None, 0)
        else:
            o = np.ascontiguousarray(order, np.int32)
            self._fn("set_bend_order")(self.h, _ip(o), o.size)

    def set_contact_order(self, mode: int):
        self._fn("set_contact_order")(self.h, int(mode))

    def set_static_colours(self, tri_colour, n_tri, edge_colour, n_edge):
        """the GPU's static colours of triangles and collision-mesh edges: check
        mode orders triangle / edge collider contacts by them"""
        t = np.ascontiguousarray(tri_colour, np.int32)
        e = np.ascontiguousarray(edge_colour, np.int32)
        self._fn("set_static_colours")(self.h, _ip(t), t.size, int(n_tri), _ip(e), e.size, int(n_edge))

    def check_mode(self, model):
        """run in the GPU model's order: constraint colour order, contact colourings"""
        self.set_tri_order(model.constraint_order(0)[0])
        self.set_bend_order(model.constraint_order(1)[0])
        self.set_contact_order(1)
        self.set_static_colours(*model.static_colours())

    def self_contact_colours(self, kind):
        n = self._fn("num_contacts")(self.h, kind)
        c = np.zeros(n, np.int32)
        self._fn("self_contact_colours")(self.h, kind, _ip(c))
        return c

    def load_topology(self, pos, inv_mass, tris, rest10, bends, links, link_rest):
        """replace the model by an explicit topology (see orc_load_topology)"""
        a = [np.ascontiguousarray(x, t) for x, t in ((pos, np.float32), (inv_mass, np.float32), (tris, np.uint32),
                                                       (rest10, np.float32), (bends, np.uint32), (links, np.uint32),
                                                       (link_rest, np.float32))]
        self._fn("load_topology")(self.h, a[0].shape[0], _fp(a[0]), _fp(a[1]), a[2].shape[0], _up(a[2]), _fp(a[3]),
                                  a[4].shape[0], _up(a[4]), a[5].shape[0], _up(a[5]), _fp(a[6]))

    def set_link_order(self, order):
        o = np.ascontiguousarray(order, np.int32)
        self._fn("set_link_order")(self.h, _ip(o), o.size)

    def residual(self) -> float:
        """max |C| over the warp, weft and shear constraints at the current positions"""
        return float(self._fn("residual")(self.h))

    def set_bruteforce_broadphase(self, on: bool):
        """True: the plain all-pairs loop instead of the (exact) sweep over sorted boxes"""
        self._fn("set_bruteforce_broadphase")(self.h, int(on))

    def ccd_broadphase(self, tol, kind, cap=1 << 24):
        out = np.zeros((cap, 2), np.int32)
        n = self._fn("ccd_broadphase")(self.h, float(tol), kind, _ip(out), cap)
        return out[:min(n, cap)].copy()


def available(kind: str = "ref") -> bool:
    return {"ref": REF_LIB, "ref_serial": REF_SERIAL_LIB}.get(kind, PORT_LIB).exists()


def ref_sdf_from_mesh(vertices, indices, cells, box6):
    """the reference's SDF::CreateFromMesh on a (cells+1)^3 grid over box6"""
    lib = _load(REF_LIB, "ref_")
    v = np.ascontiguousarray(vertices, np.float32)
    idx = np.ascontiguousarray(indices, np.uint32)
    b = np.ascontiguousarray(box6, np.float32)
    out = np.zeros((cells[0] + 1) * (cells[1] + 1) * (cells[2] + 1), np.float32)
    lib.ref_sdf_from_mesh(v.shape[0], _fp(v), idx.size // 3, _up(idx), int(cells[0]), int(cells[1]), int(cells[2]),
                          _fp(b), _fp(out))
    return out


def ref_sdf_write(cells, box6, values, path):
    lib = _load(REF_LIB, "ref_")
    b = np.ascontiguousarray(box6, np.float32)
    vals = np.ascontiguousarray(values, np.float32)
    lib.ref_sdf_write(int(cells[0]), int(cells[1]), int(cells[2]), _fp(b), _fp(vals), str(path).encode())


def ref_sdf_read(path, cap=1 << 24):
    lib = _load(REF_LIB, "ref_")
    cells = np.zeros(3, np.int32)
    box = np.zeros(6, np.float32)
    vals = np.zeros(cap, np.float32)
    n = lib.ref_sdf_read(str(path).encode(), _ip(cells), _fp(box), _fp(vals), cap)
    return cells, box, vals[:n].copy()

