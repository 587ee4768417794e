"""CPU tests: the oracle pinned to the reference, the C ABI's exports, scene shapes.

The oracle (oracle/cloth_oracle.cpp) is the checker of every GPU test. It is
pinned two ways: against golden fixtures generated from the SolidCloth
reference's own C++ (tests/golden/make_golden.py, run here where the reference
sources exist), and — when oracle/_ref is built — against the reference build
directly on the same inputs. Both comparisons are bit-exact.
"""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from solidcloth_b200 import scenes

ROOT = Path(__file__).resolve().parent.parent
GOLD = Path(__file__).resolve().parent / "golden"


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def port():
    from oracle.bridge import PortCloth, available
    if not available("port"):
        pytest.skip("oracle not built (make -C oracle port)")
    return PortCloth


def ref():
    from oracle.bridge import RefCloth, available
    if not available("ref"):
        pytest.skip("reference build absent")
    RefCloth.set_threads(1)
    return RefCloth


import importlib.util

_spec = importlib.util.spec_from_file_location("make_golden", GOLD / "make_golden.py")


def golden_module():
    m = importlib.util.module_from_spec(_spec)
    _spec.loader.exec_module(m)
    return m


# ------------------------------------------------------------------ goldens
def test_golden_cfg0():
    P = port()
    g = np.load(GOLD / "cfg0.npz")
    sc = scenes.cfg0()
    o = P.from_scene(sc)
    idx, rest = o.tris()
    assert np.array_equal(idx, g["tris"]) and np.array_equal(bits(rest), bits(g["rest"]))
    assert np.array_equal(o.bends(), g["bends"]) and np.array_equal(o.edges(), g["edges"])
    for _ in range(10):
        o.step(sc.dt)
        o.update_mesh()
    pos, prev, vel, w = o.state()
    for a, b in [(pos, g["pos"]), (prev, g["prev"]), (vel, g["vel"]), (w, g["invmass"])]:
        assert np.array_equal(bits(a), bits(b))
    assert np.array_equal(bits(o.mesh_normals(False)), bits(g["normals"]))
    assert np.array_equal(bits(o.mesh_normals(True)), bits(g["prev_normals"]))


def test_golden_sdf_contacts():
    P = port()
    m = golden_module()
    g = np.load(GOLD / "sdf.npz")
    sc = m.sdf_scene()
    o = P.from_scene(sc)
    for _ in range(3):
        o.step(sc.dt)
        o.update_mesh()
    vi, vf = o.contacts(0)
    assert len(vi) > 0
    assert np.array_equal(vi, g["vc_idx"]) and np.array_equal(bits(vf), bits(g["vc_f"]))
    assert np.array_equal(bits(o.positions()), bits(g["pos"]))


def test_golden_self_contacts():
    P = port()
    m = golden_module()
    g = np.load(GOLD / "self.npz")
    sc, st = m.folded_scene()
    o = P.from_scene(sc)
    o.set_state(*st)
    o.step(sc.dt)
    ti, tf = o.contacts(3)
    ei, ef = o.contacts(4)
    assert len(ti) > 100 and len(ei) > 100
    assert np.array_equal(ti, g["vt_idx"]) and np.array_equal(bits(tf), bits(g["vt_f"]))
    # edge-edge: the reference leaves w3 uninitialised for edge contacts; compare the rest
    sel = [0, 1, 2, 3, 4, 6]
    assert np.array_equal(ei, g["ee_idx"]) and np.array_equal(bits(ef[:, sel]), bits(g["ee_f"][:, sel]))
    assert np.array_equal(bits(o.positions()), bits(g["pos"]))


def test_golden_ccd():
    P = port()
    g = np.load(GOLD / "ccd.npz")
    sc, st = scenes.ccd_scene(16)
    o = P.from_scene(sc)
    o.set_state(*st)
    o.predict_detect(sc.dt / sc.params.substeps, ccd=False)
    tol = sc.params.thickness + 0.5 * sc.params.tolerance
    assert np.array_equal(bits(o.swept_boxes(0, tol)), bits(g["boxes_t"]))
    allvt = set(map(tuple, o.ccd_broadphase(tol, 0).tolist()))
    allee = set(map(tuple, o.ccd_broadphase(tol, 1).tolist()))
    # the reference's same-leaf midphase finds a subset of all overlapping pairs
    assert set(map(tuple, g["mid_vt"].tolist())) <= allvt
    assert set(map(tuple, g["mid_ee"].tolist())) <= allee
    o.ccd_narrow_on(g["mid_vt"], g["mid_ee"])
    hi, hf = o.contacts(3)
    ei, ef = o.contacts(4)
    assert len(hi) > 100 and len(ei) > 100
    sel = [0, 1, 2, 3, 4, 5, 6]
    assert np.array_equal(hi, g["hit_vt_idx"]) and np.array_equal(bits(hf[:, sel]), bits(g["hit_vt_f"][:, sel]))
    sel = [0, 1, 2, 3, 4, 6]
    assert np.array_equal(ei, g["hit_ee_idx"]) and np.array_equal(bits(ef[:, sel]), bits(g["hit_ee_f"][:, sel]))


def test_golden_mesh_collider():
    P = port()
    m = golden_module()
    g = np.load(GOLD / "mesh.npz")
    sc = m.mesh_scene()
    o = P.from_scene(sc)
    for _ in range(2):
        o.step(sc.dt)
        o.update_mesh()
    for k, name in [(0, "vc"), (1, "tc"), (2, "ec")]:
        a, b = o.contacts(k)
        assert len(a) > 0, name
        assert np.array_equal(a, g[name + "_idx"]) and np.array_equal(bits(b), bits(g[name + "_f"])), name
    assert np.array_equal(bits(o.positions()), bits(g["pos"]))


# --------------------------------------------------- port vs reference, live
@pytest.mark.parametrize("n", [12, 20])
def test_port_matches_reference_sdf_self(n, ref_threads):
    R, P = ref(), port()
    sc = scenes.cfg1(n=n, self_mode="proximity")
    sc.params.substeps = 2
    sc.params.iterations = 5
    sc.positions[:, 1] -= np.float32(0.4 - 0.003)
    r, o = R.from_scene(sc), P.from_scene(sc)
    for _ in range(4):
        r.step(sc.dt)
        o.step(sc.dt)
        r.update_mesh()
        o.update_mesh()
        assert np.array_equal(bits(r.positions()), bits(o.positions()))
    for k in (0, 3):
        assert np.array_equal(r.contacts(k)[0], o.contacts(k)[0])


def test_port_matches_reference_fixed_vs_early_exit(ref_threads):
    """Both the fixed-iteration mode and the reference's early exit (FEM: exits
    after one iteration without contacts, quirk of Physics/ClothPBD.cpp:357)."""
    R, P = ref(), port()
    for fixed in (True, False):
        sc = scenes.cfg0()
        sc.params.fixed_iterations = fixed
        r, o = R.from_scene(sc), P.from_scene(sc)
        for _ in range(5):
            r.step(sc.dt)
            o.step(sc.dt)
        assert np.array_equal(bits(r.positions()), bits(o.positions()))


def test_ccd_port_matches_reference_on_all_pairs(ref_threads):
    R, P = ref(), port()
    sc, st = scenes.ccd_scene(20)
    o = P.from_scene(sc)
    o.set_state(*st)
    o.predict_detect(sc.dt, ccd=False)
    tol = sc.params.thickness + 0.5 * sc.params.tolerance
    vt, ee = o.ccd_broadphase(tol, 0), o.ccd_broadphase(tol, 1)
    r = R.from_scene(sc)
    r.set_state(*st)
    r.predict_detect(sc.dt, ccd=False)
    r.ccd_narrow_on(vt, ee)
    o.ccd_narrow_on(vt, ee)
    for k in (3, 4):
        a, b = r.contacts(k), o.contacts(k)
        assert len(a[0]) > 100
        sel = [0, 1, 2, 3, 4, 6]
        assert np.array_equal(a[0], b[0]) and np.array_equal(bits(a[1][:, sel]), bits(b[1][:, sel]))


def test_contact_colouring_is_independent():
    P = port()
    m = golden_module()
    sc, st = m.folded_scene()
    o = P.from_scene(sc)
    o.set_state(*st)
    o.step(sc.dt)
    for kind in (3, 4):
        idx, _ = o.contacts(kind)
        col = o.self_contact_colours(kind)
        assert col.min() >= 0
        for c in np.unique(col):
            v = idx[col == c].reshape(-1)
            assert len(np.unique(v)) == v.size


# ------------------------------------------------------------------ C ABI
def declared_symbols():
    txt = (ROOT / "include" / "solidcloth_b200.h").read_text()
    return sorted(set(re.findall(r"SCEXP[^;(]*?\b(sc[A-Za-z0-9]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    from solidcloth_b200 import api
    if not api.LIB_PATH.exists():
        pytest.skip("CUDA library not built")
    lib = ctypes.CDLL(str(api.LIB_PATH))
    names = declared_symbols()
    assert len(names) >= 95
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers every entry point
    assert set(names) <= set(api.SIGNATURES)


def test_reference_entry_points_are_all_present():
    """Every extern "C" function of the reference's ClothAPI (Demo/ClothAPI.h:65-146)
    has a counterpart of the same name (two take C arrays instead of C++ objects)."""
    reference_api = [
        "scCreateCollisionWorld", "scFreeCollisionWorld", "scClearCollidables", "scGetNumCollidables",
        "scAddCollidable", "scGetCollidable", "scCreateWalls", "scCreateSphere", "scCreateCapsule",
        "scGetCollidableType", "scGetMeshTree", "scGetWallsInfo", "scGetSphereInfo", "scGetCapsuleInfo",
        "scCreateClothPatch", "scFreeClothPatch", "scGetClothModel", "scGetClothMesh", "scInitCloth",
        "scStepCloth", "scUpdateClothMesh", "scComputeStrainMap", "scGetNumParticles", "scGetParticlePos",
        "scGetParticleInvMass", "scGetNumTris", "scGetTriangle", "scGetTriangleInfo", "scGetNumQuads",
        "scGetQuad", "scGetNumLinks", "scGetLink", "scGetNumContacts", "scGetContact", "scGetNumTriContacts",
        "scGetTriContact", "scGetCollisionFlags", "scSetCollisionFlags", "scGetThickness", "scSetThickness",
        "scGetTolerance", "scSetTolerance", "scGetFriction", "scSetFriction", "scGetNumIterations",
        "scSetNumIterations", "scGetUseFEM", "scSetUseFEM", "scGetClothTree", "scAddMouseSpring",
        "scUpdateMouseSpring", "scRemoveMouseSpring", "scGetMeshVertexCount", "scGetMeshIndexCount",
        "scGetMeshNormalBuffer", "scGetMeshVertexBuffer", "scGetMeshIndexBuffer"]
    names = set(declared_symbols())
    assert not [n for n in reference_api if n not in names]
    assert {"scCreateSDFGrid", "scCreateMeshCollider"} <= names


# ------------------------------------------------------------------ scenes
@pytest.mark.parametrize("n,T,E,B", [(32, 1922, 2945, 2821), (128, 32258, 48641, 48133)])
def test_grid_counts(n, T, E, B):
    P = port()
    sc = scenes.cfg1(n=n) if n > 32 else scenes.cfg0()
    o = P.from_scene(sc)
    assert o.n == n * n
    assert len(o.tris()[0]) == T and len(o.edges()) == E and len(o.bends()) == B


def test_icosphere_level5():
    m = scenes.icosphere(5, 0.25, (0, 0.25, 0))
    assert m.vertices.shape == (10242, 3) and m.indices.size == 3 * 20480


def test_sphere_sdf_samples():
    g = scenes.sphere_sdf((0, 0, 0), 0.3, 63, 0.1)
    assert g.values.size == 64 ** 3
    assert abs(g.values.min() + 0.3) < 0.02


# ------------------------------------------------------- mass-spring path
def test_golden_links():
    """The mass-spring path (FEM off; SolveLinks, Physics/ClothPBD.cpp:9-50) of the
    oracle against fixtures from the reference build, with and without dihedral
    bending (without it, ClothPatch::Init adds bend links)."""
    P = port()
    P.set_portable_math(False)
    g = np.load(GOLD / "links.npz")
    mg = golden_module()
    for dih in (False, True):
        sc = mg.links_scene(dih)
        o = P.from_scene(sc)
        for _ in range(8):
            o.step(sc.dt)
        pos, prev, vel, _ = o.state()
        assert np.array_equal(bits(pos), bits(g[f"pos_dihedral{int(dih)}"])), dih
        assert np.array_equal(bits(vel), bits(g[f"vel_dihedral{int(dih)}"])), dih


@pytest.mark.parametrize("fixed", [True, False])
def test_port_matches_reference_links(fixed, ref_threads):
    """Live: links path bit-exact, in fixed-iteration mode and with the
    reference's exit test (links error below 0.05, Physics/ClothPBD.cpp:357)."""
    R, P = ref(), port()
    P.set_portable_math(False)
    mg = golden_module()
    for dih in (False, True):
        sc = mg.links_scene(dih)
        sc.params.fixed_iterations = fixed
        r, o = R.from_scene(sc), P.from_scene(sc)
        for _ in range(6):
            r.step(sc.dt)
            o.step(sc.dt)
        assert np.array_equal(bits(r.positions()), bits(o.positions())), dih


# ------------------------------------------- Jacobi and conjugate residual
def _same_or_both_nan(a, b):
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    return np.array_equal(np.isnan(a), np.isnan(b)) and np.array_equal(bits(np.nan_to_num(a)), bits(np.nan_to_num(b)))


def test_golden_solvers():
    """SolveJacobi and SolveCR (Physics/ClothPBD.cpp:371-496, 616-661), chosen by
    ClothModel::SetSolver: the oracle against fixtures from the reference build,
    bit for bit (where the reference's conjugate-residual solve diverges, NaN
    where it has NaN)."""
    P = port()
    P.set_portable_math(False)
    g = np.load(GOLD / "solvers.npz")
    for name, sc, frames in golden_module().solver_scenes():
        o = P.from_scene(sc)
        for _ in range(frames):
            o.step(sc.dt)
        pos, prev, vel, _ = o.state()
        assert _same_or_both_nan(pos, g[f"{name}_pos"]), name
        assert _same_or_both_nan(vel, g[f"{name}_vel"]), name
    assert np.isfinite(g["jacobi_pos"]).all() and np.isfinite(g["cr_pos"]).all()
    assert np.isnan(g["cr_diverging_pos"]).any()


def test_port_matches_reference_solvers(ref_threads):
    """Live: the Jacobi and conjugate-residual solves bit-exact against the
    reference build, frame by frame."""
    R, P = ref(), port()
    P.set_portable_math(False)
    for name, sc, frames in golden_module().solver_scenes():
        r, o = R.from_scene(sc), P.from_scene(sc)
        for f in range(frames):
            r.step(sc.dt)
            o.step(sc.dt)
            assert _same_or_both_nan(r.positions(), o.positions()), (name, f)


# ------------------------------------------------------------- mesh cloth
def test_port_matches_reference_mesh_cloth(ref_threads):
    """ClothPatch::Init(mesh) (Physics/ClothPatch.cpp:42-133) in the reference
    build, its topology loaded into the oracle: the oracle steps it bit for bit
    (FEM + bends, and the mass-spring path)."""
    R, P = ref(), port()
    P.set_portable_math(False)
    for fem in (True, False):
        v, idx, uv, col, prm = scenes.mesh_cloth()
        prm.fem = fem
        r = R()
        pa = prm.as_array()
        r._fn("set_params")(r.h, pa.ctypes.data_as(__import__("ctypes").POINTER(__import__("ctypes").c_float)), pa.size)
        r.init_mesh(v, idx, uv, col, (0, 0, 0), True)
        pos, prev, vel, w = r.state()
        assert 0 < pos.shape[0] < v.shape[0]          # coincident corners merged
        assert np.sum(w == 0) == 2                    # the two red corners pinned
        ti, tr = r.tris()
        li, lr = r.links()
        o = P()
        o._fn("set_params")(o.h, pa.ctypes.data_as(__import__("ctypes").POINTER(__import__("ctypes").c_float)), pa.size)
        o.load_topology(pos, w, ti, tr, r.bends(), li, lr)
        dt = 1.0 / 60
        for _ in range(6):
            r.step(dt)
            o.step(dt)
        assert np.array_equal(bits(r.positions()), bits(o.positions())), fem


# ------------------------------------------------- oracle broad phase: sweep
def _pairs(o, tol, brute):
    o.set_bruteforce_broadphase(brute)
    return o.ccd_broadphase(tol, 0), o.ccd_broadphase(tol, 1)


@pytest.mark.parametrize("case", ["ccd_thick", "drape", "nan"])
def test_oracle_sweep_broadphase_equals_all_pairs(case):
    """The oracle's sorted-sweep broad phase (used at the configuration sizes)
    returns exactly the all-pairs loop's pair lists, in the same order: on the
    demo-scale fold with boxes several cells wide, on a draped cloth after a few
    frames, and with a NaN position (whose boxes the overlap test cannot reject)."""
    P = port()
    if case == "ccd_thick":
        sc, state = scenes.ccd_scene(16)
        sc.params.thickness = 3.0
    else:
        sc = scenes.cfg1(n=40)
        state = None
    o = P.from_scene(sc)
    if state is not None:
        o.set_state(*state)
    if case != "ccd_thick":
        for _ in range(3):
            o.step(sc.dt)
    if case == "nan":
        pos, prev, vel, _ = o.state()
        pos[77, 1] = np.nan
        o.set_state(pos, prev, vel)
    o.predict_detect(sc.dt / sc.params.substeps, ccd=False)
    tol = sc.params.thickness + 0.5 * sc.params.tolerance
    fast = _pairs(o, tol, False)
    slow = _pairs(o, tol, True)
    for f, s in zip(fast, slow):
        assert len(s) > 0
        assert np.array_equal(f, s)
