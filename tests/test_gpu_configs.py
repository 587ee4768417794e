"""GPU parity at the benchmark configurations' sizes, through the C ABI.

Check mode (the oracle runs the reference's sequential sweep in the order the
coloured GPU sweep realises, with the library's portable arc cosine) on:

  * the 128x128 drape onto the 64^3 sphere SDF with continuous self-collision
    (16,384 vertices), two frames;
  * the 256x256 drape onto the level-5 icosphere mesh + ground plane with mesh
    contacts and continuous self-collision (65,536 vertices: exactly the 65,536
    vertices the reference's uint16 index casts allow,
    Geometry/ClosestPointsBetweenMeshes.cpp:78-80), one frame started 1 cm above
    the collider so that mesh contacts appear;
  * the first 64 of the 512 uneven instances as one batch, two frames, each
    instance against the oracle stepping it alone.

Positions must be bit-identical after every frame; the contact lists of the
last substep and the continuous detector's candidate-pair sets (from the same
predicted state) must be equal as sets and per query in the GPU's order. The
device status must stay clear: no pair-store, pool, stack or colour overflow.
"""
import copy

import numpy as np
import pytest

from solidcloth_b200 import scenes

pytestmark = pytest.mark.gpu


def _same(g, c):
    return np.array_equal(np.ascontiguousarray(g, np.float32).view(np.uint32),
                          np.ascontiguousarray(c, np.float32).view(np.uint32))


def _oracle_for(sc, p, state=None):
    """oracle in the GPU patch p's constraint order (check mode)"""
    from oracle.bridge import PortCloth
    PortCloth.set_portable_math(True)
    o = PortCloth.from_scene(sc)
    if state is not None:
        o.set_state(*state)
    o.set_tri_order(p.model.constraint_order(0)[0])
    o.set_bend_order(p.model.constraint_order(1)[0])
    o.set_contact_order(1)
    o.set_static_colours(*p.model.static_colours())
    return o


def _pairs_match(sc, p, pos, prev, vel):
    """The GPU's candidate pairs of its last substep against the oracle's all-pairs
    broad phase from the same start-of-substep state: the GPU predicts from
    (pos, prev, vel) of the substep before, so rebuild that state in the oracle."""
    from oracle.bridge import PortCloth
    o2 = PortCloth.from_scene(sc)
    o2.set_state(pos, prev, vel)
    o2.predict_detect(sc.dt / sc.params.substeps, ccd=False)
    tol = sc.params.thickness + 0.5 * sc.params.tolerance
    ovt, oee = o2.ccd_broadphase(tol, 0), o2.ccd_broadphase(tol, 1)
    gvt, gee = p.model.ccd_candidates(0, cap=1 << 25), p.model.ccd_candidates(1, cap=1 << 25)
    assert len(ovt) > 0 and len(oee) > 0
    # vertex-triangle pairs come from the GPU as (vertex, triangle), ascending;
    # the oracle lists (triangle, vertex) ascending: reorder it by vertex
    want_vt = ovt[np.lexsort((ovt[:, 0], ovt[:, 1]))][:, ::-1]
    assert np.array_equal(gvt, want_vt)
    assert np.array_equal(gee, oee)
    o2.close()
    return len(ovt), len(oee)


def _run_check_mode(sc, frames, per_substep_state=True, solver_mode=0):
    """GPU and oracle side by side; returns the GPU patch, the oracle and the
    state before the last substep (for the broad-phase comparison)"""
    from solidcloth_b200 import api
    w, p = api.load_scene(sc)
    if solver_mode:
        p.model.set_solver_mode(solver_mode)
    o = _oracle_for(sc, p)
    for f in range(frames):
        p.step(sc.dt)
        o.step(sc.dt)
        p.update_mesh()
        o.update_mesh()
        g, c = p.model.positions(), o.positions()
        assert _same(g, c), (f, float(np.abs(g - c).max()))
    assert p.status() & ~16 == 0, p.status()
    return w, p, o


def test_cfg1_128_drape_check_mode():
    sc = scenes.cfg1()
    # start 2 mm above the sphere so that SDF contacts appear within the frames
    sc.positions[:, 1] -= np.float32(0.398)
    w, p, o = _run_check_mode(sc, 2)
    gi, gf = p.model.contacts(0)
    oi, of = o.contacts(0)
    assert len(oi) >= 100
    assert np.array_equal(gi, oi)
    assert _same(gf[:, :6], of[:, :6])
    # normals (Mesh::ComputeNormals, Geometry/Mesh.cpp:10-63) of the updated mesh
    _, gn, _ = p.mesh_buffers()
    assert _same(gn, o.mesh_normals())
    # one more substep from a known state: the candidate pairs
    sub = copy.deepcopy(sc)
    sub.params.substeps = 1
    pos, prev, vel = p.model.positions(), p.model.prev_positions(), p.model.velocities()
    from solidcloth_b200 import api
    w1, p1 = api.load_scene(sub)
    p1.model.set_state(pos, prev, vel)
    p1.step(sub.dt)
    nvt, nee = _pairs_match(sub, p1, pos, prev, vel)
    assert nvt > 100_000 and nee > 100_000
    assert p1.status() & ~16 == 0
    p1.free()
    p.free()


@pytest.mark.parametrize("n", [128, 256])
def test_band_solver_check_mode_at_config_sizes(n):
    """The band-parallel solver (solver mode 4: one 16-CTA cluster, particle
    bands resident in shared memory, interior then boundary records) on the
    128x128 SDF drape and the 256x256 icosphere drape: bit-identical to the
    oracle run in the band order, frame by frame."""
    sc = scenes.cfg1() if n == 128 else scenes.cfg2()
    sc.positions[:, 1] -= np.float32(0.398 if n == 128 else 0.49)
    w, p, o = _run_check_mode(sc, 1, solver_mode=4)
    cs, per_band, halo, used = p.model.band_plan()
    assert used == 1 and cs == 16 and per_band * cs == n * n and 0 < halo <= 2 * n + 2
    assert p.model.solver_choice()[0][0] == 4
    p.free()


def test_cfg2_256_mesh_drape_check_mode():
    sc = scenes.cfg2()
    assert sc.num_vertices == 65536
    sc.positions[:, 1] -= np.float32(0.49)
    w, p, o = _run_check_mode(sc, 1)
    seen = 0
    for kind in (0, 1, 2):
        gi, gf = p.model.contacts(kind)
        oi, of = o.contacts(kind)
        assert np.array_equal(gi, oi), (kind, len(gi), len(oi))
        k = min(gf.shape[1], of.shape[1])
        assert _same(gf[:, :k], of[:, :k]), kind
        seen += len(oi)
    assert seen > 100
    _, gn, _ = p.mesh_buffers()
    assert _same(gn, o.mesh_normals())
    sub = copy.deepcopy(sc)
    sub.params.substeps = 1
    pos, prev, vel = p.model.positions(), p.model.prev_positions(), p.model.velocities()
    from solidcloth_b200 import api
    w1, p1 = api.load_scene(sub)
    p1.model.set_state(pos, prev, vel)
    p1.step(sub.dt)
    nvt, nee = _pairs_match(sub, p1, pos, prev, vel)
    assert nvt > 1_000_000 and nee > 1_000_000
    assert p1.status() & ~16 == 0
    p1.free()
    p.free()


def test_cfg3_64_instances_check_mode():
    """The first 64 of the 512 uneven instances as one batch: every instance
    equals the oracle stepping it alone in its own constraint order."""
    from solidcloth_b200 import api
    insts = scenes.cfg3_instances()[:64]
    b = api.load_batch(insts)
    frames = 2
    for _ in range(frames):
        b.step(insts[0].dt)
    assert b.status() == 0, b.status()
    pos = b.model.positions()
    for k, sc in enumerate(insts):
        a, n = b.instance(k)
        w, p = api.load_scene(sc)          # the instance alone: its constraint order
        o = _oracle_for(sc, p)
        p.free()
        w.free()
        for _ in range(frames):
            o.step(sc.dt)
        c = o.positions()
        assert _same(pos[a:a + n], c), (k, sc.n, float(np.abs(pos[a:a + n] - c).max()))
        o.close()
    b.free()


def test_sdf_triangle_contacts_check_mode():
    """GridSDF::QueryTriangle (Frank-Wolfe over the triangle, at most 100 steps,
    Physics/ClothCollisionSDF.h:148-205) with CF_TRIANGLES on an SDF collider:
    triangle contacts and trajectories equal the oracle's frame by frame."""
    from solidcloth_b200 import api
    sc = scenes.cfg1(n=24)
    sc.params.flags |= scenes.CF_TRIANGLES
    sc.params.substeps = 2
    sc.params.iterations = 6
    sc.positions[:, 1] -= np.float32(0.397)
    sc.ccd = False
    # unit inverse masses: the reference's triangle-contact solve divides by the
    # inverse mass (Physics/ClothCollisionHandler.cpp:302) and is only consistent
    # for inverse mass 1; with the lumped gram masses both it and the oracle blow up
    sc.masses = np.ones(sc.num_vertices, np.float32)
    w, p = api.load_scene(sc)
    o = _oracle_for(sc, p)
    seen = 0
    for f in range(5):
        p.step(sc.dt)
        o.step(sc.dt)
        p.update_mesh()
        o.update_mesh()
        assert np.isfinite(p.model.positions()).all()
        assert _same(p.model.positions(), o.positions()), f
        gi, gf = p.model.contacts(1)
        oi, of = o.contacts(1)
        assert np.array_equal(gi, oi), (f, len(gi), len(oi))
        k = min(gf.shape[1], of.shape[1])
        assert _same(gf[:, :k], of[:, :k]), f
        seen += len(oi)
    assert seen > 0
    assert p.status() & ~16 == 0
    p.free()
