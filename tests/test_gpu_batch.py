"""Batched instances (scCreateClothBatch) against the same clothes stepped one
by one, through the C ABI: the batch runs every instance's projections in the
order the instance would run alone, so trajectories are bit-identical; spatial
queries never cross instances."""
import numpy as np
import pytest

from solidcloth_b200 import scenes

pytestmark = pytest.mark.gpu


def _same(a, b):
    return np.array_equal(np.ascontiguousarray(a, np.float32).view(np.uint32),
                          np.ascontiguousarray(b, np.float32).view(np.uint32))


def _standalone(sc, frames, state=None):
    from solidcloth_b200 import api
    w, p = api.load_scene(sc)
    if state is not None:
        p.model.set_state(*state)
    for _ in range(frames):
        p.step(sc.dt)
    out = (p.model.positions(), p.model.velocities(), p.status())
    p.free()
    w.free()
    return out


@pytest.mark.parametrize("solver", ["auto", "grid", "kernels"])
def test_batch_matches_standalone(solver):
    """Uneven instances (sides 8..24, own sphere SDF, 1-4 pinned corners, the
    continuous self-collision detector on): each instance of the batch equals the
    instance stepped alone, bit for bit, whichever solver runs the batch."""
    from solidcloth_b200 import api
    insts = scenes.cfg3_instances(count=5, seed=11, lo=8, hi=24)
    frames = 6
    b = api.load_batch(insts)
    assert b.size() == len(insts)
    if solver == "grid":
        b.model.set_grid_solver(0, 1)
    elif solver == "kernels":
        b.model.set_solver_mode(3)
    for _ in range(frames):
        b.step(insts[0].dt)
    pos, vel = b.model.positions(), b.model.velocities()
    assert b.status() == 0
    for k, sc in enumerate(insts):
        a, n = b.instance(k)
        assert n == sc.num_vertices
        p1, v1, st = _standalone(sc, frames)
        assert st == 0
        assert _same(pos[a:a + n], p1), (k, float(np.abs(pos[a:a + n] - p1).max()))
        assert _same(vel[a:a + n], v1), k
    b.free()


@pytest.mark.parametrize("walk", [0, 1])
def test_batch_queries_stay_inside_instances(walk):
    """Two copies of a folded demo-scale cloth at the same place: the batch's
    continuous-collision candidate pairs are the union of each copy's own pairs
    (offset), with no pair between the copies, and its self contacts likewise."""
    from solidcloth_b200 import api
    sc, state = scenes.ccd_scene(16)
    b = api.load_batch([sc, sc])
    b.model.set_broad_phase_mode(walk)
    n = sc.num_vertices
    pos, prev, vel = state
    b.model.set_state(np.concatenate([pos, pos]), np.concatenate([prev, prev]), np.concatenate([vel, vel]))
    b.step(sc.dt)
    w, p = api.load_scene(sc, ccd=True)
    p.model.set_state(*state)
    p.step(sc.dt)
    T = p.model.num_tris()
    E = p.model.num_edges()
    one_vt, one_ee = p.model.ccd_candidates(0), p.model.ccd_candidates(1)
    assert len(one_vt) > 0 and len(one_ee) > 0
    both_vt, both_ee = b.model.ccd_candidates(0), b.model.ccd_candidates(1)
    want_vt = np.concatenate([one_vt, one_vt + np.array([n, T], np.int32)])
    want_ee = np.concatenate([one_ee, one_ee + E])
    assert np.array_equal(both_vt, want_vt)
    assert np.array_equal(both_ee, want_ee)
    # each copy moves exactly as the copy alone
    g = b.model.positions()
    assert _same(g[:n], p.model.positions()) and _same(g[n:], p.model.positions())
    p.free()
    w.free()
    b.free()
