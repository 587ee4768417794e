"""The fast build of the solver (scSetSolverPrecision(model, 1): FMA contraction,
approximate division and square root) against the CPU oracle, through the C ABI.

The projections are the reference's (Physics/ClothPBD.cpp:52-224,
Physics/ClothCollisionHandler.cpp:134-542) evaluated with shorter arithmetic
chains, so results are no longer bit-identical; the bound is the scope's
per-projection tolerance, 1e-5 relative in FP32 (relative to the cloth's
coordinate scale, max |x|), checked on the oracle in the GPU's constraint order
(check mode) from identical states. Detection is shared with the IEEE build:
contact lists stay bit-exact. Over many frames the order-drift bound of the IEEE
build applies unchanged.
"""
import copy

import numpy as np
import pytest

from solidcloth_b200 import scenes

pytestmark = pytest.mark.gpu

REL = 1e-5     # per-projection tolerance of the scope, relative to the coordinate scale


def _pair(sc, fast=True, state=None):
    from solidcloth_b200 import api
    from oracle.bridge import PortCloth
    PortCloth.set_portable_math(True)
    w, p = api.load_scene(sc)
    p.model.set_fast_math(fast)
    o = PortCloth.from_scene(sc)
    if state is not None:
        p.model.set_state(*state)
        o.set_state(*state)
    o.set_tri_order(p.model.constraint_order(0)[0])
    o.set_bend_order(p.model.constraint_order(1)[0])
    o.set_contact_order(1)
    o.set_static_colours(*p.model.static_colours())
    return w, p, o


def _rel(g, c):
    return float(np.abs(g - c).max()) / max(1.0, float(np.abs(c).max()))


def test_precision_setter_round_trips_and_rejects():
    from solidcloth_b200 import api
    w, p = api.load_scene(scenes.cfg0())
    assert p.model.fast_math() is False          # IEEE by default
    p.model.set_fast_math(True)
    assert p.model.fast_math() is True
    api.lib().scSetSolverPrecision(p.model.h, 7)
    assert api.lib().scGetLastError() == 2
    assert p.model.fast_math() is True
    p.free()


@pytest.mark.parametrize("what", ["fem", "fem_bends"])
def test_fast_projections_within_tolerance(what):
    """One substep of one iteration from the same state: one sweep of every FEM
    colour (and bend colour), each projection once."""
    sc = scenes.cfg0()
    sc.params.substeps = 1
    sc.params.iterations = 1
    sc.params.dihedral = what == "fem_bends"
    # a strained start: every constraint projects
    rng = np.random.default_rng(3)
    pos = (sc.positions + rng.uniform(-0.01, 0.01, sc.positions.shape)).astype(np.float32)
    state = (pos, pos.copy(), np.zeros_like(pos))
    w, p, o = _pair(sc, state=state)
    p.step(sc.dt)
    o.step(sc.dt)
    g, c = p.model.positions(), o.positions()
    assert not np.array_equal(g, pos)
    assert _rel(g, c) <= REL, _rel(g, c)
    assert p.status() == 0


def test_fast_steps_within_tolerance_cfg0():
    """Whole steps (4 substeps x 10 iterations, FEM + bends), frame by frame."""
    sc = scenes.cfg0()
    w, p, o = _pair(sc)
    for f in range(5):
        p.step(sc.dt)
        o.step(sc.dt)
        assert _rel(p.model.positions(), o.positions()) <= REL, (f, _rel(p.model.positions(), o.positions()))


def test_fast_sdf_drape_contacts_exact_positions_within_tolerance():
    """128x128 drape 2 mm above the SDF sphere, one frame (8 substeps x 15
    iterations): vertex contact lists stay bit-exact (detection runs in the IEEE
    build on the same predicted positions up to the solver's rounding, so the
    lists are compared where the states still agree: the first substep), positions
    within tolerance."""
    sc = scenes.cfg1()
    sc.positions[:, 1] -= np.float32(0.398)
    sub = copy.deepcopy(sc)
    sub.params.substeps = 1
    w, p, o = _pair(sub)
    p.step(sub.dt)
    o.step(sub.dt)
    gi, gf = p.model.contacts(0)
    oi, of = o.contacts(0)
    assert len(oi) > 0 and np.array_equal(gi, oi)
    assert _rel(p.model.positions(), o.positions()) <= REL
    w, p, o = _pair(sc)
    p.step(sc.dt)
    o.step(sc.dt)
    assert _rel(p.model.positions(), o.positions()) <= REL, _rel(p.model.positions(), o.positions())
    assert p.status() & ~16 == 0


@pytest.mark.parametrize("scene", ["cfg0", "sdf", "links"])
def test_fast_solvers_agree(scene):
    """In the fast build the cluster solver, every grid variant and the
    per-colour kernels run the same projections in the same order; FMA contraction may differ between the kernels they are inlined into,
    so they agree within the projection tolerance rather than bit for bit."""
    from solidcloth_b200 import api
    if scene == "cfg0":
        sc = scenes.cfg0()
    elif scene == "sdf":
        sc = scenes.cfg1(n=20)
        sc.params.substeps = 4
        sc.params.iterations = 6
        sc.positions[:, 1] -= np.float32(0.4 - 0.006)
    else:
        sc = scenes.cfg0()
        sc.params.fem = False
        sc.params.stretch, sc.params.shear, sc.params.bend = 1e3, 5e2, 2.0
    modes = [("cluster", 0), ("cluster", 1), ("kernels", None)] + [("grid", (v, 1)) for v in range(len(api.grid_variants()))]
    out = []
    for mode, arg in modes:
        w, p = api.load_scene(sc)
        p.model.set_fast_math(True)
        if mode == "cluster":
            p.model.set_cluster_variant(arg)
        elif mode == "kernels":
            p.model.set_cluster_solver(False)
        else:
            p.model.set_grid_solver(*arg)
        for _ in range(4):
            p.step(sc.dt)
        out.append(p.model.positions())
        assert p.status() & ~16 == 0, mode
        p.free()
    for g, m in zip(out[1:], modes[1:]):
        assert _rel(g, out[0]) <= REL, (m, _rel(g, out[0]))


def test_fast_order_drift():
    """The fast build, coloured order, against the oracle in the reference's own
    sequential order with libm's acosf (the reference algorithm): the same bound
    as the IEEE build's drift test (twice the chaos envelope of one extra
    iteration or a last-ulp arc cosine change), transient and damped to rest."""
    from test_gpu_step import _drift_runs       # tests/ is on sys.path (rootdir-relative imports)
    sc = scenes.cfg0()
    drift, envelope, rg, rr = _drift_runs(sc, 100, 20, fast=True)
    assert drift.max() <= 2.0 * envelope.max(), (drift, envelope)
    assert 0.5 * rr <= rg <= 2.0 * rr, (rg, rr)
    sc = scenes.cfg0()
    sc.params.drag = 0.98
    sc.params.iterations = 40
    drift, envelope, rg, rr = _drift_runs(sc, 400, 100, fast=True)
    assert drift[-1] <= 0.01, (drift, envelope)
    assert abs(rg - rr) <= 0.05 * rr, (rg, rr)


@pytest.mark.parametrize("fast", [False, True])
def test_projections_against_reference_arc_cosine_at_256(fast):
    """One sweep of every FEM and bend colour on a 256 x 256 cloth (65,536
    particles, the benchmark size) from a strained state, each constraint
    projected once, against the oracle in the GPU's order with libm's acosf — the
    reference's own arc cosine (Physics/ClothPBD.cpp:157), where the GPU evaluates
    the portable one: within the scope's 1e-5 relative per projection, for the
    IEEE and the fast build."""
    from solidcloth_b200 import api
    from oracle.bridge import PortCloth
    sc = scenes.make_grid_scene("proj_256", 256, 1.5, 0.0, scenes.Params(iterations=1, substeps=1),
                                pinned_corners=(1, 3), seed=5)
    rng = np.random.default_rng(7)
    pos = (sc.positions + rng.uniform(-0.004, 0.004, sc.positions.shape)).astype(np.float32)
    state = (pos, pos.copy(), np.zeros_like(pos))
    w, p = api.load_scene(sc)
    p.model.set_fast_math(fast)
    p.model.set_state(*state)
    PortCloth.set_portable_math(False)
    try:
        o = PortCloth.from_scene(sc)
        o.set_state(*state)
        o.set_tri_order(p.model.constraint_order(0)[0])
        o.set_bend_order(p.model.constraint_order(1)[0])
        p.step(sc.dt)
        o.step(sc.dt)
        g, c = p.model.positions(), o.positions()
    finally:
        PortCloth.set_portable_math(True)
    assert not np.array_equal(g, pos)
    assert _rel(g, c) <= REL, _rel(g, c)
    assert p.status() == 0
    o.close()
    p.free()
