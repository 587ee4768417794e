"""Warm-start network kernels (tcgen05 tensor-core forward and backward with
tensor-memory accumulators, Adam) against the CPU oracle oracle/mlp_oracle.py,
and the warm start's wiring into the step."""
import numpy as np
import pytest

from oracle import mlp_oracle as M
from solidcloth_b200 import scenes

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def _case(seed=0, S=3000):
    rng = np.random.default_rng(seed)
    p = M.init_params(seed)
    d = M.unpack(p)
    d["W4"][:] = rng.standard_normal(d["W4"].shape).astype(np.float32) * 0.2
    d["b1"][:] = rng.standard_normal(64).astype(np.float32) * 0.1
    p = M.pack(d)
    X = rng.standard_normal((S, M.IN)).astype(np.float32) * 2.0
    T = rng.standard_normal((S, M.OUT)).astype(np.float32) * 1e-3
    norm = np.concatenate([rng.standard_normal(M.IN) * 0.1, 0.5 + rng.random(M.IN), [1e-3, 2e-3, 1e-3]]).astype(np.float32)
    return p, norm, X, T


def test_forward_matches_oracle():
    """BF16 tensor-core forward vs the oracle's BF16-rounded forward: agreement to
    1 % of the output range (FP32 accumulation order differs)."""
    import torch
    from solidcloth_b200.api import lib
    p, norm, X, T = _case()
    Y = torch.zeros((X.shape[0], 3), device="cuda")
    dX, dp, dn = _dev(X), _dev(p), _dev(norm)     # kept alive while the kernel runs
    rc = lib().scMlpForward(dX.data_ptr(), X.shape[0], dp.data_ptr(), dn.data_ptr(), Y.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == 0
    want = M.predict(p, norm, X)
    got = Y.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-2 * np.abs(want).max(), float(np.abs(got - want).max())


def test_gradients_match_oracle():
    """GPU gradients (BF16 operands, FP32 accumulation on the tensor cores) vs the
    oracle's (BF16 forward, FP32 backward): relative L2 error below 2 %, loss
    within 1 %. S = 3000 is not a multiple of the 128-row tile, so the padded
    rows of the last tile are exercised."""
    import torch
    from solidcloth_b200.api import lib
    p, norm, X, T = _case(1)
    g = torch.zeros(M.NPARAM, device="cuda")
    loss = torch.zeros(1, device="cuda")
    dX, dT, dp, dn = _dev(X), _dev(T), _dev(p), _dev(norm)
    rc = lib().scMlpGradients(dX.data_ptr(), dT.data_ptr(), X.shape[0], dp.data_ptr(),
                              dn.data_ptr(), g.data_ptr(), loss.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == 0
    gw, lw = M.grad(p, norm, X, T)
    gg = g.cpu().numpy()
    assert np.linalg.norm(gg - gw) / np.linalg.norm(gw) < 2e-2, np.linalg.norm(gg - gw) / np.linalg.norm(gw)
    assert abs(float(loss.item()) - lw) <= 1e-2 * lw


def test_adam_step_matches_oracle():
    import torch
    from solidcloth_b200.api import lib
    rng = np.random.default_rng(2)
    p = rng.standard_normal(M.NPARAM).astype(np.float32)
    g = rng.standard_normal(M.NPARAM).astype(np.float32)
    m = np.zeros(M.NPARAM, np.float32)
    v = np.zeros(M.NPARAM, np.float32)
    dp, dm, dv = _dev(p), _dev(m), _dev(v)
    dg = _dev(g)
    for step in (1, 2, 3):
        assert lib().scMlpAdamStep(dp.data_ptr(), dg.data_ptr(), dm.data_ptr(), dv.data_ptr(), step, 1e-3, None) == 0
        M.adam(p, g, m, v, step, 1e-3)
    torch.cuda.synchronize()
    assert np.allclose(dp.cpu().numpy(), p, rtol=1e-5, atol=1e-6)


def test_training_reduces_loss():
    """The project's own kernels fit a smooth synthetic target: 300 Adam steps
    reduce the loss at least tenfold."""
    import torch
    from solidcloth_b200.api import lib
    rng = np.random.default_rng(4)
    S = 8192
    X = rng.standard_normal((S, M.IN)).astype(np.float32)
    T = (np.stack([np.tanh(X[:, 0]) * X[:, 1], np.sin(X[:, 2]), 0.5 * X[:, 3] * X[:, 4]], 1) * 1e-3).astype(np.float32)
    norm = np.concatenate([np.zeros(M.IN), np.ones(M.IN), [1e-3] * 3]).astype(np.float32)
    p = _dev(M.init_params(5))
    m = torch.zeros(M.NPARAM, device="cuda")
    v = torch.zeros(M.NPARAM, device="cuda")
    g = torch.zeros(M.NPARAM, device="cuda")
    loss = torch.zeros(1, device="cuda")
    dX, dT, dn = _dev(X), _dev(T), _dev(norm)
    first = None
    for step in range(1, 301):
        assert lib().scMlpGradients(dX.data_ptr(), dT.data_ptr(), S, p.data_ptr(), dn.data_ptr(), g.data_ptr(), loss.data_ptr(), None) == 0
        if first is None:
            torch.cuda.synchronize()
            first = float(loss.item())
        assert lib().scMlpAdamStep(p.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), step, 3e-3, None) == 0
    lib().scMlpGradients(dX.data_ptr(), dT.data_ptr(), S, p.data_ptr(), dn.data_ptr(), g.data_ptr(), loss.data_ptr(), None)
    torch.cuda.synchronize()
    assert float(loss.item()) < 0.1 * first, (first, float(loss.item()))


def _flat_scene():
    p = scenes.Params(thickness=0.005, tolerance=0.005, iterations=4, substeps=2, flags=scenes.CF_VERTICES)
    sc = scenes.make_grid_scene("flat_8", 8, 0.2, 0.25, p)
    sc.positions = scenes.grid_positions(8, sc.inc, sc.offset).astype(np.float32)   # exact rest shape
    sc.sdfs.append(scenes.sphere_sdf((0.0, 0.0, 0.0), 0.2, 31, 0.1))
    return sc


def test_recorded_features_match_numpy():
    """Features recorded after the prediction equal a numpy restatement of their
    definition on the recorded predicted positions."""
    import torch
    from solidcloth_b200 import api
    sc = _flat_scene()
    sc.positions = (sc.positions + np.random.default_rng(0).uniform(-2e-3, 2e-3, sc.positions.shape)).astype(np.float32)
    w, p = api.load_scene(sc)
    n = sc.num_vertices
    F = torch.zeros((sc.params.substeps, n, 12), device="cuda")
    Tg = torch.zeros((sc.params.substeps, n, 3), device="cuda")
    p.model.set_sample_buffers(F.data_ptr(), Tg.data_ptr())
    prev0 = p.model.positions()
    p.step(sc.dt)
    f = F.cpu().numpy()[0]
    h = sc.dt / sc.params.substeps
    # substep 0: prev = start positions; predicted = prev + h v with v = h g
    assert np.allclose(f[:, 3:6], np.array([0, -9.8 * h, 0], np.float32), atol=1e-6)
    assert np.allclose(f[:, 0:3], f[:, 3:6] * h, atol=1e-7)
    xp = prev0 + f[:, 0:3]
    edges = p.model.edges()
    strain = np.zeros(n)
    cnt = np.zeros(n)
    # rest lengths from the grid layout (the uv parameterisation)
    grid = scenes.grid_positions(8, sc.inc, sc.offset)
    for (a, b2, _, _) in edges:
        l0 = np.linalg.norm(grid[a] - grid[b2])
        s = np.linalg.norm(xp[a] - xp[b2]) / l0 - 1
        strain[a] += s; strain[b2] += s; cnt[a] += 1; cnt[b2] += 1
    assert np.allclose(f[:, 6], strain / cnt, atol=1e-5)
    d = np.linalg.norm(xp, axis=1) - 0.2
    assert np.allclose(f[:, 10], np.clip(d, -1, 1), atol=2e-3)     # 32^3 SDF sampling
    assert np.all(f[:, 11] == 0.0)                                  # no earlier substep
    # substep 1's twelfth feature: substep 0's correction along the normal
    f1 = F.cpu().numpy()[1]
    t0 = Tg.cpu().numpy()[0]
    assert np.allclose(f1[:, 11], np.sum(t0 * f[:, 7:10], axis=1), atol=1e-8)
    nrm = np.linalg.norm(f[:, 7:10], axis=1)
    assert np.allclose(nrm, 1.0, atol=1e-5)
    p.free()


def test_warm_start_adds_the_network_output():
    """A network with zero weights and output bias b moves every free particle of
    a rigidly falling flat cloth by b x scale; the rigid motion leaves every FEM
    and bend constraint satisfied, so the step's result is the plain result
    shifted by that correction."""
    from solidcloth_b200 import api
    sc = _flat_scene()
    sc.sdfs.clear()
    sc.params.flags = 0
    res = []
    for warm in (False, True):
        w, p = api.load_scene(sc)
        if warm:
            prm = np.zeros(M.NPARAM, np.float32)
            prm[M.NPARAM - 3:] = [1.0, -2.0, 0.5]
            norm = np.concatenate([np.zeros(12), np.ones(12), [1e-3, 1e-3, 1e-3]]).astype(np.float32)
            p.model.set_warm_start(prm, norm)
        p.step(sc.dt)
        res.append(p.model.positions())
        p.free()
    # each substep adds s; its velocity carries every earlier s into the next
    # prediction: after n substeps the shift is n (n + 1) / 2 s
    n = sc.params.substeps
    shift = np.array([1e-3, -2e-3, 0.5e-3], np.float32) * (n * (n + 1) / 2)
    assert np.allclose(res[1] - res[0], shift, atol=2e-6)
