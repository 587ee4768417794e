"""The warm-start network's CPU oracle pinned by finite differences (CPU only)."""
import numpy as np

from oracle import mlp_oracle as M


def _case(seed=0, S=40):
    rng = np.random.default_rng(seed)
    p = M.init_params(seed)
    p[M.NPARAM - 195:M.NPARAM - 3] = rng.standard_normal(192).astype(np.float32) * 0.1   # W4 non-zero
    X = rng.standard_normal((S, M.IN)).astype(np.float32)
    T = rng.standard_normal((S, M.OUT)).astype(np.float32) * 1e-3
    norm = np.concatenate([rng.standard_normal(M.IN) * 0.1, 1.0 + rng.random(M.IN), [1e-3, 2e-3, 1e-3]]).astype(np.float32)
    return p, norm, X, T


def test_layout():
    assert M.NPARAM == 9347 and M.NNORM == 27
    p = M.init_params(1)
    assert np.array_equal(M.pack(M.unpack(p)), p)


def test_gradient_matches_finite_differences():
    """Central differences of the FP32 network (float64 loss) against the
    analytic gradient, on every bias and a sample of weights: relative error
    below 2e-2 per entry where the gradient is not tiny, 1e-2 overall."""
    p, norm, X, T = _case()
    g, _ = M.grad_fp32(p, norm, X, T)
    rng = np.random.default_rng(3)
    idx = np.unique(np.concatenate([rng.choice(M.NPARAM, 300, replace=False),
                                    np.arange(768, 832), np.arange(M.NPARAM - 3, M.NPARAM)]))
    fd = np.zeros(len(idx))
    for k, j in enumerate(idx):
        h = 1e-2 * max(1.0, abs(float(p[j])))
        pp = p.astype(np.float64).copy()
        pp[j] += h
        lp = M.loss(pp.astype(np.float32), norm, X, T, rounded=False)
        pp[j] -= 2 * h
        lm = M.loss(pp.astype(np.float32), norm, X, T, rounded=False)
        fd[k] = (lp - lm) / (2 * h)
    ga = g[idx].astype(np.float64)
    big = np.abs(ga) > 1e-3 * np.abs(ga).max()
    rel = np.abs(fd - ga)[big] / np.abs(ga)[big]
    assert np.median(rel) < 1e-2, np.median(rel)
    assert np.linalg.norm(fd - ga) / np.linalg.norm(ga) < 2e-2


def test_bf16_rounding():
    # spacing at 1 is 2^-7: 1 + 2^-8 ties to even (1), 1 + 3 2^-8 ties to even (1 + 2^-6)
    x = np.array([1.0, 1.00390625, 1.01171875, 1.005859375, -3.0e-5, 65504.0], np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.015625 and r[3] == 1.0078125
    assert np.all(np.abs(r - x) <= np.abs(x) * 2 ** -8)
