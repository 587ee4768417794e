"""The trained warm start (solidcloth_b200/data/warmstart.npz: 2,000 drapes at
256 x 256) against the plain solver on a held-out 256 x 256 drape, through the C
ABI: Gauss-Seidel iterations a substep to the same update residual (the largest
particle displacement of an iteration, 1e-4 m, cap 200).

The learned warm start has no reference counterpart; it replaces iterations of
the Gauss-Seidel loop (Physics/ClothPBD.cpp:332-361). The bar is the scope's: at
least 2x fewer iterations at equal residual, here over a set of held-out drapes.
Both arms must reach the residual (below the cap), and the learned arm's final
constraint residual must not be worse than twice the plain arm's (the network
does not buy iterations with a worse state)."""
import numpy as np
import pytest

from solidcloth_b200 import learned
from solidcloth_b200.build import PKG

pytestmark = pytest.mark.gpu

CAP = 200
TOL = 1e-4        # metres


def _weights():
    z = np.load(PKG / "data" / "warmstart.npz")
    return z["params"].astype(np.float32), z["norm"].astype(np.float32), int(z["n"])


def test_trained_network_gain_on_held_out_256_drapes():
    """Eight held-out 256 x 256 drapes (learned.TEST_SEEDS: neither the training
    nor the output-scale calibration saw them): the gain varies from drape to
    drape, so the bar is on the set — median and aggregate (sum of plain over sum
    of learned iterations) iteration ratios of at least 2, no drape below 1.25 —
    with both arms at the residual on every drape and more vertex-substeps/s in
    total. The final constraint residual (max |C| over the FEM constraints, set
    by the few most strained triangles at the collider) must be no worse with the
    learned start than 1.5 times the plain arm's in the median over the drapes,
    and within 3 times on every drape."""
    params, norm, n_train = _weights()
    assert n_train == 256
    rows, plain_t, learned_t = [], 0.0, 0.0
    for seed in learned.TEST_SEEDS:
        assert seed >= 2000 and seed not in learned.CALIBRATION_SEEDS
        d = learned.drape_scene(seed, 256)
        r = learned.compare([d], params, norm, frames=3, skip=4, tol=TOL, max_iter=CAP)
        plain, warm = r["plain"], r["learned"]
        assert plain["status"] == 0 and warm["status"] == 0, (seed, r)
        assert plain["iterations_per_substep"] < CAP and warm["iterations_per_substep"] < CAP, (seed, r)
        rows.append({"seed": seed, "plain": plain["iterations_per_substep"], "learned": warm["iterations_per_substep"],
                     "residual_ratio": warm["constraint_residual_after"] / plain["constraint_residual_after"]})
        plain_t += plain["ms_per_frame"]
        learned_t += warm["ms_per_frame"]
    s = learned.summary(rows)
    assert s["median"] >= 2.0 and s["aggregate"] >= 2.0 and s["min"] >= 1.25, (s, rows)
    res = sorted(r["residual_ratio"] for r in rows)
    assert 0.5 * (res[3] + res[4]) <= 1.5 and res[-1] <= 3.0, rows
    assert learned_t < plain_t, (learned_t, plain_t)


def test_untrained_network_gives_no_gain():
    """Control: the same comparison with the correction scaled to zero runs the
    plain iteration count (the warm start's wiring adds nothing by itself)."""
    params, norm, _ = _weights()
    d = learned.drape_scene(30_000_002, 64, side=0.5)
    r = learned.compare([d], params, learned.scaled(norm, 0.0), frames=2, skip=2, tol=TOL, max_iter=CAP)
    assert abs(r["plain"]["iterations_per_substep"] - r["learned"]["iterations_per_substep"]) <= 0.5, r
