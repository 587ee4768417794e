"""Learned warm start: data generation with the GPU solver, training with the
library's own kernels, and the plain-versus-learned comparison.

The network (12 -> 64 -> 64 -> 64 -> 3, GELU, BF16 weights on the tensor cores)
predicts, per particle, the correction the Gauss-Seidel loop will apply in a
substep (solved minus predicted position) from features available right after
the prediction. The library applies it before the loop; plain iterations then
continue until the residual target, so the plain solver still decides when a
substep is done. Everything runs on the GPU: samples come from the solver through
scSetSampleBuffers, gradients from scMlpGradients, updates from scMlpAdamStep.
"""
from __future__ import annotations

import os
import time
from dataclasses import dataclass

import numpy as np

from . import api, scenes

NPARAM = 9347
NNORM = 27
IN, OUT = 12, 3


def init_params(seed: int = 0) -> np.ndarray:
    """He-style weights, zero biases, zero output layer (no correction at start)."""
    rng = np.random.default_rng(seed)
    shapes = [(64, 12), (64,), (64, 64), (64,), (64, 64), (64,), (3, 64), (3,)]
    parts = []
    for k, shp in enumerate(shapes):
        if len(shp) == 1 or k == 6:
            parts.append(np.zeros(shp, np.float32))
        else:
            parts.append((rng.standard_normal(shp) * np.sqrt(2.0 / shp[1])).astype(np.float32))
    return np.concatenate([q.ravel() for q in parts]).astype(np.float32)


def drape_scene(seed: int, n: int = 256, side: float = 1.5, ccd: bool = True) -> scenes.Scene:
    """A random drape of the 256 x 256, 1.5 m self-colliding cloth: sphere SDF
    (centre within 0.15 m of the cloth's axis, radius 0.2-0.4 m, 64^3 samples)
    under the flat cloth rotated about the vertical by a random angle and released
    3 cm above the sphere's top; no pins."""
    rng = np.random.default_rng(seed)
    r = float(rng.uniform(0.2, 0.4))
    cx, cz = (float(v) for v in rng.uniform(-0.15, 0.15, 2))
    angle = float(rng.uniform(0.0, np.pi))
    p = scenes.Params(thickness=0.005, tolerance=0.005, friction=0.3, iterations=20, substeps=8,
                      flags=scenes.CF_VERTICES)
    height = r + 0.03
    s = scenes.make_grid_scene(f"drape_{n}_s{seed}", n, side, height, p, seed=seed, frames=60)
    c, sn = np.cos(angle), np.sin(angle)
    rot = np.array([[c, 0, -sn], [0, 1, 0], [sn, 0, c]], np.float32)
    centre = s.positions.mean(0)
    s.positions = ((s.positions - centre) @ rot.T + centre).astype(np.float32)
    s.sdfs.append(scenes.sphere_sdf((cx, 0.0, cz), r, 63, 0.1))
    s.ccd = ccd
    return s


@dataclass
class Dataset:
    X: "object"       # torch float32 (S, 12) on the GPU
    T: "object"       # torch float32 (S, 3)
    drapes: int
    seconds: float


def generate(num_drapes: int, n: int = 256, per_batch: int = 32, skip_frames: int = 4, record_frames: int = 3,
             keep_every: int = 128, tol: float = 1e-4, max_iter: int = 100, seed0: int = 0, log=None) -> Dataset:
    """Simulate `num_drapes` drapes with the plain solver (update residual target
    `tol` in metres, at most `max_iter` iterations a substep) in batches, and keep
    every `keep_every`-th particle's (features, correction) of every substep of
    the recorded frames."""
    import torch
    t0 = time.time()
    xs, ts = [], []
    for b0 in range(0, num_drapes, per_batch):
        tb = time.time()
        ds = [drape_scene(seed0 + k, n) for k in range(b0, min(num_drapes, b0 + per_batch))]
        b = api.load_batch(ds)
        tl = time.time()
        b.model.set_fast_math(True)
        b.model.set_residual_target(tol, max_iter, metres=True)
        N = sum(d.num_vertices for d in ds)
        sub = ds[0].params.substeps
        for _ in range(skip_frames):
            b.step(ds[0].dt)
        F = torch.zeros((sub, N, IN), device="cuda")
        Tg = torch.zeros((sub, N, OUT), device="cuda")
        b.model.set_sample_buffers(F.data_ptr(), Tg.data_ptr())
        for f in range(record_frames):
            b.step(ds[0].dt)
            b.synchronize()
            sel = torch.arange((f * 7) % keep_every, N, keep_every, device="cuda")
            xs.append(F[:, sel].reshape(-1, IN).clone())
            ts.append(Tg[:, sel].reshape(-1, OUT).clone())
        b.model.set_sample_buffers(0, 0)
        b.free()
        if log:
            log(f"batch {b0 // per_batch}: set-up {tl - tb:.1f} s, frames {time.time() - tl:.1f} s")
    torch.cuda.synchronize()
    return Dataset(torch.cat(xs), torch.cat(ts), num_drapes, time.time() - t0)


def fit_norm(X, T) -> np.ndarray:
    """feature mean and 1/std (std floored), output scale = target std per axis"""
    mean = X.mean(0).cpu().numpy()
    std = X.std(0).cpu().numpy()
    std = np.where(std > 1e-6, std, 1.0)
    tstd = T.std(0).cpu().numpy()
    tstd = np.where(tstd > 1e-9, tstd, 1e-6)
    return np.concatenate([mean, 1.0 / std, tstd]).astype(np.float32)


def train(X, T, norm: np.ndarray, epochs: int = 20, batch: int = 65536, lr: float = 2e-3, seed: int = 0,
          params: np.ndarray | None = None, log=None):
    """Adam on mean((MLP(X) - T / scale)^2) with the library's kernels; returns
    (params, per-epoch mean losses)."""
    import torch
    lib = api.lib()
    p = torch.from_numpy(params if params is not None else init_params(seed)).cuda()
    m = torch.zeros(NPARAM, device="cuda")
    v = torch.zeros(NPARAM, device="cuda")
    g = torch.zeros(NPARAM, device="cuda")
    loss = torch.zeros(1, device="cuda")
    dn = torch.from_numpy(norm).cuda()
    S = X.shape[0]
    gen = torch.Generator(device="cuda").manual_seed(seed)
    step = 0
    history = []
    for ep in range(epochs):
        perm = torch.randperm(S, device="cuda", generator=gen)
        tot, cnt = 0.0, 0
        losses = []
        for k in range(0, S, batch):
            idx = perm[k:k + batch]
            xb, tb = X[idx].contiguous(), T[idx].contiguous()
            rc = lib.scMlpGradients(xb.data_ptr(), tb.data_ptr(), xb.shape[0], p.data_ptr(), dn.data_ptr(),
                                    g.data_ptr(), loss.data_ptr(), None)
            if rc != 0:
                raise RuntimeError(f"scMlpGradients: {rc}")
            step += 1
            lib.scMlpAdamStep(p.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), step, lr, None)
            losses.append(loss.clone())
        ep_loss = float(torch.stack(losses).mean().item())
        history.append(ep_loss)
        if log:
            log(f"epoch {ep}: loss {ep_loss:.4f}")
    return p.cpu().numpy(), history


def predict(X, params: np.ndarray, norm: np.ndarray):
    import torch
    Y = torch.zeros((X.shape[0], OUT), device="cuda")
    dp, dn = torch.from_numpy(params).cuda(), torch.from_numpy(norm).cuda()   # alive until the kernel ran
    rc = api.lib().scMlpForward(X.data_ptr(), X.shape[0], dp.data_ptr(), dn.data_ptr(), Y.data_ptr(), None)
    torch.cuda.synchronize()
    if rc != 0:
        raise RuntimeError(f"scMlpForward: {rc}")
    return Y


def compare(drapes, params: np.ndarray | None, norm: np.ndarray | None, frames: int = 6, skip: int = 4,
            tol: float = 1e-4, max_iter: int = 200, fast: bool = True):
    """Plain versus learned on the same drapes (a batch): Gauss-Seidel iterations a
    substep to reach the update residual target (the largest particle
    displacement of an iteration, in metres), and device-timed
    vertex-substeps/s over the measured frames (after `skip` untimed frames).
    constraint_residual_after is max |C| over the FEM constraints after the last
    frame (scGetResidual), a check that both arms end in states of equal quality.
    Both arms run one fixed solver kernel (the cluster solver for one drape, the
    grid solver's first variant for a batch) rather than the autotuner's choice:
    in the fast build the solvers agree only within the projection tolerance,
    and iteration counts to a max-norm residual amplify such differences, so a
    timing-dependent choice would make the counts differ from run to run."""
    import torch
    out = {}
    for label, warm in (("plain", False), ("learned", True)):
        b = api.load_batch(drapes) if len(drapes) > 1 else api.load_scene(drapes[0])[1]
        b.model.set_fast_math(fast)
        if len(drapes) > 1:
            b.model.set_grid_solver(0, 1)
        else:
            b.model.set_cluster_variant(0)
        b.model.set_residual_target(tol, max_iter, metres=True)
        if warm:
            b.model.set_warm_start(params, norm)
        dt = drapes[0].dt
        for _ in range(skip):
            b.step(dt)
        b.synchronize()
        b.model.iteration_total()
        st = torch.cuda.ExternalStream(b.cuda_stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(frames):
            b.step(dt)
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        its = b.model.iteration_total()
        sub = drapes[0].params.substeps * frames
        N = sum(d.num_vertices for d in drapes)
        out[label] = {"iterations_per_substep": its / sub, "vertex_substeps_per_s": N * sub / (ms * 1e-3),
                      "ms_per_frame": ms / frames, "constraint_residual_after": b.model.residual(), "status": b.status()}
        b.free()
    return out


def scaled(norm: np.ndarray, alpha: float) -> np.ndarray:
    """the same network with its correction multiplied by alpha"""
    out = norm.copy()
    out[2 * IN:] *= alpha
    return out


# Drape seeds of the three disjoint sets: training 0 .. drapes-1, calibration of
# the output scale, and the held-out test drapes the GPU test and the benchmark
# report (neither of the others ever sees them).
CALIBRATION_SEEDS = (30_000_000, 30_000_001, 20_000_001, 40_000_000, 10_256_000, 50_000_000, 50_000_001)
TEST_SEEDS = tuple(range(60_000_000, 60_000_008))


def calibrate(params: np.ndarray, norm: np.ndarray, seeds=CALIBRATION_SEEDS, alphas=(1.0, 0.75, 0.5), n: int = 256,
              tol: float = 1e-4, max_iter: int = 200):
    """Output scale of the correction: the network is fitted to the mean
    correction, and where it is unsure a shorter step serves the iterations that
    follow better. Each alpha runs the plain-versus-learned comparison on the
    calibration drapes; the one with the largest aggregate iteration ratio (sum of
    plain over sum of learned iterations) wins. Returns (alpha, per-alpha rows)."""
    rows = {}
    for a in alphas:
        rs = []
        for sd in seeds:
            r = compare([drape_scene(sd, n)], params, scaled(norm, a), frames=3, skip=4, tol=tol, max_iter=max_iter)
            rs.append({"seed": sd, "plain": r["plain"]["iterations_per_substep"],
                       "learned": r["learned"]["iterations_per_substep"]})
        rows[a] = rs
    agg = {a: sum(x["plain"] for x in rs) / sum(x["learned"] for x in rs) for a, rs in rows.items()}
    return max(agg, key=agg.get), rows


def summary(rows):
    """iteration ratios of plain-versus-learned rows: per drape, median, aggregate"""
    ratios = sorted(r["plain"] / r["learned"] for r in rows)
    k = len(ratios)
    med = ratios[k // 2] if k % 2 else 0.5 * (ratios[k // 2 - 1] + ratios[k // 2])
    return {"ratios": ratios, "median": med, "min": ratios[0],
            "aggregate": sum(r["plain"] for r in rows) / sum(r["learned"] for r in rows)}


def main(argv=None):
    """Generate, train, evaluate; writes the parameters (npz) and a JSON report.

    python -m solidcloth_b200.learned --drapes 2000 --out solidcloth_b200/data/warmstart.npz
    """
    import argparse
    import json
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--drapes", type=int, default=2000)
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--per-batch", type=int, default=32)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--tol", type=float, default=1e-4)
    ap.add_argument("--max-iter", type=int, default=100, help="iteration cap of the data generation")
    ap.add_argument("--eval-max-iter", type=int, default=200, help="iteration cap of the evaluation")
    ap.add_argument("--eval", type=int, default=4, help="held-out drapes per evaluation size")
    ap.add_argument("--eval-n", type=int, nargs="*", default=[256])
    ap.add_argument("--out", default="solidcloth_b200/data/warmstart.npz")
    ap.add_argument("--report", default=None)
    ap.add_argument("--calibrate", action="store_true",
                    help="only calibrate the output scale of the weights in --out (rewrites it and the report's "
                         "calibration entry)")
    a = ap.parse_args(argv)
    if a.calibrate:
        z = dict(np.load(a.out))
        alpha, rows = calibrate(z["params"].astype(np.float32), z["norm"].astype(np.float32))
        z["norm"] = scaled(z["norm"].astype(np.float32), alpha)
        z["output_scale"] = np.float32(float(z.get("output_scale", 1.0)) * alpha)
        np.savez(a.out, **z)
        entry = {"alpha": alpha, "seeds": list(CALIBRATION_SEEDS),
                 "per_alpha": {str(k): dict(summary(v), rows=v) for k, v in rows.items()}}
        if a.report:
            rep = json.load(open(a.report)) if os.path.exists(a.report) else {}
            rep["calibration"] = entry
            with open(a.report, "w") as f:
                json.dump(rep, f, indent=1)
        print(json.dumps(entry))
        return entry
    torch.cuda.init()
    ds = generate(a.drapes, n=a.n, per_batch=a.per_batch, tol=a.tol, max_iter=a.max_iter,
                  log=lambda m: print(m, flush=True))
    print(f"samples {ds.X.shape[0]} from {ds.drapes} drapes in {ds.seconds:.1f} s", flush=True)
    norm = fit_norm(ds.X, ds.T)
    t0 = time.time()
    params, hist = train(ds.X, ds.T, norm, epochs=a.epochs, log=lambda m: print(m, flush=True))
    train_s = time.time() - t0
    np.savez(a.out, params=params, norm=norm, drapes=a.drapes, n=a.n, tol=a.tol, loss=np.array(hist))
    report = {"drapes": a.drapes, "n_train": a.n, "samples": int(ds.X.shape[0]), "generate_s": ds.seconds,
              "train_s": train_s, "loss_per_epoch": hist, "tol": a.tol, "residual_unit": "m", "max_iter": a.max_iter,
              "eval_max_iter": a.eval_max_iter, "eval": {}}
    for n in a.eval_n:
        rows = []
        for k in range(a.eval):
            d = drape_scene(10_000_000 + 1000 * n + k, n)
            r = compare([d], params, norm, frames=3, skip=4, tol=a.tol, max_iter=a.eval_max_iter)
            rows.append(r)
            print(n, k, json.dumps(r), flush=True)
        report["eval"][str(n)] = rows
    if a.report:
        with open(a.report, "w") as f:
            json.dump(report, f, indent=1)
    return report


if __name__ == "__main__":
    main()
