"""CPU oracle of the learned warm start's network (test infrastructure only).

The network has no counterpart in the reference: this file is the checker for
the library's MLP kernels (solidcloth_b200/csrc/mlp_kernels.cuh). It restates,
in numpy FP32:

* the forward pass as the GPU runs it: inputs normalised in FP32, then every
  matrix operand (weights and activations) rounded to BF16 (round to nearest
  even), FP32 accumulation starting from the bias, GELU (tanh form) in FP32;
* the backward pass as the GPU runs it: FP32 master weights, FP32
  pre-activations, the mean of the squared error over S x 3 outputs against
  target / output scale;
* the same network without BF16 rounding, whose gradient `grad_fp32` is checked
  against central finite differences (tests/test_mlp_oracle.py), which pins the
  backward formulas.

Parameter layout (FP32 vector of 9347): W1[64][12], b1[64], W2[64][64], b2[64],
W3[64][64], b3[64], W4[3][64], b4[3]; norm (27): feature mean, 1/std, output scale.
"""
import numpy as np

IN, H, OUT = 12, 64, 3
SHAPES = [("W1", (H, IN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)),
          ("W3", (H, H)), ("b3", (H,)), ("W4", (OUT, H)), ("b4", (OUT,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)
NNORM = 2 * IN + OUT
C0 = np.float32(0.7978845608028654)


def unpack(p):
    out, k = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = p[k:k + n].reshape(shp)
        k += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float32).ravel() for name, _ in SHAPES]).astype(np.float32)


def init_params(seed=0):
    """He-style initialisation; the last layer starts at zero (no correction)."""
    rng = np.random.default_rng(seed)
    d = {}
    for name, shp in SHAPES:
        if name.startswith("b"):
            d[name] = np.zeros(shp, np.float32)
        else:
            d[name] = (rng.standard_normal(shp) * np.sqrt(2.0 / shp[1])).astype(np.float32)
    d["W4"][:] = 0.0
    return pack(d)


def bf16(x):
    """round FP32 to the nearest BF16 (ties to even), returned as FP32"""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def gelu(x):
    x = x.astype(np.float32)
    return (np.float32(0.5) * x * (np.float32(1) + np.tanh(C0 * (x + np.float32(0.044715) * x * x * x)))).astype(np.float32)


def gelu_grad(x):
    x = x.astype(np.float32)
    t = np.tanh(C0 * (x + np.float32(0.044715) * x * x * x))
    return (0.5 * (1 + t) + 0.5 * x * (1 - t * t) * C0 * (1 + 3 * np.float32(0.044715) * x * x)).astype(np.float32)


def normalise(X, norm):
    return ((X.astype(np.float32) - norm[:IN]) * norm[IN:2 * IN]).astype(np.float32)


def forward(p, norm, X, rounded=True):
    """network output (before the output scale) and the hidden pre-activations"""
    d = unpack(p)
    r = bf16 if rounded else (lambda a: a.astype(np.float32))
    x = normalise(X, norm)
    z1 = (r(x) @ r(d["W1"]).T + d["b1"]).astype(np.float32)
    z2 = (r(gelu(z1)) @ r(d["W2"]).T + d["b2"]).astype(np.float32)
    z3 = (r(gelu(z2)) @ r(d["W3"]).T + d["b3"]).astype(np.float32)
    y = (r(gelu(z3)) @ r(d["W4"]).T + d["b4"]).astype(np.float32)
    return y, (x, z1, z2, z3)


def predict(p, norm, X, rounded=True):
    """corrections = output x output scale (what the warm start adds)"""
    return forward(p, norm, X, rounded)[0] * norm[2 * IN:]


def loss(p, norm, X, T, rounded=True):
    y, _ = forward(p, norm, X, rounded)
    e = y - T / norm[2 * IN:]
    return float(np.mean(e.astype(np.float64) ** 2))


def grad(p, norm, X, T, rounded=True):
    """(gradient vector, loss) of mean((MLP(X) - T / scale)^2), as the GPU computes it"""
    d = unpack(p)
    y, (x, z1, z2, z3) = forward(p, norm, X, rounded)
    S = X.shape[0]
    e = (y - T / norm[2 * IN:]).astype(np.float32)
    dy = (2.0 * e / (S * OUT)).astype(np.float32)
    g = {}
    h3, h2, h1 = gelu(z3), gelu(z2), gelu(z1)
    g["W4"] = dy.T @ h3
    g["b4"] = dy.sum(0)
    dz3 = (dy @ d["W4"]) * gelu_grad(z3)
    g["W3"] = dz3.T @ h2
    g["b3"] = dz3.sum(0)
    dz2 = (dz3 @ d["W3"]) * gelu_grad(z2)
    g["W2"] = dz2.T @ h1
    g["b2"] = dz2.sum(0)
    dz1 = (dz2 @ d["W2"]) * gelu_grad(z1)
    g["W1"] = dz1.T @ x
    g["b1"] = dz1.sum(0)
    return pack(g), float(np.mean(e.astype(np.float64) ** 2))


def grad_fp32(p, norm, X, T):
    return grad(p, norm, X, T, rounded=False)


def adam(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """one Adam step (Kingma & Ba 2015), in place; returns p"""
    m[:] = b1 * m + (1 - b1) * g
    v[:] = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    p -= (lr * mh / (np.sqrt(vh) + eps)).astype(np.float32)
    return p
