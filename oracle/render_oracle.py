"""CPU oracle of the headless cloth picture (test infrastructure only).

Restates, in numpy FP32, what solidcloth_b200/csrc/render.cu computes: the
demo's Phong program (Shaders/shader_phong_vertex.glsl:21-36 — world-space
position and normalised normal, clip position = view_proj * (p, 1);
shader_phong_geometry.glsl compute_distances() — window-space heights for the
wireframe; shader_phong_fragment.glsl:166-222 main() and :67-98 orennayar()).

The raster stage (projection, edge functions, barycentrics, NDC depth, the
order-preserving depth key and the nearest-then-lowest-index rule) keeps the
kernel's FP32 operation order, so the per-pixel (depth key << 32 | triangle)
words are compared bit for bit. Shading goes through acos/sin/tan/pow/exp2,
whose last bits differ between libraries, so colours are compared within a
tolerance written in the test.
"""
import numpy as np

F = np.float32
OREN_NAYAR, MONOCHROME, WIREFRAME = 2, 8, 16
EMPTY = np.uint64(0xFFFFFFFFFFFFFFFF)


def _project(vp, p):
    """window x, y, NDC z, clip w per vertex (rows); w <= 0 marks the vertex unusable"""
    m = vp.astype(F).reshape(16)
    px, py, pz = p[:, 0].astype(F), p[:, 1].astype(F), p[:, 2].astype(F)
    cx = m[0] * px + m[1] * py + m[2] * pz + m[3]
    cy = m[4] * px + m[5] * py + m[6] * pz + m[7]
    cz = m[8] * px + m[9] * py + m[10] * pz + m[11]
    cw = m[12] * px + m[13] * py + m[14] * pz + m[15]
    with np.errstate(divide="ignore", invalid="ignore"):
        iw = F(1) / cw
    return cx, cy, cz, cw, iw


def _window(cx, cy, cz, iw, width, height):
    x = (cx * iw + F(1)) * F(0.5) * F(width)
    y = (F(1) - cy * iw) * F(0.5) * F(height)
    z = cz * iw
    return x, y, z


def _edge(ax, ay, bx, by, px, py):
    return (bx - ax) * (py - ay) - (by - ay) * (px - ax)


def _depth_key(z):
    u = z.astype(F).view(np.uint32)
    return np.where(u & np.uint32(0x80000000), ~u, u | np.uint32(0x80000000)).astype(np.uint32)


def rasterise(vp, pos, tri, width, height):
    """(height, width) uint64 words: (depth key << 32 | triangle index), all ones where empty"""
    cx, cy, cz, cw, iw = _project(vp, pos)
    x, y, z = _window(cx, cy, cz, iw, width, height)
    zb = np.full(width * height, EMPTY, np.uint64)
    for t in range(tri.shape[0]):
        v = tri[t]
        if not np.all(cw[v] > 0):
            continue
        X, Y, Z = x[v], y[v], z[v]
        area = _edge(X[0], Y[0], X[1], Y[1], X[2], Y[2])
        if area == 0:
            continue
        # the kernel's float -> int conversion saturates; clamping first is the same
        lim = lambda v: float(np.clip(v, -2.0, 2.0 * max(width, height) + 2.0))
        x0 = max(0, int(np.floor(lim(min(X[0], min(X[1], X[2]))))))
        x1 = min(width - 1, int(np.ceil(lim(max(X[0], max(X[1], X[2]))))))
        y0 = max(0, int(np.floor(lim(min(Y[0], min(Y[1], Y[2]))))))
        y1 = min(height - 1, int(np.ceil(lim(max(Y[0], max(Y[1], Y[2]))))))
        if x1 < x0 or y1 < y0:
            continue
        ia = F(1) / area
        PX, PY = np.meshgrid(np.arange(x0, x1 + 1), np.arange(y0, y1 + 1))
        qx, qy = PX.astype(F) + F(0.5), PY.astype(F) + F(0.5)
        b0 = _edge(X[1], Y[1], X[2], Y[2], qx, qy) * ia
        b1 = _edge(X[2], Y[2], X[0], Y[0], qx, qy) * ia
        b2 = _edge(X[0], Y[0], X[1], Y[1], qx, qy) * ia
        zz = b0 * Z[0] + b1 * Z[1] + b2 * Z[2]
        ok = (b0 >= 0) & (b1 >= 0) & (b2 >= 0) & (zz >= -1) & (zz <= 1)
        if not ok.any():
            continue
        idx = (PY[ok] * width + PX[ok]).astype(np.int64)
        key = (_depth_key(zz[ok]).astype(np.uint64) << np.uint64(32)) | np.uint64(t)
        zb[idx] = np.minimum(zb[idx], key)
    return zb.reshape(height, width)


def _normalize(v):
    l = np.sqrt(((v[..., 0] * v[..., 0] + v[..., 1] * v[..., 1]) + v[..., 2] * v[..., 2]))
    return (F(1) / l)[..., None] * v


def _dot(a, b):
    return (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]


def _oren_nayar(p, n, light, eye, roughness=F(1.4)):
    L, N, V = _normalize(light - p), _normalize(n), _normalize(eye - p)
    acosVN, acosLN = np.arccos(_dot(V, N)), np.arccos(_dot(L, N))
    alpha, beta = np.maximum(acosVN, acosLN), np.minimum(acosVN, acosLN)
    gamma = _dot(V - _dot(V, N)[..., None] * N, L - _dot(L, N)[..., None] * N)
    r2 = roughness * roughness
    C1 = F(1) - F(0.5) * (r2 / (r2 + F(0.33)))
    C2 = F(0.45) * (r2 / (r2 + F(0.09)))
    C2 = np.where(gamma >= 0, C2 * np.sin(alpha), C2 * (np.sin(alpha) - np.power((F(2) * beta) / F(3.14167), F(3))))
    C3 = F(1) / F(8) * (r2 / (r2 + F(0.09))) * np.power((F(4) * alpha * beta) / (F(3.14167) * F(3.14167)), F(2))
    A = gamma * C2 * np.tan(beta)
    B = (F(1) - np.abs(gamma)) * C3 * np.tan((alpha + beta) / F(2))
    return np.minimum(np.maximum(F(0), _dot(N, L)) * (C1 + A + B), F(0.99))


def shade(vp, pos, nrm, tri, zbuf, width, height, params16):
    """(height, width, 4) float32 picture for the words `zbuf` (from rasterise)"""
    prm = np.asarray(params16, F)
    light, eye, kd, ks = prm[0:3], prm[3:6], prm[6:9], prm[9:12]
    shininess, flip, background, flags = prm[12], prm[13], prm[14], int(prm[15])
    out = np.zeros((height * width, 4), F)
    out[:, 3] = 1
    zb = zbuf.reshape(-1)
    hit = zb != EMPTY
    out[~hit, :3] = background
    pix = np.nonzero(hit)[0]
    if pix.size == 0:
        return out.reshape(height, width, 4)
    t = (zb[pix] & np.uint64(0xFFFFFFFF)).astype(np.int64)
    cx, cy, cz, cw, iw = _project(vp, pos)
    x, y, _ = _window(cx, cy, cz, iw, width, height)
    V3 = tri[t]                                   # (P, 3) vertex indices
    X, Y, W = x[V3], y[V3], cw[V3]
    qx = (pix % width).astype(F) + F(0.5)
    qy = (pix // width).astype(F) + F(0.5)
    ia = F(1) / _edge(X[:, 0], Y[:, 0], X[:, 1], Y[:, 1], X[:, 2], Y[:, 2])
    b = np.stack([_edge(X[:, 1], Y[:, 1], X[:, 2], Y[:, 2], qx, qy) * ia,
                  _edge(X[:, 2], Y[:, 2], X[:, 0], Y[:, 0], qx, qy) * ia,
                  _edge(X[:, 0], Y[:, 0], X[:, 1], Y[:, 1], qx, qy) * ia], 1)
    if flags & MONOCHROME:
        col = np.broadcast_to(kd, (pix.size, 3)).astype(F)
    else:
        wb = b / W
        s = (wb[:, 0] + wb[:, 1]) + wb[:, 2]
        P = np.zeros((pix.size, 3), F)
        N = np.zeros((pix.size, 3), F)
        for k in range(3):
            wk = (wb[:, k] / s)[:, None]
            P = P + wk * pos[V3[:, k]].astype(F)
            N = N + wk * _normalize(nrm[V3[:, k]].astype(F))
        Nf = flip * _normalize(N)
        L = _normalize(light - P)
        V = _normalize(eye - P)
        ambient = F(0.2)
        diffuse = np.maximum(_dot(L, Nf), F(0))
        spec = np.zeros(pix.size, F)
        if np.sqrt(_dot(ks, ks)) > 0:
            R = -L - (F(2) * _dot(Nf, -L))[:, None] * Nf
            sp = np.power(np.maximum(_dot(V, R), F(0)), shininess)
            spec = np.where(diffuse > 0, sp, F(0)).astype(F)
        if flags & OREN_NAYAR:
            sh = _oren_nayar(P, N, light, eye)
        else:
            sh = (ambient + diffuse) / (F(1) + ambient)
        col = sh[:, None] * kd + spec[:, None] * ks
    if flags & WIREFRAME:
        d = np.full(pix.size, np.inf, F)
        for k in range(3):
            a, c = (k + 1) % 3, (k + 2) % 3
            ux, uy = X[:, a] - X[:, k], Y[:, a] - Y[:, k]
            vx, vy = X[:, c] - X[:, k], Y[:, c] - Y[:, k]
            area = np.abs(ux * vy - uy * vx)
            h = area / np.sqrt((ux - vx) * (ux - vx) + (uy - vy) * (uy - vy))
            d = np.minimum(d, b[:, k] * h)
        line_width = F(1)
        d = np.where(d > F(0.5) * line_width + F(1), F(2), d)
        d = np.minimum(np.maximum(d - (F(0.5) * line_width - F(1)), F(0)), F(2))
        I = np.exp2(F(-2) * d * d)
        col = (F(1) - I)[:, None] * col
    out[pix, :3] = col
    return out.reshape(height, width, 4)
