"""Headless pictures of a cloth: camera matrices with the demo's conventions and
an image writer, around ClothPatch.render (scRenderCloth, CUDA rasteriser of the
demo's Phong program).

The matrices follow Math::Matrix4::Perspective and Math::Matrix4::LookAt
(Math/Matrix4.h:198-208, 357-380) — OpenGL clip space, right-handed eye space
looking down -z — and are returned row-major for column vectors, the layout
scRenderCloth takes. The demo's default projection is Graphics3D::Resize's
Perspective(fov, w / h, n, f) (Graphics3D/Graphics3DGLS.cpp:139-145).

    python -m solidcloth_b200.render --out cloth.ppm
"""
from __future__ import annotations

import numpy as np


def perspective(fov_deg: float, aspect: float, near: float, far: float) -> np.ndarray:
    d = 1.0 / np.tan(np.radians(fov_deg) * 0.5)
    P = np.zeros((4, 4), np.float32)
    P[0, 0] = d / aspect
    P[1, 1] = d
    P[2, 2] = (near + far) / (near - far)
    P[2, 3] = 2 * near * far / (near - far)
    P[3, 2] = -1.0
    return P


def look_at(eye, center, up=(0.0, 1.0, 0.0)) -> np.ndarray:
    eye, center, up = (np.asarray(v, np.float64) for v in (eye, center, up))
    z = eye - center
    z /= np.linalg.norm(z)
    x = np.cross(up, z)
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    V = np.eye(4)
    V[0, :3], V[1, :3], V[2, :3] = x, y, z
    V[:3, 3] = -V[:3, :3] @ eye
    return V.astype(np.float32)


def view_proj(eye, center, width: int, height: int, fov_deg: float = 60.0, near: float = 0.05,
              far: float = 100.0, up=(0.0, 1.0, 0.0)) -> np.ndarray:
    return (perspective(fov_deg, width / height, near, far) @ look_at(eye, center, up)).astype(np.float32)


def frame(positions: np.ndarray, direction=(0.6, 0.8, 1.0), fov_deg: float = 60.0):
    """(eye, center) that fit the points' bounding sphere in the view from `direction`"""
    p = np.asarray(positions, np.float64).reshape(-1, 3)
    lo, hi = p.min(0), p.max(0)
    c = 0.5 * (lo + hi)
    r = max(0.5 * np.linalg.norm(hi - lo), 1e-3)
    d = np.asarray(direction, np.float64)
    d /= np.linalg.norm(d)
    dist = r / np.sin(np.radians(fov_deg) * 0.5) * 1.1
    return tuple(c + dist * d), tuple(c)


def write_ppm(path, rgba) -> None:
    """binary PPM (P6) of an (H, W, >=3) float image in [0, 1], row 0 at the top"""
    img = rgba.detach().cpu().numpy() if hasattr(rgba, "detach") else np.asarray(rgba)
    rgb = (np.clip(img[..., :3], 0.0, 1.0) * 255.0 + 0.5).astype(np.uint8)
    h, w = rgb.shape[:2]
    with open(path, "wb") as f:
        f.write(b"P6\n%d %d\n255\n" % (w, h))
        f.write(rgb.tobytes())


def main(argv=None):
    """Drape the sphere scene (an n x n cloth) for a number of frames and write one picture."""
    import argparse
    from . import api, scenes
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--frames", type=int, default=60)
    ap.add_argument("--width", type=int, default=640)
    ap.add_argument("--height", type=int, default=480)
    ap.add_argument("--flags", type=int, default=0)
    ap.add_argument("--out", default="cloth.ppm")
    a = ap.parse_args(argv)
    scene = scenes.cfg1(n=a.n)
    world, patch = api.load_scene(scene)
    for _ in range(a.frames):
        patch.step(scene.dt)
    patch.synchronize()
    patch.update_mesh()
    pos, nrm, _ = patch.mesh_buffers()
    eye, center = frame(pos)
    vp = view_proj(eye, center, a.width, a.height)
    # the demo's flip-normals switch: show the side whose normals face the eye
    flip = 1.0 if float(nrm.mean(0) @ (np.subtract(eye, center))) >= 0 else -1.0
    img = patch.render(vp, a.width, a.height, light=(eye[0], eye[1] + 2.0, eye[2]), eye=eye, flip=flip,
                       flags=a.flags)
    write_ppm(a.out, img)
    print(a.out)


if __name__ == "__main__":
    main()
