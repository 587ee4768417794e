"""Headless cloth picture (scRenderCloth): camera conventions of Math/Matrix4.h,
the CPU restatement of the demo's Phong program on small cases, and the CUDA
rasteriser against it on a draped cloth (GPU)."""
import numpy as np
import pytest

from oracle import render_oracle as ro
from solidcloth_b200 import render, scenes

# colours go through pow / acos / sin / tan / exp2, whose last bits differ between
# CUDA and numpy; everything else in the picture is compared bit for bit
COLOUR_ATOL = 2e-5


def test_camera_matches_matrix4_conventions():
    eye, center = (1.0, 2.0, 3.0), (0.0, 0.5, 0.0)
    V = render.look_at(eye, center)
    e = V @ np.array([*eye, 1.0])
    assert np.allclose(e[:3], 0, atol=1e-6)
    c = V @ np.array([*center, 1.0])
    d = np.linalg.norm(np.subtract(eye, center))
    assert np.allclose(c[:3], [0, 0, -d], atol=1e-5)            # looking down -z
    P = render.perspective(60.0, 4 / 3, 0.1, 10.0)
    for zeye, ndc in ((-0.1, -1.0), (-10.0, 1.0)):
        q = P @ np.array([0.0, 0.0, zeye, 1.0])
        assert q[2] / q[3] == pytest.approx(ndc, abs=1e-5)
    q = P @ np.array([0.0, np.tan(np.radians(30.0)), -1.0, 1.0])
    assert q[1] / q[3] == pytest.approx(1.0, abs=1e-5)          # vertical fov


def _quad(z=0.0, half=0.5):
    pos = np.array([[-half, -half, z], [half, -half, z], [half, half, z], [-half, half, z]], np.float32)
    tri = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    nrm = np.tile(np.array([[0, 0, 1]], np.float32), (4, 1))
    return pos, nrm, tri


def _params(light, eye, flags=0, ks=(0.0, 0.0, 0.0)):
    return np.array([*light, *eye, 0.8, 0.3, 0.3, *ks, 32.0, 1.0, 0.25, flags], np.float32)


def test_oracle_depth_rule_and_coverage():
    W = H = 32
    vp = render.view_proj((0, 0, 3), (0, 0, 0), W, H, fov_deg=45)
    p0, n0, t0 = _quad(0.0)
    p1, n1, t1 = _quad(0.5, 0.25)                 # smaller, nearer quad drawn second
    pos = np.concatenate([p0, p1])
    tri = np.concatenate([t0, t1 + 4])
    zb = ro.rasterise(vp, pos, tri, W, H)
    ids = np.where(zb == ro.EMPTY, -1, (zb & np.uint64(0xFFFFFFFF)).astype(np.int64))
    assert ids[0, 0] == -1                       # corner: background
    assert ids[H // 2, W // 2] in (2, 3)          # centre: the nearer quad wins
    assert set(np.unique(ids[ids >= 0])) == {0, 1, 2, 3}
    # equal depth: the lower triangle index wins (GL_LESS in draw order)
    zb2 = ro.rasterise(vp, np.concatenate([p0, p0]), np.concatenate([t0, t0 + 4]), W, H)
    ids2 = (zb2[zb2 != ro.EMPTY] & np.uint64(0xFFFFFFFF)).astype(np.int64)
    assert ids2.max() <= 1


def test_oracle_phong_values():
    W = H = 16
    vp = render.view_proj((0, 0, 2), (0, 0, 0), W, H, fov_deg=60)
    pos, nrm, tri = _quad(0.0, 2.0)
    zb = ro.rasterise(vp, pos, tri, W, H)
    img = ro.shade(vp, pos, nrm, tri, zb, W, H, _params((0, 0, 50.0), (0, 0, 2), ks=(0.5, 0.5, 0.5)))
    # the light far along +z: diffuse ~1, shade = (0.2 + 1) / 1.2 = 1; specular ~1 at the
    # centre where the reflection points at the eye
    c = img[H // 2, W // 2, :3]
    assert np.allclose(c, np.array([0.8, 0.3, 0.3]) + 0.5, atol=5e-2)   # pixel centres sit off the axis
    # light behind the surface: ambient only, no specular
    img = ro.shade(vp, pos, nrm, tri, zb, W, H, _params((0, 0, -50.0), (0, 0, 2), ks=(0.5, 0.5, 0.5)))
    assert np.allclose(img[H // 2, W // 2, :3], np.array([0.8, 0.3, 0.3]) * (0.2 / 1.2), atol=1e-6)
    # monochrome: kd everywhere covered; background elsewhere
    img = ro.shade(vp, pos, nrm, tri, zb, W, H, _params((0, 0, 50.0), (0, 0, 2), flags=ro.MONOCHROME))
    cov = zb != ro.EMPTY
    assert np.allclose(img[cov][:, :3], [0.8, 0.3, 0.3])


def test_oracle_wireframe_darkens_edges_only():
    W = H = 64
    vp = render.view_proj((0, 0, 2), (0, 0, 0), W, H, fov_deg=60)
    pos, nrm, tri = _quad(0.0, 0.5)
    zb = ro.rasterise(vp, pos, tri, W, H)
    prm = _params((0, 0, 50.0), (0, 0, 2))
    plain = ro.shade(vp, pos, nrm, tri, zb, W, H, prm)
    prm[15] = ro.WIREFRAME
    wire = ro.shade(vp, pos, nrm, tri, zb, W, H, prm)
    cov = zb != ro.EMPTY
    dark = (wire[..., 0] < plain[..., 0] - 5e-2) & cov     # the shader also dims interiors by exp2(-8)
    assert dark.any() and dark.sum() < 0.5 * cov.sum()
    # the diagonal (shared edge) is among the darkened pixels
    assert dark[H // 2, W // 2] or dark[H // 2 - 1, W // 2] or dark[H // 2, W // 2 - 1]


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [0, ro.OREN_NAYAR, ro.WIREFRAME, ro.MONOCHROME])
def test_gpu_render_equals_oracle(flags):
    from solidcloth_b200 import api
    scene = scenes.cfg1(n=24)
    _, patch = api.load_scene(scene)
    try:
        for _ in range(30):
            patch.step(scene.dt)
        patch.update_mesh()
        pos, nrm, idx = patch.mesh_buffers()
        tri = idx.reshape(-1, 3).astype(np.int64)
        W, H = 160, 120
        eye, center = render.frame(pos)
        vp = render.view_proj(eye, center, W, H)
        light = (eye[0] + 0.5, eye[1] + 2.0, eye[2])
        img, zb = patch.render(vp, W, H, light=light, eye=eye, ks=(0.3, 0.3, 0.3), flags=flags, return_zbuf=True)
        img = img.cpu().numpy()
        zb = zb.cpu().numpy().view(np.uint64)
        zo = ro.rasterise(vp, pos, tri, W, H)
        assert (zb != ro.EMPTY).sum() > 0.05 * W * H
        assert np.array_equal(zb, zo)
        prm = np.array([*light, *eye, 0.8, 0.3, 0.3, 0.3, 0.3, 0.3, 32.0, 1.0, 0.3, flags], np.float32)
        io = ro.shade(vp, pos, nrm, tri, zo, W, H, prm)
        assert np.allclose(img, io, atol=COLOUR_ATOL, rtol=0)
    finally:
        patch.free()


@pytest.mark.gpu
def test_gpu_render_rejects_unrestated_flags():
    from solidcloth_b200 import api
    scene = scenes.cfg1(n=8)
    _, patch = api.load_scene(scene)
    try:
        vp = render.view_proj((0, 1, 2), (0, 0, 0), 8, 8)
        with pytest.raises(RuntimeError):
            patch.render(vp, 8, 8, flags=32)       # shadows are not restated
    finally:
        patch.free()
