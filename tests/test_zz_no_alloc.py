"""scComputeVertexNormalsNoAlloc: the allocation-free normals entry point.

It exists for callers that cannot call cudaMalloc (engines that reserve all GPU
memory up front, code running inside another library's memory pool, real-time
threads); its scratch is a fixed file-scope device array instead of a device
allocation. These tests call it through the C ABI on device buffers and check
its output against the normals the existing entry point (scUpdateClothMesh ->
scGetMeshNormalBuffer) computes for the same positions, on two calls in a row
(the second must not see the first call's leftover scratch), at the exact
capacity (a 256 x 256 grid, 65,536 vertices), on a caller's own stream with a
smaller mesh after a larger one, with no triangles, with a zero-area triangle,
and with an index out of range (rejected, nothing written for it).

The file name makes pytest collect it last, so a run that stops at the first
failure has already run every other test. It passes alone in a fresh process
and after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

from solidcloth_b200 import scenes

pytestmark = pytest.mark.gpu

TOL = 1e-5   # the parity tolerance of the GPU tests; the sums here use atomics
SC_ERR_ARG = 2


def _call(L, pos, idx, stream=None, n_override=None):
    """Runs the entry point on device copies of pos / idx; returns (rc, normals)."""
    import torch
    v = torch.from_numpy(np.ascontiguousarray(pos, np.float32)).cuda()
    i = torch.from_numpy(np.ascontiguousarray(idx, np.int32).reshape(-1)).cuda()
    out = torch.full_like(v, float("nan"))
    n = v.shape[0] if n_override is None else n_override
    h = None if stream is None else ctypes.c_void_p(stream.cuda_stream)
    rc = L.scComputeVertexNormalsNoAlloc(ctypes.c_void_p(v.data_ptr()), n,
                                         ctypes.c_void_p(i.data_ptr() if i.numel() else 0),
                                         i.numel() // 3, ctypes.c_void_p(out.data_ptr()), h)
    torch.cuda.synchronize()
    return rc, out.cpu().numpy()


def _existing(sc, frames):
    """Positions, normals (scUpdateClothMesh) and indices of `sc` after `frames` frames."""
    from solidcloth_b200 import api
    w, p = api.load_scene(sc)
    for _ in range(frames):
        p.step(sc.dt)
    p.update_mesh()
    verts, normals, idx = p.mesh_buffers()
    p.free()
    w.free()
    return verts, normals, idx


def _restated_normals(v, idx):
    """Mesh::ComputeNormals (Geometry/Mesh.cpp:10-63) in float32 numpy, for meshes
    no cloth patch can hold (a zero-area triangle)."""
    v = v.astype(np.float32)
    out = np.zeros_like(v)
    with np.errstate(all="ignore"):
        for t in idx.reshape(-1, 3):
            a, b, c = v[t[0]], v[t[1]], v[t[2]]
            n = np.cross(b - a, c - a)
            nt = n * (np.float32(1) / np.float32(np.sqrt(np.dot(n, n))))
            e1, e2, e3 = b - a, c - b, a - c
            e1 = e1 / np.sqrt(np.dot(e1, e1)); e2 = e2 / np.sqrt(np.dot(e2, e2)); e3 = e3 / np.sqrt(np.dot(e3, e3))
            cs = [-np.dot(e1, e3), -np.dot(e1, e2), -np.dot(e2, e3)]
            for k, cc in enumerate(cs):
                out[t[k]] += np.float32(np.arccos(np.clip(cc, -1, 1))) * nt
        ln = np.sqrt((out * out).sum(1))
        nz = ln != 0
        out[nz] = out[nz] / ln[nz, None]
    return out


def test_no_alloc_normals_match_existing_entry_point():
    from solidcloth_b200 import api
    L = api.lib()
    sc = scenes.cfg0()
    w, p = api.load_scene(sc)
    for call in range(2):
        # move the cloth so the two calls see different geometry
        for _ in range(3 + 5 * call):
            p.step(sc.dt)
        p.update_mesh()
        verts, ref_normals, idx = p.mesh_buffers()
        rc, normals = _call(L, verts, idx)
        assert rc == 0, api.lib().scGetLastErrorString()
        assert np.isfinite(normals).all()
        err = float(np.abs(normals - ref_normals).max())
        assert err <= TOL, (call, err)
    p.free()


def test_no_alloc_at_capacity_then_smaller_mesh_on_own_stream():
    """65,536 vertices (the capacity), then a 32x32 mesh on a caller's stream:
    the second call clears exactly what it uses and reads nothing stale."""
    import torch
    from solidcloth_b200 import api
    L = api.lib()
    big = scenes.make_grid_scene("nalloc_256", 256, 1.5, 0.0, scenes.Params(iterations=4, substeps=2),
                                 pinned_corners=(1, 3), seed=11)
    verts, ref, idx = _existing(big, 2)
    assert verts.shape[0] == 65536
    rc, normals = _call(L, verts, idx)
    assert rc == 0, L.scGetLastErrorString()
    assert float(np.abs(normals - ref).max()) <= TOL
    small = scenes.cfg0(seed=4)
    verts2, ref2, idx2 = _existing(small, 3)
    s = torch.cuda.Stream()
    for _ in range(2):
        rc, normals2 = _call(L, verts2, idx2, stream=s)
        assert rc == 0, L.scGetLastErrorString()
        assert float(np.abs(normals2 - ref2).max()) <= TOL


def test_no_alloc_without_triangles_gives_zero_normals():
    from solidcloth_b200 import api
    L = api.lib()
    pos = np.random.default_rng(1).uniform(-1, 1, (100, 3)).astype(np.float32)
    rc, normals = _call(L, pos, np.zeros(0, np.int32))
    assert rc == 0, L.scGetLastErrorString()
    assert (normals == 0).all()


def test_no_alloc_zero_area_triangle_matches_restatement():
    """A zero-area triangle gives its vertices the reference's NaN normal
    (Vector3::Normalize divides by a zero length); the others are unaffected."""
    from solidcloth_b200 import api
    L = api.lib()
    # triangle 2 is collinear, with exactly representable coordinates so that its
    # edge vectors are exactly parallel and their cross product exactly zero
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0.25], [2, 2, 0.5], [3, 3, 0.75], [5, 0, 0], [6, 0, 0],
                    [5, 1, 0.125]], np.float32)
    idx = np.array([0, 1, 2, 1, 3, 2, 3, 4, 5, 6, 7, 8], np.int32)
    expect = _restated_normals(pos, idx)
    rc, normals = _call(L, pos, idx)
    assert rc == 0, L.scGetLastErrorString()
    assert (np.isnan(normals) == np.isnan(expect)).all()
    fin = ~np.isnan(expect)
    assert np.isnan(expect[3]).all() and fin[6:].all()
    assert float(np.abs(normals[fin] - expect[fin]).max()) <= TOL


def test_no_alloc_rejects_out_of_range_indices():
    """A triangle with an index >= numVertices is skipped and reported; the
    valid triangles' normals are still computed."""
    from solidcloth_b200 import api
    L = api.lib()
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0.3]], np.float32)
    good = np.array([0, 1, 2, 1, 3, 2], np.int32)
    rc, expect = _call(L, pos, good)
    assert rc == 0
    for bad_index in (4, 65536, 70000, 2 ** 31 - 1):
        idx = np.concatenate([good, np.array([0, 1, bad_index], np.int32)])
        rc, normals = _call(L, pos, idx)
        assert rc == SC_ERR_ARG, bad_index
        assert b"index >= numVertices" in L.scGetLastErrorString()
        L.scGetLastError()
        assert float(np.abs(normals - expect).max()) <= TOL
    # the entry point still works after a rejected call
    rc, normals = _call(L, pos, good)
    assert rc == 0 and float(np.abs(normals - expect).max()) <= TOL


def test_no_alloc_rejects_oversized_meshes():
    from solidcloth_b200 import api
    L = api.lib()
    n = 65536 + 1
    rc = L.scComputeVertexNormalsNoAlloc(ctypes.c_void_p(16), n, ctypes.c_void_p(16), 1, ctypes.c_void_p(16), None)
    assert rc == 2
    assert b"65536" in L.scGetLastErrorString()
    L.scGetLastError()
