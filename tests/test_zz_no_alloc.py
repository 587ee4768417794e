"""scComputeVertexNormalsNoAlloc: the allocation-free normals entry point.

It exists for callers that cannot call cudaMalloc (engines that reserve all GPU
memory up front, code running inside another library's memory pool, real-time
threads); its scratch is a fixed file-scope device array instead of a device
allocation. This test calls it through the C ABI on device buffers and checks
its output against the normals the existing entry point (scUpdateClothMesh ->
scGetMeshNormalBuffer) computes for the same positions, on two calls in a row
(the second must not see the first call's leftover scratch).

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


def _call(L, pos, idx, stream=None):
    import torch
    v = torch.from_numpy(np.ascontiguousarray(pos, np.float32)).cuda()
    i = torch.from_numpy(np.ascontiguousarray(idx, np.int32)).cuda()
    out = torch.full_like(v, float("nan"))
    rc = L.scComputeVertexNormalsNoAlloc(ctypes.c_void_p(v.data_ptr()), v.shape[0], ctypes.c_void_p(i.data_ptr()),
                                         i.numel() // 3, ctypes.c_void_p(out.data_ptr()), None)
    torch.cuda.synchronize()
    return rc, out.cpu().numpy()


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


def test_no_alloc_rejects_oversized_meshes():
    from solidcloth_b200 import api
    L = api.lib()
    n = 65536 + 1
    rc = L.scComputeVertexNormalsNoAlloc(ctypes.c_void_p(16), n, ctypes.c_void_p(16), 1, ctypes.c_void_p(16), None)
    assert rc == 2
    assert b"65536" in L.scGetLastErrorString()
    L.scGetLastError()
