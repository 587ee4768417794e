"""The C ABI rejects bad arguments before it touches the GPU: each call below
records an error code (scGetLastError) and returns, on a host without a GPU too."""
import ctypes as C

import numpy as np
import pytest

SC_ERR_ARG = 2


@pytest.fixture(scope="module")
def lib():
    from solidcloth_b200 import api
    try:
        return api.lib()
    except RuntimeError as e:       # library not built
        pytest.skip(str(e))


def _last(lib):
    return lib.scGetLastError()


def test_noalloc_normals_rejects_sizes_and_null_buffers(lib):
    lib.scGetLastError()
    buf = (C.c_float * 3)()
    idx = (C.c_uint * 3)()
    assert lib.scComputeVertexNormalsNoAlloc(None, 1, None, 0, buf, None) == SC_ERR_ARG
    assert lib.scComputeVertexNormalsNoAlloc(buf, 1, None, 1, buf, None) == SC_ERR_ARG      # triangles, no indices
    assert lib.scComputeVertexNormalsNoAlloc(buf, 0, idx, 1, buf, None) == SC_ERR_ARG
    assert lib.scComputeVertexNormalsNoAlloc(buf, 65537, idx, 1, buf, None) == SC_ERR_ARG   # above the scratch
    assert lib.scComputeVertexNormalsNoAlloc(buf, 3, idx, -1, buf, None) == SC_ERR_ARG
    assert lib.scComputeVertexNormalsNoAlloc(buf, 3, idx, 16777217, buf, None) == SC_ERR_ARG  # above the triangle cap
    assert _last(lib) == SC_ERR_ARG
    assert _last(lib) == 0                                                                # read and cleared


def test_render_and_probe_reject_bad_requests(lib):
    from solidcloth_b200 import api
    lib.scGetLastError()
    vp = np.eye(4, dtype=np.float32)
    prm = np.zeros(16, np.float32)
    img = np.zeros(4, np.float32)
    null_patch = api.scClothPatch(None)
    rc = lib.scRenderCloth(null_patch, vp.ctypes.data_as(api._f), prm.ctypes.data_as(api._f), 1, 1,
                           img.ctypes.data, img.ctypes.data)
    assert rc == SC_ERR_ARG and _last(lib) == SC_ERR_ARG
    assert lib.scProbeClusterPhase(2, 10) < 0 and _last(lib) == SC_ERR_ARG
    assert lib.scProbeClusterPhase(0, 0) < 0 and _last(lib) == SC_ERR_ARG


def test_model_setters_reject_null_models_and_bad_modes(lib):
    from solidcloth_b200 import api
    lib.scGetLastError()
    null_model = api.scModel(None)
    lib.scSetBroadPhaseMode(null_model, 0)
    assert _last(lib) == SC_ERR_ARG
    lib.scSetSolverMode(null_model, 1)
    assert _last(lib) == SC_ERR_ARG
    lib.scSetGridSolver(null_model, 0, 1)
    assert _last(lib) == SC_ERR_ARG
