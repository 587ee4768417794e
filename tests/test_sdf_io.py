"""SDF files in the reference's binary format (SDF::WriteToFile / LoadFromFile,
Geometry/SDF.cpp:78-151) and SDFs built from meshes (SDF::CreateFromMesh)."""
import struct

import numpy as np
import pytest

from solidcloth_b200 import scenes

GOLD = __import__("pathlib").Path(__file__).resolve().parent / "golden"


def _grid():
    rng = np.random.default_rng(3)
    cells = (5, 4, 3)
    box = np.array([-0.5, -0.25, 0.0, 0.75, 0.5, 0.3], np.float32)
    vals = rng.standard_normal(6 * 5 * 4).astype(np.float32)
    return cells, box, vals


def _make(cells, box, vals):
    from solidcloth_b200 import api
    b = api.scAabb3(api.v3(box[:3]), api.v3(box[3:]))
    h = api.lib().scCreateSDFGrid(cells[0], cells[1], cells[2], b, api._fp(np.ascontiguousarray(vals, np.float32)))
    return api.SDFHandle(h)


def test_save_load_round_trip_and_layout(tmp_path):
    """Own write, then own read: identical grid; the file is 3 ints, 6 doubles
    (min.x, max.x, min.y, max.y, min.z, max.z) and the values as doubles."""
    from solidcloth_b200 import api
    cells, box, vals = _grid()
    s = _make(cells, box, vals)
    path = tmp_path / "a.sdf"
    assert s.save(path)
    raw = path.read_bytes()
    assert len(raw) == 12 + 48 + 8 * vals.size
    assert struct.unpack("3i", raw[:12]) == cells
    b = struct.unpack("6d", raw[12:60])
    assert np.array_equal(np.float32(b), box[[0, 3, 1, 4, 2, 5]])
    assert np.array_equal(np.frombuffer(raw[60:], np.float64).astype(np.float32), vals)
    t = api.SDFHandle.load(path)
    c2, b2, v2 = t.grid()
    assert tuple(c2) == cells and np.array_equal(b2, box) and np.array_equal(v2, vals)
    s.free()
    t.free()


def test_files_match_the_reference_byte_for_byte(tmp_path):
    """The reference build writes the same bytes, and each side reads the other's file."""
    from oracle.bridge import available, ref_sdf_read, ref_sdf_write
    if not available("ref"):
        pytest.skip("reference build absent")
    from solidcloth_b200 import api
    cells, box, vals = _grid()
    ours, theirs = tmp_path / "ours.sdf", tmp_path / "ref.sdf"
    s = _make(cells, box, vals)
    s.save(ours)
    ref_sdf_write(cells, box, vals, theirs)
    assert ours.read_bytes() == theirs.read_bytes()
    c, b, v = ref_sdf_read(ours)
    assert tuple(c) == cells and np.array_equal(b, box) and np.array_equal(v, vals)
    c2, b2, v2 = api.SDFHandle.load(theirs).grid()
    assert np.array_equal(v2, vals)
    s.free()


def test_golden_sdf_from_mesh_pins_reference():
    """The fixture is the reference's own CreateFromMesh (live check where the build exists)."""
    from oracle.bridge import available, ref_sdf_from_mesh
    if not available("ref"):
        pytest.skip("reference build absent")
    g = np.load(GOLD / "sdf_mesh.npz")
    vals = ref_sdf_from_mesh(g["vertices"], g["indices"], (16, 16, 16), g["box"])
    assert np.array_equal(vals.view(np.uint32), g["values"].view(np.uint32))


@pytest.mark.gpu
def test_gpu_sdf_from_mesh_bitexact():
    """SDF::CreateFromMesh on the GPU equals the reference's, bit for bit (the
    field is unsigned, as the reference's default delta normal makes it)."""
    from solidcloth_b200 import api
    g = np.load(GOLD / "sdf_mesh.npz")
    s = api.SDFHandle.from_mesh(g["vertices"], g["indices"], (16, 16, 16), g["box"])
    cells, box, vals = s.grid()
    assert tuple(cells) == (16, 16, 16)
    assert np.array_equal(vals.view(np.uint32), g["values"].view(np.uint32)), float(np.abs(vals - g["values"]).max())
    assert np.all(vals >= 0)
    s.free()
