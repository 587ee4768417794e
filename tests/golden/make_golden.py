"""Generate the golden fixtures in this directory from the SolidCloth reference
itself (oracle/_ref, built from the reference's own C++ sources, single thread).

    python tests/golden/make_golden.py

The fixtures pin the CPU oracle (oracle/cloth_oracle.cpp) on machines where the
reference build is absent: tests/test_oracle.py replays each case through the
oracle and requires bit-identical results.
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle.bridge import RefCloth  # noqa: E402
from solidcloth_b200 import scenes  # noqa: E402


def case_cfg0():
    sc = scenes.cfg0()
    r = RefCloth.from_scene(sc)
    out = {}
    for f in range(10):
        r.step(sc.dt)
        r.update_mesh()
    pos, prev, vel, w = r.state()
    idx, rest = r.tris()
    return dict(pos=pos, prev=prev, vel=vel, invmass=w, tris=idx, rest=rest, bends=r.bends(), edges=r.edges(),
                normals=r.mesh_normals(False), prev_normals=r.mesh_normals(True))


def sdf_scene():
    sc = scenes.cfg1(n=20, self_mode="proximity")
    sc.params.substeps = 2
    sc.params.iterations = 6
    sc.positions[:, 1] -= np.float32(0.4 - 0.004)
    return sc


def case_sdf():
    sc = sdf_scene()
    r = RefCloth.from_scene(sc)
    for f in range(3):
        r.step(sc.dt)
        r.update_mesh()
    vi, vf = r.contacts(0)
    pos, prev, vel, _ = r.state()
    return dict(pos=pos, prev=prev, vel=vel, vc_idx=vi, vc_f=vf)


def folded_scene():
    sc = scenes.cfg1(n=16, self_mode="proximity")
    sc.sdfs.clear()
    sc.params.substeps = 1
    sc.params.iterations = 4
    return sc, scenes.folded(sc, gap=0.004)


def case_self():
    sc, st = folded_scene()
    r = RefCloth.from_scene(sc)
    r.set_state(*st)
    r.step(sc.dt)
    ti, tf = r.contacts(3)
    ei, ef = r.contacts(4)
    pos, prev, vel, _ = r.state()
    return dict(pos=pos, vt_idx=ti, vt_f=tf, ee_idx=ei, ee_f=ef)


def case_ccd():
    sc, st = scenes.ccd_scene(16)
    r = RefCloth.from_scene(sc)
    r.set_state(*st)
    r.predict_detect(sc.dt / sc.params.substeps, ccd=False)
    mid_vt, mid_ee = r.ccd_midphase()
    boxes_t = r.swept_boxes(0, sc.params.thickness + 0.5 * sc.params.tolerance)
    r2 = RefCloth.from_scene(sc)
    r2.set_state(*st)
    r2.predict_detect(sc.dt / sc.params.substeps, ccd=False)
    # narrow phase over the midphase candidates (the reference's own pair set)
    r2.ccd_narrow_on(mid_vt, mid_ee)
    hi, hf = r2.contacts(3)
    ei, ef = r2.contacts(4)
    return dict(mid_vt=mid_vt, mid_ee=mid_ee, boxes_t=boxes_t, hit_vt_idx=hi, hit_vt_f=hf, hit_ee_idx=ei, hit_ee_f=ef)


def mesh_scene():
    sc = scenes.cfg2(n=21, level=3)
    sc.params.substeps = 2
    sc.params.iterations = 4
    sc.positions[:, 1] -= np.float32(0.52)
    return sc


def case_mesh():
    sc = mesh_scene()
    r = RefCloth.from_scene(sc)
    for f in range(2):
        r.step(sc.dt)
        r.update_mesh()
    pos, prev, vel, _ = r.state()
    out = dict(pos=pos, prev=prev, vel=vel)
    for k, name in [(0, "vc"), (1, "tc"), (2, "ec")]:
        a, b = r.contacts(k)
        out[name + "_idx"], out[name + "_f"] = a, b
    return out


def links_scene(dihedral):
    """the mass-spring path (FEM off): stretch, shear and, without dihedral
    bending, bend links (ClothPatch::Init, Physics/ClothPatch.cpp:170-207)"""
    sc = scenes.cfg0()
    sc.params.fem = False
    sc.params.dihedral = dihedral
    sc.params.stretch, sc.params.shear, sc.params.bend = 1e3, 5e2, 2.0
    return sc


def case_links():
    out = {}
    for dih in (False, True):
        sc = links_scene(dih)
        r = RefCloth.from_scene(sc)
        for f in range(8):
            r.step(sc.dt)
        pos, prev, vel, _ = r.state()
        out[f"pos_dihedral{int(dih)}"] = pos
        out[f"vel_dihedral{int(dih)}"] = vel
    return out


def solver_scenes():
    """The reference's other link solvers (ClothModel::SetSolver): SolveJacobi on
    the mass-spring cloth with dihedral bending (stretch and shear links), eight
    frames; SolveCR one frame of one substep x 3 iterations (finite), and its
    default 4 x 10 frame (the solve diverges to NaN in the reference itself)."""
    jac = links_scene(True)
    jac.params.solver = 0
    cr = links_scene(True)
    cr.params.solver = 2
    cr.params.substeps, cr.params.iterations = 1, 3
    cr_div = links_scene(True)
    cr_div.params.solver = 2
    return [("jacobi", jac, 8), ("cr", cr, 1), ("cr_diverging", cr_div, 1)]


def case_solvers():
    out = {}
    for name, sc, frames in solver_scenes():
        r = RefCloth.from_scene(sc)
        for f in range(frames):
            r.step(sc.dt)
        pos, prev, vel, _ = r.state()
        out[f"{name}_pos"] = pos
        out[f"{name}_vel"] = vel
    return out


def case_sdf_mesh():
    """SDF::CreateFromMesh of a level-2 icosphere (radius 0.25) on a 16^3-cell grid"""
    from oracle.bridge import ref_sdf_from_mesh
    m = scenes.icosphere(2, 0.25, (0.0, 0.0, 0.0))
    box = np.array([-0.4, -0.4, -0.4, 0.4, 0.4, 0.4], np.float32)
    vals = ref_sdf_from_mesh(m.vertices, m.indices, (16, 16, 16), box)
    return dict(vertices=np.asarray(m.vertices, np.float32), indices=np.asarray(m.indices, np.uint32),
                box=box, values=vals)


CASES = {"cfg0": case_cfg0, "sdf": case_sdf, "self": case_self, "ccd": case_ccd, "mesh": case_mesh,
         "links": case_links, "sdf_mesh": case_sdf_mesh, "solvers": case_solvers}


if __name__ == "__main__":
    RefCloth.set_threads(1)
    only = set(sys.argv[1:])
    for name, fn in CASES.items():
        if only and name not in only:
            continue
        d = fn()
        np.savez_compressed(HERE / f"{name}.npz", **d)
        print(name, {k: v.shape for k, v in d.items()})
