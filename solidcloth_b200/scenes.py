"""Synthetic cloth workloads with the shapes of the benchmark configurations.

Every array here is float32 / uint32 and produced deterministically from a
seed, so the CUDA library, the CPU oracle and the reference build all receive
bit-identical inputs. Nothing in this module touches a GPU.

Configurations (sizes, materials and colliders of the benchmark set):
  cfg0  32x32 grid, 1 m, two corners pinned, FEM + bends, no collisions, 4 x 10
  cfg1  128x128 grid, 1 m, 0.4 m above a sphere (r 0.3) sampled as a 64^3 SDF,
        self-collision, thickness 5 mm, friction 0.3, 8 x 15
  cfg2  256x256 grid, 1.5 m, dropped 0.5 m onto a level-5 icosphere mesh
        (r 0.25) standing on a ground plane, mesh + self contacts, 8 x 20
  cfg3  512 independent cloths, side 16..128 log-uniform, sphere SDF 32^3 each,
        1-4 pinned corners, self-collision, 8 x 15
Mapping choices (documented where the reference needs an interpretation):
  * unit = 1 (SI gravity), FEM on, dihedral bends on;
  * E = 1e3 enters only the shear compliance; Poisson 0.3;
  * bend stiffness 1e-3 is the projection factor s = 0.0005 * b, so b = 2.0;
  * lumped masses from areal density 0.1 kg/m^2; pinned vertices get mass 0
    (-> inverse mass 0, as ClothModel::SetMasses does);
  * +-1e-3 m uniform noise on positions after the grid is built;
  * fixed iteration counts (the reference's FEM early exit is bypassed).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

CF_VERTICES, CF_TRIANGLES, CF_SELF, CF_WALLS, CF_EDGES = 1, 2, 4, 8, 16


@dataclass
class Params:
    unit: float = 1.0
    thickness: float = 0.3
    tolerance: float = 0.2
    shear: float = 1e3
    bend: float = 2.0
    stretch: float = 2e10
    poisson: float = 0.3
    friction: float = 0.4
    iterations: int = 10
    substeps: int = 4
    flags: int = 0
    fem: bool = True
    dihedral: bool = True
    fixed_iterations: bool = True
    drag: float = 1.0
    solver: int = 1     # ClothModel::SolverType: 0 Jacobi, 1 Gauss-Seidel, 2 conjugate residual (not in as_array)

    def as_array(self) -> np.ndarray:
        return np.array([self.unit, self.thickness, self.tolerance, self.shear, self.bend,
                         self.stretch, self.poisson, self.friction, self.iterations,
                         self.substeps, self.flags, float(self.fem), float(self.dihedral),
                         float(self.fixed_iterations), self.drag], dtype=np.float32)


@dataclass
class SDFGrid:
    cells: tuple
    box: np.ndarray          # (6,) min xyz, max xyz
    values: np.ndarray       # (cells+1)^3 float32, x fastest


@dataclass
class MeshCollider:
    vertices: np.ndarray     # (V, 3) float32
    indices: np.ndarray      # (T*3,) uint32


@dataclass
class Scene:
    name: str
    n: int                   # vertices per side
    inc: float               # grid spacing
    offset: np.ndarray       # (3,)
    attached: bool
    params: Params
    masses: np.ndarray       # (n*n,) float32, 0 at pinned vertices
    positions: np.ndarray    # (n*n, 3) float32 (noisy initial positions)
    dt: float = 1.0 / 60.0
    frames: int = 120
    walls: Optional[np.ndarray] = None
    spheres: List[tuple] = field(default_factory=list)
    sdfs: List[SDFGrid] = field(default_factory=list)
    meshes: List[MeshCollider] = field(default_factory=list)
    ccd: bool = False

    @property
    def num_vertices(self) -> int:
        return self.n * self.n


def grid_positions(n: int, inc: float, offset) -> np.ndarray:
    """Flat horizontal grid positions exactly as ClothPatch::Init(grid) computes
    them in float32 (Physics/ClothPatch.cpp:150-190): column j at
    x_j = x_{j-1} + inc starting from -0.5*n*inc, row i at startY + inc*i."""
    off = np.asarray(offset, dtype=np.float32)
    inc32 = np.float32(inc)
    start = np.float32(np.float32(np.float32(-0.5) * np.float32(n)) * inc32)
    xs = np.empty(n, dtype=np.float32)
    x = start
    for j in range(n):                 # the running float32 sum of the reference's loop
        xs[j] = x
        x = np.float32(x + inc32)
    zs = (start + (inc32 * np.arange(n, dtype=np.float32)).astype(np.float32)).astype(np.float32)
    zs[0] = start
    pos = np.empty((n, n, 3), dtype=np.float32)
    pos[:, :, 0] = (xs + off[0]).astype(np.float32)[:, None]
    pos[:, :, 1] = np.float32(np.float32(0) + off[1])
    pos[:, :, 2] = (zs + off[2]).astype(np.float32)[None, :]
    return pos.reshape(n * n, 3)


def grid_triangles(n: int) -> np.ndarray:
    """Triangle list of ClothPatch::Init(grid), alternating diagonals
    (Physics/ClothPatch.cpp:205-221)."""
    j, i = np.meshgrid(np.arange(1, n), np.arange(1, n), indexing="ij")
    idx = j * n + i
    a, b, c, d = idx - n - 1, idx - n, idx, idx - 1
    same = (i & 1) == (j & 1)
    t1 = np.where(same[..., None], np.stack([a, c, b], -1), np.stack([b, d, c], -1))
    t2 = np.where(same[..., None], np.stack([a, d, c], -1), np.stack([d, b, a], -1))
    return np.stack([t1, t2], 2).reshape(-1, 3).astype(np.uint32)


def lumped_masses(n: int, inc: float, density: float, pinned) -> np.ndarray:
    tris = grid_triangles(n)
    area = np.float32(0.5 * inc * inc)
    m = np.zeros(n * n, dtype=np.float64)
    for k in range(3):
        np.add.at(m, tris[:, k], density * float(area) / 3.0)
    m = m.astype(np.float32)
    for p in pinned:
        m[p] = 0.0
    return m


def corner_pins(n: int, corners) -> List[int]:
    """Corner vertex ids: 0 = (j=0,i=0), 1 = (j=0,i=n-1), 2 = (j=n-1,i=0), 3 = (j=n-1,i=n-1).
    ClothPatch::Init(attached=true) pins corners 1 and 3."""
    ids = [0, n - 1, (n - 1) * n, n * n - 1]
    return [ids[c] for c in corners]


def sphere_sdf(center, radius: float, cells: int, margin: float) -> SDFGrid:
    """Analytic sphere distance sampled at the grid points of SDF::Create(cells,
    cells, cells, box) (Geometry/SDF.cpp:10-40, GetPosAt SDF.h:64-70)."""
    c = np.asarray(center, dtype=np.float32)
    half = np.float32(radius + margin)
    bmin = (c - half).astype(np.float32)
    bmax = (c + half).astype(np.float32)
    ext = (bmax - bmin).astype(np.float32)
    inv = np.float32(1.0) / np.float32(cells)
    steps = (ext * inv).astype(np.float32)
    ax = np.arange(cells + 1, dtype=np.float32)
    gx = (ax * steps[0] + bmin[0]).astype(np.float32)
    gy = (ax * steps[1] + bmin[1]).astype(np.float32)
    gz = (ax * steps[2] + bmin[2]).astype(np.float32)
    Z, Y, X = np.meshgrid(gz, gy, gx, indexing="ij")
    d = np.sqrt((X.astype(np.float64) - c[0]) ** 2 + (Y.astype(np.float64) - c[1]) ** 2 +
                (Z.astype(np.float64) - c[2]) ** 2) - radius
    vals = d.astype(np.float32).reshape(-1)          # x fastest (z outermost)
    return SDFGrid((cells, cells, cells), np.concatenate([bmin, bmax]).astype(np.float32), vals)


def icosphere(level: int, radius: float, center) -> MeshCollider:
    """Icosahedron subdivided `level` times and projected to the sphere
    (level 5 -> 10,242 vertices, 20,480 triangles), outward winding."""
    t = (1.0 + 5 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
             (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(v, dtype=np.float64) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    v = (np.asarray(verts) * radius + np.asarray(center, dtype=np.float64)).astype(np.float32)
    return MeshCollider(v, np.asarray(faces, dtype=np.uint32).reshape(-1))


def _noise(rng: np.random.Generator, shape, amp: float) -> np.ndarray:
    return rng.uniform(-amp, amp, size=shape).astype(np.float32)


def make_grid_scene(name: str, n: int, side: float, height: float, params: Params,
                    pinned_corners=(), seed: int = 0, frames: int = 120,
                    center_xz=(0.0, 0.0)) -> Scene:
    inc = float(np.float32(side / (n - 1)))
    # centre the grid: column/row coordinates start at -0.5*n*inc
    off = np.array([0.5 * inc + center_xz[0], height, 0.5 * inc + center_xz[1]], dtype=np.float32)
    pins = corner_pins(n, pinned_corners)
    masses = lumped_masses(n, inc, 0.1, pins)
    rng = np.random.default_rng(seed)
    pos = grid_positions(n, inc, off)
    pos = (pos + _noise(rng, pos.shape, 1e-3)).astype(np.float32)
    attached = tuple(sorted(pinned_corners)) == (1, 3)
    return Scene(name, n, inc, off, attached, params, masses, pos, frames=frames)


def cfg0(seed: int = 0) -> Scene:
    p = Params(iterations=10, substeps=4, flags=0)
    return make_grid_scene("cfg0_32x32_pinned", 32, 1.0, 0.0, p, pinned_corners=(1, 3), seed=seed, frames=120)


def _self_flags(self_mode: str):
    """Self-collision mapping. "ccd": the continuous detector the benchmark
    configurations name (Physics/SelfCollisionDetector.cpp), CF_SELF off.
    "proximity": the reference's live CF_SELF path (brute-force closest features,
    Geometry/ClosestPointsBetweenMeshes.cpp:538-592). "both": the two together.
    At the configurations' scale (5 mm thickness + 5 mm tolerance on a 7.9 mm
    grid) the live path finds coplanar non-adjacent neighbours within radTol and
    its solve treats them as penetrating (it tests the triangle-normal component,
    ClothCollisionHandler.cpp:400-412), so the reference itself crumples the
    cloth; the continuous detector does not."""
    return {"ccd": (0, True), "proximity": (CF_SELF, False), "both": (CF_SELF, True)}[self_mode]


def cfg1(seed: int = 1, n: int = 128, ccd: bool = True, self_mode: str | None = None) -> Scene:
    mode = self_mode or ("ccd" if ccd else "proximity")
    sf, use_ccd = _self_flags(mode)
    p = Params(thickness=0.005, tolerance=0.005, friction=0.3, iterations=15, substeps=8,
               flags=CF_VERTICES | sf)
    s = make_grid_scene(f"cfg1_{n}x{n}_sphere_sdf_self_{mode}", n, 1.0, 0.3 + 0.4, p, seed=seed, frames=300)
    s.sdfs.append(sphere_sdf((0.0, 0.0, 0.0), 0.3, 63, 0.1))
    s.ccd = use_ccd
    return s


def cfg2(seed: int = 2, n: int = 256, level: int = 5, self_mode: str = "ccd") -> Scene:
    sf, use_ccd = _self_flags(self_mode)
    p = Params(thickness=0.005, tolerance=0.005, friction=0.3, iterations=20, substeps=8,
               flags=CF_VERTICES | CF_TRIANGLES | CF_EDGES | CF_WALLS | sf)
    s = make_grid_scene(f"cfg2_{n}x{n}_icosphere_mesh_self_{self_mode}", n, 1.5, 0.5 + 0.5, p, seed=seed, frames=300)
    s.ccd = use_ccd
    # Unit masses (inverse mass 1, the reference's own default after Init): the
    # reference's triangle and edge contact solves divide by the inverse mass
    # (SolveTriContacts / SolveEdgeContacts, Physics/ClothCollisionHandler.cpp:302,381),
    # which is only consistent when inverse masses are 1; with ~1 g lumped masses
    # they move vertices by kilometres. FEM, bends and the other contacts are
    # invariant to a uniform mass scale.
    s.masses = np.ones(n * n, dtype=np.float32)
    s.walls = np.array([-20.0, 0.0, -20.0, 20.0, 20.0, 20.0], dtype=np.float32)
    s.meshes.append(icosphere(level, 0.25, (0.0, 0.25, 0.0)))
    return s


def cfg3_instances(count: int = 512, seed: int = 3, lo: int = 16, hi: int = 128) -> List[Scene]:
    rng = np.random.default_rng(seed)
    sides = np.exp(rng.uniform(np.log(lo), np.log(hi), size=count)).round().astype(int)
    scenes = []
    for k in range(count):
        n = int(np.clip(sides[k], lo, hi))
        r = float(rng.uniform(0.1, 0.4))
        npins = int(rng.integers(1, 5))
        corners = tuple(sorted(rng.choice(4, size=npins, replace=False).tolist()))
        p = Params(thickness=0.005, tolerance=0.005, friction=0.3, iterations=15, substeps=8,
                   flags=CF_VERTICES)
        s = make_grid_scene(f"cfg3_inst{k}_{n}", n, 1.0, r + 0.4, p, pinned_corners=corners,
                            seed=seed * 100003 + k, frames=200)
        s.sdfs.append(sphere_sdf((0.0, 0.0, 0.0), r, 31, 0.1))
        s.ccd = True
        scenes.append(s)
    return scenes


CONFIGS = {"cfg0": cfg0, "cfg1": cfg1, "cfg2": cfg2}


def folded(scene: Scene, gap: float = 0.004, drop_speed: float = 0.0):
    """A cloth folded in half along its middle row: rows past the middle are
    mirrored onto the first half, `gap` above it, optionally moving down at
    `drop_speed` m/s. Returns (pos, prev, vel) float32 arrays (prev == pos)."""
    n = scene.n
    pos = scene.positions.copy().reshape(n, n, 3)  # [j (x), i (z), xyz]
    mid = (n - 1) / 2.0
    i = np.arange(n)
    z0 = pos[:, 0, 2].copy()
    inc = np.float32(scene.inc)
    top = i > mid
    zmir = z0[:, None] + (2 * mid - i[None, :]) * inc
    pos[:, top, 2] = zmir[:, top]
    pos[:, top, 1] = pos[:, top, 1] + np.float32(gap)
    pos = pos.reshape(-1, 3).astype(np.float32)
    vel = np.zeros_like(pos)
    if drop_speed:
        vel.reshape(n, n, 3)[:, top, 1] = -drop_speed
    return pos, pos.copy(), vel.astype(np.float32)


def ccd_scene(n: int = 16, seed: int = 5):
    """Continuous-collision test case in the reference demo's unit scale (the
    reference's CCD cut-offs are absolute: |f(0)| < 1e-3 and a 0.1 proximity,
    Physics/SelfCollisionDetector.cpp:257,300, so they only act at that scale):
    a folded 30-unit cloth whose upper layer falls through the lower one with a
    deforming (non-rigid) motion. Returns (scene, (pos, prev, vel))."""
    p = Params(unit=10, thickness=0.5, tolerance=0.4, iterations=2, substeps=1,
               flags=CF_VERTICES | CF_SELF)
    sc = make_grid_scene(f"ccd_fold_{n}", n, 30.0, 0.0, p, seed=seed)
    pos, prev, vel = folded(sc, gap=0.3, drop_speed=40.0)
    rng = np.random.default_rng(seed + 2)
    vel = (vel + rng.uniform(-20.0, 20.0, vel.shape)).astype(np.float32)
    sc.ccd = True
    return sc, (pos, prev, vel)


def mesh_cloth(n: int = 10, side: float = 0.5, height: float = 0.3, seed: int = 9):
    """A square sheet given as a triangle soup, as a mesh importer delivers it:
    every triangle has its own three vertices (coincident corners merge into
    particles in ClothPatch::Init(mesh)), with uvs = the rest-shape xz
    coordinates, and red vertex colours on the two far corners (pinned when
    attached). A little seeded noise is added to the heights. Returns
    (vertices, indices, uvs, colors, params)."""
    rng = np.random.default_rng(seed)
    inc = np.float32(side / (n - 1))
    xs = (np.arange(n, dtype=np.float32) * inc - np.float32(0.5 * side)).astype(np.float32)
    grid = np.stack(np.meshgrid(xs, xs, indexing="ij"), -1).reshape(-1, 2)
    ys = (np.float32(height) + _noise(rng, (n * n,), 1e-3)).astype(np.float32)
    verts, uvs, cols, idx = [], [], [], []
    for j in range(n - 1):
        for i in range(n - 1):
            a, b, c, d = j * n + i, j * n + i + 1, (j + 1) * n + i + 1, (j + 1) * n + i
            for tri in ((a, b, c), (a, c, d)):
                for v in tri:
                    verts.append((grid[v, 0], ys[v], grid[v, 1]))
                    uvs.append((grid[v, 0], grid[v, 1]))
                    corner = v in (n - 1, n * n - 1)
                    cols.append((1.0 if corner else 0.0, 0.0, 0.0))
                    idx.append(len(idx))
    p = Params(thickness=0.005, tolerance=0.005, iterations=8, substeps=4, flags=0)
    return (np.array(verts, np.float32), np.array(idx, np.uint32), np.array(uvs, np.float32),
            np.array(cols, np.float32), p)
