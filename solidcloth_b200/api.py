"""Python binding of the C ABI (include/solidcloth_b200.h) over ctypes.

The classes mirror the reference's C++ objects that ClothDemo drives directly
(Physics/CollisionWorld.h, Physics/ClothPatch.h, Physics/ClothModel.h) and call
the same sc* entry points a ctypes / cgo / JNI caller of the reference's
ClothLib would bind. There is no CPU fallback: if the CUDA library is not built
or no CUDA device is usable, constructing a patch raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from .scenes import Scene

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libsolidcloth_b200.so"


class scVector3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class scVector2(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float)]


class scAabb3(C.Structure):
    _fields_ = [("min", scVector3), ("max", scVector3)]


class scQuaternion(C.Structure):
    _fields_ = [("s", C.c_float), ("v", scVector3)]


class _Handle(C.Structure):
    _fields_ = [("ptr", C.c_void_p)]


scClothPatch = scCollisionWorld = scMesh = scModel = _Handle
_f = C.POINTER(C.c_float)
_i = C.POINTER(C.c_int)
_u = C.POINTER(C.c_uint)

# name -> (argtypes, restype)
SIGNATURES = {
    "scCreateCollisionWorld": ([], scCollisionWorld),
    "scFreeCollisionWorld": ([scCollisionWorld], None),
    "scClearCollidables": ([scCollisionWorld], None),
    "scGetNumCollidables": ([scCollisionWorld], C.c_int),
    "scAddCollidable": ([scCollisionWorld, C.c_void_p], None),
    "scGetCollidable": ([scCollisionWorld, C.c_int], C.c_void_p),
    "scCreateWalls": ([scAabb3], C.c_void_p),
    "scCreateSphere": ([scVector3, C.c_float], C.c_void_p),
    "scCreateCapsule": ([scVector3, C.c_float, C.c_float, scQuaternion], C.c_void_p),
    "scCreateSDFGrid": ([C.c_int, C.c_int, C.c_int, scAabb3, _f], C.c_void_p),
    "scCreateSDFFromMesh": ([_f, C.c_int, _u, C.c_int, C.c_int, C.c_int, C.c_int, scAabb3], C.c_void_p),
    "scSaveSDF": ([C.c_void_p, C.c_char_p], C.c_bool),
    "scLoadSDF": ([C.c_char_p], C.c_void_p),
    "scInitClothMesh": ([scClothPatch, _f, C.c_int, _u, C.c_int, _f, _f, scVector3, C.c_bool], None),
    "scGetMeshParticleMap": ([scClothPatch, _i, C.c_int], C.c_int),
    "scGetTriangleRest": ([scModel, _f], None),
    "scInitClothObj": ([scClothPatch, C.c_char_p, scVector3, C.c_bool], C.c_bool),
    "scGetLinkRest": ([scModel, _f], None),
    "scGetSDFGrid": ([C.c_void_p, _i, _f, _f, C.c_int], C.c_int),
    "scFreeCollidable": ([C.c_void_p], None),
    "scCreateMeshCollider": ([_f, C.c_int, _u, C.c_int], C.c_void_p),
    "scGetCollidableType": ([C.c_void_p], C.c_int),
    "scGetMeshTree": ([C.c_void_p], C.c_void_p),
    "scGetWallsInfo": ([C.c_void_p, C.POINTER(scAabb3)], None),
    "scGetSphereInfo": ([C.c_void_p, _f, C.POINTER(scVector3)], None),
    "scGetCapsuleInfo": ([C.c_void_p, _f, _f, C.POINTER(scVector3), C.POINTER(scQuaternion)], None),
    "scCreateClothPatch": ([scCollisionWorld], scClothPatch),
    "scFreeClothPatch": ([scClothPatch], None),
    "scGetClothModel": ([scClothPatch], scModel),
    "scGetClothMesh": ([scClothPatch], scMesh),
    "scInitCloth": ([scClothPatch, C.c_int, C.c_int, C.c_float, scVector3, C.c_bool, C.c_bool], None),
    "scStepCloth": ([scClothPatch, C.c_float], None),
    "scUpdateClothMesh": ([scClothPatch], None),
    "scComputeStrainMap": ([scClothPatch, C.POINTER(scVector3)], None),
    "scGetNumParticles": ([scModel], C.c_int),
    "scGetParticlePos": ([scModel, C.c_int, C.POINTER(scVector3)], None),
    "scGetParticleInvMass": ([scModel, C.c_int], C.c_float),
    "scGetNumTris": ([scModel], C.c_int),
    "scGetTriangle": ([scModel, C.c_int, _i, _i, _i], None),
    "scGetTriangleInfo": ([scModel, C.c_int, _f, C.POINTER(scVector2), C.POINTER(scVector2), C.POINTER(scVector2)], None),
    "scGetNumQuads": ([scModel], C.c_int),
    "scGetQuad": ([scModel, C.c_int, _i, _i, _i, _i], None),
    "scGetNumLinks": ([scModel], C.c_int),
    "scGetLink": ([scModel, C.c_int, _i, _i], None),
    "scGetNumContacts": ([scModel], C.c_int),
    "scGetContact": ([scModel, C.c_int, C.POINTER(scVector3), C.POINTER(scVector3)], None),
    "scGetNumTriContacts": ([scModel], C.c_int),
    "scGetTriContact": ([scModel, C.c_int, C.POINTER(scVector3), C.POINTER(scVector3)], None),
    "scGetCollisionFlags": ([scModel], C.c_int),
    "scSetCollisionFlags": ([scModel, C.c_int], None),
    "scGetThickness": ([scModel], C.c_float),
    "scSetThickness": ([scModel, C.c_float], None),
    "scGetTolerance": ([scModel], C.c_float),
    "scSetTolerance": ([scModel, C.c_float], None),
    "scGetFriction": ([scModel], C.c_float),
    "scSetFriction": ([scModel, C.c_float], None),
    "scGetNumIterations": ([scModel], C.c_int),
    "scSetNumIterations": ([scModel, C.c_int], None),
    "scGetUseFEM": ([scModel], C.c_bool),
    "scSetUseFEM": ([scModel, C.c_bool], None),
    "scSetSolverType": ([scModel, C.c_int], None),
    "scGetSolverType": ([scModel], C.c_int),
    "scGetClothTree": ([scModel], C.c_void_p),
    "scAddMouseSpring": ([scModel, C.c_int, C.c_int, C.c_int, scVector3, scVector3], None),
    "scUpdateMouseSpring": ([scModel, scVector3], None),
    "scRemoveMouseSpring": ([scModel], None),
    "scGetMeshVertexCount": ([scMesh], C.c_int),
    "scGetMeshIndexCount": ([scMesh], C.c_int),
    "scGetMeshNormalBuffer": ([scMesh], C.POINTER(scVector3)),
    "scGetMeshVertexBuffer": ([scMesh], C.POINTER(scVector3)),
    "scGetMeshIndexBuffer": ([scMesh], C.POINTER(C.c_uint)),
    "scSetUnit": ([scModel, C.c_float], None),
    "scGetUnit": ([scModel], C.c_float),
    "scSetShearStiffness": ([scModel, C.c_float], None),
    "scSetBendStiffness": ([scModel, C.c_float], None),
    "scSetStretchStiffness": ([scModel, C.c_float], None),
    "scSetPoisson": ([scModel, C.c_float], None),
    "scSetDragCoeff": ([scModel, C.c_float], None),
    "scSetDihedral": ([scModel, C.c_bool], None),
    "scSetSelfShrink": ([scModel, C.c_float], None),
    "scSetNumSteps": ([scClothPatch, C.c_int], None),
    "scGetNumSteps": ([scClothPatch], C.c_int),
    "scSetMasses": ([scModel, _f], None),
    "scSetParticleInvMass": ([scModel, C.c_int, C.c_float], None),
    "scSetParticlePositions": ([scModel, _f], None),
    "scGetParticlePositions": ([scModel, _f], None),
    "scGetParticleVelocities": ([scModel, _f], None),
    "scGetParticlePrevPositions": ([scModel, _f], None),
    "scSetParticleState": ([scModel, _f, _f, _f], None),
    "scSetFixedIterations": ([scModel, C.c_bool], None),
    "scSetSelfCCD": ([scModel, C.c_bool], None),
    "scSetClusterSolver": ([scModel, C.c_bool], None),
    "scSetClusterStaging": ([scModel, C.c_bool], None),
    "scSetSolverPrecision": ([scModel, C.c_int], None),
    "scSetResidualUnit": ([scModel, C.c_int], None),
    "scSetClusterVariant": ([scModel, C.c_int], None),
    "scGetStaticColours": ([scModel, _i, _i, _i], C.c_int),
    "scGetSolverPrecision": ([scModel], C.c_int),
    "scCreateClothBatch": ([scCollisionWorld, C.POINTER(scClothPatch), C.c_int], scClothPatch),
    "scGetBatchSize": ([scClothPatch], C.c_int),
    "scGetBatchInstance": ([scClothPatch, C.c_int, _i, _i], None),
    "scSetSolverMode": ([scModel, C.c_int], None),
    "scSetGridSolver": ([scModel, C.c_int, C.c_int], None),
    "scGetSolverChoice": ([scModel, _i, _f, C.c_int], C.c_int),
    "scGetBandPlan": ([scModel, _i], C.c_int),
    "scSetBandVariant": ([scModel, C.c_int], None),
    "scGetGridVariants": ([_i, C.c_int], C.c_int),
    "scSetBroadPhaseMode": ([scModel, C.c_int], None),
    "scGetBroadPhaseMode": ([scModel, _f], C.c_int),
    "scGetSolverIterations": ([scModel], C.c_int),
    "scGetResidual": ([scModel], C.c_float),
    "scSetResidualTarget": ([scModel, C.c_float, C.c_int], None),
    "scGetIterationTotal": ([scModel], C.c_int),
    "scSetWarmStart": ([scModel, _f, _f], C.c_bool),
    "scSetSampleBuffers": ([scModel, C.c_void_p, C.c_void_p], C.c_bool),
    "scMlpParamCount": ([], C.c_int),
    "scMlpForward": ([C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "scMlpGradients": ([C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "scMlpAdamStep": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float, C.c_void_p], C.c_int),
    "scGetConstraintOrder": ([scModel, C.c_int, _i, _i], C.c_int),
    "scGetNumBends": ([scModel], C.c_int),
    "scGetBends": ([scModel, _u], None),
    "scGetNumEdges": ([scModel], C.c_int),
    "scGetEdges": ([scModel, _i], None),
    "scGetNumContactsOfKind": ([scModel, C.c_int], C.c_int),
    "scGetSelfContacts": ([scModel, C.c_int, _i, _f], None),
    "scGetVertexContacts": ([scModel, _i, _f], None),
    "scGetTriContacts": ([scModel, _i, _f], None),
    "scGetEdgeContacts": ([scModel, _i, _f], None),
    "scGetCCDCandidates": ([scModel, C.c_int, _i, C.c_int], C.c_int),
    "scGetCollisionMeshNormals": ([scModel, _f], None),
    "scGetContactColours": ([scModel, C.c_int, _i], C.c_int),
    "scComputeVertexNormalsNoAlloc": ([C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p], C.c_int),
    "scGetLastError": ([], C.c_int),
    "scGetLastErrorString": ([], C.c_char_p),
    "scGetStatus": ([scClothPatch], C.c_int),
    "scSynchronize": ([scClothPatch], None),
    "scGetCudaStream": ([scClothPatch], C.c_void_p),
    "scGetGraphKernelCount": ([scClothPatch], C.c_int),
    "scSetDirectLaunch": ([scClothPatch, C.c_int], None),
    "scProfileSweep": ([scClothPatch, C.c_int, C.c_int], C.c_float),
    "scProbeClusterPhase": ([C.c_int, C.c_int], C.c_float),
    "scSetKernelTiming": ([scClothPatch, C.c_int], C.c_bool),
    "scGetKernelTiming": ([scClothPatch, _f, _i], C.c_int),
    "scRenderCloth": ([scClothPatch, _f, _f, C.c_int, C.c_int, C.c_void_p, C.c_void_p], C.c_int),
}

_lib = None


def lib():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m solidcloth_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def _fp(a):
    return a.ctypes.data_as(_f)


def _check(what: str):
    L = lib()
    msg = L.scGetLastErrorString()
    err = L.scGetLastError()
    if err:
        raise RuntimeError(f"{what}: error {err}: {msg.decode() if msg else ''}")


def v3(x) -> scVector3:
    return scVector3(float(x[0]), float(x[1]), float(x[2]))


class CollisionWorld:
    """Physics::CollisionWorld (Physics/CollisionWorld.h:10-29)."""

    def __init__(self):
        self.h = lib().scCreateCollisionWorld()

    def add_walls(self, box6):
        b = scAabb3(v3(box6[:3]), v3(box6[3:]))
        lib().scAddCollidable(self.h, lib().scCreateWalls(b))

    def add_sphere(self, center, radius):
        lib().scAddCollidable(self.h, lib().scCreateSphere(v3(center), float(radius)))

    def add_sdf(self, grid):
        vals = np.ascontiguousarray(grid.values, np.float32)
        b = scAabb3(v3(grid.box[:3]), v3(grid.box[3:]))
        h = lib().scCreateSDFGrid(grid.cells[0], grid.cells[1], grid.cells[2], b, _fp(vals))
        _check("scCreateSDFGrid")
        lib().scAddCollidable(self.h, h)

    def add_mesh(self, mesh):
        v = np.ascontiguousarray(mesh.vertices, np.float32)
        idx = np.ascontiguousarray(mesh.indices, np.uint32)
        h = lib().scCreateMeshCollider(_fp(v), v.shape[0], idx.ctypes.data_as(_u), idx.size)
        _check("scCreateMeshCollider")
        lib().scAddCollidable(self.h, h)

    def clear(self):
        lib().scClearCollidables(self.h)

    @property
    def num_collidables(self):
        return lib().scGetNumCollidables(self.h)

    def free(self):
        if self.h is not None:
            lib().scFreeCollisionWorld(self.h)
            self.h = None


class ClothModel:
    """Physics::ClothModel as seen through the scModel handle."""

    def __init__(self, handle, patch):
        self.h = handle
        self.patch = patch

    @property
    def num_particles(self):
        return lib().scGetNumParticles(self.h)

    def set_params(self, p):
        L = lib()
        L.scSetUnit(self.h, p.unit)
        L.scSetThickness(self.h, p.thickness)
        L.scSetTolerance(self.h, p.tolerance)
        L.scSetShearStiffness(self.h, p.shear)
        L.scSetBendStiffness(self.h, p.bend)
        L.scSetStretchStiffness(self.h, p.stretch)
        L.scSetPoisson(self.h, p.poisson)
        L.scSetFriction(self.h, p.friction)
        L.scSetNumIterations(self.h, int(p.iterations))
        L.scSetCollisionFlags(self.h, int(p.flags))
        L.scSetUseFEM(self.h, bool(p.fem))
        L.scSetDihedral(self.h, bool(p.dihedral))
        L.scSetFixedIterations(self.h, bool(p.fixed_iterations))
        L.scSetDragCoeff(self.h, p.drag)
        L.scSetSolverType(self.h, int(getattr(p, "solver", 1)))
        _check("set_params")

    def set_masses(self, masses):
        m = np.ascontiguousarray(masses, np.float32)
        lib().scSetMasses(self.h, _fp(m))
        _check("scSetMasses")

    def set_positions(self, pos):
        p = np.ascontiguousarray(pos, np.float32)
        lib().scSetParticlePositions(self.h, _fp(p))
        _check("scSetParticlePositions")

    def set_state(self, pos, prev, vel):
        a, b, c = (np.ascontiguousarray(x, np.float32) for x in (pos, prev, vel))
        lib().scSetParticleState(self.h, _fp(a), _fp(b), _fp(c))
        _check("scSetParticleState")

    def _get3(self, fn):
        out = np.zeros((self.num_particles, 3), np.float32)
        getattr(lib(), fn)(self.h, _fp(out))
        return out

    def positions(self):
        return self._get3("scGetParticlePositions")

    def velocities(self):
        return self._get3("scGetParticleVelocities")

    def prev_positions(self):
        return self._get3("scGetParticlePrevPositions")

    def collision_mesh_normals(self):
        return self._get3("scGetCollisionMeshNormals")

    def inv_masses(self):
        return np.array([lib().scGetParticleInvMass(self.h, i) for i in range(self.num_particles)], np.float32)

    def set_ccd(self, on: bool):
        lib().scSetSelfCCD(self.h, bool(on))

    def set_cluster_solver(self, on: bool):
        lib().scSetClusterSolver(self.h, bool(on))

    def solver_type(self) -> int:
        """ClothModel::GetSolver: 0 Jacobi, 1 Gauss-Seidel, 2-4 conjugate residual"""
        return int(lib().scGetSolverType(self.h))

    def set_solver_mode(self, mode: int):
        """0 autotuned (default), 1 cluster kernel, 2 grid kernel, 3 per-colour
        kernels, 4 band kernel (its own order)"""
        lib().scSetSolverMode(self.h, int(mode))
        _check("scSetSolverMode")

    def set_cluster_variant(self, variant: int):
        lib().scSetClusterVariant(self.h, int(variant))
        _check("scSetClusterVariant")

    def set_grid_solver(self, variant: int, blocks_per_sm: int):
        lib().scSetGridSolver(self.h, int(variant), int(blocks_per_sm))
        _check("scSetGridSolver")

    def set_band_variant(self, variant: int):
        """force the band kernel with 256 / 512 / 1024 threads per CTA (variant 0 / 1 / 2)"""
        lib().scSetBandVariant(self.h, int(variant))
        _check("scSetBandVariant")

    def band_plan(self):
        """(CTAs of the band solver's cluster or 0, particles per band, halo
        particles, in use) — scGetBandPlan"""
        out = np.zeros(4, np.int32)
        lib().scGetBandPlan(self.h, out.ctypes.data_as(_i))
        return tuple(int(x) for x in out)

    def solver_choice(self):
        """(kind, variant, CTAs per SM, threads) in use, and the last tuning's candidates"""
        out = np.zeros(4, np.int32)
        log = np.zeros((64, 4), np.float32)
        n = lib().scGetSolverChoice(self.h, out.ctypes.data_as(_i), log.ctypes.data_as(_f), 64)
        return tuple(int(x) for x in out), log[:min(n, 64)].copy()

    BROAD_WALKS = ("per-query stack walk", "warp packet")

    def set_broad_phase_mode(self, mode: int):
        """0 per-query walks, 1 warp packets, -1 tuned"""
        lib().scSetBroadPhaseMode(self.h, int(mode))
        _check("scSetBroadPhaseMode")

    def broad_phase_mode(self):
        """(walk in use, tuned ms of each walk in BROAD_WALKS order)"""
        ms = np.zeros(2, np.float32)
        mode = lib().scGetBroadPhaseMode(self.h, ms.ctypes.data_as(_f))
        return int(mode), ms.copy()

    def set_cluster_staging(self, on: bool):
        lib().scSetClusterStaging(self.h, bool(on))

    def set_fast_math(self, on: bool):
        """solver numerics: True = the fast build (FMA, approximate div/sqrt),
        False = IEEE, bit-exact with the reference's operation order"""
        lib().scSetSolverPrecision(self.h, int(bool(on)))
        _check("scSetSolverPrecision")

    def fast_math(self) -> bool:
        return bool(lib().scGetSolverPrecision(self.h))

    def constraint_order(self, kind):
        n = (lib().scGetNumTris(self.h), lib().scGetNumBends(self.h), lib().scGetNumLinks(self.h))[kind]
        order = np.zeros(n, np.int32)
        start = np.zeros(70, np.int32)
        nc = lib().scGetConstraintOrder(self.h, kind, order.ctypes.data_as(_i), start.ctypes.data_as(_i))
        return order, start[:nc + 1].copy()

    def tris(self):
        n = lib().scGetNumTris(self.h)
        out = np.zeros((n, 3), np.int32)
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        for t in range(n):
            lib().scGetTriangle(self.h, t, C.byref(a), C.byref(b), C.byref(c))
            out[t] = (a.value, b.value, c.value)
        return out

    def tri_rest(self):
        """(T, 10): du1 du2 dv1 dv2 invDet lu0 lv0 lu2 lv2 area"""
        out = np.zeros((lib().scGetNumTris(self.h), 10), np.float32)
        lib().scGetTriangleRest(self.h, _fp(out))
        return out

    def links(self):
        """(L, 2) indices and (L, 2) rest length / stiffness, in creation order"""
        n = lib().scGetNumLinks(self.h)
        idx = np.zeros((n, 2), np.uint32)
        a, b = C.c_int(), C.c_int()
        for k in range(n):
            lib().scGetLink(self.h, k, C.byref(a), C.byref(b))
            idx[k] = (a.value, b.value)
        rest = np.zeros((n, 2), np.float32)
        lib().scGetLinkRest(self.h, _fp(rest))
        return idx, rest

    def bends(self):
        n = lib().scGetNumBends(self.h)
        out = np.zeros((n, 4), np.uint32)
        lib().scGetBends(self.h, out.ctypes.data_as(_u))
        return out

    def num_edges(self) -> int:
        return int(lib().scGetNumEdges(self.h))

    def num_tris(self) -> int:
        return int(lib().scGetNumTris(self.h))

    def num_bends(self) -> int:
        return int(lib().scGetNumBends(self.h))

    def edges(self):
        n = lib().scGetNumEdges(self.h)
        out = np.zeros((n, 4), np.int32)
        lib().scGetEdges(self.h, out.ctypes.data_as(_i))
        return out

    def contacts(self, kind):
        """kind 0 vertex, 1 tri, 2 edge, 3 self VT, 4 self EE (oracle layout)."""
        L = lib()
        n = L.scGetNumContactsOfKind(self.h, kind)
        if kind == 0:
            a = np.zeros((n, 2), np.int32); f = np.zeros((n, 6), np.float32)
            L.scGetVertexContacts(self.h, a.ctypes.data_as(_i), _fp(f))
        elif kind == 1:
            a = np.zeros((n, 4), np.int32); f = np.zeros((n, 9), np.float32)
            L.scGetTriContacts(self.h, a.ctypes.data_as(_i), _fp(f))
        elif kind == 2:
            a = np.zeros((n, 3), np.int32); f = np.zeros((n, 8), np.float32)
            L.scGetEdgeContacts(self.h, a.ctypes.data_as(_i), _fp(f))
        else:
            a = np.zeros((n, 4), np.int32); f = np.zeros((n, 7), np.float32)
            L.scGetSelfContacts(self.h, kind, a.ctypes.data_as(_i), _fp(f))
        return a, f

    def ccd_candidates(self, kind, cap=1 << 24):
        out = np.zeros((cap, 2), np.int32)
        n = lib().scGetCCDCandidates(self.h, kind, out.ctypes.data_as(_i), cap)
        return out[:min(n, cap)].copy()

    def residual(self) -> float:
        """max |C| over the warp, weft and shear constraints at the current positions"""
        return float(lib().scGetResidual(self.h))

    def set_residual_target(self, tol: float, max_iterations: int, metres: bool = False):
        """iterate each substep until the update residual <= tol (at most
        max_iterations); the residual in metres or (default) in mean rest edges"""
        lib().scSetResidualUnit(self.h, int(bool(metres)))
        _check("scSetResidualUnit")
        lib().scSetResidualTarget(self.h, float(tol), int(max_iterations))
        _check("scSetResidualTarget")

    def set_warm_start(self, params, norm):
        """params (9347 FP32) and norm (27 FP32) host arrays; None turns it off"""
        if params is None:
            ok = lib().scSetWarmStart(self.h, None, None)
        else:
            p = np.ascontiguousarray(params, np.float32)
            n = np.ascontiguousarray(norm, np.float32)
            ok = lib().scSetWarmStart(self.h, p.ctypes.data_as(_f), n.ctypes.data_as(_f))
        _check("scSetWarmStart")
        return bool(ok)

    def set_sample_buffers(self, features_ptr, targets_ptr):
        """device pointers (numSteps x N x 12, numSteps x N x 3) or 0 to stop"""
        ok = lib().scSetSampleBuffers(self.h, C.c_void_p(features_ptr or None), C.c_void_p(targets_ptr or None))
        _check("scSetSampleBuffers")
        return bool(ok)

    def iteration_total(self) -> int:
        """Gauss-Seidel iterations of all substeps since the last call"""
        return int(lib().scGetIterationTotal(self.h))

    def solver_iterations(self):
        return lib().scGetSolverIterations(self.h)

    def static_colours(self):
        """(triangle colours, triangle colour count, edge colours, edge colour count):
        the static colouring of the triangle and edge collider contacts"""
        L = lib()
        tri = np.zeros(max(1, self.num_tris()), np.int32)
        edge = np.zeros(max(1, self.num_edges()), np.int32)
        cnt = np.zeros(2, np.int32)
        L.scGetStaticColours(self.h, tri.ctypes.data_as(_i), edge.ctypes.data_as(_i), cnt.ctypes.data_as(_i))
        return tri[:self.num_tris()].copy(), int(cnt[0]), edge[:self.num_edges()].copy(), int(cnt[1])

    def contact_colours(self, cls):
        counts = np.zeros(128, np.int32)
        used = lib().scGetContactColours(self.h, int(cls), counts.ctypes.data_as(_i))
        return counts[:used].copy()


class ClothPatch:
    """Physics::ClothPatch (Physics/ClothPatch.h:24-72) on one GPU."""

    def __init__(self, world: CollisionWorld):
        self.world = world
        self.h = lib().scCreateClothPatch(world.h)
        _check("scCreateClothPatch")
        self.model = ClothModel(lib().scGetClothModel(self.h), self)

    def init_grid(self, div_x, div_y, inc, offset, horizontal=True, attached=False):
        lib().scInitCloth(self.h, int(div_x), int(div_y), float(inc), v3(offset), bool(horizontal), bool(attached))
        _check("scInitCloth")

    def init_mesh(self, vertices, indices, uvs=None, colors=None, offset=(0, 0, 0), attached=False):
        """ClothPatch::Init(mesh, offset, attached)"""
        v = np.ascontiguousarray(vertices, np.float32)
        idx = np.ascontiguousarray(indices, np.uint32)
        u = None if uvs is None else np.ascontiguousarray(uvs, np.float32)
        c = None if colors is None else np.ascontiguousarray(colors, np.float32)
        lib().scInitClothMesh(self.h, _fp(v), v.shape[0], idx.ctypes.data_as(_u), idx.size,
                              None if u is None else _fp(u), None if c is None else _fp(c), v3(offset), bool(attached))
        _check("scInitClothMesh")

    def init_obj(self, path, offset=(0, 0, 0), attached=False):
        ok = lib().scInitClothObj(self.h, str(path).encode(), v3(offset), bool(attached))
        _check("scInitClothObj")
        return bool(ok)

    def particle_map(self):
        n = lib().scGetMeshParticleMap(self.h, None, 0)
        m = np.zeros(n, np.int32)
        lib().scGetMeshParticleMap(self.h, m.ctypes.data_as(_i), n)
        return m

    def set_num_steps(self, n):
        lib().scSetNumSteps(self.h, int(n))

    def step(self, dt):
        lib().scStepCloth(self.h, float(dt))
        _check("scStepCloth")

    def update_mesh(self):
        lib().scUpdateClothMesh(self.h)
        _check("scUpdateClothMesh")

    def synchronize(self):
        lib().scSynchronize(self.h)

    def status(self):
        return lib().scGetStatus(self.h)

    def cuda_stream(self) -> int:
        return lib().scGetCudaStream(self.h) or 0

    def graph_kernel_count(self) -> int:
        return lib().scGetGraphKernelCount(self.h)

    def set_direct_launch(self, on: bool):
        """launch each substep's kernels directly instead of replaying the frame graph"""
        lib().scSetDirectLaunch(self.h, int(bool(on)))
        _check("scSetDirectLaunch")

    def profile_sweep(self, kind: int, reps: int = 50) -> float:
        ms = lib().scProfileSweep(self.h, int(kind), int(reps))
        _check("scProfileSweep")
        return float(ms)

    def set_kernel_timing(self, frames: int):
        """bracket the solve and broad phases of the next `frames` frames with CUDA events"""
        ok = lib().scSetKernelTiming(self.h, int(frames))
        _check("scSetKernelTiming")
        return bool(ok)

    def kernel_timing(self):
        """{section: (total ms, instances)} since the last read, and the frames covered"""
        ms = np.zeros(4, np.float32)
        cnt = np.zeros(4, np.int32)
        frames = lib().scGetKernelTiming(self.h, ms.ctypes.data_as(_f), cnt.ctypes.data_as(_i))
        names = ("gs_solve", "ccd_broad_ee", "ccd_broad_vt", "colliders")
        return {n: (float(ms[k]), int(cnt[k])) for k, n in enumerate(names)}, int(frames)

    def render(self, view_proj, width: int, height: int, light=(0.0, 2.0, 2.0), eye=(0.0, 1.0, 2.0),
               kd=(0.8, 0.3, 0.3), ks=(0.2, 0.2, 0.2), shininess: float = 32.0, flip: float = 1.0,
               background: float = 0.3, flags: int = 0, return_zbuf: bool = False):
        """The current mesh drawn with the demo's Phong program into a CUDA tensor
        (height, width, 4); with return_zbuf also the per-pixel (depth key << 32 |
        triangle) words (int64, -1 where nothing was drawn)."""
        import torch
        vp = np.ascontiguousarray(view_proj, np.float32).reshape(16)
        prm = np.array([*light, *eye, *kd, *ks, shininess, flip, background, flags], np.float32)
        img = torch.empty((height, width, 4), dtype=torch.float32, device="cuda")
        z = torch.empty((height, width), dtype=torch.int64, device="cuda")
        rc = lib().scRenderCloth(self.h, _fp(vp), _fp(prm), int(width), int(height), img.data_ptr(), z.data_ptr())
        if rc != 0:
            _check("scRenderCloth")
            raise RuntimeError(f"scRenderCloth: error {rc}")
        return (img, z) if return_zbuf else img

    def mesh_buffers(self):
        L = lib()
        m = L.scGetClothMesh(self.h)
        nv, ni = L.scGetMeshVertexCount(m), L.scGetMeshIndexCount(m)
        v = np.ctypeslib.as_array(C.cast(L.scGetMeshVertexBuffer(m), _f), shape=(nv, 3)).copy()
        nb = L.scGetMeshNormalBuffer(m)
        n = np.ctypeslib.as_array(C.cast(nb, _f), shape=(nv, 3)).copy() if nb else None
        idx = np.ctypeslib.as_array(L.scGetMeshIndexBuffer(m), shape=(ni,)).copy()
        return v, n, idx

    def free(self):
        if self.h is not None:
            lib().scFreeClothPatch(self.h)
            self.h = None


class ClothBatch(ClothPatch):
    """Independent clothes stepped as one patch (scCreateClothBatch)."""

    def __init__(self, parts):
        self.world = CollisionWorld()
        arr = (scClothPatch * len(parts))(*[p.h for p in parts])
        self.h = lib().scCreateClothBatch(self.world.h, arr, len(parts))
        _check("scCreateClothBatch")
        if not self.h.ptr:
            raise RuntimeError("scCreateClothBatch failed")
        self.model = ClothModel(lib().scGetClothModel(self.h), self)

    def size(self) -> int:
        return int(lib().scGetBatchSize(self.h))

    def instance(self, k: int):
        """(first particle, particle count) of instance k"""
        a, n = C.c_int(), C.c_int()
        lib().scGetBatchInstance(self.h, int(k), C.byref(a), C.byref(n))
        _check("scGetBatchInstance")
        return a.value, n.value


def load_batch(scenes_, ccd: bool | None = None):
    """One batch patch over a list of scenes.Scene (each with its own colliders);
    the per-scene patches are built, merged and freed."""
    parts = [load_scene(s, ccd) for s in scenes_]
    b = ClothBatch([p for _, p in parts])
    for w, p in parts:
        p.free()
        w.free()
    return b


class SDFHandle:
    """An SDF collidable made outside a world (from a mesh or a file)."""

    def __init__(self, h):
        if not h:
            raise RuntimeError("SDF creation failed")
        self.h = h

    @classmethod
    def from_mesh(cls, vertices, indices, cells, box6):
        v = np.ascontiguousarray(vertices, np.float32)
        idx = np.ascontiguousarray(indices, np.uint32)
        b = scAabb3(v3(box6[:3]), v3(box6[3:]))
        h = lib().scCreateSDFFromMesh(_fp(v), v.shape[0], idx.ctypes.data_as(_u), idx.size,
                                      int(cells[0]), int(cells[1]), int(cells[2]), b)
        _check("scCreateSDFFromMesh")
        return cls(h)

    @classmethod
    def load(cls, path):
        h = lib().scLoadSDF(str(path).encode())
        _check("scLoadSDF")
        return cls(h)

    def save(self, path):
        ok = lib().scSaveSDF(self.h, str(path).encode())
        _check("scSaveSDF")
        return bool(ok)

    def grid(self):
        """(cells (3,), box (6,), values ((nx+1)(ny+1)(nz+1),) x fastest)"""
        cells = np.zeros(3, np.int32)
        box = np.zeros(6, np.float32)
        n = lib().scGetSDFGrid(self.h, cells.ctypes.data_as(_i), _fp(box), None, 0)
        vals = np.zeros(n, np.float32)
        lib().scGetSDFGrid(self.h, None, None, _fp(vals), n)
        return cells, box, vals

    def free(self):
        if self.h:
            lib().scFreeCollidable(self.h)
            self.h = None


def grid_variants():
    """(threads per CTA, FEM constraints per thread, bends per thread) per grid-solver variant"""
    info = np.zeros((64, 3), np.int32)
    n = lib().scGetGridVariants(info.ctypes.data_as(_i), 64)
    return [tuple(int(x) for x in info[k]) for k in range(n)]


def load_scene(scene: Scene, ccd: bool | None = None):
    """Build world + patch for a scenes.Scene exactly as the oracles do."""
    w = CollisionWorld()
    if scene.walls is not None:
        w.add_walls(scene.walls)
    for (c, r) in scene.spheres:
        w.add_sphere(c, r)
    for g in scene.sdfs:
        w.add_sdf(g)
    for m in scene.meshes:
        w.add_mesh(m)
    p = ClothPatch(w)
    p.model.set_params(scene.params)
    p.set_num_steps(scene.params.substeps)
    p.init_grid(scene.n, scene.n, scene.inc, scene.offset, True, scene.attached)
    p.model.set_masses(scene.masses)
    p.model.set_positions(scene.positions)
    p.model.set_ccd(scene.ccd if ccd is None else ccd)
    return w, p
