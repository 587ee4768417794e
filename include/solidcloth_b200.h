/*
 * solidcloth_b200.h — C ABI of the B200 cloth step (libsolidcloth_b200.so).
 *
 * Drop-in for the SolidCloth "ClothAPI" (Demo/ClothAPI.h:65-146): the same sc*
 * entry points, handle structs and argument meaning, so a caller that binds the
 * reference's ClothLib binds this library by changing the library name. Where
 * the reference passes C++ references (Vector3&, int&) this header declares the
 * ABI-identical pointers; Math::Vector3 is 3 packed floats (scVector3) and
 * Geometry::Aabb3 two of them (scAabb3).
 *
 * Differences, all additive or forced by the absence of C++ types in a C ABI:
 *   - scCreateSDF(Geometry::SDF*) / scCreateMesh(Geometry::Mesh*) take caller-owned
 *     C++ objects in the reference; here the grid / mesh data are passed as
 *     arrays (scCreateSDFGrid, scCreateMeshCollider).
 *   - scComputeStrainMap fills a caller array instead of a std::vector.
 *   - The step runs asynchronously on the patch's CUDA stream; every getter
 *     synchronises first, so results are visible exactly as in the reference.
 *   - Errors: the reference has none (invalid handles are UB). Every entry point
 *     here records failures; scGetLastError() returns and clears the last one.
 * Each declaration cites the reference declaration it replaces.
 */
#ifndef SOLIDCLOTH_B200_H
#define SOLIDCLOTH_B200_H

#include <stdbool.h>

#if defined(_WIN32)
#define SCEXP __declspec(dllexport)
#else
#define SCEXP __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef void* scHandle;                                 /* Demo/ClothAPI.h:9 */
typedef struct scClothPatch { void* ptr; } scClothPatch; /* Demo/ClothAPI.h:11-17 */
typedef struct scCollisionWorld { void* ptr; } scCollisionWorld; /* :19-22 */
typedef struct scMesh { void* ptr; } scMesh;            /* :24-27 */
typedef struct scModel { void* ptr; } scModel;          /* :29-32 */
typedef struct scVector3 { float x, y, z; } scVector3;  /* Math::Vector3 */
typedef struct scVector2 { float x, y; } scVector2;     /* Math::Vector2 */
typedef struct scAabb3 { scVector3 min, max; } scAabb3; /* Geometry::Aabb3 */
typedef struct scQuaternion { float s; scVector3 v; } scQuaternion; /* Math::Quaternion */

enum scCollFlags                                        /* Demo/ClothAPI.h:34-41 */
{
    scCollisionFlagVertices = 1,
    scCollisionFlagTriangles = 2,
    scCollisionFlagSelf = 4,
    scCollisionFlagWalls = 8,
    scCollisionFlagEdges = 16,
};

enum scCollidableType                                   /* Demo/ClothAPI.h:43-53 */
{
    scCollidableTypeInvalid,
    scCollidableTypeWalls,
    scCollidableTypeSlab,
    scCollidableTypeSphere,
    scCollidableTypeMesh,
    scCollidableTypeBox,
    scCollidableTypeCapsule,
    scCollidableTypeSDF,
};

/* ---- collision world (Demo/ClothAPI.h:68-74) ---- */
SCEXP scCollisionWorld scCreateCollisionWorld(void);
SCEXP void scFreeCollisionWorld(scCollisionWorld collWorld);
SCEXP void scClearCollidables(scCollisionWorld collWorld);
SCEXP int scGetNumCollidables(scCollisionWorld collWorld);
/* Transfers ownership of the collidable to the world (Demo/ClothAPI.cpp:38-43). */
SCEXP void scAddCollidable(scCollisionWorld collWorld, scHandle collidable);
SCEXP scHandle scGetCollidable(scCollisionWorld collWorld, int i);

/* ---- collidables (Demo/ClothAPI.h:77-87) ---- */
SCEXP scHandle scCreateWalls(scAabb3 box);
SCEXP scHandle scCreateSphere(scVector3 center, float radius);
/* Stored and reported by scGetCapsuleInfo; the GPU step ignores capsules. */
SCEXP scHandle scCreateCapsule(scVector3 c, float rad, float halfHeight, scQuaternion quat);
/* Replaces scCreateSDF(Geometry::SDF*) (Demo/ClothAPI.h:80): a (nx+1)(ny+1)(nz+1)
   float grid over `box`, x fastest, as Geometry::SDF::Create(nx, ny, nz, box) +
   values + ComputeGradient() (Geometry/SDF.cpp:10-56,210-256). Values are copied. */
SCEXP scHandle scCreateSDFGrid(int nx, int ny, int nz, scAabb3 box, const float* values);
/* SDF::Create(nx, ny, nz, box) + SDF::CreateFromMesh (Geometry/SDF.cpp:10-18,58-76),
   computed on the GPU: every grid node's distance to the nearest triangle found
   through the mesh tree ComputeMeshTree(mesh, ATF_TRIANGLES, 10, 0.1) builds. As
   in the reference, with its default delta normal the field is unsigned.
   Returns an SDF collidable (gradient computed). Addition. */
SCEXP scHandle scCreateSDFFromMesh(const float* vertices, int nv, const unsigned* indices, int ni,
                                   int nx, int ny, int nz, scAabb3 box);
/* SDF::WriteToFile / SDF::LoadFromFile (Geometry/SDF.cpp:78-151): the reference's
   binary format (3 ints, box and values as doubles). Additions. */
SCEXP bool scSaveSDF(scHandle sdf, const char* path);
SCEXP scHandle scLoadSDF(const char* path);
/* addition: an SDF collidable's grid (cells per side, box min / max, up to cap
   values); returns the value count */
SCEXP int scGetSDFGrid(scHandle sdf, int* cells3, float* box6, float* values, int cap);
/* addition: delete a collidable that was never added to a world (a world owns
   the collidables added to it) */
SCEXP void scFreeCollidable(scHandle collidable);
/* Replaces scCreateMesh(Geometry::Mesh*) (Demo/ClothAPI.h:81): a triangle mesh
   prepared as Demo/ClothDemo.cpp:100-103 does (normals, edges, edge one-rings).
   Arrays are copied. */
SCEXP scHandle scCreateMeshCollider(const float* vertices, int numVertices, const unsigned* indices, int numIndices);
SCEXP int scGetCollidableType(scHandle collidable);
/* Opaque here: the reference returns its Geometry::AabbTree*, a C++ type. */
SCEXP void* scGetMeshTree(scHandle collMesh);
SCEXP void scGetWallsInfo(scHandle walls, scAabb3* box);
SCEXP void scGetSphereInfo(scHandle sphere, float* radius, scVector3* center);
SCEXP void scGetCapsuleInfo(scHandle capsule, float* radius, float* halfHeight, scVector3* center, scQuaternion* rot);

/* ---- cloth patch (Demo/ClothAPI.h:91-99) ---- */
SCEXP scClothPatch scCreateClothPatch(scCollisionWorld collWorld);
SCEXP void scFreeClothPatch(scClothPatch patch);
/* Batches (additions, no reference counterpart): one patch that steps `count`
   initialised patches as independent instances in one CUDA graph per frame and
   one solver launch per substep. The parts must share every solver parameter and
   the substep count; each keeps the colliders of its own world (vertex, wall and
   self collisions; triangle / edge collider contacts are not supported). The
   parts' state is copied: they may be freed afterwards. The batch is an ordinary
   patch for scStepCloth and the getters; instance k owns particles
   [first, first + num) of its model. */
SCEXP scClothPatch scCreateClothBatch(scCollisionWorld world, const scClothPatch* parts, int count);
SCEXP int scGetBatchSize(scClothPatch batch);
SCEXP void scGetBatchInstance(scClothPatch batch, int k, int* firstParticle, int* numParticles);
SCEXP scModel scGetClothModel(scClothPatch patch);
SCEXP scMesh scGetClothMesh(scClothPatch patch);
SCEXP void scInitCloth(scClothPatch patch, int divX, int divY, float inc, scVector3 offset, bool horizontal, bool attached);
/* ClothPatch::Init(mesh, offset, attached) (Physics/ClothPatch.cpp:42-133), which
   the reference's C API does not expose: a cloth from a triangle mesh (nv
   vertices, ni indices); uvs (nv x 2) give the rest shape, colors (nv x 3) pin
   vertices whose red channel is non-zero when `attached`; both may be NULL.
   Coincident vertices merge into one particle (the reference's merge). The
   patch's mesh buffers then hold the particles and their triangles;
   scGetMeshParticleMap gives the input vertex -> particle map. Additions. */
SCEXP void scInitClothMesh(scClothPatch patch, const float* vertices, int nv, const unsigned* indices, int ni,
                           const float* uvs, const float* colors, scVector3 offset, bool attached);
SCEXP int scGetMeshParticleMap(scClothPatch patch, int* map, int cap);
/* addition: scInitClothMesh from a Wavefront OBJ file (v, vt, f; polygons fanned
   into triangles; one vertex per face corner with its uv, as the demo's mesh
   importer delivers meshes, Geometry/Assets.cpp:103); false if unreadable */
SCEXP bool scInitClothObj(scClothPatch patch, const char* path, scVector3 offset, bool attached);
/* The hot entry point: ClothPatch::Step (Demo/ClothAPI.cpp:146-150). */
SCEXP void scStepCloth(scClothPatch patch, float dt);
SCEXP void scUpdateClothMesh(scClothPatch patch);
/* Replaces scComputeStrainMap(patch, std::vector<Vector3>&): colors has one
   scVector3 per particle. */
SCEXP void scComputeStrainMap(scClothPatch patch, scVector3* colors);

/* ---- cloth model (Demo/ClothAPI.h:102-138) ---- */
SCEXP int scGetNumParticles(scModel model);
SCEXP void scGetParticlePos(scModel model, int i, scVector3* pos);
SCEXP float scGetParticleInvMass(scModel model, int i);
SCEXP int scGetNumTris(scModel model);
SCEXP void scGetTriangle(scModel model, int i, int* i1, int* i2, int* i3);
SCEXP void scGetTriangleInfo(scModel model, int i, float* invDet, scVector2* du, scVector2* dv, scVector2* s);
SCEXP int scGetNumQuads(scModel model);
SCEXP void scGetQuad(scModel model, int i, int* i1, int* i2, int* i3, int* i4);
SCEXP int scGetNumLinks(scModel model);
SCEXP void scGetLink(scModel model, int i, int* i1, int* i2);
SCEXP int scGetNumContacts(scModel model);
SCEXP void scGetContact(scModel model, int i, scVector3* point, scVector3* normal);
SCEXP int scGetNumTriContacts(scModel model);
SCEXP void scGetTriContact(scModel model, int i, scVector3* point, scVector3* normal);
SCEXP int scGetCollisionFlags(scModel model);
SCEXP void scSetCollisionFlags(scModel model, int val);
SCEXP float scGetThickness(scModel model);
SCEXP void scSetThickness(scModel model, float val);
SCEXP float scGetTolerance(scModel model);
SCEXP void scSetTolerance(scModel model, float val);
SCEXP float scGetFriction(scModel model);
SCEXP void scSetFriction(scModel model, float val);
SCEXP int scGetNumIterations(scModel model);
SCEXP void scSetNumIterations(scModel model, int val);
SCEXP bool scGetUseFEM(scModel model);
SCEXP void scSetUseFEM(scModel model, bool val);
/* Opaque here (Demo/ClothAPI.h:134 returns Geometry::AabbTree*). */
SCEXP void* scGetClothTree(scModel model);
SCEXP void scAddMouseSpring(scModel model, int i1, int i2, int i3, scVector3 coords, scVector3 p);
SCEXP void scUpdateMouseSpring(scModel model, scVector3 p);
SCEXP void scRemoveMouseSpring(scModel model);

/* ---- mesh (Demo/ClothAPI.h:141-145); borrowed pointers, valid until the next
   scUpdateClothMesh / scInitCloth / scFreeClothPatch ---- */
SCEXP int scGetMeshVertexCount(scMesh mesh);
SCEXP int scGetMeshIndexCount(scMesh mesh);
SCEXP scVector3* scGetMeshNormalBuffer(scMesh mesh);
SCEXP scVector3* scGetMeshVertexBuffer(scMesh mesh);
SCEXP unsigned int* scGetMeshIndexBuffer(scMesh mesh);

/* ---- additions: setters the reference has only on the C++ ClothModel /
   ClothPatch (Physics/ClothModel.h:110-146, Physics/ClothPatch.h:49-50) ---- */
SCEXP void scSetUnit(scModel model, float val);
SCEXP float scGetUnit(scModel model);
SCEXP void scSetShearStiffness(scModel model, float val);
SCEXP void scSetBendStiffness(scModel model, float val);
SCEXP void scSetStretchStiffness(scModel model, float val);
SCEXP void scSetPoisson(scModel model, float val);
SCEXP void scSetDragCoeff(scModel model, float val);
SCEXP void scSetDihedral(scModel model, bool val);
/* ClothModel::SetSolver / GetSolver (Physics/ClothModel.h:137-138; C++ members, not
   in the reference's C API): the SolverType ClothModelPBD::Step dispatches on
   (Physics/ClothPBD.cpp:293-298). 1 SOLVER_GAUSS_SEIDEL (default), 0 SOLVER_JACOBI
   (SolveJacobi: links only, omega 0.5), 2-4 the conjugate-residual SolveCR (links
   only). Other values are rejected (SC_ERR_ARG). */
SCEXP void scSetSolverType(scModel model, int type);
SCEXP int scGetSolverType(scModel model);
SCEXP void scSetSelfShrink(scModel model, float val);
SCEXP void scSetNumSteps(scClothPatch patch, int val);
SCEXP int scGetNumSteps(scClothPatch patch);
/* ClothModel::SetMasses (Physics/ClothModel.cpp:45-52): mass 0 pins a particle. */
SCEXP void scSetMasses(scModel model, const float* masses);
SCEXP void scSetParticleInvMass(scModel model, int i, float invMass);
/* ClothModel::SetPositions (Physics/ClothModel.cpp:38-43), bulk xyz; also sets
   the previous positions, as a freshly initialised patch has them equal. */
SCEXP void scSetParticlePositions(scModel model, const float* xyz);
SCEXP void scGetParticlePositions(scModel model, float* xyz);
SCEXP void scGetParticleVelocities(scModel model, float* xyz);
SCEXP void scGetParticlePrevPositions(scModel model, float* xyz);
SCEXP void scSetParticleState(scModel model, const float* pos, const float* prev, const float* vel);
/* Fixed iteration count: bypasses the GS early exit (Physics/ClothPBD.cpp:357),
   which in FEM mode otherwise stops after one iteration without contacts. */
SCEXP void scSetFixedIterations(scModel model, bool val);
/* Continuous vertex-triangle / edge-edge self-collision
   (Physics/SelfCollisionDetector.cpp), appended to the self contacts each substep. */
SCEXP void scSetSelfCCD(scModel model, bool val);
SCEXP int scGetSolverIterations(scModel model);
/* addition (no reference counterpart): constraint residual of the current
   positions, max |C| over every triangle's warp, weft and shear constraint (the
   quantities Physics/ClothPBD.cpp:66-99 projects); bends are excluded because a
   draped cloth holds them away from zero. -1 before the first step. */
SCEXP float scGetResidual(scModel model);
/* addition: tol > 0 makes every substep's Gauss-Seidel loop run until its update
   residual — the largest particle displacement of the last iteration divided by
   the mean rest edge length — is <= tol, at most maxIterations iterations (the
   reference's own exit test is then off); tol = 0 restores iteration counting.
   (The constraint residual above does not vanish at convergence: the shear
   constraint is compliant and contacts hold the cloth strained.) */
SCEXP void scSetResidualTarget(scModel model, float tol, int maxIterations);
/* addition: the update residual's unit: 0 (default) = mean rest edge lengths,
   1 = metres (the largest displacement of the last iteration itself) */
SCEXP void scSetResidualUnit(scModel model, int unit);
/* addition: Gauss-Seidel iterations run by all substeps since the last call */
SCEXP int scGetIterationTotal(scModel model);

/* ---- additions: learned warm start (no reference counterpart) ----
   A per-particle MLP 12 -> 64 -> 64 -> 64 -> 3 (GELU; BF16 weights and
   activations on the tensor cores, FP32 accumulation) maps a particle's features
   after the substep's prediction to a position correction that is applied before
   the Gauss-Seidel loop. Features: predicted minus previous position (3),
   velocity (3), mean strain of the incident edges (1), collision-mesh normal (3),
   distance to the first sphere / SDF collider (1, clamped to +-1), the previous
   substep's solver correction along that normal (1). params: scMlpParamCount() FP32 values, W[out][in] row-major per
   layer then the layer's bias; norm: feature mean (12), 1 / feature std (12),
   output scale (3). params = NULL turns the warm start off. */
SCEXP bool scSetWarmStart(scModel model, const float* params, const float* norm);
/* Record every substep of the next frames: features (numSteps x N x 12) after the
   prediction and targets (numSteps x N x 3) = solved minus predicted positions,
   into caller-owned DEVICE buffers; NULL stops recording. */
SCEXP bool scSetSampleBuffers(scModel model, float* features, float* targets);
SCEXP int scMlpParamCount(void);
/* Device-pointer training and inference on `stream` (a cudaStream_t, 0 = legacy):
   Y = MLP(X) * output scale for S rows; gradients of mean((MLP(X) - T / scale)^2)
   (grad and loss are overwritten); one Adam step (beta 0.9 / 0.999, eps 1e-8).
   Return 0 or an error code. */
SCEXP int scMlpForward(const float* X, int S, const float* params, const float* norm, float* Y, void* stream);
SCEXP int scMlpGradients(const float* X, const float* T, int S, const float* params, const float* norm,
                         float* grad, float* loss, void* stream);
SCEXP int scMlpAdamStep(float* params, const float* grad, float* m, float* v, int step, float lr, void* stream);
/* true (default): the Gauss-Seidel loop of a substep runs as one thread-block
   cluster with the particles in distributed shared memory, when the cloth fits
   (up to 131,072 particles); false: one kernel per colour. Same results. */
SCEXP void scSetClusterSolver(scModel model, bool val);
/* Solver for the Gauss-Seidel loop (additions, no reference counterpart).
   0 = autotuned at the first step (default: the fastest of the cluster kernel,
   the grid-resident cooperative kernel's variants and the per-colour kernels,
   timed on this cloth), 1 = cluster kernel (clothes up to 131,072 particles),
   2 = grid kernel (tuned variant), 3 = per-colour kernels, 4 = band-parallel
   kernel (clothes with a band plan, scGetBandPlan; its thread count timed at
   the first step). Modes 0-3 give identical results (the colour order); the
   band kernel sweeps in its own order (interior records of every band, then
   boundary records), which scGetConstraintOrder reports while it is in use.
   scSetClusterSolver(true/false) is mode 1 / 3. */
SCEXP void scSetSolverMode(scModel model, int mode);
/* force grid variant `variant` (0 .. scGetGridVariants()-1) with blocksPerSm CTAs per SM */
SCEXP void scSetGridSolver(scModel model, int variant, int blocksPerSm);
/* force the cluster kernel with 1 (variant 0) or 2 (variant 1) constraints per thread */
SCEXP void scSetClusterVariant(scModel model, int variant);
/* out4 = {kind, grid variant, CTAs per SM, threads per CTA} of the solver in use;
   tuneMs (4 floats per candidate: kind, variant, CTAs per SM, ms per substep)
   gets up to cap candidates of the last tuning; returns the candidate count */
SCEXP int scGetSolverChoice(scModel model, int* out4, float* tuneMs, int cap);
/* force the band-parallel kernel with 256 (variant 0), 512 (1) or 1024 (2)
   threads per CTA (addition; SC_ERR_UNSUPPORTED without a band plan) */
SCEXP void scSetBandVariant(scModel model, int variant);
/* Band plan of the band-parallel solver (addition): out4 = {CTAs of its
   cluster (0: no plan), particles per band, halo particles, 1 if it is the
   solver in use}; returns 1 if the cloth has a plan. */
SCEXP int scGetBandPlan(scModel model, int* out4);
/* Continuous-collision broad phase walk (additions): 0 = one tree walk per query
   (lane), 1 = warp packets (32 neighbouring queries walk together, broadcast
   node loads), -1 (default) = timed at the first step and the faster kept. Same
   candidate sets. Either walk stops a query at 128 candidates; those queries are
   finished by a second pass, one warp per query. scGetBroadPhaseMode returns the
   walk in use and, in ms2, the tuned times of both (ms per substep's detection). */
SCEXP void scSetBroadPhaseMode(scModel model, int mode);
SCEXP int scGetBroadPhaseMode(scModel model, float* ms2);
/* info3 = {threads per CTA, FEM constraints per thread, bends per thread} per variant */
SCEXP int scGetGridVariants(int* info3, int cap);
/* true (default): the cluster solver copies each CTA's FEM and bend records to
   shared memory once per substep when they fit; false: read them from global
   memory in every sweep. Same results. */
SCEXP void scSetClusterStaging(scModel model, bool val);
/* Numerics of the Gauss-Seidel projections and contact solves. 0 (default):
   IEEE division and square root without FMA contraction, the reference's
   operation order bit for bit. 1: the fast build of the same solver (FMA
   contraction, approximate division and square root): every projection within
   1e-5 relative of the IEEE one. Detection (boxes, candidate pairs, contacts)
   is exact in both. Other values are rejected (SC_ERR_ARG). */
SCEXP void scSetSolverPrecision(scModel model, int mode);
SCEXP int scGetSolverPrecision(scModel model);

/* ---- additions: inspection for parity checks ---- */
/* kind 0: FEM triangles, 1: bends, 2: links. Writes the solve order (a permutation) and
   returns the number of colours; colourStart gets numColours+1 offsets if not NULL. */
SCEXP int scGetConstraintOrder(scModel model, int kind, int* order, int* colourStart);
SCEXP int scGetNumBends(scModel model);
/* Static colours the triangle and edge collider contacts are solved by: each
   triangle's colour (its FEM colour; T ints) and each collision-mesh edge's
   (E ints), counts2 = {triangle colours, edge colours}; returns E. A contact's
   colour is its triangle's / edge's plus the colour count times its collider's
   index among the sphere, SDF and mesh colliders (capped at 127). */
SCEXP int scGetStaticColours(scModel model, int* triColour, int* edgeColour, int* counts2);
/* FEM rest data of every triangle: du1 du2 dv1 dv2 invDet lu0 lv0 lu2 lv2 area
   (Physics/ClothTypes.h:37-62); links' rest length and stiffness */
SCEXP void scGetTriangleRest(scModel model, float* rest10);
SCEXP void scGetLinkRest(scModel model, float* rest2);
SCEXP void scGetBends(scModel model, unsigned* idx4);
SCEXP int scGetNumEdges(scModel model);
SCEXP void scGetEdges(scModel model, int* e4);
/* kind 0 vertex, 1 triangle, 2 edge, 3 self vertex-triangle, 4 self edge-edge */
SCEXP int scGetNumContactsOfKind(scModel model, int kind);
/* self contacts (kind 3/4): idx4 = i1..i4, f7 = normal xyz, w1, w2, w3, side */
SCEXP void scGetSelfContacts(scModel model, int kind, int* idx4, float* f7);
/* vertex contacts in list order: idx2 = particle, feature; f6 = point, normal */
SCEXP void scGetVertexContacts(scModel model, int* idx2, float* f6);
/* triangle contacts: idx4 = i1 i2 i3 feature; f9 = point normal w */
SCEXP void scGetTriContacts(scModel model, int* idx4, float* f9);
/* edge contacts: idx3 = i1 i2 feature; f8 = point normal w1 w2 */
SCEXP void scGetEdgeContacts(scModel model, int* idx3, float* f8);
/* continuous-collision broad-phase pairs of the last substep:
   kind 0 -> (vertex, triangle), kind 1 -> (edge, edge), sorted; returns the number
   of pairs held (a list longer than the pair store sets status bit 4) */
SCEXP int scGetCCDCandidates(scModel model, int kind, int* pairs, int cap);
/* contact classes of the last substep (0 edge, 1 triangle, 2 self vertex-triangle,
   3 self edge-edge): writes the per-colour counts of the independent-set
   colouring into counts[0..127] (may be NULL) and returns the colours used */
SCEXP int scGetContactColours(scModel model, int cls, int* counts);
/* collision-mesh (prev positions) vertex normals as of the last mesh update */
SCEXP void scGetCollisionMeshNormals(scModel model, float* xyz);

/* ---- additions: errors and synchronisation ---- */
SCEXP int scGetLastError(void);
SCEXP const char* scGetLastErrorString(void);
/* device-side status bits of the last steps (overflow of fixed-capacity
   contact slots etc.); clears them */
SCEXP int scGetStatus(scClothPatch patch);
SCEXP void scSynchronize(scClothPatch patch);

/* ---- additions: measurement ---- */
/* the patch's CUDA stream (cudaStream_t), for events around scStepCloth */
SCEXP void* scGetCudaStream(scClothPatch patch);
/* kernel nodes in the frame graph of the last scStepCloth (launches per frame) */
SCEXP int scGetGraphKernelCount(scClothPatch patch);
/* on != 0: scStepCloth launches the substeps' kernels one by one on the patch
   stream instead of replaying the captured frame graph (same kernels, same
   results; for profilers that cannot see kernels inside graphs); section timing
   (scSetKernelTiming) records nothing meanwhile. Default 0. */
SCEXP void scSetDirectLaunch(scClothPatch patch, int on);
/* Time `reps` back-to-back constraint sweeps (kind 0: all FEM colours of one
   iteration, 1: all bend colours) captured as one graph, with CUDA events on
   the patch stream; returns milliseconds per sweep, or a negative value on error.
   Particle positions are modified. */
SCEXP float scProfileSweep(scClothPatch patch, int kind, int reps);
/* Latency floor of the cluster solver's colour phases (addition, no reference
   counterpart): runs `phases` phases on one thread-block cluster of the solver's
   size and block shape, separated by cluster barriers, with nothing else in a
   phase (kind 0) or one distributed-shared-memory read and write per thread
   (kind 1), and returns microseconds per phase (negative on error). Uses the
   current device and the legacy default stream; allocates nothing. */
SCEXP float scProbeClusterPhase(int kind, int phases);
/* Section timing inside the frame graph (additions, no reference counterpart):
   frames > 0 brackets, in every substep, the Gauss-Seidel solve (section 0), the
   edge-edge (1) and vertex-triangle (2) continuous-collision broad phases and the
   collider detection (3: walls, spheres, SDFs, meshes) with
   CUDA events, fresh ones for each of the next `frames` frames, so no host
   synchronisation enters a timed run; 0 turns it off. Re-captures the graph. */
SCEXP bool scSetKernelTiming(scClothPatch patch, int frames);
/* Synchronises; ms[4] = summed event time per section, counts[4] = timed
   instances, over the frames since the last read; returns those frames. */
SCEXP int scGetKernelTiming(scClothPatch patch, float* ms, int* counts);

/* ---- addition with no counterpart in the reference: normals without allocation ----
   For callers that cannot call cudaMalloc (engines that reserve all GPU memory up
   front and forbid allocation in their frame loop, code running inside another
   library's memory pool, real-time threads where an allocation would stall the
   frame). Computes the angle-weighted vertex normals of a triangle mesh — the
   normals scUpdateClothMesh computes — from caller-owned DEVICE buffers:
   vertices and normals are numVertices packed xyz floats, indices 3*numTriangles.
   Its only scratch is a fixed file-scope device array of SC_NOALLOC_MAX_VERTICES
   float4 accumulators (1 MiB, resident on every GPU that loads the library until
   the process exits); meshes with more vertices, or more than
   SC_NOALLOC_MAX_TRIANGLES triangles, are rejected (SC_ERR_ARG = 2).
   Every triangle index is checked on the device: a triangle with an index
   >= numVertices is skipped (nothing is written for it) and the call returns
   SC_ERR_ARG; to report that, the call waits for its work on `stream` to finish.
   Every call shares that scratch and leaves its contents behind; a call clears
   what it uses first, but calls that overlap on the GPU race and must be
   serialised by the caller. The first call on a device looks the scratch's
   device address up, so make it before any stream capture that includes later
   calls; later calls on a stream that is not capturing look it up again.
   Work is enqueued on `stream` (a cudaStream_t, NULL = legacy default).
   Returns 0 or an error code (details from scGetLastErrorString). */
#define SC_NOALLOC_MAX_VERTICES 65536
#define SC_NOALLOC_MAX_TRIANGLES 16777216
SCEXP int scComputeVertexNormalsNoAlloc(const float* vertices, int numVertices, const unsigned* indices,
                                        int numTriangles, float* normals, void* stream);

/* ---- addition: headless picture of the cloth ----
   Rasterises the patch's current mesh on the GPU with the demo's Phong program
   (Shaders/shader_phong_*.glsl; drawn by Graphics3D::DrawMesh,
   Graphics/Graphics3D.h) into `rgba` (a DEVICE buffer of width*height float4,
   row 0 at the top). viewProj16: row-major 4x4 view-projection matrix applied to
   column vectors (x, y, z, 1), OpenGL clip conventions. params16: light position
   (3), eye position (3), diffuse colour kd (3), specular colour ks (3),
   shininess, flip (+1/-1 for the normal's side), background grey, flags
   (shader bits: 2 Oren-Nayar, 8 monochrome, 16 wireframe; others are rejected
   with SC_ERR_UNSUPPORTED = 4). zscratch: a DEVICE buffer of width*height
   uint64 that the call overwrites; afterwards each word holds (depth key << 32 |
   triangle index), or all ones where no triangle covers the pixel. Blocks until
   the picture is written. Returns 0 or an error code. */
SCEXP int scRenderCloth(scClothPatch patch, const float* viewProj16, const float* params16, int width, int height,
                        float* rgba, void* zscratch);

#ifdef __cplusplus
}
#endif

#endif /* SOLIDCLOTH_B200_H */
