// launch.h — host-callable launchers for the cloth-step kernels (step_kernels.cu).
#pragma once
#include "sc_internal.cuh"

namespace sc {

constexpr int KVT = 48;        // self vertex-triangle contact slots per vertex
constexpr int KCAND = 256;     // BVH candidates kept per proximity query
constexpr int KRES = 96;       // distinct features tracked per vertex for the dedup
constexpr int KADJ = 16;       // adjacent primitives held in registers by a broad-phase query
constexpr int KCCD = 128;      // continuous-collision candidates kept in a query's own slots
// second broad-phase pass: warps per block, blocks, stack entries per depth level
constexpr int CCD_COOP_THREADS = 128, CCD_COOP_BLOCKS = 4 * 148, CCD_COOP_GROUP = 64;
// first-pass walks: one query per lane, or warp packets
enum { BROAD_LANE = 0, BROAD_PACKET = 1, BROAD_WALKS = 2 };
constexpr int CCD_VT_PAIRS = 128, CCD_EE_PAIRS = 96; // pair store per vertex / edge
constexpr int CCD_VT_HITS = 32, CCD_EE_HITS = 16;   // continuous contacts per vertex / edge
constexpr int MAX_COLOURS = 128; // independent-set colouring rounds per contact class
constexpr int WALL_SLOTS = 5;

// Vertex contact slot (walls, sphere, SDF, mesh vertex contacts).
struct VC { float4 point; float4 normal; float2 lam; int feature; int mesh; };
// Triangle contact (cloth triangle vs collider vertex / sphere / SDF).
struct TC { uint4 idx; float4 point; float4 normal; float4 w; float2 lam; int feature; int mesh; };
// Edge contact (cloth edge vs collider edge / sphere).
struct EC { uint4 idx; float4 point; float4 normal; float4 w; float2 lam; int feature; int mesh; };
// Self contact (vertex-triangle: i1..i3 triangle, i4 vertex; edge-edge: (i1,i2) x (i3,i4)).
struct SCt { uint4 idx; float4 normal; float4 w; float2 lam; float side; float error; };

// Vertex collider descriptor (world order).
struct VColl
{
    int type;        // 1 walls, 3 sphere, 7 sdf, 4 mesh
    int slotBase;    // first slot of this collider in the vertex-contact slot array
    int kmax;        // slots per vertex
    int vBegin, vCount; // particles it acts on (a batch instance's range; else all)
    int countBase;   // first of its vCount per-particle slot counts
    int mesh;        // mesh collider index for type 4
    float4 a, b;     // walls: lo, hi; sphere: centre (a.xyz), radius (a.w)
    cudaTextureObject_t val, grad; // sdf
    float4 sdfLo, sdfSteps;        // sdf box min, steps
    int4 sdfCells;
};

struct Buffers
{
    // vertex contacts: counts[coll][N] (uint8), slots[slotBase + i*kmax + k]
    uint8_t* vcCount;
    VC* vc;
    int numVColl;
    const VColl* vcoll;       // device copy
    const int2* instColl;     // batch: (first collider, count) per instance; null: all colliders act on all
    int broadWalk;            // continuous broad phase first-pass walk (BROAD_*, tuned)
    // triangle / edge contacts: per-collider slot arrays, flags, dense lists
    TC* tcSlot; int* tcFlag; TC* tcList; int* tcCount; int tcCap;
    EC* ecSlot; int* ecFlag; EC* ecList; int* ecCount; int ecCap;
    // self contacts
    int* stCnt; SCt* stSlot; SCt* stList; int* stCount; int stCap;
    int* seFlag; SCt* seSlot; SCt* seList; int* seCount; int seCap;
    // continuous collision
    int* ccdVtCnt; int* ccdVtCand; int* ccdEeCnt; int* ccdEeCand;
    int2* ccdVtPairs; int2* ccdEePairs; int* ccdVtPairCount; int* ccdEePairCount; int ccdVtCap, ccdEeCap;
    uint8_t* ccdVtHit; uint8_t* ccdEeHit;  // per pair: 1 if the narrow phase reports a contact
    int* ccdVtOff; int* ccdEeOff;          // first pair of each query
    int* ccdVtHitCnt; int* ccdEeHitCnt;    // hits per query
    int* ccdPool; int ccdPoolCap; int* ccdPoolUsed;  // candidate lists longer than KCCD
    int* ccdVtPoolOff; int* ccdEePoolOff;
    int* ccdVtOvf; int* ccdEeOvf; int* ccdOvfN;      // queries with more than KCCD candidates; counts (vt, ee)
    // colouring scratch
    unsigned long long* vmin;  // N, kept at ~0
    int* colour; int* order; int* colourStart; int colourCap;
    // scan scratch: block sums, per-item offsets, totals
    int* scanBlock; int* scanOff; int* scanTot;
    int* scanBlock2;           // second block-sum scratch for scans on the side stream
    int* scanOff2;             // second per-item offsets (side stream)
    const DevMesh* meshes;     // device array
    int numMeshes;
};

void launch_predict(cudaStream_t s, const DevCloth& c, const SolverParams& P);
// state <-> 10 N floats: positions, velocities, previous positions (xyz), inverse masses
void launch_pack_state(cudaStream_t s, const DevCloth& c, float* out);
void launch_unpack_state(cudaStream_t s, const DevCloth& c, const float* in);
void launch_velocity(cudaStream_t s, const DevCloth& c, const SolverParams& P);
void launch_fem(cudaStream_t s, const DevCloth& c, const SolverParams& P, int first, int count);
void launch_links(cudaStream_t s, const DevCloth& c, const SolverParams& P, int first, int count);
void launch_reset_link_error(cudaStream_t s, const DevCloth& c);
void launch_bends(cudaStream_t s, const DevCloth& c, const SolverParams& P, int first, int count, int resetErr);
void launch_normals(cudaStream_t s, const DevCloth& c, bool prevMesh, const float4* verts);
void launch_vertex_colliders(cudaStream_t s, const DevCloth& c, const SolverParams& P, const Buffers& b, const VColl* hostColl);
void launch_tri_edge_colliders(cudaStream_t s, const DevCloth& c, const SolverParams& P, const Buffers& b,
                               const VColl* hostColl, int numColl, int flags);
void launch_solve_vertex_contacts(cudaStream_t s, const DevCloth& c, const SolverParams& P, const Buffers& b);
void launch_solve_multi_contacts(cudaStream_t s, const DevCloth& c, const SolverParams& P, const Buffers& b, int iter);
void launch_colour_contacts(cudaStream_t s, const DevCloth& c, const Buffers& b);
void launch_bvh_refit(cudaStream_t s, const DevBVH& bvh, const DevCloth& c, int kind, float tol);
size_t ccd_coop_smem(int depth);      // dynamic shared memory of the second broad-phase pass
// microseconds a phase of the cluster solver's barrier structure costs (kind 0:
// barrier only; 1: plus one distributed-shared-memory read and write), -1 if no
// cluster of the solver's size fits
float probe_cluster_phase(int kind, int phases);
void ccd_kernel_setup();              // kernel attributes (once per device, outside capture)
void launch_self_proximity(cudaStream_t s, const DevCloth& c, const SolverParams& P, const Buffers& b,
                           const DevBVH& triBvh, const DevBVH& edgeBvh);
// swept-tree refits + continuous-collision broad and narrow phases; the
// vertex-triangle half runs on `side` (forked from / joined to s by the events);
// marks (optional, entries may be null): records around the edge-edge and the
// vertex-triangle broad phases {ee start, ee end, vt start, vt end}
void launch_ccd(cudaStream_t s, cudaStream_t side, cudaEvent_t fork, cudaEvent_t join, const DevCloth& c,
                const SolverParams& P, const Buffers& b, const DevBVH& triBvh, const DevBVH& edgeBvh,
                const cudaEvent_t* marks = nullptr);
// self-contact lists: proximity contacts (self) compacted, then the continuous
// hits appended (ccd; vertex-triangle on `side` between fork and join)
void launch_compact_self(cudaStream_t s, cudaStream_t side, cudaEvent_t fork, cudaEvent_t join, const DevCloth& c,
                         const SolverParams& P, const Buffers& b, bool self, bool ccd);
void launch_reset_gs(cudaStream_t s, const DevCloth& c);

// The reference's other link solvers (ClothModel::SetSolver, Physics/ClothPBD.cpp:293-298):
// links in index order, per-link displacements, and each particle's incident links
// in increasing link index ((link << 1) | 1 where the particle is the link's i2)
struct LinkSolve
{
    int L;
    const float4* link;     // L: i1, i2 (bits), rest length, stiffness; link index order
    float4* disp;           // L: this iteration's displacement of each link
    float* d;               // L: conjugate-residual search direction
    const int* incStart;    // N + 1
    const int* inc;         // 2 L
};
// SolveJacobi: `iterations` rounds of SolveLinksJacobi (omega 0.5)
void launch_solve_jacobi(cudaStream_t s, const DevCloth& c, const SolverParams& P, const LinkSolve& ls);
// SolveCR (alpha0 0.1): beta[k] of iteration k, (k / (iterations - 1))^0.6, computed by the caller
void launch_solve_cr(cudaStream_t s, const DevCloth& c, const SolverParams& P, const LinkSolve& ls, const float* beta);
// max |C| over warp / weft / shear constraints, as float bits into *out
void launch_residual(cudaStream_t s, const DevCloth& c, unsigned* out);
// residual-target mode for the per-colour path: residual + exit flag after an iteration
void launch_residual_exit(cudaStream_t s, const DevCloth& c, const SolverParams& P, int iter);
void launch_iteration_total(cudaStream_t s, const DevCloth& c);
void launch_gs_exit_test(cudaStream_t s, const DevCloth& c, const SolverParams& P, int iter);

// cluster-resident Gauss-Seidel solver (one cluster per cloth, one launch per substep)
constexpr int GS_THREADS = 512;
constexpr int GS_SMEM_MAX = 200 * 1024; // dynamic shared memory per CTA: particles + staged records
struct GsPlan
{
    int iterations, shift, nFemCol, nBendCol;
    int stage;               // 1: each CTA copies its constraint records to shared memory first
    int femStage, bendStage; // records per CTA when staged (max over the cluster's CTAs)
    int femStart[65];
    int bendStart[65];
    int nLinkCol;            // mass-spring path (FEM off): link colours
    int linkStart[65];
};
// cluster size usable for N particles (0: too large or unsupported); sets the
// log2 particles-per-CTA and the dynamic shared memory per CTA
int gs_cluster_size(int N, int& shift, size_t& smem);
// variant 0: one constraint per thread; 1: two (their loads overlap)
int gs_cluster_variants();
void launch_gs_cluster(cudaStream_t s, const DevCloth& c, const SolverParams& P, const Buffers& b, GsPlan plan,
                       int clusterSize, size_t smem, int variant);

// grid-resident solver (cooperative launch, any cloth or batch size); variants
// differ in threads per CTA and in constraints per thread (tiles)
int gs_grid_variants();
void gs_grid_variant_info(int variant, int& threads, int& femTile, int& bendTile);
int gs_grid_max_blocks_per_sm(int variant);
bool launch_gs_grid(cudaStream_t s, const DevCloth& c, const SolverParams& P, const Buffers& b, GsPlan plan,
                    int variant, int blocksPerSm);

// band-parallel solver (one cluster per cloth, one launch per substep): the
// particles in contiguous bands of 2^shift, one per CTA, resident in shared
// memory; each class's records split per band into interior records (every
// particle in the band) and boundary records (lowest particle in the band, the
// others in it or among the first `halo` particles of the next band)
struct BandView
{
    int shift, halo;
    int nFemCol, nBendCol, nLinkCol;
    // record offsets per (band, part, colour): [(band * 2 + part) * nCol + colour], nBands * 2 * nCol + 1 entries
    const int* femOff;
    const int* bendOff;
    const int* linkOff;
    // records in (band, part, colour, colour order) order: FEM 3 float4, bends uint4, links float4
    const float4* fem;
    const uint4* bend;
    const float4* link;
    // records staged in shared memory (1) or read through the non-coherent path (0),
    // and the most records one band holds (the staging layout)
    int stageFem, stageBend, stageLink;
    int femMax, bendMax, linkMax;
};
constexpr int BAND_SMEM_MAX = 220 * 1024;  // dynamic shared memory per CTA of the band solver
// threads-per-CTA variants of the band solver (same order, bit-identical results)
int gs_band_variants();
int gs_band_threads(int variant);
// true if a cluster of clusterSize CTAs with smem bytes each can run the band solver
bool gs_band_fits(int clusterSize, size_t smem);

// The solver's entry points as one table per build of solver.cuh: IEEE division
// and square root without FMA contraction (bit-exact with the reference's
// operation order, the check-mode build) or the fast build (FMA contraction,
// approximate division and square root). Same kernels, same order, same
// launch shapes; detection is shared and always exact.
struct SolverOps
{
    void (*fem)(cudaStream_t, const DevCloth&, const SolverParams&, int, int);
    void (*links)(cudaStream_t, const DevCloth&, const SolverParams&, int, int);
    void (*reset_link_error)(cudaStream_t, const DevCloth&);
    void (*bends)(cudaStream_t, const DevCloth&, const SolverParams&, int, int, int);
    void (*vertex_contacts)(cudaStream_t, const DevCloth&, const SolverParams&, const Buffers&);
    void (*multi_contacts)(cudaStream_t, const DevCloth&, const SolverParams&, const Buffers&, int);
    int (*cluster_size)(int, int&, size_t&);
    void (*cluster)(cudaStream_t, const DevCloth&, const SolverParams&, const Buffers&, GsPlan, int, size_t, int);
    int (*grid_max_blocks_per_sm)(int);
    bool (*grid)(cudaStream_t, const DevCloth&, const SolverParams&, const Buffers&, GsPlan, int, int);
    bool (*band)(cudaStream_t, const DevCloth&, const SolverParams&, const Buffers&, GsPlan, const BandView&, int, size_t,
                 int);
};
const SolverOps& solver_ops(bool fast);

// learned warm start (mlp_kernels.cuh): 9347 FP32 parameters, 27 normalisation values
constexpr int MLP_NPARAM = 9347, MLP_NNORM = 27, MLP_IN = 12, MLP_OUT = 3;
void launch_mlp_warm(cudaStream_t s, const DevCloth& c, const Buffers& b, const float* prm, const float* norm);
void launch_mlp_features(cudaStream_t s, const DevCloth& c, const Buffers& b, float* feat);
void launch_mlp_targets(cudaStream_t s, const DevCloth& c, float* target);
void launch_mlp_forward(cudaStream_t s, const float* X, int S, const float* prm, const float* norm, float* Y);
bool launch_mlp_grad(cudaStream_t s, const float* X, const float* T, int S, const float* prm, const float* norm,
                     float* grad, float* loss);
void launch_adam(cudaStream_t s, float* prm, const float* grad, float* m, float* v, int step, float lr);

// SDF::CreateFromMesh on the device: (nx+1)(ny+1)(nz+1) values, x fastest
bool launch_sdf_from_mesh(const DevMesh& m, int nx, int ny, int nz, float4 lo, float4 steps, float* out, int* status);

// exclusive scan of n ints (out may alias nothing); total written to *total if not null
void scan_ints(cudaStream_t s, const int* in, int* out, int n, int* total, int* tmp);

} // namespace sc
