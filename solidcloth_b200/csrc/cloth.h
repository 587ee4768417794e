// cloth.h — host-side objects behind the C ABI: collision world, collidables,
// cloth model and cloth patch (the roles of Physics/CollisionWorld.h,
// Physics/Common.h, Physics/ClothModel.h and Physics/ClothPatch.h).
#pragma once
#include "launch.h"
#include <memory>
#include <vector>
#include <map>
#include <string>
#include <cstdint>

namespace sc {

// ------------------------------------------------------------ host mesh
struct HEdge
{
    V3 n = {0, 0, 0};
    uint32_t i1 = 0, i2 = 0;
    int t1 = -1, t2 = -1;
    int origIdx = 0;
    bool swapped = false;
};

struct HMesh
{
    std::vector<V3> verts;
    std::vector<uint32_t> idx;
    std::vector<V3> normals, triN;
    std::vector<uint32_t> triE;          // 3 per triangle
    std::vector<HEdge> edges;
    std::vector<std::vector<int>> vtxRing, edgeRing;
    int ntris() const { return (int)idx.size() / 3; }
    void compute_normals();              // Mesh::ComputeNormals
    void construct_edges();              // Mesh::ConstructEdges
    void construct_rings(bool vtx, bool edge);
};

// ------------------------------------------------------------ colliders
enum CollidableType { CT_INVALID, CT_WALLS, CT_SLAB, CT_SPHERE, CT_MESH, CT_BOX, CT_CAPSULE, CT_SDF };

struct Collidable
{
    int type = CT_INVALID;
    float rot[4] = {1, 0, 0, 0};       // quaternion (s, x, y, z)
    V3 center = {0, 0, 0};
    virtual ~Collidable() {}
};

struct WallsC : Collidable { Box box; };
struct SphereC : Collidable { float radius = 0; };
struct CapsuleC : Collidable { float r = 0, hh = 0; };

struct SDFC : Collidable
{
    int nc[3] = {0, 0, 0};
    Box box;
    V3 steps = {0, 0, 0};
    std::vector<float> values;
    std::vector<V3> grad;
    // per-device texture objects
    int device = -1;
    cudaArray_t valArr = nullptr, gradArr = nullptr;
    cudaTextureObject_t valTex = 0, gradTex = 0;
    ~SDFC();
    void compute_gradient();             // SDF::ComputeGradient
    bool upload(int dev);
};

struct MeshTreeNode { Box box; std::vector<uint32_t> tris, verts, edges; int left = -1, right = -1; };

struct MeshC : Collidable
{
    HMesh mesh;
    std::vector<MeshTreeNode> tree;      // Geometry::ComputeMeshTree, built lazily
    bool built = false;
    int device = -1;
    // device copies
    void* dmem = nullptr;
    DevMesh dev{};
    ~MeshC();
    // Geometry::ComputeMeshTree(mesh, flags, maxLevel, tol): flags 1 triangles,
    // 2 vertices, 4 edges (ATF_*); the collider uses all three, maxLevel 20
    void build_tree(float tol, int maxLevel = 20, int flags = 7);
    bool upload(int dev);
};

struct CollisionWorld
{
    std::vector<std::shared_ptr<Collidable>> list;
    uint64_t version = 0;
};

// ------------------------------------------------------------ cloth
struct HostParams
{
    // defaults of ClothModel::ClothModel (Physics/ClothModel.cpp:10-36)
    float unit = 10, thickness = 0.3f, tolerance = 0.2f, shear = 5e8f, bend = 5.f, stretch = 2e10f;
    float poisson = 0.5f, friction = 0.4f, area = 10.f, drag = 1.f, selfShrink = .9f, selfSoften = .1f;
    float selfThreshold = 0.003f;
    int iterations = 50, flags = 0, bendFreq = 2;
    bool fem = false, dihedral = true, fixedIterations = false, ccd = false;
    bool stageRecords = true;    // cluster solver: constraint records in shared memory
    bool fastMath = false;       // solver build: false = IEEE (bit-exact), true = FMA + approximate div/sqrt
    float resTol = 0.f;          // > 0: Gauss-Seidel runs until the residual is <= resTol (iterations = cap)
    bool resMetres = false;      // update residual in metres (true) or in mean rest edge lengths
    int solverType = 1;          // ClothModel::SolverType: 0 Jacobi, 1 Gauss-Seidel, other: conjugate residual
};

// a collider acting on the particles [vBegin, vBegin + vCount) of batch instance `inst`
struct BatchColl { std::shared_ptr<Collidable> coll; int vBegin, vCount, inst; };

// solver selection (autotuned unless forced)
enum SolverKind { SOLVE_AUTO = 0, SOLVE_CLUSTER = 1, SOLVE_GRID = 2, SOLVE_KERNELS = 3, SOLVE_BAND = 4 };
struct SolverChoice { int kind, variant, blocksPerSm; float ms; int broad; };

struct FemHost { uint32_t i1, i2, i3; float du1, du2, dv1, dv2, det, invDet, lu0, lv0, su, sv, lu2, lv2, area; };

struct LBVHHost
{
    std::vector<int> child, escape, parent, leafNode, maxPrim;
    int numLeaves = 0, numNodes = 0, depth = 0;
    void build(const std::vector<V3>& centroids);
};

class ClothPatch;

class ClothModel
{
public:
    explicit ClothModel(ClothPatch* owner) : owner(owner) {}
    ~ClothModel();

    ClothPatch* owner;
    HostParams prm;
    uint64_t paramVersion = 1;

    // host topology and rest data
    int N = 0;
    std::vector<V3> hpos, hprev, hvel;
    std::vector<float> invMass;
    std::vector<float> uvx, uvy;
    // grid clothes (ClothPatch::Init(grid)): each particle's (column, row); empty
    // for a cloth from a mesh (and for a batch with such a part)
    std::vector<int2> gridIJ;
    std::vector<FemHost> tris;
    std::vector<uint4> bends;
    std::vector<uint2> links;
    std::vector<float2> linkRest;              // rest length, stiffness (ClothModel::AddLink)
    std::vector<int> linkOrder, linkColourStart;
    std::vector<uint4> quads;
    std::vector<int> triOrder, bendOrder;      // colour order
    std::vector<int> triColourStart, bendColourStart;
    std::vector<int> edgeColourHost;           // static colour of each collision-mesh edge (edge contacts)
    bool mouseActive = false;

    // device
    int device = -1;
    std::vector<void*> allocs;
    DevCloth dc{};
    DevBVH triBvh{}, edgeBvh{}, sweptTriBvh{}, sweptEdgeBvh{};
    Buffers buf{};
    std::vector<VColl> vcollHost;
    std::vector<void*> bufAllocs;
    uint64_t bufWorldVersion = ~0ull;
    int bufFlags = -1;
    bool bufCcd = false;

    void* dalloc(size_t bytes, bool contactBuffer = false);
    void release_device();
    void release_buffers();
    bool upload_topology(const HMesh& mesh);
    bool ensure_buffers(const CollisionWorld& world, cudaStream_t s);
    void download_state(cudaStream_t s);
    void upload_state(cudaStream_t s);
    // scSetParticleState: caller arrays (xyz triples) to the host copies and the device
    void set_state(const float* pos, const float* prev, const float* vel, cudaStream_t s);
    // pinned host / device staging of the packed state (10 N floats), made on first use
    float* stageHost = nullptr;
    float* stageDev = nullptr;
    bool ensure_stage();
    SolverParams solver_params(float h) const;
    // batch of independent clothes (empty: one cloth): first particle / triangle /
    // edge / bend of each instance (+ end), and each instance's colliders
    std::vector<int> instV, instT, instE, instB;
    std::vector<BatchColl> batchColl;
    // learned warm start: FP32 parameters + normalisation on the device (owned),
    // and optional per-substep sample recording into caller-owned device buffers
    float resScale = 1.f;                       // 1 / mean rest edge length
    float* mlpPrm = nullptr;
    bool warmStart = false;
    float* sampleFeat = nullptr;
    float* sampleTarget = nullptr;
    int solverMode = SOLVE_AUTO;                // forced solver, or the tuner's choice
    SolverChoice choice{SOLVE_CLUSTER, 0, 0, 0.f};
    bool tuned = false;
    uint64_t tunedVersion = 0;
    std::vector<SolverChoice> tuneLog;          // candidates and their times of the last tuning
    int broadWalk = 0;                          // tuned: continuous broad phase first-pass walk (BROAD_*)
    int broadMode = -1;                         // forced walk (BROAD_*) or -1: tuned
    float broadMs[BROAD_WALKS] = {};            // tuned times of the broad-phase walks
    void colour_constraints();
    void touch() { paramVersion++; }

    // band-parallel solver (k_gs_band): the plan, when the cloth admits one
    // (build_band_plan); used when solver mode 4 is set
    struct BandPlan
    {
        bool valid = false;
        int clusterSize = 0, shift = 0, halo = 0;
        int femMax = 0, bendMax = 0, linkMax = 0;          // most records of one band per class
        std::vector<int> triOrder, bendOrder, linkOrder;   // its Gauss-Seidel order, (part, colour, band, record)
        std::vector<int> triStart, bendStart, linkStart;   // (part, colour) group starts of that order
        BandView view{};                                   // device arrays (in allocs)
    } bandPlan;
    void build_band_plan();
    LinkSolve linkSolve{};                      // Jacobi / conjugate-residual link solves (uploaded with the links)
    bool band_active() const { return bandPlan.valid && solverMode == SOLVE_BAND; }
    size_t band_smem();
};

class ClothPatch
{
public:
    explicit ClothPatch(CollisionWorld& w);
    ~ClothPatch();

    CollisionWorld& world;
    ClothModel model;
    HMesh mesh, prevMesh;     // render mesh and collision mesh (host mirrors)
    int numSteps = 1;
    bool isQuadMesh = true;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;               // second branch of the captured frame graph
    cudaEvent_t evFork = nullptr, evJoin = nullptr;

    // cached CUDA graph of one frame
    cudaGraphExec_t graph = nullptr;
    cudaGraph_t graphDef = nullptr;            // the captured definition of `graph`
    float graphDt = -1.f;
    int graphSteps = -1;
    uint64_t graphParamVersion = 0, graphWorldVersion = ~0ull;
    bool hostStateDirty = false;   // host copies older than the device state
    bool directLaunch = false;     // launch the substeps' kernels directly instead of replaying the frame graph
    int graphKernelCount = 0;

    // In-graph section timing: event-record nodes bracket the Gauss-Seidel solve
    // and the two broad phases of every substep; before each replay they are
    // pointed at fresh events (cudaGraphExecEventRecordNodeSetEvent affects only
    // later launches), so a run of frames is timed with no host synchronisation.
    enum { SEC_GS = 0, SEC_BROAD_EE = 1, SEC_BROAD_VT = 2, SEC_COLLIDERS = 3, NSEC = 4 };
    int timingFrames = 0;                       // frames the pool can hold (0: off)
    int timingUsed = 0;                         // frames recorded since the last read
    std::vector<cudaEvent_t> timingCapture;     // events named at capture: [substep][section][start/end]
    std::vector<cudaGraphNode_t> timingNodes;   // their record nodes in the instantiated graph
    std::vector<cudaEvent_t> timingPool;        // [frame][substep][section][start/end]
    int recordingSubstep = 0;
    void timing_mark(int section, bool end, cudaStream_t s);
    bool set_timing(int frames);
    int read_timing(float* msPerSection, int* countPerSection);

    bool init_grid(int divX, int divY, float inc, V3 offset, bool horizontal, bool attached);
    bool init_batch(const std::vector<ClothPatch*>& parts);
    bool init_mesh(const std::vector<V3>& verts, const std::vector<uint32_t>& idx, const float* uvs,
                   const float* colors, V3 offset, bool attached);
    std::vector<int> meshMap;                  // mesh cloth: input vertex -> particle
    bool step(float dt);
    void update_mesh();
    void record_substep(float h);
    bool record_solve(cudaStream_t s, const SolverParams& P, const SolverChoice& ch);
    bool autotune(float h);
    void sync();
};

// error reporting (thread-local last error, plus device status bits)
void set_error(int code, const std::string& msg);
int last_error();
const char* last_error_string();

enum ErrorCodes { SC_OK = 0, SC_ERR_CUDA = 1, SC_ERR_ARG = 2, SC_ERR_STATE = 3, SC_ERR_UNSUPPORTED = 4, SC_ERR_DEVICE_STATUS = 5 };

} // namespace sc
