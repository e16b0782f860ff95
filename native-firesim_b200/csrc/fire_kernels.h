// fire_kernels.h -- kernel declarations of firesim-b200 (sm_100a).
#pragma once

#include "fire_device.cuh"

namespace firesim {

// One ember's screen-space splat, computed once per frame (see emberSetup).
struct EmberSplat {
    int active;
    int minX, maxX, minY, maxY;
    float screenX, screenY, trailX, trailY;
    float radius, cappedTrailLen, lifeFade;
    float3 color;
};

// Per-block partial of the frame metrics: 21 FP64 sums (the reference's
// MetricAccumulator order, src/fire_cuda.cu:70-102), 9 positive-float maxima
// as int bits, and the invalid-cell count.
struct MetricPartial {
    double sums[21];
    int maxBits[9];
    int invalidCells;
};
constexpr int kMetricBlocks = 296;

// Brick decomposition of the shared-memory-resident SOR (sorResident).
struct ResidentBrick {
    int bx, by, bz;     // brick extent, all even
    int nbx, nby, nbz;  // bricks per axis
};
// Brick-to-brick exchange of the resident SOR.  After half sweep h a brick
// publishes each of its face cells as one 64-bit word into exchange[cell]:
// the value's bits in the high half, epoch + h + 1 in the low half.  A
// neighbour that needs the cell for half sweep h + 1 polls that word until
// the tag matches; value and tag travel in one single-copy-atomic store, so
// there is no separate flag and no fence.  Every poll gives up after waitNs
// nanoseconds (or kResidentMaxPolls polls), records epoch + 1 in *status so
// the other bricks stop waiting too, writes brick + 1 into the host-mapped
// *hostStatus and returns.  silentBrick >= 0 is a host-side fault injection:
// that brick never publishes, so its neighbours' polls run out.
struct ResidentSync {
    unsigned long long* exchange;  // one word per grid cell (only face cells are written)
    unsigned* status;
    unsigned* hostStatus;
    unsigned epoch;
    int silentBrick;
    unsigned long long waitNs;
    const int* skip;               // non-null and non-zero: the solve has converged, return at once
};

// Residual gate of a solve run in chunks: after each chunk the residual
// r = div + (sum of the six neighbours) - 6 p (neighbours clamped at the walls,
// as in the update) is reduced in a fixed order, and the chunks after the one
// that reached max |r| <= tolerance return at once.
struct SorGate {
    int converged;
    int iterations;      // iterations run
    float maxResidual;   // max |r| after the last chunk run
    int pad;
    double l2Residual;   // sqrt(sum r^2), accumulated in FP64
};
constexpr int kResidualBlocks = 592;  // 4 per SM; each warp takes whole rows
constexpr int kResidualThreads = 256;
constexpr unsigned kResidentMaxPolls = 1u << 24;
constexpr int kMetricThreads = 128;

// fire_sim.cu
__global__ void fuelBedTables(float* material, float* breathing, FrameParams p, int withMaterial);
__global__ void resetCells(ScalarFields out, float* pressure, float* divergence, float* divergenceAfter, const float* material,
                           const float* breathing, FrameParams p);
__global__ void advectVelocity(FaceT* uOut, FaceT* vOut, FaceT* wOut, Velocity vel, FrameParams p);
__global__ void advectReact(ScalarFields out, ScalarFieldsIn in, Velocity vel, const float* material, const float* breathing, FrameParams p,
                            HashLattice2 sourceLattice);
__global__ void hashLatticeBuild(HashLattice2 a, HashLattice2 b);
__global__ void forceContributions(float4* contrib, ScalarFieldsIn s, Velocity vel, FrameParams p, HashLattice2 curlA, HashLattice2 curlB);
__global__ void forceApply(FaceT* uOut, FaceT* vOut, FaceT* wOut, const float4* contrib, Velocity vel, FrameParams p);
__global__ void forceProjectSetup(FaceT* uOut, FaceT* vOut, FaceT* wOut, float* divergence, float* pressure, const float4* contrib,
                                  Velocity vel, FrameParams p);
__global__ void velocityBoundary(FaceT* u, FaceT* v, FaceT* w, FrameParams p, int clampValues);
__global__ void divergenceOf(float* divergence, float* pressureOrNull, Velocity vel, FrameParams p);
// Colour-split layout of the non-resident solve: colour c, row (y, z), slot k
// holds the cell x = 2k + ((c + y + z) & 1); H = (nx + 1) / 2 slots per row,
// rows P = H rounded up to 4 floats apart (so a row starts on 16 bytes and a
// half sweep moves float4s).  Slots k >= H, and k = H - 1 where its x is nx,
// hold no cell and are never read.
struct SplitGrid {
    int nx, ny, nz, H, P;
};
inline SplitGrid splitGridOf(int nx, int ny, int nz) {
    const int h = (nx + 1) / 2;
    return SplitGrid{nx, ny, nz, h, (h + 3) & ~3};
}
__host__ __device__ inline int splitIdx(const SplitGrid& s, int c, int y, int z, int k) { return ((c * s.nz + z) * s.ny + y) * s.P + k; }
constexpr int kSplitRows = 4;  // rows (y) per block of the split half sweep; a warp covers 128 slots of one row
__global__ void sorSplitPack(float* split, float* splitDiv, const float* pressure, const float* divergence, SplitGrid s);
__global__ void sorSplitUnpack(float* pressure, const float* split, SplitGrid s);
__global__ void sorSplitHalfSweep(float* own, const float* other, const float* ownDiv, SplitGrid s, int c, float omega, const int* skip);
__global__ void sorResidualPartials(const float* pressure, const float* divergence, Grid g, const SorGate* gate, double* partialSq,
                                    float* partialMax);
__global__ void sorSplitResidualPartials(const float* split, const float* splitDiv, SplitGrid s, const SorGate* gate, double* partialSq,
                                         float* partialMax);
__global__ void sorResidualFinal(SorGate* gate, const double* partialSq, const float* partialMax, int partials, float tolerance,
                                 int chunkIterations);
// The sorResident<BX, 16, 16> instantiation for brick width bx (32 or 16),
// for cudaFuncSetAttribute / cudaLaunchCooperativeKernel.
const void* sorResidentKernel(int bx);
// Dynamic shared memory of that instantiation (padded colour planes + div).
size_t sorResidentSharedBytes(int bx);
__global__ void subtractWall(FaceT* u, FaceT* v, FaceT* w, const float* pressure, FrameParams p, int doSubtract, int doWalls);

// fire_light.cu
__global__ void lightBuild(float4* sceneLight, float* sceneShadow, ScalarFieldsIn s, FrameParams p);
__global__ void lightPropagate(float4* outLight, const float4* inLight, const float* sceneShadow, FrameParams p, float diffusion,
                               float decay);

// fire_render.cu
// Work list of the raymarch: 8x4-pixel tiles taken by warps from *counter
// (zeroed before each launch), in the order of `order` (tile ids, x fastest).
constexpr int kRayTileW = 8, kRayTileH = 4;
struct RayTiles {
    int* counter;
    const int* order;
    int tilesX;
    int count;
};
__global__ void raymarch(float4* out, ScalarFieldsIn s, Velocity vel, const float4* lightF, const float* shadowF, FrameParams p, RayTiles tiles);
// The same for one scene id (0, 1, 2) fixed at compile time, without a debug view.
__global__ void raymarchScene0(float4* out, ScalarFieldsIn s, Velocity vel, const float4* lightF, const float* shadowF, FrameParams p,
                               RayTiles tiles);
__global__ void raymarchScene1(float4* out, ScalarFieldsIn s, Velocity vel, const float4* lightF, const float* shadowF, FrameParams p,
                               RayTiles tiles);
__global__ void raymarchScene2(float4* out, ScalarFieldsIn s, Velocity vel, const float4* lightF, const float* shadowF, FrameParams p,
                               RayTiles tiles);
__global__ void emberSetup(EmberSplat* embers, ScalarFieldsIn s, Velocity vel, FrameParams p);
__global__ void emberGather(float4* hdr, const EmberSplat* embers, FrameParams p);
__global__ void tonemapOverlay(uint32_t* frame, const float4* hdr, FrameParams p, int doTonemap, int doOverlay);
__global__ void packHdr(void* dst, size_t pitchBytes, int halfFormat, const float4* hdr, FrameParams p);

// fire_metrics.cu
__global__ void metricsPartials(MetricPartial* partials, ScalarFieldsIn s, const float4* sceneLight, const float* sceneShadow,
                                const float* divergenceBefore, const float* divergenceAfter, FrameParams p);
__global__ void metricsFinal(MetricPartial* out, const MetricPartial* partials, int count);

// ---------------------------------------------------------------------------
// Config physics (FirePhysicsParams.mode 1, fire_config.cu).  Per-step
// constants are formed on the host from FirePhysicsParams in float:
// burnFrac = min(1, burnRate * dt), coolFrac = min(1, cooling * dt),
// sootFrac = min(1, sootDecay * dt), windDtX/Z = dt * windX/Z,
// invPeriod = 1 / noisePeriod, r2 = radius * radius, row = (int)centerY.
struct ConfigEmitter {
    float cx, cz, r2, fuel, heat, up, jitter;
    int row;
    unsigned seed;
};
struct ConfigParams {
    int nx, ny, nz, lx, ly, lz, frameW, frameH;
    unsigned long long step;
    float dt, burnFrac, coolFrac, sootFrac, ignition, heatRelease, sootYield;
    float buoyHeat, buoySoot, ambient, eps, windDtX, windDtZ;
    float noiseAmp, invPeriod;
    unsigned noiseSeed;
    int emitterCount;
    ConfigEmitter emitters[4];
    int primarySamples, lightSamples;
    float3 light;
    float lightIntensity, extinction, fuelExtinction, emission, albedo;
    float3 eye, forward, right, up;
    float tanHalf, aspect;
};

// SplitMix64's output function (Steele, Lea and Flood, OOPSLA 2014).
__host__ __device__ inline unsigned long long splitmix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
// Emitter jitter: uniform in [0, 1) on a 2^-24 grid, one draw per (seed, step, cell).
__host__ __device__ inline float jitterUniform(unsigned seed, unsigned long long step, unsigned cell) {
    const unsigned long long k = (static_cast<unsigned long long>(seed) << 32) ^ (step * 0xD1B54A32D192ED03ull) ^ cell;
    return static_cast<float>(splitmix64(k) >> 40) * (1.0f / 16777216.0f);
}
// Value-noise lattice value in [-1, 1) on a 2^-23 grid for component comp of the seeded field.
__host__ __device__ inline float latticeValue(unsigned seed, int comp, int ix, int iy, int iz) {
    const unsigned long long k = ((static_cast<unsigned long long>(seed) << 2) | static_cast<unsigned>(comp)) * 0xD1342543DE82EF95ull +
                                 static_cast<unsigned long long>(static_cast<unsigned>(ix)) * 0x9E3779B97F4A7C15ull +
                                 static_cast<unsigned long long>(static_cast<unsigned>(iy)) * 0xC2B2AE3D27D4EB4Full +
                                 static_cast<unsigned long long>(static_cast<unsigned>(iz)) * 0x165667B19E3779F9ull;
    return static_cast<float>(splitmix64(k) >> 40) * (1.0f / 8388608.0f) - 1.0f;
}

__global__ void cfgAdvectVelocity(FaceT* uOut, FaceT* vOut, FaceT* wOut, Velocity vel, ConfigParams p);
__global__ void cfgAdvectScalars(Rec4* aOut, const Rec4* aIn, Velocity vel, ConfigParams p);
__global__ void cfgVorticity(float4* vort, Velocity vel, ConfigParams p);
__global__ void cfgNoiseField(float4* noise, ConfigParams p);
__global__ void cfgCellForce(float4* force, const float4* vort, const Rec4* a, const float4* noise, ConfigParams p);
__global__ void cfgApplyForces(FaceT* uOut, FaceT* vOut, FaceT* wOut, Velocity vel, const float4* force, ConfigParams p);
__global__ void cfgTransmittance(float* tr, const Rec4* a, ConfigParams p);
__global__ void cfgRaymarch(float4* hdr, const Rec4* a, const float* tr, ConfigParams p);

// ---------------------------------------------------------------------------
// Multigrid pressure solve of the config physics (fire_mg.cu): the
// incremental projection (cfgPrepareIncrement, mgSolve, cfgSubtractIncrement)
// for one scene or a batch of scenes in one persistent launch.
// A level: extents, axis weights 1/h^2 (fine spacing 1), 2 (wx + wy + wz) and
// its reciprocal, and which axes were halved from the level above.
struct MgLevel {
    int nx, ny, nz;
    float wx, wy, wz, diag, invDiag;
    int cx, cy, cz;
};
constexpr int kMgMaxLevels = 10;
constexpr int kMgMaxScenes = 128;     // scenes of one batched solve
constexpr int kMgTailCells = 6144;    // the tail starts at the first level with at most this many cells
constexpr size_t kMgTailSmemMax = 200 * 1024;  // shared memory a tail may use
// Where a tail keeps its levels: all in shared memory; the tail level's rhs
// in global memory and the rest in shared memory; all in global memory.
enum MgTailMode { kMgTailShared = 0, kMgTailRhsGlobal = 1, kMgTailGlobal = 2 };
constexpr int kMgThreads = 1024;      // threads of a CTA of mgSolve (one CTA per SM)
constexpr int kMgChunkRows = 4;       // level-0 rows per residual chunk (rows whose length is not a multiple of 4)
constexpr int kMgChunkUnits = 4;      // 128-cell units per residual chunk (rows whose length is a multiple of 4)
constexpr int kMgCoarsestSweeps = 32;
constexpr int kMgHardCycleCap = 1000;  // fireCudaSetPressureMultigrid accepts at most this many cycles
constexpr unsigned kMgMaxPolls = 1u << 26;
constexpr unsigned kMgStatusFlag = 0x80000000u;  // host status word: a multigrid barrier wait ran out (low bits: phase)
// One scene of a solve.  Level l's p and rhs: level 0 is the increment and
// the divergence array; levels >= 1 are the coarse corrections.
struct MgScene {
    MgLevel lv[kMgMaxLevels];
    float* p[kMgMaxLevels];
    float* rhs[kMgMaxLevels];
    float* pressure;   // += the increment at the end of the solve
    SorGate* gate;     // zeroed before the launch
    double* chunkSq;   // per residual chunk (mgResidualChunks)
    int levels;        // number of levels
    int tail;          // first level solved by one CTA (the tail)
    int tailMode;      // MgTailMode
};
// The work lists of a solve, as prefix sums over the scenes (0 for a scene
// whose tail starts at or above the level).  smoothUnits and fineUnits count
// the units of grid level l (the smoothing's and the prolongation's): where
// the row length is a multiple of 4, 128 consecutive cells in memory, four
// per lane (mgQuadUnits); otherwise 128-cell (smoothing) or 32-cell
// (prolongation) chunks of single rows.  coarseUnits counts the restriction's
// units of level l + 1: 64 consecutive coarse cells where the fine row length
// is a multiple of 4, else 32-cell chunks of single rows.  chunks counts the
// residual's chunks of level 0 (mgResidualChunks), allUnits the units of
// level 0 as the smoothing takes them (for the first and last phases).
struct MgPlan {
    int scenes;
    int gridLevels;  // max over the scenes of tail
    int maxCycles, pre, post, gated;
    float tolerance;
    int smoothUnits[kMgMaxLevels][kMgMaxScenes + 1];
    int fineUnits[kMgMaxLevels][kMgMaxScenes + 1];
    int coarseUnits[kMgMaxLevels][kMgMaxScenes + 1];
    int chunks[kMgMaxScenes + 1];
    int allUnits[kMgMaxScenes + 1];
};
// Chunks per row of a level: 128-cell chunks (the smoothing's units, four
// cells per lane) and 32-cell chunks (the prolongation's and restriction's).
__host__ __device__ inline int mgQuadChunks(int nx) { return (nx + 127) / 128; }
__host__ __device__ inline int mgRowChunks(int nx) { return (nx + 31) / 32; }
// 128-cell units of a level whose row length is a multiple of 4.
__host__ __device__ inline int mgQuadUnits(int nx, int ny, int nz) { return (nx * ny * nz + 127) / 128; }
// The level-0 residual's chunks of one scene: kMgChunkUnits quad units, or
// kMgChunkRows rows where the row length is not a multiple of 4.
__host__ __device__ inline int mgResidualChunks(int nx, int ny, int nz) {
    return (nx & 3) == 0 ? (mgQuadUnits(nx, ny, nz) + kMgChunkUnits - 1) / kMgChunkUnits : (ny * nz + kMgChunkRows - 1) / kMgChunkRows;
}
// Grid barrier and convergence state of mgSolve (zeroed before each launch):
// the count of barrier arrivals (barrier k is passed when it reaches
// k * gridDim.x), a failure flag, and per scene the max |r| of the level-0
// residual of a cycle (float bits; cycles alternate between the two rows).
struct MgSync {
    unsigned count, failed, pad0, pad1;
    unsigned sceneMax[2][kMgMaxScenes];
};
__global__ void mgSolve(const MgScene* scenes, const MgPlan* plan, MgSync* sync, unsigned* hostStatus, unsigned long long waitNs);
__global__ void cfgPrepareIncrement(FaceT* uOut, FaceT* vOut, FaceT* wOut, Velocity vel, const float* pressure, float* rhs, int nx,
                                    int ny, int nz);
__global__ void cfgSubtractIncrement(FaceT* u, FaceT* v, FaceT* w, const float* delta, int nx, int ny, int nz, int doWalls);
__global__ void cfgTopFaces(FaceT* v, const float* p, int nx, int ny, int nz);

// ---------------------------------------------------------------------------
// Batched config physics (fire_config.cu, host side fire_batch.cu): one launch
// per stage over every scene of a batch.  A block belongs to one scene; its
// threads take consecutive elements of one index space of that scene (x
// fastest): cells, faces ((nx+1)(ny+1)(nz+1)), half-resolution light cells
// or pixels.  The per-element work is the single-scene kernels' own body, so
// a scene gives the same bits alone or in a batch.
enum BatchSpace { kBatchCells = 0, kBatchFaces = 1, kBatchLight = 2, kBatchPixels = 3, kBatchSpaces = 4 };
constexpr int kBatchThreads = 128;
// Elements per thread of a batched stage: runs of consecutive cells or faces
// (one scene lookup and one coordinate division per run); one light column or
// pixel per thread.
__host__ __device__ constexpr int batchPerThread(int space) { return space == kBatchCells || space == kBatchFaces ? 4 : 1; }
constexpr int kBatchMaxScenes = kMgMaxScenes;
struct BatchScene {
    ConfigParams c;        // this step's parameters (c.step: the emitters' jitter counter)
    Velocity vel;          // faces at the start of the step
    FaceT* adv[3];         // advected faces
    const Rec4* aIn;       // record a at the start of the step
    Rec4* aOut;            // the advanced record a
    float4* vort;
    float4* force;
    const float4* noise;   // curl-noise field (null when its amplitude is 0)
    FaceT* forced[3];      // faces after the forces
    FaceT* proj[3];        // faces of the projection (the previous pressure's gradient subtracted)
    float* pressure;
    float* divergence;
    float* delta;          // the multigrid's level-0 increment
    float* transmittance;
    float4* hdr;
    void* slot;            // the scene's HDR output buffer (null: keep the frame in hdr)
    size_t slotPitch;
    int slotFormat;        // FireHdrFormat
    int count[kBatchSpaces];  // elements of each index space
};
struct BatchPlan {
    int scenes;
    int start[kBatchSpaces][kBatchMaxScenes + 1];  // prefix sums of the blocks of each scene (0 for a scene that does not render);
                                                   // a block takes kBatchThreads * batchPerThread(space) elements
};
__global__ void batchAdvectVelocity(const BatchScene* scenes, const BatchPlan* plan);
__global__ void batchAdvectScalars(const BatchScene* scenes, const BatchPlan* plan);
__global__ void batchVorticity(const BatchScene* scenes, const BatchPlan* plan);
__global__ void batchCellForce(const BatchScene* scenes, const BatchPlan* plan);
__global__ void batchApplyForces(const BatchScene* scenes, const BatchPlan* plan);
__global__ void batchPrepareIncrement(const BatchScene* scenes, const BatchPlan* plan);
__global__ void batchSubtractIncrement(const BatchScene* scenes, const BatchPlan* plan);
__global__ void batchTransmittance(const BatchScene* scenes, const BatchPlan* plan);
__global__ void batchRaymarch(const BatchScene* scenes, const BatchPlan* plan);
__global__ void batchPackHdr(const BatchScene* scenes, const BatchPlan* plan);

}  // namespace firesim
