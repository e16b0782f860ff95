// fire_scene.h -- host-side owner of one fire scene on one GPU.
//
// A Scene holds every device buffer of the frame pipeline, its own CUDA
// stream, the captured SOR graph and the clocks, and runs any contiguous range
// of the frame's stages with the fusions of the B200 kernels.  The C ABI
// (fire_abi.cu) is a thin layer over it: the reference's singleton is one
// Scene.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "../../include/fire_cuda.h"
#include "../../include/fire_ext.h"
#include "fire_guard.h"
#include "fire_kernels.h"

namespace firesim {

struct HdrSlot {
    void* ptr = nullptr;
    size_t pitchBytes = 0;
    int format = 0;
};

// Inputs of the per-scene fuel-bed material table (fuelBedMaterial depends on nothing else).
struct MaterialKey {
    int sceneId = -1;
    float emitterRadius = 0.0f, emitterCenterX = 0.0f, emitterCenterZ = 0.0f;
    int burnerCenterCount = 0;
    float burnerX0 = 0.0f, burnerZ0 = 0.0f;
    bool operator==(const MaterialKey& o) const;
};

// The host side of one persistent multigrid solve (mgSolve) over one scene or
// a batch of scenes: the work lists and scene descriptors in device memory,
// the launch shape, and the barrier state.  plan() rebuilds them when the
// scenes or the solver settings change; launch() queues one solve.
class MgSolver {
public:
    MgSolver() = default;
    ~MgSolver();
    MgSolver(const MgSolver&) = delete;
    MgSolver& operator=(const MgSolver&) = delete;
    bool plan(int device, const std::vector<MgScene>& scenes, int maxCycles, int pre, int post, double tolerance, cudaStream_t stream,
              std::string& err);
    bool planned() const { return planned_; }
    // Queues the barrier reset and the cooperative launch on `stream`; a wait
    // that runs out writes kMgStatusFlag | phase into *hostStatus (host-mapped).
    bool launch(cudaStream_t stream, unsigned* hostStatus, std::string& err);
    void release();
    int gridBlocks() const { return grid_; }

private:
    MgScene* dScenes_ = nullptr;  // kMgMaxScenes descriptors
    MgPlan* dPlan_ = nullptr;
    MgSync* dSync_ = nullptr;
    // Pinned staging of the uploads, a ring of kStaging slots: a new plan
    // waits only for the upload made kStaging plans ago, not the last one.
    static constexpr int kStaging = 3;
    MgScene* hScenesRing_[kStaging] = {};
    MgPlan* hPlanRing_[kStaging] = {};
    cudaEvent_t uploadedRing_[kStaging] = {};
    int slot_ = 0;
    bool planned_ = false;
    size_t smem_ = 0;
    int grid_ = 0, sms_ = 0;
    unsigned long long waitNs_ = 1000000000ull;
};

// Host-side fault injection of Scene's device allocations: -1 = off; n >= 0 =
// n more allocations succeed, then every one fails with cudaErrorMemoryAllocation.
void setAllocationFault(long long succeedBeforeFailing);

// Defaults of FirePhysicsParams for a grid (fireCudaDefaultPhysicsParams).
void defaultPhysicsParams(FirePhysicsParams& params, int nx, int ny, int nz);
// Range and finiteness checks of fireCudaSetPhysicsParams.
bool validatePhysicsParams(const FirePhysicsParams& params, std::string& err);

// Autotuner of the resident SOR's brick shape (process-wide): on by default;
// the measured choice per device and grid (-1: not timed yet).
bool autotuneEnabled();
void setAutotune(bool enabled);
int tunedBrick(int device, int nx, int ny, int nz);
void rememberTunedBrick(int device, int nx, int ny, int nz, int pick, float msLarge, float msSmall);
bool tunedBrickRecord(int device, int nx, int ny, int nz, int& pick, float& msLarge, float& msSmall);

class Scene {
public:
    Scene() = default;
    ~Scene();
    Scene(const Scene&) = delete;
    Scene& operator=(const Scene&) = delete;

    bool init(int device, int frameW, int frameH, int nx, int ny, int nz, std::string& err);

    // The reference's settings clamps (src/fire_cuda.cu:3135-3179) and the
    // host-computed camera basis (:2696-2704).
    FrameParams paramsFrom(const FireSettings& s, float time) const;
    // makeParams() defaults of the reference (src/fire_cuda.cu:2655-2694), used by fireCudaReset.
    FrameParams defaultParams(float time) const;

    bool runStages(int first, int last, const FrameParams& p, std::string& err);
    // One frame with the reference's time bookkeeping (src/fire_cuda.cu:3106-3549).
    bool frame(uint32_t* hostBgra, const FireSettings& s, FireCudaFrameMetrics* metrics, bool toHdrSlot, bool advance, bool render,
               std::string& err);
    bool reset(std::string& err);

    bool getField(int field, void* host, size_t bytes, std::string& err);
    bool setField(int field, const void* host, size_t bytes, std::string& err);
    bool registerHdrSlot(int slot, void* ptr, size_t pitch, int format, std::string& err);
    bool setActiveSlot(int slot, std::string& err);
    void clearSlots();
    bool setPressureSolver(int iterations, float omega, std::string& err);
    // 0 = automatic (shared-memory-resident when the grid fits co-resident), 1 = colour-split, 2 = resident only.
    bool setPressurePath(int path, std::string& err);
    int lastPressurePath() const { return lastPressurePath_; }
    // The brick of the resident solve (after its first solve), or false.
    bool residentBrick(int& bx, int& by, int& bz) const;
    // Fault injection for the resident SOR's bounded waits: brick `silentBrick`
    // (-1 = none) never announces its half sweeps; each wait gives up after waitUs.
    bool setResidentFault(int silentBrick, long long waitUs, std::string& err);
    // Residual-gated solve: stop once max |r| <= tolerance, checked every checkEvery iterations
    // (tolerance 0 = the fixed iteration count).
    bool setPressureTolerance(double tolerance, int checkEvery, std::string& err);
    // Iterations run, max |r| and the FP64 L2 residual of the latest gated solve (waits for the stream).
    bool pressureStats(int& iterations, float& maxResidual, double& l2Residual, std::string& err);
    // Hash lattices on (default) or off: off hashes every fbm corner in place (same bits, slower).
    void setHashLattices(bool enabled) { latticesEnabled_ = enabled; }
    // Multigrid pressure solve (config physics with a Dirichlet top); maxCycles 0 = red-black SOR.
    bool setPressureMultigrid(int maxCycles, int preSmooth, int postSmooth, std::string& err);
    // Physics of the following passes (mode 0 reference, mode 1 config physics).
    bool setPhysics(const FirePhysicsParams& params, std::string& err);
    const FirePhysicsParams& physics() const { return physics_; }
    // Steps of the config physics since the last reset (the emitter jitter's counter).
    unsigned long long configStep() const { return cfgStep_; }
    bool synchronize(std::string& err);
    // After a host sync: fails once with "timed out" if a resident SOR wait ran out since the last check.
    bool checkSolverStatus(std::string& err);
    size_t deviceBytes() const { return deviceBytes_; }
    unsigned long long launchCount() const { return launches_; }

    int nx = 0, ny = 0, nz = 0, lnx = 0, lny = 0, lnz = 0, frameW = 0, frameH = 0, device = 0;
    float simTime = 0.0f, renderTime = 0.0f;
    int frameIndex = 0;
    int pressureIterations = kDefaultPressureIterations;
    float pressureOmega = kDefaultPressureOmega;
    cudaStream_t stream = nullptr;

private:
    bool check(const char* label, cudaError_t e, std::string& err);
    bool alloc(void** p, size_t bytes, const char* label, std::string& err);
    void release();
    ScalarFieldsIn scalarsIn() const;
    ScalarFields scalarsOut() const;
    Velocity velocity() const;
    bool ensureMaterial(const FrameParams& p, std::string& err);
    bool runSor(const FrameParams& p, std::string& err);
    bool runMetrics(const FrameParams& p, std::string& err);
    bool fillMetrics(FireCudaFrameMetrics* out, std::string& err);

    unsigned long long launches_ = 0;
    size_t cells_ = 0, nu_ = 0, nv_ = 0, nw_ = 0, lightCells_ = 0, pixels_ = 0, deviceBytes_ = 0;
    Rec4* sa_[2] = {};
    Rec4* sb_[2] = {};
    Rec2* sc_[2] = {};
    int cur_ = 0;
    FaceT* vel_[3][2] = {};
    int vcur_ = 0;
    float* pressure_ = nullptr;
    float* divergence_ = nullptr;
    float* divergenceAfter_ = nullptr;
    float4* contrib_ = nullptr;
    float* material_ = nullptr;
    float* breathing_ = nullptr;
    MaterialKey materialKey_;
    float4* light_ = nullptr;
    float4* lightNext_ = nullptr;
    float* shadow_ = nullptr;
    float4* hdr_ = nullptr;
    uint32_t* bgra_ = nullptr;
    EmberSplat* embers_ = nullptr;
    MetricPartial* partials_ = nullptr;
    MetricPartial* metricDevice_ = nullptr;
    MetricPartial* metricHost_ = nullptr;
    HdrSlot slots_[4];
    int activeSlot_ = 0;
    cudaEvent_t events_[9] = {};
    bool residentPlan(ResidentBrick& r, size_t& smemBytes, int& threads);
    // Times one solve with each brick shape that fits (both from the same
    // pressure, which is put back) and keeps the faster (autotuneResident).
    bool tuneResident(std::string& err);
    int planState_ = 0;  // 0 not planned, 1 resident plan, 2 no resident plan
    ResidentBrick plan_{};
    size_t planSmem_ = 0;
    int planThreads_ = 0;
    // Brick shapes that fit co-resident, for the autotuner (tuneCount_ > 1:
    // not yet timed for this grid).
    ResidentBrick tuneBricks_[2]{};
    size_t tuneSmem_[2] = {0, 0};
    int tuneThreads_[2] = {0, 0};
    int tuneCount_ = 0;
    int pressurePath_ = 0;
    int lastPressurePath_ = 0;
    cudaGraphExec_t sorExec_ = nullptr;
    // hash21 lattices of the two curl-noise fbm call sites of the force pass.
    bool latticesEnabled_ = true;
    bool curlLattices(const FrameParams& p, HashLattice2& a, HashLattice2& b) const;
    float* curlLattice_ = nullptr;
    size_t curlCapacity_[2] = {0, 0};
    // hash21 lattice of the fuel-bed source noise of the advect/react pass.
    bool sourceLattice(const FrameParams& p, HashLattice2& l) const;
    float* sourceLattice_ = nullptr;
    size_t sourceCapacity_ = 0;
    // Raymarch work list: tile order (centre first) and the tile counter.
    int* rayTileOrder_ = nullptr;
    int* rayTileCounter_ = nullptr;
    int rayTilesX_ = 0, rayTileCount_ = 0;
    int rayBlocks_[4] = {0, 0, 0, 0};  // persistent grid of raymarch, raymarchScene0..2
    double pressureTolerance_ = 0.0;
    int pressureCheckEvery_ = 10;
    bool lastSolveGated_ = false;
    SorGate* sorGate_ = nullptr;
    double* residualSq_ = nullptr;
    float* residualMax_ = nullptr;
    unsigned* sorStatus_ = nullptr;               // device: failure tag of the resident SOR
    unsigned long long* sorExchange_ = nullptr;   // device: one tagged word per cell (face cells)
    unsigned* sorHostStatus_ = nullptr;  // host-mapped: brick + 1 of a wait that ran out
    unsigned sorEpoch_ = 0;
    int sorSilentBrick_ = -1;
    unsigned long long sorWaitNs_ = 1000000000ull;
    float* split_ = nullptr;      // colour-split p of the non-resident solve (allocated on first use)
    float* splitDiv_ = nullptr;   // colour-split div
    double sorTolKey_ = -1.0;
    int sorChunkKey_ = -1;
    int sorGraphLaunches_ = 0;
    int sorIterations_ = -1;
    float sorOmega_ = 0.0f;
    // Config physics.
    FirePhysicsParams physics_{};
    float4* cfgVort_ = nullptr;   // vorticity (x, y, z, |omega|) per cell, allocated on first use
    float* cfgLight_ = nullptr;   // transmittance to the point light, half resolution
    float4* cfgNoise_ = nullptr;  // curl-noise acceleration per cell, rebuilt when its parameters change
    bool cfgNoiseValid_ = false;
    float cfgNoiseKey_[3] = {0.0f, 0.0f, 0.0f};
    unsigned cfgNoiseSeed_ = 0;
    int cfgLx_ = 0, cfgLy_ = 0, cfgLz_ = 0;
    unsigned long long cfgStep_ = 0;
    ConfigParams configParams() const;
    // Multigrid: levels, their buffers (mgP_[0] is the increment, the level-0
    // rhs is divergence_), the residual chunks, this scene's descriptor and its solver.
    int mgCycles_ = 0, mgPre_ = 2, mgPost_ = 2;
    std::vector<MgLevel> mgLevels_;
    std::vector<float*> mgP_, mgRhs_;  // mgRhs_[0] is unused (divergence_)
    double* mgChunkSq_ = nullptr;
    bool mgDeltaValid_ = false;        // mgP_[0] holds the latest solve's increment (the subtraction takes it)
    MgSolver mgSolver_;
    int mgKeyCycles_ = -1, mgKeyPre_ = -1, mgKeyPost_ = -1;
    double mgKeyTol_ = -1.0;
    bool runMultigrid(std::string& err);

public:
    // The multigrid buffers of this scene (allocated on first use) and its
    // descriptor for a batched solve.
    bool multigridScene(MgScene& out, std::string& err);
    // Incremental projection under a Dirichlet top with the multigrid solve.
    bool incrementalProjection() const { return physics_.mode == 1 && physics_.pressureTop == 1 && mgCycles_ > 0; }
    int multigridCycles() const { return mgCycles_; }
    int multigridPre() const { return mgPre_; }
    int multigridPost() const { return mgPost_; }
    double pressureTolerance() const { return pressureTolerance_; }
    unsigned* hostStatus() const { return sorHostStatus_; }
    // One step inside a FireBatch (see fire_batch.cu): bookkeeping, buffers and
    // this step's descriptor; the batch queues the kernels on `stream`.
    bool batchStep(BatchScene& d, const FireSettings& s, bool render, std::string& err);
    // Allocates every buffer batchStep can need, so that later batched steps allocate nothing.
    bool prepareBatched(std::string& err);
    void addLaunches(unsigned long long n) { launches_ += n; }
    bool hasHdrOutput() const { return slots_[activeSlot_].ptr != nullptr; }
    // The stream this scene created (`stream` is it, except while a batch holds the scene).
    cudaStream_t ownStream() const { return ownStream_; }

private:
    cudaStream_t ownStream_ = nullptr;
    bool ensureConfigBuffers(std::string& err);
    bool runConfigStages(int first, int last, const FrameParams& p, std::string& err);
};

// Steps a set of config-physics scenes (incremental multigrid projection)
// together on one stream: per sub-step one upload of their step descriptors,
// one launch per stage over all of them (fire_config.cu, batch*) and one
// persistent multigrid launch (fire_mg.cu).  The set may change between
// sub-steps (setScenes re-plans without allocating or synchronising); the
// scenes' own work must be on stream() (callers point Scene::stream at it).
class BatchRunner {
public:
    BatchRunner() = default;
    ~BatchRunner();
    BatchRunner(const BatchRunner&) = delete;
    BatchRunner& operator=(const BatchRunner&) = delete;
    bool init(int device, std::string& err);
    bool setScenes(const std::vector<Scene*>& scenes, std::string& err);
    // One sub-step of every scene of the set (settings[i] and render[i] for scene i).
    bool run(const FireSettings* settings, const int* render, std::string& err);
    void release();
    cudaStream_t stream() const { return stream_; }
    unsigned* hostStatus() const { return hostStatus_; }
    unsigned long long launches() const { return launches_; }
    const std::vector<Scene*>& scenes() const { return scenes_; }
    // After a stream sync: fails once if a multigrid barrier wait ran out since the last check.
    bool checkStatus(std::string& err);

private:
    static constexpr int kRing = 2;  // pinned descriptor buffers in flight
    int device_ = 0;
    std::vector<Scene*> scenes_;
    cudaStream_t stream_ = nullptr;
    MgSolver solver_;
    BatchScene* dScenes_ = nullptr;   // kBatchMaxScenes
    BatchPlan* dPlan_ = nullptr;
    unsigned char* host_[kRing] = {};  // pinned: kBatchMaxScenes descriptors + a plan
    cudaEvent_t copied_[kRing] = {};
    int slot_ = 0;
    unsigned* hostStatus_ = nullptr;  // host-mapped
    unsigned long long launches_ = 0;
};

}  // namespace firesim

// The opaque FireScene handle of fire_ext.h: one Scene and its device.
struct FireScene {
    std::unique_ptr<firesim::Scene> scene;
    int device = 0;
};
