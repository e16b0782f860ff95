// fire_scene.cu -- allocation, launch sequencing and clocks of one scene.
#include "fire_scene.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <atomic>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

namespace firesim {

namespace {

enum Stage {
    kAdvectVelocity = 0, kAdvectReact, kForce, kVelocityBoundary, kDivergence, kPressureSor, kSubtract, kWallBoundary,
    kLightBuild, kLightPropagate, kRender, kEmbers, kTonemap, kOverlay, kMetrics, kReset,
};

enum Event { kStart = 0, kAfterVelocity, kAfterReaction, kAfterProjection, kAfterSolve, kAfterLighting, kAfterRaymarch, kAfterPack, kAfterRender };

int clampI(int v, int lo, int hi) { return std::max(lo, std::min(hi, v)); }
float clampF(float v, float lo, float hi) { return std::max(lo, std::min(hi, v)); }

// Threads along x for a row of n cells (rows are launched one CTA row each).
int rowThreads(int n) { return n <= 32 ? 32 : (n <= 64 ? 64 : 128); }

dim3 cellGrid(int bx, int n, int ny, int nz) { return dim3((n + bx - 1) / bx, ny, nz); }

}  // namespace

bool MaterialKey::operator==(const MaterialKey& o) const {
    return sceneId == o.sceneId && emitterRadius == o.emitterRadius && emitterCenterX == o.emitterCenterX &&
           emitterCenterZ == o.emitterCenterZ && burnerCenterCount == o.burnerCenterCount && burnerX0 == o.burnerX0 &&
           burnerZ0 == o.burnerZ0;
}

Scene::~Scene() { release(); }

bool Scene::check(const char* label, cudaError_t e, std::string& err) {
    if (e != cudaSuccess) {
        err = std::string(label) + ": " + cudaGetErrorString(e);
        return false;
    }
    return true;
}

// Host-side fault injection of the scenes' device allocations
// (fireCudaSetAllocationFault): -1 = off; n >= 0 = n more allocations
// succeed, then every one fails as cudaMalloc does when memory runs out.
std::atomic<long long> g_allocationsBeforeFault{-1};

void setAllocationFault(long long succeedBeforeFailing) { g_allocationsBeforeFault.store(succeedBeforeFailing); }

bool Scene::alloc(void** p, size_t bytes, const char* label, std::string& err) {
    long long left = g_allocationsBeforeFault.load();
    while (left >= 0) {
        if (left == 0) {
            *p = nullptr;
            err = std::string(label) + ": " + cudaGetErrorString(cudaErrorMemoryAllocation) + " (injected)";
            return false;
        }
        if (g_allocationsBeforeFault.compare_exchange_weak(left, left - 1)) break;
    }
    // The buffer's name for the bounds-checking build's reports: the label without "cudaMalloc ".
    const char* name = std::strncmp(label, "cudaMalloc ", 11) == 0 ? label + 11 : label;
    if (!check(label, deviceAlloc(p, bytes, name), err)) {
        *p = nullptr;
        return false;
    }
    deviceBytes_ += bytes;
    return true;
}

void Scene::release() {
    if (device >= 0 && (stream != nullptr || sa_[0] != nullptr)) {
        cudaSetDevice(device);
    }
    if (stream != nullptr) {
        cudaStreamSynchronize(stream);
    }
    if (ownStream_ != nullptr && ownStream_ != stream) {
        cudaStreamSynchronize(ownStream_);
    }
    if (sorExec_ != nullptr) {
        cudaGraphExecDestroy(sorExec_);
        sorExec_ = nullptr;
    }
    mgSolver_.release();
    mgDeltaValid_ = false;
    for (float* b : mgP_) {
        deviceFree(b);
    }
    for (float* b : mgRhs_) {
        deviceFree(b);
    }
    deviceFree(mgChunkSq_);
    mgChunkSq_ = nullptr;
    mgP_.clear();
    mgRhs_.clear();
    mgLevels_.clear();
    mgKeyCycles_ = -1;
    void* bufs[] = {sa_[0], sa_[1], sb_[0], sb_[1], sc_[0], sc_[1], vel_[0][0], vel_[0][1], vel_[1][0], vel_[1][1], vel_[2][0],
                    vel_[2][1], pressure_, divergence_, divergenceAfter_, contrib_, material_, breathing_, light_, lightNext_,
                    shadow_, hdr_, bgra_, embers_, partials_, metricDevice_, sorStatus_, sorExchange_, curlLattice_, sourceLattice_,
                    rayTileOrder_, rayTileCounter_, sorGate_, residualSq_, residualMax_, split_, splitDiv_,
                    cfgVort_, cfgLight_, cfgNoise_};
    for (void* b : bufs) {
        deviceFree(b);
    }
    if (metricHost_ != nullptr) cudaFreeHost(metricHost_);
    if (sorHostStatus_ != nullptr) cudaFreeHost(sorHostStatus_);
    sorStatus_ = nullptr;
    sorExchange_ = nullptr;
    rayTileOrder_ = nullptr;
    rayTileCounter_ = nullptr;
    sorGate_ = nullptr;
    residualSq_ = nullptr;
    residualMax_ = nullptr;
    split_ = nullptr;
    splitDiv_ = nullptr;
    cfgVort_ = nullptr;
    cfgLight_ = nullptr;
    cfgNoise_ = nullptr;
    cfgNoiseValid_ = false;
    sorHostStatus_ = nullptr;
    curlLattice_ = nullptr;
    sourceLattice_ = nullptr;
    for (cudaEvent_t& e : events_) {
        if (e != nullptr) cudaEventDestroy(e);
        e = nullptr;
    }
    if (ownStream_ != nullptr) cudaStreamDestroy(ownStream_);
    ownStream_ = nullptr;
    stream = nullptr;
    std::memset(sa_, 0, sizeof(sa_));
    std::memset(sb_, 0, sizeof(sb_));
    std::memset(sc_, 0, sizeof(sc_));
    std::memset(vel_, 0, sizeof(vel_));
    pressure_ = divergence_ = divergenceAfter_ = material_ = breathing_ = shadow_ = nullptr;
    contrib_ = light_ = lightNext_ = hdr_ = nullptr;
    bgra_ = nullptr;
    embers_ = nullptr;
    partials_ = metricDevice_ = metricHost_ = nullptr;
    deviceBytes_ = 0;
}

bool Scene::init(int dev, int fw, int fh, int x, int y, int z, std::string& err) {
    if (x < 2 || y < 2 || z < 2 || fw < 1 || fh < 1) {
        err = "invalid grid or frame dimensions";
        return false;
    }
    const long long cells = static_cast<long long>(x) * y * z;
    if (cells > (1LL << 30) || static_cast<long long>(fw) * fh > (1LL << 28) || y > 65535 || z > 65535 || fh > 65535 * 8) {
        err = "grid or frame too large for the 32-bit index layout";
        return false;
    }
    device = dev;
    nx = x;
    ny = y;
    nz = z;
    frameW = fw;
    frameH = fh;
    defaultPhysicsParams(physics_, nx, ny, nz);
    cfgStep_ = 0;
    // Light grid, src/fire_cuda.cu:2920-2922.
    lnx = clampI((nx + 3) / 4, 18, 48);
    lny = clampI((ny + 3) / 4, 20, 56);
    lnz = clampI((nz + 3) / 4, 16, 36);
    cells_ = static_cast<size_t>(cells);
    nu_ = static_cast<size_t>(nx + 1) * ny * nz;
    nv_ = static_cast<size_t>(nx) * (ny + 1) * nz;
    nw_ = static_cast<size_t>(nx) * ny * (nz + 1);
    lightCells_ = static_cast<size_t>(lnx) * lny * lnz;
    pixels_ = static_cast<size_t>(fw) * fh;
    if (!check("cudaSetDevice", cudaSetDevice(device), err)) return false;
    if (!check("cudaStreamCreate", cudaStreamCreateWithFlags(&ownStream_, cudaStreamNonBlocking), err)) return false;
    stream = ownStream_;
    bool ok = true;
    for (int i = 0; i < 2 && ok; ++i) {
        ok = alloc(reinterpret_cast<void**>(&sa_[i]), cells_ * sizeof(Rec4), "cudaMalloc scalars a", err) &&
             alloc(reinterpret_cast<void**>(&sb_[i]), cells_ * sizeof(Rec4), "cudaMalloc scalars b", err) &&
             alloc(reinterpret_cast<void**>(&sc_[i]), cells_ * sizeof(Rec2), "cudaMalloc scalars c", err) &&
             alloc(reinterpret_cast<void**>(&vel_[0][i]), nu_ * sizeof(FaceT), "cudaMalloc u", err) &&
             alloc(reinterpret_cast<void**>(&vel_[1][i]), nv_ * sizeof(FaceT), "cudaMalloc v", err) &&
             alloc(reinterpret_cast<void**>(&vel_[2][i]), nw_ * sizeof(FaceT), "cudaMalloc w", err);
    }
    ok = ok && alloc(reinterpret_cast<void**>(&pressure_), cells_ * sizeof(float), "cudaMalloc pressure", err) &&
         alloc(reinterpret_cast<void**>(&divergence_), cells_ * sizeof(float), "cudaMalloc divergence", err) &&
         alloc(reinterpret_cast<void**>(&divergenceAfter_), cells_ * sizeof(float), "cudaMalloc divergence after", err) &&
         alloc(reinterpret_cast<void**>(&contrib_), cells_ * sizeof(float4), "cudaMalloc force scratch", err) &&
         alloc(reinterpret_cast<void**>(&material_), static_cast<size_t>(nx) * nz * sizeof(float), "cudaMalloc material", err) &&
         alloc(reinterpret_cast<void**>(&breathing_), static_cast<size_t>(nx) * nz * sizeof(float), "cudaMalloc breathing", err) &&
         alloc(reinterpret_cast<void**>(&light_), lightCells_ * sizeof(float4), "cudaMalloc scene light", err) &&
         alloc(reinterpret_cast<void**>(&lightNext_), lightCells_ * sizeof(float4), "cudaMalloc scene light next", err) &&
         alloc(reinterpret_cast<void**>(&shadow_), lightCells_ * sizeof(float), "cudaMalloc scene shadow", err) &&
         alloc(reinterpret_cast<void**>(&hdr_), pixels_ * sizeof(float4), "cudaMalloc hdr frame", err) &&
         alloc(reinterpret_cast<void**>(&bgra_), pixels_ * sizeof(uint32_t), "cudaMalloc frame", err) &&
         alloc(reinterpret_cast<void**>(&embers_), kMaxEmberCount * sizeof(EmberSplat), "cudaMalloc embers", err) &&
         alloc(reinterpret_cast<void**>(&partials_), kMetricBlocks * sizeof(MetricPartial), "cudaMalloc metric partials", err) &&
         alloc(reinterpret_cast<void**>(&metricDevice_), sizeof(MetricPartial), "cudaMalloc metrics", err) &&
         check("cudaMallocHost metrics", cudaMallocHost(reinterpret_cast<void**>(&metricHost_), sizeof(MetricPartial)), err);
    // Raymarch tiles, ordered by distance of the tile centre from the frame
    // centre (ties by id), and a persistent grid that fills every SM.
    if (ok) {
        rayTilesX_ = (fw + kRayTileW - 1) / kRayTileW;
        const int tilesY = (fh + kRayTileH - 1) / kRayTileH;
        rayTileCount_ = rayTilesX_ * tilesY;
        std::vector<int> order(rayTileCount_);
        std::vector<double> dist(rayTileCount_);
        for (int t = 0; t < rayTileCount_; ++t) {
            order[t] = t;
            const double cx = ((t % rayTilesX_) + 0.5) * kRayTileW - 0.5 * fw;
            const double cy = ((t / rayTilesX_) + 0.5) * kRayTileH - 0.5 * fh;
            dist[t] = cx * cx + cy * cy;
        }
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return dist[a] < dist[b]; });
        int sms = 0, perSm = 0;
        ok = alloc(reinterpret_cast<void**>(&rayTileOrder_), order.size() * sizeof(int), "cudaMalloc ray tiles", err) &&
             alloc(reinterpret_cast<void**>(&rayTileCounter_), sizeof(int), "cudaMalloc ray tile counter", err) &&
             check("upload ray tiles", cudaMemcpy(rayTileOrder_, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice), err) &&
             check("SM count", cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), err);
        const void* kernels[4] = {reinterpret_cast<const void*>(raymarch), reinterpret_cast<const void*>(raymarchScene0),
                                  reinterpret_cast<const void*>(raymarchScene1), reinterpret_cast<const void*>(raymarchScene2)};
        for (int k = 0; ok && k < 4; ++k) {
            ok = check("raymarch occupancy", cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernels[k], 128, 0), err);
            rayBlocks_[k] = std::max(1, sms * std::max(1, perSm));
        }
    }
    ok = ok && alloc(reinterpret_cast<void**>(&sorGate_), sizeof(SorGate), "cudaMalloc SOR gate", err) &&
         check("clear SOR gate", cudaMemsetAsync(sorGate_, 0, sizeof(SorGate), stream), err) &&
         alloc(reinterpret_cast<void**>(&residualSq_), kResidualBlocks * sizeof(double), "cudaMalloc residual partials", err) &&
         alloc(reinterpret_cast<void**>(&residualMax_), kResidualBlocks * sizeof(float), "cudaMalloc residual maxima", err);
    // Resident SOR: the tagged exchange words (zero tags never match) and the failure status.
    ok = ok && alloc(reinterpret_cast<void**>(&sorExchange_), cells_ * sizeof(unsigned long long), "cudaMalloc SOR exchange", err) &&
         check("clear SOR exchange", cudaMemsetAsync(sorExchange_, 0, cells_ * sizeof(unsigned long long), stream), err) &&
         alloc(reinterpret_cast<void**>(&sorStatus_), sizeof(unsigned), "cudaMalloc SOR status", err) &&
         check("clear SOR status", cudaMemsetAsync(sorStatus_, 0, sizeof(unsigned), stream), err) &&
         check("cudaHostAlloc SOR status", cudaHostAlloc(reinterpret_cast<void**>(&sorHostStatus_), sizeof(unsigned), cudaHostAllocMapped), err);
    if (ok) *sorHostStatus_ = 0;
    {
        // Lattice sizes do not depend on time: plan at t = 0 with one extra
        // lattice cell of slack per axis.
        FrameParams p0{};
        HashLattice2 a, b;
        curlCapacity_[0] = curlCapacity_[1] = 1u << 30;
        curlLattices(p0, a, b);
        curlCapacity_[0] = static_cast<size_t>(a.offset[kFbmOctaves - 1] + (a.sx[kFbmOctaves - 1] + 1) * (a.sy[kFbmOctaves - 1] + 1)) + 4096;
        curlCapacity_[1] = static_cast<size_t>(b.offset[kFbmOctaves - 1] + (b.sx[kFbmOctaves - 1] + 1) * (b.sy[kFbmOctaves - 1] + 1)) + 4096;
        ok = ok && alloc(reinterpret_cast<void**>(&curlLattice_), (curlCapacity_[0] + curlCapacity_[1]) * sizeof(float), "cudaMalloc curl lattices", err);
        HashLattice2 src;
        sourceCapacity_ = 1u << 30;
        sourceLattice(p0, src);
        sourceCapacity_ =
            static_cast<size_t>(src.offset[kFbmOctaves - 1] + (src.sx[kFbmOctaves - 1] + 1) * (src.sy[kFbmOctaves - 1] + 1)) + 4096;
        ok = ok && alloc(reinterpret_cast<void**>(&sourceLattice_), sourceCapacity_ * sizeof(float), "cudaMalloc source lattice", err);
    }
    for (int i = 0; i < 9 && ok; ++i) {
        ok = check("cudaEventCreate", cudaEventCreate(&events_[i]), err);
    }
    ok = ok && check("clear hdr", cudaMemsetAsync(hdr_, 0, pixels_ * sizeof(float4), stream), err) &&
         check("clear frame", cudaMemsetAsync(bgra_, 0, pixels_ * sizeof(uint32_t), stream), err);
    if (!ok) {
        release();
        return false;
    }
    return true;
}

ScalarFieldsIn Scene::scalarsIn() const { return {sa_[cur_], sb_[cur_], sc_[cur_]}; }
ScalarFields Scene::scalarsOut() const { return {sa_[1 - cur_], sb_[1 - cur_], sc_[1 - cur_]}; }
Velocity Scene::velocity() const { return {vel_[0][vcur_], vel_[1][vcur_], vel_[2][vcur_]}; }

FrameParams Scene::paramsFrom(const FireSettings& s, float time) const {
    FrameParams p{};
    p.nx = nx; p.ny = ny; p.nz = nz; p.frameW = frameW; p.frameH = frameH; p.lnx = lnx; p.lny = lny; p.lnz = lnz;
    p.dt = clampF(s.dt, 0.001f, 1.0f / 30.0f);
    p.time = time;
    p.mouseX = clampF(s.mouseX, 0.0f, 1.0f);
    p.mouseY = clampF(s.mouseY, 0.0f, 1.0f);
    p.leftDown = s.leftDown;
    p.rightDown = s.rightDown;
    p.showGizmos = s.showGizmos;
    p.activeGizmo = s.activeGizmo;
    p.sceneId = clampI(s.sceneId, 0, kSceneCount - 1);
    p.wind = clampF(s.wind, -1.0f, 1.0f);
    p.turbulence = clampF(s.turbulence, 0.05f, 1.8f);
    p.detail = clampF(s.detail, 0.1f, 1.5f);
    p.smokeGain = clampF(s.smoke, 0.0f, 1.6f);
    p.intensity = clampF(s.intensity, 0.2f, 2.4f);
    const float yaw = s.cameraYaw;
    const float pitch = clampF(s.cameraPitch, -0.75f, 0.75f);
    const float distance = clampF(s.cameraDistance, 1.5f, 6.0f);
    p.cinematicMode = s.cinematicMode != 0 ? 1 : 0;
    p.raymarchSteps = clampI(s.raymarchSteps, 24, kMaxRaymarchSteps);
    p.emberCount = clampI(s.emberCount, 0, kMaxEmberCount);
    p.renderDebugMode = clampI(s.renderDebugMode, 0, 6);
    p.exposure = clampF(s.exposure, 0.45f, 2.40f);
    p.reflectionGain = clampF(s.reflectionGain, 0.0f, 2.2f);
    p.smokeDarkness = clampF(s.smokeDarkness, 0.35f, 2.4f);
    p.emitterCenterX = clampF(s.emitterCenterX, -1.05f, 1.05f);
    p.emitterCenterZ = clampF(s.emitterCenterZ, -0.82f, 0.82f);
    p.emitterHeightNorm = clampF(s.emitterHeightNorm, 0.0f, 0.96f);
    p.emitterHeightBandNorm = clampF(s.emitterHeightBandNorm, 0.006f, 0.20f);
    p.emitterRadius = clampF(s.emitterRadius, 0.035f, 0.80f);
    p.burnerCenterCount = clampI(s.burnerCenterCount, 0, 4);
    for (int i = 0; i < 4; ++i) {
        p.burnerCenterX[i] = clampF(s.burnerCenterX[i], -1.05f, 1.05f);
        p.burnerCenterY[i] = clampF(s.burnerCenterY[i], 0.0f, 2.03f);
        p.burnerCenterZ[i] = clampF(s.burnerCenterZ[i], -0.82f, 0.82f);
    }
    if (p.sceneId == 2 && p.burnerCenterCount > 0) {
        p.emitterHeightNorm = clampF((p.burnerCenterY[0] - 0.02f) / 2.03f, 0.0f, 0.96f);
    }
    // Camera basis, evaluated on the host as the reference does (src/fire_cuda.cu:315-329).
    const float3 target = make_float3(0.0f, 0.72f, 0.0f);
    const float cp = std::cos(pitch);
    p.eye = make_float3(std::sin(yaw) * distance * cp, target.y + std::sin(pitch) * distance, std::cos(yaw) * distance * cp);
    p.forward = normalize3(sub3(target, p.eye));
    p.right = normalize3(cross3(p.forward, make_float3(0.0f, 1.0f, 0.0f)));
    p.up = normalize3(cross3(p.right, p.forward));
    p.tanHalfFov = 0.50f;
    p.aspect = static_cast<float>(frameW) / static_cast<float>(frameH);
    return p;
}

FrameParams Scene::defaultParams(float time) const {
    FireSettings s{};
    s.dt = 1.0f / 60.0f;
    s.mouseX = 0.5f;
    s.mouseY = 0.12f;
    s.sceneId = 0;
    s.turbulence = 0.72f;
    s.detail = 0.88f;
    s.smoke = 0.92f;
    s.intensity = 1.0f;
    s.cameraPitch = 0.18f;
    s.cameraDistance = 3.35f;
    s.cinematicMode = 1;
    s.raymarchSteps = 56;
    s.emberCount = 96;
    s.showGizmos = 0;
    s.activeGizmo = 0;
    return paramsFrom(s, time);
}

bool Scene::ensureMaterial(const FrameParams& p, std::string& err) {
    MaterialKey key;
    key.sceneId = p.sceneId;
    key.emitterRadius = p.emitterRadius;
    key.emitterCenterX = p.emitterCenterX;
    key.emitterCenterZ = p.emitterCenterZ;
    key.burnerCenterCount = p.burnerCenterCount;
    key.burnerX0 = p.burnerCenterX[0];
    key.burnerZ0 = p.burnerCenterZ[0];
    const int withMaterial = key == materialKey_ ? 0 : 1;
    const int bx = rowThreads(nx);
    fuelBedTables<<<dim3((nx + bx - 1) / bx, nz), bx, 0, stream>>>(material_, breathing_, p, withMaterial);
    launches_ += 1;
    if (!check("fuel bed tables launch", cudaGetLastError(), err)) return false;
    materialKey_ = key;
    return true;
}

bool Scene::setPressureSolver(int iterations, float omega, std::string& err) {
    if (iterations < 0 || iterations > 100000 || !(omega > 0.0f && omega < 2.0f)) {
        err = "pressure solver: iterations must be in [0, 100000] and omega in (0, 2)";
        return false;
    }
    pressureIterations = iterations;
    pressureOmega = omega;
    return true;
}

bool Scene::setPressurePath(int path, std::string& err) {
    if (path < 0 || path > 2) {
        err = "pressure path must be 0 (automatic), 1 (per-launch) or 2 (resident)";
        return false;
    }
    pressurePath_ = path;
    return true;
}

namespace {

// Measured brick choices of the resident solve, per device and grid, for the
// life of the process: index 0 = 32x16x16, 1 = 16x16x16, with both timings.
struct TunedBrick {
    int pick;
    float ms[2];
};
std::mutex g_tuneMutex;
std::map<std::tuple<int, int, int, int>, TunedBrick> g_tuned;
std::atomic<bool> g_autotune{true};

}  // namespace

bool autotuneEnabled() { return g_autotune.load(); }
void setAutotune(bool enabled) { g_autotune.store(enabled); }

int tunedBrick(int device, int nx, int ny, int nz) {
    std::lock_guard<std::mutex> lock(g_tuneMutex);
    const auto it = g_tuned.find(std::make_tuple(device, nx, ny, nz));
    return it == g_tuned.end() ? -1 : it->second.pick;
}

void rememberTunedBrick(int device, int nx, int ny, int nz, int pick, float msLarge, float msSmall) {
    std::lock_guard<std::mutex> lock(g_tuneMutex);
    g_tuned[std::make_tuple(device, nx, ny, nz)] = TunedBrick{pick, {msLarge, msSmall}};
}

bool tunedBrickRecord(int device, int nx, int ny, int nz, int& pick, float& msLarge, float& msSmall) {
    std::lock_guard<std::mutex> lock(g_tuneMutex);
    const auto it = g_tuned.find(std::make_tuple(device, nx, ny, nz));
    if (it == g_tuned.end()) return false;
    pick = it->second.pick;
    msLarge = it->second.ms[0];
    msSmall = it->second.ms[1];
    return true;
}

// Brick plan of the shared-memory-resident SOR: 32x16x16 bricks (256 threads,
// 93 KB of shared memory, two CTAs per SM), or 16^3 bricks (128 threads, 67 KB)
// when the larger ones do not fit co-resident; one CTA per brick.
bool Scene::residentPlan(ResidentBrick& r, size_t& smemBytes, int& threads) {
    if (planState_ != 0) {
        r = plan_;
        smemBytes = planSmem_;
        threads = planThreads_;
        return planState_ == 1;
    }
    planState_ = 2;
    int coop = 0, sms = 0;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device) != cudaSuccess || !coop ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    // Both brick shapes, each kept only if all its bricks fit on the GPU at once.
    struct Candidate {
        ResidentBrick r;
        size_t smem;
        int threads;
        long long bricks;
        bool fits;
    } cand[2];
    const int shapes[2][3] = {{32, 16, 16}, {16, 16, 16}};
    for (int c = 0; c < 2; ++c) {
        ResidentBrick b{};
        b.bx = shapes[c][0];
        b.by = shapes[c][1];
        b.bz = shapes[c][2];
        b.nbx = (nx + b.bx - 1) / b.bx;
        b.nby = (ny + b.by - 1) / b.by;
        b.nbz = (nz + b.bz - 1) / b.bz;
        cand[c] = Candidate{b, sorResidentSharedBytes(b.bx), (b.bx / 2) * b.by, static_cast<long long>(b.nbx) * b.nby * b.nbz, false};
        const void* fn = sorResidentKernel(b.bx);
        int perSm = 0;
        if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(cand[c].smem)) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, fn, cand[c].threads, cand[c].smem) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        cand[c].fits = cand[c].bricks <= static_cast<long long>(perSm) * sms;
    }
    // The larger bricks when they give every SM at least one; the smaller ones
    // when the larger would leave SMs idle (small grids) or do not fit.  When
    // both fit and the autotuner is on, the first solve times both
    // (tuneResident), unless this grid was timed before in this process.
    int pick = -1;
    if (cand[0].fits && cand[0].bricks >= sms) {
        pick = 0;
    } else if (cand[1].fits) {
        pick = 1;
    } else if (cand[0].fits) {
        pick = 0;
    }
    if (pick < 0) return false;
    tuneCount_ = 0;
    if (cand[0].fits && cand[1].fits && autotuneEnabled()) {
        const int known = tunedBrick(device, nx, ny, nz);
        if (known >= 0) {
            pick = known;
        } else {
            for (int c = 0; c < 2; ++c) {
                tuneBricks_[c] = cand[c].r;
                tuneSmem_[c] = cand[c].smem;
                tuneThreads_[c] = cand[c].threads;
            }
            tuneCount_ = 2;
        }
    }
    plan_ = cand[pick].r;
    planSmem_ = cand[pick].smem;
    planThreads_ = cand[pick].threads;
    planState_ = 1;
    r = plan_;
    smemBytes = planSmem_;
    threads = planThreads_;
    return true;
}

// Autotuner of the resident solve's brick shape.  Both shapes give the same
// bits, so the choice is speed only: one ungated solve of the configured
// iterations with each, from the same pressure (saved in divergenceAfter_, a
// scratch field until the metrics recompute it, and put back before the real
// solve), timed with CUDA events on the scene's stream.  The faster is kept
// for this grid for the life of the process (tunedBrick).  While the stream
// is being captured into a graph the heuristic's choice stands.
bool Scene::tuneResident(std::string& err) {
    const int count = tuneCount_;
    tuneCount_ = 0;
    if (sorSilentBrick_ >= 0) return true;  // an injected fault: keep the heuristic's choice
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &capture) != cudaSuccess || capture != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return true;
    }
    const size_t bytes = cells_ * sizeof(float);
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    bool ok = true;
    for (int i = 0; i < 3 && ok; ++i) ok = check("autotune event", cudaEventCreate(&ev[i]), err);
    ok = ok && check("autotune save", cudaMemcpyAsync(divergenceAfter_, pressure_, bytes, cudaMemcpyDeviceToDevice, stream), err);
    Grid g{nx, ny, nz};
    float omega = pressureOmega;
    int iterations = pressureIterations;
    for (int c = 0; c < count && ok; ++c) {
        ResidentBrick r = tuneBricks_[c];
        const unsigned bricks = static_cast<unsigned>(r.nbx * r.nby * r.nbz);
        void* fn = const_cast<void*>(sorResidentKernel(r.bx));
        ResidentSync sync{sorExchange_, sorStatus_, sorHostStatus_, sorEpoch_, sorSilentBrick_, sorWaitNs_, nullptr};
        sorEpoch_ += 2u * static_cast<unsigned>(iterations);
        void* args[] = {&pressure_, &divergence_, &g, &r, &sync, &iterations, &omega};
        ok = check("autotune restore", cudaMemcpyAsync(pressure_, divergenceAfter_, bytes, cudaMemcpyDeviceToDevice, stream), err) &&
             check("autotune event", cudaEventRecord(ev[c], stream), err) &&
             check("autotune launch", cudaLaunchCooperativeKernel(fn, dim3(bricks), dim3(tuneThreads_[c]), args, tuneSmem_[c], stream), err);
        launches_ += 1;
    }
    ok = ok && check("autotune event", cudaEventRecord(ev[2], stream), err) &&
         check("autotune restore", cudaMemcpyAsync(pressure_, divergenceAfter_, bytes, cudaMemcpyDeviceToDevice, stream), err) &&
         check("autotune wait", cudaEventSynchronize(ev[2]), err);
    if (ok) ok = checkSolverStatus(err);
    float ms[2] = {0.0f, 0.0f};
    if (ok) {
        // Each solve is timed from its own start to the next one's start (the
        // restore copy between them is the same for both).
        ok = check("autotune time", cudaEventElapsedTime(&ms[0], ev[0], ev[1]), err) &&
             check("autotune time", cudaEventElapsedTime(&ms[1], ev[1], ev[2]), err);
    }
    for (cudaEvent_t e : ev) {
        if (e != nullptr) cudaEventDestroy(e);
    }
    if (!ok) return false;
    const int best = ms[1] < ms[0] ? 1 : 0;
    rememberTunedBrick(device, nx, ny, nz, best, ms[0], ms[1]);
    plan_ = tuneBricks_[best];
    planSmem_ = tuneSmem_[best];
    planThreads_ = tuneThreads_[best];
    return true;
}

bool Scene::residentBrick(int& bx, int& by, int& bz) const {
    if (planState_ != 1) return false;
    bx = plan_.bx;
    by = plan_.by;
    bz = plan_.bz;
    return true;
}

// src/fire_cuda.cu:3280-3284 -- 2N half sweeps.  When the grid fits, one
// cooperative launch keeps p and div in shared memory for all of them
// (sorResident); otherwise they run on colour-split copies of p and div, as
// one CUDA graph per solve.
bool Scene::runSor(const FrameParams& p, std::string& err) {
    (void)p;
    const bool dirichletTop = physics_.mode == 1 && physics_.pressureTop == 1;
    if (mgCycles_ > 0 || dirichletTop) {
        if (!dirichletTop) {
            err = "multigrid pressure solve needs the config physics with a Dirichlet top (FirePhysicsParams.pressureTop = 1)";
            return false;
        }
        if (mgCycles_ == 0) {
            err = "a Dirichlet top needs the multigrid pressure solve (fireCudaSetPressureMultigrid)";
            return false;
        }
        return runMultigrid(err);
    }
    if (pressureIterations == 0) return true;
    if (pressurePath_ != 1) {
        ResidentBrick r;
        size_t smem = 0;
        int threads = 0;
        if (residentPlan(r, smem, threads)) {
            if (tuneCount_ > 1) {
                if (!tuneResident(err)) return false;
                residentPlan(r, smem, threads);
            }
            Grid g{nx, ny, nz};
            float omega = pressureOmega;
            const unsigned bricks = static_cast<unsigned>(r.nbx * r.nby * r.nbz);
            void* fn = const_cast<void*>(sorResidentKernel(r.bx));
            const bool gated = pressureTolerance_ > 0.0;
            const int chunk = gated ? std::max(1, std::min(pressureCheckEvery_, pressureIterations)) : pressureIterations;
            if (gated && !check("clear SOR gate", cudaMemsetAsync(sorGate_, 0, sizeof(SorGate), stream), err)) return false;
            for (int done = 0; done < pressureIterations; done += chunk) {
                int iterations = std::min(chunk, pressureIterations - done);
                ResidentSync sync{sorExchange_, sorStatus_, sorHostStatus_, sorEpoch_, sorSilentBrick_, sorWaitNs_,
                                  gated ? &sorGate_->converged : nullptr};
                sorEpoch_ += 2u * static_cast<unsigned>(iterations);
                void* args[] = {&pressure_, &divergence_, &g, &r, &sync, &iterations, &omega};
                if (!check("SOR cooperative launch", cudaLaunchCooperativeKernel(fn, dim3(bricks), dim3(threads), args, smem, stream), err)) {
                    return false;
                }
                ++launches_;
                if (gated) {
                    sorResidualPartials<<<kResidualBlocks, kResidualThreads, 0, stream>>>(pressure_, divergence_, g, sorGate_, residualSq_,
                                                                                        residualMax_);
                    sorResidualFinal<<<1, 32, 0, stream>>>(sorGate_, residualSq_, residualMax_, kResidualBlocks,
                                                           static_cast<float>(pressureTolerance_), iterations);
                    launches_ += 2;
                    if (!check("SOR residual launch", cudaGetLastError(), err)) return false;
                }
            }
            lastSolveGated_ = gated;
            lastPressurePath_ = 2;
            return true;
        }
        if (pressurePath_ == 2) {
            err = "resident SOR: the grid does not fit co-resident on this device";
            return false;
        }
    }
    // Grids too large for the resident solve: colour-split arrays and 2N
    // launches (in gated chunks when a tolerance is set), captured once per
    // (N, omega, tolerance, chunk) into a CUDA graph, so a step pays one launch.
    const SplitGrid sg = splitGridOf(nx, ny, nz);
    if (split_ == nullptr) {
        const size_t slots = 2ull * sg.nz * sg.ny * sg.P;
        if (!alloc(reinterpret_cast<void**>(&split_), slots * sizeof(float), "cudaMalloc SOR split pressure", err) ||
            !alloc(reinterpret_cast<void**>(&splitDiv_), slots * sizeof(float), "cudaMalloc SOR split divergence", err) ||
            !check("clear SOR split pressure", cudaMemsetAsync(split_, 0, slots * sizeof(float), stream), err) ||
            !check("clear SOR split divergence", cudaMemsetAsync(splitDiv_, 0, slots * sizeof(float), stream), err)) {
            return false;
        }
    }
    const bool gated = pressureTolerance_ > 0.0;
    const int chunk = gated ? std::max(1, std::min(pressureCheckEvery_, pressureIterations)) : pressureIterations;
    const double tolKey = gated ? pressureTolerance_ : 0.0;
    if (sorExec_ == nullptr || sorIterations_ != pressureIterations || sorOmega_ != pressureOmega || sorTolKey_ != tolKey ||
        sorChunkKey_ != chunk) {
        if (sorExec_ != nullptr) {
            cudaGraphExecDestroy(sorExec_);
            sorExec_ = nullptr;
        }
        const int bx = rowThreads(sg.H);
        const dim3 both((sg.H + bx - 1) / bx, ny, 2 * nz);
        const dim3 sweepBlock(32, kSplitRows);
        const dim3 sweep((sg.H + 127) / 128, (ny + kSplitRows - 1) / kSplitRows, nz);
        const int* skip = gated ? &sorGate_->converged : nullptr;
        const size_t colour = static_cast<size_t>(sg.nz) * sg.ny * sg.P;
        cudaGraph_t graph = nullptr;
        int count = 2;
        if (!check("SOR capture begin", cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), err)) return false;
        if (gated) cudaMemsetAsync(sorGate_, 0, sizeof(SorGate), stream);
        sorSplitPack<<<both, bx, 0, stream>>>(split_, splitDiv_, pressure_, divergence_, sg);
        for (int done = 0; done < pressureIterations; done += chunk) {
            const int iterations = std::min(chunk, pressureIterations - done);
            for (int i = 0; i < iterations; ++i) {
                sorSplitHalfSweep<<<sweep, sweepBlock, 0, stream>>>(split_, split_ + colour, splitDiv_, sg, 0, pressureOmega, skip);
                sorSplitHalfSweep<<<sweep, sweepBlock, 0, stream>>>(split_ + colour, split_, splitDiv_ + colour, sg, 1, pressureOmega,
                                                                    skip);
                count += 2;
            }
            if (gated) {
                sorSplitResidualPartials<<<kResidualBlocks, kResidualThreads, 0, stream>>>(split_, splitDiv_, sg, sorGate_, residualSq_,
                                                                                         residualMax_);
                sorResidualFinal<<<1, 32, 0, stream>>>(sorGate_, residualSq_, residualMax_, kResidualBlocks,
                                                       static_cast<float>(pressureTolerance_), iterations);
                count += 2;
            }
        }
        sorSplitUnpack<<<both, bx, 0, stream>>>(pressure_, split_, sg);
        const cudaError_t launchErr = cudaGetLastError();
        const cudaError_t endErr = cudaStreamEndCapture(stream, &graph);
        if (!check("SOR capture launch", launchErr, err) || !check("SOR capture end", endErr, err)) {
            if (graph) cudaGraphDestroy(graph);
            return false;
        }
        const cudaError_t instErr = cudaGraphInstantiate(&sorExec_, graph, 0);
        cudaGraphDestroy(graph);
        if (!check("SOR graph instantiate", instErr, err)) return false;
        sorIterations_ = pressureIterations;
        sorOmega_ = pressureOmega;
        sorTolKey_ = tolKey;
        sorChunkKey_ = chunk;
        sorGraphLaunches_ = count;
    }
    launches_ += static_cast<unsigned long long>(sorGraphLaunches_);
    lastSolveGated_ = gated;
    lastPressurePath_ = 1;
    return check("SOR graph launch", cudaGraphLaunch(sorExec_, stream), err);
}

bool Scene::setPressureMultigrid(int maxCycles, int preSmooth, int postSmooth, std::string& err) {
    if (maxCycles < 0 || maxCycles > 1000 || preSmooth < 1 || preSmooth > 8 || postSmooth < 1 || postSmooth > 8) {
        err = "multigrid: maxCycles must be in 0..1000 and the smoothing sweeps in 1..8";
        return false;
    }
    mgCycles_ = maxCycles;
    mgPre_ = preSmooth;
    mgPost_ = postSmooth;
    return true;
}

// ---------------------------------------------------------------------------
// MgSolver: the host side of mgSolve.

MgSolver::~MgSolver() { release(); }

void MgSolver::release() {
    for (cudaEvent_t e : uploadedRing_) {
        if (e != nullptr) cudaEventSynchronize(e);
    }
    deviceFree(dScenes_);
    deviceFree(dPlan_);
    deviceFree(dSync_);
    for (int k = 0; k < kStaging; ++k) {
        if (hScenesRing_[k] != nullptr) cudaFreeHost(hScenesRing_[k]);
        if (hPlanRing_[k] != nullptr) cudaFreeHost(hPlanRing_[k]);
        if (uploadedRing_[k] != nullptr) cudaEventDestroy(uploadedRing_[k]);
        hScenesRing_[k] = nullptr;
        hPlanRing_[k] = nullptr;
        uploadedRing_[k] = nullptr;
    }
    slot_ = 0;
    dScenes_ = nullptr;
    dPlan_ = nullptr;
    dSync_ = nullptr;
    planned_ = false;
    grid_ = 0;
    smem_ = 0;
}

// The work lists and descriptors are built on the host and uploaded on
// `stream` from pinned staging, so a plan (for example when a serving batch's
// scenes change) neither allocates nor synchronises after the first one; the
// staging is a ring, so a plan waits only for the upload made kStaging plans
// before it (the device copies are stream-ordered after the previous launch).
bool MgSolver::plan(int device, const std::vector<MgScene>& scenes, int maxCycles, int pre, int post, double tolerance,
                    cudaStream_t stream, std::string& err) {
    const int n = static_cast<int>(scenes.size());
    if (n < 1 || n > kMgMaxScenes) {
        err = "multigrid: a solve takes 1 to " + std::to_string(kMgMaxScenes) + " scenes";
        return false;
    }
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess && dScenes_ == nullptr) {
        int sms = 0, coop = 0;
        e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (e == cudaSuccess && !coop) {
            err = "multigrid: the device cannot run the persistent solve (no cooperative launch)";
            return false;
        }
        sms_ = sms;
        if (e == cudaSuccess) {
            e = cudaFuncSetAttribute(mgSolve, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kMgTailSmemMax));
        }
        if (e == cudaSuccess) e = deviceAlloc(reinterpret_cast<void**>(&dScenes_), kMgMaxScenes * sizeof(MgScene), "multigrid scene table");
        if (e == cudaSuccess) e = deviceAlloc(reinterpret_cast<void**>(&dPlan_), sizeof(MgPlan), "multigrid plan");
        if (e == cudaSuccess) e = deviceAlloc(reinterpret_cast<void**>(&dSync_), sizeof(MgSync), "multigrid sync");
        if (e == cudaSuccess) e = cudaMemset(dSync_, 0, sizeof(MgSync));
        for (int k = 0; k < kStaging; ++k) {
            if (e == cudaSuccess) {
                e = cudaHostAlloc(reinterpret_cast<void**>(&hScenesRing_[k]), kMgMaxScenes * sizeof(MgScene), cudaHostAllocDefault);
            }
            if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&hPlanRing_[k]), sizeof(MgPlan), cudaHostAllocDefault);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&uploadedRing_[k], cudaEventDisableTiming);
        }
        if (e != cudaSuccess) {
            err = std::string("multigrid plan: ") + cudaGetErrorString(e);
            release();
            return false;
        }
    }
    const int k = slot_;
    if (e == cudaSuccess) e = cudaEventSynchronize(uploadedRing_[k]);
    if (e != cudaSuccess) {
        err = std::string("multigrid plan: ") + cudaGetErrorString(e);
        return false;
    }
    MgScene* hScenes = hScenesRing_[k];
    MgPlan* hPlan = hPlanRing_[k];
    MgPlan& plan = *hPlan;
    std::memset(&plan, 0, sizeof(MgPlan));
    plan.scenes = n;
    plan.maxCycles = maxCycles;
    plan.pre = pre;
    plan.post = post;
    plan.gated = tolerance > 0.0 ? 1 : 0;
    plan.tolerance = static_cast<float>(tolerance);
    size_t smem = 0;
    for (int s = 0; s < n; ++s) {
        const MgScene& S = scenes[s];
        plan.gridLevels = std::max(plan.gridLevels, S.tail);
        size_t tailFloats = 0;
        for (int l = S.tail; l < S.levels; ++l) tailFloats += 2 * static_cast<size_t>(S.lv[l].nx) * S.lv[l].ny * S.lv[l].nz;
        if (S.tailMode == kMgTailShared) smem = std::max(smem, tailFloats * sizeof(float));
        if (S.tailMode == kMgTailRhsGlobal) {
            smem = std::max(smem, (tailFloats - static_cast<size_t>(S.lv[S.tail].nx) * S.lv[S.tail].ny * S.lv[S.tail].nz) * sizeof(float));
        }
    }
    for (int s = 0; s < n; ++s) {
        const int rows0 = scenes[s].lv[0].ny * scenes[s].lv[0].nz;
        plan.chunks[s + 1] = plan.chunks[s] + mgResidualChunks(scenes[s].lv[0].nx, scenes[s].lv[0].ny, scenes[s].lv[0].nz);
        const MgLevel& L0 = scenes[s].lv[0];
        plan.allUnits[s + 1] = plan.allUnits[s] + ((L0.nx & 3) == 0 ? mgQuadUnits(L0.nx, L0.ny, L0.nz) : rows0 * mgQuadChunks(L0.nx));
    }
    std::memcpy(hScenes, scenes.data(), n * sizeof(MgScene));
    int perSm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, mgSolve, kMgThreads, smem);
    if (e == cudaSuccess && perSm < 1) {
        err = "multigrid: no CTA of the persistent solve fits an SM";
        return false;
    }
    for (int l = 0; l < kMgMaxLevels; ++l) {
        for (int s = 0; s < n; ++s) {
            const MgScene& S = scenes[s];
            const bool grid = l < S.tail;
            const MgLevel& F = S.lv[l];
            const bool quad = (F.nx & 3) == 0;
            const int units = quad ? mgQuadUnits(F.nx, F.ny, F.nz) : F.ny * F.nz * mgQuadChunks(F.nx);
            plan.smoothUnits[l][s + 1] = plan.smoothUnits[l][s] + (grid ? units : 0);
            const int fine = quad ? mgQuadUnits(F.nx, F.ny, F.nz) : F.ny * F.nz * mgRowChunks(F.nx);
            plan.fineUnits[l][s + 1] = plan.fineUnits[l][s] + (grid ? fine : 0);
            if (grid) {
                const MgLevel& C = S.lv[l + 1];
                const int coarse = quad ? (C.nx * C.ny * C.nz + 63) / 64 : C.ny * C.nz * mgRowChunks(C.nx);
                plan.coarseUnits[l][s + 1] = plan.coarseUnits[l][s] + coarse;
            } else {
                plan.coarseUnits[l][s + 1] = plan.coarseUnits[l][s];
            }
        }
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(dScenes_, hScenes, n * sizeof(MgScene), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dPlan_, hPlan, sizeof(MgPlan), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaEventRecord(uploadedRing_[k], stream);
    if (e == cudaSuccess) slot_ = (k + 1) % kStaging;
    if (e != cudaSuccess) {
        err = std::string("multigrid plan: ") + cudaGetErrorString(e);
        return false;
    }
    grid_ = perSm * sms_;
    smem_ = smem;
    planned_ = true;
    return true;
}

bool MgSolver::launch(cudaStream_t stream, unsigned* hostStatus, std::string& err) {
    if (!planned()) {
        err = "multigrid: solve launched before it was planned";
        return false;
    }
    cudaError_t e = cudaMemsetAsync(dSync_, 0, sizeof(MgSync), stream);
    if (e == cudaSuccess) {
        void* args[] = {&dScenes_, &dPlan_, &dSync_, &hostStatus, &waitNs_};
        e = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(mgSolve), dim3(grid_), dim3(kMgThreads), args, smem_, stream);
    }
    if (e != cudaSuccess) {
        err = std::string("multigrid launch: ") + cudaGetErrorString(e);
        return false;
    }
    return true;
}

// The levels and buffers of this scene's multigrid (allocated once) and its
// descriptor: level 0 is the grid with weights (1, 1, 1); each next level
// halves every axis whose extent is even and at least 4; the shared-memory
// tail starts at the first level of at most kMgTailCells cells.
bool Scene::multigridScene(MgScene& out, std::string& err) {
    if (mgLevels_.empty()) {
        auto withWeights = [](MgLevel L) {
            L.diag = 2.0f * (L.wx + L.wy + L.wz);
            L.invDiag = 1.0f / L.diag;
            return L;
        };
        MgLevel L = withWeights(MgLevel{nx, ny, nz, 1.0f, 1.0f, 1.0f, 0.0f, 0.0f, 0, 0, 0});
        mgLevels_.push_back(L);
        while (static_cast<int>(mgLevels_.size()) < kMgMaxLevels) {
            const int cx = L.nx % 2 == 0 && L.nx >= 4, cy = L.ny % 2 == 0 && L.ny >= 4, cz = L.nz % 2 == 0 && L.nz >= 4;
            if (!cx && !cy && !cz) break;
            L = withWeights(MgLevel{cx ? L.nx / 2 : L.nx, cy ? L.ny / 2 : L.ny, cz ? L.nz / 2 : L.nz, cx ? L.wx * 0.25f : L.wx,
                                    cy ? L.wy * 0.25f : L.wy, cz ? L.wz * 0.25f : L.wz, 0.0f, 0.0f, cx, cy, cz});
            mgLevels_.push_back(L);
        }
        mgP_.assign(mgLevels_.size(), nullptr);
        mgRhs_.assign(mgLevels_.size(), nullptr);
        for (size_t l = 0; l < mgLevels_.size(); ++l) {
            const size_t n = static_cast<size_t>(mgLevels_[l].nx) * mgLevels_[l].ny * mgLevels_[l].nz;
            if (!alloc(reinterpret_cast<void**>(&mgP_[l]), n * sizeof(float), "cudaMalloc multigrid level", err) ||
                !check("clear multigrid level", cudaMemsetAsync(mgP_[l], 0, n * sizeof(float), stream), err)) {
                return false;
            }
            if (l > 0 && (!alloc(reinterpret_cast<void**>(&mgRhs_[l]), n * sizeof(float), "cudaMalloc multigrid level", err) ||
                          !check("clear multigrid level", cudaMemsetAsync(mgRhs_[l], 0, n * sizeof(float), stream), err))) {
                return false;
            }
        }
        const size_t chunks = static_cast<size_t>(mgResidualChunks(nx, ny, nz));
        if (!alloc(reinterpret_cast<void**>(&mgChunkSq_), chunks * sizeof(double), "cudaMalloc multigrid residual chunks", err)) {
            return false;
        }
    }
    MgScene S{};
    S.levels = static_cast<int>(mgLevels_.size());
    S.tail = S.levels - 1;
    for (int l = 0; l < S.levels; ++l) {
        S.lv[l] = mgLevels_[l];
        S.p[l] = mgP_[l];
        S.rhs[l] = l == 0 ? divergence_ : mgRhs_[l];
        if (S.tail == S.levels - 1 && static_cast<long long>(mgLevels_[l].nx) * mgLevels_[l].ny * mgLevels_[l].nz <= kMgTailCells) {
            S.tail = l;
        }
    }
    size_t tailBytes = 0;
    for (int l = S.tail; l < S.levels; ++l) tailBytes += 2 * sizeof(float) * mgLevels_[l].nx * mgLevels_[l].ny * mgLevels_[l].nz;
    const size_t tailRhs = sizeof(float) * mgLevels_[S.tail].nx * mgLevels_[S.tail].ny * mgLevels_[S.tail].nz;
    S.tailMode = tailBytes <= kMgTailSmemMax ? kMgTailShared : (tailBytes - tailRhs <= kMgTailSmemMax ? kMgTailRhsGlobal : kMgTailGlobal);
    S.pressure = pressure_;
    S.gate = sorGate_;
    S.chunkSq = mgChunkSq_;
    out = S;
    return true;
}

// The multigrid solve of this scene alone: one persistent launch (fire_mg.cu)
// for the increment, from zero; at its end pressure += increment.
bool Scene::runMultigrid(std::string& err) {
    const double tolKey = pressureTolerance_ > 0.0 ? pressureTolerance_ : 0.0;
    if (!mgSolver_.planned() || mgKeyCycles_ != mgCycles_ || mgKeyPre_ != mgPre_ || mgKeyPost_ != mgPost_ || mgKeyTol_ != tolKey) {
        MgScene S;
        if (!multigridScene(S, err)) return false;
        if (!mgSolver_.plan(device, std::vector<MgScene>{S}, mgCycles_, mgPre_, mgPost_, tolKey, stream, err)) return false;
        mgKeyCycles_ = mgCycles_;
        mgKeyPre_ = mgPre_;
        mgKeyPost_ = mgPost_;
        mgKeyTol_ = tolKey;
    }
    launches_ += 1;
    lastSolveGated_ = true;
    lastPressurePath_ = 3;
    mgDeltaValid_ = true;
    return mgSolver_.launch(stream, sorHostStatus_, err);
}

bool Scene::runMetrics(const FrameParams& p, std::string& err) {
    const int bx = rowThreads(nx);
    divergenceOf<<<cellGrid(bx, nx, ny, nz), bx, 0, stream>>>(divergenceAfter_, nullptr, velocity(), p);
    metricsPartials<<<kMetricBlocks, kMetricThreads, kMetricThreads * sizeof(MetricPartial), stream>>>(
        partials_, scalarsIn(), light_, shadow_, divergence_, divergenceAfter_, p);
    metricsFinal<<<1, kMetricThreads, kMetricThreads * sizeof(MetricPartial), stream>>>(metricDevice_, partials_, kMetricBlocks);
    launches_ += 3;
    if (!check("metrics launch", cudaGetLastError(), err)) return false;
    return check("metrics readback", cudaMemcpyAsync(metricHost_, metricDevice_, sizeof(MetricPartial), cudaMemcpyDeviceToHost, stream), err);
}

namespace {

// Lattice of one 2D fbm call site whose octave-0 inputs lie in
// [pxLo, pxHi] x [pyLo, pyHi]; later octaves map the range through the octave
// step (x * 2.03 + 17.7, y * 2.01 - 9.2, src/fire_cuda.cu:423-432), widened by
// one lattice cell per octave for rounding.  Entries past the edges are
// hashed in place by fbmLattice, so the margins only affect speed.
int planLattice(double pxLo, double pxHi, double pyLo, double pyHi, HashLattice2& L) {
    int offset = 0;
    for (int o = 0; o < kFbmOctaves; ++o) {
        L.ox[o] = static_cast<int>(std::floor(pxLo)) - 2;
        L.oy[o] = static_cast<int>(std::floor(pyLo)) - 2;
        L.sx[o] = static_cast<int>(std::floor(pxHi)) - L.ox[o] + 4;
        L.sy[o] = static_cast<int>(std::floor(pyHi)) - L.oy[o] + 4;
        L.offset[o] = offset;
        offset += L.sx[o] * L.sy[o];
        pxLo = pxLo * 2.03 + 17.7 - 1.0;
        pxHi = pxHi * 2.03 + 17.7 + 1.0;
        pyLo = pyLo * 2.01 - 9.2 - 1.0;
        pyHi = pyHi * 2.01 - 9.2 + 1.0;
    }
    return offset;
}

}  // namespace

// The curl noise of forceContributions hashes, per cell at (u, v, w) in [0, 1]^3,
//   A: (u * 9 + w * 3.7 + t * 0.22, v * 13 - t * 0.31)
//   B: (w * 10 - t * 0.19, u * 8 + v * 5.5 + t * 0.27)        (src/fire_cuda.cu:1164-1165)
bool Scene::curlLattices(const FrameParams& p, HashLattice2& a, HashLattice2& b) const {
    const double t = p.time;
    const int na = planLattice(t * 0.22 - 1.0, 12.7 + t * 0.22 + 1.0, -t * 0.31 - 1.0, 13.0 - t * 0.31 + 1.0, a);
    const int nb = planLattice(-t * 0.19 - 1.0, 10.0 - t * 0.19 + 1.0, t * 0.27 - 1.0, 13.5 + t * 0.27 + 1.0, b);
    const bool fits = latticesEnabled_ && curlLattice_ != nullptr && static_cast<size_t>(na) <= curlCapacity_[0] &&
                      static_cast<size_t>(nb) <= curlCapacity_[1];
    a.values = fits ? curlLattice_ : nullptr;
    b.values = fits ? curlLattice_ + curlCapacity_[0] : nullptr;
    return fits;
}

// The fuel-bed source noise of advectReact hashes, per cell at height v in [0, 1]
// and world position X in [-1.05, 1.05], Z in [-0.82, 0.82],
//   (X * 13 + Z * 3 + t * 0.38, v * 31 + Z * 11)               (src/fire_cuda.cu:1023)
bool Scene::sourceLattice(const FrameParams& p, HashLattice2& l) const {
    const double t = p.time;
    const int n = planLattice(-13.65 - 2.46 + t * 0.38 - 1.0, 13.65 + 2.46 + t * 0.38 + 1.0, -9.02 - 1.0, 31.0 + 9.02 + 1.0, l);
    const bool fits = latticesEnabled_ && sourceLattice_ != nullptr && static_cast<size_t>(n) <= sourceCapacity_;
    l.values = fits ? sourceLattice_ : nullptr;
    return fits;
}

bool Scene::runStages(int first, int last, const FrameParams& p, std::string& err) {
    if (first < 0 || last > kReset || first > last) {
        err = "stage range out of order";
        return false;
    }
    if (physics_.mode == 1) return runConfigStages(first, last, p, err);
    const int bx = rowThreads(nx);
    const dim3 cells = cellGrid(bx, nx, ny, nz);
    int s = first;
    while (s <= last) {
        switch (s) {
            case kAdvectVelocity:
                advectVelocity<<<cells, bx, 0, stream>>>(vel_[0][1 - vcur_], vel_[1][1 - vcur_], vel_[2][1 - vcur_], velocity(), p); ++launches_;
                vcur_ = 1 - vcur_;
                s = kAdvectReact;
                break;
            case kAdvectReact:
                if (!ensureMaterial(p, err)) return false;
            {
                HashLattice2 srcLattice{};
                if (sourceLattice(p, srcLattice)) {
                    hashLatticeBuild<<<dim3(256, 1), 256, 0, stream>>>(srcLattice, srcLattice); ++launches_;
                }
                advectReact<<<cells, bx, 0, stream>>>(scalarsOut(), scalarsIn(), velocity(), material_, breathing_, p, srcLattice); ++launches_;
            }
                cur_ = 1 - cur_;
                s = kForce;
                break;
            case kForce: {
                HashLattice2 curlA{}, curlB{};
                if (curlLattices(p, curlA, curlB)) {
                    hashLatticeBuild<<<dim3(64, 2), 256, 0, stream>>>(curlA, curlB); ++launches_;
                }
                forceContributions<<<cells, bx, 0, stream>>>(contrib_, scalarsIn(), velocity(), p, curlA, curlB); ++launches_;
                if (last >= kDivergence) {
                    forceProjectSetup<<<cells, bx, 0, stream>>>(vel_[0][1 - vcur_], vel_[1][1 - vcur_], vel_[2][1 - vcur_], divergence_,
                                                               pressure_, contrib_, velocity(), p); ++launches_;
                    vcur_ = 1 - vcur_;
                    s = kPressureSor;
                } else {
                    forceApply<<<cells, bx, 0, stream>>>(vel_[0][1 - vcur_], vel_[1][1 - vcur_], vel_[2][1 - vcur_], contrib_, velocity(), p); ++launches_;
                    vcur_ = 1 - vcur_;
                    s = kVelocityBoundary;
                }
                break;
            }
            case kVelocityBoundary:
                velocityBoundary<<<cells, bx, 0, stream>>>(vel_[0][vcur_], vel_[1][vcur_], vel_[2][vcur_], p, 1); ++launches_;
                s = kDivergence;
                break;
            case kDivergence:
                divergenceOf<<<cells, bx, 0, stream>>>(divergence_, pressure_, velocity(), p); ++launches_;
                s = kPressureSor;
                break;
            case kPressureSor:
                if (!runSor(p, err)) return false;
                s = kSubtract;
                break;
            case kSubtract:
                subtractWall<<<cells, bx, 0, stream>>>(vel_[0][vcur_], vel_[1][vcur_], vel_[2][vcur_], pressure_, p, 1, last >= kWallBoundary ? 1 : 0); ++launches_;
                s = last >= kWallBoundary ? kLightBuild : kWallBoundary;
                break;
            case kWallBoundary:
                subtractWall<<<cells, bx, 0, stream>>>(vel_[0][vcur_], vel_[1][vcur_], vel_[2][vcur_], pressure_, p, 0, 1); ++launches_;
                s = kLightBuild;
                break;
            case kLightBuild: {
                const int lbx = rowThreads(lnx);
                lightBuild<<<dim3((lnx + lbx - 1) / lbx, lny, lnz), lbx, 0, stream>>>(light_, shadow_, scalarsIn(), p); ++launches_;
                s = kLightPropagate;
                break;
            }
            case kLightPropagate: {
                const int lbx = rowThreads(lnx);
                const dim3 lg((lnx + lbx - 1) / lbx, lny, lnz);
                lightPropagate<<<lg, lbx, 0, stream>>>(lightNext_, light_, shadow_, p, 0.48f, 0.92f); ++launches_;
                lightPropagate<<<lg, lbx, 0, stream>>>(light_, lightNext_, shadow_, p, 0.34f, 0.96f); ++launches_;
                s = kRender;
                break;
            }
            case kRender:
            {
                if (!check("clear ray tile counter", cudaMemsetAsync(rayTileCounter_, 0, sizeof(int), stream), err)) return false;
                // Scenes 0-2 without a debug view take the instantiation with
                // the scene id fixed; the generic kernel draws the debug views.
                const int k = p.renderDebugMode == 0 && p.sceneId >= 0 && p.sceneId <= 2 ? 1 + p.sceneId : 0;
                const RayTiles tiles{rayTileCounter_, rayTileOrder_, rayTilesX_, rayTileCount_};
                auto kernel = k == 1 ? raymarchScene0 : (k == 2 ? raymarchScene1 : (k == 3 ? raymarchScene2 : raymarch));
                kernel<<<rayBlocks_[k], 128, 0, stream>>>(hdr_, scalarsIn(), velocity(), light_, shadow_, p, tiles); ++launches_;
            }
                s = kEmbers;
                break;
            case kEmbers:
                if (p.emberCount > 0 && p.renderDebugMode == 0) {
                    emberSetup<<<1, 256, 0, stream>>>(embers_, scalarsIn(), velocity(), p); ++launches_;
                    emberGather<<<dim3((frameW + 15) / 16, (frameH + 15) / 16), dim3(16, 16), 0, stream>>>(hdr_, embers_, p); ++launches_;
                }
                s = kTonemap;
                break;
            case kTonemap:
                tonemapOverlay<<<dim3((frameW + 15) / 16, (frameH + 15) / 16), dim3(16, 16), 0, stream>>>(bgra_, hdr_, p, 1,
                                                                                                      last >= kOverlay ? 1 : 0); ++launches_;
                s = last >= kOverlay ? kMetrics : kOverlay;
                break;
            case kOverlay:
                tonemapOverlay<<<dim3((frameW + 15) / 16, (frameH + 15) / 16), dim3(16, 16), 0, stream>>>(bgra_, hdr_, p, 0, 1); ++launches_;
                s = kMetrics;
                break;
            case kMetrics:
                if (!runMetrics(p, err)) return false;
                s = kReset;
                break;
            case kReset: {
                // src/fire_cuda.cu:3006-3048: procedural scalars, zero faces, zero light.
                if (!ensureMaterial(p, err)) return false;
                resetCells<<<cells, bx, 0, stream>>>(scalarsOut(), pressure_, divergence_, divergenceAfter_, material_, breathing_, p); ++launches_;
                cur_ = 1 - cur_;
                bool ok = true;
                for (int c = 0; c < 3 && ok; ++c) {
                    const size_t n = c == 0 ? nu_ : (c == 1 ? nv_ : nw_);
                    ok = check("reset velocity", cudaMemsetAsync(vel_[c][0], 0, n * sizeof(FaceT), stream), err) &&
                         check("reset velocity", cudaMemsetAsync(vel_[c][1], 0, n * sizeof(FaceT), stream), err);
                }
                ok = ok && check("reset scene light", cudaMemsetAsync(light_, 0, lightCells_ * sizeof(float4), stream), err) &&
                     check("reset scene light next", cudaMemsetAsync(lightNext_, 0, lightCells_ * sizeof(float4), stream), err) &&
                     check("reset scene shadow", cudaMemsetAsync(shadow_, 0, lightCells_ * sizeof(float), stream), err);
                if (!ok) return false;
                s = kReset + 1;
                break;
            }
            default:
                err = "unknown stage";
                return false;
        }
        if (!check("stage launch", cudaGetLastError(), err)) return false;
    }
    return true;
}

bool Scene::reset(std::string& err) {
    const FrameParams p = defaultParams(simTime);
    if (!runStages(kReset, kReset, p, err)) return false;
    simTime = 0.0f;
    renderTime = 0.0f;
    frameIndex = 0;
    return check("reset kernels sync", cudaStreamSynchronize(stream), err);
}

bool Scene::frame(uint32_t* hostBgra, const FireSettings& s, FireCudaFrameMetrics* metrics, bool toHdrSlot, bool advance, bool render,
                  std::string& err) {
    if (render && !toHdrSlot && hostBgra == nullptr) {
        err = "Output pixel pointer was null.";
        return false;
    }
    if (render && toHdrSlot && slots_[activeSlot_].ptr == nullptr) {
        err = "HDR output buffer slot is not registered.";
        return false;
    }
    if (!render && !advance) {
        err = "Step-only path requires simulation advancement.";
        return false;
    }
    const bool collect = metrics != nullptr;
    if (collect && !advance) {
        err = "Render-only measured path is not supported.";
        return false;
    }
    const float stepDt = std::max(0.001f, std::min(s.dt, 1.0f / 30.0f));
    renderTime += stepDt;
    if (advance) simTime += stepDt;
    FrameParams p = paramsFrom(s, advance ? simTime : renderTime);
    if (s.reset != 0) {
        // The reset zeroes the clocks, but the frame keeps the parameter block
        // built before it (src/fire_cuda.cu:3181, :3053-3055).
        if (!runStages(kReset, kReset, p, err)) return false;
        simTime = 0.0f;
        renderTime = 0.0f;
        frameIndex = 0;
    }
    auto rec = [&](int e) { return !collect || check("cudaEventRecord", cudaEventRecord(events_[e], stream), err); };
    if (!rec(kStart)) return false;
    if (advance) {
        // Event points of the reference (src/fire_cuda.cu:3188-3321).  The
        // forcing is fused with the divergence, so it is timed in the
        // projection interval rather than the reaction interval.
        if (!runStages(kAdvectVelocity, kAdvectVelocity, p, err) || !rec(kAfterVelocity)) return false;
        if (!runStages(kAdvectReact, kAdvectReact, p, err) || !rec(kAfterReaction)) return false;
        if (!runStages(kForce, kWallBoundary, p, err) || !rec(kAfterProjection) || !rec(kAfterSolve)) return false;
        // The config physics builds its light (the point light's transmittance)
        // only for a frame that is rendered.
        if ((physics_.mode != 1 && !runStages(kLightBuild, kLightPropagate, p, err)) || !rec(kAfterLighting)) return false;
    }
    if (!render) {
        return true;
    }
    p.time = renderTime;
    if (physics_.mode == 1 && !runStages(kLightBuild, kLightBuild, p, err)) return false;
    if (!runStages(kRender, kEmbers, p, err) || !rec(kAfterRaymarch)) return false;
    if (toHdrSlot) {
        const HdrSlot& slot = slots_[activeSlot_];
        packHdr<<<dim3((frameW + 15) / 16, (frameH + 15) / 16), dim3(16, 16), 0, stream>>>(slot.ptr, slot.pitchBytes, slot.format, hdr_, p); ++launches_;
        if (!check("HDR pack launch", cudaGetLastError(), err)) return false;
    } else if (!runStages(kTonemap, kOverlay, p, err)) {
        return false;
    }
    if (!rec(kAfterPack) || !rec(kAfterRender)) return false;
    if (!toHdrSlot) {
        if (!check("cudaMemcpy frame", cudaMemcpyAsync(hostBgra, bgra_, pixels_ * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream), err) ||
            !check("frame sync", cudaStreamSynchronize(stream), err) || !checkSolverStatus(err)) {
            return false;
        }
    }
    if (collect) {
        if (!runStages(kMetrics, kMetrics, p, err) || !check("metrics sync", cudaStreamSynchronize(stream), err) || !checkSolverStatus(err) ||
            !fillMetrics(metrics, err)) {
            return false;
        }
    }
    ++frameIndex;
    return true;
}

// src/fire_cuda.cu:3476-3545 -- event intervals and the accumulator into FireCudaFrameMetrics.
bool Scene::fillMetrics(FireCudaFrameMetrics* out, std::string& err) {
    float solveMs = 0, renderMs = 0, velocityMs = 0, reactionMs = 0, projectionMs = 0, lightingMs = 0, raymarchMs = 0, packMs = 0;
    if (!check("cudaEventElapsedTime solve", cudaEventElapsedTime(&solveMs, events_[kStart], events_[kAfterSolve]), err) ||
        !check("cudaEventElapsedTime render", cudaEventElapsedTime(&renderMs, events_[kAfterSolve], events_[kAfterRender]), err) ||
        !check("cudaEventElapsedTime velocity", cudaEventElapsedTime(&velocityMs, events_[kStart], events_[kAfterVelocity]), err) ||
        !check("cudaEventElapsedTime reaction", cudaEventElapsedTime(&reactionMs, events_[kAfterVelocity], events_[kAfterReaction]), err) ||
        !check("cudaEventElapsedTime projection", cudaEventElapsedTime(&projectionMs, events_[kAfterReaction], events_[kAfterProjection]), err) ||
        !check("cudaEventElapsedTime lighting", cudaEventElapsedTime(&lightingMs, events_[kAfterProjection], events_[kAfterLighting]), err) ||
        !check("cudaEventElapsedTime raymarch", cudaEventElapsedTime(&raymarchMs, events_[kAfterLighting], events_[kAfterRaymarch]), err) ||
        !check("cudaEventElapsedTime pack", cudaEventElapsedTime(&packMs, events_[kAfterRaymarch], events_[kAfterPack]), err)) {
        return false;
    }
    const MetricPartial& m = *metricHost_;
    const double cellCount = static_cast<double>(cells_);
    auto bits = [](int b) {
        float f;
        std::memcpy(&f, &b, 4);
        return f;
    };
    const float divBeforeL2 = static_cast<float>(std::sqrt(m.sums[19] / std::max(1.0, cellCount)));
    const float divAfterL2 = static_cast<float>(std::sqrt(m.sums[20] / std::max(1.0, cellCount)));
    FireCudaFrameMetrics o{};
    o.frameIndex = frameIndex;
    o.gridX = nx;
    o.gridY = ny;
    o.gridZ = nz;
    o.pressureIterations = pressureIterations;
    if (lastSolveGated_) {
        int it = 0;
        float mr = 0.0f;
        double l2 = 0.0;
        if (!pressureStats(it, mr, l2, err)) return false;
        o.pressureIterations = it;
    }
    o.invalidCells = m.invalidCells;
    o.timeSeconds = simTime;
    o.gpuSolveMs = solveMs;
    o.gpuRenderMs = renderMs;
    o.gpuVelocityMs = velocityMs;
    o.gpuReactionMs = reactionMs;
    o.gpuProjectionMs = projectionMs;
    o.gpuLightingMs = lightingMs;
    o.gpuRaymarchMs = raymarchMs;
    o.gpuPackMs = packMs;
    o.heatSum = static_cast<float>(m.sums[0]);
    o.fuelSum = static_cast<float>(m.sums[1]);
    o.oxygenSum = static_cast<float>(m.sums[2]);
    o.sootSum = static_cast<float>(m.sums[3]);
    o.charSum = static_cast<float>(m.sums[4]);
    o.ashSum = static_cast<float>(m.sums[5]);
    o.pyrolysisSum = static_cast<float>(m.sums[6]);
    o.progressSum = static_cast<float>(m.sums[7]);
    o.turbulenceEnergySum = static_cast<float>(m.sums[8]);
    o.sootOpticalDepthSum = static_cast<float>(m.sums[9]);
    o.maxHeat = bits(m.maxBits[0]);
    o.maxFuel = bits(m.maxBits[1]);
    o.maxSoot = bits(m.maxBits[2]);
    o.maxPyrolysis = bits(m.maxBits[3]);
    o.maxProgress = bits(m.maxBits[4]);
    o.maxTurbulenceEnergy = bits(m.maxBits[5]);
    o.flameHeightMeters = bits(m.maxBits[6]);
    o.meanOpticalDepth = static_cast<float>(m.sums[17] / std::max(1.0, cellCount));
    o.meanSceneLight = static_cast<float>(m.sums[10] / std::max(1.0, cellCount));
    o.meanSceneShadow = static_cast<float>(m.sums[11] / std::max(1.0, cellCount));
    o.flameMassProxy = static_cast<float>(m.sums[12]);
    o.smokeMassProxy = static_cast<float>(m.sums[13]);
    o.flameSmokeOverlapProxy = static_cast<float>(m.sums[14]);
    o.meanVolumetricShadow = static_cast<float>(m.sums[15] / std::max(1.0, cellCount));
    o.meanRoomIrradiance = static_cast<float>(m.sums[16] / std::max(1.0, cellCount));
    o.heatReleaseProxy = static_cast<float>(m.sums[18]);
    o.divergenceBeforeL2 = divBeforeL2;
    o.divergenceBeforeMax = bits(m.maxBits[7]);
    o.divergenceAfterL2 = divAfterL2;
    o.divergenceAfterMax = bits(m.maxBits[8]);
    o.divergenceReduction = divBeforeL2 > 0.000001f ? 1.0f - divAfterL2 / divBeforeL2 : 0.0f;
    *out = o;
    return true;
}

// ---------------------------------------------------------------------------
// Field access (tests, checkpoints): one field at a time, converting between
// the packed records and the reference's one-array-per-field layout.
namespace {

struct FieldView {
    void* base;
    size_t count;    // elements of `stride` values
    int stride;      // values per element in device memory
    int component;   // value offset inside the element
    int width;       // floats per element in the host layout
    int valueBytes;  // bytes of one stored value: 4 (float), or 2 for the transported fields of the half build
};

}  // namespace

static bool fieldView(int field, Rec4* sa, Rec4* sb, Rec2* sc, FaceT* const vel[3], float* pressure, float* divergence,
                      float* divergenceAfter, float4* light, float* shadow, float4* hdr, uint32_t* bgra, size_t cells, size_t nu,
                      size_t nv, size_t nw, size_t lightCells, size_t pixels, FieldView& v) {
    const int t = static_cast<int>(sizeof(FaceT));
    switch (field) {
        case 0: case 1: case 2: case 3: v = {sa, cells, 4, field, 1, t}; return true;
        case 4: case 5: case 6: case 7: v = {sb, cells, 4, field - 4, 1, t}; return true;
        case 8: case 9: v = {sc, cells, 2, field - 8, 1, t}; return true;
        case 10: v = {pressure, cells, 1, 0, 1, 4}; return true;
        case 11: v = {divergence, cells, 1, 0, 1, 4}; return true;
        case 12: v = {vel[0], nu, 1, 0, 1, t}; return true;
        case 13: v = {vel[1], nv, 1, 0, 1, t}; return true;
        case 14: v = {vel[2], nw, 1, 0, 1, t}; return true;
        case 15: v = {light, lightCells, 4, 0, 4, 4}; return true;
        case 16: v = {shadow, lightCells, 1, 0, 1, 4}; return true;
        case 17: v = {hdr, pixels, 4, 0, 4, 4}; return true;
        case 18: v = {bgra, pixels, 1, 0, 1, 4}; return true;
        case 19: v = {divergenceAfter, cells, 1, 0, 1, 4}; return true;
        default: return false;
    }
}

namespace {

float storedToFloat(const unsigned char* p, int bytes) {
    if (bytes == 4) {
        float f;
        std::memcpy(&f, p, 4);
        return f;
    }
#if defined(FIRE_HALF_STORAGE)
    Half1 h;
    std::memcpy(&h, p, 2);
    return static_cast<float>(h);
#else
    return 0.0f;
#endif
}

void floatToStored(float f, unsigned char* p, int bytes) {
    if (bytes == 4) {
        std::memcpy(p, &f, 4);
        return;
    }
#if defined(FIRE_HALF_STORAGE)
    const Half1 h(f);  // round to nearest
    std::memcpy(p, &h, 2);
#endif
}

}  // namespace

bool Scene::getField(int field, void* host, size_t bytes, std::string& err) {
    FaceT* velNow[3] = {vel_[0][vcur_], vel_[1][vcur_], vel_[2][vcur_]};
    FieldView v;
    if (field == FIRE_FIELD_CONFIG_TRANSMITTANCE) {
        if (!ensureConfigBuffers(err)) return false;
        v = {cfgLight_, static_cast<size_t>(cfgLx_) * cfgLy_ * cfgLz_, 1, 0, 1, 4};
    } else if (!fieldView(field, sa_[cur_], sb_[cur_], sc_[cur_], velNow, pressure_, divergence_, divergenceAfter_, light_, shadow_, hdr_,
                          bgra_, cells_, nu_, nv_, nw_, lightCells_, pixels_, v)) {
        err = "unknown field id";
        return false;
    }
    if (bytes != v.count * v.width * 4) {
        err = "field size mismatch";
        return false;
    }
    if (!check("field sync", cudaStreamSynchronize(stream), err)) return false;
    if (v.width == v.stride && v.valueBytes == 4) {
        return check("cudaMemcpy field", cudaMemcpy(host, v.base, bytes, cudaMemcpyDeviceToHost), err);
    }
    std::vector<unsigned char> staging(v.count * v.stride * v.valueBytes);
    if (!check("cudaMemcpy field", cudaMemcpy(staging.data(), v.base, staging.size(), cudaMemcpyDeviceToHost), err)) return false;
    float* out = static_cast<float*>(host);
    for (size_t i = 0; i < v.count; ++i) {
        for (int w = 0; w < v.width; ++w) {
            out[i * v.width + w] = storedToFloat(staging.data() + (i * v.stride + v.component + w) * v.valueBytes, v.valueBytes);
        }
    }
    return true;
}

bool Scene::setField(int field, const void* host, size_t bytes, std::string& err) {
    if (field == FIRE_FIELD_PRESSURE) mgDeltaValid_ = false;  // the field, not an older solve, is the pressure now
    FaceT* velNow[3] = {vel_[0][vcur_], vel_[1][vcur_], vel_[2][vcur_]};
    FieldView v;
    if (field == FIRE_FIELD_CONFIG_TRANSMITTANCE) {
        if (!ensureConfigBuffers(err)) return false;
        v = {cfgLight_, static_cast<size_t>(cfgLx_) * cfgLy_ * cfgLz_, 1, 0, 1, 4};
    } else if (!fieldView(field, sa_[cur_], sb_[cur_], sc_[cur_], velNow, pressure_, divergence_, divergenceAfter_, light_, shadow_, hdr_,
                          bgra_, cells_, nu_, nv_, nw_, lightCells_, pixels_, v)) {
        err = "unknown field id";
        return false;
    }
    if (bytes != v.count * v.width * 4) {
        err = "field size mismatch";
        return false;
    }
    if (!check("field sync", cudaStreamSynchronize(stream), err)) return false;
    if (v.width == v.stride && v.valueBytes == 4) {
        return check("cudaMemcpy field", cudaMemcpy(v.base, host, bytes, cudaMemcpyHostToDevice), err);
    }
    std::vector<unsigned char> staging(v.count * v.stride * v.valueBytes);
    if (!check("cudaMemcpy field", cudaMemcpy(staging.data(), v.base, staging.size(), cudaMemcpyDeviceToHost), err)) return false;
    const float* in = static_cast<const float*>(host);
    for (size_t i = 0; i < v.count; ++i) {
        for (int w = 0; w < v.width; ++w) {
            floatToStored(in[i * v.width + w], staging.data() + (i * v.stride + v.component + w) * v.valueBytes, v.valueBytes);
        }
    }
    return check("cudaMemcpy field", cudaMemcpy(v.base, staging.data(), staging.size(), cudaMemcpyHostToDevice), err);
}

bool Scene::registerHdrSlot(int slot, void* ptr, size_t pitch, int format, std::string& err) {
    if (slot < 0 || slot >= 4) {
        err = "HDR buffer slot is outside the supported slot range.";
        return false;
    }
    if (ptr == nullptr) {
        err = "HDR buffer pointer was null.";
        return false;
    }
    const size_t rowBytes = static_cast<size_t>(frameW) * (format == 1 ? 8 : 16);
    if ((format != 0 && format != 1) || pitch < rowBytes || (reinterpret_cast<uintptr_t>(ptr) & 15) != 0 || (pitch & 15) != 0) {
        err = "HDR buffer: format must be 0 or 1, pitch >= width*pixel bytes, pointer and pitch 16-byte aligned";
        return false;
    }
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, ptr) != cudaSuccess || attr.type != cudaMemoryTypeDevice || attr.device != device) {
        cudaGetLastError();
        err = "HDR buffer must be device memory of the scene's GPU";
        return false;
    }
    slots_[slot] = HdrSlot{ptr, pitch, format};
    return true;
}

bool Scene::setActiveSlot(int slot, std::string& err) {
    if (slot < 0 || slot >= 4 || slots_[slot].ptr == nullptr) {
        char buf[96];
        std::snprintf(buf, sizeof(buf), "HDR buffer slot %d is not registered.", slot);
        err = buf;
        return false;
    }
    activeSlot_ = slot;
    return true;
}

void Scene::clearSlots() {
    for (HdrSlot& s : slots_) s = HdrSlot{};
    activeSlot_ = 0;
}

bool Scene::synchronize(std::string& err) {
    return check("cudaStreamSynchronize", cudaStreamSynchronize(stream), err) && checkSolverStatus(err);
}

// A resident SOR wait that ran out leaves brick + 1 in the host-mapped status
// word; the pressure of that solve is incomplete.  Read after a stream sync.
bool Scene::checkSolverStatus(std::string& err) {
    if (sorHostStatus_ == nullptr) return true;
    const unsigned st = *reinterpret_cast<volatile unsigned*>(sorHostStatus_);
    if (st == 0) return true;
    *sorHostStatus_ = 0;
    if (st & kMgStatusFlag) {
        err = "multigrid solve: a grid barrier wait timed out in phase " + std::to_string(st & ~kMgStatusFlag);
    } else {
        err = "resident SOR: brick " + std::to_string(st - 1) + " timed out waiting for a neighbour's half sweep";
    }
    return false;
}

bool Scene::setPressureTolerance(double tolerance, int checkEvery, std::string& err) {
    if (!(tolerance >= 0.0) || checkEvery < 1) {
        err = "pressure tolerance must be >= 0 and the check interval >= 1";
        return false;
    }
    pressureTolerance_ = tolerance;
    pressureCheckEvery_ = checkEvery;
    return true;
}

bool Scene::pressureStats(int& iterations, float& maxResidual, double& l2Residual, std::string& err) {
    if (!lastSolveGated_) {
        iterations = pressureIterations;
        maxResidual = -1.0f;
        l2Residual = -1.0;
        return true;
    }
    SorGate gate{};
    if (!check("pressure stats sync", cudaStreamSynchronize(stream), err) ||
        !check("pressure stats copy", cudaMemcpy(&gate, sorGate_, sizeof(gate), cudaMemcpyDeviceToHost), err)) {
        return false;
    }
    iterations = gate.iterations;
    maxResidual = gate.maxResidual;
    l2Residual = gate.l2Residual;
    return true;
}

bool Scene::setResidentFault(int silentBrick, long long waitUs, std::string& err) {
    if (waitUs <= 0 || waitUs > 10000000) {
        err = "resident SOR wait limit must be in (0, 10 s]";
        return false;
    }
    sorSilentBrick_ = silentBrick < 0 ? -1 : silentBrick;
    sorWaitNs_ = static_cast<unsigned long long>(waitUs) * 1000ull;
    return true;
}

// ---------------------------------------------------------------------------
// Config physics (FirePhysicsParams.mode 1): parameters, buffers and stages.

void defaultPhysicsParams(FirePhysicsParams& q, int nx, int ny, int nz) {
    std::memset(&q, 0, sizeof(q));
    q.mode = 0;
    q.dt = 1.0f / 60.0f;
    q.buoyancyHeat = 1.62f;   // src/fire_cuda.cu:1176
    q.buoyancySoot = 0.095f;  // src/fire_cuda.cu:1176
    q.ambientHeat = 0.0f;
    q.burnRate = 0.5f;
    q.ignitionHeat = 0.05f;
    q.heatRelease = 1.0f;
    q.sootYield = 0.3f;
    q.cooling = 0.35f;
    q.sootDecay = 0.05f;
    q.vorticityEps = 0.0f;
    q.noisePeriod = 16.0f;
    q.noiseSeed = 7u;
    q.primarySamples = 96;
    q.lightSamples = 32;
    q.lightX = 0.5f * static_cast<float>(nx);
    q.lightY = 1.4f * static_cast<float>(ny);
    q.lightZ = 0.5f * static_cast<float>(nz);
    q.lightIntensity = 1.0f;
    q.extinction = 0.9f;
    q.fuelExtinction = 0.05f;
    q.emission = 0.6f;
    q.albedo = 0.7f;
    q.eyeX = 0.5f * static_cast<float>(nx);
    q.eyeY = 0.5f * static_cast<float>(ny);
    q.eyeZ = -1.3f * static_cast<float>(std::max(nx, std::max(ny, nz)));
    q.targetX = 0.5f * static_cast<float>(nx);
    q.targetY = 0.5f * static_cast<float>(ny);
    q.targetZ = 0.5f * static_cast<float>(nz);
    q.fovYDegrees = 45.0f;
}

bool validatePhysicsParams(const FirePhysicsParams& q, std::string& err) {
    if (q.mode != 0 && q.mode != 1) {
        err = "physics mode must be 0 (reference) or 1 (config)";
        return false;
    }
    if (q.pressureTop != 0 && q.pressureTop != 1) {
        err = "physics parameters: pressureTop must be 0 (Neumann) or 1 (Dirichlet)";
        return false;
    }
    const float vals[] = {q.dt, q.buoyancyHeat, q.buoyancySoot, q.ambientHeat, q.burnRate, q.ignitionHeat, q.heatRelease, q.sootYield,
                          q.cooling, q.sootDecay, q.vorticityEps, q.windX, q.windZ, q.noiseAmplitude, q.noisePeriod, q.lightX,
                          q.lightY, q.lightZ, q.lightIntensity, q.extinction, q.fuelExtinction, q.emission, q.albedo, q.eyeX,
                          q.eyeY, q.eyeZ, q.targetX, q.targetY, q.targetZ, q.fovYDegrees};
    for (float v : vals) {
        if (!std::isfinite(v)) {
            err = "physics parameters must be finite";
            return false;
        }
    }
    if (!(q.dt > 0.0f) || !(q.noisePeriod > 0.0f) || q.burnRate < 0.0f || q.cooling < 0.0f || q.sootDecay < 0.0f) {
        err = "physics parameters: dt and noisePeriod must be > 0, rates >= 0";
        return false;
    }
    if (q.primarySamples < 1 || q.primarySamples > 4096 || q.lightSamples < 1 || q.lightSamples > 4096) {
        err = "physics parameters: sample counts must be in 1..4096";
        return false;
    }
    if (!(q.fovYDegrees > 0.0f && q.fovYDegrees < 179.0f)) {
        err = "physics parameters: fovYDegrees must be in (0, 179)";
        return false;
    }
    if (q.emitterCount < 0 || q.emitterCount > FIRE_MAX_EMITTERS) {
        err = "physics parameters: emitterCount must be in 0..4";
        return false;
    }
    for (int e = 0; e < q.emitterCount; ++e) {
        const FireEmitterDisk& d = q.emitters[e];
        const float ev[] = {d.centerX, d.centerY, d.centerZ, d.radius, d.fuel, d.heat, d.upVelocity, d.jitterScale};
        for (float v : ev) {
            if (!std::isfinite(v)) {
                err = "emitter parameters must be finite";
                return false;
            }
        }
        if (d.radius < 0.0f || d.jitterScale < 0.0f || d.jitterScale > 1.0f || std::fabs(d.centerY) > 1.0e6f) {
            err = "emitter parameters: radius >= 0, jitterScale in [0, 1]";
            return false;
        }
    }
    const float fx = q.targetX - q.eyeX, fy = q.targetY - q.eyeY, fz = q.targetZ - q.eyeZ;
    if (!(fx * fx + fy * fy + fz * fz > 0.0f)) {
        err = "physics parameters: camera eye and target coincide";
        return false;
    }
    return true;
}

bool Scene::setPhysics(const FirePhysicsParams& params, std::string& err) {
    if (!validatePhysicsParams(params, err)) return false;
    physics_ = params;
    return true;
}

ConfigParams Scene::configParams() const {
    const FirePhysicsParams& q = physics_;
    ConfigParams c{};
    c.nx = nx;
    c.ny = ny;
    c.nz = nz;
    c.lx = (nx + 1) / 2;
    c.ly = (ny + 1) / 2;
    c.lz = (nz + 1) / 2;
    c.frameW = frameW;
    c.frameH = frameH;
    c.step = cfgStep_;
    c.dt = q.dt;
    c.burnFrac = std::min(1.0f, q.burnRate * q.dt);
    c.coolFrac = std::min(1.0f, q.cooling * q.dt);
    c.sootFrac = std::min(1.0f, q.sootDecay * q.dt);
    c.ignition = q.ignitionHeat;
    c.heatRelease = q.heatRelease;
    c.sootYield = q.sootYield;
    c.buoyHeat = q.buoyancyHeat;
    c.buoySoot = q.buoyancySoot;
    c.ambient = q.ambientHeat;
    c.eps = q.vorticityEps;
    c.windDtX = q.dt * q.windX;
    c.windDtZ = q.dt * q.windZ;
    c.noiseAmp = q.noiseAmplitude;
    c.invPeriod = 1.0f / q.noisePeriod;
    c.noiseSeed = q.noiseSeed;
    c.emitterCount = q.emitterCount;
    for (int e = 0; e < q.emitterCount; ++e) {
        const FireEmitterDisk& d = q.emitters[e];
        c.emitters[e] = ConfigEmitter{d.centerX, d.centerZ, d.radius * d.radius, d.fuel, d.heat, d.upVelocity, d.jitterScale,
                                      static_cast<int>(std::floor(d.centerY)), d.seed};
    }
    c.primarySamples = q.primarySamples;
    c.lightSamples = q.lightSamples;
    c.light = make_float3(q.lightX, q.lightY, q.lightZ);
    c.lightIntensity = q.lightIntensity;
    c.extinction = q.extinction;
    c.fuelExtinction = q.fuelExtinction;
    c.emission = q.emission;
    c.albedo = q.albedo;
    // Pinhole camera: forward to the target, right = forward x (0, 1, 0), up = right x forward.
    float fx = q.targetX - q.eyeX, fy = q.targetY - q.eyeY, fz = q.targetZ - q.eyeZ;
    const float fl = std::sqrt(fx * fx + fy * fy + fz * fz);
    fx = fx / fl;
    fy = fy / fl;
    fz = fz / fl;
    float rx = -fz, ry = 0.0f, rz = fx;
    const float rl = std::sqrt(rx * rx + rz * rz);
    if (rl > 0.0f) {
        rx = rx / rl;
        rz = rz / rl;
    } else {
        rx = 1.0f;
        rz = 0.0f;
    }
    c.eye = make_float3(q.eyeX, q.eyeY, q.eyeZ);
    c.forward = make_float3(fx, fy, fz);
    c.right = make_float3(rx, ry, rz);
    c.up = make_float3(ry * fz - rz * fy, rz * fx - rx * fz, rx * fy - ry * fx);
    c.tanHalf = std::tan(q.fovYDegrees * 0.00872664626f);
    c.aspect = static_cast<float>(frameW) / static_cast<float>(frameH);
    return c;
}

bool Scene::ensureConfigBuffers(std::string& err) {
    if (cfgVort_ != nullptr) return true;
    cfgLx_ = (nx + 1) / 2;
    cfgLy_ = (ny + 1) / 2;
    cfgLz_ = (nz + 1) / 2;
    const size_t lightCells = static_cast<size_t>(cfgLx_) * cfgLy_ * cfgLz_;
    return alloc(reinterpret_cast<void**>(&cfgVort_), cells_ * sizeof(float4), "cudaMalloc config vorticity", err) &&
           alloc(reinterpret_cast<void**>(&cfgLight_), lightCells * sizeof(float), "cudaMalloc config transmittance", err) &&
           check("clear config vorticity", cudaMemsetAsync(cfgVort_, 0, cells_ * sizeof(float4), stream), err) &&
           check("clear config transmittance", cudaMemsetAsync(cfgLight_, 0, lightCells * sizeof(float), stream), err);
}

// One step of this scene inside a FireBatch: the frame's bookkeeping (clocks,
// reset, frame index), the buffers the batched kernels need, and the
// descriptor of this step's buffers; then the host state advances as the
// step will leave it (record a and the faces swap once, the jitter counter
// advances).  Only for the config physics with the incremental multigrid
// projection; the batch queues the kernels.
bool Scene::batchStep(BatchScene& d, const FireSettings& s, bool render, std::string& err) {
    if (!incrementalProjection()) {
        err = "a batched scene needs the config physics with p = 0 on the top face and the multigrid solve";
        return false;
    }
    if (render && slots_[activeSlot_].ptr == nullptr) {
        err = "HDR output buffer slot is not registered.";
        return false;
    }
    const float stepDt = std::max(0.001f, std::min(s.dt, 1.0f / 30.0f));
    renderTime += stepDt;
    simTime += stepDt;
    FrameParams p = paramsFrom(s, simTime);
    if (s.reset != 0) {
        if (!runStages(kReset, kReset, p, err)) return false;
        simTime = 0.0f;
        renderTime = 0.0f;
        frameIndex = 0;
    }
    if (!ensureConfigBuffers(err)) return false;
    MgScene mg;
    if (!multigridScene(mg, err)) return false;
    ConfigParams c = configParams();
    if (c.noiseAmp != 0.0f) {
        const float key[3] = {c.noiseAmp, c.invPeriod, static_cast<float>(c.noiseSeed)};
        if (!cfgNoiseValid_ || std::memcmp(key, cfgNoiseKey_, sizeof(key)) != 0 || cfgNoiseSeed_ != c.noiseSeed) {
            if (cfgNoise_ == nullptr && !alloc(reinterpret_cast<void**>(&cfgNoise_), cells_ * sizeof(float4), "cudaMalloc config noise field", err)) {
                return false;
            }
            const int bx = rowThreads(nx);
            cfgNoiseField<<<cellGrid(bx, nx, ny, nz), bx, 0, stream>>>(cfgNoise_, c); ++launches_;
            if (!check("config noise field launch", cudaGetLastError(), err)) return false;
            std::memcpy(cfgNoiseKey_, key, sizeof(key));
            cfgNoiseSeed_ = c.noiseSeed;
            cfgNoiseValid_ = true;
        }
    }
    BatchScene b{};
    b.c = c;
    b.vel = velocity();
    for (int f = 0; f < 3; ++f) {
        b.adv[f] = vel_[f][1 - vcur_];     // advection: cur -> other
        b.forced[f] = vel_[f][vcur_];      // forces: other -> cur
        b.proj[f] = vel_[f][1 - vcur_];    // prepared faces: cur -> other, then projected in place
    }
    b.aIn = sa_[cur_];
    b.aOut = sa_[1 - cur_];
    b.vort = cfgVort_;
    b.force = contrib_;
    b.noise = c.noiseAmp != 0.0f ? cfgNoise_ : nullptr;
    b.pressure = pressure_;
    b.divergence = divergence_;
    b.delta = mgP_[0];
    b.transmittance = cfgLight_;
    b.hdr = hdr_;
    const HdrSlot& slot = slots_[activeSlot_];
    b.slot = slot.ptr;
    b.slotPitch = slot.pitchBytes;
    b.slotFormat = slot.format;
    b.count[kBatchCells] = static_cast<int>(cells_);
    b.count[kBatchFaces] = (nx + 1) * (ny + 1) * (nz + 1);
    b.count[kBatchLight] = render ? cfgLx_ * cfgLy_ * cfgLz_ : 0;
    b.count[kBatchPixels] = render ? frameW * frameH : 0;
    d = b;
    cur_ = 1 - cur_;
    vcur_ = 1 - vcur_;
    ++cfgStep_;
    mgDeltaValid_ = true;
    lastSolveGated_ = true;
    lastPressurePath_ = 3;
    ++frameIndex;
    return true;
}

// Every buffer a batched config-physics step can need (config fields,
// multigrid levels, the curl-noise field), so that batchStep allocates nothing.
bool Scene::prepareBatched(std::string& err) {
    if (!ensureConfigBuffers(err)) return false;
    MgScene mg;
    if (!multigridScene(mg, err)) return false;
    return cfgNoise_ != nullptr || alloc(reinterpret_cast<void**>(&cfgNoise_), cells_ * sizeof(float4), "cudaMalloc config noise field", err);
}

// The config physics on the frame's stage ids: advect velocity, advect +
// react + emit, forces (vorticity, cell accelerations, faces with the walls),
// divergence, SOR, subtract, transmittance, raymarch, camera response,
// metrics, reset.  VELOCITY_BOUNDARY, LIGHT_PROPAGATE, EMBERS and OVERLAY have
// no counterpart here and do nothing.
bool Scene::runConfigStages(int first, int last, const FrameParams& p, std::string& err) {
    if (!ensureConfigBuffers(err)) return false;
    const int bx = rowThreads(nx);
    const dim3 cells = cellGrid(bx, nx, ny, nz);
    for (int s = first; s <= last; ++s) {
        const ConfigParams c = configParams();
        switch (s) {
            case kAdvectVelocity:
                cfgAdvectVelocity<<<cells, bx, 0, stream>>>(vel_[0][1 - vcur_], vel_[1][1 - vcur_], vel_[2][1 - vcur_], velocity(), c); ++launches_;
                vcur_ = 1 - vcur_;
                break;
            case kAdvectReact:
                cfgAdvectScalars<<<cells, bx, 0, stream>>>(sa_[1 - cur_], sa_[cur_], velocity(), c); ++launches_;
                cur_ = 1 - cur_;
                ++cfgStep_;
                break;
            case kForce:
                if (c.eps != 0.0f) {
                    cfgVorticity<<<cells, bx, 0, stream>>>(cfgVort_, velocity(), c); ++launches_;
                }
                if (c.noiseAmp != 0.0f) {
                    // The curl-noise field depends only on its parameters: build it when they change.
                    const float key[3] = {c.noiseAmp, c.invPeriod, static_cast<float>(c.noiseSeed)};
                    if (!cfgNoiseValid_ || std::memcmp(key, cfgNoiseKey_, sizeof(key)) != 0 || cfgNoiseSeed_ != c.noiseSeed) {
                        if (cfgNoise_ == nullptr &&
                            !alloc(reinterpret_cast<void**>(&cfgNoise_), cells_ * sizeof(float4), "cudaMalloc config noise field", err)) {
                            return false;
                        }
                        cfgNoiseField<<<cells, bx, 0, stream>>>(cfgNoise_, c); ++launches_;
                        std::memcpy(cfgNoiseKey_, key, sizeof(key));
                        cfgNoiseSeed_ = c.noiseSeed;
                        cfgNoiseValid_ = true;
                    }
                }
                cfgCellForce<<<cells, bx, 0, stream>>>(contrib_, cfgVort_, sa_[cur_], cfgNoise_, c); ++launches_;
                cfgApplyForces<<<cells, bx, 0, stream>>>(vel_[0][1 - vcur_], vel_[1][1 - vcur_], vel_[2][1 - vcur_], velocity(), contrib_, c); ++launches_;
                vcur_ = 1 - vcur_;
                break;
            case kDivergence:
                if (incrementalProjection()) {
                    // The previous pressure's gradient first; the solve then finds the increment.
                    MgScene S;
                    if (!multigridScene(S, err)) return false;
                    cfgPrepareIncrement<<<cells, bx, 0, stream>>>(vel_[0][1 - vcur_], vel_[1][1 - vcur_], vel_[2][1 - vcur_], velocity(),
                                                                  pressure_, divergence_, nx, ny, nz); ++launches_;
                    vcur_ = 1 - vcur_;
                    mgDeltaValid_ = false;
                } else {
                    divergenceOf<<<cells, bx, 0, stream>>>(divergence_, pressure_, velocity(), p); ++launches_;
                }
                break;
            case kPressureSor:
                if (!runSor(p, err)) return false;
                break;
            case kSubtract:
                if (physics_.pressureTop == 1 && mgDeltaValid_) {
                    // The multigrid solve found the pressure increment: subtract its gradient.
                    cfgSubtractIncrement<<<cells, bx, 0, stream>>>(vel_[0][vcur_], vel_[1][vcur_], vel_[2][vcur_], mgP_[0], nx, ny, nz,
                                                                   last >= kWallBoundary ? 1 : 0); ++launches_;
                } else {
                    subtractWall<<<cells, bx, 0, stream>>>(vel_[0][vcur_], vel_[1][vcur_], vel_[2][vcur_], pressure_, p, 1, last >= kWallBoundary ? 1 : 0); ++launches_;
                    if (physics_.pressureTop == 1) {
                        cfgTopFaces<<<dim3((nx + bx - 1) / bx, nz), bx, 0, stream>>>(vel_[1][vcur_], pressure_, nx, ny, nz); ++launches_;
                    }
                }
                if (last >= kWallBoundary) ++s;
                break;
            case kWallBoundary:
                subtractWall<<<cells, bx, 0, stream>>>(vel_[0][vcur_], vel_[1][vcur_], vel_[2][vcur_], pressure_, p, 0, 1); ++launches_;
                break;
            case kLightBuild: {
                const int lbx = rowThreads(cfgLx_);
                cfgTransmittance<<<dim3((cfgLx_ + lbx - 1) / lbx, cfgLy_, cfgLz_), lbx, 0, stream>>>(cfgLight_, sa_[cur_], c); ++launches_;
                break;
            }
            case kRender:
                cfgRaymarch<<<dim3((frameW + 15) / 16, (frameH + 7) / 8), dim3(16, 8), 0, stream>>>(hdr_, sa_[cur_], cfgLight_, c); ++launches_;
                break;
            case kTonemap:
                tonemapOverlay<<<dim3((frameW + 15) / 16, (frameH + 15) / 16), dim3(16, 16), 0, stream>>>(bgra_, hdr_, p, 1, 0); ++launches_;
                break;
            case kMetrics:
                if (!runMetrics(p, err)) return false;
                break;
            case kReset: {
                bool ok = true;
                for (int b = 0; b < 2 && ok; ++b) {
                    ok = check("reset config scalars", cudaMemsetAsync(sa_[b], 0, cells_ * sizeof(Rec4), stream), err) &&
                         check("reset config scalars", cudaMemsetAsync(sb_[b], 0, cells_ * sizeof(Rec4), stream), err) &&
                         check("reset config scalars", cudaMemsetAsync(sc_[b], 0, cells_ * sizeof(Rec2), stream), err);
                }
                for (int f = 0; f < 3 && ok; ++f) {
                    const size_t n = f == 0 ? nu_ : (f == 1 ? nv_ : nw_);
                    ok = check("reset velocity", cudaMemsetAsync(vel_[f][0], 0, n * sizeof(FaceT), stream), err) &&
                         check("reset velocity", cudaMemsetAsync(vel_[f][1], 0, n * sizeof(FaceT), stream), err);
                }
                ok = ok && check("reset pressure", cudaMemsetAsync(pressure_, 0, cells_ * sizeof(float), stream), err) &&
                     check("reset divergence", cudaMemsetAsync(divergence_, 0, cells_ * sizeof(float), stream), err) &&
                     check("reset divergence after", cudaMemsetAsync(divergenceAfter_, 0, cells_ * sizeof(float), stream), err) &&
                     check("reset config transmittance",
                           cudaMemsetAsync(cfgLight_, 0, static_cast<size_t>(cfgLx_) * cfgLy_ * cfgLz_ * sizeof(float), stream), err);
                if (!ok) return false;
                cfgStep_ = 0;
                mgDeltaValid_ = false;
                break;
            }
            default:
                break;  // VELOCITY_BOUNDARY, LIGHT_PROPAGATE, EMBERS, OVERLAY
        }
        if (!check("config stage launch", cudaGetLastError(), err)) return false;
    }
    return true;
}

}  // namespace firesim
