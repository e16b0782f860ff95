// fire_abi.cu -- the C ABI of include/fire_cuda.h and include/fire_ext.h.
//
// The reference keeps one global scene (src/fire_cuda.cu:116-195) behind
// seventeen entry points that return bool and leave a message for
// fireCudaLastError() in the form "label: cudaGetErrorString" (:197-207).
// This file keeps that contract over one firesim::Scene.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>

#include "../../include/fire_ext.h"
#include "fire_scene.h"

namespace {

std::unique_ptr<firesim::Scene> g_scene;
int g_device = 0;
char g_lastError[512] = "No CUDA error.";

bool fail(const std::string& msg) {
    std::snprintf(g_lastError, sizeof(g_lastError), "%s", msg.c_str());
    return false;
}

bool requireScene() {
    if (!g_scene) {
        return fail("CUDA renderer is not initialized.");
    }
    return true;
}

bool initialize(int frameW, int frameH, int nx, int ny, int nz) {
    fireCudaShutdown();
    std::strcpy(g_lastError, "No CUDA error.");
    auto scene = std::make_unique<firesim::Scene>();
    std::string err;
    if (!scene->init(g_device, frameW, frameH, nx, ny, nz, err)) {
        return fail(err);
    }
    if (!scene->reset(err)) {
        return fail(err);
    }
    g_scene = std::move(scene);
    return true;
}

bool frame(uint32_t* bgra, const FireSettings* s, FireCudaFrameMetrics* metrics, bool toHdr, bool advance, bool render) {
    if (!requireScene()) return false;
    if (s == nullptr) return fail("Settings pointer was null.");
    std::string err;
    if (!g_scene->frame(bgra, *s, metrics, toHdr, advance, render, err)) return fail(err);
    return true;
}

}  // namespace

extern "C" {

// src/fire_cuda.cu:2912-3004 -- grid derived from the window request.
bool fireCudaInitialize(int frameWidth, int frameHeight, int gridWidth, int gridHeight) {
    const bool highQualityRequest = gridWidth >= 320 || gridHeight >= 220;
    auto clampI = [](int v, int lo, int hi) { return std::max(lo, std::min(hi, v)); };
    const int nx = clampI(gridWidth / 2, 72, highQualityRequest ? 176 : 104);
    const int ny = clampI(gridHeight - 32, 80, highQualityRequest ? 208 : 112);
    const int nz = clampI(gridWidth / 3, 48, highQualityRequest ? 132 : 72);
    return initialize(frameWidth, frameHeight, nx, ny, nz);
}

bool fireCudaInitializeGrid(int frameWidth, int frameHeight, int nx, int ny, int nz) {
    return initialize(frameWidth, frameHeight, nx, ny, nz);
}

bool fireCudaSetAllocationFault(long long succeedBeforeFailing) {
    if (succeedBeforeFailing < -1) return fail("fireCudaSetAllocationFault: the count must be -1 (off) or >= 0.");
    firesim::setAllocationFault(succeedBeforeFailing);
    return true;
}

bool fireCudaCheckGuards(int* corrupted) {
    int count = -1;
    std::string report;
    const bool ok = firesim::checkGuards(count, report);
    if (corrupted != nullptr) *corrupted = count;
    if (!ok || count != 0) return fail(report);
    return true;
}

bool fireCudaPlantGuardByte(const char* bufferLabel, size_t offset) {
    std::string err;
    if (!firesim::plantGuardByte(bufferLabel, offset, err)) return fail(err);
    return true;
}

bool fireCudaStepAndRender(uint32_t* bgraPixels, const FireSettings& settings) {
    return frame(bgraPixels, &settings, nullptr, false, true, true);
}

bool fireCudaStepAndRenderMeasured(uint32_t* bgraPixels, const FireSettings& settings, FireCudaFrameMetrics* metrics) {
    if (metrics == nullptr) return fail("Metrics output pointer was null.");
    return frame(bgraPixels, &settings, metrics, false, true, true);
}

bool fireCudaSelectDeviceForD3D11(void* d3d11Device) {
    (void)d3d11Device;
    return fail("D3D11 unavailable on headless build; use fireCudaSelectDevice.");
}

bool fireCudaSelectDevice(int device) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return fail("fireCudaSelectDevice: no such CUDA device.");
    }
    g_device = device;
    const cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    return true;
}

bool fireCudaRegisterD3D11Texture(void* d3d11Texture) {
    (void)d3d11Texture;
    return fail("D3D11 unavailable on headless build; use fireCudaRegisterHdrBufferSlot.");
}

bool fireCudaRegisterD3D11TextureSlot(int slot, void* d3d11Texture) {
    (void)slot;
    (void)d3d11Texture;
    return fail("D3D11 unavailable on headless build; use fireCudaRegisterHdrBufferSlot.");
}

bool fireCudaRegisterHdrBufferSlot(int slot, void* devicePtr, size_t pitchBytes, int format) {
    if (!requireScene()) return false;
    std::string err;
    if (!g_scene->registerHdrSlot(slot, devicePtr, pitchBytes, format, err)) return fail(err);
    return true;
}

bool fireCudaSetD3D11TextureSlot(int slot) {
    if (!requireScene()) return false;
    std::string err;
    if (!g_scene->setActiveSlot(slot, err)) return fail(err);
    return true;
}

bool fireCudaStepD3D11(const FireSettings& settings) { return frame(nullptr, &settings, nullptr, false, true, false); }

bool fireCudaStepAndRenderD3D11(const FireSettings& settings) { return frame(nullptr, &settings, nullptr, true, true, true); }

bool fireCudaStepAndRenderD3D11Measured(const FireSettings& settings, FireCudaFrameMetrics* metrics) {
    if (metrics == nullptr) return fail("Metrics output pointer was null.");
    return frame(nullptr, &settings, metrics, true, true, true);
}

bool fireCudaRenderD3D11(const FireSettings& settings) { return frame(nullptr, &settings, nullptr, true, false, true); }

void fireCudaUnregisterD3D11Texture(void) {
    if (g_scene) g_scene->clearSlots();
}

bool fireCudaSynchronize(void) {
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return fail(std::string("cudaDeviceSynchronize: ") + cudaGetErrorString(e));
    std::string err;
    if (g_scene && !g_scene->checkSolverStatus(err)) return fail(err);
    return true;
}

bool fireCudaReset(void) {
    if (!requireScene()) return false;
    std::string err;
    if (!g_scene->reset(err)) return fail(err);
    return true;
}

// src/fire_cuda.cu:3066-3104
bool fireCudaGetDiagnostics(FireCudaDiagnostics* diagnostics) {
    if (diagnostics == nullptr) return fail("Diagnostics output pointer was null.");
    FireCudaDiagnostics out{};
    cudaError_t e = cudaDriverGetVersion(&out.driverVersion);
    if (e != cudaSuccess) return fail(std::string("cudaDriverGetVersion: ") + cudaGetErrorString(e));
    e = cudaRuntimeGetVersion(&out.runtimeVersion);
    if (e != cudaSuccess) return fail(std::string("cudaRuntimeGetVersion: ") + cudaGetErrorString(e));
    e = cudaGetDeviceCount(&out.deviceCount);
    if (e != cudaSuccess) return fail(std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
    if (out.deviceCount <= 0) return fail("No CUDA-capable device was found.");
    int device = 0;
    e = cudaGetDevice(&device);
    if (e != cudaSuccess) return fail(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    cudaDeviceProp props{};
    e = cudaGetDeviceProperties(&props, device);
    if (e != cudaSuccess) return fail(std::string("cudaGetDeviceProperties: ") + cudaGetErrorString(e));
    out.activeDevice = device;
    out.computeMajor = props.major;
    out.computeMinor = props.minor;
    out.totalGlobalMem = static_cast<uint64_t>(props.totalGlobalMem);
    const size_t nameLen = strnlen(props.name, sizeof(out.deviceName) - 1);
    std::memcpy(out.deviceName, props.name, nameLen);
    out.deviceName[nameLen] = '\0';
    *diagnostics = out;
    return true;
}

void fireCudaShutdown(void) { g_scene.reset(); }

const char* fireCudaLastError(void) { return g_lastError; }

bool fireCudaSetPressureSolver(int iterations, float omega) {
    if (!requireScene()) return false;
    std::string err;
    if (!g_scene->setPressureSolver(iterations, omega, err)) return fail(err);
    return true;
}

bool fireCudaSetPressurePath(int path) {
    if (!requireScene()) return false;
    std::string err;
    if (!g_scene->setPressurePath(path, err)) return fail(err);
    return true;
}

bool fireCudaSetHashLattices(int enabled) {
    if (!requireScene()) return false;
    g_scene->setHashLattices(enabled != 0);
    return true;
}

bool fireCudaSetPressureTolerance(double maxResidual, int checkEvery) {
    if (!requireScene()) return false;
    std::string err;
    if (!g_scene->setPressureTolerance(maxResidual, checkEvery, err)) return fail(err);
    return true;
}

void fireCudaDefaultPhysicsParams(FirePhysicsParams* params, int nx, int ny, int nz) {
    if (params != nullptr) firesim::defaultPhysicsParams(*params, nx, ny, nz);
}

bool fireCudaSetPhysicsParams(const FirePhysicsParams* params) {
    if (!requireScene()) return false;
    if (params == nullptr) return fail("Physics parameter pointer was null.");
    std::string err;
    if (!g_scene->setPhysics(*params, err)) return fail(err);
    return true;
}

bool fireCudaSetPressureMultigrid(int maxCycles, int preSmooth, int postSmooth) {
    if (!requireScene()) return false;
    std::string err;
    if (!g_scene->setPressureMultigrid(maxCycles, preSmooth, postSmooth, err)) return fail(err);
    return true;
}

bool fireCudaGetPhysicsParams(FirePhysicsParams* params) {
    if (!requireScene()) return false;
    if (params == nullptr) return fail("Physics parameter pointer was null.");
    *params = g_scene->physics();
    return true;
}

bool fireCudaGetPressureStats(int* iterations, float* maxResidual, double* l2Residual) {
    if (!requireScene()) return false;
    if (iterations == nullptr || maxResidual == nullptr || l2Residual == nullptr) return fail("Pressure stats pointer was null.");
    std::string err;
    if (!g_scene->pressureStats(*iterations, *maxResidual, *l2Residual, err)) return fail(err);
    return true;
}

int fireCudaGetPressurePathUsed(void) { return g_scene ? g_scene->lastPressurePath() : 0; }

bool fireCudaSetAutotune(int enabled) {
    firesim::setAutotune(enabled != 0);
    return true;
}

bool fireCudaGetTunedBrick(int nx, int ny, int nz, int* brickX, float* msBrick32, float* msBrick16) {
    if (brickX == nullptr || msBrick32 == nullptr || msBrick16 == nullptr) return fail("fireCudaGetTunedBrick: null output");
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        cudaGetLastError();
        return fail("fireCudaGetTunedBrick: no CUDA device");
    }
    int pick = 0;
    if (!firesim::tunedBrickRecord(device, nx, ny, nz, pick, *msBrick32, *msBrick16)) return fail("fireCudaGetTunedBrick: grid not timed");
    *brickX = pick == 0 ? 32 : 16;
    return true;
}

bool fireCudaSetResidentSorFault(int silentBrick, long long waitUs) {
    if (!requireScene()) return false;
    std::string err;
    if (!g_scene->setResidentFault(silentBrick, waitUs, err)) return fail(err);
    return true;
}

bool fireCudaGetGridInfo(int* dims8) {
    if (!requireScene()) return false;
    if (dims8 == nullptr) return fail("dims pointer was null.");
    const firesim::Scene& s = *g_scene;
    const int d[8] = {s.nx, s.ny, s.nz, s.lnx, s.lny, s.lnz, s.frameW, s.frameH};
    std::memcpy(dims8, d, sizeof(d));
    return true;
}

bool fireCudaGetField(int field, void* host, size_t bytes) {
    if (!requireScene()) return false;
    if (host == nullptr) return fail("field host pointer was null.");
    std::string err;
    if (!g_scene->getField(field, host, bytes, err)) return fail(err);
    return true;
}

bool fireCudaSetField(int field, const void* host, size_t bytes) {
    if (!requireScene()) return false;
    if (host == nullptr) return fail("field host pointer was null.");
    std::string err;
    if (!g_scene->setField(field, host, bytes, err)) return fail(err);
    return true;
}

bool fireCudaRunStages(int first, int last, const FireSettings* settings, float time) {
    if (!requireScene()) return false;
    if (settings == nullptr) return fail("Settings pointer was null.");
    std::string err;
    const firesim::FrameParams p = g_scene->paramsFrom(*settings, time);
    if (!g_scene->runStages(first, last, p, err) || !g_scene->synchronize(err)) return fail(err);
    return true;
}

bool fireCudaRunStagesAsync(int first, int last, const FireSettings* settings, float time) {
    if (!requireScene()) return false;
    if (settings == nullptr) return fail("Settings pointer was null.");
    std::string err;
    const firesim::FrameParams p = g_scene->paramsFrom(*settings, time);
    if (!g_scene->runStages(first, last, p, err)) return fail(err);
    return true;
}

bool fireCudaGetTimes(float* simTime, float* renderTime, int* frameIndex) {
    if (!requireScene()) return false;
    if (simTime) *simTime = g_scene->simTime;
    if (renderTime) *renderTime = g_scene->renderTime;
    if (frameIndex) *frameIndex = g_scene->frameIndex;
    return true;
}

bool fireCudaSetTimes(float simTime, float renderTime, int frameIndex) {
    if (!requireScene()) return false;
    g_scene->simTime = simTime;
    g_scene->renderTime = renderTime;
    g_scene->frameIndex = frameIndex;
    return true;
}

bool fireCudaGetStream(void** stream) {
    if (!requireScene()) return false;
    if (stream == nullptr) return fail("stream pointer was null.");
    *stream = static_cast<void*>(g_scene->stream);
    return true;
}

bool fireCudaGetLaunchCount(unsigned long long* count) {
    if (!requireScene()) return false;
    if (count == nullptr) return fail("count pointer was null.");
    *count = g_scene->launchCount();
    return true;
}

const char* fireCudaBuildInfo(void) { return "firesim-b200 sm_100a"; }

// The reference declares its seventeen entry points with C++ linkage in the
// global namespace (src/fire_cuda.h:102-118), so a caller built against that
// header links against their mangled names.  A const FireSettings& passes as
// a pointer, so each mangled name is an alias of the C entry point above:
// such a caller links against this library without being recompiled.
#define FIRE_CXX_ALIAS(mangled, target) __attribute__((alias(#target), visibility("default")))
FIRE_API bool _Z18fireCudaInitializeiiii(int, int, int, int) FIRE_CXX_ALIAS(_, fireCudaInitialize);
FIRE_API bool _Z21fireCudaStepAndRenderPjRK12FireSettings(uint32_t*, const FireSettings&) FIRE_CXX_ALIAS(_, fireCudaStepAndRender);
FIRE_API bool _Z29fireCudaStepAndRenderMeasuredPjRK12FireSettingsP20FireCudaFrameMetrics(uint32_t*, const FireSettings&, FireCudaFrameMetrics*)
    FIRE_CXX_ALIAS(_, fireCudaStepAndRenderMeasured);
FIRE_API bool _Z28fireCudaSelectDeviceForD3D11Pv(void*) FIRE_CXX_ALIAS(_, fireCudaSelectDeviceForD3D11);
FIRE_API bool _Z28fireCudaRegisterD3D11TexturePv(void*) FIRE_CXX_ALIAS(_, fireCudaRegisterD3D11Texture);
FIRE_API bool _Z32fireCudaRegisterD3D11TextureSlotiPv(int, void*) FIRE_CXX_ALIAS(_, fireCudaRegisterD3D11TextureSlot);
FIRE_API bool _Z27fireCudaSetD3D11TextureSloti(int) FIRE_CXX_ALIAS(_, fireCudaSetD3D11TextureSlot);
FIRE_API bool _Z17fireCudaStepD3D11RK12FireSettings(const FireSettings&) FIRE_CXX_ALIAS(_, fireCudaStepD3D11);
FIRE_API bool _Z26fireCudaStepAndRenderD3D11RK12FireSettings(const FireSettings&) FIRE_CXX_ALIAS(_, fireCudaStepAndRenderD3D11);
FIRE_API bool _Z34fireCudaStepAndRenderD3D11MeasuredRK12FireSettingsP20FireCudaFrameMetrics(const FireSettings&, FireCudaFrameMetrics*)
    FIRE_CXX_ALIAS(_, fireCudaStepAndRenderD3D11Measured);
FIRE_API bool _Z19fireCudaRenderD3D11RK12FireSettings(const FireSettings&) FIRE_CXX_ALIAS(_, fireCudaRenderD3D11);
FIRE_API void _Z30fireCudaUnregisterD3D11Texturev(void) FIRE_CXX_ALIAS(_, fireCudaUnregisterD3D11Texture);
FIRE_API bool _Z19fireCudaSynchronizev(void) FIRE_CXX_ALIAS(_, fireCudaSynchronize);
FIRE_API bool _Z13fireCudaResetv(void) FIRE_CXX_ALIAS(_, fireCudaReset);
FIRE_API bool _Z22fireCudaGetDiagnosticsP19FireCudaDiagnostics(FireCudaDiagnostics*) FIRE_CXX_ALIAS(_, fireCudaGetDiagnostics);
FIRE_API void _Z16fireCudaShutdownv(void) FIRE_CXX_ALIAS(_, fireCudaShutdown);
FIRE_API const char* _Z17fireCudaLastErrorv(void) FIRE_CXX_ALIAS(_, fireCudaLastError);
#undef FIRE_CXX_ALIAS

}  // extern "C"

namespace firesim {
// Lets entry points defined in other translation units report through
// fireCudaLastError().
void setLastErrorMessage(const char* msg) { fail(msg); }
}  // namespace firesim
