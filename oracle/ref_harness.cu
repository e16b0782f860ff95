// ref_harness.cu -- test infrastructure, not product code.
//
// Drives native-firesim's own CUDA implementation (src/fire_cuda.cu, compiled
// unmodified apart from the D3D11 interop lines that oracle/build_ref.py
// removes) so that its outputs can pin the CPU oracle and check the product
// on identical inputs.  This file #includes the derived copy, so every
// anonymous-namespace kernel and global of the reference is visible here.
//
// Exposed (C linkage) for ctypes:
//   ref_init_grid     allocate the reference's globals for an explicit grid,
//                     bypassing the request clamp of src/fire_cuda.cu:2916-2922
//   ref_step          the reference's own stepAndRenderInternal (:3106-3549)
//   ref_stages        launch the reference kernels of stages [first, last] in the
//                     order and launch shapes of stepAndRenderInternal, reading
//                     the *current* fields (not the render snapshot)
//   ref_get/set_field copy a device field to/from host memory
//
// Field ids and stage ids are the ones of include/fire_ext.h (FIRE_FIELD_*,
// FIRE_STAGE_*); they are repeated as literals here because this TU sees the
// reference's own fire_cuda.h, not ours.
#include "fire_cuda_headless.cu"

namespace refh {

// Restates src/fire_cuda.cu:3135-3179 (settings -> SimParams) with an
// explicit simulation time, so one stage can be replayed at a chosen time.
SimParams paramsFrom(const FireSettings& settings, float time) {
    const float stepDt = std::max(0.001f, std::min(settings.dt, 1.0f / 30.0f));
    SimParams params = makeParams(stepDt);
    params.time = time;
    params.mouseX = std::max(0.0f, std::min(1.0f, settings.mouseX));
    params.mouseY = std::max(0.0f, std::min(1.0f, settings.mouseY));
    params.leftDown = settings.leftDown;
    params.rightDown = settings.rightDown;
    params.showGizmos = settings.showGizmos;
    params.activeGizmo = settings.activeGizmo;
    params.sceneId = std::max(0, std::min(kSceneCount - 1, settings.sceneId));
    params.wind = std::max(-1.0f, std::min(1.0f, settings.wind));
    params.turbulence = std::max(0.05f, std::min(1.8f, settings.turbulence));
    params.detail = std::max(0.1f, std::min(1.5f, settings.detail));
    params.smokeGain = std::max(0.0f, std::min(1.6f, settings.smoke));
    params.intensity = std::max(0.2f, std::min(2.4f, settings.intensity));
    params.cameraYaw = settings.cameraYaw;
    params.cameraPitch = std::max(-0.75f, std::min(0.75f, settings.cameraPitch));
    params.cameraDistance = std::max(1.5f, std::min(6.0f, settings.cameraDistance));
    params.cinematicMode = settings.cinematicMode != 0 ? 1 : 0;
    params.raymarchSteps = std::max(24, std::min(kMaxRaymarchSteps, settings.raymarchSteps));
    params.emberCount = std::max(0, std::min(kMaxEmberCount, settings.emberCount));
    params.renderDebugMode = std::max(0, std::min(6, settings.renderDebugMode));
    params.exposure = std::max(0.45f, std::min(2.40f, settings.exposure));
    params.reflectionGain = std::max(0.0f, std::min(2.2f, settings.reflectionGain));
    params.smokeDarkness = std::max(0.35f, std::min(2.4f, settings.smokeDarkness));
    params.emitterCenterX = std::max(-1.05f, std::min(1.05f, settings.emitterCenterX));
    params.emitterCenterZ = std::max(-0.82f, std::min(0.82f, settings.emitterCenterZ));
    params.emitterHeightNorm = std::max(0.0f, std::min(0.96f, settings.emitterHeightNorm));
    params.emitterHeightBandNorm = std::max(0.006f, std::min(0.20f, settings.emitterHeightBandNorm));
    params.emitterRadius = std::max(0.035f, std::min(0.80f, settings.emitterRadius));
    params.burnerCenterCount = std::max(0, std::min(4, settings.burnerCenterCount));
    for (int i = 0; i < 4; ++i) {
        params.burnerCenterX[i] = std::max(-1.05f, std::min(1.05f, settings.burnerCenterX[i]));
        params.burnerCenterY[i] = std::max(0.0f, std::min(2.03f, settings.burnerCenterY[i]));
        params.burnerCenterZ[i] = std::max(-0.82f, std::min(0.82f, settings.burnerCenterZ[i]));
    }
    if (params.sceneId == 2 && params.burnerCenterCount > 0) {
        params.emitterHeightNorm = std::max(0.0f, std::min(0.96f, (params.burnerCenterY[0] - 0.02f) / 2.03f));
    }
    updateCameraCache(params);
    return params;
}

struct FieldRef {
    void* ptr;
    size_t bytes;
};

FieldRef fieldRef(int id) {
    const size_t n = static_cast<size_t>(g_nx) * g_ny * g_nz;
    const size_t nu = static_cast<size_t>(g_nx + 1) * g_ny * g_nz;
    const size_t nv = static_cast<size_t>(g_nx) * (g_ny + 1) * g_nz;
    const size_t nw = static_cast<size_t>(g_nx) * g_ny * (g_nz + 1);
    const size_t nl = static_cast<size_t>(g_lightNx) * g_lightNy * g_lightNz;
    const size_t np = static_cast<size_t>(g_frameW) * g_frameH;
    switch (id) {
        case 0: return {g_heat, n * 4};
        case 1: return {g_fuel, n * 4};
        case 2: return {g_oxygen, n * 4};
        case 3: return {g_soot, n * 4};
        case 4: return {g_char, n * 4};
        case 5: return {g_ash, n * 4};
        case 6: return {g_pyrolysis, n * 4};
        case 7: return {g_progress, n * 4};
        case 8: return {g_turbulenceEnergy, n * 4};
        case 9: return {g_sootOptics, n * 4};
        case 10: return {g_pressure, n * 4};
        case 11: return {g_divergence, n * 4};
        case 12: return {g_u, nu * 4};
        case 13: return {g_v, nv * 4};
        case 14: return {g_w, nw * 4};
        case 15: return {g_sceneLight, nl * 16};
        case 16: return {g_sceneShadow, nl * 4};
        case 17: return {g_hdrFrameDevice, np * 16};
        case 18: return {g_frameDevice, np * 4};
        case 19: return {g_divergenceAfter, n * 4};
        default: return {nullptr, 0};
    }
}

MetricAccumulator g_lastMetrics = {};

// Stage ids (FIRE_STAGE_* in include/fire_ext.h).
enum {
    kAdvectVelocity = 0,
    kAdvectReact = 1,
    kForce = 2,
    kVelocityBoundary = 3,
    kDivergence = 4,
    kPressureSor = 5,
    kSubtract = 6,
    kWallBoundary = 7,
    kLightBuild = 8,
    kLightPropagate = 9,
    kRender = 10,
    kEmbers = 11,
    kTonemap = 12,
    kOverlay = 13,
    kMetrics = 14,
    kReset = 15,
};

bool runStage(int stage, const SimParams& params) {
    const dim3 fieldBlock(8, 8, 4);
    const dim3 scalarGrid((g_nx + 7) / 8, (g_ny + 7) / 8, (g_nz + 3) / 4);
    const int velocityMax = std::max(std::max((g_nx + 1) * g_ny * g_nz, g_nx * (g_ny + 1) * g_nz), g_nx * g_ny * (g_nz + 1));
    const dim3 lightBlock(8, 8, 4);
    const dim3 lightGrid = gridFor3d(g_lightNx, g_lightNy, g_lightNz, lightBlock);
    const dim3 frameBlock(16, 16);
    switch (stage) {
        case kReset:
            return resetSimulationFields(params);
        case kAdvectVelocity:
            for (int zStart = 0; zStart < g_nz; zStart += kVolumeLaunchDepth) {
                const int zEnd = std::min(g_nz, zStart + kVolumeLaunchDepth);
                const SimParams slice = withVolumeWindow(params, zStart, zEnd);
                advectUKernel<<<gridFor3d(g_nx + 1, g_ny, zEnd - zStart, fieldBlock), fieldBlock>>>(g_uNext, g_u, g_v, g_w, slice);
                advectVKernel<<<gridFor3d(g_nx, g_ny + 1, zEnd - zStart, fieldBlock), fieldBlock>>>(g_vNext, g_u, g_v, g_w, slice);
            }
            for (int zStart = 0; zStart < g_nz + 1; zStart += kVolumeLaunchDepth) {
                const int zEnd = std::min(g_nz + 1, zStart + kVolumeLaunchDepth);
                const SimParams slice = withVolumeWindow(params, zStart, zEnd);
                advectWKernel<<<gridFor3d(g_nx, g_ny, zEnd - zStart, fieldBlock), fieldBlock>>>(g_wNext, g_u, g_v, g_w, slice);
            }
            std::swap(g_u, g_uNext);
            std::swap(g_v, g_vNext);
            std::swap(g_w, g_wNext);
            return true;
        case kAdvectReact:
            for (int zStart = 0; zStart < g_nz; zStart += kVolumeLaunchDepth) {
                const int zEnd = std::min(g_nz, zStart + kVolumeLaunchDepth);
                const SimParams slice = withVolumeWindow(params, zStart, zEnd);
                advectReactKernel<<<gridFor3d(g_nx, g_ny, zEnd - zStart, fieldBlock), fieldBlock>>>(
                    g_heatNext, g_fuelNext, g_oxygenNext, g_sootNext, g_charNext, g_ashNext, g_pyrolysisNext,
                    g_progressNext, g_turbulenceEnergyNext, g_sootOpticsNext, g_heat, g_fuel, g_oxygen, g_soot,
                    g_char, g_ash, g_pyrolysis, g_progress, g_turbulenceEnergy, g_sootOptics, g_u, g_v, g_w, slice);
            }
            std::swap(g_heat, g_heatNext);
            std::swap(g_fuel, g_fuelNext);
            std::swap(g_oxygen, g_oxygenNext);
            std::swap(g_soot, g_sootNext);
            std::swap(g_char, g_charNext);
            std::swap(g_ash, g_ashNext);
            std::swap(g_pyrolysis, g_pyrolysisNext);
            std::swap(g_progress, g_progressNext);
            std::swap(g_turbulenceEnergy, g_turbulenceEnergyNext);
            std::swap(g_sootOptics, g_sootOpticsNext);
            return true;
        case kForce:
            for (int zStart = 0; zStart < g_nz; zStart += kVolumeLaunchDepth) {
                const int zEnd = std::min(g_nz, zStart + kVolumeLaunchDepth);
                const SimParams slice = withVolumeWindow(params, zStart, zEnd);
                forceVelocityKernel<<<gridFor3d(g_nx, g_ny, zEnd - zStart, fieldBlock), fieldBlock>>>(
                    g_u, g_v, g_w, g_heat, g_soot, g_turbulenceEnergy, g_progress, slice);
            }
            return true;
        case kVelocityBoundary:
            velocityBoundaryKernel<<<(velocityMax + 255) / 256, 256>>>(g_u, g_v, g_w, params);
            return true;
        case kDivergence:
            divergenceKernel<<<scalarGrid, fieldBlock>>>(g_divergence, g_pressure, g_u, g_v, g_w, params);
            return true;
        case kPressureSor: {
            const int cells = ((g_nx + 1) / 2) * g_ny * g_nz;
            for (int i = 0; i < kPressureIterations; ++i) {
                sorPressureParityKernel<<<(cells + kCudaBlockThreads - 1) / kCudaBlockThreads, kCudaBlockThreads>>>(g_pressure, g_divergence, params, 0, kPressureOmega);
                sorPressureParityKernel<<<(cells + kCudaBlockThreads - 1) / kCudaBlockThreads, kCudaBlockThreads>>>(g_pressure, g_divergence, params, 1, kPressureOmega);
            }
            return true;
        }
        case kSubtract:
            subtractPressureKernel<<<scalarGrid, fieldBlock>>>(g_u, g_v, g_w, g_pressure, params);
            return true;
        case kWallBoundary:
            velocityWallBoundaryKernel<<<(velocityMax + 255) / 256, 256>>>(g_u, g_v, g_w, params);
            return true;
        case kLightBuild:
            buildSceneLightKernel<<<lightGrid, lightBlock>>>(g_sceneLight, g_sceneShadow, g_heat, g_fuel, g_oxygen, g_soot,
                                                             g_char, g_ash, g_pyrolysis, g_progress, g_sootOptics, params);
            return true;
        case kLightPropagate:
            propagateSceneLightKernel<<<lightGrid, lightBlock>>>(g_sceneLightNext, g_sceneLight, g_sceneShadow, params, 0.48f, 0.92f);
            propagateSceneLightKernel<<<lightGrid, lightBlock>>>(g_sceneLight, g_sceneLightNext, g_sceneShadow, params, 0.34f, 0.96f);
            return true;
        case kRender:
            for (int yStart = 0; yStart < g_frameH; yStart += kRenderLaunchRows) {
                const int yEnd = std::min(g_frameH, yStart + kRenderLaunchRows);
                const SimParams slice = withFrameWindow(params, yStart, yEnd);
                renderKernel<<<gridForFrameRows(g_frameW, yEnd - yStart, frameBlock), frameBlock>>>(
                    g_hdrFrameDevice, g_heat, g_fuel, g_oxygen, g_soot, g_char, g_ash, g_pyrolysis, g_progress,
                    g_turbulenceEnergy, g_sootOptics, g_sceneLight, g_sceneShadow, g_u, g_v, g_w, slice);
            }
            return true;
        case kEmbers:
            if (params.emberCount > 0 && params.renderDebugMode == 0) {
                emberHdrKernel<<<(params.emberCount + kCudaBlockThreads - 1) / kCudaBlockThreads, kCudaBlockThreads>>>(
                    g_hdrFrameDevice, g_heat, g_char, g_pyrolysis, g_turbulenceEnergy, g_u, g_v, g_w, params);
            }
            return true;
        case kTonemap:
            for (int yStart = 0; yStart < g_frameH; yStart += kRenderLaunchRows) {
                const int yEnd = std::min(g_frameH, yStart + kRenderLaunchRows);
                const SimParams slice = withFrameWindow(params, yStart, yEnd);
                tonemapKernel<<<gridForFrameRows(g_frameW, yEnd - yStart, frameBlock), frameBlock>>>(g_frameDevice, g_hdrFrameDevice, slice);
            }
            return true;
        case kOverlay:
            for (int yStart = 0; yStart < g_frameH; yStart += kRenderLaunchRows) {
                const int yEnd = std::min(g_frameH, yStart + kRenderLaunchRows);
                const SimParams slice = withFrameWindow(params, yStart, yEnd);
                overlayKernel<<<gridForFrameRows(g_frameW, yEnd - yStart, frameBlock), frameBlock>>>(g_frameDevice, g_heat, slice);
            }
            return true;
        case kMetrics: {
            divergenceOnlyKernel<<<scalarGrid, fieldBlock>>>(g_divergenceAfter, g_u, g_v, g_w, params);
            if (cudaMemset(g_metricsDevice, 0, sizeof(MetricAccumulator)) != cudaSuccess) {
                return false;
            }
            accumulateMetricsKernel<<<scalarGrid, fieldBlock>>>(
                g_metricsDevice, g_heat, g_fuel, g_oxygen, g_soot, g_char, g_ash, g_pyrolysis, g_progress,
                g_turbulenceEnergy, g_sootOptics, g_sceneLight, g_sceneShadow, g_divergence, g_divergenceAfter, params);
            return cudaMemcpy(&g_lastMetrics, g_metricsDevice, sizeof(MetricAccumulator), cudaMemcpyDeviceToHost) == cudaSuccess;
        }
        default:
            std::snprintf(g_lastError, sizeof(g_lastError), "unknown stage %d", stage);
            return false;
    }
}

bool allocateAll() {
    const size_t n = static_cast<size_t>(g_nx) * g_ny * g_nz * sizeof(float);
    const size_t nu = static_cast<size_t>(g_nx + 1) * g_ny * g_nz * sizeof(float);
    const size_t nv = static_cast<size_t>(g_nx) * (g_ny + 1) * g_nz * sizeof(float);
    const size_t nw = static_cast<size_t>(g_nx) * g_ny * (g_nz + 1) * sizeof(float);
    const size_t nl = static_cast<size_t>(g_lightNx) * g_lightNy * g_lightNz;
    const size_t np = static_cast<size_t>(g_frameW) * g_frameH;
    float** scalars[] = {&g_heat, &g_heatNext, &g_fuel, &g_fuelNext, &g_oxygen, &g_oxygenNext, &g_soot, &g_sootNext,
                         &g_char, &g_charNext, &g_ash, &g_ashNext, &g_pyrolysis, &g_pyrolysisNext, &g_progress,
                         &g_progressNext, &g_turbulenceEnergy, &g_turbulenceEnergyNext, &g_sootOptics,
                         &g_sootOpticsNext, &g_pressure, &g_pressureNext, &g_divergence, &g_divergenceAfter};
    for (float** f : scalars) {
        if (cudaMalloc(f, n) != cudaSuccess) return false;
    }
    if (cudaMalloc(&g_u, nu) != cudaSuccess || cudaMalloc(&g_uNext, nu) != cudaSuccess ||
        cudaMalloc(&g_v, nv) != cudaSuccess || cudaMalloc(&g_vNext, nv) != cudaSuccess ||
        cudaMalloc(&g_w, nw) != cudaSuccess || cudaMalloc(&g_wNext, nw) != cudaSuccess ||
        cudaMalloc(&g_metricsDevice, sizeof(MetricAccumulator)) != cudaSuccess ||
        cudaMalloc(&g_frameDevice, np * 4) != cudaSuccess || cudaMalloc(&g_hdrFrameDevice, np * 16) != cudaSuccess ||
        cudaMalloc(&g_sceneLight, nl * 16) != cudaSuccess || cudaMalloc(&g_sceneLightNext, nl * 16) != cudaSuccess ||
        cudaMalloc(&g_sceneShadow, nl * 4) != cudaSuccess) {
        return false;
    }
    for (int slot = 0; slot < kRenderSnapshotSlots; ++slot) {
        if (!allocateRenderSnapshotSlot(slot, n, nu, nv, nw, nl * 16, nl * 4)) return false;
    }
    cudaEvent_t* events[] = {&g_stepStartEvent, &g_afterVelocityEvent, &g_afterReactionEvent, &g_afterProjectionEvent,
                             &g_afterLightingEvent, &g_afterRaymarchEvent, &g_afterPackEvent, &g_afterSolveEvent,
                             &g_afterRenderEvent};
    for (cudaEvent_t* e : events) {
        if (cudaEventCreate(e) != cudaSuccess) return false;
    }
    return cudaMemset(g_hdrFrameDevice, 0, np * 16) == cudaSuccess && cudaMemset(g_frameDevice, 0, np * 4) == cudaSuccess;
}

// Evaluates one of the reference's own __device__ noise/math functions on n
// input tuples (3 floats each), one thread per tuple, to compare their
// rounding with the CPU oracle's restatement.
__global__ void probeKernel(int kind, int n, const float* in, float* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const float a = in[3 * i], b = in[3 * i + 1], c = in[3 * i + 2];
    float r = 0.0f;
    switch (kind) {
        case 0: r = hash21(make_float2(a, b)); break;
        case 1: r = hash31(make_float3(a, b, c)); break;
        case 2: r = valueNoise(make_float2(a, b)); break;
        case 3: r = valueNoise3(make_float3(a, b, c)); break;
        case 4: r = fbm(make_float2(a, b)); break;
        case 5: r = fbm3(make_float3(a, b, c)); break;
        case 6: r = sinf(a); break;
        case 7: r = expf(a); break;
        case 8: r = logf(a); break;
        case 9: r = powf(a, b); break;
        case 10: r = cosf(a); break;
        case 11: r = atan2f(a, b); break;
        case 12: r = sqrtf(a); break;
        default: r = 0.0f; break;
    }
    out[i] = r;
}

}  // namespace refh

extern "C" {

int ref_probe(int kind, int n, const float* hostIn, float* hostOut) {
    float* dIn = nullptr;
    float* dOut = nullptr;
    if (n <= 0) return -2;
    if (cudaMalloc(&dIn, size_t(n) * 3 * sizeof(float)) != cudaSuccess) return -1;
    if (cudaMalloc(&dOut, size_t(n) * sizeof(float)) != cudaSuccess) {
        cudaFree(dIn);
        return -1;
    }
    int rc = 0;
    if (cudaMemcpy(dIn, hostIn, size_t(n) * 3 * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) rc = -1;
    if (rc == 0) {
        refh::probeKernel<<<(n + 255) / 256, 256>>>(kind, n, dIn, dOut);
        if (cudaDeviceSynchronize() != cudaSuccess) rc = -1;
    }
    if (rc == 0 && cudaMemcpy(hostOut, dOut, size_t(n) * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) rc = -1;
    cudaFree(dIn);
    cudaFree(dOut);
    return rc;
}

// Grid-explicit init; light grid from src/fire_cuda.cu:2920-2922.
int ref_init_grid(int frameW, int frameH, int nx, int ny, int nz) {
    fireCudaShutdown();
    g_frameW = frameW;
    g_frameH = frameH;
    g_nx = nx;
    g_ny = ny;
    g_nz = nz;
    g_lightNx = clampHost((g_nx + 3) / 4, 18, 48);
    g_lightNy = clampHost((g_ny + 3) / 4, 20, 56);
    g_lightNz = clampHost((g_nz + 3) / 4, 16, 36);
    g_time = 0.0f;
    g_renderTime = 0.0f;
    g_frameIndex = 0;
    if (cudaSetDevice(0) != cudaSuccess || !refh::allocateAll()) {
        std::snprintf(g_lastError, sizeof(g_lastError), "ref_init_grid: allocation failed");
        freeDeviceMemory();
        return -1;
    }
    return fireCudaReset() ? 0 : -1;
}

// The reference's own full step (src/fire_cuda.cu:3106); mode 0 = BGRA step,
// 1 = BGRA step + metrics, 2 = step only, 3 = render only (BGRA).
int ref_step(uint32_t* bgra, const FireSettings* settings, FireCudaFrameMetrics* metrics, int mode) {
    bool ok = false;
    switch (mode) {
        case 0: ok = stepAndRenderInternal(bgra, *settings, nullptr, false, true, true); break;
        case 1: ok = stepAndRenderInternal(bgra, *settings, metrics, false, true, true); break;
        case 2: ok = stepAndRenderInternal(nullptr, *settings, nullptr, false, true, false); break;
        case 3: ok = stepAndRenderInternal(bgra, *settings, nullptr, false, false, true); break;
        default: return -2;
    }
    if (!ok) return -1;
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

int ref_stages(int first, int last, const FireSettings* settings, float time) {
    const SimParams params = refh::paramsFrom(*settings, time);
    for (int s = first; s <= last; ++s) {
        if (!refh::runStage(s, params)) return -1;
    }
    const cudaError_t err = cudaDeviceSynchronize();
    if (err != cudaSuccess) {
        std::snprintf(g_lastError, sizeof(g_lastError), "ref_stages: %s", cudaGetErrorString(err));
        return -1;
    }
    return 0;
}

long long ref_field_bytes(int id) { return static_cast<long long>(refh::fieldRef(id).bytes); }

int ref_get_field(int id, void* host, long long bytes) {
    const refh::FieldRef f = refh::fieldRef(id);
    if (f.ptr == nullptr || static_cast<size_t>(bytes) != f.bytes) return -2;
    return cudaMemcpy(host, f.ptr, f.bytes, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -1;
}

int ref_set_field(int id, const void* host, long long bytes) {
    const refh::FieldRef f = refh::fieldRef(id);
    if (f.ptr == nullptr || static_cast<size_t>(bytes) != f.bytes) return -2;
    return cudaMemcpy(f.ptr, host, f.bytes, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : -1;
}

// MetricAccumulator of the last kMetrics stage: 21 doubles then 10 ints.
int ref_last_metrics(double* sums21, int* bits10) {
    const MetricAccumulator& m = refh::g_lastMetrics;
    const double* d = &m.heatSum;
    for (int i = 0; i < 21; ++i) sums21[i] = d[i];
    const int* b = &m.maxHeatBits;
    for (int i = 0; i < 10; ++i) bits10[i] = b[i];
    return 0;
}

void ref_get_times(float* simTime, float* renderTime, int* frameIndex) {
    *simTime = g_time;
    *renderTime = g_renderTime;
    *frameIndex = g_frameIndex;
}

void ref_light_dims(int* dims) {
    dims[0] = g_lightNx;
    dims[1] = g_lightNy;
    dims[2] = g_lightNz;
}

const char* ref_last_error() { return g_lastError; }

// Host-side parameter block of a frame (camera basis and clamped settings), for
// comparing host arithmetic; needs no GPU.
void ref_frame_params(const FireSettings* settings, float time, int frameW, int frameH, float* out16) {
    const int w = g_frameW, h = g_frameH;
    g_frameW = frameW;
    g_frameH = frameH;
    const SimParams p = refh::paramsFrom(*settings, time);
    g_frameW = w;
    g_frameH = h;
    const float v[16] = {p.cameraEye.x, p.cameraEye.y, p.cameraEye.z, p.cameraForward.x, p.cameraForward.y, p.cameraForward.z,
                         p.cameraRight.x, p.cameraRight.y, p.cameraRight.z, p.cameraUp.x, p.cameraUp.y, p.cameraUp.z,
                         p.cameraTanHalfFov, p.cameraAspect, p.time, p.dt};
    for (int i = 0; i < 16; ++i) out16[i] = v[i];
}

void ref_shutdown() { fireCudaShutdown(); }

}  // extern "C"
