/*
 * fire_cuda.h -- drop-in replacement for native-firesim's src/fire_cuda.h.
 *
 * The three structs keep the field order, types and defaults of the reference
 * header (src/fire_cuda.h:5-100), so a caller compiled against the reference
 * header sees the same memory layout.  The seventeen entry points keep their
 * names, argument meaning and error convention (bool + fireCudaLastError()),
 * src/fire_cuda.h:102-118.  They are declared with C linkage so that ctypes,
 * cgo or JNI can bind them directly; a `const FireSettings&` argument is
 * passed as a pointer at the ABI level, which is what the C view below
 * declares.
 *
 * Headless build: the D3D11 entry points keep their names and meaning, but a
 * "registered texture" is a caller-owned device buffer of float4 pixels
 * (fireCudaRegisterHdrBufferSlot in fire_ext.h).  fireCudaSelectDeviceForD3D11
 * and fireCudaRegisterD3D11Texture(Slot) return false with the message
 * "D3D11 unavailable on headless build".
 */
#pragma once

#include <stdint.h>

/* Exported symbols of libfiresim_b200.so (built with hidden default visibility). */
#if defined(__GNUC__)
#define FIRE_API __attribute__((visibility("default")))
#else
#define FIRE_API
#endif

#ifdef __cplusplus
#define FIRE_DEFAULT(v) = v
#define FIRE_DEFAULT_ARRAY = {}
extern "C" {
#else
#include <stdbool.h>
#define FIRE_DEFAULT(v)
#define FIRE_DEFAULT_ARRAY
#endif

/* src/fire_cuda.h:5-14 */
typedef struct FireCudaDiagnostics {
    int driverVersion FIRE_DEFAULT(0);
    int runtimeVersion FIRE_DEFAULT(0);
    int deviceCount FIRE_DEFAULT(0);
    int activeDevice FIRE_DEFAULT(-1);
    int computeMajor FIRE_DEFAULT(0);
    int computeMinor FIRE_DEFAULT(0);
    uint64_t totalGlobalMem FIRE_DEFAULT(0);
    char deviceName[128] FIRE_DEFAULT_ARRAY;
} FireCudaDiagnostics;

/* src/fire_cuda.h:16-62 */
typedef struct FireCudaFrameMetrics {
    int frameIndex FIRE_DEFAULT(0);
    int gridX FIRE_DEFAULT(0);
    int gridY FIRE_DEFAULT(0);
    int gridZ FIRE_DEFAULT(0);
    int pressureIterations FIRE_DEFAULT(0);
    int invalidCells FIRE_DEFAULT(0);
    float timeSeconds FIRE_DEFAULT(0.0f);
    float gpuSolveMs FIRE_DEFAULT(0.0f);
    float gpuRenderMs FIRE_DEFAULT(0.0f);
    float gpuVelocityMs FIRE_DEFAULT(0.0f);
    float gpuReactionMs FIRE_DEFAULT(0.0f);
    float gpuProjectionMs FIRE_DEFAULT(0.0f);
    float gpuLightingMs FIRE_DEFAULT(0.0f);
    float gpuRaymarchMs FIRE_DEFAULT(0.0f);
    float gpuPackMs FIRE_DEFAULT(0.0f);
    float heatSum FIRE_DEFAULT(0.0f);
    float fuelSum FIRE_DEFAULT(0.0f);
    float oxygenSum FIRE_DEFAULT(0.0f);
    float sootSum FIRE_DEFAULT(0.0f);
    float charSum FIRE_DEFAULT(0.0f);
    float ashSum FIRE_DEFAULT(0.0f);
    float pyrolysisSum FIRE_DEFAULT(0.0f);
    float progressSum FIRE_DEFAULT(0.0f);
    float turbulenceEnergySum FIRE_DEFAULT(0.0f);
    float sootOpticalDepthSum FIRE_DEFAULT(0.0f);
    float maxHeat FIRE_DEFAULT(0.0f);
    float maxFuel FIRE_DEFAULT(0.0f);
    float maxSoot FIRE_DEFAULT(0.0f);
    float maxPyrolysis FIRE_DEFAULT(0.0f);
    float maxProgress FIRE_DEFAULT(0.0f);
    float maxTurbulenceEnergy FIRE_DEFAULT(0.0f);
    float flameHeightMeters FIRE_DEFAULT(0.0f);
    float meanOpticalDepth FIRE_DEFAULT(0.0f);
    float meanSceneLight FIRE_DEFAULT(0.0f);
    float meanSceneShadow FIRE_DEFAULT(0.0f);
    float flameMassProxy FIRE_DEFAULT(0.0f);
    float smokeMassProxy FIRE_DEFAULT(0.0f);
    float flameSmokeOverlapProxy FIRE_DEFAULT(0.0f);
    float meanVolumetricShadow FIRE_DEFAULT(0.0f);
    float meanRoomIrradiance FIRE_DEFAULT(0.0f);
    float heatReleaseProxy FIRE_DEFAULT(0.0f);
    float divergenceBeforeL2 FIRE_DEFAULT(0.0f);
    float divergenceBeforeMax FIRE_DEFAULT(0.0f);
    float divergenceAfterL2 FIRE_DEFAULT(0.0f);
    float divergenceAfterMax FIRE_DEFAULT(0.0f);
    float divergenceReduction FIRE_DEFAULT(0.0f);
} FireCudaFrameMetrics;

/* src/fire_cuda.h:64-100 */
typedef struct FireSettings {
    int width FIRE_DEFAULT(1280);
    int height FIRE_DEFAULT(720);
    float dt FIRE_DEFAULT(1.0f / 60.0f);
    float mouseX FIRE_DEFAULT(0.5f);
    float mouseY FIRE_DEFAULT(0.12f);
    int leftDown FIRE_DEFAULT(0);
    int rightDown FIRE_DEFAULT(0);
    int reset FIRE_DEFAULT(0);
    int showGizmos FIRE_DEFAULT(1);
    int activeGizmo FIRE_DEFAULT(1);
    int sceneId FIRE_DEFAULT(0);
    float wind FIRE_DEFAULT(0.0f);
    float turbulence FIRE_DEFAULT(0.72f);
    float detail FIRE_DEFAULT(0.88f);
    float smoke FIRE_DEFAULT(0.92f);
    float intensity FIRE_DEFAULT(1.0f);
    float cameraYaw FIRE_DEFAULT(0.0f);
    float cameraPitch FIRE_DEFAULT(0.18f);
    float cameraDistance FIRE_DEFAULT(3.35f);
    int cinematicMode FIRE_DEFAULT(0);
    int raymarchSteps FIRE_DEFAULT(56);
    int emberCount FIRE_DEFAULT(96);
    int renderDebugMode FIRE_DEFAULT(0);
    float exposure FIRE_DEFAULT(1.0f);
    float reflectionGain FIRE_DEFAULT(1.0f);
    float smokeDarkness FIRE_DEFAULT(1.0f);
    float emitterCenterX FIRE_DEFAULT(0.0f);
    float emitterCenterZ FIRE_DEFAULT(0.0f);
    float emitterHeightNorm FIRE_DEFAULT(0.0f);
    float emitterHeightBandNorm FIRE_DEFAULT(0.06f);
    float emitterRadius FIRE_DEFAULT(0.48f);
    int burnerCenterCount FIRE_DEFAULT(0);
    float burnerCenterX[4] FIRE_DEFAULT_ARRAY;
    float burnerCenterY[4] FIRE_DEFAULT_ARRAY;
    float burnerCenterZ[4] FIRE_DEFAULT_ARRAY;
} FireSettings;

#ifdef __cplusplus
#define FIRE_SETTINGS_ARG const FireSettings&
#else
#define FIRE_SETTINGS_ARG const FireSettings*
#endif

/* src/fire_cuda.h:102 -- grid derived from the request exactly as the reference
 * does (src/fire_cuda.cu:2916-2922); fireCudaInitializeGrid in fire_ext.h takes
 * explicit dimensions. */
FIRE_API bool fireCudaInitialize(int frameWidth, int frameHeight, int gridWidth, int gridHeight);
/* src/fire_cuda.h:103 -- one step + render; writes W*H BGRA8 pixels to host memory, synchronous. */
FIRE_API bool fireCudaStepAndRender(uint32_t* bgraPixels, FIRE_SETTINGS_ARG settings);
/* src/fire_cuda.h:104 -- as above plus FireCudaFrameMetrics (FP64 sums, divergence norms, pass timings). */
FIRE_API bool fireCudaStepAndRenderMeasured(uint32_t* bgraPixels, FIRE_SETTINGS_ARG settings, FireCudaFrameMetrics* metrics);
/* src/fire_cuda.h:105 -- headless: returns false ("D3D11 unavailable on headless build"). */
FIRE_API bool fireCudaSelectDeviceForD3D11(void* d3d11Device);
/* src/fire_cuda.h:106-107 -- headless: returns false; use fireCudaRegisterHdrBufferSlot. */
FIRE_API bool fireCudaRegisterD3D11Texture(void* d3d11Texture);
FIRE_API bool fireCudaRegisterD3D11TextureSlot(int slot, void* d3d11Texture);
/* src/fire_cuda.h:108 -- selects which registered HDR buffer slot the *D3D11 paths write. */
FIRE_API bool fireCudaSetD3D11TextureSlot(int slot);
/* src/fire_cuda.h:109 -- step only (no render), asynchronous until fireCudaSynchronize. */
FIRE_API bool fireCudaStepD3D11(FIRE_SETTINGS_ARG settings);
/* src/fire_cuda.h:110-111 -- step + render into the active HDR buffer slot (float4 per pixel). */
FIRE_API bool fireCudaStepAndRenderD3D11(FIRE_SETTINGS_ARG settings);
FIRE_API bool fireCudaStepAndRenderD3D11Measured(FIRE_SETTINGS_ARG settings, FireCudaFrameMetrics* metrics);
/* src/fire_cuda.h:112 -- render only (advances render time, not simulation time). */
FIRE_API bool fireCudaRenderD3D11(FIRE_SETTINGS_ARG settings);
/* src/fire_cuda.h:113 -- forgets every registered HDR buffer slot. */
FIRE_API void fireCudaUnregisterD3D11Texture(void);
/* src/fire_cuda.h:114-118 */
FIRE_API bool fireCudaSynchronize(void);
FIRE_API bool fireCudaReset(void);
FIRE_API bool fireCudaGetDiagnostics(FireCudaDiagnostics* diagnostics);
FIRE_API void fireCudaShutdown(void);
FIRE_API const char* fireCudaLastError(void);

#ifdef __cplusplus
}
#endif
