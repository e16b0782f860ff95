/*
 * fire_ext.h -- extensions of the fire_cuda.h ABI (C linkage, plain pointers and sizes).
 *
 * None of these entry points exists in native-firesim; they cover what its
 * ABI cannot express on a headless Linux box (see each comment).  They act on
 * the same singleton scene as fire_cuda.h ("scene 0"), except the fireScene*
 * family, which manages independent scenes by handle.  Every function returns
 * false (or NULL) on error and sets fireCudaLastError().
 */
#pragma once

#include <stddef.h>

#include "fire_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Field ids for fireCudaGetField / fireCudaSetField.  Scalars and the pressure
 * and divergence fields hold nx*ny*nz floats (x fastest); the MAC faces hold
 * (nx+1)*ny*nz, nx*(ny+1)*nz and nx*ny*(nz+1) floats; SCENE_LIGHT holds four
 * floats per light cell (radiance RGB, extinction); HDR four floats per pixel;
 * BGRA one uint32 per pixel. */
enum FireFieldId {
    FIRE_FIELD_HEAT = 0,
    FIRE_FIELD_FUEL = 1,
    FIRE_FIELD_OXYGEN = 2,
    FIRE_FIELD_SOOT = 3,
    FIRE_FIELD_CHAR = 4,
    FIRE_FIELD_ASH = 5,
    FIRE_FIELD_PYROLYSIS = 6,
    FIRE_FIELD_PROGRESS = 7,
    FIRE_FIELD_TURBULENCE_ENERGY = 8,
    FIRE_FIELD_SOOT_OPTICS = 9,
    FIRE_FIELD_PRESSURE = 10,
    FIRE_FIELD_DIVERGENCE = 11,
    FIRE_FIELD_U = 12,
    FIRE_FIELD_V = 13,
    FIRE_FIELD_W = 14,
    FIRE_FIELD_SCENE_LIGHT = 15,
    FIRE_FIELD_SCENE_SHADOW = 16,
    FIRE_FIELD_HDR = 17,
    FIRE_FIELD_BGRA = 18,
    FIRE_FIELD_DIVERGENCE_AFTER = 19,
    /* Config physics: transmittance to the point light, one float per cell of
     * the half-resolution grid ((nx+1)/2 * (ny+1)/2 * (nz+1)/2). */
    FIRE_FIELD_CONFIG_TRANSMITTANCE = 20
};

/* The passes of one frame, in order (the launch sequence of
 * stepAndRenderInternal, src/fire_cuda.cu:3196-3471). */
enum FireStageId {
    FIRE_STAGE_ADVECT_VELOCITY = 0,
    FIRE_STAGE_ADVECT_REACT = 1,
    FIRE_STAGE_FORCE = 2,
    FIRE_STAGE_VELOCITY_BOUNDARY = 3,
    FIRE_STAGE_DIVERGENCE = 4,
    FIRE_STAGE_PRESSURE_SOR = 5,
    FIRE_STAGE_SUBTRACT = 6,
    FIRE_STAGE_WALL_BOUNDARY = 7,
    FIRE_STAGE_LIGHT_BUILD = 8,
    FIRE_STAGE_LIGHT_PROPAGATE = 9,
    FIRE_STAGE_RENDER = 10,
    FIRE_STAGE_EMBERS = 11,
    FIRE_STAGE_TONEMAP = 12,
    FIRE_STAGE_OVERLAY = 13,
    FIRE_STAGE_METRICS = 14,
    FIRE_STAGE_RESET = 15
};

enum FireHdrFormat {
    FIRE_HDR_RGBA32F = 0, /* float4 per pixel */
    FIRE_HDR_RGBA16F = 1  /* half4 per pixel, negatives clamped to 0 (as packFp16SurfaceKernel) */
};

/* Grid-explicit initialisation: fireCudaInitialize derives the grid from a
 * window request and clamps it to nx>=72 (src/fire_cuda.cu:2916-2922), so it
 * cannot express 64^3, 128^3 or 256^3.  The light grid follows the reference's
 * rule (ceil(n/4) clamped to [18,48] x [20,56] x [16,36]). */
FIRE_API bool fireCudaInitializeGrid(int frameWidth, int frameHeight, int nx, int ny, int nz);

/* Headless stand-in for fireCudaSelectDeviceForD3D11: picks the CUDA device by
 * ordinal for the next initialisation. */
FIRE_API bool fireCudaSelectDevice(int device);

/* Registers a caller-owned device buffer (frameWidth x frameHeight pixels,
 * pitchBytes per row, FireHdrFormat) as HDR output slot 0..3: the headless form
 * of fireCudaRegisterD3D11TextureSlot.  The *D3D11 entry points write the
 * active slot (fireCudaSetD3D11TextureSlot). */
FIRE_API bool fireCudaRegisterHdrBufferSlot(int slot, void* devicePtr, size_t pitchBytes, int format);

/* Pressure-solver policy: SOR iterations and over-relaxation factor
 * (the reference hard-codes 40 and 1.52, src/fire_cuda.cu:104-105). */
FIRE_API bool fireCudaSetPressureSolver(int iterations, float omega);

/* Execution path of the SOR solve (identical results): 0 = automatic (one
 * cooperative launch that keeps p and div in shared memory when every brick of
 * the grid can be co-resident, else the colour-split solve), 1 = colour-split
 * solve (p and div copied into per-colour arrays, one launch per half sweep,
 * replayed as one CUDA graph), 2 = shared-memory-resident only (fails if the
 * grid does not fit). */
FIRE_API bool fireCudaSetPressurePath(int path);

/* Scene/emitter contract.  Writes the emitter fields of *settings
 * (emitterCenterX/Z, emitterHeightNorm, emitterHeightBandNorm, emitterRadius,
 * burnerCenterCount, burnerCenterX/Y/Z) for scene `sceneId` (clamped to 0..2)
 * as the reference's worker does before each frame: from
 * <fireScenesDir>/<room|campfire|gas-burner-aver1>/scene.json and, for scenes
 * 1 and 2, emitter-mask.json beside it.  Replaces loadSceneEmitterParams +
 * applySceneEmitterParams (src/main.cpp:1397-1476, :433-447), whose directory
 * is the fixed relative path assets/fire-scenes.  A NULL or unreadable
 * directory gives the reference's built-in values for the scene.  Host only;
 * touches no GPU state. */
FIRE_API bool fireCudaApplySceneContract(int sceneId, const char* fireScenesDir, FireSettings* settings);

/* Hash lattices (default on): fbm fields evaluated over the whole grid or
 * frame read their sin hashes from a table built once per step or frame.
 * Off, every corner is hashed in place.  The results are the same bits either
 * way; the switch exists to test that and to measure the tables' effect.  No
 * counterpart in the reference, which always hashes in place. */
FIRE_API bool fireCudaSetHashLattices(int enabled);

/* Residual-gated pressure solve (SOR policy; the reference always runs a
 * fixed count, src/fire_cuda.cu:3280-3284).  With maxResidual > 0 the
 * solve runs in chunks of checkEvery iterations; after
 * each chunk the residual r = div + (six neighbours, clamped at the walls) - 6p
 * is reduced in a fixed order (max |r| in FP32, L2 in FP64) and once
 * max |r| <= maxResidual the remaining chunks return at once, up to the
 * iteration count of fireCudaSetPressureSolver.  The host does not wait.
 * maxResidual = 0 restores the fixed count.  A gated solve that runs m
 * iterations gives the same bits as a fixed solve of m iterations, on either
 * path. */
FIRE_API bool fireCudaSetPressureTolerance(double maxResidual, int checkEvery);
/* Iterations run, max |r| and L2 residual of the latest gated solve (waits
 * for the scene's stream); after a fixed-count solve: the count and -1. */
FIRE_API bool fireCudaGetPressureStats(int* iterations, float* maxResidual, double* l2Residual);

/* Autotuner of the shared-memory-resident SOR's brick shape (no counterpart
 * in the reference, which has no resident solve).  When both 32x16x16 and
 * 16x16x16 bricks fit co-resident, the first resident solve of a grid times
 * one solve with each, from the same pressure (the results are the same
 * bits), and keeps the faster for that grid and device for the life of the
 * process; later scenes of the grid reuse the choice.  On by default; off,
 * the fixed rule picks (32x16x16 when it gives every SM a brick).
 * Process-wide; needs no scene. */
FIRE_API bool fireCudaSetAutotune(int enabled);
/* The autotuner's record for an nx x ny x nz grid on the current device:
 * *brickX = 32 or 16 (the brick kept) and the measured time of one solve
 * with each; false when the grid has not been timed. */
FIRE_API bool fireCudaGetTunedBrick(int nx, int ny, int nz, int* brickX, float* msBrick32, float* msBrick16);

/* Path the latest pressure solve took: 0 = none yet (or no grid),
 * 1 = colour-split SOR, 2 = shared-memory-resident SOR, 3 = multigrid. */
FIRE_API int fireCudaGetPressurePathUsed(void);

/* Failure detection of the shared-memory-resident SOR (no counterpart in the
 * reference, whose solve is one launch per half sweep).  Each brick waits only
 * for its face neighbours; every wait gives up after waitUs microseconds
 * (default 1 s), records the brick and lets the whole solve return, and the
 * next fireCudaSynchronize (or synchronous step) fails with "timed out".
 * silentBrick >= 0 injects the fault from the host: that brick never
 * announces its half sweeps.  Pass (-1, 1000000) to restore the defaults. */
FIRE_API bool fireCudaSetResidentSorFault(int silentBrick, long long waitUs);

/* Host-side fault injection of device allocations (no counterpart in the
 * reference): -1 turns it off; n >= 0 lets n more of the library's scene
 * allocations succeed, after which every one fails as cudaMalloc does when
 * device memory runs out ("out of memory (injected)").  Nothing reaches the
 * GPU: the failing call is never made.  Initialisation that hits it fails
 * and frees what it had allocated, as the reference's init does
 * (src/fire_cuda.cu:2981). */
FIRE_API bool fireCudaSetAllocationFault(long long succeedBeforeFailing);

/* Bounds checks (no counterpart in the reference, whose kernels index
 * unchecked, src/fire_cuda.cu:445-487).  The FIRE_BOUNDS_CHECK build of this
 * library, libfiresim_b200_checked.so, places every device buffer it owns
 * between two 2 MiB guard zones and fills the whole allocation with 0xFF
 * bytes (NaN in every float field, -1 in every integer) when it is made.
 * fireCudaCheckGuards synchronizes the current device and scans the guard
 * zones of every live buffer on it and of those freed since the last call.
 * *corrupted = the number of buffers with a changed zone (0: every zone
 * intact; -1: this library is not the checked build).  Returns false when
 * a zone changed (fireCudaLastError names the first buffer, the side and
 * the byte), on a CUDA error, and in the default builds.  Changed zones are
 * re-armed, so each change is reported once. */
FIRE_API bool fireCudaCheckGuards(int* corrupted);

/* Checked build only: sets the byte `offset` bytes past the end of the first
 * live buffer named `bufferLabel` (e.g. "pressure") to 0 with a host-side
 * cudaMemset inside that buffer's allocation: the checker's own test. */
FIRE_API bool fireCudaPlantGuardByte(const char* bufferLabel, size_t offset);

/* nx, ny, nz, lightNx, lightNy, lightNz, frameWidth, frameHeight. */
FIRE_API bool fireCudaGetGridInfo(int* dims8);

/* Copies one field between host memory and the scene (bytes must match). */
FIRE_API bool fireCudaGetField(int field, void* host, size_t bytes);
FIRE_API bool fireCudaSetField(int field, const void* host, size_t bytes);

/* Runs stages [first, last] on the current fields at an explicit simulation
 * time, with the settings clamped as in a step (src/fire_cuda.cu:3135-3179).
 * The clocks are not advanced. */
FIRE_API bool fireCudaRunStages(int first, int last, const FireSettings* settings, float time);

/* As fireCudaRunStages, but returns once the stages are queued on the scene's
 * stream (fireCudaGetStream) instead of waiting for them; errors the GPU
 * reports surface at the next fireCudaSynchronize.  Lets a caller bracket a
 * stage range with its own events on that stream. */
FIRE_API bool fireCudaRunStagesAsync(int first, int last, const FireSettings* settings, float time);

/* Simulation clock, render clock and frame index of the singleton scene. */
FIRE_API bool fireCudaGetTimes(float* simTime, float* renderTime, int* frameIndex);
FIRE_API bool fireCudaSetTimes(float simTime, float renderTime, int frameIndex);

/* The CUDA stream (cudaStream_t) the singleton scene launches on, so callers can
 * order their own work or record events against it. */
FIRE_API bool fireCudaGetStream(void** stream);

/* Kernels launched by the singleton scene since initialisation (kernels inside
 * captured graphs are counted one by one). */
FIRE_API bool fireCudaGetLaunchCount(unsigned long long* count);

/* The force pass (stages FORCE..DIVERGENCE: force increments, their face
 * gather with the boundary clamps, divergence, pressure reset) on buffers the
 * caller owns, without any device allocation.  No counterpart in the
 * reference: it exists for callers that cannot let a library allocate --
 * engines that own all device memory through their own arena, frames being
 * captured into a CUDA graph (cudaMalloc cannot be captured), plugins whose
 * host forbids allocations after start-up.
 *
 * Inputs: the cell records in this library's packed layout (recordsA: 4-vector
 * heat, fuel, oxygen, soot; recordsB: 4-vector char, ash, pyrolysis, progress;
 * recordsC: 2-vector turbulenceEnergy, sootOptics; nx*ny*nz each, x fastest) and
 * the MAC faces u, v, w.  Outputs: uOut, vOut, wOut, divergence (nx*ny*nz) and
 * pressure (set to 0).  All device pointers; work is queued on `stream`
 * (0 = legacy default stream) and the call returns without synchronising.
 *
 * Element type: records and faces (inputs and uOut/vOut/wOut) are in the
 * storage type of the library that is loaded: float in libfiresim_b200.so,
 * IEEE half in libfiresim_b200_f16.so, bfloat16 in libfiresim_b200_bf16.so
 * (the pointer types below are float only for the FP32 build's sake);
 * divergence and pressure are float in every build.
 *
 * Physics: this is the reference physics' force pass (FirePhysicsParams mode
 * 0) only.  It takes no physics parameters and ignores any mode set with
 * fireCudaSetPhysicsParams; the config physics' FORCE..DIVERGENCE stages are
 * different kernels.
 *
 * Errors: if a CUDA error from the caller's earlier work is already pending,
 * nothing is launched and the call fails without clearing it.  ny and nz are
 * at most 65535.
 *
 * Limit: at most 1,048,576 cells (nx*ny*nz); larger grids are rejected.  The
 * per-cell increments live in one fixed 16 MiB array that every GPU loading
 * the library holds until exit.  The first call on each device resolves that
 * array's device address, so make it before any stream capture.  All calls
 * share the array: calls that overlap on the GPU (other streams, other host
 * threads) race.  Each call overwrites the first nx*ny*nz entries before
 * reading them, so nothing has to be cleared between calls. */
FIRE_API bool fireCudaForceProjectNoAlloc(const FireSettings* settings, float time, int nx, int ny, int nz,
                                          const void* recordsA, const void* recordsB, const void* recordsC,
                                          const float* u, const float* v, const float* w, float* uOut, float* vOut,
                                          float* wOut, float* divergence, float* pressure, void* stream);

/* ---- Config physics ----------------------------------------------------
 * A second physics of the same scene and kernels' projection, for workloads
 * written as a plain T/F/S smoke-and-fire model rather than the reference's
 * ten-scalar, sin-hash, fuel-bed model (which has no seeds, no disk emitters
 * and no point light).  mode 0 (the default) keeps the reference's physics
 * bit for bit and ignores every other field.  mode 1 ("config physics"):
 *   - state: heat T, fuel F, soot S (the other seven scalars stay 0); MAC
 *     faces in cells per step; cell (i,j,k) has its centre at (i+.5, j+.5, k+.5);
 *   - advection: semi-Lagrangian, one Euler backtrace of a whole step
 *     (X - velocity(X)), trilinear with clamped indices, faces and scalars;
 *   - reaction: where T > ignitionHeat, burn = F * min(1, burnRate * dt):
 *     F -= burn, T += heatRelease * burn, S += sootYield * burn; then T and S
 *     decay by min(1, cooling * dt) and min(1, sootDecay * dt);
 *   - emitters: the cells of row y = (int)centerY with (x - centerX)^2 +
 *     (z - centerZ)^2 <= radius^2 take F = max(F, fuel * j), T = max(T, heat * j),
 *     j = 1 - jitterScale * U, U uniform in [0,1) from SplitMix64 of (seed,
 *     step, cell); their two v faces are set to upVelocity;
 *   - forces (accelerations, times dt): buoyancy buoyancyHeat * (T -
 *     ambientHeat) - buoyancySoot * S upward; vorticity confinement
 *     vorticityEps * (N x omega) (Fedkiw, Stam and Jensen 2001; h = 1, central
 *     differences with clamped neighbours); noiseAmplitude * curl(psi), psi
 *     three seeded value-noise fields of period noisePeriod cells (cubic
 *     Hermite interpolation, analytic gradient); wind (windX, windZ) on u and w;
 *   - projection: the same divergence, red-black SOR and gradient subtraction
 *     as mode 0 (walls closed, top open, Neumann pressure);
 *   - render: transmittance to a point light at half grid resolution
 *     (lightSamples per ray, clipped to the grid box), then primarySamples per
 *     pixel from a pinhole camera: extinction * S + fuelExtinction * F absorbs,
 *     in-scattering albedo * lightIntensity * transmittance, emission
 *     emission * T with a fixed heat colour; HDR float4 (rgb, 1 - view
 *     transmittance); the BGRA frame is the camera response of FireSettings.
 * Times: dt is this struct's; FireSettings.dt still drives the clocks. */
typedef struct FireEmitterDisk {
    float centerX, centerY, centerZ; /* cell-index coordinates */
    float radius;                    /* cells */
    float fuel, heat;                /* injected amounts before jitter */
    float upVelocity;                /* cells per step, written to the emitter cells' v faces */
    float jitterScale;               /* 0..1 */
    unsigned int seed;
    unsigned int reserved;
} FireEmitterDisk;

#define FIRE_MAX_EMITTERS 4

typedef struct FirePhysicsParams {
    int mode;                        /* 0 reference physics, 1 config physics */
    float dt;                        /* seconds per step */
    float buoyancyHeat, buoyancySoot, ambientHeat;
    float burnRate, ignitionHeat, heatRelease, sootYield; /* 1/s, -, -, - */
    float cooling, sootDecay;        /* 1/s */
    float vorticityEps;
    float windX, windZ;              /* acceleration of u and w, cells/step per second */
    float noiseAmplitude, noisePeriod;
    unsigned int noiseSeed;
    int emitterCount;                /* 0..FIRE_MAX_EMITTERS */
    FireEmitterDisk emitters[FIRE_MAX_EMITTERS];
    int primarySamples, lightSamples;
    float lightX, lightY, lightZ, lightIntensity;
    float extinction, fuelExtinction, emission, albedo;
    float eyeX, eyeY, eyeZ, targetX, targetY, targetZ, fovYDegrees;
    int pressureTop;                 /* 0: Neumann (the reference's); 1: p = 0 above the top row
                                        (needs the multigrid solver, fireCudaSetPressureMultigrid) */
} FirePhysicsParams;

/* Multigrid pressure solve (config physics with pressureTop = 1): up to
 * maxCycles V-cycles per step, each with preSmooth / postSmooth red-black
 * Gauss-Seidel sweeps per level (1..8); with fireCudaSetPressureTolerance
 * set, the level-0 residual is checked after every cycle and the solve stops
 * once max |r| <= tolerance (fireCudaGetPressureStats counts cycles).  Level 0
 * holds the pressure in double, and each solve starts from the previous one's
 * (from zero after a reset or a write of FIRE_FIELD_PRESSURE).
 * maxCycles = 0 restores the red-black SOR. */
FIRE_API bool fireCudaSetPressureMultigrid(int maxCycles, int preSmooth, int postSmooth);

/* The defaults: mode 0; for mode 1 the reference's buoyancy constants (1.62
 * heat, 0.095 soot, src/fire_cuda.cu:1176), no wind, noise or emitters, and a
 * camera on the grid's -z side looking at its centre. */
FIRE_API void fireCudaDefaultPhysicsParams(FirePhysicsParams* params, int nx, int ny, int nz);
/* Validates (sample counts 1..4096, emitterCount 0..4, finite values, dt > 0)
 * and applies from the next pass on.  Switching modes does not clear the fields. */
FIRE_API bool fireCudaSetPhysicsParams(const FirePhysicsParams* params);
FIRE_API bool fireCudaGetPhysicsParams(FirePhysicsParams* params);

/* ---- Independent scenes, batched steps, serving ------------------------
 * No counterpart in the reference, whose scene is one process-wide singleton
 * (src/fire_cuda.cu:116-195).  A FireScene owns its fields, its stream and
 * its output; work queued on different scenes may overlap on the GPU.  The
 * entry points below return false and set fireCudaLastError() like the
 * others; they are meant to be called from one host thread. */
typedef struct FireScene FireScene;

/* Creates a scene on `device` with an nx*ny*nz grid and a frameW*frameH HDR
 * frame, reset as by fireCudaReset.  NULL on failure. */
FIRE_API FireScene* fireSceneCreate(int device, int frameW, int frameH, int nx, int ny, int nz);
/* Waits for the scene's queued work and frees it. */
FIRE_API void fireSceneDestroy(FireScene* scene);
/* Device memory the scene holds, in bytes (for admission against a budget). */
FIRE_API size_t fireSceneDeviceBytes(const FireScene* scene);
FIRE_API bool fireSceneSetPressureSolver(FireScene* scene, int iterations, float omega);
/* As fireCudaSetPressureTolerance / fireCudaSetPhysicsParams, for one scene. */
FIRE_API bool fireSceneSetPressureTolerance(FireScene* scene, double maxResidual, int checkEvery);
FIRE_API bool fireSceneSetPhysicsParams(FireScene* scene, const FirePhysicsParams* params);
FIRE_API bool fireSceneSetPressureMultigrid(FireScene* scene, int maxCycles, int preSmooth, int postSmooth);
/* Caller-owned device HDR buffer the scene renders into (as fireCudaRegisterHdrBufferSlot). */
FIRE_API bool fireSceneSetHdrBuffer(FireScene* scene, void* devicePtr, size_t pitchBytes, int format);
/* Queues one step (render = 0) or one step and a render into the HDR buffer
 * (render != 0) on the scene's stream; returns without waiting. */
FIRE_API bool fireSceneStep(FireScene* scene, const FireSettings* settings, int render);
FIRE_API bool fireSceneSynchronize(FireScene* scene);
FIRE_API bool fireSceneGetStream(FireScene* scene, void** stream);
/* Waits for the scene, then copies one field (FIRE_FIELD_*), as fireCudaGetField. */
FIRE_API bool fireSceneGetField(FireScene* scene, int field, void* host, size_t bytes);
/* As fireCudaGetPressureStats, for one scene (waits for the scene's stream). */
FIRE_API bool fireSceneGetPressureStats(FireScene* scene, int* iterations, float* maxResidual, double* l2Residual);

/* One sub-step of n scenes: queues fireSceneStep(scenes[i], &settings[i],
 * render ? render[i] : 0) for every scene, each on its own stream, so the
 * scenes' kernels run side by side on the GPU. */
FIRE_API bool fireBatchStep(FireScene* const* scenes, const FireSettings* settings, const int* render, int n);

/* A batch of scenes of the config physics stepped as one: per sub-step one
 * upload of the scenes' step descriptors, one launch per stage whose blocks
 * cover every scene, and the pressure solve of every scene in one persistent
 * multigrid launch.  No counterpart in the reference (one process-wide scene).
 * Every scene must use the config physics with p = 0 on the top face
 * (FirePhysicsParams mode 1, pressureTop 1) and the multigrid solve, with the
 * same cycles, smoothing sweeps and tolerance; sizes may differ; at most 128
 * scenes.  Each scene's result is the same bits as stepping it alone.  While
 * a scene belongs to a batch, its own calls (fireSceneGetField, ...) run on
 * the batch's stream; fireBatchDestroy gives each scene its stream back.
 * Destroy the batch before its scenes. */
typedef struct FireBatch FireBatch;
FIRE_API FireBatch* fireBatchCreate(FireScene* const* scenes, int n);
FIRE_API void fireBatchDestroy(FireBatch* batch);
/* One sub-step of every scene: settings[i] for scene i (its reset flag and dt
 * clamp as in fireSceneStep); render[i] != 0 (render may be NULL) also
 * renders scene i's frame into its HDR buffer.  Queued; returns at once. */
FIRE_API bool fireBatchRun(FireBatch* batch, const FireSettings* settings, const int* render);
FIRE_API bool fireBatchSynchronize(FireBatch* batch);
FIRE_API bool fireBatchGetStream(FireBatch* batch, void** stream);
/* Kernels (and the solve's one persistent launch) queued by the batch so far. */
FIRE_API bool fireBatchGetLaunchCount(FireBatch* batch, unsigned long long* count);

/* A serving loop over FireScenes: requests arrive over time, are admitted
 * while the device memory of the admitted scenes stays within a budget, and
 * every admitted scene advances one step per round (continuous batching:
 * a request that arrives while others run joins at the next round, and a
 * finished scene leaves and frees its memory at once). */
typedef struct FireServer FireServer;
typedef struct FireServeRequest {
    int id;
    int nx, ny, nz;             /* grid */
    int frameW, frameH;         /* HDR frame of the scene */
    int steps;                  /* steps to run */
    int renderEvery;            /* render after every renderEvery-th step (0 = never) */
    int sorIterations;          /* 0 = library default */
    float sorOmega;
    double arrivalSeconds;      /* arrival time, from the start of fireServerRun */
    FireSettings settings;      /* per-step settings (reset on the first step) */
    float* resultHeat;          /* optional host buffer (nx*ny*nz floats): final heat */
    float* resultHdr;           /* optional host buffer (frameW*frameH*4 floats): last frame */
    FirePhysicsParams physics;  /* mode 1: the scene's config physics (validated at submit);
                                   mode 0 (e.g. all zero): the reference's physics */
    int multigridCycles;        /* > 0 (config physics with pressureTop 1 only): the pressure is
                                   solved by multigrid V-cycles, at most this many per step */
    int multigridPre, multigridPost;  /* smoothing sweeps per level (0 = 2) */
    double pressureTolerance;   /* > 0: stop the solve once max |r| <= this (checked per cycle) */
} FireServeRequest;
typedef struct FireServeReport {
    int submitted, completed, admittedPeak;
    double seconds;             /* wall time of the run */
    double voxelSteps;          /* sum over completed steps of nx*ny*nz */
    double stepMsP50, stepMsP95, stepMsP99, stepMsMax;     /* per scene step, see fireServerRun */
    double frameMsP50, frameMsP95, frameMsP99;             /* per rendered frame */
    double queueMsP50, queueMsP99;                         /* arrival to admission */
    size_t deviceBytesPeak;
} FireServeReport;

/* A finished scene stays in a pool, by grid and frame shape, for the next
 * request of that shape (its first step resets it), so steady serving neither
 * allocates nor frees device memory; pooled scenes count toward the budget and
 * are freed, oldest first, when an admission needs their room. */
FIRE_API FireServer* fireServerCreate(int device, size_t budgetBytes);
FIRE_API void fireServerDestroy(FireServer* server);
/* Latency control: admit a request only while the admitted scenes hold at
 * most maxActiveVoxels cells (0 = no limit); every round steps all of them,
 * so this bounds the round time and with it the step latency.  Requests
 * beyond it wait in arrival order (their wait is queueMs). */
FIRE_API bool fireServerSetLimits(FireServer* server, long long maxActiveVoxels);
/* Latency control of the batched loop (see fireServerRun): admit a request
 * only while the admitted cells times the measured device time per cell of
 * a round (smoothed over the rounds) stays within roundMs, so a round, and
 * with it every scene's step, takes about roundMs at most.  0 = off. */
FIRE_API bool fireServerSetLatencyTarget(FireServer* server, double roundMs);

/* Adds a request; it is admitted no earlier than its arrivalSeconds. */
FIRE_API bool fireServerSubmit(FireServer* server, const FireServeRequest* request);
/* Runs rounds until every submitted request has completed or `maxSeconds`
 * of wall time have passed.  Step latency is the device time between the
 * completions of a scene's consecutive steps (its first step: from its
 * admission), measured with events; it contains the time the scene shares
 * the GPU with the others.
 *
 * When every submitted request uses the config physics with the multigrid
 * projection (physics.mode 1, pressureTop 1, multigridCycles > 0), each round
 * steps all admitted scenes as one batch (one launch per stage over all of
 * them, as FireBatch), and the scenes are created before the clock starts:
 * per grid shape as many as the active-cell limit lets run at once, within
 * the budget.  The loop then allocates no device memory; a request whose
 * shape has no free scene waits for one.  At most 128 scenes are admitted at
 * once.  Otherwise each admitted scene takes its own steps on its own stream. */
FIRE_API bool fireServerRun(FireServer* server, double maxSeconds, FireServeReport* report);

/* Name of the build and its compute capability target, for diagnostics. */
FIRE_API const char* fireCudaBuildInfo(void);

#ifdef __cplusplus
}
#endif
