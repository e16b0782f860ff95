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
    int kx;             // bx / 2: cells of one colour per brick row
    int ex, ey, ez;     // colour-plane extents with the one-cell halo: kx + 2, by + 2, bz + 2
    int nbx, nby, nbz;  // bricks per axis
};
constexpr int kMetricThreads = 128;

// fire_sim.cu
__global__ void fuelBedTables(float* material, float* breathing, FrameParams p, int withMaterial);
__global__ void resetCells(ScalarFields out, float* pressure, float* divergence, float* divergenceAfter, const float* material,
                           const float* breathing, FrameParams p);
__global__ void advectVelocity(float* uOut, float* vOut, float* wOut, Velocity vel, FrameParams p);
__global__ void advectReact(ScalarFields out, ScalarFieldsIn in, Velocity vel, const float* material, const float* breathing, FrameParams p);
__global__ void forceContributions(float4* contrib, ScalarFieldsIn s, Velocity vel, FrameParams p);
__global__ void forceApply(float* uOut, float* vOut, float* wOut, const float4* contrib, Velocity vel, FrameParams p);
__global__ void forceProjectSetup(float* uOut, float* vOut, float* wOut, float* divergence, float* pressure, const float4* contrib,
                                  Velocity vel, FrameParams p);
__global__ void velocityBoundary(float* u, float* v, float* w, FrameParams p, int clampValues);
__global__ void divergenceOf(float* divergence, float* pressureOrNull, Velocity vel, FrameParams p);
__global__ void sorHalfSweep(float* pressure, const float* divergence, Grid g, int parity, float omega);
template <int BX, int BY, int BZ>
__global__ void sorResident(float* pressure, const float* divergence, Grid g, ResidentBrick r, int iterations, float omega);
__global__ void subtractWall(float* u, float* v, float* w, const float* pressure, FrameParams p, int doSubtract, int doWalls);

// fire_light.cu
__global__ void lightBuild(float4* sceneLight, float* sceneShadow, ScalarFieldsIn s, FrameParams p);
__global__ void lightPropagate(float4* outLight, const float4* inLight, const float* sceneShadow, FrameParams p, float diffusion,
                               float decay);

// fire_render.cu
__global__ void raymarch(float4* out, ScalarFieldsIn s, Velocity vel, const float4* lightF, const float* shadowF, FrameParams p);
__global__ void emberSetup(EmberSplat* embers, ScalarFieldsIn s, Velocity vel, FrameParams p);
__global__ void emberGather(float4* hdr, const EmberSplat* embers, FrameParams p);
__global__ void tonemapOverlay(uint32_t* frame, const float4* hdr, FrameParams p, int doTonemap, int doOverlay);
__global__ void packHdr(void* dst, size_t pitchBytes, int halfFormat, const float4* hdr, FrameParams p);

// fire_metrics.cu
__global__ void metricsPartials(MetricPartial* partials, ScalarFieldsIn s, const float4* sceneLight, const float* sceneShadow,
                                const float* divergenceBefore, const float* divergenceAfter, FrameParams p);
__global__ void metricsFinal(MetricPartial* out, const MetricPartial* partials, int count);

}  // namespace firesim
