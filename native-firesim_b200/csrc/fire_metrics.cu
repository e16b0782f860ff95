// fire_metrics.cu -- per-frame metric reduction (sm_100a).
//
// Restates accumulateMetricsKernel (src/fire_cuda.cu:1319-1418): the same
// per-cell quantities, but instead of 21 FP64 atomicAdds and 9 atomicMaxes per
// cell on one global struct (a contention hot spot whose sums depend on the
// scheduling order), each thread accumulates a grid-strided slice, blocks
// reduce in shared memory in a fixed tree order, and one block reduces the
// block partials in index order -- deterministic and contention-free.
#include "fire_kernels.h"

namespace firesim {

namespace {

__device__ __forceinline__ void maxPositive(int& word, float value) {
    if (value > 0.0f && isfinite(value)) {
        word = max(word, __float_as_int(value));
    }
}

__device__ void reduceBlock(MetricPartial& mine, MetricPartial* shared, MetricPartial* out) {
    // Shared-memory tree reduction in a fixed pairing order.
    const int t = threadIdx.x;
    shared[t] = mine;
    __syncthreads();
    for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
        if (t < stride) {
            MetricPartial& a = shared[t];
            const MetricPartial& b = shared[t + stride];
#pragma unroll
            for (int k = 0; k < 21; ++k) a.sums[k] += b.sums[k];
#pragma unroll
            for (int k = 0; k < 9; ++k) a.maxBits[k] = max(a.maxBits[k], b.maxBits[k]);
            a.invalidCells += b.invalidCells;
        }
        __syncthreads();
    }
    if (t == 0) {
        *out = shared[0];
    }
}

}  // namespace

__global__ void __launch_bounds__(kMetricThreads) metricsPartials(MetricPartial* __restrict__ partials, ScalarFieldsIn s,
                                                                  const float4* __restrict__ sceneLight, const float* __restrict__ sceneShadow,
                                                                  const float* __restrict__ divergenceBefore,
                                                                  const float* __restrict__ divergenceAfter, FrameParams p) {
    extern __shared__ MetricPartial shared[];
    MetricPartial mine;
#pragma unroll
    for (int k = 0; k < 21; ++k) mine.sums[k] = 0.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) mine.maxBits[k] = 0;
    mine.invalidCells = 0;
    const LightGrid L{p.lnx, p.lny, p.lnz};
    const int cells = p.nx * p.ny * p.nz;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < cells; idx += gridDim.x * blockDim.x) {
        const int x = idx % p.nx;
        const int y = (idx / p.nx) % p.ny;
        const int z = idx / (p.nx * p.ny);
        const Cell10 c = loadCell(s, idx);
        const float divBefore = fabsf(__ldg(divergenceBefore + idx));
        const float divAfter = fabsf(__ldg(divergenceAfter + idx));
        const float u = cellCoord(x, p.nx);
        const float v = cellCoord(y, p.ny);
        const float w = cellCoord(z, p.nz);
        const float4 light = sampleSceneLight(sceneLight, L, u, v, w);
        const float shadow = sampleSceneShadow(sceneShadow, L, u, v, w);
        if (!isfinite(c.heat) || !isfinite(c.fuel) || !isfinite(c.oxygen) || !isfinite(c.soot) || !isfinite(c.charMass) ||
            !isfinite(c.ash) || !isfinite(c.pyrolysis) || !isfinite(c.progress) || !isfinite(c.turbulenceEnergy) ||
            !isfinite(c.sootOptics) || !isfinite(divBefore) || !isfinite(divAfter)) {
            mine.invalidCells += 1;
            continue;
        }
        const float tempK = 293.0f + c.heat * 335.0f;
        const float hrr = (c.fuel + c.pyrolysis * 0.42f) * c.oxygen * smoothstepf(610.0f, 1280.0f, tempK) * expf(-5200.0f / fmaxf(650.0f, tempK));
        const float opticalDepth = c.sootOptics + c.soot * (0.24f + 0.05f * sqrtf(fmaxf(0.0f, c.heat)));
        const float normalizedHeight = (static_cast<float>(y) + 0.5f) / static_cast<float>(p.ny);
        const float flameMass = smoothstepf(0.72f, 2.10f, c.heat + c.progress * 0.62f + c.pyrolysis * 0.24f) *
                                smoothstepf(0.035f, 0.66f, c.oxygen) * smoothstepf(0.012f, 0.52f, c.fuel + c.pyrolysis * 0.36f);
        const float smokeMass = smoothstepf(0.035f, 1.16f, c.sootOptics + c.soot * 0.38f + c.ash * 0.12f) *
                                smoothstepf(0.08f, 0.88f, normalizedHeight);
        const float overlap = flameMass * smokeMass;
        const float volumetricShadow = shadow * expf(-light.w * 0.80f);
        const float lightLuma = luminance3(make_float3(light.x, light.y, light.z));
        const float roomIrradiance = lightLuma * volumetricShadow;
        const float flameMarker = c.heat + c.fuel * 0.24f + c.progress * 0.55f;
        const double vals[21] = {c.heat, c.fuel, c.oxygen, c.soot, c.charMass, c.ash, c.pyrolysis, c.progress, c.turbulenceEnergy,
                                 c.sootOptics, lightLuma, shadow, flameMass, smokeMass, overlap, volumetricShadow, roomIrradiance,
                                 opticalDepth, hrr, static_cast<double>(divBefore) * static_cast<double>(divBefore),
                                 static_cast<double>(divAfter) * static_cast<double>(divAfter)};
#pragma unroll
        for (int k = 0; k < 21; ++k) mine.sums[k] += vals[k];
        maxPositive(mine.maxBits[0], c.heat);
        maxPositive(mine.maxBits[1], c.fuel);
        maxPositive(mine.maxBits[2], c.soot);
        maxPositive(mine.maxBits[3], c.pyrolysis);
        maxPositive(mine.maxBits[4], c.progress);
        maxPositive(mine.maxBits[5], c.turbulenceEnergy);
        maxPositive(mine.maxBits[7], divBefore);
        maxPositive(mine.maxBits[8], divAfter);
        if (flameMarker > 0.74f) {
            maxPositive(mine.maxBits[6], normalizedHeight * kRoomHeightMeters);
        }
    }
    reduceBlock(mine, shared, partials + blockIdx.x);
}

__global__ void __launch_bounds__(kMetricThreads) metricsFinal(MetricPartial* __restrict__ out, const MetricPartial* __restrict__ partials,
                                                               int count) {
    extern __shared__ MetricPartial shared[];
    MetricPartial mine;
#pragma unroll
    for (int k = 0; k < 21; ++k) mine.sums[k] = 0.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) mine.maxBits[k] = 0;
    mine.invalidCells = 0;
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
        const MetricPartial& b = partials[i];
#pragma unroll
        for (int k = 0; k < 21; ++k) mine.sums[k] += b.sums[k];
#pragma unroll
        for (int k = 0; k < 9; ++k) mine.maxBits[k] = max(mine.maxBits[k], b.maxBits[k]);
        mine.invalidCells += b.invalidCells;
    }
    reduceBlock(mine, shared, out);
}

}  // namespace firesim
