// fire_light.cu -- quarter-resolution light volume (sm_100a).
//
//   buildSceneLightKernel      src/fire_cuda.cu:1445-1525 -> lightBuild
//   propagateSceneLightKernel  src/fire_cuda.cu:1527-1565 -> lightPropagate (run twice per frame, :3313-3314)
#include "fire_kernels.h"

namespace firesim {

__global__ void __launch_bounds__(128) lightBuild(float4* __restrict__ sceneLight, float* __restrict__ sceneShadow, ScalarFieldsIn s,
                                                  FrameParams p) {
    const int lx = blockIdx.x * blockDim.x + threadIdx.x;
    const int ly = blockIdx.y;
    const int lz = blockIdx.z;
    if (lx >= p.lnx) {
        return;
    }
    const Grid g{p.nx, p.ny, p.nz};
    const float u = cellCoord(lx, p.lnx);
    const float v = cellCoord(ly, p.lny);
    const float w = cellCoord(lz, p.lnz);
    const float domainFade = volumeDomainFade(u, v, w);
    const Cell10 c = sampleAll(s, g, u, v, w);
    const float cellX = 1.0f / static_cast<float>(p.nx);
    const float cellY = 1.0f / static_cast<float>(p.ny);
    const float cellZ = 1.0f / static_cast<float>(p.nz);
    const float gradHeatX = sampleHeat(s, g, u + cellX, v, w) - sampleHeat(s, g, u - cellX, v, w);
    const float gradHeatY = sampleHeat(s, g, u, v + cellY, w) - sampleHeat(s, g, u, v - cellY, w);
    const float gradHeatZ = sampleHeat(s, g, u, v, w + cellZ) - sampleHeat(s, g, u, v, w - cellZ);
    const float frontGradient =
        sqrtf(gradHeatX * gradHeatX + gradHeatY * gradHeatY + gradHeatZ * gradHeatZ) + c.fuel * c.oxygen * 0.035f + c.progress * 0.16f;
    const float fineNoise = fbm3(u * 34.0f + p.time * 0.45f, v * 42.0f - p.time * 0.82f, w * 34.0f + p.time * 0.22f);
    const float shearNoise = fbm3(u * 12.0f - p.time * 0.38f, v * 11.0f - p.time * 0.62f, w * 13.0f + p.time * 0.20f);
    const float reactionFront = smoothstepf(0.035f, 0.54f, frontGradient + c.pyrolysis * 0.10f);
    const float flameHeightFade = smoothstepf(0.70f, 0.070f, v);
    const float lowerShadowColumn = smoothstepf(0.62f, 0.06f, v);
    const float plumeShadowColumn = smoothstepf(0.12f, 0.88f, v);
    const float sheetGate =
        smoothstepf(0.56f, 0.94f, fineNoise * 0.48f + shearNoise * 0.42f + reactionFront * 0.26f + c.heat * 0.018f) *
        smoothstepf(0.04f, 0.86f, reactionFront) * flameHeightFade;
    const float sheetCore = saturate(sheetGate * (0.42f + c.progress * 0.22f + c.pyrolysis * 0.34f));
    const float tempK = 293.0f + c.heat * 360.0f + c.fuel * 44.0f + c.pyrolysis * 120.0f + c.progress * 70.0f + sheetCore * 1020.0f;
    const float flameEmitter = domainFade * smoothstepf(820.0f, 1880.0f, tempK) *
                               smoothstepf(0.010f, 0.68f, c.fuel + c.pyrolysis * 0.30f + c.heat * 0.040f) *
                               smoothstepf(0.030f, 0.82f, c.oxygen) * reactionFront * sheetGate * (0.24f + sheetCore * 1.42f);
    const float emberEmitter = smoothstepf(0.002f, 0.22f, c.charMass + c.ash * 0.18f) * smoothstepf(0.09f, 0.00f, v) *
                               (0.10f + c.heat * 0.012f + c.pyrolysis * 0.050f);
    const float sootAttenuation = expf(-(c.sootOptics * 0.25f + c.soot * 0.090f + c.ash * 0.035f));
    const float3 flame = mul3(blackbodyColor(tempK), flameEmitter * sootAttenuation * 3.40f);
    const float3 coal = mul3(make_float3(1.0f, 0.22f, 0.040f), emberEmitter * p.reflectionGain * 0.20f);
    const float extinction = saturate(c.sootOptics * (0.26f + plumeShadowColumn * 0.42f) + c.soot * (0.065f + plumeShadowColumn * 0.20f) +
                                      c.ash * 0.050f + c.progress * lowerShadowColumn * 0.020f);
    const int idx = (lz * p.lny + ly) * p.lnx + lx;
    sceneLight[idx] = make_float4(flame.x + coal.x, flame.y + coal.y, flame.z + coal.z, extinction);
    const float verticalDepth = v * (1.0f + plumeShadowColumn * 0.70f);
    const float radialDepth = expf(-((u - 0.50f) * (u - 0.50f) * 5.5f + (w - 0.50f) * (w - 0.50f) * 7.0f));
    const float opticalShadow =
        c.sootOptics * (0.62f + plumeShadowColumn * 1.15f) + c.soot * (0.22f + plumeShadowColumn * 0.46f) + c.ash * 0.072f;
    sceneShadow[idx] = expf(-(opticalShadow * (0.72f + verticalDepth * 0.42f) + radialDepth * opticalShadow * 0.34f + c.progress * 0.035f));
}

__global__ void __launch_bounds__(128) lightPropagate(float4* __restrict__ outLight, const float4* __restrict__ inLight,
                                                      const float* __restrict__ sceneShadow, FrameParams p, float diffusion, float decay) {
    const int lx = blockIdx.x * blockDim.x + threadIdx.x;
    const int ly = blockIdx.y;
    const int lz = blockIdx.z;
    if (lx >= p.lnx) {
        return;
    }
    const int idx = (lz * p.lny + ly) * p.lnx + lx;
    const float4 center = __ldg(inLight + idx);
    float3 neighbor = make_float3(0.0f, 0.0f, 0.0f);
    float weight = 0.0f;
    // Neighbour order -x, +x, -y, +y, -z, +z as in the reference's loop.
    const int nbr[6] = {(lz * p.lny + ly) * p.lnx + max(lx - 1, 0),
                        (lz * p.lny + ly) * p.lnx + min(lx + 1, p.lnx - 1),
                        (lz * p.lny + max(ly - 1, 0)) * p.lnx + lx,
                        (lz * p.lny + min(ly + 1, p.lny - 1)) * p.lnx + lx,
                        (max(lz - 1, 0) * p.lny + ly) * p.lnx + lx,
                        (min(lz + 1, p.lnz - 1) * p.lny + ly) * p.lnx + lx};
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const float4 smp = __ldg(inLight + nbr[i]);
        const float occlusion = expf(-smp.w * 0.42f);
        neighbor = add3(neighbor, mul3(make_float3(smp.x, smp.y, smp.z), occlusion));
        weight += occlusion;
    }
    neighbor = mul3(neighbor, 1.0f / fmaxf(0.0001f, weight));
    const float shadow = __ldg(sceneShadow + idx);
    const float3 direct = make_float3(center.x, center.y, center.z);
    const float3 bounced = lerp3(direct, neighbor, diffusion);
    const float floorLift = smoothstepf(0.10f, 0.00f, cellCoord(ly, p.lny));
    const float3 contactBounce = mul3(make_float3(1.0f, 0.40f, 0.12f), floorLift * luminance3(direct) * 0.18f);
    const float3 next = add3(mul3(bounced, decay * (0.66f + shadow * 0.34f)), contactBounce);
    outLight[idx] = make_float4(next.x, next.y, next.z, center.w);
}

}  // namespace firesim
