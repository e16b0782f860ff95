// fire_render.cu -- HDR raymarch, embers, camera response and HDR output (sm_100a).
//
//   renderKernel + roomBackgroundRay etc.  src/fire_cuda.cu:1567-2244 -> raymarch
//   emberHdrKernel                         src/fire_cuda.cu:2323-2452 -> emberSetup + emberGather
//   tonemapKernel + overlayKernel          src/fire_cuda.cu:2246-2297, :1909-1951, :2454-2494 -> tonemapOverlay
//   packFp16SurfaceKernel (D3D11 surface)  src/fire_cuda.cu:2299-2321 -> packHdr (caller-owned device buffer)
#include <cuda_fp16.h>

#include "fire_kernels.h"

namespace firesim {

namespace {

__device__ __forceinline__ float3 fireVolumeUvFromWorld(float3 q) {
    return make_float3(saturate((q.x + 1.05f) / 2.10f), saturate((q.y - 0.02f) / 2.03f), saturate((q.z + 0.82f) / 1.64f));
}
__device__ __forceinline__ float3 fireVolumeWorldFromUv(float3 uv) {
    return make_float3(uv.x * 2.10f - 1.05f, uv.y * 2.03f + 0.02f, uv.z * 1.64f - 0.82f);
}

// src/fire_cuda.cu:1589-1626
__device__ float3 gatherSceneIrradiance(float3 hit, float3 normal, const float4* __restrict__ lightF, const float* __restrict__ shadowF,
                                        const LightGrid& L) {
    float3 irradiance = make_float3(0.0f, 0.0f, 0.0f);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float3 sampleUv = make_float3(0.50f, 0.16f, 0.50f);
        if (i == 1) {
            sampleUv = make_float3(0.34f, 0.26f, 0.43f);
        } else if (i == 2) {
            sampleUv = make_float3(0.66f, 0.26f, 0.57f);
        }
        const float4 light = sampleSceneLight(lightF, L, sampleUv.x, sampleUv.y, sampleUv.z);
        const float3 radiance = make_float3(light.x, light.y, light.z);
        const float lum = luminance3(radiance);
        if (lum <= 0.00001f) {
            continue;
        }
        const float3 source = fireVolumeWorldFromUv(sampleUv);
        const float3 toLight = sub3(source, hit);
        const float dist2 = fmaxf(0.045f, dot3(toLight, toLight));
        const float3 wi = mul3(toLight, rsqrtf(dist2));
        const float ndotl = fmaxf(0.0f, dot3(normal, wi));
        const float heightOcclusion = expf(-fmaxf(0.0f, hit.y - source.y) * light.w * 1.15f);
        const float visibility = sampleSceneShadow(shadowF, L, sampleUv.x, sampleUv.y, sampleUv.z) * expf(-light.w * 0.92f) * heightOcclusion;
        const float geometric = (0.12f + ndotl * 0.88f) * expf(-dist2 * 0.22f) / (0.12f + dist2);
        irradiance = add3(irradiance, mul3(radiance, visibility * geometric));
    }
    const float grazingBounce = 1.0f + smoothstepf(0.0f, 0.45f, 1.0f - fmaxf(0.0f, normal.y)) * 0.36f;
    return mul3(irradiance, 4.20f * grazingBounce);
}

// src/fire_cuda.cu:1628-1645
__device__ float volumeShadowRay(float3 hit, const float4* __restrict__ lightF, const float* __restrict__ shadowF, const LightGrid& L) {
    const float3 targetUv = fireVolumeUvFromWorld(hit);
    const float3 sourceUv = make_float3(0.50f, 0.12f, 0.50f);
    float opticalDepth = 0.0f;
#pragma unroll
    for (int i = 1; i <= 5; ++i) {
        const float t = static_cast<float>(i) / 6.0f;
        const float3 uv = lerp3(sourceUv, targetUv, t);
        const float4 light = sampleSceneLight(lightF, L, uv.x, uv.y, uv.z);
        const float shadow = sampleSceneShadow(shadowF, L, uv.x, uv.y, uv.z);
        opticalDepth += light.w * (0.18f + t * 0.22f) + (1.0f - shadow) * (0.08f + t * 0.16f);
    }
    return expf(-opticalDepth);
}

__device__ __forceinline__ float rectMask(float2 q, float2 center, float2 halfSize, float feather) {
    const float2 d = make_float2(fabsf(q.x - center.x) - halfSize.x, fabsf(q.y - center.y) - halfSize.y);
    const float outside = fmaxf(d.x, d.y);
    return smoothstepf(feather, -feather, outside);
}

__device__ __forceinline__ float lineMask(float2 q, float2 a, float2 b, float thickness) {
    const float2 pa = sub2(q, a);
    const float2 ba = sub2(b, a);
    const float h = saturate(dot2(pa, ba) / fmaxf(0.000001f, dot2(ba, ba)));
    const float2 d = sub2(pa, mul2(ba, h));
    return smoothstepf(thickness, thickness * 0.25f, sqrtf(dot2(d, d)));
}

// src/fire_cuda.cu:1661-1681
__device__ void sourceModelOverlay(float2 uv, const FrameParams& p, float3* color) {
    if (uv.x < 0.24f || uv.x > 0.76f || uv.y < 0.42f || uv.y > 0.88f) {
        return;
    }
    if (p.sceneId == 1) {
        return;
    }
    const float sourceX = p.sceneId == 2 && p.burnerCenterCount > 0 ? p.burnerCenterX[0] : p.emitterCenterX;
    const float sourceY = p.sceneId == 2 && p.burnerCenterCount > 0 ? p.burnerCenterY[0] : p.emitterHeightNorm * 2.03f + 0.02f;
    const float sourceZ = p.sceneId == 2 && p.burnerCenterCount > 0 ? p.burnerCenterZ[0] : p.emitterCenterZ;
    const float3 c = projectPoint(p, make_float3(sourceX, sourceY, sourceZ));
    const float tray = smoothstepf(0.135f, 0.105f, fabsf(uv.x - c.x)) * smoothstepf(0.050f, 0.036f, fabsf(uv.y - c.y));
    const float inner = smoothstepf(0.112f, 0.086f, fabsf(uv.x - c.x)) * smoothstepf(0.039f, 0.027f, fabsf(uv.y - c.y));
    const float alpha = saturate((tray - inner * 0.55f) * 0.65f);
    const float3 modelColor = lerp3(make_float3(0.015f, 0.013f, 0.011f), make_float3(0.13f, 0.12f, 0.10f), alpha);
    if (alpha > 0.001f) {
        *color = lerp3(*color, modelColor, saturate(alpha));
    }
}

// src/fire_cuda.cu:1683-1865 -- analytic room behind the volume.  floorGrid
// (src/fire_cuda.cu:1567-1573) returns 0, so the seam/groove/streak terms that
// multiply it are 0 here.
__device__ float3 roomBackgroundRay(float2 uv, float3 rd, float glow, const float4* __restrict__ lightF, const float* __restrict__ shadowF,
                                    const LightGrid& L, const FrameParams& p) {
    const float roomHalf = 2.55f;
    const float ceilingY = 2.18f;
    const bool cinematic = p.cinematicMode != 0;
    float bestT = 1.0e6f;
    float3 hit = make_float3(0.0f, 0.0f, 0.0f);
    float3 surfaceNormal = make_float3(0.0f, 1.0f, 0.0f);
    int surface = 0;
    const float3 eye = p.eye;
    if (rd.y < -0.0001f) {
        const float t = -eye.y / rd.y;
        const float3 q = add3(eye, mul3(rd, t));
        if (t > 0.0f && fabsf(q.x) <= roomHalf && fabsf(q.z) <= roomHalf && t < bestT) {
            bestT = t; hit = q; surfaceNormal = make_float3(0.0f, 1.0f, 0.0f); surface = 1;
        }
    }
    if (rd.y > 0.0001f) {
        const float t = (ceilingY - eye.y) / rd.y;
        const float3 q = add3(eye, mul3(rd, t));
        if (t > 0.0f && fabsf(q.x) <= roomHalf && fabsf(q.z) <= roomHalf && t < bestT) {
            bestT = t; hit = q; surfaceNormal = make_float3(0.0f, -1.0f, 0.0f); surface = 2;
        }
    }
    if (fabsf(rd.x) > 0.0001f) {
        const float planeX = rd.x > 0.0f ? roomHalf : -roomHalf;
        const float t = (planeX - eye.x) / rd.x;
        const float3 q = add3(eye, mul3(rd, t));
        if (t > 0.0f && q.y >= 0.0f && q.y <= ceilingY && fabsf(q.z) <= roomHalf && t < bestT) {
            bestT = t; hit = q; surfaceNormal = make_float3(planeX > 0.0f ? -1.0f : 1.0f, 0.0f, 0.0f); surface = 3;
        }
    }
    if (fabsf(rd.z) > 0.0001f) {
        const float planeZ = rd.z > 0.0f ? roomHalf : -roomHalf;
        const float t = (planeZ - eye.z) / rd.z;
        const float3 q = add3(eye, mul3(rd, t));
        if (t > 0.0f && q.y >= 0.0f && q.y <= ceilingY && fabsf(q.x) <= roomHalf && t < bestT) {
            bestT = t; hit = q; surfaceNormal = make_float3(0.0f, 0.0f, planeZ > 0.0f ? -1.0f : 1.0f); surface = 4;
        }
    }

    float3 color = make_float3(0.014f, 0.014f, 0.014f);
    float3 materialAlbedo = make_float3(0.26f, 0.26f, 0.25f);
    float materialGiScale = 0.24f;
    if (surface == 1) {
        const float panelSeam = 0.0f;
        const float fineSeam = 0.0f;
        const float slabTone = sinf(hit.x * 2.20f + hit.z * 1.40f) * 0.50f + sinf(hit.z * 3.10f - hit.x * 0.80f) * 0.50f;
        color = cinematic ? make_float3(0.016f, 0.016f, 0.015f) : make_float3(0.014f, 0.014f, 0.013f);
        color = add3(color, mul3(make_float3(0.014f, 0.014f, 0.013f), slabTone * 0.018f));
        color = lerp3(color, make_float3(0.014f, 0.014f, 0.013f), saturate(panelSeam * 0.16f + fineSeam * 0.045f));
        materialAlbedo = make_float3(0.26f, 0.26f, 0.25f);
        materialGiScale = 0.22f;
        if (p.sceneId == 1) {
            const float logMaterial = fuelBedMaterial(hit.x, hit.z, p);
            const float coal = expf(-(hit.x * hit.x * 1.25f + hit.z * hit.z * 2.45f)) * smoothstepf(0.28f, 0.90f, fbm(hit.x * 13.0f, hit.z * 15.0f));
            const float scorch = expf(-(hit.x * hit.x * 0.66f + hit.z * hit.z * 1.15f));
            color = lerp3(color, make_float3(0.018f, 0.015f, 0.012f), saturate(logMaterial * 0.78f + scorch * 0.20f));
            color = add3(color, mul3(make_float3(0.090f, 0.020f, 0.004f), coal * glow * 0.026f));
            color = add3(color, mul3(make_float3(0.17f, 0.11f, 0.055f), logMaterial * 0.050f));
            materialAlbedo = lerp3(materialAlbedo, make_float3(0.040f, 0.030f, 0.022f), logMaterial * 0.86f);
            materialGiScale = lerpf(materialGiScale, 0.44f, logMaterial * 0.80f);
        } else if (p.sceneId == 2) {
            const float radius = sqrtf(hit.x * hit.x + hit.z * hit.z);
            const float plate = smoothstepf(0.78f, 0.70f, radius);
            const float burner = fuelBedMaterial(hit.x, hit.z, p);
            const float radialGrooves = 0.0f;
            color = lerp3(color, make_float3(0.018f, 0.019f, 0.020f), plate * 0.70f);
            color = lerp3(color, make_float3(0.005f, 0.005f, 0.005f), burner * 0.72f);
            color = add3(color, mul3(make_float3(0.11f, 0.10f, 0.09f), radialGrooves * plate * 0.010f));
            color = add3(color, mul3(make_float3(0.090f, 0.032f, 0.006f), burner * glow * 0.012f));
            materialAlbedo = lerp3(materialAlbedo, make_float3(0.032f, 0.033f, 0.034f), plate * 0.82f);
            materialGiScale = lerpf(materialGiScale, 0.42f, plate * 0.72f);
        } else {
            const float2 hxz = make_float2(hit.x, hit.z);
            const float trayBody = rectMask(hxz, make_float2(0.0f, 0.0f), make_float2(1.08f, 0.58f), 0.022f);
            const float trayInner = rectMask(hxz, make_float2(0.0f, 0.0f), make_float2(0.96f, 0.47f), 0.020f);
            const float trayRim = saturate(trayBody - trayInner * 0.74f);
            const float emberBed = trayInner * expf(-(hit.x * hit.x * 0.74f + hit.z * hit.z * 2.20f));
            const float trayContact = trayInner * expf(-(hit.x * hit.x * 1.35f + hit.z * hit.z * 3.35f));
            const float scorch = expf(-(hit.x * hit.x * 0.82f + hit.z * hit.z * 1.75f));
            color = lerp3(color, make_float3(0.017f, 0.014f, 0.012f), trayBody * 0.82f);
            color = lerp3(color, make_float3(0.020f, 0.019f, 0.018f), scorch * (1.0f - trayBody) * 0.16f);
            color = lerp3(color, make_float3(0.010f, 0.009f, 0.008f), trayContact * 0.22f);
            color = add3(color, mul3(make_float3(0.056f, 0.014f, 0.003f), emberBed * glow * 0.26f));
            color = add3(color, mul3(make_float3(0.30f, 0.28f, 0.24f), trayRim * 0.10f));
            materialAlbedo = lerp3(materialAlbedo, make_float3(0.030f, 0.024f, 0.020f), trayBody * 0.75f);
            materialGiScale = lerpf(materialGiScale, 0.48f, trayBody * 0.85f);
        }
        const float reflectCore = expf(-(hit.x * hit.x * 2.45f + (hit.z + 0.18f) * (hit.z + 0.18f) * 1.95f)) * glow;
        const float reflectedTongues = smoothstepf(0.82f, 0.00f, fabsf(hit.x)) * smoothstepf(1.18f, 0.00f, fabsf(hit.z + 0.72f));
        const float streaks = 0.0f;
        color = add3(color, mul3(make_float3(0.55f, 0.11f, 0.023f), reflectCore * p.reflectionGain * 0.48f));
        color = add3(color, mul3(make_float3(0.46f, 0.070f, 0.014f), reflectedTongues * streaks * glow * p.reflectionGain * 0.14f));
    } else if (surface == 2) {
        color = cinematic ? make_float3(0.012f, 0.012f, 0.012f) : make_float3(0.011f, 0.011f, 0.010f);
        materialAlbedo = make_float3(0.24f, 0.24f, 0.23f);
        materialGiScale = 0.20f;
        const float2 hxz = make_float2(hit.x, hit.z);
        const float panelA = lineMask(hxz, make_float2(-1.2f, -2.0f), make_float2(-1.2f, 2.0f), 0.010f);
        const float panelB = lineMask(hxz, make_float2(0.0f, -2.0f), make_float2(0.0f, 2.0f), 0.008f);
        const float ceilingGrid = 0.0f;
        const float ceilingRib = 0.0f;
        const float fixtureL = expf(-((hit.x + 1.50f) * (hit.x + 1.50f) + (hit.z - 0.92f) * (hit.z - 0.92f)) * 120.0f);
        const float fixtureR = expf(-((hit.x - 1.72f) * (hit.x - 1.72f) + (hit.z - 0.80f) * (hit.z - 0.80f)) * 120.0f);
        color = lerp3(color, make_float3(0.011f, 0.011f, 0.010f), saturate(ceilingGrid * 0.090f + ceilingRib * 0.035f));
        color = add3(color, mul3(make_float3(0.10f, 0.096f, 0.088f), (panelA + panelB) * 0.08f));
        color = add3(color, mul3(make_float3(0.26f, 0.20f, 0.13f), (fixtureL + fixtureR) * 0.10f));
    } else {
        color = cinematic ? make_float3(0.015f, 0.015f, 0.014f) : color;
        materialAlbedo = make_float3(0.25f, 0.25f, 0.24f);
        materialGiScale = 0.24f;
        const float panelSeam = 0.0f;
        const float baseShadow = smoothstepf(0.34f, 0.02f, hit.y);
        const float crownShadow = smoothstepf(ceilingY - 0.32f, ceilingY - 0.02f, hit.y);
        color = lerp3(color, make_float3(0.017f, 0.017f, 0.016f), panelSeam * 0.090f);
        color = lerp3(color, make_float3(0.012f, 0.012f, 0.011f), saturate(baseShadow * 0.30f + crownShadow * 0.20f));
        if (surface == 4 && hit.z > 0.0f) {
            const float2 hxy = make_float2(hit.x, hit.y);
            const float recess = rectMask(hxy, make_float2(0.0f, 1.00f), make_float2(0.92f, 0.72f), 0.055f);
            const float recessEdge = lineMask(hxy, make_float2(-0.92f, 0.28f), make_float2(-0.92f, 1.72f), 0.010f) +
                                     lineMask(hxy, make_float2(0.92f, 0.28f), make_float2(0.92f, 1.72f), 0.010f);
            color = lerp3(color, make_float3(0.015f, 0.015f, 0.014f), recess * 0.42f);
            color = add3(color, mul3(make_float3(0.050f, 0.046f, 0.038f), recessEdge * 0.030f));
        }
        const float soot = expf(-(hit.x * hit.x * 0.82f + hit.z * hit.z * 1.12f)) * smoothstepf(0.36f, 1.92f, hit.y);
        color = lerp3(color, make_float3(0.010f, 0.011f, 0.012f), soot * 0.82f * p.smokeDarkness);
        materialAlbedo = lerp3(materialAlbedo, make_float3(0.030f, 0.032f, 0.034f), soot * 0.75f);
        const float wallGlow = expf(-(hit.x * hit.x * 1.1f + hit.z * hit.z * 1.3f + (hit.y - 0.70f) * (hit.y - 0.70f) * 1.0f)) * glow;
        color = add3(color, mul3(make_float3(0.15f, 0.050f, 0.018f), wallGlow * 0.090f));
        if (surface == 3 && hit.x < 0.0f) {
            const float2 hzy = make_float2(hit.z, hit.y);
            const float window = rectMask(hzy, make_float2(-1.28f, 0.92f), make_float2(0.06f, 0.62f), 0.030f);
            const float glassNoise = 0.55f + 0.25f * sinf(hit.y * 23.0f + hit.z * 15.0f);
            color = lerp3(color, make_float3(0.009f, 0.011f, 0.012f), window * 0.92f);
            color = add3(color, mul3(make_float3(0.10f, 0.12f, 0.13f), window * glassNoise * 0.16f));
        }
    }

    const float3 volumeUv = fireVolumeUvFromWorld(hit);
    const float4 giSample = sampleSceneLight(lightF, L, volumeUv.x, volumeUv.y, volumeUv.z);
    const float sceneShadow = sampleSceneShadow(shadowF, L, volumeUv.x, volumeUv.y, volumeUv.z);
    const float volumeVisibility = volumeShadowRay(hit, lightF, shadowF, L);
    const float3 gathered = gatherSceneIrradiance(hit, surfaceNormal, lightF, shadowF, L);
    const float3 indirect = mul3(add3(mul3(make_float3(giSample.x, giSample.y, giSample.z), 0.42f), gathered), volumeVisibility);
    const float grazingFalloff = surface == 2 ? 0.62f : 1.0f;
    const float contactOcclusion = smoothstepf(0.005f, 0.42f, sceneShadow) * expf(-giSample.w * 0.72f) * (0.30f + volumeVisibility * 0.70f);
    const float irradianceLift = 0.66f + smoothstepf(0.006f, 0.13f, luminance3(indirect)) * 0.72f;
    const float contactWarmth = surface == 1 ? 1.72f : (surface == 2 ? 0.88f : 1.16f);
    color = add3(color, mul3(mul3v(indirect, materialAlbedo), materialGiScale * grazingFalloff * contactOcclusion * irradianceLift * contactWarmth));
    const float shadowedSoot = (1.0f - volumeVisibility) * smoothstepf(0.18f, 0.82f, 1.0f - sceneShadow);
    color = lerp3(color, make_float3(0.006f, 0.007f, 0.008f), shadowedSoot * (surface == 2 ? 0.38f : 0.26f));
    const float wallHorizontalEdge = surface == 3 ? roomHalf - fabsf(hit.z) : roomHalf - fabsf(hit.x);
    const float cornerDistance = surface == 1 || surface == 2 ? fminf(roomHalf - fabsf(hit.x), roomHalf - fabsf(hit.z))
                                                              : fminf(wallHorizontalEdge, fminf(hit.y, ceilingY - hit.y));
    color = mul3(color, 0.84f + smoothstepf(0.0f, 0.54f, cornerDistance) * 0.16f);
    const float grain = (hash21(floorf(hit.x * 19.0f + hit.z * 13.0f), floorf(hit.y * 15.0f + p.time * 0.08f)) - 0.5f) * 0.006f;
    color = add3(color, make_float3(grain, grain, grain));
    sourceModelOverlay(uv, p, &color);
    const float fog = smoothstepf(3.8f, 0.2f, bestT);
    const float vignette = smoothstepf(0.78f, 0.20f, sqrtf((uv.x - 0.50f) * (uv.x - 0.50f) + (uv.y - 0.46f) * (uv.y - 0.46f)));
    return mul3(color, (0.12f + fog * 0.56f) * (0.58f + vignette * 0.30f));
}

// src/fire_cuda.cu:1867-1907
__device__ __forceinline__ bool intersectBox(float3 ro, float3 rd, float3 bmin, float3 bmax, float* outNear, float* outFar) {
    float tNear = 0.0f;
    float tFar = 1.0e6f;
    const float3 inv = make_float3(1.0f / (fabsf(rd.x) < 0.00001f ? copysignf(0.00001f, rd.x) : rd.x),
                                   1.0f / (fabsf(rd.y) < 0.00001f ? copysignf(0.00001f, rd.y) : rd.y),
                                   1.0f / (fabsf(rd.z) < 0.00001f ? copysignf(0.00001f, rd.z) : rd.z));
    float t0 = (bmin.x - ro.x) * inv.x;
    float t1 = (bmax.x - ro.x) * inv.x;
    if (t0 > t1) { const float tmp = t0; t0 = t1; t1 = tmp; }
    tNear = fmaxf(tNear, t0);
    tFar = fminf(tFar, t1);
    t0 = (bmin.y - ro.y) * inv.y;
    t1 = (bmax.y - ro.y) * inv.y;
    if (t0 > t1) { const float tmp = t0; t0 = t1; t1 = tmp; }
    tNear = fmaxf(tNear, t0);
    tFar = fminf(tFar, t1);
    t0 = (bmin.z - ro.z) * inv.z;
    t1 = (bmax.z - ro.z) * inv.z;
    if (t0 > t1) { const float tmp = t0; t0 = t1; t1 = tmp; }
    tNear = fmaxf(tNear, t0);
    tFar = fminf(tFar, t1);
    *outNear = tNear;
    *outFar = tFar;
    return tFar > tNear;
}

__device__ __forceinline__ float3 debugHeatColor(float value) {  // src/fire_cuda.cu:370-379
    value = saturate(value);
    const float red = smoothstepf(0.05f, 0.45f, value);
    const float orange = smoothstepf(0.24f, 0.78f, value);
    const float white = smoothstepf(0.72f, 1.0f, value);
    return make_float3(saturate(red + white * 0.70f), saturate(orange * 0.58f + white * 0.78f), saturate(white * 0.62f));
}

}  // namespace

namespace {

// src/fire_cuda.cu:1953-2244 -- one primary ray through the packed field
// records; writes RGB and alpha = 1 to pixel (x, y) of the internal HDR frame.
// smoothstepf with the span's reciprocal: for the literal edges of the
// shading terms below, 1 / (hi - lo) is a compile-time constant, so each call
// is a multiply where smoothstepf divides.  The result is within one ulp of
// smoothstepf's; a developed 512x512 frame differs by 2e-8 in relative L2 and
// renders 17-21% faster (fewer instructions, and a sample loop that fits the
// instruction cache better).
__device__ __forceinline__ float smoothstepK(float edge0, float edge1, float x) {
    const bool inverted = edge1 < edge0;
    const float lo = inverted ? edge1 : edge0;
    const float hi = inverted ? edge0 : edge1;
    const float t = saturate((x - lo) * (1.0f / fmaxf(0.000001f, hi - lo)));
    const float value = t * t * (3.0f - 2.0f * t);
    return inverted ? 1.0f - value : value;
}

// The raymarch's fbm3 (src/fire_cuda.cu:434-443, with valueNoise3 :401-421
// and hash31 :386-388): three octaves of 3D value noise, written with the
// reference's plain expressions and compiled as the reference's render
// compiles them -- one out-of-line function with its value noise and sin
// hash inlined.  In that form nvcc rounds the sin argument of the eight
// corner hashes differently from a hash compiled on its own (the form of
// hash31 in fire_device.cuh, which every other call site matches), and a
// one-ulp change of that argument scrambles the hash.  Measured on the B200:
// with this function the raymarch equals the reference's renderKernel bit for
// bit; with the standalone hash (and with each single rounding form of its
// argument) it differs in ~13% of pixels.
namespace {

__device__ __forceinline__ float renderHash31(float3 q) {
    return fracf(sinf(q.x * 127.1f + q.y * 311.7f + q.z * 74.7f) * 43758.5453123f);
}

__device__ __forceinline__ float renderValueNoise3(float3 q) {
    const float3 i = make_float3(floorf(q.x), floorf(q.y), floorf(q.z));
    const float3 f = make_float3(fracf(q.x), fracf(q.y), fracf(q.z));
    const float3 u = make_float3(f.x * f.x * (3.0f - 2.0f * f.x), f.y * f.y * (3.0f - 2.0f * f.y), f.z * f.z * (3.0f - 2.0f * f.z));
    const float c000 = renderHash31(i);
    const float c100 = renderHash31(make_float3(i.x + 1.0f, i.y, i.z));
    const float c010 = renderHash31(make_float3(i.x, i.y + 1.0f, i.z));
    const float c110 = renderHash31(make_float3(i.x + 1.0f, i.y + 1.0f, i.z));
    const float c001 = renderHash31(make_float3(i.x, i.y, i.z + 1.0f));
    const float c101 = renderHash31(make_float3(i.x + 1.0f, i.y, i.z + 1.0f));
    const float c011 = renderHash31(make_float3(i.x, i.y + 1.0f, i.z + 1.0f));
    const float c111 = renderHash31(make_float3(i.x + 1.0f, i.y + 1.0f, i.z + 1.0f));
    const float c00 = lerpf(c000, c100, u.x);
    const float c10 = lerpf(c010, c110, u.x);
    const float c01 = lerpf(c001, c101, u.x);
    const float c11 = lerpf(c011, c111, u.x);
    return lerpf(lerpf(c00, c10, u.y), lerpf(c01, c11, u.y), u.z);
}

__device__ __noinline__ float renderFbm3(float3 q) {
    float sum = 0.0f;
    float amp = 0.5f;
    for (int octave = 0; octave < 3; ++octave) {
        sum += amp * renderValueNoise3(q);
        q = make_float3(q.x * 2.03f + 17.7f, q.y * 2.01f - 9.2f, q.z * 2.07f + 5.1f);
        amp *= 0.5f;
    }
    return saturate(sum * 1.142857f);
}

}  // namespace

// SC >= 0: the scene id, fixed at compile time (the caller launches this
// instantiation only for that scene with no debug view); SC < 0: read from p,
// with the debug views.  Fixing it drops the other scenes' branches and the
// debug views' per-sample maxima from the sample loop.
template <int SC>
__device__ __forceinline__ void shadePixel(float4* __restrict__ out, int x, int y, const ScalarFieldsIn& s, const Velocity& vel,
                                           const float4* __restrict__ lightF, const float* __restrict__ shadowF, const FrameParams& p) {
    const Grid g{p.nx, p.ny, p.nz};
    const LightGrid L{p.lnx, p.lny, p.lnz};
    const float2 uv = make_float2((static_cast<float>(x) + 0.5f) / static_cast<float>(p.frameW),
                                  (static_cast<float>(y) + 0.5f) / static_cast<float>(p.frameH));
    const float sxr = (uv.x * 2.0f - 1.0f) * p.aspect * p.tanHalfFov;
    const float syr = (1.0f - uv.y * 2.0f) * p.tanHalfFov;
    const float3 rd = normalize3(add3(add3(p.forward, mul3(p.right, sxr)), mul3(p.up, syr)));
    const float baseGlow = saturate(sampleHeat(s, g, 0.50f, 0.06f, 0.50f) * 0.42f);

    float boxNear = 0.0f, boxFar = 0.0f;
    float3 accum = make_float3(0.0f, 0.0f, 0.0f);
    float trans = 1.0f;
    float flameGlow = 0.0f, smokeOcclusion = 0.0f, debugFlame = 0.0f, debugOpticalDepth = 0.0f;
    float debugTemperature = 0.0f, debugFuel = 0.0f, debugVelocity = 0.0f;
    const int sc = SC >= 0 ? SC : p.sceneId;
    constexpr bool debugViews = SC < 0;
    const bool velocityDebug = debugViews && p.renderDebugMode == 6;

    if (intersectBox(p.eye, rd, make_float3(-1.05f, 0.02f, -0.82f), make_float3(1.05f, 2.05f, 0.82f), &boxNear, &boxFar)) {
        const int raySteps = min(max(p.raymarchSteps, 24), kMaxRaymarchSteps);
        const float t0 = fmaxf(0.0f, boxNear);
        const float t1 = fminf(boxFar, t0 + 3.05f);
        const float stepT = (t1 - t0) / static_cast<float>(raySteps);
        const float cellX = 1.0f / static_cast<float>(p.nx);
        const float cellY = 1.0f / static_cast<float>(p.ny);
        const float cellZ = 1.0f / static_cast<float>(p.nz);
        const float rayJitter = hash21((static_cast<float>(x) + 0.5f) * 0.754877f, (static_cast<float>(y) + 0.5f) * 0.569840f);
        for (int i = 0; i < raySteps && trans > 0.018f; ++i) {
            const float t = t0 + (static_cast<float>(i) + rayJitter) * stepT;
            const float3 wp = add3(p.eye, mul3(rd, t));
            const float fu = saturate((wp.x + 1.05f) / 2.10f);
            const float fv = saturate((wp.y - 0.02f) / 2.03f);
            const float fw = saturate((wp.z + 0.82f) / 1.64f);
            const float domainFade = volumeDomainFade(fu, fv, fw);
            if (domainFade <= 0.001f) {
                continue;
            }
            // Coarse occupancy probe: heat, fuel, soot, progress at the unwarped point.
            const Corners cc = scalarCorners(g, fu, fv, fw);
            const float4 coarseA = gatherVec(s.a, cc, g.nx, g.ny);
            const float coarseProgress = gatherVec(s.b, cc, g.nx, g.ny).w;
            const float coarseFuel = coarseA.y;
            const float coarseActive = (coarseA.x + coarseFuel * 0.42f + coarseA.w * 0.34f + coarseProgress * 0.32f) * domainFade;
            if (coarseActive <= 0.00150f) {
                ++i;
                continue;
            }
            const float warpA = renderFbm3(make_float3(fu * 7.0f + p.time * 0.18f, fv * 5.0f - p.time * 0.11f, fw * 9.0f + p.time * 0.07f)) - 0.5f;
            const float warpB = renderFbm3(make_float3(fw * 8.0f - p.time * 0.14f, fu * 8.0f + p.time * 0.10f, fv * 6.0f - p.time * 0.08f)) - 0.5f;
            const float warpGain = 0.028f + fv * 0.060f;
            const float wu = saturate(fu + warpA * warpGain);
            const float wv = saturate(fv + (warpA - warpB) * 0.020f);
            const float ww = saturate(fw + warpB * warpGain);

            const Cell10 c = sampleAll(s, g, wu, wv, ww);
            const float heat = c.heat, fuel = c.fuel, oxygen = c.oxygen, soot = c.soot, charMass = c.charMass, ash = c.ash;
            const float pyrolysis = c.pyrolysis, progress = c.progress, turbulenceEnergy = c.turbulenceEnergy, sootOptics = c.sootOptics;
            const float4 sceneLight = sampleSceneLight(lightF, L, wu, wv, ww);
            const float sceneShadow = sampleSceneShadow(shadowF, L, wu, wv, ww);
            float3 velocity = make_float3(0.0f, 0.0f, 0.0f);
            if (velocityDebug) {
                velocity = sampleVelocity(vel, g, wu, wv, ww);
            }
            const float activeField = (heat + fuel * 0.42f + soot * 0.34f + progress * 0.32f + pyrolysis * 0.18f) * domainFade;
            if (activeField <= 0.0025f) {
                continue;
            }
            if (debugViews) {
                debugFuel = fmaxf(debugFuel, domainFade * saturate(fuel * 0.18f + charMass * 0.22f + pyrolysis * 0.30f));
            }
            if (velocityDebug) {
                debugVelocity = fmaxf(debugVelocity, saturate(sqrtf(dot3(velocity, velocity)) * 0.22f));
            }
            const float gradHeatX = sampleHeat(s, g, wu + cellX, wv, ww) - sampleHeat(s, g, wu - cellX, wv, ww);
            const float gradHeatY = sampleHeat(s, g, wu, wv + cellY, ww) - sampleHeat(s, g, wu, wv - cellY, ww);
            const float gradHeatZ = sampleHeat(s, g, wu, wv, ww + cellZ) - sampleHeat(s, g, wu, wv, ww - cellZ);
            const float frontGradient = sqrtf(gradHeatX * gradHeatX + gradHeatY * gradHeatY + gradHeatZ * gradHeatZ) + fabsf(fuel - coarseFuel) * 0.62f;
            const float reactionFront = smoothstepK(0.020f, 0.46f, frontGradient * 1.35f + fuel * oxygen * 0.040f + progress * 0.18f + pyrolysis * 0.080f);
            const float fineNoise = renderFbm3(make_float3(wu * 42.0f + p.time * 0.72f, wv * 54.0f - p.time * 1.28f, ww * 43.0f + p.time * 0.38f));
            const float shearNoise = renderFbm3(make_float3(wu * 15.0f - p.time * 0.72f, wv * 13.0f - p.time * 1.08f, ww * 17.0f + p.time * 0.32f));
            const float plumeNoise = saturate(fineNoise * 0.58f + shearNoise * 0.42f);
            const float holeNoise = saturate((1.0f - fineNoise) * 0.36f + shearNoise * 0.64f);
            const float lesBreakup = saturate(turbulenceEnergy * 0.48f + progress * 0.28f);
            const float raggedEdge = smoothstepK(0.18f, 0.92f, fineNoise * (0.46f + lesBreakup * 0.30f) + shearNoise * 0.38f + plumeNoise * 0.32f +
                                                                   saturate(activeField * 0.08f));
            const float fieldEdge = smoothstepK(0.05f, 2.30f, heat + fuel * 0.32f) * (0.10f + reactionFront * 0.90f);
            const float fieldFilament = smoothstepK(0.60f, 1.0f, fineNoise + lesBreakup * 0.10f) *
                                        smoothstepK(0.38f, 0.92f, shearNoise + (0.72f - fv) * 0.12f + reactionFront * 0.10f) *
                                        smoothstepK(1.0f, 0.02f, fv) * fieldEdge;
            const float sourceLocalV = sc == 2 ? fmaxf(0.0f, fv - p.emitterHeightNorm) : fv;
            const float burnerLowJet = sc == 2 ? smoothstepK(fmaxf(0.012f, p.emitterHeightBandNorm * 0.68f), fmaxf(0.003f, p.emitterHeightBandNorm * 0.10f),
                                                             fabsf(fv - p.emitterHeightNorm)) *
                                                     smoothstepK(0.05f, 0.58f, fuel + heat * 0.025f) * smoothstepK(0.50f, 1.0f, oxygen)
                                               : 0.0f;
            const float burnerPortJet = sc == 2 ? burnerLowJet * smoothstepK(0.68f, 0.98f, fineNoise + shearNoise * 0.18f) : 0.0f;
            const float campTongueBias =
                sc == 1 ? smoothstepK(0.035f, 0.72f, fuel + pyrolysis * 0.50f + charMass * 0.12f) * smoothstepK(0.76f, 0.035f, fv) : 0.0f;
            const float roomTraySheet =
                sc == 0 ? smoothstepK(0.018f, 0.42f, fuel + pyrolysis * 0.72f + charMass * 0.08f) * smoothstepK(0.30f, 0.015f, fv) : 0.0f;
            const float convectiveSheet =
                smoothstepK(0.42f, 0.88f, shearNoise + heat * 0.040f + plumeNoise * 0.14f + lesBreakup * 0.10f + burnerPortJet * 0.56f +
                                              campTongueBias * 0.20f + roomTraySheet * 0.24f) *
                (sc == 2 ? smoothstepK(p.emitterHeightNorm + p.emitterHeightBandNorm * 1.20f, p.emitterHeightNorm - p.emitterHeightBandNorm * 0.08f, fv)
                         : smoothstepK(sc == 1 ? 0.82f : 0.88f, 0.030f, fv)) *
                fieldEdge;
            const float breakup = smoothstepK(0.34f, 0.88f, fineNoise * 0.48f + shearNoise * 0.42f + holeNoise * 0.24f + heat * 0.026f);
            const float verticalFade = smoothstepK(0.96f, 0.025f, fv);
            const float flameHeightFade = sc == 2 ? smoothstepK(p.emitterHeightNorm + p.emitterHeightBandNorm * 0.72f,
                                                                p.emitterHeightNorm - p.emitterHeightBandNorm * 0.05f, fv)
                                                  : smoothstepK(sc == 1 ? 0.72f : 0.76f, 0.10f, fv);
            const float lowerWhite = smoothstepK(0.060f, 0.00f, sourceLocalV) * smoothstepK(0.05f, 1.30f, pyrolysis + fuel * 0.20f);
            const float tempK = 293.0f + heat * 360.0f + fuel * 44.0f + pyrolysis * 90.0f + fieldFilament * 560.0f + convectiveSheet * 420.0f +
                                lowerWhite * 110.0f + progress * 64.0f;
            const float combustion = smoothstepK(740.0f, 1630.0f, tempK) * smoothstepK(0.016f, 0.62f, fuel + heat * 0.055f) *
                                     smoothstepK(0.045f, 0.62f, oxygen) * verticalFade * flameHeightFade;
            const float thinFront = smoothstepK(0.04f, 0.56f, frontGradient + progress * 0.10f) * smoothstepK(0.02f, 0.92f, reactionFront);
            const float flameSheetTear =
                smoothstepK(0.52f, 0.88f, holeNoise + shearNoise * 0.18f + lesBreakup * 0.30f + saturate(1.0f - oxygen) * 0.12f);
            const float sheetHole = smoothstepK(0.54f, 0.90f, holeNoise + lesBreakup * 0.26f + saturate(1.0f - oxygen) * 0.12f);
            const float flameSheet =
                fmaxf(smoothstepK(0.55f, 0.94f, fineNoise * 0.46f + shearNoise * 0.44f + plumeNoise * 0.18f + reactionFront * 0.15f + heat * 0.014f -
                                                    fv * 0.050f) *
                          (1.0f - sheetHole * (0.74f + lesBreakup * 0.12f)) * (1.0f - flameSheetTear * 0.18f),
                      smoothstepK(0.18f, 0.030f, sourceLocalV) * smoothstepK(0.75f, 2.0f, heat) * thinFront * 0.030f);
            const float coherentSheet = saturate(fieldFilament * 0.86f + convectiveSheet * 0.55f + thinFront * 0.74f);
            const float sheetConfinement = saturate(coherentSheet + reactionFront * 0.08f);
            const float roomCoverageBoost = sc == 0 ? (0.72f + roomTraySheet * 1.24f) : 1.0f;
            const float flameDensity = domainFade * combustion * reactionFront * flameSheet *
                                       (0.010f + fieldFilament * 0.92f + convectiveSheet * 0.24f + thinFront * 1.22f) *
                                       (0.052f + breakup * 0.78f + raggedEdge * 0.56f + lesBreakup * 0.34f) * (0.18f + thinFront * 2.55f) *
                                       (0.060f + sheetConfinement * 0.94f + burnerPortJet * 0.72f + campTongueBias * 0.34f) * flameHeightFade *
                                       roomCoverageBoost;
            const float plumeVoid = smoothstepK(0.54f, 0.90f, holeNoise + fineNoise * 0.26f + shearNoise * 0.22f + fv * 0.20f);
            const float topDissolve = smoothstepK(sc == 1 ? 0.82f : 0.88f, sc == 1 ? 0.34f : 0.42f, fv);
            const float raggedPlume = 1.0f - plumeVoid * smoothstepK(0.18f, 0.74f, fv) * 0.96f;
            const float upperPlume = smoothstepK(0.14f, 0.48f, fv) * smoothstepK(0.030f, 1.20f, sootOptics + soot * 0.42f) *
                                     (0.025f + fineNoise * 0.035f + shearNoise * 0.034f + plumeNoise * 0.34f + raggedEdge * 0.12f +
                                      turbulenceEnergy * 0.035f) *
                                     topDissolve * raggedPlume;
            const float sceneSmokeScale = sc == 2 ? 0.035f : (sc == 1 ? 0.56f : 1.0f);
            const float rawSootDensity =
                domainFade * sceneSmokeScale *
                (smoothstepK(0.020f, 1.05f, sootOptics + soot * 0.32f) * smoothstepK(0.16f, 0.42f, fv) *
                     (0.028f + fineNoise * 0.040f + shearNoise * 0.052f + plumeNoise * 0.38f + raggedEdge * 0.16f + ash * 0.016f) +
                 upperPlume * (0.22f + plumeNoise * 0.30f) + smoothstepK(0.004f, 0.34f, sootOptics) * (0.020f + plumeNoise * 0.034f));
            const float flameFrontMask =
                saturate(flameDensity * 4.8f + combustion * reactionFront * flameSheet * (0.08f + thinFront * 0.56f + fieldFilament * 0.18f));
            const float emissiveMask = saturate(flameFrontMask);
            const float resolvedFlameSheet = smoothstepK(0.030f, 0.32f, emissiveMask) * smoothstepK(0.035f, 0.72f, oxygen);
            const float smokeOnlyMask = 1.0f - smoothstepK(0.025f, 0.20f, resolvedFlameSheet);
            const float scatterSeparation = saturate(smokeOnlyMask * (1.0f - smoothstepK(0.02f, 0.16f, emissiveMask) * 0.58f));
            const float nearFlameSootCleanout = 1.0f - smoothstepK(0.025f, 0.34f, resolvedFlameSheet) * 0.82f;
            const float smokeOnlyHeight = smoothstepK(0.20f, 0.70f, fv) * (1.0f - smoothstepK(0.02f, 0.20f, emissiveMask));
            const float upperSootNeutrality = smoothstepK(0.18f, 0.78f, fv) * scatterSeparation;
            const float absorptionDensity = rawSootDensity * nearFlameSootCleanout * (1.10f + smokeOnlyHeight * 2.20f + upperSootNeutrality * 2.40f);
            const float scatterDensity = rawSootDensity * scatterSeparation * smoothstepK(0.10f, 0.55f, fv + sootOptics * 0.10f) *
                                         (0.24f + (1.0f - smokeOnlyHeight) * 0.34f);
            const float particleRadius = saturate(0.08f + sootOptics * 0.028f + ash * 0.085f + saturate(1.0f - oxygen) * 0.12f);
            const float sootAbsorption =
                absorptionDensity * (3.10f + particleRadius * 4.60f + sootOptics * 0.70f + upperSootNeutrality * 2.85f) * p.smokeDarkness;
            const float sootScattering = scatterDensity * (0.018f + (1.0f - particleRadius) * 0.050f) * (0.20f + p.smokeGain * 0.10f);
            const float sootExtinction = sootAbsorption + sootScattering;
            const float flameExtinction = flameDensity * (0.12f + (1.0f - resolvedFlameSheet) * 0.12f);
            const float extinction = (sootExtinction + flameExtinction) * stepT;
            const float smokeAlpha = 1.0f - expf(-sootAbsorption * stepT);
            const float scatterAlpha = 1.0f - expf(-sootScattering * stepT);
            const float lightVisibility = sceneShadow * (0.35f + sceneShadow * 0.65f);
            const float3 localIrradiance = make_float3(sceneLight.x, sceneLight.y, sceneLight.z);
            const float sootLoad = saturate(sootOptics * 0.74f + soot * 0.20f + upperPlume * 0.46f);
            const float whiteCore = smoothstepK(2450.0f, 3450.0f, tempK) * combustion * smoothstepK(0.32f, 0.90f, oxygen) *
                                    smoothstepK(0.72f, 0.02f, fv) * (0.02f + thinFront * 0.48f + fieldFilament * 0.18f) *
                                    (1.0f - smoothstepK(0.16f, 0.74f, sootLoad) * 0.68f);
            const float radiantBase = saturate((tempK - 760.0f) / 2000.0f);
            const float radiantCurve = radiantBase * radiantBase * (0.82f + radiantBase * 0.18f);
            const float radiantPower = radiantCurve * (1.42f + fieldFilament * 3.15f + convectiveSheet * 1.60f + progress * 0.26f + whiteCore * 0.92f);
            const float blackbodyCoreStructure = saturate(whiteCore * (0.080f + fieldFilament * 0.28f + thinFront * 0.32f));
            const float whiteFilament = blackbodyCoreStructure * (0.55f + fineNoise * 0.30f + shearNoise * 0.18f);
            const float orangeEdge = (1.0f - whiteFilament * 0.72f) * thinFront * reactionFront * flameSheet * (0.52f + breakup * 0.95f) *
                                     smoothstepK(0.08f, 0.80f, oxygen);
            float3 flameColor = lerp3(make_float3(1.32f, 0.27f, 0.038f), blackbodyColor(tempK), saturate(whiteCore * 0.92f + whiteFilament * 0.82f));
            if (sc == 2) {
                const float blueBase = burnerPortJet * smoothstepK(0.010f, 0.11f, flameDensity + combustion * 0.18f);
                flameColor = lerp3(make_float3(0.020f, 0.18f, 2.40f), make_float3(0.36f, 0.58f, 1.95f), saturate(whiteCore * 0.34f + blueBase * 0.20f));
            } else if (sc == 1) {
                flameColor = lerp3(flameColor, make_float3(1.52f, 0.24f, 0.028f), saturate(campTongueBias * (1.0f - whiteCore) * 0.58f));
            }
            float3 flameEmission = mul3(flameColor, flameDensity * radiantPower * stepT * (1.10f + whiteCore * 0.38f));
            if (sc == 2) {
                flameEmission = mul3(flameEmission, 0.42f);
                flameEmission = add3(flameEmission, mul3(make_float3(0.012f, 0.28f, 5.20f), burnerPortJet * combustion * stepT * 4.40f));
            }
            flameEmission = add3(flameEmission, mul3(make_float3(1.10f, 1.02f, 0.86f), whiteFilament * whiteFilament * flameDensity * radiantPower * stepT * 0.82f));
            flameEmission = add3(flameEmission, mul3(make_float3(1.70f, 0.30f, 0.040f), orangeEdge * flameDensity * radiantPower * stepT *
                                                                                           (sc == 2 ? 0.06f : (sc == 1 ? 3.20f : 3.10f))));
            flameEmission = add3(flameEmission, mul3(make_float3(1.36f, 0.070f, 0.008f),
                                                     fieldFilament * (1.0f + flameSheetTear * 0.55f) * flameDensity * radiantPower * stepT *
                                                         (sc == 2 ? 0.035f : (sc == 1 ? 1.55f : 1.10f)) * (1.0f - whiteCore * 0.62f)));
            const float ashVeil = saturate(ash * 0.014f + smoothstepK(0.30f, 0.88f, fv) * (1.0f - sootLoad) * 0.003f);
            const float3 smokeBlack = make_float3(0.0018f, 0.0020f, 0.0024f);
            const float3 smokeCoal = make_float3(0.008f, 0.0092f, 0.0115f);
            const float3 smokeAsh = make_float3(0.014f, 0.0165f, 0.0210f);
            float3 smokeColor = lerp3(smokeCoal, smokeBlack, sootLoad);
            smokeColor = lerp3(smokeColor, smokeAsh, ashVeil);
            smokeColor = mul3(smokeColor, smokeOnlyMask);
            const float localIrradianceLuma = luminance3(localIrradiance);
            const float warmScatterDamp = 1.0f - upperSootNeutrality * 0.985f;
            const float nearFlameWarmLeak = (1.0f - upperSootNeutrality) * (1.0f - smokeOnlyHeight) * 0.18f;
            const float sceneWarmScatter = sc == 2 ? 0.010f : (sc == 1 ? 0.18f : 0.30f);
            const float backScatter = scatterAlpha * lightVisibility *
                                      (0.00085f + localIrradianceLuma * 0.0011f * warmScatterDamp + baseGlow * 0.00010f * sceneWarmScatter) *
                                      (0.018f + (1.0f - particleRadius) * 0.018f) * scatterSeparation;
            smokeColor = add3(smokeColor, mul3(make_float3(0.010f, 0.012f, 0.016f), backScatter));
            const float scatterGain = scatterAlpha *
                                      (0.00046f + lightVisibility * 0.00072f * warmScatterDamp + flameDensity * 0.00008f * sceneWarmScatter +
                                       turbulenceEnergy * 0.00018f) *
                                      (0.038f + (1.0f - particleRadius) * 0.045f) * scatterSeparation;
            const float sceneScatter = scatterAlpha * scatterSeparation * (0.0065f + (1.0f - particleRadius) * 0.014f) * lightVisibility;
            const float3 neutralScatterLight =
                make_float3(localIrradianceLuma * 0.052f, localIrradianceLuma * 0.064f, localIrradianceLuma * 0.086f);
            const float3 smokeScatterLight = lerp3(neutralScatterLight, localIrradiance, nearFlameWarmLeak);
            const float coalGlow = smoothstepK(0.004f, 0.18f, charMass) * smoothstepK(0.54f, 0.02f, fv) * (0.070f + pyrolysis * 0.12f + heat * 0.009f);

            if (debugViews) {
                debugFlame = fmaxf(debugFlame, saturate(flameDensity * radiantPower * 0.26f));
                debugOpticalDepth = saturate(debugOpticalDepth + sootExtinction * stepT);
                debugTemperature = fmaxf(debugTemperature, saturate((tempK - 520.0f) / 1900.0f));
            }
            accum = add3(accum, mul3(flameEmission, trans));
            accum = add3(accum, mul3(make_float3(1.0f, 0.24f, 0.035f), trans * coalGlow * stepT));
            accum = add3(accum, mul3(smokeColor, trans * scatterGain * smokeOnlyMask));
            accum = add3(accum, mul3(smokeScatterLight, trans * sceneScatter * (0.18f + warmScatterDamp * 0.42f)));
            flameGlow = fmaxf(flameGlow, flameDensity * radiantPower * (0.12f + fieldFilament * 0.18f + whiteFilament * 0.20f));
            smokeOcclusion = saturate(smokeOcclusion + smokeAlpha * trans);
            trans *= expf(-extinction);
        }
    }

    if (debugViews && p.renderDebugMode != 0) {
        float3 dc = make_float3(0.0f, 0.0f, 0.0f);
        if (p.renderDebugMode == 1) {
            dc = debugHeatColor(debugFlame);
        } else if (p.renderDebugMode == 2) {
            const float od = saturate(debugOpticalDepth);
            dc = make_float3(od, od * 0.90f, od * 0.78f);
        } else if (p.renderDebugMode == 3) {
            dc = make_float3(trans, trans, trans);
        } else if (p.renderDebugMode == 4) {
            dc = debugHeatColor(debugTemperature);
        } else if (p.renderDebugMode == 5) {
            dc = make_float3(debugFuel * 0.82f, debugFuel * 0.48f, debugFuel * 0.18f);
        } else {
            dc = make_float3(debugVelocity * 0.20f, debugVelocity * 0.72f, debugVelocity);
        }
        out[y * p.frameW + x] = make_float4(dc.x, dc.y, dc.z, 1.0f);
        return;
    }
    float3 color = accum;
    if (trans > 0.006f) {
        const float3 roomColor = roomBackgroundRay(uv, rd, baseGlow, lightF, shadowF, L, p);
        color = add3(mul3(roomColor, trans), accum);
    }
    const float bloom = saturate(flameGlow * 0.10f) * (1.0f - saturate(smokeOcclusion * 0.95f));
    color = add3(color, mul3(make_float3(1.0f, 0.25f, 0.045f), bloom * bloom * 0.017f * p.reflectionGain));
    out[y * p.frameW + x] = make_float4(fmaxf(0.0f, color.x), fmaxf(0.0f, color.y), fmaxf(0.0f, color.z), 1.0f);
}

}  // namespace

// Rays through the flame cost many times more than rays that miss it, so a
// static grid leaves most SMs idle while the last blocks finish.  Here every
// warp repeatedly takes the next 8x4-pixel tile from a counter, in an order
// that starts at the centre of the frame (where the fire box projects) and
// ends at the corners, until no tile is left.  The kernels ask for 4 blocks of
// 128 threads per SM: 128 registers and no spills.  At 5 blocks (96
// registers, spills) a 512^2 frame of a developed 128^3 fire took 1.42 ms
// instead of 1.27 ms; at 3 or 2 blocks it was no faster.
template <int SC>
__device__ __forceinline__ void raymarchBody(float4* __restrict__ out, const ScalarFieldsIn& s, const Velocity& vel,
                                             const float4* __restrict__ lightF, const float* __restrict__ shadowF, const FrameParams& p,
                                             const RayTiles& tiles) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        int t = 0;
        if (lane == 0) {
            t = atomicAdd(tiles.counter, 1);
        }
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= tiles.count) {
            break;
        }
        const int tile = __ldg(tiles.order + t);
        const int x = (tile % tiles.tilesX) * kRayTileW + (lane % kRayTileW);
        const int y = (tile / tiles.tilesX) * kRayTileH + (lane / kRayTileW);
        if (x < p.frameW && y < p.frameH) {
            shadePixel<SC>(out, x, y, s, vel, lightF, shadowF, p);
        }
    }
}

// Any scene and debug mode.
__global__ void __launch_bounds__(128, 4) raymarch(float4* __restrict__ out, ScalarFieldsIn s, Velocity vel,
                                                   const float4* __restrict__ lightF, const float* __restrict__ shadowF, FrameParams p,
                                                   RayTiles tiles) {
    raymarchBody<-1>(out, s, vel, lightF, shadowF, p, tiles);
}
// Scenes 0, 1, 2 without a debug view (renderDebugMode 0).
__global__ void __launch_bounds__(128, 4) raymarchScene0(float4* __restrict__ out, ScalarFieldsIn s, Velocity vel,
                                                         const float4* __restrict__ lightF, const float* __restrict__ shadowF, FrameParams p,
                                                         RayTiles tiles) {
    raymarchBody<0>(out, s, vel, lightF, shadowF, p, tiles);
}
__global__ void __launch_bounds__(128, 4) raymarchScene1(float4* __restrict__ out, ScalarFieldsIn s, Velocity vel,
                                                         const float4* __restrict__ lightF, const float* __restrict__ shadowF, FrameParams p,
                                                         RayTiles tiles) {
    raymarchBody<1>(out, s, vel, lightF, shadowF, p, tiles);
}
__global__ void __launch_bounds__(128, 4) raymarchScene2(float4* __restrict__ out, ScalarFieldsIn s, Velocity vel,
                                                         const float4* __restrict__ lightF, const float* __restrict__ shadowF, FrameParams p,
                                                         RayTiles tiles) {
    raymarchBody<2>(out, s, vel, lightF, shadowF, p, tiles);
}

// ---------------------------------------------------------------------------
// Embers (src/fire_cuda.cu:2323-2452).  emberSetup computes one descriptor per
// ember; emberGather adds, per pixel, every ember that covers it in ember
// order -- the splat of the reference without its float atomics.
__global__ void __launch_bounds__(256) emberSetup(EmberSplat* __restrict__ embers, ScalarFieldsIn s, Velocity vel, FrameParams p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int emberCount = min(max(p.emberCount, 0), kMaxEmberCount);
    if (i >= emberCount) {
        return;
    }
    EmberSplat e{};
    e.active = 0;
    const Grid g{p.nx, p.ny, p.nz};
    if (p.renderDebugMode != 0) {
        embers[i] = e;
        return;
    }
    const float baseGlow = saturate(sampleHeat(s, g, 0.50f, 0.06f, 0.50f) * 0.42f);
    const float sparkGate = smoothstepf(0.02f, 0.30f, baseGlow);
    const int sc = p.sceneId;
    const float seed = static_cast<float>(i);
    const float h0 = hash21(seed, 3.7f);
    const float h1 = hash21(seed, 9.1f);
    const float h2 = hash21(seed, 19.4f);
    const float h3 = hash21(seed, 31.6f);
    if (sparkGate <= 0.0001f || (sc == 1 && h2 > 0.34f) || (sc == 2 && h0 > 0.14f)) {
        embers[i] = e;
        return;
    }
    const float life = fracf(p.time * (0.20f + h2 * 0.18f + (sc == 2 ? 0.36f : 0.0f)) + h0);
    const float spawnAngle = h0 * 6.2831853f;
    float startX = 0.0f, startZ = 0.0f;
    if (sc == 2) {
        const float sourceRadius = fmaxf(0.04f, p.emitterRadius);
        const float cx = p.burnerCenterCount > 0 ? p.burnerCenterX[0] : p.emitterCenterX;
        const float cz = p.burnerCenterCount > 0 ? p.burnerCenterZ[0] : p.emitterCenterZ;
        startX = cx + cosf(spawnAngle) * sourceRadius * (0.82f + h1 * 0.18f);
        startZ = cz + sinf(spawnAngle) * sourceRadius * (0.82f + h1 * 0.18f);
    } else if (sc == 1) {
        const float logA = orientedCapsuleMask(cosf(spawnAngle) * 0.34f, sinf(spawnAngle) * 0.25f, -0.06f, 0.01f, 0.38f, 0.34f, 0.095f);
        const float logB = orientedCapsuleMask(cosf(spawnAngle + 1.7f) * 0.35f, sinf(spawnAngle + 1.7f) * 0.25f, 0.07f, -0.02f, -0.58f, 0.33f, 0.092f);
        const float contactBlend = saturate(logA + logB + h3 * 0.35f);
        const float spawnRadius = lerpf(0.16f, 0.46f, sqrtf(h1));
        startX = cosf(spawnAngle) * spawnRadius * (0.64f + contactBlend * 0.36f);
        startZ = sinf(spawnAngle) * spawnRadius * (0.46f + contactBlend * 0.26f);
    } else {
        const float spawnRadius = 0.48f;
        const float ringBias = sqrtf(h1);
        startX = cosf(spawnAngle) * spawnRadius * ringBias;
        startZ = sinf(spawnAngle) * spawnRadius * ringBias;
    }
    const float startU = saturate((startX / 2.10f) + 0.50f);
    const float startW = saturate((startZ / 1.64f) + 0.50f);
    const float startV = sc == 2 ? p.emitterHeightNorm : (sc == 1 ? 0.035f + h2 * 0.055f : 0.045f);
    const Cell10 local = sampleAll(s, g, startU, startV, startW);
    const float localHeat = local.heat;
    const float localChar = local.charMass;
    const float localPyrolysis = local.pyrolysis;
    const float localTurbulence = local.turbulenceEnergy;
    const float3 localVelocity = sampleVelocity(vel, g, startU, startV, startW);
    const float materialGate = smoothstepf(0.018f, 0.40f, localChar + localPyrolysis * 0.34f + localHeat * 0.075f);
    if (materialGate <= 0.0001f) {
        embers[i] = e;
        return;
    }
    const float temperatureK = 620.0f + localHeat * 330.0f + localPyrolysis * 210.0f + localChar * 42.0f;
    const float sceneLift = sc == 1 ? 0.86f : (sc == 2 ? 0.16f : 0.80f);
    const float t = life * (sc == 1 ? 1.24f : (sc == 2 ? 0.34f : 1.10f));
    const float drag = expf(-t * (sc == 2 ? 4.8f : 1.35f));
    const float buoyantRise = (0.26f + h3 * 0.62f + localTurbulence * 0.11f) * t * sceneLift;
    const float3 sparkWorld = make_float3(startX + (localVelocity.x * 0.34f + (h1 - 0.5f) * 0.20f + p.wind * 0.26f) * t * drag,
                                          startV * 2.03f + 0.02f + buoyantRise - (0.22f + h2 * 0.16f) * t * t,
                                          startZ + (localVelocity.z * 0.28f + (h2 - 0.5f) * 0.18f) * t * drag);
    const float prevT = fmaxf(0.0f, t - 0.045f);
    const float prevDrag = expf(-prevT * (sc == 2 ? 4.8f : 1.35f));
    const float3 prevWorld = make_float3(startX + (localVelocity.x * 0.34f + (h1 - 0.5f) * 0.20f + p.wind * 0.26f) * prevT * prevDrag,
                                         startV * 2.03f + 0.02f + (0.26f + h3 * 0.62f + localTurbulence * 0.11f) * prevT * sceneLift -
                                             (0.22f + h2 * 0.16f) * prevT * prevT,
                                         startZ + (localVelocity.z * 0.28f + (h2 - 0.5f) * 0.18f) * prevT * prevDrag);
    const float3 sparkScreen = projectPoint(p, sparkWorld);
    const float3 prevScreen = projectPoint(p, prevWorld);
    if (sparkScreen.z <= 0.0f || sparkScreen.x < -0.05f || sparkScreen.x > 1.05f || sparkScreen.y < -0.05f || sparkScreen.y > 1.05f) {
        embers[i] = e;
        return;
    }
    const float emberSize = smoothstepf(720.0f, 1580.0f, temperatureK) * materialGate;
    const float radius = ((sc == 2 ? 0.00042f : 0.00086f) + h3 * (sc == 2 ? 0.00042f : 0.00145f)) * (0.72f + emberSize * 0.90f) /
                         fmaxf(0.55f, sparkScreen.z);
    const float centerX = sparkScreen.x * static_cast<float>(p.frameW) - 0.5f;
    const float centerY = sparkScreen.y * static_cast<float>(p.frameH) - 0.5f;
    const float2 rawTrail = sub2(make_float2(sparkScreen.x, sparkScreen.y), make_float2(prevScreen.x, prevScreen.y));
    const float rawTrailLen = sqrtf(dot2(rawTrail, rawTrail));
    const float cappedTrailLen = fminf(rawTrailLen, sc == 1 ? 0.016f : 0.005f);
    const float2 trailDir = rawTrailLen > 0.000001f ? mul2(rawTrail, 1.0f / rawTrailLen) : make_float2(0.0f, -1.0f);
    const int pad = max(2, static_cast<int>(ceilf((radius + cappedTrailLen) * static_cast<float>(max(p.frameW, p.frameH)) * 3.0f)));
    const float3 hotCore = sc == 2 ? make_float3(0.36f, 0.58f, 1.04f) : make_float3(1.0f, 0.42f, 0.090f);
    const float3 cooled = sc == 2 ? make_float3(0.055f, 0.10f, 0.18f) : make_float3(0.18f, 0.026f, 0.008f);
    const float cooling = smoothstepf(0.16f, 0.92f, life) * (1.0f - saturate(localHeat * 0.045f));
    e.active = 1;
    e.minX = max(0, static_cast<int>(floorf(centerX)) - pad);
    e.maxX = min(p.frameW - 1, static_cast<int>(ceilf(centerX)) + pad);
    e.minY = max(0, static_cast<int>(floorf(centerY)) - pad);
    e.maxY = min(p.frameH - 1, static_cast<int>(ceilf(centerY)) + pad);
    e.screenX = sparkScreen.x;
    e.screenY = sparkScreen.y;
    e.trailX = trailDir.x;
    e.trailY = trailDir.y;
    e.radius = radius;
    e.cappedTrailLen = cappedTrailLen;
    e.color = lerp3(hotCore, cooled, cooling);
    e.lifeFade = smoothstepf(1.0f, 0.08f, life) * smoothstepf(0.0f, 0.16f, life) * sparkGate * materialGate * emberSize *
                 (sc == 2 ? 0.055f : (sc == 1 ? 0.58f : 0.82f));
    embers[i] = e;
}

__global__ void __launch_bounds__(256) emberGather(float4* __restrict__ hdr, const EmberSplat* __restrict__ embers, FrameParams p) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= p.frameW || y >= p.frameH) {
        return;
    }
    const int emberCount = min(max(p.emberCount, 0), kMaxEmberCount);
    float4 px = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    bool loaded = false;
    const float uy = (static_cast<float>(y) + 0.5f) / static_cast<float>(p.frameH);
    const float ux = (static_cast<float>(x) + 0.5f) / static_cast<float>(p.frameW);
    for (int i = 0; i < emberCount; ++i) {
        const EmberSplat& e = embers[i];
        if (!e.active || x < e.minX || x > e.maxX || y < e.minY || y > e.maxY) {
            continue;
        }
        const float2 trailDir = make_float2(e.trailX, e.trailY);
        const float2 d = sub2(make_float2(ux, uy), make_float2(e.screenX, e.screenY));
        const float along = dot2(d, trailDir);
        const float2 acrossVec = sub2(d, mul2(trailDir, along));
        const float across2 = dot2(acrossVec, acrossVec);
        const float streakRadius = e.radius * (1.0f + e.cappedTrailLen * 130.0f);
        const float emberCore = expf(-(across2 / fmaxf(0.0000002f, e.radius * e.radius) + along * along / fmaxf(0.0000002f, streakRadius * streakRadius)));
        const float emberHalo = expf(-dot2(d, d) / fmaxf(0.0000002f, e.radius * e.radius * 8.0f)) * 0.16f;
        const float spark = (emberCore + emberHalo) * e.lifeFade;
        if (spark > 0.00001f) {
            if (!loaded) {
                px = hdr[y * p.frameW + x];
                loaded = true;
            }
            px.x += e.color.x * spark;
            px.y += e.color.y * spark;
            px.z += e.color.z * spark;
        }
    }
    if (loaded) {
        hdr[y * p.frameW + x] = px;
    }
}

// ---------------------------------------------------------------------------
namespace {

__device__ __forceinline__ float acesToneCurve(float value) {  // src/fire_cuda.cu:2246-2253
    const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
    return saturate((value * (a * value + b)) / (value * (c * value + d) + e));
}

__device__ __forceinline__ float3 cameraResponse(float3 radiance, float exposure) {  // src/fire_cuda.cu:2255-2274
    float3 color = mul3(make_float3(fmaxf(0.0f, radiance.x), fmaxf(0.0f, radiance.y), fmaxf(0.0f, radiance.z)), exposure);
    {
        const float luma = fmaxf(0.000001f, luminance3(color));
        const float mappedLuma = acesToneCurve(luma);
        color = mul3(color, mappedLuma / luma);
    }
    const float luma = luminance3(color);
    const float toe = smoothstepf(0.000f, 0.055f, luma);
    const float hdrShoulderPreserve = smoothstepf(0.78f, 1.08f, luma);
    color = lerp3(mul3(color, 0.82f), color, toe);
    color = lerp3(color, mul3(color, 1.0f / fmaxf(1.0f, luma / 0.94f)), hdrShoulderPreserve * 0.10f);
    const float blackbodyHighlightLift = smoothstepf(0.56f, 0.90f, luma);
    color = mul3(color, 1.0f + blackbodyHighlightLift * 0.28f);
    return make_float3(powf(saturate(color.x), 1.0f / 2.2f), powf(saturate(color.y), 1.0f / 2.2f), powf(saturate(color.z), 1.0f / 2.2f));
}

__device__ __forceinline__ uint32_t packBgra(float3 color) {  // src/fire_cuda.cu:2461-2466
    const uint32_t r = static_cast<uint32_t>(saturate(color.x) * 255.0f);
    const uint32_t g = static_cast<uint32_t>(saturate(color.y) * 255.0f);
    const uint32_t b = static_cast<uint32_t>(saturate(color.z) * 255.0f);
    return 0xff000000u | (r << 16) | (g << 8) | b;
}

__device__ __forceinline__ float3 unpackBgra(uint32_t px) {
    return make_float3(static_cast<float>((px >> 16) & 0xff) / 255.0f, static_cast<float>((px >> 8) & 0xff) / 255.0f,
                       static_cast<float>(px & 0xff) / 255.0f);
}

__device__ __forceinline__ float lineAlpha(float2 q, float2 a, float2 b, float thickness) {
    const float2 pa = sub2(q, a);
    const float2 ba = sub2(b, a);
    const float h = saturate(dot2(pa, ba) / fmaxf(0.000001f, dot2(ba, ba)));
    const float2 d = sub2(pa, mul2(ba, h));
    return smoothstepf(thickness, thickness * 0.35f, sqrtf(dot2(d, d)));
}

__device__ __forceinline__ float3 drawGizmos(float3 color, float2 uv, const FrameParams& p) {  // src/fire_cuda.cu:1931-1951
    auto blend = [&](float3 g, float alpha) { color = lerp3(color, g, saturate(alpha)); };
    const float sourceX = p.sceneId == 2 && p.burnerCenterCount > 0 ? p.burnerCenterX[0] : p.emitterCenterX;
    const float sourceY = p.sceneId == 2 && p.burnerCenterCount > 0 ? p.burnerCenterY[0] : p.emitterHeightNorm * 2.03f + 0.02f;
    const float sourceZ = p.sceneId == 2 && p.burnerCenterCount > 0 ? p.burnerCenterZ[0] : p.emitterCenterZ;
    const float3 source = projectPoint(p, make_float3(sourceX, sourceY, sourceZ));
    if (source.z > 0.0f) {
        const float2 c = make_float2(source.x, source.y);
        const float2 d = sub2(uv, c);
        const float dist = sqrtf(dot2(d, d));
        const float ring = smoothstepf(0.006f, 0.006f * 0.25f, fabsf(dist - 0.125f / source.z));
        const float disk = smoothstepf(0.012f, 0.012f * 0.45f, dist);
        blend(p.activeGizmo == 1 ? make_float3(1.0f, 0.34f, 0.055f) : make_float3(0.45f, 0.18f, 0.055f), (ring + disk) * 0.85f);
    }
    const float2 axisBase = make_float2(0.90f, 0.84f);
    const float2 xAxis = add2(axisBase, mul2(make_float2(dot3(make_float3(1.0f, 0.0f, 0.0f), p.right), -dot3(make_float3(1.0f, 0.0f, 0.0f), p.up)), 0.070f));
    const float2 yAxis = add2(axisBase, mul2(make_float2(dot3(make_float3(0.0f, 1.0f, 0.0f), p.right), -dot3(make_float3(0.0f, 1.0f, 0.0f), p.up)), 0.070f));
    const float2 zAxis = add2(axisBase, mul2(make_float2(dot3(make_float3(0.0f, 0.0f, 1.0f), p.right), -dot3(make_float3(0.0f, 0.0f, 1.0f), p.up)), 0.070f));
    blend(make_float3(1.0f, 0.12f, 0.08f), lineAlpha(uv, axisBase, xAxis, 0.005f));
    blend(make_float3(0.22f, 1.0f, 0.30f), lineAlpha(uv, axisBase, yAxis, 0.005f));
    blend(make_float3(0.20f, 0.48f, 1.0f), lineAlpha(uv, axisBase, zAxis, 0.005f));
    return color;
}

}  // namespace

// Camera response to BGRA8 (doTonemap) and/or the gizmo overlay (doOverlay).
__global__ void __launch_bounds__(256) tonemapOverlay(uint32_t* __restrict__ frame, const float4* __restrict__ hdr, FrameParams p,
                                                      int doTonemap, int doOverlay) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= p.frameW || y >= p.frameH) {
        return;
    }
    const int i = y * p.frameW + x;
    uint32_t px = 0;
    if (doTonemap) {
        const float4 radiance = __ldg(hdr + i);
        float3 color = cameraResponse(make_float3(radiance.x, radiance.y, radiance.z), p.exposure);
        const float dither = (hash21(static_cast<float>(x) * 0.754877f, static_cast<float>(y) * 0.569840f) - 0.5f) / 255.0f;
        color = add3(color, make_float3(dither, dither, dither));
        px = packBgra(color);
    } else {
        px = frame[i];
    }
    if (doOverlay && p.renderDebugMode == 0 && p.showGizmos != 0) {
        const float2 uv = make_float2((static_cast<float>(x) + 0.5f) / static_cast<float>(p.frameW),
                                      (static_cast<float>(y) + 0.5f) / static_cast<float>(p.frameH));
        px = packBgra(drawGizmos(unpackBgra(px), uv, p));
    }
    frame[i] = px;
}

// Copies the HDR frame into a caller-owned device buffer (the headless form of
// packFp16SurfaceKernel, src/fire_cuda.cu:2303-2321): float4 RGBA32F, or RGBA16F
// with negative values clamped to 0 as the reference's halfBits does.
__global__ void __launch_bounds__(256) packHdr(void* __restrict__ dst, size_t pitchBytes, int halfFormat, const float4* __restrict__ hdr,
                                               FrameParams p) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= p.frameW || y >= p.frameH) {
        return;
    }
    packHdrPixel(dst, pitchBytes, halfFormat, __ldg(hdr + y * p.frameW + x), x, y);
}

}  // namespace firesim
