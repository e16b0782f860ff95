// fire_sim.cu -- simulation kernels of one frame (sm_100a).
//
// Stage map against native-firesim's src/fire_cuda.cu:
//   resetScalarsKernel            :805-848   -> resetCells (+ fuel-bed tables)
//   advectU/V/WKernel             :880-932   -> advectVelocity (all three face grids, one launch)
//   advectReactKernel             :934-1126  -> advectReact (packed records, tabled fuel bed)
//   forceVelocityKernel           :1128-1183 -> forceContributions + face gathers (no atomics)
//   velocityBoundaryKernel        :1261-1291 -> velocityBoundary / fused into forceProject
//   divergenceKernel              :1185-1199 -> divergence / fused into forceProject
//   sorPressureParityKernel       :1201-1227 -> sorResident / sorSplitHalfSweep
//   subtractPressureKernel        :1229-1245 -> subtractWall (fused with the wall zeroing)
//   velocityWallBoundaryKernel    :1293-1317
#include "fire_kernels.h"

namespace firesim {

namespace {

__device__ __forceinline__ int uAt(const Grid& g, int x, int y, int z) { return (z * g.ny + y) * (g.nx + 1) + x; }
__device__ __forceinline__ int vAt(const Grid& g, int x, int y, int z) { return (z * (g.ny + 1) + y) * g.nx + x; }
__device__ __forceinline__ int wAt(const Grid& g, int x, int y, int z) { return (z * g.ny + y) * g.nx + x; }
__device__ __forceinline__ int sAt(const Grid& g, int x, int y, int z) { return (z * g.ny + y) * g.nx + x; }
__device__ __forceinline__ int sClamped(const Grid& g, int x, int y, int z) {
    x = min(max(x, 0), g.nx - 1);
    y = min(max(y, 0), g.ny - 1);
    z = min(max(z, 0), g.nz - 1);
    return (z * g.ny + y) * g.nx + x;
}

__device__ __forceinline__ float worldXOf(int x, int nx) { return (cellCoord(x, nx) - 0.50f) * 2.10f; }
__device__ __forceinline__ float worldZOf(int z, int nz) { return (cellCoord(z, nz) - 0.50f) * 1.64f; }

}  // namespace

// ---------------------------------------------------------------------------
// Fuel-bed tables: material(x, z) per scene, breathing(x, z, time) per frame.
__global__ void __launch_bounds__(256) fuelBedTables(float* __restrict__ material, float* __restrict__ breathing,
                                                     FrameParams p, int withMaterial) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y;
    if (x >= p.nx || z >= p.nz) {
        return;
    }
    const float wx = worldXOf(x, p.nx);
    const float wz = worldZOf(z, p.nz);
    if (withMaterial) {
        material[z * p.nx + x] = fuelBedMaterial(wx, wz, p);
    }
    breathing[z * p.nx + x] = emberBreathing(wx, wz, p.time);
}

// src/fire_cuda.cu:805-848 -- procedural initial state of every cell.
__global__ void __launch_bounds__(256) resetCells(ScalarFields out, float* __restrict__ pressure, float* __restrict__ divergence,
                                                  float* __restrict__ divergenceAfter, const float* __restrict__ material,
                                                  const float* __restrict__ breathing, FrameParams p) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= p.nx) {
        return;
    }
    const Grid g{p.nx, p.ny, p.nz};
    const int idx = sAt(g, x, y, z);
    const float v = cellCoord(y, p.ny);
    const float worldX = worldXOf(x, p.nx);
    const float worldZ = worldZOf(z, p.nz);
    const float mat = __ldg(material + z * p.nx + x);
    const float chunkNoise = fbm(worldX * 18.0f + worldZ * 2.0f, worldZ * 22.0f - worldX * 5.0f);
    const float bed = fuelBedSourceFrom(mat, __ldg(breathing + z * p.nx + x), v, p);
    const int sc = p.sceneId;
    const float charScale = sc == 2 ? 0.004f : (sc == 1 ? 1.18f : 1.0f);
    const float sootScale = sc == 2 ? 0.004f : (sc == 1 ? 0.92f : 1.0f);
    const float heat = bed * (sc == 2 ? 1.34f : (sc == 1 ? 0.78f + chunkNoise * 0.26f : 0.86f + chunkNoise * 0.24f));
    const float fuel = bed * (sc == 2 ? 1.42f : (sc == 1 ? 1.05f + chunkNoise * 0.30f : 1.08f + chunkNoise * 0.26f));
    const float soot = bed * (sc == 2 ? 0.00065f : 0.018f) * sootScale;
    const float charMass = mat * (0.92f + chunkNoise * 0.72f) * charScale;
    const float ash = mat * (0.018f + smoothstepf(0.56f, 0.86f, chunkNoise) * 0.055f) * (sc == 2 ? 0.10f : 1.0f);
    const float pyrolysis = bed * (sc == 2 ? 0.018f : (sc == 1 ? 0.060f + chunkNoise * 0.034f : 0.058f + chunkNoise * 0.028f));
    const float progress = bed * (sc == 2 ? 0.11f : (sc == 1 ? 0.24f : 0.21f));
    const float turbulence = bed * (sc == 2 ? 0.012f : (sc == 1 ? 0.082f : 0.065f));
    const float sootOptics = bed * (sc == 2 ? 0.00050f : 0.018f) * sootScale;
    stv(out.a + idx, make_float4(heat, fuel, 1.0f, soot));
    stv(out.b + idx, make_float4(charMass, ash, pyrolysis, progress));
    stv(out.c + idx, make_float2(turbulence, sootOptics));
    pressure[idx] = 0.0f;
    divergence[idx] = 0.0f;
    divergenceAfter[idx] = 0.0f;
}

// ---------------------------------------------------------------------------
// The face kernels run on the cell grid: the thread of cell (x, y, z) takes
// the u, v and w faces of index (x, y, z) and, as the last cell of its row,
// column or plane, the far wall's faces of index (nx, y, z), (x, ny, z) and
// (x, y, nz).  Every face index of the (nx + 1) x (ny + 1) x (nz + 1) space
// that holds a face is visited once; a face grid of nx + 1 columns would
// leave a nearly empty block per row.
template <class Face>
__device__ __forceinline__ void facesOfCell(const FrameParams& p, int x, int y, int z, Face face) {
    face(x, y, z);
    if (x == p.nx - 1) face(p.nx, y, z);
    if (y == p.ny - 1) face(x, p.ny, z);
    if (z == p.nz - 1) face(x, y, p.nz);
}

// ---------------------------------------------------------------------------
// src/fire_cuda.cu:880-932 -- self-advection of the three face grids.  One
// thread owns the u, v and w faces that share its (x, y, z) index.
__device__ __forceinline__ void advectVelocityAt(FaceT* __restrict__ uOut, FaceT* __restrict__ vOut, FaceT* __restrict__ wOut,
                                                 const Velocity& vel, const FrameParams& p, int x, int y, int z) {
    const Grid g{p.nx, p.ny, p.nz};
    const float back = p.dt;
    if (x <= p.nx && y < p.ny && z < p.nz) {
        float r = 0.0f;
        if (x != 0 && x != p.nx) {
            const float fu = static_cast<float>(x) / static_cast<float>(p.nx);
            const float fv = cellCoord(y, p.ny);
            const float fw = cellCoord(z, p.nz);
            const float3 c = sampleVelocity(vel, g, fu, fv, fw);
            r = sampleU(vel.u, g, fu - c.x * back * kAdvectionScale, fv - c.y * back * kAdvectionScale,
                        fw - c.z * back * kAdvectionScale) * 0.995f;
        }
        stv(uOut + uAt(g, x, y, z), r);
    }
    if (x < p.nx && y <= p.ny && z < p.nz) {
        float r = 0.0f;
        if (y != 0) {
            const float fu = cellCoord(x, p.nx);
            const float fv = static_cast<float>(y) / static_cast<float>(p.ny);
            const float fw = cellCoord(z, p.nz);
            const float3 c = sampleVelocity(vel, g, fu, fv, fw);
            r = sampleV(vel.v, g, fu - c.x * back * kAdvectionScale, fv - c.y * back * kAdvectionScale,
                        fw - c.z * back * kAdvectionScale) * 0.996f;
        }
        stv(vOut + vAt(g, x, y, z), r);
    }
    if (x < p.nx && y < p.ny && z <= p.nz) {
        float r = 0.0f;
        if (z != 0 && z != p.nz) {
            const float fu = cellCoord(x, p.nx);
            const float fv = cellCoord(y, p.ny);
            const float fw = static_cast<float>(z) / static_cast<float>(p.nz);
            const float3 c = sampleVelocity(vel, g, fu, fv, fw);
            r = sampleW(vel.w, g, fu - c.x * back * kAdvectionScale, fv - c.y * back * kAdvectionScale,
                        fw - c.z * back * kAdvectionScale) * 0.995f;
        }
        stv(wOut + wAt(g, x, y, z), r);
    }
}

__global__ void __launch_bounds__(256) advectVelocity(FaceT* __restrict__ uOut, FaceT* __restrict__ vOut, FaceT* __restrict__ wOut,
                                                      Velocity vel, FrameParams p) {
    const int cx = blockIdx.x * blockDim.x + threadIdx.x;
    if (cx >= p.nx) return;
    facesOfCell(p, cx, blockIdx.y, blockIdx.z, [&](int x, int y, int z) { advectVelocityAt(uOut, vOut, wOut, vel, p, x, y, z); });
}

// ---------------------------------------------------------------------------
// MacCormack gathers of the packed records (src/fire_cuda.cu:666-732): the
// first-order sample and the clamp bounds share the eight corners.
namespace {

struct PackedSample {
    float4 a, b;
    float2 c;
};

struct PackedBounded {
    PackedSample value, lo, hi;
};

__device__ __forceinline__ float4 min4(float4 a, float4 b) {
    return make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), fminf(a.w, b.w));
}
__device__ __forceinline__ float4 max4(float4 a, float4 b) {
    return make_float4(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z), fmaxf(a.w, b.w));
}
__device__ __forceinline__ float2 min2(float2 a, float2 b) { return make_float2(fminf(a.x, b.x), fminf(a.y, b.y)); }
__device__ __forceinline__ float2 max2(float2 a, float2 b) { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }

// First-order sample of a packed record and the componentwise min/max of its
// eight corners (float4 / float2 records, or their half forms).
__device__ __forceinline__ float4 minv(float4 a, float4 b) { return min4(a, b); }
__device__ __forceinline__ float4 maxv(float4 a, float4 b) { return max4(a, b); }
__device__ __forceinline__ float2 minv(float2 a, float2 b) { return min2(a, b); }
__device__ __forceinline__ float2 maxv(float2 a, float2 b) { return max2(a, b); }

template <class P, class V>
__device__ __forceinline__ void gatherBounded(const P* __restrict__ f, const Corners& c, int sx, int sy, V& value, V& lo, V& hi) {
    const V c000 = ldv(f + (c.z0 * sy + c.y0) * sx + c.x0);
    const V c100 = ldv(f + (c.z0 * sy + c.y0) * sx + c.x1);
    const V c010 = ldv(f + (c.z0 * sy + c.y1) * sx + c.x0);
    const V c110 = ldv(f + (c.z0 * sy + c.y1) * sx + c.x1);
    const V c001 = ldv(f + (c.z1 * sy + c.y0) * sx + c.x0);
    const V c101 = ldv(f + (c.z1 * sy + c.y0) * sx + c.x1);
    const V c011 = ldv(f + (c.z1 * sy + c.y1) * sx + c.x0);
    const V c111 = ldv(f + (c.z1 * sy + c.y1) * sx + c.x1);
    value = lerpv(lerpv(lerpv(c000, c100, c.tx), lerpv(c010, c110, c.tx), c.ty),
                  lerpv(lerpv(c001, c101, c.tx), lerpv(c011, c111, c.tx), c.ty), c.tz);
    lo = minv(minv(minv(c000, c100), minv(c010, c110)), minv(minv(c001, c101), minv(c011, c111)));
    hi = maxv(maxv(maxv(c000, c100), maxv(c010, c110)), maxv(maxv(c001, c101), maxv(c011, c111)));
}

__device__ __forceinline__ float macCormack(float firstOrder, float lo, float hi, float current, float roundTrip, float blend) {
    const float corrected = fminf(hi, fmaxf(lo, firstOrder + 0.5f * (current - roundTrip)));
    return lerpf(firstOrder, corrected, saturate(blend));
}

}  // namespace

// src/fire_cuda.cu:934-1126 -- advection of the ten scalars plus the reaction network.
__global__ void __launch_bounds__(128, 6) advectReact(ScalarFields out, ScalarFieldsIn in, Velocity vel,
                                                   const float* __restrict__ material, const float* __restrict__ breathing,
                                                   FrameParams p, HashLattice2 sourceLattice) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= p.nx) {
        return;
    }
    const Grid g{p.nx, p.ny, p.nz};
    const float u = cellCoord(x, p.nx);
    const float v = cellCoord(y, p.ny);
    const float w = cellCoord(z, p.nz);
    const int idx = sAt(g, x, y, z);
    const Cell10 cur = loadCell(in, idx);
    const float currentActivity = cur.heat + cur.fuel * 0.18f + cur.soot * 0.24f + cur.pyrolysis * 0.20f + cur.progress * 0.14f +
                                  cur.sootOptics * 0.08f + cur.turbulenceEnergy * 0.06f;
    const float sourceDx = u - p.mouseX;
    const float sourceDy = v - p.mouseY;
    const float sourceDz = w - 0.5f;
    const bool outsideInteractiveSource =
        p.leftDown == 0 || (sourceDx * sourceDx + sourceDy * sourceDy + sourceDz * sourceDz) > 0.090f;
    if (v > 0.18f && currentActivity < 0.00035f && cur.charMass < 0.00010f && cur.ash < 0.00010f && outsideInteractiveSource &&
        p.rightDown == 0) {
        // Cold-air early out (src/fire_cuda.cu:984-1001).
        stv(out.a + idx, make_float4(0.0f, 0.0f, fminf(1.0f, cur.oxygen + (1.0f - cur.oxygen) * p.dt * 0.08f), 0.0f));
        stv(out.b + idx, make_float4(cur.charMass, cur.ash, 0.0f, 0.0f));
        stv(out.c + idx, make_float2(cur.turbulenceEnergy * fmaxf(0.0f, 1.0f - p.dt * 0.54f), 0.0f));
        return;
    }
    const float3 velHere = sampleVelocity(vel, g, u, v, w);
    const float prevU = u - velHere.x * p.dt * kAdvectionScale;
    const float prevV = v - velHere.y * p.dt * kAdvectionScale;
    const float prevW = w - velHere.z * p.dt * kAdvectionScale;
    const float3 prevVel = sampleVelocity(vel, g, prevU, prevV, prevW);

    // First-order samples with their clamp bounds, and the forward round trip.
    const Corners cp = scalarCorners(g, prevU, prevV, prevW);
    PackedBounded f1;
    gatherBounded(in.a, cp, g.nx, g.ny, f1.value.a, f1.lo.a, f1.hi.a);
    gatherBounded(in.b, cp, g.nx, g.ny, f1.value.b, f1.lo.b, f1.hi.b);
    gatherBounded(in.c, cp, g.nx, g.ny, f1.value.c, f1.lo.c, f1.hi.c);
    const float fwdU = prevU + prevVel.x * p.dt * kAdvectionScale;
    const float fwdV = prevV + prevVel.y * p.dt * kAdvectionScale;
    const float fwdW = prevW + prevVel.z * p.dt * kAdvectionScale;
    const Corners cf = scalarCorners(g, fwdU, fwdV, fwdW);
    const float4 rtA = gatherVec(in.a, cf, g.nx, g.ny);
    const float4 rtB = gatherVec(in.b, cf, g.nx, g.ny);
    const float2 rtC = gatherVec(in.c, cf, g.nx, g.ny);

    const float antiDiffusion = saturate(0.30f + p.detail * 0.34f);
    float heat = macCormack(f1.value.a.x, f1.lo.a.x, f1.hi.a.x, cur.heat, rtA.x, antiDiffusion);
    float fuel = macCormack(f1.value.a.y, f1.lo.a.y, f1.hi.a.y, cur.fuel, rtA.y, antiDiffusion * 0.92f);
    float oxygen = macCormack(f1.value.a.z, f1.lo.a.z, f1.hi.a.z, cur.oxygen, rtA.z, antiDiffusion * 0.70f);
    float soot = macCormack(f1.value.a.w, f1.lo.a.w, f1.hi.a.w, cur.soot, rtA.w, antiDiffusion);
    float charMass = cur.charMass;
    float ash = cur.ash;
    float pyrolysisRate = macCormack(f1.value.b.z, f1.lo.b.z, f1.hi.b.z, cur.pyrolysis, rtB.z, antiDiffusion * 0.72f) * 0.55f;
    float progress = macCormack(f1.value.b.w, f1.lo.b.w, f1.hi.b.w, cur.progress, rtB.w, antiDiffusion * 0.82f);
    float turbulenceEnergy = macCormack(f1.value.c.x, f1.lo.c.x, f1.hi.c.x, cur.turbulenceEnergy, rtC.x, antiDiffusion * 0.52f);
    float sootOptics = macCormack(f1.value.c.y, f1.lo.c.y, f1.hi.c.y, cur.sootOptics, rtC.y, antiDiffusion * 0.72f);

    const int sc = p.sceneId;
    const float worldX = (u - 0.50f) * 2.10f;
    const float worldZ = (w - 0.50f) * 1.64f;
    const float mat = __ldg(material + z * p.nx + x);
    // The source noise only matters where the bed profile or the char release
    // is non-zero: elsewhere it multiplies a zero, and the zero (with its sign)
    // is the same for any finite positive noise.  It is evaluated lazily, at
    // most once, from this step's hash lattice.
    auto evalSourceNoise = [&]() {
        return 0.70f + 0.48f * fbmLattice(worldX * 13.0f + worldZ * 3.0f + p.time * 0.38f, v * 31.0f + worldZ * 11.0f, sourceLattice);
    };
    const float exposedChar = saturate(charMass / fmaxf(0.055f, charMass + ash * 1.75f));
    const float charEdges = smoothstepf(0.06f, 0.78f, mat) * smoothstepf(0.92f, 0.02f, ash);
    const float gasFeed = sc == 2 ? 1.18f : exposedChar * charEdges;
    const float scenePyrolysisGain = sc == 2 ? 0.42f : (sc == 1 ? 1.34f : 1.0f);
    const float sceneFuelGain = sc == 2 ? 0.46f : (sc == 1 ? 1.18f : 1.0f);
    const float sceneHeatGain = sc == 2 ? 1.18f : (sc == 1 ? 1.08f : 1.0f);
    const float sceneSootGain = sc == 2 ? 0.18f : (sc == 1 ? 1.22f : 1.0f);
    const float bedProfile = fuelBedSourceFrom(mat, __ldg(breathing + z * p.nx + x), v, p);
    float sourceNoise = 1.0f;
    bool haveSourceNoise = false;
    if (bedProfile != 0.0f) {
        sourceNoise = evalSourceNoise();
        haveSourceNoise = true;
    }
    const float bed = bedProfile * sourceNoise * gasFeed * p.intensity;
    const float ambientK = 293.0f;
    float tempK = ambientK + heat * 335.0f;
    const float radiativeFeedback = smoothstepf(430.0f, 980.0f, tempK);
    const float solidOxygen = saturate(oxygen * 1.28f - soot * 0.030f);
    const float heatFlux = saturate((tempK - 405.0f) / 900.0f) + bed * 0.34f + sootOptics * 0.024f;
    const float charRelease = fminf(charMass, charMass * heatFlux * solidOxygen * (0.14f + radiativeFeedback * 1.38f) * p.dt);
    if (!haveSourceNoise && charRelease != 0.0f) {
        sourceNoise = evalSourceNoise();
    }
    pyrolysisRate += (bed * (0.34f + radiativeFeedback * 1.05f) * p.dt + charRelease * (2.45f + sourceNoise * 0.72f)) * scenePyrolysisGain;
    charMass += mat * p.dt * (sc == 2 ? 0.00005f : (sc == 1 ? 0.050f : 0.026f));
    charMass -= charRelease * 0.92f;
    ash += charRelease * (sc == 2 ? 0.025f : 0.16f + 0.22f * saturate(1.0f - oxygen));

    heat += (bed * (sc == 2 ? 10.40f : 6.20f) * p.dt * (1.0f + radiativeFeedback * 1.12f) + charRelease * 3.35f) * sceneHeatGain;
    fuel += pyrolysisRate * (sc == 2 ? 1.34f : 3.70f) * sceneFuelGain;
    soot += pyrolysisRate * (0.090f + ash * 0.032f + saturate(1.0f - oxygen) * 0.13f) * p.smokeGain *
            (sc == 2 ? 0.010f : (sc == 1 ? 0.92f : 1.0f)) * sceneSootGain;

    if (p.leftDown != 0) {
        const float mx = p.mouseX;
        const float my = p.mouseY;
        const float source = expf(-((u - mx) * (u - mx)) / 0.0180f - ((w - 0.5f) * (w - 0.5f)) / 0.0550f - ((v - my) * (v - my)) / 0.0020f);
        heat += source * p.dt * 2.8f;
        fuel += source * p.dt * 1.4f;
        pyrolysisRate += source * p.dt * 0.45f;
        progress += source * p.dt * 0.75f;
        turbulenceEnergy += source * p.dt * 0.28f;
        oxygen = fmaxf(oxygen, 0.72f + source * 0.20f);
    }
    if (p.rightDown != 0) {
        const float source =
            expf(-((u - p.mouseX) * (u - p.mouseX) + (w - 0.5f) * (w - 0.5f)) / 0.0100f - (v - p.mouseY) * (v - p.mouseY) / 0.0100f);
        soot += source * p.dt * 8.0f;
        heat *= 1.0f - source * p.dt * 1.2f;
        fuel *= 1.0f - source * p.dt * 0.7f;
    }

    tempK = ambientK + heat * 335.0f;
    const float thermalActivation = smoothstepf(575.0f, 1220.0f, tempK);
    const float arrhenius = expf(-3800.0f / fmaxf(640.0f, tempK));
    const float oxygenLimited = fminf(fuel, oxygen * 1.42f);
    const float burnMass = fminf(oxygenLimited, oxygenLimited * thermalActivation * arrhenius * (118.0f + p.intensity * 34.0f) * p.dt);
    const float incomplete = saturate(1.0f - oxygen * 1.30f + fuel * 0.065f + soot * 0.015f);
    const float heatRelease = burnMass * 7.0f;
    const float sootYield = burnMass * (0.035f + incomplete * 0.34f) * p.smokeGain * (sc == 2 ? 0.006f : (sc == 1 ? 0.96f : 1.0f));
    const float sootOxidation = soot * oxygen * smoothstepf(760.0f, 1540.0f, tempK) * p.dt * 0.82f;
    const float frontProduction = burnMass * (9.8f + turbulenceEnergy * 3.4f) + pyrolysisRate * 0.70f + charRelease * 2.10f;
    const float boundaryAir = smoothstepf(0.70f, 0.96f, v) + smoothstepf(0.11f, 0.03f, u) + smoothstepf(0.89f, 0.97f, u) +
                              smoothstepf(0.11f, 0.03f, w) + smoothstepf(0.89f, 0.97f, w);
    const float upperEntrainment = smoothstepf(0.52f, 0.98f, v);

    heat += heatRelease;
    fuel -= burnMass * 1.20f;
    oxygen -= burnMass * 0.98f;
    soot += sootYield;
    soot -= sootOxidation;
    progress += frontProduction;
    progress *= expf(-p.dt * (0.72f + v * 0.45f + oxygen * 0.16f + saturate(boundaryAir) * 1.05f + upperEntrainment * 0.26f));

    oxygen = lerpf(oxygen, 1.0f, saturate(boundaryAir) * p.dt * 1.7f);
    oxygen += (1.0f - oxygen) * p.dt * 0.08f;

    tempK = ambientK + heat * 335.0f;
    const float radiationBase = fmaxf(0.0f, (tempK - ambientK) / 1560.0f);
    const float radiationSq = radiationBase * radiationBase;
    const float radiationLoss = radiationSq * radiationSq;
    heat -= radiationLoss * p.dt * (0.88f + soot * 0.085f + sootOptics * 0.018f);
    heat *= expf(-p.dt * (0.31f + v * 0.64f + soot * 0.022f + saturate(boundaryAir) * 0.26f + upperEntrainment * 0.18f));
    fuel *= expf(-p.dt * (0.58f + heat * 0.20f + v * 0.92f + saturate(boundaryAir) * 0.18f));
    soot *= expf(-p.dt * (0.060f + v * 0.092f + oxygen * 0.028f + saturate(boundaryAir) * 0.96f + upperEntrainment * 0.22f));
    pyrolysisRate *= expf(-p.dt * (1.55f + v * 0.58f + saturate(boundaryAir) * 0.18f));

    const float uL = ldv(vel.u + uAt(g, x, y, z));
    const float uR = ldv(vel.u + uAt(g, x + 1, y, z));
    const float vD = ldv(vel.v + vAt(g, x, y, z));
    const float vU = ldv(vel.v + vAt(g, x, y + 1, z));
    const float wB = ldv(vel.w + wAt(g, x, y, z));
    const float wF = ldv(vel.w + wAt(g, x, y, z + 1));
    const float shear = fabsf(uR - uL) + fabsf(vU - vD) + fabsf(wF - wB);
    const float flameActivity = saturate(progress * 0.64f + burnMass * 5.2f + heat * 0.065f);
    turbulenceEnergy += p.dt * (shear * (0.72f + progress * 0.06f) + flameActivity * p.turbulence * 0.62f + frontProduction * 0.085f + soot * 0.018f);
    turbulenceEnergy *= expf(-p.dt * (0.54f + v * 0.24f + saturate(boundaryAir) * 0.42f + upperEntrainment * 0.16f));
    const float particleGrowth =
        saturate(incomplete * 0.36f + ash * 0.13f + soot * 0.055f + smoothstepf(0.65f, 1.55f, tempK / 1000.0f) * 0.18f);
    sootOptics = soot * (1.04f + 0.28f * sqrtf(fmaxf(0.0f, heat)) + 0.24f * ash + 0.46f * particleGrowth);
    sootOptics = lerpf(sootOptics, sootOptics * 0.48f, saturate(sootOxidation * 0.92f));

    stv(out.a + idx, make_float4(fminf(8.8f, fmaxf(0.0f, heat)), fminf(5.5f, fmaxf(0.0f, fuel)), fminf(1.0f, fmaxf(0.0f, oxygen)),
                             fminf(7.4f, fmaxf(0.0f, soot))));
    stv(out.b + idx, make_float4(fminf(2.8f, fmaxf(0.0f, charMass)), fminf(1.9f, fmaxf(0.0f, ash)), fminf(3.6f, fmaxf(0.0f, pyrolysisRate)),
                             fminf(3.4f, fmaxf(0.0f, progress))));
    stv(out.c + idx, make_float2(fminf(4.2f, fmaxf(0.0f, turbulenceEnergy)), fminf(10.0f, fmaxf(0.0f, sootOptics))));
}

// ---------------------------------------------------------------------------
// hash21 at every entry of the curl-noise lattices of this step (blockIdx.y
// selects the table).  The same function as the direct evaluation, so every
// table entry is the same bits as hashing its lattice point in place.
__global__ void __launch_bounds__(256) hashLatticeBuild(HashLattice2 a, HashLattice2 b) {
    const HashLattice2& L = blockIdx.y == 0 ? a : b;
    float* out = const_cast<float*>(L.values);
    const int total = L.offset[kFbmOctaves - 1] + L.sx[kFbmOctaves - 1] * L.sy[kFbmOctaves - 1];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        int o = 0;
        while (o + 1 < kFbmOctaves && i >= L.offset[o + 1]) ++o;
        const int local = i - L.offset[o];
        const int tx = local % L.sx[o];
        const int ty = local / L.sx[o];
        out[i] = hash21(static_cast<float>(L.ox[o] + tx), static_cast<float>(L.oy[o] + ty));
    }
}

// ---------------------------------------------------------------------------
// src/fire_cuda.cu:1128-1183 -- per-cell forcing.  Every face is read before
// any force is added; the per-cell increments go to `contrib` and the faces
// gather them (lower cell first), which makes the result deterministic.
__global__ void __launch_bounds__(128) forceContributions(float4* __restrict__ contrib, ScalarFieldsIn s, Velocity vel, FrameParams p,
                                                         HashLattice2 curlA, HashLattice2 curlB) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= p.nx) {
        return;
    }
    const Grid g{p.nx, p.ny, p.nz};
    const int idx = sAt(g, x, y, z);
    const float4 here = ldv(s.a + idx);
    const float h = here.x;
    const float sv = here.w;
    const float k = ldX(s.c + idx);
    const float c = ldW(s.b + idx);
    const float u = cellCoord(x, p.nx);
    const float v = cellCoord(y, p.ny);
    const float w = cellCoord(z, p.nz);
    auto heatAt = [&](int xx, int yy, int zz) { return ldX(s.a + sClamped(g, xx, yy, zz)); };
    const float gradX = heatAt(x + 1, y, z) - heatAt(x - 1, y, z);
    const float gradY = heatAt(x, y + 1, z) - heatAt(x, y - 1, z);
    const float gradZ = heatAt(x, y, z + 1) - heatAt(x, y, z - 1);
    const float uL = ldv(vel.u + uAt(g, x, y, z));
    const float uR = ldv(vel.u + uAt(g, x + 1, y, z));
    const float vD = ldv(vel.v + vAt(g, x, y, z));
    const float vU = ldv(vel.v + vAt(g, x, y + 1, z));
    const float wB = ldv(vel.w + wAt(g, x, y, z));
    const float wF = ldv(vel.w + wAt(g, x, y, z + 1));
    const float curlX = (wF - wB) - (vU - vD);
    const float curlY = (uR - uL) - (wF - wB);
    const float curlZ = (vU - vD) - (uR - uL);
    const float curlMagnitude = fabsf(curlX) + fabsf(curlY) + fabsf(curlZ);
    const float curlNoiseA = fbmLattice(u * 9.0f + w * 3.7f + p.time * 0.22f, v * 13.0f - p.time * 0.31f, curlA) - 0.5f;
    const float curlNoiseB = fbmLattice(w * 10.0f - p.time * 0.19f, u * 8.0f + v * 5.5f + p.time * 0.27f, curlB) - 0.5f;
    const float thermalActivity = smoothstepf(0.04f, 4.20f, h + sv * 0.28f);
    const float upperDrag = smoothstepf(0.26f, 0.94f, v);
    const float lesGain = sqrtf(fmaxf(0.0f, k)) * (0.30f + c * 0.54f);
    const int sc = p.sceneId;
    const float sceneCurlScale = sc == 2 ? 0.38f : (sc == 1 ? 1.18f : 1.0f);
    const float sceneBuoyancyScale = sc == 2 ? 0.42f : (sc == 1 ? 1.06f : 1.0f);
    const float curlGain = p.turbulence * sceneCurlScale * (0.18f + thermalActivity * 0.82f + lesGain * 1.12f);
    const float vortexGain = p.turbulence * sceneCurlScale * thermalActivity * saturate(curlMagnitude * 0.46f) * 0.68f;
    const float buoyancyFade = sc == 2 ? smoothstepf(0.24f, 0.035f, v) : smoothstepf(0.96f, 0.08f, v);
    const float verticalVelocity = 0.5f * (vD + vU);
    const float verticalDamping = verticalVelocity * (0.10f + upperDrag * 0.72f + sv * 0.020f);
    const float buoyancy =
        h * sceneBuoyancyScale * (1.62f + p.turbulence * 0.34f + c * 0.16f) * buoyancyFade - sv * 0.095f - gradY * 0.18f - verticalDamping;
    const float dv = p.dt * (buoyancy + curlY * vortexGain * 0.22f);
    const float du = p.dt * (p.wind * (0.34f + v * 0.96f) + (-gradZ * 1.36f + curlNoiseA * (0.20f + upperDrag * 0.16f) + curlX * vortexGain) * curlGain);
    const float dw = p.dt * ((gradX * 1.36f + curlNoiseB * (0.20f + upperDrag * 0.16f) + curlZ * vortexGain) * curlGain);
    contrib[idx] = make_float4(du, dv, dw, 0.0f);
}

namespace {

// Velocity of one face after the force gather and, optionally, the boundary
// clamp of src/fire_cuda.cu:1261-1291.
__device__ __forceinline__ float forcedU(const FaceT* __restrict__ u, const float4* __restrict__ contrib, const Grid& g, int x, int y,
                                         int z, bool clampWalls) {
    float val = ldv(u + uAt(g, x, y, z));
    if (x > 0) val += __ldg(&contrib[sAt(g, x - 1, y, z)].x);
    if (x < g.nx) val += __ldg(&contrib[sAt(g, x, y, z)].x);
    if (clampWalls) val = (x == 0 || x == g.nx) ? 0.0f : fminf(4.0f, fmaxf(-4.0f, val));
    return val;
}
__device__ __forceinline__ float forcedV(const FaceT* __restrict__ v, const float4* __restrict__ contrib, const Grid& g, int x, int y,
                                         int z, bool clampWalls) {
    float val = ldv(v + vAt(g, x, y, z));
    if (y > 0) val += __ldg(&contrib[sAt(g, x, y - 1, z)].y);
    if (clampWalls) val = y == 0 ? 0.0f : fminf(6.4f, fmaxf(-0.9f, val));
    return val;
}
__device__ __forceinline__ float forcedW(const FaceT* __restrict__ w, const float4* __restrict__ contrib, const Grid& g, int x, int y,
                                         int z, bool clampWalls) {
    float val = ldv(w + wAt(g, x, y, z));
    if (z > 0) val += __ldg(&contrib[sAt(g, x, y, z - 1)].z);
    if (z < g.nz) val += __ldg(&contrib[sAt(g, x, y, z)].z);
    if (clampWalls) val = (z == 0 || z == g.nz) ? 0.0f : fminf(4.0f, fmaxf(-4.0f, val));
    return val;
}

}  // namespace

// The force gather alone (stage "force"): every face adds its cells' increments.
__global__ void __launch_bounds__(256) forceApply(FaceT* __restrict__ uOut, FaceT* __restrict__ vOut, FaceT* __restrict__ wOut,
                                                  const float4* __restrict__ contrib, Velocity vel, FrameParams p) {
    const int cx = blockIdx.x * blockDim.x + threadIdx.x;
    if (cx >= p.nx) return;
    const Grid g{p.nx, p.ny, p.nz};
    facesOfCell(p, cx, blockIdx.y, blockIdx.z, [&](int x, int y, int z) {
        if (x <= p.nx && y < p.ny && z < p.nz) stv(uOut + uAt(g, x, y, z), forcedU(vel.u, contrib, g, x, y, z, false));
        if (x < p.nx && y <= p.ny && z < p.nz) stv(vOut + vAt(g, x, y, z), forcedV(vel.v, contrib, g, x, y, z, false));
        if (x < p.nx && y < p.ny && z <= p.nz) stv(wOut + wAt(g, x, y, z), forcedW(vel.w, contrib, g, x, y, z, false));
    });
}

// Fused force gather + boundary clamp + divergence (+ pressure reset): one cell
// per thread computes its six faces, writes the faces it owns (lower faces, and
// the upper ones on the last layer) and div = -(sum of differences).
__global__ void __launch_bounds__(256) forceProjectSetup(FaceT* __restrict__ uOut, FaceT* __restrict__ vOut, FaceT* __restrict__ wOut,
                                                         float* __restrict__ divergence, float* __restrict__ pressure,
                                                         const float4* __restrict__ contrib, Velocity vel, FrameParams p) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= p.nx) {
        return;
    }
    const Grid g{p.nx, p.ny, p.nz};
    const float uL = forcedU(vel.u, contrib, g, x, y, z, true);
    const float uR = forcedU(vel.u, contrib, g, x + 1, y, z, true);
    const float vD = forcedV(vel.v, contrib, g, x, y, z, true);
    const float vU = forcedV(vel.v, contrib, g, x, y + 1, z, true);
    const float wB = forcedW(vel.w, contrib, g, x, y, z, true);
    const float wF = forcedW(vel.w, contrib, g, x, y, z + 1, true);
    stv(uOut + uAt(g, x, y, z), uL);
    stv(vOut + vAt(g, x, y, z), vD);
    stv(wOut + wAt(g, x, y, z), wB);
    if (x == p.nx - 1) stv(uOut + uAt(g, x + 1, y, z), uR);
    if (y == p.ny - 1) stv(vOut + vAt(g, x, y + 1, z), vU);
    if (z == p.nz - 1) stv(wOut + wAt(g, x, y, z + 1), wF);
    const float div = uR - uL + vU - vD + wF - wB;
    const int idx = sAt(g, x, y, z);
    divergence[idx] = -div;
    pressure[idx] = 0.0f;
}

// src/fire_cuda.cu:1261-1317 -- wall zeroing, with (clampValues) or without the value clamps.
__global__ void __launch_bounds__(256) velocityBoundary(FaceT* __restrict__ u, FaceT* __restrict__ v, FaceT* __restrict__ w,
                                                        FrameParams p, int clampValues) {
    const int cx = blockIdx.x * blockDim.x + threadIdx.x;
    if (cx >= p.nx) return;
    const Grid g{p.nx, p.ny, p.nz};
    facesOfCell(p, cx, blockIdx.y, blockIdx.z, [&](int x, int y, int z) {
    if (x <= p.nx && y < p.ny && z < p.nz) {
        FaceT* f = u + uAt(g, x, y, z);
        if (x == 0 || x == p.nx) stv(f, 0.0f);
        else if (clampValues) stv(f, fminf(4.0f, fmaxf(-4.0f, ldv(f))));
    }
    if (x < p.nx && y <= p.ny && z < p.nz) {
        FaceT* f = v + vAt(g, x, y, z);
        if (y == 0) stv(f, 0.0f);
        else if (clampValues) stv(f, fminf(6.4f, fmaxf(-0.9f, ldv(f))));
    }
    if (x < p.nx && y < p.ny && z <= p.nz) {
        FaceT* f = w + wAt(g, x, y, z);
        if (z == 0 || z == p.nz) stv(f, 0.0f);
        else if (clampValues) stv(f, fminf(4.0f, fmaxf(-4.0f, ldv(f))));
    }
    });
}

// src/fire_cuda.cu:1185-1199 / :1247-1259.
__global__ void __launch_bounds__(256) divergenceOf(float* __restrict__ divergence, float* __restrict__ pressureOrNull, Velocity vel,
                                                    FrameParams p) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= p.nx) {
        return;
    }
    const Grid g{p.nx, p.ny, p.nz};
    const float div = ldv(vel.u + uAt(g, x + 1, y, z)) - ldv(vel.u + uAt(g, x, y, z)) + ldv(vel.v + vAt(g, x, y + 1, z)) -
                      ldv(vel.v + vAt(g, x, y, z)) + ldv(vel.w + wAt(g, x, y, z + 1)) - ldv(vel.w + wAt(g, x, y, z));
    const int idx = sAt(g, x, y, z);
    divergence[idx] = -div;
    if (pressureOrNull != nullptr) pressureOrNull[idx] = 0.0f;
}

// ---------------------------------------------------------------------------
// The solve for grids too large to stay in shared memory: p and div are copied
// once per solve into colour-split arrays (colour c, row (y, z), slot k holds
// x = 2k + ((c + y + z) & 1)), so every half sweep reads the other colour and
// reads and writes its own colour in contiguous runs; the natural layout of the
// reference's kernel reads both colours and writes every other float.  The
// update is the reference's arithmetic in the reference's order
// (src/fire_cuda.cu:1201-1227), so the result is the same bits.
__global__ void __launch_bounds__(256) sorSplitPack(float* __restrict__ split, float* __restrict__ splitDiv, const float* __restrict__ pressure,
                                                    const float* __restrict__ divergence, SplitGrid s) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z % s.nz;
    const int c = blockIdx.z / s.nz;
    const int x = 2 * k + ((c + y + z) & 1);
    if (k >= s.H || x >= s.nx) return;
    const int src = (z * s.ny + y) * s.nx + x;
    split[splitIdx(s, c, y, z, k)] = __ldg(pressure + src);
    splitDiv[splitIdx(s, c, y, z, k)] = __ldg(divergence + src);
}

__global__ void __launch_bounds__(256) sorSplitUnpack(float* __restrict__ pressure, const float* __restrict__ split, SplitGrid s) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z % s.nz;
    const int c = blockIdx.z / s.nz;
    const int x = 2 * k + ((c + y + z) & 1);
    if (k >= s.H || x >= s.nx) return;
    pressure[(z * s.ny + y) * s.nx + x] = __ldg(split + splitIdx(s, c, y, z, k));
}

// The four cells in slots k0..k0+3 of one colour-c row (y, z) of the split
// arrays (own: this colour, other: the other colour, i: the row start + k0):
// their values and the sums div + pL + pR + pD + pU + pB + pF, in the
// reference's order (src/fire_cuda.cu:1201-1227), with Neumann walls (the cell
// itself).  Own cells, their div and the four other-colour rows beside them
// are one float4 each; the x-neighbours are the other colour's float4 of the
// same row shifted by one slot (sx = 0: left = slot k - 1, right = slot k;
// sx = 1: left = slot k, right = slot k + 1), whose missing end is one scalar.
__device__ __forceinline__ void splitQuad(const float* __restrict__ own, const float* __restrict__ other, const float* __restrict__ div,
                                          int i, int k0, int sx, int y, int z, const SplitGrid& s, float self[4], float sum[4]) {
    const int plane = s.ny * s.P;
    const float4 me = *reinterpret_cast<const float4*>(own + i);
    const float4 mid = __ldg(reinterpret_cast<const float4*>(other + i));
    const float4 dn = y == 0 ? me : __ldg(reinterpret_cast<const float4*>(other + i - s.P));
    const float4 up = y == s.ny - 1 ? me : __ldg(reinterpret_cast<const float4*>(other + i + s.P));
    const float4 bk = z == 0 ? me : __ldg(reinterpret_cast<const float4*>(other + i - plane));
    const float4 ft = z == s.nz - 1 ? me : __ldg(reinterpret_cast<const float4*>(other + i + plane));
    const float4 dv = __ldg(reinterpret_cast<const float4*>(div + i));
    float edge = 0.0f;
    if (sx == 0 && k0 > 0) edge = __ldg(other + i - 1);
    if (sx == 1 && 2 * (k0 + 4) < s.nx) edge = __ldg(other + i + 4);
    const float sv[4] = {me.x, me.y, me.z, me.w};
    const float mv[4] = {mid.x, mid.y, mid.z, mid.w};
    const float dnv[4] = {dn.x, dn.y, dn.z, dn.w};
    const float upv[4] = {up.x, up.y, up.z, up.w};
    const float bkv[4] = {bk.x, bk.y, bk.z, bk.w};
    const float ftv[4] = {ft.x, ft.y, ft.z, ft.w};
    const float dvv[4] = {dv.x, dv.y, dv.z, dv.w};
    const int x0 = 2 * k0 + sx;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int x = x0 + 2 * j;
        const float c = sv[j];
        const float left = sx == 0 ? (j == 0 ? edge : mv[j - 1]) : mv[j];
        const float right = sx == 0 ? mv[j] : (j == 3 ? edge : mv[j + 1]);
        const float pL = x == 0 ? c : left;
        const float pR = x == s.nx - 1 ? c : right;
        const float pD = y == 0 ? c : dnv[j];
        const float pU = y == s.ny - 1 ? c : upv[j];
        const float pB = z == 0 ? c : bkv[j];
        const float pF = z == s.nz - 1 ? c : ftv[j];
        self[j] = c;
        sum[j] = dvv[j] + pL + pR + pD + pU + pB + pF;
    }
}

// One colour of a half sweep on the split arrays: thread (t, y, z) updates
// the four slots 4t..4t+3 of colour c in row (y, z).  own and other are the
// two colour halves of one split array: disjoint, and other is read-only for
// the whole launch.
__global__ void __launch_bounds__(128) sorSplitHalfSweep(float* __restrict__ own, const float* __restrict__ other,
                                                         const float* __restrict__ ownDiv, SplitGrid s, int c, float omega,
                                                         const int* skip) {
    // The gate is written only between launches, so every SM may cache it.
    if (skip != nullptr && __ldg(skip) != 0) return;
    const int k0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (k0 >= s.H || y >= s.ny) return;
    const int sx = (c + y + z) & 1;
    const int x0 = 2 * k0 + sx;
    const int i = (z * s.ny + y) * s.P + k0;
    float self[4], sum[4], out[4];
    splitQuad(own, other, ownDiv, i, k0, sx, y, z, s, self, sum);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float projected = sum[j] * (1.0f / 6.0f);
        out[j] = x0 + 2 * j < s.nx ? self[j] + omega * (projected - self[j]) : self[j];
    }
    *reinterpret_cast<float4*>(own + i) = make_float4(out[0], out[1], out[2], out[3]);
}

// Residual of the split arrays, as sorResidualPartials: each warp takes whole
// rows (colour, y, z); lane l covers the slot groups 4l, 4l + 128, ... of a row.
__global__ void __launch_bounds__(kResidualThreads) sorSplitResidualPartials(const float* __restrict__ split,
                                                                            const float* __restrict__ splitDiv, SplitGrid s,
                                                                            const SorGate* gate, double* __restrict__ partialSq,
                                                                            float* __restrict__ partialMax) {
    if (gate->converged) return;
    const int lane = threadIdx.x & 31;
    const int warps = kResidualThreads / 32;
    const int rowsPerColour = s.ny * s.nz;
    const int colour = s.nz * s.ny * s.P;
    double acc = 0.0;
    float m = 0.0f;
    for (int row = blockIdx.x * warps + (threadIdx.x >> 5); row < 2 * rowsPerColour; row += gridDim.x * warps) {
        const int c = row / rowsPerColour;
        const int yz = row - c * rowsPerColour;
        const int y = yz % s.ny;
        const int z = yz / s.ny;
        const int sx = (c + y + z) & 1;
        const float* own = split + c * colour;
        const float* other = split + (1 - c) * colour;
        const float* dv = splitDiv + c * colour;
        for (int k0 = 4 * lane; k0 < s.H; k0 += 128) {
            float self[4], sum[4];
            splitQuad(own, other, dv, yz * s.P + k0, k0, sx, y, z, s, self, sum);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (2 * (k0 + j) + sx >= s.nx || k0 + j >= s.H) continue;
                const float r = __fsub_rn(sum[j], __fmul_rn(6.0f, self[j]));
                m = fmaxf(m, fabsf(r));
                acc += static_cast<double>(r) * static_cast<double>(r);
            }
        }
    }
    __shared__ double sq[kResidualThreads];
    __shared__ float mx[kResidualThreads];
    sq[threadIdx.x] = acc;
    mx[threadIdx.x] = m;
    __syncthreads();
    for (int w = kResidualThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            sq[threadIdx.x] += sq[threadIdx.x + w];
            mx[threadIdx.x] = fmaxf(mx[threadIdx.x], mx[threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partialSq[blockIdx.x] = sq[0];
        partialMax[blockIdx.x] = mx[0];
    }
}

// src/fire_cuda.cu:1229-1245 + :1293-1317 -- u -= grad p on interior faces,
// then the wall faces are zeroed (doSubtract / doWalls select either half).
__global__ void __launch_bounds__(256) subtractWall(FaceT* __restrict__ u, FaceT* __restrict__ v, FaceT* __restrict__ w,
                                                    const float* __restrict__ pressure, FrameParams p, int doSubtract, int doWalls) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= p.nx) {
        return;
    }
    const Grid g{p.nx, p.ny, p.nz};
    const int idx = sAt(g, x, y, z);
    if (doSubtract) {
        const float pc = __ldg(pressure + idx);
        if (x > 0) stv(u + uAt(g, x, y, z), ldv(u + uAt(g, x, y, z)) - (pc - __ldg(pressure + idx - 1)));
        if (y > 0) stv(v + vAt(g, x, y, z), ldv(v + vAt(g, x, y, z)) - (pc - __ldg(pressure + idx - g.nx)));
        if (z > 0) stv(w + wAt(g, x, y, z), ldv(w + wAt(g, x, y, z)) - (pc - __ldg(pressure + idx - g.nx * g.ny)));
    }
    if (doWalls) {
        if (x == 0) stv(u + uAt(g, 0, y, z), 0.0f);
        if (x == p.nx - 1) stv(u + uAt(g, p.nx, y, z), 0.0f);
        if (y == 0) stv(v + vAt(g, x, 0, z), 0.0f);
        if (z == 0) stv(w + wAt(g, x, y, 0), 0.0f);
        if (z == p.nz - 1) stv(w + wAt(g, x, y, p.nz), 0.0f);
    }
}

}  // namespace firesim

namespace firesim {

// ---------------------------------------------------------------------------
// Shared-memory-resident red-black SOR: all 2N half sweeps in one cooperative
// launch.  Each CTA owns one brick of BX*BY*BZ cells (all even, so a brick's
// colour pattern equals the global one) and keeps its p and div in shared
// memory, split by colour: for colour c, row (y, z) holds the cells
// x = 2k + ((c + y + z) & 1), k = 0..BX/2-1, so a cell's x/y/z-neighbour reads
// of the other colour are unit-stride.  Each thread owns one (k, y) column
// of both colours and walks z.  A half sweep publishes its updated face cells
// as tagged 64-bit words (value, half sweep) in an exchange array
// (ResidentSync); a neighbour that needs them polls those words until the tag
// matches -- no grid-wide barrier, no flags, no fences -- and copies them into
// its one-cell halo.  The cooperative launch guarantees that all bricks are
// resident, so every poll is for a running CTA; each poll is still bounded in
// time.  Walls are Neumann through the clamped neighbour (the cell itself), as
// in sorPressureParityKernel.  Per-cell arithmetic is identical to
// sorSplitHalfSweep, so the result is bit-identical to the split path.
namespace {

__device__ __forceinline__ unsigned loadVolatile(const unsigned* p) { return *reinterpret_cast<const volatile unsigned*>(p); }
__device__ __forceinline__ void storeVolatile(unsigned* p, unsigned v) { *reinterpret_cast<volatile unsigned*>(p) = v; }
__device__ __forceinline__ unsigned long long globalTimerNs() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned long long loadExchange(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void storeExchange(unsigned long long* p, float value, unsigned tag) {
    const unsigned long long v = (static_cast<unsigned long long>(__float_as_uint(value)) << 32) | tag;
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Bounded poll of the halo words whose prefetched copy was stale (bit j of
// `stale`: words[j], at exchange + cell[j]) until each carries tag `want`;
// every round reloads all words still stale, so their L2 round trips overlap.
// False when the poll ran out (time or kResidentMaxPolls rounds) or another
// brick's did.
template <int N>
__device__ __forceinline__ bool residentAwait(unsigned long long (&words)[N], const int (&cell)[N], unsigned stale, unsigned want,
                                              const ResidentSync& sync, int brick) {
    const unsigned failTag = sync.epoch + 1u;
    unsigned long long start = 0;
    for (unsigned n = 0; n < kResidentMaxPolls; ++n) {
#pragma unroll
        for (int j = 0; j < N; ++j) {
            if (stale & (1u << j)) {
                const unsigned long long w = loadExchange(sync.exchange + cell[j]);
                if (static_cast<unsigned>(w) == want) {
                    words[j] = w;
                    stale &= ~(1u << j);
                }
            }
        }
        if (stale == 0) {
            return true;
        }
        if ((n & 15u) == 15u) {
            if (loadVolatile(sync.status) == failTag) {
                return false;
            }
            const unsigned long long now = globalTimerNs();
            if (start == 0) {
                start = now;
            } else if (now - start > sync.waitNs) {
                break;
            }
            __nanosleep(64);
        }
    }
    storeVolatile(sync.status, failTag);
    storeVolatile(sync.hostStatus, static_cast<unsigned>(brick) + 1u);
    __threadfence_system();
    return false;
}

// Halo cells of one colour: both x faces (BY*BZ/2 each), both y faces
// (KX*BZ each), both z faces (KX*BY each).
template <int BX, int BY, int BZ>
struct ResidentShape {
    static constexpr int KX = BX / 2;
    // A warp covers KX cells of each of RPW rows y0, y0 + 2, ...: rows of the
    // same parity, so all of its lanes read at the same x shift.  The row
    // pitch EX is padded until 2 * EX == KX (mod 32), which puts those rows
    // in disjoint bank windows: every shared access of the update is
    // conflict-free.
    static constexpr int RPW = 32 / KX;
    static constexpr int EX = ((KX + 2) + ((KX / 2 - (KX + 2) % 16) % 16 + 16) % 16);
    static constexpr int EY = BY + 2, EZ = BZ + 2;
    static constexpr int PLANE = EZ * EY * EX;
    static constexpr int THREADS = KX * BY;
    // div plane pitch: one z plane apart is 16 banks apart, so a warp that
    // reads two z rows of face cells (the y faces) does not conflict.
    static constexpr int DPITCH = THREADS + 16;
    static constexpr size_t SHARED_BYTES = (2ull * PLANE + 2ull * BZ * DPITCH) * sizeof(float);
    static_assert((2 * EX) % 32 == KX % 32 && EX >= KX + 2, "row pitch");
    static_assert(BY % (2 * RPW) == 0 && THREADS % 32 == 0, "warp-to-row mapping");
    static constexpr int HX = BY * BZ;
    static constexpr int HY = 2 * KX * BZ;
    static constexpr int HZ = 2 * KX * BY;
    static constexpr int HALO = HX + HY + HZ;
    static constexpr int PER_THREAD = (HALO + THREADS - 1) / THREADS;
    __device__ static int pidx(int c, int z, int y, int k) { return c * PLANE + ((z + 1) * EY + (y + 1)) * EX + (k + 1); }
    // div of the thread's own cells, laid out by thread: [colour][z][thread].
    __device__ static int didx(int c, int z, int t) { return (c * BZ + z) * DPITCH + t; }
};

// Global and shared index of halo cell i of colour c, or gi = -1 when the
// cell lies outside the grid (a wall: the update uses the cell itself).
template <int BX, int BY, int BZ>
__device__ __forceinline__ void residentHaloCell(int i, int c, int ox, int oy, int oz, const Grid& g, int& gi, int& si) {
    using S = ResidentShape<BX, BY, BZ>;
    int lx, ly, lz, k;
    if (i < S::HX) {
        const int side = i / (S::HX / 2);
        const int r = i % (S::HX / 2);
        lz = r / (BY / 2);
        lx = side ? BX : -1;
        ly = 2 * (r % (BY / 2)) + ((c + lx + lz) & 1);
        k = side ? S::KX : -1;
    } else if (i < S::HX + S::HY) {
        const int j = i - S::HX;
        const int side = j / (S::KX * BZ);
        const int r = j % (S::KX * BZ);
        k = r % S::KX;
        lz = r / S::KX;
        ly = side ? BY : -1;
        lx = 2 * k + ((c + ly + lz) & 1);
    } else {
        const int j = i - S::HX - S::HY;
        const int side = j / (S::KX * BY);
        const int r = j % (S::KX * BY);
        k = r % S::KX;
        ly = r / S::KX;
        lz = side ? BZ : -1;
        lx = 2 * k + ((c + ly + lz) & 1);
    }
    const int gx = ox + lx, gy = oy + ly, gz = oz + lz;
    si = S::pidx(c, lz, ly, k);
    gi = (gx >= 0 && gx < g.nx && gy >= 0 && gy < g.ny && gz >= 0 && gz < g.nz) ? (gz * g.ny + gy) * g.nx + gx : -1;
}

// Face cells of one colour in a brick, updated after the halo has arrived:
// both z faces (all k, y: each thread takes its own column at z = 0 and
// z = BZ - 1), and from a list shared out over the threads, both y faces
// (inner z) and in every inner (y, z) row the one x-face cell of that colour
// (x = 0 when the row's offset is 0, else x = BX - 1).  All other cells of
// the colour are the brick interior, whose neighbours all lie in the brick.
template <int BX, int BY, int BZ>
struct ResidentFaces {
    static constexpr int KX = BX / 2;
    static constexpr int FY = 2 * KX * (BZ - 2);
    static constexpr int FX = (BY - 2) * (BZ - 2);
    static constexpr int COUNT = FY + FX;  // the z faces are each thread's own column (z = 0, BZ - 1)
    static constexpr int PER_THREAD = (COUNT + KX * BY - 1) / (KX * BY);
};

// Row y of thread t in the conflict-free warp mapping (see ResidentShape), and its inverse.
template <int BX, int BY, int BZ>
__device__ __forceinline__ void residentColumn(int t, int& k, int& y) {
    using S = ResidentShape<BX, BY, BZ>;
    const int lane = t & 31, warp = t >> 5;
    k = lane % S::KX;
    y = (warp >> 1) * 2 * S::RPW + (warp & 1) + 2 * (lane / S::KX);
}
template <int BX, int BY, int BZ>
__device__ __forceinline__ int residentOwner(int k, int y) {
    using S = ResidentShape<BX, BY, BZ>;
    const int q = y / (2 * S::RPW), rem = y % (2 * S::RPW);
    return (2 * q + (rem & 1)) * 32 + (rem >> 1) * S::KX + k;
}

// (k, y, z) of face cell i of colour c, packed k | y << 8 | z << 16.
template <int BX, int BY, int BZ>
__device__ __forceinline__ int residentFaceCell(int i, int c) {
    using F = ResidentFaces<BX, BY, BZ>;
    int k, y, z;
    if (i < F::FY) {
        const int j = i;
        const int side = j / (F::KX * (BZ - 2));
        const int r = j % (F::KX * (BZ - 2));
        k = r % F::KX;
        z = 1 + r / F::KX;
        y = side ? BY - 1 : 0;
    } else {
        const int j = i - F::FY;
        y = 1 + j % (BY - 2);
        z = 1 + j / (BY - 2);
        k = ((c + y + z) & 1) ? F::KX - 1 : 0;
    }
    return k | (y << 8) | (z << 16);
}

// Interior cells of colour C in z0 <= z < z1 of this thread's column.  Their
// neighbours all lie in the brick; only in a brick that the grid's upper
// walls cut (FULL == false) can a neighbour lie past a wall.
template <int BX, int BY, int BZ, int C, int Z0, int Z1, bool FULL>
__device__ __forceinline__ void residentInterior(float* planes, const float* divs, int k, int y, int ox, int oy, int oz, const Grid& g,
                                                 float omega) {
    using S = ResidentShape<BX, BY, BZ>;
    constexpr int O = 1 - C;
    if (y == 0 || y == BY - 1) return;
    const int gy = oy + y;
    if (!FULL && gy >= g.ny) return;
    // The two colour planes never overlap: stores to this colour cannot
    // change the other colour's values, so their loads may run ahead.
    float* __restrict__ mine = planes + C * S::PLANE;
    const float* __restrict__ other = planes + O * S::PLANE;
    const float* __restrict__ dv = divs;
    auto at = [](int z, int yy, int kk) { return ((z + 1) * S::EY + (yy + 1)) * S::EX + (kk + 1); };
    const int sy = (C + y) & 1;
    // The other colour's (y, k) column at z - 1, z, z + 1 slides along z in
    // registers: it is the back, front and one of the x neighbours.
    float below = other[at(Z0 - 1, y, k)];
    float centre = other[at(Z0, y, k)];
#pragma unroll
    for (int z = Z0; z < Z1; ++z) {
        const float above = other[at(z + 1, y, k)];
        const int s = sy ^ (z & 1);
        const int x = 2 * k + s;
        const int gx = ox + x, gz = oz + z;
        if (x != 0 && x != BX - 1 && (FULL || (gx < g.nx && gz < g.nz))) {
            const float self = mine[at(z, y, k)];
            const float side = other[at(z, y, s ? k + 1 : k - 1)];
            const float pL = s ? centre : side;
            const float pR = (!FULL && gx == g.nx - 1) ? self : (s ? side : centre);
            const float pD = other[at(z, y - 1, k)];
            const float pU = (!FULL && gy == g.ny - 1) ? self : other[at(z, y + 1, k)];
            const float pB = below;
            const float pF = (!FULL && gz == g.nz - 1) ? self : above;
            const float d = dv[S::didx(C, z, threadIdx.x)];
            const float projected = (d + pL + pR + pD + pU + pB + pF) * (1.0f / 6.0f);
            mine[at(z, y, k)] = self + omega * (projected - self);
        }
        below = centre;
        centre = above;
    }
}

template <int BX, int BY, int BZ, int C, int Z0, int Z1>
__device__ __forceinline__ void residentInteriorAny(bool full, float* planes, const float* divs, int k, int y, int ox, int oy, int oz,
                                                    const Grid& g, float omega) {
    if (full) {
        residentInterior<BX, BY, BZ, C, Z0, Z1, true>(planes, divs, k, y, ox, oy, oz, g, omega);
    } else {
        residentInterior<BX, BY, BZ, C, Z0, Z1, false>(planes, divs, k, y, ox, oy, oz, g, omega);
    }
}

}  // namespace

// One half sweep h (colour c) of a brick runs as
//   interior cells, first three quarters of z
//   issue the loads of the neighbours' face cells (colour 1 - c) of half
//     sweep h - 1 from the tagged exchange words
//   interior cells, last quarter of z     (hides the loads' latency)
//   words whose tag is not yet h: poll them, all together each round, until
//     every tag is h; values -> halo; barrier
//   face cells, each also published as a tagged word; barrier
// so the exchange overlaps the interior update and costs one L2 round trip.
// For a 40-iteration 128^3 solve: issuing the loads after three quarters of
// the interior rather than half (the neighbours' stores have longer to land)
// took 256 -> 250 us, and polling a thread's stale words together rather
// than one after another 250 -> 238 us.
template <int BX, int BY, int BZ>
__global__ void __launch_bounds__((BX / 2) * BY, 2) sorResident(float* __restrict__ pressure, const float* __restrict__ divergence, Grid g,
                                                               ResidentBrick r, ResidentSync sync, int iterations, float omega) {
    using S = ResidentShape<BX, BY, BZ>;
    using F = ResidentFaces<BX, BY, BZ>;
    constexpr int ZMID = 3 * BZ / 4;
    if (sync.skip != nullptr && *reinterpret_cast<const volatile int*>(sync.skip) != 0) {
        return;  // an earlier chunk of this solve converged (the same word for every block)
    }
    extern __shared__ float smem[];
    float* planes = smem;                // [2][EZ][EY][EX]
    float* divs = smem + 2 * S::PLANE;   // [2][BZ][THREADS]
    const int brick = blockIdx.x;
    const int bi = brick % r.nbx, bj = (brick / r.nbx) % r.nby, bk = brick / (r.nbx * r.nby);
    const int ox = bi * BX;
    const int oy = bj * BY;
    const int oz = bk * BZ;
    const bool full = ox + BX <= g.nx && oy + BY <= g.ny && oz + BZ <= g.nz;
    const bool silent = brick == sync.silentBrick;
    int k, y;
    residentColumn<BX, BY, BZ>(threadIdx.x, k, y);
    const int gy = oy + y;

    // This thread's halo cells and face cells of each colour, fixed for the whole solve.
    int haloG[2][S::PER_THREAD], haloS[2][S::PER_THREAD], face[2][F::PER_THREAD];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
#pragma unroll
        for (int j = 0; j < S::PER_THREAD; ++j) {
            const int i = threadIdx.x + j * S::THREADS;
            haloG[c][j] = -1;
            haloS[c][j] = 0;
            if (i < S::HALO) {
                residentHaloCell<BX, BY, BZ>(i, c, ox, oy, oz, g, haloG[c][j], haloS[c][j]);
            }
        }
#pragma unroll
        for (int j = 0; j < F::PER_THREAD; ++j) {
            const int i = threadIdx.x + j * S::THREADS;
            face[c][j] = i < F::COUNT ? residentFaceCell<BX, BY, BZ>(i, c) : -1;
        }
    }

    // Load both colours of the brick column, then the halo.
#pragma unroll 4
    for (int z = 0; z < BZ; ++z) {
        const int gz = oz + z;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const int gx = ox + 2 * k + ((c + y + z) & 1);
            if (gx < g.nx && gy < g.ny && gz < g.nz) {
                const int gi = (gz * g.ny + gy) * g.nx + gx;
                planes[S::pidx(c, z, y, k)] = __ldcg(pressure + gi);
                divs[S::didx(c, z, threadIdx.x)] = __ldg(divergence + gi);
            }
        }
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
#pragma unroll
        for (int j = 0; j < S::PER_THREAD; ++j) {
            if (haloG[c][j] >= 0) planes[haloS[c][j]] = __ldcg(pressure + haloG[c][j]);
        }
    }
    __syncthreads();

    for (int it = 0; it < iterations; ++it) {
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const int o = 1 - c;
            const int h = 2 * it + c;
            const bool last = it == iterations - 1 && c == 1;
            if (c == 0) {
                residentInteriorAny<BX, BY, BZ, 0, 1, ZMID>(full, planes, divs, k, y, ox, oy, oz, g, omega);
            } else {
                residentInteriorAny<BX, BY, BZ, 1, 1, ZMID>(full, planes, divs, k, y, ox, oy, oz, g, omega);
            }
            // The neighbours' face cells of colour o from half sweep h - 1, in flight during the second half.
            unsigned long long haloW[S::PER_THREAD];
            const unsigned want = sync.epoch + static_cast<unsigned>(h);
            if (h > 0) {
#pragma unroll
                for (int j = 0; j < S::PER_THREAD; ++j) {
                    haloW[j] = haloG[o][j] >= 0 ? loadExchange(sync.exchange + haloG[o][j]) : 0ull;
                }
            }
            if (c == 0) {
                residentInteriorAny<BX, BY, BZ, 0, ZMID, BZ - 1>(full, planes, divs, k, y, ox, oy, oz, g, omega);
            } else {
                residentInteriorAny<BX, BY, BZ, 1, ZMID, BZ - 1>(full, planes, divs, k, y, ox, oy, oz, g, omega);
            }
            bool failed = false;
            if (h > 0) {
                unsigned stale = 0;
#pragma unroll
                for (int j = 0; j < S::PER_THREAD; ++j) {
                    if (haloG[o][j] >= 0 && static_cast<unsigned>(haloW[j]) != want) stale |= 1u << j;
                }
                if (stale != 0) {
                    failed = !residentAwait(haloW, haloG[o], stale, want, sync, brick);
                }
#pragma unroll
                for (int j = 0; j < S::PER_THREAD; ++j) {
                    if (haloG[o][j] >= 0) planes[haloS[o][j]] = __uint_as_float(static_cast<unsigned>(haloW[j] >> 32));
                }
            }
            if (__syncthreads_or(failed)) {
                return;
            }
            // Face cells, with the walls of the grid.
            float* __restrict__ mineF = planes + c * S::PLANE;
            const float* __restrict__ otherF = planes + o * S::PLANE;
            const float* __restrict__ divF = divs;
            auto faceUpdate = [&](int fk, int fy, int fz, int owner) {
                const int s = (c + fy + fz) & 1;
                const int fx = 2 * fk + s;
                const int gx = ox + fx, fgy = oy + fy, gz = oz + fz;
                if (gx >= g.nx || fgy >= g.ny || gz >= g.nz) return;
                const float self = mineF[S::pidx(0, fz, fy, fk)];
                const float pL = gx == 0 ? self : otherF[S::pidx(0, fz, fy, fk + s - 1)];
                const float pR = gx == g.nx - 1 ? self : otherF[S::pidx(0, fz, fy, fk + s)];
                const float pD = fgy == 0 ? self : otherF[S::pidx(0, fz, fy - 1, fk)];
                const float pU = fgy == g.ny - 1 ? self : otherF[S::pidx(0, fz, fy + 1, fk)];
                const float pB = gz == 0 ? self : otherF[S::pidx(0, fz - 1, fy, fk)];
                const float pF = gz == g.nz - 1 ? self : otherF[S::pidx(0, fz + 1, fy, fk)];
                const float d = divF[S::didx(c, fz, owner)];
                const float projected = (d + pL + pR + pD + pU + pB + pF) * (1.0f / 6.0f);
                const float next = self + omega * (projected - self);
                mineF[S::pidx(0, fz, fy, fk)] = next;
                if (!last && !silent) {
                    storeExchange(sync.exchange + (gz * g.ny + fgy) * g.nx + gx, next, sync.epoch + static_cast<unsigned>(h + 1));
                }
            };
            faceUpdate(k, y, 0, threadIdx.x);
            faceUpdate(k, y, BZ - 1, threadIdx.x);
#pragma unroll
            for (int j = 0; j < F::PER_THREAD; ++j) {
                const int cell = face[c][j];
                if (cell < 0) continue;
                const int fk = cell & 0xff, fy = (cell >> 8) & 0xff;
                faceUpdate(fk, fy, cell >> 16, residentOwner<BX, BY, BZ>(fk, fy));
            }
            if (last) {
                break;
            }
            __syncthreads();
        }
    }
    __syncthreads();
#pragma unroll 4
    for (int z = 0; z < BZ; ++z) {
        const int gz = oz + z;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const int gx = ox + 2 * k + ((c + y + z) & 1);
            if (gx < g.nx && gy < g.ny && gz < g.nz) {
                pressure[(gz * g.ny + gy) * g.nx + gx] = planes[S::pidx(c, z, y, k)];
            }
        }
    }
}

// Residual of the red-black system, per block over a fixed set of cells
// (grid-stride with a fixed grid), so the reduction order never changes.
__global__ void __launch_bounds__(kResidualThreads) sorResidualPartials(const float* __restrict__ pressure,
                                                                       const float* __restrict__ divergence, Grid g,
                                                                       const SorGate* gate, double* __restrict__ partialSq,
                                                                       float* __restrict__ partialMax) {
    if (gate->converged) return;
    // Each warp takes whole rows (y, z); its lanes stride along x.  Every
    // partial sums a fixed set of cells in a fixed order.
    const int lane = threadIdx.x & 31;
    const int warps = kResidualThreads / 32;
    const int rows = g.ny * g.nz;
    const int plane = g.nx * g.ny;
    double s = 0.0;
    float m = 0.0f;
    for (int row = blockIdx.x * warps + (threadIdx.x >> 5); row < rows; row += gridDim.x * warps) {
        const int y = row % g.ny;
        const int z = row / g.ny;
        const float* pr = pressure + row * g.nx;
        const float* dv = divergence + row * g.nx;
        for (int x = lane; x < g.nx; x += 32) {
            const float self = __ldg(pr + x);
            const float pL = x > 0 ? __ldg(pr + x - 1) : self;
            const float pR = x < g.nx - 1 ? __ldg(pr + x + 1) : self;
            const float pD = y > 0 ? __ldg(pr + x - g.nx) : self;
            const float pU = y < g.ny - 1 ? __ldg(pr + x + g.nx) : self;
            const float pB = z > 0 ? __ldg(pr + x - plane) : self;
            const float pF = z < g.nz - 1 ? __ldg(pr + x + plane) : self;
            const float r = __fsub_rn(__ldg(dv + x) + pL + pR + pD + pU + pB + pF, __fmul_rn(6.0f, self));
            m = fmaxf(m, fabsf(r));
            s += static_cast<double>(r) * static_cast<double>(r);
        }
    }
    __shared__ double sq[kResidualThreads];
    __shared__ float mx[kResidualThreads];
    sq[threadIdx.x] = s;
    mx[threadIdx.x] = m;
    __syncthreads();
    for (int w = kResidualThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            sq[threadIdx.x] += sq[threadIdx.x + w];
            mx[threadIdx.x] = fmaxf(mx[threadIdx.x], mx[threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partialSq[blockIdx.x] = sq[0];
        partialMax[blockIdx.x] = mx[0];
    }
}

// One warp: lane l sums partials l, l + 32, ... in order, then the lanes are
// combined by a fixed butterfly; max |r| decides the gate.
__global__ void sorResidualFinal(SorGate* gate, const double* __restrict__ partialSq, const float* __restrict__ partialMax, int partials,
                                 float tolerance, int chunkIterations) {
    if (blockIdx.x != 0 || gate->converged) return;
    const int lane = threadIdx.x;
    double s = 0.0;
    float m = 0.0f;
    for (int b = lane; b < partials; b += 32) {
        s += partialSq[b];
        m = fmaxf(m, partialMax[b]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    if (lane != 0) return;
    gate->iterations += chunkIterations;
    gate->maxResidual = m;
    gate->l2Residual = sqrt(s);
    if (m <= tolerance) gate->converged = 1;
}

const void* sorResidentKernel(int bx) {
    return bx == 32 ? reinterpret_cast<const void*>(sorResident<32, 16, 16>) : reinterpret_cast<const void*>(sorResident<16, 16, 16>);
}

size_t sorResidentSharedBytes(int bx) {
    return bx == 32 ? ResidentShape<32, 16, 16>::SHARED_BYTES : ResidentShape<16, 16, 16>::SHARED_BYTES;
}

}  // namespace firesim
