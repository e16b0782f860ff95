// fire_device.cuh -- per-frame parameter block, state layout and device math
// shared by the sm_100a kernels of firesim-b200.
//
// Arithmetic follows native-firesim's src/fire_cuda.cu expression by
// expression (same operand order, same constants), so the compiled kernels
// round like the reference's and the product matches the reference's own
// output.  The sin hashes pin their rounding with __fmaf_rn/__fmul_rn/
// __fsub_rn: their argument is formed with the fused multiply-adds the
// reference binary uses, and the fract is not fused -- measured by evaluating
// the reference's hash21/hash31 on the B200, where this form matches it bit for
// bit.  A one-ulp change there would scramble the noise pattern.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#if defined(FIRE_STORAGE_BF16)
#include <cuda_bf16.h>
#endif

namespace firesim {

constexpr int kMaxRaymarchSteps = 120;   // src/fire_cuda.cu:109
constexpr int kMaxEmberCount = 192;      // src/fire_cuda.cu:110
constexpr int kSceneCount = 3;           // src/fire_cuda.cu:114
constexpr float kAdvectionScale = 0.62f; // src/fire_cuda.cu:107
constexpr float kRoomHeightMeters = 2.03f;
constexpr int kDefaultPressureIterations = 40;  // src/fire_cuda.cu:104
constexpr float kDefaultPressureOmega = 1.52f;  // src/fire_cuda.cu:105

// Per-frame constant block (the content of the reference's SimParams,
// src/fire_cuda.cu:16-68, without its launch windows).  Passed by value.
struct FrameParams {
    int nx, ny, nz;
    int frameW, frameH;
    int lnx, lny, lnz;
    float dt, time, mouseX, mouseY;
    int leftDown, rightDown, showGizmos, activeGizmo, sceneId;
    float wind, turbulence, detail, smokeGain, intensity;
    float3 eye, forward, right, up;
    float tanHalfFov, aspect;
    int cinematicMode, raymarchSteps, emberCount, renderDebugMode;
    float exposure, reflectionGain, smokeDarkness;
    float emitterCenterX, emitterCenterZ, emitterHeightNorm, emitterHeightBandNorm, emitterRadius;
    int burnerCenterCount;
    float burnerCenterX[4], burnerCenterY[4], burnerCenterZ[4];
};

// Storage of the transported fields.  The default build stores the ten
// scalars and the three face grids in FP32.  The FIRE_STORAGE_F16 build
// (libfiresim_b200_f16.so) stores them as IEEE half and the FIRE_STORAGE_BF16
// build (libfiresim_b200_bf16.so) as bfloat16, converted on every load and
// rounded to nearest on every store; all arithmetic stays FP32, and pressure,
// divergence, forcing, light and frames stay FP32.  ldv/stv are the only
// accessors of these buffers, so in the FP32 build they are the plain loads
// and stores they replace.
#if defined(FIRE_STORAGE_F16) || defined(FIRE_STORAGE_BF16)
#if defined(FIRE_STORAGE_F16)
using Half1 = __half;
using Half2 = __half2;
__device__ __forceinline__ float2 halfToFloat2(Half2 v) { return __half22float2(v); }
__device__ __forceinline__ Half2 float2ToHalf(float a, float b) { return __floats2half2_rn(a, b); }
__device__ __forceinline__ float halfToFloat(Half1 v) { return __half2float(v); }
__device__ __forceinline__ Half1 floatToHalf(float v) { return __float2half_rn(v); }
#else
using Half1 = __nv_bfloat16;
using Half2 = __nv_bfloat162;
__device__ __forceinline__ float2 halfToFloat2(Half2 v) { return __bfloat1622float2(v); }
__device__ __forceinline__ Half2 float2ToHalf(float a, float b) { return __floats2bfloat162_rn(a, b); }
__device__ __forceinline__ float halfToFloat(Half1 v) { return __bfloat162float(v); }
__device__ __forceinline__ Half1 floatToHalf(float v) { return __float2bfloat16_rn(v); }
#endif
#define FIRE_HALF_STORAGE 1
struct __align__(8) Rec4 {
    Half2 xy, zw;
};
using Rec2 = Half2;
using FaceT = Half1;
constexpr bool kHalfStorage = true;
#else
using Rec4 = float4;
using Rec2 = float2;
using FaceT = float;
constexpr bool kHalfStorage = false;
#endif

__device__ __forceinline__ float ldv(const float* p) { return __ldg(p); }
__device__ __forceinline__ void stv(float* p, float v) { *p = v; }
// One pixel of the HDR frame into a caller-owned buffer (the headless form of
// packFp16SurfaceKernel, src/fire_cuda.cu:2303-2321): float4 RGBA32F, or
// RGBA16F with negative values clamped to 0 as the reference's halfBits does;
// alpha is 1.
__device__ __forceinline__ void packHdrPixel(void* dst, size_t pitchBytes, int halfFormat, float4 r, int x, int y) {
    char* row = static_cast<char*>(dst) + static_cast<size_t>(y) * pitchBytes;
    if (halfFormat) {
        const __half2 rg = __floats2half2_rn(fmaxf(0.0f, r.x), fmaxf(0.0f, r.y));
        const __half2 ba = __floats2half2_rn(fmaxf(0.0f, r.z), 1.0f);
        reinterpret_cast<__half2*>(row)[2 * x] = rg;
        reinterpret_cast<__half2*>(row)[2 * x + 1] = ba;
    } else {
        reinterpret_cast<float4*>(row)[x] = make_float4(r.x, r.y, r.z, 1.0f);
    }
}

// The value a face or scalar store of v leaves in this build's storage.
__device__ __forceinline__ float storageRound(float v) {
#if defined(FIRE_STORAGE_F16) || defined(FIRE_STORAGE_BF16)
    return halfToFloat(floatToHalf(v));
#else
    return v;
#endif
}
#if defined(FIRE_HALF_STORAGE)
__device__ __forceinline__ float4 ldv(const Rec4* p) {
    const uint2 raw = __ldg(reinterpret_cast<const uint2*>(p));
    const float2 xy = halfToFloat2(*reinterpret_cast<const Half2*>(&raw.x));
    const float2 zw = halfToFloat2(*reinterpret_cast<const Half2*>(&raw.y));
    return make_float4(xy.x, xy.y, zw.x, zw.y);
}
__device__ __forceinline__ float2 ldv(const Rec2* p) {
    const unsigned raw = __ldg(reinterpret_cast<const unsigned*>(p));
    return halfToFloat2(*reinterpret_cast<const Half2*>(&raw));
}
__device__ __forceinline__ float ldv(const Half1* p) {
    const unsigned short raw = __ldg(reinterpret_cast<const unsigned short*>(p));
    return halfToFloat(*reinterpret_cast<const Half1*>(&raw));
}
__device__ __forceinline__ void stv(Rec4* p, float4 v) {
    Rec4 r;
    r.xy = float2ToHalf(v.x, v.y);
    r.zw = float2ToHalf(v.z, v.w);
    *p = r;
}
__device__ __forceinline__ void stv(Rec2* p, float2 v) { *p = float2ToHalf(v.x, v.y); }
__device__ __forceinline__ void stv(Half1* p, float v) { *p = floatToHalf(v); }
__device__ __forceinline__ float4 ldv(const float4* p) { return __ldg(p); }
__device__ __forceinline__ float2 ldv(const float2* p) { return __ldg(p); }
// Single components of a packed record.
__device__ __forceinline__ float ldX(const Rec4* p) { return ldv(reinterpret_cast<const Half1*>(p)); }
__device__ __forceinline__ float ldW(const Rec4* p) { return ldv(reinterpret_cast<const Half1*>(p) + 3); }
__device__ __forceinline__ float ldX(const Rec2* p) { return ldv(reinterpret_cast<const Half1*>(p)); }
#else
__device__ __forceinline__ float4 ldv(const float4* p) { return __ldg(p); }
__device__ __forceinline__ float2 ldv(const float2* p) { return __ldg(p); }
__device__ __forceinline__ void stv(float4* p, float4 v) { *p = v; }
__device__ __forceinline__ void stv(float2* p, float2 v) { *p = v; }
__device__ __forceinline__ float ldX(const float4* p) { return __ldg(&p->x); }
__device__ __forceinline__ float ldW(const float4* p) { return __ldg(&p->w); }
__device__ __forceinline__ float ldX(const float2* p) { return __ldg(&p->x); }
#endif

// Packed cell record of the ten transported scalars: every consumer gathers
// many of them at the same trilinear corners, so one corner is three vector
// loads instead of ten scalar ones.
//   a = (heat, fuel, oxygen, soot)
//   b = (char, ash, pyrolysis, progress)
//   c = (turbulenceEnergy, sootOptics)
struct ScalarFields {
    Rec4* a;
    Rec4* b;
    Rec2* c;
};
struct ScalarFieldsIn {
    const Rec4* __restrict__ a;
    const Rec4* __restrict__ b;
    const Rec2* __restrict__ c;
};

struct Cell10 {
    float heat, fuel, oxygen, soot, charMass, ash, pyrolysis, progress, turbulenceEnergy, sootOptics;
};

__device__ __forceinline__ Cell10 loadCell(const ScalarFieldsIn& s, int idx) {
    const float4 a = ldv(s.a + idx);
    const float4 b = ldv(s.b + idx);
    const float2 c = ldv(s.c + idx);
    return {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y};
}

// --- small vector helpers (src/fire_cuda.cu:219-304) --------------------------
__host__ __device__ __forceinline__ float saturate(float v) { return fminf(1.0f, fmaxf(0.0f, v)); }
__host__ __device__ __forceinline__ float lerpf(float a, float b, float t) { return a + (b - a) * t; }
__device__ __forceinline__ float smoothstepf(float edge0, float edge1, float x) {
    const bool inverted = edge1 < edge0;
    const float lo = inverted ? edge1 : edge0;
    const float hi = inverted ? edge0 : edge1;
    const float t = saturate((x - lo) / fmaxf(0.000001f, hi - lo));
    const float value = t * t * (3.0f - 2.0f * t);
    return inverted ? 1.0f - value : value;
}
__device__ __forceinline__ float fracf(float v) { return v - floorf(v); }
__host__ __device__ __forceinline__ float3 add3(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ float3 mul3(float3 a, float b) { return make_float3(a.x * b, a.y * b, a.z * b); }
__host__ __device__ __forceinline__ float3 mul3v(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
__host__ __device__ __forceinline__ float3 lerp3(float3 a, float3 b, float t) { return add3(a, mul3(sub3(b, a), t)); }
__host__ __device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ float luminance3(float3 c) { return c.x * 0.2126f + c.y * 0.7152f + c.z * 0.0722f; }
__host__ __device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ float3 normalize3(float3 v) {
    const float len = sqrtf(fmaxf(0.000001f, dot3(v, v)));
    return make_float3(v.x / len, v.y / len, v.z / len);
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 mul2(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float dot2(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }

// --- sin hashes and value noise (src/fire_cuda.cu:381-443) ---------------------
__device__ __forceinline__ float hashFract(float q) {
    const float s = __fmul_rn(sinf(q), 43758.5453123f);
    return __fsub_rn(s, floorf(s));
}
__device__ __forceinline__ float hash21(float x, float y) {
    const float qx = __fmaf_rn(x, 127.1f, __fmul_rn(y, 311.7f));
    const float qy = __fmaf_rn(x, 269.5f, __fmul_rn(y, 183.3f));
    return hashFract(__fadd_rn(qx, qy));
}
__device__ __forceinline__ float hash31(float x, float y, float z) {
    return hashFract(__fmaf_rn(z, 74.7f, __fmaf_rn(x, 127.1f, __fmul_rn(y, 311.7f))));
}
__device__ __forceinline__ float noiseLerp(float a, float b, float t) { return __fmaf_rn(b - a, t, a); }
__device__ __forceinline__ float smoothWeight(float f) { return f * f * (3.0f - 2.0f * f); }

// Bilinear blend of the four lattice hashes around (px, py) with weights from the fractions.
__device__ __forceinline__ float valueNoiseFromCorners(float a, float b, float c, float d, float fx, float fy) {
    const float ux = smoothWeight(fx), uy = smoothWeight(fy);
    return noiseLerp(noiseLerp(a, b, ux), noiseLerp(c, d, ux), uy);
}

__device__ __forceinline__ float valueNoise(float px, float py) {
    const float ix = floorf(px), iy = floorf(py);
    const float fx = fracf(px), fy = fracf(py);
    const float a = hash21(ix, iy);
    const float b = hash21(ix + 1.0f, iy);
    const float c = hash21(ix, iy + 1.0f);
    const float d = hash21(ix + 1.0f, iy + 1.0f);
    return valueNoiseFromCorners(a, b, c, d, fx, fy);
}

// Trilinear blend of the eight lattice hashes around a point (hXYZ: corner offsets).
__device__ __forceinline__ float valueNoise3FromCorners(float h000, float h100, float h010, float h110, float h001, float h101, float h011,
                                                        float h111, float ux, float uy, float uz) {
    const float c00 = noiseLerp(h000, h100, ux);
    const float c10 = noiseLerp(h010, h110, ux);
    const float c01 = noiseLerp(h001, h101, ux);
    const float c11 = noiseLerp(h011, h111, ux);
    return noiseLerp(noiseLerp(c00, c10, uy), noiseLerp(c01, c11, uy), uz);
}

__device__ __forceinline__ float valueNoise3(float px, float py, float pz) {
    const float ix = floorf(px), iy = floorf(py), iz = floorf(pz);
    const float ux = smoothWeight(fracf(px)), uy = smoothWeight(fracf(py)), uz = smoothWeight(fracf(pz));
    const float jx = ix + 1.0f, jy = iy + 1.0f, jz = iz + 1.0f;
    return valueNoise3FromCorners(hash31(ix, iy, iz), hash31(jx, iy, iz), hash31(ix, jy, iz), hash31(jx, jy, iz), hash31(ix, iy, jz),
                                  hash31(jx, iy, jz), hash31(ix, jy, jz), hash31(jx, jy, jz), ux, uy, uz);
}

// Five octaves (src/fire_cuda.cu:423-432).  Inlined: its callers combine the
// result with other terms, and the fused multiply-adds the compiler forms
// there match the reference's build only in the inlined form.
__device__ __forceinline__ float fbm(float px, float py) {
    float sum = 0.0f;
    float amp = 0.5f;
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        sum = __fmaf_rn(amp, valueNoise(px, py), sum);
        px = __fmaf_rn(px, 2.03f, 17.7f);
        py = __fmaf_rn(py, 2.01f, -9.2f);
        amp *= 0.5f;
    }
    return sum;
}

// Three octaves, rescaled and saturated (src/fire_cuda.cu:434-443).  Kept out
// of line with a rolled octave loop, so one copy of the hash (and of sinf with
// its large-argument path) serves every call site: inlined and unrolled, the
// raymarch's four fbm3 calls put 96 copies of sinf in its sample loop, which
// then stalls on instruction fetch.  The result is the same bits either way
// (its callers only saturate or offset it).
static __device__ __noinline__ float fbm3(float px, float py, float pz) {
    float sum = 0.0f;
    float amp = 0.5f;
#pragma unroll 1
    for (int i = 0; i < 3; ++i) {
        sum = __fmaf_rn(amp, valueNoise3(px, py, pz), sum);
        px = __fmaf_rn(px, 2.03f, 17.7f);
        py = __fmaf_rn(py, 2.01f, -9.2f);
        pz = __fmaf_rn(pz, 2.07f, 5.1f);
        amp *= 0.5f;
    }
    return saturate(sum * 1.142857f);
}

// --- hash lattices of 2D fbm call sites ---------------------------------------
// A 2D fbm evaluated at every cell of the grid hashes the same integer
// lattice points many times over (at the lowest octave a lattice cell spans
// ten grid cells).  A HashLattice2 holds hash21 at every lattice point one
// call site can reach in this step, per octave; fbmLattice reads its four
// corners there instead of evaluating four sines.  The values are the same
// bits (hash21 of the same integral coordinates), so fbmLattice(px, py, L)
// equals fbm(px, py) exactly.  A corner outside the table, or a table with
// no storage, is hashed directly.
constexpr int kFbmOctaves = 5;
struct HashLattice2 {
    const float* values;  // octave o: sx[o] * sy[o] values at offset[o], x fastest
    int ox[kFbmOctaves], oy[kFbmOctaves];  // lattice coordinate of entry (0, 0)
    int sx[kFbmOctaves], sy[kFbmOctaves];
    int offset[kFbmOctaves];
};

static __device__ __noinline__ float hash21OutOfLine(float x, float y) { return hash21(x, y); }

__device__ __forceinline__ float fbmLattice(float px, float py, const HashLattice2& L) {
    float sum = 0.0f;
    float amp = 0.5f;
#pragma unroll
    for (int i = 0; i < kFbmOctaves; ++i) {
        const float ix = floorf(px), iy = floorf(py);
        const float fx = fracf(px), fy = fracf(py);
        const int tx = static_cast<int>(ix) - L.ox[i];
        const int ty = static_cast<int>(iy) - L.oy[i];
        float a, b, c, d;
        if (L.values != nullptr && tx >= 0 && tx < L.sx[i] - 1 && ty >= 0 && ty < L.sy[i] - 1) {
            const float* q = L.values + L.offset[i] + ty * L.sx[i] + tx;
            a = __ldg(q);
            b = __ldg(q + 1);
            c = __ldg(q + L.sx[i]);
            d = __ldg(q + L.sx[i] + 1);
        } else {
            a = hash21OutOfLine(ix, iy);
            b = hash21OutOfLine(ix + 1.0f, iy);
            c = hash21OutOfLine(ix, iy + 1.0f);
            d = hash21OutOfLine(ix + 1.0f, iy + 1.0f);
        }
        sum = __fmaf_rn(amp, valueNoiseFromCorners(a, b, c, d, fx, fy), sum);
        px = __fmaf_rn(px, 2.03f, 17.7f);
        py = __fmaf_rn(py, 2.01f, -9.2f);
        amp *= 0.5f;
    }
    return sum;
}

// --- lattice sampling -------------------------------------------------------
// Trilinear corner set of a sample in normalized coordinates on a lattice whose
// largest node index per axis is (ex, ey, ez) (src/fire_cuda.cu:489-600):
// scalars use (nx-1, ny-1, nz-1); the face grids use nx, ny or nz on their axis.
struct Corners {
    int x0, x1, y0, y1, z0, z1;
    float tx, ty, tz;
};

__device__ __forceinline__ Corners cornersOf(float u, float v, float w, int ex, int ey, int ez) {
    u = saturate(u);
    v = saturate(v);
    w = saturate(w);
    const float fx = u * static_cast<float>(ex);
    const float fy = v * static_cast<float>(ey);
    const float fz = w * static_cast<float>(ez);
    Corners c;
    c.x0 = static_cast<int>(floorf(fx));
    c.y0 = static_cast<int>(floorf(fy));
    c.z0 = static_cast<int>(floorf(fz));
    c.x1 = min(c.x0 + 1, ex);
    c.y1 = min(c.y0 + 1, ey);
    c.z1 = min(c.z0 + 1, ez);
    c.tx = fx - static_cast<float>(c.x0);
    c.ty = fy - static_cast<float>(c.y0);
    c.tz = fz - static_cast<float>(c.z0);
    return c;
}

// Gather of one scalar lattice (float, or a half face grid) with row pitch sx
// and slice pitch sx*sy.
template <class T>
__device__ __forceinline__ float gather1(const T* __restrict__ f, const Corners& c, int sx, int sy) {
    const float c000 = ldv(f + (c.z0 * sy + c.y0) * sx + c.x0);
    const float c100 = ldv(f + (c.z0 * sy + c.y0) * sx + c.x1);
    const float c010 = ldv(f + (c.z0 * sy + c.y1) * sx + c.x0);
    const float c110 = ldv(f + (c.z0 * sy + c.y1) * sx + c.x1);
    const float c001 = ldv(f + (c.z1 * sy + c.y0) * sx + c.x0);
    const float c101 = ldv(f + (c.z1 * sy + c.y0) * sx + c.x1);
    const float c011 = ldv(f + (c.z1 * sy + c.y1) * sx + c.x0);
    const float c111 = ldv(f + (c.z1 * sy + c.y1) * sx + c.x1);
    return lerpf(lerpf(lerpf(c000, c100, c.tx), lerpf(c010, c110, c.tx), c.ty),
                 lerpf(lerpf(c001, c101, c.tx), lerpf(c011, c111, c.tx), c.ty), c.tz);
}

struct Grid {
    int nx, ny, nz;
};

__device__ __forceinline__ float sampleU(const FaceT* __restrict__ u, const Grid& g, float a, float b, float c) {
    return gather1(u, cornersOf(a, b, c, g.nx, g.ny - 1, g.nz - 1), g.nx + 1, g.ny);
}
__device__ __forceinline__ float sampleV(const FaceT* __restrict__ v, const Grid& g, float a, float b, float c) {
    return gather1(v, cornersOf(a, b, c, g.nx - 1, g.ny, g.nz - 1), g.nx, g.ny + 1);
}
__device__ __forceinline__ float sampleW(const FaceT* __restrict__ w, const Grid& g, float a, float b, float c) {
    return gather1(w, cornersOf(a, b, c, g.nx - 1, g.ny - 1, g.nz), g.nx, g.ny);
}

struct Velocity {
    const FaceT* __restrict__ u;
    const FaceT* __restrict__ v;
    const FaceT* __restrict__ w;
};

__device__ __forceinline__ float3 sampleVelocity(const Velocity& vel, const Grid& g, float a, float b, float c) {
    return make_float3(sampleU(vel.u, g, a, b, c), sampleV(vel.v, g, a, b, c), sampleW(vel.w, g, a, b, c));
}

__device__ __forceinline__ float sampleScalar1(const float* __restrict__ f, const Grid& g, float a, float b, float c) {
    return gather1(f, cornersOf(a, b, c, g.nx - 1, g.ny - 1, g.nz - 1), g.nx, g.ny);
}

// Trilinear blend of packed float4 / float2 corners, component-wise in the
// same operation order as the scalar sampler.
__device__ __forceinline__ float4 lerp4(float4 a, float4 b, float t) {
    return make_float4(lerpf(a.x, b.x, t), lerpf(a.y, b.y, t), lerpf(a.z, b.z, t), lerpf(a.w, b.w, t));
}
__device__ __forceinline__ float2 lerp2v(float2 a, float2 b, float t) { return make_float2(lerpf(a.x, b.x, t), lerpf(a.y, b.y, t)); }

__device__ __forceinline__ float4 lerpv(float4 a, float4 b, float t) { return lerp4(a, b, t); }
__device__ __forceinline__ float2 lerpv(float2 a, float2 b, float t) { return lerp2v(a, b, t); }

// Gather of a packed lattice (float4 / float2, or a half record), blended
// component-wise in FP32.
template <class P>
__device__ __forceinline__ auto gatherVec(const P* __restrict__ f, const Corners& c, int sx, int sy) -> decltype(ldv(f)) {
    const auto c000 = ldv(f + (c.z0 * sy + c.y0) * sx + c.x0);
    const auto c100 = ldv(f + (c.z0 * sy + c.y0) * sx + c.x1);
    const auto c010 = ldv(f + (c.z0 * sy + c.y1) * sx + c.x0);
    const auto c110 = ldv(f + (c.z0 * sy + c.y1) * sx + c.x1);
    const auto c001 = ldv(f + (c.z1 * sy + c.y0) * sx + c.x0);
    const auto c101 = ldv(f + (c.z1 * sy + c.y0) * sx + c.x1);
    const auto c011 = ldv(f + (c.z1 * sy + c.y1) * sx + c.x0);
    const auto c111 = ldv(f + (c.z1 * sy + c.y1) * sx + c.x1);
    return lerpv(lerpv(lerpv(c000, c100, c.tx), lerpv(c010, c110, c.tx), c.ty),
                 lerpv(lerpv(c001, c101, c.tx), lerpv(c011, c111, c.tx), c.ty), c.tz);
}

__device__ __forceinline__ Corners scalarCorners(const Grid& g, float u, float v, float w) {
    return cornersOf(u, v, w, g.nx - 1, g.ny - 1, g.nz - 1);
}

// All ten scalars at one point (the light pass and the raymarch sample them together).
__device__ __forceinline__ Cell10 sampleAll(const ScalarFieldsIn& s, const Grid& g, float u, float v, float w) {
    const Corners c = scalarCorners(g, u, v, w);
    const float4 a = gatherVec(s.a, c, g.nx, g.ny);
    const float4 b = gatherVec(s.b, c, g.nx, g.ny);
    const float2 d = gatherVec(s.c, c, g.nx, g.ny);
    return {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, d.x, d.y};
}

// Heat alone (gradients, the glow probe): the x component of the packed record.
__device__ __forceinline__ float sampleHeat(const ScalarFieldsIn& s, const Grid& g, float u, float v, float w) {
    const Corners c = scalarCorners(g, u, v, w);
    const int sx = g.nx, sy = g.ny;
    auto h = [&](int x, int y, int z) { return ldX(s.a + (z * sy + y) * sx + x); };
    return lerpf(lerpf(lerpf(h(c.x0, c.y0, c.z0), h(c.x1, c.y0, c.z0), c.tx), lerpf(h(c.x0, c.y1, c.z0), h(c.x1, c.y1, c.z0), c.tx), c.ty),
                 lerpf(lerpf(h(c.x0, c.y0, c.z1), h(c.x1, c.y0, c.z1), c.tx), lerpf(h(c.x0, c.y1, c.z1), h(c.x1, c.y1, c.z1), c.tx), c.ty),
                 c.tz);
}

// --- light volume sampling (src/fire_cuda.cu:618-664) --------------------------
struct LightGrid {
    int lnx, lny, lnz;
};

__device__ __forceinline__ float4 sampleSceneLight(const float4* __restrict__ f, const LightGrid& L, float u, float v, float w) {
    if (f == nullptr || L.lnx <= 1 || L.lny <= 1 || L.lnz <= 1) {
        return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    return gatherVec(f, cornersOf(u, v, w, L.lnx - 1, L.lny - 1, L.lnz - 1), L.lnx, L.lny);
}

__device__ __forceinline__ float sampleSceneShadow(const float* __restrict__ f, const LightGrid& L, float u, float v, float w) {
    if (f == nullptr || L.lnx <= 1 || L.lny <= 1 || L.lnz <= 1) {
        return 1.0f;
    }
    u = saturate(u);
    v = saturate(v);
    w = saturate(w);
    const int x = min(max(static_cast<int>(u * static_cast<float>(L.lnx - 1) + 0.5f), 0), L.lnx - 1);
    const int y = min(max(static_cast<int>(v * static_cast<float>(L.lny - 1) + 0.5f), 0), L.lny - 1);
    const int z = min(max(static_cast<int>(w * static_cast<float>(L.lnz - 1) + 0.5f), 0), L.lnz - 1);
    return __ldg(f + (z * L.lny + y) * L.lnx + x);
}

// --- scene geometry helpers -----------------------------------------------------
__device__ __forceinline__ float volumeDomainFade(float u, float v, float w) {  // src/fire_cuda.cu:359-368
    const float side = smoothstepf(0.000f, 0.095f, u) * smoothstepf(1.000f, 0.905f, u) * smoothstepf(0.000f, 0.100f, w) *
                       smoothstepf(1.000f, 0.900f, w);
    const float floorFade = smoothstepf(0.000f, 0.018f, v);
    const float topFade = smoothstepf(1.000f, 0.520f, v);
    return saturate(side * floorFade * topFade);
}

__device__ __forceinline__ float3 blackbodyColor(float tempK) {  // src/fire_cuda.cu:1420-1443
    const float t = fmaxf(1000.0f, fminf(12000.0f, tempK)) / 100.0f;
    float r = 0.0f, g = 0.0f, b = 0.0f;
    if (t <= 66.0f) {
        r = 1.0f;
        g = saturate((99.4708025861f * logf(t) - 161.1195681661f) / 255.0f);
    } else {
        r = saturate(329.698727446f * powf(t - 60.0f, -0.1332047592f) / 255.0f);
        g = saturate(288.1221695283f * powf(t - 60.0f, -0.0755148492f) / 255.0f);
    }
    if (t >= 66.0f) {
        b = 1.0f;
    } else if (t <= 19.0f) {
        b = 0.0f;
    } else {
        b = saturate((138.5177312231f * logf(t - 10.0f) - 305.0447927307f) / 255.0f);
    }
    return make_float3(r, g, b);
}

__device__ __forceinline__ float3 projectPoint(const FrameParams& p, float3 point) {  // src/fire_cuda.cu:348-357
    const float3 view = sub3(point, p.eye);
    const float depth = dot3(view, p.forward);
    if (depth <= 0.02f) {
        return make_float3(-10.0f, -10.0f, -1.0f);
    }
    const float px = dot3(view, p.right) / (depth * p.tanHalfFov * p.aspect);
    const float py = dot3(view, p.up) / (depth * p.tanHalfFov);
    return make_float3(0.5f + px * 0.5f, 0.5f - py * 0.5f, depth);
}

__device__ __forceinline__ float orientedCapsuleMask(float x, float z, float cx, float cz, float angle, float halfLength, float radius) {
    const float ca = cosf(angle);  // src/fire_cuda.cu:734-744
    const float sa = sinf(angle);
    const float px = x - cx;
    const float pz = z - cz;
    const float qx = px * ca + pz * sa;
    const float qz = -px * sa + pz * ca;
    const float over = fmaxf(fabsf(qx) - halfLength, 0.0f);
    const float dist = sqrtf(over * over + qz * qz);
    return smoothstepf(radius, radius * 0.22f, dist);
}

// Procedural fuel bed of each scene (src/fire_cuda.cu:746-793).  It depends
// only on the scene and its emitter parameters, so the step reads it from a
// per-scene (x, z) table built once; the raymarch's floor shading calls it at
// arbitrary points.
__device__ __forceinline__ float fuelBedMaterial(float x, float z, const FrameParams& p) {
    if (p.sceneId == 1) {
        const float logA = orientedCapsuleMask(x, z, -0.06f, 0.01f, 0.38f, 0.34f, 0.060f);
        const float logB = orientedCapsuleMask(x, z, 0.07f, -0.02f, -0.58f, 0.33f, 0.058f);
        const float logC = orientedCapsuleMask(x, z, 0.01f, 0.08f, 1.34f, 0.24f, 0.050f);
        const float contactAB = fminf(logA, logB) * 1.25f;
        const float contactBC = fminf(logB, logC) * 1.10f;
        const float contactCA = fminf(logC, logA) * 0.92f;
        const float coalNoise = fbm(x * 9.4f + z * 1.7f, z * 11.2f - x * 3.1f);
        const float coalBed = smoothstepf(0.38f, 0.08f, sqrtf(x * x * 1.35f + z * z * 2.40f)) * smoothstepf(0.34f, 0.88f, coalNoise);
        const float cracks = smoothstepf(0.65f, 0.93f, fbm(x * 21.0f - z * 6.0f, z * 24.0f + x * 4.0f));
        const float contactPyrolysis = saturate(contactAB + contactBC + contactCA);
        return saturate((logA * 0.72f + logB * 0.70f + logC * 0.54f + coalBed * 0.84f + contactPyrolysis * 1.18f) * (1.0f - cracks * 0.24f));
    }
    if (p.sceneId == 2) {
        const float sourceRadius = fmaxf(0.04f, p.emitterRadius);
        float source = 0.0f;
        const float cx = p.burnerCenterCount > 0 ? p.burnerCenterX[0] : p.emitterCenterX;
        const float cz = p.burnerCenterCount > 0 ? p.burnerCenterZ[0] : p.emitterCenterZ;
        const float px = x - cx;
        const float pz = z - cz;
        const float radius = sqrtf(px * px + pz * pz);
        const float angle = atan2f(pz, px);
        const float ring = smoothstepf(sourceRadius * 0.072f, sourceRadius * 0.014f, fabsf(radius - sourceRadius));
        const float innerRing = smoothstepf(sourceRadius * 0.052f, sourceRadius * 0.012f, fabsf(radius - sourceRadius * 0.52f));
        const float ports = 0.5f + 0.5f * cosf(angle * 32.0f);
        const float portMask = smoothstepf(0.80f, 0.992f, ports);
        const float centerPilot = smoothstepf(sourceRadius * 0.22f, 0.000f, radius) * 0.045f;
        source = fmaxf(source, (ring * (0.035f + portMask * 1.72f) + innerRing * 0.055f + centerPilot) *
                                   smoothstepf(sourceRadius * 1.28f, sourceRadius * 1.05f, radius));
        return saturate(source);
    }
    const float tray = smoothstepf(1.08f, 0.030f, fabsf(x)) * smoothstepf(0.56f, 0.026f, fabsf(z));
    const float emberMat = smoothstepf(1.00f, 0.018f, fabsf(x)) * smoothstepf(0.50f, 0.020f, fabsf(z));
    const float mound = expf(-(x * x * 0.70f + z * z * 2.15f));
    const float logMass = fbm(x * 3.7f + z * 0.9f, z * 5.4f - x * 0.6f);
    const float chips = fbm(x * 15.0f + z * 4.0f, z * 18.0f - x * 5.0f);
    const float strand = 0.5f + 0.5f * sinf((x * 19.0f + z * 7.0f) + fbm(z * 4.0f, x * 3.0f) * 4.2f);
    const float cracks = smoothstepf(0.44f, 0.74f, chips) * smoothstepf(0.20f, 0.84f, logMass);
    const float voids = smoothstepf(0.70f, 0.93f, chips * 0.72f + strand * 0.34f);
    const float clumps = smoothstepf(0.22f, 0.86f, logMass * 0.82f + chips * 0.36f + strand * 0.18f);
    const float porousFuel = (0.24f + clumps * 0.94f + emberMat * 0.20f) * (0.64f + mound * 0.46f);
    return saturate(tray * porousFuel * (1.0f - cracks * 0.46f) * (1.0f - voids * 0.34f));
}

// Height profile of the fuel bed source (first factor of src/fire_cuda.cu:797-799).
__device__ __forceinline__ float fuelBedHeight(float h, const FrameParams& p) {
    return p.sceneId == 2 ? smoothstepf(fmaxf(0.005f, p.emitterHeightBandNorm * 0.34f), fmaxf(0.0015f, p.emitterHeightBandNorm * 0.055f),
                                        fabsf(h - p.emitterHeightNorm))
                          : smoothstepf(p.sceneId == 1 ? 0.245f : 0.145f, 0.00f, h);
}

// Ember breathing of the bed (src/fire_cuda.cu:800): depends on (x, z, time) only.
__device__ __forceinline__ float emberBreathing(float x, float z, float time) {
    return 0.84f + 0.16f * fbm(x * 9.0f + time * 0.035f, z * 11.0f - time * 0.025f);
}

// fuelBedSource (src/fire_cuda.cu:795-803) from a material value and breathing factor.
__device__ __forceinline__ float fuelBedSourceFrom(float material, float breathing, float h, const FrameParams& p) {
    const float height = fuelBedHeight(h, p);
    const float exposedFuel = saturate(material * breathing);
    return saturate(height * exposedFuel);
}

__device__ __forceinline__ float cellCoord(int i, int n) { return (static_cast<float>(i) + 0.5f) / static_cast<float>(n); }

}  // namespace firesim
