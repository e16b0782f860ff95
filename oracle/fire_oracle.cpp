// fire_oracle.cpp -- CPU oracle for the native-firesim frame pipeline.
//
// TEST INFRASTRUCTURE, NOT PRODUCT CODE (see fire_oracle.h).  Each function
// restates one function of the reference, src/fire_cuda.cu, and cites the
// lines it follows.  Everything is templated on the arithmetic type T:
//   T = float   reproduces the reference's single-precision arithmetic
//               (without FMA contraction: this file is built with
//               -ffp-contract=off, so every operation rounds as written);
//   T = double  is the precision oracle.
// The pseudo-random hashes (hash21/hash31) are always evaluated in float,
// because they define the noise pattern itself; in the double oracle only the
// interpolation and everything downstream is widened.
//
// Deliberate restatement choices (each documented where it happens):
//   * forceVelocityKernel (src/fire_cuda.cu:1128-1183) reads the face
//     velocities while other threads atomically add to them.  The oracle reads
//     every face before any force is added and adds the two contributions of a
//     shared face lower cell first -- the reference's result whenever its loads
//     precede its atomics, which is what it does at the sizes of the golden
//     fixtures (one wave of blocks).
//   * atomic FP64 metric sums are summed in cell order.
//   * ember splats (src/fire_cuda.cu:2446-2448) are added in ember order.
//   * the render snapshot copies (src/fire_cuda.cu:2871-2908) are not made;
//     rendering reads the current fields, which hold the same values whenever
//     step and render run in sequence.
#include "fire_oracle.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

namespace {

char g_error[256] = "no error";

int setError(const char* msg) {
    std::snprintf(g_error, sizeof(g_error), "%s", msg);
    return -1;
}

// Constants, src/fire_cuda.cu:104-114.
constexpr int kPressureIterations = 40;
constexpr float kPressureOmega = 1.52f;
constexpr float kRoomHeightMeters = 2.03f;
constexpr float kAdvectionScale = 0.62f;
constexpr int kMaxRaymarchSteps = 120;
constexpr int kMaxEmberCount = 192;
constexpr int kSceneCount = 3;

#define F(x) T(x##f)

template <class T>
struct V2 {
    T x, y;
};
template <class T>
struct V3 {
    T x, y, z;
};
template <class T>
struct V4 {
    T x, y, z, w;
};

template <class T> inline V2<T> v2(T x, T y) { return {x, y}; }
template <class T> inline V3<T> v3(T x, T y, T z) { return {x, y, z}; }

// src/fire_cuda.cu:219-304 -- small vector helpers.
template <class T> inline T saturate(T v) { return std::fmin(T(1), std::fmax(T(0), v)); }
template <class T> inline T lerpf(T a, T b, T t) { return a + (b - a) * t; }
template <class T> inline T smoothstepf(T edge0, T edge1, T x) {
    const bool inverted = edge1 < edge0;
    const T lo = inverted ? edge1 : edge0;
    const T hi = inverted ? edge0 : edge1;
    const T t = saturate((x - lo) / std::fmax(F(0.000001), hi - lo));
    const T value = t * t * (F(3.0) - F(2.0) * t);
    return inverted ? F(1.0) - value : value;
}
template <class T> inline T fracf(T v) { return v - std::floor(v); }
template <class T> inline V3<T> add3(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> inline V3<T> sub3(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline V3<T> mul3(V3<T> a, T b) { return {a.x * b, a.y * b, a.z * b}; }
template <class T> inline V3<T> mul3v(V3<T> a, V3<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T> inline V3<T> lerp3(V3<T> a, V3<T> b, T t) { return add3(a, mul3(sub3(b, a), t)); }
template <class T> inline T dot3(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline T luminance3(V3<T> c) { return c.x * F(0.2126) + c.y * F(0.7152) + c.z * F(0.0722); }
template <class T> inline V3<T> cross3(V3<T> a, V3<T> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> inline V3<T> normalize3(V3<T> v) {
    const T len = std::sqrt(std::fmax(F(0.000001), dot3(v, v)));
    return {v.x / len, v.y / len, v.z / len};
}
template <class T> inline V2<T> sub2(V2<T> a, V2<T> b) { return {a.x - b.x, a.y - b.y}; }
template <class T> inline V2<T> add2(V2<T> a, V2<T> b) { return {a.x + b.x, a.y + b.y}; }
template <class T> inline V2<T> mul2(V2<T> a, T s) { return {a.x * s, a.y * s}; }
template <class T> inline T dot2(V2<T> a, V2<T> b) { return a.x * b.x + a.y * b.y; }

// src/fire_cuda.cu:381-388 -- sin hashes, always in float (they define the pattern).
// A one-ulp change of the sine's argument scrambles the hash, so the argument
// is formed with the fused multiply-adds the reference's compiled device code
// uses (every product feeding a sum is fused; established by evaluating the
// reference's own hash21/hash31 on the GPU over 2x10^5 inputs: this form
// matches bit for bit wherever CUDA's sinf equals the correctly rounded sine).
inline float hash21f(float px, float py) {
    const float qx = std::fma(px, 127.1f, py * 311.7f);
    const float qy = std::fma(px, 269.5f, py * 183.3f);
    const float s = std::sin(qx + qy) * 43758.5453123f;
    return s - std::floor(s);
}
inline float hash31f(float px, float py, float pz) {
    const float s = std::sin(std::fma(pz, 74.7f, std::fma(px, 127.1f, py * 311.7f))) * 43758.5453123f;
    return s - std::floor(s);
}

// Interpolation inside the noise functions, fused as in the reference binary.
template <class T> inline T nlerp(T a, T b, T t) { return std::fma(b - a, t, a); }

// src/fire_cuda.cu:390-399
template <class T> T valueNoise(V2<T> p) {
    const V2<T> i = {std::floor(p.x), std::floor(p.y)};
    const V2<T> f = {fracf(p.x), fracf(p.y)};
    const T a = T(hash21f(float(i.x), float(i.y)));
    const T b = T(hash21f(float(i.x + F(1.0)), float(i.y)));
    const T c = T(hash21f(float(i.x), float(i.y + F(1.0))));
    const T d = T(hash21f(float(i.x + F(1.0)), float(i.y + F(1.0))));
    const V2<T> u = {f.x * f.x * (F(3.0) - F(2.0) * f.x), f.y * f.y * (F(3.0) - F(2.0) * f.y)};
    return nlerp(nlerp(a, b, u.x), nlerp(c, d, u.x), u.y);
}

// src/fire_cuda.cu:401-421
template <class T> T valueNoise3(V3<T> p) {
    const V3<T> i = {std::floor(p.x), std::floor(p.y), std::floor(p.z)};
    const V3<T> f = {fracf(p.x), fracf(p.y), fracf(p.z)};
    const V3<T> u = {f.x * f.x * (F(3.0) - F(2.0) * f.x), f.y * f.y * (F(3.0) - F(2.0) * f.y),
                     f.z * f.z * (F(3.0) - F(2.0) * f.z)};
    const float ix = float(i.x), iy = float(i.y), iz = float(i.z);
    const float jx = float(i.x + F(1.0)), jy = float(i.y + F(1.0)), jz = float(i.z + F(1.0));
    const T c000 = T(hash31f(ix, iy, iz));
    const T c100 = T(hash31f(jx, iy, iz));
    const T c010 = T(hash31f(ix, jy, iz));
    const T c110 = T(hash31f(jx, jy, iz));
    const T c001 = T(hash31f(ix, iy, jz));
    const T c101 = T(hash31f(jx, iy, jz));
    const T c011 = T(hash31f(ix, jy, jz));
    const T c111 = T(hash31f(jx, jy, jz));
    const T c00 = nlerp(c000, c100, u.x);
    const T c10 = nlerp(c010, c110, u.x);
    const T c01 = nlerp(c001, c101, u.x);
    const T c11 = nlerp(c011, c111, u.x);
    return nlerp(nlerp(c00, c10, u.y), nlerp(c01, c11, u.y), u.z);
}

// src/fire_cuda.cu:423-432 -- five octaves.
template <class T> T fbm(V2<T> p) {
    T sum = F(0.0);
    T amp = F(0.5);
    for (int i = 0; i < 5; ++i) {
        sum = std::fma(amp, valueNoise(p), sum);
        p = {std::fma(p.x, F(2.03), F(17.7)), std::fma(p.y, F(2.01), F(-9.2))};
        amp *= F(0.5);
    }
    return sum;
}

// src/fire_cuda.cu:434-443 -- three octaves, rescaled and saturated.
template <class T> T fbm3(V3<T> p) {
    T sum = F(0.0);
    T amp = F(0.5);
    for (int i = 0; i < 3; ++i) {
        sum = std::fma(amp, valueNoise3(p), sum);
        p = {std::fma(p.x, F(2.03), F(17.7)), std::fma(p.y, F(2.01), F(-9.2)), std::fma(p.z, F(2.07), F(5.1))};
        amp *= F(0.5);
    }
    return saturate(sum * F(1.142857));
}

// SimParams, src/fire_cuda.cu:16-68 (the launch-window fields are not needed).
template <class T>
struct Params {
    int nx, ny, nz, frameW, frameH, lnx, lny, lnz;
    T dt, time, mouseX, mouseY;
    int leftDown, rightDown, showGizmos, activeGizmo, sceneId;
    T wind, turbulence, detail, smokeGain, intensity, cameraYaw, cameraPitch, cameraDistance;
    V3<T> eye, forward, right, up;
    T tanHalfFov, aspect;
    int cinematicMode, raymarchSteps, emberCount, renderDebugMode;
    T exposure, reflectionGain, smokeDarkness;
    T emitterCenterX, emitterCenterZ, emitterHeightNorm, emitterHeightBandNorm, emitterRadius;
    int burnerCenterCount;
    T burnerCenterX[4], burnerCenterY[4], burnerCenterZ[4];
};

// src/fire_cuda.cu:315-329 (evaluated on the host by the reference as well).
template <class T> void computeCamera(Params<T>& p) {
    const V3<T> target = {F(0.0), F(0.72), F(0.0)};
    const T cp = std::cos(p.cameraPitch);
    p.eye = {std::sin(p.cameraYaw) * p.cameraDistance * cp, target.y + std::sin(p.cameraPitch) * p.cameraDistance,
             std::cos(p.cameraYaw) * p.cameraDistance * cp};
    p.forward = normalize3(sub3(target, p.eye));
    p.right = normalize3(cross3(p.forward, V3<T>{F(0.0), F(1.0), F(0.0)}));
    p.up = normalize3(cross3(p.right, p.forward));
    p.tanHalfFov = F(0.50);
    p.aspect = T(static_cast<float>(p.frameW) / static_cast<float>(p.frameH));
}

// The grid and the fields of one scene.
template <class T>
struct State {
    int nx, ny, nz, lnx, lny, lnz, frameW, frameH;
    std::vector<T> scalar[10];
    std::vector<T> pressure, divergence, divergenceAfter;
    std::vector<T> u, v, w;
    std::vector<V4<T>> light, lightNext;
    std::vector<T> shadow;
    std::vector<V4<T>> hdr;
    std::vector<uint32_t> bgra;
    float simTime = 0.0f, renderTime = 0.0f;
    int frameIndex = 0;
    int pressureIterations = kPressureIterations;
    float pressureOmega = kPressureOmega;
    double metricSums[21] = {};
    int metricWords[10] = {};

    size_t cells() const { return size_t(nx) * ny * nz; }
    size_t lightCells() const { return size_t(lnx) * lny * lnz; }
};

enum { HEAT, FUEL, OXYGEN, SOOT, CHAR, ASH, PYRO, PROGRESS, TURB, SOOTOPT };

// Index maps, src/fire_cuda.cu:445-487.
template <class T> inline int sIdx(const Params<T>& p, int x, int y, int z) {
    x = std::min(std::max(x, 0), p.nx - 1);
    y = std::min(std::max(y, 0), p.ny - 1);
    z = std::min(std::max(z, 0), p.nz - 1);
    return (z * p.ny + y) * p.nx + x;
}
template <class T> inline int uIdx(const Params<T>& p, int x, int y, int z) {
    x = std::min(std::max(x, 0), p.nx);
    y = std::min(std::max(y, 0), p.ny - 1);
    z = std::min(std::max(z, 0), p.nz - 1);
    return (z * p.ny + y) * (p.nx + 1) + x;
}
template <class T> inline int vIdx(const Params<T>& p, int x, int y, int z) {
    x = std::min(std::max(x, 0), p.nx - 1);
    y = std::min(std::max(y, 0), p.ny);
    z = std::min(std::max(z, 0), p.nz - 1);
    return (z * (p.ny + 1) + y) * p.nx + x;
}
template <class T> inline int wIdx(const Params<T>& p, int x, int y, int z) {
    x = std::min(std::max(x, 0), p.nx - 1);
    y = std::min(std::max(y, 0), p.ny - 1);
    z = std::min(std::max(z, 0), p.nz);
    return (z * p.ny + y) * p.nx + x;
}

// Trilinear gather on a lattice of (ex+1) x (ey+1) x (ez+1) nodes with row
// pitches sx, sy: the common form of sampleScalar/sampleU/sampleV/sampleW,
// src/fire_cuda.cu:489-600.  ex, ey, ez are the largest node index per axis.
template <class T>
inline T trilinear(const T* f, int ex, int ey, int ez, int sx, int sy, T u, T v, T w) {
    u = saturate(u);
    v = saturate(v);
    w = saturate(w);
    const T fx = u * T(static_cast<float>(ex));
    const T fy = v * T(static_cast<float>(ey));
    const T fz = w * T(static_cast<float>(ez));
    const int x0 = static_cast<int>(std::floor(fx));
    const int y0 = static_cast<int>(std::floor(fy));
    const int z0 = static_cast<int>(std::floor(fz));
    const int x1 = std::min(x0 + 1, ex);
    const int y1 = std::min(y0 + 1, ey);
    const int z1 = std::min(z0 + 1, ez);
    const T tx = fx - T(static_cast<float>(x0));
    const T ty = fy - T(static_cast<float>(y0));
    const T tz = fz - T(static_cast<float>(z0));
    auto at = [&](int x, int y, int z) { return f[(size_t(z) * sy + y) * sx + x]; };
    const T c000 = at(x0, y0, z0), c100 = at(x1, y0, z0), c010 = at(x0, y1, z0), c110 = at(x1, y1, z0);
    const T c001 = at(x0, y0, z1), c101 = at(x1, y0, z1), c011 = at(x0, y1, z1), c111 = at(x1, y1, z1);
    // The reference's sm_100a build contracts each lerp a + (b - a) t into
    // fma(b - a, t, a); with this form the velocity advection equals its
    // output bit for bit (golden fixtures).
    auto L = [](T a, T b, T t) { return std::fma(b - a, t, a); };
    return L(L(L(c000, c100, tx), L(c010, c110, tx), ty), L(L(c001, c101, tx), L(c011, c111, tx), ty), tz);
}

template <class T> inline T sampleScalar(const T* f, const Params<T>& p, T u, T v, T w) {
    return trilinear(f, p.nx - 1, p.ny - 1, p.nz - 1, p.nx, p.ny, u, v, w);
}
template <class T> inline T sampleU(const T* f, const Params<T>& p, T u, T v, T w) {
    return trilinear(f, p.nx, p.ny - 1, p.nz - 1, p.nx + 1, p.ny, u, v, w);
}
template <class T> inline T sampleV(const T* f, const Params<T>& p, T u, T v, T w) {
    return trilinear(f, p.nx - 1, p.ny, p.nz - 1, p.nx, p.ny + 1, u, v, w);
}
template <class T> inline T sampleW(const T* f, const Params<T>& p, T u, T v, T w) {
    return trilinear(f, p.nx - 1, p.ny - 1, p.nz, p.nx, p.ny, u, v, w);
}
// src/fire_cuda.cu:602-604
template <class T>
inline V3<T> sampleVelocity(const State<T>& s, const Params<T>& p, T u, T v, T w) {
    return {sampleU(s.u.data(), p, u, v, w), sampleV(s.v.data(), p, u, v, w), sampleW(s.w.data(), p, u, v, w)};
}

// src/fire_cuda.cu:618-651
template <class T> V4<T> sampleSceneLight(const V4<T>* f, const Params<T>& p, T u, T v, T w) {
    if (f == nullptr || p.lnx <= 1 || p.lny <= 1 || p.lnz <= 1) return {F(0.0), F(0.0), F(0.0), F(0.0)};
    u = saturate(u);
    v = saturate(v);
    w = saturate(w);
    const T fx = u * T(static_cast<float>(p.lnx - 1));
    const T fy = v * T(static_cast<float>(p.lny - 1));
    const T fz = w * T(static_cast<float>(p.lnz - 1));
    const int x0 = static_cast<int>(std::floor(fx));
    const int y0 = static_cast<int>(std::floor(fy));
    const int z0 = static_cast<int>(std::floor(fz));
    const int x1 = std::min(x0 + 1, p.lnx - 1);
    const int y1 = std::min(y0 + 1, p.lny - 1);
    const int z1 = std::min(z0 + 1, p.lnz - 1);
    const T tx = fx - T(static_cast<float>(x0));
    const T ty = fy - T(static_cast<float>(y0));
    const T tz = fz - T(static_cast<float>(z0));
    auto at = [&](int x, int y, int z) { return f[(size_t(z) * p.lny + y) * p.lnx + x]; };
    auto l4 = [](V4<T> a, V4<T> b, T t) {
        return V4<T>{lerpf(a.x, b.x, t), lerpf(a.y, b.y, t), lerpf(a.z, b.z, t), lerpf(a.w, b.w, t)};
    };
    const V4<T> c00 = l4(at(x0, y0, z0), at(x1, y0, z0), tx);
    const V4<T> c10 = l4(at(x0, y1, z0), at(x1, y1, z0), tx);
    const V4<T> c01 = l4(at(x0, y0, z1), at(x1, y0, z1), tx);
    const V4<T> c11 = l4(at(x0, y1, z1), at(x1, y1, z1), tx);
    return l4(l4(c00, c10, ty), l4(c01, c11, ty), tz);
}

// src/fire_cuda.cu:653-664 -- nearest light cell.
template <class T> T sampleSceneShadow(const T* f, const Params<T>& p, T u, T v, T w) {
    if (f == nullptr || p.lnx <= 1 || p.lny <= 1 || p.lnz <= 1) return F(1.0);
    u = saturate(u);
    v = saturate(v);
    w = saturate(w);
    const int x = std::min(std::max(static_cast<int>(u * T(static_cast<float>(p.lnx - 1)) + F(0.5)), 0), p.lnx - 1);
    const int y = std::min(std::max(static_cast<int>(v * T(static_cast<float>(p.lny - 1)) + F(0.5)), 0), p.lny - 1);
    const int z = std::min(std::max(static_cast<int>(w * T(static_cast<float>(p.lnz - 1)) + F(0.5)), 0), p.lnz - 1);
    return f[(size_t(z) * p.lny + y) * p.lnx + x];
}

// src/fire_cuda.cu:666-732 -- MacCormack: first-order sample, forward round
// trip, clamp to the eight corners of the first-order cell, blend.
template <class T>
T sampleScalarMacCormack(const T* field, const Params<T>& p, T current, V3<T> prevVel, T prevU, T prevV, T prevW,
                         T blend) {
    const T firstOrder = sampleScalar(field, p, prevU, prevV, prevW);
    const T fwdU = prevU + prevVel.x * p.dt * T(kAdvectionScale);
    const T fwdV = prevV + prevVel.y * p.dt * T(kAdvectionScale);
    const T fwdW = prevW + prevVel.z * p.dt * T(kAdvectionScale);
    const T roundTrip = sampleScalar(field, p, fwdU, fwdV, fwdW);
    const T u = saturate(prevU), v = saturate(prevV), w = saturate(prevW);
    const T fx = u * T(static_cast<float>(p.nx - 1));
    const T fy = v * T(static_cast<float>(p.ny - 1));
    const T fz = w * T(static_cast<float>(p.nz - 1));
    const int x0 = static_cast<int>(std::floor(fx));
    const int y0 = static_cast<int>(std::floor(fy));
    const int z0 = static_cast<int>(std::floor(fz));
    const int x1 = std::min(x0 + 1, p.nx - 1);
    const int y1 = std::min(y0 + 1, p.ny - 1);
    const int z1 = std::min(z0 + 1, p.nz - 1);
    auto at = [&](int x, int y, int z) { return field[(size_t(z) * p.ny + y) * p.nx + x]; };
    T lo = at(x0, y0, z0);
    T hi = lo;
    const T c[7] = {at(x1, y0, z0), at(x0, y1, z0), at(x1, y1, z0), at(x0, y0, z1),
                    at(x1, y0, z1), at(x0, y1, z1), at(x1, y1, z1)};
    for (int i = 0; i < 7; ++i) lo = std::fmin(lo, c[i]);
    for (int i = 0; i < 7; ++i) hi = std::fmax(hi, c[i]);
    const T corrected = std::fmin(hi, std::fmax(lo, firstOrder + F(0.5) * (current - roundTrip)));
    return lerpf(firstOrder, corrected, saturate(blend));
}

// src/fire_cuda.cu:734-744
template <class T> T orientedCapsuleMask(T x, T z, T cx, T cz, T angle, T halfLength, T radius) {
    const T ca = std::cos(angle);
    const T sa = std::sin(angle);
    const T px = x - cx;
    const T pz = z - cz;
    const T qx = px * ca + pz * sa;
    const T qz = -px * sa + pz * ca;
    const T over = std::fmax(std::fabs(qx) - halfLength, F(0.0));
    const T dist = std::sqrt(over * over + qz * qz);
    return smoothstepf(radius, radius * F(0.22), dist);
}

// src/fire_cuda.cu:746-793 -- procedural fuel-bed material per scene.
template <class T> T fuelBedMaterial(T x, T z, const Params<T>& p) {
    if (p.sceneId == 1) {
        const T logA = orientedCapsuleMask(x, z, F(-0.06), F(0.01), F(0.38), F(0.34), F(0.060));
        const T logB = orientedCapsuleMask(x, z, F(0.07), F(-0.02), F(-0.58), F(0.33), F(0.058));
        const T logC = orientedCapsuleMask(x, z, F(0.01), F(0.08), F(1.34), F(0.24), F(0.050));
        const T contactAB = std::fmin(logA, logB) * F(1.25);
        const T contactBC = std::fmin(logB, logC) * F(1.10);
        const T contactCA = std::fmin(logC, logA) * F(0.92);
        const T coalNoise = fbm(v2(x * F(9.4) + z * F(1.7), z * F(11.2) - x * F(3.1)));
        const T coalBed = smoothstepf(F(0.38), F(0.08), std::sqrt(x * x * F(1.35) + z * z * F(2.40))) *
                          smoothstepf(F(0.34), F(0.88), coalNoise);
        const T cracks = smoothstepf(F(0.65), F(0.93), fbm(v2(x * F(21.0) - z * F(6.0), z * F(24.0) + x * F(4.0))));
        const T contactPyrolysis = saturate(contactAB + contactBC + contactCA);
        return saturate((logA * F(0.72) + logB * F(0.70) + logC * F(0.54) + coalBed * F(0.84) +
                         contactPyrolysis * F(1.18)) *
                        (F(1.0) - cracks * F(0.24)));
    }
    if (p.sceneId == 2) {
        const T sourceRadius = std::fmax(F(0.04), p.emitterRadius);
        T source = F(0.0);
        const T cx = p.burnerCenterCount > 0 ? p.burnerCenterX[0] : p.emitterCenterX;
        const T cz = p.burnerCenterCount > 0 ? p.burnerCenterZ[0] : p.emitterCenterZ;
        const T px = x - cx;
        const T pz = z - cz;
        const T radius = std::sqrt(px * px + pz * pz);
        const T angle = std::atan2(pz, px);
        const T ring = smoothstepf(sourceRadius * F(0.072), sourceRadius * F(0.014), std::fabs(radius - sourceRadius));
        const T innerRing =
            smoothstepf(sourceRadius * F(0.052), sourceRadius * F(0.012), std::fabs(radius - sourceRadius * F(0.52)));
        const T ports = F(0.5) + F(0.5) * std::cos(angle * F(32.0));
        const T portMask = smoothstepf(F(0.80), F(0.992), ports);
        const T centerPilot = smoothstepf(sourceRadius * F(0.22), F(0.000), radius) * F(0.045);
        source = std::fmax(source, (ring * (F(0.035) + portMask * F(1.72)) + innerRing * F(0.055) + centerPilot) *
                                       smoothstepf(sourceRadius * F(1.28), sourceRadius * F(1.05), radius));
        return saturate(source);
    }
    const T tray = smoothstepf(F(1.08), F(0.030), std::fabs(x)) * smoothstepf(F(0.56), F(0.026), std::fabs(z));
    const T emberMat = smoothstepf(F(1.00), F(0.018), std::fabs(x)) * smoothstepf(F(0.50), F(0.020), std::fabs(z));
    const T mound = std::exp(-(x * x * F(0.70) + z * z * F(2.15)));
    const T logMass = fbm(v2(x * F(3.7) + z * F(0.9), z * F(5.4) - x * F(0.6)));
    const T chips = fbm(v2(x * F(15.0) + z * F(4.0), z * F(18.0) - x * F(5.0)));
    const T strand = F(0.5) + F(0.5) * std::sin((x * F(19.0) + z * F(7.0)) + fbm(v2(z * F(4.0), x * F(3.0))) * F(4.2));
    const T cracks = smoothstepf(F(0.44), F(0.74), chips) * smoothstepf(F(0.20), F(0.84), logMass);
    const T voids = smoothstepf(F(0.70), F(0.93), chips * F(0.72) + strand * F(0.34));
    const T clumps = smoothstepf(F(0.22), F(0.86), logMass * F(0.82) + chips * F(0.36) + strand * F(0.18));
    const T porousFuel = (F(0.24) + clumps * F(0.94) + emberMat * F(0.20)) * (F(0.64) + mound * F(0.46));
    return saturate(tray * porousFuel * (F(1.0) - cracks * F(0.46)) * (F(1.0) - voids * F(0.34)));
}

// src/fire_cuda.cu:795-803
template <class T> T fuelBedSource(T x, T z, T h, const Params<T>& p) {
    const T material = fuelBedMaterial(x, z, p);
    const T height =
        p.sceneId == 2
            ? smoothstepf(std::fmax(F(0.005), p.emitterHeightBandNorm * F(0.34)),
                          std::fmax(F(0.0015), p.emitterHeightBandNorm * F(0.055)), std::fabs(h - p.emitterHeightNorm))
            : smoothstepf(p.sceneId == 1 ? F(0.245) : F(0.145), F(0.00), h);
    const T emberBreathing =
        F(0.84) + F(0.16) * fbm(v2(x * F(9.0) + p.time * F(0.035), z * F(11.0) - p.time * F(0.025)));
    const T exposedFuel = saturate(material * emberBreathing);
    return saturate(height * exposedFuel);
}

template <class T> inline T cellU(int x, const Params<T>& p) {
    return (T(static_cast<float>(x)) + F(0.5)) / T(static_cast<float>(p.nx));
}
template <class T> inline T cellV(int y, const Params<T>& p) {
    return (T(static_cast<float>(y)) + F(0.5)) / T(static_cast<float>(p.ny));
}
template <class T> inline T cellW(int z, const Params<T>& p) {
    return (T(static_cast<float>(z)) + F(0.5)) / T(static_cast<float>(p.nz));
}

// src/fire_cuda.cu:805-878 + the memsets of :3043-3048 -- seeds every field.
template <class T> void stageReset(State<T>& s, const Params<T>& p) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < p.nz; ++z) {
        for (int y = 0; y < p.ny; ++y) {
            for (int x = 0; x < p.nx; ++x) {
                const size_t idx = size_t(sIdx(p, x, y, z));
                const T u = cellU(x, p), v = cellV(y, p), w = cellW(z, p);
                const T worldX = (u - F(0.50)) * F(2.10);
                const T worldZ = (w - F(0.50)) * F(1.64);
                const T material = fuelBedMaterial(worldX, worldZ, p);
                const T chunkNoise =
                    fbm(v2(worldX * F(18.0) + worldZ * F(2.0), worldZ * F(22.0) - worldX * F(5.0)));
                const T bed = fuelBedSource(worldX, worldZ, v, p);
                const int sc = p.sceneId;
                const T charScale = sc == 2 ? F(0.004) : (sc == 1 ? F(1.18) : F(1.0));
                const T sootScale = sc == 2 ? F(0.004) : (sc == 1 ? F(0.92) : F(1.0));
                s.scalar[HEAT][idx] =
                    bed * (sc == 2 ? F(1.34) : (sc == 1 ? F(0.78) + chunkNoise * F(0.26) : F(0.86) + chunkNoise * F(0.24)));
                s.scalar[FUEL][idx] =
                    bed * (sc == 2 ? F(1.42) : (sc == 1 ? F(1.05) + chunkNoise * F(0.30) : F(1.08) + chunkNoise * F(0.26)));
                s.scalar[OXYGEN][idx] = F(1.0);
                s.scalar[SOOT][idx] = bed * (sc == 2 ? F(0.00065) : F(0.018)) * sootScale;
                s.scalar[CHAR][idx] = material * (F(0.92) + chunkNoise * F(0.72)) * charScale;
                s.scalar[ASH][idx] = material * (F(0.018) + smoothstepf(F(0.56), F(0.86), chunkNoise) * F(0.055)) *
                                     (sc == 2 ? F(0.10) : F(1.0));
                s.scalar[PYRO][idx] = bed * (sc == 2 ? F(0.018)
                                                     : (sc == 1 ? F(0.060) + chunkNoise * F(0.034)
                                                                : F(0.058) + chunkNoise * F(0.028)));
                s.scalar[PROGRESS][idx] = bed * (sc == 2 ? F(0.11) : (sc == 1 ? F(0.24) : F(0.21)));
                s.scalar[TURB][idx] = bed * (sc == 2 ? F(0.012) : (sc == 1 ? F(0.082) : F(0.065)));
                s.scalar[SOOTOPT][idx] = bed * (sc == 2 ? F(0.00050) : F(0.018)) * sootScale;
                s.pressure[idx] = F(0.0);
                s.divergence[idx] = F(0.0);
                s.divergenceAfter[idx] = F(0.0);
            }
        }
    }
    std::fill(s.u.begin(), s.u.end(), F(0.0));
    std::fill(s.v.begin(), s.v.end(), F(0.0));
    std::fill(s.w.begin(), s.w.end(), F(0.0));
    std::fill(s.light.begin(), s.light.end(), V4<T>{});
    std::fill(s.lightNext.begin(), s.lightNext.end(), V4<T>{});
    std::fill(s.shadow.begin(), s.shadow.end(), F(0.0));
}

// src/fire_cuda.cu:880-932 -- semi-Lagrangian self-advection of the three face
// grids.  The backtrace f - vel * dt * 0.62 is one fused multiply-add in the
// reference's build, fma(-(vel * dt), 0.62, f).
template <class T> void stageAdvectVelocity(State<T>& s, const Params<T>& p) {
    std::vector<T> un(s.u.size()), vn(s.v.size()), wn(s.w.size());
    const T back = p.dt * T(kAdvectionScale);
    (void)back;
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < p.nz; ++z) {
        for (int y = 0; y < p.ny; ++y) {
            for (int x = 0; x <= p.nx; ++x) {
                const int o = uIdx(p, x, y, z);
                if (x == 0 || x == p.nx) {
                    un[o] = F(0.0);
                    continue;
                }
                const T fu = T(static_cast<float>(x)) / T(static_cast<float>(p.nx));
                const T fv = cellV(y, p), fw = cellW(z, p);
                const V3<T> vel = sampleVelocity(s, p, fu, fv, fw);
                un[o] = sampleU(s.u.data(), p, std::fma(-(vel.x * p.dt), T(kAdvectionScale), fu),
                                std::fma(-(vel.y * p.dt), T(kAdvectionScale), fv), std::fma(-(vel.z * p.dt), T(kAdvectionScale), fw)) *
                        F(0.995);
            }
        }
    }
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < p.nz; ++z) {
        for (int y = 0; y <= p.ny; ++y) {
            for (int x = 0; x < p.nx; ++x) {
                const int o = vIdx(p, x, y, z);
                if (y == 0) {
                    vn[o] = F(0.0);
                    continue;
                }
                const T fu = cellU(x, p);
                const T fv = T(static_cast<float>(y)) / T(static_cast<float>(p.ny));
                const T fw = cellW(z, p);
                const V3<T> vel = sampleVelocity(s, p, fu, fv, fw);
                vn[o] = sampleV(s.v.data(), p, std::fma(-(vel.x * p.dt), T(kAdvectionScale), fu),
                                std::fma(-(vel.y * p.dt), T(kAdvectionScale), fv), std::fma(-(vel.z * p.dt), T(kAdvectionScale), fw)) *
                        F(0.996);
            }
        }
    }
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z <= p.nz; ++z) {
        for (int y = 0; y < p.ny; ++y) {
            for (int x = 0; x < p.nx; ++x) {
                const int o = wIdx(p, x, y, z);
                if (z == 0 || z == p.nz) {
                    wn[o] = F(0.0);
                    continue;
                }
                const T fu = cellU(x, p), fv = cellV(y, p);
                const T fw = T(static_cast<float>(z)) / T(static_cast<float>(p.nz));
                const V3<T> vel = sampleVelocity(s, p, fu, fv, fw);
                wn[o] = sampleW(s.w.data(), p, std::fma(-(vel.x * p.dt), T(kAdvectionScale), fu),
                                std::fma(-(vel.y * p.dt), T(kAdvectionScale), fv), std::fma(-(vel.z * p.dt), T(kAdvectionScale), fw)) *
                        F(0.995);
            }
        }
    }
    s.u.swap(un);
    s.v.swap(vn);
    s.w.swap(wn);
}

// src/fire_cuda.cu:934-1126 -- advection of the ten scalars and the reaction network.
template <class T> void stageAdvectReact(State<T>& s, const Params<T>& p) {
    std::vector<T> out[10];
    for (int i = 0; i < 10; ++i) out[i].resize(s.cells());
    const T* in[10];
    for (int i = 0; i < 10; ++i) in[i] = s.scalar[i].data();
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (int z = 0; z < p.nz; ++z) {
        for (int y = 0; y < p.ny; ++y) {
            for (int x = 0; x < p.nx; ++x) {
                const T u = cellU(x, p), v = cellV(y, p), w = cellW(z, p);
                const size_t idx = (size_t(z) * p.ny + y) * p.nx + x;
                const T currentActivity = in[HEAT][idx] + in[FUEL][idx] * F(0.18) + in[SOOT][idx] * F(0.24) +
                                          in[PYRO][idx] * F(0.20) + in[PROGRESS][idx] * F(0.14) +
                                          in[SOOTOPT][idx] * F(0.08) + in[TURB][idx] * F(0.06);
                const T sourceDx = u - p.mouseX;
                const T sourceDy = v - p.mouseY;
                const T sourceDz = w - F(0.5);
                const bool outsideInteractiveSource =
                    p.leftDown == 0 || (sourceDx * sourceDx + sourceDy * sourceDy + sourceDz * sourceDz) > F(0.090);
                if (v > F(0.18) && currentActivity < F(0.00035) && in[CHAR][idx] < F(0.00010) &&
                    in[ASH][idx] < F(0.00010) && outsideInteractiveSource && p.rightDown == 0) {
                    out[HEAT][idx] = F(0.0);
                    out[FUEL][idx] = F(0.0);
                    out[OXYGEN][idx] = std::fmin(F(1.0), in[OXYGEN][idx] + (F(1.0) - in[OXYGEN][idx]) * p.dt * F(0.08));
                    out[SOOT][idx] = F(0.0);
                    out[CHAR][idx] = in[CHAR][idx];
                    out[ASH][idx] = in[ASH][idx];
                    out[PYRO][idx] = F(0.0);
                    out[PROGRESS][idx] = F(0.0);
                    out[TURB][idx] = in[TURB][idx] * std::fmax(F(0.0), F(1.0) - p.dt * F(0.54));
                    out[SOOTOPT][idx] = F(0.0);
                    continue;
                }
                const V3<T> vel = sampleVelocity(s, p, u, v, w);
                const T prevU = u - vel.x * p.dt * T(kAdvectionScale);
                const T prevV = v - vel.y * p.dt * T(kAdvectionScale);
                const T prevW = w - vel.z * p.dt * T(kAdvectionScale);
                const V3<T> prevVel = sampleVelocity(s, p, prevU, prevV, prevW);

                const T antiDiffusion = saturate(F(0.30) + p.detail * F(0.34));
                auto mc = [&](int f, T blend) {
                    return sampleScalarMacCormack(in[f], p, in[f][idx], prevVel, prevU, prevV, prevW, blend);
                };
                T heat = mc(HEAT, antiDiffusion);
                T fuel = mc(FUEL, antiDiffusion * F(0.92));
                T oxygen = mc(OXYGEN, antiDiffusion * F(0.70));
                T soot = mc(SOOT, antiDiffusion);
                T charMass = in[CHAR][idx];
                T ash = in[ASH][idx];
                T pyrolysisRate = mc(PYRO, antiDiffusion * F(0.72)) * F(0.55);
                T progress = mc(PROGRESS, antiDiffusion * F(0.82));
                T turbulenceEnergy = mc(TURB, antiDiffusion * F(0.52));
                T sootOptics = mc(SOOTOPT, antiDiffusion * F(0.72));

                const int sc = p.sceneId;
                const T worldX = (u - F(0.50)) * F(2.10);
                const T worldZ = (w - F(0.50)) * F(1.64);
                const T material = fuelBedMaterial(worldX, worldZ, p);
                const T sourceNoise =
                    F(0.70) + F(0.48) * fbm(v2(worldX * F(13.0) + worldZ * F(3.0) + p.time * F(0.38),
                                               v * F(31.0) + worldZ * F(11.0)));
                const T exposedChar = saturate(charMass / std::fmax(F(0.055), charMass + ash * F(1.75)));
                const T charEdges = smoothstepf(F(0.06), F(0.78), material) * smoothstepf(F(0.92), F(0.02), ash);
                const T gasFeed = sc == 2 ? F(1.18) : exposedChar * charEdges;
                const T scenePyrolysisGain = sc == 2 ? F(0.42) : (sc == 1 ? F(1.34) : F(1.0));
                const T sceneFuelGain = sc == 2 ? F(0.46) : (sc == 1 ? F(1.18) : F(1.0));
                const T sceneHeatGain = sc == 2 ? F(1.18) : (sc == 1 ? F(1.08) : F(1.0));
                const T sceneSootGain = sc == 2 ? F(0.18) : (sc == 1 ? F(1.22) : F(1.0));
                const T bed = fuelBedSource(worldX, worldZ, v, p) * sourceNoise * gasFeed * p.intensity;
                const T ambientK = F(293.0);
                T tempK = ambientK + heat * F(335.0);
                const T radiativeFeedback = smoothstepf(F(430.0), F(980.0), tempK);
                const T solidOxygen = saturate(oxygen * F(1.28) - soot * F(0.030));
                const T heatFlux = saturate((tempK - F(405.0)) / F(900.0)) + bed * F(0.34) + sootOptics * F(0.024);
                const T charRelease = std::fmin(
                    charMass, charMass * heatFlux * solidOxygen * (F(0.14) + radiativeFeedback * F(1.38)) * p.dt);
                pyrolysisRate += (bed * (F(0.34) + radiativeFeedback * F(1.05)) * p.dt +
                                  charRelease * (F(2.45) + sourceNoise * F(0.72))) *
                                 scenePyrolysisGain;
                charMass += material * p.dt * (sc == 2 ? F(0.00005) : (sc == 1 ? F(0.050) : F(0.026)));
                charMass -= charRelease * F(0.92);
                ash += charRelease * (sc == 2 ? F(0.025) : F(0.16) + F(0.22) * saturate(F(1.0) - oxygen));

                heat += (bed * (sc == 2 ? F(10.40) : F(6.20)) * p.dt * (F(1.0) + radiativeFeedback * F(1.12)) +
                         charRelease * F(3.35)) *
                        sceneHeatGain;
                fuel += pyrolysisRate * (sc == 2 ? F(1.34) : F(3.70)) * sceneFuelGain;
                soot += pyrolysisRate * (F(0.090) + ash * F(0.032) + saturate(F(1.0) - oxygen) * F(0.13)) * p.smokeGain *
                        (sc == 2 ? F(0.010) : (sc == 1 ? F(0.92) : F(1.0))) * sceneSootGain;

                if (p.leftDown != 0) {
                    const T mx = p.mouseX;
                    const T my = p.mouseY;
                    const T source = std::exp(-((u - mx) * (u - mx)) / F(0.0180) -
                                              ((w - F(0.5)) * (w - F(0.5))) / F(0.0550) -
                                              ((v - my) * (v - my)) / F(0.0020));
                    heat += source * p.dt * F(2.8);
                    fuel += source * p.dt * F(1.4);
                    pyrolysisRate += source * p.dt * F(0.45);
                    progress += source * p.dt * F(0.75);
                    turbulenceEnergy += source * p.dt * F(0.28);
                    oxygen = std::fmax(oxygen, F(0.72) + source * F(0.20));
                }
                if (p.rightDown != 0) {
                    const T source = std::exp(
                        -((u - p.mouseX) * (u - p.mouseX) + (w - F(0.5)) * (w - F(0.5))) / F(0.0100) -
                        (v - p.mouseY) * (v - p.mouseY) / F(0.0100));
                    soot += source * p.dt * F(8.0);
                    heat *= F(1.0) - source * p.dt * F(1.2);
                    fuel *= F(1.0) - source * p.dt * F(0.7);
                }

                tempK = ambientK + heat * F(335.0);
                const T thermalActivation = smoothstepf(F(575.0), F(1220.0), tempK);
                const T arrhenius = std::exp(F(-3800.0) / std::fmax(F(640.0), tempK));
                const T oxygenLimited = std::fmin(fuel, oxygen * F(1.42));
                const T burnMass = std::fmin(oxygenLimited, oxygenLimited * thermalActivation * arrhenius *
                                                                (F(118.0) + p.intensity * F(34.0)) * p.dt);
                const T incomplete = saturate(F(1.0) - oxygen * F(1.30) + fuel * F(0.065) + soot * F(0.015));
                const T heatRelease = burnMass * F(7.0);
                const T sootYield = burnMass * (F(0.035) + incomplete * F(0.34)) * p.smokeGain *
                                    (sc == 2 ? F(0.006) : (sc == 1 ? F(0.96) : F(1.0)));
                const T sootOxidation = soot * oxygen * smoothstepf(F(760.0), F(1540.0), tempK) * p.dt * F(0.82);
                const T frontProduction =
                    burnMass * (F(9.8) + turbulenceEnergy * F(3.4)) + pyrolysisRate * F(0.70) + charRelease * F(2.10);
                const T boundaryAir = smoothstepf(F(0.70), F(0.96), v) + smoothstepf(F(0.11), F(0.03), u) +
                                      smoothstepf(F(0.89), F(0.97), u) + smoothstepf(F(0.11), F(0.03), w) +
                                      smoothstepf(F(0.89), F(0.97), w);
                const T upperEntrainment = smoothstepf(F(0.52), F(0.98), v);

                heat += heatRelease;
                fuel -= burnMass * F(1.20);
                oxygen -= burnMass * F(0.98);
                soot += sootYield;
                soot -= sootOxidation;
                progress += frontProduction;
                progress *= std::exp(-p.dt * (F(0.72) + v * F(0.45) + oxygen * F(0.16) + saturate(boundaryAir) * F(1.05) +
                                              upperEntrainment * F(0.26)));

                oxygen = lerpf(oxygen, F(1.0), saturate(boundaryAir) * p.dt * F(1.7));
                oxygen += (F(1.0) - oxygen) * p.dt * F(0.08);

                tempK = ambientK + heat * F(335.0);
                const T radiationBase = std::fmax(F(0.0), (tempK - ambientK) / F(1560.0));
                const T radiationSq = radiationBase * radiationBase;
                const T radiationLoss = radiationSq * radiationSq;
                heat -= radiationLoss * p.dt * (F(0.88) + soot * F(0.085) + sootOptics * F(0.018));
                heat *= std::exp(-p.dt * (F(0.31) + v * F(0.64) + soot * F(0.022) + saturate(boundaryAir) * F(0.26) +
                                          upperEntrainment * F(0.18)));
                fuel *= std::exp(-p.dt * (F(0.58) + heat * F(0.20) + v * F(0.92) + saturate(boundaryAir) * F(0.18)));
                soot *= std::exp(-p.dt * (F(0.060) + v * F(0.092) + oxygen * F(0.028) + saturate(boundaryAir) * F(0.96) +
                                          upperEntrainment * F(0.22)));
                pyrolysisRate *= std::exp(-p.dt * (F(1.55) + v * F(0.58) + saturate(boundaryAir) * F(0.18)));

                const T uL = s.u[(size_t(z) * p.ny + y) * (p.nx + 1) + x];
                const T uR = s.u[(size_t(z) * p.ny + y) * (p.nx + 1) + x + 1];
                const T vD = s.v[(size_t(z) * (p.ny + 1) + y) * p.nx + x];
                const T vU = s.v[(size_t(z) * (p.ny + 1) + y + 1) * p.nx + x];
                const T wB = s.w[(size_t(z) * p.ny + y) * p.nx + x];
                const T wF = s.w[(size_t(z + 1) * p.ny + y) * p.nx + x];
                const T shear = std::fabs(uR - uL) + std::fabs(vU - vD) + std::fabs(wF - wB);
                const T flameActivity = saturate(progress * F(0.64) + burnMass * F(5.2) + heat * F(0.065));
                turbulenceEnergy += p.dt * (shear * (F(0.72) + progress * F(0.06)) +
                                            flameActivity * p.turbulence * F(0.62) + frontProduction * F(0.085) +
                                            soot * F(0.018));
                turbulenceEnergy *= std::exp(-p.dt * (F(0.54) + v * F(0.24) + saturate(boundaryAir) * F(0.42) +
                                                      upperEntrainment * F(0.16)));
                const T particleGrowth =
                    saturate(incomplete * F(0.36) + ash * F(0.13) + soot * F(0.055) +
                             smoothstepf(F(0.65), F(1.55), tempK / F(1000.0)) * F(0.18));
                sootOptics = soot * (F(1.04) + F(0.28) * std::sqrt(std::fmax(F(0.0), heat)) + F(0.24) * ash +
                                     F(0.46) * particleGrowth);
                sootOptics = lerpf(sootOptics, sootOptics * F(0.48), saturate(sootOxidation * F(0.92)));

                out[HEAT][idx] = std::fmin(F(8.8), std::fmax(F(0.0), heat));
                out[FUEL][idx] = std::fmin(F(5.5), std::fmax(F(0.0), fuel));
                out[OXYGEN][idx] = std::fmin(F(1.0), std::fmax(F(0.0), oxygen));
                out[SOOT][idx] = std::fmin(F(7.4), std::fmax(F(0.0), soot));
                out[CHAR][idx] = std::fmin(F(2.8), std::fmax(F(0.0), charMass));
                out[ASH][idx] = std::fmin(F(1.9), std::fmax(F(0.0), ash));
                out[PYRO][idx] = std::fmin(F(3.6), std::fmax(F(0.0), pyrolysisRate));
                out[PROGRESS][idx] = std::fmin(F(3.4), std::fmax(F(0.0), progress));
                out[TURB][idx] = std::fmin(F(4.2), std::fmax(F(0.0), turbulenceEnergy));
                out[SOOTOPT][idx] = std::fmin(F(10.0), std::fmax(F(0.0), sootOptics));
            }
        }
    }
    for (int i = 0; i < 10; ++i) s.scalar[i].swap(out[i]);
}

// src/fire_cuda.cu:1128-1183 -- buoyancy, curl noise, vortex feedback, wind.
// All face velocities are read before any force is added; shared faces
// receive their two contributions lower cell first (see the file header).
template <class T> void stageForce(State<T>& s, const Params<T>& p) {
    const size_t n = s.cells();
    std::vector<T> dv(n), du(n), dw(n);
    const T* heat = s.scalar[HEAT].data();
    const T* soot = s.scalar[SOOT].data();
    const T* turb = s.scalar[TURB].data();
    const T* prog = s.scalar[PROGRESS].data();
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < p.nz; ++z) {
        for (int y = 0; y < p.ny; ++y) {
            for (int x = 0; x < p.nx; ++x) {
                const size_t idx = size_t(sIdx(p, x, y, z));
                const T h = heat[idx];
                const T sv = soot[idx];
                const T k = turb[idx];
                const T c = prog[idx];
                const T u = cellU(x, p), v = cellV(y, p), w = cellW(z, p);
                const T gradX = heat[sIdx(p, x + 1, y, z)] - heat[sIdx(p, x - 1, y, z)];
                const T gradY = heat[sIdx(p, x, y + 1, z)] - heat[sIdx(p, x, y - 1, z)];
                const T gradZ = heat[sIdx(p, x, y, z + 1)] - heat[sIdx(p, x, y, z - 1)];
                const T uL = s.u[uIdx(p, x, y, z)];
                const T uR = s.u[uIdx(p, x + 1, y, z)];
                const T vD = s.v[vIdx(p, x, y, z)];
                const T vU = s.v[vIdx(p, x, y + 1, z)];
                const T wB = s.w[wIdx(p, x, y, z)];
                const T wF = s.w[wIdx(p, x, y, z + 1)];
                const T curlX = (wF - wB) - (vU - vD);
                const T curlY = (uR - uL) - (wF - wB);
                const T curlZ = (vU - vD) - (uR - uL);
                const T curlMagnitude = std::fabs(curlX) + std::fabs(curlY) + std::fabs(curlZ);
                const T curlNoiseA =
                    fbm(v2(u * F(9.0) + w * F(3.7) + p.time * F(0.22), v * F(13.0) - p.time * F(0.31))) - F(0.5);
                const T curlNoiseB =
                    fbm(v2(w * F(10.0) - p.time * F(0.19), u * F(8.0) + v * F(5.5) + p.time * F(0.27))) - F(0.5);
                const T thermalActivity = smoothstepf(F(0.04), F(4.20), h + sv * F(0.28));
                const T upperDrag = smoothstepf(F(0.26), F(0.94), v);
                const T lesGain = std::sqrt(std::fmax(F(0.0), k)) * (F(0.30) + c * F(0.54));
                const int sc = p.sceneId;
                const T sceneCurlScale = sc == 2 ? F(0.38) : (sc == 1 ? F(1.18) : F(1.0));
                const T sceneBuoyancyScale = sc == 2 ? F(0.42) : (sc == 1 ? F(1.06) : F(1.0));
                const T curlGain = p.turbulence * sceneCurlScale * (F(0.18) + thermalActivity * F(0.82) + lesGain * F(1.12));
                const T vortexGain =
                    p.turbulence * sceneCurlScale * thermalActivity * saturate(curlMagnitude * F(0.46)) * F(0.68);
                const T buoyancyFade = sc == 2 ? smoothstepf(F(0.24), F(0.035), v) : smoothstepf(F(0.96), F(0.08), v);
                const T verticalVelocity = F(0.5) * (vD + vU);
                const T verticalDamping = verticalVelocity * (F(0.10) + upperDrag * F(0.72) + sv * F(0.020));
                const T buoyancy = h * sceneBuoyancyScale * (F(1.62) + p.turbulence * F(0.34) + c * F(0.16)) * buoyancyFade -
                                   sv * F(0.095) - gradY * F(0.18) - verticalDamping;
                dv[idx] = p.dt * (buoyancy + curlY * vortexGain * F(0.22));
                du[idx] = p.dt * (p.wind * (F(0.34) + v * F(0.96)) +
                                  (-gradZ * F(1.36) + curlNoiseA * (F(0.20) + upperDrag * F(0.16)) + curlX * vortexGain) *
                                      curlGain);
                dw[idx] = p.dt * ((gradX * F(1.36) + curlNoiseB * (F(0.20) + upperDrag * F(0.16)) + curlZ * vortexGain) *
                                  curlGain);
            }
        }
    }
    // Face gathers in a fixed order (lower cell first).
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < p.nz; ++z) {
        for (int y = 0; y < p.ny; ++y) {
            for (int x = 0; x <= p.nx; ++x) {
                T val = s.u[uIdx(p, x, y, z)];
                if (x > 0) val += du[sIdx(p, x - 1, y, z)];
                if (x < p.nx) val += du[sIdx(p, x, y, z)];
                s.u[uIdx(p, x, y, z)] = val;
            }
        }
    }
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < p.nz; ++z) {
        for (int y = 1; y <= p.ny; ++y) {
            for (int x = 0; x < p.nx; ++x) {
                s.v[vIdx(p, x, y, z)] += dv[sIdx(p, x, y - 1, z)];
            }
        }
    }
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z <= p.nz; ++z) {
        for (int y = 0; y < p.ny; ++y) {
            for (int x = 0; x < p.nx; ++x) {
                T val = s.w[wIdx(p, x, y, z)];
                if (z > 0) val += dw[sIdx(p, x, y, z - 1)];
                if (z < p.nz) val += dw[sIdx(p, x, y, z)];
                s.w[wIdx(p, x, y, z)] = val;
            }
        }
    }
}

// src/fire_cuda.cu:1261-1291 -- wall zeroing and clamps.
template <class T> void stageVelocityBoundary(State<T>& s, const Params<T>& p, bool clampValues) {
    const long nu = long(p.nx + 1) * p.ny * p.nz, nv = long(p.nx) * (p.ny + 1) * p.nz, nw = long(p.nx) * p.ny * (p.nz + 1);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < nu; ++i) {
        const int x = int(i % (p.nx + 1));
        if (x == 0 || x == p.nx) s.u[i] = F(0.0);
        else if (clampValues) s.u[i] = std::fmin(F(4.0), std::fmax(F(-4.0), s.u[i]));
    }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < nv; ++i) {
        const int y = int((i / p.nx) % (p.ny + 1));
        if (y == 0) s.v[i] = F(0.0);
        else if (clampValues) s.v[i] = std::fmin(F(6.4), std::fmax(F(-0.9), s.v[i]));
    }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < nw; ++i) {
        const int z = int(i / (long(p.nx) * p.ny));
        if (z == 0 || z == p.nz) s.w[i] = F(0.0);
        else if (clampValues) s.w[i] = std::fmin(F(4.0), std::fmax(F(-4.0), s.w[i]));
    }
}

// src/fire_cuda.cu:1185-1199 and :1247-1259 -- div = -(sum of face differences), h = 1.
template <class T> void computeDivergence(const State<T>& s, const Params<T>& p, std::vector<T>& div) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < p.nz; ++z) {
        for (int y = 0; y < p.ny; ++y) {
            for (int x = 0; x < p.nx; ++x) {
                const T d = s.u[uIdx(p, x + 1, y, z)] - s.u[uIdx(p, x, y, z)] + s.v[vIdx(p, x, y + 1, z)] -
                            s.v[vIdx(p, x, y, z)] + s.w[wIdx(p, x, y, z + 1)] - s.w[wIdx(p, x, y, z)];
                div[sIdx(p, x, y, z)] = -d;
            }
        }
    }
}

// src/fire_cuda.cu:1201-1227 + loop :3280-3284 -- in-place red-black SOR,
// Neumann walls through the clamped index map.  The reference's sm_100a build
// evaluates pressure + omega * (sum / 6 - pressure) as two fused multiply-adds,
// fma(omega, fma(sum, 1/6, -p), p): every cell of a B200 half sweep matches
// that form and none of the unfused ones, so the float oracle rounds it so.
template <class T> void stagePressureSor(State<T>& s, const Params<T>& p) {
    T* pr = s.pressure.data();
    const T* div = s.divergence.data();
    const T omega = T(s.pressureOmega);
    for (int it = 0; it < s.pressureIterations; ++it) {
        for (int parity = 0; parity < 2; ++parity) {
#pragma omp parallel for collapse(2) schedule(static)
            for (int z = 0; z < p.nz; ++z) {
                for (int y = 0; y < p.ny; ++y) {
                    const int firstX = (parity ^ y ^ z) & 1;
                    for (int x = firstX; x < p.nx; x += 2) {
                        const int idx = sIdx(p, x, y, z);
                        const T pL = pr[sIdx(p, x - 1, y, z)];
                        const T pR = pr[sIdx(p, x + 1, y, z)];
                        const T pD = pr[sIdx(p, x, y - 1, z)];
                        const T pU = pr[sIdx(p, x, y + 1, z)];
                        const T pB = pr[sIdx(p, x, y, z - 1)];
                        const T pF = pr[sIdx(p, x, y, z + 1)];
                        const T sum = div[idx] + pL + pR + pD + pU + pB + pF;
                        pr[idx] = std::fma(omega, std::fma(sum, T(1.0f / 6.0f), -pr[idx]), pr[idx]);
                    }
                }
            }
        }
    }
}

// src/fire_cuda.cu:1229-1245 -- u -= grad p on interior faces.
template <class T> void stageSubtract(State<T>& s, const Params<T>& p) {
    const T* pr = s.pressure.data();
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < p.nz; ++z) {
        for (int y = 0; y < p.ny; ++y) {
            for (int x = 0; x < p.nx; ++x) {
                if (x > 0) s.u[uIdx(p, x, y, z)] -= pr[sIdx(p, x, y, z)] - pr[sIdx(p, x - 1, y, z)];
                if (y > 0) s.v[vIdx(p, x, y, z)] -= pr[sIdx(p, x, y, z)] - pr[sIdx(p, x, y - 1, z)];
                if (z > 0) s.w[wIdx(p, x, y, z)] -= pr[sIdx(p, x, y, z)] - pr[sIdx(p, x, y, z - 1)];
            }
        }
    }
}

// src/fire_cuda.cu:359-368
template <class T> T volumeDomainFade(T u, T v, T w) {
    const T side = smoothstepf(F(0.000), F(0.095), u) * smoothstepf(F(1.000), F(0.905), u) *
                   smoothstepf(F(0.000), F(0.100), w) * smoothstepf(F(1.000), F(0.900), w);
    const T floorFade = smoothstepf(F(0.000), F(0.018), v);
    const T topFade = smoothstepf(F(1.000), F(0.520), v);
    return saturate(side * floorFade * topFade);
}

// src/fire_cuda.cu:1420-1443
template <class T> V3<T> blackbodyColor(T tempK) {
    const T t = std::fmax(F(1000.0), std::fmin(F(12000.0), tempK)) / F(100.0);
    T r = F(0.0), g = F(0.0), b = F(0.0);
    if (t <= F(66.0)) {
        r = F(1.0);
        g = saturate((F(99.4708025861) * std::log(t) - F(161.1195681661)) / F(255.0));
    } else {
        r = saturate(F(329.698727446) * std::pow(t - F(60.0), F(-0.1332047592)) / F(255.0));
        g = saturate(F(288.1221695283) * std::pow(t - F(60.0), F(-0.0755148492)) / F(255.0));
    }
    if (t >= F(66.0)) b = F(1.0);
    else if (t <= F(19.0)) b = F(0.0);
    else b = saturate((F(138.5177312231) * std::log(t - F(10.0)) - F(305.0447927307)) / F(255.0));
    return {r, g, b};
}

// src/fire_cuda.cu:1445-1525 -- quarter-resolution radiance/extinction and shadow volume.
template <class T> void stageLightBuild(State<T>& s, const Params<T>& p) {
    const T* f[10];
    for (int i = 0; i < 10; ++i) f[i] = s.scalar[i].data();
#pragma omp parallel for collapse(2) schedule(static)
    for (int lz = 0; lz < p.lnz; ++lz) {
        for (int ly = 0; ly < p.lny; ++ly) {
            for (int lx = 0; lx < p.lnx; ++lx) {
                const T u = (T(static_cast<float>(lx)) + F(0.5)) / T(static_cast<float>(p.lnx));
                const T v = (T(static_cast<float>(ly)) + F(0.5)) / T(static_cast<float>(p.lny));
                const T w = (T(static_cast<float>(lz)) + F(0.5)) / T(static_cast<float>(p.lnz));
                const T domainFade = volumeDomainFade(u, v, w);
                const T heat = sampleScalar(f[HEAT], p, u, v, w);
                const T fuel = sampleScalar(f[FUEL], p, u, v, w);
                const T oxygen = sampleScalar(f[OXYGEN], p, u, v, w);
                const T soot = sampleScalar(f[SOOT], p, u, v, w);
                const T charMass = sampleScalar(f[CHAR], p, u, v, w);
                const T ash = sampleScalar(f[ASH], p, u, v, w);
                const T pyrolysis = sampleScalar(f[PYRO], p, u, v, w);
                const T progress = sampleScalar(f[PROGRESS], p, u, v, w);
                const T sootOptics = sampleScalar(f[SOOTOPT], p, u, v, w);
                const T cellX = F(1.0) / T(static_cast<float>(p.nx));
                const T cellY = F(1.0) / T(static_cast<float>(p.ny));
                const T cellZ = F(1.0) / T(static_cast<float>(p.nz));
                const T gradHeatX = sampleScalar(f[HEAT], p, u + cellX, v, w) - sampleScalar(f[HEAT], p, u - cellX, v, w);
                const T gradHeatY = sampleScalar(f[HEAT], p, u, v + cellY, w) - sampleScalar(f[HEAT], p, u, v - cellY, w);
                const T gradHeatZ = sampleScalar(f[HEAT], p, u, v, w + cellZ) - sampleScalar(f[HEAT], p, u, v, w - cellZ);
                const T frontGradient = std::sqrt(gradHeatX * gradHeatX + gradHeatY * gradHeatY + gradHeatZ * gradHeatZ) +
                                        fuel * oxygen * F(0.035) + progress * F(0.16);
                const T fineNoise = fbm3(v3(u * F(34.0) + p.time * F(0.45), v * F(42.0) - p.time * F(0.82),
                                            w * F(34.0) + p.time * F(0.22)));
                const T shearNoise = fbm3(v3(u * F(12.0) - p.time * F(0.38), v * F(11.0) - p.time * F(0.62),
                                             w * F(13.0) + p.time * F(0.20)));
                const T reactionFront = smoothstepf(F(0.035), F(0.54), frontGradient + pyrolysis * F(0.10));
                const T flameHeightFade = smoothstepf(F(0.70), F(0.070), v);
                const T lowerShadowColumn = smoothstepf(F(0.62), F(0.06), v);
                const T plumeShadowColumn = smoothstepf(F(0.12), F(0.88), v);
                const T sheetGate = smoothstepf(F(0.56), F(0.94), fineNoise * F(0.48) + shearNoise * F(0.42) +
                                                                     reactionFront * F(0.26) + heat * F(0.018)) *
                                    smoothstepf(F(0.04), F(0.86), reactionFront) * flameHeightFade;
                const T sheetCore = saturate(sheetGate * (F(0.42) + progress * F(0.22) + pyrolysis * F(0.34)));
                const T tempK = F(293.0) + heat * F(360.0) + fuel * F(44.0) + pyrolysis * F(120.0) + progress * F(70.0) +
                                sheetCore * F(1020.0);
                const T flameEmitter = domainFade * smoothstepf(F(820.0), F(1880.0), tempK) *
                                       smoothstepf(F(0.010), F(0.68), fuel + pyrolysis * F(0.30) + heat * F(0.040)) *
                                       smoothstepf(F(0.030), F(0.82), oxygen) * reactionFront * sheetGate *
                                       (F(0.24) + sheetCore * F(1.42));
                const T emberEmitter = smoothstepf(F(0.002), F(0.22), charMass + ash * F(0.18)) *
                                       smoothstepf(F(0.09), F(0.00), v) *
                                       (F(0.10) + heat * F(0.012) + pyrolysis * F(0.050));
                const T sootAttenuation = std::exp(-(sootOptics * F(0.25) + soot * F(0.090) + ash * F(0.035)));
                const V3<T> flame = mul3(blackbodyColor(tempK), flameEmitter * sootAttenuation * F(3.40));
                const V3<T> coal = mul3(V3<T>{F(1.0), F(0.22), F(0.040)}, emberEmitter * p.reflectionGain * F(0.20));
                const T extinction = saturate(sootOptics * (F(0.26) + plumeShadowColumn * F(0.42)) +
                                              soot * (F(0.065) + plumeShadowColumn * F(0.20)) + ash * F(0.050) +
                                              progress * lowerShadowColumn * F(0.020));
                const size_t idx = (size_t(lz) * p.lny + ly) * p.lnx + lx;
                s.light[idx] = {flame.x + coal.x, flame.y + coal.y, flame.z + coal.z, extinction};
                const T verticalDepth = v * (F(1.0) + plumeShadowColumn * F(0.70));
                const T radialDepth = std::exp(-((u - F(0.50)) * (u - F(0.50)) * F(5.5) + (w - F(0.50)) * (w - F(0.50)) * F(7.0)));
                const T opticalShadow = sootOptics * (F(0.62) + plumeShadowColumn * F(1.15)) +
                                        soot * (F(0.22) + plumeShadowColumn * F(0.46)) + ash * F(0.072);
                s.shadow[idx] = std::exp(-(opticalShadow * (F(0.72) + verticalDepth * F(0.42)) +
                                           radialDepth * opticalShadow * F(0.34) + progress * F(0.035)));
            }
        }
    }
}

// src/fire_cuda.cu:1527-1565, run twice per step (:3313-3314).
template <class T>
void propagateLight(std::vector<V4<T>>& out, const std::vector<V4<T>>& in, const std::vector<T>& shadow,
                    const Params<T>& p, T diffusion, T decay) {
    static const int dx[6] = {-1, 1, 0, 0, 0, 0};
    static const int dy[6] = {0, 0, -1, 1, 0, 0};
    static const int dz[6] = {0, 0, 0, 0, -1, 1};
#pragma omp parallel for collapse(2) schedule(static)
    for (int lz = 0; lz < p.lnz; ++lz) {
        for (int ly = 0; ly < p.lny; ++ly) {
            for (int lx = 0; lx < p.lnx; ++lx) {
                const size_t idx = (size_t(lz) * p.lny + ly) * p.lnx + lx;
                const V4<T> center = in[idx];
                V3<T> neighbor = {F(0.0), F(0.0), F(0.0)};
                T weight = F(0.0);
                for (int i = 0; i < 6; ++i) {
                    const int sx = std::min(std::max(lx + dx[i], 0), p.lnx - 1);
                    const int sy = std::min(std::max(ly + dy[i], 0), p.lny - 1);
                    const int sz = std::min(std::max(lz + dz[i], 0), p.lnz - 1);
                    const V4<T> smp = in[(size_t(sz) * p.lny + sy) * p.lnx + sx];
                    const T occlusion = std::exp(-smp.w * F(0.42));
                    neighbor = add3(neighbor, mul3(V3<T>{smp.x, smp.y, smp.z}, occlusion));
                    weight += occlusion;
                }
                neighbor = mul3(neighbor, F(1.0) / std::fmax(F(0.0001), weight));
                const T sh = shadow[idx];
                const V3<T> direct = {center.x, center.y, center.z};
                const V3<T> bounced = lerp3(direct, neighbor, diffusion);
                const T floorLift =
                    smoothstepf(F(0.10), F(0.00), (T(static_cast<float>(ly)) + F(0.5)) / T(static_cast<float>(p.lny)));
                const V3<T> contactBounce = mul3(V3<T>{F(1.0), F(0.40), F(0.12)}, floorLift * luminance3(direct) * F(0.18));
                const V3<T> next = add3(mul3(bounced, decay * (F(0.66) + sh * F(0.34))), contactBounce);
                out[idx] = {next.x, next.y, next.z, center.w};
            }
        }
    }
}

template <class T> void stageLightPropagate(State<T>& s, const Params<T>& p) {
    propagateLight(s.lightNext, s.light, s.shadow, p, F(0.48), F(0.92));
    propagateLight(s.light, s.lightNext, s.shadow, p, F(0.34), F(0.96));
}

// src/fire_cuda.cu:1575-1587
template <class T> V3<T> fireVolumeUvFromWorld(V3<T> q) {
    return {saturate((q.x + F(1.05)) / F(2.10)), saturate((q.y - F(0.02)) / F(2.03)), saturate((q.z + F(0.82)) / F(1.64))};
}
template <class T> V3<T> fireVolumeWorldFromUv(V3<T> uv) {
    return {uv.x * F(2.10) - F(1.05), uv.y * F(2.03) + F(0.02), uv.z * F(1.64) - F(0.82)};
}

// src/fire_cuda.cu:1589-1626
template <class T>
V3<T> gatherSceneIrradiance(V3<T> hit, V3<T> normal, const V4<T>* lightF, const T* shadowF, const Params<T>& p) {
    V3<T> irradiance = {F(0.0), F(0.0), F(0.0)};
    for (int i = 0; i < 3; ++i) {
        V3<T> sampleUv = {F(0.50), F(0.16), F(0.50)};
        if (i == 1) sampleUv = {F(0.34), F(0.26), F(0.43)};
        else if (i == 2) sampleUv = {F(0.66), F(0.26), F(0.57)};
        const V4<T> light = sampleSceneLight(lightF, p, sampleUv.x, sampleUv.y, sampleUv.z);
        const V3<T> radiance = {light.x, light.y, light.z};
        const T lum = luminance3(radiance);
        if (lum <= F(0.00001)) continue;
        const V3<T> source = fireVolumeWorldFromUv(sampleUv);
        const V3<T> toLight = sub3(source, hit);
        const T dist2 = std::fmax(F(0.045), dot3(toLight, toLight));
        const V3<T> wi = mul3(toLight, F(1.0) / std::sqrt(dist2));
        const T ndotl = std::fmax(F(0.0), dot3(normal, wi));
        const T heightOcclusion = std::exp(-std::fmax(F(0.0), hit.y - source.y) * light.w * F(1.15));
        const T visibility = sampleSceneShadow(shadowF, p, sampleUv.x, sampleUv.y, sampleUv.z) *
                             std::exp(-light.w * F(0.92)) * heightOcclusion;
        const T geometric = (F(0.12) + ndotl * F(0.88)) * std::exp(-dist2 * F(0.22)) / (F(0.12) + dist2);
        irradiance = add3(irradiance, mul3(radiance, visibility * geometric));
    }
    const T grazingBounce = F(1.0) + smoothstepf(F(0.0), F(0.45), F(1.0) - std::fmax(F(0.0), normal.y)) * F(0.36);
    return mul3(irradiance, F(4.20) * grazingBounce);
}

// src/fire_cuda.cu:1628-1645
template <class T> T volumeShadowRay(V3<T> hit, const V4<T>* lightF, const T* shadowF, const Params<T>& p) {
    const V3<T> targetUv = fireVolumeUvFromWorld(hit);
    const V3<T> sourceUv = {F(0.50), F(0.12), F(0.50)};
    T opticalDepth = F(0.0);
    for (int i = 1; i <= 5; ++i) {
        const T t = T(static_cast<float>(i)) / F(6.0);
        const V3<T> uv = lerp3(sourceUv, targetUv, t);
        const V4<T> light = sampleSceneLight(lightF, p, uv.x, uv.y, uv.z);
        const T shadow = sampleSceneShadow(shadowF, p, uv.x, uv.y, uv.z);
        opticalDepth += light.w * (F(0.18) + t * F(0.22)) + (F(1.0) - shadow) * (F(0.08) + t * F(0.16));
    }
    return std::exp(-opticalDepth);
}

// src/fire_cuda.cu:1647-1659
template <class T> T rectMask(V2<T> q, V2<T> center, V2<T> halfSize, T feather) {
    const V2<T> d = {std::fabs(q.x - center.x) - halfSize.x, std::fabs(q.y - center.y) - halfSize.y};
    const T outside = std::fmax(d.x, d.y);
    return smoothstepf(feather, -feather, outside);
}
template <class T> T lineMask(V2<T> q, V2<T> a, V2<T> b, T thickness) {
    const V2<T> pa = sub2(q, a);
    const V2<T> ba = sub2(b, a);
    const T h = saturate(dot2(pa, ba) / std::fmax(F(0.000001), dot2(ba, ba)));
    const V2<T> d = sub2(pa, mul2(ba, h));
    return smoothstepf(thickness, thickness * F(0.25), std::sqrt(dot2(d, d)));
}

// src/fire_cuda.cu:348-357
template <class T> V3<T> projectPoint(const Params<T>& cam, V3<T> point) {
    const V3<T> view = sub3(point, cam.eye);
    const T depth = dot3(view, cam.forward);
    if (depth <= F(0.02)) return {F(-10.0), F(-10.0), F(-1.0)};
    const T px = dot3(view, cam.right) / (depth * cam.tanHalfFov * cam.aspect);
    const T py = dot3(view, cam.up) / (depth * cam.tanHalfFov);
    return {F(0.5) + px * F(0.5), F(0.5) - py * F(0.5), depth};
}

// src/fire_cuda.cu:1661-1681
template <class T> void sourceModelOverlay(V2<T> uv, const Params<T>& p, V3<T>* color) {
    if (uv.x < F(0.24) || uv.x > F(0.76) || uv.y < F(0.42) || uv.y > F(0.88)) return;
    if (p.sceneId == 1) return;
    const T sourceX = p.sceneId == 2 && p.burnerCenterCount > 0 ? p.burnerCenterX[0] : p.emitterCenterX;
    const T sourceY = p.sceneId == 2 && p.burnerCenterCount > 0 ? p.burnerCenterY[0]
                                                                : p.emitterHeightNorm * F(2.03) + F(0.02);
    const T sourceZ = p.sceneId == 2 && p.burnerCenterCount > 0 ? p.burnerCenterZ[0] : p.emitterCenterZ;
    const V3<T> c = projectPoint(p, V3<T>{sourceX, sourceY, sourceZ});
    const T tray = smoothstepf(F(0.135), F(0.105), std::fabs(uv.x - c.x)) * smoothstepf(F(0.050), F(0.036), std::fabs(uv.y - c.y));
    const T inner = smoothstepf(F(0.112), F(0.086), std::fabs(uv.x - c.x)) * smoothstepf(F(0.039), F(0.027), std::fabs(uv.y - c.y));
    const T alpha = saturate((tray - inner * F(0.55)) * F(0.65));
    const V3<T> modelColor = lerp3(V3<T>{F(0.015), F(0.013), F(0.011)}, V3<T>{F(0.13), F(0.12), F(0.10)}, alpha);
    if (alpha > F(0.001)) *color = lerp3(*color, modelColor, saturate(alpha));
}

// src/fire_cuda.cu:1683-1865 -- analytic room (floor, ceiling, walls) with GI gather.
// floorGrid (src/fire_cuda.cu:1567-1573) always returns 0, so its terms are 0 here.
template <class T>
V3<T> roomBackgroundRay(V2<T> uv, V3<T> rd, T glow, const V4<T>* lightF, const T* shadowF, const Params<T>& p) {
    const T roomHalf = F(2.55);
    const T ceilingY = F(2.18);
    const bool cinematic = p.cinematicMode != 0;
    T bestT = F(1.0e6);
    V3<T> hit = {F(0.0), F(0.0), F(0.0)};
    V3<T> surfaceNormal = {F(0.0), F(1.0), F(0.0)};
    int surface = 0;
    const V3<T> eye = p.eye;
    if (rd.y < F(-0.0001)) {
        const T t = -eye.y / rd.y;
        const V3<T> q = add3(eye, mul3(rd, t));
        if (t > F(0.0) && std::fabs(q.x) <= roomHalf && std::fabs(q.z) <= roomHalf && t < bestT) {
            bestT = t; hit = q; surfaceNormal = {F(0.0), F(1.0), F(0.0)}; surface = 1;
        }
    }
    if (rd.y > F(0.0001)) {
        const T t = (ceilingY - eye.y) / rd.y;
        const V3<T> q = add3(eye, mul3(rd, t));
        if (t > F(0.0) && std::fabs(q.x) <= roomHalf && std::fabs(q.z) <= roomHalf && t < bestT) {
            bestT = t; hit = q; surfaceNormal = {F(0.0), F(-1.0), F(0.0)}; surface = 2;
        }
    }
    if (std::fabs(rd.x) > F(0.0001)) {
        const T planeX = rd.x > F(0.0) ? roomHalf : -roomHalf;
        const T t = (planeX - eye.x) / rd.x;
        const V3<T> q = add3(eye, mul3(rd, t));
        if (t > F(0.0) && q.y >= F(0.0) && q.y <= ceilingY && std::fabs(q.z) <= roomHalf && t < bestT) {
            bestT = t; hit = q; surfaceNormal = {planeX > F(0.0) ? F(-1.0) : F(1.0), F(0.0), F(0.0)}; surface = 3;
        }
    }
    if (std::fabs(rd.z) > F(0.0001)) {
        const T planeZ = rd.z > F(0.0) ? roomHalf : -roomHalf;
        const T t = (planeZ - eye.z) / rd.z;
        const V3<T> q = add3(eye, mul3(rd, t));
        if (t > F(0.0) && q.y >= F(0.0) && q.y <= ceilingY && std::fabs(q.x) <= roomHalf && t < bestT) {
            bestT = t; hit = q; surfaceNormal = {F(0.0), F(0.0), planeZ > F(0.0) ? F(-1.0) : F(1.0)}; surface = 4;
        }
    }

    V3<T> color = {F(0.014), F(0.014), F(0.014)};
    V3<T> materialAlbedo = {F(0.26), F(0.26), F(0.25)};
    T materialGiScale = F(0.24);
    if (surface == 1) {
        const T panelSeam = F(0.0);
        const T fineSeam = F(0.0);
        const T slabTone = std::sin(hit.x * F(2.20) + hit.z * F(1.40)) * F(0.50) + std::sin(hit.z * F(3.10) - hit.x * F(0.80)) * F(0.50);
        color = cinematic ? V3<T>{F(0.016), F(0.016), F(0.015)} : V3<T>{F(0.014), F(0.014), F(0.013)};
        color = add3(color, mul3(V3<T>{F(0.014), F(0.014), F(0.013)}, slabTone * F(0.018)));
        color = lerp3(color, V3<T>{F(0.014), F(0.014), F(0.013)}, saturate(panelSeam * F(0.16) + fineSeam * F(0.045)));
        materialAlbedo = {F(0.26), F(0.26), F(0.25)};
        materialGiScale = F(0.22);
        if (p.sceneId == 1) {
            const T logMaterial = fuelBedMaterial(hit.x, hit.z, p);
            const T coal = std::exp(-(hit.x * hit.x * F(1.25) + hit.z * hit.z * F(2.45))) *
                           smoothstepf(F(0.28), F(0.90), fbm(v2(hit.x * F(13.0), hit.z * F(15.0))));
            const T scorch = std::exp(-(hit.x * hit.x * F(0.66) + hit.z * hit.z * F(1.15)));
            color = lerp3(color, V3<T>{F(0.018), F(0.015), F(0.012)}, saturate(logMaterial * F(0.78) + scorch * F(0.20)));
            color = add3(color, mul3(V3<T>{F(0.090), F(0.020), F(0.004)}, coal * glow * F(0.026)));
            color = add3(color, mul3(V3<T>{F(0.17), F(0.11), F(0.055)}, logMaterial * F(0.050)));
            materialAlbedo = lerp3(materialAlbedo, V3<T>{F(0.040), F(0.030), F(0.022)}, logMaterial * F(0.86));
            materialGiScale = lerpf(materialGiScale, F(0.44), logMaterial * F(0.80));
        } else if (p.sceneId == 2) {
            const T radius = std::sqrt(hit.x * hit.x + hit.z * hit.z);
            const T plate = smoothstepf(F(0.78), F(0.70), radius);
            const T burner = fuelBedMaterial(hit.x, hit.z, p);
            const T radialGrooves = F(0.0);
            color = lerp3(color, V3<T>{F(0.018), F(0.019), F(0.020)}, plate * F(0.70));
            color = lerp3(color, V3<T>{F(0.005), F(0.005), F(0.005)}, burner * F(0.72));
            color = add3(color, mul3(V3<T>{F(0.11), F(0.10), F(0.09)}, radialGrooves * plate * F(0.010)));
            color = add3(color, mul3(V3<T>{F(0.090), F(0.032), F(0.006)}, burner * glow * F(0.012)));
            materialAlbedo = lerp3(materialAlbedo, V3<T>{F(0.032), F(0.033), F(0.034)}, plate * F(0.82));
            materialGiScale = lerpf(materialGiScale, F(0.42), plate * F(0.72));
        } else {
            const V2<T> hxz = {hit.x, hit.z};
            const T trayBody = rectMask(hxz, V2<T>{F(0.0), F(0.0)}, V2<T>{F(1.08), F(0.58)}, F(0.022));
            const T trayInner = rectMask(hxz, V2<T>{F(0.0), F(0.0)}, V2<T>{F(0.96), F(0.47)}, F(0.020));
            const T trayRim = saturate(trayBody - trayInner * F(0.74));
            const T emberBed = trayInner * std::exp(-(hit.x * hit.x * F(0.74) + hit.z * hit.z * F(2.20)));
            const T trayContact = trayInner * std::exp(-(hit.x * hit.x * F(1.35) + hit.z * hit.z * F(3.35)));
            const T scorch = std::exp(-(hit.x * hit.x * F(0.82) + hit.z * hit.z * F(1.75)));
            color = lerp3(color, V3<T>{F(0.017), F(0.014), F(0.012)}, trayBody * F(0.82));
            color = lerp3(color, V3<T>{F(0.020), F(0.019), F(0.018)}, scorch * (F(1.0) - trayBody) * F(0.16));
            color = lerp3(color, V3<T>{F(0.010), F(0.009), F(0.008)}, trayContact * F(0.22));
            color = add3(color, mul3(V3<T>{F(0.056), F(0.014), F(0.003)}, emberBed * glow * F(0.26)));
            color = add3(color, mul3(V3<T>{F(0.30), F(0.28), F(0.24)}, trayRim * F(0.10)));
            materialAlbedo = lerp3(materialAlbedo, V3<T>{F(0.030), F(0.024), F(0.020)}, trayBody * F(0.75));
            materialGiScale = lerpf(materialGiScale, F(0.48), trayBody * F(0.85));
        }
        const T reflectCore = std::exp(-(hit.x * hit.x * F(2.45) + (hit.z + F(0.18)) * (hit.z + F(0.18)) * F(1.95))) * glow;
        const T reflectedTongues = smoothstepf(F(0.82), F(0.00), std::fabs(hit.x)) * smoothstepf(F(1.18), F(0.00), std::fabs(hit.z + F(0.72)));
        const T streaks = F(0.0);
        color = add3(color, mul3(V3<T>{F(0.55), F(0.11), F(0.023)}, reflectCore * p.reflectionGain * F(0.48)));
        color = add3(color, mul3(V3<T>{F(0.46), F(0.070), F(0.014)}, reflectedTongues * streaks * glow * p.reflectionGain * F(0.14)));
    } else if (surface == 2) {
        color = cinematic ? V3<T>{F(0.012), F(0.012), F(0.012)} : V3<T>{F(0.011), F(0.011), F(0.010)};
        materialAlbedo = {F(0.24), F(0.24), F(0.23)};
        materialGiScale = F(0.20);
        const V2<T> hxz = {hit.x, hit.z};
        const T panelA = lineMask(hxz, V2<T>{F(-1.2), F(-2.0)}, V2<T>{F(-1.2), F(2.0)}, F(0.010));
        const T panelB = lineMask(hxz, V2<T>{F(0.0), F(-2.0)}, V2<T>{F(0.0), F(2.0)}, F(0.008));
        const T ceilingGrid = F(0.0);
        const T ceilingRib = F(0.0);
        const T fixtureL = std::exp(-((hit.x + F(1.50)) * (hit.x + F(1.50)) + (hit.z - F(0.92)) * (hit.z - F(0.92))) * F(120.0));
        const T fixtureR = std::exp(-((hit.x - F(1.72)) * (hit.x - F(1.72)) + (hit.z - F(0.80)) * (hit.z - F(0.80))) * F(120.0));
        color = lerp3(color, V3<T>{F(0.011), F(0.011), F(0.010)}, saturate(ceilingGrid * F(0.090) + ceilingRib * F(0.035)));
        color = add3(color, mul3(V3<T>{F(0.10), F(0.096), F(0.088)}, (panelA + panelB) * F(0.08)));
        color = add3(color, mul3(V3<T>{F(0.26), F(0.20), F(0.13)}, (fixtureL + fixtureR) * F(0.10)));
    } else {
        color = cinematic ? V3<T>{F(0.015), F(0.015), F(0.014)} : color;
        materialAlbedo = {F(0.25), F(0.25), F(0.24)};
        materialGiScale = F(0.24);
        const T panelSeam = F(0.0);
        const T baseShadow = smoothstepf(F(0.34), F(0.02), hit.y);
        const T crownShadow = smoothstepf(ceilingY - F(0.32), ceilingY - F(0.02), hit.y);
        color = lerp3(color, V3<T>{F(0.017), F(0.017), F(0.016)}, panelSeam * F(0.090));
        color = lerp3(color, V3<T>{F(0.012), F(0.012), F(0.011)}, saturate(baseShadow * F(0.30) + crownShadow * F(0.20)));
        if (surface == 4 && hit.z > F(0.0)) {
            const V2<T> hxy = {hit.x, hit.y};
            const T recess = rectMask(hxy, V2<T>{F(0.0), F(1.00)}, V2<T>{F(0.92), F(0.72)}, F(0.055));
            const T recessEdge = lineMask(hxy, V2<T>{F(-0.92), F(0.28)}, V2<T>{F(-0.92), F(1.72)}, F(0.010)) +
                                 lineMask(hxy, V2<T>{F(0.92), F(0.28)}, V2<T>{F(0.92), F(1.72)}, F(0.010));
            color = lerp3(color, V3<T>{F(0.015), F(0.015), F(0.014)}, recess * F(0.42));
            color = add3(color, mul3(V3<T>{F(0.050), F(0.046), F(0.038)}, recessEdge * F(0.030)));
        }
        const T soot = std::exp(-(hit.x * hit.x * F(0.82) + hit.z * hit.z * F(1.12))) * smoothstepf(F(0.36), F(1.92), hit.y);
        color = lerp3(color, V3<T>{F(0.010), F(0.011), F(0.012)}, soot * F(0.82) * p.smokeDarkness);
        materialAlbedo = lerp3(materialAlbedo, V3<T>{F(0.030), F(0.032), F(0.034)}, soot * F(0.75));
        const T wallGlow = std::exp(-(hit.x * hit.x * F(1.1) + hit.z * hit.z * F(1.3) + (hit.y - F(0.70)) * (hit.y - F(0.70)) * F(1.0))) * glow;
        color = add3(color, mul3(V3<T>{F(0.15), F(0.050), F(0.018)}, wallGlow * F(0.090)));
        if (surface == 3 && hit.x < F(0.0)) {
            const V2<T> hzy = {hit.z, hit.y};
            const T window = rectMask(hzy, V2<T>{F(-1.28), F(0.92)}, V2<T>{F(0.06), F(0.62)}, F(0.030));
            const T glassNoise = F(0.55) + F(0.25) * std::sin(hit.y * F(23.0) + hit.z * F(15.0));
            color = lerp3(color, V3<T>{F(0.009), F(0.011), F(0.012)}, window * F(0.92));
            color = add3(color, mul3(V3<T>{F(0.10), F(0.12), F(0.13)}, window * glassNoise * F(0.16)));
        }
    }

    const V3<T> volumeUv = fireVolumeUvFromWorld(hit);
    const V4<T> giSample = sampleSceneLight(lightF, p, volumeUv.x, volumeUv.y, volumeUv.z);
    const T sceneShadow = sampleSceneShadow(shadowF, p, volumeUv.x, volumeUv.y, volumeUv.z);
    const T volumeVisibility = volumeShadowRay(hit, lightF, shadowF, p);
    const V3<T> gathered = gatherSceneIrradiance(hit, surfaceNormal, lightF, shadowF, p);
    const V3<T> indirect = mul3(add3(mul3(V3<T>{giSample.x, giSample.y, giSample.z}, F(0.42)), gathered), volumeVisibility);
    const T grazingFalloff = surface == 2 ? F(0.62) : F(1.0);
    const T contactOcclusion = smoothstepf(F(0.005), F(0.42), sceneShadow) * std::exp(-giSample.w * F(0.72)) *
                               (F(0.30) + volumeVisibility * F(0.70));
    const T irradianceLift = F(0.66) + smoothstepf(F(0.006), F(0.13), luminance3(indirect)) * F(0.72);
    const T contactWarmth = surface == 1 ? F(1.72) : (surface == 2 ? F(0.88) : F(1.16));
    color = add3(color, mul3(mul3v(indirect, materialAlbedo),
                             materialGiScale * grazingFalloff * contactOcclusion * irradianceLift * contactWarmth));
    const T shadowedSoot = (F(1.0) - volumeVisibility) * smoothstepf(F(0.18), F(0.82), F(1.0) - sceneShadow);
    color = lerp3(color, V3<T>{F(0.006), F(0.007), F(0.008)}, shadowedSoot * (surface == 2 ? F(0.38) : F(0.26)));
    const T wallHorizontalEdge = surface == 3 ? roomHalf - std::fabs(hit.z) : roomHalf - std::fabs(hit.x);
    const T cornerDistance = surface == 1 || surface == 2
                                 ? std::fmin(roomHalf - std::fabs(hit.x), roomHalf - std::fabs(hit.z))
                                 : std::fmin(wallHorizontalEdge, std::fmin(hit.y, ceilingY - hit.y));
    color = mul3(color, F(0.84) + smoothstepf(F(0.0), F(0.54), cornerDistance) * F(0.16));
    const T grain = (T(hash21f(float(std::floor(hit.x * F(19.0) + hit.z * F(13.0))),
                               float(std::floor(hit.y * F(15.0) + p.time * F(0.08))))) - F(0.5)) * F(0.006);
    color = add3(color, V3<T>{grain, grain, grain});
    sourceModelOverlay(uv, p, &color);
    const T fog = smoothstepf(F(3.8), F(0.2), bestT);
    const T vignette = smoothstepf(F(0.78), F(0.20), std::sqrt((uv.x - F(0.50)) * (uv.x - F(0.50)) + (uv.y - F(0.46)) * (uv.y - F(0.46))));
    return mul3(color, (F(0.12) + fog * F(0.56)) * (F(0.58) + vignette * F(0.30)));
}

// src/fire_cuda.cu:1867-1907
template <class T> bool intersectBox(V3<T> ro, V3<T> rd, V3<T> bmin, V3<T> bmax, T* outNear, T* outFar) {
    T tNear = F(0.0);
    T tFar = F(1.0e6);
    auto inv1 = [](T d) { return F(1.0) / (std::fabs(d) < F(0.00001) ? std::copysign(F(0.00001), d) : d); };
    const V3<T> inv = {inv1(rd.x), inv1(rd.y), inv1(rd.z)};
    auto slab = [&](T lo, T hi, T o, T iv) {
        T t0 = (lo - o) * iv;
        T t1 = (hi - o) * iv;
        if (t0 > t1) std::swap(t0, t1);
        tNear = std::fmax(tNear, t0);
        tFar = std::fmin(tFar, t1);
    };
    slab(bmin.x, bmax.x, ro.x, inv.x);
    slab(bmin.y, bmax.y, ro.y, inv.y);
    slab(bmin.z, bmax.z, ro.z, inv.z);
    *outNear = tNear;
    *outFar = tFar;
    return tFar > tNear;
}

// src/fire_cuda.cu:370-379
template <class T> V3<T> debugHeatColor(T value) {
    value = saturate(value);
    const T red = smoothstepf(F(0.05), F(0.45), value);
    const T orange = smoothstepf(F(0.24), F(0.78), value);
    const T white = smoothstepf(F(0.72), F(1.0), value);
    return {saturate(red + white * F(0.70)), saturate(orange * F(0.58) + white * F(0.78)), saturate(white * F(0.62))};
}

// src/fire_cuda.cu:1953-2244 -- the HDR raymarch, one pixel.
template <class T> V4<T> renderPixel(const State<T>& s, const Params<T>& p, int x, int y) {
    const T* f[10];
    for (int i = 0; i < 10; ++i) f[i] = s.scalar[i].data();
    const V4<T>* lightF = s.light.data();
    const T* shadowF = s.shadow.data();
    const V2<T> uv = {(T(static_cast<float>(x)) + F(0.5)) / T(static_cast<float>(p.frameW)),
                      (T(static_cast<float>(y)) + F(0.5)) / T(static_cast<float>(p.frameH))};
    // cameraRayDirection, src/fire_cuda.cu:342-346
    const T sx = (uv.x * F(2.0) - F(1.0)) * p.aspect * p.tanHalfFov;
    const T sy = (F(1.0) - uv.y * F(2.0)) * p.tanHalfFov;
    const V3<T> rd = normalize3(add3(add3(p.forward, mul3(p.right, sx)), mul3(p.up, sy)));
    const T baseGlow = saturate(sampleScalar(f[HEAT], p, F(0.50), F(0.06), F(0.50)) * F(0.42));

    T boxNear = F(0.0), boxFar = F(0.0);
    V3<T> accum = {F(0.0), F(0.0), F(0.0)};
    T trans = F(1.0);
    T flameGlow = F(0.0), smokeOcclusion = F(0.0), debugFlame = F(0.0), debugOpticalDepth = F(0.0);
    T debugTemperature = F(0.0), debugFuel = F(0.0), debugVelocity = F(0.0);
    const int sc = p.sceneId;

    if (intersectBox(p.eye, rd, V3<T>{F(-1.05), F(0.02), F(-0.82)}, V3<T>{F(1.05), F(2.05), F(0.82)}, &boxNear, &boxFar)) {
        const int raySteps = std::min(std::max(p.raymarchSteps, 24), kMaxRaymarchSteps);
        const T t0 = std::fmax(F(0.0), boxNear);
        const T t1 = std::fmin(boxFar, t0 + F(3.05));
        const T stepT = (t1 - t0) / T(static_cast<float>(raySteps));
        const T rayJitter = T(hash21f((static_cast<float>(x) + 0.5f) * 0.754877f, (static_cast<float>(y) + 0.5f) * 0.569840f));
        for (int i = 0; i < raySteps && trans > F(0.018); ++i) {
            const T t = t0 + (T(static_cast<float>(i)) + rayJitter) * stepT;
            const V3<T> wp = add3(p.eye, mul3(rd, t));
            const T fu = saturate((wp.x + F(1.05)) / F(2.10));
            const T fv = saturate((wp.y - F(0.02)) / F(2.03));
            const T fw = saturate((wp.z + F(0.82)) / F(1.64));
            const T domainFade = volumeDomainFade(fu, fv, fw);
            if (domainFade <= F(0.001)) continue;
            const T coarseHeat = sampleScalar(f[HEAT], p, fu, fv, fw);
            const T coarseFuel = sampleScalar(f[FUEL], p, fu, fv, fw);
            const T coarseSoot = sampleScalar(f[SOOT], p, fu, fv, fw);
            const T coarseProgress = sampleScalar(f[PROGRESS], p, fu, fv, fw);
            const T coarseActive = (coarseHeat + coarseFuel * F(0.42) + coarseSoot * F(0.34) + coarseProgress * F(0.32)) * domainFade;
            if (coarseActive <= F(0.00150)) {
                ++i;
                continue;
            }
            const T warpA = fbm3(v3(fu * F(7.0) + p.time * F(0.18), fv * F(5.0) - p.time * F(0.11), fw * F(9.0) + p.time * F(0.07))) - F(0.5);
            const T warpB = fbm3(v3(fw * F(8.0) - p.time * F(0.14), fu * F(8.0) + p.time * F(0.10), fv * F(6.0) - p.time * F(0.08))) - F(0.5);
            const T warpGain = F(0.028) + fv * F(0.060);
            const T wu = saturate(fu + warpA * warpGain);
            const T wv = saturate(fv + (warpA - warpB) * F(0.020));
            const T ww = saturate(fw + warpB * warpGain);

            const T heat = sampleScalar(f[HEAT], p, wu, wv, ww);
            const T fuel = sampleScalar(f[FUEL], p, wu, wv, ww);
            const T oxygen = sampleScalar(f[OXYGEN], p, wu, wv, ww);
            const T soot = sampleScalar(f[SOOT], p, wu, wv, ww);
            const T charMass = sampleScalar(f[CHAR], p, wu, wv, ww);
            const T ash = sampleScalar(f[ASH], p, wu, wv, ww);
            const T pyrolysis = sampleScalar(f[PYRO], p, wu, wv, ww);
            const T progress = sampleScalar(f[PROGRESS], p, wu, wv, ww);
            const T turbulenceEnergy = sampleScalar(f[TURB], p, wu, wv, ww);
            const T sootOptics = sampleScalar(f[SOOTOPT], p, wu, wv, ww);
            const V4<T> sceneLight = sampleSceneLight(lightF, p, wu, wv, ww);
            const T sceneShadow = sampleSceneShadow(shadowF, p, wu, wv, ww);
            V3<T> velocity = {F(0.0), F(0.0), F(0.0)};
            if (p.renderDebugMode == 6) velocity = sampleVelocity(s, p, wu, wv, ww);
            const T activeField = (heat + fuel * F(0.42) + soot * F(0.34) + progress * F(0.32) + pyrolysis * F(0.18)) * domainFade;
            if (activeField <= F(0.0025)) continue;
            debugFuel = std::fmax(debugFuel, domainFade * saturate(fuel * F(0.18) + charMass * F(0.22) + pyrolysis * F(0.30)));
            if (p.renderDebugMode == 6) {
                debugVelocity = std::fmax(debugVelocity, saturate(std::sqrt(dot3(velocity, velocity)) * F(0.22)));
            }
            const T cellX = F(1.0) / T(static_cast<float>(p.nx));
            const T cellY = F(1.0) / T(static_cast<float>(p.ny));
            const T cellZ = F(1.0) / T(static_cast<float>(p.nz));
            const T gradHeatX = sampleScalar(f[HEAT], p, wu + cellX, wv, ww) - sampleScalar(f[HEAT], p, wu - cellX, wv, ww);
            const T gradHeatY = sampleScalar(f[HEAT], p, wu, wv + cellY, ww) - sampleScalar(f[HEAT], p, wu, wv - cellY, ww);
            const T gradHeatZ = sampleScalar(f[HEAT], p, wu, wv, ww + cellZ) - sampleScalar(f[HEAT], p, wu, wv, ww - cellZ);
            const T frontGradient = std::sqrt(gradHeatX * gradHeatX + gradHeatY * gradHeatY + gradHeatZ * gradHeatZ) +
                                    std::fabs(fuel - coarseFuel) * F(0.62);
            const T reactionFront = smoothstepf(F(0.020), F(0.46), frontGradient * F(1.35) + fuel * oxygen * F(0.040) +
                                                                     progress * F(0.18) + pyrolysis * F(0.080));
            const T fineNoise = fbm3(v3(wu * F(42.0) + p.time * F(0.72), wv * F(54.0) - p.time * F(1.28), ww * F(43.0) + p.time * F(0.38)));
            const T shearNoise = fbm3(v3(wu * F(15.0) - p.time * F(0.72), wv * F(13.0) - p.time * F(1.08), ww * F(17.0) + p.time * F(0.32)));
            const T plumeNoise = saturate(fineNoise * F(0.58) + shearNoise * F(0.42));
            const T holeNoise = saturate((F(1.0) - fineNoise) * F(0.36) + shearNoise * F(0.64));
            const T lesBreakup = saturate(turbulenceEnergy * F(0.48) + progress * F(0.28));
            const T raggedEdge = smoothstepf(F(0.18), F(0.92), fineNoise * (F(0.46) + lesBreakup * F(0.30)) + shearNoise * F(0.38) +
                                                                 plumeNoise * F(0.32) + saturate(activeField * F(0.08)));
            const T fieldEdge = smoothstepf(F(0.05), F(2.30), heat + fuel * F(0.32)) * (F(0.10) + reactionFront * F(0.90));
            const T fieldFilament = smoothstepf(F(0.60), F(1.0), fineNoise + lesBreakup * F(0.10)) *
                                    smoothstepf(F(0.38), F(0.92), shearNoise + (F(0.72) - fv) * F(0.12) + reactionFront * F(0.10)) *
                                    smoothstepf(F(1.0), F(0.02), fv) * fieldEdge;
            const T sourceLocalV = sc == 2 ? std::fmax(F(0.0), fv - p.emitterHeightNorm) : fv;
            const T burnerLowJet = sc == 2 ? smoothstepf(std::fmax(F(0.012), p.emitterHeightBandNorm * F(0.68)),
                                                         std::fmax(F(0.003), p.emitterHeightBandNorm * F(0.10)),
                                                         std::fabs(fv - p.emitterHeightNorm)) *
                                                 smoothstepf(F(0.05), F(0.58), fuel + heat * F(0.025)) *
                                                 smoothstepf(F(0.50), F(1.0), oxygen)
                                           : F(0.0);
            const T burnerPortJet = sc == 2 ? burnerLowJet * smoothstepf(F(0.68), F(0.98), fineNoise + shearNoise * F(0.18)) : F(0.0);
            const T campTongueBias = sc == 1 ? smoothstepf(F(0.035), F(0.72), fuel + pyrolysis * F(0.50) + charMass * F(0.12)) *
                                                   smoothstepf(F(0.76), F(0.035), fv)
                                             : F(0.0);
            const T roomTraySheet = sc == 0 ? smoothstepf(F(0.018), F(0.42), fuel + pyrolysis * F(0.72) + charMass * F(0.08)) *
                                                  smoothstepf(F(0.30), F(0.015), fv)
                                            : F(0.0);
            const T convectiveSheet =
                smoothstepf(F(0.42), F(0.88), shearNoise + heat * F(0.040) + plumeNoise * F(0.14) + lesBreakup * F(0.10) +
                                                  burnerPortJet * F(0.56) + campTongueBias * F(0.20) + roomTraySheet * F(0.24)) *
                (sc == 2 ? smoothstepf(p.emitterHeightNorm + p.emitterHeightBandNorm * F(1.20),
                                       p.emitterHeightNorm - p.emitterHeightBandNorm * F(0.08), fv)
                         : smoothstepf(sc == 1 ? F(0.82) : F(0.88), F(0.030), fv)) *
                fieldEdge;
            const T breakup = smoothstepf(F(0.34), F(0.88), fineNoise * F(0.48) + shearNoise * F(0.42) + holeNoise * F(0.24) + heat * F(0.026));
            const T verticalFade = smoothstepf(F(0.96), F(0.025), fv);
            const T flameHeightFade = sc == 2 ? smoothstepf(p.emitterHeightNorm + p.emitterHeightBandNorm * F(0.72),
                                                            p.emitterHeightNorm - p.emitterHeightBandNorm * F(0.05), fv)
                                              : smoothstepf(sc == 1 ? F(0.72) : F(0.76), F(0.10), fv);
            const T lowerWhite = smoothstepf(F(0.060), F(0.00), sourceLocalV) * smoothstepf(F(0.05), F(1.30), pyrolysis + fuel * F(0.20));
            const T tempK = F(293.0) + heat * F(360.0) + fuel * F(44.0) + pyrolysis * F(90.0) + fieldFilament * F(560.0) +
                            convectiveSheet * F(420.0) + lowerWhite * F(110.0) + progress * F(64.0);
            const T combustion = smoothstepf(F(740.0), F(1630.0), tempK) * smoothstepf(F(0.016), F(0.62), fuel + heat * F(0.055)) *
                                 smoothstepf(F(0.045), F(0.62), oxygen) * verticalFade * flameHeightFade;
            const T thinFront = smoothstepf(F(0.04), F(0.56), frontGradient + progress * F(0.10)) * smoothstepf(F(0.02), F(0.92), reactionFront);
            const T flameSheetTear = smoothstepf(F(0.52), F(0.88), holeNoise + shearNoise * F(0.18) + lesBreakup * F(0.30) +
                                                                     saturate(F(1.0) - oxygen) * F(0.12));
            const T sheetHole = smoothstepf(F(0.54), F(0.90), holeNoise + lesBreakup * F(0.26) + saturate(F(1.0) - oxygen) * F(0.12));
            const T flameSheet = std::fmax(
                smoothstepf(F(0.55), F(0.94), fineNoise * F(0.46) + shearNoise * F(0.44) + plumeNoise * F(0.18) +
                                                  reactionFront * F(0.15) + heat * F(0.014) - fv * F(0.050)) *
                    (F(1.0) - sheetHole * (F(0.74) + lesBreakup * F(0.12))) * (F(1.0) - flameSheetTear * F(0.18)),
                smoothstepf(F(0.18), F(0.030), sourceLocalV) * smoothstepf(F(0.75), F(2.0), heat) * thinFront * F(0.030));
            const T coherentSheet = saturate(fieldFilament * F(0.86) + convectiveSheet * F(0.55) + thinFront * F(0.74));
            const T sheetConfinement = saturate(coherentSheet + reactionFront * F(0.08));
            const T roomCoverageBoost = sc == 0 ? (F(0.72) + roomTraySheet * F(1.24)) : F(1.0);
            const T flameDensity = domainFade * combustion * reactionFront * flameSheet *
                                   (F(0.010) + fieldFilament * F(0.92) + convectiveSheet * F(0.24) + thinFront * F(1.22)) *
                                   (F(0.052) + breakup * F(0.78) + raggedEdge * F(0.56) + lesBreakup * F(0.34)) *
                                   (F(0.18) + thinFront * F(2.55)) *
                                   (F(0.060) + sheetConfinement * F(0.94) + burnerPortJet * F(0.72) + campTongueBias * F(0.34)) *
                                   flameHeightFade * roomCoverageBoost;
            const T plumeVoid = smoothstepf(F(0.54), F(0.90), holeNoise + fineNoise * F(0.26) + shearNoise * F(0.22) + fv * F(0.20));
            const T topDissolve = smoothstepf(sc == 1 ? F(0.82) : F(0.88), sc == 1 ? F(0.34) : F(0.42), fv);
            const T raggedPlume = F(1.0) - plumeVoid * smoothstepf(F(0.18), F(0.74), fv) * F(0.96);
            const T upperPlume = smoothstepf(F(0.14), F(0.48), fv) * smoothstepf(F(0.030), F(1.20), sootOptics + soot * F(0.42)) *
                                 (F(0.025) + fineNoise * F(0.035) + shearNoise * F(0.034) + plumeNoise * F(0.34) +
                                  raggedEdge * F(0.12) + turbulenceEnergy * F(0.035)) *
                                 topDissolve * raggedPlume;
            const T sceneSmokeScale = sc == 2 ? F(0.035) : (sc == 1 ? F(0.56) : F(1.0));
            const T rawSootDensity =
                domainFade * sceneSmokeScale *
                (smoothstepf(F(0.020), F(1.05), sootOptics + soot * F(0.32)) * smoothstepf(F(0.16), F(0.42), fv) *
                     (F(0.028) + fineNoise * F(0.040) + shearNoise * F(0.052) + plumeNoise * F(0.38) + raggedEdge * F(0.16) + ash * F(0.016)) +
                 upperPlume * (F(0.22) + plumeNoise * F(0.30)) +
                 smoothstepf(F(0.004), F(0.34), sootOptics) * (F(0.020) + plumeNoise * F(0.034)));
            const T flameFrontMask = saturate(flameDensity * F(4.8) + combustion * reactionFront * flameSheet *
                                                                          (F(0.08) + thinFront * F(0.56) + fieldFilament * F(0.18)));
            const T emissiveMask = saturate(flameFrontMask);
            const T resolvedFlameSheet = smoothstepf(F(0.030), F(0.32), emissiveMask) * smoothstepf(F(0.035), F(0.72), oxygen);
            const T smokeOnlyMask = F(1.0) - smoothstepf(F(0.025), F(0.20), resolvedFlameSheet);
            const T scatterSeparation = saturate(smokeOnlyMask * (F(1.0) - smoothstepf(F(0.02), F(0.16), emissiveMask) * F(0.58)));
            const T nearFlameSootCleanout = F(1.0) - smoothstepf(F(0.025), F(0.34), resolvedFlameSheet) * F(0.82);
            const T smokeOnlyHeight = smoothstepf(F(0.20), F(0.70), fv) * (F(1.0) - smoothstepf(F(0.02), F(0.20), emissiveMask));
            const T upperSootNeutrality = smoothstepf(F(0.18), F(0.78), fv) * scatterSeparation;
            const T absorptionDensity = rawSootDensity * nearFlameSootCleanout * (F(1.10) + smokeOnlyHeight * F(2.20) + upperSootNeutrality * F(2.40));
            const T scatterDensity = rawSootDensity * scatterSeparation * smoothstepf(F(0.10), F(0.55), fv + sootOptics * F(0.10)) *
                                     (F(0.24) + (F(1.0) - smokeOnlyHeight) * F(0.34));
            const T particleRadius = saturate(F(0.08) + sootOptics * F(0.028) + ash * F(0.085) + saturate(F(1.0) - oxygen) * F(0.12));
            const T sootAbsorption = absorptionDensity * (F(3.10) + particleRadius * F(4.60) + sootOptics * F(0.70) + upperSootNeutrality * F(2.85)) *
                                     p.smokeDarkness;
            const T sootScattering = scatterDensity * (F(0.018) + (F(1.0) - particleRadius) * F(0.050)) * (F(0.20) + p.smokeGain * F(0.10));
            const T sootExtinction = sootAbsorption + sootScattering;
            const T flameExtinction = flameDensity * (F(0.12) + (F(1.0) - resolvedFlameSheet) * F(0.12));
            const T extinction = (sootExtinction + flameExtinction) * stepT;
            const T smokeAlpha = F(1.0) - std::exp(-sootAbsorption * stepT);
            const T scatterAlpha = F(1.0) - std::exp(-sootScattering * stepT);
            const T lightVisibility = sceneShadow * (F(0.35) + sceneShadow * F(0.65));
            const V3<T> localIrradiance = {sceneLight.x, sceneLight.y, sceneLight.z};
            const T sootLoad = saturate(sootOptics * F(0.74) + soot * F(0.20) + upperPlume * F(0.46));
            const T whiteCore = smoothstepf(F(2450.0), F(3450.0), tempK) * combustion * smoothstepf(F(0.32), F(0.90), oxygen) *
                                smoothstepf(F(0.72), F(0.02), fv) * (F(0.02) + thinFront * F(0.48) + fieldFilament * F(0.18)) *
                                (F(1.0) - smoothstepf(F(0.16), F(0.74), sootLoad) * F(0.68));
            const T radiantBase = saturate((tempK - F(760.0)) / F(2000.0));
            const T radiantCurve = radiantBase * radiantBase * (F(0.82) + radiantBase * F(0.18));
            const T radiantPower = radiantCurve * (F(1.42) + fieldFilament * F(3.15) + convectiveSheet * F(1.60) + progress * F(0.26) + whiteCore * F(0.92));
            const T blackbodyCoreStructure = saturate(whiteCore * (F(0.080) + fieldFilament * F(0.28) + thinFront * F(0.32)));
            const T whiteFilament = blackbodyCoreStructure * (F(0.55) + fineNoise * F(0.30) + shearNoise * F(0.18));
            const T orangeEdge = (F(1.0) - whiteFilament * F(0.72)) * thinFront * reactionFront * flameSheet *
                                 (F(0.52) + breakup * F(0.95)) * smoothstepf(F(0.08), F(0.80), oxygen);
            V3<T> flameColor = lerp3(V3<T>{F(1.32), F(0.27), F(0.038)}, blackbodyColor(tempK), saturate(whiteCore * F(0.92) + whiteFilament * F(0.82)));
            if (sc == 2) {
                const T blueBase = burnerPortJet * smoothstepf(F(0.010), F(0.11), flameDensity + combustion * F(0.18));
                flameColor = lerp3(V3<T>{F(0.020), F(0.18), F(2.40)}, V3<T>{F(0.36), F(0.58), F(1.95)}, saturate(whiteCore * F(0.34) + blueBase * F(0.20)));
            } else if (sc == 1) {
                flameColor = lerp3(flameColor, V3<T>{F(1.52), F(0.24), F(0.028)}, saturate(campTongueBias * (F(1.0) - whiteCore) * F(0.58)));
            }
            V3<T> flameEmission = mul3(flameColor, flameDensity * radiantPower * stepT * (F(1.10) + whiteCore * F(0.38)));
            if (sc == 2) {
                flameEmission = mul3(flameEmission, F(0.42));
                flameEmission = add3(flameEmission, mul3(V3<T>{F(0.012), F(0.28), F(5.20)}, burnerPortJet * combustion * stepT * F(4.40)));
            }
            flameEmission = add3(flameEmission, mul3(V3<T>{F(1.10), F(1.02), F(0.86)}, whiteFilament * whiteFilament * flameDensity * radiantPower * stepT * F(0.82)));
            flameEmission = add3(flameEmission, mul3(V3<T>{F(1.70), F(0.30), F(0.040)},
                                                     orangeEdge * flameDensity * radiantPower * stepT *
                                                         (sc == 2 ? F(0.06) : (sc == 1 ? F(3.20) : F(3.10)))));
            flameEmission = add3(flameEmission, mul3(V3<T>{F(1.36), F(0.070), F(0.008)},
                                                     fieldFilament * (F(1.0) + flameSheetTear * F(0.55)) * flameDensity * radiantPower * stepT *
                                                         (sc == 2 ? F(0.035) : (sc == 1 ? F(1.55) : F(1.10))) * (F(1.0) - whiteCore * F(0.62))));
            const T upperSmokeMask = smoothstepf(F(0.18), F(0.72), fv) * scatterSeparation;
            (void)upperSmokeMask;
            const T ashVeil = saturate(ash * F(0.014) + smoothstepf(F(0.30), F(0.88), fv) * (F(1.0) - sootLoad) * F(0.003));
            const V3<T> smokeBlack = {F(0.0018), F(0.0020), F(0.0024)};
            const V3<T> smokeCoal = {F(0.008), F(0.0092), F(0.0115)};
            const V3<T> smokeAsh = {F(0.014), F(0.0165), F(0.0210)};
            V3<T> smokeColor = lerp3(smokeCoal, smokeBlack, sootLoad);
            smokeColor = lerp3(smokeColor, smokeAsh, ashVeil);
            smokeColor = mul3(smokeColor, smokeOnlyMask);
            const T localIrradianceLuma = luminance3(localIrradiance);
            const T warmScatterDamp = F(1.0) - upperSootNeutrality * F(0.985);
            const T nearFlameWarmLeak = (F(1.0) - upperSootNeutrality) * (F(1.0) - smokeOnlyHeight) * F(0.18);
            const T sceneWarmScatter = sc == 2 ? F(0.010) : (sc == 1 ? F(0.18) : F(0.30));
            const T backScatter = scatterAlpha * lightVisibility *
                                  (F(0.00085) + localIrradianceLuma * F(0.0011) * warmScatterDamp + baseGlow * F(0.00010) * sceneWarmScatter) *
                                  (F(0.018) + (F(1.0) - particleRadius) * F(0.018)) * scatterSeparation;
            smokeColor = add3(smokeColor, mul3(V3<T>{F(0.010), F(0.012), F(0.016)}, backScatter));
            const T scatterGain = scatterAlpha *
                                  (F(0.00046) + lightVisibility * F(0.00072) * warmScatterDamp + flameDensity * F(0.00008) * sceneWarmScatter +
                                   turbulenceEnergy * F(0.00018)) *
                                  (F(0.038) + (F(1.0) - particleRadius) * F(0.045)) * scatterSeparation;
            const T sceneScatter = scatterAlpha * scatterSeparation * (F(0.0065) + (F(1.0) - particleRadius) * F(0.014)) * lightVisibility;
            const V3<T> neutralScatterLight = {localIrradianceLuma * F(0.052), localIrradianceLuma * F(0.064), localIrradianceLuma * F(0.086)};
            const V3<T> smokeScatterLight = lerp3(neutralScatterLight, localIrradiance, nearFlameWarmLeak);
            const T coalGlow = smoothstepf(F(0.004), F(0.18), charMass) * smoothstepf(F(0.54), F(0.02), fv) *
                               (F(0.070) + pyrolysis * F(0.12) + heat * F(0.009));

            debugFlame = std::fmax(debugFlame, saturate(flameDensity * radiantPower * F(0.26)));
            debugOpticalDepth = saturate(debugOpticalDepth + sootExtinction * stepT);
            debugTemperature = std::fmax(debugTemperature, saturate((tempK - F(520.0)) / F(1900.0)));
            accum = add3(accum, mul3(flameEmission, trans));
            accum = add3(accum, mul3(V3<T>{F(1.0), F(0.24), F(0.035)}, trans * coalGlow * stepT));
            accum = add3(accum, mul3(smokeColor, trans * scatterGain * smokeOnlyMask));
            accum = add3(accum, mul3(smokeScatterLight, trans * sceneScatter * (F(0.18) + warmScatterDamp * F(0.42))));
            flameGlow = std::fmax(flameGlow, flameDensity * radiantPower * (F(0.12) + fieldFilament * F(0.18) + whiteFilament * F(0.20)));
            smokeOcclusion = saturate(smokeOcclusion + smokeAlpha * trans);
            trans *= std::exp(-extinction);
        }
    }

    if (p.renderDebugMode != 0) {
        V3<T> dc = {F(0.0), F(0.0), F(0.0)};
        if (p.renderDebugMode == 1) dc = debugHeatColor(debugFlame);
        else if (p.renderDebugMode == 2) {
            const T od = saturate(debugOpticalDepth);
            dc = {od, od * F(0.90), od * F(0.78)};
        } else if (p.renderDebugMode == 3) dc = {trans, trans, trans};
        else if (p.renderDebugMode == 4) dc = debugHeatColor(debugTemperature);
        else if (p.renderDebugMode == 5) dc = {debugFuel * F(0.82), debugFuel * F(0.48), debugFuel * F(0.18)};
        else dc = {debugVelocity * F(0.20), debugVelocity * F(0.72), debugVelocity};
        return {dc.x, dc.y, dc.z, F(1.0)};
    }
    V3<T> color = accum;
    if (trans > F(0.006)) {
        const V3<T> roomColor = roomBackgroundRay(uv, rd, baseGlow, lightF, shadowF, p);
        color = add3(mul3(roomColor, trans), accum);
    }
    const T bloom = saturate(flameGlow * F(0.10)) * (F(1.0) - saturate(smokeOcclusion * F(0.95)));
    color = add3(color, mul3(V3<T>{F(1.0), F(0.25), F(0.045)}, bloom * bloom * F(0.017) * p.reflectionGain));
    return {std::fmax(F(0.0), color.x), std::fmax(F(0.0), color.y), std::fmax(F(0.0), color.z), F(1.0)};
}

template <class T> void stageRender(State<T>& s, const Params<T>& p) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < p.frameH; ++y) {
        for (int x = 0; x < p.frameW; ++x) {
            s.hdr[size_t(y) * p.frameW + x] = renderPixel(s, p, x, y);
        }
    }
}

// src/fire_cuda.cu:2323-2452 -- ember splats, added in ember order.
template <class T> void stageEmbers(State<T>& s, const Params<T>& p) {
    const int emberCount = std::min(std::max(p.emberCount, 0), kMaxEmberCount);
    if (emberCount <= 0 || p.renderDebugMode != 0) return;
    const T* heatF = s.scalar[HEAT].data();
    const T baseGlow = saturate(sampleScalar(heatF, p, F(0.50), F(0.06), F(0.50)) * F(0.42));
    const T sparkGate = smoothstepf(F(0.02), F(0.30), baseGlow);
    if (sparkGate <= F(0.0001)) return;
    const int sc = p.sceneId;
    for (int i = 0; i < emberCount; ++i) {
        const float seed = static_cast<float>(i);
        const T h0 = T(hash21f(seed, 3.7f));
        const T h1 = T(hash21f(seed, 9.1f));
        const T h2 = T(hash21f(seed, 19.4f));
        const T h3 = T(hash21f(seed, 31.6f));
        if (sc == 1 && h2 > F(0.34)) continue;
        if (sc == 2 && h0 > F(0.14)) continue;
        const T life = fracf(p.time * (F(0.20) + h2 * F(0.18) + (sc == 2 ? F(0.36) : F(0.0))) + h0);
        const T spawnAngle = h0 * F(6.2831853);
        T startX = F(0.0), startZ = F(0.0);
        if (sc == 2) {
            const T sourceRadius = std::fmax(F(0.04), p.emitterRadius);
            const T cx = p.burnerCenterCount > 0 ? p.burnerCenterX[0] : p.emitterCenterX;
            const T cz = p.burnerCenterCount > 0 ? p.burnerCenterZ[0] : p.emitterCenterZ;
            startX = cx + std::cos(spawnAngle) * sourceRadius * (F(0.82) + h1 * F(0.18));
            startZ = cz + std::sin(spawnAngle) * sourceRadius * (F(0.82) + h1 * F(0.18));
        } else if (sc == 1) {
            const T logA = orientedCapsuleMask(std::cos(spawnAngle) * F(0.34), std::sin(spawnAngle) * F(0.25), F(-0.06), F(0.01), F(0.38), F(0.34), F(0.095));
            const T logB = orientedCapsuleMask(std::cos(spawnAngle + F(1.7)) * F(0.35), std::sin(spawnAngle + F(1.7)) * F(0.25), F(0.07), F(-0.02), F(-0.58), F(0.33), F(0.092));
            const T contactBlend = saturate(logA + logB + h3 * F(0.35));
            const T spawnRadius = lerpf(F(0.16), F(0.46), std::sqrt(h1));
            startX = std::cos(spawnAngle) * spawnRadius * (F(0.64) + contactBlend * F(0.36));
            startZ = std::sin(spawnAngle) * spawnRadius * (F(0.46) + contactBlend * F(0.26));
        } else {
            const T spawnRadius = F(0.48);
            const T ringBias = std::sqrt(h1);
            startX = std::cos(spawnAngle) * spawnRadius * ringBias;
            startZ = std::sin(spawnAngle) * spawnRadius * ringBias;
        }
        const T startU = saturate((startX / F(2.10)) + F(0.50));
        const T startW = saturate((startZ / F(1.64)) + F(0.50));
        const T startV = sc == 2 ? p.emitterHeightNorm : (sc == 1 ? F(0.035) + h2 * F(0.055) : F(0.045));
        const T localHeat = sampleScalar(heatF, p, startU, startV, startW);
        const T localChar = sampleScalar(s.scalar[CHAR].data(), p, startU, startV, startW);
        const T localPyrolysis = sampleScalar(s.scalar[PYRO].data(), p, startU, startV, startW);
        const T localTurbulence = sampleScalar(s.scalar[TURB].data(), p, startU, startV, startW);
        const V3<T> localVelocity = sampleVelocity(s, p, startU, startV, startW);
        const T materialGate = smoothstepf(F(0.018), F(0.40), localChar + localPyrolysis * F(0.34) + localHeat * F(0.075));
        if (materialGate <= F(0.0001)) continue;
        const T temperatureK = F(620.0) + localHeat * F(330.0) + localPyrolysis * F(210.0) + localChar * F(42.0);
        const T sceneLift = sc == 1 ? F(0.86) : (sc == 2 ? F(0.16) : F(0.80));
        const T t = life * (sc == 1 ? F(1.24) : (sc == 2 ? F(0.34) : F(1.10)));
        const T drag = std::exp(-t * (sc == 2 ? F(4.8) : F(1.35)));
        const T buoyantRise = (F(0.26) + h3 * F(0.62) + localTurbulence * F(0.11)) * t * sceneLift;
        const V3<T> sparkWorld = {startX + (localVelocity.x * F(0.34) + (h1 - F(0.5)) * F(0.20) + p.wind * F(0.26)) * t * drag,
                                  startV * F(2.03) + F(0.02) + buoyantRise - (F(0.22) + h2 * F(0.16)) * t * t,
                                  startZ + (localVelocity.z * F(0.28) + (h2 - F(0.5)) * F(0.18)) * t * drag};
        const T prevT = std::fmax(F(0.0), t - F(0.045));
        const T prevDrag = std::exp(-prevT * (sc == 2 ? F(4.8) : F(1.35)));
        const V3<T> prevWorld = {startX + (localVelocity.x * F(0.34) + (h1 - F(0.5)) * F(0.20) + p.wind * F(0.26)) * prevT * prevDrag,
                                 startV * F(2.03) + F(0.02) + (F(0.26) + h3 * F(0.62) + localTurbulence * F(0.11)) * prevT * sceneLift -
                                     (F(0.22) + h2 * F(0.16)) * prevT * prevT,
                                 startZ + (localVelocity.z * F(0.28) + (h2 - F(0.5)) * F(0.18)) * prevT * prevDrag};
        const V3<T> sparkScreen = projectPoint(p, sparkWorld);
        const V3<T> prevScreen = projectPoint(p, prevWorld);
        if (sparkScreen.z <= F(0.0) || sparkScreen.x < F(-0.05) || sparkScreen.x > F(1.05) || sparkScreen.y < F(-0.05) ||
            sparkScreen.y > F(1.05)) continue;
        const T emberSize = smoothstepf(F(720.0), F(1580.0), temperatureK) * materialGate;
        const T radius = ((sc == 2 ? F(0.00042) : F(0.00086)) + h3 * (sc == 2 ? F(0.00042) : F(0.00145))) *
                         (F(0.72) + emberSize * F(0.90)) / std::fmax(F(0.55), sparkScreen.z);
        const T centerX = sparkScreen.x * T(static_cast<float>(p.frameW)) - F(0.5);
        const T centerY = sparkScreen.y * T(static_cast<float>(p.frameH)) - F(0.5);
        const V2<T> rawTrail = sub2(V2<T>{sparkScreen.x, sparkScreen.y}, V2<T>{prevScreen.x, prevScreen.y});
        const T rawTrailLen = std::sqrt(dot2(rawTrail, rawTrail));
        const T cappedTrailLen = std::fmin(rawTrailLen, sc == 1 ? F(0.016) : F(0.005));
        const V2<T> trailDir = rawTrailLen > F(0.000001) ? mul2(rawTrail, F(1.0) / rawTrailLen) : V2<T>{F(0.0), F(-1.0)};
        const int pad = std::max(2, static_cast<int>(std::ceil((radius + cappedTrailLen) *
                                                               T(static_cast<float>(std::max(p.frameW, p.frameH))) * F(3.0))));
        const int minX = std::max(0, static_cast<int>(std::floor(centerX)) - pad);
        const int maxX = std::min(p.frameW - 1, static_cast<int>(std::ceil(centerX)) + pad);
        const int minY = std::max(0, static_cast<int>(std::floor(centerY)) - pad);
        const int maxY = std::min(p.frameH - 1, static_cast<int>(std::ceil(centerY)) + pad);
        const V3<T> hotCore = sc == 2 ? V3<T>{F(0.36), F(0.58), F(1.04)} : V3<T>{F(1.0), F(0.42), F(0.090)};
        const V3<T> cooled = sc == 2 ? V3<T>{F(0.055), F(0.10), F(0.18)} : V3<T>{F(0.18), F(0.026), F(0.008)};
        const T cooling = smoothstepf(F(0.16), F(0.92), life) * (F(1.0) - saturate(localHeat * F(0.045)));
        const V3<T> sparkColor = lerp3(hotCore, cooled, cooling);
        const T lifeFade = smoothstepf(F(1.0), F(0.08), life) * smoothstepf(F(0.0), F(0.16), life) * sparkGate * materialGate *
                           emberSize * (sc == 2 ? F(0.055) : (sc == 1 ? F(0.58) : F(0.82)));
        for (int py = minY; py <= maxY; ++py) {
            const T uy = (T(static_cast<float>(py)) + F(0.5)) / T(static_cast<float>(p.frameH));
            for (int px = minX; px <= maxX; ++px) {
                const T ux = (T(static_cast<float>(px)) + F(0.5)) / T(static_cast<float>(p.frameW));
                const V2<T> d = sub2(V2<T>{ux, uy}, V2<T>{sparkScreen.x, sparkScreen.y});
                const T along = dot2(d, trailDir);
                const V2<T> acrossVec = sub2(d, mul2(trailDir, along));
                const T across2 = dot2(acrossVec, acrossVec);
                const T streakRadius = radius * (F(1.0) + cappedTrailLen * F(130.0));
                const T emberCore = std::exp(-(across2 / std::fmax(F(0.0000002), radius * radius) +
                                               along * along / std::fmax(F(0.0000002), streakRadius * streakRadius)));
                const T emberHalo = std::exp(-dot2(d, d) / std::fmax(F(0.0000002), radius * radius * F(8.0))) * F(0.16);
                const T spark = (emberCore + emberHalo) * lifeFade;
                if (spark > F(0.00001)) {
                    V4<T>& px4 = s.hdr[size_t(py) * p.frameW + px];
                    px4.x += sparkColor.x * spark;
                    px4.y += sparkColor.y * spark;
                    px4.z += sparkColor.z * spark;
                }
            }
        }
    }
}

// src/fire_cuda.cu:2246-2274 -- hue-preserving ACES and the camera response curve.
template <class T> T acesToneCurve(T value) {
    const T a = F(2.51), b = F(0.03), c = F(2.43), d = F(0.59), e = F(0.14);
    return saturate((value * (a * value + b)) / (value * (c * value + d) + e));
}
template <class T> V3<T> cameraResponse(V3<T> radiance, T exposure) {
    V3<T> color = mul3(V3<T>{std::fmax(F(0.0), radiance.x), std::fmax(F(0.0), radiance.y), std::fmax(F(0.0), radiance.z)}, exposure);
    {
        const T luma = std::fmax(F(0.000001), luminance3(color));
        const T mappedLuma = acesToneCurve(luma);
        color = mul3(color, mappedLuma / luma);
    }
    const T luma = luminance3(color);
    const T toe = smoothstepf(F(0.000), F(0.055), luma);
    const T hdrShoulderPreserve = smoothstepf(F(0.78), F(1.08), luma);
    color = lerp3(mul3(color, F(0.82)), color, toe);
    color = lerp3(color, mul3(color, F(1.0) / std::fmax(F(1.0), luma / F(0.94))), hdrShoulderPreserve * F(0.10));
    const T blackbodyHighlightLift = smoothstepf(F(0.56), F(0.90), luma);
    color = mul3(color, F(1.0) + blackbodyHighlightLift * F(0.28));
    return {std::pow(saturate(color.x), F(1.0) / F(2.2)), std::pow(saturate(color.y), F(1.0) / F(2.2)),
            std::pow(saturate(color.z), F(1.0) / F(2.2))};
}

inline uint32_t packChannel(float v) { return static_cast<uint32_t>(std::fmin(1.0f, std::fmax(0.0f, v)) * 255.0f); }

// src/fire_cuda.cu:2276-2297 -- exposure, camera response, dither, BGRA8.
template <class T> void stageTonemap(State<T>& s, const Params<T>& p) {
#pragma omp parallel for schedule(static)
    for (int y = 0; y < p.frameH; ++y) {
        for (int x = 0; x < p.frameW; ++x) {
            const size_t i = size_t(y) * p.frameW + x;
            const V4<T> r = s.hdr[i];
            V3<T> color = cameraResponse(V3<T>{r.x, r.y, r.z}, p.exposure);
            const T dither = (T(hash21f(static_cast<float>(x) * 0.754877f, static_cast<float>(y) * 0.569840f)) - F(0.5)) / F(255.0);
            color = add3(color, V3<T>{dither, dither, dither});
            s.bgra[i] = 0xff000000u | (packChannel(float(color.x)) << 16) | (packChannel(float(color.y)) << 8) |
                        packChannel(float(color.z));
        }
    }
}

// src/fire_cuda.cu:1909-1951 -- gizmo helpers.
template <class T> T lineAlpha(V2<T> q, V2<T> a, V2<T> b, T thickness) {
    const V2<T> pa = sub2(q, a);
    const V2<T> ba = sub2(b, a);
    const T h = saturate(dot2(pa, ba) / std::fmax(F(0.000001), dot2(ba, ba)));
    const V2<T> d = sub2(pa, mul2(ba, h));
    return smoothstepf(thickness, thickness * F(0.35), std::sqrt(dot2(d, d)));
}
template <class T> T ringAlpha(V2<T> q, V2<T> c, T radius, T thickness) {
    const V2<T> d = sub2(q, c);
    return smoothstepf(thickness, thickness * F(0.25), std::fabs(std::sqrt(dot2(d, d)) - radius));
}
template <class T> T diskAlpha(V2<T> q, V2<T> c, T radius) {
    const V2<T> d = sub2(q, c);
    return smoothstepf(radius, radius * F(0.45), std::sqrt(dot2(d, d)));
}

// src/fire_cuda.cu:2454-2494 -- gizmo overlay on the BGRA8 frame.
template <class T> void stageOverlay(State<T>& s, const Params<T>& p) {
    if (p.renderDebugMode != 0 || p.showGizmos == 0) return;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < p.frameH; ++y) {
        for (int x = 0; x < p.frameW; ++x) {
            const size_t i = size_t(y) * p.frameW + x;
            const uint32_t px = s.bgra[i];
            V3<T> color = {T(static_cast<float>((px >> 16) & 0xff) / 255.0f), T(static_cast<float>((px >> 8) & 0xff) / 255.0f),
                           T(static_cast<float>(px & 0xff) / 255.0f)};
            const V2<T> uv = {(T(static_cast<float>(x)) + F(0.5)) / T(static_cast<float>(p.frameW)),
                              (T(static_cast<float>(y)) + F(0.5)) / T(static_cast<float>(p.frameH))};
            auto blend = [&](V3<T> g, T alpha) { color = lerp3(color, g, saturate(alpha)); };
            const T sourceX = p.sceneId == 2 && p.burnerCenterCount > 0 ? p.burnerCenterX[0] : p.emitterCenterX;
            const T sourceY = p.sceneId == 2 && p.burnerCenterCount > 0 ? p.burnerCenterY[0] : p.emitterHeightNorm * F(2.03) + F(0.02);
            const T sourceZ = p.sceneId == 2 && p.burnerCenterCount > 0 ? p.burnerCenterZ[0] : p.emitterCenterZ;
            const V3<T> source = projectPoint(p, V3<T>{sourceX, sourceY, sourceZ});
            if (source.z > F(0.0)) {
                const V2<T> c = {source.x, source.y};
                const T a = ringAlpha(uv, c, F(0.125) / source.z, F(0.006)) + diskAlpha(uv, c, F(0.012));
                blend(p.activeGizmo == 1 ? V3<T>{F(1.0), F(0.34), F(0.055)} : V3<T>{F(0.45), F(0.18), F(0.055)}, a * F(0.85));
            }
            const V2<T> axisBase = {F(0.90), F(0.84)};
            const V3<T> ex = {F(1.0), F(0.0), F(0.0)}, ey = {F(0.0), F(1.0), F(0.0)}, ez = {F(0.0), F(0.0), F(1.0)};
            const V2<T> xAxis = add2(axisBase, mul2(V2<T>{dot3(ex, p.right), -dot3(ex, p.up)}, F(0.070)));
            const V2<T> yAxis = add2(axisBase, mul2(V2<T>{dot3(ey, p.right), -dot3(ey, p.up)}, F(0.070)));
            const V2<T> zAxis = add2(axisBase, mul2(V2<T>{dot3(ez, p.right), -dot3(ez, p.up)}, F(0.070)));
            blend(V3<T>{F(1.0), F(0.12), F(0.08)}, lineAlpha(uv, axisBase, xAxis, F(0.005)));
            blend(V3<T>{F(0.22), F(1.0), F(0.30)}, lineAlpha(uv, axisBase, yAxis, F(0.005)));
            blend(V3<T>{F(0.20), F(0.48), F(1.0)}, lineAlpha(uv, axisBase, zAxis, F(0.005)));
            s.bgra[i] = 0xff000000u | (packChannel(float(color.x)) << 16) | (packChannel(float(color.y)) << 8) | packChannel(float(color.z));
        }
    }
}

inline int floatBits(float v) {
    int b;
    std::memcpy(&b, &v, 4);
    return b;
}
inline float bitsFloat(int b) {
    float v;
    std::memcpy(&v, &b, 4);
    return v;
}

// src/fire_cuda.cu:1319-1418 + :3443-3471 -- post-projection divergence and
// the per-frame sums/maxima, summed in cell order in double.
template <class T> void stageMetrics(State<T>& s, const Params<T>& p) {
    computeDivergence(s, p, s.divergenceAfter);
    double sums[21] = {};
    int words[10] = {};
    auto maxPos = [](int& word, T value) {
        const float fv = float(value);
        if (fv > 0.0f && std::isfinite(fv)) word = std::max(word, floatBits(fv));
    };
    for (int z = 0; z < p.nz; ++z) {
        for (int y = 0; y < p.ny; ++y) {
            for (int x = 0; x < p.nx; ++x) {
                const size_t idx = (size_t(z) * p.ny + y) * p.nx + x;
                const T heat = s.scalar[HEAT][idx], fuel = s.scalar[FUEL][idx], oxygen = s.scalar[OXYGEN][idx];
                const T soot = s.scalar[SOOT][idx], charMass = s.scalar[CHAR][idx], ash = s.scalar[ASH][idx];
                const T pyrolysis = s.scalar[PYRO][idx], progress = s.scalar[PROGRESS][idx];
                const T turbulenceEnergy = s.scalar[TURB][idx], sootOptics = s.scalar[SOOTOPT][idx];
                const T divBefore = std::fabs(s.divergence[idx]);
                const T divAfter = std::fabs(s.divergenceAfter[idx]);
                const T u = cellU(x, p), v = cellV(y, p), w = cellW(z, p);
                const V4<T> sceneLight = sampleSceneLight(s.light.data(), p, u, v, w);
                const T sceneShadow = sampleSceneShadow(s.shadow.data(), p, u, v, w);
                if (!std::isfinite(heat) || !std::isfinite(fuel) || !std::isfinite(oxygen) || !std::isfinite(soot) ||
                    !std::isfinite(charMass) || !std::isfinite(ash) || !std::isfinite(pyrolysis) || !std::isfinite(progress) ||
                    !std::isfinite(turbulenceEnergy) || !std::isfinite(sootOptics) || !std::isfinite(divBefore) ||
                    !std::isfinite(divAfter)) {
                    words[9] += 1;
                    continue;
                }
                const T tempK = F(293.0) + heat * F(335.0);
                const T hrr = (fuel + pyrolysis * F(0.42)) * oxygen * smoothstepf(F(610.0), F(1280.0), tempK) *
                              std::exp(F(-5200.0) / std::fmax(F(650.0), tempK));
                const T opticalDepth = sootOptics + soot * (F(0.24) + F(0.05) * std::sqrt(std::fmax(F(0.0), heat)));
                const T normalizedHeight = (T(static_cast<float>(y)) + F(0.5)) / T(static_cast<float>(p.ny));
                const T flameMass = smoothstepf(F(0.72), F(2.10), heat + progress * F(0.62) + pyrolysis * F(0.24)) *
                                    smoothstepf(F(0.035), F(0.66), oxygen) * smoothstepf(F(0.012), F(0.52), fuel + pyrolysis * F(0.36));
                const T smokeMass = smoothstepf(F(0.035), F(1.16), sootOptics + soot * F(0.38) + ash * F(0.12)) *
                                    smoothstepf(F(0.08), F(0.88), normalizedHeight);
                const T overlap = flameMass * smokeMass;
                const T volumetricShadow = sceneShadow * std::exp(-sceneLight.w * F(0.80));
                const T roomIrradiance = luminance3(V3<T>{sceneLight.x, sceneLight.y, sceneLight.z}) * volumetricShadow;
                const T flameMarker = heat + fuel * F(0.24) + progress * F(0.55);
                const double vals[21] = {
                    double(heat), double(fuel), double(oxygen), double(soot), double(charMass), double(ash),
                    double(pyrolysis), double(progress), double(turbulenceEnergy), double(sootOptics),
                    double(luminance3(V3<T>{sceneLight.x, sceneLight.y, sceneLight.z})), double(sceneShadow),
                    double(flameMass), double(smokeMass), double(overlap), double(volumetricShadow), double(roomIrradiance),
                    double(opticalDepth), double(hrr), double(divBefore) * double(divBefore), double(divAfter) * double(divAfter)};
                for (int k = 0; k < 21; ++k) sums[k] += vals[k];
                maxPos(words[0], heat);
                maxPos(words[1], fuel);
                maxPos(words[2], soot);
                maxPos(words[3], pyrolysis);
                maxPos(words[4], progress);
                maxPos(words[5], turbulenceEnergy);
                maxPos(words[7], divBefore);
                maxPos(words[8], divAfter);
                if (flameMarker > F(0.74)) maxPos(words[6], normalizedHeight * T(kRoomHeightMeters));
            }
        }
    }
    std::memcpy(s.metricSums, sums, sizeof(sums));
    std::memcpy(s.metricWords, words, sizeof(words));
}

// src/fire_cuda.cu:3135-3179 -- settings clamps into the per-launch constant block.
template <class T> Params<T> makeParams(const State<T>& s, const FireSettings& st, float time) {
    Params<T> p{};
    p.nx = s.nx; p.ny = s.ny; p.nz = s.nz; p.frameW = s.frameW; p.frameH = s.frameH;
    p.lnx = s.lnx; p.lny = s.lny; p.lnz = s.lnz;
    auto cf = [](float v, float lo, float hi) { return std::max(lo, std::min(hi, v)); };
    auto ci = [](int v, int lo, int hi) { return std::max(lo, std::min(hi, v)); };
    p.dt = T(cf(st.dt, 0.001f, 1.0f / 30.0f));
    p.time = T(time);
    p.mouseX = T(cf(st.mouseX, 0.0f, 1.0f));
    p.mouseY = T(cf(st.mouseY, 0.0f, 1.0f));
    p.leftDown = st.leftDown;
    p.rightDown = st.rightDown;
    p.showGizmos = st.showGizmos;
    p.activeGizmo = st.activeGizmo;
    p.sceneId = ci(st.sceneId, 0, kSceneCount - 1);
    p.wind = T(cf(st.wind, -1.0f, 1.0f));
    p.turbulence = T(cf(st.turbulence, 0.05f, 1.8f));
    p.detail = T(cf(st.detail, 0.1f, 1.5f));
    p.smokeGain = T(cf(st.smoke, 0.0f, 1.6f));
    p.intensity = T(cf(st.intensity, 0.2f, 2.4f));
    p.cameraYaw = T(st.cameraYaw);
    p.cameraPitch = T(cf(st.cameraPitch, -0.75f, 0.75f));
    p.cameraDistance = T(cf(st.cameraDistance, 1.5f, 6.0f));
    p.cinematicMode = st.cinematicMode != 0 ? 1 : 0;
    p.raymarchSteps = ci(st.raymarchSteps, 24, kMaxRaymarchSteps);
    p.emberCount = ci(st.emberCount, 0, kMaxEmberCount);
    p.renderDebugMode = ci(st.renderDebugMode, 0, 6);
    p.exposure = T(cf(st.exposure, 0.45f, 2.40f));
    p.reflectionGain = T(cf(st.reflectionGain, 0.0f, 2.2f));
    p.smokeDarkness = T(cf(st.smokeDarkness, 0.35f, 2.4f));
    p.emitterCenterX = T(cf(st.emitterCenterX, -1.05f, 1.05f));
    p.emitterCenterZ = T(cf(st.emitterCenterZ, -0.82f, 0.82f));
    float heightNorm = cf(st.emitterHeightNorm, 0.0f, 0.96f);
    p.emitterHeightBandNorm = T(cf(st.emitterHeightBandNorm, 0.006f, 0.20f));
    p.emitterRadius = T(cf(st.emitterRadius, 0.035f, 0.80f));
    p.burnerCenterCount = ci(st.burnerCenterCount, 0, 4);
    float by0 = 0.0f;
    for (int i = 0; i < 4; ++i) {
        p.burnerCenterX[i] = T(cf(st.burnerCenterX[i], -1.05f, 1.05f));
        const float by = cf(st.burnerCenterY[i], 0.0f, 2.03f);
        if (i == 0) by0 = by;
        p.burnerCenterY[i] = T(by);
        p.burnerCenterZ[i] = T(cf(st.burnerCenterZ[i], -0.82f, 0.82f));
    }
    if (p.sceneId == 2 && p.burnerCenterCount > 0) heightNorm = cf((by0 - 0.02f) / 2.03f, 0.0f, 0.96f);
    p.emitterHeightNorm = T(heightNorm);
    // The camera basis is computed on the host in float by the reference
    // (updateCameraCache, src/fire_cuda.cu:2696-2704); computeCamera<float>
    // reproduces it, and the double oracle widens the float result.
    Params<float> pf{};
    pf.frameW = p.frameW; pf.frameH = p.frameH;
    pf.cameraYaw = float(p.cameraYaw); pf.cameraPitch = float(p.cameraPitch); pf.cameraDistance = float(p.cameraDistance);
    computeCamera(pf);
    p.eye = {T(pf.eye.x), T(pf.eye.y), T(pf.eye.z)};
    p.forward = {T(pf.forward.x), T(pf.forward.y), T(pf.forward.z)};
    p.right = {T(pf.right.x), T(pf.right.y), T(pf.right.z)};
    p.up = {T(pf.up.x), T(pf.up.y), T(pf.up.z)};
    p.tanHalfFov = T(pf.tanHalfFov);
    p.aspect = T(pf.aspect);
    return p;
}

template <class T> int runStage(State<T>& s, int stage, const Params<T>& p) {
    switch (stage) {
        case 0: stageAdvectVelocity(s, p); return 0;
        case 1: stageAdvectReact(s, p); return 0;
        case 2: stageForce(s, p); return 0;
        case 3: stageVelocityBoundary(s, p, true); return 0;
        case 4:
            computeDivergence(s, p, s.divergence);
            std::fill(s.pressure.begin(), s.pressure.end(), F(0.0));
            return 0;
        case 5: stagePressureSor(s, p); return 0;
        case 6: stageSubtract(s, p); return 0;
        case 7: stageVelocityBoundary(s, p, false); return 0;
        case 8: stageLightBuild(s, p); return 0;
        case 9: stageLightPropagate(s, p); return 0;
        case 10: stageRender(s, p); return 0;
        case 11: stageEmbers(s, p); return 0;
        case 12: stageTonemap(s, p); return 0;
        case 13: stageOverlay(s, p); return 0;
        case 14: stageMetrics(s, p); return 0;
        case 15: stageReset(s, p); return 0;
        default: return setError("unknown stage");
    }
}

// src/fire_cuda.cu:3106-3549 -- one frame with the reference's time bookkeeping.
template <class T>
int runFrame(State<T>& s, uint32_t* bgra, const FireSettings& st, FireCudaFrameMetrics* metrics, int mode) {
    const bool advance = mode != 3;
    const bool render = mode != 2;
    const bool collect = mode == 1;
    const float stepDt = std::max(0.001f, std::min(st.dt, 1.0f / 30.0f));
    s.renderTime += stepDt;
    if (advance) s.simTime += stepDt;
    Params<T> p = makeParams(s, st, advance ? s.simTime : s.renderTime);
    if (st.reset != 0) {
        // resetSimulationFields zeroes both clocks but the step keeps using
        // the parameter block built before the reset (src/fire_cuda.cu:3181, :3053-3055).
        stageReset(s, p);
        s.simTime = 0.0f;
        s.renderTime = 0.0f;
        s.frameIndex = 0;
    }
    if (advance) {
        for (int stage = 0; stage <= 9; ++stage) runStage(s, stage, p);
    }
    if (!render) return 0;
    p.time = T(s.renderTime);
    stageRender(s, p);
    stageEmbers(s, p);
    stageTonemap(s, p);
    stageOverlay(s, p);
    if (bgra != nullptr) std::memcpy(bgra, s.bgra.data(), s.bgra.size() * 4);
    if (collect && metrics != nullptr) {
        stageMetrics(s, p);
        const double cellCount = double(s.cells());
        const double* m = s.metricSums;
        const int* wd = s.metricWords;
        FireCudaFrameMetrics out{};
        const float divBeforeL2 = float(std::sqrt(m[19] / std::max(1.0, cellCount)));
        const float divAfterL2 = float(std::sqrt(m[20] / std::max(1.0, cellCount)));
        out.frameIndex = s.frameIndex;
        out.gridX = s.nx; out.gridY = s.ny; out.gridZ = s.nz;
        out.pressureIterations = s.pressureIterations;
        out.invalidCells = wd[9];
        out.timeSeconds = s.simTime;
        out.heatSum = float(m[0]); out.fuelSum = float(m[1]); out.oxygenSum = float(m[2]); out.sootSum = float(m[3]);
        out.charSum = float(m[4]); out.ashSum = float(m[5]); out.pyrolysisSum = float(m[6]); out.progressSum = float(m[7]);
        out.turbulenceEnergySum = float(m[8]); out.sootOpticalDepthSum = float(m[9]);
        out.maxHeat = bitsFloat(wd[0]); out.maxFuel = bitsFloat(wd[1]); out.maxSoot = bitsFloat(wd[2]);
        out.maxPyrolysis = bitsFloat(wd[3]); out.maxProgress = bitsFloat(wd[4]); out.maxTurbulenceEnergy = bitsFloat(wd[5]);
        out.flameHeightMeters = bitsFloat(wd[6]);
        out.meanOpticalDepth = float(m[17] / std::max(1.0, cellCount));
        out.meanSceneLight = float(m[10] / std::max(1.0, cellCount));
        out.meanSceneShadow = float(m[11] / std::max(1.0, cellCount));
        out.flameMassProxy = float(m[12]); out.smokeMassProxy = float(m[13]); out.flameSmokeOverlapProxy = float(m[14]);
        out.meanVolumetricShadow = float(m[15] / std::max(1.0, cellCount));
        out.meanRoomIrradiance = float(m[16] / std::max(1.0, cellCount));
        out.heatReleaseProxy = float(m[18]);
        out.divergenceBeforeL2 = divBeforeL2;
        out.divergenceBeforeMax = bitsFloat(wd[7]);
        out.divergenceAfterL2 = divAfterL2;
        out.divergenceAfterMax = bitsFloat(wd[8]);
        out.divergenceReduction = divBeforeL2 > 0.000001f ? 1.0f - divAfterL2 / divBeforeL2 : 0.0f;
        *metrics = out;
    }
    ++s.frameIndex;
    return 0;
}

struct Oracle {
    int precision;
    std::unique_ptr<State<float>> f;
    std::unique_ptr<State<double>> d;
};

template <class T> void initState(State<T>& s, int fw, int fh, int nx, int ny, int nz) {
    s.nx = nx; s.ny = ny; s.nz = nz; s.frameW = fw; s.frameH = fh;
    auto clampI = [](int v, int lo, int hi) { return std::max(lo, std::min(hi, v)); };
    // Light grid, src/fire_cuda.cu:2920-2922.
    s.lnx = clampI((nx + 3) / 4, 18, 48);
    s.lny = clampI((ny + 3) / 4, 20, 56);
    s.lnz = clampI((nz + 3) / 4, 16, 36);
    const size_t n = s.cells();
    for (auto& v : s.scalar) v.assign(n, T(0));
    s.pressure.assign(n, T(0));
    s.divergence.assign(n, T(0));
    s.divergenceAfter.assign(n, T(0));
    s.u.assign(size_t(nx + 1) * ny * nz, T(0));
    s.v.assign(size_t(nx) * (ny + 1) * nz, T(0));
    s.w.assign(size_t(nx) * ny * (nz + 1), T(0));
    s.light.assign(s.lightCells(), V4<T>{});
    s.lightNext.assign(s.lightCells(), V4<T>{});
    s.shadow.assign(s.lightCells(), T(0));
    s.hdr.assign(size_t(fw) * fh, V4<T>{});
    s.bgra.assign(size_t(fw) * fh, 0u);
}

// Generic field access: returns element pointer, element count and components.
template <class T> T* fieldData(State<T>& s, int id, size_t* count, int* comps) {
    *comps = 1;
    switch (id) {
        case 0: case 1: case 2: case 3: case 4: case 5: case 6: case 7: case 8: case 9:
            *count = s.scalar[id].size(); return s.scalar[id].data();
        case 10: *count = s.pressure.size(); return s.pressure.data();
        case 11: *count = s.divergence.size(); return s.divergence.data();
        case 12: *count = s.u.size(); return s.u.data();
        case 13: *count = s.v.size(); return s.v.data();
        case 14: *count = s.w.size(); return s.w.data();
        case 15: *comps = 4; *count = s.light.size(); return &s.light[0].x;
        case 16: *count = s.shadow.size(); return s.shadow.data();
        case 17: *comps = 4; *count = s.hdr.size(); return &s.hdr[0].x;
        case 19: *count = s.divergenceAfter.size(); return s.divergenceAfter.data();
        default: *count = 0; return nullptr;
    }
}

template <class T> int setField(State<T>& s, int id, const void* host, long long bytes) {
    if (id == 18) {
        if (size_t(bytes) != s.bgra.size() * 4) return setError("bgra size mismatch");
        std::memcpy(s.bgra.data(), host, size_t(bytes));
        return 0;
    }
    size_t count = 0;
    int comps = 1;
    T* dst = fieldData(s, id, &count, &comps);
    if (dst == nullptr) return setError("unknown field");
    const size_t n = count * comps;
    if (size_t(bytes) != n * 4) return setError("field size mismatch");
    const float* src = static_cast<const float*>(host);
    for (size_t i = 0; i < n; ++i) dst[i] = T(src[i]);
    return 0;
}

template <class T> int getField(State<T>& s, int id, void* host, long long bytes) {
    if (id == 18) {
        if (size_t(bytes) != s.bgra.size() * 4) return setError("bgra size mismatch");
        std::memcpy(host, s.bgra.data(), size_t(bytes));
        return 0;
    }
    size_t count = 0;
    int comps = 1;
    T* src = fieldData(s, id, &count, &comps);
    if (src == nullptr) return setError("unknown field");
    const size_t n = count * comps;
    if (size_t(bytes) != n * 4) return setError("field size mismatch");
    float* dst = static_cast<float*>(host);
    for (size_t i = 0; i < n; ++i) dst[i] = float(src[i]);
    return 0;
}

template <class T> int getFieldF64(State<T>& s, int id, double* host, long long count64) {
    size_t count = 0;
    int comps = 1;
    T* src = fieldData(s, id, &count, &comps);
    if (src == nullptr) return setError("unknown field");
    if (size_t(count64) != count * comps) return setError("field size mismatch");
    for (size_t i = 0; i < count * comps; ++i) host[i] = double(src[i]);
    return 0;
}

}  // namespace

extern "C" {

void* oracle_create(int precision, int frameW, int frameH, int nx, int ny, int nz) {
    if (nx < 2 || ny < 2 || nz < 2 || frameW < 1 || frameH < 1) {
        setError("oracle_create: invalid dimensions");
        return nullptr;
    }
    auto* o = new Oracle{precision, nullptr, nullptr};
    if (precision == 0) {
        o->f.reset(new State<float>());
        initState(*o->f, frameW, frameH, nx, ny, nz);
    } else {
        o->d.reset(new State<double>());
        initState(*o->d, frameW, frameH, nx, ny, nz);
    }
    return o;
}

void oracle_destroy(void* h) { delete static_cast<Oracle*>(h); }

#define DISPATCH(h, expr_f, expr_d)        \
    Oracle* o = static_cast<Oracle*>(h);   \
    if (o->precision == 0) {               \
        auto& s = *o->f;                   \
        (void)s;                           \
        expr_f;                            \
    } else {                               \
        auto& s = *o->d;                   \
        (void)s;                           \
        expr_d;                            \
    }

void oracle_light_dims(void* h, int* dims) {
    DISPATCH(h, (dims[0] = s.lnx, dims[1] = s.lny, dims[2] = s.lnz), (dims[0] = s.lnx, dims[1] = s.lny, dims[2] = s.lnz))
}

int oracle_set_field(void* h, int id, const void* host, long long bytes) {
    DISPATCH(h, return setField(s, id, host, bytes), return setField(s, id, host, bytes))
}

int oracle_get_field(void* h, int id, void* host, long long bytes) {
    DISPATCH(h, return getField(s, id, host, bytes), return getField(s, id, host, bytes))
}

int oracle_get_field_f64(void* h, int id, double* host, long long count) {
    DISPATCH(h, return getFieldF64(s, id, host, count), return getFieldF64(s, id, host, count))
}

int oracle_stages(void* h, int first, int last, const FireSettings* st, float time) {
    DISPATCH(
        h,
        {
            const Params<float> p = makeParams(s, *st, time);
            for (int k = first; k <= last; ++k)
                if (runStage(s, k, p) != 0) return -1;
            return 0;
        },
        {
            const Params<double> p = makeParams(s, *st, time);
            for (int k = first; k <= last; ++k)
                if (runStage(s, k, p) != 0) return -1;
            return 0;
        })
}

void oracle_set_pressure_solver(void* h, int iterations, float omega) {
    DISPATCH(h, (s.pressureIterations = iterations, s.pressureOmega = omega),
             (s.pressureIterations = iterations, s.pressureOmega = omega))
}

int oracle_step(void* h, uint32_t* bgra, const FireSettings* st, FireCudaFrameMetrics* metrics, int mode) {
    DISPATCH(h, return runFrame(s, bgra, *st, metrics, mode), return runFrame(s, bgra, *st, metrics, mode))
}

void oracle_last_metrics(void* h, double* sums21, int* words10) {
    DISPATCH(h, (std::memcpy(sums21, s.metricSums, sizeof(s.metricSums)), std::memcpy(words10, s.metricWords, sizeof(s.metricWords))),
             (std::memcpy(sums21, s.metricSums, sizeof(s.metricSums)), std::memcpy(words10, s.metricWords, sizeof(s.metricWords))))
}

void oracle_times(void* h, float* simTime, float* renderTime, int* frameIndex) {
    DISPATCH(h, (*simTime = s.simTime, *renderTime = s.renderTime, *frameIndex = s.frameIndex),
             (*simTime = s.simTime, *renderTime = s.renderTime, *frameIndex = s.frameIndex))
}

void oracle_set_times(void* h, float simTime, float renderTime, int frameIndex) {
    DISPATCH(h, (s.simTime = simTime, s.renderTime = renderTime, s.frameIndex = frameIndex),
             (s.simTime = simTime, s.renderTime = renderTime, s.frameIndex = frameIndex))
}

int oracle_threads(void) { return omp_get_max_threads(); }
void oracle_set_threads(int n) { omp_set_num_threads(n); }
const char* oracle_last_error(void) { return g_error; }

}  // extern "C"
