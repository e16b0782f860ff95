// config_oracle.cpp -- CPU oracle of the config physics (see config_oracle.h).
//
// TEST INFRASTRUCTURE, NOT PRODUCT CODE.  A plain restatement of the model of
// include/fire_ext.h ("Config physics"), written independently of the CUDA
// kernels.  Every expression is evaluated in the order the model states it
// (lerp(a, b, t) = fma(t, b - a, a); trilinear along x, then y, then z; sums
// left to right), so T = float reproduces the product's rounding.  The
// projection (divergence, red-black SOR, gradient subtraction, wall zeroing)
// restates the reference's, src/fire_cuda.cu:1185-1245 and :1293-1317,
// which the config physics shares with the reference physics.
#include "config_oracle.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

namespace {

char g_error[256] = "no error";

int setError(const char* msg) {
    std::snprintf(g_error, sizeof(g_error), "%s", msg);
    return -1;
}

// SplitMix64 output function (Steele, Lea and Flood, OOPSLA 2014).
uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Emitter jitter U in [0, 1): the top 24 bits of mix64((seed << 32) ^ step * K ^ cell), times 2^-24.
float jitter(unsigned seed, uint64_t step, unsigned cell) {
    const uint64_t k = (uint64_t(seed) << 32) ^ (step * 0xD1B54A32D192ED03ull) ^ uint64_t(cell);
    return float(mix64(k) >> 40) * (1.0f / 16777216.0f);
}

// Lattice value in [-1, 1): the top 24 bits of mix64 of the seeded lattice key, times 2^-23, minus 1.
float lattice(unsigned seed, int comp, int ix, int iy, int iz) {
    const uint64_t k = ((uint64_t(seed) << 2) | uint64_t(unsigned(comp))) * 0xD1342543DE82EF95ull +
                       uint64_t(unsigned(ix)) * 0x9E3779B97F4A7C15ull + uint64_t(unsigned(iy)) * 0xC2B2AE3D27D4EB4Full +
                       uint64_t(unsigned(iz)) * 0x165667B19E3779F9ull;
    return float(mix64(k) >> 40) * (1.0f / 8388608.0f) - 1.0f;
}

template <class T>
struct Vec3 {
    T x, y, z;
};

template <class T>
struct Emitter {
    T cx, cz, r2, fuel, heat, up, jit;
    int row;
    unsigned seed;
};

template <class T>
struct Derived {
    T dt, burnFrac, coolFrac, sootFrac, ignition, heatRelease, sootYield, buoyHeat, buoySoot, ambient, eps, windDtX, windDtZ;
    T noiseAmp, invPeriod;
    unsigned noiseSeed;
    std::vector<Emitter<T>> emitters;
    int primary, lightSamples;
    Vec3<T> light, eye, fwd, right, up;
    T lightIntensity, extinction, fuelExtinction, emission, albedo, tanHalf, aspect;
};

template <class T>
struct Scene {
    int nx, ny, nz, lx, ly, lz, W, H;
    std::vector<T> heat, fuel, soot, u, v, w, pressure, divergence, transmittance, hdr;
    std::vector<T> delta;  // the latest multigrid solve's pressure increment (Dirichlet top)
    std::vector<T> vort;   // 4 per cell
    std::vector<T> force;  // 3 per cell
    FirePhysicsParams phys;
    int iterations = 40;
    float omega = 1.52f;
    uint64_t step = 0;
    // Multigrid (Dirichlet top): cycles per solve, smoothing sweeps, tolerance on max |r| (0 = none).
    int mgCycles = 0, mgPre = 2, mgPost = 2;
    float mgTolerance = 0.0f;
    int mgCyclesRun = 0;
    float mgMaxResidual = -1.0f;

    int cells() const { return nx * ny * nz; }
    int sI(int x, int y, int z) const { return (z * ny + y) * nx + x; }
    int uI(int x, int y, int z) const { return (z * ny + y) * (nx + 1) + x; }
    int vI(int x, int y, int z) const { return (z * (ny + 1) + y) * nx + x; }
    int wI(int x, int y, int z) const { return (z * ny + y) * nx + x; }

    void resize() {
        const size_t n = size_t(cells());
        heat.assign(n, T(0));
        fuel.assign(n, T(0));
        soot.assign(n, T(0));
        pressure.assign(n, T(0));
        divergence.assign(n, T(0));
        u.assign(size_t(nx + 1) * ny * nz, T(0));
        v.assign(size_t(nx) * (ny + 1) * nz, T(0));
        w.assign(size_t(nx) * ny * (nz + 1), T(0));
        transmittance.assign(size_t(lx) * ly * lz, T(0));
        hdr.assign(size_t(W) * H * 4, T(0));
        vort.assign(n * 4, T(0));
        delta.clear();
        force.assign(n * 3, T(0));
        step = 0;
    }

    // The per-step constants, formed from the float parameters in T.
    Derived<T> derive() const {
        const FirePhysicsParams& q = phys;
        Derived<T> d;
        const T dt = T(q.dt);
        d.dt = dt;
        d.burnFrac = std::min(T(1), T(q.burnRate) * dt);
        d.coolFrac = std::min(T(1), T(q.cooling) * dt);
        d.sootFrac = std::min(T(1), T(q.sootDecay) * dt);
        d.ignition = T(q.ignitionHeat);
        d.heatRelease = T(q.heatRelease);
        d.sootYield = T(q.sootYield);
        d.buoyHeat = T(q.buoyancyHeat);
        d.buoySoot = T(q.buoyancySoot);
        d.ambient = T(q.ambientHeat);
        d.eps = T(q.vorticityEps);
        d.windDtX = dt * T(q.windX);
        d.windDtZ = dt * T(q.windZ);
        d.noiseAmp = T(q.noiseAmplitude);
        d.invPeriod = T(1) / T(q.noisePeriod);
        d.noiseSeed = q.noiseSeed;
        for (int e = 0; e < q.emitterCount; ++e) {
            const FireEmitterDisk& k = q.emitters[e];
            d.emitters.push_back(Emitter<T>{T(k.centerX), T(k.centerZ), T(k.radius) * T(k.radius), T(k.fuel), T(k.heat),
                                            T(k.upVelocity), T(k.jitterScale), int(std::floor(k.centerY)), k.seed});
        }
        d.primary = q.primarySamples;
        d.lightSamples = q.lightSamples;
        d.light = {T(q.lightX), T(q.lightY), T(q.lightZ)};
        d.lightIntensity = T(q.lightIntensity);
        d.extinction = T(q.extinction);
        d.fuelExtinction = T(q.fuelExtinction);
        d.emission = T(q.emission);
        d.albedo = T(q.albedo);
        // Pinhole camera: forward to the target, right = forward x (0,1,0), up = right x forward.
        T fx = T(q.targetX) - T(q.eyeX), fy = T(q.targetY) - T(q.eyeY), fz = T(q.targetZ) - T(q.eyeZ);
        const T fl = std::sqrt(fx * fx + fy * fy + fz * fz);
        fx = fx / fl;
        fy = fy / fl;
        fz = fz / fl;
        T rx = -fz, ry = T(0), rz = fx;
        const T rl = std::sqrt(rx * rx + rz * rz);
        if (rl > T(0)) {
            rx = rx / rl;
            rz = rz / rl;
        } else {
            rx = T(1);
            rz = T(0);
        }
        d.eye = {T(q.eyeX), T(q.eyeY), T(q.eyeZ)};
        d.fwd = {fx, fy, fz};
        d.right = {rx, ry, rz};
        d.up = {ry * fz - rz * fy, rz * fx - rx * fz, rx * fy - ry * fx};
        d.tanHalf = T(std::tan(q.fovYDegrees * 0.00872664626f));
        d.aspect = T(W) / T(H);
        return d;
    }
};

template <class T>
struct Axis {
    int i0, i1;
    T t;
};

template <class T> Axis<T> axis(T q, int m) {
    q = std::fmin(std::fmax(q, T(0)), T(m - 1));
    Axis<T> a;
    a.i0 = int(q);
    a.i1 = std::min(a.i0 + 1, m - 1);
    a.t = q - T(a.i0);
    return a;
}

// One fused multiply-add, as the kernels' lerp1 (__fmaf_rn).
template <class T> T lerp(T a, T b, T t) { return std::fma(t, b - a, a); }

// Clamped trilinear sample of grid f (mx * my * mz, x fastest) at index position (qx, qy, qz).
template <class T> T trilinear(const std::vector<T>& f, int mx, int my, int mz, T qx, T qy, T qz) {
    const Axis<T> ax = axis(qx, mx), ay = axis(qy, my), az = axis(qz, mz);
    auto at = [&](int x, int y, int z) { return f[size_t((z * my + y) * mx + x)]; };
    const T a00 = lerp(at(ax.i0, ay.i0, az.i0), at(ax.i1, ay.i0, az.i0), ax.t);
    const T a10 = lerp(at(ax.i0, ay.i1, az.i0), at(ax.i1, ay.i1, az.i0), ax.t);
    const T a01 = lerp(at(ax.i0, ay.i0, az.i1), at(ax.i1, ay.i0, az.i1), ax.t);
    const T a11 = lerp(at(ax.i0, ay.i1, az.i1), at(ax.i1, ay.i1, az.i1), ax.t);
    const T b0 = lerp(a00, a10, ay.t);
    const T b1 = lerp(a01, a11, ay.t);
    return lerp(b0, b1, az.t);
}

template <class T> Vec3<T> velocityAt(const Scene<T>& s, T x, T y, T z) {
    const T h = T(0.5f);
    return {trilinear(s.u, s.nx + 1, s.ny, s.nz, x, y - h, z - h), trilinear(s.v, s.nx, s.ny + 1, s.nz, x - h, y, z - h),
            trilinear(s.w, s.nx, s.ny, s.nz + 1, x - h, y - h, z)};
}

// (heat, fuel, soot) at a position in cell units (cell centres at i + 0.5).
template <class T> Vec3<T> scalarsAt(const Scene<T>& s, T x, T y, T z) {
    const T h = T(0.5f);
    return {trilinear(s.heat, s.nx, s.ny, s.nz, x - h, y - h, z - h), trilinear(s.fuel, s.nx, s.ny, s.nz, x - h, y - h, z - h),
            trilinear(s.soot, s.nx, s.ny, s.nz, x - h, y - h, z - h)};
}

template <class T> bool inDisk(const Emitter<T>& e, int x, int y, int z) {
    if (y != e.row) return false;
    const T dx = T(x) - e.cx;
    const T dz = T(z) - e.cz;
    return dx * dx + dz * dz <= e.r2;
}

// Stage ADVECT_VELOCITY: every face from its one-step backtrace.
template <class T> void advectVelocity(Scene<T>& s) {
    std::vector<T> un(s.u.size()), vn(s.v.size()), wn(s.w.size());
    const T h = T(0.5f);
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z <= s.nz; ++z) {
        for (int y = 0; y <= s.ny; ++y) {
            for (int x = 0; x <= s.nx; ++x) {
                if (y < s.ny && z < s.nz) {
                    const T px = T(x), py = T(y) + h, pz = T(z) + h;
                    const Vec3<T> d = velocityAt(s, px, py, pz);
                    un[size_t(s.uI(x, y, z))] = trilinear(s.u, s.nx + 1, s.ny, s.nz, px - d.x, (py - d.y) - h, (pz - d.z) - h);
                }
                if (x < s.nx && z < s.nz) {
                    const T px = T(x) + h, py = T(y), pz = T(z) + h;
                    const Vec3<T> d = velocityAt(s, px, py, pz);
                    vn[size_t(s.vI(x, y, z))] = trilinear(s.v, s.nx, s.ny + 1, s.nz, (px - d.x) - h, py - d.y, (pz - d.z) - h);
                }
                if (x < s.nx && y < s.ny) {
                    const T px = T(x) + h, py = T(y) + h, pz = T(z);
                    const Vec3<T> d = velocityAt(s, px, py, pz);
                    wn[size_t(s.wI(x, y, z))] = trilinear(s.w, s.nx, s.ny, s.nz + 1, (px - d.x) - h, (py - d.y) - h, pz - d.z);
                }
            }
        }
    }
    s.u.swap(un);
    s.v.swap(vn);
    s.w.swap(wn);
}

// Stage ADVECT_REACT: backtrace of (T, F, S), burn, decay, emitters; the step counter advances.
template <class T> void advectScalars(Scene<T>& s, const Derived<T>& d) {
    const size_t n = size_t(s.cells());
    std::vector<T> hn(n), fn(n), sn(n);
    const T h = T(0.5f);
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < s.nz; ++z) {
        for (int y = 0; y < s.ny; ++y) {
            for (int x = 0; x < s.nx; ++x) {
                const T px = T(x) + h, py = T(y) + h, pz = T(z) + h;
                const Vec3<T> vel = velocityAt(s, px, py, pz);
                const Vec3<T> a = scalarsAt(s, px - vel.x, py - vel.y, pz - vel.z);
                T heat = a.x, fuel = a.y, soot = a.z;
                if (heat > d.ignition) {
                    const T burn = fuel * d.burnFrac;
                    fuel = fuel - burn;
                    heat = heat + d.heatRelease * burn;
                    soot = soot + d.sootYield * burn;
                }
                heat = heat - heat * d.coolFrac;
                soot = soot - soot * d.sootFrac;
                const unsigned cell = unsigned(s.sI(x, y, z));
                for (const Emitter<T>& e : d.emitters) {
                    if (!inDisk(e, x, y, z)) continue;
                    const T j = T(1) - e.jit * T(jitter(e.seed, s.step, cell));
                    fuel = std::fmax(fuel, e.fuel * j);
                    heat = std::fmax(heat, e.heat * j);
                }
                hn[cell] = heat;
                fn[cell] = fuel;
                sn[cell] = soot;
            }
        }
    }
    s.heat.swap(hn);
    s.fuel.swap(fn);
    s.soot.swap(sn);
    ++s.step;
}

// Value noise psi_comp at (x, y, z) and its gradient (cubic Hermite weights, analytic derivative).
template <class T> Vec3<T> noiseGrad(const Derived<T>& d, int comp, T x, T y, T z) {
    const T qx = x * d.invPeriod, qy = y * d.invPeriod, qz = z * d.invPeriod;
    const T fx0 = std::floor(qx), fy0 = std::floor(qy), fz0 = std::floor(qz);
    const int ix = int(fx0), iy = int(fy0), iz = int(fz0);
    const T fx = qx - fx0, fy = qy - fy0, fz = qz - fz0;
    const T sx = fx * fx * (T(3) - T(2) * fx), sy = fy * fy * (T(3) - T(2) * fy), sz = fz * fz * (T(3) - T(2) * fz);
    const T dsx = T(6) * fx * (T(1) - fx), dsy = T(6) * fy * (T(1) - fy), dsz = T(6) * fz * (T(1) - fz);
    auto L = [&](int a, int b, int c) { return T(lattice(d.noiseSeed, comp, ix + a, iy + b, iz + c)); };
    const T c000 = L(0, 0, 0), c100 = L(1, 0, 0), c010 = L(0, 1, 0), c110 = L(1, 1, 0);
    const T c001 = L(0, 0, 1), c101 = L(1, 0, 1), c011 = L(0, 1, 1), c111 = L(1, 1, 1);
    const T a00 = lerp(c000, c100, sx), a10 = lerp(c010, c110, sx), a01 = lerp(c001, c101, sx), a11 = lerp(c011, c111, sx);
    const T b0 = lerp(a00, a10, sy), b1 = lerp(a01, a11, sy);
    const T e0 = lerp(c100 - c000, c110 - c010, sy), e1 = lerp(c101 - c001, c111 - c011, sy);
    const T gx = dsx * lerp(e0, e1, sz);
    const T gy = dsy * lerp(a10 - a00, a11 - a01, sz);
    const T gz = dsz * (b1 - b0);
    return {gx * d.invPeriod, gy * d.invPeriod, gz * d.invPeriod};
}

// Stage FORCE: vorticity, cell accelerations, faces with wind, emitter velocity and walls.
template <class T> void forces(Scene<T>& s, const Derived<T>& d) {
    const T h = T(0.5f);
    auto ccx = [&](int i, int j, int k) { return h * (s.u[size_t(s.uI(i, j, k))] + s.u[size_t(s.uI(i + 1, j, k))]); };
    auto ccy = [&](int i, int j, int k) { return h * (s.v[size_t(s.vI(i, j, k))] + s.v[size_t(s.vI(i, j + 1, k))]); };
    auto ccz = [&](int i, int j, int k) { return h * (s.w[size_t(s.wI(i, j, k))] + s.w[size_t(s.wI(i, j, k + 1))]); };
    if (d.eps != T(0)) {
#pragma omp parallel for collapse(2) schedule(static)
        for (int z = 0; z < s.nz; ++z) {
            for (int y = 0; y < s.ny; ++y) {
                for (int x = 0; x < s.nx; ++x) {
                    const int xm = std::max(x - 1, 0), xp = std::min(x + 1, s.nx - 1);
                    const int ym = std::max(y - 1, 0), yp = std::min(y + 1, s.ny - 1);
                    const int zm = std::max(z - 1, 0), zp = std::min(z + 1, s.nz - 1);
                    const T ox = h * (ccz(x, yp, z) - ccz(x, ym, z)) - h * (ccy(x, y, zp) - ccy(x, y, zm));
                    const T oy = h * (ccx(x, y, zp) - ccx(x, y, zm)) - h * (ccz(xp, y, z) - ccz(xm, y, z));
                    const T oz = h * (ccy(xp, y, z) - ccy(xm, y, z)) - h * (ccx(x, yp, z) - ccx(x, ym, z));
                    T* o = &s.vort[size_t(s.sI(x, y, z)) * 4];
                    o[0] = ox;
                    o[1] = oy;
                    o[2] = oz;
                    o[3] = std::sqrt(ox * ox + oy * oy + oz * oz);
                }
            }
        }
    }
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < s.nz; ++z) {
        for (int y = 0; y < s.ny; ++y) {
            for (int x = 0; x < s.nx; ++x) {
                const int idx = s.sI(x, y, z);
                T cx = T(0), cy = T(0), cz = T(0);
                if (d.eps != T(0)) {
                    const int xm = std::max(x - 1, 0), xp = std::min(x + 1, s.nx - 1);
                    const int ym = std::max(y - 1, 0), yp = std::min(y + 1, s.ny - 1);
                    const int zm = std::max(z - 1, 0), zp = std::min(z + 1, s.nz - 1);
                    auto mag = [&](int i, int j, int k) { return s.vort[size_t(s.sI(i, j, k)) * 4 + 3]; };
                    const T* o = &s.vort[size_t(idx) * 4];
                    const T ex = h * (mag(xp, y, z) - mag(xm, y, z));
                    const T ey = h * (mag(x, yp, z) - mag(x, ym, z));
                    const T ez = h * (mag(x, y, zp) - mag(x, y, zm));
                    const T len = std::sqrt(ex * ex + ey * ey + ez * ez);
                    T nx = T(0), ny = T(0), nz = T(0);
                    if (len > T(1e-20f)) {
                        nx = ex / len;
                        ny = ey / len;
                        nz = ez / len;
                    }
                    cx = d.eps * (ny * o[2] - nz * o[1]);
                    cy = d.eps * (nz * o[0] - nx * o[2]);
                    cz = d.eps * (nx * o[1] - ny * o[0]);
                }
                T fx = T(0), fy = T(0), fz = T(0);
                if (d.noiseAmp != T(0)) {
                    const T px = T(x) + h, py = T(y) + h, pz = T(z) + h;
                    const Vec3<T> g0 = noiseGrad(d, 0, px, py, pz);
                    const Vec3<T> g1 = noiseGrad(d, 1, px, py, pz);
                    const Vec3<T> g2 = noiseGrad(d, 2, px, py, pz);
                    fx = d.noiseAmp * (g2.y - g1.z);
                    fy = d.noiseAmp * (g0.z - g2.x);
                    fz = d.noiseAmp * (g1.x - g0.y);
                }
                const T buoyancy = d.buoyHeat * (s.heat[size_t(idx)] - d.ambient) - d.buoySoot * s.soot[size_t(idx)];
                T* f = &s.force[size_t(idx) * 3];
                f[0] = cx + fx;
                f[1] = buoyancy + cy + fy;
                f[2] = cz + fz;
            }
        }
    }
    auto F = [&](int x, int y, int z, int c) { return s.force[size_t(s.sI(x, y, z)) * 3 + c]; };
    std::vector<T> un(s.u.size()), vn(s.v.size()), wn(s.w.size());
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z <= s.nz; ++z) {
        for (int y = 0; y <= s.ny; ++y) {
            for (int x = 0; x <= s.nx; ++x) {
                if (y < s.ny && z < s.nz) {
                    T uu = T(0);
                    if (x > 0 && x < s.nx) uu = s.u[size_t(s.uI(x, y, z))] + (d.dt * (h * (F(x - 1, y, z, 0) + F(x, y, z, 0))) + d.windDtX);
                    un[size_t(s.uI(x, y, z))] = uu;
                }
                if (x < s.nx && z < s.nz) {
                    T vv = T(0);
                    if (y > 0) {
                        const T vo = s.v[size_t(s.vI(x, y, z))];
                        vv = y < s.ny ? vo + d.dt * (h * (F(x, y - 1, z, 1) + F(x, y, z, 1))) : vo + d.dt * F(x, y - 1, z, 1);
                        for (const Emitter<T>& e : d.emitters) {
                            if ((y < s.ny && inDisk(e, x, y, z)) || inDisk(e, x, y - 1, z)) vv = e.up;
                        }
                    }
                    vn[size_t(s.vI(x, y, z))] = vv;
                }
                if (x < s.nx && y < s.ny) {
                    T ww = T(0);
                    if (z > 0 && z < s.nz) ww = s.w[size_t(s.wI(x, y, z))] + (d.dt * (h * (F(x, y, z - 1, 2) + F(x, y, z, 2))) + d.windDtZ);
                    wn[size_t(s.wI(x, y, z))] = ww;
                }
            }
        }
    }
    s.u.swap(un);
    s.v.swap(vn);
    s.w.swap(wn);
}

// src/fire_cuda.cu:1185-1199 -- divergence = -(sum of face differences); p = 0.
// With p = 0 on the top face and the multigrid solve, the projection is
// incremental: the previous step's pressure gradient is subtracted from the
// faces first (interior faces, and the top faces with the ghost -p), the
// divergence of those faces becomes the rhs, and the solve finds only the
// increment (from zero), so float carries it without the rounding floor of
// the whole pressure.  The pressure field keeps the previous pressure.
template <class T> void prepareIncrement(Scene<T>& s) {
    const T* pr = s.pressure.data();
    for (int z = 0; z < s.nz; ++z)
        for (int y = 0; y < s.ny; ++y)
            for (int x = 0; x < s.nx; ++x) {
                const T pc = pr[s.sI(x, y, z)];
                if (x > 0) s.u[size_t(s.uI(x, y, z))] -= pc - pr[s.sI(x - 1, y, z)];
                if (y > 0) s.v[size_t(s.vI(x, y, z))] -= pc - pr[s.sI(x, y - 1, z)];
                if (z > 0) s.w[size_t(s.wI(x, y, z))] -= pc - pr[s.sI(x, y, z - 1)];
                if (y == s.ny - 1) s.v[size_t(s.vI(x, s.ny, z))] -= (T(0) - pc) - pc;
            }
    for (int z = 0; z < s.nz; ++z)
        for (int y = 0; y < s.ny; ++y)
            for (int x = 0; x < s.nx; ++x) {
                const T dv = s.u[size_t(s.uI(x + 1, y, z))] - s.u[size_t(s.uI(x, y, z))] + s.v[size_t(s.vI(x, y + 1, z))] -
                             s.v[size_t(s.vI(x, y, z))] + s.w[size_t(s.wI(x, y, z + 1))] - s.w[size_t(s.wI(x, y, z))];
                s.divergence[size_t(s.sI(x, y, z))] = -dv;
            }
    s.delta.clear();
}

template <class T> void divergence(Scene<T>& s) {
    if (s.phys.pressureTop == 1 && s.mgCycles > 0) {
        prepareIncrement(s);
        return;
    }
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < s.nz; ++z) {
        for (int y = 0; y < s.ny; ++y) {
            for (int x = 0; x < s.nx; ++x) {
                const T dv = s.u[size_t(s.uI(x + 1, y, z))] - s.u[size_t(s.uI(x, y, z))] + s.v[size_t(s.vI(x, y + 1, z))] -
                             s.v[size_t(s.vI(x, y, z))] + s.w[size_t(s.wI(x, y, z + 1))] - s.w[size_t(s.wI(x, y, z))];
                s.divergence[size_t(s.sI(x, y, z))] = -dv;
                s.pressure[size_t(s.sI(x, y, z))] = T(0);
            }
        }
    }
}

// src/fire_cuda.cu:1201-1227 -- in-place red-black SOR, Neumann walls (clamped
// neighbours).  The GPU evaluates p + omega * (sum / 6 - p) as two fused
// multiply-adds, fma(omega, fma(sum, 1/6, -p), p) (measured: every cell of a
// B200 half sweep matches this form, none of the unfused ones), so this
// restatement rounds the same way.
template <class T> void sor(Scene<T>& s) {
    T* pr = s.pressure.data();
    const T* div = s.divergence.data();
    const T omega = T(s.omega);
    for (int it = 0; it < s.iterations; ++it) {
        for (int parity = 0; parity < 2; ++parity) {
#pragma omp parallel for collapse(2) schedule(static)
            for (int z = 0; z < s.nz; ++z) {
                for (int y = 0; y < s.ny; ++y) {
                    for (int x = (parity ^ y ^ z) & 1; x < s.nx; x += 2) {
                        const int i = s.sI(x, y, z);
                        const T pL = pr[s.sI(std::max(x - 1, 0), y, z)];
                        const T pR = pr[s.sI(std::min(x + 1, s.nx - 1), y, z)];
                        const T pD = pr[s.sI(x, std::max(y - 1, 0), z)];
                        const T pU = pr[s.sI(x, std::min(y + 1, s.ny - 1), z)];
                        const T pB = pr[s.sI(x, y, std::max(z - 1, 0))];
                        const T pF = pr[s.sI(x, y, std::min(z + 1, s.nz - 1))];
                        const T sum = div[i] + pL + pR + pD + pU + pB + pF;
                        pr[i] = std::fma(omega, std::fma(sum, T(1.0f / 6.0f), -pr[i]), pr[i]);
                    }
                }
            }
        }
    }
}

// src/fire_cuda.cu:1229-1245 -- u -= grad p on interior faces.
template <class T> void subtract(Scene<T>& s) {
    const T* pr = s.pressure.data();
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < s.nz; ++z) {
        for (int y = 0; y < s.ny; ++y) {
            for (int x = 0; x < s.nx; ++x) {
                const T pc = pr[s.sI(x, y, z)];
                if (x > 0) s.u[size_t(s.uI(x, y, z))] -= pc - pr[s.sI(x - 1, y, z)];
                if (y > 0) s.v[size_t(s.vI(x, y, z))] -= pc - pr[s.sI(x, y - 1, z)];
                if (z > 0) s.w[size_t(s.wI(x, y, z))] -= pc - pr[s.sI(x, y, z - 1)];
            }
        }
    }
}

// src/fire_cuda.cu:1293-1317 -- closed walls: u at x = 0, nx; v at y = 0; w at z = 0, nz.
// ---- Multigrid for the Dirichlet top (the product's fire_mg.cu) ----------
// Level equation: sum over axes of w_a (2p - p_a- - p_a+) = rhs; walls and
// floor Neumann (the cell itself), the antisymmetric ghost -p above the top
// row.  Level 0: w = (1, 1, 1).  The next level halves every axis whose extent
// is even and at least 4 and divides its weight by 4; at most 10 levels.
template <class T>
struct Lvl {
    int nx, ny, nz;
    T wx, wy, wz, diag, invDiag;
    int cx, cy, cz;
    int at(int x, int y, int z) const { return (z * ny + y) * nx + x; }
};

template <class T> Lvl<T> withWeights(Lvl<T> L) {
    L.diag = T(2) * (L.wx + L.wy + L.wz);
    L.invDiag = T(1) / L.diag;
    return L;
}

// The level operations (every level in T), as the product's fire_mg.cu.
template <class P, class T> P wsum(const std::vector<P>& p, const std::vector<T>& rhs, const Lvl<T>& L, int x, int y, int z, P self) {
    const int i = L.at(x, y, z);
    const P pL = x > 0 ? p[i - 1] : self;
    const P pR = x < L.nx - 1 ? p[i + 1] : self;
    const P pD = y > 0 ? p[i - L.nx] : self;
    const P pU = y < L.ny - 1 ? p[i + L.nx] : P(0) - self;
    const P pB = z > 0 ? p[i - L.nx * L.ny] : self;
    const P pF = z < L.nz - 1 ? p[i + L.nx * L.ny] : self;
    return P(rhs[i]) + P(L.wx) * (pL + pR) + P(L.wy) * (pD + pU) + P(L.wz) * (pB + pF);
}

template <class P, class T> P resAt(const std::vector<P>& p, const std::vector<T>& rhs, const Lvl<T>& L, int x, int y, int z) {
    const P self = p[L.at(x, y, z)];
    return wsum(p, rhs, L, x, y, z, self) - P(L.diag) * self;
}

template <class P, class T> void mgSmooth(std::vector<P>& p, const std::vector<T>& rhs, const Lvl<T>& L, int sweeps) {
    for (int k = 0; k < sweeps; ++k) {
        for (int colour = 0; colour < 2; ++colour) {
#pragma omp parallel for collapse(2) schedule(static)
            for (int z = 0; z < L.nz; ++z) {
                for (int y = 0; y < L.ny; ++y) {
                    for (int x = (colour + y + z) & 1; x < L.nx; x += 2) {
                        const int i = L.at(x, y, z);
                        p[i] = wsum(p, rhs, L, x, y, z, p[i]) * P(L.invDiag);
                    }
                }
            }
        }
    }
}

// max |r| as the GPU reduces it: |r| in the level's type, rounded to float.
template <class P, class T> float residualMax(const std::vector<P>& p, const std::vector<T>& rhs, const Lvl<T>& L) {
    float m = 0.0f;
    for (int z = 0; z < L.nz; ++z)
        for (int y = 0; y < L.ny; ++y)
            for (int x = 0; x < L.nx; ++x) m = std::fmax(m, float(std::fabs(double(resAt(p, rhs, L, x, y, z)))));
    return m;
}

// Coarse rhs at (X, Y, Z): the mean residual of the covered fine cells in the fine level's type.
template <class P, class T>
T restrictMean(const std::vector<P>& pf, const std::vector<T>& rf, const Lvl<T>& F, const Lvl<T>& C, int X, int Y, int Z) {
    const int x0 = C.cx ? 2 * X : X, y0 = C.cy ? 2 * Y : Y, z0 = C.cz ? 2 * Z : Z;
    const P half = P(0.5f);
    P az[2] = {P(0), P(0)};
    for (int dz = 0; dz <= C.cz; ++dz) {
        P ay[2] = {P(0), P(0)};
        for (int dy = 0; dy <= C.cy; ++dy) {
            const P a = resAt(pf, rf, F, x0, y0 + dy, z0 + dz);
            ay[dy] = C.cx ? half * (a + resAt(pf, rf, F, x0 + 1, y0 + dy, z0 + dz)) : a;
        }
        az[dz] = C.cy ? half * (ay[0] + ay[1]) : ay[0];
    }
    return T(C.cz ? half * (az[0] + az[1]) : az[0]);
}

// p += the coarse correction (evaluated in T) interpolated along the halved axes.
template <class P, class T> void prolong(std::vector<P>& pf, const std::vector<T>& pc, const Lvl<T>& F, const Lvl<T>& C) {
    const T ux = C.cx ? T(0.75f) : T(1), vx = C.cx ? T(0.25f) : T(0);
    const T uy = C.cy ? T(0.75f) : T(1), vy = C.cy ? T(0.25f) : T(0);
    const T uz = C.cz ? T(0.75f) : T(1), vz = C.cz ? T(0.25f) : T(0);
    for (int z = 0; z < F.nz; ++z)
        for (int y = 0; y < F.ny; ++y)
            for (int x = 0; x < F.nx; ++x) {
                const int X0 = C.cx ? x >> 1 : x, Y0 = C.cy ? y >> 1 : y, Z0 = C.cz ? z >> 1 : z;
                const int X1 = !C.cx ? X0 : ((x & 1) ? std::min(X0 + 1, C.nx - 1) : std::max(X0 - 1, 0));
                const int Y1 = !C.cy ? Y0 : ((y & 1) ? std::min(Y0 + 1, C.ny - 1) : std::max(Y0 - 1, 0));
                const int Z1 = !C.cz ? Z0 : ((z & 1) ? std::min(Z0 + 1, C.nz - 1) : std::max(Z0 - 1, 0));
                const T a0 = ux * pc[C.at(X0, Y0, Z0)] + vx * pc[C.at(X1, Y0, Z0)];
                const T a1 = ux * pc[C.at(X0, Y1, Z0)] + vx * pc[C.at(X1, Y1, Z0)];
                const T a2 = ux * pc[C.at(X0, Y0, Z1)] + vx * pc[C.at(X1, Y0, Z1)];
                const T a3 = ux * pc[C.at(X0, Y1, Z1)] + vx * pc[C.at(X1, Y1, Z1)];
                const T b0 = uy * a0 + vy * a1, b1 = uy * a2 + vy * a3;
                const int i = F.at(x, y, z);
                pf[i] = pf[i] + P(uz * b0 + vz * b1);
            }
}

template <class T> void multigrid(Scene<T>& s) {
    std::vector<Lvl<T>> lv{withWeights(Lvl<T>{s.nx, s.ny, s.nz, T(1), T(1), T(1), T(0), T(0), 0, 0, 0})};
    while (lv.size() < 10) {
        const Lvl<T> b = lv.back();
        const int cx = b.nx % 2 == 0 && b.nx >= 4, cy = b.ny % 2 == 0 && b.ny >= 4, cz = b.nz % 2 == 0 && b.nz >= 4;
        if (!cx && !cy && !cz) break;
        lv.push_back(withWeights(Lvl<T>{cx ? b.nx / 2 : b.nx, cy ? b.ny / 2 : b.ny, cz ? b.nz / 2 : b.nz,
                                        cx ? b.wx * T(0.25f) : b.wx, cy ? b.wy * T(0.25f) : b.wy, cz ? b.wz * T(0.25f) : b.wz,
                                        T(0), T(0), cx, cy, cz}));
    }
    const int n = int(lv.size());
    std::vector<std::vector<T>> P(n), R(n);
    for (int l = 1; l < n; ++l) {
        P[l].assign(size_t(lv[l].nx) * lv[l].ny * lv[l].nz, T(0));
        R[l].assign(P[l].size(), T(0));
    }
    // Level 0: the pressure increment, from zero; rhs the divergence array
    // (the divergence after the previous pressure's gradient was subtracted).
    std::vector<T> p0(size_t(s.cells()), T(0));
    const std::vector<T>& r0 = s.divergence;
    s.mgCyclesRun = 0;
    s.mgMaxResidual = -1.0f;
    for (int c = 0; c < s.mgCycles; ++c) {
        for (int l = 0; l + 1 < n; ++l) {
            const Lvl<T>& F = lv[l];
            const Lvl<T>& C = lv[l + 1];
            if (l == 0) {
                mgSmooth(p0, r0, F, s.mgPre);
            } else {
                mgSmooth(P[l], R[l], F, s.mgPre);
            }
            for (int Z = 0; Z < C.nz; ++Z)
                for (int Y = 0; Y < C.ny; ++Y)
                    for (int X = 0; X < C.nx; ++X) {
                        R[l + 1][C.at(X, Y, Z)] = l == 0 ? restrictMean(p0, r0, F, C, X, Y, Z) : restrictMean(P[l], R[l], F, C, X, Y, Z);
                        P[l + 1][C.at(X, Y, Z)] = T(0);
                    }
        }
        if (n == 1) {
            mgSmooth(p0, r0, lv[0], 32);
        } else {
            mgSmooth(P[n - 1], R[n - 1], lv[n - 1], 32);
        }
        for (int l = n - 2; l >= 0; --l) {
            if (l == 0) {
                prolong(p0, P[1], lv[0], lv[1]);
                mgSmooth(p0, r0, lv[0], s.mgPost);
            } else {
                prolong(P[l], P[l + 1], lv[l], lv[l + 1]);
                mgSmooth(P[l], R[l], lv[l], s.mgPost);
            }
        }
        ++s.mgCyclesRun;
        if (s.mgTolerance > 0.0f) {
            s.mgMaxResidual = residualMax(p0, r0, lv[0]);
            if (s.mgMaxResidual <= s.mgTolerance) break;
        }
    }
    // The new pressure is the previous one plus the increment; the gradient
    // subtraction takes the increment.
    for (size_t i = 0; i < p0.size(); ++i) s.pressure[i] = s.pressure[i] + p0[i];
    s.delta = std::move(p0);
}

// The gradient subtraction of the multigrid's pressure increment (Dirichlet
// top): interior faces, and the top faces with the antisymmetric ghost -delta.
template <class T> void subtractIncrement(Scene<T>& s) {
    const std::vector<T>& pr = s.delta;
    for (int z = 0; z < s.nz; ++z)
        for (int y = 0; y < s.ny; ++y)
            for (int x = 0; x < s.nx; ++x) {
                const T pc = pr[size_t(s.sI(x, y, z))];
                if (x > 0) s.u[size_t(s.uI(x, y, z))] -= pc - pr[size_t(s.sI(x - 1, y, z))];
                if (y > 0) s.v[size_t(s.vI(x, y, z))] -= pc - pr[size_t(s.sI(x, y - 1, z))];
                if (z > 0) s.w[size_t(s.wI(x, y, z))] -= pc - pr[size_t(s.sI(x, y, z - 1))];
                if (y == s.ny - 1) s.v[size_t(s.vI(x, s.ny, z))] -= (T(0) - pc) - pc;
            }
}

template <class T> void walls(Scene<T>& s) {
    for (int z = 0; z < s.nz; ++z) {
        for (int y = 0; y < s.ny; ++y) {
            s.u[size_t(s.uI(0, y, z))] = T(0);
            s.u[size_t(s.uI(s.nx, y, z))] = T(0);
        }
    }
    for (int z = 0; z < s.nz; ++z) {
        for (int x = 0; x < s.nx; ++x) s.v[size_t(s.vI(x, 0, z))] = T(0);
    }
    for (int y = 0; y < s.ny; ++y) {
        for (int x = 0; x < s.nx; ++x) {
            s.w[size_t(s.wI(x, y, 0))] = T(0);
            s.w[size_t(s.wI(x, y, s.nz))] = T(0);
        }
    }
}

template <class T> T sigmaAt(const Scene<T>& s, const Derived<T>& d, T x, T y, T z) {
    const Vec3<T> a = scalarsAt(s, x, y, z);
    return d.extinction * a.z + d.fuelExtinction * a.y;
}

// Stage LIGHT_BUILD: transmittance to the point light from each 2x2x2 block centre.
template <class T> void transmittance(Scene<T>& s, const Derived<T>& d) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int lz = 0; lz < s.lz; ++lz) {
        for (int ly = 0; ly < s.ly; ++ly) {
            for (int lx = 0; lx < s.lx; ++lx) {
                const T px = T(2) * T(lx) + T(1), py = T(2) * T(ly) + T(1), pz = T(2) * T(lz) + T(1);
                const T dx = d.light.x - px, dy = d.light.y - py, dz = d.light.z - pz;
                const T dist = std::sqrt(dx * dx + dy * dy + dz * dz);
                T t = T(1);
                if (dist > T(1e-6f)) {
                    const T rx = dx / dist, ry = dy / dist, rz = dz / dist;
                    T seg = dist;
                    if (rx > T(0)) seg = std::fmin(seg, (T(s.nx) - px) / rx);
                    if (rx < T(0)) seg = std::fmin(seg, (T(0) - px) / rx);
                    if (ry > T(0)) seg = std::fmin(seg, (T(s.ny) - py) / ry);
                    if (ry < T(0)) seg = std::fmin(seg, (T(0) - py) / ry);
                    if (rz > T(0)) seg = std::fmin(seg, (T(s.nz) - pz) / rz);
                    if (rz < T(0)) seg = std::fmin(seg, (T(0) - pz) / rz);
                    seg = std::fmax(seg, T(0));
                    const T ds = seg / T(d.lightSamples);
                    T tau = T(0);
                    for (int k = 0; k < d.lightSamples; ++k) {
                        const T at = (T(k) + T(0.5f)) * ds;
                        tau = tau + sigmaAt(s, d, px + rx * at, py + ry * at, pz + rz * at) * ds;
                    }
                    t = std::exp(-tau);
                }
                s.transmittance[size_t((lz * s.ly + ly) * s.lx + lx)] = t;
            }
        }
    }
}

// Stage RENDER: one camera ray per pixel through the grid box.
template <class T> void raymarch(Scene<T>& s, const Derived<T>& d) {
#pragma omp parallel for schedule(static)
    for (int py = 0; py < s.H; ++py) {
        for (int px = 0; px < s.W; ++px) {
            const T sx = (T(2) * (T(px) + T(0.5f)) / T(s.W) - T(1)) * d.tanHalf * d.aspect;
            const T sy = (T(1) - T(2) * (T(py) + T(0.5f)) / T(s.H)) * d.tanHalf;
            T dx = d.fwd.x + d.right.x * sx + d.up.x * sy;
            T dy = d.fwd.y + d.right.y * sx + d.up.y * sy;
            T dz = d.fwd.z + d.right.z * sx + d.up.z * sy;
            const T len = std::sqrt(dx * dx + dy * dy + dz * dz);
            dx = dx / len;
            dy = dy / len;
            dz = dz / len;
            T t0 = T(0), t1 = T(3.0e38f);
            bool hit = true;
            const T eye[3] = {d.eye.x, d.eye.y, d.eye.z};
            const T dir[3] = {dx, dy, dz};
            const T hiB[3] = {T(s.nx), T(s.ny), T(s.nz)};
            for (int k = 0; k < 3; ++k) {
                if (dir[k] == T(0)) {
                    if (eye[k] < T(0) || eye[k] > hiB[k]) hit = false;
                } else {
                    const T ta = (T(0) - eye[k]) / dir[k];
                    const T tb = (hiB[k] - eye[k]) / dir[k];
                    t0 = std::fmax(t0, std::fmin(ta, tb));
                    t1 = std::fmin(t1, std::fmax(ta, tb));
                }
            }
            T r = T(0), g = T(0), b = T(0), view = T(1);
            if (hit && t1 > t0) {
                const T ds = (t1 - t0) / T(d.primary);
                for (int k = 0; k < d.primary; ++k) {
                    const T at = t0 + (T(k) + T(0.5f)) * ds;
                    const T qx = d.eye.x + dx * at, qy = d.eye.y + dy * at, qz = d.eye.z + dz * at;
                    const Vec3<T> a = scalarsAt(s, qx, qy, qz);
                    const T sigma = d.extinction * a.z + d.fuelExtinction * a.y;
                    const T alpha = T(1) - std::exp(-(sigma * ds));
                    const T lt = trilinear(s.transmittance, s.lx, s.ly, s.lz, qx * T(0.5f) - T(0.5f), qy * T(0.5f) - T(0.5f),
                                           qz * T(0.5f) - T(0.5f));
                    const T scatter = d.albedo * d.lightIntensity * lt * alpha;
                    const T heat = std::fmax(a.x, T(0));
                    const T hh = heat / (heat + T(1));
                    const T e = d.emission * heat * ds;
                    r = r + view * (scatter + e);
                    g = g + view * (scatter + e * (T(0.35f) + T(0.45f) * hh));
                    b = b + view * (scatter + e * (T(0.08f) + T(0.50f) * hh * hh));
                    view = view * (T(1) - alpha);
                }
            }
            T* o = &s.hdr[size_t(py * s.W + px) * 4];
            o[0] = r + view * T(0.015f);
            o[1] = g + view * T(0.016f);
            o[2] = b + view * T(0.020f);
            o[3] = T(1) - view;
        }
    }
}

template <class T> int runStages(Scene<T>& s, int first, int last) {
    if (first < 0 || last > FIRE_STAGE_RESET || first > last) return setError("stage range out of order");
    for (int st = first; st <= last; ++st) {
        const Derived<T> d = s.derive();
        switch (st) {
            case FIRE_STAGE_ADVECT_VELOCITY: advectVelocity(s); break;
            case FIRE_STAGE_ADVECT_REACT: advectScalars(s, d); break;
            case FIRE_STAGE_FORCE: forces(s, d); break;
            case FIRE_STAGE_DIVERGENCE: divergence(s); break;
            case FIRE_STAGE_PRESSURE_SOR:
                if (s.phys.pressureTop == 1) {
                    multigrid(s);
                } else {
                    sor(s);
                }
                break;
            case FIRE_STAGE_SUBTRACT:
                if (s.phys.pressureTop == 1 && s.delta.size() == size_t(s.cells())) {
                    subtractIncrement(s);
                } else {
                    subtract(s);
                    if (s.phys.pressureTop == 1) {
                        // No multigrid pressure: the top faces from the float field, ghost -p.
                        for (int z = 0; z < s.nz; ++z)
                            for (int x = 0; x < s.nx; ++x) {
                                T& v = s.v[size_t(s.vI(x, s.ny, z))];
                                const T top = s.pressure[size_t(s.sI(x, s.ny - 1, z))];
                                v = v - ((T(0) - top) - top);
                            }
                    }
                }
                if (last >= FIRE_STAGE_WALL_BOUNDARY) {
                    walls(s);
                    ++st;
                }
                break;
            case FIRE_STAGE_WALL_BOUNDARY: walls(s); break;
            case FIRE_STAGE_LIGHT_BUILD: transmittance(s, d); break;
            case FIRE_STAGE_RENDER: raymarch(s, d); break;
            case FIRE_STAGE_RESET: {
                const FirePhysicsParams keep = s.phys;
                s.resize();
                s.phys = keep;
                break;
            }
            default: break;
        }
    }
    return 0;
}

struct Handle {
    int precision;
    Scene<float> f;
    Scene<double> d;
};

template <class T> std::vector<T>* fieldOf(Scene<T>& s, int field) {
    switch (field) {
        case FIRE_FIELD_HEAT: return &s.heat;
        case FIRE_FIELD_FUEL: return &s.fuel;
        case FIRE_FIELD_SOOT: return &s.soot;
        case FIRE_FIELD_PRESSURE: return &s.pressure;
        case FIRE_FIELD_DIVERGENCE: return &s.divergence;
        case FIRE_FIELD_U: return &s.u;
        case FIRE_FIELD_V: return &s.v;
        case FIRE_FIELD_W: return &s.w;
        case FIRE_FIELD_HDR: return &s.hdr;
        case FIRE_FIELD_CONFIG_TRANSMITTANCE: return &s.transmittance;
        default: return nullptr;
    }
}

template <class T> void init(Scene<T>& s, int W, int H, int nx, int ny, int nz) {
    s.nx = nx;
    s.ny = ny;
    s.nz = nz;
    s.lx = (nx + 1) / 2;
    s.ly = (ny + 1) / 2;
    s.lz = (nz + 1) / 2;
    s.W = W;
    s.H = H;
    std::memset(&s.phys, 0, sizeof(s.phys));
    s.resize();
}

#define CFG_DISPATCH(h, expr)                          \
    do {                                               \
        Handle* hd = static_cast<Handle*>(h);          \
        if (hd->precision == 0) {                      \
            auto& s = hd->f;                           \
            expr;                                      \
        } else {                                       \
            auto& s = hd->d;                           \
            expr;                                      \
        }                                              \
    } while (0)

}  // namespace

extern "C" {

void* cfg_oracle_create(int precision, int frameW, int frameH, int nx, int ny, int nz) {
    if (nx < 2 || ny < 2 || nz < 2 || frameW < 1 || frameH < 1 || (precision != 0 && precision != 1)) {
        setError("invalid dimensions or precision");
        return nullptr;
    }
    Handle* h = new Handle;
    h->precision = precision;
    if (precision == 0) {
        init(h->f, frameW, frameH, nx, ny, nz);
    } else {
        init(h->d, frameW, frameH, nx, ny, nz);
    }
    return h;
}

void cfg_oracle_destroy(void* o) { delete static_cast<Handle*>(o); }

int cfg_oracle_set_physics(void* o, const FirePhysicsParams* params) {
    if (params == nullptr) return setError("null parameters");
    if (params->emitterCount < 0 || params->emitterCount > FIRE_MAX_EMITTERS || params->primarySamples < 1 ||
        params->lightSamples < 1 || !(params->noisePeriod > 0.0f)) {
        return setError("parameters out of range");
    }
    CFG_DISPATCH(o, s.phys = *params);
    return 0;
}

void cfg_oracle_set_pressure_solver(void* o, int iterations, float omega) { CFG_DISPATCH(o, (s.iterations = iterations, s.omega = omega)); }

void cfg_oracle_set_multigrid(void* o, int maxCycles, int preSmooth, int postSmooth, float tolerance) {
    CFG_DISPATCH(o, (s.mgCycles = maxCycles, s.mgPre = preSmooth, s.mgPost = postSmooth, s.mgTolerance = tolerance));
}

void cfg_oracle_multigrid_stats(void* o, int* cycles, float* maxResidual) {
    CFG_DISPATCH(o, (*cycles = s.mgCyclesRun, *maxResidual = s.mgMaxResidual));
}

int cfg_oracle_set_field(void* o, int field, const void* host, long long bytes) {
    int rc = 0;
    CFG_DISPATCH(o, {
        auto* f = fieldOf(s, field);
        if (f == nullptr) {
            rc = setError("unknown field");
        } else if (bytes != static_cast<long long>(f->size() * sizeof(float))) {
            rc = setError("field size mismatch");
        } else {
            const float* in = static_cast<const float*>(host);
            for (size_t i = 0; i < f->size(); ++i) (*f)[i] = in[i];
            if (field == FIRE_FIELD_PRESSURE) s.delta.clear();
        }
    });
    return rc;
}

int cfg_oracle_get_field(void* o, int field, void* host, long long bytes) {
    int rc = 0;
    CFG_DISPATCH(o, {
        auto* f = fieldOf(s, field);
        if (f == nullptr) {
            rc = setError("unknown field");
        } else if (bytes != static_cast<long long>(f->size() * sizeof(float))) {
            rc = setError("field size mismatch");
        } else {
            float* out = static_cast<float*>(host);
            for (size_t i = 0; i < f->size(); ++i) out[i] = static_cast<float>((*f)[i]);
        }
    });
    return rc;
}

int cfg_oracle_get_field_f64(void* o, int field, double* host, long long count) {
    int rc = 0;
    CFG_DISPATCH(o, {
        auto* f = fieldOf(s, field);
        if (f == nullptr) {
            rc = setError("unknown field");
        } else if (count != static_cast<long long>(f->size())) {
            rc = setError("field size mismatch");
        } else {
            for (size_t i = 0; i < f->size(); ++i) host[i] = static_cast<double>((*f)[i]);
        }
    });
    return rc;
}

int cfg_oracle_stages(void* o, int first, int last) {
    int rc = 0;
    CFG_DISPATCH(o, rc = runStages(s, first, last));
    return rc;
}

int cfg_oracle_step(void* o, int render) {
    int rc = 0;
    CFG_DISPATCH(o, {
        rc = runStages(s, FIRE_STAGE_ADVECT_VELOCITY, FIRE_STAGE_WALL_BOUNDARY);
        if (rc == 0 && render) rc = runStages(s, FIRE_STAGE_LIGHT_BUILD, FIRE_STAGE_RENDER);
    });
    return rc;
}

unsigned long long cfg_oracle_step_count(void* o) {
    unsigned long long n = 0;
    CFG_DISPATCH(o, n = s.step);
    return n;
}

const char* cfg_oracle_last_error(void) { return g_error; }

}  // extern "C"
