// fire_config.cu -- kernels of the config physics (FirePhysicsParams.mode 1).
//
// A plain T/F/S smoke-and-fire model on the same MAC grid and projection as
// the reference physics: semi-Lagrangian advection in cell units, first-order
// burn, seeded disk emitters, vorticity confinement, curl of seeded value
// noise, wind, and a point-light transmittance render.  The reference has
// none of these (its model is the ten-scalar fuel bed of src/fire_cuda.cu);
// the equations are stated in include/fire_ext.h.  The divergence, the SOR
// solve and the gradient subtraction are the reference-physics kernels.
//
// This file is compiled with -fmad=false: every product and sum rounds as
// written, and the only fused multiply-adds are the explicit ones of the
// interpolations (lerp1), so a CPU restatement that evaluates the same
// expressions in the same order in IEEE float, with std::fma where the
// kernels fuse, gives the same bits for the whole simulation step (only +, -,
// *, /, fma, sqrt, floor, min/max and integer hashing occur there).
// The render uses expf and is compared within a tolerance.
//
// Memory: records are read and written through the storage accessors
// (ldv/stv), so the FP16 and BF16 storage builds apply unchanged.  Only record
// a = (heat, fuel, oxygen, soot) is advanced; b and c are not touched.
#include "fire_kernels.h"

namespace firesim {

namespace {

__device__ __forceinline__ int faceIndex(int x, int y, int z, int mx, int my) { return (z * my + y) * mx + x; }

// Clamped trilinear sample of a grid of mx*my*mz values (x fastest) at index-space
// position q: q clamped to [0, m-1] per axis, i0 = (int)q, i1 = min(i0 + 1, m - 1),
// t = q - i0; lerp(a, b, t) = fma(t, b - a, a), along x, then y, then z.
struct Corners {
    int x0, x1, y0, y1, z0, z1;
    float tx, ty, tz;
};

__device__ __forceinline__ void axisOf(float q, int m, int& i0, int& i1, float& t) {
    q = fminf(fmaxf(q, 0.0f), static_cast<float>(m - 1));
    i0 = static_cast<int>(q);
    i1 = min(i0 + 1, m - 1);
    t = q - static_cast<float>(i0);
}

__device__ __forceinline__ Corners cornersAt(float qx, float qy, float qz, int mx, int my, int mz) {
    Corners c;
    axisOf(qx, mx, c.x0, c.x1, c.tx);
    axisOf(qy, my, c.y0, c.y1, c.ty);
    axisOf(qz, mz, c.z0, c.z1, c.tz);
    return c;
}

// One fused multiply-add (explicit, as the file is built without contraction).
__device__ __forceinline__ float lerp1(float a, float b, float t) { return __fmaf_rn(t, b - a, a); }

__device__ __forceinline__ float4 lerp4(float4 a, float4 b, float t) {
    return make_float4(lerp1(a.x, b.x, t), lerp1(a.y, b.y, t), lerp1(a.z, b.z, t), lerp1(a.w, b.w, t));
}

// The eight corner loads address one base cell plus fixed offsets (0 or 1
// cell along each axis, 0 where the clamp merges the corners), which saves
// the index arithmetic of a full (z * my + y) * mx + x per corner.
template <typename P>
__device__ __forceinline__ float trilinear1(const P* f, const Corners& c, int mx, int my) {
    const P* b = f + faceIndex(c.x0, c.y0, c.z0, mx, my);
    const int dx = c.x1 - c.x0, dy = (c.y1 - c.y0) * mx, dz = (c.z1 - c.z0) * mx * my;
    const float a00 = lerp1(ldv(b), ldv(b + dx), c.tx);
    const float a10 = lerp1(ldv(b + dy), ldv(b + dy + dx), c.tx);
    const float a01 = lerp1(ldv(b + dz), ldv(b + dz + dx), c.tx);
    const float a11 = lerp1(ldv(b + dz + dy), ldv(b + dz + dy + dx), c.tx);
    const float b0 = lerp1(a00, a10, c.ty);
    const float b1 = lerp1(a01, a11, c.ty);
    return lerp1(b0, b1, c.tz);
}

__device__ __forceinline__ float4 trilinearRec(const Rec4* f, const Corners& c, int mx, int my) {
    const Rec4* b = f + faceIndex(c.x0, c.y0, c.z0, mx, my);
    const int dx = c.x1 - c.x0, dy = (c.y1 - c.y0) * mx, dz = (c.z1 - c.z0) * mx * my;
    const float4 a00 = lerp4(ldv(b), ldv(b + dx), c.tx);
    const float4 a10 = lerp4(ldv(b + dy), ldv(b + dy + dx), c.tx);
    const float4 a01 = lerp4(ldv(b + dz), ldv(b + dz + dx), c.tx);
    const float4 a11 = lerp4(ldv(b + dz + dy), ldv(b + dz + dy + dx), c.tx);
    const float4 b0 = lerp4(a00, a10, c.ty);
    const float4 b1 = lerp4(a01, a11, c.ty);
    return lerp4(b0, b1, c.tz);
}

// Velocity (cells per step) at the faces and cell centres the advection
// traces back from.  u lives at (i, j+.5, k+.5), v at (i+.5, j, k+.5), w at
// (i+.5, j+.5, k); the velocity at a point is the clamped trilinear sample of
// each face grid (x, then y, then z).  At these points one or two of each
// sample's weights are 0, and lerp(a, b, 0) = a, so those axes are skipped and
// the remaining lerps are taken in the same order: for finite velocities the
// values equal the full trilinear samples, except possibly in the sign of a
// zero, which the callers (position - velocity, position >= 0) cannot see.
__device__ __forceinline__ float faceAt(const FaceT* f, int x, int y, int z, int mx, int my) { return ldv(f + faceIndex(x, y, z, mx, my)); }

// At the u face (x, y + .5, z + .5).
__device__ __forceinline__ float3 velocityAtUFace(const Velocity& vel, const ConfigParams& p, int x, int y, int z) {
    int x0, x1;
    float tx;
    axisOf(static_cast<float>(x) - 0.5f, p.nx, x0, x1, tx);
    // v at y and y + 1 (weight 1/2), w at z and z + 1 (weight 1/2), x0 and x1 along x.
    const int dx = x1 - x0;
    const FaceT* vb = vel.v + faceIndex(x0, y, z, p.nx, p.ny + 1);
    const FaceT* wb = vel.w + faceIndex(x0, y, z, p.nx, p.ny);
    const int vy = p.nx, wz = p.nx * p.ny;
    const float v = lerp1(lerp1(ldv(vb), ldv(vb + dx), tx), lerp1(ldv(vb + vy), ldv(vb + vy + dx), tx), 0.5f);
    const float w = lerp1(lerp1(ldv(wb), ldv(wb + dx), tx), lerp1(ldv(wb + wz), ldv(wb + wz + dx), tx), 0.5f);
    return make_float3(faceAt(vel.u, x, y, z, p.nx + 1, p.ny), v, w);
}

// At the v face (x + .5, y, z + .5).
__device__ __forceinline__ float3 velocityAtVFace(const Velocity& vel, const ConfigParams& p, int x, int y, int z) {
    int y0, y1;
    float ty;
    axisOf(static_cast<float>(y) - 0.5f, p.ny, y0, y1, ty);
    const FaceT* ub = vel.u + faceIndex(x, y0, z, p.nx + 1, p.ny);
    const FaceT* wb = vel.w + faceIndex(x, y0, z, p.nx, p.ny);
    const int du = (y1 - y0) * (p.nx + 1), dw = (y1 - y0) * p.nx, wz = p.nx * p.ny;
    const float u = lerp1(lerp1(ldv(ub), ldv(ub + 1), 0.5f), lerp1(ldv(ub + du), ldv(ub + du + 1), 0.5f), ty);
    const float w = lerp1(lerp1(ldv(wb), ldv(wb + dw), ty), lerp1(ldv(wb + wz), ldv(wb + wz + dw), ty), 0.5f);
    return make_float3(u, faceAt(vel.v, x, y, z, p.nx, p.ny + 1), w);
}

// At the w face (x + .5, y + .5, z).
__device__ __forceinline__ float3 velocityAtWFace(const Velocity& vel, const ConfigParams& p, int x, int y, int z) {
    int z0, z1;
    float tz;
    axisOf(static_cast<float>(z) - 0.5f, p.nz, z0, z1, tz);
    const FaceT* ub = vel.u + faceIndex(x, y, z0, p.nx + 1, p.ny);
    const FaceT* vb = vel.v + faceIndex(x, y, z0, p.nx, p.ny + 1);
    const int du = (z1 - z0) * (p.nx + 1) * p.ny, dv = (z1 - z0) * p.nx * (p.ny + 1), vy = p.nx;
    const float u = lerp1(lerp1(ldv(ub), ldv(ub + 1), 0.5f), lerp1(ldv(ub + du), ldv(ub + du + 1), 0.5f), tz);
    const float v = lerp1(lerp1(ldv(vb), ldv(vb + vy), 0.5f), lerp1(ldv(vb + dv), ldv(vb + dv + vy), 0.5f), tz);
    return make_float3(u, v, faceAt(vel.w, x, y, z, p.nx, p.ny));
}

// At the cell centre (x + .5, y + .5, z + .5): the mean of the two faces along each axis.
__device__ __forceinline__ float3 velocityAtCentre(const Velocity& vel, const ConfigParams& p, int x, int y, int z) {
    const FaceT* ub = vel.u + faceIndex(x, y, z, p.nx + 1, p.ny);
    const FaceT* vb = vel.v + faceIndex(x, y, z, p.nx, p.ny + 1);
    const FaceT* wb = vel.w + faceIndex(x, y, z, p.nx, p.ny);
    return make_float3(lerp1(ldv(ub), ldv(ub + 1), 0.5f), lerp1(ldv(vb), ldv(vb + p.nx), 0.5f), lerp1(ldv(wb), ldv(wb + p.nx * p.ny), 0.5f));
}

__device__ __forceinline__ float4 recordAt(const Rec4* a, const ConfigParams& p, float x, float y, float z) {
    return trilinearRec(a, cornersAt(x - 0.5f, y - 0.5f, z - 0.5f, p.nx, p.ny, p.nz), p.nx, p.ny);
}

__device__ __forceinline__ bool inDisk(const ConfigEmitter& e, int x, int y, int z) {
    if (y != e.row) return false;
    const float dx = static_cast<float>(x) - e.cx;
    const float dz = static_cast<float>(z) - e.cz;
    return dx * dx + dz * dz <= e.r2;
}

// psi_c at position (x, y, z) (cell units) and its gradient: value noise on a
// lattice of period 1/invPeriod cells, cubic Hermite weights s = f^2 (3 - 2f),
// ds/df = 6 f (1 - f).
__device__ __forceinline__ float3 noiseGradient(const ConfigParams& p, int comp, float x, float y, float z) {
    const float qx = x * p.invPeriod, qy = y * p.invPeriod, qz = z * p.invPeriod;
    const float fx0 = floorf(qx), fy0 = floorf(qy), fz0 = floorf(qz);
    const int ix = static_cast<int>(fx0), iy = static_cast<int>(fy0), iz = static_cast<int>(fz0);
    const float fx = qx - fx0, fy = qy - fy0, fz = qz - fz0;
    const float sx = fx * fx * (3.0f - 2.0f * fx), sy = fy * fy * (3.0f - 2.0f * fy), sz = fz * fz * (3.0f - 2.0f * fz);
    const float dsx = 6.0f * fx * (1.0f - fx), dsy = 6.0f * fy * (1.0f - fy), dsz = 6.0f * fz * (1.0f - fz);
    const float c000 = latticeValue(p.noiseSeed, comp, ix, iy, iz), c100 = latticeValue(p.noiseSeed, comp, ix + 1, iy, iz);
    const float c010 = latticeValue(p.noiseSeed, comp, ix, iy + 1, iz), c110 = latticeValue(p.noiseSeed, comp, ix + 1, iy + 1, iz);
    const float c001 = latticeValue(p.noiseSeed, comp, ix, iy, iz + 1), c101 = latticeValue(p.noiseSeed, comp, ix + 1, iy, iz + 1);
    const float c011 = latticeValue(p.noiseSeed, comp, ix, iy + 1, iz + 1), c111 = latticeValue(p.noiseSeed, comp, ix + 1, iy + 1, iz + 1);
    const float a00 = lerp1(c000, c100, sx), a10 = lerp1(c010, c110, sx), a01 = lerp1(c001, c101, sx), a11 = lerp1(c011, c111, sx);
    const float b0 = lerp1(a00, a10, sy), b1 = lerp1(a01, a11, sy);
    const float e0 = lerp1(c100 - c000, c110 - c010, sy), e1 = lerp1(c101 - c001, c111 - c011, sy);
    const float gx = dsx * lerp1(e0, e1, sz);
    const float gy = dsy * lerp1(a10 - a00, a11 - a01, sz);
    const float gz = dsz * (b1 - b0);
    return make_float3(gx * p.invPeriod, gy * p.invPeriod, gz * p.invPeriod);
}

__device__ __forceinline__ float cellCentred(const FaceT* f, int lo, int hi) { return 0.5f * (ldv(f + lo) + ldv(f + hi)); }

}  // namespace

// Each thread owns u(x,y,z), v(x,y,z) and w(x,y,z) where they exist and
// writes each as the face grid sampled at its one-step backtrace.
__device__ __forceinline__ void cfgAdvectVelocityAt(FaceT* __restrict__ uOut, FaceT* __restrict__ vOut, FaceT* __restrict__ wOut,
                                                         const Velocity& vel, const ConfigParams& p, int x, int y, int z) {
    const float fx = static_cast<float>(x), fy = static_cast<float>(y), fz = static_cast<float>(z);
    if (y < p.ny && z < p.nz) {
        const float px = fx, py = fy + 0.5f, pz = fz + 0.5f;
        const float3 d = velocityAtUFace(vel, p, x, y, z);
        const float bx = px - d.x, by = py - d.y, bz = pz - d.z;
        stv(uOut + faceIndex(x, y, z, p.nx + 1, p.ny),
            trilinear1(vel.u, cornersAt(bx, by - 0.5f, bz - 0.5f, p.nx + 1, p.ny, p.nz), p.nx + 1, p.ny));
    }
    if (x < p.nx && z < p.nz) {
        const float px = fx + 0.5f, py = fy, pz = fz + 0.5f;
        const float3 d = velocityAtVFace(vel, p, x, y, z);
        const float bx = px - d.x, by = py - d.y, bz = pz - d.z;
        stv(vOut + faceIndex(x, y, z, p.nx, p.ny + 1), trilinear1(vel.v, cornersAt(bx - 0.5f, by, bz - 0.5f, p.nx, p.ny + 1, p.nz), p.nx, p.ny + 1));
    }
    if (x < p.nx && y < p.ny) {
        const float px = fx + 0.5f, py = fy + 0.5f, pz = fz;
        const float3 d = velocityAtWFace(vel, p, x, y, z);
        const float bx = px - d.x, by = py - d.y, bz = pz - d.z;
        stv(wOut + faceIndex(x, y, z, p.nx, p.ny), trilinear1(vel.w, cornersAt(bx - 0.5f, by - 0.5f, bz, p.nx, p.ny, p.nz + 1), p.nx, p.ny));
    }
}

// The single-scene face kernels run on the cell grid: the thread of cell
// (x, y, z) owns its u, v and w faces and, as the last cell of its row,
// column or plane, the far wall's face beside it (x = nx, y = ny, z = nz).
// A face grid of nx + 1 columns would leave a nearly empty block per row.
template <class Face>
__device__ __forceinline__ void facesOfCell(const ConfigParams& p, int x, int y, int z, Face face) {
    face(x, y, z);
    if (x == p.nx - 1) face(p.nx, y, z);
    if (y == p.ny - 1) face(x, p.ny, z);
    if (z == p.nz - 1) face(x, y, p.nz);
}

__global__ void __launch_bounds__(128) cfgAdvectVelocity(FaceT* __restrict__ uOut, FaceT* __restrict__ vOut, FaceT* __restrict__ wOut,
                                                         Velocity vel, ConfigParams p) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= p.nx) return;
    facesOfCell(p, x, blockIdx.y, blockIdx.z, [&](int fx, int fy, int fz) { cfgAdvectVelocityAt(uOut, vOut, wOut, vel, p, fx, fy, fz); });
}

// Backtrace of record a from the cell centre, then burn, decay and emitters.
__device__ __forceinline__ void cfgAdvectScalarsAt(Rec4* __restrict__ aOut, const Rec4* __restrict__ aIn, const Velocity& vel, const ConfigParams& p, int x, int y, int z) {
    const float px = static_cast<float>(x) + 0.5f, py = static_cast<float>(y) + 0.5f, pz = static_cast<float>(z) + 0.5f;
    const float3 d = velocityAtCentre(vel, p, x, y, z);
    const float4 s = recordAt(aIn, p, px - d.x, py - d.y, pz - d.z);
    float heat = s.x, fuel = s.y, soot = s.w;
    if (heat > p.ignition) {
        const float burn = fuel * p.burnFrac;
        fuel = fuel - burn;
        heat = heat + p.heatRelease * burn;
        soot = soot + p.sootYield * burn;
    }
    heat = heat - heat * p.coolFrac;
    soot = soot - soot * p.sootFrac;
    const unsigned cell = static_cast<unsigned>((z * p.ny + y) * p.nx + x);
    for (int e = 0; e < p.emitterCount; ++e) {
        const ConfigEmitter& em = p.emitters[e];
        if (!inDisk(em, x, y, z)) continue;
        const float j = 1.0f - em.jitter * jitterUniform(em.seed, p.step, cell);
        fuel = fmaxf(fuel, em.fuel * j);
        heat = fmaxf(heat, em.heat * j);
    }
    stv(aOut + cell, make_float4(heat, fuel, 0.0f, soot));
}

__global__ void __launch_bounds__(128) cfgAdvectScalars(Rec4* __restrict__ aOut, const Rec4* __restrict__ aIn, Velocity vel, ConfigParams p) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= p.nx) return;
    cfgAdvectScalarsAt(aOut, aIn, vel, p, x, y, z);
}

// omega = curl of the cell-centred velocity (central differences, clamped
// neighbours), and |omega|.
__device__ __forceinline__ void cfgVorticityAt(float4* __restrict__ vort, const Velocity& vel, const ConfigParams& p, int x, int y, int z) {
    const int xm = max(x - 1, 0), xp = min(x + 1, p.nx - 1);
    const int ym = max(y - 1, 0), yp = min(y + 1, p.ny - 1);
    const int zm = max(z - 1, 0), zp = min(z + 1, p.nz - 1);
    const int ux = p.nx + 1, vy = p.ny + 1;
    auto ccx = [&](int i, int j, int k) { return cellCentred(vel.u, faceIndex(i, j, k, ux, p.ny), faceIndex(i + 1, j, k, ux, p.ny)); };
    auto ccy = [&](int i, int j, int k) { return cellCentred(vel.v, faceIndex(i, j, k, p.nx, vy), faceIndex(i, j + 1, k, p.nx, vy)); };
    auto ccz = [&](int i, int j, int k) { return cellCentred(vel.w, faceIndex(i, j, k, p.nx, p.ny), faceIndex(i, j, k + 1, p.nx, p.ny)); };
    const float ox = 0.5f * (ccz(x, yp, z) - ccz(x, ym, z)) - 0.5f * (ccy(x, y, zp) - ccy(x, y, zm));
    const float oy = 0.5f * (ccx(x, y, zp) - ccx(x, y, zm)) - 0.5f * (ccz(xp, y, z) - ccz(xm, y, z));
    const float oz = 0.5f * (ccy(xp, y, z) - ccy(xm, y, z)) - 0.5f * (ccx(x, yp, z) - ccx(x, ym, z));
    vort[(z * p.ny + y) * p.nx + x] = make_float4(ox, oy, oz, sqrtf(ox * ox + oy * oy + oz * oz));
}

__global__ void __launch_bounds__(128) cfgVorticity(float4* __restrict__ vort, Velocity vel, ConfigParams p) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= p.nx) return;
    cfgVorticityAt(vort, vel, p, x, y, z);
}

// The curl-noise acceleration amplitude * curl(psi) at every cell centre.  It
// depends only on the noise parameters and the grid, so the scene builds it
// once per parameter set and cfgCellForce reads it.
__device__ __forceinline__ void cfgNoiseFieldAt(float4* __restrict__ noise, const ConfigParams& p, int x, int y, int z) {
    const float px = static_cast<float>(x) + 0.5f, py = static_cast<float>(y) + 0.5f, pz = static_cast<float>(z) + 0.5f;
    const float3 g0 = noiseGradient(p, 0, px, py, pz);
    const float3 g1 = noiseGradient(p, 1, px, py, pz);
    const float3 g2 = noiseGradient(p, 2, px, py, pz);
    noise[(z * p.ny + y) * p.nx + x] = make_float4(p.noiseAmp * (g2.y - g1.z), p.noiseAmp * (g0.z - g2.x), p.noiseAmp * (g1.x - g0.y), 0.0f);
}

__global__ void __launch_bounds__(128) cfgNoiseField(float4* __restrict__ noise, ConfigParams p) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= p.nx) return;
    cfgNoiseFieldAt(noise, p, x, y, z);
}

// Cell-centred acceleration: buoyancy + confinement + curl noise (read from
// the field cfgNoiseField built; null when the amplitude is 0).
__device__ __forceinline__ void cfgCellForceAt(float4* __restrict__ force, const float4* __restrict__ vort, const Rec4* __restrict__ a,
                                                    const float4* __restrict__ noise, const ConfigParams& p, int x, int y, int z) {
    const int idx = (z * p.ny + y) * p.nx + x;
    const float4 s = ldv(a + idx);
    float cx = 0.0f, cy = 0.0f, cz = 0.0f;
    if (p.eps != 0.0f) {
        const int xm = max(x - 1, 0), xp = min(x + 1, p.nx - 1);
        const int ym = max(y - 1, 0), yp = min(y + 1, p.ny - 1);
        const int zm = max(z - 1, 0), zp = min(z + 1, p.nz - 1);
        const float4 o = vort[idx];
        const float ex = 0.5f * (vort[(z * p.ny + y) * p.nx + xp].w - vort[(z * p.ny + y) * p.nx + xm].w);
        const float ey = 0.5f * (vort[(z * p.ny + yp) * p.nx + x].w - vort[(z * p.ny + ym) * p.nx + x].w);
        const float ez = 0.5f * (vort[(zp * p.ny + y) * p.nx + x].w - vort[(zm * p.ny + y) * p.nx + x].w);
        const float len = sqrtf(ex * ex + ey * ey + ez * ez);
        float nx = 0.0f, ny = 0.0f, nz = 0.0f;
        if (len > 1e-20f) {
            nx = ex / len;
            ny = ey / len;
            nz = ez / len;
        }
        cx = p.eps * (ny * o.z - nz * o.y);
        cy = p.eps * (nz * o.x - nx * o.z);
        cz = p.eps * (nx * o.y - ny * o.x);
    }
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    if (p.noiseAmp != 0.0f) {
        const float4 n = __ldg(noise + idx);
        fx = n.x;
        fy = n.y;
        fz = n.z;
    }
    const float buoyancy = p.buoyHeat * (s.x - p.ambient) - p.buoySoot * s.w;
    force[idx] = make_float4(cx + fx, buoyancy + cy + fy, cz + fz, 0.0f);
}

__global__ void __launch_bounds__(128) cfgCellForce(float4* __restrict__ force, const float4* __restrict__ vort, const Rec4* __restrict__ a,
                                                    const float4* __restrict__ noise, ConfigParams p) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= p.nx) return;
    cfgCellForceAt(force, vort, a, noise, p, x, y, z);
}

// Faces += dt * (mean of the two adjacent cells' accelerations) + wind; the
// emitter cells' v faces take upVelocity; walls (u at x = 0, nx; v at y = 0;
// w at z = 0, nz) are zero; the top v faces keep the cell below's acceleration.
__device__ __forceinline__ void cfgApplyForcesAt(FaceT* __restrict__ uOut, FaceT* __restrict__ vOut, FaceT* __restrict__ wOut,
                                                      const Velocity& vel, const float4* __restrict__ force, const ConfigParams& p, int x, int y, int z) {
    if (y < p.ny && z < p.nz) {
        const int i = faceIndex(x, y, z, p.nx + 1, p.ny);
        float u = 0.0f;
        if (x > 0 && x < p.nx) {
            const float fa = force[(z * p.ny + y) * p.nx + x - 1].x, fb = force[(z * p.ny + y) * p.nx + x].x;
            u = ldv(vel.u + i) + (p.dt * (0.5f * (fa + fb)) + p.windDtX);
        }
        stv(uOut + i, u);
    }
    if (x < p.nx && z < p.nz) {
        const int i = faceIndex(x, y, z, p.nx, p.ny + 1);
        float v = 0.0f;
        if (y > 0) {
            const float fd = force[(z * p.ny + y - 1) * p.nx + x].y;
            v = y < p.ny ? ldv(vel.v + i) + p.dt * (0.5f * (fd + force[(z * p.ny + y) * p.nx + x].y)) : ldv(vel.v + i) + p.dt * fd;
            for (int e = 0; e < p.emitterCount; ++e) {
                const ConfigEmitter& em = p.emitters[e];
                if ((y < p.ny && inDisk(em, x, y, z)) || inDisk(em, x, y - 1, z)) v = em.up;
            }
        }
        stv(vOut + i, v);
    }
    if (x < p.nx && y < p.ny) {
        const int i = faceIndex(x, y, z, p.nx, p.ny);
        float w = 0.0f;
        if (z > 0 && z < p.nz) {
            const float fb = force[((z - 1) * p.ny + y) * p.nx + x].z, ff = force[(z * p.ny + y) * p.nx + x].z;
            w = ldv(vel.w + i) + (p.dt * (0.5f * (fb + ff)) + p.windDtZ);
        }
        stv(wOut + i, w);
    }
}

__global__ void __launch_bounds__(128) cfgApplyForces(FaceT* __restrict__ uOut, FaceT* __restrict__ vOut, FaceT* __restrict__ wOut,
                                                      Velocity vel, const float4* __restrict__ force, ConfigParams p) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= p.nx) return;
    facesOfCell(p, x, blockIdx.y, blockIdx.z,
                [&](int fx, int fy, int fz) { cfgApplyForcesAt(uOut, vOut, wOut, vel, force, p, fx, fy, fz); });
}

// Transmittance toward the point light from the centre of each 2x2x2 block of
// cells: lightSamples midpoint samples of extinction * S + fuelExtinction * F
// along the segment, clipped where it leaves the grid box.
__device__ __forceinline__ void cfgTransmittanceAt(float* __restrict__ tr, const Rec4* __restrict__ a, const ConfigParams& p, int lx, int ly, int lz) {
    const float px = 2.0f * static_cast<float>(lx) + 1.0f, py = 2.0f * static_cast<float>(ly) + 1.0f, pz = 2.0f * static_cast<float>(lz) + 1.0f;
    const float dx = p.light.x - px, dy = p.light.y - py, dz = p.light.z - pz;
    const float dist = sqrtf(dx * dx + dy * dy + dz * dz);
    float t = 1.0f;
    if (dist > 1e-6f) {
        const float rx = dx / dist, ry = dy / dist, rz = dz / dist;
        float seg = dist;
        if (rx > 0.0f) seg = fminf(seg, (static_cast<float>(p.nx) - px) / rx);
        if (rx < 0.0f) seg = fminf(seg, (0.0f - px) / rx);
        if (ry > 0.0f) seg = fminf(seg, (static_cast<float>(p.ny) - py) / ry);
        if (ry < 0.0f) seg = fminf(seg, (0.0f - py) / ry);
        if (rz > 0.0f) seg = fminf(seg, (static_cast<float>(p.nz) - pz) / rz);
        if (rz < 0.0f) seg = fminf(seg, (0.0f - pz) / rz);
        seg = fmaxf(seg, 0.0f);
        const float ds = seg / static_cast<float>(p.lightSamples);
        float tau = 0.0f;
        for (int s = 0; s < p.lightSamples; ++s) {
            const float at = (static_cast<float>(s) + 0.5f) * ds;
            const float4 r = recordAt(a, p, px + rx * at, py + ry * at, pz + rz * at);
            tau = tau + (p.extinction * r.w + p.fuelExtinction * r.y) * ds;
        }
        t = expf(-tau);
    }
    tr[(lz * p.ly + ly) * p.lx + lx] = t;
}

__global__ void __launch_bounds__(128) cfgTransmittance(float* __restrict__ tr, const Rec4* __restrict__ a, ConfigParams p) {
    const int lx = blockIdx.x * blockDim.x + threadIdx.x;
    const int ly = blockIdx.y;
    const int lz = blockIdx.z;
    if (lx >= p.lx) return;
    cfgTransmittanceAt(tr, a, p, lx, ly, lz);
}

// One pixel: the camera ray's chord through the grid box in primarySamples
// midpoint samples; absorption, in-scattering of the point light (its
// transmittance volume) and emission; a dark background behind.
__device__ __forceinline__ void cfgRaymarchAt(float4* __restrict__ hdr, const Rec4* __restrict__ a, const float* __restrict__ tr,
                                                   const ConfigParams& p, int px, int py) {
    const float sx = (2.0f * (static_cast<float>(px) + 0.5f) / static_cast<float>(p.frameW) - 1.0f) * p.tanHalf * p.aspect;
    const float sy = (1.0f - 2.0f * (static_cast<float>(py) + 0.5f) / static_cast<float>(p.frameH)) * p.tanHalf;
    float dx = p.forward.x + p.right.x * sx + p.up.x * sy;
    float dy = p.forward.y + p.right.y * sx + p.up.y * sy;
    float dz = p.forward.z + p.right.z * sx + p.up.z * sy;
    const float len = sqrtf(dx * dx + dy * dy + dz * dz);
    dx = dx / len;
    dy = dy / len;
    dz = dz / len;
    float t0 = 0.0f, t1 = 3.0e38f;
    bool hit = true;
    const float eye[3] = {p.eye.x, p.eye.y, p.eye.z};
    const float dir[3] = {dx, dy, dz};
    const float hiB[3] = {static_cast<float>(p.nx), static_cast<float>(p.ny), static_cast<float>(p.nz)};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (dir[k] == 0.0f) {
            if (eye[k] < 0.0f || eye[k] > hiB[k]) hit = false;
        } else {
            const float ta = (0.0f - eye[k]) / dir[k];
            const float tb = (hiB[k] - eye[k]) / dir[k];
            t0 = fmaxf(t0, fminf(ta, tb));
            t1 = fminf(t1, fmaxf(ta, tb));
        }
    }
    float r = 0.0f, g = 0.0f, b = 0.0f, view = 1.0f;
    if (hit && t1 > t0) {
        const float ds = (t1 - t0) / static_cast<float>(p.primarySamples);
        for (int s = 0; s < p.primarySamples; ++s) {
            const float at = t0 + (static_cast<float>(s) + 0.5f) * ds;
            const float qx = p.eye.x + dx * at, qy = p.eye.y + dy * at, qz = p.eye.z + dz * at;
            const float4 rec = recordAt(a, p, qx, qy, qz);
            const float sigma = p.extinction * rec.w + p.fuelExtinction * rec.y;
            const float alpha = 1.0f - expf(-(sigma * ds));
            const float lt = trilinear1(tr, cornersAt(qx * 0.5f - 0.5f, qy * 0.5f - 0.5f, qz * 0.5f - 0.5f, p.lx, p.ly, p.lz), p.lx, p.ly);
            const float scatter = p.albedo * p.lightIntensity * lt * alpha;
            const float heat = fmaxf(rec.x, 0.0f);
            const float h = heat / (heat + 1.0f);
            const float e = p.emission * heat * ds;
            r = r + view * (scatter + e);
            g = g + view * (scatter + e * (0.35f + 0.45f * h));
            b = b + view * (scatter + e * (0.08f + 0.50f * h * h));
            view = view * (1.0f - alpha);
        }
    }
    hdr[py * p.frameW + px] = make_float4(r + view * 0.015f, g + view * 0.016f, b + view * 0.020f, 1.0f - view);
}

__global__ void __launch_bounds__(128) cfgRaymarch(float4* __restrict__ hdr, const Rec4* __restrict__ a, const float* __restrict__ tr,
                                                   ConfigParams p) {
    const int px = blockIdx.x * blockDim.x + threadIdx.x;
    const int py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= p.frameW || py >= p.frameH) return;
    cfgRaymarchAt(hdr, a, tr, p, px, py);
}

// ---- the incremental projection of the multigrid solve (fire_mg.cu) ----

// The incremental projection's first half (see the file comment), out of
// place: per cell, the faces it owns (u at x, v at y, w at z, and the last
// face of each axis for the last cell) are written to the other velocity
// buffer, the interior ones and the top ones minus the previous pressure's
// gradient, rounded to storage, the wall ones as they are; rhs = -div of the
// cell's six updated faces (those it does not own recomputed the same way).
__device__ __forceinline__ void cfgPrepareIncrementAt(FaceT* __restrict__ uOut, FaceT* __restrict__ vOut, FaceT* __restrict__ wOut,
                                                      const Velocity& vel, const float* __restrict__ pressure, float* __restrict__ rhs,
                                                      int nx, int ny, int nz, int x, int y, int z) {
    const int i = (z * ny + y) * nx + x;
    const int ui = (z * ny + y) * (nx + 1) + x;
    const int vi = (z * (ny + 1) + y) * nx + x;
    const int wi = (z * ny + y) * nx + x;
    const float pc = pressure[i];
    const float u0 = x > 0 ? storageRound(ldv(vel.u + ui) - (pc - pressure[i - 1])) : ldv(vel.u + ui);
    const float u1 = x + 1 < nx ? storageRound(ldv(vel.u + ui + 1) - (pressure[i + 1] - pc)) : ldv(vel.u + ui + 1);
    const float v0 = y > 0 ? storageRound(ldv(vel.v + vi) - (pc - pressure[i - nx])) : ldv(vel.v + vi);
    const float v1 = y + 1 < ny ? storageRound(ldv(vel.v + vi + nx) - (pressure[i + nx] - pc))
                                : storageRound(ldv(vel.v + vi + nx) - ((0.0f - pc) - pc));
    const float w0 = z > 0 ? storageRound(ldv(vel.w + wi) - (pc - pressure[i - nx * ny])) : ldv(vel.w + wi);
    const float w1 = z + 1 < nz ? storageRound(ldv(vel.w + wi + nx * ny) - (pressure[i + nx * ny] - pc)) : ldv(vel.w + wi + nx * ny);
    const float div = u1 - u0 + v1 - v0 + w1 - w0;
    rhs[i] = -div;
    stv(uOut + ui, u0);
    stv(vOut + vi, v0);
    stv(wOut + wi, w0);
    if (x == nx - 1) stv(uOut + ui + 1, u1);
    if (y == ny - 1) stv(vOut + vi + nx, v1);
    if (z == nz - 1) stv(wOut + wi + nx * ny, w1);
}

// The incremental projection's second half: u -= grad delta on the interior
// faces and the top faces (ghost -delta); with doWalls the closed walls are
// zeroed as in subtractWall.
__device__ __forceinline__ void cfgSubtractIncrementAt(FaceT* __restrict__ u, FaceT* __restrict__ v, FaceT* __restrict__ w,
                                                       const float* __restrict__ delta, int nx, int ny, int nz, int doWalls, int x, int y,
                                                       int z) {
    const int i = (z * ny + y) * nx + x;
    const float dc = delta[i];
    const int ui = (z * ny + y) * (nx + 1) + x;
    const int vi = (z * (ny + 1) + y) * nx + x;
    const int wi = (z * ny + y) * nx + x;
    if (x > 0) stv(u + ui, ldv(u + ui) - (dc - delta[i - 1]));
    if (y > 0) stv(v + vi, ldv(v + vi) - (dc - delta[i - nx]));
    if (z > 0) stv(w + wi, ldv(w + wi) - (dc - delta[i - nx * ny]));
    if (y == ny - 1) {
        const int top = (z * (ny + 1) + ny) * nx + x;
        stv(v + top, ldv(v + top) - ((0.0f - dc) - dc));
    }
    if (doWalls) {
        if (x == 0) stv(u + ui, 0.0f);
        if (x == nx - 1) stv(u + ui + 1, 0.0f);
        if (y == 0) stv(v + vi, 0.0f);
        if (z == 0) stv(w + wi, 0.0f);
        if (z == nz - 1) stv(w + (nz * ny + y) * nx + x, 0.0f);
    }
}

__global__ void __launch_bounds__(128) cfgPrepareIncrement(FaceT* __restrict__ uOut, FaceT* __restrict__ vOut, FaceT* __restrict__ wOut,
                                                           Velocity vel, const float* __restrict__ pressure, float* __restrict__ rhs,
                                                           int nx, int ny, int nz) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= nx) return;
    cfgPrepareIncrementAt(uOut, vOut, wOut, vel, pressure, rhs, nx, ny, nz, x, blockIdx.y, blockIdx.z);
}

__global__ void __launch_bounds__(128) cfgSubtractIncrement(FaceT* __restrict__ u, FaceT* __restrict__ v, FaceT* __restrict__ w,
                                                            const float* __restrict__ delta, int nx, int ny, int nz, int doWalls) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= nx) return;
    cfgSubtractIncrementAt(u, v, w, delta, nx, ny, nz, doWalls, x, blockIdx.y, blockIdx.z);
}

// ---- batched stages (BatchScene, BatchPlan in fire_kernels.h) ----------

namespace {

// The scene of this block: the last s with start[s] <= blockIdx.x.
__device__ __forceinline__ int batchSceneOf(const int* start, int n) {
    const int b = static_cast<int>(blockIdx.x);
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(start + mid) <= b) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    return lo;
}

// This thread's batchPerThread(space) elements of index space `space`, in
// rows of w elements and planes of h rows: body(B, i, x, y, z) for each.  A
// block takes kBatchThreads * K consecutive elements and thread t the
// elements t, t + kBatchThreads, ... of them (so that every pass of the
// block is coalesced); the scene lookup and the division of the first index
// into coordinates happen once per thread, later coordinates step from it.
template <int SPACE, class Dims, class Body>
__device__ __forceinline__ void batchForEach(const BatchScene* scenes, const BatchPlan* plan, Dims dims, Body body) {
    constexpr int K = batchPerThread(SPACE);
    const int n = plan->scenes;
    const int s = batchSceneOf(plan->start[SPACE], n);
    const BatchScene& B = scenes[s];
    const int count = B.count[SPACE];
    const int first = (static_cast<int>(blockIdx.x) - __ldg(plan->start[SPACE] + s)) * kBatchThreads * K + static_cast<int>(threadIdx.x);
    if (first >= count) return;
    int w, h;
    dims(B, w, h);
    const int row = first / w;
    int x = first - row * w, y = row % h, z = row / h;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int i = first + k * kBatchThreads;
        if (i >= count) break;
        body(B, i, x, y, z);
        x += kBatchThreads;
        while (x >= w) {
            x -= w;
            if (++y == h) {
                y = 0;
                ++z;
            }
        }
    }
}

__device__ __forceinline__ void cellDims(const BatchScene& B, int& w, int& h) {
    w = B.c.nx;
    h = B.c.ny;
}
__device__ __forceinline__ void faceDims(const BatchScene& B, int& w, int& h) {
    w = B.c.nx + 1;
    h = B.c.ny + 1;
}

__device__ __forceinline__ Velocity velocityOf(FaceT* const (&f)[3]) { return Velocity{f[0], f[1], f[2]}; }

}  // namespace

__global__ void __launch_bounds__(kBatchThreads) batchAdvectVelocity(const BatchScene* __restrict__ scenes, const BatchPlan* __restrict__ plan) {
    batchForEach<kBatchFaces>(scenes, plan, faceDims, [](const BatchScene& B, int, int x, int y, int z) {
        cfgAdvectVelocityAt(B.adv[0], B.adv[1], B.adv[2], B.vel, B.c, x, y, z);
    });
}

__global__ void __launch_bounds__(kBatchThreads) batchAdvectScalars(const BatchScene* __restrict__ scenes, const BatchPlan* __restrict__ plan) {
    batchForEach<kBatchCells>(scenes, plan, cellDims, [](const BatchScene& B, int, int x, int y, int z) {
        cfgAdvectScalarsAt(B.aOut, B.aIn, velocityOf(B.adv), B.c, x, y, z);
    });
}

__global__ void __launch_bounds__(kBatchThreads) batchVorticity(const BatchScene* __restrict__ scenes, const BatchPlan* __restrict__ plan) {
    batchForEach<kBatchCells>(scenes, plan, cellDims, [](const BatchScene& B, int, int x, int y, int z) {
        if (B.c.eps == 0.0f) return;
        cfgVorticityAt(B.vort, velocityOf(B.adv), B.c, x, y, z);
    });
}

__global__ void __launch_bounds__(kBatchThreads) batchCellForce(const BatchScene* __restrict__ scenes, const BatchPlan* __restrict__ plan) {
    batchForEach<kBatchCells>(scenes, plan, cellDims, [](const BatchScene& B, int, int x, int y, int z) {
        cfgCellForceAt(B.force, B.vort, B.aOut, B.noise, B.c, x, y, z);
    });
}

__global__ void __launch_bounds__(kBatchThreads) batchApplyForces(const BatchScene* __restrict__ scenes, const BatchPlan* __restrict__ plan) {
    batchForEach<kBatchFaces>(scenes, plan, faceDims, [](const BatchScene& B, int, int x, int y, int z) {
        cfgApplyForcesAt(B.forced[0], B.forced[1], B.forced[2], velocityOf(B.adv), B.force, B.c, x, y, z);
    });
}

__global__ void __launch_bounds__(kBatchThreads) batchPrepareIncrement(const BatchScene* __restrict__ scenes,
                                                                      const BatchPlan* __restrict__ plan) {
    batchForEach<kBatchCells>(scenes, plan, cellDims, [](const BatchScene& B, int, int x, int y, int z) {
        cfgPrepareIncrementAt(B.proj[0], B.proj[1], B.proj[2], velocityOf(B.forced), B.pressure, B.divergence, B.c.nx, B.c.ny, B.c.nz, x,
                              y, z);
    });
}

__global__ void __launch_bounds__(kBatchThreads) batchSubtractIncrement(const BatchScene* __restrict__ scenes,
                                                                       const BatchPlan* __restrict__ plan) {
    batchForEach<kBatchCells>(scenes, plan, cellDims, [](const BatchScene& B, int, int x, int y, int z) {
        cfgSubtractIncrementAt(B.proj[0], B.proj[1], B.proj[2], B.delta, B.c.nx, B.c.ny, B.c.nz, 1, x, y, z);
    });
}

__global__ void __launch_bounds__(kBatchThreads) batchTransmittance(const BatchScene* __restrict__ scenes, const BatchPlan* __restrict__ plan) {
    batchForEach<kBatchLight>(
        scenes, plan,
        [](const BatchScene& B, int& w, int& h) {
            w = B.c.lx;
            h = B.c.ly;
        },
        [](const BatchScene& B, int, int x, int y, int z) { cfgTransmittanceAt(B.transmittance, B.aOut, B.c, x, y, z); });
}

__global__ void __launch_bounds__(kBatchThreads) batchRaymarch(const BatchScene* __restrict__ scenes, const BatchPlan* __restrict__ plan) {
    batchForEach<kBatchPixels>(
        scenes, plan,
        [](const BatchScene& B, int& w, int& h) {
            w = B.c.frameW;
            h = B.c.frameH;
        },
        [](const BatchScene& B, int, int x, int y, int) { cfgRaymarchAt(B.hdr, B.aOut, B.transmittance, B.c, x, y); });
}

__global__ void __launch_bounds__(kBatchThreads) batchPackHdr(const BatchScene* __restrict__ scenes, const BatchPlan* __restrict__ plan) {
    batchForEach<kBatchPixels>(
        scenes, plan,
        [](const BatchScene& B, int& w, int& h) {
            w = B.c.frameW;
            h = B.c.frameH;
        },
        [](const BatchScene& B, int i, int x, int y, int) {
            if (B.slot == nullptr) return;
            packHdrPixel(B.slot, B.slotPitch, B.slotFormat, B.hdr[i], x, y);
        });
}

}  // namespace firesim
