// fire_mg.cu -- geometric multigrid for the pressure equation of the config
// physics with a Dirichlet top (p = 0 on the top face).
//
// Level equation: sum over axes a of w_a (2p - p_a- - p_a+) = rhs, with
// Neumann walls and floor (a missing neighbour is the cell itself) and an
// antisymmetric ghost above the top row (-p), which keeps the boundary on the
// top face at every level.  Level 0 is the grid with w = (1, 1, 1) and rhs =
// the projection's divergence array (-div u).  Level l + 1 halves every axis
// whose extent is even and at least 4 (semi-coarsening keeps odd extents) and
// divides that axis's weight by 4 (the doubled spacing squared).  A V-cycle:
// pre-smoothing (red-black Gauss-Seidel), the residual averaged onto the
// coarse cells, the coarse correction from zero, its cell-centred
// interpolation (3/4, 1/4 along each halved axis, neighbours clamped) added
// back, post-smoothing; the coarsest level is relaxed by one block.  After
// each cycle the level-0 residual is reduced into the solve's gate
// (sorResidualFinal); once max |r| is within the tolerance every later kernel
// of the solve returns at once.
//
// Level 0 holds p in double (its smoothing, residuals and prolongation run in
// double; rhs stays float): in float, the rounding of p itself floors the
// residual near 6 ulp(|p|), ~1e-4 for |p| ~ 140, and with it |div u| after
// the projection.  The coarser levels carry small corrections in float.  The
// solve ends by writing the float pressure field; under a Dirichlet top the
// gradient subtraction reads the double pressure (cfgSubtractWide).
//
// Compiled with -fmad=false: every operation rounds as written, so a CPU
// restatement in the same order gives the same bits.
#include "fire_kernels.h"

namespace firesim {

namespace {

__device__ __forceinline__ int mgAt(const MgLevel& L, int x, int y, int z) { return (z * L.ny + y) * L.nx + x; }

__device__ __forceinline__ bool skipped(const int* skip) { return skip != nullptr && __ldg(skip) != 0; }

// rhs + wx (pL + pR) + wy (pD + pU) + wz (pB + pF), in the level's pressure
// type P (double on level 0), in this order.
template <typename P>
__device__ __forceinline__ P combine(float rhs, P pL, P pR, P pD, P pU, P pB, P pF, const MgLevel& L) {
    return static_cast<P>(rhs) + static_cast<P>(L.wx) * (pL + pR) + static_cast<P>(L.wy) * (pD + pU) + static_cast<P>(L.wz) * (pB + pF);
}

// The weighted sum for cell (x, y, z) with the boundary rules.
template <typename P>
__device__ __forceinline__ P weightedSum(const P* p, const float* rhs, const MgLevel& L, int x, int y, int z, P self) {
    const int i = mgAt(L, x, y, z);
    const P pL = x > 0 ? p[i - 1] : self;
    const P pR = x < L.nx - 1 ? p[i + 1] : self;
    const P pD = y > 0 ? p[i - L.nx] : self;
    const P pU = y < L.ny - 1 ? p[i + L.nx] : static_cast<P>(0) - self;
    const P pB = z > 0 ? p[i - L.nx * L.ny] : self;
    const P pF = z < L.nz - 1 ? p[i + L.nx * L.ny] : self;
    return combine(rhs[i], pL, pR, pD, pU, pB, pF, L);
}

template <typename P>
__device__ __forceinline__ P residualAt(const P* p, const float* rhs, const MgLevel& L, int x, int y, int z) {
    const P self = p[mgAt(L, x, y, z)];
    return weightedSum(p, rhs, L, x, y, z, self) - static_cast<P>(L.diag) * self;
}

template <typename P>
__device__ __forceinline__ void smoothCell(P* p, const float* rhs, const MgLevel& L, int x, int y, int z) {
    const int i = mgAt(L, x, y, z);
    p[i] = weightedSum(p, rhs, L, x, y, z, p[i]) * static_cast<P>(L.invDiag);
}

}  // namespace

// One colour of red-black Gauss-Seidel: cells with (x + y + z) % 2 == colour.
template <typename P>
__device__ __forceinline__ void mgSmoothBody(P* __restrict__ p, const float* __restrict__ rhs, const MgLevel& L, int colour, const int* skip) {
    if (skipped(skip)) return;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (y >= L.ny) return;
    const int x = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + ((colour + y + z) & 1);
    if (x >= L.nx) return;
    smoothCell(p, rhs, L, x, y, z);
}

// Coarse rhs = the mean residual of the covered fine cells (averaged along x,
// then y, then z over the halved axes, in the fine level's type), coarse p = 0.
template <typename P>
__device__ __forceinline__ void mgRestrictBody(float* __restrict__ rhsC, float* __restrict__ pC, const P* __restrict__ p,
                                               const float* __restrict__ rhs, const MgLevel& F, const MgLevel& C, const int* skip) {
    if (skipped(skip)) return;
    const int X = blockIdx.x * blockDim.x + threadIdx.x;
    const int Y = blockIdx.y;
    const int Z = blockIdx.z;
    if (X >= C.nx) return;
    const int x0 = C.cx ? 2 * X : X, y0 = C.cy ? 2 * Y : Y, z0 = C.cz ? 2 * Z : Z;
    const P half = static_cast<P>(0.5f);
    P az[2];
    for (int dz = 0; dz <= C.cz; ++dz) {
        P ay[2];
        for (int dy = 0; dy <= C.cy; ++dy) {
            const P r0 = residualAt(p, rhs, F, x0, y0 + dy, z0 + dz);
            ay[dy] = C.cx ? half * (r0 + residualAt(p, rhs, F, x0 + 1, y0 + dy, z0 + dz)) : r0;
        }
        az[dz] = C.cy ? half * (ay[0] + ay[1]) : ay[0];
    }
    const int c = mgAt(C, X, Y, Z);
    rhsC[c] = static_cast<float>(C.cz ? half * (az[0] + az[1]) : az[0]);
    pC[c] = 0.0f;
}

// p += the coarse correction interpolated along the halved axes (weights 3/4
// and 1/4, neighbour clamped; weights 1 and 0 along kept axes), x, then y, then z.
template <typename P>
__device__ __forceinline__ void mgProlongBody(P* __restrict__ p, const float* __restrict__ pC, const MgLevel& F, const MgLevel& C,
                                              const int* skip) {
    if (skipped(skip)) return;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= F.nx || y >= F.ny) return;
    const int X0 = C.cx ? x >> 1 : x, Y0 = C.cy ? y >> 1 : y, Z0 = C.cz ? z >> 1 : z;
    const int X1 = !C.cx ? X0 : ((x & 1) ? min(X0 + 1, C.nx - 1) : max(X0 - 1, 0));
    const int Y1 = !C.cy ? Y0 : ((y & 1) ? min(Y0 + 1, C.ny - 1) : max(Y0 - 1, 0));
    const int Z1 = !C.cz ? Z0 : ((z & 1) ? min(Z0 + 1, C.nz - 1) : max(Z0 - 1, 0));
    const float ux = C.cx ? 0.75f : 1.0f, vx = C.cx ? 0.25f : 0.0f;
    const float uy = C.cy ? 0.75f : 1.0f, vy = C.cy ? 0.25f : 0.0f;
    const float uz = C.cz ? 0.75f : 1.0f, vz = C.cz ? 0.25f : 0.0f;
    const float a0 = ux * pC[mgAt(C, X0, Y0, Z0)] + vx * pC[mgAt(C, X1, Y0, Z0)];
    const float a1 = ux * pC[mgAt(C, X0, Y1, Z0)] + vx * pC[mgAt(C, X1, Y1, Z0)];
    const float a2 = ux * pC[mgAt(C, X0, Y0, Z1)] + vx * pC[mgAt(C, X1, Y0, Z1)];
    const float a3 = ux * pC[mgAt(C, X0, Y1, Z1)] + vx * pC[mgAt(C, X1, Y1, Z1)];
    const float b0 = uy * a0 + vy * a1, b1 = uy * a2 + vy * a3;
    const int i = mgAt(F, x, y, z);
    p[i] = p[i] + static_cast<P>(uz * b0 + vz * b1);
}

// `sweeps` red-black Gauss-Seidel iterations over cells first, first + stride,
// ... (at most four of them) of a level, whose coordinates are worked out once;
// each colour ends with a barrier of the warp (warpOnly) or of the block.
template <typename P>
__device__ __forceinline__ void smoothCells(P* __restrict__ p, const float* __restrict__ rhs, const MgLevel& L, int sweeps, int first,
                                            int stride, bool warpOnly) {
    const int cells = L.nx * L.ny * L.nz;
    int xs[4], ys[4], zs[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int i = first + k * stride;
        xs[k] = i < cells ? i % L.nx : -1;
        ys[k] = (i / L.nx) % L.ny;
        zs[k] = i / (L.nx * L.ny);
    }
    for (int s = 0; s < sweeps; ++s) {
        for (int colour = 0; colour < 2; ++colour) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (xs[k] >= 0 && ((xs[k] + ys[k] + zs[k]) & 1) == colour) smoothCell(p, rhs, L, xs[k], ys[k], zs[k]);
            }
            if (warpOnly) {
                __syncwarp();
            } else {
                __syncthreads();
            }
        }
    }
}

// The coarsest level: `sweeps` red-black Gauss-Seidel iterations by one
// block.  A level of at most 128 cells is relaxed by the first warp alone,
// with warp barriers between the colours; one of at most four cells per
// thread works out each thread's cells once.
template <typename P>
__device__ __forceinline__ void mgCoarsestBody(P* __restrict__ p, const float* __restrict__ rhs, const MgLevel& L, int sweeps,
                                               const int* skip) {
    if (skipped(skip)) return;
    const int cells = L.nx * L.ny * L.nz;
    if (cells <= 4 * 32) {
        if (threadIdx.x < 32) smoothCells(p, rhs, L, sweeps, static_cast<int>(threadIdx.x), 32, true);
        return;
    }
    if (cells <= 4 * static_cast<int>(blockDim.x)) {
        smoothCells(p, rhs, L, sweeps, static_cast<int>(threadIdx.x), static_cast<int>(blockDim.x), false);
        return;
    }
    for (int s = 0; s < sweeps; ++s) {
        for (int colour = 0; colour < 2; ++colour) {
            for (int i = threadIdx.x; i < cells; i += blockDim.x) {
                const int x = i % L.nx;
                const int y = (i / L.nx) % L.ny;
                const int z = i / (L.nx * L.ny);
                if (((x + y + z) & 1) != colour) continue;
                smoothCell(p, rhs, L, x, y, z);
            }
            __syncthreads();
        }
    }
}

// Level-0 residual r = (weighted neighbour sum) - 6p with the Dirichlet top,
// per block over whole rows (as sorResidualPartials).
template <typename P>
__device__ __forceinline__ void mgResidualPartialsBody(const P* __restrict__ p, const float* __restrict__ rhs, const MgLevel& L,
                                                       const SorGate* gate, double* __restrict__ partialSq, float* __restrict__ partialMax) {
    if (gate->converged) return;
    const int lane = threadIdx.x & 31;
    const int warps = kResidualThreads / 32;
    double s = 0.0;
    float m = 0.0f;
    for (int row = blockIdx.x * warps + (threadIdx.x >> 5); row < L.ny * L.nz; row += gridDim.x * warps) {
        const int y = row % L.ny;
        const int z = row / L.ny;
        for (int x = lane; x < L.nx; x += 32) {
            const double r = static_cast<double>(residualAt(p, rhs, L, x, y, z));
            m = fmaxf(m, static_cast<float>(fabs(r)));
            s += r * r;
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

// The kernels, one per pressure type (F: float, the coarser levels; D: double, level 0).
__global__ void __launch_bounds__(kMgRowBlockThreads) mgSmoothF(float* p, const float* rhs, MgLevel L, int colour, const int* skip) {
    mgSmoothBody(p, rhs, L, colour, skip);
}
__global__ void __launch_bounds__(kMgRowBlockThreads) mgSmoothD(double* p, const float* rhs, MgLevel L, int colour, const int* skip) {
    mgSmoothBody(p, rhs, L, colour, skip);
}
__global__ void __launch_bounds__(128) mgRestrictF(float* rhsC, float* pC, const float* p, const float* rhs, MgLevel F, MgLevel C,
                                                   const int* skip) {
    mgRestrictBody(rhsC, pC, p, rhs, F, C, skip);
}
__global__ void __launch_bounds__(128) mgRestrictD(float* rhsC, float* pC, const double* p, const float* rhs, MgLevel F, MgLevel C,
                                                   const int* skip) {
    mgRestrictBody(rhsC, pC, p, rhs, F, C, skip);
}
__global__ void __launch_bounds__(kMgRowBlockThreads) mgProlongF(float* p, const float* pC, MgLevel F, MgLevel C, const int* skip) {
    mgProlongBody(p, pC, F, C, skip);
}
__global__ void __launch_bounds__(kMgRowBlockThreads) mgProlongD(double* p, const float* pC, MgLevel F, MgLevel C, const int* skip) {
    mgProlongBody(p, pC, F, C, skip);
}
__global__ void __launch_bounds__(256) mgCoarsestF(float* p, const float* rhs, MgLevel L, int sweeps, const int* skip) {
    mgCoarsestBody(p, rhs, L, sweeps, skip);
}
__global__ void __launch_bounds__(256) mgCoarsestD(double* p, const float* rhs, MgLevel L, int sweeps, const int* skip) {
    mgCoarsestBody(p, rhs, L, sweeps, skip);
}
__global__ void __launch_bounds__(kResidualThreads) mgResidualPartialsD(const double* p, const float* rhs, MgLevel L, const SorGate* gate,
                                                                        double* partialSq, float* partialMax) {
    mgResidualPartialsBody(p, rhs, L, gate, partialSq, partialMax);
}

// The float pressure field from the double level-0 pressure of the solve.
__global__ void __launch_bounds__(256) mgStoreFloat(float* __restrict__ dst, const double* __restrict__ src, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = static_cast<float>(src[i]);
}

// The gradient subtraction under a Dirichlet top from the double pressure:
// each face's difference is formed in double and rounded once before the
// float update; the top faces use the antisymmetric ghost -p; with doWalls
// the closed walls are zeroed as in subtractWall.
__global__ void __launch_bounds__(128) cfgSubtractWide(FaceT* __restrict__ u, FaceT* __restrict__ v, FaceT* __restrict__ w,
                                                       const double* __restrict__ p, int nx, int ny, int nz, int doWalls) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= nx) return;
    const int i = (z * ny + y) * nx + x;
    const double pc = p[i];
    const int ui = (z * ny + y) * (nx + 1) + x;
    const int vi = (z * (ny + 1) + y) * nx + x;
    const int wi = (z * ny + y) * nx + x;
    if (x > 0) stv(u + ui, ldv(u + ui) - static_cast<float>(pc - p[i - 1]));
    if (y > 0) stv(v + vi, ldv(v + vi) - static_cast<float>(pc - p[i - nx]));
    if (z > 0) stv(w + wi, ldv(w + wi) - static_cast<float>(pc - p[i - nx * ny]));
    if (y == ny - 1) {
        const int top = (z * (ny + 1) + ny) * nx + x;
        stv(v + top, ldv(v + top) - static_cast<float>((0.0 - pc) - pc));
    }
    if (doWalls) {
        if (x == 0) stv(u + ui, 0.0f);
        if (x == nx - 1) stv(u + ui + 1, 0.0f);
        if (y == 0) stv(v + vi, 0.0f);
        if (z == 0) stv(w + wi, 0.0f);
        if (z == nz - 1) stv(w + (nz * ny + y) * nx + x, 0.0f);
    }
}

// End of one V-cycle inside the solve's conditional WHILE node: one warp
// reduces the level-0 residual partials (when gated, as sorResidualFinal),
// counts the cycle and sets the loop condition, which is cleared once the
// residual is within the tolerance or maxCycles cycles have run.  The count
// always advances, so the loop ends after at most maxCycles bodies.
__global__ void mgCycleEnd(SorGate* gate, const double* __restrict__ partialSq, const float* __restrict__ partialMax, int partials,
                           float tolerance, int gated, int maxCycles, cudaGraphConditionalHandle loop) {
    const int lane = threadIdx.x;
    if (gated) {
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
        if (lane == 0) {
            gate->maxResidual = m;
            gate->l2Residual = sqrt(s);
            if (m <= tolerance) gate->converged = 1;
        }
    }
    if (lane != 0) return;
    if (!gated) {
        gate->maxResidual = -1.0f;
        gate->l2Residual = -1.0;
    }
    gate->iterations += 1;
    const bool more = gate->converged == 0 && gate->iterations < maxCycles && gate->iterations < kMgHardCycleCap;
    cudaGraphSetConditional(loop, more ? 1u : 0u);
}

// The top faces under a Dirichlet top: v(x, ny, z) -= (ghost - p) with the
// antisymmetric ghost -p of the top cell.
__global__ void __launch_bounds__(128) cfgTopFaces(FaceT* __restrict__ v, const float* __restrict__ p, int nx, int ny, int nz) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y;
    if (x >= nx) return;
    const int face = (z * (ny + 1) + ny) * nx + x;
    const float top = p[(z * ny + ny - 1) * nx + x];
    stv(v + face, ldv(v + face) - ((0.0f - top) - top));
}

}  // namespace firesim
