// fire_mg.cu -- geometric multigrid for the pressure equation of the config
// physics with a Dirichlet top (p = 0 on the top face), for one scene or for
// a batch of scenes of any sizes in one persistent launch.
//
// Incremental projection.  Before the solve, cfgPrepareIncrement subtracts
// the previous step's pressure gradient from the faces (interior faces, and
// the top faces with the antisymmetric ghost -p) and writes the divergence of
// those faces as the rhs; the solve then finds only the increment delta,
// from zero (its first phase clears it).  The increment is small next to the pressure (|p| ~ 1e2 in a
// developed 128^3 fire), so float carries it without the rounding floor that
// float pressure itself would put on |div u| (~6 ulp of |p|); every level is
// float.  At the end of the solve pressure += delta, and the gradient
// subtraction (cfgSubtractIncrement) takes delta.
//
// Level equation: sum over axes a of w_a (2p - p_a- - p_a+) = rhs, with
// Neumann walls and floor (a missing neighbour is the cell itself) and the
// antisymmetric ghost -p above the top row, which keeps the boundary on the
// top face at every level.  Level 0 is the grid with w = (1, 1, 1).  Level
// l + 1 halves every axis whose extent is even and at least 4 (semi-
// coarsening keeps odd extents) and divides that axis's weight by 4.  A
// V-cycle: pre-smoothing (red-black Gauss-Seidel), the residual averaged onto
// the coarse cells, the coarse correction from zero, its cell-centred
// interpolation (3/4, 1/4 along each halved axis, neighbours clamped) added
// back, post-smoothing; the coarsest level gets kMgCoarsestSweeps sweeps.
// After each cycle the level-0 residual is reduced per scene in a fixed order
// (max |r| in float, sum r^2 in double); a scene whose max |r| is within the
// tolerance stops, and the solve ends when every scene has stopped or
// maxCycles cycles have run.
//
// One launch (mgSolve) runs every cycle of every scene of the batch.  Its
// CTAs are all co-resident (cooperative launch); the phases of a cycle are
// separated by a grid barrier whose waits are bounded in time.  Within a
// phase, warps take rows of all scenes at that level from one work list.
// The coarse end of each scene's hierarchy (from the first level of at most
// kMgTailCells cells down) is solved by one CTA in shared memory (in its
// global buffers if it does not fit, as for a grid that cannot coarsen).  Reads of
// data written inside the launch go through L2 (ld.global.cg), as L1 is not
// coherent between SMs.
//
// Compiled with -fmad=false: every operation rounds as written, so a CPU
// restatement in the same order gives the same bits, and a scene gives the
// same bits alone or in any batch.
#include "fire_kernels.h"

namespace firesim {

namespace {

__device__ __forceinline__ int mgAt(const MgLevel& L, int x, int y, int z) { return (z * L.ny + y) * L.nx + x; }

__device__ __forceinline__ unsigned loadVolatileU(const unsigned* p) { return *reinterpret_cast<const volatile unsigned*>(p); }
__device__ __forceinline__ int loadVolatileI(const int* p) { return *reinterpret_cast<const volatile int*>(p); }
__device__ __forceinline__ unsigned long long mgTimerNs() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// rhs + wx (pL + pR) + wy (pD + pU) + wz (pB + pF), in this order.
__device__ __forceinline__ float combine(float rhs, float pL, float pR, float pD, float pU, float pB, float pF, const MgLevel& L) {
    return rhs + L.wx * (pL + pR) + L.wy * (pD + pU) + L.wz * (pB + pF);
}

// Neighbour sums with the boundary rules, reading p through `load`.
template <class Load>
__device__ __forceinline__ float weightedSum(Load load, float rhs, const MgLevel& L, int i, int x, int y, int z, float self) {
    const float pL = x > 0 ? load(i - 1) : self;
    const float pR = x < L.nx - 1 ? load(i + 1) : self;
    const float pD = y > 0 ? load(i - L.nx) : self;
    const float pU = y < L.ny - 1 ? load(i + L.nx) : 0.0f - self;
    const float pB = z > 0 ? load(i - L.nx * L.ny) : self;
    const float pF = z < L.nz - 1 ? load(i + L.nx * L.ny) : self;
    return combine(rhs, pL, pR, pD, pU, pB, pF, L);
}

// The scene of work item `item` in a prefix array of n + 1 offsets: the last
// s with off[s] <= item (empty ranges are skipped over).
__device__ __forceinline__ int sceneOf(const int* off, int n, int item) {
    int lo = 0, hi = n;  // off[lo] <= item < off[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(off + mid) <= item) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    return lo;
}

// Grid barrier of the persistent solve: the last CTA to arrive resets the
// count and advances the generation; the others poll the generation.  Every
// wait gives up after waitNs (or a poll cap), marks the sync failed so the
// other CTAs stop too, and records the phase in the host-mapped status word.
__device__ bool gridBarrier(MgSync* sync, unsigned& generation, unsigned long long waitNs, unsigned* hostStatus, int phase) {
    __syncthreads();
    __shared__ int sFailed;
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned target = generation + 1u;
        bool failed = false;
        if (atomicAdd(&sync->count, 1u) == gridDim.x - 1u) {
            sync->count = 0u;
            __threadfence();
            atomicExch(&sync->generation, target);
        } else {
            const unsigned long long start = mgTimerNs();
            for (unsigned n = 0;; ++n) {
                if (loadVolatileU(&sync->generation) == target) break;
                if ((n & 7u) == 7u) {
                    if (loadVolatileU(&sync->failed) != 0u) {
                        failed = true;
                        break;
                    }
                    if (mgTimerNs() - start > waitNs || n > kMgMaxPolls) {
                        atomicExch(&sync->failed, 1u);
                        *reinterpret_cast<volatile unsigned*>(hostStatus) = kMgStatusFlag | static_cast<unsigned>(phase);
                        __threadfence_system();
                        failed = true;
                        break;
                    }
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        sFailed = (failed || loadVolatileU(&sync->failed) != 0u) ? 1 : 0;
    }
    __syncthreads();
    generation += 1u;
    return sFailed == 0;
}

// ---- the tail: levels tail..levels-1 of one scene in one CTA ------------
// The levels' p and rhs live in shared memory, except where the tail's mode
// puts them in their global buffers (read through L2): kMgTailShared keeps
// everything in shared memory; kMgTailRhsGlobal keeps the tail level's rhs
// (read-only within the tail) in global memory; kMgTailGlobal keeps all of it
// there, for a tail too large for shared memory.

template <bool kGlobal>
__device__ __forceinline__ float tailLoad(const float* a, int i) {
    if constexpr (kGlobal) {
        return __ldcg(a + i);
    } else {
        return a[i];
    }
}

constexpr int kTailSlots = 4;  // cells per thread of the slot path of tailSmooth

// `sweeps` red-black sweeps of one tail level.  A level of at most 128 cells
// is relaxed by the first warp alone, with warp barriers; otherwise by the
// whole CTA.  In shared memory a level of at most kTailSlots cells per
// thread keeps each thread's cells, their coordinates and their rhs in
// registers for all the sweeps; a larger one is walked by columns (x, y)
// along z, one division per column.  The level is passed by value and p and
// rhs do not alias, so the level's fields and the rhs loads are not reloaded
// or held back by the stores to p.
template <bool PG, bool RG>
__device__ __noinline__ void tailSmooth(float* __restrict__ p, const float* __restrict__ rhs, const MgLevel L, int sweeps) {
    const int cols = L.nx * L.ny;
    const int cells = cols * L.nz;
    const bool warpOnly = cells <= 4 * 32;
    const int stride = warpOnly ? 32 : static_cast<int>(blockDim.x);
    const bool active = !warpOnly || threadIdx.x < 32;
    auto load = [&](int j) { return tailLoad<PG>(p, j); };
    if (!PG && cells <= kTailSlots * stride) {
        int packed[kTailSlots];
        float rh[kTailSlots];
#pragma unroll
        for (int k = 0; k < kTailSlots; ++k) {
            const int i = static_cast<int>(threadIdx.x) + k * stride;
            packed[k] = -1;
            rh[k] = 0.0f;
            if (active && i < cells) {
                const int x = i % L.nx, y = (i / L.nx) % L.ny, z = i / cols;
                packed[k] = x | (y << 10) | (z << 20);
                rh[k] = tailLoad<RG>(rhs, i);
            }
        }
        for (int s = 0; s < sweeps; ++s) {
            for (int colour = 0; colour < 2; ++colour) {
#pragma unroll
                for (int k = 0; k < kTailSlots; ++k) {
                    const int c = packed[k];
                    if (c < 0) continue;
                    const int x = c & 1023, y = (c >> 10) & 1023, z = c >> 20;
                    if (((x + y + z) & 1) != colour) continue;
                    const int i = static_cast<int>(threadIdx.x) + k * stride;
                    p[i] = weightedSum(load, rh[k], L, i, x, y, z, p[i]) * L.invDiag;
                }
                if (warpOnly) {
                    __syncwarp();
                } else {
                    __syncthreads();
                }
            }
        }
        __syncthreads();
        return;
    }
    for (int s = 0; s < sweeps; ++s) {
        for (int colour = 0; colour < 2; ++colour) {
            if (active) {
                for (int col = threadIdx.x; col < cols; col += stride) {
                    const int y = col / L.nx, x = col - y * L.nx;
#pragma unroll 4
                    for (int z = (colour + x + y) & 1; z < L.nz; z += 2) {
                        const int i = col + z * cols;
                        p[i] = weightedSum(load, tailLoad<RG>(rhs, i), L, i, x, y, z, load(i)) * L.invDiag;
                    }
                }
            }
            if constexpr (PG) __threadfence_block();
            if (warpOnly) {
                __syncwarp();
            } else {
                __syncthreads();
            }
        }
    }
    __syncthreads();
}

// Coarse rhs = the mean residual of the covered fine cells (averaged along x,
// then y, then z over the halved axes), coarse p = 0.
template <class Load>
__device__ __forceinline__ float restrictAt(Load loadP, const float* rhsF, bool rhsViaL2, const MgLevel& F, const MgLevel& C, int X, int Y,
                                           int Z) {
    const int x0 = C.cx ? 2 * X : X, y0 = C.cy ? 2 * Y : Y, z0 = C.cz ? 2 * Z : Z;
    float az[2] = {0.0f, 0.0f};
    for (int dz = 0; dz <= C.cz; ++dz) {
        float ay[2] = {0.0f, 0.0f};
        for (int dy = 0; dy <= C.cy; ++dy) {
            float r[2] = {0.0f, 0.0f};
            for (int dx = 0; dx <= C.cx; ++dx) {
                const int x = x0 + dx, y = y0 + dy, z = z0 + dz;
                const int i = mgAt(F, x, y, z);
                const float self = loadP(i);
                const float rh = rhsViaL2 ? __ldcg(rhsF + i) : rhsF[i];
                r[dx] = weightedSum(loadP, rh, F, i, x, y, z, self) - F.diag * self;
            }
            ay[dy] = C.cx ? 0.5f * (r[0] + r[1]) : r[0];
        }
        az[dz] = C.cy ? 0.5f * (ay[0] + ay[1]) : ay[0];
    }
    return C.cz ? 0.5f * (az[0] + az[1]) : az[0];
}

// p += the coarse correction interpolated along the halved axes (weights 3/4
// and 1/4, neighbour clamped; weights 1 and 0 along kept axes), x, then y, then z.
template <class LoadC>
__device__ __forceinline__ float prolongAt(LoadC loadC, const MgLevel& F, const MgLevel& C, int x, int y, int z) {
    const int X0 = C.cx ? x >> 1 : x, Y0 = C.cy ? y >> 1 : y, Z0 = C.cz ? z >> 1 : z;
    const int X1 = !C.cx ? X0 : ((x & 1) ? min(X0 + 1, C.nx - 1) : max(X0 - 1, 0));
    const int Y1 = !C.cy ? Y0 : ((y & 1) ? min(Y0 + 1, C.ny - 1) : max(Y0 - 1, 0));
    const int Z1 = !C.cz ? Z0 : ((z & 1) ? min(Z0 + 1, C.nz - 1) : max(Z0 - 1, 0));
    const float ux = C.cx ? 0.75f : 1.0f, vx = C.cx ? 0.25f : 0.0f;
    const float uy = C.cy ? 0.75f : 1.0f, vy = C.cy ? 0.25f : 0.0f;
    const float uz = C.cz ? 0.75f : 1.0f, vz = C.cz ? 0.25f : 0.0f;
    const float a0 = ux * loadC(mgAt(C, X0, Y0, Z0)) + vx * loadC(mgAt(C, X1, Y0, Z0));
    const float a1 = ux * loadC(mgAt(C, X0, Y1, Z0)) + vx * loadC(mgAt(C, X1, Y1, Z0));
    const float a2 = ux * loadC(mgAt(C, X0, Y0, Z1)) + vx * loadC(mgAt(C, X1, Y0, Z1));
    const float a3 = ux * loadC(mgAt(C, X0, Y1, Z1)) + vx * loadC(mgAt(C, X1, Y1, Z1));
    const float b0 = uy * a0 + vy * a1, b1 = uy * a2 + vy * a3;
    return uz * b0 + vz * b1;
}

// The V-cycle of levels tail..levels-1 of scene S by this CTA.  The tail
// level's p comes from global memory (it is zero there unless the tail is
// level 0) and goes back to it at the end.
template <int MODE>
__device__ __noinline__ void tailCycle(const MgScene& S, int pre, int post, float* smem) {
    constexpr bool PG = MODE == kMgTailGlobal;
    const int t = S.tail;
    float* p[kMgMaxLevels];
    float* r[kMgMaxLevels];
    int off = 0;
    for (int l = t; l < S.levels; ++l) {
        const int n = S.lv[l].nx * S.lv[l].ny * S.lv[l].nz;
        if (PG) {
            p[l] = S.p[l];
            r[l] = S.rhs[l];
        } else {
            p[l] = smem + off;
            off += n;
            if (MODE == kMgTailRhsGlobal && l == t) {
                r[l] = S.rhs[l];
            } else {
                r[l] = smem + off;
                off += n;
            }
        }
    }
    const MgLevel T0 = S.lv[t];
    const int n0 = T0.nx * T0.ny * T0.nz;
    if constexpr (!PG) {
        for (int i = threadIdx.x; i < n0; i += blockDim.x) {
            p[t][i] = __ldcg(S.p[t] + i);
            if (MODE == kMgTailShared) r[t][i] = __ldcg(S.rhs[t] + i);
        }
    }
    __syncthreads();
    const int last = S.levels - 1;
    for (int l = t; l < last; ++l) {
        const MgLevel F = S.lv[l];
        const MgLevel C = S.lv[l + 1];
        const bool rg = PG || (MODE == kMgTailRhsGlobal && l == t);
        if (rg) {
            tailSmooth<PG, true>(p[l], r[l], F, pre);
        } else {
            tailSmooth<PG, false>(p[l], r[l], F, pre);
        }
        const float* pf = p[l];
        auto loadF = [&](int j) { return tailLoad<PG>(pf, j); };
        const int cols = C.nx * C.ny;
        for (int col = threadIdx.x; col < cols; col += blockDim.x) {
            const int Y = col / C.nx, X = col - Y * C.nx;
            for (int Z = 0; Z < C.nz; ++Z) {
                const int i = col + Z * cols;
                r[l + 1][i] = restrictAt(loadF, r[l], rg, F, C, X, Y, Z);
                p[l + 1][i] = 0.0f;
            }
        }
        if constexpr (PG) __threadfence_block();
        __syncthreads();
    }
    if (PG || (MODE == kMgTailRhsGlobal && last == t)) {
        tailSmooth<PG, true>(p[last], r[last], S.lv[last], kMgCoarsestSweeps);
    } else {
        tailSmooth<PG, false>(p[last], r[last], S.lv[last], kMgCoarsestSweeps);
    }
    for (int l = last - 1; l >= t; --l) {
        const MgLevel F = S.lv[l];
        const MgLevel C = S.lv[l + 1];
        const float* pc = p[l + 1];
        auto loadC = [&](int j) { return tailLoad<PG>(pc, j); };
        const int cols = F.nx * F.ny;
        for (int col = threadIdx.x; col < cols; col += blockDim.x) {
            const int y = col / F.nx, x = col - y * F.nx;
            for (int z = 0; z < F.nz; ++z) {
                const int i = col + z * cols;
                p[l][i] = tailLoad<PG>(p[l], i) + prolongAt(loadC, F, C, x, y, z);
            }
        }
        if constexpr (PG) __threadfence_block();
        __syncthreads();
        if (PG || (MODE == kMgTailRhsGlobal && l == t)) {
            tailSmooth<PG, true>(p[l], r[l], F, post);
        } else {
            tailSmooth<PG, false>(p[l], r[l], F, post);
        }
    }
    if constexpr (!PG) {
        for (int i = threadIdx.x; i < n0; i += blockDim.x) S.p[t][i] = p[t][i];
    }
}

}  // namespace

// The persistent batched solve (see the file comment).  Work items of the
// grid levels are rows of one level of one scene, one warp per row; the
// tail is one CTA per scene; the residual is one warp per chunk of
// kMgChunkRows level-0 rows; the gate is one warp per scene.
__global__ void __launch_bounds__(kMgThreads, 1) mgSolve(const MgScene* __restrict__ scenes, const MgPlan* __restrict__ plan, MgSync* sync,
                                                        unsigned* hostStatus, unsigned long long waitNs) {
    extern __shared__ float smem[];
    __shared__ int sActive;
    const int n = plan->scenes;
    const int gridLevels = plan->gridLevels;
    const int maxCycles = plan->maxCycles, pre = plan->pre, post = plan->post, gated = plan->gated;
    const float tolerance = plan->tolerance;
    const int lane = threadIdx.x & 31;
    const int warpsPerBlock = blockDim.x >> 5;
    const int gwarp = blockIdx.x * warpsPerBlock + (threadIdx.x >> 5);
    const int nwarps = gridDim.x * warpsPerBlock;
    unsigned generation = loadVolatileU(&sync->generation);
    int phase = 0;
    // The scenes still running, read once after each gate (converged flags
    // change only in the gate phase).
    __shared__ unsigned char sRunning[kMgMaxScenes];
    auto refreshRunning = [&]() {
        for (int s = threadIdx.x; s < n; s += blockDim.x) sRunning[s] = loadVolatileI(&scenes[s].gate->converged) == 0 ? 1 : 0;
        __syncthreads();
    };
    auto converged = [&](int s) { return sRunning[s] == 0; };
    // Units are processed kMgUnroll at a time per warp, every load of them
    // issued before any store, so that their L2 round trips overlap.
    constexpr int U = kMgUnroll;

    // One colour of red-black Gauss-Seidel on level l of every scene that has
    // it as a grid level.  A unit is 128 consecutive cells of a row, four per
    // lane: the lane loads its four cells and the same four of the rows above,
    // below, behind and in front (one float4 each when the row length is a
    // multiple of 4, else element by element), the rhs and the two cells
    // beside them, updates the two of its cells of the colour and stores the
    // four back (the other two unchanged: no thread writes them in this phase).
    auto smooth = [&](int l, int colour) {
        const int* off = plan->smoothUnits[l];
        const int total = __ldg(off + n);
        for (int unit = gwarp; unit < total; unit += nwarps) {
            const int s = sceneOf(off, n, unit);
            if (converged(s)) continue;
            const MgScene& S = scenes[s];
            const MgLevel L = S.lv[l];
            const int u = unit - __ldg(off + s);
            const int cpr = mgQuadChunks(L.nx);
            const int row = u / cpr, chunk = u - row * cpr;
            const int y = row % L.ny, z = row / L.ny;
            const int x0 = chunk * 128 + 4 * lane;
            if (x0 >= L.nx) continue;
            float* p = S.p[l];
            const float* rhs = S.rhs[l];
            const int i0 = row * L.nx + x0;
            const int plane = L.nx * L.ny;
            float c[4], dn[4], up[4], bk[4], fr[4], rh[4];
            const bool quad = (L.nx & 3) == 0;
            if (quad) {
                const float4 v = __ldcg(reinterpret_cast<const float4*>(p + i0));
                c[0] = v.x; c[1] = v.y; c[2] = v.z; c[3] = v.w;
                const float4 vd = y > 0 ? __ldcg(reinterpret_cast<const float4*>(p + i0 - L.nx)) : v;
                const float4 vu = y < L.ny - 1 ? __ldcg(reinterpret_cast<const float4*>(p + i0 + L.nx))
                                               : make_float4(0.0f - v.x, 0.0f - v.y, 0.0f - v.z, 0.0f - v.w);
                const float4 vb = z > 0 ? __ldcg(reinterpret_cast<const float4*>(p + i0 - plane)) : v;
                const float4 vf = z < L.nz - 1 ? __ldcg(reinterpret_cast<const float4*>(p + i0 + plane)) : v;
                const float4 vr = l == 0 ? __ldg(reinterpret_cast<const float4*>(rhs + i0)) : __ldcg(reinterpret_cast<const float4*>(rhs + i0));
                dn[0] = vd.x; dn[1] = vd.y; dn[2] = vd.z; dn[3] = vd.w;
                up[0] = vu.x; up[1] = vu.y; up[2] = vu.z; up[3] = vu.w;
                bk[0] = vb.x; bk[1] = vb.y; bk[2] = vb.z; bk[3] = vb.w;
                fr[0] = vf.x; fr[1] = vf.y; fr[2] = vf.z; fr[3] = vf.w;
                rh[0] = vr.x; rh[1] = vr.y; rh[2] = vr.z; rh[3] = vr.w;
            } else {
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int i = i0 + e;
                    if (x0 + e < L.nx) {
                        c[e] = __ldcg(p + i);
                        dn[e] = y > 0 ? __ldcg(p + i - L.nx) : c[e];
                        up[e] = y < L.ny - 1 ? __ldcg(p + i + L.nx) : 0.0f - c[e];
                        bk[e] = z > 0 ? __ldcg(p + i - plane) : c[e];
                        fr[e] = z < L.nz - 1 ? __ldcg(p + i + plane) : c[e];
                        rh[e] = l == 0 ? __ldg(rhs + i) : __ldcg(rhs + i);
                    } else {
                        c[e] = dn[e] = up[e] = bk[e] = fr[e] = rh[e] = 0.0f;
                    }
                }
            }
            const float left = x0 > 0 ? __ldcg(p + i0 - 1) : 0.0f;
            const float right = x0 + 4 < L.nx ? __ldcg(p + i0 + 4) : 0.0f;
            const int e0 = (colour + x0 + y + z) & 1;  // the colour's cells are e0 and e0 + 2
            float o[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int x = x0 + e;
                o[e] = c[e];
                if ((e & 1) != e0 || x >= L.nx) continue;
                const float self = c[e];
                const float pL = x > 0 ? (e > 0 ? c[e - 1] : left) : self;
                const float pR = x < L.nx - 1 ? (e < 3 ? c[e + 1] : right) : self;
                o[e] = (rh[e] + L.wx * (pL + pR) + L.wy * (dn[e] + up[e]) + L.wz * (bk[e] + fr[e])) * L.invDiag;
            }
            if (quad) {
                *reinterpret_cast<float4*>(p + i0) = make_float4(o[0], o[1], o[2], o[3]);
            } else {
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    if ((e & 1) == e0 && x0 + e < L.nx) p[i0 + e] = o[e];
                }
            }
        }
    };
    auto restrictTo = [&](int l) {
        const int* off = plan->coarseUnits[l];
        const int total = __ldg(off + n);
        for (int unit = gwarp; unit < total; unit += nwarps) {
            const int s = sceneOf(off, n, unit);
            if (converged(s)) continue;
            const MgScene& S = scenes[s];
            const MgLevel F = S.lv[l], C = S.lv[l + 1];
            const int u = unit - __ldg(off + s);
            const int cpr = mgRowChunks(C.nx);
            const int row = u / cpr, chunk = u - row * cpr;
            const int Y = row % C.ny, Z = row / C.ny;
            const int X = chunk * 32 + lane;
            if (X >= C.nx) continue;
            const float* pf = S.p[l];
            auto loadF = [&](int j) { return __ldcg(pf + j); };
            const int c = mgAt(C, X, Y, Z);
            const float r = restrictAt(loadF, S.rhs[l], l > 0, F, C, X, Y, Z);
            S.rhs[l + 1][c] = r;
            S.p[l + 1][c] = 0.0f;
        }
    };
    auto prolongFrom = [&](int l) {
        const int* off = plan->fineUnits[l];
        const int total = __ldg(off + n);
        for (int base = gwarp * U; base < total; base += nwarps * U) {
            int sc[U], idx[U];
            float cur[U], add[U];
#pragma unroll
            for (int k = 0; k < U; ++k) {
                const int unit = base + k;
                sc[k] = -1;
                if (unit >= total) continue;
                const int s = sceneOf(off, n, unit);
                if (converged(s)) continue;
                const MgScene& S = scenes[s];
                const MgLevel F = S.lv[l], C = S.lv[l + 1];
                const int u = unit - __ldg(off + s);
                const int cpr = mgRowChunks(F.nx);
                const int row = u / cpr, chunk = u - row * cpr;
                const int y = row % F.ny, z = row / F.ny;
                const int x = chunk * 32 + lane;
                if (x >= F.nx) continue;
                const float* pc = S.p[l + 1];
                auto loadC = [&](int j) { return __ldcg(pc + j); };
                const int i = mgAt(F, x, y, z);
                sc[k] = s;
                idx[k] = i;
                cur[k] = __ldcg(S.p[l] + i);
                add[k] = prolongAt(loadC, F, C, x, y, z);
            }
#pragma unroll
            for (int k = 0; k < U; ++k) {
                if (sc[k] >= 0) scenes[sc[k]].p[l][idx[k]] = cur[k] + add[k];
            }
        }
    };

    // Every scene starts unconverged with no cycles run, from a zero increment.
    for (int s = gwarp; s < n; s += nwarps) {
        if (lane == 0) *scenes[s].gate = SorGate{0, 0, 0.0f, 0, 0.0};
    }
    {
        const int total = __ldg(plan->allRows + n);
        for (int item = gwarp; item < total; item += nwarps) {
            const int s = sceneOf(plan->allRows, n, item);
            const MgScene& S = scenes[s];
            const int base = (item - __ldg(plan->allRows + s)) * S.lv[0].nx;
            for (int x = lane; x < S.lv[0].nx; x += 32) S.p[0][base + x] = 0.0f;
        }
    }
    if (!gridBarrier(sync, generation, waitNs, hostStatus, ++phase)) return;
    refreshRunning();
    for (int cycle = 0; cycle < maxCycles; ++cycle) {
        for (int l = 0; l < gridLevels; ++l) {
            for (int k = 0; k < 2 * pre; ++k) {
                smooth(l, k & 1);
                if (!gridBarrier(sync, generation, waitNs, hostStatus, ++phase)) return;
            }
            restrictTo(l);
            if (!gridBarrier(sync, generation, waitNs, hostStatus, ++phase)) return;
        }
        for (int s = blockIdx.x; s < n; s += gridDim.x) {
            if (!converged(s)) {
                const int mode = scenes[s].tailMode;
                if (mode == kMgTailShared) {
                    tailCycle<kMgTailShared>(scenes[s], pre, post, smem);
                } else if (mode == kMgTailRhsGlobal) {
                    tailCycle<kMgTailRhsGlobal>(scenes[s], pre, post, smem);
                } else {
                    tailCycle<kMgTailGlobal>(scenes[s], pre, post, smem);
                }
            }
            __syncthreads();
        }
        if (!gridBarrier(sync, generation, waitNs, hostStatus, ++phase)) return;
        for (int l = gridLevels - 1; l >= 0; --l) {
            prolongFrom(l);
            if (!gridBarrier(sync, generation, waitNs, hostStatus, ++phase)) return;
            for (int k = 0; k < 2 * post; ++k) {
                smooth(l, k & 1);
                if (!gridBarrier(sync, generation, waitNs, hostStatus, ++phase)) return;
            }
        }
        if (gated) {
            // Level-0 residual, one warp per chunk of rows (a fixed partition, so
            // the sums do not depend on the launch shape).
            const int total = __ldg(plan->chunks + n);
            for (int item = gwarp; item < total; item += nwarps) {
                const int s = sceneOf(plan->chunks, n, item);
                if (converged(s)) continue;
                const MgScene& S = scenes[s];
                const MgLevel L = S.lv[0];
                const float* p = S.p[0];
                auto load = [&](int j) { return __ldcg(p + j); };
                const int chunk = item - __ldg(plan->chunks + s);
                const int rows = L.ny * L.nz;
                // The chunk's cells in order (rows of x), lane-strided; no
                // stores in the loop, so the unrolled loads overlap.
                const int first = chunk * kMgChunkRows;
                const int count = (min(rows, first + kMgChunkRows) - first) * L.nx;
                double sq = 0.0;
                float mx = 0.0f;
#pragma unroll 4
                for (int j = lane; j < count; j += 32) {
                    const int row = first + j / L.nx, x = j - (j / L.nx) * L.nx;
                    const int y = row % L.ny, z = row / L.ny;
                    const int i = row * L.nx + x;
                    const float self = __ldcg(p + i);
                    const float r = weightedSum(load, __ldg(S.rhs[0] + i), L, i, x, y, z, self) - L.diag * self;
                    mx = fmaxf(mx, fabsf(r));
                    sq += static_cast<double>(r) * static_cast<double>(r);
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    sq += __shfl_xor_sync(0xffffffffu, sq, o);
                    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
                }
                if (lane == 0) {
                    S.chunkSq[chunk] = sq;
                    S.chunkMax[chunk] = mx;
                }
            }
            if (!gridBarrier(sync, generation, waitNs, hostStatus, ++phase)) return;
        }
        // Gate: one warp per scene that was still running this cycle.
        for (int s = gwarp; s < n; s += nwarps) {
            if (converged(s)) continue;
            const MgScene& S = scenes[s];
            if (gated) {
                const int first = __ldg(plan->chunks + s), count = __ldg(plan->chunks + s + 1) - first;
                double sq = 0.0;
                float mx = 0.0f;
                for (int c = lane; c < count; c += 32) {
                    sq += __ldcg(S.chunkSq + c);
                    mx = fmaxf(mx, __ldcg(S.chunkMax + c));
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    sq += __shfl_xor_sync(0xffffffffu, sq, o);
                    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
                }
                if (lane == 0) {
                    S.gate->maxResidual = mx;
                    S.gate->l2Residual = sqrt(sq);
                    S.gate->iterations = cycle + 1;
                    if (mx <= tolerance) S.gate->converged = 1;
                }
            } else if (lane == 0) {
                S.gate->maxResidual = -1.0f;
                S.gate->l2Residual = -1.0;
                S.gate->iterations = cycle + 1;
            }
        }
        if (!gridBarrier(sync, generation, waitNs, hostStatus, ++phase)) return;
        refreshRunning();
        if (threadIdx.x == 0) sActive = 0;
        __syncthreads();
        for (int s = threadIdx.x; s < n; s += blockDim.x) {
            if (!converged(s)) atomicOr(&sActive, 1);
        }
        __syncthreads();
        if (sActive == 0) break;
    }
    // pressure += delta on every cell of every scene.
    const int total = __ldg(plan->allRows + n);
    for (int item = gwarp; item < total; item += nwarps) {
        const int s = sceneOf(plan->allRows, n, item);
        const MgScene& S = scenes[s];
        const MgLevel L = S.lv[0];
        const int row = item - __ldg(plan->allRows + s);
        const int base = row * L.nx;
        for (int x = lane; x < L.nx; x += 32) S.pressure[base + x] = S.pressure[base + x] + __ldcg(S.p[0] + base + x);
    }
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
