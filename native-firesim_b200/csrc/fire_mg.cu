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
// separated by a grid barrier (a monotonic arrival count with release and
// acquire semantics) whose waits are bounded in time.  Within a phase, warps
// take the units of all scenes at that level from one work list.  A level's
// first colour-0 half sweep from p = 0 is written with its rhs (by the
// restriction, or the first phase for level 0 in the first cycle), as its
// arithmetic reduces to (rhs + 0) / diag there.
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

// Grid barrier of the persistent solve.  Thread 0 of each CTA adds its
// arrival to a monotonic count with release semantics (after __syncthreads,
// so the whole CTA's writes of the phase are published with it) and polls
// the count with acquire loads until every CTA has arrived at this barrier.
// Every wait gives up after waitNs (or a poll cap), marks the sync failed so
// the other CTAs stop too, and records the phase in the host-mapped status
// word.
__device__ __forceinline__ unsigned loadAcquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ bool gridBarrier(MgSync* sync, unsigned& generation, unsigned long long waitNs, unsigned* hostStatus, int phase) {
    __syncthreads();
    __shared__ int sFailed;
    if (threadIdx.x == 0) {
        const unsigned target = (generation + 1u) * gridDim.x;
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(&sync->count) : "memory");
        bool failed = false;
        const unsigned long long start = mgTimerNs();
        for (unsigned n = 0;; ++n) {
            if (loadAcquire(&sync->count) >= target) break;
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
            __nanosleep(20);
        }
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

// A tail level's cells as columns (x, y) along z: with at least as many
// columns as threads, thread t takes columns t, t + threads, ... whole;
// otherwise the columns are split along z into `zsplit` groups, thread t
// taking column t % cols and z group t / cols (every zsplit-th cell of the
// column, or of its cells of one colour).  Threads past cols * zsplit idle.
struct TailMap {
    int col, colStride, zg, zsplit;
    bool active;
};

__device__ __forceinline__ TailMap tailMap(int cols, int threads) {
    TailMap m;
    const int t = static_cast<int>(threadIdx.x);
    if (cols >= threads) {
        m.col = t;
        m.colStride = threads;
        m.zg = 0;
        m.zsplit = 1;
        m.active = t < threads;
    } else {
        m.zsplit = threads / cols;
        m.zg = t / cols;
        m.col = t - m.zg * cols;
        m.colStride = cols;
        m.active = m.zg < m.zsplit;
    }
    return m;
}

// `sweeps` red-black sweeps of a level of at most 32 cells by the first
// warp, a cell per lane, p in registers: the neighbours' values come by warp
// shuffles (a Neumann side reads the lane's own value), with the same
// arithmetic as weightedSum.
template <bool RG>
__device__ __forceinline__ void tailSmoothLanes(float* __restrict__ p, const float* __restrict__ rhs, const MgLevel L, int sweeps,
                                                bool skipFirst) {
    if (threadIdx.x < 32) {
        const int lane = static_cast<int>(threadIdx.x);
        const int plane = L.nx * L.ny;
        const bool own = lane < plane * L.nz;
        const int z = lane / plane, y = (lane - z * plane) / L.nx, x = lane - z * plane - y * L.nx;
        const int nL = own && x > 0 ? lane - 1 : lane;
        const int nR = own && x < L.nx - 1 ? lane + 1 : lane;
        const int nD = own && y > 0 ? lane - L.nx : lane;
        const int nU = own && y < L.ny - 1 ? lane + L.nx : lane;
        const int nB = own && z > 0 ? lane - plane : lane;
        const int nF = own && z < L.nz - 1 ? lane + plane : lane;
        const bool top = y == L.ny - 1;
        const int parity = (x + y + z) & 1;
        const float rh = own ? tailLoad<RG>(rhs, lane) : 0.0f;
        float v = own ? p[lane] : 0.0f;
        for (int s = 0; s < sweeps; ++s) {
            for (int colour = skipFirst && s == 0 ? 1 : 0; colour < 2; ++colour) {
                const float pL = __shfl_sync(0xffffffffu, v, nL);
                const float pR = __shfl_sync(0xffffffffu, v, nR);
                const float pD = __shfl_sync(0xffffffffu, v, nD);
                const float up = __shfl_sync(0xffffffffu, v, nU);
                const float pB = __shfl_sync(0xffffffffu, v, nB);
                const float pF = __shfl_sync(0xffffffffu, v, nF);
                const float pU = top ? 0.0f - v : up;
                const float next = combine(rh, pL, pR, pD, pU, pB, pF, L) * L.invDiag;
                if (own && parity == colour) v = next;
            }
        }
        if (own) p[lane] = v;
    }
    __syncthreads();
}

// `sweeps` red-black sweeps of one tail level.  A level of at most 32 cells
// goes to tailSmoothLanes; one of at most 128 cells is relaxed by the first
// warp alone, with warp barriers; otherwise by the whole CTA.  skipFirst:
// the first colour-0 half sweep was already done (from p = 0, by whoever
// wrote the level's rhs).
template <bool PG, bool RG>
__device__ __forceinline__ void tailSmooth(float* __restrict__ p, const float* __restrict__ rhs, const MgLevel L, int sweeps,
                                           bool skipFirst) {
    const int cols = L.nx * L.ny;
    if (!PG && cols * L.nz <= 32) {
        tailSmoothLanes<RG>(p, rhs, L, sweeps, skipFirst);
        return;
    }
    const bool warpOnly = cols * L.nz <= 4 * 32;
    auto load = [&](int j) { return tailLoad<PG>(p, j); };
    auto sync = [&]() {
        if constexpr (PG) __threadfence_block();
        if (warpOnly) {
            __syncwarp();
        } else {
            __syncthreads();
        }
    };
    if (!warpOnly || threadIdx.x < 32) {
        const TailMap m = tailMap(cols, warpOnly ? 32 : static_cast<int>(blockDim.x));
        if (m.colStride >= cols) {
            // At most one column per thread: its coordinates once.
            const int y = m.col / L.nx, x = m.col - y * L.nx;
            const int z0 = 2 * m.zg + ((x + y) & 1), dz = 2 * m.zsplit;
            for (int s = 0; s < sweeps; ++s) {
                for (int colour = skipFirst && s == 0 ? 1 : 0; colour < 2; ++colour) {
                    if (m.active) {
#pragma unroll 4
                        for (int z = z0 ^ colour; z < L.nz; z += dz) {
                            const int i = m.col + z * cols;
                            p[i] = weightedSum(load, tailLoad<RG>(rhs, i), L, i, x, y, z, load(i)) * L.invDiag;
                        }
                    }
                    sync();
                }
            }
        } else {
            for (int s = 0; s < sweeps; ++s) {
                for (int colour = skipFirst && s == 0 ? 1 : 0; colour < 2; ++colour) {
                    for (int col = m.col; col < cols; col += m.colStride) {
                        const int y = col / L.nx, x = col - y * L.nx;
#pragma unroll 4
                        for (int z = (colour + x + y) & 1; z < L.nz; z += 2) {
                            const int i = col + z * cols;
                            p[i] = weightedSum(load, tailLoad<RG>(rhs, i), L, i, x, y, z, load(i)) * L.invDiag;
                        }
                    }
                    sync();
                }
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
    auto residual = [&](int x, int y, int z) {
        const int i = mgAt(F, x, y, z);
        const float self = loadP(i);
        const float rh = rhsViaL2 ? __ldcg(rhsF + i) : rhsF[i];
        return weightedSum(loadP, rh, F, i, x, y, z, self) - F.diag * self;
    };
    auto rowMean = [&](int y, int z) {
        const float r0 = residual(x0, y, z);
        return C.cx ? 0.5f * (r0 + residual(x0 + 1, y, z)) : r0;
    };
    auto planeMean = [&](int z) {
        const float a0 = rowMean(y0, z);
        return C.cy ? 0.5f * (a0 + rowMean(y0 + 1, z)) : a0;
    };
    const float b0 = planeMean(z0);
    return C.cz ? 0.5f * (b0 + planeMean(z0 + 1)) : b0;
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
// level 0) and goes back to it at the end.  The levels' array addresses are
// kept in shared memory, so that no per-thread array holds them.
template <int MODE>
__device__ __forceinline__ void tailCycle(const MgScene& S, int pre, int post, float* smem) {
    constexpr bool PG = MODE == kMgTailGlobal;
    __shared__ float* sP[kMgMaxLevels];
    __shared__ float* sR[kMgMaxLevels];
    const int t = S.tail;
    const int last = S.levels - 1;
    if (threadIdx.x == 0) {
        int off = 0;
        for (int l = t; l <= last; ++l) {
            const int n = S.lv[l].nx * S.lv[l].ny * S.lv[l].nz;
            if (PG) {
                sP[l] = S.p[l];
                sR[l] = S.rhs[l];
            } else {
                sP[l] = smem + off;
                off += n;
                if (MODE == kMgTailRhsGlobal && l == t) {
                    sR[l] = S.rhs[l];
                } else {
                    sR[l] = smem + off;
                    off += n;
                }
            }
        }
    }
    __syncthreads();
    const int threads = static_cast<int>(blockDim.x);
    // A level whose p starts at 0 gets its first colour-0 half sweep where its
    // rhs is written: (rhs + 0) / diag on colour-0 cells, 0 elsewhere (every
    // neighbour sum is +0, so this is the half sweep's result to the bit).
    // That holds for every level below the tail level, and for the tail level
    // itself unless it is level 0 (whose p carries over between cycles).
    auto firstRed = [&](int l, int sweeps) { return sweeps > 0 && (l > t || t > 0); };
    {
        const MgLevel T = S.lv[t];
        const bool fuse = firstRed(t, t == last ? kMgCoarsestSweeps : pre);
        const int cols = T.nx * T.ny;
        const TailMap m = tailMap(cols, threads);
        if (m.active && (!PG || fuse)) {
            for (int col = m.col; col < cols; col += m.colStride) {
                const int y = col / T.nx, x = col - y * T.nx;
                for (int z = m.zg; z < T.nz; z += m.zsplit) {
                    const int i = col + z * cols;
                    const float r = __ldcg(S.rhs[t] + i);
                    if (MODE == kMgTailShared) sR[t][i] = r;
                    const float v = !fuse ? __ldcg(S.p[t] + i) : (((x + y + z) & 1) == 0 ? (r + 0.0f) * T.invDiag : 0.0f);
                    sP[t][i] = v;
                }
            }
        }
        if constexpr (PG) __threadfence_block();
        __syncthreads();
    }
    for (int l = t; l < last; ++l) {
        const MgLevel F = S.lv[l];
        const MgLevel C = S.lv[l + 1];
        const bool rg = PG || (MODE == kMgTailRhsGlobal && l == t);
        float* pf = sP[l];
        const float* rf = sR[l];
        if (rg) {
            tailSmooth<PG, true>(pf, rf, F, pre, firstRed(l, pre));
        } else {
            tailSmooth<PG, false>(pf, rf, F, pre, firstRed(l, pre));
        }
        const bool fuseC = firstRed(l + 1, l + 1 == last ? kMgCoarsestSweeps : pre);
        auto loadF = [&](int j) { return tailLoad<PG>(pf, j); };
        float* pc = sP[l + 1];
        float* rc = sR[l + 1];
        const int cols = C.nx * C.ny;
        const TailMap m = tailMap(cols, threads);
        if (m.active) {
            for (int col = m.col; col < cols; col += m.colStride) {
                const int Y = col / C.nx, X = col - Y * C.nx;
                for (int Z = m.zg; Z < C.nz; Z += m.zsplit) {
                    const int i = col + Z * cols;
                    const float r = restrictAt(loadF, rf, rg, F, C, X, Y, Z);
                    rc[i] = r;
                    pc[i] = fuseC && ((X + Y + Z) & 1) == 0 ? (r + 0.0f) * C.invDiag : 0.0f;
                }
            }
        }
        if constexpr (PG) __threadfence_block();
        __syncthreads();
    }
    {
        const MgLevel B = S.lv[last];
        const bool skip = firstRed(last, kMgCoarsestSweeps);
        if (PG || (MODE == kMgTailRhsGlobal && last == t)) {
            tailSmooth<PG, true>(sP[last], sR[last], B, kMgCoarsestSweeps, skip);
        } else {
            tailSmooth<PG, false>(sP[last], sR[last], B, kMgCoarsestSweeps, skip);
        }
    }
    for (int l = last - 1; l >= t; --l) {
        const MgLevel F = S.lv[l];
        const MgLevel C = S.lv[l + 1];
        float* pf = sP[l];
        const float* pc = sP[l + 1];
        auto loadC = [&](int j) { return tailLoad<PG>(pc, j); };
        const int cols = F.nx * F.ny;
        const TailMap m = tailMap(cols, threads);
        if (m.active) {
            for (int col = m.col; col < cols; col += m.colStride) {
                const int y = col / F.nx, x = col - y * F.nx;
                for (int z = m.zg; z < F.nz; z += m.zsplit) {
                    const int i = col + z * cols;
                    pf[i] = tailLoad<PG>(pf, i) + prolongAt(loadC, F, C, x, y, z);
                }
            }
        }
        if constexpr (PG) __threadfence_block();
        __syncthreads();
        if (PG || (MODE == kMgTailRhsGlobal && l == t)) {
            tailSmooth<PG, true>(pf, sR[l], F, post, false);
        } else {
            tailSmooth<PG, false>(pf, sR[l], F, post, false);
        }
    }
    if constexpr (!PG) {
        const int n0 = S.lv[t].nx * S.lv[t].ny * S.lv[t].nz;
        const float* p0 = sP[t];
        for (int i = threadIdx.x; i < n0; i += blockDim.x) S.p[t][i] = p0[i];
    }
}

// ---- quads: four consecutive cells of a row, one float4 per lane ----------
// Used where the row length is a multiple of 4 (rows, and so every quad,
// start 16-byte aligned).  A lane's edge neighbours (x0 - 1, x0 + 4) come from
// the lanes beside it by shuffles; lanes 0 and 31 load them.

__device__ __forceinline__ float4 ldcg4(const float* a) { return __ldcg(reinterpret_cast<const float4*>(a)); }
__device__ __forceinline__ float4 ldg4(const float* a) { return __ldg(reinterpret_cast<const float4*>(a)); }
__device__ __forceinline__ float at4(const float4& v, int e) { return e == 0 ? v.x : e == 1 ? v.y : e == 2 ? v.z : v.w; }

// The operands of a lane's quad: the quad, the quads below, above, behind
// and in front (the quad itself, or minus it above the top row, where the
// level has none), the rhs, and the values left and right of the quad.
struct Quad {
    float4 c, dn, up, bk, fr, rh;
    float left, right;
};

// The cells of a level whose row length is a multiple of 4 are taken in
// memory order, 128 per warp (a unit), four per lane: the lane's quad starts
// at flat index i and lies within one row.  quadLoad loads its operands; the
// values left and right of the quad come from the lanes beside it when they
// hold the same row (lanes 0 and 31 load them).  Every lane of the warp calls
// it (the shuffles are warp-wide); a lane past the level's end (live false)
// gets zeros.
__device__ __forceinline__ void quadLoad(Quad& q, const float* p, const float* rhs, bool rhsLdg, const MgLevel& L, int i, int x0, int y,
                                         int z, int lane, bool live) {
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const int plane = L.nx * L.ny;
    q.c = live ? ldcg4(p + i) : zero;
    q.dn = live && y > 0 ? ldcg4(p + i - L.nx) : zero;
    q.up = live && y < L.ny - 1 ? ldcg4(p + i + L.nx) : zero;
    q.bk = live && z > 0 ? ldcg4(p + i - plane) : zero;
    q.fr = live && z < L.nz - 1 ? ldcg4(p + i + plane) : zero;
    q.rh = live ? (rhsLdg ? ldg4(rhs + i) : ldcg4(rhs + i)) : zero;
    const float eL = lane == 0 && live && x0 > 0 ? __ldcg(p + i - 1) : 0.0f;
    const float eR = lane == 31 && live && x0 + 4 < L.nx ? __ldcg(p + i + 4) : 0.0f;
    q.left = __shfl_up_sync(0xffffffffu, q.c.w, 1);
    q.right = __shfl_down_sync(0xffffffffu, q.c.x, 1);
    if (lane == 0) q.left = eL;
    if (lane == 31) q.right = eR;
}

// weightedSum for cell e of a quad (same boundary rules and order).
__device__ __forceinline__ float quadSum(const MgLevel& L, const Quad& q, int e, int x, int y, int z) {
    const float self = at4(q.c, e);
    const float pL = x > 0 ? (e > 0 ? at4(q.c, e - 1) : q.left) : self;
    const float pR = x < L.nx - 1 ? (e < 3 ? at4(q.c, e + 1) : q.right) : self;
    const float pD = y > 0 ? at4(q.dn, e) : self;
    const float pU = y < L.ny - 1 ? at4(q.up, e) : 0.0f - self;
    const float pB = z > 0 ? at4(q.bk, e) : self;
    const float pF = z < L.nz - 1 ? at4(q.fr, e) : self;
    return combine(at4(q.rh, e), pL, pR, pD, pU, pB, pF, L);
}

// Asks L2 to fetch the line holding a (no register or shared memory holds
// the data; the load that follows finds it there).
__device__ __forceinline__ void prefetchLineL2(const float* a) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(__cvta_generic_to_global(a)));
}

// Coordinates of flat index i of a level.
__device__ __forceinline__ void flatCoords(const MgLevel& L, int i, int& x, int& y, int& z) {
    const int row = i / L.nx;
    x = i - row * L.nx;
    z = row / L.ny;
    y = row - z * L.ny;
}

}  // namespace

// The persistent batched solve (see the file comment).  Work items of the
// grid levels are units of one level of one scene (128 cells in memory order,
// a quad per lane, where the row length is a multiple of 4; else chunks of
// one row), one warp per unit; the tail is one CTA per scene; the residual is
// one warp per chunk (mgResidualChunks); every CTA decides convergence from
// the per-scene maxima, and one CTA per scene writes its gate record at the
// end.
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
    unsigned generation = 0;
    int phase = 0;
    // The scenes still running, with the cycles run and the last cycle's max
    // |r| of each: every CTA keeps the same copy, updated from the per-scene
    // maxima in sync after each cycle's residual phase (no gate phase).
    __shared__ unsigned char sRunning[kMgMaxScenes];
    __shared__ int sCycles[kMgMaxScenes];
    __shared__ float sMax[kMgMaxScenes];
    for (int s = threadIdx.x; s < n; s += blockDim.x) {
        sRunning[s] = 1;
        sCycles[s] = 0;
        sMax[s] = -1.0f;
    }
    __syncthreads();
    auto converged = [&](int s) { return sRunning[s] == 0; };
    // One colour of red-black Gauss-Seidel on level l of every scene that has
    // it as a grid level.  Where the row length is a multiple of 4, a unit is
    // 128 consecutive cells in memory (several short rows, or part of a long
    // one), four per lane: each lane updates the two of its four cells of the
    // colour and stores all four (the other two unchanged: no thread writes
    // them in this phase).  Otherwise a unit is a 128-cell chunk of one row,
    // taken cell by cell.
    auto smooth = [&](int l, int colour) {
        const int* off = plan->smoothUnits[l];
        const int total = __ldg(off + n);
        for (int unit = gwarp; unit < total; unit += nwarps) {
            const int s = sceneOf(off, n, unit);
            if (converged(s)) continue;
            const MgScene& S = scenes[s];
            const MgLevel L = S.lv[l];
            const int u = unit - __ldg(off + s);
            float* p = S.p[l];
            const float* rhs = S.rhs[l];
            if ((L.nx & 3) == 0) {
                const int i = u * 128 + 4 * lane;
                const bool live = i < L.nx * L.ny * L.nz;
                // Ask L2 for this lane's cells of the warp's next unit (when it
                // is in the same scene), so that its loads find them there.
                const int ahead = i + nwarps * 128;
                if (ahead < L.nx * L.ny * L.nz) {
                    prefetchLineL2(rhs + ahead);
                    prefetchLineL2(p + ahead);
                }
                int x0, y, z;
                flatCoords(L, live ? i : 0, x0, y, z);
                Quad q;
                quadLoad(q, p, rhs, l == 0, L, i, x0, y, z, lane, live);
                if (!live) continue;
                const int e0 = (colour + x0 + y + z) & 1;  // the colour's cells are e0 and e0 + 2
                const float a = quadSum(L, q, e0, x0 + e0, y, z) * L.invDiag;
                const float b = quadSum(L, q, e0 + 2, x0 + e0 + 2, y, z) * L.invDiag;
                float4 o = q.c;
                if (e0 == 0) {
                    o.x = a;
                    o.z = b;
                } else {
                    o.y = a;
                    o.w = b;
                }
                *reinterpret_cast<float4*>(p + i) = o;
            } else {
                const int cpr = mgQuadChunks(L.nx);
                const int row = u / cpr, chunk = u - row * cpr;
                const int y = row % L.ny, z = row / L.ny;
                const int base = row * L.nx;
                auto load = [&](int j) { return __ldcg(p + j); };
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int x = chunk * 128 + 4 * lane + e;
                    if (x >= L.nx || ((colour + x + y + z) & 1) != 0) continue;
                    const int i = base + x;
                    const float rh = l == 0 ? __ldg(rhs + i) : __ldcg(rhs + i);
                    p[i] = weightedSum(load, rh, L, i, x, y, z, load(i)) * L.invDiag;
                }
            }
        }
    };
    // Coarse rhs = the mean residual of the covered fine cells, and coarse p
    // = 0, or, when `red` (the coarse level is a grid level whose
    // pre-smoothing starts with the colour-0 half sweep), that half sweep's
    // result from p = 0: (rhs + 0) / diag on colour-0 cells (every neighbour
    // sum is +0, so the sweep's arithmetic reduces to this exactly) and 0 on
    // the others.  Where the fine row length is a multiple of 4, a unit is 64
    // consecutive coarse cells in memory, two per lane, whose fine quad is
    // loaded row by row (quadLoad) for each of the fine rows covered;
    // otherwise a unit is a 32-cell chunk of a coarse row, a cell per lane.
    auto restrictTo = [&](int l, bool redFirst) {
        const int* off = plan->coarseUnits[l];
        const int total = __ldg(off + n);
        for (int unit = gwarp; unit < total; unit += nwarps) {
            const int s = sceneOf(off, n, unit);
            if (converged(s)) continue;
            const MgScene& S = scenes[s];
            const MgLevel F = S.lv[l], C = S.lv[l + 1];
            const bool red = redFirst && l + 1 < S.tail;
            const int u = unit - __ldg(off + s);
            const float* pf = S.p[l];
            const float* rf = S.rhs[l];
            if ((F.nx & 3) == 0) {
                const int j = u * 64 + 2 * lane;
                const bool live = j < C.nx * C.ny * C.nz;
                int X0, Y, Z;
                flatCoords(C, live ? j : 0, X0, Y, Z);
                const int x0 = 2 * X0;
                float az[2][2] = {{0.0f, 0.0f}, {0.0f, 0.0f}};
#pragma unroll
                for (int dz = 0; dz < 2; ++dz) {
                    if (dz > C.cz) break;
                    float ay[2][2] = {{0.0f, 0.0f}, {0.0f, 0.0f}};
#pragma unroll
                    for (int dy = 0; dy < 2; ++dy) {
                        if (dy > C.cy) break;
                        const int y = C.cy ? 2 * Y + dy : Y, z = C.cz ? 2 * Z + dz : Z;
                        const int i = (z * F.ny + y) * F.nx + x0;
                        Quad q;
                        quadLoad(q, pf, rf, l == 0, F, i, x0, y, z, lane, live);
                        float r[4];
#pragma unroll
                        for (int e = 0; e < 4; ++e) r[e] = quadSum(F, q, e, x0 + e, y, z) - F.diag * at4(q.c, e);
                        ay[dy][0] = 0.5f * (r[0] + r[1]);
                        ay[dy][1] = 0.5f * (r[2] + r[3]);
                    }
#pragma unroll
                    for (int k = 0; k < 2; ++k) az[dz][k] = C.cy ? 0.5f * (ay[0][k] + ay[1][k]) : ay[0][k];
                }
                if (!live) continue;
                float rc[2], pc[2];
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    rc[k] = C.cz ? 0.5f * (az[0][k] + az[1][k]) : az[0][k];
                    pc[k] = red && ((X0 + k + Y + Z) & 1) == 0 ? (rc[k] + 0.0f) * C.invDiag : 0.0f;
                }
                *reinterpret_cast<float2*>(S.rhs[l + 1] + j) = make_float2(rc[0], rc[1]);
                *reinterpret_cast<float2*>(S.p[l + 1] + j) = make_float2(pc[0], pc[1]);
            } else {
                const int cpr = mgRowChunks(C.nx);
                const int row = u / cpr, chunk = u - row * cpr;
                const int Y = row % C.ny, Z = row / C.ny;
                const int X = chunk * 32 + lane;
                if (X >= C.nx) continue;
                auto loadF = [&](int k) { return __ldcg(pf + k); };
                const int c = mgAt(C, X, Y, Z);
                const float r = restrictAt(loadF, rf, l > 0, F, C, X, Y, Z);
                S.rhs[l + 1][c] = r;
                S.p[l + 1][c] = red && ((X + Y + Z) & 1) == 0 ? (r + 0.0f) * C.invDiag : 0.0f;
            }
        }
    };
    // p += the interpolated coarse correction.  Where the fine row length is
    // a multiple of 4, units are 128 consecutive fine cells in memory, a quad
    // per lane: for each of the four coarse rows the quad interpolates from,
    // the lane loads the coarse values at x0/2 and x0/2 + 1 and takes those
    // at x0/2 - 1 and x0/2 + 2 from the lanes beside it (clamped at the row's
    // ends).  Otherwise a unit is a 32-cell chunk of a row, a cell per lane.
    auto prolongFrom = [&](int l) {
        const int* off = plan->fineUnits[l];
        const int total = __ldg(off + n);
        for (int unit = gwarp; unit < total; unit += nwarps) {
            const int s = sceneOf(off, n, unit);
            if (converged(s)) continue;
            const MgScene& S = scenes[s];
            const MgLevel F = S.lv[l], C = S.lv[l + 1];
            const int u = unit - __ldg(off + s);
            float* pf = S.p[l];
            const float* pc = S.p[l + 1];
            if ((F.nx & 3) == 0) {
                const int i = u * 128 + 4 * lane;
                const bool live = i < F.nx * F.ny * F.nz;
                int x0, y, z;
                flatCoords(F, live ? i : 0, x0, y, z);
                const int Y0 = C.cy ? y >> 1 : y, Z0 = C.cz ? z >> 1 : z;
                const int Y1 = !C.cy ? Y0 : ((y & 1) ? min(Y0 + 1, C.ny - 1) : max(Y0 - 1, 0));
                const int Z1 = !C.cz ? Z0 : ((z & 1) ? min(Z0 + 1, C.nz - 1) : max(Z0 - 1, 0));
                const float4 cur = live ? ldcg4(pf + i) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                // v[k][e] = the coarse values at X0 and X1 of fine cell e in
                // coarse row k: (Y0, Z0), (Y1, Z0), (Y0, Z1), (Y1, Z1).
                float v[4][4][2];
                const bool sameRowLeft = lane > 0 && x0 > 0, sameRowRight = lane < 31 && x0 + 4 < F.nx;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int base = ((k >> 1 ? Z1 : Z0) * C.ny + (k & 1 ? Y1 : Y0)) * C.nx;
                    if (C.cx) {
                        const int b = x0 >> 1;  // coarse x of fine x0 and x0 + 1; b + 1 of x0 + 2 and x0 + 3
                        float2 bc = make_float2(0.0f, 0.0f);
                        if (live) bc = __ldcg(reinterpret_cast<const float2*>(pc + base + b));
                        float a = __shfl_up_sync(0xffffffffu, bc.y, 1);    // b - 1
                        float d = __shfl_down_sync(0xffffffffu, bc.x, 1);  // b + 2
                        if (!sameRowLeft) a = live && x0 > 0 ? __ldcg(pc + base + b - 1) : bc.x;
                        if (!sameRowRight) d = live && x0 + 4 < F.nx ? __ldcg(pc + base + b + 2) : bc.y;
                        v[k][0][0] = bc.x;
                        v[k][0][1] = a;
                        v[k][1][0] = bc.x;
                        v[k][1][1] = bc.y;
                        v[k][2][0] = bc.y;
                        v[k][2][1] = bc.x;
                        v[k][3][0] = bc.y;
                        v[k][3][1] = d;
                    } else {
                        float4 w = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                        if (live) w = ldcg4(pc + base + x0);
#pragma unroll
                        for (int e = 0; e < 4; ++e) v[k][e][0] = v[k][e][1] = at4(w, e);
                    }
                }
                if (!live) continue;
                const float ux = C.cx ? 0.75f : 1.0f, vx = C.cx ? 0.25f : 0.0f;
                const float uy = C.cy ? 0.75f : 1.0f, vy = C.cy ? 0.25f : 0.0f;
                const float uz = C.cz ? 0.75f : 1.0f, vz = C.cz ? 0.25f : 0.0f;
                float out[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const float a0 = ux * v[0][e][0] + vx * v[0][e][1];
                    const float a1 = ux * v[1][e][0] + vx * v[1][e][1];
                    const float a2 = ux * v[2][e][0] + vx * v[2][e][1];
                    const float a3 = ux * v[3][e][0] + vx * v[3][e][1];
                    const float b0 = uy * a0 + vy * a1, b1 = uy * a2 + vy * a3;
                    out[e] = at4(cur, e) + (uz * b0 + vz * b1);
                }
                *reinterpret_cast<float4*>(pf + i) = make_float4(out[0], out[1], out[2], out[3]);
            } else {
                const int cpr = mgRowChunks(F.nx);
                const int row = u / cpr, chunk = u - row * cpr;
                const int y = row % F.ny, z = row / F.ny;
                const int x = chunk * 32 + lane;
                if (x >= F.nx) continue;
                auto loadC = [&](int j) { return __ldcg(pc + j); };
                const int i = mgAt(F, x, y, z);
                pf[i] = __ldcg(pf + i) + prolongAt(loadC, F, C, x, y, z);
            }
        }
    };

    // Every scene starts from a zero increment.  With pre-smoothing, the
    // first cycle's colour-0 half sweep of level 0 is done here, as in
    // restrictTo: (rhs + 0) / diag on colour-0 cells, 0 elsewhere (scenes
    // whose level 0 is in the tail start from 0).  Units as the smoothing's.
    const bool redFirst = pre > 0;
    {
        const int total = __ldg(plan->allUnits + n);
        for (int unit = gwarp; unit < total; unit += nwarps) {
            const int s = sceneOf(plan->allUnits, n, unit);
            const MgScene& S = scenes[s];
            const MgLevel L = S.lv[0];
            const int u = unit - __ldg(plan->allUnits + s);
            const bool red = redFirst && S.tail > 0;
            float* p = S.p[0];
            const float* rhs = S.rhs[0];
            if ((L.nx & 3) == 0) {
                const int i = u * 128 + 4 * lane;
                if (i >= L.nx * L.ny * L.nz) continue;
                int x0, y, z;
                flatCoords(L, i, x0, y, z);
                float4 o = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                if (red) {
                    const float4 r = ldg4(rhs + i);
                    const int e0 = (x0 + y + z) & 1;  // colour-0 cells: e0 and e0 + 2
                    if (e0 == 0) {
                        o.x = (r.x + 0.0f) * L.invDiag;
                        o.z = (r.z + 0.0f) * L.invDiag;
                    } else {
                        o.y = (r.y + 0.0f) * L.invDiag;
                        o.w = (r.w + 0.0f) * L.invDiag;
                    }
                }
                *reinterpret_cast<float4*>(p + i) = o;
            } else {
                const int cpr = mgQuadChunks(L.nx);
                const int row = u / cpr, chunk = u - row * cpr;
                const int y = row % L.ny, z = row / L.ny;
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int x = chunk * 128 + 4 * lane + e;
                    if (x >= L.nx) continue;
                    const int i = row * L.nx + x;
                    p[i] = red && ((x + y + z) & 1) == 0 ? (__ldg(rhs + i) + 0.0f) * L.invDiag : 0.0f;
                }
            }
        }
    }
    if (!gridBarrier(sync, generation, waitNs, hostStatus, ++phase)) return;
    for (int cycle = 0; cycle < maxCycles; ++cycle) {
        for (int l = 0; l < gridLevels; ++l) {
            // The colour-0 half sweep of a coarse level, and of level 0 in the
            // first cycle, was done with the restriction (the initialisation).
            for (int k = redFirst && (l > 0 || cycle == 0) ? 1 : 0; k < 2 * pre; ++k) {
                smooth(l, k & 1);
                if (!gridBarrier(sync, generation, waitNs, hostStatus, ++phase)) return;
            }
            restrictTo(l, redFirst);
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
            // Level-0 residual, one warp per chunk (mgResidualChunk: a fixed
            // partition of each scene's cells, so the sums do not depend on
            // the launch shape or the batch).  Where the row length is a
            // multiple of 4 a chunk is kMgChunkUnits 128-cell units in memory
            // order, a quad per lane; otherwise kMgChunkRows rows, a cell per
            // lane.  A lane sums its cells in order, then the warp by a
            // shuffle tree.
            const int total = __ldg(plan->chunks + n);
            for (int item = gwarp; item < total; item += nwarps) {
                const int s = sceneOf(plan->chunks, n, item);
                if (converged(s)) continue;
                const MgScene& S = scenes[s];
                const MgLevel L = S.lv[0];
                const float* p = S.p[0];
                const float* rhs = S.rhs[0];
                const int chunk = item - __ldg(plan->chunks + s);
                double sq = 0.0;
                float mx = 0.0f;
                auto accumulate = [&](float r) {
                    mx = fmaxf(mx, fabsf(r));
                    sq += static_cast<double>(r) * static_cast<double>(r);
                };
                if ((L.nx & 3) == 0) {
                    const int cells = L.nx * L.ny * L.nz;
#pragma unroll 1
                    for (int k = 0; k < kMgChunkUnits; ++k) {
                        const int i = (chunk * kMgChunkUnits + k) * 128 + 4 * lane;
                        if (i - 4 * lane >= cells) break;
                        const bool live = i < cells;
                        int x0, y, z;
                        flatCoords(L, live ? i : 0, x0, y, z);
                        Quad q;
                        quadLoad(q, p, rhs, true, L, i, x0, y, z, lane, live);
                        if (live) {
#pragma unroll
                            for (int e = 0; e < 4; ++e) accumulate(quadSum(L, q, e, x0 + e, y, z) - L.diag * at4(q.c, e));
                        }
                    }
                } else {
                    auto load = [&](int j) { return __ldcg(p + j); };
                    const int rows = L.ny * L.nz;
                    const int first = chunk * kMgChunkRows;
                    const int count = (min(rows, first + kMgChunkRows) - first) * L.nx;
#pragma unroll 4
                    for (int j = lane; j < count; j += 32) {
                        const int row = first + j / L.nx, x = j - (j / L.nx) * L.nx;
                        const int y = row % L.ny, z = row / L.ny;
                        const int i = row * L.nx + x;
                        const float self = __ldcg(p + i);
                        accumulate(weightedSum(load, __ldg(rhs + i), L, i, x, y, z, self) - L.diag * self);
                    }
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    sq += __shfl_xor_sync(0xffffffffu, sq, o);
                    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
                }
                if (lane == 0) {
                    S.chunkSq[chunk] = sq;
                    atomicMax(&sync->sceneMax[cycle & 1][s], __float_as_uint(mx));  // mx >= 0: its bits order as the value
                }
            }
            // The other row of per-scene maxima, last read after the previous
            // cycle's residual (several barriers ago), is cleared for the next.
            if (blockIdx.x == 0) {
                for (int s = threadIdx.x; s < n; s += blockDim.x) sync->sceneMax[(cycle + 1) & 1][s] = 0u;
            }
            if (!gridBarrier(sync, generation, waitNs, hostStatus, ++phase)) return;
        }
        // Convergence, the same in every CTA: a scene still running has run
        // this cycle; with a tolerance, it stops once its max |r| is within it.
        for (int s = threadIdx.x; s < n; s += blockDim.x) {
            if (!sRunning[s]) continue;
            sCycles[s] = cycle + 1;
            if (gated) {
                const float m = __uint_as_float(__ldcg(&sync->sceneMax[cycle & 1][s]));
                sMax[s] = m;
                if (m <= tolerance) sRunning[s] = 0;
            }
        }
        if (threadIdx.x == 0) sActive = 0;
        __syncthreads();
        for (int s = threadIdx.x; s < n; s += blockDim.x) {
            if (!converged(s)) atomicOr(&sActive, 1);
        }
        __syncthreads();
        if (sActive == 0) break;
    }
    // Each scene's gate, by CTA s % gridDim.x: the cycles run, the last
    // cycle's max |r| and sqrt(sum r^2) of its chunks (summed in a fixed
    // order: thread t takes chunks t, t + blockDim.x, ..., then shuffle trees
    // over each warp and over the warps).
    __shared__ double sSum[kMgThreads / 32];
    for (int s = blockIdx.x; s < n; s += gridDim.x) {
        const MgScene& S = scenes[s];
        double sq = 0.0;
        if (gated) {
            const int first = __ldg(plan->chunks + s), count = __ldg(plan->chunks + s + 1) - first;
            for (int c = threadIdx.x; c < count; c += blockDim.x) sq += __ldcg(S.chunkSq + c);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
        if (lane == 0) sSum[threadIdx.x >> 5] = sq;
        __syncthreads();
        if (threadIdx.x < 32) {
            sq = static_cast<int>(threadIdx.x) < warpsPerBlock ? sSum[threadIdx.x] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
            if (threadIdx.x == 0) {
                S.gate->iterations = sCycles[s];
                S.gate->maxResidual = gated ? sMax[s] : -1.0f;
                S.gate->l2Residual = gated ? sqrt(sq) : -1.0;
                S.gate->converged = gated && sMax[s] >= 0.0f && sMax[s] <= tolerance ? 1 : 0;
            }
        }
        __syncthreads();
    }
    // pressure += delta on every cell of every scene (units as the smoothing's).
    const int total = __ldg(plan->allUnits + n);
    for (int unit = gwarp; unit < total; unit += nwarps) {
        const int s = sceneOf(plan->allUnits, n, unit);
        const MgScene& S = scenes[s];
        const MgLevel L = S.lv[0];
        const int u = unit - __ldg(plan->allUnits + s);
        if ((L.nx & 3) == 0) {
            const int i = u * 128 + 4 * lane;
            if (i >= L.nx * L.ny * L.nz) continue;
            const float4 p = *reinterpret_cast<const float4*>(S.pressure + i);
            const float4 d = ldcg4(S.p[0] + i);
            *reinterpret_cast<float4*>(S.pressure + i) = make_float4(p.x + d.x, p.y + d.y, p.z + d.z, p.w + d.w);
        } else {
            const int cpr = mgQuadChunks(L.nx);
            const int row = u / cpr, chunk = u - row * cpr;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int x = chunk * 128 + 4 * lane + e;
                if (x >= L.nx) continue;
                const int i = row * L.nx + x;
                S.pressure[i] = S.pressure[i] + __ldcg(S.p[0] + i);
            }
        }
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
