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
// In shared memory (kGlobal false) or, for a tail too large for it, in the
// levels' own global buffers (kGlobal true, read through L2).

template <bool kGlobal>
__device__ __forceinline__ float tailLoad(const float* a, int i) {
    if constexpr (kGlobal) {
        return __ldcg(a + i);
    } else {
        return a[i];
    }
}

template <bool kGlobal>
__device__ void tailSmooth(float* p, const float* rhs, const MgLevel& L, int sweeps) {
    const int cells = L.nx * L.ny * L.nz;
    auto load = [&](int j) { return tailLoad<kGlobal>(p, j); };
    for (int s = 0; s < sweeps; ++s) {
        for (int colour = 0; colour < 2; ++colour) {
            if (cells <= 4 * 32) {
                // A tiny level: the first warp alone, with warp barriers.
                if (threadIdx.x < 32) {
                    for (int i = threadIdx.x; i < cells; i += 32) {
                        const int x = i % L.nx, y = (i / L.nx) % L.ny, z = i / (L.nx * L.ny);
                        if (((x + y + z) & 1) == colour) {
                            p[i] = weightedSum(load, tailLoad<kGlobal>(rhs, i), L, i, x, y, z, load(i)) * L.invDiag;
                        }
                    }
                    if constexpr (kGlobal) __threadfence_block();
                    __syncwarp();
                }
            } else {
                for (int i = threadIdx.x; i < cells; i += blockDim.x) {
                    const int x = i % L.nx, y = (i / L.nx) % L.ny, z = i / (L.nx * L.ny);
                    if (((x + y + z) & 1) == colour) {
                        p[i] = weightedSum(load, tailLoad<kGlobal>(rhs, i), L, i, x, y, z, load(i)) * L.invDiag;
                    }
                }
                if constexpr (kGlobal) __threadfence_block();
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

// The V-cycle of levels tail..levels-1 of scene S by this CTA.  In shared
// memory, rhs and p of the tail level come from global memory (p is zero
// there unless the tail is level 0), everything below lives in shared memory,
// and the tail level's p goes back to global memory.
template <bool kGlobal>
__device__ void tailCycle(const MgScene& S, int pre, int post, float* smem) {
    const int t = S.tail;
    float* p[kMgMaxLevels];
    float* r[kMgMaxLevels];
    int off = 0;
    for (int l = t; l < S.levels; ++l) {
        const int n = S.lv[l].nx * S.lv[l].ny * S.lv[l].nz;
        if constexpr (kGlobal) {
            p[l] = S.p[l];
            r[l] = S.rhs[l];
        } else {
            p[l] = smem + off;
            r[l] = smem + off + n;
        }
        off += 2 * n;
    }
    const MgLevel& T0 = S.lv[t];
    const int n0 = T0.nx * T0.ny * T0.nz;
    if constexpr (!kGlobal) {
        for (int i = threadIdx.x; i < n0; i += blockDim.x) {
            p[t][i] = __ldcg(S.p[t] + i);
            r[t][i] = __ldcg(S.rhs[t] + i);
        }
    }
    __syncthreads();
    const int last = S.levels - 1;
    for (int l = t; l < last; ++l) {
        const MgLevel& F = S.lv[l];
        const MgLevel& C = S.lv[l + 1];
        tailSmooth<kGlobal>(p[l], r[l], F, pre);
        const float* pf = p[l];
        auto loadF = [&](int j) { return tailLoad<kGlobal>(pf, j); };
        const int nc = C.nx * C.ny * C.nz;
        for (int i = threadIdx.x; i < nc; i += blockDim.x) {
            const int X = i % C.nx, Y = (i / C.nx) % C.ny, Z = i / (C.nx * C.ny);
            r[l + 1][i] = restrictAt(loadF, r[l], kGlobal, F, C, X, Y, Z);
            p[l + 1][i] = 0.0f;
        }
        if constexpr (kGlobal) __threadfence_block();
        __syncthreads();
    }
    tailSmooth<kGlobal>(p[last], r[last], S.lv[last], kMgCoarsestSweeps);
    for (int l = last - 1; l >= t; --l) {
        const MgLevel& F = S.lv[l];
        const MgLevel& C = S.lv[l + 1];
        const float* pc = p[l + 1];
        auto loadC = [&](int j) { return tailLoad<kGlobal>(pc, j); };
        const int nf = F.nx * F.ny * F.nz;
        for (int i = threadIdx.x; i < nf; i += blockDim.x) {
            const int x = i % F.nx, y = (i / F.nx) % F.ny, z = i / (F.nx * F.ny);
            p[l][i] = tailLoad<kGlobal>(p[l], i) + prolongAt(loadC, F, C, x, y, z);
        }
        if constexpr (kGlobal) __threadfence_block();
        __syncthreads();
        tailSmooth<kGlobal>(p[l], r[l], F, post);
    }
    if constexpr (!kGlobal) {
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
    auto converged = [&](int s) { return loadVolatileI(&scenes[s].gate->converged) != 0; };

    // One colour of red-black Gauss-Seidel on level l of every scene that has it as a grid level.
    auto smooth = [&](int l, int colour) {
        const int* off = plan->rows[l];
        const int total = __ldg(off + n);
        for (int item = gwarp; item < total; item += nwarps) {
            const int s = sceneOf(off, n, item);
            if (converged(s)) continue;
            const MgScene& S = scenes[s];
            const MgLevel L = S.lv[l];
            float* p = S.p[l];
            const float* rhs = S.rhs[l];
            const int row = item - __ldg(off + s);
            const int y = row % L.ny, z = row / L.ny;
            auto load = [&](int j) { return __ldcg(p + j); };
            for (int x = 2 * lane + ((colour + y + z) & 1); x < L.nx; x += 64) {
                const int i = mgAt(L, x, y, z);
                const float rh = l == 0 ? __ldg(rhs + i) : __ldcg(rhs + i);
                p[i] = weightedSum(load, rh, L, i, x, y, z, __ldcg(p + i)) * L.invDiag;
            }
        }
    };
    auto restrictTo = [&](int l) {
        const int* off = plan->coarseRows[l];
        const int total = __ldg(off + n);
        for (int item = gwarp; item < total; item += nwarps) {
            const int s = sceneOf(off, n, item);
            if (converged(s)) continue;
            const MgScene& S = scenes[s];
            const MgLevel F = S.lv[l], C = S.lv[l + 1];
            const float* pf = S.p[l];
            auto loadF = [&](int j) { return __ldcg(pf + j); };
            const int row = item - __ldg(off + s);
            const int Y = row % C.ny, Z = row / C.ny;
            for (int X = lane; X < C.nx; X += 32) {
                const int c = mgAt(C, X, Y, Z);
                S.rhs[l + 1][c] = restrictAt(loadF, S.rhs[l], l > 0, F, C, X, Y, Z);
                S.p[l + 1][c] = 0.0f;
            }
        }
    };
    auto prolongFrom = [&](int l) {
        const int* off = plan->rows[l];
        const int total = __ldg(off + n);
        for (int item = gwarp; item < total; item += nwarps) {
            const int s = sceneOf(off, n, item);
            if (converged(s)) continue;
            const MgScene& S = scenes[s];
            const MgLevel F = S.lv[l], C = S.lv[l + 1];
            const float* pc = S.p[l + 1];
            auto loadC = [&](int j) { return __ldcg(pc + j); };
            float* pf = S.p[l];
            const int row = item - __ldg(off + s);
            const int y = row % F.ny, z = row / F.ny;
            for (int x = lane; x < F.nx; x += 32) {
                const int i = mgAt(F, x, y, z);
                pf[i] = __ldcg(pf + i) + prolongAt(loadC, F, C, x, y, z);
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
                if (scenes[s].tailInGlobal) {
                    tailCycle<true>(scenes[s], pre, post, smem);
                } else {
                    tailCycle<false>(scenes[s], pre, post, smem);
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
                double sq = 0.0;
                float mx = 0.0f;
                for (int row = chunk * kMgChunkRows; row < min(rows, (chunk + 1) * kMgChunkRows); ++row) {
                    const int y = row % L.ny, z = row / L.ny;
                    for (int x = lane; x < L.nx; x += 32) {
                        const int i = mgAt(L, x, y, z);
                        const float self = __ldcg(p + i);
                        const float r = weightedSum(load, __ldg(S.rhs[0] + i), L, i, x, y, z, self) - L.diag * self;
                        mx = fmaxf(mx, fabsf(r));
                        sq += static_cast<double>(r) * static_cast<double>(r);
                    }
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
