// fire_noalloc.cu -- the force pass for callers that cannot allocate device memory.
//
// The regular force pass (Scene::runStages, stages FORCE..DIVERGENCE) keeps its
// per-cell force increments in a buffer the scene allocated with cudaMalloc.
// Some callers cannot let a library allocate: an engine that owns every byte
// of device memory through its own arena, a caller capturing its frame into a
// CUDA graph (cudaMalloc is not capturable), or a plugin whose host forbids
// third-party allocations after start-up.  fireCudaForceProjectNoAlloc runs
// the same two kernels (forceContributions, forceProjectSetup) on buffers the
// caller owns, and keeps the increments in the fixed array below instead.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <string>

#include "../../include/fire_ext.h"
#include "fire_scene.h"

namespace {

// Per-cell force increments (du, dv, dw, unused) for at most kNoAllocMaxCells
// cells: 16 MiB, held by every GPU that loads the library until the process exits.
constexpr int kNoAllocMaxCells = 1 << 20;
static __device__ __align__(256) float4 g_forceScratch[kNoAllocMaxCells];

// Device address of g_forceScratch per device ordinal.  In host code the
// symbol is only a host-side stand-in, so the address is resolved with
// cudaGetSymbolAddress on each device, once, while that device is current.
// Several host threads may resolve it at once; they store the same value, and
// the atomics keep that free of data races.  A cudaDeviceReset (or a reset of
// the primary context) unloads the module, so the cached address is stale
// after one: a process that resets a device must reload the library.
constexpr int kMaxDevices = 64;
std::atomic<float4*> g_scratchAddress[kMaxDevices] = {};

}  // namespace

namespace firesim {
void setLastErrorMessage(const char* msg);
}  // namespace firesim

namespace {

bool fail(const std::string& msg) {
    firesim::setLastErrorMessage(msg.c_str());
    return false;
}

}  // namespace

extern "C" bool fireCudaForceProjectNoAlloc(const FireSettings* settings, float time, int nx, int ny, int nz,
                                            const void* recordsA, const void* recordsB, const void* recordsC,
                                            const float* u, const float* v, const float* w, float* uOut, float* vOut,
                                            float* wOut, float* divergence, float* pressure, void* stream) {
    if (settings == nullptr || recordsA == nullptr || recordsB == nullptr || recordsC == nullptr || u == nullptr ||
        v == nullptr || w == nullptr || uOut == nullptr || vOut == nullptr || wOut == nullptr || divergence == nullptr ||
        pressure == nullptr) {
        return fail("fireCudaForceProjectNoAlloc: a pointer argument was null.");
    }
    if (nx < 2 || ny < 2 || nz < 2) {
        return fail("fireCudaForceProjectNoAlloc: grid dimensions must be at least 2.");
    }
    // The launch grid is (ceil(nx / block), ny, nz): y and z are capped at 65535 blocks.
    if (ny > 65535 || nz > 65535) {
        return fail("fireCudaForceProjectNoAlloc: ny and nz must be at most 65535.");
    }
    const long long cells = static_cast<long long>(nx) * ny * nz;
    if (cells > kNoAllocMaxCells) {
        char buf[200];
        std::snprintf(buf, sizeof(buf),
                      "fireCudaForceProjectNoAlloc: grid of %lld cells exceeds the %d-cell scratch of this entry point.",
                      cells, kNoAllocMaxCells);
        return fail(buf);
    }
    if ((reinterpret_cast<uintptr_t>(recordsA) & 15) != 0 || (reinterpret_cast<uintptr_t>(recordsB) & 15) != 0 ||
        (reinterpret_cast<uintptr_t>(recordsC) & 7) != 0) {
        return fail("fireCudaForceProjectNoAlloc: records A/B must be 16-byte aligned and records C 8-byte aligned.");
    }
    // An error left pending by the caller's own earlier work is not this call's
    // to clear or to report as its own: refuse to launch and leave it in place.
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        return fail(std::string("fireCudaForceProjectNoAlloc: an earlier CUDA error is pending (") + cudaGetErrorString(e) +
                    "); nothing was launched.");
    }
    int device = 0;
    e = cudaGetDevice(&device);
    if (e != cudaSuccess) return fail(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (device < 0 || device >= kMaxDevices) return fail("fireCudaForceProjectNoAlloc: device ordinal out of range.");
    float4* scratch = g_scratchAddress[device].load(std::memory_order_acquire);
    if (scratch == nullptr) {
        void* addr = nullptr;
        e = cudaGetSymbolAddress(&addr, g_forceScratch);
        if (e != cudaSuccess) return fail(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        scratch = static_cast<float4*>(addr);
        g_scratchAddress[device].store(scratch, std::memory_order_release);
    }

    // The settings clamps of a step; Scene allocates nothing until init().
    firesim::Scene dims;
    dims.nx = nx;
    dims.ny = ny;
    dims.nz = nz;
    dims.frameW = 1;
    dims.frameH = 1;
    const firesim::FrameParams p = dims.paramsFrom(*settings, time);
    // Records and faces in this build's storage format (float, or half in the FP16 build).
    const firesim::ScalarFieldsIn in{static_cast<const firesim::Rec4*>(recordsA), static_cast<const firesim::Rec4*>(recordsB),
                                     static_cast<const firesim::Rec2*>(recordsC)};
    const firesim::Velocity vel{reinterpret_cast<const firesim::FaceT*>(u), reinterpret_cast<const firesim::FaceT*>(v),
                                reinterpret_cast<const firesim::FaceT*>(w)};
    const int bx = nx <= 32 ? 32 : (nx <= 64 ? 64 : 128);
    const dim3 grid((nx + bx - 1) / bx, ny, nz);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // No lattice storage here: every curl-noise corner is hashed in place.
    const firesim::HashLattice2 noLattice{};
    firesim::forceContributions<<<grid, bx, 0, s>>>(scratch, in, vel, p, noLattice, noLattice);
    e = cudaGetLastError();  // nothing was pending on entry, so an error here is this launch's
    if (e != cudaSuccess) return fail(std::string("force pass launch: ") + cudaGetErrorString(e));
    firesim::forceProjectSetup<<<grid, bx, 0, s>>>(reinterpret_cast<firesim::FaceT*>(uOut), reinterpret_cast<firesim::FaceT*>(vOut),
                                                   reinterpret_cast<firesim::FaceT*>(wOut), divergence, pressure, scratch, vel, p);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(std::string("force pass launch: ") + cudaGetErrorString(e));
    return true;
}
