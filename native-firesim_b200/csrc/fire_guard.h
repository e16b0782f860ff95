// fire_guard.h -- the library's device allocations, and the bounds-checking build.
//
// Every device buffer the library owns comes from deviceAlloc and goes back
// through deviceFree.  In the default builds they are cudaMalloc and cudaFree.
//
// In the FIRE_BOUNDS_CHECK build (libfiresim_b200_checked.so) each buffer
// sits between two guard zones of kGuardBytes, and the whole allocation,
// payload included, starts as 0xFF bytes: a NaN in every float, half and
// bfloat16 field and -1 in every integer.  Then
//   - a kernel that writes up to kGuardBytes past either end of a buffer
//     changes a guard byte, which checkGuards finds and names (the buffer's
//     label, the side, the first changed byte);
//   - a kernel that reads past an end, or reads a cell that nothing has
//     written yet, takes a NaN or a -1 into its result, which shows as a
//     difference from the default build's result on the same inputs.
// No access leaves the allocation, so a stray index costs no memory fault.
// The reference has no counterpart: its kernels index unchecked
// (src/fire_cuda.cu:445-487), and compute-sanitizer is the usual tool.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <string>

namespace firesim {

#ifdef FIRE_BOUNDS_CHECK
constexpr bool kBoundsChecked = true;
#else
constexpr bool kBoundsChecked = false;
#endif

// One guard zone: a plane of a 256^3 grid of 32-byte records is 2 MiB.
constexpr size_t kGuardBytes = size_t(2) << 20;

// cudaMalloc on the current device; `label` names the buffer in reports.
cudaError_t deviceAlloc(void** p, size_t bytes, const char* label);
// cudaFree of a deviceAlloc pointer (null is ignored).  The checked build
// scans the buffer's guard zones first and keeps what it finds for the next
// checkGuards.
void deviceFree(void* p);

// Checked build: synchronizes the current device, scans the guard zones of
// its live allocations, re-arms every zone found changed, and sets
// `corrupted` to the number of buffers with a changed zone (those freed
// since the last call included) and `report` to a description of the first.
// Returns false only on a CUDA error (described in `report`).
// Default builds: corrupted = -1 and a report that says so; returns true.
bool checkGuards(int& corrupted, std::string& report);

// Checked build: sets the byte `offset` bytes past the end of the first live
// buffer labelled `label` to 0 with a host-side cudaMemset.  The byte lies
// inside that buffer's allocation; this is how the checker's own test makes
// a change for checkGuards to find.  Default builds: returns false.
bool plantGuardByte(const char* label, size_t offset, std::string& err);

}  // namespace firesim
