// fire_oracle.h -- CPU oracle for the native-firesim frame pipeline.
//
// TEST INFRASTRUCTURE, NOT PRODUCT CODE.  Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg load this library, and only as the checker
// or the timed CPU baseline.  The product library never links or calls it.
//
// The oracle restates the reference's per-frame pipeline (src/fire_cuda.cu of
// native-firesim) as plain scalar C++ with OpenMP, instantiated in float (the
// reference's arithmetic) and double (the precision oracle).  It is pinned
// against the reference's own CUDA code by the fixtures in tests/golden/,
// which tests/golden/make_golden.py records from oracle/_ref/libfire_ref.so.
//
// Field and stage ids are the FIRE_FIELD_* / FIRE_STAGE_* ids of
// include/fire_ext.h.
#pragma once

#include <stddef.h>
#include <stdint.h>

#include "../include/fire_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

// precision: 0 = float (the reference's arithmetic), 1 = double.
void* oracle_create(int precision, int frameW, int frameH, int nx, int ny, int nz);
void oracle_destroy(void* o);
void oracle_light_dims(void* o, int* dims3);
// Copies a field as float32 (uint32 for the BGRA frame); bytes must match.
int oracle_set_field(void* o, int field, const void* host, long long bytes);
int oracle_get_field(void* o, int field, void* host, long long bytes);
// Double-precision view of a field (only for the double oracle; float oracle widens).
int oracle_get_field_f64(void* o, int field, double* host, long long count);
// Runs stages [first, last] at an explicit time, reading the current fields.
int oracle_stages(void* o, int first, int last, const FireSettings* settings, float time);
// Overrides the projection's SOR iteration count and omega (defaults 40, 1.52).
void oracle_set_pressure_solver(void* o, int iterations, float omega);
// The whole frame with the reference's time bookkeeping (src/fire_cuda.cu:3106-3549).
// mode 0 = step + BGRA, 1 = step + BGRA + metrics, 2 = step only, 3 = render only (BGRA).
int oracle_step(void* o, uint32_t* bgra, const FireSettings* settings, FireCudaFrameMetrics* metrics, int mode);
// The metric accumulator of the last metrics stage: 21 double sums and 10 int words.
void oracle_last_metrics(void* o, double* sums21, int* words10);
void oracle_times(void* o, float* simTime, float* renderTime, int* frameIndex);
void oracle_set_times(void* o, float simTime, float renderTime, int frameIndex);
int oracle_threads(void);
void oracle_set_threads(int n);
const char* oracle_last_error(void);

#ifdef __cplusplus
}
#endif
