// config_oracle.h -- CPU oracle of the config physics (FirePhysicsParams.mode 1).
//
// TEST INFRASTRUCTURE, NOT PRODUCT CODE.  Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg load this library, and only as the checker
// or the timed CPU baseline.  The product library never links or calls it.
//
// The config physics is this project's own model (the reference has no disk
// emitters, seeds, vorticity confinement or point light); the equations are
// stated in include/fire_ext.h.  This file restates them as plain scalar C++
// with OpenMP, instantiated in float (the product's arithmetic: the product
// compiles these kernels without FMA contraction and this oracle is built
// with -ffp-contract=off, so the simulation matches bit for bit) and double
// (the precision oracle).  Field and stage ids are the FIRE_FIELD_* /
// FIRE_STAGE_* ids of include/fire_ext.h.
#pragma once

#include <stdint.h>

#include "../include/fire_ext.h"

#ifdef __cplusplus
extern "C" {
#endif

// precision: 0 = float, 1 = double.  The scene starts empty (all fields 0).
void* cfg_oracle_create(int precision, int frameW, int frameH, int nx, int ny, int nz);
void cfg_oracle_destroy(void* o);
int cfg_oracle_set_physics(void* o, const FirePhysicsParams* params);
void cfg_oracle_set_pressure_solver(void* o, int iterations, float omega);
// Multigrid solve of the Dirichlet top (FirePhysicsParams.pressureTop = 1): up
// to maxCycles V-cycles, stopping once max |r| <= tolerance (0: all cycles).
void cfg_oracle_set_multigrid(void* o, int maxCycles, int preSmooth, int postSmooth, float tolerance);
void cfg_oracle_multigrid_stats(void* o, int* cycles, float* maxResidual);
// Fields: HEAT, FUEL, SOOT, PRESSURE, DIVERGENCE, U, V, W, HDR, CONFIG_TRANSMITTANCE (float32).
int cfg_oracle_set_field(void* o, int field, const void* host, long long bytes);
int cfg_oracle_get_field(void* o, int field, void* host, long long bytes);
int cfg_oracle_get_field_f64(void* o, int field, double* host, long long count);
// Stages [first, last] with the product's stage ids; ADVECT_REACT advances the step counter.
int cfg_oracle_stages(void* o, int first, int last);
// One step (ADVECT_VELOCITY .. WALL_BOUNDARY), then LIGHT_BUILD and RENDER if render != 0.
int cfg_oracle_step(void* o, int render);
unsigned long long cfg_oracle_step_count(void* o);
const char* cfg_oracle_last_error(void);

#ifdef __cplusplus
}
#endif
