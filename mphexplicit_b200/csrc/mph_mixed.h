// mph_mixed.h — the mixed-precision form (k_mixed.cu): FP32 pair arithmetic
// on cell-relative coordinates with compensated per-particle sums; FP64 kept
// for position/velocity integration (the buffers of DevFP64) and for the
// global mass/momentum/energy sums.  mph_host.cpp sequences the launches.
#pragma once
#include <string>
#include "mph_internal.h"

namespace mph {

struct MixedState;

// Allocate, sort, build the table and run the start-up density sweep.
// fp64_pressure: the density sweep's short-range pairs (DensityP,
// DivergenceP, hence the PressureP values) in FP64, the rest in FP32
// (MPH_MODE_MIXED_P64).
int mixed_create(MixedState** out, const SimConst& c, const mph_constants& k, DevFP64& d, bool fp64_pressure,
                 cudaStream_t s, std::string* err);
// Convection/wall/periodic + displacement maximum + FP32 copies (1 launch).
void mixed_move(MixedState* m, const SimConst& c, DevFP64& d, cudaStream_t s);
// Counting sort by cell, reorder, neighbour table; *launches gets the count.
int mixed_rebuild(MixedState* m, const SimConst& c, DevFP64& d, cudaStream_t s, std::string* err, int* launches);
// Density sweep (1 launch); advance_wall moves the wall centres one step.
void mixed_sweep_a(MixedState* m, const SimConst& c, DevFP64& d, bool advance_wall, cudaStream_t s);
// Force sweep (FP32 pairs) + FP64 velocity update into d.vel[1 - d.vcur];
// returns the number of launches (1).
int mixed_sweep_b(MixedState* m, const SimConst& c, DevFP64& d, cudaStream_t s);
// Force sweep by cell walk (no long table read) instead of the table sweep.
void mixed_set_cell_walk(MixedState* m, bool on);
// Fill the output-only fields (DensityA, wall forces, neighbour counts).
int mixed_export(MixedState* m, const SimConst& c, DevFP64& d, cudaStream_t s, std::string* err, int* launches);
// VirialPressureAtParticle into d.virial_p (FP32 pair terms, output only).
int mixed_virial(MixedState* m, const SimConst& c, DevFP64& d, cudaStream_t s, std::string* err);
// Positions/velocities were overwritten in `d` (mph_set_state): refresh.
int mixed_import(MixedState* m, const SimConst& c, DevFP64& d, cudaStream_t s, std::string* err);
void mixed_mark_stale(MixedState* m);
int mixed_max_neighbors(const MixedState* m);
int mixed_capacity(const MixedState* m);
void mixed_destroy(MixedState* m);

}  // namespace mph
