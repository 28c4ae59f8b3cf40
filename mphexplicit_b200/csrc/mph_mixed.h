// mph_mixed.h — the mixed-precision form (FP32 pair arithmetic on cell-relative
// coordinates, compensated sums, FP64 integration), k_mixed.cu.
#pragma once
#include <string>
#include "mph_internal.h"

namespace mph {

struct MixedState;

int mixed_create(MixedState** out, const SimConst& c, const mph_constants& k, DevFP64& d, cudaStream_t s,
                 std::string* err);
// Advance nsteps; the FP64 buffers of `d` are stale until mixed_export.
int mixed_step(MixedState* m, const SimConst& c, DevFP64& d, int nsteps, cudaStream_t s, std::string* err);
// Write the mixed state back into the FP64 buffers (current order, fields).
int mixed_export(MixedState* m, const SimConst& c, DevFP64& d, cudaStream_t s, std::string* err);
// Take positions/velocities from the FP64 buffers (after mph_set_state).
int mixed_import(MixedState* m, const SimConst& c, DevFP64& d, cudaStream_t s, std::string* err);
long long mixed_rebuilds(const MixedState* m);
void mixed_destroy(MixedState* m);

}  // namespace mph
