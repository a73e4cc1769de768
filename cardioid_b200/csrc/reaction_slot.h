// Constant-memory reaction slots for the plugin Reaction (plugins.cu).
//
// The compiled reaction kernels read a reaction type's scalars and fit
// coefficients from one of CDB_MAX_REACTION_TYPES constant-memory slots
// per device (engine_host.cu).  Engines and plugin reactions share the
// slots; registrations with identical content (scalars, fit shapes and
// coefficients) share one slot, reference counted.  A plugin reaction whose
// fits have the compiled shapes (fit_shapes.h) runs the unrolled
// per-slot kernel; otherwise, or when every slot is taken, it keeps the
// generic kernel in plugins.cu.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/cardioid_b200.h"

namespace cdb {

// The slot of this reaction type (taken and uploaded when new), or -1.
int reaction_slot_acquire(int device, const cdb_tt06_params& params, const cdb_fit* fits);
void reaction_slot_release(int device, int slot);

// dVm[index[i]] = -Iion of cell i, i < n, with Vm[index[i]] and the state
// rows s64 / s32 (pitch n) of the plugin layout, on the slot's kernel.
cudaError_t reaction_slot_calc(int slot, bool mixed, int64_t n, double dt, const int32_t* index, const double* Vm,
                               double* dVm, double* s64, float* s32, cudaStream_t stream);

}  // namespace cdb
