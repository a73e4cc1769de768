/* Force-included when the oracle build compiles the reference's
 * CUDADiffusion.cc (elec/CUDADiffusion.cc), so that its constructor, which
 * builds the face-conductivity table on the host (:73-122), runs in the CPU
 * build: the GPU space is the host space (the build has no USE_CUDA, so
 * lazy_array has one space), and the constructor's final cudaMemset of the
 * Vm block becomes a host memset under a name of its own (no CUDA runtime
 * symbol is defined).  Test infrastructure. */
#pragma once
#include <cuda_runtime_api.h>
cudaError_t oracle_host_cudaMemset(void* p, int value, size_t bytes);
#define cudaMemset oracle_host_cudaMemset
#define GPU CPU
