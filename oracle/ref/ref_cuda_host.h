/* Force-included when the oracle build compiles the reference's
 * CUDADiffusion.cc and ECGSensor.cc, so that their host code runs in the CPU
 * build (CUDADiffusion's constructor builds the face-conductivity table on
 * the host, elec/CUDADiffusion.cc:73-122; ECGSensor.cc holds the CPU ECG sum
 * calcEcg, :231-246): the GPU space is the host space (the build has no
 * USE_CUDA, so lazy_array has one space), and cudaMemset becomes a host
 * memset under a name of its own (no CUDA runtime symbol is defined).
 * Test infrastructure. */
#pragma once
#include <cuda_runtime_api.h>
cudaError_t oracle_host_cudaMemset(void* p, int value, size_t bytes);
#define cudaMemset oracle_host_cudaMemset
#define GPU CPU
