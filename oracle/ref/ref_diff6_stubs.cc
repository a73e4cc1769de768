// Host stand-ins for the pieces of the reference's CUDADiffusion that live
// in its CUDA kernel file (elec/CUDADiffusion_ker.cu), so that the oracle
// build can construct a CUDADiffusion and read the face-conductivity table
// its constructor builds on the host.  The kernels themselves are not run
// (the oracle never calls CUDADiffusion::updateLocalVoltage or calc): these
// stand-ins abort if reached.  Test infrastructure.
#include <cuda_runtime_api.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "lazy_array.hh"

typedef double Real;

void call_cuda_kernels(ro_mgarray_ptr<Real>, rw_mgarray_ptr<Real>, ro_mgarray_ptr<Real>, int, int, int,
                       wo_mgarray_ptr<Real>, ro_mgarray_ptr<int>, int)
{
  std::fprintf(stderr, "oracle build: CUDADiffusion::calc is not available (host-only build)\n");
  std::abort();
}

void copy_to_block(wo_mgarray_ptr<double>, ro_mgarray_ptr<int>, ro_mgarray_ptr<double>, const int, const int)
{
  std::fprintf(stderr, "oracle build: CUDADiffusion voltage updates are not available (host-only build)\n");
  std::abort();
}

cudaError_t oracle_host_cudaMemset(void* p, int value, size_t bytes)
{
  std::memset(p, value, bytes);
  return cudaSuccess;
}
