// Host stand-ins for the pieces of the reference's CUDADiffusion and
// ECGSensor that live in CUDA kernel files (elec/CUDADiffusion_ker.cu,
// elec/ECGSensor.cu), so that the oracle build can link those classes'
// host code: the face-conductivity table CUDADiffusion's constructor builds
// on the host, and ECGSensor's CPU sum calcEcg.  The kernels themselves are
// not run (the oracle never calls CUDADiffusion's voltage updates or calc,
// nor constructs or evaluates an ECGSensor): these stand-ins abort if
// reached.  Test infrastructure.
#include <cuda_runtime_api.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "Long64.hh"
#include "PioHeaderData.hh"
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

void calcInvrCUDA(wo_mgarray_ptr<double>, ro_mgarray_ptr<Long64>, ro_mgarray_ptr<double>, const int, const int,
                  const int, const int, const double, const double, const double)
{
  std::fprintf(stderr, "oracle build: the ECG 1/r kernel is not available (host-only build)\n");
  std::abort();
}

void calcEcgCUDA(wo_mgarray_ptr<double>, ro_mgarray_ptr<double>, ro_mgarray_ptr<double>, const int)
{
  std::fprintf(stderr, "oracle build: the ECG sum kernel is not available (host-only build)\n");
  std::abort();
}

// ECGSensor::print's file header (elec/PioHeaderData.cc, which needs the
// reference's generated build-version record); print is never called.
void PioHeaderData::writeHeader(pfile_st*, int, double)
{
  std::fprintf(stderr, "oracle build: ECG file output is not available\n");
  std::abort();
}
void PioHeaderData::addItem(const std::string&, int) { std::abort(); }

cudaError_t oracle_host_cudaMemset(void* p, int value, size_t bytes)
{
  std::memset(p, value, bytes);
  return cudaSuccess;
}
