// FGR stencil entry point that allocates nothing: cdb_fgr_calc_static.
//
// Some callers cannot allocate device memory: code that runs inside another
// framework's memory pool or allocator hooks, code that must not change the
// device's allocation state between two measurements, or a host that has
// handed all free memory to a long-lived workspace.  This entry point takes
// every input and output from the caller and keeps its one piece of working
// memory — the zero-padded Vm block the 19-point stencil reads — in a
// file-scope __device__ array that the library's module holds on every GPU
// that loads it, until the process exits.
//
// The block holds at most kStaticVoxels doubles (16 MiB): a box of
// nx*ny*nz cells fits when (nx+2)*(ny+2)*(nz+2) <= 2,097,152, e.g. 126^3.
// Every call shares the one array and leaves its contents behind; the call
// clears the whole block it uses before filling it.  Two calls whose
// kernels overlap on the GPU (different streams, or different host threads)
// race on the block: a caller serialises them, e.g. on one stream.
//
// The array's device address is looked up on the first call on each device
// and kept: a cudaDeviceReset on that device after the first call (which
// unloads the module, so the array may come back elsewhere) is not
// supported.  The call leaves the calling thread's current device as it
// found it.
#include <cuda_runtime.h>

#include <mutex>

#include "common.cuh"
#include "fgr_device.cuh"

namespace cdb {

constexpr int64_t kStaticVoxels = int64_t(1) << 21;   // 16 MiB of doubles

static __device__ __align__(256) double g_static_block[kStaticVoxels];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_static_mutex;
double* g_static_ptr[kMaxDevices] = {nullptr};

// The device address of the block on the current device.  In host code
// g_static_block names a host-side stand-in, not device memory, so the
// address is looked up once per device, with that device current.
cudaError_t static_block(int device, double** out)
{
  std::lock_guard<std::mutex> lock(g_static_mutex);
  if (!g_static_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_block);
    if (e != cudaSuccess) return e;
    g_static_ptr[device] = (double*)p;
  }
  *out = g_static_ptr[device];
  return cudaSuccess;
}

__global__ void static_clear_kernel(double* __restrict__ blk, int64_t nvox)
{
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nvox; v += (int64_t)gridDim.x * blockDim.x)
    blk[v] = 0.0;
}

__global__ void static_scatter_kernel(const double* __restrict__ Vm, double* __restrict__ blk, int nx, int ny,
                                      int64_t n, int64_t bx, int64_t bxy)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t x = i % nx, y = (i / nx) % ny, z = i / ((int64_t)nx * ny);
  blk[(x + 1) + bx * (y + 1) + bxy * (z + 1)] = Vm[i];
}

// dVm[i] = scale (A0 phi0 + sum_{k=1..18} A_k phi_k), the reference's order
// (elec/FGRDiffusionOMP.cc:109-131); weights are 19 rows of n (A0 first).
__global__ void static_stencil_kernel(const double* __restrict__ w19, const double* __restrict__ blk, int nx, int ny,
                                      int64_t n, int64_t bx, int64_t bxy, double scale, double* __restrict__ dVm)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t x = i % nx, y = (i / nx) % ny, z = i / ((int64_t)nx * ny);
  const int64_t v = (x + 1) + bx * (y + 1) + bxy * (z + 1);
  double tmp = w19[i] * blk[v];
#pragma unroll
  for (int k = 1; k < 19; ++k) tmp += w19[k * n + i] * blk[v + node_dx(k) + bx * node_dy(k) + bxy * node_dz(k)];
  dVm[i] = tmp * scale;
}

// Makes `device` current for the call and restores the caller's current
// device when the call returns (the entry point runs inside other
// frameworks' code, whose device choice it must not change).
struct DeviceScope {
  int prev = -1;
  cudaError_t enter(int device)
  {
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) {
      prev = -1;
      return e;
    }
    return prev == device ? cudaSuccess : cudaSetDevice(device);
  }
  ~DeviceScope()
  {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace
}  // namespace cdb

using namespace cdb;

extern "C" cdb_status cdb_fgr_calc_static(int device, int32_t nx, int32_t ny, int32_t nz, const double* weights19,
                                          const double* Vm, double* dVm, double diffusionScale, void* stream)
{
  CDB_CHECK(weights19 && Vm && dVm, CDB_INVALID_ARG, "null argument");
  CDB_CHECK(nx > 0 && ny > 0 && nz > 0, CDB_INVALID_ARG, "grid dimensions must be positive");
  CDB_CHECK(device >= 0 && device < kMaxDevices, CDB_INVALID_ARG, "device index out of range");
  const int64_t bx = (int64_t)nx + 2, bxy = bx * ((int64_t)ny + 2), nvox = bxy * ((int64_t)nz + 2);
  CDB_CHECK(nvox <= kStaticVoxels, CDB_INVALID_ARG,
            "box too large for cdb_fgr_calc_static: (nx+2)(ny+2)(nz+2) = " + std::to_string(nvox) +
                " voxels exceeds the static block of " + std::to_string(kStaticVoxels) + " voxels (16 MiB)");
  DeviceScope scope;
  CDB_CUDA(scope.enter(device));
  double* blk = nullptr;
  CDB_CUDA(static_block(device, &blk));
  const int64_t n = (int64_t)nx * ny * nz;
  cudaStream_t s = (cudaStream_t)stream;
  // the block keeps the previous call's values: clear all of it (the halo
  // must read zero) before the scatter
  static_clear_kernel<<<(unsigned)std::min<int64_t>((nvox + 255) / 256, 4096), 256, 0, s>>>(blk, nvox);
  static_scatter_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(Vm, blk, nx, ny, n, bx, bxy);
  static_stencil_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(weights19, blk, nx, ny, n, bx, bxy,
                                                                    diffusionScale, dVm);
  CDB_CUDA(cudaGetLastError());
  return CDB_OK;
}
