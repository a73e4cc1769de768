// Drop-in plugins behind the reference's split interfaces:
//   cdb_reaction_*  BetterTT06 as a Reaction (elec/Reaction.hh:10-40): calc
//                   gathers Vm[indexArray[i]] and scatters dVm[indexArray[i]]
//                   exactly as the reference's kernel (elec/BetterTT06.cc:1075-1298,
//                   launch :1320-1364) but in hand-written sm_100a code;
//   cdb_fgr_*       the FGR stencil as a Diffusion (elec/Diffusion.hh:19-39,
//                   elec/FGRDiffusionOMP.cc:75-131): updateLocalVoltage scatters
//                   Vm into the padded block, calc assigns dVm.
// They keep the reference's data flow (Vm crosses HBM several times per
// step); the fused engine (engine_host.cu) is the fast path.
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "fgr_device.cuh"
#include "reaction_slot.h"
#include "tt06_step.cuh"

namespace cdb {

struct ReactionArgs {
  TT06Scalars p;
  FitShape sh;
  const double* coef64;
  const float* coef32;
  double* s64;
  float* s32;
  int64_t n;
};

template <bool MIXED>
__global__ void __launch_bounds__(128) reaction_calc_kernel(ReactionArgs a, double dt, const int32_t* __restrict__ index,
                                                            const double* __restrict__ Vm, double* __restrict__ dVm)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const int64_t n = a.n;
  const int32_t e = index[i];
  const double V = Vm[e];
  const BlockScale none{1.0, 1.0, 1.0};
  if (MIXED) {
    IOMixed io{a.s64 + i, a.s32 + i, n};
    GenericFits fits{a.coef64, a.coef32, &a.sh};
    dVm[e] = (double)tt06_step_mixed(a.p, none, fits, (float)dt, V, io);
  } else {
    IO64 io{a.s64 + i, n};
    GenericFits fits{a.coef64, nullptr, &a.sh};
    dVm[e] = tt06_step(a.p, none, fits, dt, V, io);
  }
}

__global__ void reaction_init_kernel(int64_t n, double* s64, float* s32, int mixed, const int32_t* index, double* Vm)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (mixed) {
    for (int k = 0; k < 5; ++k) s64[k * n + i] = tt06_initial_state(k);
    for (int k = 5; k < kNumStates; ++k) s32[(k - 5) * n + i] = (float)tt06_initial_state(k);
  } else {
    for (int k = 0; k < kNumStates; ++k) s64[k * n + i] = tt06_initial_state(k);
  }
  if (index && Vm) Vm[index[i]] = kInitialVm;
}

__global__ void fgr_scatter_kernel(int64_t n, const double* __restrict__ Vm, const int64_t* __restrict__ voxel,
                                   double* __restrict__ blk)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) blk[voxel[i]] = Vm[i];
}

// dVm[i] = scale (A0 phi0 + sum_{k=1..18} A_k phi_k), elec/FGRDiffusionOMP.cc:109-131.
__global__ void fgr_calc_kernel(int64_t n, const double* __restrict__ w19, const int64_t* __restrict__ voxel,
                                const double* __restrict__ blk, int64_t bx, int64_t bxy, double scale,
                                double* __restrict__ dVm)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t v = voxel[i];
  double tmp = w19[i] * blk[v];
#pragma unroll
  for (int k = 1; k < 19; ++k) tmp += w19[k * n + i] * blk[v + node_dx(k) + bx * node_dy(k) + bxy * node_dz(k)];
  dVm[i] = tmp * scale;
}

__global__ void plugin_voxel_map_kernel(int64_t n, const int64_t* __restrict__ gid, int nx, int ny, int64_t bx,
                                        int64_t bxy, int64_t* __restrict__ map, int64_t* __restrict__ cellVoxel)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t g = gid[i];
  const int64_t x = g % nx, y = (g / nx) % ny, z = g / ((int64_t)nx * ny);
  const int64_t v = (x + 1) + bx * (y + 1) + bxy * (z + 1);
  map[v] = i;
  cellVoxel[i] = v;
}

__global__ void plugin_weights_kernel(int64_t n, const int64_t* __restrict__ map, const int64_t* __restrict__ cellVoxel,
                                      const double* __restrict__ sigma6, const int32_t* __restrict__ cellType,
                                      int64_t bx, int64_t bxy, double hx, double hy, double hz, double* __restrict__ w19)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t v = cellVoxel[i];
  int tissue[19];
  int64_t nbr[19];
  for (int k = 0; k < 19; ++k) {
    const int64_t c = map[v + node_dx(k) + bx * node_dy(k) + bxy * node_dz(k)];
    nbr[k] = c;
    tissue[k] = c >= 0 && cellType[c] > 0;   // isTissue(cellType), elec/FGRUtils.hh:42
  }
  double W[19];
  fgr_cell_weights(tissue, [&](int k, int c) { return sigma6[6 * nbr[k] + c]; }, hx, hy, hz, W);
  for (int k = 0; k < 19; ++k) w19[k * n + i] = W[k];
}

struct Buf {
  void* p = nullptr;
  ~Buf() { if (p) cudaFree(p); }
  cudaError_t alloc(size_t b) { return b ? cudaMalloc(&p, b) : cudaSuccess; }
  template <typename T> T* as() const { return (T*)p; }
};

}  // namespace cdb

using namespace cdb;

struct cdb_reaction {
  int device = 0;
  cdb_precision prec = CDB_FP64;
  int64_t n = 0;
  double dt = 0;
  TT06Scalars p{};
  FitShape sh{};
  Buf coef64, coef32, s64, s32;
  int slot = -1;   // constant-memory slot with the compiled fit shapes, or -1: the generic kernel
  ~cdb_reaction() { reaction_slot_release(device, slot); }
};

struct cdb_fgr {
  int device = 0;
  int64_t n = 0;
  int64_t bx = 0, bxy = 0, nvox = 0;
  double scale = 0;
  Buf w19, voxel, blk;
};

extern "C" {

cdb_status cdb_reaction_create(int device, cdb_precision precision, const cdb_tt06_params* params,
                               const cdb_fit fits[CDB_NUM_FITS], int64_t nCells, double dt, cdb_reaction** out)
{
  CDB_CHECK(params && fits && out, CDB_INVALID_ARG, "null argument");
  CDB_CHECK(nCells >= 0 && nCells < (int64_t(1) << 31), CDB_INVALID_ARG, "nCells out of range");
  CDB_CHECK(dt > 0, CDB_INVALID_ARG, "dt must be > 0");
  CDB_CHECK(precision == CDB_FP64 || precision == CDB_MIXED, CDB_INVALID_ARG, "unknown precision");
  CDB_CUDA(cudaSetDevice(device));
  std::unique_ptr<cdb_reaction> r(new cdb_reaction);
  r->device = device;
  r->prec = precision;
  r->n = nCells;
  r->dt = dt;
  r->p = to_scalars(*params);
  std::vector<double> pool(kFitPoolPerType, 0.0);
  std::string err;
  CDB_CHECK(pack_fits(fits, r->sh, pool.data(), kFitPoolPerType, err), CDB_INVALID_ARG, err);
  std::vector<float> pool32(pool.begin(), pool.end());
  CDB_CUDA(r->coef64.alloc(pool.size() * 8));
  CDB_CUDA(r->coef32.alloc(pool32.size() * 4));
  CDB_CUDA(cudaMemcpy(r->coef64.p, pool.data(), pool.size() * 8, cudaMemcpyHostToDevice));
  CDB_CUDA(cudaMemcpy(r->coef32.p, pool32.data(), pool32.size() * 4, cudaMemcpyHostToDevice));
  r->slot = reaction_slot_acquire(device, *params, fits);
  const int64_t n = std::max<int64_t>(nCells, 1);
  if (precision == CDB_MIXED) {
    CDB_CUDA(r->s64.alloc(n * 5 * 8));
    CDB_CUDA(r->s32.alloc(n * 13 * 4));
  } else {
    CDB_CUDA(r->s64.alloc(n * 18 * 8));
  }
  reaction_init_kernel<<<(unsigned)((n + 255) / 256), 256>>>(nCells, r->s64.as<double>(), r->s32.as<float>(),
                                                             precision == CDB_MIXED, nullptr, nullptr);
  CDB_CUDA(cudaDeviceSynchronize());
  *out = r.release();
  return CDB_OK;
}

cdb_status cdb_reaction_init(cdb_reaction* r, const int32_t* indexArray, double* Vm, void* stream)
{
  CDB_CHECK(r, CDB_INVALID_ARG, "null argument");
  // a reaction with no cells (its cellTypes absent from the tissue) has
  // nothing to do, whatever its (possibly null, empty) arrays
  if (r->n == 0) return CDB_OK;
  CDB_CHECK(indexArray && Vm, CDB_INVALID_ARG, "null argument");
  CDB_CUDA(cudaSetDevice(r->device));
  reaction_init_kernel<<<(unsigned)((r->n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      r->n, r->s64.as<double>(), r->s32.as<float>(), r->prec == CDB_MIXED, indexArray, Vm);
  CDB_CUDA(cudaGetLastError());
  return CDB_OK;
}

cdb_status cdb_reaction_calc(cdb_reaction* r, double dt, const int32_t* indexArray, const double* Vm,
                             const double* iStim, double* dVm, void* stream)
{
  (void)iStim;   // unused by BetterTT06::calc, as in the reference (elec/BetterTT06.cc:1429)
  CDB_CHECK(r, CDB_INVALID_ARG, "null argument");
  CDB_CHECK(dt == r->dt, CDB_INVALID_ARG, "dt differs from the dt the fits were made for");
  if (r->n == 0) return CDB_OK;   // no cells: nothing to read or write (arrays may be null)
  CDB_CHECK(indexArray && Vm && dVm, CDB_INVALID_ARG, "null argument");
  CDB_CUDA(cudaSetDevice(r->device));
  if (r->slot >= 0) {
    CDB_CUDA(reaction_slot_calc(r->slot, r->prec == CDB_MIXED, r->n, dt, indexArray, Vm, dVm, r->s64.as<double>(),
                                r->s32.as<float>(), (cudaStream_t)stream));
    return CDB_OK;
  }
  ReactionArgs a;
  a.p = r->p;
  a.sh = r->sh;
  a.coef64 = r->coef64.as<double>();
  a.coef32 = r->coef32.as<float>();
  a.s64 = r->s64.as<double>();
  a.s32 = r->s32.as<float>();
  a.n = r->n;
  const unsigned grid = (unsigned)((r->n + 127) / 128);
  if (r->prec == CDB_MIXED)
    reaction_calc_kernel<true><<<grid, 128, 0, (cudaStream_t)stream>>>(a, dt, indexArray, Vm, dVm);
  else
    reaction_calc_kernel<false><<<grid, 128, 0, (cudaStream_t)stream>>>(a, dt, indexArray, Vm, dVm);
  CDB_CUDA(cudaGetLastError());
  return CDB_OK;
}

cdb_status cdb_reaction_get_state(cdb_reaction* r, int var, double* host)
{
  CDB_CHECK(r, CDB_INVALID_ARG, "null argument");
  CDB_CHECK(var >= 0 && var < kNumStates, CDB_INVALID_ARG, "state index out of range");
  if (r->n == 0) return CDB_OK;
  CDB_CHECK(host, CDB_INVALID_ARG, "null argument");
  CDB_CUDA(cudaSetDevice(r->device));
  CDB_CUDA(cudaDeviceSynchronize());
  const int64_t n = r->n;
  if (r->prec == CDB_MIXED && var >= 5) {
    std::vector<float> tmp(n);
    CDB_CUDA(cudaMemcpy(tmp.data(), r->s32.as<float>() + (var - 5) * n, n * 4, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < n; ++i) host[i] = tmp[i];
  } else {
    CDB_CUDA(cudaMemcpy(host, r->s64.as<double>() + var * n, n * 8, cudaMemcpyDeviceToHost));
  }
  return CDB_OK;
}

cdb_status cdb_reaction_set_state(cdb_reaction* r, int var, const double* host)
{
  CDB_CHECK(r, CDB_INVALID_ARG, "null argument");
  CDB_CHECK(var >= 0 && var < kNumStates, CDB_INVALID_ARG, "state index out of range");
  if (r->n == 0) return CDB_OK;
  CDB_CHECK(host, CDB_INVALID_ARG, "null argument");
  CDB_CUDA(cudaSetDevice(r->device));
  CDB_CUDA(cudaDeviceSynchronize());
  const int64_t n = r->n;
  if (r->prec == CDB_MIXED && var >= 5) {
    std::vector<float> tmp(host, host + n);
    CDB_CUDA(cudaMemcpy(r->s32.as<float>() + (var - 5) * n, tmp.data(), n * 4, cudaMemcpyHostToDevice));
  } else {
    CDB_CUDA(cudaMemcpy(r->s64.as<double>() + var * n, host, n * 8, cudaMemcpyHostToDevice));
  }
  return CDB_OK;
}

cdb_status cdb_reaction_destroy(cdb_reaction* r)
{
  if (!r) return CDB_OK;
  cudaSetDevice(r->device);
  cudaDeviceSynchronize();
  delete r;
  return CDB_OK;
}

cdb_status cdb_fgr_create(int device, int32_t nx, int32_t ny, int32_t nz, double dx, double dy, double dz,
                          int64_t nCells, const int64_t* gid, const int32_t* cellType, const double* sigma6,
                          double diffusionScale, cdb_fgr** out)
{
  CDB_CHECK(out && gid && cellType && sigma6, CDB_INVALID_ARG, "null argument");
  CDB_CHECK(nx > 0 && ny > 0 && nz > 0 && dx > 0 && dy > 0 && dz > 0, CDB_INVALID_ARG, "bad grid");
  const int64_t grid = (int64_t)nx * ny * nz;
  CDB_CHECK(nCells > 0 && nCells <= grid, CDB_INVALID_ARG, "nCells out of range");
  for (int64_t i = 0; i < nCells; ++i) {
    CDB_CHECK(gid[i] >= 0 && gid[i] < grid, CDB_INVALID_ARG, "gid outside the grid");
  }
  CDB_CUDA(cudaSetDevice(device));
  std::unique_ptr<cdb_fgr> d(new cdb_fgr);
  d->device = device;
  d->n = nCells;
  d->scale = diffusionScale;
  d->bx = nx + 2;
  d->bxy = d->bx * (ny + 2);
  d->nvox = d->bxy * (nz + 2);
  CDB_CUDA(d->w19.alloc(nCells * 19 * 8));
  CDB_CUDA(d->voxel.alloc(nCells * 8));
  CDB_CUDA(d->blk.alloc(d->nvox * 8));
  CDB_CUDA(cudaMemset(d->blk.p, 0, d->nvox * 8));
  Buf map, g, ct, sig;
  CDB_CUDA(map.alloc(d->nvox * 8));
  CDB_CUDA(g.alloc(nCells * 8));
  CDB_CUDA(ct.alloc(nCells * 4));
  CDB_CUDA(sig.alloc(nCells * 48));
  CDB_CUDA(cudaMemset(map.p, 0xff, d->nvox * 8));
  CDB_CUDA(cudaMemcpy(g.p, gid, nCells * 8, cudaMemcpyHostToDevice));
  CDB_CUDA(cudaMemcpy(ct.p, cellType, nCells * 4, cudaMemcpyHostToDevice));
  CDB_CUDA(cudaMemcpy(sig.p, sigma6, nCells * 48, cudaMemcpyHostToDevice));
  const unsigned grid256 = (unsigned)((nCells + 255) / 256);
  plugin_voxel_map_kernel<<<grid256, 256>>>(nCells, g.as<int64_t>(), nx, ny, d->bx, d->bxy, map.as<int64_t>(),
                                            d->voxel.as<int64_t>());
  plugin_weights_kernel<<<(unsigned)((nCells + 127) / 128), 128>>>(nCells, map.as<int64_t>(), d->voxel.as<int64_t>(),
                                                                   sig.as<double>(), ct.as<int32_t>(), d->bx, d->bxy,
                                                                   dx, dy, dz, d->w19.as<double>());
  CDB_CUDA(cudaDeviceSynchronize());
  *out = d.release();
  return CDB_OK;
}

cdb_status cdb_fgr_update_local_voltage(cdb_fgr* d, const double* Vm, void* stream)
{
  CDB_CHECK(d && Vm, CDB_INVALID_ARG, "null argument");
  CDB_CUDA(cudaSetDevice(d->device));
  fgr_scatter_kernel<<<(unsigned)((d->n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(d->n, Vm, d->voxel.as<int64_t>(),
                                                                                      d->blk.as<double>());
  CDB_CUDA(cudaGetLastError());
  return CDB_OK;
}

cdb_status cdb_fgr_calc(cdb_fgr* d, double* dVm, void* stream)
{
  CDB_CHECK(d && dVm, CDB_INVALID_ARG, "null argument");
  CDB_CUDA(cudaSetDevice(d->device));
  fgr_calc_kernel<<<(unsigned)((d->n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      d->n, d->w19.as<double>(), d->voxel.as<int64_t>(), d->blk.as<double>(), d->bx, d->bxy, d->scale, dVm);
  CDB_CUDA(cudaGetLastError());
  return CDB_OK;
}

cdb_status cdb_fgr_get_weights(cdb_fgr* d, double* host19)
{
  CDB_CHECK(d && host19, CDB_INVALID_ARG, "null argument");
  CDB_CUDA(cudaSetDevice(d->device));
  CDB_CUDA(cudaDeviceSynchronize());
  std::vector<double> w(d->n * 19);
  CDB_CUDA(cudaMemcpy(w.data(), d->w19.p, w.size() * 8, cudaMemcpyDeviceToHost));
  for (int64_t i = 0; i < d->n; ++i)
    for (int k = 0; k < 19; ++k) host19[i * 19 + k] = w[k * d->n + i];
  return CDB_OK;
}

cdb_status cdb_fgr_destroy(cdb_fgr* d)
{
  if (!d) return CDB_OK;
  cudaSetDevice(d->device);
  cudaDeviceSynchronize();
  delete d;
  return CDB_OK;
}

}  // extern "C"

// ---- diagnostics ----

namespace cdb {
__global__ void diag_div64_kernel(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                                  double* __restrict__ q)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) q[i] = div64(a[i], b[i]);
}
}  // namespace cdb

extern "C" cdb_status cdb_diag_div64(int device, int64_t n, const double* a, const double* b, double* q, void* stream)
{
  CDB_CHECK(a && b && q && n >= 0, CDB_INVALID_ARG, "bad argument");
  CDB_CUDA(cudaSetDevice(device));
  if (n == 0) return CDB_OK;
  diag_div64_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(n, a, b, q);
  CDB_CUDA(cudaGetLastError());
  return CDB_OK;
}
