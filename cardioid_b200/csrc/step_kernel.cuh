// The fused time-step kernel and its set-up kernels.
//
// One launch per (time step, reaction type present): each warp takes one
// warp tile, a run of up to 32 consecutive cells of one tissue that share a
// reaction type, so the type — and with it the coefficient pool — is a
// kernel parameter, uniform across the launch.  Per cell, in the order of
// the reference's omp loop (elec/simulationLoop.cc:183-231):
//   FGR stencil on Vm(t) (elec/FGRDiffusionOMP.cc:109-131),
//   BetterTT06 update (elec/BetterTT06.cc:1426-1649),
//   box stimuli, assigned in order (elec/BoxStimulus.cc:56-64),
//   Vm(t+dt) = Vm + dt (dVmR + dVmD + iStim) (elec/simulationLoop.cc:221-228),
//   activation time: first post-step time with Vm > 0 (elec/ActivationTimeSensor.cc:99-111),
//   min/max Vm (elec/MinMaxSensor.cc:44-67) on request.
// Vm is read from one padded block and written to the other.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"
#include "fgr_device.cuh"
#include "tt06_step.cuh"

namespace cdb {

constexpr int kWarpsPerCta = 4;
constexpr int kCta = 32 * kWarpsPerCta;

struct TissueDev {
  double* vm[2];
  double* s64;
  float* s32;
  const void* w;
  const int64_t* voxel;
  double* act;
  int64_t n;
  int64_t px, pxy;        // padded strides
  int nx, ny, nz;
  int py0, pz0;           // 1 when y (z) is padded
  int cls;
  int nstim, stim0;
  int parity;             // buffer holding Vm at the start of the next launch batch
  int64_t step0;          // steps taken at the start of the next launch batch
  double scale;           // diffusionScale (0: no diffusion)
  BlockScale blk;
  unsigned long long* minmax;   // 2 slots
};

struct WarpTile {
  int tissue;
  int count;
  int64_t first;
};

struct StepArgs {
  TissueDev* tissues;
  const WarpTile* tiles;      // this launch's tiles
  int nTiles;
  int rt;                     // reaction type (constant-memory slot)
  const cdb_stimulus* stims;
  const double* times;
  double dt;
  int k;                      // step within the launch batch
  int minmax;                 // reduce min/max this step
};

__constant__ TT06Scalars c_scal[CDB_MAX_REACTION_TYPES];
__constant__ FitShape c_shape[CDB_MAX_REACTION_TYPES];
__constant__ double c_coef64[CDB_MAX_REACTION_TYPES * kFitPoolPerType];
__constant__ float c_coef32[CDB_MAX_REACTION_TYPES * kFitPoolPerType];

__device__ __forceinline__ double pulse_value(const cdb_stimulus& s, double time)
{
  if (!(time > s.t0 && time < s.tf)) return 0.0;
  const double t = time - floor(time / s.period) * s.period;
  return (t >= s.phase && t < s.phase + s.duration) ? s.amplitude : 0.0;
}

// Geometry of one tissue, held in registers by the step kernel.
struct Geom {
  const int64_t* voxel;
  int64_t px, pxy;
  int nx, ny, py0, pz0;
};

__device__ __forceinline__ void cell_coords(const Geom& g, int64_t i, int64_t& vox, int& x, int& y, int& z)
{
  if (g.voxel) {
    vox = g.voxel[i];
    const int64_t yz = vox / g.px;
    x = (int)(vox - yz * g.px) - 1;
    const int64_t py = g.pxy / g.px;
    const int64_t zz = yz / py;
    y = (int)(yz - zz * py) - g.py0;
    z = (int)zz - g.pz0;
  } else {
    const int nxy = g.nx * g.ny;
    const int ii = (int)i;
    z = ii / nxy;
    const int r = ii - z * nxy;
    y = r / g.nx;
    x = r - y * g.nx;
    vox = (int64_t)(x + 1) + g.px * (int64_t)(y + g.py0) + g.pxy * (int64_t)(z + g.pz0);
  }
}

__device__ __forceinline__ int64_t node_offset(int64_t px, int64_t pxy, int node)
{
  return (int64_t)node_dx(node) + px * node_dy(node) + pxy * node_dz(node);
}

// FP64 stencil in the reference's order: A0 phi0 + sum_k A_k phi_k.
template <int CLS>
__device__ __forceinline__ double stencil64(const double* __restrict__ w, int64_t n, int64_t px, int64_t pxy,
                                            const double* __restrict__ vin, int64_t vox, double phi0, int64_t i)
{
  double tmp = __ldg(w + i) * phi0;
#pragma unroll
  for (int r = 1; r < class_rows(CLS); ++r) {
    const int node = class_node(CLS, r);
    tmp += __ldg(w + r * n + i) * __ldg(vin + vox + node_offset(px, pxy, node));
  }
  return tmp;
}

// Mixed stencil: sum_k A_k (phi_k - phi0) with FP32 weights; the
// differences are taken in FP64 (A0 = -sum A_k).
template <int CLS>
__device__ __forceinline__ double stencil32(const float* __restrict__ w, int64_t n, int64_t px, int64_t pxy,
                                            const double* __restrict__ vin, int64_t vox, double phi0, int64_t i)
{
  float tmp = 0.f;
#pragma unroll
  for (int r = 1; r < class_rows(CLS); ++r) {
    const int node = class_node(CLS, r);
    const float d = (float)(__ldg(vin + vox + node_offset(px, pxy, node)) - phi0);
    tmp = fmaf(__ldg(w + (r - 1) * n + i), d, tmp);
  }
  return (double)tmp;
}

// Resident CTAs per SM the register budget aims at: 4 CTAs (16 warps, 128
// registers).  The mixed step fits without spilling; the FP64 step spills
// ~90 bytes per thread to L1 there, and still runs 1.2x faster on B200 than
// at 3 CTAs (168 registers, no spill) because latency hiding dominates.
#ifndef CDB_FP64_MIN_CTAS
#define CDB_FP64_MIN_CTAS 4
#endif
template <bool MIXED>
constexpr int min_ctas() { return MIXED ? 4 : CDB_FP64_MIN_CTAS; }

// SLOT >= 0: the launch's reaction type is constant-memory slot SLOT and its
// fits have the compiled shapes (fit_shapes.h); SLOT < 0: any slot (a.rt)
// with run-time shapes.
template <bool MIXED, int SLOT>
__global__ void __launch_bounds__(kCta, min_ctas<MIXED>()) fused_step_kernel(StepArgs a)
{
  constexpr bool SPEC = SLOT >= 0;
  const int warp = blockIdx.x * kWarpsPerCta + (threadIdx.x >> 5);
  if (warp >= a.nTiles) return;   // whole warps leave together
  const int lane = threadIdx.x & 31;
  const WarpTile tile = a.tiles[warp];
  const TissueDev* __restrict__ Tp = a.tissues + tile.tissue;
  const int64_t lstep = Tp->step0 + a.k;
  const double time = a.times[lstep];
  const double tnext = a.times[lstep + 1];
  const int nstim = Tp->nstim;
  const int stim0 = Tp->stim0;
  // lane s holds stimulus s's value at this time
  const double stimVal = lane < nstim ? pulse_value(a.stims[stim0 + lane], time) : 0.0;
  const bool active = lane < tile.count;
  // lanes past the tile's end stand in for its first cell until the end
  const int64_t i = tile.first + (active ? lane : 0);
  Geom g;
  g.voxel = Tp->voxel; g.px = Tp->px; g.pxy = Tp->pxy; g.nx = Tp->nx; g.ny = Tp->ny;
  g.py0 = Tp->py0; g.pz0 = Tp->pz0;
  int64_t vox;
  int x, y, z;
  cell_coords(g, i, vox, x, y, z);
  // iStim = 0, then every stimulus that is on assigns its value inside its box
  double istim = 0.0;
  for (int k = 0; k < nstim; ++k) {
    const double v = __shfl_sync(0xffffffffu, stimVal, k);
    if (v != 0.0) {
      const cdb_stimulus* b = a.stims + stim0 + k;
      if (x > b->xMin && x < b->xMax && y > b->yMin && y < b->yMax && z > b->zMin && z < b->zMax) istim = v;
    }
  }
  double vnew = 0.0;
  if (active) {
    const int cur = (Tp->parity + a.k) & 1;
    const double* __restrict__ vin = Tp->vm[cur];
    double* __restrict__ vout = Tp->vm[cur ^ 1];
    const int64_t n = Tp->n;   // tissues hold fewer than 2^31 cells
    const double scale = Tp->scale;
    const int cls = Tp->cls;
    const void* wp = Tp->w;
    const BlockScale blk = Tp->blk;
    double* const s64 = Tp->s64 + i;
    float* const s32 = Tp->s32 + i;
    double* const act = Tp->act;
    const double phi0 = vin[vox];

    double dvmD = 0.0;
    if (scale != 0.0) {
      double acc;
      if (MIXED) {
        const float* w = (const float*)wp;
        acc = cls == kVolume ? stencil32<kVolume>(w, n, g.px, g.pxy, vin, vox, phi0, i)
            : cls == kSheet ? stencil32<kSheet>(w, n, g.px, g.pxy, vin, vox, phi0, i)
                            : stencil32<kCable>(w, n, g.px, g.pxy, vin, vox, phi0, i);
      } else {
        const double* w = (const double*)wp;
        acc = cls == kVolume ? stencil64<kVolume>(w, n, g.px, g.pxy, vin, vox, phi0, i)
            : cls == kSheet ? stencil64<kSheet>(w, n, g.px, g.pxy, vin, vox, phi0, i)
                            : stencil64<kCable>(w, n, g.px, g.pxy, vin, vox, phi0, i);
      }
      dvmD = acc * scale;
    }

    // With SPEC the slot is a template parameter, so every coefficient is
    // an immediate constant-bank operand of its FMA (no load instruction).
    const int rt = SPEC ? SLOT : a.rt;
    const double* c64 = c_coef64 + rt * kFitPoolPerType;
    double dvmR;
    if (MIXED) {
      IOMixed io{s64, s32, n};
      const float* c32 = c_coef32 + rt * kFitPoolPerType;
      if (SPEC) {
        SpecFits fits{c64, c32};
        dvmR = (double)tt06_step_mixed(c_scal[rt], blk, fits, (float)a.dt, phi0, io);
      } else {
        GenericFits fits{c64, c32, &c_shape[rt]};
        dvmR = (double)tt06_step_mixed(c_scal[rt], blk, fits, (float)a.dt, phi0, io);
      }
    } else {
      IO64 io{s64, n};
      if (SPEC) {
        SpecFits fits{c64, nullptr};
        dvmR = tt06_step(c_scal[rt], blk, fits, a.dt, phi0, io);
      } else {
        GenericFits fits{c64, nullptr, &c_shape[rt]};
        dvmR = tt06_step(c_scal[rt], blk, fits, a.dt, phi0, io);
      }
    }

    vnew = phi0 + a.dt * (dvmR + dvmD + istim);
    vout[vox] = vnew;
    if (vnew > 0.0) {
      double* ap = act + i;
      if (*ap < 0.0) *ap = tnext;
    }
  }
  if (a.minmax) {
    double lo = active ? vnew : __longlong_as_double(0x7ff0000000000000ll);
    double hi = active ? vnew : -__longlong_as_double(0x7ff0000000000000ll);
    for (int o = 16; o > 0; o >>= 1) {
      lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (lane == 0) {
      atomicMin(Tp->minmax, ordered_bits(lo));
      atomicMax(Tp->minmax + 1, ordered_bits(hi));
    }
  }
}

// One step of one reaction type: the compiled kernel of its slot when the
// type has the compiled fit shapes (slot >= 0), else the generic kernel.
template <bool MIXED>
inline void launch_step(int slot, unsigned grid, cudaStream_t stream, const StepArgs& a)
{
  static_assert(CDB_MAX_REACTION_TYPES == 6, "one compiled kernel per slot");
  switch (slot) {
    case 0: fused_step_kernel<MIXED, 0><<<grid, kCta, 0, stream>>>(a); break;
    case 1: fused_step_kernel<MIXED, 1><<<grid, kCta, 0, stream>>>(a); break;
    case 2: fused_step_kernel<MIXED, 2><<<grid, kCta, 0, stream>>>(a); break;
    case 3: fused_step_kernel<MIXED, 3><<<grid, kCta, 0, stream>>>(a); break;
    case 4: fused_step_kernel<MIXED, 4><<<grid, kCta, 0, stream>>>(a); break;
    case 5: fused_step_kernel<MIXED, 5><<<grid, kCta, 0, stream>>>(a); break;
    default: fused_step_kernel<MIXED, -1><<<grid, kCta, 0, stream>>>(a); break;
  }
}

// After a launch batch of k steps: every tissue is k steps further.
__global__ void advance_kernel(TissueDev* tissues, int nTissues, int k)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nTissues) {
    tissues[t].step0 += k;
    tissues[t].parity = (tissues[t].parity + k) & 1;
  }
}

__global__ void reset_minmax_kernel(TissueDev* tissues, int nTissues)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nTissues) {
    tissues[t].minmax[0] = ordered_bits(__longlong_as_double(0x7ff0000000000000ll));
    tissues[t].minmax[1] = ordered_bits(-__longlong_as_double(0x7ff0000000000000ll));
  }
}

// ---- set-up kernels ----

// Marks tissue voxels of the full-padded build block with their cell index.
__global__ void build_voxel_map_kernel(int64_t n, const int64_t* __restrict__ gid, int nx, int ny, int64_t bx,
                                       int64_t bxy, int64_t* __restrict__ map, int64_t* __restrict__ cellVoxel)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t g = gid ? gid[i] : i;
  const int64_t x = g % nx, y = (g / nx) % ny, z = g / ((int64_t)nx * ny);
  const int64_t v = (x + 1) + bx * (y + 1) + bxy * (z + 1);
  map[v] = i;
  cellVoxel[i] = v;
}

// Weights of every cell (fgr_cell_weights), written in the tissue's class
// layout: FP64 rows = A0 then the class nodes; mixed rows = class nodes.
__global__ void build_weights_kernel(int64_t n, const int64_t* __restrict__ map, const int64_t* __restrict__ cellVoxel,
                                     const double* __restrict__ sigma6, int64_t bx, int64_t bxy, double hx, double hy,
                                     double hz, int cls, int mixed, void* __restrict__ wout)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t v = cellVoxel[i];
  int tissue[19];
  int64_t nbrCell[19];
  for (int k = 0; k < 19; ++k) {
    const int64_t c = map[v + node_dx(k) + bx * node_dy(k) + bxy * node_dz(k)];
    nbrCell[k] = c;
    tissue[k] = c >= 0;
  }
  double W[19];
  fgr_cell_weights(tissue, [&](int k, int c) { return sigma6[6 * nbrCell[k] + c]; }, hx, hy, hz, W);
  const int rows = class_rows(cls);
  if (mixed) {
    float* w = (float*)wout;
    for (int r = 1; r < rows; ++r) w[(r - 1) * n + i] = (float)W[class_node(cls, r)];
  } else {
    double* w = (double*)wout;
    w[i] = W[0];
    for (int r = 1; r < rows; ++r) w[r * n + i] = W[class_node(cls, r)];
  }
}

// Scatter / gather between cell order and the padded block.
__device__ __forceinline__ int64_t cell_voxel(int64_t i, const int64_t* __restrict__ voxel, int nx, int ny,
                                              int64_t px, int64_t pxy, int py0, int pz0)
{
  if (voxel) return voxel[i];
  const int64_t x = i % nx, y = (i / nx) % ny, z = i / ((int64_t)nx * ny);
  return (x + 1) + px * (y + py0) + pxy * (z + pz0);
}

__global__ void scatter_vm_kernel(int64_t n, const double* __restrict__ src, double* __restrict__ blk,
                                  const int64_t* __restrict__ voxel, int nx, int ny, int64_t px, int64_t pxy, int py0,
                                  int pz0)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) blk[cell_voxel(i, voxel, nx, ny, px, pxy, py0, pz0)] = src[i];
}

__global__ void gather_vm_kernel(int64_t n, const double* __restrict__ blk, double* __restrict__ dst,
                                 const int64_t* __restrict__ voxel, int nx, int ny, int64_t px, int64_t pxy, int py0,
                                 int pz0)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = blk[cell_voxel(i, voxel, nx, ny, px, pxy, py0, pz0)];
}

__global__ void init_state_kernel(int64_t n, double* s64, float* s32, int mixed, double* act)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (mixed) {
    for (int k = 0; k < 5; ++k) s64[k * n + i] = tt06_initial_state(k);
    for (int k = 5; k < kNumStates; ++k) s32[(k - 5) * n + i] = (float)tt06_initial_state(k);
  } else {
    for (int k = 0; k < kNumStates; ++k) s64[k * n + i] = tt06_initial_state(k);
  }
  act[i] = -1.0;
}

__global__ void fill_kernel(int64_t n, double* p, double v)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

inline unsigned grid_for(int64_t n, int block) { return (unsigned)((n + block - 1) / block); }

}  // namespace cdb
