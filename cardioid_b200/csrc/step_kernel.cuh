// The fused time-step kernel and its set-up kernels.
//
// One launch per (time step, reaction type present): each warp takes warp
// tiles, runs of up to 32 consecutive cells of one tissue that share a
// reaction type and lie in one 32-cell block, so the type — and with it the
// coefficient pool — is a kernel parameter, uniform across the launch.  Per
// cell, in the order of the reference's omp loop (elec/simulationLoop.cc:183-231):
//   FGR stencil on Vm(t) (elec/FGRDiffusionOMP.cc:109-131),
//   BetterTT06 update (elec/BetterTT06.cc:1426-1649),
//   stimuli in order: box assigns (elec/BoxStimulus.cc:56-64), point adds
//   (elec/PointStimulus.cc:26-36),
//   Vm(t+dt) = Vm + dt (dVmR + dVmD + iStim) (elec/simulationLoop.cc:221-228),
//   activation time: first post-step time with Vm > 0 (elec/ActivationTimeSensor.cc:99-111),
//   min/max Vm (elec/MinMaxSensor.cc:44-67) on request.
// Vm is read from one padded block and written to the other.
//
// State and weights are stored in AoSoA blocks of 32 cells (block b holds
// row r of its 32 cells contiguously at [b][r][0..31]), so a tile's inputs
// are a few contiguous, 16-byte-aligned runs.  The kernel is persistent over
// its tiles: while a warp computes one tile it has the next tile's state
// block (and, for the mixed path, weight block) copied into shared memory
// with cp.async (double buffering), so the DRAM latency of those loads
// overlaps the reaction's arithmetic.
#pragma once
#include <cuda.h>            // CUtensorMap (the type only: tensor maps are encoded through the runtime's driver entry point)
#include <cuda_runtime.h>

#include <cfloat>

#include "common.cuh"
#include "fgr_device.cuh"
#include "tt06_step.cuh"

namespace cdb {

constexpr int kWarpsPerCta = 4;
constexpr int kCta = 32 * kWarpsPerCta;
constexpr int kBlk = 32;   // cells per AoSoA block

struct TissueDev {
  double* vm[2];
  double* s64;            // AoSoA: FP64 [nb][18][32]; mixed [nb][5][32]
  float* s32;             // AoSoA: mixed [nb][13][32]
  const void* w;          // AoSoA: FP64 [nb][rows][32] doubles; mixed [nb][rows-1][32] floats
  const int64_t* voxel;    // masked tissues: padded voxel of every cell, in cell order
  const int* vrel;         // per slot: voxel offset from its tile's vox0
  double* act;             // per slot
  int64_t n;
  int64_t nSlots, nVox;   // sizes of the slot arrays and of each padded Vm block (checked builds)
  int64_t px, pxy;        // padded strides
  int nx, ny, nz;
  int py0, pz0;           // 1 when y (z) is padded
  int cls;
  int nstim, stim0;
  int parity;             // buffer holding Vm at the start of the next launch batch
  int actAll;             // Vm was written by the host since the last step
  int64_t step0;          // steps taken at the start of the next launch batch
  int64_t timeOff;        // time at step s is StepArgs::times[timeOff + s]
  double scale;           // diffusionScale (0: no diffusion)
  BlockScale blk;
  unsigned long long* minmax;   // 2 slots
  // ECG pseudo-sensor (off when ecgN == 0): electrodes at ecgPts (x y z, mm),
  // evaluated when the step count reaches a multiple of ecgRate into entry
  // (count / ecgRate) % kEcgRing of ecgTrace ([kEcgRing][ecgN]); ecgInvr
  // holds 1 / |r - p_j| per slot ([block][electrode][32], double on the
  // FP64 path, float on the mixed path; the reference's 1/r table,
  // elec/ECGSensor.cu:9-40).
  int ecgN, ecgRate;
  const double* ecgPts;
  double* ecgTrace;
  const void* ecgInvr;
  double hx, hy, hz;          // voxel spacing, mm
  // Stage 3: a TMA tensor map over each padded Vm block (x, y, z extents
  // px, ny + 2, nz + 2; box 36 x 3 x 3 doubles), for volume tissues with
  // even strides (zero otherwise).
  CUtensorMap vmMap[2];
};

// A warp tile: one 32-slot AoSoA block of one tissue, whose slots hold
// cells of one reaction type (count of them, the rest are padding).  Lane l
// works on slot first + l, whose voxel in the padded Vm block is vox0 plus
// the slot's offset (TissueDev::vrel).  Bit k of stimMask is set when
// stimulus k's box holds a cell of the tile.  flags: kTileRow when the
// tile's cells are the consecutive voxels vox0, vox0 + 1, ... of one x-row
// of a volume tissue whose padded strides are even: its stencil reads the
// 3 x 3 rows of 34 voxels around them, which stage 3 loads into shared
// memory as one TMA box of 36 x 3 x 3 at padded coordinates (wx, wy, wz):
// wx = the even x at or below the first cell's x - 1, wy and wz the row's
// y - 1 and z - 1.
constexpr int kTileRow = 1;
struct __align__(16) WarpTile {
  int tissue;
  int count;
  int64_t first;
  int64_t vox0;
  unsigned stimMask;
  int flags;
  int wx, wy, wz;
  int pad;
};
constexpr int kDescBytes = sizeof(WarpTile);
static_assert(kDescBytes == 48, "tile descriptors are copied as three 16-byte chunks");

constexpr int kEcgRing = 1024;
constexpr int kEcgMaxPoints = 32;

// A lane's running min/max of Vm for one tissue over the warp's tiles of a
// min/max step; the warp reduces it and adds it to the tissue's sensor when
// the tissue changes and at the end (two atomics per warp, not per tile).
struct MinMaxAcc {
  double lo, hi;
  int tissue;
};

// A warp's running ECG sums for one tissue and one evaluation entry, in
// shared memory (acc[j]: electrode j), added to the trace when either
// changes.
struct EcgAcc {
  double* acc;
  int tissue;
  int entry;
  int seen = -1;        // tissue whose evaluation entry is evalEntry (-1: none this launch)
  int evalEntry = -1;
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
  int stage;                  // 1: stage the next tile through shared memory (cp.async), 2: with bulk copies
  int* err;                   // set to CDB_TIMEOUT when a bounded wait gives up
  int withhold;               // test of the bounded waits (stage 2): issue no copies after each warp's first tile
  int nTissues;               // sizes of the tissue and time tables (checked builds)
  int64_t nTimes;
};

// Index guard of the checked build (compiled with CDB_BOUNDS_CHECK, the
// stand-in for a memory checker on a pool where compute-sanitizer is
// closed): an index outside [0, n) records CDB_BOUNDS_FAULT in the engine's
// error word (cdb_engine_sync returns it) and is replaced by 0, so the
// access stays inside the array.  In the normal build it is the identity.
struct IndexCheck {
  int64_t n;
  int* err;
  __device__ __forceinline__ int64_t operator()(int64_t i) const
  {
#ifdef CDB_BOUNDS_CHECK
    if ((unsigned long long)i >= (unsigned long long)n) {
      atomicCAS(err, 0, (int)CDB_BOUNDS_FAULT);
      return 0;
    }
#endif
    return i;
  }
};

__constant__ TT06Scalars c_scal[CDB_MAX_REACTION_TYPES];
__constant__ FitShape c_shape[CDB_MAX_REACTION_TYPES];
__constant__ double c_coef64[CDB_MAX_REACTION_TYPES * kFitPoolPerType];
__constant__ __align__(16) float c_coef32[CDB_MAX_REACTION_TYPES * kFitPoolPerType];   // paired layout for compiled slots (fit_pair32)

// AoSoA row sizes
constexpr int kRows64 = kNumStates;                 // FP64 state rows
constexpr int kRowsMixed64 = 5, kRowsMixed32 = 13;  // mixed state rows
__host__ __device__ constexpr int weight_rows(int cls, bool mixed) { return mixed ? class_rows(cls) - 1 : class_rows(cls); }

// Shared-memory staging per warp and buffer: the mixed path stages its state
// block and its weight block (up to 18 float rows), the FP64 path its state
// block (its weights are read directly); both stage the slots' voxel offsets.
// WGT: the mixed path's weight block is staged too (not in stage 3, whose
// Vm window takes its shared memory; there the weights stream from global
// memory).
template <bool MIXED, bool WGT = true>
__host__ __device__ constexpr int vrel_offset()
{
  return MIXED ? (kRowsMixed64 * kBlk * 8 + kRowsMixed32 * kBlk * 4 + (WGT ? 18 * kBlk * 4 : 0)) : kRows64 * kBlk * 8;
}
template <bool MIXED, bool WGT = true>
__host__ __device__ constexpr int stage_bytes()
{
  return vrel_offset<MIXED, WGT>() + kBlk * 4 + kDescBytes;   // + the next tile's descriptor
}

// Stage 3's Vm window of a row tile: rows (dy, dz) in {-1, 0, 1}^2, row
// r = (dy + 1) + 3 (dz + 1), each kWinRow doubles from the even x at or
// below the tile's first x - 1 (the TMA box, [z][y][x] in shared memory);
// the tile's cells and their x neighbours lie within the first 35 of them.
constexpr int kWinRow = 36;
constexpr int kWinBytes = 9 * kWinRow * 8;
// A TMA tensor copy's shared-memory destination must be 128-byte aligned:
// the window region starts on a 128-byte boundary of the (128-byte aligned)
// dynamic shared memory and each warp's window takes a multiple of 128.
__host__ __device__ constexpr int align128(int b) { return (b + 127) / 128 * 128; }
constexpr int kWinStride = align128(kWinBytes);

// Dynamic shared memory of a launch: per warp two staging buffers (stages
// 1-3), three mbarriers (stages 2-3: the two buffers and the window) and,
// for the window variant (win), one Vm window and no staged weights.
template <bool MIXED, bool WGT>
__host__ __device__ constexpr int win_base()
{
  return align128(kWarpsPerCta * (2 * stage_bytes<MIXED, WGT>() + 3 * 8));
}
template <bool MIXED>
__host__ __device__ constexpr int step_smem_bytes(int stage, bool win)
{
  return stage == 0 ? 0
                    : win ? win_base<MIXED, false>() + kWarpsPerCta * kWinStride
                          : kWarpsPerCta * (2 * stage_bytes<MIXED>() + 3 * 8);
}

__device__ __forceinline__ double pulse_value(const cdb_stimulus& s, double time)
{
  if (!(time > s.t0 && time < s.tf)) return 0.0;
  const double t = time - floor(time / s.period) * s.period;
  return (t >= s.phase && t < s.phase + s.duration) ? s.amplitude : 0.0;
}

__device__ __forceinline__ int64_t node_offset(int64_t px, int64_t pxy, int node)
{
  return (int64_t)node_dx(node) + px * node_dy(node) + pxy * node_dz(node);
}

// FP64 stencil in the reference's order: A0 phi0 + sum_k A_k phi_k; w points
// at the cell's row-0 weight, rows kBlk apart.
template <int CLS>
__device__ __forceinline__ double stencil64(const double* __restrict__ w, int64_t px, int64_t pxy,
                                            const double* __restrict__ vin, int64_t vox, double phi0,
                                            const IndexCheck& vchk)
{
  double tmp = __ldg(w) * phi0;
#pragma unroll
  for (int r = 1; r < class_rows(CLS); ++r) {
    const int node = class_node(CLS, r);
    tmp += __ldg(w + r * kBlk) * __ldg(vin + vchk(vox + node_offset(px, pxy, node)));
  }
  return tmp;
}

// Mixed stencil: sum_k A_k (phi_k - phi0) with FP32 weights (from shared
// memory); the differences are taken in FP64 (A0 = -sum A_k).
template <int CLS>
__device__ __forceinline__ double stencil32(const float* __restrict__ w, int64_t px, int64_t pxy,
                                            const double* __restrict__ vin, int64_t vox, double phi0,
                                            const IndexCheck& vchk)
{
  float tmp = 0.f;
#pragma unroll
  for (int r = 1; r < class_rows(CLS); ++r) {
    const int node = class_node(CLS, r);
    const float d = (float)(__ldg(vin + vchk(vox + node_offset(px, pxy, node))) - phi0);
    tmp = fmaf(w[(r - 1) * kBlk], d, tmp);
  }
  return (double)tmp;
}

// The same two stencils reading the neighbours from a stage-3 window: c
// points at the cell's own voxel in the centre row, so neighbour (dx, dy,
// dz) is c[dx + kWinRow (dy + 3 dz)], a compile-time offset.  Same
// operands and order as the global versions, so the same results bit for
// bit.
__host__ __device__ constexpr int win_offset(int node)
{
  return node_dx(node) + kWinRow * (node_dy(node) + 3 * node_dz(node));
}
__device__ __forceinline__ double stencil64_win(const double* __restrict__ w, const double* c, double phi0)
{
  double tmp = __ldg(w) * phi0;
#pragma unroll
  for (int r = 1; r < class_rows(kVolume); ++r) tmp += __ldg(w + r * kBlk) * c[win_offset(class_node(kVolume, r))];
  return tmp;
}
__device__ __forceinline__ double stencil32_win(const float* __restrict__ w, const double* c, double phi0)
{
  float tmp = 0.f;
#pragma unroll
  for (int r = 1; r < class_rows(kVolume); ++r) {
    const float d = (float)(c[win_offset(class_node(kVolume, r))] - phi0);
    tmp = fmaf(w[(r - 1) * kBlk], d, tmp);
  }
  return (double)tmp;
}

// State access of one cell in an AoSoA block: reads from the staged copy,
// writes to the global block.
struct IOBlock64 {
  const double* __restrict__ src;   // [18][32], at the cell's column
  double* __restrict__ dst;
  template <int K> __device__ __forceinline__ double get() const { return src[K * kBlk]; }
  template <int K> __device__ __forceinline__ void put(double v) const { dst[K * kBlk] = v; }
};

struct IOBlockMixed {
  const double* __restrict__ src64;   // [5][32]
  const float* __restrict__ src32;    // [13][32]
  double* __restrict__ dst64;
  float* __restrict__ dst32;
  template <int K> __device__ __forceinline__ double get() const
  {
    if (K < 5) return src64[K * kBlk];
    return (double)src32[(K - 5) * kBlk];
  }
  template <int K> __device__ __forceinline__ void put(double v) const
  {
    if (K < 5) dst64[K * kBlk] = v;
    else dst32[(K - 5) * kBlk] = (float)v;
  }
};

__device__ __forceinline__ void cp_async16(void* smemDst, const void* gmemSrc)
{
  const unsigned d = (unsigned)__cvta_generic_to_shared(smemDst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmemSrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// The warp copies `bytes` (a multiple of 16) from global to shared memory,
// 16 bytes per lane per round.
__device__ __forceinline__ void warp_copy(unsigned char* dst, const unsigned char* src, int bytes, int lane)
{
  for (int c = lane * 16; c < bytes; c += 32 * 16) cp_async16(dst + c, src + c);
}

// Copies a tile descriptor into shared memory (16 bytes per lane).
__device__ __forceinline__ void stage_desc(const WarpTile* src, WarpTile* dst, int lane)
{
  if (lane < kDescBytes / 16) cp_async16((unsigned char*)dst + lane * 16, (const unsigned char*)src + lane * 16);
}

// Copies a tile's state block (and, mixed, weight block) into buf.
template <bool MIXED>
__device__ __forceinline__ void stage_tile(const StepArgs& a, const WarpTile& tile, int lane, unsigned char* buf)
{
  const TissueDev* __restrict__ Tp = a.tissues + IndexCheck{a.nTissues, a.err}(tile.tissue);
  const int64_t b = IndexCheck{Tp->nSlots, a.err}(tile.first) / kBlk;
  if (MIXED) {
    warp_copy(buf, (const unsigned char*)(Tp->s64 + b * kRowsMixed64 * kBlk), kRowsMixed64 * kBlk * 8, lane);
    warp_copy(buf + kRowsMixed64 * kBlk * 8, (const unsigned char*)(Tp->s32 + b * kRowsMixed32 * kBlk),
              kRowsMixed32 * kBlk * 4, lane);
    if (Tp->scale != 0.0) {
      const int wr = weight_rows(Tp->cls, true);
      warp_copy(buf + kRowsMixed64 * kBlk * 8 + kRowsMixed32 * kBlk * 4,
                (const unsigned char*)((const float*)Tp->w + b * wr * kBlk), wr * kBlk * 4, lane);
    }
  } else {
    warp_copy(buf, (const unsigned char*)(Tp->s64 + b * kRows64 * kBlk), kRows64 * kBlk * 8, lane);
  }
  warp_copy(buf + vrel_offset<MIXED>(), (const unsigned char*)(Tp->vrel + b * kBlk), kBlk * 4, lane);
}

__device__ __forceinline__ void minmax_flush(const StepArgs& a, MinMaxAcc& acc, int lane)
{
  if (acc.tissue >= 0) {
    double lo = acc.lo, hi = acc.hi;
    for (int o = 16; o > 0; o >>= 1) {
      lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (lane == 0) {
      unsigned long long* mm = a.tissues[acc.tissue].minmax;
      atomicMin(mm, ordered_bits(lo));
      atomicMax(mm + 1, ordered_bits(hi));
    }
  }
  acc.tissue = -1;
  acc.lo = __longlong_as_double(0x7ff0000000000000ll);
  acc.hi = -__longlong_as_double(0x7ff0000000000000ll);
}

__device__ __forceinline__ void ecg_flush(const StepArgs& a, EcgAcc& acc, int lane)
{
  __syncwarp();
  if (acc.tissue >= 0) {
    const TissueDev* __restrict__ T = a.tissues + acc.tissue;
    if (lane < T->ecgN) atomicAdd(T->ecgTrace + (int64_t)acc.entry * T->ecgN + lane, acc.acc[lane]);
  }
  acc.acc[lane] = 0.0;
  __syncwarp();
  acc.tissue = -1;
}

// Sums 8 values per lane over the warp with 9 shuffles (instead of 8 x 5):
// each round halves the values a lane keeps and swaps the other half with
// the partner lane.  Lane l ends with the sum of value (l >> 2) & 7.
__device__ __forceinline__ double warp_sum8(const double (&v)[8], int lane)
{
  const bool h4 = lane & 16, h3 = lane & 8, h2 = lane & 4;
  double w[4], u[2];
#pragma unroll
  for (int q = 0; q < 4; ++q)
    w[q] = (h4 ? v[q + 4] : v[q]) + __shfl_xor_sync(0xffffffffu, h4 ? v[q] : v[q + 4], 16);
#pragma unroll
  for (int q = 0; q < 2; ++q)
    u[q] = (h3 ? w[q + 2] : w[q]) + __shfl_xor_sync(0xffffffffu, h3 ? w[q] : w[q + 2], 8);
  double r = (h2 ? u[1] : u[0]) + __shfl_xor_sync(0xffffffffu, h2 ? u[0] : u[1], 4);
  r += __shfl_xor_sync(0xffffffffu, r, 2);
  r += __shfl_xor_sync(0xffffffffu, r, 1);
  return r;
}

// ---- bulk (TMA) staging: one lane issues cp.async.bulk copies of the
// tile's contiguous blocks, completing on the buffer's mbarrier ----

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity)
{
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void bulk_copy(void* dst, const void* src, unsigned bytes, unsigned long long* bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Bounded wait for a buffer's copies (every lane): false once about a
// second has passed on the GPU's global timer (checked every 64 polls), or
// after 2^20 polls, each of which the hardware may suspend for a while.
constexpr int kWaitPolls = 1 << 20;
constexpr unsigned long long kWaitNs = 1000000000ull;
__device__ __forceinline__ unsigned long long global_ns()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity)
{
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (int i = 0; i < kWaitPolls; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 63) == 63 && global_ns() - t0 > kWaitNs) return false;
  }
  return false;
}

// Lane 0: copies a tile's state block, weight block (mixed) and voxel
// offsets, and the descriptor of the tile after it (when there is one),
// into buf, all completing on bar.
template <bool MIXED, bool WGT = true>
__device__ __forceinline__ void stage_tile_bulk(const StepArgs& a, const WarpTile& tile, unsigned char* buf,
                                                const WarpTile* nextDesc, WarpTile* descDst, unsigned long long* bar)
{
  const TissueDev* __restrict__ Tp = a.tissues + IndexCheck{a.nTissues, a.err}(tile.tissue);
  const int64_t b = IndexCheck{Tp->nSlots, a.err}(tile.first) / kBlk;
  unsigned bytes = kBlk * 4 + (nextDesc ? (unsigned)kDescBytes : 0u);
  int wr = 0;
  if (MIXED) {
    bytes += kRowsMixed64 * kBlk * 8 + kRowsMixed32 * kBlk * 4;
    if (WGT && Tp->scale != 0.0) wr = weight_rows(Tp->cls, true);
    bytes += wr * kBlk * 4;
  } else {
    bytes += kRows64 * kBlk * 8;
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // after this warp's reads of buf
  mbar_expect_tx(bar, bytes);
  if (MIXED) {
    bulk_copy(buf, Tp->s64 + b * kRowsMixed64 * kBlk, kRowsMixed64 * kBlk * 8, bar);
    bulk_copy(buf + kRowsMixed64 * kBlk * 8, Tp->s32 + b * kRowsMixed32 * kBlk, kRowsMixed32 * kBlk * 4, bar);
    if (wr)
      bulk_copy(buf + kRowsMixed64 * kBlk * 8 + kRowsMixed32 * kBlk * 4, (const float*)Tp->w + b * wr * kBlk,
                wr * kBlk * 4, bar);
  } else {
    bulk_copy(buf, Tp->s64 + b * kRows64 * kBlk, kRows64 * kBlk * 8, bar);
  }
  bulk_copy(buf + vrel_offset<MIXED, WGT>(), Tp->vrel + b * kBlk, kBlk * 4, bar);
  if (nextDesc) bulk_copy(descDst, nextDesc, kDescBytes, bar);
}

// A tile's stage-3 window: where its rows are copied and how the warp
// waits for them (win null: the tile reads its neighbours from global
// memory).
struct TileWindow {
  const double* win;            // the warp's window buffer
  unsigned long long* bar;      // its mbarrier
  unsigned parity;              // phase parity of this tile's copies
};

// Lane 0: loads the stencil window of row tile `tile` from Vm buffer `cur`
// into the warp's window buffer with one TMA tensor copy (the box of 36 x 3
// x 3 doubles at the tile's (wx, wy, wz); its x coordinate is even, so the
// copy starts on a 16-byte boundary), completing on bar (stage 3).  Box
// parts past the block's x extent read as zero: the stencil never uses them.
// False, with CDB_BOUNDS_FAULT recorded and no copy issued, when the
// destination (128 bytes), the tensor map (64 bytes) or the box's x
// coordinate (16 bytes of doubles) is not aligned: the tile then reads its
// neighbours from global memory.
__device__ __forceinline__ bool stage_window(const TissueDev* __restrict__ Tp, const WarpTile* tile, int cur,
                                             double* win, unsigned long long* bar, int* err)
{
  const int wx = tile->wx, wy = tile->wy, wz = tile->wz;
  if ((smem_u32(win) & 127u) || ((unsigned long long)&Tp->vmMap[cur] & 63ull) || (wx & 1)) {
    atomicCAS(err, 0, (int)CDB_BOUNDS_FAULT);
    return false;
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // after the warp's reads of the last window
  mbar_expect_tx(bar, kWinBytes);
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_u32(win)), "l"(&Tp->vmMap[cur]), "r"(wx), "r"(wy), "r"(wz), "r"(smem_u32(bar))
      : "memory");
  return true;
}

// The BetterTT06 update of one cell (state through the staged block or
// global memory); returns dVm = -Iion.  With SPEC the slot is a template
// parameter, so every coefficient address is a compile-time constant.
template <bool MIXED, int SLOT>
__device__ __forceinline__ double react_cell(const StepArgs& a, const TissueDev* __restrict__ Tp, int64_t b, int pos,
                                             const unsigned char* buf, bool staged, double phi0)
{
  constexpr bool SPEC = SLOT >= 0;
  const BlockScale blk = Tp->blk;
  const int rt = SPEC ? SLOT : a.rt;
  const double* c64 = c_coef64 + rt * kFitPoolPerType;
  if (MIXED) {
    double* g64 = Tp->s64 + b * kRowsMixed64 * kBlk + pos;
    float* g32 = Tp->s32 + b * kRowsMixed32 * kBlk + pos;
    IOBlockMixed io{staged ? (const double*)buf + pos : g64,
                    staged ? (const float*)(buf + kRowsMixed64 * kBlk * 8) + pos : g32, g64, g32};
    const float* c32 = c_coef32 + rt * kFitPoolPerType;
    if (SPEC) {
      SpecFits fits{c64, c32};
      return (double)tt06_step_mixed(c_scal[rt], blk, fits, (float)a.dt, phi0, io);
    }
    GenericFits fits{c64, c32, &c_shape[rt]};
    return (double)tt06_step_mixed(c_scal[rt], blk, fits, (float)a.dt, phi0, io);
  }
  double* g64 = Tp->s64 + b * kRows64 * kBlk + pos;
  IOBlock64 io{staged ? (const double*)buf + pos : g64, g64};
  if (SPEC) {
    SpecFits fits{c64, nullptr};
    return tt06_step(c_scal[rt], blk, fits, a.dt, phi0, io);
  }
  GenericFits fits{c64, nullptr, &c_shape[rt]};
  return tt06_step(c_scal[rt], blk, fits, a.dt, phi0, io);
}

// dVmD of one cell, neighbours from global memory: scale (A0 phi0 +
// sum_k A_k phi_k) (FP64) or scale sum_k A_k (phi_k - phi0) (mixed).
template <bool MIXED, bool WGT = true>
__device__ __forceinline__ double stencil_global(const TissueDev* __restrict__ Tp, int64_t b, int pos,
                                                 const unsigned char* buf, bool staged, const double* vin,
                                                 int64_t vox, double phi0, const IndexCheck& vchk)
{
  const int cls = Tp->cls;
  const int64_t px = Tp->px, pxy = Tp->pxy;
  double acc;
  if (MIXED) {
    const float* w = WGT && staged ? (const float*)(buf + kRowsMixed64 * kBlk * 8 + kRowsMixed32 * kBlk * 4) + pos
                                   : (const float*)Tp->w + b * weight_rows(cls, true) * kBlk + pos;
    acc = cls == kVolume ? stencil32<kVolume>(w, px, pxy, vin, vox, phi0, vchk)
        : cls == kSheet ? stencil32<kSheet>(w, px, pxy, vin, vox, phi0, vchk)
                        : stencil32<kCable>(w, px, pxy, vin, vox, phi0, vchk);
  } else {
    const double* w = (const double*)Tp->w + b * weight_rows(cls, false) * kBlk + pos;
    acc = cls == kVolume ? stencil64<kVolume>(w, px, pxy, vin, vox, phi0, vchk)
        : cls == kSheet ? stencil64<kSheet>(w, px, pxy, vin, vox, phi0, vchk)
                        : stencil64<kCable>(w, px, pxy, vin, vox, phi0, vchk);
  }
  return acc * Tp->scale;
}

// Vm(t + dt) of one cell, written to vout, and its activation time
// (ActivationTimeSensor::eval, elec/ActivationTimeSensor.cc:99-111).
__device__ __forceinline__ double integrate_cell(const StepArgs& a, const TissueDev* __restrict__ Tp, int64_t i,
                                                 double* vout, int64_t vox, double phi0, double dvmR, double dvmD,
                                                 double istim, double tnext)
{
  const double vnew = phi0 + a.dt * (dvmR + dvmD + istim);
  vout[vox] = vnew;
  // Once Vm has gone above 0 the cell's activation time is set, so a cell
  // with Vm > 0 at the start of the step already has one; only upward
  // crossings need to read it, except in the first step after the host
  // wrote Vm.
  if (vnew > 0.0 && (phi0 <= 0.0 || (a.k == 0 && Tp->actAll))) {
    double* ap = Tp->act + i;
    if (*ap < 0.0) *ap = tnext;
  }
  return vnew;
}

// One tile.  With `staged` the tile's state (and mixed weights) are read
// from buf; otherwise straight from global memory.  WIN (stage 3): the
// stencil runs after the reaction, on a row tile's rows copied into shared
// memory while the reaction computed (tw.win; other tiles read global
// memory); false when the wait for them gave up (the engine's error word
// says CDB_TIMEOUT).
template <bool MIXED, int SLOT, bool ECG, bool WIN>
__device__ __forceinline__ bool step_tile(const StepArgs& a, const WarpTile& tile, int lane, const unsigned char* buf,
                                          bool staged, const TileWindow& tw, EcgAcc& ecg, MinMaxAcc& mm)
{
  const TissueDev* __restrict__ Tp = a.tissues + IndexCheck{a.nTissues, a.err}(tile.tissue);
  const IndexCheck tchk{a.nTimes, a.err};
  const int64_t lstep = Tp->step0 + a.k;
  const double time = a.times[tchk(Tp->timeOff + lstep)];
  const double tnext = a.times[tchk(Tp->timeOff + lstep + 1)];
  const bool active = lane < tile.count;
  // lanes past the tile's end stand in for its first cell until the end
  const int l = active ? lane : 0;
  const IndexCheck schk{Tp->nSlots, a.err}, vchk{Tp->nVox, a.err};
  const int64_t i = schk(tile.first + l);
  constexpr bool WGT = !WIN;     // stage 3 streams the weights from global memory
  const int rel = staged ? ((const int*)(buf + vrel_offset<MIXED, WGT>()))[l] : Tp->vrel[i];
  const int64_t vox = vchk(tile.vox0 + rel);
  const int64_t px = Tp->px, pxy = Tp->pxy;
  // iStim = 0, then the stimuli whose boxes hold a cell of the tile, in order
  double istim = 0.0;
  if (tile.stimMask) {
    const int stim0 = Tp->stim0;
    // lane s holds stimulus s's value at this time
    const double stimVal = lane < Tp->nstim ? pulse_value(a.stims[stim0 + lane], time) : 0.0;
    const int64_t zz = vox / pxy, rem = vox - zz * pxy, yy = rem / px;
    const int x = (int)(rem - yy * px) - 1, y = (int)yy - Tp->py0, z = (int)zz - Tp->pz0;
    for (unsigned m = tile.stimMask; m; m &= m - 1) {
      const int k = __ffs(m) - 1;
      const double v = __shfl_sync(0xffffffffu, stimVal, k);
      if (v != 0.0) {
        const cdb_stimulus* bx = a.stims + stim0 + k;
        if (x > bx->xMin && x < bx->xMax && y > bx->yMin && y < bx->yMax && z > bx->zMin && z < bx->zMax)
          istim = bx->mode == CDB_STIM_POINT ? istim + v : v;
      }
    }
  }
  const int64_t b = i / kBlk;
  const int pos = (int)(i - b * kBlk);
  const int cur = (Tp->parity + a.k) & 1;
  const double* __restrict__ vin = Tp->vm[cur];
  double* __restrict__ vout = Tp->vm[cur ^ 1];
  double vnew = 0.0;
  double ecgSrc = 0.0;        // the cell's dVmD, the ECG's source term
  if (!WIN) {
    if (active) {
      const double phi0 = vin[vox];
      const double dvmD = Tp->scale != 0.0 ? stencil_global<MIXED>(Tp, b, pos, buf, staged, vin, vox, phi0, vchk) : 0.0;
      ecgSrc = dvmD;
      const double dvmR = react_cell<MIXED, SLOT>(a, Tp, b, pos, buf, staged, phi0);
      vnew = integrate_cell(a, Tp, i, vout, vox, phi0, dvmR, dvmD, istim, tnext);
    }
  } else {
    double phi0 = 0.0, dvmR = 0.0, dvmD = 0.0;
    if (active) {
      phi0 = vin[vox];
      dvmR = react_cell<MIXED, SLOT>(a, Tp, b, pos, buf, staged, phi0);
    }
    if (tw.win) {
      // the row tile's window, copied while the reaction computed (every lane waits)
      if (!__all_sync(0xffffffffu, mbar_wait(tw.bar, tw.parity))) {
        if (lane == 0) atomicExch(a.err, (int)CDB_TIMEOUT);
        mbar_wait(tw.bar, tw.parity);      // let its copies land before the warp leaves
        return false;
      }
      if (active && Tp->scale != 0.0) {
        const double* c = tw.win + 4 * kWinRow + (int)((tile.vox0 - 1) & 1) + 1 + l;
        if (MIXED)
          dvmD = stencil32_win((const float*)Tp->w + b * weight_rows(kVolume, true) * kBlk + pos, c, phi0);
        else
          dvmD = stencil64_win((const double*)Tp->w + b * weight_rows(kVolume, false) * kBlk + pos, c, phi0);
        dvmD *= Tp->scale;
      }
    } else if (active && Tp->scale != 0.0) {
      dvmD = stencil_global<MIXED, WGT>(Tp, b, pos, buf, staged, vin, vox, phi0, vchk);
    }
    ecgSrc = dvmD;
    if (active) vnew = integrate_cell(a, Tp, i, vout, vox, phi0, dvmR, dvmD, istim, tnext);
  }
  if (a.minmax) {
    if (mm.tissue != tile.tissue) {
      minmax_flush(a, mm, lane);
      mm.tissue = tile.tissue;
    }
    if (active) {
      mm.lo = fmin(mm.lo, vnew);
      mm.hi = fmax(mm.hi, vnew);
      // a non-finite Vm stays non-finite, so checking at the batch's last
      // step catches it; the first error recorded is kept
      if (!(fabs(vnew) <= DBL_MAX)) atomicCAS(a.err, 0, (int)CDB_NUMERIC_FAULT);
    }
  }
  // ECG (ECGSensor::eval / calcEcg, elec/ECGSensor.cc:231-320 and
  // elec/ECGSensor.cu:9-168): after the step, on evaluation steps, electrode
  // j gets sum over cells of dVmD / |r - p_j| with r = (x dx, y dy, z dz).
  // Whether this launch evaluates a tissue is fixed per tissue: the warp
  // works it out when its tiles move to another tissue.
  if (ECG && ecg.seen != tile.tissue) {
    ecg.seen = tile.tissue;
    ecg.evalEntry = Tp->ecgN && (lstep + 1) % Tp->ecgRate == 0 ? (int)(((lstep + 1) / Tp->ecgRate) % kEcgRing) : -1;
  }
  if (ECG && ecg.evalEntry >= 0) {
    const int ecgN = Tp->ecgN;
    const int entry = ecg.evalEntry;
    if (ecg.tissue != tile.tissue || ecg.entry != entry) {
      ecg_flush(a, ecg, lane);
      ecg.tissue = tile.tissue;
      ecg.entry = entry;
    }
    const int64_t at = b * ecgN * kBlk + pos;
    const double* __restrict__ inv64 = (const double*)Tp->ecgInvr + at;
    const float* __restrict__ inv32 = (const float*)Tp->ecgInvr + at;
    for (int g = 0; g < ecgN; g += 8) {
      double v[8];
#pragma unroll
      for (int q = 0; q < 8; ++q)
        v[q] = active && g + q < ecgN ? ecgSrc * (MIXED ? (double)inv32[(g + q) * kBlk] : inv64[(g + q) * kBlk])
                                      : 0.0;
      const double sum = warp_sum8(v, lane);
      const int e = g + ((lane >> 2) & 7);
      if ((lane & 3) == 0 && e < ecgN) ecg.acc[e] += sum;
    }
    // the tissue's first tile clears the entry the next evaluation fills
    if (tile.first == 0 && lane < ecgN)
      Tp->ecgTrace[(int64_t)((entry + 1) % kEcgRing) * ecgN + lane] = 0.0;
  }
  return true;
}

// Resident CTAs per SM the register budget aims at: 4 for FP64 (16 warps,
// at most 128 registers) and 5 for mixed (20 warps, at most 102 registers,
// which its shared-memory buffers also allow).  The default launches (mixed
// bulk-staged, FP64 direct loads) do not spill; within this budget the
// mixed window variant spills 4-12 bytes per thread, the mixed ECG
// variants 4, the FP64 window variant 32 and the generic kernels (run-time
// fit shapes) 12-116 (ptxas -v).
#ifndef CDB_FP64_MIN_CTAS
#define CDB_FP64_MIN_CTAS 4
#endif
#ifndef CDB_MIXED_MIN_CTAS
#define CDB_MIXED_MIN_CTAS 5
#endif
template <bool MIXED>
constexpr int min_ctas() { return MIXED ? CDB_MIXED_MIN_CTAS : CDB_FP64_MIN_CTAS; }

// Persistent over the launch's warp tiles: warp w takes tiles w, w + W,
// w + 2W, ... (W warps in the grid).  With a.stage set, the next tile's
// state (and mixed weights) is in flight to shared memory while the current
// one computes.
// SLOT >= 0: the launch's reaction type is constant-memory slot SLOT and its
// fits have the compiled shapes (fit_shapes.h); SLOT < 0: any slot (a.rt)
// with run-time shapes.
// WIN: the stage-3 variant (Vm windows of row tiles; only stage-3 launches
// of the compiled slots without ECG use it).
template <bool MIXED, int SLOT, bool ECG, bool WIN>
__global__ void __launch_bounds__(kCta, min_ctas<MIXED>()) fused_step_kernel(StepArgs a)
{
  constexpr bool WGT = !WIN;
  constexpr int kBuf = stage_bytes<MIXED, WGT>();
  // dynamic: step_smem_bytes<MIXED>(a.stage, WIN) bytes (none for stage 0)
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ double ecgSmem[ECG ? kWarpsPerCta * 32 : 1];   // each warp's ECG sums
  const int lane = threadIdx.x & 31;
  const int warpInCta = threadIdx.x >> 5;
  double* const ecgMine = ecgSmem + (ECG ? warpInCta * 32 : 0);
  if (ECG) {
    ecgMine[lane] = 0.0;
    __syncwarp();
  }
  unsigned char* mine = smem + warpInCta * 2 * kBuf;
  const int stride = gridDim.x * kWarpsPerCta;
  int t = blockIdx.x * kWarpsPerCta + warpInCta;
  const TileWindow noWin{nullptr, nullptr, 0};
  if (!WIN && !a.stage) {
    // the next tile's descriptor is in flight while this tile computes; a
    // warp past its last tile takes an empty descriptor (never an
    // uninitialised one, whose copy the compiler may treat as any value)
    EcgAcc ecg{ecgMine, -1, 0};
    MinMaxAcc mm{__longlong_as_double(0x7ff0000000000000ll), -__longlong_as_double(0x7ff0000000000000ll), -1};
    WarpTile cur = t < a.nTiles ? a.tiles[t] : WarpTile{};
    for (; t < a.nTiles; t += stride) {
      const WarpTile nxt = t + stride < a.nTiles ? a.tiles[t + stride] : WarpTile{};
      step_tile<MIXED, SLOT, ECG, false>(a, cur, lane, nullptr, false, noWin, ecg, mm);
      cur = nxt;
    }
    if (ECG) ecg_flush(a, ecg, lane);
    if (a.minmax) minmax_flush(a, mm, lane);
    return;
  }
  if (WIN || a.stage >= 2) {
    // Bulk copies: lane 0 issues, for tile t + stride, cp.async.bulk copies
    // of its contiguous blocks (and of the descriptor after it) into the
    // other buffer while the warp computes tile t; every lane waits on the
    // buffer's mbarrier, phase (iteration / 2) & 1.  Stage 3 also copies a
    // row tile's nine stencil rows into the warp's window at the start of
    // its iteration (third mbarrier, phase = windows so far & 1), read after
    // the reaction.
    unsigned long long* bars = (unsigned long long*)(smem + kWarpsPerCta * 2 * kBuf) + warpInCta * 3;
    double* const win = WIN ? (double*)(smem + win_base<MIXED, WGT>() + warpInCta * kWinStride) : nullptr;
    WarpTile* const desc0 = (WarpTile*)(mine + vrel_offset<MIXED, WGT>() + kBlk * 4);
    WarpTile* const desc1 = (WarpTile*)(mine + kBuf + vrel_offset<MIXED, WGT>() + kBlk * 4);
    if (lane == 0) {
      mbar_init(bars, 1);
      mbar_init(bars + 1, 1);
      mbar_init(bars + 2, 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    EcgAcc ecg{ecgMine, -1, 0};
    MinMaxAcc mm{__longlong_as_double(0x7ff0000000000000ll), -__longlong_as_double(0x7ff0000000000000ll), -1};
    WarpTile cur = t < a.nTiles ? a.tiles[t] : WarpTile{};
    if (t < a.nTiles && lane == 0)
      stage_tile_bulk<MIXED, WGT>(a, cur, mine, t + stride < a.nTiles ? a.tiles + t + stride : nullptr, desc0, bars);
    unsigned windows = 0;
    for (int it = 0; t < a.nTiles; ++it, t += stride) {
      const int tn = t + stride;
      const int bi = it & 1;
      if (!__all_sync(0xffffffffu, mbar_wait(bars + bi, (it >> 1) & 1))) {
        if (lane == 0) atomicExch(a.err, (int)CDB_TIMEOUT);
        mbar_wait(bars + bi, (it >> 1) & 1);    // let its copies land before the warp leaves
        return;
      }
      __syncwarp();           // every lane is past the wait and done with the other buffer (and the window)
      const WarpTile nxt = tn < a.nTiles ? *(bi ? desc1 : desc0) : WarpTile{};
      const bool next = tn < a.nTiles && !a.withhold;
      TileWindow tw = noWin;
      if (WIN && (cur.flags & kTileRow)) {
        // the window's box origin, from this tile's descriptor: in global
        // memory for the first tile, else still in the slot the next copy
        // overwrites (so before that copy is issued)
        bool issued = false;
        if (lane == 0) {
          const TissueDev* __restrict__ Tp = a.tissues + IndexCheck{a.nTissues, a.err}(cur.tissue);
          issued = stage_window(Tp, it == 0 ? a.tiles + t : (bi ? desc0 : desc1), (Tp->parity + a.k) & 1, win,
                                bars + 2, a.err);
        }
        if (__shfl_sync(0xffffffffu, issued, 0)) {
          tw = TileWindow{win, bars + 2, windows & 1u};
          ++windows;
        }
      }
      if (next && lane == 0)
        stage_tile_bulk<MIXED, WGT>(a, nxt, mine + (bi ^ 1) * kBuf,
                               tn + stride < a.nTiles ? a.tiles + tn + stride : nullptr, bi ? desc0 : desc1,
                               bars + (bi ^ 1));
      if (!step_tile<MIXED, SLOT, ECG, WIN>(a, cur, lane, mine + bi * kBuf, true, tw, ecg, mm)) {
        if (next) mbar_wait(bars + (bi ^ 1), ((it + 1) >> 1) & 1);   // the next tile's copies, in flight
        return;
      }
      cur = nxt;
    }
    if (ECG) ecg_flush(a, ecg, lane);
    if (a.minmax) minmax_flush(a, mm, lane);
    return;
  }
  if (WIN) return;
  // Buffer i holds tile t's inputs and the descriptor of tile t + stride,
  // copied together one iteration ahead.
  WarpTile* desc0 = (WarpTile*)(mine + vrel_offset<MIXED>() + kBlk * 4);
  WarpTile* desc1 = (WarpTile*)(mine + kBuf + vrel_offset<MIXED>() + kBlk * 4);
  if (t < a.nTiles) {
    const WarpTile first = a.tiles[t];
    stage_tile<MIXED>(a, first, lane, mine);
    if (t + stride < a.nTiles) stage_desc(a.tiles + t + stride, desc0, lane);
  }
  cp_async_commit();
  WarpTile cur = t < a.nTiles ? a.tiles[t] : WarpTile{};
  EcgAcc ecg{ecgMine, -1, 0};
  MinMaxAcc mm{__longlong_as_double(0x7ff0000000000000ll), -__longlong_as_double(0x7ff0000000000000ll), -1};
  for (int it = 0; t < a.nTiles; ++it, t += stride) {
    const int tn = t + stride;
    WarpTile* mineDesc = (it & 1) ? desc1 : desc0;        // descriptor of tile tn, copied with tile t
    WarpTile* nextDesc = (it & 1) ? desc0 : desc1;
    cp_async_wait_all();    // tile t's inputs and tile tn's descriptor (copied during the last tile) have landed
    __syncwarp();           // for every lane, and every lane is done with the other buffer
    const WarpTile nxt = tn < a.nTiles ? *mineDesc : WarpTile{};
    if (tn < a.nTiles) {
      stage_tile<MIXED>(a, nxt, lane, mine + ((it + 1) & 1) * kBuf);
      if (tn + stride < a.nTiles) stage_desc(a.tiles + tn + stride, nextDesc, lane);
    }
    cp_async_commit();
    step_tile<MIXED, SLOT, ECG, false>(a, cur, lane, mine + (it & 1) * kBuf, true, noWin, ecg, mm);
    cur = nxt;
  }
  cp_async_wait_all();
  if (ECG) ecg_flush(a, ecg, lane);
  if (a.minmax) minmax_flush(a, mm, lane);
}

// The compiled kernel of a slot when the type has the compiled fit shapes
// (slot >= 0), else the generic kernel; with the ECG sensor compiled in or
// out (only launches that hold a tissue with electrodes pay for it); for
// stage 3, the compiled slots without ECG run the window variant (the
// others run stage 3 as stage 2).
template <bool MIXED, bool ECG, bool WIN>
inline void (*step_kernel_of(int slot))(StepArgs)
{
  static_assert(CDB_MAX_REACTION_TYPES == 6, "one compiled kernel per slot");
  switch (slot) {
    case 0: return fused_step_kernel<MIXED, 0, ECG, WIN>;
    case 1: return fused_step_kernel<MIXED, 1, ECG, WIN>;
    case 2: return fused_step_kernel<MIXED, 2, ECG, WIN>;
    case 3: return fused_step_kernel<MIXED, 3, ECG, WIN>;
    case 4: return fused_step_kernel<MIXED, 4, ECG, WIN>;
    case 5: return fused_step_kernel<MIXED, 5, ECG, WIN>;
    default: return fused_step_kernel<MIXED, -1, ECG, false>;
  }
}

// Whether a launch runs the window variant.
inline bool step_uses_window(int slot, bool ecg, int stage) { return stage == 3 && !ecg && slot >= 0; }

template <bool MIXED>
inline void (*step_kernel_for(int slot, bool ecg, int stage))(StepArgs)
{
  if (ecg) return step_kernel_of<MIXED, true, false>(slot);
  return stage == 3 ? step_kernel_of<MIXED, false, true>(slot) : step_kernel_of<MIXED, false, false>(slot);
}

template <bool MIXED>
inline int step_launch_smem(int slot, bool ecg, int stage)
{
  return step_smem_bytes<MIXED>(stage, step_uses_window(slot, ecg, stage));
}

// One step of one reaction type (dynamic shared memory for a.stage).
template <bool MIXED>
inline void launch_step(int slot, bool ecg, unsigned grid, cudaStream_t stream, const StepArgs& a)
{
  step_kernel_for<MIXED>(slot, ecg, a.stage)<<<grid, kCta, step_launch_smem<MIXED>(slot, ecg, a.stage), stream>>>(a);
}

// Lets every step kernel of a precision take stage 3's dynamic shared
// memory (above the default 48 KB limit); once per device, before any
// launch or capture.
template <bool MIXED>
inline cudaError_t allow_step_smem()
{
  for (int slot = -1; slot < CDB_MAX_REACTION_TYPES; ++slot)
    for (int v = 0; v < 3; ++v) {        // ECG, no ECG, window variant
      const cudaError_t e = cudaFuncSetAttribute(step_kernel_for<MIXED>(slot, v == 0, v == 2 ? 3 : 2),
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 step_launch_smem<MIXED>(slot, v == 0, v == 2 ? 3 : 2));
      if (e != cudaSuccess) return e;
    }
  return cudaSuccess;
}

// CTAs of a slot's kernel that are resident on one SM at once with the
// stage's shared memory (0 on error).
template <bool MIXED>
inline int resident_ctas(int slot, bool ecg, int stage)
{
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, step_kernel_for<MIXED>(slot, ecg, stage), kCta,
                                                    step_launch_smem<MIXED>(slot, ecg, stage)) != cudaSuccess)
    return 0;
  return n;
}

__global__ void advance_kernel(TissueDev* tissues, int nTissues, int k)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nTissues) {
    tissues[t].step0 += k;
    tissues[t].parity = (tissues[t].parity + k) & 1;
    tissues[t].actAll = 0;
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

// AoSoA index of row r of cell i
__host__ __device__ inline int64_t aosoa(int64_t i, int rows, int r)
{
  return ((i / kBlk) * rows + r) * kBlk + (i % kBlk);
}

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

// Weights of every cell (fgr_cell_weights), written AoSoA at the cell's
// slot in the tissue's class layout: FP64 rows = A0 then the class nodes;
// mixed rows = class nodes.
__global__ void build_weights_kernel(int64_t n, const int64_t* __restrict__ map, const int64_t* __restrict__ cellVoxel,
                                     const double* __restrict__ sigma6, int64_t bx, int64_t bxy, double hx, double hy,
                                     double hz, int cls, int mixed, const int64_t* __restrict__ slot,
                                     void* __restrict__ wout)
{
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  const int64_t v = cellVoxel[c];
  const int64_t i = slot[c];
  int tissue[19];
  int64_t nbrCell[19];
  for (int k = 0; k < 19; ++k) {
    const int64_t nb = map[v + node_dx(k) + bx * node_dy(k) + bxy * node_dz(k)];
    nbrCell[k] = nb;
    tissue[k] = nb >= 0;
  }
  double W[19];
  fgr_cell_weights(tissue, [&](int k, int e) { return sigma6[6 * nbrCell[k] + e]; }, hx, hy, hz, W);
  const int rows = class_rows(cls);
  if (mixed) {
    float* w = (float*)wout;
    for (int r = 1; r < rows; ++r) w[aosoa(i, rows - 1, r - 1)] = (float)W[class_node(cls, r)];
  } else {
    double* w = (double*)wout;
    w[aosoa(i, rows, 0)] = W[0];
    for (int r = 1; r < rows; ++r) w[aosoa(i, rows, r)] = W[class_node(cls, r)];
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

// 1 / |r - p_j| for every cell and electrode, at the cell's slot
// (invr[block][electrode][32], float when mixed); r = (x hx, y hy, z hz) as the step's
// voxel decomposition gives it (ECGSensor's calcInvr_kernel,
// elec/ECGSensor.cu:9-40).
__global__ void ecg_invr_kernel(int64_t n, const int64_t* __restrict__ slot, const int64_t* __restrict__ voxel, int nx,
                                int ny, int64_t px, int64_t pxy, int py0, int pz0, double hx, double hy, double hz,
                                const double* __restrict__ pts, int nPts, int mixed, void* __restrict__ invr)
{
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  const int64_t vox = cell_voxel(c, voxel, nx, ny, px, pxy, py0, pz0);
  const int64_t zz = vox / pxy, rem = vox - zz * pxy, yy = rem / px;
  const double xr = (double)((int)(rem - yy * px) - 1) * hx;
  const double yr = (double)((int)yy - py0) * hy;
  const double zr = (double)((int)zz - pz0) * hz;
  const int64_t i = slot[c], b = i / kBlk;
  const int64_t at = b * nPts * kBlk + (i - b * kBlk);
  for (int j = 0; j < nPts; ++j) {
    const double ex = xr - pts[3 * j], ey = yr - pts[3 * j + 1], ez = zr - pts[3 * j + 2];
    const double r = 1.0 / sqrt(ex * ex + ey * ey + ez * ez);
    if (mixed) ((float*)invr)[at + j * kBlk] = (float)r;
    else ((double*)invr)[at + j * kBlk] = r;
  }
}

// Writes host-given Vm of cells c0 .. c0+n-1 into a padded block; sets
// *actAll (when given) so the next step checks every cell's activation time.
__global__ void scatter_vm_kernel(int64_t c0, int64_t n, const double* __restrict__ src, double* __restrict__ blk,
                                  const int64_t* __restrict__ voxel, int nx, int ny, int64_t px, int64_t pxy, int py0,
                                  int pz0, int* actAll)
{
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t i = c0 + j;
  if (j < n) blk[cell_voxel(i, voxel, nx, ny, px, pxy, py0, pz0)] = src[i];
  if (j == 0 && actAll) *actAll = 1;
}

__global__ void gather_vm_kernel(int64_t c0, int64_t n, const double* __restrict__ blk, double* __restrict__ dst,
                                 const int64_t* __restrict__ voxel, int nx, int ny, int64_t px, int64_t pxy, int py0,
                                 int pz0)
{
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t i = c0 + j;
  if (j < n) dst[i] = blk[cell_voxel(i, voxel, nx, ny, px, pxy, py0, pz0)];
}

// Row var of the AoSoA state to / from a cell-order array of doubles
// (slot[c]: the slot of cell c).
__global__ void gather_state_kernel(int64_t n, const int64_t* __restrict__ slot, const double* __restrict__ s64,
                                    const float* __restrict__ s32, int mixed, int var, double* __restrict__ dst)
{
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  const int64_t i = slot[c];
  if (!mixed) dst[c] = s64[aosoa(i, kRows64, var)];
  else if (var < kRowsMixed64) dst[c] = s64[aosoa(i, kRowsMixed64, var)];
  else dst[c] = (double)s32[aosoa(i, kRowsMixed32, var - kRowsMixed64)];
}

__global__ void scatter_state_kernel(int64_t n, const int64_t* __restrict__ slot, double* __restrict__ s64,
                                     float* __restrict__ s32, int mixed, int var, const double* __restrict__ src)
{
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  const int64_t i = slot[c];
  if (!mixed) s64[aosoa(i, kRows64, var)] = src[c];
  else if (var < kRowsMixed64) s64[aosoa(i, kRowsMixed64, var)] = src[c];
  else s32[aosoa(i, kRowsMixed32, var - kRowsMixed64)] = (float)src[c];
}

// Per-slot values (activation times) to cell order.
__global__ void gather_slots_kernel(int64_t n, const int64_t* __restrict__ slot, const double* __restrict__ src,
                                    double* __restrict__ dst)
{
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c < n) dst[c] = src[slot[c]];
}

// Initial state and activation time of every slot (padding slots too).
__global__ void init_state_kernel(int64_t nSlots, double* s64, float* s32, int mixed, double* act)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nSlots) return;
  if (mixed) {
    for (int k = 0; k < kRowsMixed64; ++k) s64[aosoa(i, kRowsMixed64, k)] = tt06_initial_state(k);
    for (int k = kRowsMixed64; k < kNumStates; ++k)
      s32[aosoa(i, kRowsMixed32, k - kRowsMixed64)] = (float)tt06_initial_state(k);
  } else {
    for (int k = 0; k < kNumStates; ++k) s64[aosoa(i, kRows64, k)] = tt06_initial_state(k);
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
