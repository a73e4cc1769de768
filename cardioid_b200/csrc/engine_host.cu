// Fused monodomain engine: one kernel per time step does, for every tissue
// cell, the FGR stencil on Vm(t), the BetterTT06 update, the box stimuli,
// the integrator Vm(t+dt) = Vm + dt (dVmR + dVmD + iStim) and the sensors
// (activation time, min/max Vm), in the order of the reference's omp loop
// (elec/simulationLoop.cc:183-231), reading Vm from one buffer and writing
// the other so Vm crosses HBM once per step.
//
// HBM layout, per tissue (all arrays separate cudaMalloc allocations, so
// tissues join and retire between steps without moving anyone else):
//   vm[2]      padded Vm blocks (halo of one voxel, zero, never written)
//              in x-fastest order; only dimensions longer than one voxel
//              are padded (a cable is nx+2 long, a sheet (nx+2)(ny+2));
//   slots      cells grouped by reaction type, each group padded to whole
//              32-slot blocks (slot map: cell -> slot);
//   s64, s32   state, AoSoA blocks of 32 slots: FP64 path 18 rows of
//              double; mixed path 5 rows of double (Ca_SR Ca_i Ca_ss K_i
//              Na_i) and 13 of float (R_prime and the 12 gates);
//   w          stencil weights, AoSoA (FP64: A0 and the class's nodes in
//              double; mixed: the class's nodes without A0 in float);
//   vrel       per slot, int32 voxel offset from its block's first voxel;
//   voxel      (masked tissues only) int64 padded-voxel index per cell;
//   act        activation time per slot.
// A warp-tile table, grouped by reaction type, maps each warp to one block
// (step_kernel.cuh).
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <array>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "fgr_device.cuh"
#include "reaction_slot.h"
#include "step_kernel.cuh"

namespace cdb {

thread_local std::string t_last_error;

// A named NVTX range over one entry point, so the engine's phases show in a
// timeline profiler (the counterpart of the reference's PerformanceTimers /
// USE_NVTX ranges, elec/PerformanceTimers.hh:72-84, cudaNVTX.h:3-25); free
// when no tool is attached.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};
void set_error(const std::string& msg) { t_last_error = msg; }
int64_t g_launches = 0;

// ---- host engine ----

struct DeviceBuffer {
  void* p = nullptr;
  size_t bytes = 0;
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  ~DeviceBuffer() { release(); }
  cudaError_t alloc(size_t b)
  {
    release();
    bytes = b;
    return b ? cudaMalloc(&p, b) : cudaSuccess;
  }
  void release()
  {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <typename T>
  T* as() const { return (T*)p; }
};

struct HostTissue {
  TissueDev dev{};
  std::vector<cdb_stimulus> stims;
  DeviceBuffer vm0, vm1, s64, s32, w, voxel, act, minmax;
  std::vector<WarpTile> tiles[CDB_MAX_REACTION_TYPES];   // by slot; .tissue set at rebuild
  int64_t nSlots = 0;               // AoSoA slots (cells plus padding)
  std::vector<int64_t> slot;        // slot of every cell
  DeviceBuffer slotMap, vrel;       // device copies: cell -> slot; per-slot voxel offsets
  DeviceBuffer ecgPts, ecgTrace;    // ECG electrodes and trace ring (cdb_engine_set_ecg)
  DeviceBuffer ecgInvr;             // 1/r per slot and electrode
  double ecgK = 0;                  // kconst * dx dy dz
  int64_t ecgNext = 0;              // next evaluation (step / rate) to hand to the host
  int64_t steps = 0;       // steps taken
  int clock = 0;           // its time sequence (Engine::clocks)
  int parity = 0;
  int64_t n = 0;
  int nx = 0, ny = 0, nz = 0;
  // Chunked host step (cdb_engine_step_host): chunk j holds cells
  // pipeCell[j] .. pipeCell[j+1]-1, whole planes of the slowest grid axis;
  // its compute launches take the tiles whose stencil needs no later chunk
  // (per slot, local tiles up to pipeTiles[j][slot]).  Output range j,
  // cells outCell[j] .. outCell[j+1]-1, is final once compute chunk
  // pipeOut[j] has run.  pipeK = 1: one chunk.
  int pipeK = 1;
  std::vector<int64_t> pipeCell, outCell;
  std::vector<int> pipeOut;
  std::vector<std::array<int64_t, CDB_MAX_REACTION_TYPES>> pipeTiles;
};

// Constant-memory reaction slots are a per-device resource shared by every
// engine and plugin reaction of the process.  Registrations with identical
// content (scalars, fit shape, coefficient pool) share a slot, reference
// counted; a slot is uploaded when it is taken and reused once released.
struct SlotEntry {
  int refs = 0;
  bool spec = false;                 // pool packed for the compiled fit shapes
  std::vector<unsigned char> key;    // the uploaded content
};
std::mutex g_slot_mutex;
std::map<int, std::vector<SlotEntry>> g_slots;

// The slot holding this content (uploaded when new); -1 when every slot is
// taken (err stays cudaSuccess) or the upload failed (err set).  The
// caller has made `device` current.
int acquire_slot(int device, const TT06Scalars& scal, const FitShape& shape, const std::vector<double>& pool,
                 bool spec, cudaError_t& err)
{
  std::vector<unsigned char> key(sizeof(scal) + sizeof(shape) + pool.size() * sizeof(double) + 1);
  unsigned char* k = key.data();
  std::memcpy(k, &scal, sizeof(scal));
  std::memcpy(k + sizeof(scal), &shape, sizeof(shape));
  std::memcpy(k + sizeof(scal) + sizeof(shape), pool.data(), pool.size() * sizeof(double));
  key.back() = spec ? 1 : 0;
  std::lock_guard<std::mutex> lock(g_slot_mutex);
  std::vector<SlotEntry>& used = g_slots[device];
  used.resize(CDB_MAX_REACTION_TYPES);
  for (int s = 0; s < CDB_MAX_REACTION_TYPES; ++s)
    if (used[s].refs > 0 && used[s].key == key) {
      ++used[s].refs;
      return s;
    }
  for (int s = 0; s < CDB_MAX_REACTION_TYPES; ++s) {
    if (used[s].refs > 0) continue;
    // the compiled kernels' FP32 forms (shifted fits) for a specialised
    // pool, in the paired layout of fit_pair32
    std::vector<float> pool32(pool.begin(), pool.end());
    if (spec) {
      if (!spec_pool32(pool.data(), pool32.data(), (int)pool.size())) return -1;
      std::vector<float> paired(pool32.size());
      spec_pair_pool32(pool32.data(), paired.data(), (int)paired.size());
      pool32.swap(paired);
    }
    err = cudaMemcpyToSymbol(c_scal, &scal, sizeof(scal), s * sizeof(TT06Scalars));
    if (err == cudaSuccess) err = cudaMemcpyToSymbol(c_shape, &shape, sizeof(shape), s * sizeof(FitShape));
    if (err == cudaSuccess)
      err = cudaMemcpyToSymbol(c_coef64, pool.data(), pool.size() * sizeof(double),
                               (size_t)s * kFitPoolPerType * sizeof(double));
    if (err == cudaSuccess)
      err = cudaMemcpyToSymbol(c_coef32, pool32.data(), pool32.size() * sizeof(float),
                               (size_t)s * kFitPoolPerType * sizeof(float));
    if (err != cudaSuccess) return -1;
    used[s].refs = 1;
    used[s].spec = spec;
    used[s].key = std::move(key);
    return s;
  }
  return -1;
}

void release_slot(int device, int slot)
{
  std::lock_guard<std::mutex> lock(g_slot_mutex);
  std::vector<SlotEntry>& used = g_slots[device];
  if (slot >= 0 && slot < (int)used.size() && used[slot].refs > 0) --used[slot].refs;
}

struct Engine {
  cdb_engine_config cfg{};
  cudaStream_t stream = nullptr;
  int nTypes = 0;
  int slots[CDB_MAX_REACTION_TYPES] = {0};   // constant-memory slot of each reaction id
  bool spec[CDB_MAX_REACTION_TYPES] = {false};   // slot packed for the compiled fit shapes
  std::map<int, std::unique_ptr<HostTissue>> tissues;
  int nextId = 0;
  bool dirty = true;
  // tables
  DeviceBuffer dTissues, dTiles, dStims, dTimes, dStage, dErr;
  // Time sequences: clock c gives time[s] = clocks[c].times[s - base] for
  // step s >= base, accumulated as time += dt like the reference
  // (elec/simulationLoop.cc:230).  Clock 0 starts at step 0, time 0; a
  // restarted tissue (cdb_engine_set_clock) may need its own.  dTimes holds
  // all of them back to back, clock c from offset clocks[c].off.
  struct Clock {
    int64_t base;
    std::vector<double> times;
    int64_t off;
  };
  std::vector<Clock> clocks{Clock{0, {0.0}, 0}};
  std::vector<int> order;         // tissue ids in table order
  int64_t nTiles = 0;
  std::vector<std::pair<int, std::pair<int, int>>> slotTiles;   // slot -> (first tile, tile count)
  int64_t launches = 0;
  // graph of a launch batch
  cudaGraphExec_t graph = nullptr;
  int graphSteps = 0;
  bool graphMinmax = false;
  // launch tuning (cdb_engine_set_tuning; the autotuner picks them)
  int stage = 0;           // staging mode (set per precision at creation)
  bool withhold = false;   // cdb_engine_test_bounded_wait: the next batch withholds its bulk copies
  int ctasPerSm = 0;       // persistent grid: SMs x this; 0 = as many as are resident
  int layout = CDB_LAYOUT_ROWS;    // warp-tile layout of tissues added from here on
  int numSms = 148;
  // resident CTAs per SM by [stage][ECG][slot] (last: generic)
  int resident[4][2][CDB_MAX_REACTION_TYPES + 1] = {};
  bool anyEcg = false;     // a tissue has ECG electrodes: launch the kernels with the sensor
  bool windowSlot[CDB_MAX_REACTION_TYPES] = {};   // stage 3 runs this type's launches with Vm windows

  int grid_ctas_per_sm(int slot, int st)
  {
    if (ctasPerSm > 0) return ctasPerSm;
    int& r = resident[st][anyEcg ? 1 : 0][slot < 0 ? CDB_MAX_REACTION_TYPES : slot];
    if (r == 0)
      r = cfg.precision == CDB_MIXED ? resident_ctas<true>(slot, anyEcg, st) : resident_ctas<false>(slot, anyEcg, st);
    return r > 0 ? r : 4;
  }

  // copy streams and events of the chunked host step
  cudaStream_t sIn = nullptr, sOut = nullptr;
  cudaEvent_t evStart = nullptr, evOut = nullptr;
  std::vector<cudaEvent_t> evIn, evComp;
  DeviceBuffer dStageOut;
  // graphs of the chunked host step with page-locked host buffers, one per
  // (Vm in, Vm out, parity): a time loop that alternates two buffers uses two
  struct HostStepGraph {
    const double* in;
    double* out;
    int parity;
    cudaGraphExec_t exec;
    int64_t launches;
  };
  std::vector<HostStepGraph> hostGraphs;

  // Every captured graph goes whenever what it captured may change (tables,
  // time table, tuning, staging buffers).
  void drop_graphs()
  {
    if (graph) cudaGraphExecDestroy(graph);
    graph = nullptr;
    for (const HostStepGraph& g : hostGraphs) cudaGraphExecDestroy(g.exec);
    hostGraphs.clear();
  }

  cudaError_t ensure_pipe(int K)
  {
    cudaError_t err = cudaSuccess;
    if (!sIn) err = cudaStreamCreateWithFlags(&sIn, cudaStreamNonBlocking);
    if (err == cudaSuccess && !sOut) err = cudaStreamCreateWithFlags(&sOut, cudaStreamNonBlocking);
    if (err == cudaSuccess && !evStart) err = cudaEventCreateWithFlags(&evStart, cudaEventDisableTiming);
    if (err == cudaSuccess && !evOut) err = cudaEventCreateWithFlags(&evOut, cudaEventDisableTiming);
    while (err == cudaSuccess && (int)evIn.size() < K) {
      cudaEvent_t a = nullptr, b = nullptr;
      err = cudaEventCreateWithFlags(&a, cudaEventDisableTiming);
      if (err == cudaSuccess) err = cudaEventCreateWithFlags(&b, cudaEventDisableTiming);
      if (a) evIn.push_back(a);
      if (b) evComp.push_back(b);
    }
    return err;
  }

  ~Engine()
  {
    drop_graphs();
    tissues.clear();
    for (cudaEvent_t ev : evIn) cudaEventDestroy(ev);
    for (cudaEvent_t ev : evComp) cudaEventDestroy(ev);
    if (evStart) cudaEventDestroy(evStart);
    if (evOut) cudaEventDestroy(evOut);
    if (sIn) cudaStreamDestroy(sIn);
    if (sOut) cudaStreamDestroy(sOut);
    if (stream) cudaStreamDestroy(stream);
    for (int t = 0; t < nTypes; ++t) release_slot(cfg.device, slots[t]);
  }

  // Every tissue's clock covers `extra` steps past its current step (+1 for
  // the time after the last of them); re-uploads dTimes when a clock grew.
  cdb_status ensure_times(int64_t extra)
  {
    std::vector<int64_t> need(clocks.size(), 1);
    for (auto& kv : tissues) {
      const Clock& c = clocks[kv.second->clock];
      need[kv.second->clock] = std::max(need[kv.second->clock], kv.second->steps - c.base + extra + 1);
    }
    bool grew = dTimes.p == nullptr;
    for (size_t c = 0; c < clocks.size(); ++c) {
      std::vector<double>& t = clocks[c].times;
      if ((int64_t)t.size() >= need[c]) continue;
      // at least 2^16 steps at a time: a re-upload drains the stream and
      // re-captures the step graph, so it must stay rare in long runs
      const int64_t want = std::max<int64_t>(need[c], std::max<int64_t>((int64_t)t.size() * 2, int64_t(1) << 16));
      t.reserve(want);
      while ((int64_t)t.size() < want) t.push_back(t.back() + cfg.dt);
      grew = true;
    }
    if (!grew) return CDB_OK;
    std::vector<double> all;
    for (Clock& c : clocks) {
      c.off = (int64_t)all.size();
      all.insert(all.end(), c.times.begin(), c.times.end());
    }
    CDB_CUDA(cudaStreamSynchronize(stream));
    CDB_CUDA(dTimes.alloc(all.size() * sizeof(double)));
    CDB_CUDA(cudaMemcpy(dTimes.p, all.data(), all.size() * sizeof(double), cudaMemcpyHostToDevice));
    drop_graphs();
    dirty = true;   // tissues' time offsets
    return CDB_OK;
  }

  double tissue_time(const HostTissue& t) const
  {
    const Clock& c = clocks[t.clock];
    return c.times[t.steps - c.base];
  }

  cdb_status rebuild()
  {
    if (!dirty) return CDB_OK;
    CDB_CUDA(cudaStreamSynchronize(stream));
    order.clear();
    std::vector<TissueDev> devs;
    std::vector<WarpTile> tiles;
    std::vector<WarpTile> bySlot[CDB_MAX_REACTION_TYPES];
    std::vector<cdb_stimulus> stims;
    anyEcg = false;
    for (auto& kv : tissues) {
      HostTissue& t = *kv.second;
      anyEcg = anyEcg || t.dev.ecgN > 0;
      t.dev.stim0 = (int)stims.size();
      t.dev.nstim = (int)t.stims.size();
      stims.insert(stims.end(), t.stims.begin(), t.stims.end());
      t.dev.step0 = t.steps;
      t.dev.parity = t.parity;
      t.dev.timeOff = clocks[t.clock].off - clocks[t.clock].base;
      const int idx = (int)devs.size();
      devs.push_back(t.dev);
      order.push_back(kv.first);
      for (int sl = 0; sl < CDB_MAX_REACTION_TYPES; ++sl)
        for (WarpTile tl : t.tiles[sl]) {
          tl.tissue = idx;
          bySlot[sl].push_back(tl);
        }
    }
    slotTiles.clear();
    for (int sl = 0; sl < CDB_MAX_REACTION_TYPES; ++sl) {
      // stage 3 uses the window variant for a type's launches only when at
      // least half of its tiles are row tiles (the variant runs the others
      // slower than stage 2: stencil after the reaction, weights unstaged)
      int64_t rows = 0;
      for (const WarpTile& tl : bySlot[sl]) rows += (tl.flags & kTileRow) ? 1 : 0;
      windowSlot[sl] = !bySlot[sl].empty() && 2 * rows >= (int64_t)bySlot[sl].size();
      if (bySlot[sl].empty()) continue;
      slotTiles.push_back({sl, {(int)tiles.size(), (int)bySlot[sl].size()}});
      tiles.insert(tiles.end(), bySlot[sl].begin(), bySlot[sl].end());
    }
    nTiles = (int64_t)tiles.size();
    CDB_CUDA(dTissues.alloc(std::max<size_t>(1, devs.size()) * sizeof(TissueDev)));
    CDB_CUDA(dTiles.alloc(std::max<size_t>(1, tiles.size()) * sizeof(WarpTile)));
    CDB_CUDA(dStims.alloc(std::max<size_t>(1, stims.size()) * sizeof(cdb_stimulus)));
    if (!devs.empty())
      CDB_CUDA(cudaMemcpy(dTissues.p, devs.data(), devs.size() * sizeof(TissueDev), cudaMemcpyHostToDevice));
    if (!tiles.empty())
      CDB_CUDA(cudaMemcpy(dTiles.p, tiles.data(), tiles.size() * sizeof(WarpTile), cudaMemcpyHostToDevice));
    if (!stims.empty())
      CDB_CUDA(cudaMemcpy(dStims.p, stims.data(), stims.size() * sizeof(cdb_stimulus), cudaMemcpyHostToDevice));
    drop_graphs();
    dirty = false;
    return CDB_OK;
  }

  // Host copies of step0/parity/actAll follow the device ones (advance_kernel).
  void advance_host(int k)
  {
    for (auto& kv : tissues) {
      kv.second->steps += k;
      kv.second->parity = (kv.second->parity + k) & 1;
      kv.second->dev.actAll = 0;
    }
  }

  // Device address of a tissue's actAll flag; null while the tables are
  // stale (the next rebuild uploads the host copy).
  int* act_all_flag(int id)
  {
    if (dirty) return nullptr;
    for (size_t k = 0; k < order.size(); ++k)
      if (order[k] == id) return &dTissues.as<TissueDev>()[k].actAll;
    return nullptr;
  }

  // Step s of a batch for tiles first .. first+count-1 of the table (all
  // of slot rt).
  void launch_tiles(int rt, int64_t first, int64_t count, int s, bool minmax, cudaStream_t st)
  {
    StepArgs a;
    a.tissues = dTissues.as<TissueDev>();
    a.tiles = dTiles.as<WarpTile>() + first;
    a.nTiles = (int)count;
    a.rt = rt;
    a.stims = dStims.as<cdb_stimulus>();
    a.times = dTimes.as<double>();
    a.dt = cfg.dt;
    a.k = s;
    a.minmax = minmax ? 1 : 0;
    a.stage = withhold ? 2 : (stage == 3 && !windowSlot[rt]) ? 2 : stage;
    a.err = dErr.as<int>();
    a.withhold = withhold ? 1 : 0;
    a.nTissues = (int)order.size();
    a.nTimes = (int64_t)(dTimes.bytes / sizeof(double));
    const int slot = spec[rt] ? rt : -1;
    const unsigned grid = (unsigned)std::min<int64_t>(grid_for(a.nTiles, kWarpsPerCta),
                                                      (int64_t)numSms * grid_ctas_per_sm(slot, a.stage));
    if (cfg.precision == CDB_MIXED) launch_step<true>(slot, anyEcg, grid, st, a);
    else launch_step<false>(slot, anyEcg, grid, st, a);
    ++launches;
  }

  cdb_status launch_batch(int k, bool minmax)
  {
    const int nT = (int)order.size();
    if (minmax) {
      reset_minmax_kernel<<<grid_for(nT, 128), 128, 0, stream>>>(dTissues.as<TissueDev>(), nT);
      ++launches;
    }
    for (int s = 0; s < k; ++s)
      for (const auto& st : slotTiles)
        launch_tiles(st.first, st.second.first, st.second.second, s, minmax && s == k - 1, stream);
    advance_kernel<<<grid_for(nT, 128), 128, 0, stream>>>(dTissues.as<TissueDev>(), nT, k);
    ++launches;
    return CDB_OK;
  }

  cdb_status step(int k, bool minmax = true)
  {
    CDB_CHECK(k >= 0, CDB_INVALID_ARG, "nSteps must be >= 0");
    if (k == 0 || tissues.empty()) return CDB_OK;
    cdb_status st = ensure_times(k);
    if (st != CDB_OK) return st;
    st = rebuild();
    if (st != CDB_OK) return st;
    if (withhold) {
      // one batch, launched directly (never captured), then back to normal
      launch_batch(k, minmax);
      withhold = false;
      CDB_CUDA(cudaGetLastError());
      advance_host(k);
      return CDB_OK;
    }
    if (cfg.use_graphs) {
      if (!graph || graphSteps != k || graphMinmax != minmax) {
        if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
        cudaGraph_t g;
        CDB_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        const int64_t before = launches;
        launch_batch(k, minmax);
        const int64_t perBatch = launches - before;
        launches = before;
        CDB_CUDA(cudaStreamEndCapture(stream, &g));
        cudaError_t e = cudaGraphInstantiate(&graph, g, 0);
        cudaGraphDestroy(g);
        CDB_CUDA(e);
        graphSteps = k;
        graphMinmax = minmax;
        graphLaunches = perBatch;
      }
      CDB_CUDA(cudaGraphLaunch(graph, stream));
      launches += graphLaunches;
    } else {
      launch_batch(k, minmax);
    }
    CDB_CUDA(cudaGetLastError());
    advance_host(k);
    return CDB_OK;
  }
  int64_t graphLaunches = 0;
};

// ---- plugin reactions on constant-memory slots (reaction_slot.h) ----

// One cell per thread in the plugin's layout (state rows of pitch n, Vm and
// dVm through the index array), the slot's scalars and coefficients with
// the compiled fit shapes: the same arithmetic as the fused step's reaction.
template <bool MIXED, int SLOT>
__global__ void __launch_bounds__(kCta, min_ctas<MIXED>())
    reaction_slot_kernel(int64_t n, double dt, const int32_t* __restrict__ index, const double* __restrict__ Vm,
                         double* __restrict__ dVm, double* __restrict__ s64, float* __restrict__ s32)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t e = index[i];
  const double V = Vm[e];
  const BlockScale none{1.0, 1.0, 1.0};
  const double* c64 = c_coef64 + SLOT * kFitPoolPerType;
  if (MIXED) {
    IOMixed io{s64 + i, s32 + i, n};
    SpecFits fits{c64, c_coef32 + SLOT * kFitPoolPerType};
    dVm[e] = (double)tt06_step_mixed(c_scal[SLOT], none, fits, (float)dt, V, io);
  } else {
    IO64 io{s64 + i, n};
    SpecFits fits{c64, nullptr};
    dVm[e] = tt06_step(c_scal[SLOT], none, fits, dt, V, io);
  }
}

template <bool MIXED>
cudaError_t launch_reaction_slot(int slot, int64_t n, double dt, const int32_t* index, const double* Vm, double* dVm,
                                 double* s64, float* s32, cudaStream_t stream)
{
  static_assert(CDB_MAX_REACTION_TYPES == 6, "one compiled kernel per slot");
  void (*k)(int64_t, double, const int32_t*, const double*, double*, double*, float*) = nullptr;
  switch (slot) {
    case 0: k = reaction_slot_kernel<MIXED, 0>; break;
    case 1: k = reaction_slot_kernel<MIXED, 1>; break;
    case 2: k = reaction_slot_kernel<MIXED, 2>; break;
    case 3: k = reaction_slot_kernel<MIXED, 3>; break;
    case 4: k = reaction_slot_kernel<MIXED, 4>; break;
    case 5: k = reaction_slot_kernel<MIXED, 5>; break;
    default: return cudaErrorInvalidValue;
  }
  k<<<(unsigned)((n + kCta - 1) / kCta), kCta, 0, stream>>>(n, dt, index, Vm, dVm, s64, s32);
  return cudaGetLastError();
}

int reaction_slot_acquire(int device, const cdb_tt06_params& params, const cdb_fit* fits)
{
  FitShape shape{};
  std::vector<double> pool(kFitPoolPerType, 0.0);
  std::string err;
  if (!pack_fits(fits, shape, pool.data(), kFitPoolPerType, err)) return -1;
  if (!pack_fits_spec(fits, pool.data(), kFitPoolPerType)) return -1;
  if (cudaSetDevice(device) != cudaSuccess) return -1;
  cudaError_t up = cudaSuccess;
  const int slot = acquire_slot(device, to_scalars(params), shape, pool, true, up);
  return up == cudaSuccess ? slot : -1;
}

void reaction_slot_release(int device, int slot) { release_slot(device, slot); }

cudaError_t reaction_slot_calc(int slot, bool mixed, int64_t n, double dt, const int32_t* index, const double* Vm,
                               double* dVm, double* s64, float* s32, cudaStream_t stream)
{
  return mixed ? launch_reaction_slot<true>(slot, n, dt, index, Vm, dVm, s64, s32, stream)
               : launch_reaction_slot<false>(slot, n, dt, index, Vm, dVm, s64, s32, stream);
}

}  // namespace cdb

using namespace cdb;

struct cdb_engine {
  Engine e;
};

namespace {

HostTissue* find_tissue(cdb_engine* e, int32_t id)
{
  auto it = e->e.tissues.find(id);
  return it == e->e.tissues.end() ? nullptr : it->second.get();
}

int tissue_class(int nx, int ny, int nz, bool masked)
{
  if (masked) return kVolume;
  if (ny == 1 && nz == 1) return kCable;
  if (nz == 1) return kSheet;
  return kVolume;
}

cdb_status validate_desc(const Engine& E, const cdb_tissue_desc* t)
{
  CDB_CHECK(t, CDB_INVALID_ARG, "null tissue descriptor");
  CDB_CHECK(t->nx > 0 && t->ny > 0 && t->nz > 0, CDB_INVALID_ARG, "grid dimensions must be positive");
  CDB_CHECK(t->dx > 0 && t->dy > 0 && t->dz > 0, CDB_INVALID_ARG, "grid spacing must be positive");
  const int64_t grid = (int64_t)t->nx * t->ny * t->nz;
  CDB_CHECK(t->nCells > 0 && t->nCells <= grid, CDB_INVALID_ARG, "nCells must be in [1, nx*ny*nz]");
  CDB_CHECK(t->nCells < (int64_t(1) << 31), CDB_INVALID_ARG, "a tissue holds fewer than 2^31 cells");
  CDB_CHECK(t->gid || t->nCells == grid, CDB_INVALID_ARG, "gid may be NULL only for a full grid");
  CDB_CHECK(t->cellType && t->reaction && t->sigma6, CDB_INVALID_ARG, "cellType, reaction and sigma6 are required");
  CDB_CHECK(t->nStim >= 0 && t->nStim <= CDB_MAX_STIM_PER_TISSUE, CDB_INVALID_ARG, "too many stimuli for one tissue");
  CDB_CHECK(t->nStim == 0 || t->stim, CDB_INVALID_ARG, "stim is NULL");
  for (int64_t i = 0; i < t->nCells; ++i) {
    CDB_CHECK(t->cellType[i] > 0, CDB_INVALID_ARG, "cellType must be > 0 (tissue) for every cell");
    CDB_CHECK(t->reaction[i] < E.nTypes, CDB_INVALID_ARG, "reaction id out of range");
    if (t->gid) {
      CDB_CHECK(t->gid[i] >= 0 && t->gid[i] < grid, CDB_INVALID_ARG, "gid outside the grid");
      CDB_CHECK(i == 0 || t->gid[i] > t->gid[i - 1], CDB_INVALID_ARG, "gids must be strictly increasing");
    }
  }
  for (int s = 0; s < t->nStim; ++s) {
    CDB_CHECK(t->stim[s].period > 0 && t->stim[s].duration > 0, CDB_INVALID_ARG, "stimulus period and duration must be > 0");
    CDB_CHECK(t->stim[s].mode == CDB_STIM_BOX || t->stim[s].mode == CDB_STIM_POINT, CDB_INVALID_ARG,
              "stimulus mode must be CDB_STIM_BOX or CDB_STIM_POINT");
  }
  return CDB_OK;
}

int64_t padded_voxels(int nx, int ny, int nz, int cls, int64_t* px, int64_t* pxy, int* py0, int* pz0)
{
  const int64_t Px = nx + 2;
  const int64_t Py = cls >= kSheet ? ny + 2 : 1;
  const int64_t Pz = cls == kVolume ? nz + 2 : 1;
  if (px) *px = Px;
  if (pxy) *pxy = Px * Py;
  if (py0) *py0 = cls >= kSheet ? 1 : 0;
  if (pz0) *pz0 = cls == kVolume ? 1 : 0;
  return Px * Py * Pz;
}

// Slots per reaction type of a tissue: its cells grouped by type, each
// group rounded up to whole 32-slot blocks.
int64_t count_slots(int64_t n, const uint8_t* reaction, const int* slots, int64_t count[CDB_MAX_REACTION_TYPES])
{
  for (int k = 0; k < CDB_MAX_REACTION_TYPES; ++k) count[k] = 0;
  for (int64_t c = 0; c < n; ++c) ++count[slots[reaction[c]]];
  int64_t total = 0;
  for (int k = 0; k < CDB_MAX_REACTION_TYPES; ++k) total += (count[k] + kBlk - 1) / kBlk * kBlk;
  return total;
}

// The slot layout and warp tiles of a tissue.  Cells are grouped by reaction
// type (constant-memory slot, ascending), in cell order within a type, each
// group starting on a 32-slot block, so every AoSoA block holds one type and
// every warp tile is full but the last of its type (the per-type cell
// grouping of ReactionManager::create, elec/ReactionManager.cc:74-371).
// The chunk plan of cdb_engine_step_host.  Cells must be in grid order
// (non-decreasing gid), so a chunk of whole planes of the slowest axis is a
// range of cells and every reaction type's tiles reach those planes in
// order; a tile needs the planes of its cells and one past them (the
// stencil), so it is computed by the chunk holding its last cell's next
// plane.  One chunk when the tissue is small or out of grid order.
void build_pipe(HostTissue& h, const int64_t* gid, const std::vector<int64_t>& cellOf)
{
  h.pipeK = 1;
  h.pipeCell = {0, h.n};
  h.outCell = {0, h.n};
  h.pipeOut = {0};
  h.pipeTiles.assign(1, {});
  for (int k = 0; k < CDB_MAX_REACTION_TYPES; ++k) h.pipeTiles[0][k] = (int64_t)h.tiles[k].size();
  const int64_t n = h.n;
  int64_t stride = 1, planes = h.nx;
  if (h.nz > 1) {
    stride = (int64_t)h.nx * h.ny;
    planes = h.nz;
  } else if (h.ny > 1) {
    stride = h.nx;
    planes = h.ny;
  }
  // Chunks of planes/16 planes measured best on the 256^3 box (3.4 ms per
  // step against 3.8 with planes/8 and 3.7 with planes/32: smaller chunks
  // shorten the pipeline's head and tail, larger ones keep the step launches
  // long); the first and the last are half as long (head and tail shorter
  // again: 3.66 against 3.72 ms), so there are KF + 1 chunks.
  const int KF = (int)std::min<int64_t>(16, planes / 16);
  if (KF < 2 || n < (int64_t(1) << 16)) return;
  const int K = KF + 1;
  auto g = [&](int64_t c) { return gid ? gid[c] : c; };
  for (int64_t c = 1; c < n; ++c)
    if (g(c) < g(c - 1)) return;
  auto plane = [&](int64_t c) { return g(c) / stride; };
  std::vector<int64_t> P(K + 1);   // chunk j: planes P[j] .. P[j+1]-1
  for (int j = 0; j <= K; ++j) P[j] = j == 0 ? 0 : j == K ? planes : (2 * j - 1) * planes / (2 * KF);
  // Output range j: planes Q[j] .. Q[j+1]-1, one plane behind the chunks
  // (a chunk's last plane waits for the next chunk's first), so compute
  // chunk j completes output range j and its copy down starts a chunk
  // earlier than chunk j's own would.
  std::vector<int64_t> Q(K + 1);
  for (int j = 0; j <= K; ++j) Q[j] = j == 0 || j == K ? P[j] : P[j] - 1;
  auto range_of = [&](const std::vector<int64_t>& B, int64_t p) {
    int j = 0;
    while (j + 1 < K && B[j + 1] <= p) ++j;
    return j;
  };
  auto chunk_of = [&](int64_t p) { return range_of(P, p); };
  auto first_cells = [&](const std::vector<int64_t>& B) {
    std::vector<int64_t> cells(K + 1, n);
    for (int j = 1; j < K; ++j) {
      int64_t lo = 0, hi = n;   // first cell with plane >= B[j]
      while (lo < hi) {
        const int64_t mid = (lo + hi) / 2;
        if (plane(mid) >= B[j]) hi = mid;
        else lo = mid + 1;
      }
      cells[j] = lo;
    }
    cells[0] = 0;
    return cells;
  };
  std::vector<int64_t> cells = first_cells(P), outCells = first_cells(Q);
  std::vector<int> out(K, 0);
  std::vector<std::array<int64_t, CDB_MAX_REACTION_TYPES>> ends(K);
  for (int k = 0; k < CDB_MAX_REACTION_TYPES; ++k) {
    // a tile needs the chunk holding the plane after its last cell; tiles
    // are reordered (stably) by that chunk, so each chunk launches a prefix
    // of its type's tiles (the kernel takes tiles in any order)
    auto lastCell = [&](const WarpTile& tl) {
      int64_t c = cellOf[tl.first];
      for (int l = 1; l < tl.count; ++l) c = std::max(c, cellOf[tl.first + l]);
      return c;
    };
    auto firstCell = [&](const WarpTile& tl) {
      int64_t c = cellOf[tl.first];
      for (int l = 1; l < tl.count; ++l) c = std::min(c, cellOf[tl.first + l]);
      return c;
    };
    auto req = [&](const WarpTile& tl) { return chunk_of(std::min<int64_t>(plane(lastCell(tl)) + 1, planes - 1)); };
    std::stable_sort(h.tiles[k].begin(), h.tiles[k].end(),
                     [&](const WarpTile& a, const WarpTile& b) { return req(a) < req(b); });
    std::vector<int64_t> count(K, 0);
    for (const WarpTile& tl : h.tiles[k]) {
      const int r = req(tl);
      ++count[r];
      for (int o = range_of(Q, plane(firstCell(tl))); o <= range_of(Q, plane(lastCell(tl))); ++o)
        out[o] = std::max(out[o], r);
    }
    int64_t acc = 0;
    for (int j = 0; j < K; ++j) ends[j][k] = acc += count[j];
  }
  h.pipeK = K;
  h.pipeCell = std::move(cells);
  h.outCell = std::move(outCells);
  h.pipeOut = std::move(out);
  h.pipeTiles = std::move(ends);
}

// The driver's tensor-map encoder, through the runtime's entry point (so the
// library links only the runtime); null when the driver does not offer it.
PFN_cuTensorMapEncodeTiled tensor_map_encoder()
{
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled)p;
  });
  return fn;
}

// Stage 3's tensor maps over a volume tissue's two padded Vm blocks: FP64,
// extents (px, ny + 2, nz + 2), row and plane strides px and pxy doubles
// (multiples of 16 bytes: px is even), box 36 x 3 x 3 (kWinRow x 3 x 3),
// no interleave, swizzle or multicast, zero fill outside the block.  False
// (maps zeroed) when the strides are odd or the encoder is missing or
// refuses.
bool encode_vm_maps(TissueDev& d, void* vm0, void* vm1)
{
  std::memset(d.vmMap, 0, sizeof(d.vmMap));
  if (d.cls != kVolume || d.px % 2 || d.pxy % 2) return false;
  PFN_cuTensorMapEncodeTiled enc = tensor_map_encoder();
  if (!enc) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)d.px, (cuuint64_t)d.ny + 2, (cuuint64_t)d.nz + 2};
  const cuuint64_t strides[2] = {(cuuint64_t)d.px * 8, (cuuint64_t)d.pxy * 8};
  const cuuint32_t box[3] = {kWinRow, 3, 3};
  const cuuint32_t elem[3] = {1, 1, 1};
  void* base[2] = {vm0, vm1};
  for (int k = 0; k < 2; ++k)
    if (enc(&d.vmMap[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base[k], dims, strides, box, elem,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
      std::memset(d.vmMap, 0, sizeof(d.vmMap));
      return false;
    }
  return true;
}

// Fills h.slot, h.tiles, h.nSlots and vrel (per slot: voxel offset from its
// tile's first voxel; 0 for padding).  With windows (the tissue has stage
// 3's tensor maps) row tiles are flagged kTileRow with their box origin.
// Layout (the warp tiles' shape): CDB_LAYOUT_CELLS fills each type's blocks
// with its cells in cell order; CDB_LAYOUT_ROWS cuts every x-row run of a
// type (consecutive gids in one x-row) into whole 32-cell blocks from the
// run's start, one row tile each, and packs the runs' remainders, in cell
// order, into shared blocks (one open at a time).  Either way a type takes
// ceil(cells / 32) blocks and every block's occupied slots are a prefix.
cdb_status build_layout(HostTissue& h, const int64_t* gid, const uint8_t* reaction, const int* slots,
                        const cdb_stimulus* stim, int nStim, std::vector<int32_t>& vrel, bool windows, int layout)
{
  const TissueDev& d = h.dev;
  const int64_t n = h.n;
  int64_t count[CDB_MAX_REACTION_TYPES], start[CDB_MAX_REACTION_TYPES], next[CDB_MAX_REACTION_TYPES];
  h.nSlots = count_slots(n, reaction, slots, count);
  int64_t total = 0;
  for (int k = 0; k < CDB_MAX_REACTION_TYPES; ++k) {
    start[k] = next[k] = total;
    total += (count[k] + kBlk - 1) / kBlk * kBlk;
  }
  h.slot.resize(n);
  std::vector<int64_t> voxOf(h.nSlots, 0), cellOf(h.nSlots, -1);
  std::vector<unsigned> mask(h.nSlots / kBlk, 0u);
  std::vector<int> fill(h.nSlots / kBlk, 0);
  auto g = [&](int64_t c) { return gid ? gid[c] : c; };
  auto assign = [&](int64_t c, int64_t i) {
    h.slot[c] = i;
    cellOf[i] = c;
    ++fill[i / kBlk];
    const int64_t gc = g(c);
    const int x = (int)(gc % h.nx);
    const int64_t yz = gc / h.nx;
    const int y = (int)(yz % h.ny), z = (int)(yz / h.ny);
    voxOf[i] = (int64_t)(x + 1) + d.px * (int64_t)(y + d.py0) + d.pxy * (int64_t)(z + d.pz0);
    for (int k = 0; k < nStim; ++k) {
      const cdb_stimulus& b = stim[k];
      if (x > b.xMin && x < b.xMax && y > b.yMin && y < b.yMax && z > b.zMin && z < b.zMax) mask[i / kBlk] |= 1u << k;
    }
  };
  if (layout == CDB_LAYOUT_ROWS) {
    std::vector<std::vector<int64_t>> cellsOf(CDB_MAX_REACTION_TYPES);
    for (int64_t c = 0; c < n; ++c) cellsOf[slots[reaction[c]]].push_back(c);
    for (int k = 0; k < CDB_MAX_REACTION_TYPES; ++k) {
      const std::vector<int64_t>& cs = cellsOf[k];
      int64_t shared = -1;
      int sfill = kBlk;
      for (size_t a = 0; a < cs.size();) {
        size_t e = a + 1;
        while (e < cs.size() && g(cs[e]) == g(cs[e - 1]) + 1 && g(cs[e]) % h.nx != 0) ++e;
        const size_t full = (e - a) / kBlk;
        for (size_t q = 0; q < full; ++q) {
          const int64_t blk = next[k];
          next[k] += kBlk;
          for (int l = 0; l < kBlk; ++l) assign(cs[a + q * kBlk + l], blk + l);
        }
        for (size_t r = a + full * kBlk; r < e; ++r) {
          if (sfill == kBlk) {
            shared = next[k];
            next[k] += kBlk;
            sfill = 0;
          }
          assign(cs[r], shared + sfill++);
        }
        a = e;
      }
    }
  } else {
    for (int64_t c = 0; c < n; ++c) assign(c, next[slots[reaction[c]]]++);
  }
  vrel.assign(h.nSlots, 0);
  for (auto& v : h.tiles) v.clear();
  for (int k = 0; k < CDB_MAX_REACTION_TYPES; ++k)
    for (int64_t f = start[k]; f < start[k] + count[k]; f += kBlk) {
      WarpTile tl{};
      tl.first = f;
      tl.count = fill[f / kBlk];
      tl.vox0 = voxOf[f];
      tl.stimMask = mask[f / kBlk];
      bool row = windows;
      for (int l = 0; l < tl.count; ++l) {
        const int64_t r = voxOf[f + l] - tl.vox0;
        CDB_CHECK(r >= INT32_MIN && r <= INT32_MAX, CDB_INVALID_ARG,
                  "grid too large: 32 consecutive cells of one type span more than 2^31 voxels");
        vrel[f + l] = (int32_t)r;
        row = row && r == l;
      }
      tl.flags = row ? kTileRow : 0;
      if (row) {
        const int64_t zp = tl.vox0 / d.pxy, rem = tl.vox0 - zp * d.pxy, yp = rem / d.px, xp = rem - yp * d.px;
        tl.wx = (int)((xp - 1) & ~int64_t(1));
        tl.wy = (int)(yp - 1);
        tl.wz = (int)(zp - 1);
      }
      h.tiles[k].push_back(tl);
    }
  build_pipe(h, gid, cellOf);
  return CDB_OK;
}

int64_t tissue_bytes(const Engine& E, const cdb_tissue_desc* t)
{
  const bool masked = t->gid && t->nCells != (int64_t)t->nx * t->ny * t->nz;
  const int cls = tissue_class(t->nx, t->ny, t->nz, masked);
  const int64_t vox = padded_voxels(t->nx, t->ny, t->nz, cls, nullptr, nullptr, nullptr, nullptr);
  const int64_t n = t->nCells;
  int64_t count[CDB_MAX_REACTION_TYPES];
  const int64_t nSlots = count_slots(n, t->reaction, E.slots, count);
  const bool mixed = E.cfg.precision == CDB_MIXED;
  int64_t b = 2 * vox * 8;                                                   // Vm blocks
  b += mixed ? nSlots * (kRowsMixed64 * 8 + kRowsMixed32 * 4) : nSlots * kRows64 * 8;   // state
  b += nSlots * weight_rows(cls, mixed) * (mixed ? 4 : 8);                   // weights
  b += nSlots * (8 + 4) + n * 8 + (masked ? n * 8 : 0) + 64;                 // act, vrel, slot map, voxel
  return b;
}

}  // namespace

extern "C" {

const char* cdb_last_error(void) { return t_last_error.c_str(); }
const char* cdb_version(void) { return "cardioid_b200 0.1 (sm_100a)"; }

double cdb_fit_eval(const cdb_fit* f, double x)
{
  const double* c = f->coeff;
  double num = c[f->numer - 1];
  for (int k = f->numer - 2; k >= 0; --k) num = c[k] + x * num;
  if (f->denom == 1) return num;
  const double* d = c + f->numer;
  double den = d[f->denom - 2];
  for (int k = f->denom - 3; k >= 0; --k) den = d[k] + x * den;
  den = 1 + x * den;
  return num / den;
}

cdb_status cdb_diag_fit_forms(const cdb_fit fits[CDB_NUM_FITS], int32_t poolSize, float* pool32, float* shift,
                              float* scale, int32_t* compiled)
{
  CDB_CHECK(fits && pool32 && shift && scale && compiled, CDB_INVALID_ARG, "null argument");
  CDB_CHECK(poolSize >= kSpecPool, CDB_INVALID_ARG, "pool32 holds fewer than the compiled pool's coefficients");
  std::vector<double> pool(kFitPoolPerType, 0.0);
  *compiled = pack_fits_spec(fits, pool.data(), kFitPoolPerType) ? 1 : 0;
  if (*compiled) {
    std::vector<float> p32(kFitPoolPerType);
    CDB_CHECK(spec_pool32(pool.data(), p32.data(), kFitPoolPerType), CDB_INVALID_ARG, "shifted denominator vanishes");
    for (int k = 0; k < kSpecPool; ++k) pool32[k] = p32[k];
  }
  for (int f = 0; f < kNumFits; ++f) shift[f] = kSpecShift[f];
  *scale = kSpecShiftScale;
  return CDB_OK;
}

cdb_status cdb_engine_create(const cdb_engine_config* cfg, cdb_engine** out)
{
  CDB_CHECK(cfg && out, CDB_INVALID_ARG, "null argument");
  CDB_CHECK(cfg->dt > 0, CDB_INVALID_ARG, "dt must be > 0");
  CDB_CHECK(cfg->precision == CDB_FP64 || cfg->precision == CDB_MIXED, CDB_INVALID_ARG, "unknown precision");
  int nDev = 0;
  CDB_CUDA(cudaGetDeviceCount(&nDev));
  CDB_CHECK(cfg->device >= 0 && cfg->device < nDev, CDB_INVALID_ARG, "no such device");
  CDB_CUDA(cudaSetDevice(cfg->device));
  std::unique_ptr<cdb_engine> e(new cdb_engine);
  e->e.cfg = *cfg;
  CDB_CUDA(cudaStreamCreateWithFlags(&e->e.stream, cudaStreamNonBlocking));
  CDB_CUDA(cudaDeviceGetAttribute(&e->e.numSms, cudaDevAttrMultiProcessorCount, cfg->device));
  CDB_CUDA(e->e.dErr.alloc(sizeof(int)));
  CDB_CUDA(cudaMemset(e->e.dErr.p, 0, sizeof(int)));
  // defaults, from the autotuner's tables on the 256^3 box (rows layout):
  // mixed, bulk-copy staging (stage 2; 1-3 % ahead of stage 3's Vm windows
  // and 6-8 % ahead of direct loads over five boxes); FP64, direct loads
  e->e.stage = cfg->precision == CDB_MIXED ? 2 : 0;
  CDB_CUDA(cfg->precision == CDB_MIXED ? allow_step_smem<true>() : allow_step_smem<false>());
  *out = e.release();
  return CDB_OK;
}

cdb_status cdb_engine_set_tuning(cdb_engine* e, int32_t stage, int32_t ctasPerSm)
{
  CDB_CHECK(e, CDB_INVALID_ARG, "null engine");
  CDB_CHECK(stage >= 0 && stage <= 3, CDB_INVALID_ARG, "stage must be 0, 1, 2 or 3");
  CDB_CHECK(ctasPerSm >= 0 && ctasPerSm <= 64, CDB_INVALID_ARG, "ctasPerSm must be in [0, 64]");
  Engine& E = e->e;
  CDB_CUDA(cudaSetDevice(E.cfg.device));
  CDB_CUDA(cudaStreamSynchronize(E.stream));
  E.stage = stage;
  E.ctasPerSm = ctasPerSm;
  E.drop_graphs();
  return CDB_OK;
}

cdb_status cdb_engine_set_layout(cdb_engine* e, int32_t layout)
{
  CDB_CHECK(e, CDB_INVALID_ARG, "null engine");
  CDB_CHECK(layout == CDB_LAYOUT_CELLS || layout == CDB_LAYOUT_ROWS, CDB_INVALID_ARG, "unknown layout");
  e->e.layout = layout;
  return CDB_OK;
}

cdb_status cdb_engine_get_layout(cdb_engine* e, int32_t* layout)
{
  CDB_CHECK(e && layout, CDB_INVALID_ARG, "null argument");
  *layout = e->e.layout;
  return CDB_OK;
}

cdb_status cdb_engine_get_tuning(cdb_engine* e, int32_t* stage, int32_t* ctasPerSm)
{
  CDB_CHECK(e, CDB_INVALID_ARG, "null engine");
  if (stage) *stage = e->e.stage;
  if (ctasPerSm) *ctasPerSm = e->e.ctasPerSm;
  return CDB_OK;
}

cdb_status cdb_engine_destroy(cdb_engine* e)
{
  if (!e) return CDB_OK;
  cudaSetDevice(e->e.cfg.device);
  cudaStreamSynchronize(e->e.stream);
  delete e;
  return CDB_OK;
}

cdb_status cdb_engine_add_reaction(cdb_engine* e, const cdb_tt06_params* params, const cdb_fit fits[CDB_NUM_FITS],
                                   int32_t* id)
{
  CDB_CHECK(e && params && fits && id, CDB_INVALID_ARG, "null argument");
  Engine& E = e->e;
  CDB_CHECK(E.nTypes < CDB_MAX_REACTION_TYPES, CDB_INVALID_ARG, "too many reaction types");
  FitShape shape{};
  std::vector<double> pool(kFitPoolPerType, 0.0);
  std::string err;
  CDB_CHECK(pack_fits(fits, shape, pool.data(), kFitPoolPerType, err), CDB_INVALID_ARG, err);
  // fits no longer than the compiled shapes run the unrolled kernel
  const bool specialised = pack_fits_spec(fits, pool.data(), kFitPoolPerType);
  const TT06Scalars scal = to_scalars(*params);
  CDB_CUDA(cudaSetDevice(E.cfg.device));
  CDB_CUDA(cudaStreamSynchronize(E.stream));
  cudaError_t up = cudaSuccess;
  const int slot = acquire_slot(E.cfg.device, scal, shape, pool, specialised, up);
  CDB_CUDA(up);
  CDB_CHECK(slot >= 0, CDB_INVALID_ARG,
            "every constant-memory reaction slot of this device is in use (at most " +
                std::to_string(CDB_MAX_REACTION_TYPES) +
                " distinct reaction types across the process's engines and plugin reactions)");
  E.slots[E.nTypes] = slot;
  E.spec[slot] = specialised;
  E.nTypes += 1;   // the engine holds the slot from here on; destroy releases it
  *id = E.nTypes - 1;
  return CDB_OK;
}

cdb_status cdb_engine_tissue_bytes(cdb_engine* e, const cdb_tissue_desc* t, int64_t* bytes)
{
  CDB_CHECK(e && t && bytes, CDB_INVALID_ARG, "null argument");
  *bytes = tissue_bytes(e->e, t);
  return CDB_OK;
}

cdb_status cdb_engine_free_bytes(cdb_engine* e, int64_t* freeBytes, int64_t* totalBytes)
{
  CDB_CHECK(e, CDB_INVALID_ARG, "null engine");
  CDB_CUDA(cudaSetDevice(e->e.cfg.device));
  size_t f = 0, t = 0;
  CDB_CUDA(cudaMemGetInfo(&f, &t));
  if (freeBytes) *freeBytes = (int64_t)f;
  if (totalBytes) *totalBytes = (int64_t)t;
  return CDB_OK;
}

cdb_status cdb_engine_add_tissue(cdb_engine* e, const cdb_tissue_desc* t, int32_t* id)
{
  NvtxRange range("cdb_engine_add_tissue");
  CDB_CHECK(e && id, CDB_INVALID_ARG, "null argument");
  Engine& E = e->e;
  cdb_status st = validate_desc(E, t);
  if (st != CDB_OK) return st;
  CDB_CUDA(cudaSetDevice(E.cfg.device));
  const bool mixed = E.cfg.precision == CDB_MIXED;
  const int64_t n = t->nCells;
  const int64_t gridN = (int64_t)t->nx * t->ny * t->nz;
  const bool masked = t->gid && n != gridN;
  const int cls = tissue_class(t->nx, t->ny, t->nz, masked);
  std::unique_ptr<HostTissue> h(new HostTissue);
  h->n = n;
  h->nx = t->nx; h->ny = t->ny; h->nz = t->nz;
  TissueDev& d = h->dev;
  d.n = n;
  d.nx = t->nx; d.ny = t->ny; d.nz = t->nz;
  d.cls = cls;
  const int64_t vox = padded_voxels(t->nx, t->ny, t->nz, cls, &d.px, &d.pxy, &d.py0, &d.pz0);
  d.scale = t->diffusionScale;
  d.blk.g_Kr = t->g_Kr_scale; d.blk.g_CaL = t->g_CaL_scale; d.blk.g_Na = t->g_Na_scale;
  h->stims.assign(t->stim, t->stim + t->nStim);

  cudaStream_t s = E.stream;
  CDB_CUDA(cudaStreamSynchronize(s));
  CDB_CUDA(h->vm0.alloc(vox * 8));
  CDB_CUDA(h->vm1.alloc(vox * 8));
  CDB_CUDA(cudaMemsetAsync(h->vm0.p, 0, vox * 8, s));
  CDB_CUDA(cudaMemsetAsync(h->vm1.p, 0, vox * 8, s));
  // slots grouped by reaction type; AoSoA arrays cover whole 32-slot blocks
  std::vector<int32_t> vrel;
  {
    const bool windows = encode_vm_maps(d, h->vm0.p, h->vm1.p);
    const cdb_status ls = build_layout(*h, t->gid, t->reaction, E.slots, t->stim, t->nStim, vrel, windows, E.layout);
    if (ls != CDB_OK) return ls;
  }
  const int64_t nSlots = h->nSlots;
  if (mixed) {
    CDB_CUDA(h->s64.alloc(nSlots * kRowsMixed64 * 8));
    CDB_CUDA(h->s32.alloc(nSlots * kRowsMixed32 * 4));
  } else {
    CDB_CUDA(h->s64.alloc(nSlots * kRows64 * 8));
  }
  const int wrows = weight_rows(cls, mixed);
  CDB_CUDA(h->w.alloc(nSlots * wrows * (mixed ? 4 : 8)));
  CDB_CUDA(cudaMemsetAsync(h->w.p, 0, nSlots * wrows * (mixed ? 4 : 8), s));
  CDB_CUDA(h->act.alloc(nSlots * 8));
  CDB_CUDA(h->vrel.alloc(nSlots * 4));
  CDB_CUDA(h->slotMap.alloc(n * 8));
  CDB_CUDA(cudaMemcpyAsync(h->vrel.p, vrel.data(), nSlots * 4, cudaMemcpyHostToDevice, s));
  CDB_CUDA(cudaMemcpyAsync(h->slotMap.p, h->slot.data(), n * 8, cudaMemcpyHostToDevice, s));
  CDB_CUDA(h->minmax.alloc(16));
  if (masked) CDB_CUDA(h->voxel.alloc(n * 8));

  // set-up scratch: full-padded voxel map, cell voxels, sigma, gids
  {
    const int64_t bx = t->nx + 2, bxy = bx * (t->ny + 2);
    const int64_t bvox = bxy * (t->nz + 2);
    DeviceBuffer map, cellVoxel, sig, gid, host64;
    CDB_CUDA(map.alloc(bvox * 8));
    CDB_CUDA(cellVoxel.alloc(n * 8));
    CDB_CUDA(sig.alloc(n * 6 * 8));
    if (t->gid) {
      CDB_CUDA(gid.alloc(n * 8));
      CDB_CUDA(cudaMemcpyAsync(gid.p, t->gid, n * 8, cudaMemcpyHostToDevice, s));
    }
    CDB_CUDA(cudaMemsetAsync(map.p, 0xff, bvox * 8, s));   // -1: no cell
    CDB_CUDA(cudaMemcpyAsync(sig.p, t->sigma6, n * 6 * 8, cudaMemcpyHostToDevice, s));
    build_voxel_map_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, gid.as<int64_t>(), t->nx, t->ny, bx, bxy,
                                                            map.as<int64_t>(), cellVoxel.as<int64_t>());
    build_weights_kernel<<<grid_for(n, 128), 128, 0, s>>>(n, map.as<int64_t>(), cellVoxel.as<int64_t>(),
                                                          sig.as<double>(), bx, bxy, t->dx, t->dy, t->dz, cls,
                                                          mixed ? 1 : 0, h->slotMap.as<int64_t>(), h->w.p);
    E.launches += 2;
    if (masked) {
      // cell voxels in the engine's (class-padded) block; masked tissues are kVolume
      std::vector<int64_t> v(n);
      const int64_t Px = d.px, Pxy = d.pxy;
      for (int64_t i = 0; i < n; ++i) {
        const int64_t g = t->gid[i];
        const int64_t x = g % t->nx, y = (g / t->nx) % t->ny, z = g / ((int64_t)t->nx * t->ny);
        v[i] = (x + 1) + Px * (y + d.py0) + Pxy * (z + d.pz0);
      }
      CDB_CUDA(cudaMemcpyAsync(h->voxel.p, v.data(), n * 8, cudaMemcpyHostToDevice, s));
      CDB_CUDA(cudaStreamSynchronize(s));
    }
    CDB_CUDA(cudaStreamSynchronize(s));
  }
  d.vm[0] = h->vm0.as<double>();
  d.vm[1] = h->vm1.as<double>();
  d.s64 = h->s64.as<double>();
  d.s32 = h->s32.as<float>();
  d.w = h->w.p;
  d.voxel = masked ? h->voxel.as<int64_t>() : nullptr;
  d.act = h->act.as<double>();
  d.minmax = h->minmax.as<unsigned long long>();
  d.actAll = 1;
  d.hx = t->dx; d.hy = t->dy; d.hz = t->dz;
  d.vrel = h->vrel.as<int>();
  d.nSlots = nSlots;
  d.nVox = vox;
  init_state_kernel<<<grid_for(nSlots, 256), 256, 0, s>>>(nSlots, d.s64, d.s32, mixed ? 1 : 0, d.act);
  E.launches += 1;
  {
    DeviceBuffer v0;
    CDB_CUDA(v0.alloc(n * 8));
    if (t->vm0) {
      CDB_CUDA(cudaMemcpyAsync(v0.p, t->vm0, n * 8, cudaMemcpyHostToDevice, s));
    } else {
      fill_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, v0.as<double>(), kInitialVm);
      E.launches += 1;
    }
    scatter_vm_kernel<<<grid_for(n, 256), 256, 0, s>>>(0, n, v0.as<double>(), d.vm[0], d.voxel, d.nx, d.ny, d.px,
                                                       d.pxy, d.py0, d.pz0, nullptr);
    E.launches += 1;
    CDB_CUDA(cudaStreamSynchronize(s));
  }
  CDB_CUDA(cudaGetLastError());
  const int newId = E.nextId++;
  E.tissues[newId] = std::move(h);
  E.dirty = true;
  *id = newId;
  return CDB_OK;
}

cdb_status cdb_engine_remove_tissue(cdb_engine* e, int32_t id)
{
  CDB_CHECK(e, CDB_INVALID_ARG, "null engine");
  Engine& E = e->e;
  auto it = E.tissues.find(id);
  CDB_CHECK(it != E.tissues.end(), CDB_NOT_FOUND, "no tissue with that id");
  CDB_CUDA(cudaSetDevice(E.cfg.device));
  CDB_CUDA(cudaStreamSynchronize(E.stream));
  E.tissues.erase(it);
  E.dirty = true;
  return CDB_OK;
}

cdb_status cdb_engine_step(cdb_engine* e, int32_t nSteps)
{
  NvtxRange range("cdb_engine_step");
  CDB_CHECK(e, CDB_INVALID_ARG, "null engine");
  CDB_CUDA(cudaSetDevice(e->e.cfg.device));
  return e->e.step(nSteps, true);
}

cdb_status cdb_engine_sync(cdb_engine* e)
{
  CDB_CHECK(e, CDB_INVALID_ARG, "null engine");
  CDB_CUDA(cudaSetDevice(e->e.cfg.device));
  CDB_CUDA(cudaStreamSynchronize(e->e.stream));
  int err = 0;
  CDB_CUDA(cudaMemcpy(&err, e->e.dErr.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    CDB_CUDA(cudaMemset(e->e.dErr.p, 0, sizeof(int)));
    CDB_CHECK(false, (cdb_status)err,
              err == CDB_NUMERIC_FAULT  ? "a non-finite Vm was found at the end of a launch batch"
              : err == CDB_BOUNDS_FAULT ? "the bounds-checked build found an index out of range"
                                        : "a bounded wait in the step kernel gave up (its copies did not arrive)");
  }
  return CDB_OK;
}

cdb_status cdb_engine_tissue_time(cdb_engine* e, int32_t id, int64_t* steps, double* time)
{
  CDB_CHECK(e, CDB_INVALID_ARG, "null engine");
  HostTissue* t = find_tissue(e, id);
  CDB_CHECK(t, CDB_NOT_FOUND, "no tissue with that id");
  Engine& E = e->e;
  cdb_status st = E.ensure_times(0);
  if (st != CDB_OK) return st;
  if (steps) *steps = t->steps;
  if (time) *time = E.tissue_time(*t);
  return CDB_OK;
}

cdb_status cdb_engine_set_ecg(cdb_engine* e, int32_t id, int32_t nPoints, const double* xyz, int32_t evalRate,
                              double kconst)
{
  CDB_CHECK(e, CDB_INVALID_ARG, "null engine");
  HostTissue* t = find_tissue(e, id);
  CDB_CHECK(t, CDB_NOT_FOUND, "no tissue with that id");
  CDB_CHECK(nPoints >= 0 && nPoints <= kEcgMaxPoints, CDB_INVALID_ARG, "ECG needs 0..32 electrodes");
  CDB_CHECK(nPoints == 0 || (xyz && evalRate >= 1), CDB_INVALID_ARG, "ECG electrodes and an evalRate >= 1 are required");
  Engine& E = e->e;
  CDB_CUDA(cudaSetDevice(E.cfg.device));
  CDB_CUDA(cudaStreamSynchronize(E.stream));
  TissueDev& d = t->dev;
  if (nPoints == 0) {
    d.ecgN = 0;
    t->ecgPts.release();
    t->ecgTrace.release();
    t->ecgInvr.release();
  } else {
    CDB_CUDA(t->ecgPts.alloc(nPoints * 3 * sizeof(double)));
    CDB_CUDA(cudaMemcpy(t->ecgPts.p, xyz, nPoints * 3 * sizeof(double), cudaMemcpyHostToDevice));
    const bool mixed = E.cfg.precision == CDB_MIXED;
    const size_t invrBytes = (size_t)t->nSlots * nPoints * (mixed ? sizeof(float) : sizeof(double));
    CDB_CUDA(t->ecgInvr.alloc(invrBytes));
    CDB_CUDA(cudaMemset(t->ecgInvr.p, 0, invrBytes));
    if (t->n > 0) {
      ecg_invr_kernel<<<grid_for(t->n, 256), 256, 0, E.stream>>>(
          t->n, t->slotMap.as<int64_t>(), d.voxel, d.nx, d.ny, d.px, d.pxy, d.py0, d.pz0, d.hx, d.hy, d.hz,
          t->ecgPts.as<double>(), nPoints, mixed ? 1 : 0, t->ecgInvr.p);
      E.launches += 1;
      CDB_CUDA(cudaGetLastError());
      CDB_CUDA(cudaStreamSynchronize(E.stream));
    }
    CDB_CUDA(t->ecgTrace.alloc((size_t)kEcgRing * nPoints * sizeof(double)));
    CDB_CUDA(cudaMemset(t->ecgTrace.p, 0, (size_t)kEcgRing * nPoints * sizeof(double)));
    d.ecgN = nPoints;
    d.ecgRate = evalRate;
    t->ecgK = kconst * d.hx * d.hy * d.hz;
    t->ecgNext = t->steps / evalRate + 1;
  }
  d.ecgPts = t->ecgPts.as<double>();
  d.ecgTrace = t->ecgTrace.as<double>();
  d.ecgInvr = t->ecgInvr.p;
  E.dirty = true;
  return CDB_OK;
}

cdb_status cdb_engine_read_ecg(cdb_engine* e, int32_t id, int64_t maxEntries, int64_t* nEntries, int64_t* loops,
                               double* values)
{
  CDB_CHECK(e && nEntries, CDB_INVALID_ARG, "null argument");
  HostTissue* t = find_tissue(e, id);
  CDB_CHECK(t, CDB_NOT_FOUND, "no tissue with that id");
  *nEntries = 0;
  const TissueDev& d = t->dev;
  if (d.ecgN == 0) return CDB_OK;
  CDB_CHECK(maxEntries >= 0 && (maxEntries == 0 || (loops && values)), CDB_INVALID_ARG, "output arrays are required");
  Engine& E = e->e;
  CDB_CUDA(cudaSetDevice(E.cfg.device));
  CDB_CUDA(cudaStreamSynchronize(E.stream));
  const int64_t last = t->steps / d.ecgRate;                  // last completed evaluation
  // the ring holds the last kEcgRing - 1 evaluations (each one clears the next entry)
  const int64_t first = std::max(t->ecgNext, last - kEcgRing + 2);
  const int64_t n = std::min<int64_t>(std::max<int64_t>(0, last - first + 1), maxEntries);
  std::vector<double> ring((size_t)kEcgRing * d.ecgN);
  if (n > 0) CDB_CUDA(cudaMemcpy(ring.data(), t->ecgTrace.p, ring.size() * sizeof(double), cudaMemcpyDeviceToHost));
  for (int64_t k = 0; k < n; ++k) {
    const int64_t ev = first + k;
    loops[k] = ev * d.ecgRate;
    for (int j = 0; j < d.ecgN; ++j) values[k * d.ecgN + j] = ring[(size_t)(ev % kEcgRing) * d.ecgN + j] * t->ecgK;
  }
  t->ecgNext = first + n;
  *nEntries = n;
  return CDB_OK;
}

cdb_status cdb_engine_set_clock(cdb_engine* e, int32_t id, int64_t loop, double time)
{
  CDB_CHECK(e, CDB_INVALID_ARG, "null engine");
  HostTissue* t = find_tissue(e, id);
  CDB_CHECK(t, CDB_NOT_FOUND, "no tissue with that id");
  CDB_CHECK(loop >= 0, CDB_INVALID_ARG, "loop must be >= 0");
  Engine& E = e->e;
  CDB_CUDA(cudaSetDevice(E.cfg.device));
  CDB_CUDA(cudaStreamSynchronize(E.stream));
  t->steps = loop;
  // clock 0 if its accumulated time at this step is exactly `time`
  t->clock = 0;
  cdb_status st = E.ensure_times(0);
  if (st != CDB_OK) return st;
  if (E.tissue_time(*t) != time) {
    int c = -1;
    for (size_t k = 1; k < E.clocks.size(); ++k)
      if (E.clocks[k].base == loop && E.clocks[k].times[0] == time) c = (int)k;
    if (c < 0) {
      E.clocks.push_back(Engine::Clock{loop, {time}, 0});
      c = (int)E.clocks.size() - 1;
    }
    t->clock = c;
    st = E.ensure_times(0);
    if (st != CDB_OK) return st;
  }
  E.dirty = true;
  return CDB_OK;
}

cdb_status cdb_engine_read_vm(cdb_engine* e, int32_t id, double* host)
{
  CDB_CHECK(e && host, CDB_INVALID_ARG, "null argument");
  HostTissue* t = find_tissue(e, id);
  CDB_CHECK(t, CDB_NOT_FOUND, "no tissue with that id");
  Engine& E = e->e;
  CDB_CUDA(cudaSetDevice(E.cfg.device));
  DeviceBuffer tmp;
  CDB_CUDA(tmp.alloc(t->n * 8));
  const TissueDev& d = t->dev;
  gather_vm_kernel<<<grid_for(t->n, 256), 256, 0, E.stream>>>(0, t->n, d.vm[t->parity], tmp.as<double>(), d.voxel,
                                                             d.nx, d.ny, d.px, d.pxy, d.py0, d.pz0);
  E.launches += 1;
  CDB_CUDA(cudaMemcpyAsync(host, tmp.p, t->n * 8, cudaMemcpyDeviceToHost, E.stream));
  CDB_CUDA(cudaStreamSynchronize(E.stream));
  return CDB_OK;
}

cdb_status cdb_engine_write_vm(cdb_engine* e, int32_t id, const double* host)
{
  CDB_CHECK(e && host, CDB_INVALID_ARG, "null argument");
  HostTissue* t = find_tissue(e, id);
  CDB_CHECK(t, CDB_NOT_FOUND, "no tissue with that id");
  Engine& E = e->e;
  CDB_CUDA(cudaSetDevice(E.cfg.device));
  DeviceBuffer tmp;
  CDB_CUDA(tmp.alloc(t->n * 8));
  CDB_CUDA(cudaMemcpyAsync(tmp.p, host, t->n * 8, cudaMemcpyHostToDevice, E.stream));
  const TissueDev& d = t->dev;
  t->dev.actAll = 1;
  scatter_vm_kernel<<<grid_for(t->n, 256), 256, 0, E.stream>>>(0, t->n, tmp.as<double>(), d.vm[t->parity], d.voxel,
                                                              d.nx, d.ny, d.px, d.pxy, d.py0, d.pz0,
                                                              E.act_all_flag(id));
  E.launches += 1;
  CDB_CUDA(cudaStreamSynchronize(E.stream));
  return CDB_OK;
}

cdb_status cdb_engine_read_state(cdb_engine* e, int32_t id, int var, double* host)
{
  CDB_CHECK(e && host, CDB_INVALID_ARG, "null argument");
  CDB_CHECK(var >= 0 && var < kNumStates, CDB_INVALID_ARG, "state index out of range");
  HostTissue* t = find_tissue(e, id);
  CDB_CHECK(t, CDB_NOT_FOUND, "no tissue with that id");
  Engine& E = e->e;
  CDB_CUDA(cudaSetDevice(E.cfg.device));
  CDB_CUDA(cudaStreamSynchronize(E.stream));
  const int64_t n = t->n;
  DeviceBuffer tmp;
  CDB_CUDA(tmp.alloc(n * 8));
  gather_state_kernel<<<grid_for(n, 256), 256, 0, E.stream>>>(n, t->slotMap.as<int64_t>(), t->dev.s64, t->dev.s32,
                                                              E.cfg.precision == CDB_MIXED, var, tmp.as<double>());
  E.launches += 1;
  CDB_CUDA(cudaMemcpyAsync(host, tmp.p, n * 8, cudaMemcpyDeviceToHost, E.stream));
  CDB_CUDA(cudaStreamSynchronize(E.stream));
  return CDB_OK;
}

cdb_status cdb_engine_write_state(cdb_engine* e, int32_t id, int var, const double* host)
{
  CDB_CHECK(e && host, CDB_INVALID_ARG, "null argument");
  CDB_CHECK(var >= 0 && var < kNumStates, CDB_INVALID_ARG, "state index out of range");
  HostTissue* t = find_tissue(e, id);
  CDB_CHECK(t, CDB_NOT_FOUND, "no tissue with that id");
  Engine& E = e->e;
  CDB_CUDA(cudaSetDevice(E.cfg.device));
  CDB_CUDA(cudaStreamSynchronize(E.stream));
  const int64_t n = t->n;
  DeviceBuffer tmp;
  CDB_CUDA(tmp.alloc(n * 8));
  CDB_CUDA(cudaMemcpyAsync(tmp.p, host, n * 8, cudaMemcpyHostToDevice, E.stream));
  scatter_state_kernel<<<grid_for(n, 256), 256, 0, E.stream>>>(n, t->slotMap.as<int64_t>(), t->dev.s64, t->dev.s32,
                                                               E.cfg.precision == CDB_MIXED, var, tmp.as<double>());
  E.launches += 1;
  CDB_CUDA(cudaStreamSynchronize(E.stream));
  return CDB_OK;
}

cdb_status cdb_engine_read_activation(cdb_engine* e, int32_t id, double* host)
{
  CDB_CHECK(e && host, CDB_INVALID_ARG, "null argument");
  HostTissue* t = find_tissue(e, id);
  CDB_CHECK(t, CDB_NOT_FOUND, "no tissue with that id");
  Engine& E = e->e;
  CDB_CUDA(cudaSetDevice(E.cfg.device));
  CDB_CUDA(cudaStreamSynchronize(E.stream));
  DeviceBuffer tmp;
  CDB_CUDA(tmp.alloc(t->n * 8));
  gather_slots_kernel<<<grid_for(t->n, 256), 256, 0, E.stream>>>(t->n, t->slotMap.as<int64_t>(), t->dev.act,
                                                                 tmp.as<double>());
  E.launches += 1;
  CDB_CUDA(cudaMemcpyAsync(host, tmp.p, t->n * 8, cudaMemcpyDeviceToHost, E.stream));
  CDB_CUDA(cudaStreamSynchronize(E.stream));
  return CDB_OK;
}

cdb_status cdb_engine_minmax(cdb_engine* e, int32_t id, double* vmin, double* vmax)
{
  CDB_CHECK(e, CDB_INVALID_ARG, "null engine");
  HostTissue* t = find_tissue(e, id);
  CDB_CHECK(t, CDB_NOT_FOUND, "no tissue with that id");
  Engine& E = e->e;
  CDB_CUDA(cudaSetDevice(E.cfg.device));
  CDB_CUDA(cudaStreamSynchronize(E.stream));
  unsigned long long mm[2];
  CDB_CUDA(cudaMemcpy(mm, t->dev.minmax, 16, cudaMemcpyDeviceToHost));
  if (vmin) *vmin = from_ordered_bits(mm[0]);
  if (vmax) *vmax = from_ordered_bits(mm[1]);
  return CDB_OK;
}

cdb_status cdb_engine_read_weights(cdb_engine* e, int32_t id, double* host19)
{
  CDB_CHECK(e && host19, CDB_INVALID_ARG, "null argument");
  HostTissue* t = find_tissue(e, id);
  CDB_CHECK(t, CDB_NOT_FOUND, "no tissue with that id");
  Engine& E = e->e;
  CDB_CUDA(cudaSetDevice(E.cfg.device));
  CDB_CUDA(cudaStreamSynchronize(E.stream));
  const int64_t n = t->n;
  const int cls = t->dev.cls;
  const int rows = class_rows(cls);
  const bool mixed = E.cfg.precision == CDB_MIXED;
  std::vector<double> out(n * 19, 0.0);
  if (mixed) {
    std::vector<float> w((size_t)t->nSlots * (rows - 1));
    CDB_CUDA(cudaMemcpy(w.data(), t->dev.w, w.size() * 4, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < n; ++i) {
      double a0 = 0;
      for (int r = 1; r < rows; ++r) {
        const float v = w[aosoa(t->slot[i], rows - 1, r - 1)];
        out[i * 19 + class_node(cls, r)] = v;
        a0 -= v;
      }
      out[i * 19] = a0;
    }
  } else {
    std::vector<double> w((size_t)t->nSlots * rows);
    CDB_CUDA(cudaMemcpy(w.data(), t->dev.w, w.size() * 8, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < n; ++i)
      for (int r = 0; r < rows; ++r) out[i * 19 + class_node(cls, r)] = w[aosoa(t->slot[i], rows, r)];
  }
  std::memcpy(host19, out.data(), out.size() * 8);
  return CDB_OK;
}

// Whether n doubles at p lie in page-locked host memory (both ends: an
// array is one allocation), which a captured copy needs.
static bool host_locked(const void* p, int64_t n)
{
  cudaPointerAttributes a;
  for (const void* q : {p, (const void*)((const double*)p + (n > 0 ? n - 1 : 0))}) {
    if (cudaPointerGetAttributes(&a, q) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    if (a.type != cudaMemoryTypeHost) return false;
  }
  return true;
}

cdb_status cdb_engine_step_host(cdb_engine* e, int32_t id, const double* vm_in, double* vm_out)
{
  NvtxRange range("cdb_engine_step_host");
  CDB_CHECK(e && vm_in && vm_out, CDB_INVALID_ARG, "null argument");
  HostTissue* t = find_tissue(e, id);
  CDB_CHECK(t, CDB_NOT_FOUND, "no tissue with that id");
  Engine& E = e->e;
  CDB_CHECK(E.tissues.size() == 1, CDB_INVALID_ARG, "cdb_engine_step_host needs an engine with one tissue");
  CDB_CUDA(cudaSetDevice(E.cfg.device));
  const int64_t n = t->n;
  if (E.dStage.bytes < (size_t)n * 8) {
    E.drop_graphs();
    CDB_CUDA(E.dStage.alloc(n * 8));
  }
  cudaStream_t s = E.stream;
  if (t->pipeK < 2) {
    const TissueDev& d = t->dev;
    CDB_CUDA(cudaMemcpyAsync(E.dStage.p, vm_in, n * 8, cudaMemcpyHostToDevice, s));
    t->dev.actAll = 1;
    scatter_vm_kernel<<<grid_for(n, 256), 256, 0, s>>>(0, n, E.dStage.as<double>(), d.vm[t->parity], d.voxel, d.nx,
                                                       d.ny, d.px, d.pxy, d.py0, d.pz0, E.act_all_flag(id));
    E.launches += 1;
    cdb_status st = E.step(1, false);
    if (st != CDB_OK) return st;
    gather_vm_kernel<<<grid_for(n, 256), 256, 0, s>>>(0, n, d.vm[t->parity], E.dStage.as<double>(), d.voxel, d.nx,
                                                      d.ny, d.px, d.pxy, d.py0, d.pz0);
    E.launches += 1;
    CDB_CUDA(cudaMemcpyAsync(vm_out, E.dStage.p, n * 8, cudaMemcpyDeviceToHost, s));
    CDB_CUDA(cudaStreamSynchronize(s));
    return CDB_OK;
  }
  // Chunked: Vm goes up chunk by chunk on one copy stream; on the engine's
  // stream each chunk is scattered into the padded block once it has
  // landed, the tiles whose stencil reads no later chunk are computed, and
  // the chunks whose new Vm is then final are gathered; a second copy
  // stream takes each of those down.  Both copy directions and the step
  // overlap, and every kernel stays on the engine's stream (the persistent
  // step kernels hold every SM while they run).  With page-locked host
  // buffers the whole pattern (about ten API calls per chunk) is captured
  // once as a graph and replayed by one launch: the same device time, and
  // the host thread issues one call per step instead of some 170.
  cdb_status st = E.ensure_times(1);
  if (st != CDB_OK) return st;
  st = E.rebuild();
  if (st != CDB_OK) return st;
  const int K = t->pipeK;
  CDB_CUDA(E.ensure_pipe(K));
  if (E.dStageOut.bytes < (size_t)n * 8) {
    E.drop_graphs();
    CDB_CUDA(E.dStageOut.alloc(n * 8));
  }
  const TissueDev& d = t->dev;
  double* const vin = d.vm[t->parity];
  double* const vout = d.vm[t->parity ^ 1];
  int* const flag = E.act_all_flag(id);
  t->dev.actAll = 1;
  double* const stIn = E.dStage.as<double>();
  double* const stOut = E.dStageOut.as<double>();
  auto enqueue = [&]() -> cudaError_t {
    cudaError_t err = cudaEventRecord(E.evStart, s);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(E.sIn, E.evStart, 0);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(E.sOut, E.evStart, 0);
    for (int j = 0; j < K && err == cudaSuccess; ++j) {
      const int64_t c0 = t->pipeCell[j], m = t->pipeCell[j + 1] - c0;
      if (m > 0) err = cudaMemcpyAsync(stIn + c0, vm_in + c0, m * 8, cudaMemcpyHostToDevice, E.sIn);
      if (err == cudaSuccess) err = cudaEventRecord(E.evIn[j], E.sIn);
    }
    for (int j = 0; j < K && err == cudaSuccess; ++j) {
      err = cudaStreamWaitEvent(s, E.evIn[j], 0);
      if (err != cudaSuccess) break;
      const int64_t c0 = t->pipeCell[j], m = t->pipeCell[j + 1] - c0;
      if (m > 0) {
        scatter_vm_kernel<<<grid_for(m, 256), 256, 0, s>>>(c0, m, stIn, vin, d.voxel, d.nx, d.ny, d.px, d.pxy, d.py0,
                                                           d.pz0, flag);
        E.launches += 1;
      }
      for (const auto& sl : E.slotTiles) {
        const int64_t lo = j ? t->pipeTiles[j - 1][sl.first] : 0, hi = t->pipeTiles[j][sl.first];
        if (hi > lo) E.launch_tiles(sl.first, sl.second.first + lo, hi - lo, 0, false, s);
      }
      bool down = false;
      for (int i = 0; i < K; ++i) {
        const int64_t g0 = t->outCell[i], gm = t->outCell[i + 1] - g0;
        if (t->pipeOut[i] != j || gm == 0) continue;
        gather_vm_kernel<<<grid_for(gm, 256), 256, 0, s>>>(g0, gm, vout, stOut, d.voxel, d.nx, d.ny, d.px, d.pxy,
                                                           d.py0, d.pz0);
        E.launches += 1;
        down = true;
      }
      err = cudaEventRecord(E.evComp[j], s);
      if (err == cudaSuccess && down) err = cudaStreamWaitEvent(E.sOut, E.evComp[j], 0);
      // the chunks this compute chunk completed go down at once
      for (int i = 0; i < K && err == cudaSuccess && down; ++i) {
        const int64_t g0 = t->outCell[i], gm = t->outCell[i + 1] - g0;
        if (t->pipeOut[i] != j || gm == 0) continue;
        err = cudaMemcpyAsync(vm_out + g0, stOut + g0, gm * 8, cudaMemcpyDeviceToHost, E.sOut);
      }
    }
    if (err != cudaSuccess) return err;
    advance_kernel<<<1, 128, 0, s>>>(E.dTissues.as<TissueDev>(), 1, 1);
    E.launches += 1;
    err = cudaEventRecord(E.evOut, E.sOut);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(s, E.evOut, 0);
    return err;
  };
  if (E.cfg.use_graphs && !E.withhold && host_locked(vm_in, n) && host_locked(vm_out, n)) {
    Engine::HostStepGraph* g = nullptr;
    for (Engine::HostStepGraph& h : E.hostGraphs)
      if (h.in == vm_in && h.out == vm_out && h.parity == t->parity) g = &h;
    if (!g) {
      cudaGraph_t cg = nullptr;
      CDB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      const int64_t before = E.launches;
      const cudaError_t err = enqueue();
      const int64_t per = E.launches - before;
      E.launches = before;
      const cudaError_t end = cudaStreamEndCapture(s, &cg);
      CDB_CUDA(err);
      CDB_CUDA(end);
      cudaGraphExec_t exec = nullptr;
      const cudaError_t inst = cudaGraphInstantiate(&exec, cg, 0);
      cudaGraphDestroy(cg);
      CDB_CUDA(inst);
      E.hostGraphs.push_back(Engine::HostStepGraph{vm_in, vm_out, t->parity, exec, per});
      g = &E.hostGraphs.back();
    }
    CDB_CUDA(cudaGraphLaunch(g->exec, s));
    E.launches += g->launches;
  } else {
    CDB_CUDA(enqueue());
  }
  E.advance_host(1);
  CDB_CUDA(cudaGetLastError());
  CDB_CUDA(cudaStreamSynchronize(s));
  return CDB_OK;
}

cdb_status cdb_engine_test_bounded_wait(cdb_engine* e)
{
  CDB_CHECK(e, CDB_INVALID_ARG, "null engine");
  e->e.withhold = true;
  return CDB_OK;
}

cdb_status cdb_engine_launch_count(cdb_engine* e, int64_t* launches)
{
  CDB_CHECK(e && launches, CDB_INVALID_ARG, "null argument");
  *launches = e->e.launches;
  return CDB_OK;
}

cdb_status cdb_engine_stream(cdb_engine* e, void** stream)
{
  CDB_CHECK(e && stream, CDB_INVALID_ARG, "null argument");
  *stream = (void*)e->e.stream;
  return CDB_OK;
}

}  // extern "C"
