// The reference's own GPU reaction path, run and timed on the device.
//
// BetterTT06 compiled with USE_CUDA builds its NVRTC kernel at creation
// (ThisReaction::constructKernel, elec/BetterTT06.cc:1045-1318: the fit
// coefficients and parameters printed into the kernel source, one thread per
// cell, state in SoA rows of nCells) and launches it from calc on the default
// stream (elec/BetterTT06.cc:1320-1364).  This driver creates the reactions
// through the reference's ReactionManager and calls ReactionManager::calc
// (elec/ReactionManager.cc:14-27) once per step, the call simulationLoop makes
// (elec/simulationLoop.cc:198-202), with Vm and iStim held fixed (a
// reaction-only loop: the state advances every step, Vm does not).
//
// TEST AND MEASUREMENT INFRASTRUCTURE ONLY: compiled with the reference
// sources it drives into oracle/_ref/ref_gpu_reaction by oracle/ref/Makefile;
// the product never links or runs it.
//
// Usage: ref_gpu_reaction OBJECTS DT STEPS WARMUP CELLTYPES VM OUT NAME...
//   OBJECTS    object-database file (REACTION, FIT and FUNCTION objects)
//   CELLTYPES  int32 anatomy cellType per cell (binary)
//   VM         float64 Vm per cell (binary), or "-" for the reactions' own
//              initial Vm (initializeMembraneState)
//   OUT        "-", or a file that receives dVm (N float64) followed by the
//              checkpoint states (N float64 each, getCheckpointInfo order)
//   NAME...    REACTION object names, as the reference's reaction list
// Prints one JSON line: cells, steps, ms per step (CUDA events around the
// STEPS calls on the default stream, after WARMUP calls) and cell-steps/s.
#include <mpi.h>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "ReactionManager.hh"
#include "Reaction.hh"
#include "ThreadServer.hh"
#include "lazy_array.hh"
#include "object_cc.hh"
#include "units.h"

void registerBuiltinReactions();

namespace {

bool readFile(const char* path, void* dst, size_t bytes)
{
   FILE* f = std::fopen(path, "rb");
   if (!f) return false;
   const size_t got = std::fread(dst, 1, bytes, f);
   std::fclose(f);
   return got == bytes;
}

long fileBytes(const char* path)
{
   FILE* f = std::fopen(path, "rb");
   if (!f) return -1;
   std::fseek(f, 0, SEEK_END);
   const long n = std::ftell(f);
   std::fclose(f);
   return n;
}

#define CHECK_CUDA(x)                                                                    \
   do {                                                                                  \
      cudaError_t e_ = (x);                                                              \
      if (e_ != cudaSuccess) {                                                           \
         std::fprintf(stderr, "ref_gpu_reaction: %s: %s\n", #x, cudaGetErrorString(e_)); \
         return 3;                                                                       \
      }                                                                                  \
   } while (0)

}  // namespace

int main(int argc, char** argv)
{
   if (argc < 9) {
      std::fprintf(stderr, "usage: %s OBJECTS DT STEPS WARMUP CELLTYPES VM OUT NAME...\n", argv[0]);
      return 2;
   }
   const char* objects = argv[1];
   const double dt = std::atof(argv[2]);
   const int steps = std::atoi(argv[3]);
   const int warmup = std::atoi(argv[4]);
   const char* ctPath = argv[5];
   const char* vmPath = argv[6];
   const char* outPath = argv[7];

   MPI_Init(&argc, &argv);
   // Cardioid's unit system (elec/cardioid.cc:84-85)
   units_internal(1e-3, 1e-9, 1e-3, 1e-3, 1, 1e-9, 1);
   units_external(1e-3, 1e-9, 1e-3, 1e-3, 1, 1e-9, 1);
   object_compilefile(objects);
   registerBuiltinReactions();

   const long ctBytes = fileBytes(ctPath);
   if (ctBytes <= 0 || ctBytes % 4) {
      std::fprintf(stderr, "ref_gpu_reaction: bad cell-type file %s\n", ctPath);
      return 2;
   }
   const long n = ctBytes / 4;
   std::vector<int> cellType(n);
   if (!readFile(ctPath, cellType.data(), ctBytes)) return 2;

   // BetterTT06's factory loads its NVRTC module through the driver API
   // (cuModuleLoadDataEx, elec/BetterTT06.cc:1316), which needs a current
   // context: create the runtime's primary context first, as the
   // reference's own earlier device allocations do.
   CHECK_CUDA(cudaFree(0));
   ReactionManager reaction;
   for (int a = 8; a < argc; ++a) reaction.addReaction(argv[a]);
   ThreadTeam group = ThreadServer::getInstance().getThreadTeam(std::vector<unsigned>());
   reaction.create(dt, ro_array_ptr<int>(cellType.data(), n), group);

   lazy_array<double> Vm, iStim, dVm;
   Vm.resize(n);
   iStim.resize(n);
   dVm.resize(n);
   {
      wo_array_ptr<double> v = Vm.useOn(CPU);
      wo_array_ptr<double> s = iStim.useOn(CPU);
      wo_array_ptr<double> d = dVm.useOn(CPU);
      for (long ii = 0; ii < n; ++ii) { v[ii] = 0; s[ii] = 0; d[ii] = 0; }
   }
   reaction.initializeMembraneState(Vm);
   if (std::string(vmPath) != "-") {
      wo_array_ptr<double> v = Vm.useOn(CPU);
      if (fileBytes(vmPath) != n * 8 || !readFile(vmPath, v.raw(), n * 8)) {
         std::fprintf(stderr, "ref_gpu_reaction: bad Vm file %s\n", vmPath);
         return 2;
      }
   }

   for (int k = 0; k < warmup; ++k) reaction.calc(dt, Vm, iStim, dVm);
   CHECK_CUDA(cudaDeviceSynchronize());
   cudaEvent_t e0, e1;
   CHECK_CUDA(cudaEventCreate(&e0));
   CHECK_CUDA(cudaEventCreate(&e1));
   CHECK_CUDA(cudaEventRecord(e0, 0));
   for (int k = 0; k < steps; ++k) reaction.calc(dt, Vm, iStim, dVm);
   CHECK_CUDA(cudaEventRecord(e1, 0));
   CHECK_CUDA(cudaEventSynchronize(e1));
   CHECK_CUDA(cudaGetLastError());
   float ms = 0.f;
   CHECK_CUDA(cudaEventElapsedTime(&ms, e0, e1));

   if (std::string(outPath) != "-") {
      FILE* f = std::fopen(outPath, "wb");
      if (!f) return 2;
      {
         ro_array_ptr<double> d = dVm.useOn(CPU);
         std::fwrite(d.raw(), 8, n, f);
      }
      std::vector<std::string> names, units;
      reaction.getCheckpointInfo(names, units);
      std::vector<double> col(n);
      for (const std::string& name : names) {
         const int h = reaction.getVarHandle(name);
         for (long ii = 0; ii < n; ++ii) col[ii] = reaction.getValue((int)ii, h);
         std::fwrite(col.data(), 8, n, f);
      }
      std::fclose(f);
   }
   const double perStep = steps > 0 ? ms / steps : 0.0;
   std::printf("{\"cells\": %ld, \"steps\": %d, \"warmup\": %d, \"ms_per_step\": %.6f, \"cell_steps_per_s\": %.6e}\n",
               n, steps, warmup, perStep, perStep > 0 ? n / (perStep * 1e-3) : 0.0);
   return 0;
}
