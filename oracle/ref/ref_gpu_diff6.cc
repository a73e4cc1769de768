// The reference's own "cuda" Diffusion run on the device: CUDADiffusion
// (elec/CUDADiffusion.cc: the face-conductivity table built on the host,
// updateLocalVoltage / calc) with its kernels diff_6face_v1, map_dVm and
// copy_to_block_kernel (elec/CUDADiffusion_ker.cu:16-221), compiled with nvcc.
//
// diff_6face_v1 runs 32 x 32 thread blocks over tiles of 30 x 30 (y, z)
// voxels and returns from the threads past the last tile's extent before
// its __syncthreads (elec/CUDADiffusion_ker.cu:52-53).  When the local
// grid's y and z sizes are 30 k + 2 (tissue extents in y and z that are
// multiples of 30) the last tiles are full and no thread returns, so every
// thread reaches every barrier; this driver refuses every other grid.
//
// TEST INFRASTRUCTURE ONLY: built with the reference sources it drives into
// oracle/_ref/ref_gpu_diff6 by oracle/ref/Makefile; the product never links
// or runs it.
//
// Usage: ref_gpu_diff6 NX NY NZ DX DY DZ SCALE GIDS CELLTYPES SIGMA VM OUT [STEPS]
//   GIDS int64 gid per cell (gid = x + nx (y + ny z)), CELLTYPES int32,
//   SIGMA float64 [n][6] (a11 a12 a13 a22 a23 a33), VM float64 [n], all
//   binary; OUT receives dVm (float64 [n]) from one updateLocalVoltage +
//   calc, as the reference's omp loop calls them.  With STEPS, that pair is
//   then timed STEPS times (CUDA events on the default stream, after 3
//   untimed pairs) and one JSON line gives ms per pair.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include <cuda_runtime.h>

#include "Anatomy.hh"
#include "AnatomyCell.hh"
#include "CUDADiffusion.hh"
#include "DiffusionUtils.hh"
#include "lazy_array.hh"

namespace {

long fileBytes(const char* path)
{
   FILE* f = std::fopen(path, "rb");
   if (!f) return -1;
   std::fseek(f, 0, SEEK_END);
   const long n = std::ftell(f);
   std::fclose(f);
   return n;
}

bool readFile(const char* path, void* dst, size_t bytes)
{
   FILE* f = std::fopen(path, "rb");
   if (!f) return false;
   const size_t got = std::fread(dst, 1, bytes, f);
   std::fclose(f);
   return got == bytes;
}

}  // namespace

int main(int argc, char** argv)
{
   if (argc != 13 && argc != 14) {
      std::fprintf(stderr, "usage: %s NX NY NZ DX DY DZ SCALE GIDS CELLTYPES SIGMA VM OUT [STEPS]\n", argv[0]);
      return 2;
   }
   const int nx = std::atoi(argv[1]), ny = std::atoi(argv[2]), nz = std::atoi(argv[3]);
   const double dx = std::atof(argv[4]), dy = std::atof(argv[5]), dz = std::atof(argv[6]);
   const double scale = std::atof(argv[7]);
   const long n = fileBytes(argv[8]) / 8;
   if (n <= 0 || fileBytes(argv[9]) != n * 4 || fileBytes(argv[10]) != n * 48 || fileBytes(argv[11]) != n * 8) {
      std::fprintf(stderr, "ref_gpu_diff6: bad input sizes\n");
      return 2;
   }
   std::vector<long long> gid(n);
   std::vector<int> cellType(n);
   std::vector<double> sigma(6 * n), vm(n);
   if (!readFile(argv[8], gid.data(), n * 8) || !readFile(argv[9], cellType.data(), n * 4) ||
       !readFile(argv[10], sigma.data(), n * 48) || !readFile(argv[11], vm.data(), n * 8))
      return 2;

   Anatomy a;
   a.setGridSize(nx, ny, nz);
   a.dx() = dx; a.dy() = dy; a.dz() = dz;
   a.offset_x() = 0; a.offset_y() = 0; a.offset_z() = 0;
   std::vector<AnatomyCell>& cells = a.cellArray();
   cells.resize(n);
   for (long ii = 0; ii < n; ++ii) {
      AnatomyCell& c = cells[ii];
      c.gid_ = gid[ii];
      c.cellType_ = cellType[ii];
      c.sigma_.a11 = sigma[6 * ii + 0];
      c.sigma_.a12 = sigma[6 * ii + 1];
      c.sigma_.a13 = sigma[6 * ii + 2];
      c.sigma_.a22 = sigma[6 * ii + 3];
      c.sigma_.a23 = sigma[6 * ii + 4];
      c.sigma_.a33 = sigma[6 * ii + 5];
      c.dest_ = 0;
      c.sortind_ = (int)ii;
   }
   a.nRemote() = 0;
   a.nGlobal() = n;

   const LocalGrid grid = DiffusionUtils::findBoundingBox(a, false);
   if ((grid.ny() - 2) % 30 != 0 || (grid.nz() - 2) % 30 != 0) {
      std::fprintf(stderr, "ref_gpu_diff6: local grid %d x %d x %d: the reference kernel needs y and z sizes of "
                   "30 k + 2 (otherwise threads return before its barriers)\n", grid.nx(), grid.ny(), grid.nz());
      return 2;
   }

   CUDADiffusion diffusion(a, 0, scale);   // loop type 0: the omp loop
   lazy_array<double> Vm, dVm;
   Vm.resize(n);
   dVm.resize(n);
   {
      wo_array_ptr<double> v = Vm.useOn(CPU);
      for (long ii = 0; ii < n; ++ii) v[ii] = vm[ii];
   }
   diffusion.updateLocalVoltage(Vm);
   diffusion.calc(dVm);
   if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess) {
      std::fprintf(stderr, "ref_gpu_diff6: a kernel failed\n");
      return 3;
   }
   FILE* f = std::fopen(argv[12], "wb");
   if (!f) return 2;
   {
      ro_array_ptr<double> d = dVm.useOn(CPU);
      std::fwrite(d.raw(), 8, n, f);
   }
   std::fclose(f);
   const int steps = argc == 14 ? std::atoi(argv[13]) : 0;
   float ms = 0.f;
   if (steps > 0) {
      for (int k = 0; k < 3; ++k) {
         diffusion.updateLocalVoltage(Vm);
         diffusion.calc(dVm);
      }
      cudaEvent_t e0, e1;
      if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return 3;
      cudaDeviceSynchronize();
      cudaEventRecord(e0, 0);
      for (int k = 0; k < steps; ++k) {
         diffusion.updateLocalVoltage(Vm);
         diffusion.calc(dVm);
      }
      cudaEventRecord(e1, 0);
      if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) return 3;
      cudaEventElapsedTime(&ms, e0, e1);
   }
   std::printf("{\"cells\": %ld, \"grid\": [%d, %d, %d], \"steps\": %d, \"ms_per_step\": %.6f}\n", n, grid.nx(),
               grid.ny(), grid.nz(), steps, steps > 0 ? ms / steps : 0.0);
   return 0;
}
