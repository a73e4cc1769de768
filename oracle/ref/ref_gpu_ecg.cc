// The reference's own ECG kernels, run on the device: calcInvrCUDA (the
// 1/|r - p| table, elec/ECGSensor.cu:9-61) and calcEcgCUDA (the sum over
// cells of dVmD times that table, elec/ECGSensor.cu:79-160), compiled from
// elec/ECGSensor.cu with nvcc and called as ECGSensor::calcInvR and
// ECGSensor::eval call them (elec/ECGSensor.cc:47-78, 285-300).
//
// TEST INFRASTRUCTURE ONLY: built with the reference sources it drives into
// oracle/_ref/ref_gpu_ecg by oracle/ref/Makefile; the product never links or
// runs it.
//
// Usage: ref_gpu_ecg NX NY NZ DX DY DZ GIDS POINTS DVMD OUT
//   GIDS    int64 gid per cell (gid = x + nx (y + ny z)), binary
//   POINTS  float64 electrode positions [m][3] (mm), binary
//   DVMD    float64 dVmD per cell, binary, or "-" (no sum)
//   OUT     receives the table (n x m float64, cell-major, as the reference
//           stores it) and, with DVMD, the m sums
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "ECGSensor.hh"
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
   if (argc != 11) {
      std::fprintf(stderr, "usage: %s NX NY NZ DX DY DZ GIDS POINTS DVMD OUT\n", argv[0]);
      return 2;
   }
   const int nx = std::atoi(argv[1]), ny = std::atoi(argv[2]), nz = std::atoi(argv[3]);
   const double dx = std::atof(argv[4]), dy = std::atof(argv[5]), dz = std::atof(argv[6]);
   const char* gidPath = argv[7];
   const char* ptsPath = argv[8];
   const char* dvmPath = argv[9];
   const char* outPath = argv[10];
   const long gb = fileBytes(gidPath), pb = fileBytes(ptsPath);
   if (gb <= 0 || gb % 8 || pb <= 0 || pb % 24) {
      std::fprintf(stderr, "ref_gpu_ecg: bad input sizes\n");
      return 2;
   }
   const long n = gb / 8;
   const int m = (int)(pb / 24);
   if (m > 32) {
      std::fprintf(stderr, "ref_gpu_ecg: at most 32 electrodes (the reference kernel's block is 32 x m threads)\n");
      return 2;
   }
   lazy_array<Long64> gids;
   lazy_array<double> points, invr, dVmD, ecgs;
   gids.resize(n);
   points.resize(3 * m);
   invr.resize(n * m);
   ecgs.resize(m);
   {
      wo_array_ptr<Long64> g = gids.useOn(CPU);
      wo_array_ptr<double> p = points.useOn(CPU);
      if (!readFile(gidPath, g.raw(), gb) || !readFile(ptsPath, p.raw(), pb)) return 2;
   }
   {
      // as ECGSensor::calcInvR: the table starts at zero on the device
      wo_array_ptr<double> t = invr.useOn(GPU);
      if (cudaMemset(t.raw(), 0, sizeof(double) * t.size()) != cudaSuccess) return 3;
   }
   calcInvrCUDA(invr, gids, points, m, nx, ny, nz, dx, dy, dz);
   const bool sum = std::string(dvmPath) != "-";
   // calcEcg_kernel gives its first 111 blocks ceil(n / 112) cells each and
   // does not check them against n (elec/ECGSensor.cu:89-101): run it only
   // where those ranges stay inside the cells
   if (sum && 111 * ((n + 111) / 112) > n) {
      std::fprintf(stderr, "ref_gpu_ecg: the reference's ECG sum reads past %ld cells; use a multiple of 112\n", n);
      return 2;
   }
   if (sum) {
      dVmD.resize(n);
      {
         wo_array_ptr<double> d = dVmD.useOn(CPU);
         if (fileBytes(dvmPath) != n * 8 || !readFile(dvmPath, d.raw(), n * 8)) return 2;
      }
      {
         // calcEcg_kernel adds into the sums: zeroed on the device first, as
         // ECGSensor::eval does (elec/ECGSensor.cc:248-252)
         wo_array_ptr<double> e = ecgs.useOn(GPU);
         if (cudaMemset(e.raw(), 0, sizeof(double) * e.size()) != cudaSuccess) return 3;
      }
      calcEcgCUDA(ecgs, invr, dVmD, m);
   }
   if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess) {
      std::fprintf(stderr, "ref_gpu_ecg: a kernel failed\n");
      return 3;
   }
   FILE* f = std::fopen(outPath, "wb");
   if (!f) return 2;
   {
      ro_array_ptr<double> t = invr.useOn(CPU);
      std::fwrite(t.raw(), 8, n * m, f);
   }
   if (sum) {
      ro_array_ptr<double> e = ecgs.useOn(CPU);
      std::fwrite(e.raw(), 8, m, f);
   }
   std::fclose(f);
   std::printf("{\"cells\": %ld, \"electrodes\": %d}\n", n, m);
   return 0;
}
