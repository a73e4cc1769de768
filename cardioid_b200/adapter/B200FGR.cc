// B200FGR (B200FGR.hh): FGR diffusion of the reference code on the B200.
//
// This build of the reference keeps its arrays on the host, so
// updateLocalVoltage copies the local Vm to the device and calc copies dVm
// back; a CUDA build of the reference would hand the device pointers
// (useOn(GPU)) straight to cdb_fgr_update_local_voltage / cdb_fgr_calc.
// Errors end in assert, as the reference's own factories and CUDA paths do.
#include "B200FGR.hh"

#include <cuda_runtime.h>

#include <cassert>
#include <cstdio>
#include <vector>

#include "Anatomy.hh"
#include "../../include/cardioid_b200.h"

namespace {

void check(cdb_status s, const char* what)
{
   if (s != CDB_OK) {
      std::fprintf(stderr, "B200FGR: %s failed: %s\n", what, cdb_last_error());
      assert(false && "B200FGR");
   }
}

void checkCuda(cudaError_t e, const char* what)
{
   if (e != cudaSuccess) {
      std::fprintf(stderr, "B200FGR: %s: %s\n", what, cudaGetErrorString(e));
      assert(false && "B200FGR");
   }
}

}  // namespace

B200FGR::B200FGR(const FGRUtils::FGRDiffusionParms& parms, const Anatomy& anatomy, int device)
: Diffusion(parms.diffusionScale_), device_(device), nLocal_(anatomy.nLocal()), scale0_(parms.diffusionScale_)
{
   // one GPU holds every cell: halo cells from other ranks have no place here
   assert(anatomy.nRemote() == 0 && "B200FGR: remote cells are not supported");
   const unsigned n = nLocal_;
   std::vector<int64_t> gid(n);
   std::vector<int32_t> type(n);
   std::vector<double> sigma(6 * (size_t)n);
   for (unsigned ii = 0; ii < n; ++ii) {
      gid[ii] = anatomy.gid(ii);
      type[ii] = anatomy.cellType(ii);
      const SymmetricTensor s = anatomy.conductivity(ii);
      double* o = &sigma[6 * (size_t)ii];
      o[0] = s.a11; o[1] = s.a12; o[2] = s.a13; o[3] = s.a22; o[4] = s.a23; o[5] = s.a33;
   }
   check(cdb_fgr_create(device, (int32_t)anatomy.nx(), (int32_t)anatomy.ny(), (int32_t)anatomy.nz(), anatomy.dx(),
                        anatomy.dy(), anatomy.dz(), n, gid.data(), type.data(), sigma.data(), scale0_, &d_),
         "cdb_fgr_create");
   checkCuda(cudaSetDevice(device), "cudaSetDevice");
   checkCuda(cudaMalloc(&dVmIn_, sizeof(double) * (n ? n : 1)), "cudaMalloc");
   checkCuda(cudaMalloc(&dVmOut_, sizeof(double) * (n ? n : 1)), "cudaMalloc");
}

B200FGR::~B200FGR()
{
   cudaSetDevice(device_);
   cudaFree(dVmIn_);
   cudaFree(dVmOut_);
   cdb_fgr_destroy(d_);
}

void B200FGR::updateLocalVoltage(ro_mgarray_ptr<double> VmLocal)
{
   ro_array_ptr<double> vm = VmLocal.useOn(CPU);
   assert(vm.size() >= nLocal_);
   checkCuda(cudaSetDevice(device_), "cudaSetDevice");
   checkCuda(cudaMemcpy(dVmIn_, vm.raw(), sizeof(double) * nLocal_, cudaMemcpyHostToDevice), "cudaMemcpy");
   check(cdb_fgr_update_local_voltage(d_, dVmIn_, nullptr), "cdb_fgr_update_local_voltage");
}

void B200FGR::updateRemoteVoltage(ro_mgarray_ptr<double> VmRemote)
{
   assert(VmRemote.size() == 0 && "B200FGR: remote cells are not supported");
}

void B200FGR::calc(rw_mgarray_ptr<double> dVm)
{
   check(cdb_fgr_calc(d_, dVmOut_, nullptr), "cdb_fgr_calc");
   rw_array_ptr<double> out = dVm.useOn(CPU);
   assert(out.size() >= nLocal_);
   checkCuda(cudaMemcpy(out.raw(), dVmOut_, sizeof(double) * nLocal_, cudaMemcpyDeviceToHost), "cudaMemcpy");
   // setDiffusionScale after construction rescales the result
   if (diffusionScale_ != scale0_) {
      const double r = diffusionScale_ / scale0_;
      double* p = out.raw();
      for (unsigned ii = 0; ii < nLocal_; ++ii) p[ii] *= r;
   }
}

extern "C" Diffusion* b200DiffusionFactory(const FGRUtils::FGRDiffusionParms& parms, const Anatomy& anatomy)
{
   return new B200FGR(parms, anatomy, 0);
}
