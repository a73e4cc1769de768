// B200FGR: the FGR stencil as a Diffusion of the reference code
// (elec/Diffusion.hh:19-39) that computes on the B200 through the C ABI
// (cdb_fgr_*, include/cardioid_b200.h).  Weights are built on the device by
// the same rule as FGRDiffusionOMP::precomputeCoefficients
// (elec/FGRDiffusionOMP.cc:166-223); calc assigns dVm for every local cell,
// as FGRDiffusionOMP::calc does in the omp loop (elec/FGRDiffusionOMP.cc:109-131).
//
// diffusionFactory (elec/diffusionFactory.cc:37-66) is a closed if-chain;
// the one line a maintainer adds there is
//     else if (method == "b200") return new B200FGR(fgrParms, anatomy);
// and the built library also exports b200DiffusionFactory (below) for a
// driver that loads it at run time.
#ifndef B200FGR_HH
#define B200FGR_HH

#include "Diffusion.hh"
#include "FGRUtils.hh"

class Anatomy;
struct cdb_fgr;

class B200FGR : public Diffusion
{
 public:
   B200FGR(const FGRUtils::FGRDiffusionParms& parms, const Anatomy& anatomy, int device = 0);
   ~B200FGR();
   void updateLocalVoltage(ro_mgarray_ptr<double> VmLocal);
   void updateRemoteVoltage(ro_mgarray_ptr<double> VmRemote);
   void calc(rw_mgarray_ptr<double> dVm);

 private:
   B200FGR(const B200FGR&);
   B200FGR& operator=(const B200FGR&);

   cdb_fgr* d_ = nullptr;
   int device_;
   unsigned nLocal_;
   double scale0_;            // the diffusionScale the weights were built with
   double* dVmIn_ = nullptr;  // device copies of the local Vm and of dVm
   double* dVmOut_ = nullptr;
};

// The same construction behind a C symbol, for drivers that dlopen this
// library (the reference's own dynamic-plugin pattern, elec/reactionFactory.cc:48-70).
extern "C" Diffusion* b200DiffusionFactory(const FGRUtils::FGRDiffusionParms& parms, const Anatomy& anatomy);

#endif
