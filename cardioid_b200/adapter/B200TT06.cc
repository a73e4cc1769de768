// B200TT06: BetterTT06 as a Reaction of the reference code
// (elec/Reaction.hh:10-40) that computes on the B200 through the C ABI
// (cdb_reaction_*, include/cardioid_b200.h).
//
// A maintainer builds it against a Cardioid checkout either as a dynamic
// reaction (-DDYNAMIC_REACTION=1: reactionFactory dlopens the shared object
// named by the REACTION's `method` and calls its `factory`,
// elec/reactionFactory.cc:48-70) or as a built-in (registered as
// "B200TT06", elec/registerBuiltinReactions.pl:32-63).  oracle/ref/Makefile
// builds the dynamic form next to the reference's own code, and
// tests/test_adapter_gpu.py runs it inside the reference's ReactionManager.
//
// REACTION keys as BetterTT06 (reactionFactoryForBetterTT06,
// elec/BetterTT06.cc:69-160): celltype, g_CaL g_K1 g_Kr g_Ks g_Na g_bca
// g_bna g_pCa g_pK g_to, and fit, a FIT object whose dt, celltype and g_K1
// match (required: this reaction does not generate fits; the reference's
// BetterTT06 or cardioid_b200.fitgen writes them).  Extra keys: precision
// (fp64 | mixed) and device.
//
// This build of the reference keeps its arrays on the host, so every calc
// copies Vm in and the reaction's dVm entries out; a CUDA build of the
// reference would hand the device pointers (useOn(GPU)) straight through.
#include <cuda_runtime.h>

#include <algorithm>
#include <cassert>
#include <cstdio>
#include <string>
#include <vector>

#include "Reaction.hh"
#include "object_cc.hh"
#include "reactionFactory.hh"
#include "../../include/cardioid_b200.h"

namespace {

const char* const kStateNames[CDB_NUM_STATES] = {"Ca_SR", "Ca_i", "Ca_ss", "K_i", "Na_i", "R_prime",
                                                "Xr1",   "Xr2",  "Xs",    "d",   "f",    "f2",
                                                "fCass", "h",    "j",     "m",   "r",    "s"};
const char* const kStateUnits[CDB_NUM_STATES] = {"uM", "uM", "uM", "mM", "mM", "1", "1", "1", "1",
                                                 "1",  "1",  "1",  "1",  "1",  "1", "1", "1", "1"};

void check(cdb_status s, const char* what)
{
  if (s != CDB_OK) {
    std::fprintf(stderr, "B200TT06: %s failed: %s\n", what, cdb_last_error());
    assert(false && "B200TT06");   // the reference asserts on such errors
  }
}

void checkCuda(cudaError_t e, const char* what)
{
  if (e != cudaSuccess) {
    std::fprintf(stderr, "B200TT06: %s: %s\n", what, cudaGetErrorString(e));
    assert(false && "B200TT06");
  }
}

}  // namespace

class B200TT06 : public Reaction
{
 public:
  B200TT06(const cdb_tt06_params& p, const std::vector<cdb_fit>& fits, int nCells, double dt, int device,
           cdb_precision prec)
  : n_(nCells), device_(device)
  {
    check(cdb_reaction_create(device, prec, &p, fits.data(), nCells, dt, &r_), "cdb_reaction_create");
    checkCuda(cudaSetDevice(device), "cudaSetDevice");
    checkCuda(cudaMalloc(&dIndex_, sizeof(int) * (n_ > 0 ? n_ : 1)), "cudaMalloc");
    state_.assign(CDB_NUM_STATES, std::vector<double>());
    fresh_.assign(CDB_NUM_STATES, false);
    dirty_.assign(CDB_NUM_STATES, false);
  }

  ~B200TT06()
  {
    cudaSetDevice(device_);
    cudaFree(dIndex_);
    cudaFree(dVm_);
    cudaFree(dDVm_);
    cdb_reaction_destroy(r_);
  }

  std::string methodName() const { return "BetterTT06"; }   // SINGLECELL objects for BetterTT06 apply

  void calc(double dt, ro_mgarray_ptr<int> indexArray, ro_mgarray_ptr<double> Vm, ro_mgarray_ptr<double> iStim,
            wo_mgarray_ptr<double> dVm)
  {
    flushStates();
    ro_array_ptr<int> idx = indexArray.useOn(CPU);
    ro_array_ptr<double> vm = Vm.useOn(CPU);
    wo_array_ptr<double> dvm = dVm.useOn(CPU);
    upload(idx.raw(), (int)idx.size(), vm.raw(), (int)vm.size());
    check(cdb_reaction_calc(r_, dt, dIndex_, dVm_, nullptr, dDVm_, nullptr), "cdb_reaction_calc");
    (void)iStim;   // unused, as in BetterTT06
    scatter(idx.raw(), (int)idx.size(), dDVm_, dvm.raw(), (int)dvm.size());
    for (size_t k = 0; k < fresh_.size(); ++k) fresh_[k] = false;
  }

  void initializeMembraneVoltage(ro_mgarray_ptr<int> indexArray, wo_mgarray_ptr<double> Vm)
  {
    ro_array_ptr<int> idx = indexArray.useOn(CPU);
    wo_array_ptr<double> vm = Vm.useOn(CPU);
    upload(idx.raw(), (int)idx.size(), nullptr, (int)vm.size());
    check(cdb_reaction_init(r_, dIndex_, dVm_, nullptr), "cdb_reaction_init");
    scatter(idx.raw(), (int)idx.size(), dVm_, vm.raw(), (int)vm.size());
  }

  void getCheckpointInfo(std::vector<std::string>& names, std::vector<std::string>& units) const
  {
    names.assign(kStateNames, kStateNames + CDB_NUM_STATES);
    units.assign(kStateUnits, kStateUnits + CDB_NUM_STATES);
  }

  int getVarHandle(const std::string& name) const
  {
    for (int k = 0; k < CDB_NUM_STATES; ++k)
      if (name == kStateNames[k]) return k;
    return -1;
  }

  void setValue(int iCell, int handle, double value)
  {
    // initializeMembraneState (elec/Reaction.cc:42-53) passes indices up to
    // the whole tissue's size; only this reaction's cells exist here
    if (handle < 0 || handle >= CDB_NUM_STATES || iCell < 0 || iCell >= n_) return;
    load(handle)[iCell] = value;
    dirty_[handle] = true;
  }

  double getValue(int iCell, int handle) const
  {
    if (handle < 0 || handle >= CDB_NUM_STATES || iCell < 0 || iCell >= n_) return 0.0;
    return const_cast<B200TT06*>(this)->load(handle)[iCell];
  }

  const std::string getUnit(const std::string& name) const
  {
    const int k = getVarHandle(name);
    return k >= 0 ? kStateUnits[k] : "INVALID";
  }

 private:
  // Device copies of the index slice and of the whole Vm / dVm arrays.
  void upload(const int* idx, int nIdx, const double* vm, int nVm)
  {
    assert(nIdx == n_);
    checkCuda(cudaSetDevice(device_), "cudaSetDevice");
    if (nVm > cap_) {
      cudaFree(dVm_);
      cudaFree(dDVm_);
      checkCuda(cudaMalloc(&dVm_, sizeof(double) * nVm), "cudaMalloc");
      checkCuda(cudaMalloc(&dDVm_, sizeof(double) * nVm), "cudaMalloc");
      cap_ = nVm;
    }
    if (hostIndex_.size() != (size_t)nIdx || !std::equal(idx, idx + nIdx, hostIndex_.begin())) {
      hostIndex_.assign(idx, idx + nIdx);
      checkCuda(cudaMemcpy(dIndex_, idx, sizeof(int) * nIdx, cudaMemcpyHostToDevice), "cudaMemcpy");
    }
    if (vm) checkCuda(cudaMemcpy(dVm_, vm, sizeof(double) * nVm, cudaMemcpyHostToDevice), "cudaMemcpy");
  }

  // host[idx[i]] = device[idx[i]] for this reaction's cells only: other
  // reactions own the rest of the array.
  void scatter(const int* idx, int nIdx, const double* device, double* host, int nHost)
  {
    tmp_.resize(nHost);
    checkCuda(cudaMemcpy(tmp_.data(), device, sizeof(double) * nHost, cudaMemcpyDeviceToHost), "cudaMemcpy");
    for (int i = 0; i < nIdx; ++i) host[idx[i]] = tmp_[idx[i]];
  }

  std::vector<double>& load(int k)
  {
    if (!fresh_[k]) {
      state_[k].resize(n_);
      check(cdb_reaction_get_state(r_, k, state_[k].data()), "cdb_reaction_get_state");
      fresh_[k] = true;
    }
    return state_[k];
  }

  void flushStates()
  {
    for (int k = 0; k < CDB_NUM_STATES; ++k)
      if (dirty_[k]) {
        check(cdb_reaction_set_state(r_, k, state_[k].data()), "cdb_reaction_set_state");
        dirty_[k] = false;
      }
  }

  cdb_reaction* r_ = nullptr;
  int n_;
  int device_;
  int* dIndex_ = nullptr;
  double* dVm_ = nullptr;
  double* dDVm_ = nullptr;
  int cap_ = 0;
  std::vector<int> hostIndex_;
  std::vector<double> tmp_;
  std::vector<std::vector<double>> state_;   // host copies of the states, cell order of the reaction
  std::vector<bool> fresh_, dirty_;
};

REACTION_FACTORY(B200TT06)(OBJECT* obj, const double dt, const int numPoints, const ThreadTeam&)
{
  cdb_tt06_params p;
  objectGet(obj, "celltype", p.celltype, "0");
  // BetterTT06's defaults, g_Ks and g_to by celltype (elec/BetterTT06.cc:75-116)
  objectGet(obj, "g_CaL", p.g_CaL, "3.98e-5");
  objectGet(obj, "g_K1", p.g_K1, "5.405");
  objectGet(obj, "g_Kr", p.g_Kr, "0.153");
  objectGet(obj, "g_Ks", p.g_Ks, p.celltype == 1 ? "0.098" : "0.392");
  objectGet(obj, "g_Na", p.g_Na, "14.838");
  objectGet(obj, "g_bca", p.g_bca, "0.000592");
  objectGet(obj, "g_bna", p.g_bna, "0.00029");
  objectGet(obj, "g_pCa", p.g_pCa, "0.1238");
  objectGet(obj, "g_pK", p.g_pK, "0.0146");
  objectGet(obj, "g_to", p.g_to, p.celltype == 0 ? "0.073" : "0.294");
  std::string fitName, precision;
  int device = 0;
  objectGet(obj, "fit", fitName, "");
  objectGet(obj, "precision", precision, "fp64");
  objectGet(obj, "device", device, "0");
  OBJECT* fitObj = fitName.empty() ? nullptr : objectFind(fitName, "FIT");
  double fdt, fct, fgk1;
  std::vector<std::string> functions;
  if (fitObj) {
    objectGet(fitObj, "dt", fdt, "nan");
    objectGet(fitObj, "celltype", fct, "nan");
    objectGet(fitObj, "g_K1", fgk1, "nan");
    objectGet(fitObj, "functions", functions);
  }
  if (!fitObj || fdt != dt || fct != p.celltype || fgk1 != p.g_K1 || functions.size() != CDB_NUM_FITS) {
    std::fprintf(stderr, "B200TT06: REACTION needs a FIT object matching its dt, celltype and g_K1\n");
    assert(false && "B200TT06 fit");
  }
  std::vector<cdb_fit> fits(CDB_NUM_FITS);
  for (int k = 0; k < CDB_NUM_FITS; ++k) {
    OBJECT* f = objectFind(functions[k], "FUNCTION");
    std::vector<double> coeff;
    objectGet(f, "numer", fits[k].numer, "-1");
    objectGet(f, "denom", fits[k].denom, "-1");
    objectGet(f, "coeff", coeff);
    assert(coeff.size() <= CDB_MAX_COEFF);
    for (size_t c = 0; c < coeff.size(); ++c) fits[k].coeff[c] = coeff[c];
  }
  return new B200TT06(p, fits, numPoints, dt, device, precision == "mixed" ? CDB_MIXED : CDB_FP64);
}
