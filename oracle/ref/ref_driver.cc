// Thin driver that runs the reference's own CPU path (BetterTT06 through
// ReactionManager, FGRDiffusionOMP, BoxStimulus) on an in-memory anatomy and
// exposes it through a small C API for the tests and the CPU baseline.
//
// TEST INFRASTRUCTURE ONLY.  It is compiled, together with the reference
// sources it drives, into oracle/_ref/ by oracle/ref/Makefile.  The product
// never links or loads it.
//
// The step restates the body of the reference's "omp" time loop
// (elec/simulationLoop.cc:183-231) in the same order:
//   iStim = 0; stimulus[i]->stim(time, iStim); reaction->calc(dt, Vm, iStim, dVmR);
//   diffusion->updateLocalVoltage(Vm); diffusion->calc(dVmD);
//   Vm += dt*(dVmR + dVmD + iStim); time += dt;
// and then applies the activation-time rule of ActivationTimeSensor::eval
// (elec/ActivationTimeSensor.cc:99-111): first post-step time with Vm > 0.
#include <mpi.h>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <sstream>
#include <omp.h>
#include <cstdlib>
#include <unistd.h>
#include <dlfcn.h>

#include "Anatomy.hh"
#include "AnatomyCell.hh"
#include "JHUConductivity.hh"
// CUDADiffusion keeps its face-conductivity table private; the oracle
// reads it back to pin the 6-face plugin's table.
#define private public
#include "CUDADiffusion.hh"
#undef private
#include "FGRDiffusionOMP.hh"
#include "FGRUtils.hh"
#include "ReactionManager.hh"
#include "Reaction.hh"
#include "Stimulus.hh"
#include "ThreadServer.hh"
#include "lazy_array.hh"
#include "object_cc.hh"
#include "units.h"
#include "PerformanceTimers.hh"
#include "BucketOfBits.hh"
#include "readPioFile.hh"
#include "pio.h"

Stimulus* stimulusFactory(const std::string& name, const Anatomy& anatomy);
// The reference's CPU ECG sum (elec/ECGSensor.cc:231-246; not in a header).
void calcEcg(rw_mgarray_ptr<double> ecgs, ro_mgarray_ptr<double> invr, ro_mgarray_ptr<double> dVmDiffusion,
             const int nEcgPoints);

namespace {

struct RefSim {
   Anatomy anatomy;
   ReactionManager reaction;
   Diffusion* diffusion = nullptr;
   double diffusionScale = 0;
   std::vector<Stimulus*> stimulus;
   lazy_array<double> Vm, dVmR, dVmD, iStim;
   lazy_array<double> remote;
   std::vector<double> actTime;
   std::vector<char> activated;
   double dt = 0, time = 0;
   long loop = 0;
   bool useDiffusion = true;
};

std::vector<std::string> splitWords(const char* s)
{
   std::vector<std::string> out;
   if (!s) return out;
   std::istringstream in(s);
   std::string w;
   while (in >> w) out.push_back(w);
   return out;
}

}  // namespace

extern "C" {

// Compiles object-database text (REACTION, FIT, FUNCTION, STIMULUS objects,
// in the reference's object.data syntax) into the global object database.
int ref_objects_compile(const char* text)
{
   static bool once = false;
   if (!once) {
      int argc = 0; char** argv = nullptr;
      MPI_Init(&argc, &argv);
      // Cardioid's unit system: internal and external units are the same
      // (mm, ug, ms, mA, K, nmol, cd), as set in elec/cardioid.cc:84-85.
      units_internal(1e-3, 1e-9, 1e-3, 1e-3, 1, 1e-9, 1);
      units_external(1e-3, 1e-9, 1e-3, 1e-3, 1, 1e-9, 1);
      // The stencil wraps its loops in the reference timers (elec/cardioid.cc:87).
      profileInit();
      once = true;
   }
   // object_compilestring takes one object; a file takes many.
   char path[] = "/tmp/oracle_objects_XXXXXX";
   int fd = mkstemp(path);
   if (fd < 0) return -1;
   FILE* f = fdopen(fd, "w");
   std::fputs(text, f);
   std::fclose(f);
   object_compilefile(path);
   std::remove(path);
   return 0;
}

// Builds the simulation.  Cells are given in local order with their gid on
// an nx*ny*nz grid (gid = x + nx*(y + ny*z)), their anatomy cellType and
// their conductivity tensor as 6 doubles (a11 a12 a13 a22 a23 a33).
void* ref_sim_create(const char* reactionNames, const char* stimulusNames,
                     int nx, int ny, int nz, double dx, double dy, double dz,
                     long nCells, const long long* gid, const int* cellType,
                     const double* sigma6, double dt, double diffusionScale,
                     int useDiffusion)
{
   RefSim* sim = new RefSim;
   sim->dt = dt;
   sim->useDiffusion = useDiffusion != 0;
   Anatomy& a = sim->anatomy;
   a.setGridSize(nx, ny, nz);
   a.dx() = dx; a.dy() = dy; a.dz() = dz;
   a.offset_x() = 0; a.offset_y() = 0; a.offset_z() = 0;
   std::vector<AnatomyCell>& cells = a.cellArray();
   cells.resize(nCells);
   for (long ii = 0; ii < nCells; ++ii) {
      AnatomyCell& c = cells[ii];
      c.gid_ = gid[ii];
      c.cellType_ = cellType[ii];
      c.sigma_.a11 = sigma6[6 * ii + 0];
      c.sigma_.a12 = sigma6[6 * ii + 1];
      c.sigma_.a13 = sigma6[6 * ii + 2];
      c.sigma_.a22 = sigma6[6 * ii + 3];
      c.sigma_.a23 = sigma6[6 * ii + 4];
      c.sigma_.a33 = sigma6[6 * ii + 5];
      c.dest_ = 0;
      c.sortind_ = (int)ii;
   }
   a.nRemote() = 0;
   a.nGlobal() = nCells;

   for (const std::string& r : splitWords(reactionNames)) sim->reaction.addReaction(r);
   {
      std::vector<int> ct(cellType, cellType + nCells);
      ro_array_ptr<int> ctp(&ct[0], ct.size());
      // The thread server hands each team its own threads and runs out, so
      // every simulation shares one team (BetterTT06 ignores it).
      static ThreadTeam group = ThreadServer::getInstance().getThreadTeam(std::vector<unsigned>());
      sim->reaction.create(dt, ctp, group);
   }
   sim->Vm.resize(nCells);
   sim->dVmR.resize(nCells);
   sim->dVmD.resize(nCells);
   sim->iStim.resize(nCells);
   sim->remote.resize(0);
   {
      wo_array_ptr<double> v = sim->Vm.useOn(CPU);
      wo_array_ptr<double> r = sim->dVmR.useOn(CPU);
      wo_array_ptr<double> d = sim->dVmD.useOn(CPU);
      for (long ii = 0; ii < nCells; ++ii) { v[ii] = 0; r[ii] = 0; d[ii] = 0; }
   }
   sim->reaction.initializeMembraneState(sim->Vm);
   sim->diffusionScale = diffusionScale;
   if (sim->useDiffusion) {
      FGRUtils::FGRDiffusionParms p;
      p.printBBox_ = false;
      p.diffusionScale_ = diffusionScale;
      sim->diffusion = new FGRDiffusionOMP(p, a);
   }
   for (const std::string& s : splitWords(stimulusNames))
      sim->stimulus.push_back(stimulusFactory(s, a));
   sim->actTime.assign(nCells, 0.0);
   sim->activated.assign(nCells, 0);
   return sim;
}

// Replaces the simulation's FGRDiffusionOMP by the Diffusion that the shared
// library at `path` builds through its b200DiffusionFactory symbol (a
// driver-side stand-in for the one-line diffusionFactory addition); 0 on
// success.
int ref_sim_use_diffusion_plugin(void* h, const char* path)
{
   RefSim* sim = static_cast<RefSim*>(h);
   void* lib = dlopen(path, RTLD_NOW);
   if (!lib) { std::fprintf(stderr, "dlopen %s: %s\n", path, dlerror()); return 1; }
   typedef Diffusion* (*Factory)(const FGRUtils::FGRDiffusionParms&, const Anatomy&);
   Factory f = (Factory)dlsym(lib, "b200DiffusionFactory");
   if (!f) { std::fprintf(stderr, "dlsym b200DiffusionFactory: %s\n", dlerror()); return 2; }
   FGRUtils::FGRDiffusionParms p;
   p.printBBox_ = false;
   p.diffusionScale_ = sim->diffusionScale;
   delete sim->diffusion;
   sim->diffusion = f(p, sim->anatomy);
   sim->useDiffusion = true;
   return 0;
}

// The face-conductivity table that the reference's "cuda" Diffusion builds
// on the host for the simulation's anatomy (CUDADiffusion constructor,
// elec/CUDADiffusion.cc:30-130): dims[0..2] = its local grid (the anatomy's
// bounding box, findBoundingBox(anatomy, false)), dims[3..5] = the grid
// offset of that box, and out[9 nx ny nz] in its layout, entry
// z + nz (y + ny (x + nx (j + 3 i))) for face normal i and gradient
// direction j.  Returns nx ny nz, or -(nx ny nz) (dims still set, out
// untouched) when out holds fewer than 9 nx ny nz entries.
long ref_sim_diff6_face_sigma(void* h, int* dims, double* out, long capacity)
{
   RefSim* sim = static_cast<RefSim*>(h);
   CUDADiffusion d(sim->anatomy, 0, sim->diffusionScale);
   const long n = (long)d.nx_ * d.ny_ * d.nz_;
   dims[0] = d.nx_; dims[1] = d.ny_; dims[2] = d.nz_;
   Tuple lo = d.localGrid_.localTuple(Tuple(0, 0, 0));
   dims[3] = -lo.x(); dims[4] = -lo.y(); dims[5] = -lo.z();
   if (capacity < 9 * n) return -n;
   ro_array_ptr<double> f = d.sigmaFaceNormal_.readonly(CPU);
   for (long k = 0; k < 9 * n; ++k) out[k] = f[k];
   return n;
}

// ecgs[j] = sum over cells i of invr[i nPoints + j] dVmD[i], by the
// reference's CPU ECG sum calcEcg (elec/ECGSensor.cc:231-246) on arrays in
// its layout; ecgs starts at zero (ECGSensor::eval zeroes it first).
void ref_calc_ecg(long nCells, int nPoints, const double* invr, const double* dVmD, double* ecgs)
{
   lazy_array<double> e, r, d;
   e.resize(nPoints);
   r.resize(nCells * nPoints);
   d.resize(nCells);
   {
      wo_array_ptr<double> ee = e.writeonly(CPU), rr = r.writeonly(CPU), dd = d.writeonly(CPU);
      for (int j = 0; j < nPoints; ++j) ee[j] = 0;
      for (long k = 0; k < nCells * nPoints; ++k) rr[k] = invr[k];
      for (long k = 0; k < nCells; ++k) dd[k] = dVmD[k];
   }
   calcEcg(e, r, d, nPoints);
   ro_array_ptr<double> out = e.readonly(CPU);
   for (int j = 0; j < nPoints; ++j) ecgs[j] = out[j];
}

// Conductivity tensors of the reference's JHU rule (JHUConductivity::compute,
// elec/JHUConductivity.cc:26-120) for cells `gid` of an nx*ny*nz grid, with
// the parameters setConductivity gives it (elec/setConductivity.cc:207-226,
// transmural axis ny - 2); out[6 n] = a11 a12 a13 a22 a23 a33 per cell.
void ref_jhu_sigma(int nx, int ny, int nz, double sigmaLi, double sigmaTi, double sheetAngle, int rotationMatrix,
                   int homogeneousFiber, long n, const long long* gid, double* out)
{
   JHUConductivityParms p;
   p.nx = nx; p.ny = ny; p.nz = nz;
   p.transmuralAxis = ny - 2;
   p.sigmaLi = sigmaLi;
   p.sigmaTi = sigmaTi;
   p.sheetAngle = sheetAngle;
   p.rotatationMatrix = rotationMatrix;
   p.homogeneousFiber = homogeneousFiber != 0;
   JHUConductivity jhu(p);
   for (long ii = 0; ii < n; ++ii) {
      AnatomyCell c;
      c.gid_ = gid[ii];
      jhu.compute(c);
      const double v[6] = {c.sigma_.a11, c.sigma_.a12, c.sigma_.a13, c.sigma_.a22, c.sigma_.a23, c.sigma_.a33};
      for (int k = 0; k < 6; ++k) out[6 * ii + k] = v[k];
   }
}

void ref_sim_destroy(void* h)
{
   RefSim* sim = static_cast<RefSim*>(h);
   delete sim->diffusion;
   for (Stimulus* s : sim->stimulus) delete s;
   delete sim;
}

long ref_sim_ncells(void* h) { return (long)static_cast<RefSim*>(h)->anatomy.nLocal(); }
double ref_sim_time(void* h) { return static_cast<RefSim*>(h)->time; }

void ref_sim_get_vm(void* h, double* out)
{
   RefSim* sim = static_cast<RefSim*>(h);
   ro_array_ptr<double> v = sim->Vm.useOn(CPU);
   for (size_t ii = 0; ii < v.size(); ++ii) out[ii] = v[ii];
}

void ref_sim_set_vm(void* h, const double* in)
{
   RefSim* sim = static_cast<RefSim*>(h);
   wo_array_ptr<double> v = sim->Vm.useOn(CPU);
   for (size_t ii = 0; ii < v.size(); ++ii) v[ii] = in[ii];
}

void ref_sim_get_dvm(void* h, double* dVmR, double* dVmD, double* iStim)
{
   RefSim* sim = static_cast<RefSim*>(h);
   ro_array_ptr<double> r = sim->dVmR.useOn(CPU);
   ro_array_ptr<double> d = sim->dVmD.useOn(CPU);
   ro_array_ptr<double> s = sim->iStim.useOn(CPU);
   for (size_t ii = 0; ii < r.size(); ++ii) {
      if (dVmR) dVmR[ii] = r[ii];
      if (dVmD) dVmD[ii] = d[ii];
      if (iStim) iStim[ii] = s[ii];
   }
}

void ref_sim_get_activation(void* h, double* out)
{
   RefSim* sim = static_cast<RefSim*>(h);
   for (size_t ii = 0; ii < sim->actTime.size(); ++ii)
      out[ii] = sim->activated[ii] ? sim->actTime[ii] : -1.0;
}

// Field names in checkpoint order, space separated (the reference's
// ReactionManager::getCheckpointInfo order).
int ref_sim_field_names(void* h, char* buf, int bufLen)
{
   RefSim* sim = static_cast<RefSim*>(h);
   std::vector<std::string> names, units;
   sim->reaction.getCheckpointInfo(names, units);
   std::string all;
   for (size_t ii = 0; ii < names.size(); ++ii) {
      if (ii) all += " ";
      all += names[ii];
   }
   if ((int)all.size() + 1 > bufLen) return -1;
   std::strcpy(buf, all.c_str());
   return (int)names.size();
}

int ref_sim_get_state(void* h, const char* name, double* out)
{
   RefSim* sim = static_cast<RefSim*>(h);
   int handle = sim->reaction.getVarHandle(name);
   if (handle < 0) return -1;
   long n = sim->anatomy.nLocal();
   for (long ii = 0; ii < n; ++ii) out[ii] = sim->reaction.getValue((int)ii, handle);
   return 0;
}

int ref_sim_set_state(void* h, const char* name, const double* in)
{
   RefSim* sim = static_cast<RefSim*>(h);
   int handle = sim->reaction.getVarHandle(name);
   if (handle < 0) return -1;
   long n = sim->anatomy.nLocal();
   for (long ii = 0; ii < n; ++ii) sim->reaction.setValue((int)ii, handle, in[ii]);
   return 0;
}

void ref_set_threads(int n) { omp_set_num_threads(n); }

// Advances nSteps time steps.
void ref_sim_step(void* h, int nSteps)
{
   RefSim* sim = static_cast<RefSim*>(h);
   const long nLocal = sim->anatomy.nLocal();
   for (int step = 0; step < nSteps; ++step) {
      {
         wo_array_ptr<double> iStim = sim->iStim.useOn(CPU);
         for (long ii = 0; ii < nLocal; ++ii) iStim[ii] = 0;
      }
      for (Stimulus* s : sim->stimulus) s->stim(sim->time, sim->iStim);
      sim->reaction.calc(sim->dt, sim->Vm, sim->iStim, sim->dVmR);
      if (sim->diffusion) {
         sim->diffusion->updateLocalVoltage(sim->Vm);
         if (sim->anatomy.nRemote() > 0) sim->diffusion->updateRemoteVoltage(sim->remote);
         sim->diffusion->calc(sim->dVmD);
      }
      {
         rw_array_ptr<double> Vm = sim->Vm.useOn(CPU);
         ro_array_ptr<double> dVmR = sim->dVmR.useOn(CPU);
         ro_array_ptr<double> dVmD = sim->dVmD.useOn(CPU);
         ro_array_ptr<double> iStim = sim->iStim.useOn(CPU);
         double dt = sim->dt;
         for (long ii = 0; ii < nLocal; ++ii) Vm[ii] += dt * (dVmR[ii] + dVmD[ii] + iStim[ii]);
      }
      sim->time += sim->dt;
      ++sim->loop;
      {
         ro_array_ptr<double> Vm = sim->Vm.useOn(CPU);
         for (long ii = 0; ii < nLocal; ++ii) {
            if (sim->activated[ii]) continue;
            if (Vm[ii] > 0) { sim->activated[ii] = 1; sim->actTime[ii] = sim->time; }
         }
      }
   }
}

// Reads a pio file (name ends in '#', e.g. snapshot.000000000010/state#)
// through the reference's own reader (simUtil/src/pio.c,
// elec/readPioFile.cc, elec/BucketOfBits.cc), as readCheckpoint does
// (elec/checkpointIO.cc:213-268).  Returns the record count (-1 if the file
// cannot be opened); field names go space-separated into names; with values
// given (capacity >= records x fields) every field of every record as a
// double, record-major (u8 and int fields converted).
long ref_read_pio(const char* name, int* nFields, char* names, int namesLen, double* values, long capacity)
{
   std::string first = std::string(name) + "000000";
   if (access(first.c_str(), R_OK) != 0) return -1;
   PFILE* file = Popen(name, "r", MPI_COMM_WORLD);
   if (!file) return -1;
   BucketOfBits* data = readPioFile(file);
   Pclose(file);
   const long n = data->nRecords();
   const int nf = data->nFields();
   *nFields = nf;
   std::string all;
   for (int f = 0; f < nf; ++f) all += (f ? " " : "") + data->fieldName(f);
   if (names && namesLen > 0) {
      std::strncpy(names, all.c_str(), namesLen - 1);
      names[namesLen - 1] = 0;
   }
   if (values && capacity >= n * nf)
      for (long r = 0; r < n; ++r) {
         BucketOfBits::Record rec = data->getRecord(r);
         for (int f = 0; f < nf; ++f) {
            double v = 0;
            switch (data->dataType(f)) {
              case BucketOfBits::intType: { int t; rec.getValue(f, t); v = t; break; }
              case BucketOfBits::u8Type: { uint64_t t; rec.getValue(f, t); v = (double)t; break; }
              default: rec.getValue(f, v);
            }
            values[r * nf + f] = v;
         }
      }
   delete data;
   return n;
}

}  // extern "C"
