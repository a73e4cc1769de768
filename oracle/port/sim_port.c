/* FGR diffusion, box stimulus and the omp-loop integrator restated on the
 * CPU.  TEST INFRASTRUCTURE (see oracle_port.h). */
#include "oracle_port.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* The 19 stencil nodes in the reference's NodeLocation order
 * (elec/FGRUtils.hh:22-24): offsets in (x, y, z). */
static const int kNode[19][3] = {
   {0, 0, 0},   {-1, 0, 0},  {0, -1, 0}, {1, 0, 0},   {0, 1, 0},   {0, 0, -1}, {0, 0, 1},
   {-1, -1, 0}, {1, -1, 0},  {1, 1, 0},  {-1, 1, 0},  {-1, 0, -1}, {0, -1, -1}, {1, 0, -1},
   {0, 1, -1},  {-1, 0, 1},  {0, -1, 1}, {1, 0, 1},   {0, 1, 1}};

/* Faces in the reference's iFace order (elec/FGRDiffusionOMP.cc:64-69):
 * -x, -y, +x, +y, -z, +z, as (axis, sign). */
static const int kFace[6][2] = {{0, -1}, {1, -1}, {0, 1}, {1, 1}, {2, -1}, {2, 1}};

static int node_of(int ox, int oy, int oz)
{
   for (int k = 0; k < 19; ++k)
      if (kNode[k][0] == ox && kNode[k][1] == oy && kNode[k][2] == oz) return k;
   return -1;
}

struct op_sim {
   int nx, ny, nz;
   double dx, dy, dz;
   int64_t n;
   int64_t* gid;
   uint8_t* reaction;
   int nParams;
   op_params_t* params;
   int nStim;
   op_stim_t* stim;
   double dt, scale, time;
   int useDiffusion;
   /* bounding box with a one-voxel halo, z fastest (elec/Array3d.hh:173-177) */
   int bx, by, bz, ox, oy, oz;
   int64_t nBlock;
   int64_t* blockIndex;
   double* vmBlock;
   double* A;        /* 19 per cell: A0, A[1..18] */
   long off[19];
   double *vm, *dvmR, *dvmD, *iStim, *state, *act;
   char* activated;
};

static int64_t block_index(const op_sim_t* s, int x, int y, int z)
{
   return (int64_t)(z - s->oz) + (int64_t)s->bz * ((int64_t)(y - s->oy) + (int64_t)s->by * (x - s->ox));
}

/* The gradient weights of one face component (elec/FGRUtils.cc:10-148):
 * the normal component is the two-point difference across the face; a
 * tangential component is the four-node average difference (+1/4 on the
 * nodes one step along the axis on both sides of the face, -1/4 one step
 * against it), and only when all four nodes are tissue. */
static void face_gradient(int face, const int tissue[19], double grad[3][19])
{
   memset(grad, 0, sizeof(double) * 3 * 19);
   const int axis = kFace[face][0], sign = kFace[face][1];
   int nbr[3] = {0, 0, 0};
   nbr[axis] = sign;
   const int nbrNode = node_of(nbr[0], nbr[1], nbr[2]);
   if (sign > 0) { grad[axis][nbrNode] = 1.0; grad[axis][0] = -1.0; }
   else { grad[axis][0] = 1.0; grad[axis][nbrNode] = -1.0; }
   for (int b = 0; b < 3; ++b) {
      if (b == axis) continue;
      int cp[3] = {0, 0, 0}, cm[3] = {0, 0, 0}, np_[3], nm[3];
      cp[b] = 1; cm[b] = -1;
      for (int k = 0; k < 3; ++k) { np_[k] = nbr[k] + cp[k]; nm[k] = nbr[k] + cm[k]; }
      int kcp = node_of(cp[0], cp[1], cp[2]), kcm = node_of(cm[0], cm[1], cm[2]);
      int knp = node_of(np_[0], np_[1], np_[2]), knm = node_of(nm[0], nm[1], nm[2]);
      if (tissue[kcp] && tissue[kcm] && tissue[knp] && tissue[knm]) {
         grad[b][kcp] = 0.25; grad[b][knp] = 0.25;
         grad[b][kcm] = -0.25; grad[b][knm] = -0.25;
      }
   }
}

/* precomputeCoefficients + f1, elec/FGRDiffusionOMP.cc:166-265. */
static void build_weights(op_sim_t* s, const int* cellType, const double* sigma6)
{
   const double h[3] = {s->dx, s->dy, s->dz};
   const double hInv[3] = {1.0 / s->dx, 1.0 / s->dy, 1.0 / s->dz};
   const double vol = h[0] * h[1] * h[2];
   int* tissueBlk = calloc(s->nBlock, sizeof(int));
   double* sigBlk = calloc(s->nBlock * 6, sizeof(double));
   for (int64_t i = 0; i < s->n; ++i) {
      int64_t b = s->blockIndex[i];
      memcpy(sigBlk + 6 * b, sigma6 + 6 * i, 6 * sizeof(double));
      tissueBlk[b] = cellType[i] > 0;
   }
   for (int64_t i = 0; i < s->n; ++i) {
      int64_t b = s->blockIndex[i];
      double* A = s->A + 19 * i;
      double W[19] = {0};
      int tissue[19];
      for (int k = 0; k < 19; ++k) tissue[k] = tissueBlk[b + s->off[k]];
      for (int face = 0; face < 6; ++face) {
         const int axis = kFace[face][0], sign = kFace[face][1];
         int64_t nb = b + s->off[node_of(axis == 0 ? sign : 0, axis == 1 ? sign : 0, axis == 2 ? sign : 0)];
         if (tissueBlk[nb] == 0) continue;
         const double* sa = sigBlk + 6 * b;
         const double* sb = sigBlk + 6 * nb;
         /* (sigma_a + sigma_b) / 2.0, componentwise (elec/SymmetricTensor.cc) */
         double a11 = (sa[0] + sb[0]) / 2.0, a12 = (sa[1] + sb[1]) / 2.0, a13 = (sa[2] + sb[2]) / 2.0;
         double a22 = (sa[3] + sb[3]) / 2.0, a23 = (sa[4] + sb[4]) / 2.0, a33 = (sa[5] + sb[5]) / 2.0;
         double S[3] = {0, 0, 0};
         if (axis == 0) S[0] = sign * (h[1] * h[2]);
         if (axis == 1) S[1] = sign * (h[0] * h[2]);
         if (axis == 2) S[2] = sign * (h[0] * h[1]);
         double sts[3];
         sts[0] = (a11 * S[0] + a12 * S[1] + a13 * S[2]) / vol;
         sts[1] = (a12 * S[0] + a22 * S[1] + a23 * S[2]) / vol;
         sts[2] = (a13 * S[0] + a23 * S[1] + a33 * S[2]) / vol;
         double grad[3][19];
         face_gradient(face, tissue, grad);
         for (int k = 0; k < 19; ++k)
            for (int j = 0; j < 3; ++j) W[k] += sts[j] * grad[j][k] * hInv[j];
      }
      double a0 = 0;
      for (int k = 1; k < 19; ++k) a0 -= W[k];
      A[0] = a0;
      for (int k = 1; k < 19; ++k) A[k] = W[k];
   }
   free(tissueBlk);
   free(sigBlk);
}

op_sim_t* op_sim_create(int nx, int ny, int nz, double dx, double dy, double dz,
                        int64_t nCells, const int64_t* gid, const int* cellType,
                        const uint8_t* reaction, const double* sigma6,
                        int nParams, const op_params_t* params,
                        int nStim, const op_stim_t* stim,
                        double dt, double diffusionScale, int useDiffusion)
{
   op_sim_t* s = calloc(1, sizeof(op_sim_t));
   s->nx = nx; s->ny = ny; s->nz = nz;
   s->dx = dx; s->dy = dy; s->dz = dz;
   s->n = nCells;
   s->dt = dt; s->scale = diffusionScale; s->useDiffusion = useDiffusion;
   s->gid = malloc(nCells * sizeof(int64_t));
   memcpy(s->gid, gid, nCells * sizeof(int64_t));
   s->reaction = malloc(nCells);
   memcpy(s->reaction, reaction, nCells);
   s->nParams = nParams;
   s->params = malloc(nParams * sizeof(op_params_t));
   memcpy(s->params, params, nParams * sizeof(op_params_t));
   s->nStim = nStim;
   s->stim = malloc((nStim ? nStim : 1) * sizeof(op_stim_t));
   if (nStim) memcpy(s->stim, stim, nStim * sizeof(op_stim_t));

   /* bounding box of the cells plus one voxel (elec/DiffusionUtils.cc:19-66) */
   int xmin = 1 << 30, ymin = 1 << 30, zmin = 1 << 30, xmax = -1, ymax = -1, zmax = -1;
   for (int64_t i = 0; i < nCells; ++i) {
      int x = (int)(gid[i] % nx), y = (int)((gid[i] / nx) % ny), z = (int)(gid[i] / nx / ny);
      if (x < xmin) xmin = x; if (x > xmax) xmax = x;
      if (y < ymin) ymin = y; if (y > ymax) ymax = y;
      if (z < zmin) zmin = z; if (z > zmax) zmax = z;
   }
   s->bx = xmax - xmin + 3; s->by = ymax - ymin + 3; s->bz = zmax - zmin + 3;
   s->ox = xmin - 1; s->oy = ymin - 1; s->oz = zmin - 1;
   s->nBlock = (int64_t)s->bx * s->by * s->bz;
   for (int k = 0; k < 19; ++k)
      s->off[k] = kNode[k][2] + (long)s->bz * (kNode[k][1] + (long)s->by * kNode[k][0]);
   s->blockIndex = malloc(nCells * sizeof(int64_t));
   for (int64_t i = 0; i < nCells; ++i) {
      int x = (int)(gid[i] % nx), y = (int)((gid[i] / nx) % ny), z = (int)(gid[i] / nx / ny);
      s->blockIndex[i] = block_index(s, x, y, z);
   }
   s->vmBlock = calloc(s->nBlock, sizeof(double));
   s->A = calloc(nCells * 19, sizeof(double));
   build_weights(s, cellType, sigma6);

   s->vm = calloc(nCells, sizeof(double));
   s->dvmR = calloc(nCells, sizeof(double));
   s->dvmD = calloc(nCells, sizeof(double));
   s->iStim = calloc(nCells, sizeof(double));
   s->state = calloc(nCells * OP_NSTATE, sizeof(double));
   s->act = calloc(nCells, sizeof(double));
   s->activated = calloc(nCells, 1);
   for (int64_t i = 0; i < nCells; ++i) op_state_init(s->state + OP_NSTATE * i, s->vm + i);
   return s;
}

void op_sim_destroy(op_sim_t* s)
{
   if (!s) return;
   free(s->gid); free(s->reaction); free(s->params); free(s->stim);
   free(s->blockIndex); free(s->vmBlock); free(s->A);
   free(s->vm); free(s->dvmR); free(s->dvmD); free(s->iStim); free(s->state);
   free(s->act); free(s->activated);
   free(s);
}

/* PeriodicPulse::eval, elec/PeriodicPulse.cc:22-28. */
static double pulse_value(const op_stim_t* p, double time)
{
   double t = time - floor(time / p->period) * p->period;
   if (t >= p->phase && t < p->phase + p->duration) return p->amplitude;
   return 0.0;
}

void op_sim_step(op_sim_t* s, int nSteps)
{
   const int64_t n = s->n;
   for (int step = 0; step < nSteps; ++step) {
      memset(s->iStim, 0, n * sizeof(double));
      for (int k = 0; k < s->nStim; ++k) {
         const op_stim_t* p = &s->stim[k];
         if (!(s->time > p->t0 && s->time < p->tf)) continue;
         double value = pulse_value(p, s->time);
         if (value == 0) continue;
         for (int64_t i = 0; i < n; ++i) {
            int x = (int)(s->gid[i] % s->nx), y = (int)((s->gid[i] / s->nx) % s->ny),
                z = (int)(s->gid[i] / s->nx / s->ny);
            if (x > p->xMin && x < p->xMax && y > p->yMin && y < p->yMax && z > p->zMin && z < p->zMax)
               s->iStim[i] = p->mode ? s->iStim[i] + value : value;
         }
      }
      /* Cells are independent within each phase, so threading the loops
       * changes no result. */
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < n; ++i)
         s->dvmR[i] = op_tt06_step(&s->params[s->reaction[i]], s->dt, s->vm[i], s->state + OP_NSTATE * i);
      if (s->useDiffusion) {
         for (int64_t i = 0; i < n; ++i) s->vmBlock[s->blockIndex[i]] = s->vm[i];
#pragma omp parallel for schedule(static)
         for (int64_t i = 0; i < n; ++i) {
            const double* phi = s->vmBlock + s->blockIndex[i];
            const double* A = s->A + 19 * i;
            double tmp = A[0] * phi[0];
            for (int k = 1; k < 19; ++k) tmp += A[k] * phi[s->off[k]];
            s->dvmD[i] = tmp * s->scale;
         }
      }
      for (int64_t i = 0; i < n; ++i) s->vm[i] += s->dt * (s->dvmR[i] + s->dvmD[i] + s->iStim[i]);
      s->time += s->dt;
      for (int64_t i = 0; i < n; ++i) {
         if (s->activated[i]) continue;
         if (s->vm[i] > 0) { s->activated[i] = 1; s->act[i] = s->time; }
      }
   }
}

double op_sim_time(const op_sim_t* s) { return s->time; }
void op_sim_get_vm(const op_sim_t* s, double* out) { memcpy(out, s->vm, s->n * sizeof(double)); }
void op_sim_set_vm(op_sim_t* s, const double* in) { memcpy(s->vm, in, s->n * sizeof(double)); }

void op_sim_get_dvm(const op_sim_t* s, double* dVmR, double* dVmD, double* iStim)
{
   if (dVmR) memcpy(dVmR, s->dvmR, s->n * sizeof(double));
   if (dVmD) memcpy(dVmD, s->dvmD, s->n * sizeof(double));
   if (iStim) memcpy(iStim, s->iStim, s->n * sizeof(double));
}

void op_sim_get_state(const op_sim_t* s, int var, double* out)
{
   for (int64_t i = 0; i < s->n; ++i) out[i] = s->state[OP_NSTATE * i + var];
}

void op_sim_set_state(op_sim_t* s, int var, const double* in)
{
   for (int64_t i = 0; i < s->n; ++i) s->state[OP_NSTATE * i + var] = in[i];
}

void op_sim_get_activation(const op_sim_t* s, double* out)
{
   for (int64_t i = 0; i < s->n; ++i) out[i] = s->activated[i] ? s->act[i] : -1.0;
}

void op_sim_get_weights(const op_sim_t* s, double* out19)
{
   memcpy(out19, s->A, s->n * 19 * sizeof(double));
}
