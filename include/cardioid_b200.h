/*
 * cardioid_b200 — C ABI of the B200 engine for Cardioid's monodomain hot path.
 *
 * Plain pointers and sizes only; every call returns a cdb_status and never
 * throws or aborts.  cdb_last_error() gives the message of the calling
 * thread's last failure.  Pointers documented as "device" are CUDA device
 * pointers on the engine's device; all others are host pointers.
 *
 * Three groups of entry points, each standing in for one reference
 * interface (paths are relative to the LLNL/Cardioid checkout):
 *
 *   cdb_reaction_*  — the Reaction plugin (elec/Reaction.hh:10-40) for
 *                     BetterTT06 (elec/BetterTT06.hh, elec/BetterTT06.cc).
 *   cdb_fgr_*       — the Diffusion plugin (elec/Diffusion.hh:19-39) for the
 *                     FGR stencil (elec/FGRDiffusionOMP.hh/.cc).
 *   cdb_engine_*    — the omp time loop (elec/simulationLoop.cc:150-243) with
 *                     reaction, diffusion, box stimuli, integrator and the
 *                     activation/min-max sensors fused into one kernel per
 *                     step, over one or many tissues.
 */
#ifndef CARDIOID_B200_H
#define CARDIOID_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  CDB_OK = 0,
  CDB_INVALID_ARG = 1,   /* a size, index, key or pointer the call cannot accept */
  CDB_OOM = 2,           /* device memory could not be allocated */
  CDB_CUDA_ERROR = 3,    /* a CUDA runtime call or kernel launch failed */
  CDB_NUMERIC_FAULT = 4, /* a non-finite Vm was detected */
  CDB_TIMEOUT = 5,       /* a bounded device wait gave up */
  CDB_NOT_FOUND = 6,     /* no tissue or reaction with that id */
  CDB_BOUNDS_FAULT = 7   /* the bounds-checked build found an index out of range */
} cdb_status;

typedef enum { CDB_FP64 = 0, CDB_MIXED = 1 } cdb_precision;

#define CDB_NUM_FITS 30
#define CDB_NUM_STATES 18
#define CDB_MAX_COEFF 64
#define CDB_MAX_REACTION_TYPES 6
#define CDB_MAX_STIM_PER_TISSUE 32

/* One rational fit in the reference's FUNCTION-object form
 * (elec/Interpolation.hh:11-99): numer numerator coefficients then denom-1
 * denominator coefficients, monomial, denominator constant 1. */
typedef struct {
  int32_t numer;
  int32_t denom;
  double coeff[CDB_MAX_COEFF];
} cdb_fit;

/* Scalar parameters of one BetterTT06 REACTION object
 * (reactionFactoryForBetterTT06, elec/BetterTT06.cc:69-121). */
typedef struct {
  double celltype, g_CaL, g_K1, g_Kr, g_Ks, g_Na, g_bca, g_bna, g_pCa, g_pK, g_to;
} cdb_tt06_params;

/* A stimulus with a PeriodicPulse (elec/PeriodicPulse.cc:22-28,
 * elec/Stimulus.hh:21-27): on while t0 < time < tf and
 * phase <= time mod period < phase + duration, for the cells with
 * xMin < x < xMax, yMin < y < yMax, zMin < z < zMax.  Stimuli apply in list
 * order to iStim, which starts each step at 0:
 *   mode CDB_STIM_BOX   — BoxStimulus (elec/BoxStimulus.cc:11-70): iStim =
 *                         amplitude (= -vStim), overwriting earlier stimuli;
 *   mode CDB_STIM_POINT — PointStimulus (elec/PointStimulus.cc:26-36):
 *                         iStim += amplitude; its box is (x-1, x+1) x
 *                         (y-1, y+1) x (z-1, z+1) around the target cell. */
#define CDB_STIM_BOX 0
#define CDB_STIM_POINT 1
typedef struct {
  double t0, tf, period, duration, amplitude, phase;
  double xMin, xMax, yMin, yMax, zMin, zMax;
  int32_t mode;
  int32_t reserved;   /* 0 */
} cdb_stimulus;

/* ------------------------------------------------------------------ */
/* Library                                                              */
/* ------------------------------------------------------------------ */
const char* cdb_last_error(void);
const char* cdb_version(void);
/* Evaluates one fit on the host (Interpolation::eval). */
double cdb_fit_eval(const cdb_fit* fit, double x);

/* ------------------------------------------------------------------ */
/* Reaction plugin: BetterTT06 on the device.                           */
/* Replaces BetterTT06::ThisReaction (elec/BetterTT06.hh:49-112):       */
/*   constructor + reactionFactoryForBetterTT06   -> cdb_reaction_create */
/*   initializeMembraneVoltage (BetterTT06.cc:1657) -> cdb_reaction_init */
/*   calc (Reaction.hh:15-19, BetterTT06.cc:1320)   -> cdb_reaction_calc */
/*   getValue / setValue (BetterTT06.cc:1860-2210)  -> cdb_reaction_{get,set}_state */
/* ------------------------------------------------------------------ */
typedef struct cdb_reaction cdb_reaction;

/* A reaction whose fits have the compiled shapes (the shipped fit files'
 * term counts or fewer) runs the unrolled kernel of one of the device's
 * CDB_MAX_REACTION_TYPES constant-memory slots, which engines and plugin
 * reactions share (identical parameters and fits share one slot); other fit
 * sets, or a reaction created when every slot is taken, run the generic
 * kernel.  Both compute the same model; the slot kernel is faster. */

cdb_status cdb_reaction_create(int device, cdb_precision precision, const cdb_tt06_params* params,
                               const cdb_fit fits[CDB_NUM_FITS], int64_t nCells, double dt,
                               cdb_reaction** out);
/* indexArray (device, int32[nCells]) lists this reaction's cells in the
 * caller's Vm array; Vm (device) gets V_init at those positions. */
cdb_status cdb_reaction_init(cdb_reaction* r, const int32_t* indexArray, double* Vm, void* stream);
/* dVm[indexArray[i]] = -Iion(Vm[indexArray[i]], state_i); state advanced
 * by dt.  iStim is accepted and unused, as in the reference.  All device
 * pointers; stream is a cudaStream_t (NULL = default stream).  A reaction
 * created with nCells = 0 (a REACTION whose cellTypes the tissue lacks, as
 * ReactionManager::create can make) returns CDB_OK from init and calc
 * without touching its arrays, which may then be NULL. */
cdb_status cdb_reaction_calc(cdb_reaction* r, double dt, const int32_t* indexArray, const double* Vm,
                             const double* iStim, double* dVm, void* stream);
/* var in checkpoint order (Ca_SR Ca_i Ca_ss K_i Na_i R_prime Xr1 Xr2 Xs d f
 * f2 fCass h j m r s); host arrays of nCells doubles. */
cdb_status cdb_reaction_get_state(cdb_reaction* r, int var, double* host);
cdb_status cdb_reaction_set_state(cdb_reaction* r, int var, const double* host);
cdb_status cdb_reaction_destroy(cdb_reaction* r);

/* ------------------------------------------------------------------ */
/* Diffusion plugin: FGR 19-point stencil on the device.                */
/* Replaces FGRDiffusionOMP (elec/FGRDiffusionOMP.hh:13-44):            */
/*   constructor + precomputeCoefficients    -> cdb_fgr_create          */
/*   updateLocalVoltage (FGRDiffusionOMP.cc:75) -> cdb_fgr_update_local_voltage */
/*   calc (FGRDiffusionOMP.cc:109, assigns dVm) -> cdb_fgr_calc         */
/* ------------------------------------------------------------------ */
typedef struct cdb_fgr cdb_fgr;

/* Cells (host arrays) in local order: gid = x + nx*(y + ny*z) on the
 * nx*ny*nz grid, anatomy cellType (> 0 is tissue) and the conductivity
 * tensor as a11 a12 a13 a22 a23 a33 (S/mm); spacing in mm;
 * diffusionScale in mm^3/mF. */
cdb_status cdb_fgr_create(int device, int32_t nx, int32_t ny, int32_t nz, double dx, double dy, double dz,
                          int64_t nCells, const int64_t* gid, const int32_t* cellType, const double* sigma6,
                          double diffusionScale, cdb_fgr** out);
cdb_status cdb_fgr_update_local_voltage(cdb_fgr* d, const double* Vm, void* stream);
cdb_status cdb_fgr_calc(cdb_fgr* d, double* dVm, void* stream);
/* The weights the stencil uses (host, nCells x 19: A0 then A[1..18] in the
 * reference's NodeLocation order). */
cdb_status cdb_fgr_get_weights(cdb_fgr* d, double* host19);
cdb_status cdb_fgr_destroy(cdb_fgr* d);

/* ------------------------------------------------------------------ */
/* Diffusion plugin: the reference's "cuda" 6-face stencil.             */
/* Replaces CUDADiffusion (elec/CUDADiffusion.cc:30-160, kernel         */
/* diff_6face_v1, elec/CUDADiffusion_ker.cu:16-140) for users of        */
/* method = cuda: each face carries the conductivity of the cell on its */
/* + side (sigma area / h diffusionScale / volume), tangential terms    */
/* only when their four nodes exist; dVm = sum of face flux             */
/* differences (assigned).  Same cell and grid arguments as             */
/* cdb_fgr_create; every given cell is present (cellType not checked,   */
/* as in the reference).  cdb_diff6_get_face_sigma: host nCells x 9,    */
/* the - face of axis i, component j at [9 c + 3 i + j].                */
/* ------------------------------------------------------------------ */
typedef struct cdb_diff6 cdb_diff6;
cdb_status cdb_diff6_create(int device, int32_t nx, int32_t ny, int32_t nz, double dx, double dy, double dz,
                            int64_t nCells, const int64_t* gid, const double* sigma6, double diffusionScale,
                            cdb_diff6** out);
cdb_status cdb_diff6_update_local_voltage(cdb_diff6* d, const double* Vm, void* stream);
cdb_status cdb_diff6_calc(cdb_diff6* d, double* dVm, void* stream);
cdb_status cdb_diff6_get_face_sigma(cdb_diff6* d, double* host9);
cdb_status cdb_diff6_destroy(cdb_diff6* d);

/* The FGR stencil for callers that cannot allocate device memory (code
 * inside another framework's allocator, or measurement code that must leave
 * the allocation state unchanged).  No counterpart in the reference.
 * dVm[i] = diffusionScale (A0 phi0 + sum_k A_k phi_k) on a full nx*ny*nz box
 * in gid order (x fastest); weights19 (device) is 19 rows of nCells doubles,
 * row 0 = A0 and rows 1..18 = A[1..18] in NodeLocation order (the rows of
 * cdb_fgr_get_weights, transposed); Vm and dVm are device arrays of nCells.
 * The padded Vm block lives in a static device array of 16 MiB
 * ((nx+2)(ny+2)(nz+2) <= 2,097,152 voxels, e.g. 126^3); larger boxes are
 * rejected with CDB_INVALID_ARG.  The call allocates nothing: no cudaMalloc,
 * no cudaFree.  Its first call on a device looks up that array's device
 * address (cudaGetSymbolAddress); make that first call before any stream
 * capture, and do not cudaDeviceReset that device afterwards (the address
 * is kept for the life of the process).  Every call shares the one array
 * and clears it first; calls that overlap on the GPU (other streams, other
 * threads) race on it.  The calling thread's current device is the same on
 * return as on entry. */
cdb_status cdb_fgr_calc_static(int device, int32_t nx, int32_t ny, int32_t nz, const double* weights19,
                               const double* Vm, double* dVm, double diffusionScale, void* stream);

/* ------------------------------------------------------------------ */
/* Fused engine                                                          */
/* ------------------------------------------------------------------ */
typedef struct cdb_engine cdb_engine;

typedef struct {
  int device;
  cdb_precision precision;
  double dt;               /* ms */
  int use_graphs;          /* capture step batches as CUDA graphs */
} cdb_engine_config;

typedef struct {
  int32_t nx, ny, nz;          /* grid; gid = x + nx*(y + ny*z) */
  double dx, dy, dz;           /* mm */
  int64_t nCells;
  const int64_t* gid;          /* NULL: all nx*ny*nz cells in gid order */
  const int32_t* cellType;     /* anatomy cellType per cell, > 0 */
  const uint8_t* reaction;     /* reaction-type id per cell */
  const double* sigma6;        /* nCells x 6 */
  const double* vm0;           /* initial Vm per cell; NULL: V_init */
  double diffusionScale;       /* mm^3/mF; 0 disables diffusion */
  float g_Kr_scale, g_CaL_scale, g_Na_scale;   /* drug block multipliers (1 = none) */
  int32_t nStim;
  const cdb_stimulus* stim;
} cdb_tissue_desc;

cdb_status cdb_engine_create(const cdb_engine_config* cfg, cdb_engine** out);
cdb_status cdb_engine_destroy(cdb_engine* e);
/* Registers a BetterTT06 parameter set; *id is used in cdb_tissue_desc.reaction. */
cdb_status cdb_engine_add_reaction(cdb_engine* e, const cdb_tt06_params* params,
                                   const cdb_fit fits[CDB_NUM_FITS], int32_t* id);
/* Device bytes a tissue would take (for admission by free memory). */
cdb_status cdb_engine_tissue_bytes(cdb_engine* e, const cdb_tissue_desc* t, int64_t* bytes);
cdb_status cdb_engine_free_bytes(cdb_engine* e, int64_t* free_bytes, int64_t* total_bytes);
/* Adds a tissue between steps; its time starts at 0. */
cdb_status cdb_engine_add_tissue(cdb_engine* e, const cdb_tissue_desc* t, int32_t* id);
cdb_status cdb_engine_remove_tissue(cdb_engine* e, int32_t id);
/* Advances every tissue by nSteps steps of dt (one fused kernel per step). */
cdb_status cdb_engine_step(cdb_engine* e, int32_t nSteps);
/* Blocks until the engine's stream is idle; CDB_TIMEOUT if a bounded wait
 * inside the step gave up since the last call (the affected steps are
 * incomplete); CDB_NUMERIC_FAULT if a cell's Vm was NaN or infinite at the
 * end of a launch batch of cdb_engine_step (checked with the min/max
 * sensor, on each batch's last step). */
cdb_status cdb_engine_sync(cdb_engine* e);
/* Test of the failure path (no counterpart in the reference): the next
 * cdb_engine_step batch runs with bulk-copy staging and issues no copies
 * after each warp's first tile, so those warps' bounded waits (about a
 * second each) run out, the batch is left incomplete and cdb_engine_sync
 * returns CDB_TIMEOUT; nothing faults, and later batches run normally. */
cdb_status cdb_engine_test_bounded_wait(cdb_engine* e);
/* Number of steps a tissue has taken and its time (ms, accumulated as
 * time += dt like the reference). */
cdb_status cdb_engine_tissue_time(cdb_engine* e, int32_t id, int64_t* steps, double* time);
/* Sets a tissue's step count and time, as a restart does (the SIMULATE
 * object's loop and time, written by writeRestart, elec/checkpointIO.cc:
 * 104-117, and the checkpoint header): later steps continue time += dt from
 * `time`.  Vm and state are unchanged (cdb_engine_write_vm/_write_state). */
cdb_status cdb_engine_set_clock(cdb_engine* e, int32_t id, int64_t loop, double time);
/* The ECG pseudo-sensor fused into the step (ECGSensor, elec/ECGSensor.cc:
 * 20-320, elec/ECGSensor.cu:9-168): every evalRate steps, electrode j
 * (xyz[3j..3j+2], mm) records kconst dx dy dz sum over cells of
 * dVmD / |r - p_j|, r = (x dx, y dy, z dz) from the cell's gid.  At most 32
 * electrodes; nPoints = 0 turns it off.  The device keeps the last 1023
 * evaluations; cdb_engine_read_ecg hands out those not read yet (oldest
 * first): loops[k] is the step count of evaluation k and values[k*nPoints+j]
 * its electrode j. */
cdb_status cdb_engine_set_ecg(cdb_engine* e, int32_t id, int32_t nPoints, const double* xyz, int32_t evalRate,
                              double kconst);
cdb_status cdb_engine_read_ecg(cdb_engine* e, int32_t id, int64_t maxEntries, int64_t* nEntries, int64_t* loops,
                               double* values);
/* Host copies, cell order of the tissue. */
cdb_status cdb_engine_read_vm(cdb_engine* e, int32_t id, double* host);
cdb_status cdb_engine_write_vm(cdb_engine* e, int32_t id, const double* host);
cdb_status cdb_engine_read_state(cdb_engine* e, int32_t id, int var, double* host);
cdb_status cdb_engine_write_state(cdb_engine* e, int32_t id, int var, const double* host);
/* First post-step time with Vm > 0 per cell, -1 if never
 * (ActivationTimeSensor::eval, elec/ActivationTimeSensor.cc:99-111). */
cdb_status cdb_engine_read_activation(cdb_engine* e, int32_t id, double* host);
/* min/max Vm of a tissue after the last step (MinMaxSensor, elec/MinMaxSensor.cc:44-67). */
cdb_status cdb_engine_minmax(cdb_engine* e, int32_t id, double* vmin, double* vmax);
/* Weights of a tissue (host, nCells x 19, A0 then A[1..18]), as built. */
cdb_status cdb_engine_read_weights(cdb_engine* e, int32_t id, double* host19);
/* One step through host buffers: copies vm_in (host) to the device, takes
 * one fused step of the tissue and copies the new Vm to vm_out (host).
 * The reaction state stays on the device, as a Reaction object keeps its
 * own state; this is the per-step cost a caller that owns Vm on the host
 * pays.  The engine must hold only this tissue.  When its cells are in grid
 * order (non-decreasing gid) and it has at least 32 planes along its
 * slowest axis and 65536 cells, the step runs in chunks of planes so the
 * upload, the step and the download overlap (both copy directions need
 * page-locked host buffers to overlap; with page-locked buffers the chunked
 * step is captured once per (vm_in, vm_out, Vm parity) as a CUDA graph and
 * replayed); vm_in and vm_out may be the same buffer. */
cdb_status cdb_engine_step_host(cdb_engine* e, int32_t id, const double* vm_in, double* vm_out);
/* ------------------------------------------------------------------ */
/* Diagnostics                                                           */
/* ------------------------------------------------------------------ */
/* q[i] = a[i] / b[i] (device arrays) computed with the engine's branch-free
 * FP64 quotient (Newton-refined reciprocal with a residual correction), for
 * measuring it against IEEE division.  No counterpart in the reference. */
cdb_status cdb_diag_div64(int device, int64_t n, const double* a, const double* b, double* q, void* stream);

/* The fit forms the compiled mixed kernels evaluate (host only, no device
 * needed): *compiled = 1 when the 30 fits run the compiled (unrolled)
 * kernels, else 0 (the generic kernel); when compiled, pool32[0..poolSize)
 * receives their FP32 coefficient pool (the compiled offsets; shifted fits
 * rewritten in t = (x - shift) / scale), and shift[30] / *scale the
 * shift of each fit (0 when it is evaluated as written).  No counterpart in
 * the reference. */
cdb_status cdb_diag_fit_forms(const cdb_fit fits[CDB_NUM_FITS], int32_t poolSize, float* pool32, float* shift,
                              float* scale, int32_t* compiled);

/* Launch tuning of the step kernel (no counterpart in the reference):
 * stage 1 = each warp copies its next tile's state (mixed: and weights)
 * into shared memory with cp.async while it computes the current one, 2 =
 * the same with bulk (TMA) copies completing on an mbarrier, 3 = stage 2
 * plus the Vm tile and halo of every row tile (32 consecutive voxels of one
 * x-row of a volume tissue with even padded strides): its nine stencil rows
 * are loaded into shared memory by one TMA tensor copy while the reaction
 * computes and the stencil reads them there (a reaction type's launches run
 * as stage 2 when fewer than half of its tiles are row tiles), 0 = direct
 * loads; ctasPerSm sizes the
 * persistent grid (SMs x ctasPerSm CTAs of 128 threads), 0 = as many CTAs as
 * are resident on an SM at once.  All stages give the same results bit for
 * bit.  Defaults: stage 2 for CDB_MIXED, 0 for CDB_FP64, ctasPerSm 0;
 * cardioid_b200.autotune picks them by timing. */
cdb_status cdb_engine_set_tuning(cdb_engine* e, int32_t stage, int32_t ctasPerSm);
cdb_status cdb_engine_get_tuning(cdb_engine* e, int32_t* stage, int32_t* ctasPerSm);

/* Warp-tile layout of the tissues added after the call (no counterpart in
 * the reference): CDB_LAYOUT_CELLS fills each reaction type's 32-slot
 * blocks with its cells in cell order; CDB_LAYOUT_ROWS (default) cuts every
 * x-row run of a type into whole 32-cell row tiles (stage 3 stages their
 * Vm tile and halo) and packs the runs' remainders into shared blocks.  Same
 * results bit for bit; cardioid_b200.autotune picks it by timing. */
#define CDB_LAYOUT_CELLS 0
#define CDB_LAYOUT_ROWS 1
cdb_status cdb_engine_set_layout(cdb_engine* e, int32_t layout);
cdb_status cdb_engine_get_layout(cdb_engine* e, int32_t* layout);

/* Kernels launched by this engine since creation. */
cdb_status cdb_engine_launch_count(cdb_engine* e, int64_t* launches);
/* The CUDA stream (cudaStream_t) the engine launches on. */
cdb_status cdb_engine_stream(cdb_engine* e, void** stream);

#ifdef __cplusplus
}
#endif
#endif
