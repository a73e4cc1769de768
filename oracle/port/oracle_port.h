/* CPU restatement of the monodomain hot path of LLNL/Cardioid, used as the
 * correctness oracle for the B200 engine.
 *
 * TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load it, as the checker; the product never links it.
 *
 * What it restates (reference paths are relative to the Cardioid checkout):
 *   - Interpolation::eval            elec/Interpolation.hh:11-99
 *   - BetterTT06 factory defaults    elec/BetterTT06.cc:69-121
 *   - BetterTT06 initial state       elec/BetterTT06.cc:1657-1712
 *   - BetterTT06 CPU calc (1 cell)   elec/BetterTT06.cc:1426-1649
 *   - FGR weights                    elec/FGRDiffusionOMP.cc:166-265, elec/FGRUtils.cc:10-148
 *   - FGR stencil                    elec/FGRDiffusionOMP.cc:109-131
 *   - Box/PointStimulus, PeriodicPulse elec/BoxStimulus.cc:11-70, elec/PointStimulus.cc:26-36,
 *                                    elec/PeriodicPulse.cc:22-28,
 *                                    elec/Stimulus.hh:21-27
 *   - omp-loop integrator            elec/simulationLoop.cc:183-231
 *   - activation-time sensor         elec/ActivationTimeSensor.cc:99-111
 * The arithmetic keeps the reference's operation order and is compiled with
 * -ffp-contract=off, so on x86-64 it reproduces the reference bit for bit.
 */
#ifndef ORACLE_PORT_H
#define ORACLE_PORT_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OP_NFIT 30
#define OP_NSTATE 18
#define OP_MAXCOEF 64

/* Fit slots, in the order of the reference's _interpolant[] array
 * (elec/BetterTT06.cc:35-66). */
enum op_fit {
   OPF_fCass_RLA, OPF_Xr1_RLA, OPF_Xr1_RLB, OPF_Xr2_RLA, OPF_Xr2_RLB, OPF_Xs_RLA, OPF_Xs_RLB,
   OPF_d_RLA, OPF_d_RLB, OPF_f2_RLA, OPF_f2_RLB, OPF_f_RLA, OPF_f_RLB, OPF_h_RLA, OPF_h_RLB,
   OPF_j_RLA, OPF_j_RLB, OPF_m_RLA, OPF_m_RLB, OPF_r_RLA, OPF_r_RLB, OPF_s_RLA, OPF_s_RLB,
   OPF_exp_gamma_VFRT, OPF_exp_gamma_m1_VFRT, OPF_i_CalTerm3, OPF_i_CalTerm4, OPF_i_NaK_term,
   OPF_i_p_K_term, OPF_i_K1
};

/* State slots, in checkpoint (alphabetical) order, which is also the
 * reference GPU kernel's SoA order (elec/BetterTT06.cc:1052-1073). */
enum op_state {
   OPS_Ca_SR, OPS_Ca_i, OPS_Ca_ss, OPS_K_i, OPS_Na_i, OPS_R_prime, OPS_Xr1, OPS_Xr2, OPS_Xs,
   OPS_d, OPS_f, OPS_f2, OPS_fCass, OPS_h, OPS_j, OPS_m, OPS_r, OPS_s
};

typedef struct {
   int numer, denom;            /* term counts; denom == 1 means a polynomial */
   double coeff[OP_MAXCOEF];    /* numer coefficients, then denom-1 coefficients */
} op_fit_t;

typedef struct {
   double celltype, g_CaL, g_K1, g_Kr, g_Ks, g_Na, g_bca, g_bna, g_pCa, g_pK, g_to;
   op_fit_t fit[OP_NFIT];
} op_params_t;

double op_fit_eval(const op_fit_t* f, double x);
void op_params_defaults(op_params_t* p, double celltype);
void op_state_init(double state[OP_NSTATE], double* Vm);
/* One BetterTT06 step of one cell: updates state in place, returns dVm = -Iion. */
double op_tt06_step(const op_params_t* p, double dt, double V, double state[OP_NSTATE]);

/* ---- tissue ---- */
typedef struct {
   double t0, tf;                       /* Stimulus on while t0 < time < tf */
   double period, duration, amplitude, phase;  /* PeriodicPulse */
   double xMin, xMax, yMin, yMax, zMin, zMax;  /* strict box on the global tuple */
   int mode;      /* 0: BoxStimulus assigns (elec/BoxStimulus.cc:56-64);
                     1: PointStimulus adds (elec/PointStimulus.cc:26-36) */
   int reserved;
} op_stim_t;

typedef struct op_sim op_sim_t;

/* Cells in local order with gid = x + nx*(y + ny*z).  reaction[i] selects
 * params[reaction[i]]; cellType[i] > 0 marks tissue for the FGR mask. */
op_sim_t* op_sim_create(int nx, int ny, int nz, double dx, double dy, double dz,
                        int64_t nCells, const int64_t* gid, const int* cellType,
                        const uint8_t* reaction, const double* sigma6,
                        int nParams, const op_params_t* params,
                        int nStim, const op_stim_t* stim,
                        double dt, double diffusionScale, int useDiffusion);
void op_sim_destroy(op_sim_t* s);
void op_sim_step(op_sim_t* s, int nSteps);
double op_sim_time(const op_sim_t* s);
void op_sim_get_vm(const op_sim_t* s, double* out);
void op_sim_set_vm(op_sim_t* s, const double* in);
void op_sim_get_dvm(const op_sim_t* s, double* dVmR, double* dVmD, double* iStim);
void op_sim_get_state(const op_sim_t* s, int var, double* out);
void op_sim_set_state(op_sim_t* s, int var, const double* in);
void op_sim_get_activation(const op_sim_t* s, double* out);
/* FGR weights of every cell: A0 then A[1..18] in NodeLocation order. */
void op_sim_get_weights(const op_sim_t* s, double* out19);

#ifdef __cplusplus
}
#endif
#endif
