/* BetterTT06 restated for one cell.  TEST INFRASTRUCTURE (see oracle_port.h).
 *
 * The operation order of every expression follows the reference CPU loop
 * (elec/BetterTT06.cc:1426-1649) as built with simdops at width 1, where
 * float64v converts implicitly to and from double, so arithmetic is the
 * built-in double arithmetic except where a long double literal promotes a
 * whole expression (the Ca_i and Ca_ss derivatives).
 */
#include "oracle_port.h"
#include <math.h>
#include <string.h>

/* Interpolation::eval: Horner numerator over (1 + x * Horner denominator),
 * elec/Interpolation.hh:11-99. */
double op_fit_eval(const op_fit_t* f, double x)
{
   const double* c = f->coeff;
   double num = c[f->numer - 1];
   for (int k = f->numer - 2; k >= 0; --k) num = c[k] + x * num;
   if (f->denom == 1) return num;
   const double* d = c + f->numer;
   double den = d[f->denom - 2];
   for (int k = f->denom - 3; k >= 0; --k) den = d[k] + x * den;
   den = 1 + x * den;
   return num / den;
}

/* reactionFactoryForBetterTT06 defaults, elec/BetterTT06.cc:86-121. */
void op_params_defaults(op_params_t* p, double celltype)
{
   memset(p, 0, sizeof(*p));
   p->celltype = celltype;
   p->g_CaL = 3.98000000000000e-5;
   p->g_bca = 0.000592000000000000;
   p->g_pCa = 0.123800000000000;
   p->g_Na = 14.8380000000000;
   p->g_K1 = 5.40500000000000;
   p->g_pK = 0.0146000000000000;
   p->g_Kr = 0.153000000000000;
   p->g_Ks = (celltype == 1) ? 0.0980000000000000 : 0.392000000000000;
   p->g_bna = 0.000290000000000000;
   p->g_to = (celltype == 0) ? 0.0730000000000000 : 0.294000000000000;
}

/* initializeMembraneVoltage, elec/BetterTT06.cc:1657-1712. */
void op_state_init(double s[OP_NSTATE], double* Vm)
{
   s[OPS_Ca_SR] = 3.15500000000000;
   s[OPS_Ca_i] = 2.00000000000000e-5;
   s[OPS_Ca_ss] = 0.000170000000000000;
   s[OPS_K_i] = 138.400000000000;
   s[OPS_Na_i] = 10.3550000000000;
   s[OPS_R_prime] = 0.986800000000000;
   s[OPS_Xr1] = 0.00448000000000000;
   s[OPS_Xr2] = 0.476000000000000;
   s[OPS_Xs] = 0.00870000000000000;
   s[OPS_d] = 3.16400000000000e-5;
   s[OPS_f] = 0.960900000000000;
   s[OPS_f2] = 0.977800000000000;
   s[OPS_fCass] = 0.995300000000000;
   s[OPS_h] = 0.550000000000000;
   s[OPS_j] = 0.660000000000000;
   s[OPS_m] = 0.00155000000000000;
   s[OPS_r] = 2.23500000000000e-8;
   s[OPS_s] = 0.601200000000000;
   if (Vm) *Vm = -83;
}

/* Model constants of the BetterTT06 calc (elec/BetterTT06.cc:1438-1474). */
static const double kCm = 0.185, kF = 96485.3415, kR = 8314.472, kT = 310;
static const double kVc = 0.016404, kFactorFix = 1, kCao = 2;
static const double kBufC = 0.2, kBufSr = 10, kBufSs = 0.4, kEC = 1.5;
static const double kKbufC = 0.001, kKbufSr = 0.3, kKbufSs = 0.00025, kKup = 0.00025;
static const double kVleak = 0.00036, kVrel = 0.102, kVsr = 0.001094, kVss = 5.468e-5;
static const double kVxfer = 0.0038, kVmaxUp = 0.006375;
static const double kK1p = 0.15, kK2p = 0.045, kK3 = 0.06, kK4 = 0.005, kMaxSr = 2.5, kMinSr = 1;
static const double kKpCa = 0.0005, kKNaCa = 1000, kKsat = 0.1, kKmCa = 1.38, kKmNai = 87.5;
static const double kAlpha = 2.5, kKo = 5.4, kPkna = 0.03, kNao = 140, kKmNa = 40;

double op_tt06_step(const op_params_t* p, double dt, double V, double st[OP_NSTATE])
{
   const op_fit_t* fit = p->fit;
   const double sqrtKo = sqrt(kKo);
   const double RT = kR * kT;
   double caSR = st[OPS_Ca_SR], caI = st[OPS_Ca_i], caSS = st[OPS_Ca_ss];
   double kI = st[OPS_K_i], naI = st[OPS_Na_i], rPrime = st[OPS_R_prime];

   /* gate coefficients */
   double fCassInf = 0.4 + 0.6 / (400.0 * (caSS * caSS) + 1);
   double aXr1 = op_fit_eval(&fit[OPF_Xr1_RLA], V), bXr1 = op_fit_eval(&fit[OPF_Xr1_RLB], V);
   double aXr2 = op_fit_eval(&fit[OPF_Xr2_RLA], V), bXr2 = op_fit_eval(&fit[OPF_Xr2_RLB], V);
   double aXs = op_fit_eval(&fit[OPF_Xs_RLA], V), bXs = op_fit_eval(&fit[OPF_Xs_RLB], V);
   double ad = op_fit_eval(&fit[OPF_d_RLA], V), bd = op_fit_eval(&fit[OPF_d_RLB], V);
   double af = op_fit_eval(&fit[OPF_f_RLA], V), bf = op_fit_eval(&fit[OPF_f_RLB], V);
   double af2 = op_fit_eval(&fit[OPF_f2_RLA], V), bf2 = op_fit_eval(&fit[OPF_f2_RLB], V);
   double aFc = op_fit_eval(&fit[OPF_fCass_RLA], caSS), bFc = -fCassInf;
   double ah = op_fit_eval(&fit[OPF_h_RLA], V), bh = op_fit_eval(&fit[OPF_h_RLB], V);
   double aj = op_fit_eval(&fit[OPF_j_RLA], V), bj = op_fit_eval(&fit[OPF_j_RLB], V);
   double am = op_fit_eval(&fit[OPF_m_RLA], V), bm = op_fit_eval(&fit[OPF_m_RLB], V);
   double ar = op_fit_eval(&fit[OPF_r_RLA], V), br = op_fit_eval(&fit[OPF_r_RLB], V);
   double as = op_fit_eval(&fit[OPF_s_RLA], V), bs = op_fit_eval(&fit[OPF_s_RLB], V);

   /* currents and fluxes */
   double calT3 = op_fit_eval(&fit[OPF_i_CalTerm3], V);
   double calT4 = op_fit_eval(&fit[OPF_i_CalTerm4], V);
   double eCa = 0.5 * kR * kT * log(kCao / caI) / kF;
   double iBCa = p->g_bca * (V - eCa);
   double iPCa = caI * p->g_pCa / (caI + kKpCa);
   double expG = op_fit_eval(&fit[OPF_exp_gamma_VFRT], V);
   double expGm1 = op_fit_eval(&fit[OPF_exp_gamma_m1_VFRT], V);
   double pKterm = op_fit_eval(&fit[OPF_i_p_K_term], V);
   double eK = RT * log(kKo / kI) / kF;
   double naKterm = op_fit_eval(&fit[OPF_i_NaK_term], V);
   double iNaK = naI * naKterm / (naI + kKmNa);
   double naFromNaK = 3 * iNaK;
   double kFromNaK = -2 * iNaK;
   double vEK = -eK + V;
   double bufC = (1.0 / (kBufC * kKbufC / ((caI + kKbufC) * (caI + kKbufC)) + 1));
   double bufSR = (1.0 / (kBufSr * kKbufSr / ((caSR + kKbufSr) * (caSR + kKbufSr)) + 1));
   double bufSS = (1.0 / (kBufSs * kKbufSs / ((caSS + kKbufSs) * (caSS + kKbufSs)) + 1));
   double iLeak = kVleak * (caSR - caI);
   double iUp = kVmaxUp / (1 + (kKup * kKup) / (caI * caI));
   double iXfer = kVxfer * (-caI + caSS);
   double kcasr = kMaxSr - (kMaxSr - kMinSr) / (1 + (kEC * kEC) / (caSR * caSR));
   double k1 = kK1p / kcasr;
   double k2 = kK2p * kcasr;
   double O = (caSS * caSS) * rPrime * k1 / ((caSS * caSS) * k1 + kK3);
   double dRprime = -caSS * rPrime * k2 + kK4 * (-rPrime + 1);
   double iRel = O * kVrel * (caSR - caSS);
   double dCaSR = bufSR * (-iLeak - iRel + iUp);
   double iCaL = st[OPS_d] * st[OPS_f] * st[OPS_f2] * st[OPS_fCass] * p->g_CaL *
                 (-kCao * calT3 + 0.25 * caSS * calT4);
   double iNaCa = kKNaCa * ((naI * naI * naI) * kCao * expG - (kNao * kNao * kNao) * caI * kAlpha * expGm1) /
                  (((kNao * kNao * kNao) + (kKmNai * kKmNai * kKmNai)) * (kCao + kKmCa) * (kKsat * expGm1 + 1));
   double naFromNaCa = 3 * iNaCa;
   double iK1 = op_fit_eval(&fit[OPF_i_K1], vEK);
   double iPK = vEK * p->g_pK * pKterm;
   double iKr = 0.430331482911935 * vEK * sqrtKo * st[OPS_Xr1] * st[OPS_Xr2] * p->g_Kr;
   double eNa = RT * log(kNao / naI) / kF;
   double eKs = RT * log((kKo + kNao * kPkna) / (kI + naI * kPkna)) / kF;
   double iKs = (st[OPS_Xs] * st[OPS_Xs]) * p->g_Ks * (V - eKs);
   double iBNa = p->g_bna * (-eNa + V);
   double iTo = vEK * p->g_to * st[OPS_r] * st[OPS_s];
   double kTot = kFromNaK + iK1 + iPK + iKr + iKs + iTo;
   /* The reference writes these two with a long double factor -1.0L/2.0L;
    * under the simdops width-1 build float64v converts to double, so the
    * whole bracket and its product with the buffer factor are evaluated in
    * long double and rounded once on assignment. */
   const long double halfCm = -1.0L / 2.0L * kCm;
   double dCaI = bufC * (halfCm * (-2 * iNaCa + iBCa + iPCa) / (kF * kVc) + iXfer + kVsr * (iLeak - iUp) / kVc);
   double dCaSS = bufSS * (halfCm * iCaL / (kF * kVss) - kVc * iXfer / kVss + kVsr * iRel / kVss);
   double m = st[OPS_m];
   double iNa = (m * m * m) * p->g_Na * st[OPS_h] * st[OPS_j] * (-eNa + V);
   double dKi = -kCm * kFactorFix * kTot / (kF * kVc);
   double naTot = iNa + naFromNaK + iBNa + naFromNaCa;
   double dNai = -kCm * kFactorFix * naTot / (kF * kVc);
   double caTot = iCaL + iPCa + iBCa + -2 * iNaCa;
   double iIon = caTot + kTot + naTot;

   /* forward Euler on the concentrations, Rush-Larsen on the gates */
   st[OPS_Ca_SR] = caSR + dt * dCaSR;
   st[OPS_Ca_i] = caI + dt * dCaI;
   st[OPS_Ca_ss] = caSS + dt * dCaSS;
   st[OPS_K_i] = kI + dt * dKi;
   st[OPS_Na_i] = naI + dt * dNai;
   st[OPS_R_prime] = rPrime + dt * dRprime;
#define RL(slot, a, b) st[slot] += a * (st[slot] + b)
   RL(OPS_Xr1, aXr1, bXr1);
   RL(OPS_Xr2, aXr2, bXr2);
   RL(OPS_Xs, aXs, bXs);
   RL(OPS_d, ad, bd);
   RL(OPS_f, af, bf);
   RL(OPS_f2, af2, bf2);
   RL(OPS_fCass, aFc, bFc);
   RL(OPS_h, ah, bh);
   RL(OPS_j, aj, bj);
   RL(OPS_m, am, bm);
   RL(OPS_r, ar, br);
   RL(OPS_s, as, bs);
#undef RL
   return -iIon;
}
