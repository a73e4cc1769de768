// BetterTT06 ionic update of one cell on the device.
//
// Model: elec/BetterTT06.cc (LLNL/Cardioid) — CPU calc :1426-1649, the same
// equations as the reference's NVRTC kernel :1075-1298.  Per cell and step:
// 30 rational fits (Interpolation::eval, elec/Interpolation.hh:11-99), the
// currents, forward Euler on Ca_SR, Ca_i, Ca_ss, K_i, Na_i, R_prime and
// Rush-Larsen (X += a*(X + b)) on 12 gates; returns dVm = -Iion.
//
// Two precisions:
//   tt06_step        FP64; every operation in double, expressions in the
//                    reference's order (the compiler contracts a*b+c into an
//                    FMA, which only changes last bits).
//   tt06_step_mixed  fits, gates, currents and R_prime in FP32; Vm and the
//                    five concentrations in FP64 (their per-step increments
//                    are ~1e-7 of their values); the few fits whose monomial
//                    form loses accuracy in FP32 are evaluated in FP64.
// Fit evaluation is a policy: GenericFits reads term counts at run time;
// SpecFits has them as compile-time constants (fit_shapes.h), so every
// Horner chain unrolls and the 30 independent chains interleave.
#pragma once
#include <cstdint>

#include "fit_shapes.h"

namespace cdb {

constexpr int kNumFits = 30;
constexpr int kNumStates = 18;
constexpr int kMaxCoeff = 64;        // per fit (numer + denom - 1 <= 63)
constexpr int kMaxReactionTypes = 8;

// Fit slots, in the order of the reference's _interpolant[] (elec/BetterTT06.cc:35-66).
enum FitSlot {
  F_fCass_a, F_Xr1_a, F_Xr1_b, F_Xr2_a, F_Xr2_b, F_Xs_a, F_Xs_b, F_d_a, F_d_b, F_f2_a, F_f2_b,
  F_f_a, F_f_b, F_h_a, F_h_b, F_j_a, F_j_b, F_m_a, F_m_b, F_r_a, F_r_b, F_s_a, F_s_b,
  F_expG, F_expGm1, F_CalT3, F_CalT4, F_NaKterm, F_pKterm, F_K1
};

// State slots in checkpoint order (also the SoA order).
enum StateSlot {
  S_Ca_SR, S_Ca_i, S_Ca_ss, S_K_i, S_Na_i, S_R_prime, S_Xr1, S_Xr2, S_Xs, S_d, S_f, S_f2,
  S_fCass, S_h, S_j, S_m, S_r, S_s
};

// Scalar parameters of one reaction type (REACTION object).
struct TT06Scalars {
  double celltype, g_CaL, g_K1, g_Kr, g_Ks, g_Na, g_bca, g_bna, g_pCa, g_pK, g_to;
};

// Shape of the 30 fits of one reaction type: term counts and the offset of
// each fit's coefficients inside the type's coefficient pool.
struct FitShape {
  int16_t numer[kNumFits];
  int16_t denom[kNumFits];
  int16_t offset[kNumFits];
  // Fits the mixed path evaluates in FP64: those whose monomial Horner form
  // loses more than 1e-5 of their range in FP32 (set at registration).
  uint32_t fp64mask;
};

// Per-tissue multipliers of the unfitted conductances (drug block).
struct BlockScale {
  float g_Kr, g_CaL, g_Na;
};

// Horner numerator over (1 + x * Horner denominator); the monomial form
// of the FIT files (elec/Interpolation.hh:11-99).
template <typename Real>
__device__ __forceinline__ Real fit_eval(const Real* __restrict__ c, int numer, int denom, Real x)
{
  Real num = c[numer - 1];
#pragma unroll 2
  for (int k = numer - 2; k >= 0; --k) num = c[k] + x * num;
  if (denom == 1) return num;
  const Real* d = c + numer;
  Real den = d[denom - 2];
#pragma unroll 2
  for (int k = denom - 3; k >= 0; --k) den = d[k] + x * den;
  den = Real(1) + x * den;
  return num / den;
}

__device__ __forceinline__ float fit_eval_fast(const float* __restrict__ c, int numer, int denom, float x)
{
  float num = c[numer - 1];
#pragma unroll 2
  for (int k = numer - 2; k >= 0; --k) num = fmaf(x, num, c[k]);
  if (denom == 1) return num;
  const float* d = c + numer;
  float den = d[denom - 2];
#pragma unroll 2
  for (int k = denom - 3; k >= 0; --k) den = fmaf(x, den, d[k]);
  den = fmaf(x, den, 1.0f);
  return __fdividef(num, den);
}

// The same with compile-time term counts and offsets (fully unrolled).
template <int SLOT>
__device__ __forceinline__ double fit_spec64(const double* __restrict__ c, double x)
{
  constexpr int N = kSpecNumer[SLOT], D = kSpecDenom[SLOT], O = kSpecOffset[SLOT];
  double num = c[O + N - 1];
#pragma unroll
  for (int k = N - 2; k >= 0; --k) num = c[O + k] + x * num;
  if (D == 1) return num;
  double den = c[O + N + D - 2];
#pragma unroll
  for (int k = D - 3; k >= 0; --k) den = c[O + N + k] + x * den;
  den = 1.0 + x * den;
  return num / den;
}

template <int SLOT>
__device__ __forceinline__ float fit_spec32(const float* __restrict__ c, float x)
{
  constexpr int N = kSpecNumer[SLOT], D = kSpecDenom[SLOT], O = kSpecOffset[SLOT];
  float num = c[O + N - 1];
#pragma unroll
  for (int k = N - 2; k >= 0; --k) num = fmaf(x, num, c[O + k]);
  if (D == 1) return num;
  float den = c[O + N + D - 2];
#pragma unroll
  for (int k = D - 3; k >= 0; --k) den = fmaf(x, den, c[O + N + k]);
  den = fmaf(x, den, 1.0f);
  return __fdividef(num, den);
}

// Fit evaluation policies.  c64 / c32 point at one reaction type's
// coefficient pool (FP64 and FP32 copies).
struct GenericFits {
  const double* __restrict__ c64;
  const float* __restrict__ c32;
  const FitShape* sh;
  template <int SLOT>
  __device__ __forceinline__ double f64(double x) const
  {
    return fit_eval<double>(c64 + sh->offset[SLOT], sh->numer[SLOT], sh->denom[SLOT], x);
  }
  template <int SLOT>
  __device__ __forceinline__ float fmix(float xf, double xd) const
  {
    if ((sh->fp64mask >> SLOT) & 1u) return (float)f64<SLOT>(xd);
    return fit_eval_fast(c32 + sh->offset[SLOT], sh->numer[SLOT], sh->denom[SLOT], xf);
  }
};

struct SpecFits {
  const double* __restrict__ c64;
  const float* __restrict__ c32;
  template <int SLOT>
  __device__ __forceinline__ double f64(double x) const { return fit_spec64<SLOT>(c64, x); }
  template <int SLOT>
  __device__ __forceinline__ float fmix(float xf, double xd) const
  {
    if ((kSpecFp64Mask >> SLOT) & 1u) return (float)fit_spec64<SLOT>(c64, xd);
    return fit_spec32<SLOT>(c32, xf);
  }
};

// The state vector of one cell: concentrations in double, the other 13 in Real.
template <typename Real>
struct CellState {
  double caSR, caI, caSS, kI, naI;
  Real rPrime, Xr1, Xr2, Xs, d, f, f2, fCass, h, j, m, r, s;
};

struct ConstsD {
  static constexpr double Cm = 0.185, F = 96485.3415, R = 8314.472, T = 310;
  static constexpr double Vc = 0.016404, Cao = 2, BufC = 0.2, BufSr = 10, BufSs = 0.4, EC = 1.5;
  static constexpr double KbufC = 0.001, KbufSr = 0.3, KbufSs = 0.00025, Kup = 0.00025;
  static constexpr double Vleak = 0.00036, Vrel = 0.102, Vsr = 0.001094, Vss = 5.468e-5;
  static constexpr double Vxfer = 0.0038, VmaxUp = 0.006375, K1p = 0.15, K2p = 0.045, K3 = 0.06;
  static constexpr double K4 = 0.005, MaxSr = 2.5, MinSr = 1, KpCa = 0.0005, KNaCa = 1000;
  static constexpr double Ksat = 0.1, KmCa = 1.38, KmNai = 87.5, Alpha = 2.5, Ko = 5.4;
  static constexpr double Pkna = 0.03, Nao = 140, KmNa = 40;
};

// FP64 step, the reference's expression order.
template <class Fits>
__device__ __forceinline__ double tt06_step(const TT06Scalars& p, const BlockScale& blk, const Fits& fits,
                                            double dt, double V, CellState<double>& st)
{
  using C = ConstsD;
#define FIT(slot, x) fits.template f64<slot>(x)
  const double gKr = p.g_Kr * (double)blk.g_Kr, gCaL = p.g_CaL * (double)blk.g_CaL, gNa = p.g_Na * (double)blk.g_Na;
  const double sqrtKo = 2.32379000772445;   // sqrt(5.4) in double
  const double RT = C::R * C::T;
  const double caSR = st.caSR, caI = st.caI, caSS = st.caSS, kI = st.kI, naI = st.naI, rPrime = st.rPrime;

  const double fCassInf = 0.4 + 0.6 / (400.0 * (caSS * caSS) + 1);
  const double aXr1 = FIT(F_Xr1_a, V), bXr1 = FIT(F_Xr1_b, V);
  const double aXr2 = FIT(F_Xr2_a, V), bXr2 = FIT(F_Xr2_b, V);
  const double aXs = FIT(F_Xs_a, V), bXs = FIT(F_Xs_b, V);
  const double ad = FIT(F_d_a, V), bd = FIT(F_d_b, V);
  const double af = FIT(F_f_a, V), bf = FIT(F_f_b, V);
  const double af2 = FIT(F_f2_a, V), bf2 = FIT(F_f2_b, V);
  const double aFc = FIT(F_fCass_a, caSS), bFc = -fCassInf;
  const double ah = FIT(F_h_a, V), bh = FIT(F_h_b, V);
  const double aj = FIT(F_j_a, V), bj = FIT(F_j_b, V);
  const double am = FIT(F_m_a, V), bm = FIT(F_m_b, V);
  const double ar = FIT(F_r_a, V), br = FIT(F_r_b, V);
  const double as = FIT(F_s_a, V), bs = FIT(F_s_b, V);

  const double calT3 = FIT(F_CalT3, V), calT4 = FIT(F_CalT4, V);
  const double eCa = 0.5 * C::R * C::T * log(C::Cao / caI) / C::F;
  const double iBCa = p.g_bca * (V - eCa);
  const double iPCa = caI * p.g_pCa / (caI + C::KpCa);
  const double expG = FIT(F_expG, V), expGm1 = FIT(F_expGm1, V);
  const double pKterm = FIT(F_pKterm, V);
  const double eK = RT * log(C::Ko / kI) / C::F;
  const double naKterm = FIT(F_NaKterm, V);
  const double iNaK = naI * naKterm / (naI + C::KmNa);
  const double vEK = -eK + V;
  const double bufC = 1.0 / (C::BufC * C::KbufC / ((caI + C::KbufC) * (caI + C::KbufC)) + 1);
  const double bufSR = 1.0 / (C::BufSr * C::KbufSr / ((caSR + C::KbufSr) * (caSR + C::KbufSr)) + 1);
  const double bufSS = 1.0 / (C::BufSs * C::KbufSs / ((caSS + C::KbufSs) * (caSS + C::KbufSs)) + 1);
  const double iLeak = C::Vleak * (caSR - caI);
  const double iUp = C::VmaxUp / (1 + (C::Kup * C::Kup) / (caI * caI));
  const double iXfer = C::Vxfer * (-caI + caSS);
  const double kcasr = C::MaxSr - (C::MaxSr - C::MinSr) / (1 + (C::EC * C::EC) / (caSR * caSR));
  const double k1 = C::K1p / kcasr, k2 = C::K2p * kcasr;
  const double O = (caSS * caSS) * rPrime * k1 / ((caSS * caSS) * k1 + C::K3);
  const double dRprime = -caSS * rPrime * k2 + C::K4 * (-rPrime + 1);
  const double iRel = O * C::Vrel * (caSR - caSS);
  const double dCaSR = bufSR * (-iLeak - iRel + iUp);
  const double iCaL = st.d * st.f * st.f2 * st.fCass * gCaL * (-C::Cao * calT3 + 0.25 * caSS * calT4);
  const double nao3 = C::Nao * C::Nao * C::Nao, kmnai3 = C::KmNai * C::KmNai * C::KmNai;
  const double iNaCa = C::KNaCa * ((naI * naI * naI) * C::Cao * expG - nao3 * caI * C::Alpha * expGm1) /
                       ((nao3 + kmnai3) * (C::Cao + C::KmCa) * (C::Ksat * expGm1 + 1));
  const double iK1 = FIT(F_K1, vEK);
  const double iPK = vEK * p.g_pK * pKterm;
  const double iKr = 0.430331482911935 * vEK * sqrtKo * st.Xr1 * st.Xr2 * gKr;
  const double eNa = RT * log(C::Nao / naI) / C::F;
  const double eKs = RT * log((C::Ko + C::Nao * C::Pkna) / (kI + naI * C::Pkna)) / C::F;
  const double iKs = (st.Xs * st.Xs) * p.g_Ks * (V - eKs);
  const double iBNa = p.g_bna * (-eNa + V);
  const double iTo = vEK * p.g_to * st.r * st.s;
  const double kTot = -2 * iNaK + iK1 + iPK + iKr + iKs + iTo;
  const double halfCm = -0.5 * C::Cm;
  const double dCaI = bufC * (halfCm * (-2 * iNaCa + iBCa + iPCa) / (C::F * C::Vc) + iXfer + C::Vsr * (iLeak - iUp) / C::Vc);
  const double dCaSS = bufSS * (halfCm * iCaL / (C::F * C::Vss) - C::Vc * iXfer / C::Vss + C::Vsr * iRel / C::Vss);
  const double m = st.m;
  const double iNa = (m * m * m) * gNa * st.h * st.j * (-eNa + V);
  const double dKi = -C::Cm * kTot / (C::F * C::Vc);
  const double naTot = iNa + 3 * iNaK + iBNa + 3 * iNaCa;
  const double dNai = -C::Cm * naTot / (C::F * C::Vc);
  const double caTot = iCaL + iPCa + iBCa + -2 * iNaCa;
  const double iIon = caTot + kTot + naTot;

  st.caSR = caSR + dt * dCaSR;
  st.caI = caI + dt * dCaI;
  st.caSS = caSS + dt * dCaSS;
  st.kI = kI + dt * dKi;
  st.naI = naI + dt * dNai;
  st.rPrime = rPrime + dt * dRprime;
  st.Xr1 += aXr1 * (st.Xr1 + bXr1);
  st.Xr2 += aXr2 * (st.Xr2 + bXr2);
  st.Xs += aXs * (st.Xs + bXs);
  st.d += ad * (st.d + bd);
  st.f += af * (st.f + bf);
  st.f2 += af2 * (st.f2 + bf2);
  st.fCass += aFc * (st.fCass + bFc);
  st.h += ah * (st.h + bh);
  st.j += aj * (st.j + bj);
  st.m += am * (st.m + bm);
  st.r += ar * (st.r + br);
  st.s += as * (st.s + bs);
#undef FIT
  return -iIon;
}

// Mixed step.  Returns dVm = -Iion in float.
template <class Fits>
__device__ __forceinline__ float tt06_step_mixed(const TT06Scalars& p, const BlockScale& blk, const Fits& fits,
                                                 float dtf, double V, CellState<float>& st)
{
  // every V-fit takes V; its FP32 argument is Vf
#define FIT(slot, x) fits.template fmix<slot>(x, V)
#define FITX(slot, xf, xd) fits.template fmix<slot>(xf, xd)
  constexpr float Cm = 0.185f, F = 96485.3415f, RT = 8314.472f * 310.0f, Vc = 0.016404f, Cao = 2.0f;
  constexpr float BufC = 0.2f, BufSr = 10.0f, BufSs = 0.4f, EC2 = 1.5f * 1.5f;
  constexpr float KbufC = 0.001f, KbufSr = 0.3f, KbufSs = 0.00025f, Kup2 = 0.00025f * 0.00025f;
  constexpr float Vleak = 0.00036f, Vrel = 0.102f, Vsr = 0.001094f, Vss = 5.468e-5f, Vxfer = 0.0038f;
  constexpr float VmaxUp = 0.006375f, K1p = 0.15f, K2p = 0.045f, K3 = 0.06f, K4 = 0.005f;
  constexpr float MaxSr = 2.5f, MinSr = 1.0f, KpCa = 0.0005f, KNaCa = 1000.0f, Ksat = 0.1f;
  constexpr float KmCa = 1.38f, KmNai = 87.5f, Alpha = 2.5f, Ko = 5.4f, Pkna = 0.03f, Nao = 140.0f;
  constexpr float KmNa = 40.0f;
  constexpr float RT_F = RT / F;
  const float gKr = (float)p.g_Kr * blk.g_Kr, gCaL = (float)p.g_CaL * blk.g_CaL, gNa = (float)p.g_Na * blk.g_Na;
  const float Vf = (float)V;
  const float caSR = (float)st.caSR, caI = (float)st.caI, caSS = (float)st.caSS;
  const float kI = (float)st.kI, naI = (float)st.naI, rPrime = st.rPrime;

  const float fCassInf = 0.4f + __fdividef(0.6f, 400.0f * (caSS * caSS) + 1.0f);
  const float aXr1 = FIT(F_Xr1_a, Vf), bXr1 = FIT(F_Xr1_b, Vf);
  const float aXr2 = FIT(F_Xr2_a, Vf), bXr2 = FIT(F_Xr2_b, Vf);
  const float aXs = FIT(F_Xs_a, Vf), bXs = FIT(F_Xs_b, Vf);
  const float ad = FIT(F_d_a, Vf), bd = FIT(F_d_b, Vf);
  const float af = FIT(F_f_a, Vf), bf = FIT(F_f_b, Vf);
  const float af2 = FIT(F_f2_a, Vf), bf2 = FIT(F_f2_b, Vf);
  const float aFc = FITX(F_fCass_a, caSS, st.caSS), bFc = -fCassInf;
  const float ah = FIT(F_h_a, Vf), bh = FIT(F_h_b, Vf);
  const float aj = FIT(F_j_a, Vf), bj = FIT(F_j_b, Vf);
  const float am = FIT(F_m_a, Vf), bm = FIT(F_m_b, Vf);
  const float ar = FIT(F_r_a, Vf), br = FIT(F_r_b, Vf);
  const float as = FIT(F_s_a, Vf), bs = FIT(F_s_b, Vf);

  const float calT3 = FIT(F_CalT3, Vf), calT4 = FIT(F_CalT4, Vf);
  const float eCa = 0.5f * RT_F * logf(__fdividef(Cao, caI));
  const float iBCa = (float)p.g_bca * (Vf - eCa);
  const float iPCa = __fdividef(caI * (float)p.g_pCa, caI + KpCa);
  const float expG = FIT(F_expG, Vf), expGm1 = FIT(F_expGm1, Vf);
  const float pKterm = FIT(F_pKterm, Vf);
  const float eK = RT_F * logf(__fdividef(Ko, kI));
  const float naKterm = FIT(F_NaKterm, Vf);
  const float iNaK = __fdividef(naI * naKterm, naI + KmNa);
  const float vEK = Vf - eK;
  const float cC = caI + KbufC, cSR = caSR + KbufSr, cSS = caSS + KbufSs;
  const float bufC = __fdividef(1.0f, __fdividef(BufC * KbufC, cC * cC) + 1.0f);
  const float bufSR = __fdividef(1.0f, __fdividef(BufSr * KbufSr, cSR * cSR) + 1.0f);
  const float bufSS = __fdividef(1.0f, __fdividef(BufSs * KbufSs, cSS * cSS) + 1.0f);
  const float iLeak = Vleak * (caSR - caI);
  const float iUp = __fdividef(VmaxUp, 1.0f + __fdividef(Kup2, caI * caI));
  const float iXfer = Vxfer * (caSS - caI);
  const float kcasr = MaxSr - __fdividef(MaxSr - MinSr, 1.0f + __fdividef(EC2, caSR * caSR));
  const float k1 = __fdividef(K1p, kcasr), k2 = K2p * kcasr;
  const float ss2 = caSS * caSS;
  const float O = __fdividef(ss2 * rPrime * k1, ss2 * k1 + K3);
  const float dRprime = -caSS * rPrime * k2 + K4 * (1.0f - rPrime);
  const float iRel = O * Vrel * (caSR - caSS);
  const float dCaSR = bufSR * (iUp - iLeak - iRel);
  const float iCaL = st.d * st.f * st.f2 * st.fCass * gCaL * (0.25f * caSS * calT4 - Cao * calT3);
  constexpr float nao3 = Nao * Nao * Nao, kmnai3 = KmNai * KmNai * KmNai;
  constexpr float naCaDen0 = (nao3 + kmnai3) * (Cao + KmCa);
  const float iNaCa = __fdividef(KNaCa * ((naI * naI * naI) * Cao * expG - nao3 * caI * Alpha * expGm1),
                                 naCaDen0 * (Ksat * expGm1 + 1.0f));
  const float iK1 = FITX(F_K1, vEK, V - (double)eK);
  const float iPK = vEK * (float)p.g_pK * pKterm;
  const float iKr = 0.430331482911935f * 2.3237900077f * vEK * st.Xr1 * st.Xr2 * gKr;
  const float eNa = RT_F * logf(__fdividef(Nao, naI));
  const float eKs = RT_F * logf(__fdividef(Ko + Nao * Pkna, kI + naI * Pkna));
  const float iKs = (st.Xs * st.Xs) * (float)p.g_Ks * (Vf - eKs);
  const float iBNa = (float)p.g_bna * (Vf - eNa);
  const float iTo = vEK * (float)p.g_to * st.r * st.s;
  const float kTot = -2.0f * iNaK + iK1 + iPK + iKr + iKs + iTo;
  constexpr float halfCm_FVc = -0.5f * Cm / (F * Vc), halfCm_FVss = -0.5f * Cm / (F * Vss);
  const float dCaI = bufC * (halfCm_FVc * (iBCa + iPCa - 2.0f * iNaCa) + iXfer + (Vsr / Vc) * (iLeak - iUp));
  const float dCaSS = bufSS * (halfCm_FVss * iCaL - (Vc / Vss) * iXfer + (Vsr / Vss) * iRel);
  const float m = st.m;
  const float iNa = (m * m * m) * gNa * st.h * st.j * (Vf - eNa);
  constexpr float mCm_FVc = -Cm / (F * Vc);
  const float dKi = mCm_FVc * kTot;
  const float naTot = iNa + 3.0f * iNaK + iBNa + 3.0f * iNaCa;
  const float dNai = mCm_FVc * naTot;
  const float caTot = iCaL + iPCa + iBCa - 2.0f * iNaCa;
  const float iIon = caTot + kTot + naTot;

  st.caSR += (double)(dtf * dCaSR);
  st.caI += (double)(dtf * dCaI);
  st.caSS += (double)(dtf * dCaSS);
  st.kI += (double)(dtf * dKi);
  st.naI += (double)(dtf * dNai);
  st.rPrime = rPrime + dtf * dRprime;
  st.Xr1 += aXr1 * (st.Xr1 + bXr1);
  st.Xr2 += aXr2 * (st.Xr2 + bXr2);
  st.Xs += aXs * (st.Xs + bXs);
  st.d += ad * (st.d + bd);
  st.f += af * (st.f + bf);
  st.f2 += af2 * (st.f2 + bf2);
  st.fCass += aFc * (st.fCass + bFc);
  st.h += ah * (st.h + bh);
  st.j += aj * (st.j + bj);
  st.m += am * (st.m + bm);
  st.r += ar * (st.r + br);
  st.s += as * (st.s + bs);
#undef FIT
#undef FITX
  return -iIon;
}

}  // namespace cdb
