// The BetterTT06 step of one cell (elec/BetterTT06.cc:1426-1649) on the
// device, reading and writing its state through an IO policy.
//
// Order: the currents and concentration derivatives first (they need the old
// gate values, V and seven fits), the concentrations and R_prime stored as
// soon as they are known, then each gate's two Rush-Larsen fits, its update
// and its store, one gate at a time.  Only independent work moves relative
// to the reference's listing; the short live ranges keep the register count
// (and with it the number of resident warps) in check.  In the FP64 step a
// division by a model constant is a product with its reciprocal and every
// other division is div64 (branch-free), which moves results by a few ulp.
//
// IO policy: get<k>() loads state k (checkpoint order), put<k>(v) stores it.
#pragma once
#include "tt06_device.cuh"

namespace cdb {

// FP64 step, the reference's expression order.
template <class Fits, class IO>
__device__ __forceinline__ double tt06_step(const TT06Scalars& p, const BlockScale& blk, const Fits& fits,
                                            double dt, double V, IO& io)
{
  using C = ConstsD;
#define FIT(slot, x) fits.template f64<slot>(x)
  const double gKr = p.g_Kr * blk.g_Kr, gCaL = p.g_CaL * blk.g_CaL, gNa = p.g_Na * blk.g_Na;
  const double sqrtKo = 2.32379000772445;   // sqrt(5.4) in double
  const double RT = C::R * C::T;
  const double caSR = io.template get<S_Ca_SR>(), caI = io.template get<S_Ca_i>();
  const double caSS = io.template get<S_Ca_ss>(), kI = io.template get<S_K_i>();
  const double naI = io.template get<S_Na_i>(), rPrime = io.template get<S_R_prime>();
  const double Xr1 = io.template get<S_Xr1>(), Xr2 = io.template get<S_Xr2>(), Xs = io.template get<S_Xs>();
  const double d = io.template get<S_d>(), f = io.template get<S_f>(), f2 = io.template get<S_f2>();
  const double fCass = io.template get<S_fCass>(), h = io.template get<S_h>(), j = io.template get<S_j>();
  const double m = io.template get<S_m>(), r = io.template get<S_r>(), s = io.template get<S_s>();

  // currents
  // (divisions by constants are products with their reciprocals; the rest
  // go through div64, so no division takes a branch)
  const double calT3 = FIT(F_CalT3, V), calT4 = FIT(F_CalT4, V);
  const double eCa = 0.5 * C::R * C::T * log(div64(C::Cao, caI)) * C::InvF;
  const double iBCa = p.g_bca * (V - eCa);
  const double iPCa = div64(caI * p.g_pCa, caI + C::KpCa);
  const double expG = FIT(F_expG, V), expGm1 = FIT(F_expGm1, V);
  const double pKterm = FIT(F_pKterm, V);
  const double eK = RT * log(div64(C::Ko, kI)) * C::InvF;
  const double naKterm = FIT(F_NaKterm, V);
  const double iNaK = div64(naI * naKterm, naI + C::KmNa);
  const double vEK = -eK + V;
  const double bufC = rcp64(div64(C::BufC * C::KbufC, (caI + C::KbufC) * (caI + C::KbufC)) + 1);
  const double bufSR = rcp64(div64(C::BufSr * C::KbufSr, (caSR + C::KbufSr) * (caSR + C::KbufSr)) + 1);
  const double bufSS = rcp64(div64(C::BufSs * C::KbufSs, (caSS + C::KbufSs) * (caSS + C::KbufSs)) + 1);
  const double iLeak = C::Vleak * (caSR - caI);
  const double iUp = div64(C::VmaxUp, 1 + div64(C::Kup * C::Kup, caI * caI));
  const double iXfer = C::Vxfer * (-caI + caSS);
  const double kcasr = C::MaxSr - div64(C::MaxSr - C::MinSr, 1 + div64(C::EC * C::EC, caSR * caSR));
  const double k1 = div64(C::K1p, kcasr), k2 = C::K2p * kcasr;
  const double O = div64((caSS * caSS) * rPrime * k1, (caSS * caSS) * k1 + C::K3);
  const double dRprime = -caSS * rPrime * k2 + C::K4 * (-rPrime + 1);
  const double iRel = O * C::Vrel * (caSR - caSS);
  const double dCaSR = bufSR * (-iLeak - iRel + iUp);
  const double iCaL = d * f * f2 * fCass * gCaL * (-C::Cao * calT3 + 0.25 * caSS * calT4);
  const double nao3 = C::Nao * C::Nao * C::Nao, kmnai3 = C::KmNai * C::KmNai * C::KmNai;
  const double iNaCa = div64(C::KNaCa * ((naI * naI * naI) * C::Cao * expG - nao3 * caI * C::Alpha * expGm1),
                             (nao3 + kmnai3) * (C::Cao + C::KmCa) * (C::Ksat * expGm1 + 1));
  const double iK1 = FIT(F_K1, vEK);
  const double iPK = vEK * p.g_pK * pKterm;
  const double iKr = 0.430331482911935 * vEK * sqrtKo * Xr1 * Xr2 * gKr;
  const double eNa = RT * log(div64(C::Nao, naI)) * C::InvF;
  const double eKs = RT * log(div64(C::Ko + C::Nao * C::Pkna, kI + naI * C::Pkna)) * C::InvF;
  const double iKs = (Xs * Xs) * p.g_Ks * (V - eKs);
  const double iBNa = p.g_bna * (-eNa + V);
  const double iTo = vEK * p.g_to * r * s;
  const double kTot = -2 * iNaK + iK1 + iPK + iKr + iKs + iTo;
  const double halfCm = -0.5 * C::Cm;
  const double dCaI = bufC * (halfCm * (-2 * iNaCa + iBCa + iPCa) * C::InvFVc + iXfer + C::Vsr * (iLeak - iUp) * C::InvVc);
  const double dCaSS = bufSS * (halfCm * iCaL * C::InvFVss - C::Vc * iXfer * C::InvVss + C::Vsr * iRel * C::InvVss);
  const double iNa = (m * m * m) * gNa * h * j * (-eNa + V);
  const double dKi = -C::Cm * kTot * C::InvFVc;
  const double naTot = iNa + 3 * iNaK + iBNa + 3 * iNaCa;
  const double dNai = -C::Cm * naTot * C::InvFVc;
  const double caTot = iCaL + iPCa + iBCa + -2 * iNaCa;
  const double iIon = caTot + kTot + naTot;

  // forward Euler on the concentrations and R_prime
  io.template put<S_Ca_SR>(caSR + dt * dCaSR);
  io.template put<S_Ca_i>(caI + dt * dCaI);
  io.template put<S_Ca_ss>(caSS + dt * dCaSS);
  io.template put<S_K_i>(kI + dt * dKi);
  io.template put<S_Na_i>(naI + dt * dNai);
  io.template put<S_R_prime>(rPrime + dt * dRprime);

  // Rush-Larsen on the gates, X += a (X + b), one gate at a time
#define GATE(S, X, FA, FB, x)                     \
  {                                               \
    const double ga = FIT(FA, x), gb = FIT(FB, x); \
    io.template put<S>(X + ga * (X + gb));        \
  }
  GATE(S_Xr1, Xr1, F_Xr1_a, F_Xr1_b, V)
  GATE(S_Xr2, Xr2, F_Xr2_a, F_Xr2_b, V)
  GATE(S_Xs, Xs, F_Xs_a, F_Xs_b, V)
  GATE(S_d, d, F_d_a, F_d_b, V)
  GATE(S_f, f, F_f_a, F_f_b, V)
  GATE(S_f2, f2, F_f2_a, F_f2_b, V)
  {
    const double fCassInf = 0.4 + div64(0.6, 400.0 * (caSS * caSS) + 1);
    const double ga = FIT(F_fCass_a, caSS), gb = -fCassInf;
    io.template put<S_fCass>(fCass + ga * (fCass + gb));
  }
  GATE(S_h, h, F_h_a, F_h_b, V)
  GATE(S_j, j, F_j_a, F_j_b, V)
  GATE(S_m, m, F_m_a, F_m_b, V)
  GATE(S_r, r, F_r_a, F_r_b, V)
  GATE(S_s, s, F_s_a, F_s_b, V)
#undef GATE
#undef FIT
  return -iIon;
}

// Mixed step.  Returns dVm = -Iion in float.
template <class Fits, class IO>
__device__ __forceinline__ float tt06_step_mixed(const TT06Scalars& p, const BlockScale& blk, Fits& fits,
                                                 float dtf, double V, IO& io)
{
  // every V-fit takes V (fv: the policy evaluates it in V or in its shifted argument)
#define FIT(slot, x) fits.template fv<slot>(V)
#define FITX(slot, xf, xd) fits.template fmix<slot>(xf, xd)
  fits.set_v((float)V);
  constexpr float Cm = 0.185f, F = 96485.3415f, RT = 8314.472f * 310.0f, Vc = 0.016404f, Cao = 2.0f;
  constexpr float BufC = 0.2f, BufSr = 10.0f, BufSs = 0.4f, EC2 = 1.5f * 1.5f;
  constexpr float KbufC = 0.001f, KbufSr = 0.3f, KbufSs = 0.00025f, Kup2 = 0.00025f * 0.00025f;
  constexpr float Vleak = 0.00036f, Vrel = 0.102f, Vsr = 0.001094f, Vss = 5.468e-5f, Vxfer = 0.0038f;
  constexpr float VmaxUp = 0.006375f, K1p = 0.15f, K2p = 0.045f, K3 = 0.06f, K4 = 0.005f;
  constexpr float MaxSr = 2.5f, MinSr = 1.0f, KpCa = 0.0005f, KNaCa = 1000.0f, Ksat = 0.1f;
  constexpr float KmCa = 1.38f, KmNai = 87.5f, Alpha = 2.5f, Ko = 5.4f, Pkna = 0.03f, Nao = 140.0f;
  constexpr float KmNa = 40.0f;
  constexpr float RT_F = RT / F;
  const float gKr = (float)(p.g_Kr * blk.g_Kr), gCaL = (float)(p.g_CaL * blk.g_CaL), gNa = (float)(p.g_Na * blk.g_Na);
  const float Vf = (float)V;
  const double caSRd = io.template get<S_Ca_SR>(), caId = io.template get<S_Ca_i>();
  const double caSSd = io.template get<S_Ca_ss>(), kId = io.template get<S_K_i>();
  const double naId = io.template get<S_Na_i>();
  const float rPrime = io.template get<S_R_prime>();
  const float Xr1 = io.template get<S_Xr1>(), Xr2 = io.template get<S_Xr2>(), Xs = io.template get<S_Xs>();
  const float d = io.template get<S_d>(), f = io.template get<S_f>(), f2 = io.template get<S_f2>();
  const float fCass = io.template get<S_fCass>(), h = io.template get<S_h>(), j = io.template get<S_j>();
  const float m = io.template get<S_m>(), r = io.template get<S_r>(), s = io.template get<S_s>();
  const float caSR = (float)caSRd, caI = (float)caId, caSS = (float)caSSd, kI = (float)kId, naI = (float)naId;

  // currents
  const float calT3 = FIT(F_CalT3, Vf), calT4 = FIT(F_CalT4, Vf);
  // __logf (hardware log2, ~2^-21 relative): the Nernst potentials need
  // ~1e-6 mV, and their arguments are positive concentration ratios
  const float eCa = 0.5f * RT_F * __logf(fdiv(Cao, caI));
  const float iBCa = p.f_bca * (Vf - eCa);
  const float iPCa = fdiv(caI * p.f_pCa, caI + KpCa);
  const float expG = FIT(F_expG, Vf), expGm1 = FIT(F_expGm1, Vf);
  const float pKterm = FIT(F_pKterm, Vf);
  const float eK = RT_F * __logf(fdiv(Ko, kI));
  const float naKterm = FIT(F_NaKterm, Vf);
  const float iNaK = fdiv(naI * naKterm, naI + KmNa);
  const float vEK = Vf - eK;
  const float cC = caI + KbufC, cSR = caSR + KbufSr, cSS = caSS + KbufSs;
  const float bufC = fdiv(1.0f, fdiv(BufC * KbufC, cC * cC) + 1.0f);
  const float bufSR = fdiv(1.0f, fdiv(BufSr * KbufSr, cSR * cSR) + 1.0f);
  const float bufSS = fdiv(1.0f, fdiv(BufSs * KbufSs, cSS * cSS) + 1.0f);
  const float iLeak = Vleak * (caSR - caI);
  const float iUp = fdiv(VmaxUp, 1.0f + fdiv(Kup2, caI * caI));
  const float iXfer = Vxfer * (caSS - caI);
  const float kcasr = MaxSr - fdiv(MaxSr - MinSr, 1.0f + fdiv(EC2, caSR * caSR));
  const float k1 = fdiv(K1p, kcasr), k2 = K2p * kcasr;
  const float ss2 = caSS * caSS;
  const float O = fdiv(ss2 * rPrime * k1, ss2 * k1 + K3);
  const float dRprime = -caSS * rPrime * k2 + K4 * (1.0f - rPrime);
  const float iRel = O * Vrel * (caSR - caSS);
  const float dCaSR = bufSR * (iUp - iLeak - iRel);
  const float iCaL = d * f * f2 * fCass * gCaL * (0.25f * caSS * calT4 - Cao * calT3);
  constexpr float nao3 = Nao * Nao * Nao, kmnai3 = KmNai * KmNai * KmNai;
  constexpr float naCaDen0 = (nao3 + kmnai3) * (Cao + KmCa);
  const float iNaCa = fdiv(KNaCa * ((naI * naI * naI) * Cao * expG - nao3 * caI * Alpha * expGm1),
                                 naCaDen0 * (Ksat * expGm1 + 1.0f));
  const float iK1 = FITX(F_K1, vEK, V - (double)eK);
  const float iPK = vEK * p.f_pK * pKterm;
  const float iKr = 0.430331482911935f * 2.3237900077f * vEK * Xr1 * Xr2 * gKr;
  const float eNa = RT_F * __logf(fdiv(Nao, naI));
  const float eKs = RT_F * __logf(fdiv(Ko + Nao * Pkna, kI + naI * Pkna));
  const float iKs = (Xs * Xs) * p.f_Ks * (Vf - eKs);
  const float iBNa = p.f_bna * (Vf - eNa);
  const float iTo = vEK * p.f_to * r * s;
  const float kTot = -2.0f * iNaK + iK1 + iPK + iKr + iKs + iTo;
  constexpr float halfCm_FVc = -0.5f * Cm / (F * Vc), halfCm_FVss = -0.5f * Cm / (F * Vss);
  const float dCaI = bufC * (halfCm_FVc * (iBCa + iPCa - 2.0f * iNaCa) + iXfer + (Vsr / Vc) * (iLeak - iUp));
  const float dCaSS = bufSS * (halfCm_FVss * iCaL - (Vc / Vss) * iXfer + (Vsr / Vss) * iRel);
  const float iNa = (m * m * m) * gNa * h * j * (Vf - eNa);
  constexpr float mCm_FVc = -Cm / (F * Vc);
  const float dKi = mCm_FVc * kTot;
  const float naTot = iNa + 3.0f * iNaK + iBNa + 3.0f * iNaCa;
  const float dNai = mCm_FVc * naTot;
  const float caTot = iCaL + iPCa + iBCa - 2.0f * iNaCa;
  const float iIon = caTot + kTot + naTot;

  // concentrations accumulate in FP64
  io.template put<S_Ca_SR>(caSRd + (double)(dtf * dCaSR));
  io.template put<S_Ca_i>(caId + (double)(dtf * dCaI));
  io.template put<S_Ca_ss>(caSSd + (double)(dtf * dCaSS));
  io.template put<S_K_i>(kId + (double)(dtf * dKi));
  io.template put<S_Na_i>(naId + (double)(dtf * dNai));
  io.template put<S_R_prime>(rPrime + dtf * dRprime);

#define GATE(S, X, FA, FB)                          \
  {                                                 \
    const float ga = FIT(FA, Vf), gb = FIT(FB, Vf); \
    io.template put<S>(X + ga * (X + gb));          \
  }
  GATE(S_Xr1, Xr1, F_Xr1_a, F_Xr1_b)
  GATE(S_Xr2, Xr2, F_Xr2_a, F_Xr2_b)
  GATE(S_Xs, Xs, F_Xs_a, F_Xs_b)
  GATE(S_d, d, F_d_a, F_d_b)
  GATE(S_f, f, F_f_a, F_f_b)
  GATE(S_f2, f2, F_f2_a, F_f2_b)
  {
    const float fCassInf = 0.4f + fdiv(0.6f, 400.0f * (caSS * caSS) + 1.0f);
    const float ga = FITX(F_fCass_a, caSS, caSSd), gb = -fCassInf;
    io.template put<S_fCass>(fCass + ga * (fCass + gb));
  }
  GATE(S_h, h, F_h_a, F_h_b)
  GATE(S_j, j, F_j_a, F_j_b)
  GATE(S_m, m, F_m_a, F_m_b)
  GATE(S_r, r, F_r_a, F_r_b)
  GATE(S_s, s, F_s_a, F_s_b)
#undef GATE
#undef FIT
#undef FITX
  return -iIon;
}

// State IO on structure-of-arrays rows with pitch n.
// FP64: 18 rows of double.  Mixed: 5 rows of double (the concentrations)
// and 13 rows of float (R_prime and the gates).
struct IO64 {
  double* __restrict__ s;
  int64_t n;
  template <int K> __device__ __forceinline__ double get() const { return s[K * n]; }
  template <int K> __device__ __forceinline__ void put(double v) const { s[K * n] = v; }
};

struct IOMixed {
  double* __restrict__ s64;
  float* __restrict__ s32;
  int64_t n;
  template <int K> __device__ __forceinline__ double get() const
  {
    if (K < 5) return s64[K * n];
    return (double)s32[(K - 5) * n];
  }
  template <int K> __device__ __forceinline__ void put(double v) const
  {
    if (K < 5) s64[K * n] = v;
    else s32[(K - 5) * n] = (float)v;
  }
};

}  // namespace cdb
