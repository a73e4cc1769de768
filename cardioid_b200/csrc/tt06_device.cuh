// BetterTT06 ionic update of one cell on the device.
//
// Model: elec/BetterTT06.cc (LLNL/Cardioid) — CPU calc :1426-1649, the same
// equations as the reference's NVRTC kernel :1075-1298.  Per cell and step:
// 30 rational fits (Interpolation::eval, elec/Interpolation.hh:11-99), the
// currents, forward Euler on Ca_SR, Ca_i, Ca_ss, K_i, Na_i, R_prime and
// Rush-Larsen (X += a*(X + b)) on 12 gates; returns dVm = -Iion.
//
// This header holds the model's tables, constants and fit evaluation; the
// step itself is in tt06_step.cuh.  Two precisions:
//   FP64   every operation in double, expressions in the reference's order
//          (the compiler contracts a*b+c into an FMA, which only changes
//          last bits);
//   mixed  fits, gates, currents and R_prime in FP32; Vm and the five
//          concentrations in FP64 (their per-step increments are ~1e-7 of
//          their values).  The compiled kernels evaluate the few fits whose
//          monomial form loses accuracy in FP32 in a shifted argument
//          (fit_form32); the generic kernel evaluates them in FP64.
// Fit evaluation is a policy: GenericFits reads term counts at run time;
// SpecFits has them as compile-time constants (fit_shapes.h), so every
// Horner chain unrolls and the 30 independent chains interleave; its FP32
// fits run each numerator and denominator chain pair in two-lane FMAs
// (fit_pair32).
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
  // FP32 copies for the mixed step (constant operands, no conversion)
  float f_Ks, f_bca, f_bna, f_pCa, f_pK, f_to;
};

// FP32 quotient from the hardware reciprocal approximation
// (rcp.approx.ftz.f32, within 1 ulp): a * (1/b), no range handling.
__device__ __forceinline__ float fdiv(float a, float b)
{
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(b));
  return a * r;
}

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
  double g_Kr, g_CaL, g_Na;
};

// FP64 quotient without the slow-path branch of the IEEE division: the
// hardware reciprocal approximation (PTX rcp.approx.ftz.f64) refined by one
// Newton-Raphson step r <- r + r (1 - b r), then the quotient corrected
// once by its residual, q <- q + r (a - b q) (Markstein's method, IBM J.
// Res. Dev. 34(1), 1990): the correction squares the reciprocal's relative
// error, so one refinement of the seed is enough for a faithful quotient.  Within a few ulp of a / b for the normal,
// finite operands of the model (tests/test_division_gpu.py measures it
// against CUDA's a / b); subnormal divisors flush to zero.  Defining
// CDB_IEEE_DIV restores a / b.
// The seed refined once (relative error about the square of the seed's).
__device__ __forceinline__ double rcp64_1(double b)
{
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(b));
  const double e = fma(-b, r, 1.0);
  return fma(r, e, r);
}

// A reciprocal on its own: refined twice.
__device__ __forceinline__ double rcp64(double b)
{
#ifdef CDB_IEEE_DIV
  return 1.0 / b;
#else
  const double r = rcp64_1(b);
  const double e = fma(-b, r, 1.0);
  return fma(r, e, r);
#endif
}

__device__ __forceinline__ double div64(double a, double b)
{
#ifdef CDB_IEEE_DIV
  return a / b;
#else
  const double r = rcp64_1(b);
  const double q = a * r;
  return fma(r, fma(-b, q, a), q);
#endif
}

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
  return fdiv(num, den);
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
  return div64(num, den);
}

__host__ __device__ constexpr bool spec_shifted(int slot) { return (kSpecShiftMask >> slot) & 1u; }

// ---- the compiled mixed kernels' FP32 fits: paired Horner chains ----
//
// A rational fit num(x) / (1 + x den'(x)) is two Horner chains in the same
// argument, num <- fma(x, num, c) and den <- fma(x, den, d), independent
// of each other.  sm_100's two-lane FP32 FMA (__ffma2_rn, each lane rounded
// as fmaf) takes one step of both, so the chains run together for as many
// steps as the shorter one has, after the longer one's first steps run
// alone: one instruction per pair of FMAs, with the same operations and
// rounding as the two scalar chains.  Every fit runs this way: the fits in
// kSpecShiftMask in the shifted argument t = (x - s) / h of fit_shapes.h
// (their monomial form loses accuracy in FP32: numerator and denominator
// span many decades over the domain, and about the shift point the Taylor
// coefficients no longer cancel; h is a power of two, so t is one FMA with
// immediate operands and no extra rounding; registration rewrote their
// coefficients in t, spec_pool32), the others as written.
//
// Pool layout (built at registration from the FP32 pool, spec_pair_pool32):
// per fit a 16-byte aligned block holding the numerator's and the
// denominator's top coefficients, the coefficients of the longer chain's
// lone steps (top first), padding to a 16-byte boundary, then one
// (numerator, denominator) coefficient pair per joint step, two per
// 16-byte load; the denominator's last coefficient is the 1 of its form
// 1 + x (...).  A polynomial fit (denominator 1) holds its top coefficient,
// one pad and its remaining coefficients, top first.  (16-byte pairs of
// pairs measured 1 % faster on the 256^3 step than 8-byte pairs, same bits.)
//
// The layout per fit, for the device (compile-time F) and for the host
// (run-time f, spec_pair_pool32); the two agree (static_assert below).
template <int F>
struct PairShape {
  static constexpr int N = kSpecNumer[F], D = kSpecDenom[F];
  static constexpr int steps = D == 1 ? 0 : (N < D ? N : D) - 1;          // joint steps
  static constexpr int lead = D == 1 ? N - 1 : (N > D ? N : D) - 1 - steps;   // lone steps of the longer chain
  static constexpr int first = (2 + lead + 3) & ~3;                        // first pair, 16-byte aligned
  static constexpr int block = (first + 2 * steps + 3) & ~3;               // blocks start 16-byte aligned
};
template <int F>
struct PairOffset {
  static constexpr int value = PairOffset<F - 1>::value + PairShape<F - 1>::block;
};
template <>
struct PairOffset<0> {
  static constexpr int value = 0;
};
constexpr int kPairPool = PairOffset<30>::value;

constexpr int pair_steps(int f)
{
  return kSpecDenom[f] == 1 ? 0 : (kSpecNumer[f] < kSpecDenom[f] ? kSpecNumer[f] : kSpecDenom[f]) - 1;
}
constexpr int pair_lead(int f)
{
  return kSpecDenom[f] == 1 ? kSpecNumer[f] - 1
                            : (kSpecNumer[f] > kSpecDenom[f] ? kSpecNumer[f] : kSpecDenom[f]) - 1 - pair_steps(f);
}
constexpr int pair_first(int f) { return (2 + pair_lead(f) + 3) & ~3; }
constexpr int pair_offset(int f)
{
  int o = 0;
  for (int g = 0; g < f; ++g) o += (pair_first(g) + 2 * pair_steps(g) + 3) & ~3;
  return o;
}
static_assert(pair_offset(30) == kPairPool && pair_offset(29) == PairOffset<29>::value &&
                  pair_offset(13) == PairOffset<13>::value,
              "host and device pool layouts agree");

// FP32 fit F of the paired pool c (16-byte aligned) at argument x.
template <int F>
__device__ __forceinline__ float fit_pair32(const float* __restrict__ c, float x)
{
  constexpr int N = kSpecNumer[F], D = kSpecDenom[F], B = PairOffset<F>::value;
  constexpr int L = PairShape<F>::lead, S = PairShape<F>::steps, P0 = PairShape<F>::first;
  if (D == 1) {
    float num = c[B];
#pragma unroll
    for (int i = 0; i < L; ++i) num = fmaf(x, num, c[B + 2 + i]);
    return num;
  }
  float num = c[B], den = c[B + 1];
#pragma unroll
  for (int i = 0; i < L; ++i) {
    if (N > D) num = fmaf(x, num, c[B + 2 + i]);
    else den = fmaf(x, den, c[B + 2 + i]);
  }
  float2 nd = make_float2(num, den);
  const float2 xx = make_float2(x, x);
  // two joint steps' coefficient pairs per 16-byte load
#pragma unroll
  for (int k = 0; k + 1 < S; k += 2) {
    const float4 q = *reinterpret_cast<const float4*>(c + B + P0 + 2 * k);
    nd = __ffma2_rn(xx, nd, make_float2(q.x, q.y));
    nd = __ffma2_rn(xx, nd, make_float2(q.z, q.w));
  }
  if (S & 1) nd = __ffma2_rn(xx, nd, *reinterpret_cast<const float2*>(c + B + P0 + 2 * (S - 1)));
  return fdiv(nd.x, nd.y);
}

// The same in the fit's shifted argument when it has one.
template <int F>
__device__ __forceinline__ float fit_form32(const float* __restrict__ c, float x)
{
  if (!spec_shifted(F)) return fit_pair32<F>(c, x);
  constexpr float inv = 1.0f / kSpecShiftScale, off = -kSpecShift[F] / kSpecShiftScale;
  return fit_pair32<F>(c, fmaf(x, inv, off));
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
  __device__ __forceinline__ void set_v(float) {}
  template <int SLOT>
  __device__ __forceinline__ float fv(double vd) const { return fmix<SLOT>((float)vd, vd); }
};

struct SpecFits {
  const double* __restrict__ c64;
  const float* __restrict__ c32;   // the paired FP32 pool (fit_pair32)
  float v;                         // V in FP32 (set_v)
  __device__ __forceinline__ void set_v(float vf) { v = vf; }
  template <int SLOT>
  __device__ __forceinline__ double f64(double x) const { return fit_spec64<SLOT>(c64, x); }
  // a fit of another argument (Ca_ss, V - E_K)
  template <int SLOT>
  __device__ __forceinline__ float fmix(float xf, double) const { return fit_form32<SLOT>(c32, xf); }
  // a fit of V
  template <int SLOT>
  __device__ __forceinline__ float fv(double) const { return fit_form32<SLOT>(c32, v); }
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
  // reciprocals of the constant divisors (x / c becomes x * (1/c))
  static constexpr double InvF = 1.0 / F, InvFVc = 1.0 / (F * Vc), InvVc = 1.0 / Vc;
  static constexpr double InvFVss = 1.0 / (F * Vss), InvVss = 1.0 / Vss;
};

}  // namespace cdb
