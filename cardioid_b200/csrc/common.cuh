// Shared host/device plumbing of the cardioid_b200 library: error status,
// device allocations, reaction-type tables in constant memory.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cardioid_b200.h"
#include "tt06_device.cuh"

namespace cdb {

constexpr int kFitPoolPerType = 640;   // coefficients of one reaction type's 30 fits
static_assert(kMaxReactionTypes >= CDB_MAX_REACTION_TYPES, "type table size");

void set_error(const std::string& msg);

// Reaction-type tables, uploaded once per type (constant memory: every
// thread of a warp reads the same coefficient).
struct TypeTables {
  TT06Scalars scal[CDB_MAX_REACTION_TYPES];
  FitShape shape[CDB_MAX_REACTION_TYPES];
};

struct Status {
  cdb_status code = CDB_OK;
  bool ok() const { return code == CDB_OK; }
};

#define CDB_CUDA(call)                                                                     \
  do {                                                                                     \
    cudaError_t _e = (call);                                                               \
    if (_e != cudaSuccess) {                                                               \
      ::cdb::set_error(std::string(#call) + ": " + cudaGetErrorString(_e));                \
      return (_e == cudaErrorMemoryAllocation) ? CDB_OOM : CDB_CUDA_ERROR;                 \
    }                                                                                      \
  } while (0)

#define CDB_CHECK(cond, code, msg)                                                         \
  do {                                                                                     \
    if (!(cond)) {                                                                         \
      ::cdb::set_error(msg);                                                               \
      return code;                                                                         \
    }                                                                                      \
  } while (0)

// Which fits lose accuracy when their monomial Horner form is evaluated in
// FP32 (as the mixed path does): the FP32 value (FMA Horner, float
// coefficients) is compared with the FP64 one over the fit's domain (V in
// [-100, 100] mV; Ca_ss in [1e-7, 0.1] mM for slot 0), and a fit whose
// largest error exceeds 1e-5 of its largest magnitude is flagged for FP64.
// High-degree rational fits whose denominator spans many decades (h and m
// Rush-Larsen rates, the K1 current) are the ones flagged.
inline uint32_t fp64_fit_mask(const cdb_fit* fits)
{
  uint32_t mask = 0;
  for (int f = 0; f < kNumFits; ++f) {
    const cdb_fit& F = fits[f];
    const double lo = f == 0 ? 1e-7 : -100.0, hi = f == 0 ? 0.1 : 100.0;
    double maxErr = 0, maxVal = 0;
    const int nPts = 4001;
    for (int i = 0; i < nPts; ++i) {
      const double x = lo + (hi - lo) * i / (nPts - 1);
      double num = F.coeff[F.numer - 1];
      for (int k = F.numer - 2; k >= 0; --k) num = F.coeff[k] + x * num;
      double v = num;
      const float xf = (float)x;
      float numf = (float)F.coeff[F.numer - 1];
      for (int k = F.numer - 2; k >= 0; --k) numf = std::fma(xf, numf, (float)F.coeff[k]);
      float vf = numf;
      if (F.denom > 1) {
        const double* d = F.coeff + F.numer;
        double den = d[F.denom - 2];
        for (int k = F.denom - 3; k >= 0; --k) den = d[k] + x * den;
        den = 1 + x * den;
        v = num / den;
        float denf = (float)d[F.denom - 2];
        for (int k = F.denom - 3; k >= 0; --k) denf = std::fma(xf, denf, (float)d[k]);
        denf = std::fma(xf, denf, 1.0f);
        vf = numf / denf;
      }
      maxVal = std::max(maxVal, std::fabs(v));
      const double e = std::fabs((double)vf - v);
      maxErr = std::isfinite(e) ? std::max(maxErr, e) : 1e300;
    }
    if (maxErr > 1e-5 * maxVal) mask |= 1u << f;
  }
  return mask;
}

// Packs 30 fits into a coefficient pool; fails when they do not fit.
inline bool pack_fits(const cdb_fit* fits, FitShape& sh, double* pool, int poolSize, std::string& err)
{
  int off = 0;
  for (int f = 0; f < kNumFits; ++f) {
    const int nn = fits[f].numer, nd = fits[f].denom;
    if (nn < 1 || nd < 1 || nn + nd - 1 > CDB_MAX_COEFF) {
      err = "fit " + std::to_string(f) + " has invalid term counts";
      return false;
    }
    if (off + nn + nd - 1 > poolSize) {
      err = "fits of one reaction type exceed " + std::to_string(poolSize) + " coefficients";
      return false;
    }
    sh.numer[f] = (int16_t)nn;
    sh.denom[f] = (int16_t)nd;
    sh.offset[f] = (int16_t)off;
    for (int k = 0; k < nn + nd - 1; ++k) pool[off + k] = fits[f].coeff[k];
    off += nn + nd - 1;
  }
  sh.fp64mask = fp64_fit_mask(fits);
  return true;
}

// Taylor shift and scale of a polynomial: q with sum_k c_k x^k =
// sum_j q_j t^j, t = (x - s) / h.  Repeated synthetic division by (x - s)
// in long double (each coefficient to about 1e-12 relative even where the
// monomial coefficients cancel strongly), then q_j = a_j h^j.
inline void taylor_shift(const double* c, int n, double s, double h, long double* q)
{
  for (int k = 0; k < n; ++k) q[k] = c[k];
  for (int i = 0; i < n; ++i)
    for (int k = n - 2; k >= i; --k) q[k] += (long double)s * q[k + 1];
  long double hp = 1;
  for (int j = 0; j < n; ++j, hp *= h) q[j] *= hp;
}

// FP32 coefficient pool of the mixed kernels from a pool packed at the
// compiled offsets (pack_fits_spec): a fit in kSpecShiftMask is rewritten in
// t = (x - kSpecShift) / kSpecShiftScale, numerator and denominator divided
// by the denominator's constant term so that the denominator keeps the form
// 1 + t (...); every other fit is the FP32 rounding of its coefficients.
// False when a shifted denominator vanishes at the shift point.
inline bool spec_pool32(const double* pool, float* out, int poolSize)
{
  for (int k = 0; k < poolSize; ++k) out[k] = (float)pool[k];
  long double qn[CDB_MAX_COEFF + 1], qd[CDB_MAX_COEFF + 1];
  double den[CDB_MAX_COEFF + 1];
  for (int f = 0; f < kNumFits; ++f) {
    if (!((kSpecShiftMask >> f) & 1u)) continue;
    const int O = kSpecOffset[f], N = kSpecNumer[f], D = kSpecDenom[f];
    den[0] = 1.0;
    for (int k = 1; k < D; ++k) den[k] = pool[O + N + k - 1];
    taylor_shift(pool + O, N, kSpecShift[f], kSpecShiftScale, qn);
    taylor_shift(den, D, kSpecShift[f], kSpecShiftScale, qd);
    if (!(std::fabs((double)qd[0]) > 0.0) || !std::isfinite((double)qd[0])) return false;
    for (int k = 0; k < N; ++k) out[O + k] = (float)(qn[k] / qd[0]);
    for (int k = 1; k < D; ++k) out[O + N + k - 1] = (float)(qd[k] / qd[0]);
  }
  return true;
}

// One fit's FP32 numerator or denominator polynomial (n coefficients,
// c[0] the constant term) as the compiled mixed kernels evaluate it: Horner
// with one rounding per step (fit_pair32 runs the numerator's and the
// denominator's chains in the two lanes of one FMA, each lane rounded as
// fmaf, so each chain's value is this one).
inline float spec_poly32(const float* c, int n, float x)
{
  float r = c[n - 1];
  for (int k = n - 2; k >= 0; --k) r = std::fma(x, r, c[k]);
  return r;
}

// The paired FP32 pool of the compiled mixed kernels (fit_pair32's layout,
// tt06_device.cuh) from the FP32 pool at the compiled offsets
// (spec_pool32); out holds at least kPairPool floats, zero outside the
// fits' blocks.
inline void spec_pair_pool32(const float* spec32, float* out, int outSize)
{
  for (int k = 0; k < outSize; ++k) out[k] = 0.0f;
  for (int f = 0; f < kNumFits; ++f) {
    const int O = kSpecOffset[f], N = kSpecNumer[f], D = kSpecDenom[f], B = pair_offset(f);
    const int L = pair_lead(f), S = pair_steps(f), P0 = pair_first(f);
    // coefficient of step i of the numerator chain (top first), and of
    // step j of the denominator chain (its last step adds the form's 1)
    auto num = [&](int i) { return spec32[O + N - 2 - i]; };
    auto den = [&](int j) { return j < D - 2 ? spec32[O + N + D - 3 - j] : 1.0f; };
    out[B] = spec32[O + N - 1];
    if (D == 1) {
      for (int i = 0; i < L; ++i) out[B + 2 + i] = num(i);
      continue;
    }
    out[B + 1] = spec32[O + N + D - 2];
    for (int i = 0; i < L; ++i) out[B + 2 + i] = N > D ? num(i) : den(i);
    const int i0 = N > D ? L : 0, j0 = N > D ? 0 : L;
    for (int k = 0; k < S; ++k) {
      out[B + P0 + 2 * k] = num(i0 + k);
      out[B + P0 + 2 * k + 1] = den(j0 + k);
    }
  }
}
static_assert(kPairPool <= kFitPoolPerType, "the paired pool exceeds the per-type pool");

// Whether the paired pool gives every fit's numerator and denominator the
// same values, bit for bit, as the Horner chains of spec_poly32 on the
// FP32 pool, at 41 points of each fit's domain: fit_pair32's steps
// restated on the host, one std::fma per lane (a check of the layout).
inline bool spec_pair_ok(const float* spec32, const float* paired)
{
  float dc[CDB_MAX_COEFF + 1];
  for (int f = 0; f < kNumFits; ++f) {
    const int O = kSpecOffset[f], N = kSpecNumer[f], D = kSpecDenom[f], B = pair_offset(f);
    const int L = pair_lead(f), S = pair_steps(f), P0 = pair_first(f);
    const bool shifted = (kSpecShiftMask >> f) & 1u;
    dc[0] = 1.0f;
    for (int k = 1; k < D; ++k) dc[k] = spec32[O + N + k - 1];
    const double lo = f == 0 ? 1e-7 : -100.0, hi = f == 0 ? 0.1 : 100.0;
    for (int i = 0; i <= 40; ++i) {
      const double xd = lo + (hi - lo) * i / 40;
      const float x = shifted ? std::fma((float)xd, 1.0f / kSpecShiftScale, -kSpecShift[f] / kSpecShiftScale)
                              : (float)xd;
      float num = paired[B], den = 1.0f;
      if (D == 1) {
        for (int k = 0; k < L; ++k) num = std::fma(x, num, paired[B + 2 + k]);
      } else {
        den = paired[B + 1];
        for (int k = 0; k < L; ++k) {
          if (N > D) num = std::fma(x, num, paired[B + 2 + k]);
          else den = std::fma(x, den, paired[B + 2 + k]);
        }
        for (int k = 0; k < S; ++k) {
          num = std::fma(x, num, paired[B + P0 + 2 * k]);
          den = std::fma(x, den, paired[B + P0 + 2 * k + 1]);
        }
      }
      const float wn = spec_poly32(spec32 + O, N, x), wd = D > 1 ? spec_poly32(dc, D, x) : 1.0f;
      if (std::memcmp(&num, &wn, sizeof(float)) != 0 || std::memcmp(&den, &wd, sizeof(float)) != 0) return false;
    }
  }
  return true;
}

// Whether the FP32 forms of spec_pool32, evaluated as the mixed kernels do
// (spec_poly32, FP32 quotient), stay within 1e-5 of each
// fit's largest magnitude against the FP64 monomial form over the fit's
// domain (V in [-100, 100] mV; Ca_ss in [1e-7, 0.1] mM for slot 0).
inline bool spec_fp32_ok(const double* pool, const float* pool32)
{
  float dc[CDB_MAX_COEFF + 1];
  for (int f = 0; f < kNumFits; ++f) {
    const int O = kSpecOffset[f], N = kSpecNumer[f], D = kSpecDenom[f];
    const bool shifted = (kSpecShiftMask >> f) & 1u;
    dc[0] = 1.0f;
    for (int k = 1; k < D; ++k) dc[k] = pool32[O + N + k - 1];
    const double lo = f == 0 ? 1e-7 : -100.0, hi = f == 0 ? 0.1 : 100.0;
    double maxErr = 0, maxVal = 0;
    const int nPts = 4001;
    for (int i = 0; i < nPts; ++i) {
      const double x = lo + (hi - lo) * i / (nPts - 1);
      double num = pool[O + N - 1];
      for (int k = N - 2; k >= 0; --k) num = pool[O + k] + x * num;
      double den = 1;
      if (D > 1) {
        den = pool[O + N + D - 2];
        for (int k = D - 3; k >= 0; --k) den = pool[O + N + k] + x * den;
        den = 1 + x * den;
      }
      const double v = num / den;
      const float xf = shifted ? std::fma((float)x, 1.0f / kSpecShiftScale, -kSpecShift[f] / kSpecShiftScale)
                               : (float)x;
      const float vf = spec_poly32(pool32 + O, N, xf) / spec_poly32(dc, D, xf);
      maxVal = std::max(maxVal, std::fabs(v));
      const double e = std::fabs((double)vf - v);
      maxErr = std::isfinite(e) ? std::max(maxErr, e) : 1e300;
    }
    if (maxErr > 1e-5 * maxVal) return false;
  }
  return true;
}

// Packs 30 fits at the compile-time offsets of fit_shapes.h, zero-padded,
// when every fit is no longer than the compiled shape, the mixed kernels'
// FP32 forms of them are accurate (spec_fp32_ok) and their paired pool
// reproduces those forms (spec_pair_ok); false otherwise.
inline bool pack_fits_spec(const cdb_fit* fits, double* pool, int poolSize)
{
  static_assert(kSpecPool <= kFitPoolPerType, "compiled fit pool exceeds the per-type pool");
  for (int f = 0; f < kNumFits; ++f) {
    const int nn = fits[f].numer, nd = fits[f].denom;
    if (nn < 1 || nd < 1 || nn > kSpecNumer[f]) return false;
    if (nd > 1 && nd > kSpecDenom[f]) return false;
  }
  for (int k = 0; k < poolSize; ++k) pool[k] = 0.0;
  for (int f = 0; f < kNumFits; ++f) {
    const int nn = fits[f].numer, nd = fits[f].denom;
    const int O = kSpecOffset[f], N = kSpecNumer[f];
    for (int k = 0; k < nn; ++k) pool[O + k] = fits[f].coeff[k];
    for (int k = 0; k < nd - 1; ++k) pool[O + N + k] = fits[f].coeff[nn + k];
  }
  std::vector<float> pool32(poolSize), paired(poolSize);
  if (!spec_pool32(pool, pool32.data(), poolSize) || !spec_fp32_ok(pool, pool32.data())) return false;
  spec_pair_pool32(pool32.data(), paired.data(), poolSize);
  return spec_pair_ok(pool32.data(), paired.data());
}

inline TT06Scalars to_scalars(const cdb_tt06_params& p)
{
  TT06Scalars s;
  s.celltype = p.celltype; s.g_CaL = p.g_CaL; s.g_K1 = p.g_K1; s.g_Kr = p.g_Kr; s.g_Ks = p.g_Ks;
  s.g_Na = p.g_Na; s.g_bca = p.g_bca; s.g_bna = p.g_bna; s.g_pCa = p.g_pCa; s.g_pK = p.g_pK; s.g_to = p.g_to;
  s.f_Ks = (float)p.g_Ks; s.f_bca = (float)p.g_bca; s.f_bna = (float)p.g_bna; s.f_pCa = (float)p.g_pCa;
  s.f_pK = (float)p.g_pK; s.f_to = (float)p.g_to;
  return s;
}

// Initial state of BetterTT06 (initializeMembraneVoltage, elec/BetterTT06.cc:1657-1712),
// checkpoint order.
__host__ __device__ inline double tt06_initial_state(int k)
{
  switch (k) {
    case S_Ca_SR: return 3.155;
    case S_Ca_i: return 2.0e-5;
    case S_Ca_ss: return 0.00017;
    case S_K_i: return 138.4;
    case S_Na_i: return 10.355;
    case S_R_prime: return 0.9868;
    case S_Xr1: return 0.00448;
    case S_Xr2: return 0.476;
    case S_Xs: return 0.0087;
    case S_d: return 3.164e-5;
    case S_f: return 0.9609;
    case S_f2: return 0.9778;
    case S_fCass: return 0.9953;
    case S_h: return 0.55;
    case S_j: return 0.66;
    case S_m: return 0.00155;
    case S_r: return 2.235e-8;
    default: return 0.6012;   // s
  }
}
constexpr double kInitialVm = -83.0;

// Order-preserving map of doubles onto unsigned 64-bit integers, for
// atomicMin / atomicMax reductions.
__host__ __device__ inline unsigned long long ordered_bits(double v)
{
#ifdef __CUDA_ARCH__
  long long b = __double_as_longlong(v);
#else
  long long b;
  std::memcpy(&b, &v, 8);
#endif
  return b >= 0 ? (unsigned long long)b ^ 0x8000000000000000ull : ~(unsigned long long)b;
}
__host__ __device__ inline double from_ordered_bits(unsigned long long u)
{
  unsigned long long b = (u & 0x8000000000000000ull) ? (u ^ 0x8000000000000000ull) : ~u;
  double v;
#ifdef __CUDA_ARCH__
  v = __longlong_as_double((long long)b);
#else
  std::memcpy(&v, &b, 8);
#endif
  return v;
}

// Device-side counter of launches made by this library (for reporting).
extern int64_t g_launches;

}  // namespace cdb
