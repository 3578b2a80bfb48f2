// pf_common.cuh -- arithmetic shared by the engine and the stateless kernels.
//
// * Philox4x32-10 counter-based RNG, written from Salmon, Moraes, Dror, Shaw,
//   "Parallel random numbers: as easy as 1, 2, 3" (SC'11).  It replaces the
//   reference's cuRAND Philox states (src/particle_filter/predict.cu:14-20,
//   resampling.cu:183-205).
// * Box-Muller normals.
// * Deterministic weight quantisation: exp(lw - max) evaluated with IEEE
//   double-precision operations that round identically on host and device,
//   then scaled to a 64-bit integer, and the exact rescaling of integer sums
//   by such exponentials (scale_floor).  The systematic resampler's CDF is an
//   exact integer prefix sum of these values, so the ancestor indices are a
//   function of (log-weights, offset) alone, independent of scan order.
// * The systematic predicate of resampling.cu:69-77,
//       cdf[i] < (u + k) / N
//   evaluated exactly as  C_i * N * 2^32  <  (k * 2^32 + u32) * W
//   with C the integer inclusive CDF and W its total.
#pragma once
#include <stdint.h>
#include <math.h>
#include <string.h>
#include <cuda_runtime.h>

#define PF_HD __host__ __device__ __forceinline__

namespace pfb {

// ---------------------------------------------------------------- Philox
struct U4 {
  uint32_t x, y, z, w;
};

PF_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
#ifdef __CUDA_ARCH__
  lo = a * b;
  hi = __umulhi(a, b);
#else
  uint64_t p = (uint64_t)a * (uint64_t)b;
  lo = (uint32_t)p;
  hi = (uint32_t)(p >> 32);
#endif
}

// Ten rounds; round multipliers and Weyl key increments from the paper.
PF_HD U4 philox10(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(0xD2511F53u, c.x, hi0, lo0);
    mulhilo32(0xCD9E8D57u, c.z, hi1, lo1);
    U4 n;
    n.x = hi1 ^ c.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ c.w ^ k1;
    n.w = lo0;
    c = n;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// Stream tags (third counter word, high byte) keep the draws of different
// purposes disjoint for the same (particle, epoch, filter).
enum : uint32_t {
  TAG_INIT = 0x01000000u,
  TAG_PREDICT = 0x02000000u,
  TAG_SYS_U = 0x03000000u,
  TAG_MEGO_OFF = 0x04000000u,
  TAG_MEGO_U = 0x05000000u,
  TAG_COMPAT_INIT = 0x11000000u,
  TAG_COMPAT_PREDICT = 0x12000000u,
  TAG_COMPAT_MEGO = 0x13000000u,
};

#ifdef __CUDACC__
// Two standard normals from two 32-bit words (Box-Muller) with
// u1 = (a + 1/2) 2^-32 in (0, 1) and angle 2*pi*u2 in [-pi, pi), where the
// fast sine/cosine are accurate to about 2^-21.
// log(u1) keeps r = sqrt(-2 log u1) accurate to ~4e-6 absolute or better:
// the fast logarithm (absolute error ~2^-21) wherever |log u1| >= 2^-8;
// above 1 - 2^-8, u1 = 1 - v with v = (~a + 1/2) 2^-32 formed exactly and
// log(1 - v) = -v (1 + v/2 + v^2/3) (next term v^4/4 < 6e-11).
__device__ __forceinline__ float bm_log_u1(uint32_t a) {
  const float two_m32 = 2.3283064365386963e-10f;
  const float half_ulp = 1.1641532182693481e-10f;
  if (a >= 0xFF000000u) {
    const float v = fmaf((float)(~a), two_m32, half_ulp);
    return -v * fmaf(v, fmaf(v, 1.0f / 3.0f, 0.5f), 1.0f);
  }
  return __logf(fmaf((float)a, two_m32, half_ulp));
}

// The angle uses the top 24 bits of b: u2 = (b >> 8) 2^-24 - 1/2 is exact in
// FP32.
__device__ __forceinline__ float2 box_muller_f32(uint32_t a, uint32_t b) {
  float u2 = fmaf((float)(b >> 8), 5.9604644775390625e-08f, -0.5f);
  // r = sqrt(q) as q * rsqrt(q) (two instructions; q >= 2^-32 here, the
  // relative error of about 2^-22 is far below the noise tolerance)
  const float q = fmaxf(-2.0f * bm_log_u1(a), 0.0f);
  const float r = q > 0.0f ? q * rsqrtf(q) : 0.0f;
  float s, c;
  __sincosf(6.283185307179586f * u2, &s, &c);
  return make_float2(r * c, r * s);
}

__device__ __forceinline__ double2 box_muller_f64(uint32_t a, uint32_t b) {
  const double two_m32 = 2.3283064365386963e-10;
  double u1 = ((double)a + 0.5) * two_m32;
  double u2 = (double)b * two_m32 - 0.5;
  double r = sqrt(-2.0 * log(u1));
  double s, c;
  sincospi(2.0 * u2, &s, &c);
  return make_double2(r * c, r * s);
}
#endif

// ------------------------------------------------ deterministic quantiser
// Double-precision operations with round-to-nearest that neither the host
// compiler nor nvcc may contract or reorder, so host and device produce the
// same bits.
PF_HD double det_mul(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b);
#else
  volatile double r = a * b;
  return r;
#endif
}
PF_HD double det_sub(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dsub_rn(a, b);
#else
  volatile double r = a - b;
  return r;
#endif
}
PF_HD double det_fma(double a, double b, double c) {
#ifdef __CUDA_ARCH__
  return __fma_rn(a, b, c);
#else
  return fma(a, b, c);
#endif
}

// Exponent K of the fixed-point scale: the largest weight maps to about
// 2^K, and N * 2^(K+1) stays below 2^63.
PF_HD int quant_exponent(int n) {
  int lg = 0;
  while ((1ll << lg) < (long long)n) ++lg;
  int k = 62 - lg;
  return k < 40 ? k : 40;
}

// e^t for t in [0, ln 2): the Taylor series of the exponential
// (coefficients 1/j!, degree 13, truncation error < 1e-13) in Horner form
// with fma.
PF_HD double exp_poly(double t) {
  double q = 1.6059043836821615e-10;  // 1/13!
  q = det_fma(q, t, 2.0876756987868099e-09);  // 1/12!
  q = det_fma(q, t, 2.5052108385441720e-08);  // 1/11!
  q = det_fma(q, t, 2.7557319223985893e-07);  // 1/10!
  q = det_fma(q, t, 2.7557319223985888e-06);  // 1/9!
  q = det_fma(q, t, 2.4801587301587302e-05);  // 1/8!
  q = det_fma(q, t, 1.9841269841269841e-04);  // 1/7!
  q = det_fma(q, t, 1.3888888888888889e-03);  // 1/6!
  q = det_fma(q, t, 8.3333333333333333e-03);  // 1/5!
  q = det_fma(q, t, 4.1666666666666667e-02);  // 1/4!
  q = det_fma(q, t, 1.6666666666666667e-01);  // 1/3!
  q = det_fma(q, t, 0.5);
  q = det_fma(q, t, 1.0);
  q = det_fma(q, t, 1.0);  // e^t = 2^f in [1, 2]
  return q;
}

// q = floor(2^K * exp(d)) for a shifted log-weight d = lw - max <= 0.
// x = d * log2(e), n = floor(x), f = x - n (exact), t = f * ln 2, and
// e^t = 2^f from exp_poly; 2^n scales exactly.  Weights below 2^-40 of the
// largest quantise to zero.
PF_HD uint64_t quantize_shifted(double d, int K) {
  const double x = det_mul(d, 1.4426950408889634074);
  if (!(x > -40.0)) return 0ull;  // also catches NaN
  const double n = floor(x);
  const double f = det_sub(x, n);  // exact: f in [0, 1)
  const double t = det_mul(f, 0.69314718055994530942);
  const double v = ldexp(exp_poly(t), K + (int)n);  // exact scaling, <= 2^(K+1)
  return (uint64_t)v;                               // truncation
}

// floor(v * r) for an integer v < 2^53 and 0 <= r <= 1: one rounded product
// (exact conversion of v), then truncation.
PF_HD uint64_t scale_floor(uint64_t v, double r) { return (uint64_t)det_mul((double)v, r); }
// The same on an integer-valued double v < 2^53.
PF_HD double scale_trunc(double v, double r) { return trunc(det_mul(v, r)); }

// ------------------------------------- deterministic FP32 exponential
// The engine's log-weights are FP32 (about 1e-7 relative), so its integer
// CDF evaluates e^d in FP32 with round-to-nearest operations that neither
// compiler may contract, identical on host and device: x = d log2(e) (one
// rounded product), n = floor(x), f = x - n (one rounded difference), 2^f
// from the Taylor series of e^(f ln 2) (coefficients (ln 2)^k / k! rounded to
// FP32, degree 9, Horner with fma; within 2 ulp of 2^f), and 2^n applied
// exactly.
PF_HD float det_fmul(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fmul_rn(a, b);
#else
  volatile float r = a * b;
  return r;
#endif
}
PF_HD float det_fsub(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fsub_rn(a, b);
#else
  volatile float r = a - b;
  return r;
#endif
}
PF_HD float det_ffma(float a, float b, float c) {
#ifdef __CUDA_ARCH__
  return __fmaf_rn(a, b, c);
#else
  return fmaf(a, b, c);
#endif
}
PF_HD float exp2_frac_f32(float f) {
  float q = 0x1.b5253ep-24f;  // (ln 2)^9 / 9!
  q = det_ffma(q, f, 0x1.62c022p-20f);  // (ln 2)^8 / 8!
  q = det_ffma(q, f, 0x1.ffcbfcp-17f);  // (ln 2)^7 / 7!
  q = det_ffma(q, f, 0x1.430912p-13f);  // (ln 2)^6 / 6!
  q = det_ffma(q, f, 0x1.5d87fep-10f);  // (ln 2)^5 / 5!
  q = det_ffma(q, f, 0x1.3b2ab6p-7f);  // (ln 2)^4 / 4!
  q = det_ffma(q, f, 0x1.c6b08ep-5f);  // (ln 2)^3 / 3!
  q = det_ffma(q, f, 0x1.ebfbep-3f);  // (ln 2)^2 / 2!
  q = det_ffma(q, f, 0x1.62e43p-1f);  // ln 2
  q = det_ffma(q, f, 0x1.0p+0f);
  return q;
}

// 2^m as a float, exact for -126 <= m <= 127.
PF_HD float pow2_f32(int m) {
  const uint32_t b = (uint32_t)(127 + m) << 23;
#ifdef __CUDA_ARCH__
  return __uint_as_float(b);
#else
  float r;
  memcpy(&r, &b, sizeof(r));
  return r;
#endif
}

// floor(2^K e^d) for a shifted FP32 log-weight d = lw - max <= 0, as an
// integer-valued float (exact: 2^f 2^(K+n) < 2^41 is a float, its
// truncation too); weights below 2^-40 of the maximum quantise to zero.
PF_HD float quantize_f32(float d, int K) {
  const float x = det_fmul(d, 0x1.715476p+0f /* log2(e) */);
  if (!(x > -40.0f)) return 0.0f;  // also catches NaN
  const float n = floorf(x);
  const float p = exp2_frac_f32(det_fsub(x, n));
  return truncf(p * pow2_f32(K + (int)n));
}

// e^d for d <= 0 (0 below 2^-126), the scale factors of the tiled CDF.
PF_HD float det_expf(float d) {
  const float x = det_fmul(d, 0x1.715476p+0f /* log2(e) */);
  if (!(x > -126.0f)) return 0.0f;
  const float n = floorf(x);
  return exp2_frac_f32(det_fsub(x, n)) * pow2_f32((int)n);  // exact: a normal float
}

// ------------------------------------------------ 128-bit exact compare
PF_HD void mul_64x64(uint64_t a, uint64_t b, uint64_t& hi, uint64_t& lo) {
#ifdef __CUDA_ARCH__
  lo = a * b;
  hi = __umul64hi(a, b);
#else
  unsigned __int128 p = (unsigned __int128)a * b;
  lo = (uint64_t)p;
  hi = (uint64_t)(p >> 64);
#endif
}

// (k * 2^32 + u) * W  <=  C * N * 2^32 ?
PF_HD bool slot_at_or_below(uint64_t k, uint32_t u, uint64_t W, uint64_t C,
                            uint32_t N) {
  uint64_t T = (k << 32) | (uint64_t)u;
  uint64_t lh, ll;
  mul_64x64(T, W, lh, ll);
  uint64_t ch, cl;
  mul_64x64(C, (uint64_t)N, ch, cl);  // < 2^94
  uint64_t rh = (ch << 32) | (cl >> 32);
  uint64_t rl = cl << 32;
  return (lh < rh) || (lh == rh && ll <= rl);
}

// F(C) = #{k in [0, N) : (k * 2^32 + u) * W <= C * N * 2^32}.
// Slots [F(C_{i-1}), F(C_i)) are the offspring of particle i; equivalently
// the lower-bound search of resampling.cu:72-77 returns i for those slots.
PF_HD uint32_t offspring_end(uint64_t C, uint64_t W, uint32_t N, uint32_t u) {
  double est = (double)C / (double)W * (double)N - (double)u * 2.3283064365386963e-10;
  long long k = (long long)floor(est);
  if (k < -1) k = -1;
  if (k > (long long)N - 1) k = (long long)N - 1;
  while (k >= 0 && !slot_at_or_below((uint64_t)k, u, W, C, N)) --k;
  while (k + 1 < (long long)N && slot_at_or_below((uint64_t)(k + 1), u, W, C, N)) ++k;
  return (uint32_t)(k + 1);
}

// Exact F from an estimate k of the last slot at or below C (moved to the
// right value by the 128-bit predicate).  Out of line: it runs only for
// estimates close to a slot boundary.
static __host__ __device__ __noinline__ uint32_t offspring_end_settle(long long k, uint64_t C, uint64_t W, uint32_t N,
                                                              uint32_t u) {
  while (k >= 0 && !slot_at_or_below((uint64_t)k, u, W, C, N)) --k;
  while (k + 1 < (long long)N && slot_at_or_below((uint64_t)(k + 1), u, W, C, N)) ++k;
  return (uint32_t)(k + 1);
}

// offspring_end with the FP64 estimate x = C * (N / W) - u 2^-32 from a
// precomputed scale.  F = clamp(floor(x_exact), -1, N-1) + 1 where x_exact
// is the real-valued x.  For C <= W and N <= 2^30 the estimate is off by
// less than 2^-20 (four roundings of relative size 2^-53 on |x| < 2^31), so
// when x lies more than 2^-16 from an integer its floor is exact and the
// 128-bit checks are skipped; otherwise they decide.  The result is the
// exact F either way.
PF_HD uint32_t offspring_end_scaled(uint64_t C, uint64_t W, uint32_t N, uint32_t u, double scale,
                                    double uf) {
  const double x = (double)C * scale - uf;
  const double fl = floor(x);
  long long k = (long long)fl;
  if (k < -1) k = -1;
  if (k > (long long)N - 1) k = (long long)N - 1;
  const double fr = x - fl;
  if (fr > 0x1p-16 && fr < 1.0 - 0x1p-16) return (uint32_t)(k + 1);
  return offspring_end_settle(k, C, W, N, u);
}

// offspring_end_scaled for C = P + t2 with P exact (and Pd its double) and t2
// an integer-valued double: the estimate uses (Pd + t2) (relative error
// 2^-52, the same bound as above), the exact checks the 64-bit sum.
PF_HD uint32_t offspring_end_split(uint64_t P, double Pd, double t2, uint64_t W, uint32_t N, uint32_t u,
                                   double scale, double uf) {
  const double x = (Pd + t2) * scale - uf;
  const double fl = floor(x);
  long long k = (long long)fl;
  if (k < -1) k = -1;
  if (k > (long long)N - 1) k = (long long)N - 1;
  const double fr = x - fl;
  if (fr > 0x1p-16 && fr < 1.0 - 0x1p-16) return (uint32_t)(k + 1);
  return offspring_end_settle(k, P + (uint64_t)t2, W, N, u);
}

}  // namespace pfb
