/*
 * pf_oracle.c -- FP64 CPU restatement of the particle-filter step of
 * rsasaki0109/gnss_gpu, used ONLY as test infrastructure: by tests/, by
 * __graft_entry__.smoke() as the checker, and by bench.py's CPU-baseline leg.
 * Nothing in the product links or calls it.
 *
 * Sources restated (paths inside the reference project):
 *   predict.cu:7-21        init_kernel        -> orc_init
 *   predict.cu:23-38       predict_kernel     -> orc_predict, orc_pf_predict
 *   weight.cu:13-57        weight_kernel      -> orc_weight_*, orc_pf_weight
 *   pf_device.cu:19-26     Huber cost         -> orc_weight_* (mode 1)
 *   weight.cu:61-160       ESS                -> orc_stats, orc_pf_ess
 *   weight.cu:163-328      weighted mean      -> orc_stats, orc_pf_estimate
 *   resampling.cu:60-83,152 systematic search -> orc_systematic, orc_systematic_tiled
 *   resampling.cu:175-272  reference Megopolis -> orc_pf_megopolis_ref
 *   Chesser et al. arXiv:2109.13504, canonical Megopolis -> orc_megopolis
 *   particle_filter.py:129-175 update order   -> orc_epoch
 *   weight_3d.cu:14-177    building-aware likelihood (brute-force ray
 *                          casting, LOS/NLOS mixture) -> orc_los, orc_weight_3d
 * Random numbers: Philox4x32-10 from Salmon et al., SC'11, with this
 * project's counter layout (particle, epoch, tag, filter), so the oracle and
 * the CUDA path draw identical 32-bit words.  Normals: Box-Muller in FP64.
 *
 * Compile with -ffp-contract=off: orc_quantize must round exactly like the
 * device's sequence of IEEE double multiply, subtract and fma.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define TAG_INIT 0x01000000u
#define TAG_PREDICT 0x02000000u
#define TAG_SYS_U 0x03000000u
#define TAG_MEGO_OFF 0x04000000u
#define TAG_MEGO_U 0x05000000u
#define TAG_COMPAT_INIT 0x11000000u
#define TAG_COMPAT_PREDICT 0x12000000u
#define TAG_COMPAT_MEGO 0x13000000u

/* ------------------------------------------------------------ Philox */
void orc_philox10(const uint32_t in[4], uint32_t k0, uint32_t k1, uint32_t out[4]) {
  uint32_t c0 = in[0], c1 = in[1], c2 = in[2], c3 = in[3];
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    uint32_t n1 = (uint32_t)p1;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    uint32_t n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Box-Muller of the stateless (FP64) path: u1 = (a + 1/2) 2^-32,
 * u2 = b 2^-32 - 1/2. */
static void bm(uint32_t a, uint32_t b, double* n0, double* n1) {
  const double two_m32 = 2.3283064365386963e-10;
  double u1 = ((double)a + 0.5) * two_m32;
  double u2 = (double)b * two_m32 - 0.5;
  double r = sqrt(-2.0 * log(u1));
  double th = 6.283185307179586476925286766559 * u2;
  *n0 = r * cos(th);
  *n1 = r * sin(th);
}

/* Box-Muller of the engine (FP32 on the device): same u1, angle from the
 * top 24 bits of b, u2 = (b >> 8) 2^-24 - 1/2. */
static void bm24(uint32_t a, uint32_t b, double* n0, double* n1) {
  const double two_m32 = 2.3283064365386963e-10;
  double u1 = ((double)a + 0.5) * two_m32;
  double u2 = (double)(b >> 8) * 5.9604644775390625e-08 - 0.5;
  double r = sqrt(-2.0 * log(u1));
  double th = 6.283185307179586476925286766559 * u2;
  *n0 = r * cos(th);
  *n1 = r * sin(th);
}

/* Eight normals of one particle: words of (p, epoch, tag|0) then (tag|1). */
static void normals8(uint32_t p, uint32_t epoch, uint32_t tag, uint32_t fid, uint32_t k0,
                     uint32_t k1, int need, double nz[8]) {
  uint32_t c[4] = {p, epoch, tag, fid}, w[4];
  orc_philox10(c, k0, k1, w);
  bm24(w[0], w[1], &nz[0], &nz[1]);
  bm24(w[2], w[3], &nz[2], &nz[3]);
  if (need > 4) {
    c[2] = tag | 1u;
    orc_philox10(c, k0, k1, w);
    bm24(w[0], w[1], &nz[4], &nz[5]);
    bm24(w[2], w[3], &nz[6], &nz[7]);
  } else {
    nz[4] = nz[5] = nz[6] = nz[7] = 0.0;
  }
}

/* ------------------------------------------------ deterministic quantiser
 * q = floor(2^K exp(d)) for d = lw - max <= 0, with exactly the operation
 * sequence of the device (every step an IEEE-rounded double operation):
 * x = d log2(e), n = floor(x), f = x - n, t = f ln 2, e^t by its Taylor
 * series (1/j!, degree 13) in Horner form with fma, times 2^(K+n),
 * truncated.  Weights below 2^-40 of the largest quantise to zero. */
static double dmul(double a, double b) { volatile double r = a * b; return r; }
static double dsub(double a, double b) { volatile double r = a - b; return r; }

int orc_quant_exponent(int n) {
  int lg = 0;
  while ((1ll << lg) < (long long)n) ++lg;
  int k = 62 - lg;
  return k < 40 ? k : 40;
}

/* e^t for t in [0, ln 2): Taylor series of degree 13 in Horner form. */
static double exp_poly(double t) {
  double q = 1.6059043836821615e-10;
  q = fma(q, t, 2.0876756987868099e-09);
  q = fma(q, t, 2.5052108385441720e-08);
  q = fma(q, t, 2.7557319223985893e-07);
  q = fma(q, t, 2.7557319223985888e-06);
  q = fma(q, t, 2.4801587301587302e-05);
  q = fma(q, t, 1.9841269841269841e-04);
  q = fma(q, t, 1.3888888888888889e-03);
  q = fma(q, t, 8.3333333333333333e-03);
  q = fma(q, t, 4.1666666666666667e-02);
  q = fma(q, t, 1.6666666666666667e-01);
  q = fma(q, t, 0.5);
  q = fma(q, t, 1.0);
  q = fma(q, t, 1.0);
  return q;
}

uint64_t orc_quantize(double d, int K) {
  const double x = dmul(d, 1.4426950408889634074);
  if (!(x > -40.0)) return 0;
  const double n = floor(x);
  const double f = dsub(x, n);
  const double t = dmul(f, 0.69314718055994530942);
  return (uint64_t)ldexp(exp_poly(t), K + (int)n);
}

/* floor(v * r) for an integer v < 2^53 and 0 <= r <= 1, one rounded product. */
static uint64_t scale_floor(uint64_t v, double r) { return (uint64_t)dmul((double)v, r); }

/* Deterministic FP32 exponential of the engine's tiled CDF (the device's
 * exp2_frac_f32 / quantize_f32 / det_expf): x = d log2(e) (one rounded
 * product), n = floor(x), f = x - n (one rounded difference), 2^f from the
 * Taylor series of e^(f ln 2) (coefficients (ln 2)^k / k! rounded to FP32,
 * degree 9, Horner with fma), 2^n applied exactly. */
static float fmul32(float a, float b) { volatile float r = a * b; return r; }
static float fsub32(float a, float b) { volatile float r = a - b; return r; }
static float exp2_frac32(float f) {
  float q = 0x1.b5253ep-24f;
  q = fmaf(q, f, 0x1.62c022p-20f);
  q = fmaf(q, f, 0x1.ffcbfcp-17f);
  q = fmaf(q, f, 0x1.430912p-13f);
  q = fmaf(q, f, 0x1.5d87fep-10f);
  q = fmaf(q, f, 0x1.3b2ab6p-7f);
  q = fmaf(q, f, 0x1.c6b08ep-5f);
  q = fmaf(q, f, 0x1.ebfbep-3f);
  q = fmaf(q, f, 0x1.62e43p-1f);
  q = fmaf(q, f, 0x1.0p+0f);
  return q;
}
static float pow2f32(int m) {
  const uint32_t b = (uint32_t)(127 + m) << 23;
  float r;
  memcpy(&r, &b, sizeof(r));
  return r;
}
uint64_t orc_quantize_f32(float d, int K) {
  const float x = fmul32(d, 0x1.715476p+0f);
  if (!(x > -40.0f)) return 0;
  const float n = floorf(x);
  const float p = exp2_frac32(fsub32(x, n));
  volatile float v = p * pow2f32(K + (int)n);
  return (uint64_t)v;
}
float orc_det_expf(float d) {
  const float x = fmul32(d, 0x1.715476p+0f);
  if (!(x > -126.0f)) return 0.0f;
  const float n = floorf(x);
  volatile float v = exp2_frac32(fsub32(x, n)) * pow2f32((int)n);
  return v;
}

/* FP32 log-weights of the engine: the shift lw - max is exact in FP64. */
void orc_quantize_all(const float* lw, int n, float max_lw, uint64_t* q) {
  const int K = orc_quant_exponent(n);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) q[i] = orc_quantize((double)lw[i] - (double)max_lw, K);
}

void orc_quantize_all64(const double* lw, int n, double max_lw, uint64_t* q) {
  const int K = orc_quant_exponent(n);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) q[i] = orc_quantize(lw[i] - max_lw, K);
}

/* ------------------------------------------------------------ systematic
 * resampling.cu:69-77: for slot k the lower-bound search over [0, N-1]
 * for the first i with !(cdf[i] < (u + k)/N).  With an integer CDF C and
 * total W the comparison is exact: C_i*N*2^32 < (k*2^32 + u32)*W.
 * Returns 0 on success, -1 if every weight quantised to zero. */
static int systematic_from_q(uint64_t* C, int n, uint32_t u32, int* anc, uint64_t* wq_out) {
  uint64_t acc = 0;
  for (int i = 0; i < n; ++i) {
    acc += C[i];
    C[i] = acc;
  }
  const uint64_t W = acc;
  if (wq_out) *wq_out = W;
  if (W == 0) return -1;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < n; ++k) {
    const unsigned __int128 rhs = (unsigned __int128)((((uint64_t)k) << 32) | u32) * W;
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      int mid = (lo + hi) / 2;
      unsigned __int128 lhs = ((unsigned __int128)C[mid] * (uint64_t)n) << 32;
      if (lhs < rhs) lo = mid + 1;
      else hi = mid;
    }
    anc[k] = lo;
  }
  return 0;
}

int orc_systematic(const float* lw, int n, float max_lw, uint32_t u32, int* anc, uint64_t* wq_out) {
  uint64_t* C = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
  if (!C) return -2;
  orc_quantize_all(lw, n, max_lw, C);
  int r = systematic_from_q(C, n, u32, anc, wq_out);
  free(C);
  return r;
}

int orc_systematic64(const double* lw, int n, double max_lw, uint32_t u32, int* anc, uint64_t* wq_out) {
  uint64_t* C = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
  if (!C) return -2;
  orc_quantize_all64(lw, n, max_lw, C);
  int r = systematic_from_q(C, n, u32, anc, wq_out);
  free(C);
  return r;
}

/* ------------------------------------------- tiled integer CDF (engine)
 * The engine quantises each 128-particle segment (one warp) against its own
 * maximum wm_s and rescales exactly, with one rounded product and a floor
 * per level (tiles of 1024 particles = 8 segments, then the filter):
 *   q_i   = floor(2^K e^(lw_i - wm_s)),       c_i = prefix of q inside s
 *   (e^ here the deterministic FP32 exponential orc_quantize_f32 /
 *   orc_det_expf; products with it one rounded FP64 multiply)
 *   S_s   = c at the segment's end,            rho_s = e^(wm_s - tm_t)
 *   Q_s   = floor(S_s rho_s),                  E_s = prefix of Q over s in t
 *   S_t   = sum of Q_s,                        r_t = e^(tm_t - M)
 *   Q_t   = floor(S_t r_t),                    P_t = prefix of Q_t
 *   C_i   = P_t + floor((E_s + floor(c_i rho_s)) r_t),  W = sum of Q_t
 * (tm_t the tile maximum, M the filter maximum).  C is non-decreasing and ends at W; slot k's ancestor
 * is the first i with (k 2^32 + u) W <= C_i N 2^32, the predicate of
 * resampling.cu:69-77 as for the plain integer CDF. */
int orc_systematic_tiled(const float* lw, int n, uint32_t u32, int* anc, uint64_t* wq_out, float* max_out) {
  const int K = orc_quant_exponent(n);
  const int nt = (n + 1023) / 1024;
  uint64_t* C = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
  float* tm = (float*)malloc(sizeof(float) * (size_t)nt);
  uint64_t* St = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)nt);
  double* rho = (double*)malloc(sizeof(double) * (size_t)nt * 8);
  uint64_t* E = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)nt * 8);
  if (!C || !tm || !St || !rho || !E) {
    free(C); free(tm); free(St); free(rho); free(E);
    return -2;
  }
  float M = -INFINITY;
#pragma omp parallel for schedule(static) reduction(max : M)
  for (int t = 0; t < nt; ++t) {
    float wm[8];
    uint64_t S[8];
    float tmax = -INFINITY;
    for (int s = 0; s < 8; ++s) {
      const int a = t * 1024 + s * 128, b = a + 128 < n ? a + 128 : n;
      float m = -INFINITY;
      for (int i = a; i < b; ++i) m = fmaxf(m, lw[i]);
      uint64_t run = 0;
      for (int i = a; i < b; ++i) {
        run += orc_quantize_f32(fsub32(lw[i], m), K);
        C[i] = run;
      }
      wm[s] = m;
      S[s] = run;
      tmax = fmaxf(tmax, m);
    }
    uint64_t acc = 0;
    for (int s = 0; s < 8; ++s) {
      const double r = S[s] ? (double)orc_det_expf(fsub32(wm[s], tmax)) : 0.0;
      rho[t * 8 + s] = r;
      E[t * 8 + s] = acc;
      acc += S[s] ? scale_floor(S[s], r) : 0;
    }
    St[t] = acc;
    tm[t] = tmax;
    M = fmaxf(M, tmax);
  }
  if (max_out) *max_out = M;
  uint64_t W = 0;
  double* rt = (double*)malloc(sizeof(double) * (size_t)nt);
  uint64_t* P = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)nt);
  for (int t = 0; t < nt; ++t) {
    rt[t] = St[t] ? (double)orc_det_expf(fsub32(tm[t], M)) : 0.0;
    P[t] = W;
    W += St[t] ? scale_floor(St[t], rt[t]) : 0;
  }
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    const int t = i / 1024, s = (i % 1024) / 128;
    const uint64_t inner = E[t * 8 + s] + scale_floor(C[i], rho[t * 8 + s]);
    C[i] = P[t] + scale_floor(inner, rt[t]);
  }
  free(rt); free(P); free(tm); free(St); free(rho); free(E);
  if (wq_out) *wq_out = W;
  int r = 0;
  if (W == 0) {
    r = -1;
  } else {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n; ++k) {
      const unsigned __int128 rhs = (unsigned __int128)((((uint64_t)k) << 32) | u32) * W;
      int lo = 0, hi = n - 1;
      while (lo < hi) {
        int mid = (lo + hi) / 2;
        unsigned __int128 lhs = ((unsigned __int128)C[mid] * (uint64_t)n) << 32;
        if (lhs < rhs) lo = mid + 1;
        else hi = mid;
      }
      anc[k] = lo;
    }
  }
  free(C);
  return r;
}

/* ------------------------------------------------------ canonical Megopolis
 * Chesser et al. (arXiv:2109.13504): for each slot k the chain starts at
 * ancestor k; iteration b proposes j = (k + o_{b,g}) mod N with an offset
 * shared by the 32-slot segment g = k / 32 and accepts with probability
 * min(1, w_j / w_ancestor).  Draws (the engine's layout): the offsets of
 * iteration b for the four segments g = 32 t + 8 r + w (tile t, r = 0..3)
 * are the words r of Philox (8 t + w, epoch, TAG_MEGO_OFF | b, filter); the
 * acceptance uniform of slot k at iteration b is the 16-bit half (b even:
 * low) of word (b % 8) / 2 of Philox (k, epoch, TAG_MEGO_U | b / 8, filter),
 * as (h + 1/2) 2^-16. */
void orc_megopolis(const float* lw, int n, int iters, uint32_t k0, uint32_t k1, uint32_t epoch,
                   uint32_t fid, int* anc) {
#pragma omp parallel for schedule(static)
  for (int k = 0; k < n; ++k) {
    const uint32_t g = (uint32_t)(k / 32);
    const uint32_t quad = (g / 32) * 8 + (g % 8), r = (g % 32) / 8;
    int a = k;
    double la = (double)lw[k];
    uint32_t uw[4];
    for (int b = 0; b < iters; ++b) {
      uint32_t ow[4];
      uint32_t co[4] = {quad, epoch, TAG_MEGO_OFF | (uint32_t)b, fid};
      orc_philox10(co, k0, k1, ow);
      if ((b & 7) == 0) {
        uint32_t cu[4] = {(uint32_t)k, epoch, TAG_MEGO_U | (uint32_t)(b >> 3), fid};
        orc_philox10(cu, k0, k1, uw);
      }
      const uint32_t w32 = uw[(b & 7) >> 1];
      const uint32_t h = (b & 1) ? (w32 >> 16) : (w32 & 0xFFFFu);
      const uint32_t o = (uint32_t)(((uint64_t)ow[r] * (uint64_t)(uint32_t)n) >> 32);
      int cand = k + (int)o;
      if (cand >= n) cand -= n;
      const double lc = (double)lw[cand];
      const double u = ((double)h + 0.5) * 1.52587890625e-05;
      if (log(u) < lc - la) {
        a = cand;
        la = lc;
      }
    }
    anc[k] = a;
  }
}

/* ------------------------------------------------------ engine-semantics step
 * State: D = 3 + nclk components (local E, N, U offsets about an ECEF anchor
 * with rotation rot (rows E, N, U), then clock offsets about clk_anchor).
 */
void orc_local_to_ecef(const double rot[9], const double anchor[3], double e, double nn, double u,
                       double out[3]) {
  out[0] = anchor[0] + rot[0] * e + rot[3] * nn + rot[6] * u;
  out[1] = anchor[1] + rot[1] * e + rot[4] * nn + rot[7] * u;
  out[2] = anchor[2] + rot[2] * e + rot[5] * nn + rot[8] * u;
}

/* predict.cu:7-21 -- N(0, spread) about the anchor. */
void orc_init(int n, int D, float spread_pos, float spread_clk, uint32_t k0, uint32_t k1,
              uint32_t fid, double* x) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    double nz[8];
    normals8((uint32_t)i, 0u, TAG_INIT, fid, k0, k1, D, nz);
    for (int d = 0; d < D; ++d) x[(size_t)d * n + i] = (d < 3 ? (double)spread_pos : (double)spread_clk) * nz[d];
  }
}

/* predict.cu:23-38 -- x += v dt + N(0, sigma), with the re-centring shift
 * subtracted; src may be gathered through anc (the previous resample). */
void orc_predict(int n, int D, const double* x_prev, const int* anc, const double* disp,
                 const double* shift, const float* sigma, int do_predict, uint32_t k0, uint32_t k1,
                 uint32_t epoch, uint32_t fid, double* x_out) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    const int a = anc ? anc[i] : i;
    double nz[8];
    if (do_predict) normals8((uint32_t)i, epoch, TAG_PREDICT, fid, k0, k1, D, nz);
    for (int d = 0; d < D; ++d) {
      double v = x_prev[(size_t)d * n + a] - shift[d];
      if (do_predict) v += (d < 3 ? disp[d] : 0.0) + (double)sigma[d] * nz[d];
      x_out[(size_t)d * n + i] = v;
    }
  }
}

/* weight.cu:13-57 (mode 0, Gaussian) and pf_device.cu:19-26 (mode 1, Huber):
 * the residual pr - (|sat - p| + cb) in FP64 with p = anchor + R^T d.
 * sats: [n_sat][5] = x, y, z, pr, w; clk[s] picks the clock state. */
void orc_weight(int n, int D, const double* x, const double anchor[3], const double* clk_anchor,
                const double rot[9], int n_sat, const double* sats, const int* clk, double sigma_pr,
                int mode, double huber_k, const double* lw_base, double* lw_out) {
  const double inv_s2 = 1.0 / (sigma_pr * sigma_pr);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    double p[3];
    orc_local_to_ecef(rot, anchor, x[i], x[(size_t)n + i], x[(size_t)2 * n + i], p);
    double acc = lw_base ? lw_base[i] : 0.0;
    for (int s = 0; s < n_sat; ++s) {
      const double* sv = sats + 5 * s;
      const double dx = p[0] - sv[0], dy = p[1] - sv[1], dz = p[2] - sv[2];
      const double r = sqrt(dx * dx + dy * dy + dz * dz);
      const int c = clk[s];
      const double cb = clk_anchor[c] + x[(size_t)(3 + c) * n + i];
      const double res = sv[3] - (r + cb);
      if (mode == 0) {
        acc += -0.5 * sv[4] * res * res * inv_s2;
      } else {
        const double z = fabs(res) / sigma_pr;
        const double rho = (z < huber_k) ? 0.5 * z * z : huber_k * z - 0.5 * huber_k * huber_k;
        acc += -sv[4] * rho;
      }
    }
    lw_out[i] = acc;
  }
  (void)D;
}

/* weight.cu:61-160,163-328 -- max-shifted sums.  out:
 * [0] max lw, [1] W, [2] W2, [3] ESS, [4..4+D) weighted mean offsets,
 * [11..14) ECEF estimate, [14..18) clock estimates, [18..24) 3x3 covariance
 * (xx, xy, xz, yy, yz, zz) of the local frame. */
void orc_stats(int n, int D, const double* x, const double* lw, const double anchor[3],
               const double* clk_anchor, const double rot[9], double* out) {
  double m = -INFINITY;
  for (int i = 0; i < n; ++i)
    if (lw[i] > m) m = lw[i];
  double W = 0, W2 = 0, sx[7] = {0}, sxx[6] = {0};
#pragma omp parallel
  {
    double w_ = 0, w2_ = 0, sx_[7] = {0}, sxx_[6] = {0};
#pragma omp for schedule(static) nowait
    for (int i = 0; i < n; ++i) {
      const double w = exp(lw[i] - m);
      w_ += w;
      w2_ += w * w;
      for (int d = 0; d < D; ++d) sx_[d] += w * x[(size_t)d * n + i];
      const double e = x[i], nn = x[(size_t)n + i], u = x[(size_t)2 * n + i];
      sxx_[0] += w * e * e; sxx_[1] += w * e * nn; sxx_[2] += w * e * u;
      sxx_[3] += w * nn * nn; sxx_[4] += w * nn * u; sxx_[5] += w * u * u;
    }
#pragma omp critical
    {
      W += w_;
      W2 += w2_;
      for (int d = 0; d < 7; ++d) sx[d] += sx_[d];
      for (int k = 0; k < 6; ++k) sxx[k] += sxx_[k];
    }
  }
  memset(out, 0, sizeof(double) * 24);
  out[0] = m;
  out[1] = W;
  out[2] = W2;
  out[3] = W * W / W2;
  double mu[7] = {0};
  for (int d = 0; d < D; ++d) mu[d] = sx[d] / W;
  for (int d = 0; d < D; ++d) out[4 + d] = mu[d];
  orc_local_to_ecef(rot, anchor, mu[0], mu[1], mu[2], out + 11);
  for (int c = 0; c < D - 3; ++c) out[14 + c] = clk_anchor[c] + mu[3 + c];
  out[18] = sxx[0] / W - mu[0] * mu[0];
  out[19] = sxx[1] / W - mu[0] * mu[1];
  out[20] = sxx[2] / W - mu[0] * mu[2];
  out[21] = sxx[3] / W - mu[1] * mu[1];
  out[22] = sxx[4] / W - mu[1] * mu[2];
  out[23] = sxx[5] / W - mu[2] * mu[2];
}

/* ------------------------------------------------------- full CPU epoch
 * particle_filter.py:102-175 order on an FP64 state (the CPU baseline):
 * predict, weight (overwrite), ESS, systematic resample (gather) when
 * ESS < thr * N, weighted-mean estimate.  Returns 1 if it resampled. */
int orc_epoch(int n, int D, double* x, double* x_tmp, double* lw, float* lw32, int* anc,
              const double anchor[3], const double* clk_anchor, const double rot[9],
              const double disp[3], const float* sigma, uint32_t k0, uint32_t k1, uint32_t epoch,
              int n_sat, const double* sats, const int* clk, double sigma_pr, double ess_thr,
              double* stats_out) {
  static const double zero_shift[8] = {0};
  orc_predict(n, D, x, NULL, disp, zero_shift, sigma, 1, k0, k1, epoch, 0u, x_tmp);
  orc_weight(n, D, x_tmp, anchor, clk_anchor, rot, n_sat, sats, clk, sigma_pr, 0, 0.0, NULL, lw);
  orc_stats(n, D, x_tmp, lw, anchor, clk_anchor, rot, stats_out);
  int rs = stats_out[3] < ess_thr * (double)n;
  if (rs) {
    uint32_t c[4] = {0u, epoch, TAG_SYS_U, 0u}, w[4];
    orc_philox10(c, k0, k1, w);
    orc_systematic64(lw, n, stats_out[0], w[0], anc, NULL);
    (void)lw32;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i)
      for (int d = 0; d < D; ++d) x[(size_t)d * n + i] = x_tmp[(size_t)d * n + anc[i]];
  } else {
    memcpy(x, x_tmp, sizeof(double) * (size_t)D * n);
  }
  return rs;
}

/* --------------------------------------- reference host-array semantics */
void orc_pf_initialize(double* px, double* py, double* pz, double* pcb, double ix, double iy,
                       double iz, double icb, double sp, double scb, int n, unsigned long long seed) {
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    uint32_t c[4] = {(uint32_t)i, 0u, TAG_COMPAT_INIT, 0u}, w[4];
    orc_philox10(c, k0, k1, w);
    double a0, a1, b0, b1;
    bm(w[0], w[1], &a0, &a1);
    bm(w[2], w[3], &b0, &b1);
    px[i] = ix + a0 * sp;
    py[i] = iy + a1 * sp;
    pz[i] = iz + b0 * sp;
    pcb[i] = icb + b1 * scb;
  }
}

void orc_pf_predict(double* px, double* py, double* pz, double* pcb, double vx, double vy,
                    double vz, double dt, double sp, double scb, int n, unsigned long long seed,
                    int step) {
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    uint32_t c[4] = {(uint32_t)i, (uint32_t)step, TAG_COMPAT_PREDICT, 0u}, w[4];
    orc_philox10(c, k0, k1, w);
    double a0, a1, b0, b1;
    bm(w[0], w[1], &a0, &a1);
    bm(w[2], w[3], &b0, &b1);
    px[i] += vx * dt + a0 * sp;
    py[i] += vy * dt + a1 * sp;
    pz[i] += vz * dt + b0 * sp;
    pcb[i] += b1 * scb;
  }
}

void orc_pf_weight(const double* px, const double* py, const double* pz, const double* pcb,
                   const double* sat, const double* pr, const double* ws, double* lw, int n,
                   int n_sat, double sigma_pr) {
  const double inv_s2 = 1.0 / (sigma_pr * sigma_pr);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    double acc = 0.0;
    for (int s = 0; s < n_sat; ++s) {
      const double dx = px[i] - sat[3 * s], dy = py[i] - sat[3 * s + 1], dz = pz[i] - sat[3 * s + 2];
      const double r = sqrt(dx * dx + dy * dy + dz * dz);
      const double res = pr[s] - (r + pcb[i]);
      acc += -0.5 * ws[s] * res * res * inv_s2;
    }
    lw[i] = acc;
  }
}

double orc_pf_ess(const double* lw, int n) {
  double m = -INFINITY;
  for (int i = 0; i < n; ++i)
    if (lw[i] > m) m = lw[i];
  double s = 0, s2 = 0;
  for (int i = 0; i < n; ++i) {
    double w = exp(lw[i] - m);
    s += w;
    s2 += w * w;
  }
  return s * s / s2;
}

void orc_pf_estimate(const double* px, const double* py, const double* pz, const double* pcb,
                     const double* lw, double* out, int n) {
  double m = -INFINITY;
  for (int i = 0; i < n; ++i)
    if (lw[i] > m) m = lw[i];
  double s = 0, a = 0, b = 0, c = 0, d = 0;
  for (int i = 0; i < n; ++i) {
    double w = exp(lw[i] - m);
    s += w;
    a += w * px[i];
    b += w * py[i];
    c += w * pz[i];
    d += w * pcb[i];
  }
  out[0] = a / s;
  out[1] = b / s;
  out[2] = c / s;
  out[3] = d / s;
}

/* resampling.cu:152 offset and :60-83 search, ancestors only. */
int orc_pf_systematic_ancestors(const double* lw, int n, unsigned long long seed, int* anc) {
  double m = -INFINITY;
  for (int i = 0; i < n; ++i)
    if (lw[i] > m) m = lw[i];
  double u0 = (double)(seed % 1000000ull) / (1000000.0 * (double)n);
  double v = floor(u0 * 4294967296.0);
  uint32_t u32 = (uint32_t)(v < 0 ? 0 : (v > 4294967295.0 ? 4294967295.0 : v));
  return orc_systematic64(lw, n, m, u32, anc, NULL);
}

/* resampling.cu:175-272 chain on ancestor indices (the reference's
 * acceptance against the slot's own weight), same Philox words as the
 * CUDA stateless path. */
static double u53(uint32_t a, uint32_t b) {
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

void orc_pf_megopolis_ref_ancestors(const double* lw, int n, int iters, unsigned long long seed,
                                    int* anc) {
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  int* a = (int*)malloc(sizeof(int) * (size_t)n);
  int* b = (int*)malloc(sizeof(int) * (size_t)n);
  for (int k = 0; k < n; ++k) a[k] = k;
  for (int it = 0; it < iters; ++it) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n; ++k) {
      uint32_t c[4] = {(uint32_t)k, (uint32_t)it, TAG_COMPAT_MEGO, 0u}, w[4];
      orc_philox10(c, k0, k1, w);
      const double U1 = u53(w[0], w[1]), U2 = u53(w[2], w[3]);
      const long long off = (long long)(U1 * (double)(n - 1)) + 1;
      const int j = (int)(((long long)k + off) % n);
      const double alpha = fmin(1.0, exp(lw[j] - lw[k]));
      b[k] = (U2 < alpha) ? a[j] : a[k];
    }
    int* t = a;
    a = b;
    b = t;
  }
  memcpy(anc, a, sizeof(int) * (size_t)n);
  free(a);
  free(b);
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* ----------------------------------------------------------------------
 * Building-aware likelihood (weight_3d.cu:14-177): Moller-Trumbore in FP64
 * against every triangle, then the LOS/NLOS mixture per satellite.
 * tris: n_tri x 9 (v0, v1, v2, ECEF). */
static int orc_tri_hit(const double o[3], const double d[3], const double* t, double max_t) {
  const double e1[3] = {t[3] - t[0], t[4] - t[1], t[5] - t[2]};
  const double e2[3] = {t[6] - t[0], t[7] - t[1], t[8] - t[2]};
  const double h[3] = {d[1] * e2[2] - d[2] * e2[1], d[2] * e2[0] - d[0] * e2[2], d[0] * e2[1] - d[1] * e2[0]};
  const double a = e1[0] * h[0] + e1[1] * h[1] + e1[2] * h[2];
  if (fabs(a) < 1e-12) return 0;
  const double f = 1.0 / a;
  const double s[3] = {o[0] - t[0], o[1] - t[1], o[2] - t[2]};
  const double u = f * (s[0] * h[0] + s[1] * h[1] + s[2] * h[2]);
  if (u < 0.0 || u > 1.0) return 0;
  const double q[3] = {s[1] * e1[2] - s[2] * e1[1], s[2] * e1[0] - s[0] * e1[2], s[0] * e1[1] - s[1] * e1[0]};
  const double v = f * (d[0] * q[0] + d[1] * q[1] + d[2] * q[2]);
  if (v < 0.0 || u + v > 1.0) return 0;
  const double tt = f * (e2[0] * q[0] + e2[1] * q[1] + e2[2] * q[2]);
  return tt > 1e-6 && tt < max_t;
}

static int orc_blocked(const double p[3], const double sat[3], const double* tris, int n_tri) {
  const double v[3] = {sat[0] - p[0], sat[1] - p[1], sat[2] - p[2]};
  const double dist = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  const double d[3] = {v[0] / dist, v[1] / dist, v[2] / dist};
  for (int t = 0; t < n_tri; ++t)
    if (orc_tri_hit(p, d, tris + 9 * (size_t)t, dist)) return 1;
  return 0;
}

/* los[r * n_sat + s] = 1 when rx[r] sees sat[r * n_sat + s]. */
void orc_los(const double* rx, const double* sat, int n_rx, int n_sat, const double* tris, int n_tri,
             unsigned char* los) {
#pragma omp parallel for schedule(dynamic, 16)
  for (long long i = 0; i < (long long)n_rx * n_sat; ++i)
    los[i] = orc_blocked(rx + 3 * (i / n_sat), sat + 3 * i, tris, n_tri) ? 0 : 1;
}

static double orc_mix(double los, double nlos, double p) {
  if (p <= 0.0) return los;
  if (p >= 1.0) return nlos;
  const double a = log(1.0 - p) + los, b = log(p) + nlos;
  const double m = a > b ? a : b;
  return m + log(exp(a - m) + exp(b - m));
}

/* pos: n x 3 ECEF, cb: n; sats: n_sat x 5 (x, y, z, pr, w).  lw_out: n;
 * blocked_out (n x n_sat, may be NULL). */
void orc_weight_3d(int n, const double* pos, const double* cb, int n_sat, const double* sats, const double* tris,
                   int n_tri, double sigma_los, double sigma_nlos, double nlos_bias, double p_blocked,
                   double p_clear, double* lw_out, unsigned char* blocked_out) {
  const double il = 1.0 / (sigma_los * sigma_los), in = 1.0 / (sigma_nlos * sigma_nlos);
#pragma omp parallel for schedule(dynamic, 16)
  for (int j = 0; j < n; ++j) {
    double acc = 0.0;
    for (int s = 0; s < n_sat; ++s) {
      const double* sv = sats + 5 * (size_t)s;
      const int blk = orc_blocked(pos + 3 * (size_t)j, sv, tris, n_tri);
      if (blocked_out) blocked_out[(size_t)j * n_sat + s] = (unsigned char)blk;
      const double dx = pos[3 * j] - sv[0], dy = pos[3 * j + 1] - sv[1], dz = pos[3 * j + 2] - sv[2];
      const double r = sv[3] - (sqrt(dx * dx + dy * dy + dz * dz) + cb[j]);
      const double los = -0.5 * sv[4] * r * r * il;
      const double rn = r > 0.0 ? r - nlos_bias : r;
      const double nlos = -0.5 * sv[4] * rn * rn * in;
      acc += orc_mix(los, nlos, blk ? p_blocked : p_clear);
    }
    lw_out[j] = acc;
  }
}
