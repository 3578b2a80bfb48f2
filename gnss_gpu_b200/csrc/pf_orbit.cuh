// pf_orbit.cuh -- satellite positions and clocks from broadcast navigation
// records, and the Sagnac-corrected geometric range: the input formation
// upstream of the filter step.
//
//  * Kepler broadcasts (GPS, Galileo, QZSS, BeiDou MEO/IGSO): IS-GPS-200
//    orbit with per-system gravitational parameter, earth rotation rate and
//    relativistic constant (src/ephemeris/ephemeris.cu:14-104 for GPS;
//    python/gnss_gpu/ephemeris.py:36-64,428-512 for the other systems and the
//    BDT offset).
//  * GLONASS: RK4 integration of the PZ-90 equations of motion from the
//    broadcast state, fixed steps plus one residual step
//    (python/gnss_gpu/orbit_glonass.py:67-170).
//  * Sagnac: rotation of the satellite about the earth axis by the signal
//    transit time (python/gnss_gpu/range_model.py:12-40).
//
// One thread per (epoch, satellite); FP64 throughout.  The work is O(S) per
// epoch and tiny next to the filter step, so the kernels are written for
// batching many epochs into one launch, not for bandwidth.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "../../include/gnss_pf_b200.h"

namespace pfb {

constexpr double kWeekSec = 604800.0;
constexpr double kGpstMinusBdt = 14.0;  // gnss_time_scales.py:25
constexpr double kGpstMinusUtc = 18.0;  // gnss_time_scales.py:28
constexpr double kCLight = 299792458.0;
constexpr double kOmegaSagnac = 7.2921151467e-5;  // range_model.py:8

// GLONASS PZ-90 constants (orbit_glonass.py:26-36).
constexpr double kGloRe = 6378136.0;
constexpr double kGloMu = 3.9860044e14;
constexpr double kGloJ2 = 1.0826257e-3;
constexpr double kGloOmega = 7.292115e-5;
constexpr double kGloStep = 60.0;
// Integration steps one record may take: half a week at 1 s per step.
constexpr long kGloMaxSteps = 1L << 20;
// Stored GLONASS states per record and direction (k_glo_table) and the
// scratch they may take per call.
constexpr int kGloTable = 64;
constexpr size_t kGloTableBytes = 64u << 20;

struct OrbitConsts {
  double mu, omega_e, rel_f;
};

// ephemeris.py:55-63: Galileo, QZSS and BeiDou constants; GPS otherwise.
__host__ __device__ inline OrbitConsts orbit_consts(int system) {
  if (system == 'E') return {3.986004418e14, 7.2921151467e-5, -4.442807309e-10};
  if (system == 'C') return {3.986004418e14, 7.292115e-5, -4.442807309e-10};
  return {3.986005e14, 7.2921151467e-5, -4.442807633e-10};  // 'G', 'J' and the rest
}

// gnss_time_scales.py:34-47 (fold into [0, week)).  Finite values only; the
// folding loops are bounded, with fmod past 64 weeks.
__host__ __device__ inline double unwrap_week(double v) {
  if (!isfinite(v)) return v;
  if (fabs(v) > 64.0 * kWeekSec) {
    v = fmod(v, kWeekSec);
    if (v < 0.0) v += kWeekSec;
    return v;
  }
  while (v < 0.0) v += kWeekSec;
  while (v >= kWeekSec) v -= kWeekSec;
  return v;
}

// gnss_time_scales.py:50-63: GPST receive time in the record's time scale.
__host__ __device__ inline double broadcast_rx_sow(int system, double t) {
  if (system == 'C') return unwrap_week(t - kGpstMinusBdt);
  if (system == 'R') return unwrap_week(t - kGpstMinusUtc);
  return t;
}

__host__ __device__ inline double wrap_half_week(double dt) {
  if (dt > kWeekSec / 2.0) dt -= kWeekSec;
  if (dt < -kWeekSec / 2.0) dt += kWeekSec;
  return dt;
}

// Kepler's equation by Newton's method from E = M, at most 10 updates,
// stopping once |dE| < 1e-15 (ephemeris.cu:14-22, ephemeris.py:417-425).
__device__ inline double kepler_solve(double M, double e) {
  double E = M;
  for (int k = 0; k < 10; ++k) {
    const double dE = (M - E + e * sin(E)) / (1.0 - e * cos(E));
    E += dE;
    if (fabs(dE) < 1e-15) break;
  }
  return E;
}

// Position (ECEF, m) and clock correction (s) of a Kepler record at GPST
// second of week t (ephemeris.py:428-512; the GPS-only kernel of
// ephemeris.cu:24-104 is system 'G').  The record's tgd is subtracted as
// stored; callers put the group delay they want there (0 to omit it).
__device__ inline void kepler_orbit(const pf_ephemeris_t& k, int system, double t, double* pos,
                                    double* clk) {
  const OrbitConsts c = orbit_consts(system);
  const double a = k.sqrt_a * k.sqrt_a;
  const double n = sqrt(c.mu / (a * a * a)) + k.delta_n;
  const double rx = broadcast_rx_sow(system, t);
  const double tk = wrap_half_week(rx - k.toe);
  const double E = kepler_solve(k.M0 + n * tk, k.e);
  const double sE = sin(E), cE = cos(E);
  const double den = 1.0 - k.e * cE;
  const double v = atan2(sqrt(1.0 - k.e * k.e) * sE / den, (cE - k.e) / den);
  const double phi = v + k.omega;
  const double s2 = sin(2.0 * phi), c2 = cos(2.0 * phi);
  const double u = phi + (k.cuc * c2 + k.cus * s2);
  const double r = a * (1.0 - k.e * cE) + (k.crc * c2 + k.crs * s2);
  const double inc = k.i0 + k.idot * tk + (k.cic * c2 + k.cis * s2);
  const double xp = r * cos(u), yp = r * sin(u);
  const double Om = k.omega0 + (k.omega_dot - c.omega_e) * tk - c.omega_e * k.toe;
  const double cO = cos(Om), sO = sin(Om), ci = cos(inc), si = sin(inc);
  pos[0] = xp * cO - yp * ci * sO;
  pos[1] = xp * sO + yp * ci * cO;
  pos[2] = yp * si;
  const double dt = wrap_half_week(rx - k.toc);
  const double dtr = c.rel_f * k.e * k.sqrt_a * sE;
  *clk = k.af0 + k.af1 * dt + k.af2 * dt * dt + dtr - k.tgd;
}

// PZ-90 equations of motion with the broadcast luni-solar acceleration
// (orbit_glonass.py:67-92): x = (p, v), returns dx/dt.
__device__ inline void glo_deriv(const double* x, const double* acc, double* d) {
  const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
  if (!(r2 > 0.0) || !isfinite(r2)) {
    for (int i = 0; i < 6; ++i) d[i] = 0.0;
    return;
  }
  const double r3 = r2 * sqrt(r2);
  const double w2 = kGloOmega * kGloOmega;
  const double at = 1.5 * kGloJ2 * kGloMu * (kGloRe * kGloRe) / r2 / r3;
  const double bt = 5.0 * x[2] * x[2] / r2;
  const double ct = -kGloMu / r3 - at * (1.0 - bt);
  d[0] = x[3];
  d[1] = x[4];
  d[2] = x[5];
  d[3] = (ct + w2) * x[0] + 2.0 * kGloOmega * x[4] + acc[0];
  d[4] = (ct + w2) * x[1] - 2.0 * kGloOmega * x[3] + acc[1];
  d[5] = (ct - 2.0 * at) * x[2] + acc[2];
}

// One classic RK4 step of h seconds in place (orbit_glonass.py:95-111).
__device__ inline void glo_rk4(double h, double* x, const double* acc) {
  double k1[6], k2[6], k3[6], k4[6], w[6];
  glo_deriv(x, acc, k1);
  for (int i = 0; i < 6; ++i) w[i] = x[i] + k1[i] * (h / 2.0);
  glo_deriv(w, acc, k2);
  for (int i = 0; i < 6; ++i) w[i] = x[i] + k2[i] * (h / 2.0);
  glo_deriv(w, acc, k3);
  for (int i = 0; i < 6; ++i) w[i] = x[i] + k3[i] * h;
  glo_deriv(w, acc, k4);
  for (int i = 0; i < 6; ++i) x[i] += (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]) * (h / 6.0);
}

// Full steps of the GLONASS integration of a record at GPST second of
// week t and what is left for the residual step: the loop of
// orbit_glonass.py:122-150 without the arithmetic (rem decremented in the
// same order, so it is bit-identical).  Returns false past kGloMaxSteps.
__device__ inline bool glo_plan(const pf_glonass_state_t& g, double t, double step, double& el, double& base,
                                long& k, double& rem) {
  el = wrap_half_week(broadcast_rx_sow('R', t) - g.toe);
  base = el < 0.0 ? -step : step;
  rem = el;
  k = 0;
  // a NaN time takes no step (the reference returns the broadcast position
  // with a NaN clock); an infinite one runs into the step bound
  while (fabs(rem) >= fabs(base)) {  // |base| >= 1 s, so |rem| > 1e-9 here
    if (++k > kGloMaxSteps) return false;
    rem -= base;
  }
  return true;
}

// GLONASS position and clock at GPST second of week t: align to the
// record's UTC-based scale, integrate from toe in steps of `step` seconds
// with one residual step (orbit_glonass.py:122-170).  `tbl` (may be null)
// holds the states after 1..kc full steps from toe in this direction, shared
// by every epoch of the record: the walk starts from the deepest stored
// state instead of from toe, with the same RK4 steps in the same order, so
// the result is the same bit for bit.  Returns false (outputs NaN) past
// kGloMaxSteps steps.
__device__ inline bool glonass_orbit(const pf_glonass_state_t& g, double t, double step, const double* tbl,
                                     int kc, double* pos, double* clk) {
  double el, base, rem;
  long k;
  if (!glo_plan(g, t, step, el, base, k, rem)) {
    pos[0] = pos[1] = pos[2] = *clk = nan("");
    return false;
  }
  double x[6] = {g.pos[0], g.pos[1], g.pos[2], g.vel[0], g.vel[1], g.vel[2]};
  long done = 0;
  if (tbl && k > 0 && kc > 0) {
    done = k < kc ? k : kc;
    const double* st = tbl + 6 * (done - 1);
    for (int i = 0; i < 6; ++i) x[i] = st[i];
  }
  for (; done < k; ++done) glo_rk4(base, x, g.acc);
  if (fabs(rem) > 1.0e-9) glo_rk4(rem, x, g.acc);
  pos[0] = x[0];
  pos[1] = x[1];
  pos[2] = x[2];
  *clk = -g.tau_n + g.gamma_n * el;
  return true;
}

// Record index of output i (idx null: record s); -1 when out of range.
__device__ inline int orbit_record(const int* idx, long i, int s, int n_recs) {
  const int r = idx ? idx[i] : s;
  return (r < 0 || r >= n_recs) ? -1 : r;
}

// Deepest stored state each (GLONASS record, direction) needs: kmax[2r + d]
// = max over its satellite-epochs of min(full steps, kc).
__global__ void k_glo_need(const pf_broadcast_t* __restrict__ recs, int n_recs, const int* __restrict__ idx,
                           const double* __restrict__ times, int n_epoch, int n_sat, double step, int kc,
                           int* __restrict__ kmax) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  int slot = -1, need = 0;
  if (t < (long)n_epoch * n_sat) {
    const int s = (int)(t / n_epoch), e = (int)(t - (long)s * n_epoch);
    const int r = orbit_record(idx, (long)e * n_sat + s, s, n_recs);
    double el, base, rem;
    long k;
    if (r >= 0 && recs[r].system == 'R' && glo_plan(recs[r].u.glonass, times[e], step, el, base, k, rem) && k > 0) {
      slot = 2 * r + (base < 0.0 ? 1 : 0);
      need = (int)(k < kc ? k : kc);
    }
  }
  // satellite-major order: a warp's lanes are consecutive epochs of one
  // satellite and mostly share a slot, so one atomic per group of lanes
  const unsigned grp = __match_any_sync(0xffffffffu, slot);
  const int m = (int)__reduce_max_sync(grp, (unsigned)need);
  if (slot >= 0 && (threadIdx.x & 31) == __ffs(grp) - 1) atomicMax(kmax + slot, m);
}

// The stored states: one thread per (record, direction) integrates kmax
// full steps from toe and keeps every state (6 doubles each, kc per slot).
__global__ void k_glo_table(const pf_broadcast_t* __restrict__ recs, int n_recs, double step,
                            const int* __restrict__ kmax, int kc, double* __restrict__ tbl) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * n_recs) return;
  const int K = kmax[t];
  if (K <= 0) return;
  const pf_glonass_state_t& g = recs[t >> 1].u.glonass;
  const double h = (t & 1) ? -step : step;
  double x[6] = {g.pos[0], g.pos[1], g.pos[2], g.vel[0], g.vel[1], g.vel[2]};
  double* out = tbl + (size_t)t * kc * 6;
  for (int k = 0; k < K; ++k) {
    glo_rk4(h, x, g.acc);
    for (int c = 0; c < 6; ++c) out[6 * k + c] = x[c];
  }
}

// Multi-system records: out[e][s] from recs[idx[e*S+s]] (or recs[s] when idx
// is null) at times[e]; an index outside [0, n_recs) gives NaN, and so does a
// GLONASS integration past kGloMaxSteps steps (also flagged in *err if given).
// tbl / kc: the GLONASS state table of k_glo_table, or null / 0.
// Three CTAs of 256 per SM (80 registers): the walk is FP64-latency bound,
// and the extra warps hide more of it than the few spilled values cost.
__global__ void __launch_bounds__(256, 3) k_broadcast_orbits(const pf_broadcast_t* __restrict__ recs, int n_recs,
                                   const int* __restrict__ idx, const double* __restrict__ times,
                                   int n_epoch, int n_sat, double glo_step, const double* __restrict__ tbl, int kc,
                                   double* __restrict__ pos, double* __restrict__ clk, int* __restrict__ err) {
  // Satellite-major thread order: a warp covers 32 consecutive epochs of one
  // satellite, so its lanes run the same orbit model (Kepler or the longer
  // GLONASS integration) with similar step counts.
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)n_epoch * n_sat) return;
  const int s = (int)(t / n_epoch), e = (int)(t - (long)s * n_epoch);
  const long i = (long)e * n_sat + s;
  const int r = orbit_record(idx, i, s, n_recs);
  double p[3], c;
  if (r < 0) {
    p[0] = p[1] = p[2] = c = nan("");
  } else {
    const pf_broadcast_t& rec = recs[r];
    if (rec.system == 'R') {
      const double el = wrap_half_week(broadcast_rx_sow('R', times[e]) - rec.u.glonass.toe);
      const double* tb = tbl ? tbl + ((size_t)2 * r + (el < 0.0 ? 1 : 0)) * kc * 6 : nullptr;
      if (!glonass_orbit(rec.u.glonass, times[e], glo_step, tb, kc, p, &c) && err) atomicOr(err, 1);
    } else {
      kepler_orbit(rec.u.kepler, rec.system, times[e], p, &c);
    }
  }
  if (pos) {
    pos[3 * i] = p[0];
    pos[3 * i + 1] = p[1];
    pos[3 * i + 2] = p[2];
  }
  if (clk) clk[i] = c;
}

// GPS-constant batch over the reference's parameter array
// (ephemeris.cu:106-180): out[e][s] from params[s] at times[e].
__global__ void k_sat_pos_gps(const pf_ephemeris_t* __restrict__ params, const double* __restrict__ times,
                              int n_epoch, int n_sat, double* __restrict__ pos, double* __restrict__ clk) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)n_epoch * n_sat) return;
  const int e = (int)(i / n_sat), s = (int)(i - (long)e * n_sat);
  double p[3], c;
  kepler_orbit(params[s], 'G', times[e], p, &c);
  pos[3 * i] = p[0];
  pos[3 * i + 1] = p[1];
  pos[3 * i + 2] = p[2];
  clk[i] = c;
}

// Sagnac rotation and range (range_model.py:12-40) for receivers rx[e] and
// satellites sat[e][s]: theta = omega_e |rx - sat| / c about the z axis.
__global__ void k_sagnac(const double* __restrict__ rx, const double* __restrict__ sat, int n_epoch, int n_sat,
                         double* __restrict__ sat_rot, double* __restrict__ range) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)n_epoch * n_sat) return;
  const long e = i / n_sat;
  const double r0 = rx[3 * e], r1 = rx[3 * e + 1], r2 = rx[3 * e + 2];
  const double s0 = sat[3 * i], s1 = sat[3 * i + 1], s2 = sat[3 * i + 2];
  const double d0 = r0 - s0, d1 = r1 - s1, d2 = r2 - s2;
  const double th = kOmegaSagnac * (sqrt(d0 * d0 + d1 * d1 + d2 * d2) / kCLight);
  const double ct = cos(th), st = sin(th);
  const double x = s0 * ct + s1 * st, y = -s0 * st + s1 * ct;
  if (sat_rot) {
    sat_rot[3 * i] = x;
    sat_rot[3 * i + 1] = y;
    sat_rot[3 * i + 2] = s2;
  }
  if (range) {
    const double q0 = r0 - x, q1 = r1 - y, q2 = r2 - s2;
    range[i] = sqrt(q0 * q0 + q1 * q1 + q2 * q2);
  }
}

// WGS84 geodetic latitude, longitude (rad) and height of ECEF points by
// Bowring's closed form (src/utils/coordinates.cu:7-27): one auxiliary
// angle, no iteration.
constexpr double kWgsA = 6378137.0;
constexpr double kWgsF = 1.0 / 298.257223563;
constexpr double kWgsB = kWgsA * (1.0 - kWgsF);
constexpr double kWgsE2 = 2.0 * kWgsF - kWgsF * kWgsF;

__global__ void k_ecef_to_lla(const double* __restrict__ x, const double* __restrict__ y,
                              const double* __restrict__ z, double* __restrict__ lat, double* __restrict__ lon,
                              double* __restrict__ alt, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double X = x[i], Y = y[i], Z = z[i];
  const double p = sqrt(X * X + Y * Y);
  const double th = atan2(Z * kWgsA, p * kWgsB);
  const double st = sin(th), ct = cos(th);
  const double la = atan2(Z + kWgsE2 / (1.0 - kWgsE2) * kWgsB * st * st * st, p - kWgsE2 * kWgsA * ct * ct * ct);
  const double sl = sin(la);
  lat[i] = la;
  lon[i] = atan2(Y, X);
  alt[i] = p / cos(la) - kWgsA / sqrt(1.0 - kWgsE2 * sl * sl);
}

}  // namespace pfb
