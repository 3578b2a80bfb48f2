// pf_velocity.cuh -- per-particle velocity states of the device filter
// (the reference's RBPF-style states, pf_device.cu:67-187 and 610-887):
// a velocity (ECEF, m/s) and its 3x3 covariance per particle, in FP64, held
// in caller-owned device memory beside the engine's particles.
//
// Buffer layout (pf_vel_state_t): two buffers of kVelComp x n doubles,
// component c of particle j at buf[c * n + j]: c = 0..2 velocity, 3..11
// the covariance row-major.  Kernels work on buffer `sel`; the resample
// gather writes the other one.
//
// All arithmetic is FP64 as in the reference.  Particle positions are the
// engine's FP32 offsets about its FP64 anchor (exact in FP64), current
// (gathered through the last resample, if pending).
#pragma once
#include "pf_engine_kernels.cuh"

namespace pfb {

constexpr int kVelComp = 12;
constexpr int kMaxDopplerRows = 64;
constexpr uint32_t TAG_VEL_INIT = 0x06000000u;
constexpr uint32_t TAG_VEL_PREDICT = 0x07000000u;

struct DopplerRow {
  double sat[3];
  double sat_vel[3];
  double doppler_hz;
  double weight;
};

// Two standard normals from two 32-bit words (Box-Muller in FP64).
__device__ __forceinline__ void normals2_f64(uint32_t a, uint32_t b, double& z0, double& z1) {
  const double two_m32 = 2.3283064365386963e-10;
  const double u1 = ((double)a + 0.5) * two_m32;
  const double u2 = (double)b * two_m32 - 0.5;
  const double r = sqrt(-2.0 * log(u1));
  double s, c;
  sincospi(2.0 * u2, &s, &c);
  z0 = r * c;
  z1 = r * s;
}

// Eight normals for particle slot j from two Philox blocks.
__device__ __forceinline__ void vel_normals(uint32_t j, uint32_t step, uint32_t tag, const FilterDesc* fd,
                                            double (&z)[8]) {
  const U4 r0 = philox10(U4{j, step, tag, (uint32_t)fd->filter_id}, fd->key0, fd->key1);
  const U4 r1 = philox10(U4{j, step, tag | 1u, (uint32_t)fd->filter_id}, fd->key0, fd->key1);
  normals2_f64(r0.x, r0.y, z[0], z[1]);
  normals2_f64(r0.z, r0.w, z[2], z[3]);
  normals2_f64(r1.x, r1.y, z[4], z[5]);
  normals2_f64(r1.z, r1.w, z[6], z[7]);
}

// Velocity v0 (+ spread_vel noise when > 0), covariance init_var * I.
__global__ void __launch_bounds__(kThreads) k_vel_init(EngineDev e, int f, double* vb, double vx, double vy, double vz,
                                                       double spread_vel, double init_var, uint32_t step) {
  const FilterDesc* fd = e.desc + f;
  const int n = fd->n;
  for (int j = blockIdx.x * kThreads + threadIdx.x; j < n; j += gridDim.x * kThreads) {
    double v[3] = {vx, vy, vz};
    if (spread_vel > 0.0) {
      double z[8];
      vel_normals((uint32_t)j, step, TAG_VEL_INIT, fd, z);
      for (int i = 0; i < 3; ++i) v[i] += z[i] * spread_vel;
    }
    for (int i = 0; i < 3; ++i) vb[(size_t)i * n + j] = v[i];
    for (int c = 0; c < 9; ++c) vb[(size_t)(3 + c) * n + j] = (c == 0 || c == 4 || c == 8) ? init_var : 0.0;
  }
}

// Resample gather: out[:, j] = in[:, anc[j]].
__global__ void __launch_bounds__(kThreads) k_vel_gather(EngineDev e, int f, const double* vin, double* vout) {
  const FilterDesc* fd = e.desc + f;
  const int n = fd->n;
  const long long base = fd->p_off;
  const int* seg = seg_markers(e, fd);
  for (int j = blockIdx.x * kThreads + threadIdx.x; j < n; j += gridDim.x * kThreads) {
    int a = ancestor_at(e, seg, base, j);
    a = a < 0 ? 0 : (a >= n ? n - 1 : a);
    for (int c = 0; c < kVelComp; ++c) vout[(size_t)c * n + j] = vin[(size_t)c * n + a];
  }
}

struct VelPredict {
  double guide[3];
  double rot[9];  // ECEF -> local rows (E, N, U)
  double dt, sigma_pos, sigma_vel, alpha, q;
  int kf;
  uint32_t step;
};

// Velocity predict (pf_device.cu:106-187): v = (1 - a) v + a g (+ sigma_vel
// noise unless KF); positions move by v dt + noise, the noise N(0,
// sigma_pos^2 I + dt^2 P_v) (Cholesky) in KF mode, else N(0, sigma_pos^2 I);
// KF mode adds q * dt to the velocity variances.  The positions are read
// through the pending resample gather and written to the other state
// buffer (the caller flips the parity); clocks are copied.
template <int D>
__global__ void __launch_bounds__(kThreads) k_vel_predict(EngineDev e, int f, double* vb, VelPredict vp) {
  const FilterDesc* fd = e.desc + f;
  const FilterCtrl* fc = e.ctrl + f;
  const int n = fd->n;
  const long long base = fd->p_off;
  const float* src = fc->parity ? e.state1 : e.state0;
  float* dst = fc->parity ? e.state0 : e.state1;
  const double alpha = fmin(1.0, fmax(0.0, vp.alpha));
  for (int p0 = (blockIdx.x * kThreads + threadIdx.x) * 4; p0 < n; p0 += gridDim.x * kThreads * 4) {
    float x[D][4];
    load_particles<D>(e, fd, src, base, p0, n, fc->resample_flag != 0, x);
#pragma unroll 1
    for (int k = 0; k < 4; ++k) {
      const int j = p0 + k;
      if (j >= n) break;
      double z[8];
      vel_normals((uint32_t)j, vp.step, TAG_VEL_PREDICT, fd, z);
      double v[3];
      for (int i = 0; i < 3; ++i) v[i] = (1.0 - alpha) * vb[(size_t)i * n + j] + alpha * vp.guide[i];
      int zi = 0;
      if (!vp.kf && vp.sigma_vel > 0.0)
        for (int i = 0; i < 3; ++i) v[i] += z[zi++] * vp.sigma_vel;
      for (int i = 0; i < 3; ++i) vb[(size_t)i * n + j] = v[i];
      double nz[3];
      if (vp.kf) {
        double P[9];
        for (int c = 0; c < 9; ++c) P[c] = vb[(size_t)(3 + c) * n + j];
        const double dt2 = vp.dt * vp.dt, s2 = vp.sigma_pos * vp.sigma_pos;
        const double a00 = s2 + dt2 * P[0], a01 = dt2 * P[1], a02 = dt2 * P[2];
        const double a11 = s2 + dt2 * P[4], a12 = dt2 * P[5], a22 = s2 + dt2 * P[8];
        const double l00 = sqrt(fmax(a00, 0.0));
        double l10 = 0.0, l20 = 0.0;
        if (l00 > 1e-12) {
          l10 = a01 / l00;
          l20 = a02 / l00;
        }
        const double l11 = sqrt(fmax(a11 - l10 * l10, 0.0));
        double l21 = 0.0;
        if (l11 > 1e-12) l21 = (a12 - l20 * l10) / l11;
        const double l22 = sqrt(fmax(a22 - l20 * l20 - l21 * l21, 0.0));
        nz[0] = l00 * z[0];
        nz[1] = l10 * z[0] + l11 * z[1];
        nz[2] = l20 * z[0] + l21 * z[1] + l22 * z[2];
        const double qdt = fmax(vp.q, 0.0) * fmax(vp.dt, 0.0);
        vb[(size_t)3 * n + j] = P[0] + qdt;
        vb[(size_t)7 * n + j] = P[4] + qdt;
        vb[(size_t)11 * n + j] = P[8] + qdt;
      } else {
        for (int i = 0; i < 3; ++i) nz[i] = z[zi++] * vp.sigma_pos;
      }
      double d[3];
      for (int i = 0; i < 3; ++i) d[i] = v[i] * vp.dt + nz[i];
      for (int r = 0; r < 3; ++r)
        x[r][k] = (float)((double)x[r][k] + vp.rot[3 * r] * d[0] + vp.rot[3 * r + 1] * d[1] + vp.rot[3 * r + 2] * d[2]);
    }
#pragma unroll
    for (int d = 0; d < D; ++d)
      *reinterpret_cast<float4*>(dst + (size_t)d * e.p_total + base + p0) = make_float4(x[d][0], x[d][1], x[d][2], x[d][3]);
  }
}

// ECEF position of local offsets (x, y, z) about the filter's anchor.
__device__ __forceinline__ void particle_ecef(const FilterDesc* fd, const FilterCtrl* fc, float x, float y, float z,
                                              double (&p)[3]) {
  local_to_ecef(fd->rot, fc->anchor, (double)x, (double)y, (double)z, p);
}

// Solves the 4x4 system A[:, :4] x = A[:, 4] by Gaussian elimination with
// partial pivoting (pf_device.cu:28-58); false if a pivot is below 1e-12.
__device__ bool solve4(double (&A)[4][5], double (&x)[4]) {
  for (int col = 0; col < 4; ++col) {
    int mr = col;
    for (int row = col + 1; row < 4; ++row)
      if (fabs(A[row][col]) > fabs(A[mr][col])) mr = row;
    if (mr != col)
      for (int k = 0; k < 5; ++k) {
        const double t = A[col][k];
        A[col][k] = A[mr][k];
        A[mr][k] = t;
      }
    if (fabs(A[col][col]) < 1e-12) return false;
    for (int row = col + 1; row < 4; ++row) {
      const double fct = A[row][col] / A[col][col];
      for (int k = col; k < 5; ++k) A[row][k] -= fct * A[col][k];
    }
  }
  for (int row = 3; row >= 0; --row) {
    double v = A[row][4];
    for (int col = row + 1; col < 4; ++col) v -= A[row][col] * x[col];
    x[row] = v / A[row][row];
  }
  return true;
}

struct DopplerArgs {
  int n_sat;
  int kf;           // 1: velocity Kalman update (pf_device.cu:750-887)
  double wavelength, sigma, gain, max_update;
};

// Doppler terms: pf_device.cu:610-748 (kf == 0: likelihood with the
// particle's clock drift, then a blend toward its WLS velocity) and
// pf_device.cu:750-887 (kf == 1: sequential velocity KF, innovation
// likelihood).  Log-weights accumulate (read as zero when reset).
template <int D>
__global__ void __launch_bounds__(kThreads) k_doppler(EngineDev e, int f, double* vb, const DopplerRow* rows,
                                                      DopplerArgs a) {
  __shared__ DopplerRow s_rows[kMaxDopplerRows];
  for (int i = threadIdx.x; i < a.n_sat; i += kThreads) s_rows[i] = rows[i];
  __syncthreads();
  const FilterDesc* fd = e.desc + f;
  const FilterCtrl* fc = e.ctrl + f;
  const int n = fd->n;
  const long long base = fd->p_off;
  const float* src = fc->parity ? e.state1 : e.state0;
  const bool keep = fc->lw_zero == 0;
  const double wl = a.wavelength;
  for (int p0 = (blockIdx.x * kThreads + threadIdx.x) * 4; p0 < n; p0 += gridDim.x * kThreads * 4) {
    float x[D][4];
    load_particles<D>(e, fd, src, base, p0, n, fc->resample_flag != 0, x);
    const float4 l4 = keep ? *reinterpret_cast<const float4*>(e.lw + base + p0) : make_float4(0.f, 0.f, 0.f, 0.f);
    float lv[4] = {l4.x, l4.y, l4.z, l4.w};
#pragma unroll 1
    for (int k = 0; k < 4; ++k) {
      const int j = p0 + k;
      if (j >= n) break;
      double pos[3];
      particle_ecef(fd, fc, x[0][k], x[1][k], x[2][k], pos);
      double v[3] = {vb[j], vb[(size_t)n + j], vb[(size_t)2 * n + j]};
      double log_w = 0.0;
      if (!a.kf) {
        double wcd = 0.0, wsum = 0.0;
        for (int s = 0; s < a.n_sat; ++s) {
          const DopplerRow& r = s_rows[s];
          const double dx = r.sat[0] - pos[0], dy = r.sat[1] - pos[1], dz = r.sat[2] - pos[2];
          const double rr = sqrt(dx * dx + dy * dy + dz * dz);
          if (rr < 1.0) continue;
          const double lx = dx / rr, ly = dy / rr, lz = dz / rr;
          const double obs = -r.doppler_hz * wl;
          const double svr = r.sat_vel[0] * lx + r.sat_vel[1] * ly + r.sat_vel[2] * lz;
          const double rxr = v[0] * lx + v[1] * ly + v[2] * lz;
          const double w = fmax(r.weight, 0.0);
          wcd += w * (obs - svr + rxr);
          wsum += w;
        }
        if (wsum > 0.0) {
          const double cd = wcd / wsum, inv_s2 = 1.0 / (a.sigma * a.sigma);
          for (int s = 0; s < a.n_sat; ++s) {
            const DopplerRow& r = s_rows[s];
            const double dx = r.sat[0] - pos[0], dy = r.sat[1] - pos[1], dz = r.sat[2] - pos[2];
            const double rr = sqrt(dx * dx + dy * dy + dz * dz);
            if (rr < 1.0) continue;
            const double lx = dx / rr, ly = dy / rr, lz = dz / rr;
            const double obs = -r.doppler_hz * wl;
            const double pred = (r.sat_vel[0] - v[0]) * lx + (r.sat_vel[1] - v[1]) * ly + (r.sat_vel[2] - v[2]) * lz + cd;
            const double res = obs - pred;
            log_w += -0.5 * fmax(r.weight, 0.0) * res * res * inv_s2;
          }
          const double gain = fmin(1.0, fmax(0.0, a.gain));
          if (gain > 0.0 && a.n_sat >= 4) {
            double A[4][5];
            for (int r0 = 0; r0 < 4; ++r0)
              for (int c0 = 0; c0 < 5; ++c0) A[r0][c0] = 0.0;
            for (int s = 0; s < a.n_sat; ++s) {
              const DopplerRow& r = s_rows[s];
              const double dx = r.sat[0] - pos[0], dy = r.sat[1] - pos[1], dz = r.sat[2] - pos[2];
              const double rr = sqrt(dx * dx + dy * dy + dz * dz);
              if (rr < 1.0) continue;
              const double lx = dx / rr, ly = dy / rr, lz = dz / rr;
              const double h[4] = {-lx, -ly, -lz, 1.0};
              const double svr = r.sat_vel[0] * lx + r.sat_vel[1] * ly + r.sat_vel[2] * lz;
              const double rhs = -r.doppler_hz * wl - svr;
              const double w = fmax(r.weight, 0.0);
              for (int q = 0; q < 4; ++q) {
                A[q][4] += h[q] * w * rhs;
                for (int b = 0; b < 4; ++b) A[q][b] += h[q] * w * h[b];
              }
            }
            for (int q = 0; q < 4; ++q) A[q][q] += 1e-9;
            double sol[4] = {0.0, 0.0, 0.0, 0.0};
            if (solve4(A, sol)) {
              double dv[3] = {sol[0] - v[0], sol[1] - v[1], sol[2] - v[2]};
              const double nrm = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
              if (a.max_update > 0.0 && nrm > a.max_update) {
                const double sc = a.max_update / fmax(nrm, 1e-9);
                for (int i = 0; i < 3; ++i) dv[i] *= sc;
              }
              for (int i = 0; i < 3; ++i) vb[(size_t)i * n + j] = v[i] + gain * dv[i];
            }
          }
        }
      } else {
        double P[9];
        for (int c = 0; c < 9; ++c) P[c] = vb[(size_t)(3 + c) * n + j];
        double hm[3] = {0.0, 0.0, 0.0}, ym = 0.0, wsum = 0.0;
        for (int s = 0; s < a.n_sat; ++s) {
          const DopplerRow& r = s_rows[s];
          const double w = fmax(r.weight, 0.0);
          if (w <= 0.0) continue;
          const double dx = r.sat[0] - pos[0], dy = r.sat[1] - pos[1], dz = r.sat[2] - pos[2];
          const double rr = sqrt(dx * dx + dy * dy + dz * dz);
          if (rr < 1.0) continue;
          const double lx = dx / rr, ly = dy / rr, lz = dz / rr;
          const double svr = r.sat_vel[0] * lx + r.sat_vel[1] * ly + r.sat_vel[2] * lz;
          hm[0] += w * -lx;
          hm[1] += w * -ly;
          hm[2] += w * -lz;
          ym += w * (-r.doppler_hz * wl - svr);
          wsum += w;
        }
        if (wsum > 0.0) {
          for (int i = 0; i < 3; ++i) hm[i] /= wsum;
          ym /= wsum;
          const double s2 = a.sigma * a.sigma;
          for (int s = 0; s < a.n_sat; ++s) {
            const DopplerRow& r = s_rows[s];
            const double ow = fmax(r.weight, 0.0);
            if (ow <= 0.0) continue;
            const double dx = r.sat[0] - pos[0], dy = r.sat[1] - pos[1], dz = r.sat[2] - pos[2];
            const double rr = sqrt(dx * dx + dy * dy + dz * dz);
            if (rr < 1.0) continue;
            const double lx = dx / rr, ly = dy / rr, lz = dz / rr;
            const double h[3] = {-lx - hm[0], -ly - hm[1], -lz - hm[2]};
            const double svr = r.sat_vel[0] * lx + r.sat_vel[1] * ly + r.sat_vel[2] * lz;
            const double yc = (-r.doppler_hz * wl - svr) - ym;
            const double ph0 = P[0] * h[0] + P[1] * h[1] + P[2] * h[2];
            const double ph1 = P[3] * h[0] + P[4] * h[1] + P[5] * h[2];
            const double ph2 = P[6] * h[0] + P[7] * h[1] + P[8] * h[2];
            const double S = h[0] * ph0 + h[1] * ph1 + h[2] * ph2 + s2 / ow;
            if (!(S > 1e-18) || !isfinite(S)) continue;
            const double innov = yc - (h[0] * v[0] + h[1] * v[1] + h[2] * v[2]);
            const double K[3] = {ph0 / S, ph1 / S, ph2 / S};
            for (int i = 0; i < 3; ++i) v[i] += K[i] * innov;
            const double hp0 = h[0] * P[0] + h[1] * P[3] + h[2] * P[6];
            const double hp1 = h[0] * P[1] + h[1] * P[4] + h[2] * P[7];
            const double hp2 = h[0] * P[2] + h[1] * P[5] + h[2] * P[8];
            P[0] -= K[0] * hp0; P[1] -= K[0] * hp1; P[2] -= K[0] * hp2;
            P[3] -= K[1] * hp0; P[4] -= K[1] * hp1; P[5] -= K[1] * hp2;
            P[6] -= K[2] * hp0; P[7] -= K[2] * hp1; P[8] -= K[2] * hp2;
            const double p01 = 0.5 * (P[1] + P[3]), p02 = 0.5 * (P[2] + P[6]), p12 = 0.5 * (P[5] + P[7]);
            P[1] = P[3] = isfinite(p01) ? p01 : 0.0;
            P[2] = P[6] = isfinite(p02) ? p02 : 0.0;
            P[5] = P[7] = isfinite(p12) ? p12 : 0.0;
            P[0] = (isfinite(P[0]) && P[0] > 1e-12) ? P[0] : 1e-12;
            P[4] = (isfinite(P[4]) && P[4] > 1e-12) ? P[4] : 1e-12;
            P[8] = (isfinite(P[8]) && P[8] > 1e-12) ? P[8] : 1e-12;
            log_w += -0.5 * (innov * innov / S + log(S));
          }
          for (int i = 0; i < 3; ++i) vb[(size_t)i * n + j] = v[i];
          for (int c = 0; c < 9; ++c) vb[(size_t)(3 + c) * n + j] = P[c];
        }
      }
      lv[k] = (float)((double)lv[k] + log_w);
    }
    *reinterpret_cast<float4*>(e.lw + base + p0) = make_float4(lv[0], lv[1], lv[2], lv[3]);
  }
}

}  // namespace pfb
