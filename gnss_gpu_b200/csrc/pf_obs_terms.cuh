// pf_obs_terms.cuh -- differenced and carrier-phase observation terms of the
// device filter, one pass over a filter's current particles:
//
//   PF_OBS_DD_PSEUDORANGE  r = dd - (|p - s_k| - |p - s_ref| - b_k + b_ref)   (pf_device.cu:282-368)
//   PF_OBS_CARRIER_AFV     a = afv(cp - (|p - s| + cb) / lambda)              (pf_device.cu:439-494)
//   PF_OBS_DD_CARRIER_AFV  a = afv(dd - (|p - s_k| - |p - s_ref| - b_k + b_ref) / lambda_k)
//                                                                             (pf_device.cu:496-604)
// with afv(v) = v - rint(v), a term -w r^2 / (2 sigma^2) (or the Huber cost
// when huber_k > 0) per row, and for the DD kinds the per-particle gate:
// rows with |r| > gate are dropped unless fewer than min(n, 3) would remain.
//
// Carrier terms resolve centimetres out of 2e7 m ranges, so this kernel
// works in FP64 (the FP32 offsets are exact in FP64; satellites are given
// in the filter's local frame about its anchor, computed on the host in
// FP64).  Each row's constant part is folded on the host:
//   DD pseudorange    c = dd + b_k - b_ref,               r = c - (r_k - r_ref)
//   carrier           c = cp - clk_anchor / lambda,       a = afv(c - (r + x_clk) / lambda)
//   DD carrier        c = dd + (b_k - b_ref) / lambda_k,  a = afv(c - (r_k - r_ref) / lambda_k)
#pragma once
#include "pf_engine_kernels.cuh"

namespace pfb {

constexpr int kMaxObsRows = 128;

struct ObsRow {
  double sk[3];   // satellite (k) in the local frame
  double sr[3];   // reference satellite in the local frame (DD kinds)
  double c;       // constant part of the residual
  double inv_wl;  // 1 / wavelength (carrier kinds), 1 otherwise
  double w;       // row weight
  double pad_;
};

struct ObsBlock {
  int n;
  int kind;
  int accumulate;   // 1: add to the current log-weights, 0: overwrite them
  int gate_min;     // rows that must stay inside the gate
  double inv_sigma2;
  double inv_sigma;
  double gate;      // 0: no gate
  double huber_k;   // 0: Gaussian
};

__device__ __forceinline__ double obs_residual(const ObsRow& r, int kind, double px, double py, double pz,
                                               double clk) {
  const double ax = r.sk[0] - px, ay = r.sk[1] - py, az = r.sk[2] - pz;
  const double rk = sqrt(ax * ax + ay * ay + az * az);
  if (kind == PF_OBS_CARRIER_AFV) {
    const double v = r.c - (rk + clk) * r.inv_wl;
    return v - rint(v);
  }
  const double bx = r.sr[0] - px, by = r.sr[1] - py, bz = r.sr[2] - pz;
  const double rr = sqrt(bx * bx + by * by + bz * bz);
  if (kind == PF_OBS_DD_PSEUDORANGE) return r.c - (rk - rr);
  const double v = r.c - (rk - rr) * r.inv_wl;
  return v - rint(v);
}

__device__ __forceinline__ double obs_cost(const ObsBlock& b, double w, double v) {
  if (b.huber_k > 0.0) {
    const double z = fabs(v) * b.inv_sigma, k = b.huber_k;
    return w * (z < k ? 0.5 * z * z : k * z - 0.5 * k * k);
  }
  return 0.5 * w * v * v * b.inv_sigma2;
}

template <int D>
__global__ void __launch_bounds__(kThreads) k_obs_term(EngineDev e, int f, ObsBlock b, const ObsRow* rows) {
  __shared__ ObsRow s_rows[kMaxObsRows];
  for (int i = threadIdx.x; i < b.n; i += kThreads) s_rows[i] = rows[i];
  __syncthreads();
  const FilterDesc* fd = e.desc + f;
  const FilterCtrl* fc = e.ctrl + f;
  const int n = fd->n;
  const long long base = fd->p_off;
  const float* src = fc->parity ? e.state1 : e.state0;
  const bool keep = b.accumulate && fc->lw_zero == 0;
  for (int p0 = (blockIdx.x * kThreads + threadIdx.x) * 4; p0 < n; p0 += gridDim.x * kThreads * 4) {
    float x[D][4];
    load_particles<D>(e, fd, src, base, p0, n, fc->resample_flag != 0, x);
    const float4 l = keep ? *reinterpret_cast<const float4*>(e.lw + base + p0) : make_float4(0.f, 0.f, 0.f, 0.f);
    float lv[4] = {l.x, l.y, l.z, l.w};
#pragma unroll 1
    for (int k = 0; k < 4; ++k) {
      const double px = x[0][k], py = x[1][k], pz = x[2][k], clk = x[3][k];
      bool gated = b.gate > 0.0;
      if (gated) {
        int kept = 0;
        for (int i = 0; i < b.n; ++i) kept += fabs(obs_residual(s_rows[i], b.kind, px, py, pz, clk)) <= b.gate;
        gated = kept >= b.gate_min;
      }
      double acc = 0.0;
      for (int i = 0; i < b.n; ++i) {
        const double v = obs_residual(s_rows[i], b.kind, px, py, pz, clk);
        if (gated && fabs(v) > b.gate) continue;
        acc -= obs_cost(b, s_rows[i].w, v);
      }
      lv[k] = (float)((double)lv[k] + acc);
    }
    *reinterpret_cast<float4*>(e.lw + base + p0) = make_float4(lv[0], lv[1], lv[2], lv[3]);
  }
}

}  // namespace pfb
