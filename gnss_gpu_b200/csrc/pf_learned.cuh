// pf_learned.cuh -- the learned two-component likelihood of the epoch
// kernel (weight mode PF_WEIGHT_MIXTURE).
//
// Per (filter, satellite) and epoch the CTA forms 12 features from the
// filter's prior mean (the last weighted mean moved by the known
// displacement), runs the NLOS network on the tensor cores (pf_mlp.cuh) and
// turns its outputs p (NLOS probability) and mu (NLOS bias mean) into the
// constants of
//   l(r) = log((1 - p) N(r; 0, s2) + p N(r; mu, s2 + mu^2)),  s2 = sigma_pr^2 / w,
// evaluated per particle as max(a, b) + log(1 + exp(min(a, b) - max(a, b)))
// with a = log(1-p) - log(s2)/2 - r^2/(2 s2), b likewise.  Satellites whose
// inputs leave the training range (C/N0 outside [10, 70] dB-Hz, centred
// residual above 150 m, fewer than 4 satellites) fall back to the plain
// robust (Huber) likelihood.
//
// Features (mirrored in gnss_gpu_b200/learned.py, which builds the training
// set): with e the unit line of sight in E/N/U at the prior mean,
//   f0 = e_U (sin el), f1 = |e_EN| (cos el), f2 = e_E/|e_EN| (sin az),
//   f3 = e_N/|e_EN| (cos az), f4 = (C/N0 - 40)/10,
//   f5 = clamp(rc/20, -8, 8), f6 = min(|rc|/20, 8), f7 = blocked flag,
//   f8 = n_sat/40, f9 = min(median |rc| / 20, 8), f10 = blocked fraction,
//   f11 = (C/N0 - mean C/N0)/10,
// where r = pr - |s - prior| - clock prior is the residual against the prior
// mean and rc = r - (median r of the satellite's clock group).
#pragma once
#include "pf_engine_kernels.cuh"
#include "pf_mlp.cuh"

namespace pfb {

constexpr int kMixStride = 12;  // float2 per satellite entry in mixture mode (six float4)
constexpr int kSatDbg = 16;     // floats per satellite in the debug export

struct MixSmem {
  MlpSmem w;
  float feat[PF_MAX_SATS * kMlpIn];
  float res[PF_MAX_SATS];
  float absr[PF_MAX_SATS];
  float out[PF_MAX_SATS * 2];
  float med[PF_MAX_CLK];
  float ctx[3];  // median |rc|, blocked fraction, mean C/N0
};

__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

// Builds the mixture satellite table of filter f (all threads of the CTA).
// Entry layout (each value stored twice): eE eN | eU g/2 | y w | ca ia |
// cb ib | mu mode, mode 0 = mixture, 1 = Huber fallback, 2 = unused.
template <int NCLK>
__device__ __forceinline__ void build_mixture_table(const EngineDev& e, const FilterDesc* fd, const FilterCtrl* fc,
                                                    const pf_filter_epoch_t* fe, const pf_sat_t* sats, int n_sat,
                                                    bool do_weight, bool export_dbg, int f, float2* s_sat,
                                                    int* s_grp, unsigned char* s_clk, MixSmem& M) {
  const int s = threadIdx.x;
  const bool mine = do_weight && s < n_sat;
  const pf_sat_t* sp = sats + fe->sat_offset + s;
  __syncthreads();  // nobody still reads the previous filter's table
  int c = 0;
  if (mine) {
    c = sp->clk;
    c = c < 0 ? 0 : (c >= NCLK ? NCLK - 1 : c);
    s_clk[s] = (unsigned char)c;
  }
  mlp_stage(e.mlp, M.w, kThreads);
  float eE = 0.f, eN = 0.f, eU = 0.f, g = 0.f, y = 0.f, res = 0.f, cn0 = 0.f, blk = 0.f;
  double fE = 0.0, fN = 0.0, fU = 0.0;
  if (mine) {
    const double* rot = fd->rot;
    double A[3];
    local_to_ecef(rot, fc->anchor, fc->shift[0], fc->shift[1], fc->shift[2], A);
    const double clkA = fc->clk_anchor[c] + (double)fc->shift[3 + c];
    double vx = sp->x - A[0], vy = sp->y - A[1], vz = sp->z - A[2];
    const double r0 = sqrt(vx * vx + vy * vy + vz * vz);
    const double inv = 1.0 / r0;
    vx *= inv; vy *= inv; vz *= inv;
    fE = rot[0] * vx + rot[1] * vy + rot[2] * vz;
    fN = rot[3] * vx + rot[4] * vy + rot[5] * vz;
    fU = rot[6] * vx + rot[7] * vy + rot[8] * vz;
    eE = (float)fE; eN = (float)fN; eU = (float)fU;
    g = (float)inv;
    const double yd = sp->pr - r0 - clkA;
    y = (float)yd;
    // against the prior mean A + disp: the range shortens by e . disp
    res = (float)(yd + fE * fe->disp[0] + fN * fe->disp[1] + fU * fe->disp[2]);
    cn0 = sp->cn0;
    blk = sp->blocked;
    M.res[s] = res;
  }
  __syncthreads();
  // median residual of each clock group (element of rank (m - 1) / 2)
  if (mine) {
    int m = 0, rk = 0;
    for (int j = 0; j < n_sat; ++j) {
      if (s_clk[j] != c) continue;
      ++m;
      const float rj = M.res[j];
      rk += (rj < res) || (rj == res && j < s);
    }
    if (rk == (m - 1) / 2) M.med[c] = res;
  }
  __syncthreads();
  float rc = 0.f;
  if (mine) {
    rc = res - M.med[c];
    M.absr[s] = fabsf(rc);
  }
  __syncthreads();
  if (mine) {
    int rk = 0;
    for (int j = 0; j < n_sat; ++j) {
      const float aj = M.absr[j];
      rk += (aj < fabsf(rc)) || (aj == fabsf(rc) && j < s);
    }
    if (rk == (n_sat - 1) / 2) M.ctx[0] = fabsf(rc);
  }
  if (s == 0) {
    float nb = 0.f, sc = 0.f;
    for (int j = 0; j < n_sat; ++j) {
      nb += sats[fe->sat_offset + j].blocked;
      sc += sats[fe->sat_offset + j].cn0;
    }
    M.ctx[1] = n_sat > 0 ? nb / (float)n_sat : 0.f;
    M.ctx[2] = n_sat > 0 ? sc / (float)n_sat : 0.f;
  }
  __syncthreads();
  const int rows = (n_sat + 15) & ~15;
  bool fallback = false;
  if (s < rows) {
    float* x = M.feat + s * kMlpIn;
    if (mine) {
      const float ch = (float)sqrt(fE * fE + fN * fN);
      const float inv_ch = ch > 0.f ? 1.f / ch : 0.f;
      x[0] = eU;
      x[1] = ch;
      x[2] = eE * inv_ch;
      x[3] = eN * inv_ch;
      x[4] = (cn0 - 40.f) * 0.1f;
      x[5] = clampf(rc / 20.f, -8.f, 8.f);
      x[6] = fminf(fabsf(rc) / 20.f, 8.f);
      x[7] = blk;
      x[8] = (float)n_sat / 40.f;
      x[9] = fminf(M.ctx[0] / 20.f, 8.f);
      x[10] = M.ctx[1];
      x[11] = (cn0 - M.ctx[2]) * 0.1f;
      fallback = !(cn0 >= 10.f && cn0 <= 70.f) || !(fabsf(rc) <= 150.f) || n_sat < 4;
    } else {
#pragma unroll
      for (int k = 0; k < kMlpFeat; ++k) x[k] = 0.f;
    }
#pragma unroll
    for (int k = kMlpFeat; k < kMlpIn; ++k) x[k] = 0.f;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (warp * 16 < rows) {
    MlpTile T;
    mlp_forward_tile(M.feat + warp * 16 * kMlpIn, M.w, lane, T);
    if ((lane & 3) == 0) {
      const int gr = lane >> 2;
      M.out[2 * (warp * 16 + gr)] = T.o[0];
      M.out[2 * (warp * 16 + gr) + 1] = T.o[1];
      M.out[2 * (warp * 16 + gr + 8)] = T.o[2];
      M.out[2 * (warp * 16 + gr + 8) + 1] = T.o[3];
    }
  }
  __syncthreads();
  if (mine) {
    const float p = clampf(sigmoidf_(M.out[2 * s]), 1e-4f, 1.f - 1e-4f);
    const float mu = kMuScale * softplusf(M.out[2 * s + 1]);
    const double w = sp->w;
    const float mode = (w > 0.0) ? (fallback ? 1.f : 0.f) : 2.f;
    const float s2 = (w > 0.0) ? (float)((double)fd->sigma_pr * (double)fd->sigma_pr / w) : 1.f;
    const float sn2 = s2 + mu * mu;
    const float ia = -0.5f / s2, ib = -0.5f / sn2;
    const float ca = logf(1.f - p) - 0.5f * logf(s2), cb = logf(p) - 0.5f * logf(sn2);
    int rank = 0;
    for (int s2i = 0; s2i < n_sat; ++s2i) {
      const int c2 = s_clk[s2i];
      rank += (c2 < c) || (c2 == c && s2i < s);
    }
    float2* o = s_sat + kMixStride * rank;
    o[0] = bc(eE); o[1] = bc(eN); o[2] = bc(eU); o[3] = bc(0.5f * g);
    o[4] = bc(y); o[5] = bc((float)w);
    o[6] = bc(ca); o[7] = bc(ia); o[8] = bc(cb); o[9] = bc(ib);
    o[10] = bc(mu); o[11] = bc(mode);
    if (export_dbg) {
      float* d = e.sat_dbg + ((size_t)f * e.max_sats + s) * kSatDbg;
#pragma unroll
      for (int k = 0; k < kMlpFeat; ++k) d[k] = M.feat[s * kMlpIn + k];
      d[12] = p;
      d[13] = mu;
      d[14] = mode;
      d[15] = res;
    }
  }
  if (threadIdx.x <= NCLK) {
    int cnt = 0;
    if (do_weight)
      for (int s2i = 0; s2i < n_sat; ++s2i) cnt += s_clk[s2i] < (int)threadIdx.x;
    s_grp[threadIdx.x] = cnt;
  }
  __syncthreads();
}

// Log-likelihood update of two particles for one satellite in mixture mode
// (the residual as in sat_pair_update).
__device__ __forceinline__ void sat_pair_mixture(const float2* entry, float2 dx, float2 dy, float2 dz, float2 nbb,
                                                 float2 ncb, float2& lw, const FilterDesc* fd) {
  const float4* sv = reinterpret_cast<const float4*>(entry);
  const float4 q0 = sv[0], q1 = sv[1], q2 = sv[2], q5 = sv[5];
  const float mode = q5.z;
  if (mode > 1.5f) return;  // weight 0: no contribution
  const float2 eE = f2(q0.x, q0.y), eN = f2(q0.z, q0.w), eU = f2(q1.x, q1.y), g2 = f2(q1.z, q1.w);
  const float2 yy = f2(q2.x, q2.y);
  const float2 yc = __fadd2_rn(yy, ncb);
  float2 ye = __ffma2_rn(eE, dx, yc);
  ye = __ffma2_rn(eN, dy, ye);
  ye = __ffma2_rn(eU, dz, ye);
  const float2 ed = __ffma2_rn(yc, bc(-1.0f), ye);
  const float2 sq = __ffma2_rn(ed, ed, nbb);
  const float2 r = __ffma2_rn(sq, g2, ye);
  if (mode > 0.5f) {  // Huber fallback (uniform over the warp: one satellite at a time)
    const float wq = q2.z;
    const float ks = fd->huber_k;
    const float z0 = fabsf(r.x) * fd->inv_sigma_pr, z1 = fabsf(r.y) * fd->inv_sigma_pr;
    const float rho0 = z0 < ks ? 0.5f * z0 * z0 : fmaf(ks, z0, -0.5f * ks * ks);
    const float rho1 = z1 < ks ? 0.5f * z1 * z1 : fmaf(ks, z1, -0.5f * ks * ks);
    lw.x = fmaf(-wq, rho0, lw.x);
    lw.y = fmaf(-wq, rho1, lw.y);
    return;
  }
  const float4 q3 = sv[3], q4 = sv[4];
  const float2 ca = f2(q3.x, q3.y), ia = f2(q3.z, q3.w), cb = f2(q4.x, q4.y), ib = f2(q4.z, q4.w);
  const float2 mu = f2(q5.x, q5.y);
  const float2 a = __ffma2_rn(__fmul2_rn(r, r), ia, ca);
  const float2 dm = __ffma2_rn(mu, bc(-1.0f), r);
  const float2 b = __ffma2_rn(__fmul2_rn(dm, dm), ib, cb);
  const float hi0 = fmaxf(a.x, b.x), lo0 = fminf(a.x, b.x);
  const float hi1 = fmaxf(a.y, b.y), lo1 = fminf(a.y, b.y);
  lw.x += hi0 + __logf(1.0f + __expf(lo0 - hi0));
  lw.y += hi1 + __logf(1.0f + __expf(lo1 - hi1));
}

}  // namespace pfb
