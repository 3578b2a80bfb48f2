// pf_generic.cuh -- the device filter's likelihood family (weight mode
// PF_WEIGHT_GENERIC), selected per call with pfe_set_likelihood:
//
//   Gaussian      -w r^2 / (2 sigma^2)                                     (pf_device.cu:273-275)
//   Student's t   -(nu + 1)/2 log(1 + w r^2 / (nu sigma^2))                (pf_device.cu:265-266)
//   Huber         -w rho_k(|r| / sigma)                                    (pf_device.cu:19-26,267-268)
//   GMM           log(w_los N(r; 0, sigma) + (1 - w_los) N(r; mu, s_nlos)),
//                 each quadratic term scaled by w                           (pf_device.cu:373-436)
//
// with an optional per-particle NLOS gate (pf_device.cu:236-258): a particle
// drops the satellites whose |r| exceeds the gate, unless fewer than
// min(n_sat, 4) would remain, in which case it keeps all of them.
//
// The residual r is the epoch kernel's second-order form (sat_pair_update).
// Satellite table entries use the mixture layout (kMixStride float2):
//   eE eN | eU g/2 | y w | c0 c1 | c2 c3 | mu mode
// mode 0 GMM (c0 = log w_los - log sigma, c1 = -w/(2 sigma^2), c2, c3 the
// NLOS pair), 1 Huber (c0 = k, c1 = 1/sigma), 2 unused, 3 Student's t
// (c0 = -(nu+1)/2, c1 = w/(nu sigma^2)), 4 Gaussian (c1 = -w/(2 sigma^2)).
#pragma once
#include "pf_learned.cuh"

namespace pfb {

// Table entry of one satellite for the generic likelihood.
__device__ __forceinline__ void write_generic_entry(float2* o, const EngineDev& e, float sigma, float eE, float eN,
                                                    float eU, float g, float y, float w) {
  o[0] = bc(eE); o[1] = bc(eN); o[2] = bc(eU); o[3] = bc(0.5f * g);
  o[4] = bc(y); o[5] = bc(w);
  float mode = 4.f, c0 = 0.f, c1 = 0.f, c2 = 0.f, c3 = 0.f, mu = 0.f;
  const float s2 = sigma * sigma;
  if (!(w > 0.f)) {
    mode = 2.f;
  } else if (e.lk_type == PF_LIK_STUDENT_T) {
    mode = 3.f;
    c0 = -0.5f * (e.lk_nu + 1.f);
    c1 = w / (e.lk_nu * s2);
  } else if (e.lk_type == PF_LIK_HUBER) {
    mode = 1.f;
    c0 = e.lk_huber_k;
    c1 = 1.f / sigma;
  } else if (e.lk_type == PF_LIK_GMM) {
    mode = 0.f;
    const float sn = e.lk_sigma_nlos;
    c0 = logf(e.lk_w_los) - logf(sigma);
    c1 = -0.5f * w / s2;
    c2 = logf(1.f - e.lk_w_los) - logf(sn);
    c3 = -0.5f * w / (sn * sn);
    mu = e.lk_mu_nlos;
  } else {
    c1 = -0.5f * w / s2;
  }
  o[6] = bc(c0); o[7] = bc(c1); o[8] = bc(c2); o[9] = bc(c3);
  o[10] = bc(mu); o[11] = bc(mode);
}

// Residual of two particles for one table entry (as sat_pair_update).
__device__ __forceinline__ float2 entry_residual(const float2* entry, float2 dx, float2 dy, float2 dz, float2 nbb,
                                                 float2 ncb) {
  const float4* sv = reinterpret_cast<const float4*>(entry);
  const float4 q0 = sv[0], q1 = sv[1], q2 = sv[2];
  const float2 eE = f2(q0.x, q0.y), eN = f2(q0.z, q0.w), eU = f2(q1.x, q1.y), g2 = f2(q1.z, q1.w);
  const float2 yc = __fadd2_rn(f2(q2.x, q2.y), ncb);
  float2 ye = __ffma2_rn(eE, dx, yc);
  ye = __ffma2_rn(eN, dy, ye);
  ye = __ffma2_rn(eU, dz, ye);
  const float2 ed = __ffma2_rn(yc, bc(-1.0f), ye);
  const float2 sq = __ffma2_rn(ed, ed, nbb);
  return __ffma2_rn(sq, g2, ye);
}

// Log-likelihood term of one satellite for one particle.
__device__ __forceinline__ float generic_term(const float4 q3, const float4 q4, const float4 q5, float w, float r) {
  const float mode = q5.z;
  if (mode > 3.5f) return q3.z * r * r;                              // Gaussian
  if (mode > 2.5f) return q3.x * __logf(fmaf(q3.z * r, r, 1.f));     // Student's t
  if (mode > 0.5f) {                                                  // Huber
    const float z = fabsf(r) * q3.z, k = q3.x;
    return -w * (z < k ? 0.5f * z * z : fmaf(k, z, -0.5f * k * k));
  }
  const float a = fmaf(q3.z * r, r, q3.x);                            // GMM
  const float dm = r - q5.x;
  const float b = fmaf(q4.z * dm, dm, q4.x);
  const float hi = fmaxf(a, b), lo = fminf(a, b);
  return hi + __logf(1.f + __expf(lo - hi));
}

// Adds the satellites [s0, s1) of the table to the log-weights of two
// particle pairs (with the per-particle gate when gate > 0).
__device__ __forceinline__ void generic_pairs(const float2* s_sat, int s0, int s1, const float2 (&dx)[2],
                                              const float2 (&dy)[2], const float2 (&dz)[2], const float2 (&nbb)[2],
                                              const float2 (&ncb)[2], float2 (&lwp)[2], bool (&gated)[4],
                                              float gate) {
  for (int s = s0; s < s1; ++s) {
    const float2* entry = s_sat + kMixStride * s;
    const float4* sv = reinterpret_cast<const float4*>(entry);
    const float4 q2 = sv[2], q3 = sv[3], q4 = sv[4], q5 = sv[5];
    if (q5.z > 1.5f && q5.z < 2.5f) continue;  // weight 0
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      const float2 r = entry_residual(entry, dx[p], dy[p], dz[p], nbb[p], ncb[p]);
      if (!(gated[2 * p] && fabsf(r.x) > gate)) lwp[p].x += generic_term(q3, q4, q5, q2.z, r.x);
      if (!(gated[2 * p + 1] && fabsf(r.y) > gate)) lwp[p].y += generic_term(q3, q4, q5, q2.z, r.y);
    }
  }
}

// Satellites of [s0, s1) with |r| <= gate, per particle (for the gate).
__device__ __forceinline__ void generic_kept(const float2* s_sat, int s0, int s1, const float2 (&dx)[2],
                                             const float2 (&dy)[2], const float2 (&dz)[2], const float2 (&nbb)[2],
                                             const float2 (&ncb)[2], int (&kept)[4], int& used, float gate) {
  for (int s = s0; s < s1; ++s) {
    const float2* entry = s_sat + kMixStride * s;
    ++used;  // every satellite counts, as in the reference
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      const float2 r = entry_residual(entry, dx[p], dy[p], dz[p], nbb[p], ncb[p]);
      kept[2 * p] += fabsf(r.x) <= gate;
      kept[2 * p + 1] += fabsf(r.y) <= gate;
    }
  }
}

}  // namespace pfb
