// pf_engine_kernels.cuh -- sm_100a kernels of the resident engine.
//
// One epoch of every filter is a short chain of persistent kernels, each a
// loop over (filter, tile) work items taken from an atomic queue:
//
//   k_step   fused predict + likelihood + tile statistics (+ the segment
//            and tile levels of the systematic resampler's tiled integer
//            CDF); the last tile of a filter merges the tile statistics into
//            max log-weight, ESS, weighted mean and covariance and decides
//            on the device whether the filter resamples (reference:
//            predict.cu:23-38, weight.cu:13-57,61-108,163-220,
//            particle_filter.py:153-161).
//   k_scan   tile sums scaled to the filter maximum and a decoupled
//            look-back scan of them (systematic only).
//   k_offs   filter-wide CDF of every particle, its offspring end F(i) and
//            the merge-path partition points.
//   k_merge  merge-path offspring assignment: ancestor index of every slot.
//   k_mego   Megopolis chain per slot, ancestor in registers.
//
// The resampled state is never copied here: the next k_step (or the
// estimate / export kernels) reads state[ancestor[k]].
#pragma once
#include "pf_engine_dev.cuh"

namespace pfb {

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 bc(float a) { return make_float2(a, a); }

// ---- satellite table of the likelihood (shared memory, one entry per
// satellite, every constant stored twice so the packed f32x2 operations
// read it without register moves): e_E, e_N, e_U (unit line of sight in the
// local frame), g/2 with g = 1/r0, y = pr - r0 - clock anchor, weight.
constexpr int kSatStride = 6;  // float2 per satellite entry (three float4)

__device__ __forceinline__ void write_sat_entry(float2* o, float eE, float eN, float eU, float g, float y, float wq) {
  o[0] = bc(eE);
  o[1] = bc(eN);
  o[2] = bc(eU);
  o[3] = bc(0.5f * g);
  o[4] = bc(y);
  o[5] = bc(wq);
}

// Log-weight update of two particles for one satellite.  With d the
// particle offset from the anchor, ed = e.d and the receiver clock cb, the
// range residual to second order in |d|/r0 is
//   r = (y - cb + ed) + (g/2) (ed^2 - |d|^2)
// (the next term, of order |d|^3 g^2, is below 1e-8 m for |d| < 1 km).
// ye = y - cb + ed is formed first and ed recovered as ye - (y - cb): both
// are of the size of the residual, so no large range is ever subtracted.
// nbb = -|d|^2 and ncb = -cb of the pair.
template <int WMODE>
__device__ __forceinline__ void sat_pair_update(const float2* entry, float2 dx, float2 dy, float2 dz, float2 nbb,
                                                float2 ncb, float2& lw, const FilterDesc* fd) {
  const float4* sv = reinterpret_cast<const float4*>(entry);
  const float4 q0 = sv[0], q1 = sv[1], q2 = sv[2];
  const float2 eE = f2(q0.x, q0.y), eN = f2(q0.z, q0.w), eU = f2(q1.x, q1.y), g2 = f2(q1.z, q1.w);
  const float2 yy = f2(q2.x, q2.y), wq = f2(q2.z, q2.w);
  const float2 yc = __fadd2_rn(yy, ncb);
  float2 ye = __ffma2_rn(eE, dx, yc);
  ye = __ffma2_rn(eN, dy, ye);
  ye = __ffma2_rn(eU, dz, ye);
  const float2 ed = __ffma2_rn(yc, bc(-1.0f), ye);
  const float2 sq = __ffma2_rn(ed, ed, nbb);
  const float2 r = __ffma2_rn(sq, g2, ye);
  if (WMODE == PF_WEIGHT_GAUSSIAN) {
    const float2 rw = __fmul2_rn(r, wq);
    lw = __ffma2_rn(rw, r, lw);
  } else {
    const float ks = fd->huber_k;
    const float z0 = fabsf(r.x) * fd->inv_sigma_pr, z1 = fabsf(r.y) * fd->inv_sigma_pr;
    const float rho0 = z0 < ks ? 0.5f * z0 * z0 : fmaf(ks, z0, -0.5f * ks * ks);
    const float rho1 = z1 < ks ? 0.5f * z1 * z1 : fmaf(ks, z1, -0.5f * ks * ks);
    lw.x = fmaf(-wq.x, rho0, lw.x);
    lw.y = fmaf(-wq.x, rho1, lw.y);
  }
}

// Programmatic dependent launch (sm_90+): a kernel lets the next kernel of
// the stream start launching as soon as all of its CTAs are running, and
// waits for the previous kernel's completion (and memory flush) before it
// reads anything that kernel wrote.  Both are no-ops without a programmatic
// dependency.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ int dequeue(unsigned* q, int* s_slot) {
  if (threadIdx.x == 0) *s_slot = (int)atomicAdd(q, 1u);
  __syncthreads();
  int v = *s_slot;
  __syncthreads();
  return v;
}

// The last CTA to leave resets the queue for the next launch.
__device__ __forceinline__ void queue_exit(unsigned* q) {
  if (threadIdx.x == 0) {
    unsigned old = atomicAdd(q + 1, 1u);
    if (old == gridDim.x - 1) {
      q[0] = 0u;
      q[1] = 0u;
      __threadfence();
    }
  }
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sums 16 per-lane values over a warp with 16 shuffles (a transpose-style
// butterfly: every step halves the values a lane holds).  Afterwards v[0]
// of lane l holds the warp total of value index
//   ((l >> 4) & 1) * 8 + ((l >> 3) & 1) * 4 + ((l >> 2) & 1) * 2 + ((l >> 1) & 1),
// which is returned; lanes l and l ^ 1 hold the same total.
template <typename T>
__device__ __forceinline__ int warp_transpose_sum16(T (&v)[16]) {
  const int lane = threadIdx.x & 31;
  {
    const bool up = (lane & 16) != 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const T send = up ? v[i] : v[i + 8];
      const T keep = up ? v[i + 8] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
  }
  {
    const bool up = (lane & 8) != 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const T send = up ? v[i] : v[i + 4];
      const T keep = up ? v[i + 4] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
  }
  {
    const bool up = (lane & 4) != 0;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const T send = up ? v[i] : v[i + 2];
      const T keep = up ? v[i + 2] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    }
  }
  {
    const bool up = (lane & 2) != 0;
    const T send = up ? v[0] : v[1];
    const T keep = up ? v[1] : v[0];
    v[0] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
  }
  v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
  return ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
}

// Inclusive warp scan of 64-bit integers.
__device__ __forceinline__ unsigned long long warp_incl_scan_u64(unsigned long long v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    unsigned long long t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Block-wide max over kThreads threads.
__device__ __forceinline__ float block_max(float v, float* s_tmp) {
  v = warp_max(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) s_tmp[warp] = v;
  __syncthreads();
  float r = s_tmp[0];
#pragma unroll
  for (int w = 1; w < kThreads / 32; ++w) r = fmaxf(r, s_tmp[w]);
  return r;
}

// Block exclusive scan of one 64-bit value per thread; returns the exclusive
// prefix and writes the block total to *total.
__device__ __forceinline__ unsigned long long block_excl_scan_u64(
    unsigned long long v, unsigned long long* s_tmp, unsigned long long* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long incl = warp_incl_scan_u64(v);
  __syncthreads();
  if (lane == 31) s_tmp[warp] = incl;
  __syncthreads();
  unsigned long long wpre = 0, tot = 0;
#pragma unroll
  for (int w = 0; w < kThreads / 32; ++w) {
    unsigned long long x = s_tmp[w];
    if (w < warp) wpre += x;
    tot += x;
  }
  *total = tot;
  return wpre + incl - v;
}

// -------------------------------------------------------------------------
// Tile statistics: max log-weight, sum w, sum w^2, sum w x_d, sum w x_i x_j
// (positions) with w = exp(lw - tile max).  Written as one 16-float row.
template <int D>
__device__ __forceinline__ void tile_stats(const float (&x)[D][4], const float (&lwv)[4],
                                           bool cov, float* part_row, float* s_maxtmp,
                                           float (*s_red)[kPartStride]) {
  constexpr int NV = 2 + D + 6;  // s, s2, sx[D], cov6
  float tmax = fmaxf(fmaxf(lwv[0], lwv[1]), fmaxf(lwv[2], lwv[3]));
  const float bmax = block_max(tmax, s_maxtmp);
  float acc[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) acc[i] = 0.f;
  if (bmax > -INFINITY) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      float w = exp2f((lwv[k] - bmax) * 1.4426950408889634f);
      acc[0] += w;
      acc[1] = fmaf(w, w, acc[1]);
#pragma unroll
      for (int d = 0; d < D; ++d) acc[2 + d] = fmaf(w, x[d][k], acc[2 + d]);
      if (cov) {
        float wx = w * x[0][k], wy = w * x[1][k], wz = w * x[2][k];
        acc[2 + D + 0] = fmaf(wx, x[0][k], acc[2 + D + 0]);
        acc[2 + D + 1] = fmaf(wx, x[1][k], acc[2 + D + 1]);
        acc[2 + D + 2] = fmaf(wx, x[2][k], acc[2 + D + 2]);
        acc[2 + D + 3] = fmaf(wy, x[1][k], acc[2 + D + 3]);
        acc[2 + D + 4] = fmaf(wy, x[2][k], acc[2 + D + 4]);
        acc[2 + D + 5] = fmaf(wz, x[2][k], acc[2 + D + 5]);
      }
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i) acc[i] = warp_sum(acc[i]);
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) s_red[warp][i] = acc[i];
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    float s = 0.f;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) s += s_red[w][threadIdx.x];
    part_row[1 + threadIdx.x] = s;
  }
  if (threadIdx.x == 0) part_row[0] = bmax;
  __syncthreads();
}

struct MergedStats {
  float max_lw;
  double w, w2;
  double sx[kMaxD];
  double sxx[6];
};

// Order-preserving code of a float (larger float, larger code; 0 is below
// every code, so a zeroed word means "no finite value seen").
__device__ __forceinline__ unsigned ord_code(float f) {
  const unsigned b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord_decode(unsigned c) {
  if (c == 0u) return -INFINITY;
  return __uint_as_float((c & 0x80000000u) ? (c & 0x7FFFFFFFu) : ~c);
}

// Merge the tile rows [tb, tb + nt) of one filter whose maximum tile
// log-weight M is known (executed by a whole CTA, result valid in thread
// 0).  Rows written by other CTAs are read through L2.  Each thread folds
// rows i, i + kThreads, ... in FP64 (rescaled to M), a transpose butterfly
// sums the 16 accumulators over the warp, and NV threads add the warp
// totals; the order is fixed, so the result does not depend on how the
// tiles were scheduled.
template <int D>
__device__ __forceinline__ MergedStats merge_tiles_at(const float* part, int tb, int nt, float M, double* s_dred) {
  constexpr int NV = 2 + D + 6;
  static_assert(NV <= 16, "row layout");
  double acc[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) acc[i] = 0.0;
  auto fold = [&](const float4 a0, const float4 a1, const float4 a2, const float4 a3) {
    const float r[16] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w,
                         a2.x, a2.y, a2.z, a2.w, a3.x, a3.y, a3.z, a3.w};
    if (!(r[0] > -INFINITY)) return;
    const double sc = exp((double)r[0] - (double)M);
    acc[0] += sc * (double)r[1];
    acc[1] += sc * sc * (double)r[2];
#pragma unroll
    for (int v = 2; v < NV; ++v) acc[v] += sc * (double)r[1 + v];
  };
  if (M > -INFINITY) {
    // two rows in flight per thread (rows i and i + kThreads, folded in
    // that order, the order of the plain loop)
    for (int i = threadIdx.x; i < nt; i += 2 * kThreads) {
      const int j = i + kThreads;
      const float4* ra = reinterpret_cast<const float4*>(part + (size_t)(tb + i) * kPartStride);
      const float4* rb = reinterpret_cast<const float4*>(part + (size_t)(tb + (j < nt ? j : i)) * kPartStride);
      const float4 a0 = __ldcg(ra), a1 = __ldcg(ra + 1), a2 = __ldcg(ra + 2), a3 = __ldcg(ra + 3);
      const float4 b0 = __ldcg(rb), b1 = __ldcg(rb + 1), b2 = __ldcg(rb + 2), b3 = __ldcg(rb + 3);
      fold(a0, a1, a2, a3);
      if (j < nt) fold(b0, b1, b2, b3);
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int idx = warp_transpose_sum16(acc);
  __syncthreads();  // s_dred is free
  if ((lane & 1) == 0) s_dred[warp * 16 + idx] = acc[0];
  __syncthreads();
  if (threadIdx.x < NV) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) t += s_dred[w * 16 + threadIdx.x];
    s_dred[threadIdx.x] = t;  // column threadIdx.x is read by this thread only
  }
  __syncthreads();
  MergedStats r;
  r.max_lw = M;
  if (threadIdx.x == 0) {
    r.w = s_dred[0];
    r.w2 = s_dred[1];
#pragma unroll
    for (int d = 0; d < kMaxD; ++d) r.sx[d] = d < D ? s_dred[2 + d] : 0.0;
#pragma unroll
    for (int i = 0; i < 6; ++i) r.sxx[i] = s_dred[2 + D + i];
  }
  return r;
}

// Maximum tile log-weight of the rows [tb, tb + nt) (whole CTA).
__device__ __forceinline__ float rows_max(const float* part, int tb, int nt, float* s_maxtmp) {
  float m = -INFINITY;
  for (int i = threadIdx.x; i < nt; i += kThreads) m = fmaxf(m, __ldcg(part + (size_t)(tb + i) * kPartStride));
  return block_max(m, s_maxtmp);
}

// As merge_tiles_at, with the maximum taken over the rows first.
template <int D>
__device__ __forceinline__ MergedStats merge_tiles(const float* part, int tb, int nt,
                                                   float* s_maxtmp, double* s_dred) {
  return merge_tiles_at<D>(part, tb, nt, rows_max(part, tb, nt, s_maxtmp), s_dred);
}

// Local offsets -> ECEF: anchor + R^T v.
__device__ __forceinline__ void local_to_ecef(const double* rot, const double* anchor,
                                              double e, double n, double u, double* out) {
  out[0] = anchor[0] + rot[0] * e + rot[3] * n + rot[6] * u;
  out[1] = anchor[1] + rot[1] * e + rot[4] * n + rot[7] * u;
  out[2] = anchor[2] + rot[2] * e + rot[5] * n + rot[8] * u;
}

// -------------------------------------------------------------------------
// Ancestors after a resample.  When the engine keeps segment markers
// (e.anc_seg), a 128-slot segment whose slots all share one ancestor holds
// it in its marker and its slots are not written; other segments' markers
// are -1 and their slots hold the ancestors.  seg_markers is null when every
// slot is written.
__device__ __forceinline__ const int* seg_markers(const EngineDev& e, const FilterDesc* fd) {
  return e.anc_seg ? e.seg_anc + (size_t)fd->tile_begin * kSubTiles : nullptr;
}
__device__ __forceinline__ int ancestor_at(const EngineDev& e, const int* seg, long long base, int j) {
  if (seg) {
    const int u = __ldcg(seg + j / kWarpTile);
    if (u >= 0) return u;
  }
  return __ldcg(e.anc + base + j);
}

// The ancestors of slots [p0, p0+4) (one 128-slot segment).  The marker and
// the slots are loaded together (the slots of a marked segment are stale and
// ignored): one memory latency.
struct AncLoad {
  int4 a;
  int u;
};
__device__ __forceinline__ AncLoad issue_ancestors4(const EngineDev& e, const FilterDesc* fd, long long base, int p0) {
  const int* seg = seg_markers(e, fd);
  AncLoad r;
  r.u = seg ? __ldcg(seg + p0 / kWarpTile) : -1;
  r.a = __ldcg(reinterpret_cast<const int4*>(e.anc + base + p0));
  return r;
}

// Load the 4 particles [p0, p0+4) of the current state (gathering through
// the ancestors when the last step resampled), with the ancestors' loads
// already issued.
template <int D>
__device__ __forceinline__ void load_particles_from(const EngineDev& e, const float* src, long long base, int p0,
                                                    int n, bool gather, const AncLoad& al, float (&x)[D][4]) {
  if (gather) {
    const int4 a = al.u >= 0 ? make_int4(al.u, al.u, al.u, al.u) : al.a;
    int ai[4] = {a.x, a.y, a.z, a.w};
    // slots past the filter's end hold no ancestor; keep every index in range
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (p0 + k >= n || !PF_BOUNDS_OK(e, (unsigned)ai[k] < (unsigned)n)) ai[k] = p0;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      const float* s = src + (size_t)d * e.p_total + base;
#pragma unroll
      for (int k = 0; k < 4; ++k) x[d][k] = __ldcg(s + ai[k]);
    }
  } else {
#pragma unroll
    for (int d = 0; d < D; ++d) {
      float4 v = __ldcs(reinterpret_cast<const float4*>(src + (size_t)d * e.p_total + base + p0));
      x[d][0] = v.x; x[d][1] = v.y; x[d][2] = v.z; x[d][3] = v.w;
    }
  }
}
template <int D>
__device__ __forceinline__ void load_particles(const EngineDev& e, const FilterDesc* fd, const float* src,
                                               long long base, int p0, int n, bool gather,
                                               float (&x)[D][4]) {
  AncLoad al{make_int4(0, 0, 0, 0), -1};
  if (gather) al = issue_ancestors4(e, fd, base, p0);
  load_particles_from<D>(e, src, base, p0, n, gather, al, x);
}


// The systematic offset u (a 32-bit slot fraction) of the step `epoch`:
// the reference's fixed (seed % 1e6)/(1e6 N) (resampling.cu:152) or one
// Philox draw per filter and step.
__device__ __forceinline__ uint32_t sys_offset_u(const EngineDev& e, const FilterDesc* fd, unsigned epoch) {
  if (e.sys_offset == PF_SYS_OFFSET_RANDOM)
    return philox10(U4{0u, epoch, TAG_SYS_U, (uint32_t)fd->filter_id}, fd->key0, fd->key1).x;
  return fd->sys_ref_u;
}

// Tiled integer CDF of the systematic resampler.  Every quantity below is
// an integer smaller than 2^53 (K <= 40: q < 2^41, a segment sum < 2^48, a
// tile sum < 2^51), so it is held exactly as a double and sums are exact.
//
// Segment level (one warp, 128 particles, four per lane): q = floor(2^K
// e^(lw - wm)) against the warp maximum wm (quantize_f32), stored as
// inclusive prefixes inside the segment; returns the segment sum in every
// lane.  lwv is -inf past the filter's end.
__device__ __forceinline__ double warp_incl_scan_f64(double v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}
__device__ __forceinline__ double sys_segment_prefix(const EngineDev& e, long long base, int p0, bool active,
                                                     const float (&lwv)[4], float wm, int K) {
  double q[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) q[k] = (double)quantize_f32(det_fsub(lwv[k], wm), K);
  const double ts = (q[0] + q[1]) + (q[2] + q[3]);
  const double incl = warp_incl_scan_f64(ts);
  const double c0 = (incl - ts) + q[0], c1 = c0 + q[1], c2 = c1 + q[2];
  if (active) {  // the filter's slots are padded to a multiple of 4
    double2* dst = reinterpret_cast<double2*>(e.seg_c + base + p0);
    dst[0] = make_double2(c0, c1);
    dst[1] = make_double2(c2, incl);
  }
  return __shfl_sync(0xffffffffu, incl, 31);
}

// Tile level (one warp; lane w < kThreads/32 holds segment w's sum S and
// maximum mw, tm is the tile maximum): rho_w = e^(mw - tm) (det_expf), the
// rescaled sums floor(S rho_w), their exclusive prefix E_w inside the tile,
// the tile sum S_t and the tile maximum.
__device__ __forceinline__ void sys_tile_scale(const EngineDev& e, int t, double S, float mw, float tm) {
  constexpr int kWarps = kThreads / 32;
  const int lane = threadIdx.x & 31;
  const double rho = S > 0.0 ? (double)det_expf(det_fsub(mw, tm)) : 0.0;
  const double Q = S > 0.0 ? scale_trunc(S, rho) : 0.0;
  double inc = Q;
#pragma unroll
  for (int o = 1; o < kWarps; o <<= 1) {
    const double v = __shfl_up_sync(0xffffffffu, inc, o, kWarps);
    if ((lane & (kWarps - 1)) >= o) inc += v;
  }
  if (lane < kWarps) {
    e.seg_rho[(size_t)t * kSubTiles + lane] = rho;
    e.seg_E[(size_t)t * kSubTiles + lane] = inc - Q;
  }
  if (lane == kWarps - 1) {
    e.tile_S[t] = inc;
    e.tile_m[t] = tm;
  }
}

// The filter-level scale of tile t: Q_t = floor(S_t e^(tm_t - M)) (r_t on
// return) from its sum and maximum.
__device__ __forceinline__ double sys_tile_total(double S, float tm, float M, double& r) {
  r = S > 0.0 ? (double)det_expf(det_fsub(tm, M)) : 0.0;
  return S > 0.0 ? scale_trunc(S, r) : 0.0;
}
__device__ __forceinline__ double sys_tile_total(const EngineDev& e, int t, float M, double& r) {
  return sys_tile_total(__ldcg(e.tile_S + t), __ldcg(e.tile_m + t), M, r);
}

// Particle i of tile t, warp segment s: its filter-wide inclusive prefix is
// C = P_t + floor((E_s + floor(c_i rho_s)) r_t); this returns the second
// term (an integer-valued double).
__device__ __forceinline__ double sys_inner(double E, double rho, double r, double c) {
  return scale_trunc(E + scale_trunc(c, rho), r);
}

// The last tile of a filter: merged statistics -> estimate, covariance,
// ESS, the device-side resample decision (particle_filter.py:159-161), the
// next re-centring shift, the systematic offset, and the epoch/parity step.
// Executed by one thread.
// The device-side resample decision of particle_filter.py:159-161 (ESS
// below threshold x N, or forced; never without finite weights) from the
// merged statistics and the step's epoch flags.  A function of its inputs
// alone, so any CTA holding the same merge reaches the same decision.
__device__ __forceinline__ bool resample_decision(const EngineDev& e, const FilterDesc* fd, const MergedStats& ms,
                                                  int eflags) {
  const bool do_weight = (eflags & PF_EP_WEIGHT) != 0;
  const double W = ms.w;
  const double ess = (ms.w2 > 0.0) ? (W * W) / ms.w2 : 0.0;
  if (!(W > 0.0) || !(ms.max_lw > -INFINITY)) return false;
  return (do_weight || (eflags & PF_EP_RESAMPLE_CHECK)) && !(eflags & PF_EP_NO_RESAMPLE) &&
         ((eflags & PF_EP_FORCE_RESAMPLE) || ess < (double)e.ess_threshold * (double)fd->n);
}

template <int D>
__device__ __forceinline__ void finalize_filter(const EngineDev& e, const FilterDesc* fd, FilterCtrl* fc,
                                                const MergedStats& ms, unsigned epoch, int parity,
                                                bool lw_zero, int eflags, bool do_weight) {
  constexpr int NCLK = D - 3;
  const double W = ms.w;
  const double ess = (ms.w2 > 0.0) ? (W * W) / ms.w2 : 0.0;
  double mu[kMaxD];
#pragma unroll
  for (int d = 0; d < kMaxD; ++d) mu[d] = (W > 0.0 && d < D) ? ms.sx[d] / W : 0.0;
  double A[3];
  local_to_ecef(fd->rot, fc->anchor, fc->shift[0], fc->shift[1], fc->shift[2], A);
  double est[3];
  local_to_ecef(fd->rot, A, mu[0], mu[1], mu[2], est);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    fc->anchor[i] = A[i];
    fc->est_ecef[i] = est[i];
  }
#pragma unroll
  for (int c = 0; c < PF_MAX_CLK; ++c) {
    if (c < NCLK) {
      const double ca = fc->clk_anchor[c] + (double)fc->shift[3 + c];
      fc->clk_anchor[c] = ca;
      fc->est_clk[c] = ca + mu[3 + c];
    } else {
      fc->est_clk[c] = 0.0;
    }
  }
  if ((e.flags & PF_FLAG_COVARIANCE) && W > 0.0) {
    fc->cov[0] = ms.sxx[0] / W - mu[0] * mu[0];
    fc->cov[1] = ms.sxx[1] / W - mu[0] * mu[1];
    fc->cov[2] = ms.sxx[2] / W - mu[0] * mu[2];
    fc->cov[3] = ms.sxx[3] / W - mu[1] * mu[1];
    fc->cov[4] = ms.sxx[4] / W - mu[1] * mu[2];
    fc->cov[5] = ms.sxx[5] / W - mu[2] * mu[2];
  }
  fc->ess = ess;
  fc->sum_w = W;
  fc->max_lw = ms.max_lw;
  const bool recenter = (e.flags & PF_FLAG_RECENTER) != 0 && W > 0.0;
#pragma unroll
  for (int d = 0; d < 8; ++d) fc->shift[d] = (recenter && d < D) ? (float)mu[d] : 0.f;
  const bool rs = resample_decision(e, fd, ms, eflags);
  if ((!(W > 0.0) || !(ms.max_lw > -INFINITY)) && do_weight) atomicOr(e.err, ERR_BAD_WEIGHTS);
  fc->resample_flag = rs ? 1 : 0;
  fc->lw_zero = rs ? 1 : (do_weight ? 0 : (lw_zero ? 1 : 0));
  if (rs) {
    fc->rs_seq = fc->rs_seq + 1u;
    fc->sys_u = sys_offset_u(e, fd, epoch);
  }
  fc->parity = parity ^ 1;
  fc->epoch = epoch + 1u;
  fc->ticket = 0u;
  __threadfence();
}

// -------------------------------------------------------------------------
// k_step: fused predict + weight + statistics (+ per-filter finalize).
//
// Per tile (1024 particles, 4 per thread as one float4 per component):
//   load (gathered through the last resample's ancestors if any) ->
//   predict with Philox/Box-Muller noise -> store -> likelihood over the
//   filter's satellites -> store log-weights -> per-warp statistics with a
//   transpose-style butterfly reduction -> one barrier -> warp 0 merges the
//   eight warp rows into the tile row, takes the filter's ticket and the
//   next tile -> one barrier.  The last tile of a filter merges all tile
//   rows in FP64 and writes the filter's control block.
//
// Satellite constants sit in shared memory as pre-broadcast pairs, so the
// packed f32x2 operations read them without register moves.
#ifndef PF_KSTEP_MINB
#define PF_KSTEP_MINB 2  // resident CTAs per SM the fused step is compiled for
#endif
template <int NCLK, int WMODE>
__global__ void __launch_bounds__(kThreads, PF_KSTEP_MINB) k_step(EngineDev e, int t0, int count) {
  constexpr int D = 3 + NCLK;
  constexpr int NV = 2 + D + 6;  // s, s2, sx[D], xx, xy, xz, yy, yz, zz
  constexpr int kWarps = kThreads / 32;
  __shared__ __align__(16) float2 s_sat[kSatStride * PF_MAX_SATS];
  __shared__ int s_grp[PF_MAX_CLK + 1];
  __shared__ unsigned char s_clk[PF_MAX_SATS];
  __shared__ float s_wrow[kWarps][17];       // per-warp max + NV sums
  __shared__ double s_wq[kWarps];            // per-warp quantised weight sums
  __shared__ float s_maxtmp[kWarps];
  __shared__ double s_dred[kWarps * 16];
  __shared__ int s_next, s_last;

  unsigned* q = e.queue + 2 * Q_STEP;
  pdl_trigger();
  pdl_wait();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_next = (int)atomicAdd(q, 1u);
  __syncthreads();
  int tq = s_next;
  int cached = -1;
  while (tq < count) {
    const int t = t0 + tq;
    const int f = __ldg(e.tile_filter + t);
    const FilterDesc* fd = e.desc + f;
    FilterCtrl* fc = e.ctrl + f;
    const unsigned epoch = fc->epoch;
    const int parity = fc->parity;
    const bool gather = fc->resample_flag != 0;
    const bool lw_zero = fc->lw_zero != 0;
    const unsigned char* ob = e.obs + (size_t)(epoch % (unsigned)e.obs_slots) * e.obs_slot_bytes;
    const pf_filter_epoch_t* fe = reinterpret_cast<const pf_filter_epoch_t*>(ob) + f;
    const pf_sat_t* sats = reinterpret_cast<const pf_sat_t*>(ob + sizeof(pf_filter_epoch_t) * e.n_filters);
    const int eflags = fe->flags;
    int n_sat = fe->n_sat;
    if (n_sat > e.max_sats) {
      if (threadIdx.x == 0) atomicOr(e.err, ERR_SAT_CAP);
      n_sat = e.max_sats;
    }
    if (n_sat < 0) n_sat = 0;
    const bool do_predict = (eflags & PF_EP_PREDICT) != 0;
    const bool do_weight = (eflags & PF_EP_WEIGHT) != 0;
    const bool sys_q = e.resampler == PF_RESAMPLE_SYSTEMATIC &&
                       (do_weight || (eflags & PF_EP_RESAMPLE_CHECK)) && !(eflags & PF_EP_NO_RESAMPLE);

    // ---- per-filter satellite geometry in FP64, stored as FP32 pairs in
    //      smem, grouped by clock state (stable order).
    if (f != cached) {
      int my_c = 0;
      const pf_sat_t* sp = sats + fe->sat_offset + threadIdx.x;
      if (do_weight && threadIdx.x < n_sat) {
        my_c = sp->clk;
        my_c = my_c < 0 ? 0 : (my_c >= NCLK ? NCLK - 1 : my_c);
        s_clk[threadIdx.x] = (unsigned char)my_c;
      }
      __syncthreads();
      if (do_weight && threadIdx.x < n_sat) {
        const double* rot = fd->rot;
        double A[3];
        local_to_ecef(rot, fc->anchor, fc->shift[0], fc->shift[1], fc->shift[2], A);
        const int c = my_c;
        const double clkA = fc->clk_anchor[c] + (double)fc->shift[3 + c];
        double vx = sp->x - A[0], vy = sp->y - A[1], vz = sp->z - A[2];
        const double r0 = sqrt(vx * vx + vy * vy + vz * vz);
        const double inv = 1.0 / r0;
        vx *= inv; vy *= inv; vz *= inv;
        const float eE = (float)(rot[0] * vx + rot[1] * vy + rot[2] * vz);
        const float eN = (float)(rot[3] * vx + rot[4] * vy + rot[5] * vz);
        const float eU = (float)(rot[6] * vx + rot[7] * vy + rot[8] * vz);
        const float g = (float)inv;
        const float y = (float)(sp->pr - r0 - clkA);
        const float wq = WMODE == PF_WEIGHT_GAUSSIAN ? (float)((double)fd->wscale * sp->w) : (float)sp->w;
        int rank = 0;
        for (int s2 = 0; s2 < n_sat; ++s2) {
          const int c2 = s_clk[s2];
          rank += (c2 < c) || (c2 == c && s2 < (int)threadIdx.x);
        }
        write_sat_entry(s_sat + kSatStride * rank, eE, eN, eU, g, y, wq);
      }
      if (threadIdx.x <= NCLK) {
        int cnt = 0;
        if (do_weight)
          for (int s2 = 0; s2 < n_sat; ++s2) cnt += s_clk[s2] < (int)threadIdx.x;
        s_grp[threadIdx.x] = cnt;
      }
      cached = f;
      __syncthreads();
    }

    const int n = fd->n;
    const int j = t - fd->tile_begin;
    const int p0 = j * kTile + (int)threadIdx.x * 4;
    const bool active = p0 < n;
    const long long base = fd->p_off;
    const float* src = parity ? e.state1 : e.state0;
    float* dst = parity ? e.state0 : e.state1;

    float x[D][4];
    float lwv[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
#pragma unroll
    for (int d = 0; d < D; ++d)
#pragma unroll
      for (int k = 0; k < 4; ++k) x[d][k] = 0.f;
    if (active) {
      load_particles<D>(e, fd, src, base, p0, n, gather, x);
      float lw0[4] = {0.f, 0.f, 0.f, 0.f};
      const bool need_prev = !lw_zero && (!do_weight || e.lw_mode == PF_LW_ACCUMULATE);
      if (need_prev) {
        float4 v = __ldcs(reinterpret_cast<const float4*>(e.lw + base + p0));
        lw0[0] = v.x; lw0[1] = v.y; lw0[2] = v.z; lw0[3] = v.w;
      }
      // predict: x += disp - shift + sigma * N(0,1)
      float ds[D];
#pragma unroll
      for (int d = 0; d < D; ++d) ds[d] = -fc->shift[d];
      if (do_predict) {
        ds[0] += (float)fe->disp[0];
        ds[1] += (float)fe->disp[1];
        ds[2] += (float)fe->disp[2];
        const uint32_t fid = (uint32_t)fd->filter_id;
        const uint32_t k0 = fd->key0, k1 = fd->key1;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          float nz[8];
          U4 r = philox10(U4{(uint32_t)(p0 + k), epoch, TAG_PREDICT, fid}, k0, k1);
          float2 a = box_muller_f32(r.x, r.y), b = box_muller_f32(r.z, r.w);
          nz[0] = a.x; nz[1] = a.y; nz[2] = b.x; nz[3] = b.y;
          if (D > 4) {
            U4 r2 = philox10(U4{(uint32_t)(p0 + k), epoch, TAG_PREDICT | 1u, fid}, k0, k1);
            float2 c = box_muller_f32(r2.x, r2.y), dd = box_muller_f32(r2.z, r2.w);
            nz[4] = c.x; nz[5] = c.y; nz[6] = dd.x; nz[7] = dd.y;
          } else {
            nz[4] = nz[5] = nz[6] = nz[7] = 0.f;
          }
#pragma unroll
          for (int d = 0; d < D; ++d) x[d][k] = fmaf(fd->sigma[d], nz[d], x[d][k] + ds[d]);
        }
      } else {
#pragma unroll
        for (int d = 0; d < D; ++d)
#pragma unroll
          for (int k = 0; k < 4; ++k) x[d][k] += ds[d];
      }
#pragma unroll
      for (int d = 0; d < D; ++d)
        __stcs(reinterpret_cast<float4*>(dst + (size_t)d * e.p_total + base + p0),
               make_float4(x[d][0], x[d][1], x[d][2], x[d][3]));

      if (do_weight) {
        float2 lwp[2] = {f2(lw0[0], lw0[1]), f2(lw0[2], lw0[3])};
        float2 dx[2], dy[2], dz[2], nbb[2];
#pragma unroll
        for (int p = 0; p < 2; ++p) {
          dx[p] = f2(x[0][2 * p], x[0][2 * p + 1]);
          dy[p] = f2(x[1][2 * p], x[1][2 * p + 1]);
          dz[p] = f2(x[2][2 * p], x[2][2 * p + 1]);
          float2 bb = __fmul2_rn(dx[p], dx[p]);
          bb = __ffma2_rn(dy[p], dy[p], bb);
          bb = __ffma2_rn(dz[p], dz[p], bb);
          nbb[p] = f2(-bb.x, -bb.y);
        }
#pragma unroll
        for (int c = 0; c < NCLK; ++c) {
          const float2 ncb[2] = {f2(-x[3 + c][0], -x[3 + c][1]), f2(-x[3 + c][2], -x[3 + c][3])};
          const int s_end = s_grp[c + 1];
#pragma unroll 2
          for (int s = s_grp[c]; s < s_end; ++s) {
#pragma unroll
            for (int p = 0; p < 2; ++p)
              sat_pair_update<WMODE>(s_sat + kSatStride * s, dx[p], dy[p], dz[p], nbb[p], ncb[p], lwp[p], fd);
          }
        }
        lwv[0] = lwp[0].x; lwv[1] = lwp[0].y; lwv[2] = lwp[1].x; lwv[3] = lwp[1].y;
        __stcs(reinterpret_cast<float4*>(e.lw + base + p0), make_float4(lwv[0], lwv[1], lwv[2], lwv[3]));
      } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) lwv[k] = lw0[k];
        // reset weights live only in the control block: a resample test of
        // them (no weight pass) reads the array, so it is zeroed first
        if (lw_zero && (eflags & PF_EP_RESAMPLE_CHECK) && !(eflags & PF_EP_NO_RESAMPLE))
          __stcs(reinterpret_cast<float4*>(e.lw + base + p0), make_float4(0.f, 0.f, 0.f, 0.f));
      }
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (p0 + k >= n) lwv[k] = -INFINITY;
    }

    // ---- per-warp statistics (own max), butterfly-transposed sums
    {
      float wm = fmaxf(fmaxf(lwv[0], lwv[1]), fmaxf(lwv[2], lwv[3]));
      wm = warp_max(wm);
      float v[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = 0.f;
      if (wm > -INFINITY) {
        const bool cov = (e.flags & PF_FLAG_COVARIANCE) != 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const float w = exp2f((lwv[k] - wm) * 1.4426950408889634f);
          v[0] += w;
          v[1] = fmaf(w, w, v[1]);
#pragma unroll
          for (int d = 0; d < D; ++d) v[2 + d] = fmaf(w, x[d][k], v[2 + d]);
          if (cov) {
            const float wx = w * x[0][k], wy = w * x[1][k], wz = w * x[2][k];
            v[2 + D + 0] = fmaf(wx, x[0][k], v[2 + D + 0]);
            v[2 + D + 1] = fmaf(wx, x[1][k], v[2 + D + 1]);
            v[2 + D + 2] = fmaf(wx, x[2][k], v[2 + D + 2]);
            v[2 + D + 3] = fmaf(wy, x[1][k], v[2 + D + 3]);
            v[2 + D + 4] = fmaf(wy, x[2][k], v[2 + D + 4]);
            v[2 + D + 5] = fmaf(wz, x[2][k], v[2 + D + 5]);
          }
        }
      }
      const int idx = warp_transpose_sum16(v);  // lane holds the warp total of value idx
      if ((lane & 1) == 0 && idx < NV) s_wrow[warp][1 + idx] = v[0];
      if (lane == 0) s_wrow[warp][0] = wm;
      // tiled integer CDF of the systematic resampler, segment level
      double seg_sum = 0.0;
      if (sys_q) seg_sum = sys_segment_prefix(e, base, p0, active, lwv, wm, fd->K);
      if (lane == 0) s_wq[warp] = seg_sum;
    }
    __syncthreads();
    if (warp == 0) {
      // merge the warp rows: lane i < NV sums value i with max-shift scales
      float tm = lane < kWarps ? s_wrow[lane][0] : -INFINITY;
      tm = warp_max(tm);
      float acc = 0.f;
      if (lane < NV && tm > -INFINITY) {
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
          const float mw = s_wrow[w][0];
          if (mw > -INFINITY) {
            float sc = exp2f((mw - tm) * 1.4426950408889634f);
            if (lane == 1) sc *= sc;
            acc = fmaf(sc, s_wrow[w][1 + lane], acc);
          }
        }
      }
      float* row = e.part + (size_t)t * kPartStride;
      if (lane < NV) row[1 + lane] = acc;
      if (lane == 0) row[0] = tm;
      if (sys_q)
        sys_tile_scale(e, t, lane < kWarps ? s_wq[lane] : 0.0, lane < kWarps ? s_wrow[lane][0] : -INFINITY, tm);
      __syncwarp();
      if (lane == 0) {
        __threadfence();
        const unsigned old = atomicAdd(&fc->ticket, 1u);
        s_last = (old == (unsigned)fd->n_tiles - 1u);
        s_next = (int)atomicAdd(q, 1u);
      }
    }
    __syncthreads();
    const int next = s_next;
    if (s_last) {
      __threadfence();
      MergedStats ms = merge_tiles<D>(e.part, fd->tile_begin, fd->n_tiles, s_maxtmp, s_dred);
      if (threadIdx.x == 0) finalize_filter<D>(e, fd, fc, ms, epoch, parity, lw_zero, eflags, do_weight);
      __syncthreads();
    }
    tq = next;
  }
  queue_exit(q);
}

// -------------------------------------------------------------------------
// Quantised weights of particles [p0, p0+4): from the FP32 log-weights of
// the engine, or from FP64 log-weights when the stateless API set lw64.
// The shift lw - max is exact in FP64 for FP32 inputs.
__device__ __forceinline__ void load_q4(const EngineDev& e, long long base, int p0, int n, float M,
                                        int K, unsigned long long (&q)[4]) {
  q[0] = q[1] = q[2] = q[3] = 0ull;
  if (p0 >= n) return;
  if (e.lw64) {
    const double m64 = __ldcg(e.lw64_max);
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (p0 + k < n) q[k] = quantize_shifted(__ldcg(e.lw64 + base + p0 + k) - m64, K);
  } else {
    const float4 v = __ldcg(reinterpret_cast<const float4*>(e.lw + base + p0));
    const float l[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (p0 + k < n) q[k] = quantize_shifted((double)l[k] - (double)M, K);
  }
}

// -------------------------------------------------------------------------
// k_scan: tile sums of the integer CDF, decoupled look-back over tiles.  The
// stateless API's FP64 log-weights (lw64) use the plain integer CDF against
// the global maximum instead: quantised weights summed per tile here.
__global__ void __launch_bounds__(kThreads) k_scan(EngineDev e, int t0, int count) {
  __shared__ unsigned long long s_u64[kThreads / 32];
  __shared__ int s_slot, s_first;
  unsigned* q = e.queue + 2 * Q_SCAN;
  pdl_trigger();
  pdl_wait();
  for (;;) {
    const int tq = dequeue(q, &s_slot);
    if (tq >= count) break;
    const int t = t0 + tq;
    const int f = __ldg(e.tile_filter + t);
    const FilterDesc* fd = e.desc + f;
    FilterCtrl* fc = e.ctrl + f;
    if (!fc->resample_flag) continue;
    const int n = fd->n, K = fd->K;
    const float M = fc->max_lw;
    const unsigned tag = (fc->rs_seq & 0x3FFFFFFFu) << 2;
    const int tb = fd->tile_begin, j = t - tb;
    const int p0 = j * kTile + (int)threadIdx.x * 4;
    const long long base = fd->p_off;
    unsigned long long tot;
    if (e.lw64) {  // stateless API: the plain integer CDF of the FP64 log-weights
      unsigned long long qv[4];
      load_q4(e, base, p0, n, M, K, qv);
      block_excl_scan_u64(qv[0] + qv[1] + qv[2] + qv[3], s_u64, &tot);
    } else {  // engine: the tile's sum of the tiled integer CDF, scaled to the filter maximum
      double r;
      tot = (unsigned long long)sys_tile_total(e, t, M, r);
    }
    unsigned long long excl = 0;
    if (j == 0) {
      if (threadIdx.x == 0) {
        e.lb_inc[t] = tot;
        __threadfence();
        atomicExch(e.lb_flag + t, tag | 2u);
      }
    } else {
      if (threadIdx.x == 0) {
        e.lb_agg[t] = tot;
        __threadfence();
        atomicExch(e.lb_flag + t, tag | 1u);
      }
      // Look back over a window of kThreads predecessors per round: thread
      // i inspects tile pred - i.  The sum stops at the closest predecessor
      // that published an inclusive prefix.  Spins are bounded; when the
      // limit is reached the error word is set and the scan moves on.
      const unsigned want = e.lookback_poison ? ((tag + 4u) >> 2) : (tag >> 2);
      int pred = t - 1;
      for (;;) {
        const int idx = pred - (int)threadIdx.x;
        const bool inr = idx >= tb;
        unsigned fl = 0;
        bool ok = !inr;
        unsigned long long spins = 0;
        bool timed_out = false;
        for (;;) {
          if (!ok) {
            fl = *(volatile unsigned*)(e.lb_flag + idx);
            ok = ((fl >> 2) == want) && ((fl & 3u) != 0u);
          }
          if (__syncthreads_and(ok)) break;
          if (++spins > e.spin_limit) {  // uniform across the CTA
            timed_out = true;
            break;
          }
          if (spins > 32) __nanosleep(64);
        }
        if (timed_out) {
          if (threadIdx.x == 0) atomicOr(e.err, ERR_LOOKBACK_TIMEOUT);
          break;
        }
        __threadfence();
        const bool is_inc = inr && ((fl & 3u) == 2u);
        if (threadIdx.x == 0) s_first = kThreads;
        __syncthreads();
        if (is_inc) atomicMin(&s_first, (int)threadIdx.x);
        __syncthreads();
        const int first = s_first;  // closest predecessor with a prefix
        unsigned long long val = 0;
        if (inr && (int)threadIdx.x <= first)
          val = is_inc ? *(volatile unsigned long long*)(e.lb_inc + idx)
                       : *(volatile unsigned long long*)(e.lb_agg + idx);
        unsigned long long round_sum;
        block_excl_scan_u64(val, s_u64, &round_sum);
        excl += round_sum;
        pred -= kThreads;
        if (first < kThreads || pred < tb) break;
      }
      if (threadIdx.x == 0) {
        e.lb_inc[t] = excl + tot;
        __threadfence();
        atomicExch(e.lb_flag + t, tag | 2u);
      }
    }
    if (threadIdx.x == 0) {
      e.tile_excl[t] = excl;
      if (j == fd->n_tiles - 1) fc->wq_total = excl + tot;
    }
  }
  queue_exit(q);
}

// -------------------------------------------------------------------------
// k_offs: inclusive CDF of every particle, its offspring end F(i), and the
// merge-path partition points of the filter's diagonal tiles.
__global__ void __launch_bounds__(kThreads) k_offs(EngineDev e, int t0, int count) {
  __shared__ unsigned long long s_u64[kThreads / 32];
  __shared__ int s_slot;
  unsigned* q = e.queue + 2 * Q_OFFS;
  pdl_trigger();
  pdl_wait();
  for (;;) {
    const int tq = dequeue(q, &s_slot);
    if (tq >= count) break;
    const int t = t0 + tq;
    const int f = __ldg(e.tile_filter + t);
    const FilterDesc* fd = e.desc + f;
    const FilterCtrl* fc = e.ctrl + f;
    if (!fc->resample_flag) continue;
    const int n = fd->n, K = fd->K;
    const float M = fc->max_lw;
    const unsigned long long W = fc->wq_total;
    const uint32_t u = fc->sys_u;
    const int tb = fd->tile_begin, j = t - tb;
    const int p0 = j * kTile + (int)threadIdx.x * 4;
    const long long base = fd->p_off;
    // inclusive CDF before this thread's particles (Cp) and after each (Ck)
    unsigned long long Cp = 0ull, Ck[4] = {0ull, 0ull, 0ull, 0ull};
    const int lane = threadIdx.x & 31;
    if (e.lw64) {  // stateless API: plain integer CDF
      unsigned long long qv[4];
      load_q4(e, base, p0, n, M, K, qv);
      unsigned long long tot;
      Cp = __ldcg(e.tile_excl + t) + block_excl_scan_u64(qv[0] + qv[1] + qv[2] + qv[3], s_u64, &tot);
      unsigned long long C = Cp;
#pragma unroll
      for (int k = 0; k < 4; ++k) Ck[k] = (C += qv[k]);
    } else {  // engine: tiled integer CDF (segment prefixes written by k_step)
      const int w = threadIdx.x >> 5;
      double r;
      (void)sys_tile_total(e, t, M, r);
      const double rho = __ldcg(e.seg_rho + (size_t)t * kSubTiles + w);
      const double E = __ldcg(e.seg_E + (size_t)t * kSubTiles + w);
      const unsigned long long P = __ldcg(e.tile_excl + t);
      double c[4] = {0.0, 0.0, 0.0, 0.0};
      if (p0 < n) {
        const double2* src = reinterpret_cast<const double2*>(e.seg_c + base + p0);
        const double2 a = __ldcg(src), b = __ldcg(src + 1);
        c[0] = a.x; c[1] = a.y; c[2] = b.x; c[3] = b.y;
      }
      double cprev = __shfl_up_sync(0xffffffffu, c[3], 1);
      if (lane == 0) cprev = 0.0;
      Cp = P + (unsigned long long)sys_inner(E, rho, r, cprev);
#pragma unroll
      for (int k = 0; k < 4; ++k) Ck[k] = P + (unsigned long long)sys_inner(E, rho, r, c[k]);
    }
    if (W == 0ull) {  // uniform over the CTA (one filter per tile)
      if (threadIdx.x == 0) atomicOr(e.err, ERR_BAD_WEIGHTS);
      continue;
    }
    uint32_t Fprev = 0u, Fk[4] = {0u, 0u, 0u, 0u};
    if (p0 < n) {
      const double scale = (double)n / (double)W, uf = (double)u * 2.3283064365386963e-10;
      Fprev = (p0 == 0) ? 0u : offspring_end_scaled(Cp, W, (uint32_t)n, u, scale, uf);
#pragma unroll
      for (int k = 0; k < 4; ++k)
        Fk[k] = (p0 + k < n) ? offspring_end_scaled(Ck[k], W, (uint32_t)n, u, scale, uf) : (uint32_t)n;
      *reinterpret_cast<uint4*>(e.offs + base + p0) = make_uint4(Fk[0], Fk[1], Fk[2], Fk[3]);
    }
    // merge-path tile starts: tile c begins in particle i when
    // i - 1 + F(i-1) < c * kMergeDiag <= i + F(i); each lane's run of starts
    // is written by the whole warp (heavy particles start many tiles)
#pragma unroll 1
    for (int k = 0; k < 4; ++k) {
      long long c_lo = 0, c_hi = 0;
      if (p0 + k < n) {
        const long long i = p0 + k;
        const long long hprev = i - 1 + (long long)(k == 0 ? Fprev : Fk[k - 1]);
        const long long h = i + (long long)Fk[k];
        c_lo = (hprev < 0) ? 0 : hprev / kMergeDiag + 1;
        c_hi = h / kMergeDiag + 1;
      }
      unsigned runs = __ballot_sync(0xffffffffu, c_hi > c_lo);
      while (runs) {
        const int src = __ffs(runs) - 1;
        runs &= runs - 1u;
        const long long lo = __shfl_sync(0xffffffffu, c_lo, src), hi = __shfl_sync(0xffffffffu, c_hi, src);
        const uint32_t iv = (uint32_t)(p0 - lane * 4 + src * 4 + k);
        for (long long c = lo + lane; c < hi; c += 32) e.mp_part[tb + c] = iv;
      }
    }
  }
  queue_exit(q);
}

// -------------------------------------------------------------------------
// Merge path of one diagonal tile (t - tile_begin = c): walk the merge of
// (offspring ends F, slots) over diagonals [c*2*kTile, (c+1)*2*kTile); slot
// k gets ancestor i when F(i-1) <= k < F(i).  s_F: 2*kTile+1 words of smem.
__device__ __forceinline__ void merge_tile(const EngineDev& e, const FilterDesc* fd, int t, uint32_t* s_F) {
  constexpr int kSteps = kMergeDiag / kThreads;  // 8
  const int n = fd->n;
  const int tb = fd->tile_begin, c = t - tb;
  const long long base = fd->p_off;
  const long long d0 = (long long)c * kMergeDiag;
  const long long dend = min(d0 + kMergeDiag, 2ll * n);
  const int i0 = (int)__ldcg(e.mp_part + t);
  if (i0 < 0 || i0 >= n) {  // cannot happen with valid weights; never index with it
    if (threadIdx.x == 0) atomicOr(e.err, ERR_BAD_WEIGHTS);
    return;
  }
  const int win = min(kMergeDiag + 1, n - i0);
  __syncthreads();  // the window buffer is free
  for (int w = threadIdx.x; w < win; w += kThreads) s_F[w] = __ldcg(e.offs + base + i0 + w);
  __syncthreads();
  const long long d = d0 + (long long)threadIdx.x * kSteps;
  if (d < dend) {
    int lo = 0, hi = (int)min((long long)(win - 1), d - d0);
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if ((long long)(i0 + mid) + (long long)s_F[mid] >= d) hi = mid;
      else lo = mid + 1;
    }
    int i = i0 + lo;
    long long k = d - i;
    const int steps = (int)min((long long)kSteps, dend - d);
    for (int s = 0; s < steps; ++s) {
      const int wi = i - i0;
      if (wi >= win) break;
      if (k < (long long)s_F[wi]) {
        if (k >= 0 && k < n) e.anc[base + k] = i;
        ++k;
      } else {
        ++i;
      }
    }
  }
}

// k_merge: merge_tile over the launch's tiles.
__global__ void __launch_bounds__(kThreads) k_merge(EngineDev e, int t0, int count) {
  __shared__ uint32_t s_F[kMergeDiag + 1];
  __shared__ int s_slot;
  unsigned* q = e.queue + 2 * Q_MERGE;
  pdl_trigger();
  pdl_wait();
  for (;;) {
    const int tq = dequeue(q, &s_slot);
    if (tq >= count) break;
    const int t = t0 + tq;
    const int f = __ldg(e.tile_filter + t);
    const FilterDesc* fd = e.desc + f;
    const FilterCtrl* fc = e.ctrl + f;
    if (!fc->resample_flag) continue;
    merge_tile(e, fd, t, s_F);
  }
  queue_exit(q);
}

// -------------------------------------------------------------------------
// Megopolis (Chesser et al., arXiv:2109.13504) for the slots of one tile,
// the ancestor and its log-weight in registers.  Iteration b proposes
// j = (k + o_{b,g}) mod N with one random offset per (iteration, 32-slot
// segment g), so a warp reads 32 consecutive candidate weights, and accepts
// with probability min(1, w_j / w_ancestor).  `epoch` is the step that
// decided to resample.  Log-weights are read through L2 (another CTA of the
// same launch may have written them).
__device__ __forceinline__ void mego_tile(const EngineDev& e, const FilterDesc* fd, unsigned epoch, int t) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int n = fd->n;
  const int j = t - fd->tile_begin;
  const long long base = fd->p_off;
  const uint32_t fid = (uint32_t)fd->filter_id;
  const int B = e.mego_iters;
  const float* lw = e.lw + base;
  // The warp's four 32-slot segments r (slots j*1024 + r*256 + warp*32 +
  // lane) run their chains side by side (four independent dependency chains
  // per lane).  Iteration b's offsets of all four come from one Philox call,
  // counter (quad, epoch, TAG_MEGO_OFF | b, filter) with quad = j*8 + warp,
  // word r for segment r, computed by lane b % 32; slot k's acceptance
  // uniforms are 16-bit halves, eight per call with counter (k, epoch,
  // TAG_MEGO_U | b/8, filter): word (b % 8)/2, low half for even b.  The
  // candidates do not depend on the chain, so a block of eight iterations
  // loads its 32 candidate log-weights per lane before any comparison.
  const uint32_t quad = (uint32_t)(j * kSubTiles + warp);
  int k[4], a[4];
  float la[4];
  bool valid[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int seg0 = j * kTile + r * kThreads + warp * 32;  // segment's first slot
    const bool act = seg0 < n;                               // warp-uniform
    const int k_real = seg0 + lane;
    valid[r] = act && k_real < n;
    k[r] = valid[r] ? k_real : (act ? seg0 : 0);  // lanes past the end shadow a valid slot
    a[r] = k[r];
    la[r] = __ldcg(lw + k[r]);
  }
#pragma unroll 1
  for (int c0 = 0; c0 < B; c0 += 32) {
    // lane b % 32 draws iteration b's four offsets and scales them to [0, n)
    const U4 ol = philox10(U4{quad, epoch, TAG_MEGO_OFF | (uint32_t)(c0 + lane), fid}, fd->key0, fd->key1);
    const uint32_t osc[4] = {__umulhi(ol.x, (uint32_t)n), __umulhi(ol.y, (uint32_t)n), __umulhi(ol.z, (uint32_t)n),
                             __umulhi(ol.w, (uint32_t)n)};
#pragma unroll 1
    for (int b0 = c0; b0 < min(B, c0 + 32); b0 += 8) {
      U4 ur[4];
#pragma unroll
      for (int r = 0; r < 4; ++r)
        ur[r] = philox10(U4{(uint32_t)k[r], epoch, TAG_MEGO_U | (uint32_t)(b0 >> 3), fid}, fd->key0, fd->key1);
      const int nb = min(8, B - b0);
      if (nb == 8) {
        // a full block of eight iterations: every candidate's log-weight is
        // loaded first (they do not depend on the chain), then the chains run
        float lc[8][4];
        int cand[8][4];
#pragma unroll
        for (int bb = 0; bb < 8; ++bb)
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            int c = k[r] + (int)__shfl_sync(0xffffffffu, osc[r], (b0 + bb) & 31);
            if (c >= n) c -= n;
            cand[bb][r] = c;
            lc[bb][r] = __ldcg(lw + c);
          }
#pragma unroll
        for (int bb = 0; bb < 8; ++bb)
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const uint32_t w32 = (bb >> 1) == 0 ? ur[r].x : (bb >> 1) == 1 ? ur[r].y : (bb >> 1) == 2 ? ur[r].z : ur[r].w;
            const uint32_t h = (bb & 1) ? (w32 >> 16) : (w32 & 0xFFFFu);
            const float lu = __logf(fmaf((float)h, 1.52587890625e-05f, 7.62939453125e-06f));  // (h + 1/2) 2^-16
            if (lc[bb][r] - la[r] > lu) {
              a[r] = cand[bb][r];
              la[r] = lc[bb][r];
            }
          }
      } else {
        for (int bb = 0; bb < nb; ++bb) {
          const int src_lane = (b0 + bb) & 31;
          uint32_t ow[4];
#pragma unroll
          for (int r = 0; r < 4; ++r) ow[r] = __shfl_sync(0xffffffffu, osc[r], src_lane);
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const uint32_t w32 = (bb >> 1) == 0 ? ur[r].x : (bb >> 1) == 1 ? ur[r].y : (bb >> 1) == 2 ? ur[r].z : ur[r].w;
            const uint32_t h = (bb & 1) ? (w32 >> 16) : (w32 & 0xFFFFu);
            int cand = k[r] + (int)ow[r];
            if (cand >= n) cand -= n;
            const float lc = __ldcg(lw + cand);
            const float lu = __logf(fmaf((float)h, 1.52587890625e-05f, 7.62939453125e-06f));
            if (lc - la[r] > lu) {
              a[r] = cand;
              la[r] = lc;
            }
          }
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < 4; ++r)
    if (valid[r]) e.anc[base + k[r]] = a[r];
}

// k_mego: mego_tile over the launch's tiles.
__global__ void __launch_bounds__(kThreads) k_mego(EngineDev e, int t0, int count) {
  __shared__ int s_slot;
  unsigned* q = e.queue + 2 * Q_MEGO;
  pdl_trigger();
  pdl_wait();
  for (;;) {
    const int tq = dequeue(q, &s_slot);
    if (tq >= count) break;
    const int t = t0 + tq;
    const int f = __ldg(e.tile_filter + t);
    const FilterDesc* fd = e.desc + f;
    const FilterCtrl* fc = e.ctrl + f;
    if (!fc->resample_flag) continue;
    mego_tile(e, fd, fc->epoch - 1u, t);
  }
  queue_exit(q);
}

// -------------------------------------------------------------------------
// k_init: N(0, spread) offsets about the anchor into state buffer 0.
template <int D>
__global__ void __launch_bounds__(kThreads) k_init(EngineDev e, int t0, int count,
                                                    float spread_pos, float spread_clk) {
  __shared__ int s_slot;
  unsigned* q = e.queue + 2 * Q_INIT;
  pdl_trigger();
  pdl_wait();
  for (;;) {
    const int tq = dequeue(q, &s_slot);
    if (tq >= count) break;
    const int t = t0 + tq;
    const int f = __ldg(e.tile_filter + t);
    const FilterDesc* fd = e.desc + f;
    const int n = fd->n, j = t - fd->tile_begin;
    const int p0 = j * kTile + (int)threadIdx.x * 4;
    if (p0 >= n) continue;
    const long long base = fd->p_off;
    const uint32_t fid = (uint32_t)fd->filter_id;
    float x[D][4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      float nz[8];
      U4 r = philox10(U4{(uint32_t)(p0 + k), 0u, TAG_INIT, fid}, fd->key0, fd->key1);
      float2 a = box_muller_f32(r.x, r.y), b = box_muller_f32(r.z, r.w);
      nz[0] = a.x; nz[1] = a.y; nz[2] = b.x; nz[3] = b.y;
      if (D > 4) {
        U4 r2 = philox10(U4{(uint32_t)(p0 + k), 0u, TAG_INIT | 1u, fid}, fd->key0, fd->key1);
        float2 c = box_muller_f32(r2.x, r2.y), dd = box_muller_f32(r2.z, r2.w);
        nz[4] = c.x; nz[5] = c.y; nz[6] = dd.x; nz[7] = dd.y;
      } else {
        nz[4] = nz[5] = nz[6] = nz[7] = 0.f;
      }
#pragma unroll
      for (int d = 0; d < D; ++d) x[d][k] = (d < 3 ? spread_pos : spread_clk) * nz[d];
    }
#pragma unroll
    for (int d = 0; d < D; ++d)
      *reinterpret_cast<float4*>(e.state0 + (size_t)d * e.p_total + base + p0) =
          make_float4(x[d][0], x[d][1], x[d][2], x[d][3]);
    *reinterpret_cast<float4*>(e.lw + base + p0) = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  queue_exit(q);
}

// -------------------------------------------------------------------------
// k_estimate: weighted mean over the current particle set with the current
// log-weights (zeros after a resample) -- the reference's pf_estimate
// semantics (weight.cu:163-220,301-321) -- plus the ESS of those weights
// (pf_device.cu:924) and the weighted second moments of the local position
// offsets (for the position spread, pf_device.cu:1025).
template <int D>
__global__ void __launch_bounds__(kThreads) k_estimate(EngineDev e, int t0, int count) {
  __shared__ float s_red[kThreads / 32][kPartStride];
  __shared__ float s_maxtmp[kThreads / 32];
  __shared__ double s_dred[(kThreads / 32) * 16];
  __shared__ int s_slot, s_last;
  unsigned* q = e.queue + 2 * Q_EST;
  pdl_trigger();
  pdl_wait();
  for (;;) {
    const int tq = dequeue(q, &s_slot);
    if (tq >= count) break;
    const int t = t0 + tq;
    const int f = __ldg(e.tile_filter + t);
    const FilterDesc* fd = e.desc + f;
    FilterCtrl* fc = e.ctrl + f;
    const int n = fd->n, j = t - fd->tile_begin;
    const int p0 = j * kTile + (int)threadIdx.x * 4;
    const long long base = fd->p_off;
    const float* src = fc->parity ? e.state1 : e.state0;
    float x[D][4];
    float lwv[4];
#pragma unroll
    for (int d = 0; d < D; ++d)
#pragma unroll
      for (int k = 0; k < 4; ++k) x[d][k] = 0.f;
    if (p0 < n) {
      load_particles<D>(e, fd, src, base, p0, n, fc->resample_flag != 0, x);
      if (fc->lw_zero) {
        lwv[0] = lwv[1] = lwv[2] = lwv[3] = 0.f;
      } else {
        float4 v = __ldcg(reinterpret_cast<const float4*>(e.lw + base + p0));
        lwv[0] = v.x; lwv[1] = v.y; lwv[2] = v.z; lwv[3] = v.w;
      }
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (p0 + k >= n) lwv[k] = -INFINITY;
    } else {
      lwv[0] = lwv[1] = lwv[2] = lwv[3] = -INFINITY;
    }
    tile_stats<D>(x, lwv, true, e.part + (size_t)t * kPartStride, s_maxtmp, s_red);
    if (threadIdx.x == 0) {
      __threadfence();
      unsigned old = atomicAdd(&fc->est_ticket, 1u);
      s_last = (old == (unsigned)fd->n_tiles - 1u);
    }
    __syncthreads();
    if (s_last) {
      __threadfence();
      MergedStats ms = merge_tiles<D>(e.part, fd->tile_begin, fd->n_tiles, s_maxtmp, s_dred);
      if (threadIdx.x == 0) {
        const double W = ms.w;
        double est[3];
        local_to_ecef(fd->rot, fc->anchor, ms.sx[0] / W, ms.sx[1] / W, ms.sx[2] / W, est);
        fc->api_est[0] = est[0];
        fc->api_est[1] = est[1];
        fc->api_est[2] = est[2];
#pragma unroll
        for (int c = 0; c < D - 3; ++c) fc->api_est[3 + c] = fc->clk_anchor[c] + ms.sx[3 + c] / W;
        fc->api_est[7] = (ms.w2 > 0.0) ? W * W / ms.w2 : 0.0;
#pragma unroll
        for (int i = 0; i < 6; ++i) fc->api_m2[i] = ms.sxx[i] / W;
        fc->est_ticket = 0u;
        __threadfence();
      }
      __syncthreads();
    }
  }
  queue_exit(q);
}

// -------------------------------------------------------------------------
// k_position_term: adds log sum_j pi_j exp(-|p - ref_j|^2 / (2 sigma^2)) to
// the log-weights of filter f's current particles (gathered through the
// last resample, if any; weights read as zero when the filter's weights
// were reset).  References are in the filter's local frame relative to its
// anchor (pf_device.cu:889-900 for one reference).
constexpr int kMaxPosRefs = 64;
struct PosTerm {
  float ref[kMaxPosRefs][3];
  float logpi[kMaxPosRefs];
  int K;
  float inv_2s2;
};

template <int D>
__global__ void __launch_bounds__(kThreads) k_position_term(EngineDev e, int f, PosTerm pt) {
  const FilterDesc* fd = e.desc + f;
  const FilterCtrl* fc = e.ctrl + f;
  const int n = fd->n;
  const long long base = fd->p_off;
  const float* src = fc->parity ? e.state1 : e.state0;
  const bool zero = fc->lw_zero != 0;
  for (int p0 = (blockIdx.x * kThreads + threadIdx.x) * 4; p0 < n; p0 += gridDim.x * kThreads * 4) {
    float x[D][4];
    load_particles<D>(e, fd, src, base, p0, n, fc->resample_flag != 0, x);
    float4 l = zero ? make_float4(0.f, 0.f, 0.f, 0.f) : *reinterpret_cast<const float4*>(e.lw + base + p0);
    float lv[4] = {l.x, l.y, l.z, l.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      float m = -INFINITY, acc = 0.f;
      for (int j = 0; j < pt.K; ++j) {
        const float dx = x[0][k] - pt.ref[j][0], dy = x[1][k] - pt.ref[j][1], dz = x[2][k] - pt.ref[j][2];
        const float v = pt.logpi[j] - pt.inv_2s2 * (dx * dx + dy * dy + dz * dz);
        if (!(v > -INFINITY)) continue;  // a component of weight zero
        if (v > m) {
          acc = acc * __expf(m - v) + 1.f;
          m = v;
        } else {
          acc += __expf(v - m);
        }
      }
      lv[k] += (m > -INFINITY) ? m + __logf(acc) : -INFINITY;
    }
    *reinterpret_cast<float4*>(e.lw + base + p0) = make_float4(lv[0], lv[1], lv[2], lv[3]);
  }
}

// -------------------------------------------------------------------------
// k_export: current particles as FP64 ECEF rows [n][D] (x, y, z, clocks),
// the reference's pf_get_particles layout (weight.cu:331-340).
template <int D>
__global__ void __launch_bounds__(kThreads) k_export(EngineDev e, int t0, int count, double* out) {
  __shared__ int s_slot;
  unsigned* q = e.queue + 2 * Q_EXPORT;
  pdl_trigger();
  pdl_wait();
  for (;;) {
    const int tq = dequeue(q, &s_slot);
    if (tq >= count) break;
    const int t = t0 + tq;
    const int f = __ldg(e.tile_filter + t);
    const FilterDesc* fd = e.desc + f;
    const FilterCtrl* fc = e.ctrl + f;
    const int n = fd->n, j = t - fd->tile_begin;
    const int p0 = j * kTile + (int)threadIdx.x * 4;
    if (p0 >= n) continue;
    const long long base = fd->p_off;
    const float* src = fc->parity ? e.state1 : e.state0;
    float x[D][4];
    load_particles<D>(e, fd, src, base, p0, n, fc->resample_flag != 0, x);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (p0 + k >= n) break;
      double p[3];
      local_to_ecef(fd->rot, fc->anchor, (double)x[0][k], (double)x[1][k], (double)x[2][k], p);
      double* o = out + (size_t)(p0 + k) * D;
      o[0] = p[0];
      o[1] = p[1];
      o[2] = p[2];
#pragma unroll
      for (int c = 0; c < D - 3; ++c) o[3 + c] = fc->clk_anchor[c] + (double)x[3 + c][k];
    }
  }
  queue_exit(q);
}

}  // namespace pfb
