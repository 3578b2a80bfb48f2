// pf_epoch_kernel.cuh -- one cooperative persistent kernel per epoch.
//
// All CTAs are co-resident (cooperative launch); each owns a contiguous
// chunk of (filter, tile) work items and the phases of the epoch are
// separated by one grid barrier with bounded spins:
//
//   1  predict + likelihood + tile statistics (particles loaded straight
//      into registers, gathered through the last resample's ancestors;
//      measured faster than staging them through shared memory with
//      cp.async).  Systematic: also the segment and tile levels of the
//      tiled integer CDF -- each warp quantises its 128 particles against
//      its own maximum and stores their prefixes inside the segment, warp 0
//      rescales the segment sums exactly to the tile maximum.
//   -- barrier
//   2  per-filter merge of the tile rows (filter f_first + j by CTA j mod G):
//      ESS, weighted mean / covariance, device-side resample decision.
//      At the same time, systematic only, on the CTAs that own no filter
//      (when filters are fewer than a quarter of the CTAs; otherwise every
//      CTA after its merges):
//   4  the filter maximum from the tile maxima, tile sums rescaled to it,
//      the filter prefix of each tile, then per particle its filter-wide CDF
//      and offspring end F(i); slots [F(i-1), F(i)) get ancestor i, written
//      by the lane when the run is short and by the warp when it is long,
//      where a 128-slot segment the run covers gets one marker word instead
//      of 128 slots (speculative for every filter that may resample: the
//      decision is taken meanwhile).  The kernel ends there.
//   Megopolis instead: every CTA takes the resample decision for the
//   filters of its tiles from the owner's merge (recomputed, bit-identical),
//   then runs the chain per slot of its tiles.  The kernel ends there.
//
// Compared with one kernel per phase this removes the launch/drain gaps and
// every per-tile queue atomic; the prefixes reread in phase 4 come from L2
// (the epoch just wrote them).  Phase 4 needs no CTA barrier per tile: warps
// work on independent segments.
#pragma once
#include "pf_engine_kernels.cuh"
#include "pf_learned.cuh"
#include "pf_generic.cuh"

namespace pfb {

__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned ld_relaxed(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// Grid barrier for co-resident CTAs (sense reversal on one arrival counter).
// bar[1] is the generation (the count of barriers passed over all launches),
// bar[kBarCount] the arrivals at the current barrier; `gen` is this CTA's
// copy of the generation.  Thread 0 of every CTA adds its arrival with one
// acquire-release atomic (the release publishes the writes its CTA ordered
// before it with __syncthreads); the CTA that arrives last resets the
// counter and releases the grid with one store of the next generation,
// which the others poll (relaxed loads, then one fence).  One hop from the
// last arrival to the release: measured 1.6-3.1 us per barrier at 296 CTAs
// against 2.8-5.1 us for per-CTA arrival flags collected by CTA 0.  Waits
// are bounded: on timeout the error word is set and the CTA goes on (results
// are then invalid, and the host reports PF_ETIMEOUT).
__device__ __forceinline__ void grid_barrier(const EngineDev& e, unsigned* bar, unsigned& gen) {
  const unsigned target = gen + 1u;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(bar + kBarCount) : "memory");
    if (old == gridDim.x - 1u) {  // the last CTA to arrive releases the grid
      bar[kBarCount] = 0u;
      st_release(bar + 1, target);
    }
    const unsigned want = e.lookback_poison ? target + 1u : target;
    unsigned long long spins = 0;
    while (ld_relaxed(bar + 1) != want) {
      if (++spins > e.spin_limit) {
        atomicOr(e.err, ERR_BARRIER_TIMEOUT);
        break;
      }
      if (spins > 64) __nanosleep(32);
    }
    fence_acq_rel();
  }
  gen = target;
  __syncthreads();
}

// Named CTA barriers over all kThreads threads: arrive without waiting,
// or wait for the barrier to complete.
template <int ID>
__device__ __forceinline__ void named_arrive() {
  asm volatile("bar.arrive %0, %1;" ::"n"(ID), "n"(kThreads) : "memory");
}
template <int ID>
__device__ __forceinline__ void named_sync() {
  asm volatile("bar.sync %0, %1;" ::"n"(ID), "n"(kThreads) : "memory");
}

// Reads through L2 of control-block fields that another CTA wrote before a
// grid barrier (L1 is not coherent across SMs).
__device__ __forceinline__ int ld_cg_int(const int* p) { return __ldcg(p); }
__device__ __forceinline__ unsigned ld_cg_u(const unsigned* p) { return __ldcg(p); }
__device__ __forceinline__ float ld_cg_f(const float* p) { return __ldcg(p); }

// Chunk of worker w out of nw over the work items [t0, t0 + count).
__device__ __forceinline__ void chunk_of(int t0, int count, int w, int nw, int& b, int& e) {
  const int per = count / nw, rem = count % nw;
  b = t0 + w * per + min(w, rem);
  e = b + per + (w < rem ? 1 : 0);
}
__device__ __forceinline__ void cta_chunk(int t0, int count, int& b, int& e) {
  chunk_of(t0, count, (int)blockIdx.x, (int)gridDim.x, b, e);
}

// Block-wide sums of two 64-bit values (s_tmp: 2 * kWarps words).
__device__ __forceinline__ void block_sum2_u64(unsigned long long a, unsigned long long b,
                                               unsigned long long* s_tmp, unsigned long long& ra,
                                               unsigned long long& rb) {
  constexpr int kWarps = kThreads / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  a = warp_sum_u64(a);
  b = warp_sum_u64(b);
  __syncthreads();
  if (lane == 0) {
    s_tmp[warp] = a;
    s_tmp[kWarps + warp] = b;
  }
  __syncthreads();
  ra = 0ull;
  rb = 0ull;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) {
    ra += s_tmp[w];
    rb += s_tmp[kWarps + w];
  }
}


// The systematic resampler's phase 4 walks a chunk of tiles filter segment
// by filter segment (the tiles of one filter inside the chunk).  Every warp
// works on its own 128-particle segment without CTA barriers; only the
// per-filter maximum and prefix are CTA reductions.  The loops are kept
// compact (not unrolled over tiles): this code runs a few times per CTA and
// epoch, so instruction fetch, not arithmetic, sets its speed.  Integer sums
// are exact, so the result does not depend on the chunking.

// Phase 4's inputs of one tile for one lane: the tile's integer sum and
// maximum, its warp segment's scale and prefix, the lane's four in-segment
// prefixes (zero past the filter's end).
struct OffspringTileIn {
  double S, rho, E;
  double2 ca, cb;
  float m;
};
__device__ __forceinline__ OffspringTileIn load_offspring_tile(const EngineDev& e, int g, int tb, int n,
                                                               long long base, int warp, int lane) {
  OffspringTileIn o;
  o.S = __ldcg(e.tile_S + g);
  o.m = __ldcg(e.tile_m + g);
  o.rho = 0.0;
  o.E = 0.0;
  o.ca = make_double2(0.0, 0.0);
  o.cb = o.ca;
  const int pw = (g - tb) * kTile + warp * kWarpTile, p0 = pw + lane * 4;
  if (pw < n) {
    o.rho = __ldcg(e.seg_rho + (size_t)g * kSubTiles + warp);
    o.E = __ldcg(e.seg_E + (size_t)g * kSubTiles + warp);
    if (p0 < n) {
      const double2* src = reinterpret_cast<const double2*>(e.seg_c + base + p0);
      o.ca = __ldcg(src);
      o.cb = __ldcg(src + 1);
    }
  }
  return o;
}

// The run [lo, hi) of ancestor i, written by the whole warp (its values
// broadcast from one lane): the marker of every 128-slot segment that starts
// inside the run -- i when the run covers the segment, else -1 (only the
// last one can be partial) -- and the slots of the segments the run covers
// in part.  `seg` is the filter's marker array, n its slot count.
__device__ __forceinline__ void write_heavy_run(const EngineDev& e, int* anc, int* seg, uint32_t lo, uint32_t hi,
                                                int i, uint32_t n, int lane) {
  if (!PF_BOUNDS_OK(e, lo < hi && hi <= n)) return;
  const uint32_t s_first = (lo + kWarpTile - 1) / kWarpTile, s_last = (hi - 1) / kWarpTile;
  const bool last_full = s_first <= s_last && min((s_last + 1) * (uint32_t)kWarpTile, n) <= hi;
  for (uint32_t sg = s_first + lane; sg <= s_last; sg += 32) seg[sg] = (sg < s_last || last_full) ? i : -1;
  const uint32_t head_end = min(hi, s_first * (uint32_t)kWarpTile);
  for (uint32_t j = lo + lane; j < head_end; j += 32) anc[j] = i;
  if (s_first <= s_last && !last_full)
    for (uint32_t j = s_last * (uint32_t)kWarpTile + lane; j < hi; j += 32) anc[j] = i;
}

// Phase 4, right after the grid barrier and speculative (the filters'
// owners decide at the same time whether they resample; when one does not,
// this work is unused): for every filter that may resample this step (the
// flag phase 1 left in its control block), the filter maximum from the tile
// maxima, the filter prefix of each tile of the chunk from the tile sums
// scaled to that maximum, then per particle its filter-wide CDF C_i and
// offspring end F(i); slots [F(i-1), F(i)) get ancestor i.  A run of up to
// kLightRun slots is written by its lane (with the marker of a segment
// starting inside it); a longer one by the whole warp (write_heavy_run).
// The marker of each segment is written by the run holding the segment's
// first slot, so every resampling step rewrites all of them, and the step
// needs no second grid barrier: the next step's gather is the first reader.
__device__ __forceinline__ void epoch_sys_offspring(const EngineDev& e, int cb, int ce, unsigned long long* s_u64) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int t = cb; t < ce;) {
    const int f = __ldg(e.tile_filter + t);
    const FilterDesc* fd = e.desc + f;
    FilterCtrl* fc = e.ctrl + f;
    const int tb = fd->tile_begin, nt = fd->n_tiles, se = min(ce, tb + nt);
    if (ld_cg_int(&fc->sys_q_cur)) {  // CTA-uniform
      const int n = fd->n;
      const long long base = fd->p_off;
      // the first tile's inputs load while the filter prefix is formed; in
      // the loop below the next tile's load while this one is worked on
      // (every load is independent of the previous tile)
      OffspringTileIn nxt{};
      if (t < se) nxt = load_offspring_tile(e, t, tb, n, base, warp, lane);
      // the filter maximum M (the largest tile maximum), then the prefix of
      // tile t inside its filter and the filter total, from the tile sums
      // scaled to M; four tiles per thread and round, their loads issued
      // together, one round kept in registers for filters of up to
      // kB * kThreads tiles
      constexpr int kB = 4;
      double S[kB];
      float m[kB];
      auto load_round = [&](int i0) {
#pragma unroll
        for (int j = 0; j < kB; ++j) {
          const int i = i0 + j * kThreads;
          S[j] = i < nt ? __ldcg(e.tile_S + tb + i) : 0.0;
          m[j] = i < nt ? __ldcg(e.tile_m + tb + i) : -INFINITY;
        }
      };
      float mx = -INFINITY;
#pragma unroll 1
      for (int i0 = threadIdx.x; i0 < nt; i0 += kB * kThreads) {
        load_round(i0);
#pragma unroll
        for (int j = 0; j < kB; ++j) mx = fmaxf(mx, m[j]);
      }
      const float M = block_max(mx, reinterpret_cast<float*>(s_u64));
      if (M == -INFINITY) {  // CTA-uniform: no finite weight (the owner reports it)
        t = se;
        continue;
      }
      unsigned long long P = 0, W = 0;
      {
        unsigned long long pre = 0, all = 0;
#pragma unroll 1
        for (int i0 = threadIdx.x; i0 < nt; i0 += kB * kThreads) {
          if (nt > kB * kThreads) load_round(i0);  // else the registers hold the only round
#pragma unroll
          for (int j = 0; j < kB; ++j) {
            double r;
            const unsigned long long v = (unsigned long long)sys_tile_total(S[j], m[j], M, r);
            all += v;
            if (tb + i0 + j * kThreads < t) pre += v;
          }
        }
        block_sum2_u64(pre, all, s_u64, P, W);
      }
      if (threadIdx.x == 0) {
        if (se == tb + nt) fc->wq_total = W;  // the chunk holding the filter's last tile
        if (W == 0ull) atomicOr(e.err, ERR_BAD_WEIGHTS);
      }
      if (W > 0ull) {
        const uint32_t u = ld_cg_u(&fc->sys_u_cur);
        const double scale = (double)n / (double)W, uf = (double)u * 2.3283064365386963e-10;
        int* anc = e.anc + base;
        int* seg = e.seg_anc + (size_t)tb * kSubTiles;
#pragma unroll 1
        for (int g = t; g < se; ++g) {
          const int pw = (g - tb) * kTile + warp * kWarpTile;
          const int p0 = pw + lane * 4;
          const OffspringTileIn cur = nxt;
          if (g + 1 < se) nxt = load_offspring_tile(e, g + 1, tb, n, base, warp, lane);
          double r;
          const unsigned long long ts = (unsigned long long)sys_tile_total(cur.S, cur.m, M, r);
          if (pw < n) {  // warp-uniform
            const double rho = cur.rho, E = cur.E;
            // segment prefixes of this lane's particles and of the one before
            const double c[4] = {cur.ca.x, cur.ca.y, cur.cb.x, cur.cb.y};
            double cprev = __shfl_up_sync(0xffffffffu, c[3], 1);
            if (lane == 0) cprev = 0.0;
            const double Pd = (double)P;
            uint32_t Fprev = 0u, Fk[4] = {0u, 0u, 0u, 0u};
            if (p0 < n) {
              Fprev = (p0 == 0) ? 0u
                                : offspring_end_split(P, Pd, sys_inner(E, rho, r, cprev), W, (uint32_t)n, u, scale, uf);
#pragma unroll
              for (int k = 0; k < 4; ++k)
                Fk[k] = (p0 + k < n)
                            ? offspring_end_split(P, Pd, sys_inner(E, rho, r, c[k]), W, (uint32_t)n, u, scale, uf)
                            : (uint32_t)n;
            }
#pragma unroll 1
            for (int k = 0; k < 4; ++k) {
              const uint32_t lo = (k == 0) ? Fprev : Fk[k - 1], hi = Fk[k];
              const int i = p0 + k;
              const bool run = i < n && hi > lo;
              const bool heavy = run && hi - lo > (uint32_t)kLightRun;
              if (run && !heavy && PF_BOUNDS_OK(e, hi <= (uint32_t)n)) {
                for (uint32_t j = lo; j < hi; ++j) anc[j] = i;
                const uint32_t sg = (lo + kWarpTile - 1) / kWarpTile;  // a segment starting inside the run
                if (sg * (uint32_t)kWarpTile < hi)
                  seg[sg] = min((sg + 1) * (uint32_t)kWarpTile, (uint32_t)n) <= hi ? i : -1;
              }
              unsigned todo = __ballot_sync(0xffffffffu, heavy);
              while (todo) {  // warp-uniform
                const int src = __ffs(todo) - 1;
                todo &= todo - 1u;
                write_heavy_run(e, anc, seg, __shfl_sync(0xffffffffu, lo, src), __shfl_sync(0xffffffffu, hi, src),
                                pw + src * 4 + k, (uint32_t)n, lane);
              }
            }
          }
          P += ts;
        }
      }
    }
    t = se;
  }
}

#ifndef PF_EPOCH_MINB
#define PF_EPOCH_MINB 2  // resident CTAs per SM the epoch kernel is compiled for
#endif
template <int NCLK, int WMODE, int RESAMPLER>
__global__ void __launch_bounds__(kThreads, PF_EPOCH_MINB) k_epoch(EngineDev e, int t0, int count, unsigned* bar) {
  constexpr int D = 3 + NCLK;
  constexpr int NV = 2 + D + 6;
  constexpr int kWarps = kThreads / 32;
  constexpr int kStride = (WMODE == PF_WEIGHT_MIXTURE || WMODE == PF_WEIGHT_GENERIC) ? kMixStride : kSatStride;
  __shared__ __align__(16) float2 s_sat[kStride * PF_MAX_SATS];
  __shared__ int s_grp[PF_MAX_CLK + 1];
  __shared__ unsigned char s_clk[PF_MAX_SATS];
  __shared__ float s_wrow[2][kWarps][17];
  __shared__ float s_maxtmp[kWarps];
  __shared__ double s_dred[kWarps * 16];
  __shared__ unsigned long long s_u64[2 * kWarps];
  __shared__ double s_wq[2][kWarps];  // per-warp sums of the tiled integer CDF
  __shared__ int s_dec_f, s_dec_rs;  // the filter this CTA owns in phase 2 and its decision

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // generation of the last barrier (every thread reads it before its CTA
  // first arrives, so no CTA can have moved it on yet).  A relaxed load: the
  // kernel boundary already orders the previous launch's release, and an
  // acquire here would hold every later load of the CTA behind it.
  unsigned gen = ld_relaxed(bar + 1);
  if (threadIdx.x == 0) s_dec_f = -1;
  int cb, ce;
  cta_chunk(t0, count, cb, ce);

  // ---------------------------------------------------------------- phase 1
  int cached = -1;
  int it = 0;
  for (int t = cb; t < ce; ++t, ++it) {

    const int f = __ldg(e.tile_filter + t);
    const FilterDesc* fd = e.desc + f;
    FilterCtrl* fc = e.ctrl + f;
    const unsigned epoch = fc->epoch;
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
    // the filter may resample this epoch: systematic builds its tiled integer CDF
    const bool may_rs = (do_weight || (eflags & PF_EP_RESAMPLE_CHECK)) && !(eflags & PF_EP_NO_RESAMPLE);
    const bool sys_q = RESAMPLER == PF_RESAMPLE_SYSTEMATIC && may_rs;
    if (t == fd->tile_begin && threadIdx.x == 0) {  // read after the barrier (phase 4, Megopolis)
      fc->sys_q_cur = sys_q ? 1 : 0;
      fc->eflags_cur = eflags;
      fc->epoch_cur = epoch;
      if (sys_q) fc->sys_u_cur = sys_offset_u(e, fd, epoch);
    }

    // the particles' loads are issued first: their memory latency overlaps the
    // satellite table of a new filter (FP64 geometry, two CTA barriers)
    const int n = fd->n;
    const int p0 = (t - fd->tile_begin) * kTile + (int)threadIdx.x * 4;
    const bool active = p0 < n;
    const long long base = fd->p_off;
    float* dst = fc->parity ? e.state0 : e.state1;
    float x[D][4];
    float lwv[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
    if (active) {
      load_particles<D>(e, fd, fc->parity ? e.state1 : e.state0, base, p0, n, fc->resample_flag != 0, x);
    } else {
#pragma unroll
      for (int d = 0; d < D; ++d)
#pragma unroll
        for (int k = 0; k < 4; ++k) x[d][k] = 0.f;
    }
    if constexpr (WMODE == PF_WEIGHT_MIXTURE) {
      if (f != cached) {
        __shared__ MixSmem s_mix;
        build_mixture_table<NCLK>(e, fd, fc, fe, sats, n_sat, do_weight, t == fd->tile_begin, f, s_sat, s_grp, s_clk,
                                  s_mix);
        cached = f;
      }
    }
    if (WMODE != PF_WEIGHT_MIXTURE && f != cached) {  // satellite geometry of this filter (FP64 -> FP32 pairs)
      __syncthreads();   // nobody still reads the previous filter's table
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
        if constexpr (WMODE == PF_WEIGHT_GENERIC)
          write_generic_entry(s_sat + kMixStride * rank, e, fd->sigma_pr, eE, eN, eU, g, y, (float)sp->w);
        else
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

    if (active) {
      float lw0[4] = {0.f, 0.f, 0.f, 0.f};
      const bool need_prev = !lw_zero && (!do_weight || e.lw_mode == PF_LW_ACCUMULATE);
      if (need_prev) {
        const float4 v = __ldcs(reinterpret_cast<const float4*>(e.lw + base + p0));
        lw0[0] = v.x; lw0[1] = v.y; lw0[2] = v.z; lw0[3] = v.w;
      }
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
          const U4 r = philox10(U4{(uint32_t)(p0 + k), epoch, TAG_PREDICT, fid}, k0, k1);
          const float2 a = box_muller_f32(r.x, r.y), b = box_muller_f32(r.z, r.w);
          nz[0] = a.x; nz[1] = a.y; nz[2] = b.x; nz[3] = b.y;
          if (D > 4) {
            const U4 r2 = philox10(U4{(uint32_t)(p0 + k), epoch, TAG_PREDICT | 1u, fid}, k0, k1);
            const float2 c = box_muller_f32(r2.x, r2.y), dd = box_muller_f32(r2.z, r2.w);
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
        if constexpr (WMODE == PF_WEIGHT_GENERIC) {
          bool gated[4] = {false, false, false, false};
          const float gate = e.lk_gate_m;
          if (gate > 0.f) {  // per-particle NLOS gate: drop |r| > gate unless too few satellites remain
            int kept[4] = {0, 0, 0, 0}, used = 0;
#pragma unroll
            for (int c = 0; c < NCLK; ++c) {
              const float2 ncb[2] = {f2(-x[3 + c][0], -x[3 + c][1]), f2(-x[3 + c][2], -x[3 + c][3])};
              generic_kept(s_sat, s_grp[c], s_grp[c + 1], dx, dy, dz, nbb, ncb, kept, used, gate);
            }
            const int need = used < 4 ? used : 4;
#pragma unroll
            for (int k = 0; k < 4; ++k) gated[k] = kept[k] >= need;
          }
#pragma unroll
          for (int c = 0; c < NCLK; ++c) {
            const float2 ncb[2] = {f2(-x[3 + c][0], -x[3 + c][1]), f2(-x[3 + c][2], -x[3 + c][3])};
            generic_pairs(s_sat, s_grp[c], s_grp[c + 1], dx, dy, dz, nbb, ncb, lwp, gated, gate);
          }
        }
#pragma unroll
        for (int c = 0; c < NCLK && WMODE != PF_WEIGHT_GENERIC; ++c) {
          const float2 ncb[2] = {f2(-x[3 + c][0], -x[3 + c][1]), f2(-x[3 + c][2], -x[3 + c][3])};
          const int s_end = s_grp[c + 1];
#pragma unroll 2
          for (int s = s_grp[c]; s < s_end; ++s) {
#pragma unroll
            for (int p = 0; p < 2; ++p) {
              if constexpr (WMODE == PF_WEIGHT_MIXTURE)
                sat_pair_mixture(s_sat + kMixStride * s, dx[p], dy[p], dz[p], nbb[p], ncb[p], lwp[p], fd);
              else
                sat_pair_update<WMODE>(s_sat + kSatStride * s, dx[p], dy[p], dz[p], nbb[p], ncb[p], lwp[p], fd);
            }
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

    // per-warp statistics, then warp 0 merges the warp rows into the tile row
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
      const int idx = warp_transpose_sum16(v);
      // Warp rows go to buffer it & 1; warp 0 merges them while the other
      // warps move on (named barriers: FULL[b] = 1 + b, EMPTY[b] = 3 + b).
      const int b = it & 1;
      float (*wr)[17] = s_wrow[b];
      if (warp != 0 && it >= 2) {  // warp 0 has merged tile it - 2 from this buffer
        if (b) named_sync<4>();
        else named_sync<3>();
      }
      // tiled integer CDF of the systematic resampler, segment level
      const double seg_sum = sys_q ? sys_segment_prefix(e, base, p0, active, lwv, wm, fd->K) : 0.0;
      if ((lane & 1) == 0 && idx < NV) wr[warp][1 + idx] = v[0];
      if (lane == 0) {
        wr[warp][0] = wm;
        s_wq[b][warp] = seg_sum;
      }
      if (warp != 0) {
        if (b) named_arrive<2>();
        else named_arrive<1>();
      } else {
        if (b) named_sync<2>();
        else named_sync<1>();
      }
      if (warp == 0) {
        float tm = lane < kWarps ? wr[lane][0] : -INFINITY;
        tm = warp_max(tm);
        float acc = 0.f;
        if (lane < NV && tm > -INFINITY) {
#pragma unroll
          for (int w = 0; w < kWarps; ++w) {
            const float mw = wr[w][0];
            if (mw > -INFINITY) {
              float sc = exp2f((mw - tm) * 1.4426950408889634f);
              if (lane == 1) sc *= sc;
              acc = fmaf(sc, wr[w][1 + lane], acc);
            }
          }
        }
        float* row = e.part + (size_t)t * kPartStride;
        if (lane < NV) row[1 + lane] = acc;
        if (lane == 0) {
          row[0] = tm;
          // filter maximum for the one-pass merge and the integer CDF, kept
          // only when the filter may resample this epoch
        }
        // tile level of the tiled integer CDF
        if (sys_q) sys_tile_scale(e, t, lane < kWarps ? s_wq[b][lane] : 0.0, lane < kWarps ? wr[lane][0] : -INFINITY, tm);
        if (it + 2 < ce - cb) {  // buffer b is free again
          if (b) named_arrive<4>();
          else named_arrive<3>();
        }
      }
    }
  }
  grid_barrier(e, bar, gen);

  // ---------------------------------------------------------------- phase 2
  // Filter f_first + j is merged and decided by CTA j mod G.  With fewer
  // filters than CTAs the other CTAs start phase 4 (systematic) meanwhile.
  const int f_first = __ldg(e.tile_filter + t0), nf = __ldg(e.tile_filter + t0 + count - 1) - f_first + 1;
  for (int j = blockIdx.x; j < nf; j += gridDim.x) {
    const int f = f_first + j;
    const FilterDesc* fd = e.desc + f;
    FilterCtrl* fc = e.ctrl + f;
    const unsigned epoch = fc->epoch;
    const unsigned char* ob = e.obs + (size_t)(epoch % (unsigned)e.obs_slots) * e.obs_slot_bytes;
    const pf_filter_epoch_t* fe = reinterpret_cast<const pf_filter_epoch_t*>(ob) + f;
    const int eflags = fe->flags;
    MergedStats ms = merge_tiles<D>(e.part, fd->tile_begin, fd->n_tiles, s_maxtmp, s_dred);
    if (threadIdx.x == 0) {
      finalize_filter<D>(e, fd, fc, ms, epoch, fc->parity, fc->lw_zero != 0, eflags, (eflags & PF_EP_WEIGHT) != 0);
      s_dec_f = f;
      s_dec_rs = fc->resample_flag;
    }
    __syncthreads();
  }
  if constexpr (RESAMPLER == PF_RESAMPLE_SYSTEMATIC) {
    // Phase 4 needs only the first barrier: the tiled integer CDF is
    // complete once every tile is (speculative, as the owners decide at the
    // same time).  With few filters their owners sit it out (it overlaps
    // their merges); with many, every CTA takes a share after its merges.
    const int h0 = 4 * nf <= (int)gridDim.x ? nf : 0;  // first CTA of phase 4
    if ((int)blockIdx.x >= h0) {
      int b4, e4;
      chunk_of(t0, count, (int)blockIdx.x - h0, (int)gridDim.x - h0, b4, e4);
      epoch_sys_offspring(e, b4, e4, s_u64);
    }
    // no second barrier: the ancestors and segment markers are read first by
    // the next step, after this kernel has ended
  } else {
    // Megopolis: no second barrier either.  A CTA decides for the filter of
    // its tiles itself, with the owner's merge (the same function on the
    // same rows gives the same bits, hence the same decision) or, for the
    // filter it owns, with the owner's decision; epoch and flags come from
    // the snapshot phase 1 left (the owner advances the epoch meanwhile).
    int cf = -1;
    bool crs = false;
    for (int t = cb; t < ce; ++t) {
      const int f = __ldg(e.tile_filter + t);
      const FilterDesc* fd = e.desc + f;
      const FilterCtrl* fc = e.ctrl + f;
      if (f != cf) {  // CTA-uniform
        cf = f;
        if (f == s_dec_f) {
          crs = s_dec_rs != 0;
        } else {
          const MergedStats ms = merge_tiles<D>(e.part, fd->tile_begin, fd->n_tiles, s_maxtmp, s_dred);
          if (threadIdx.x == 0) s_dec_rs = resample_decision(e, fd, ms, ld_cg_int(&fc->eflags_cur)) ? 1 : 0;
          __syncthreads();
          crs = s_dec_rs != 0;
          __syncthreads();  // s_dec_rs is rewritten for the next filter
        }
      }
      if (crs) mego_tile(e, fd, ld_cg_u(&fc->epoch_cur), t);
    }
  }
}

}  // namespace pfb
