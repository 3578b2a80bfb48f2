// pf_engine.cu -- host side of the resident engine (the pfe_* C ABI).
#include <cuda_runtime.h>
#include <stddef.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "pf_epoch_kernel.cuh"
#include "pf_obs_terms.cuh"
#include "pf_velocity.cuh"
#include "pf_weight3d.cuh"
#include "pf_status.h"

using namespace pfb;

struct pf_engine {
  pf_engine_config_t cfg;
  std::vector<pf_filter_params_t> params;
  std::vector<FilterDesc> hdesc;
  std::vector<int> tile_filter;
  int D = 0;
  int T = 0;
  long long P = 0;
  int max_n = 0;
  EngineDev dev;
  unsigned char* ws = nullptr;
  size_t ws_bytes = 0;
  double* export_buf = nullptr;
  FilterCtrl* ctrl_dev = nullptr;
  FilterDesc* desc_dev = nullptr;
  cudaStream_t stream = nullptr;
  unsigned char* pinned[2] = {nullptr, nullptr};
  cudaEvent_t pin_ev[2] = {nullptr, nullptr};
  int pin_cur = 0;
  FilterCtrl* ctrl_host = nullptr;  // pinned mirror of the control blocks, then the error word
  unsigned* err_host = nullptr;     // pinned copy of the device error word (inside ctrl_host's block)
  size_t ctrl_span = 0;             // bytes from the first control block to the end of the error word
  // pfe_step_io: per pinned staging buffer a graph of upload copy, epoch
  // kernel and result copy, re-captured when the launch parameters change
  cudaGraph_t io_graph[2] = {nullptr, nullptr};
  cudaGraphExec_t io_exec[2] = {nullptr, nullptr};
  cudaGraphNode_t io_h2d[2] = {nullptr, nullptr};
  size_t io_h2d_bytes[2] = {0, 0};
  std::vector<unsigned char> io_key[2];
  size_t obs_slot_bytes = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  int resident[Q_COUNT];
  int epoch_resident = 0;     // co-resident CTAs of the cooperative epoch kernel
  bool mlp_set = false;       // mixture mode: network parameters uploaded
  int epoch_cap = 0;          // > 0: at most this many CTAs per launch of the epoch kernel (tuning)
  size_t epoch_smem = 0;      // its dynamic shared memory
  unsigned* bar = nullptr;    // grid barrier words (count, generation, any-resample)
  ObsRow* obs_rows = nullptr; // rows of pfe_add_obs_term
  int sm_count = 0;
  int last_launches = 0;
  std::vector<int> initialized;
  // timing ring (pfe_enable_timing)
  std::vector<cudaEvent_t> tev;  // kTimingEvents per slot
  std::vector<float> t_kernel_ms; // per-kernel durations of the last read
  int t_slots = 0;
  int t_detailed = 0;  // events after every resampling kernel too
  int t_next = 0;
  int t_pending = 0;
};

namespace {

// events per timed step: before k_step, after k_step, after each of the
// three resampling kernels
constexpr int kTimingEvents = 5;

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

struct Layout {
  size_t off_state0, off_state1, off_lw, off_anc, off_offs, off_mp, off_part, off_agg, off_inc,
      off_flag, off_excl, off_wq, off_seg_rho, off_seg_E, off_tile_S, off_tile_m, off_seg_anc, off_mlp, off_satdbg, off_obsrows, off_desc, off_ctrl, off_tf, off_queue, off_err, off_obs, off_export,
      total;
  size_t obs_slot_bytes;
  long long P;
  int T, D, max_n;
};

int validate_config(const pf_engine_config_t* cfg, const pf_filter_params_t* fp) {
  if (!cfg || !fp) return set_err(PF_EINVAL, "null config");
  if (cfg->n_filters <= 0) return set_err(PF_EINVAL, "n_filters must be > 0");
  if (cfg->n_clk < 1 || cfg->n_clk > PF_MAX_CLK) return set_err(PF_EINVAL, "n_clk must be 1..%d", PF_MAX_CLK);
  if (cfg->resampler != PF_RESAMPLE_SYSTEMATIC && cfg->resampler != PF_RESAMPLE_MEGOPOLIS)
    return set_err(PF_EINVAL, "unknown resampler %d", cfg->resampler);
  if (cfg->resampler == PF_RESAMPLE_MEGOPOLIS && (cfg->megopolis_iters < 1 || cfg->megopolis_iters > 128))
    return set_err(PF_EINVAL, "megopolis_iters must be 1..128");
  if (cfg->weight_mode < PF_WEIGHT_GAUSSIAN || cfg->weight_mode > PF_WEIGHT_GENERIC)
    return set_err(PF_EINVAL, "unknown weight_mode %d", cfg->weight_mode);
  if ((cfg->weight_mode == PF_WEIGHT_MIXTURE || cfg->weight_mode == PF_WEIGHT_GENERIC) &&
      (cfg->flags & PF_FLAG_KERNEL_CHAIN))
    return set_err(PF_EINVAL, "this likelihood runs in the epoch kernel only (no PF_FLAG_KERNEL_CHAIN)");
  if (cfg->lw_mode != PF_LW_OVERWRITE && cfg->lw_mode != PF_LW_ACCUMULATE)
    return set_err(PF_EINVAL, "unknown lw_mode %d", cfg->lw_mode);
  if (cfg->sys_offset != PF_SYS_OFFSET_RANDOM && cfg->sys_offset != PF_SYS_OFFSET_REFERENCE)
    return set_err(PF_EINVAL, "unknown sys_offset %d", cfg->sys_offset);
  if (cfg->max_sats < 1 || cfg->max_sats > PF_MAX_SATS)
    return set_err(PF_ECAP, "max_sats must be 1..%d", PF_MAX_SATS);
  if (cfg->obs_slots < 1) return set_err(PF_EINVAL, "obs_slots must be >= 1");
  if (!(cfg->ess_threshold >= 0.0) || !isfinite(cfg->ess_threshold))
    return set_err(PF_EINVAL, "ess_threshold must be finite and >= 0");
  if ((cfg->weight_mode == PF_WEIGHT_HUBER || cfg->weight_mode == PF_WEIGHT_MIXTURE) && !(cfg->huber_k > 0.0))
    return set_err(PF_EINVAL, "huber_k must be > 0");
  for (int f = 0; f < cfg->n_filters; ++f) {
    const pf_filter_params_t& p = fp[f];
    if (p.n_particles <= 0 || p.n_particles > (1 << 30))
      return set_err(PF_EINVAL, "filter %d: n_particles must be 1..2^30", f);
    for (int a = 0; a < 3; ++a)
      if (!(p.sigma_pos[a] >= 0.0) || !isfinite(p.sigma_pos[a]))
        return set_err(PF_EINVAL, "filter %d: sigma_pos must be finite and >= 0", f);
    if (!(p.sigma_clk >= 0.0) || !isfinite(p.sigma_clk))
      return set_err(PF_EINVAL, "filter %d: sigma_clk must be finite and >= 0", f);
    if (!(p.sigma_pr > 0.0) || !isfinite(p.sigma_pr))
      return set_err(PF_EINVAL, "filter %d: sigma_pr must be finite and > 0", f);
  }
  return PF_OK;
}

Layout make_layout(const pf_engine_config_t* cfg, const pf_filter_params_t* fp) {
  Layout L{};
  L.D = 3 + cfg->n_clk;
  long long P = 0;
  int T = 0, max_n = 0;
  for (int f = 0; f < cfg->n_filters; ++f) {
    int n = fp[f].n_particles;
    P += (long long)align_up((size_t)n, 4);
    T += (n + PF_TILE - 1) / PF_TILE;
    max_n = std::max(max_n, n);
  }
  P = (long long)align_up((size_t)P, 64);
  L.P = P;
  L.T = T;
  L.max_n = max_n;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    size_t at = o;
    o = align_up(o + bytes, 256);
    return at;
  };
  L.off_state0 = take((size_t)L.D * P * 4);
  L.off_state1 = take((size_t)L.D * P * 4);
  L.off_lw = take((size_t)P * 4);
  L.off_anc = take((size_t)P * 4);
  L.off_offs = take((size_t)P * 4);
  L.off_mp = take((size_t)T * 4);
  L.off_part = take((size_t)T * kPartStride * 4);
  L.off_agg = take((size_t)T * 8);
  L.off_inc = take((size_t)T * 8);
  L.off_flag = take((size_t)T * 4);
  L.off_excl = take((size_t)T * 8);
  L.off_wq = take((size_t)P * 8);
  L.off_seg_rho = take((size_t)T * kSubTiles * 8);
  L.off_seg_E = take((size_t)T * kSubTiles * 8);
  L.off_tile_S = take((size_t)T * 8);
  L.off_tile_m = take((size_t)T * 4);
  L.off_seg_anc = take((size_t)T * kSubTiles * 4);
  const bool mix = cfg->weight_mode == PF_WEIGHT_MIXTURE;
  L.off_mlp = take(mix ? (size_t)kMlpParams * 4 : 0);
  L.off_satdbg = take(mix ? (size_t)cfg->n_filters * cfg->max_sats * kSatDbg * 4 : 0);
  L.off_obsrows = take(sizeof(ObsRow) * kMaxObsRows);
  L.off_desc = take(sizeof(FilterDesc) * cfg->n_filters);
  // the error word follows the control blocks, so one copy returns both
  L.off_ctrl = take(sizeof(FilterCtrl) * cfg->n_filters);
  L.off_err = take(sizeof(unsigned) * 4);
  L.off_tf = take((size_t)T * 4);
  L.off_queue = take(sizeof(unsigned) * (2 * Q_COUNT + kBarWords));
  L.obs_slot_bytes = align_up(sizeof(pf_filter_epoch_t) * cfg->n_filters +
                                  sizeof(pf_sat_t) * (size_t)cfg->n_filters * cfg->max_sats,
                              256);
  L.off_obs = take(L.obs_slot_bytes * cfg->obs_slots);
  L.off_export = take((size_t)max_n * L.D * 8);
  L.total = o;
  return L;
}

// ECEF -> local E/N/U rotation at an ECEF point (geodetic latitude from the
// WGS-84 ellipsoid by Bowring's iteration).
void enu_rotation(const double* p, double* rot) {
  const double a = 6378137.0, f = 1.0 / 298.257223563;
  const double e2 = f * (2.0 - f);
  const double x = p[0], y = p[1], z = p[2];
  const double lon = atan2(y, x);
  const double rho = sqrt(x * x + y * y);
  double lat = atan2(z, rho * (1.0 - e2));
  for (int it = 0; it < 8; ++it) {
    const double s = sin(lat);
    const double Nr = a / sqrt(1.0 - e2 * s * s);
    const double h = (fabs(cos(lat)) > 1e-12) ? rho / cos(lat) - Nr : fabs(z) - Nr * (1.0 - e2);
    lat = atan2(z, rho * (1.0 - e2 * Nr / (Nr + h)));
  }
  if (rho < 1e-6) lat = z >= 0 ? M_PI / 2 : -M_PI / 2;
  const double sl = sin(lat), cl = cos(lat), so = sin(lon), co = cos(lon);
  rot[0] = -so;      rot[1] = co;       rot[2] = 0.0;
  rot[3] = -sl * co; rot[4] = -sl * so; rot[5] = cl;
  rot[6] = cl * co;  rot[7] = cl * so;  rot[8] = sl;
}

uint32_t reference_sys_offset(unsigned long long seed, int n) {
  // resampling.cu:152 sets u0 = (seed % 1e6) / (1e6 * N) and searches for the
  // target (u0 + k) / N (resampling.cu:69).  In units of one slot the target
  // of slot k is k + u0, so the slot fraction is u0 itself, kept here as a
  // 32-bit fixed-point fraction.
  double u0 = (double)(seed % 1000000ull) / (1000000.0 * (double)n);
  double v = floor(u0 * 4294967296.0);
  if (v < 0) v = 0;
  if (v > 4294967295.0) v = 4294967295.0;
  return (uint32_t)v;
}

void fill_desc(pf_engine* eng, int f) {
  const pf_filter_params_t& p = eng->params[f];
  FilterDesc& d = eng->hdesc[f];
  for (int i = 0; i < 8; ++i) d.sigma[i] = 0.f;
  d.sigma[0] = (float)p.sigma_pos[0];
  d.sigma[1] = (float)p.sigma_pos[1];
  d.sigma[2] = (float)p.sigma_pos[2];
  for (int c = 0; c < eng->cfg.n_clk; ++c) d.sigma[3 + c] = (float)p.sigma_clk;
  d.sigma_pr = (float)p.sigma_pr;
  d.inv_sigma_pr = (float)(1.0 / p.sigma_pr);
  d.wscale = (float)(-0.5 / (p.sigma_pr * p.sigma_pr));
  d.huber_k = (float)eng->cfg.huber_k;
  d.key0 = (uint32_t)(p.seed & 0xffffffffull);
  d.key1 = (uint32_t)(p.seed >> 32);
  d.sys_ref_u = reference_sys_offset(p.seed, p.n_particles);
}

int check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) return set_err(PF_ECUDA, "%s: %s", what, cudaGetErrorString(e));
  return PF_OK;
}

#define CK(call)                                   \
  do {                                             \
    int _s = check_cuda((call), #call);            \
    if (_s != PF_OK) return _s;                    \
  } while (0)

template <typename K>
int occupancy(K kernel, int sm_count, int* out) {
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0);
  if (e != cudaSuccess) return set_err(PF_ECUDA, "occupancy: %s", cudaGetErrorString(e));
  *out = std::max(1, per_sm) * sm_count;
  return PF_OK;
}

inline int grid_for(const pf_engine* eng, int slot, int count) {
  return std::max(1, std::min(count, eng->resident[slot]));
}

// Kernel launch with programmatic dependent launch: the kernel may start
// while the previous kernel of the stream drains; it waits
// (griddepcontrol.wait) before reading that kernel's results.  PF_B200_NO_PDL=1
// in the environment turns it off (plain stream order).
bool pdl_enabled() {
  static const bool on = [] {
    const char* v = getenv("PF_B200_NO_PDL");
    return !(v && v[0] == '1');
  }();
  return on;
}

template <typename... KArgs, typename... Args>
int launch_k(void (*kernel)(KArgs...), int grid, cudaStream_t st, const char* what, Args... args) {
  cudaLaunchConfig_t lc;
  memset(&lc, 0, sizeof(lc));
  lc.gridDim = dim3((unsigned)grid);
  lc.blockDim = dim3(kThreads);
  lc.dynamicSmemBytes = 0;
  lc.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = attr;
  lc.numAttrs = pdl_enabled() ? 1 : 0;
  cudaError_t e = cudaLaunchKernelEx(&lc, kernel, args...);
  if (e != cudaSuccess) return set_err(PF_ECUDA, "%s launch: %s", what, cudaGetErrorString(e));
  return PF_OK;
}

template <int NCLK>
int launch_step_t(pf_engine* eng, int t0, int count) {
  const int g = grid_for(eng, Q_STEP, count);
  if (eng->cfg.weight_mode == PF_WEIGHT_GAUSSIAN)
    return launch_k(k_step<NCLK, PF_WEIGHT_GAUSSIAN>, g, eng->stream, "k_step", eng->dev, t0, count);
  return launch_k(k_step<NCLK, PF_WEIGHT_HUBER>, g, eng->stream, "k_step", eng->dev, t0, count);
}

int launch_step(pf_engine* eng, int t0, int count) {
  switch (eng->cfg.n_clk) {
    case 1: return launch_step_t<1>(eng, t0, count);
    case 2: return launch_step_t<2>(eng, t0, count);
    case 3: return launch_step_t<3>(eng, t0, count);
    default: return launch_step_t<4>(eng, t0, count);
  }
}

// ev (optional): events recorded after each resampling kernel (3 entries).
int launch_resample(pf_engine* eng, int t0, int count, int* n_launch, cudaEvent_t* ev = nullptr) {
  int s;
  if (eng->cfg.resampler == PF_RESAMPLE_SYSTEMATIC) {
    if ((s = launch_k(k_scan, grid_for(eng, Q_SCAN, count), eng->stream, "k_scan", eng->dev, t0, count)) != PF_OK)
      return s;
    if (ev) cudaEventRecord(ev[0], eng->stream);
    if ((s = launch_k(k_offs, grid_for(eng, Q_OFFS, count), eng->stream, "k_offs", eng->dev, t0, count)) != PF_OK)
      return s;
    if (ev) cudaEventRecord(ev[1], eng->stream);
    if ((s = launch_k(k_merge, grid_for(eng, Q_MERGE, count), eng->stream, "k_merge", eng->dev, t0, count)) != PF_OK)
      return s;
    if (ev) cudaEventRecord(ev[2], eng->stream);
    *n_launch += 3;
  } else {
    if ((s = launch_k(k_mego, grid_for(eng, Q_MEGO, count), eng->stream, "k_mego", eng->dev, t0, count)) != PF_OK)
      return s;
    if (ev) {
      cudaEventRecord(ev[0], eng->stream);
      cudaEventRecord(ev[1], eng->stream);
      cudaEventRecord(ev[2], eng->stream);
    }
    *n_launch += 1;
  }
  return check_cuda(cudaGetLastError(), "resample launch");
}

// ---- cooperative epoch kernel: instantiation table, occupancy, launch
typedef void (*EpochKernel)(EngineDev, int, int, unsigned*);

template <int NCLK, int WMODE>
EpochKernel epoch_kernel_r(int resampler) {
  return resampler == PF_RESAMPLE_SYSTEMATIC ? (EpochKernel)k_epoch<NCLK, WMODE, PF_RESAMPLE_SYSTEMATIC>
                                             : (EpochKernel)k_epoch<NCLK, WMODE, PF_RESAMPLE_MEGOPOLIS>;
}
template <int NCLK>
EpochKernel epoch_kernel_w(int wmode, int resampler) {
  if (wmode == PF_WEIGHT_GAUSSIAN) return epoch_kernel_r<NCLK, PF_WEIGHT_GAUSSIAN>(resampler);
  if (wmode == PF_WEIGHT_HUBER) return epoch_kernel_r<NCLK, PF_WEIGHT_HUBER>(resampler);
  if (wmode == PF_WEIGHT_MIXTURE) return epoch_kernel_r<NCLK, PF_WEIGHT_MIXTURE>(resampler);
  return epoch_kernel_r<NCLK, PF_WEIGHT_GENERIC>(resampler);
}
EpochKernel epoch_kernel(const pf_engine* eng) {
  const int w = eng->cfg.weight_mode, r = eng->cfg.resampler;
  switch (eng->cfg.n_clk) {
    case 1: return epoch_kernel_w<1>(w, r);
    case 2: return epoch_kernel_w<2>(w, r);
    case 3: return epoch_kernel_w<3>(w, r);
    default: return epoch_kernel_w<4>(w, r);
  }
}

int prepare_epoch_kernel(pf_engine* eng) {
  EpochKernel k = epoch_kernel(eng);
  eng->epoch_smem = 0;  // no dynamic shared memory
  CK(cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)eng->epoch_smem));
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, eng->epoch_smem));
  if (per_sm < 1) return set_err(PF_ECUDA, "epoch kernel does not fit on an SM");
  eng->epoch_resident = per_sm * eng->sm_count;
  return PF_OK;
}

// One cooperative launch over work items [t0, t0 + count): every CTA is
// resident at once, which the grid barriers require (the driver refuses the
// launch otherwise).
int launch_epoch(pf_engine* eng, int t0, int count) {
  int cap = std::min(eng->epoch_resident, kMaxEpochGrid);
  if (eng->epoch_cap > 0) cap = std::min(cap, eng->epoch_cap);
  const int grid = std::max(1, std::min(count, cap));
  cudaLaunchConfig_t lc;
  memset(&lc, 0, sizeof(lc));
  lc.gridDim = dim3((unsigned)grid);
  lc.blockDim = dim3(kThreads);
  lc.dynamicSmemBytes = eng->epoch_smem;
  lc.stream = eng->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  lc.attrs = attr;
  lc.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&lc, epoch_kernel(eng), eng->dev, t0, count, eng->bar);
  if (e != cudaSuccess) return set_err(PF_ECUDA, "k_epoch cooperative launch: %s", cudaGetErrorString(e));
  return PF_OK;
}

bool use_chain(const pf_engine* eng) { return (eng->cfg.flags & PF_FLAG_KERNEL_CHAIN) != 0; }

int err_status(unsigned w) {
  if (w & ERR_LOOKBACK_TIMEOUT) return set_err(PF_ETIMEOUT, "device look-back spin limit reached (error word 0x%x)", w);
  if (w & ERR_BARRIER_TIMEOUT) return set_err(PF_ETIMEOUT, "device grid-barrier spin limit reached (error word 0x%x)", w);
  if (w & ERR_SAT_CAP) return set_err(PF_ECAP, "n_sat above max_sats (error word 0x%x)", w);
  if (w & ERR_BAD_WEIGHTS) return set_err(PF_EINVAL, "all log-weights non-finite (error word 0x%x)", w);
  if (w & ERR_INTERNAL_CAP) return set_err(PF_ECUDA, "internal capacity exceeded (error word 0x%x)", w);
  if (w & ERR_BOUNDS) return set_err(PF_ECUDA, "index out of bounds caught by the checked build (error word 0x%x)", w);
  return PF_OK;
}

int sync_and_check(pf_engine* eng) {
  // the error word rides on the same stream as the caller's reads: one sync
  CK(cudaMemcpyAsync(eng->err_host, eng->dev.err, sizeof(unsigned), cudaMemcpyDeviceToHost, eng->stream));
  CK(cudaStreamSynchronize(eng->stream));
  return err_status(*eng->err_host);
}

int read_ctrl(pf_engine* eng) {
  // control blocks and the error word that follows them, in one copy
  CK(cudaMemcpyAsync(eng->ctrl_host, eng->ctrl_dev, eng->ctrl_span, cudaMemcpyDeviceToHost, eng->stream));
  CK(cudaStreamSynchronize(eng->stream));
  return err_status(*eng->err_host);
}

int check_filter(pf_engine* eng, int f) {
  if (!eng) return set_err(PF_EINVAL, "null engine");
  if (f < 0 || f >= eng->cfg.n_filters) return set_err(PF_EINVAL, "filter index %d out of range", f);
  return PF_OK;
}

int filter_dims(pf_engine* eng, int f, int* n, long long* base, int* tb, int* nt) {
  const FilterDesc& d = eng->hdesc[f];
  *n = d.n;
  *base = d.p_off;
  *tb = d.tile_begin;
  *nt = d.n_tiles;
  return PF_OK;
}

// The ancestors of filter f's last resample, one per slot, on the host:
// the slot array with every 128-slot segment that carries a marker
// (systematic resampling in the epoch kernel) filled from it.
int read_ancestors(pf_engine* eng, int f, int* out) {
  int n, tb, nt;
  long long base;
  filter_dims(eng, f, &n, &base, &tb, &nt);
  CK(cudaMemcpy(out, eng->dev.anc + base, sizeof(int) * n, cudaMemcpyDeviceToHost));
  if (eng->dev.anc_seg) {
    std::vector<int> mk((size_t)nt * kSubTiles);
    CK(cudaMemcpy(mk.data(), eng->dev.seg_anc + (size_t)tb * kSubTiles, sizeof(int) * mk.size(),
                  cudaMemcpyDeviceToHost));
    for (int k = 0; k < n; ++k)
      if (mk[k / kWarpTile] >= 0) out[k] = mk[k / kWarpTile];
  }
  return PF_OK;
}

// After the host wrote every slot of filter f's ancestors: no segment marker
// may override them.
int clear_segment_markers(pf_engine* eng, int f) {
  if (!eng->dev.anc_seg) return PF_OK;
  const FilterDesc& d = eng->hdesc[f];
  CK(cudaMemset(eng->dev.seg_anc + (size_t)d.tile_begin * kSubTiles, 0xFF, sizeof(int) * (size_t)d.n_tiles * kSubTiles));
  return PF_OK;
}

}  // namespace

extern "C" {

int pfe_workspace_bytes(const pf_engine_config_t* cfg, const pf_filter_params_t* filters,
                        size_t* bytes) {
  clear_err();
  int s = validate_config(cfg, filters);
  if (s != PF_OK) return s;
  if (!bytes) return set_err(PF_EINVAL, "null bytes");
  *bytes = make_layout(cfg, filters).total;
  return PF_OK;
}

int pfe_create(const pf_engine_config_t* cfg, const pf_filter_params_t* filters,
               void* dev_workspace, size_t workspace_bytes, void* stream, pf_engine_t** out) {
  clear_err();
  int s = validate_config(cfg, filters);
  if (s != PF_OK) return s;
  if (!out) return set_err(PF_EINVAL, "null out");
  Layout L = make_layout(cfg, filters);
  if (!dev_workspace) return set_err(PF_EINVAL, "null workspace");
  if (workspace_bytes < L.total)
    return set_err(PF_ENOMEM, "workspace %zu bytes < required %zu", workspace_bytes, L.total);
  if (((uintptr_t)dev_workspace & 255u) != 0) return set_err(PF_EINVAL, "workspace must be 256-byte aligned");

  pf_engine* eng = new pf_engine();
  eng->cfg = *cfg;
  eng->params.assign(filters, filters + cfg->n_filters);
  eng->D = L.D;
  eng->T = L.T;
  eng->P = L.P;
  eng->max_n = L.max_n;
  eng->ws = (unsigned char*)dev_workspace;
  eng->ws_bytes = workspace_bytes;
  eng->stream = (cudaStream_t)stream;
  eng->obs_slot_bytes = L.obs_slot_bytes;
  eng->initialized.assign(cfg->n_filters, 0);

  eng->hdesc.assign(cfg->n_filters, FilterDesc{});
  eng->tile_filter.resize(L.T);
  long long poff = 0;
  int tb = 0;
  for (int f = 0; f < cfg->n_filters; ++f) {
    FilterDesc& d = eng->hdesc[f];
    d.n = filters[f].n_particles;
    d.tile_begin = tb;
    d.n_tiles = (d.n + PF_TILE - 1) / PF_TILE;
    d.K = quant_exponent(d.n);
    d.p_off = poff;
    d.filter_id = f;
    for (int i = 0; i < 9; ++i) d.rot[i] = (i % 4 == 0) ? 1.0 : 0.0;
    fill_desc(eng, f);
    for (int t = 0; t < d.n_tiles; ++t) eng->tile_filter[tb + t] = f;
    tb += d.n_tiles;
    poff += (long long)align_up((size_t)d.n, 4);
  }

  unsigned char* w = eng->ws;
  EngineDev& e = eng->dev;
  e.state0 = (float*)(w + L.off_state0);
  e.state1 = (float*)(w + L.off_state1);
  e.lw = (float*)(w + L.off_lw);
  e.anc = (int*)(w + L.off_anc);
  e.offs = (uint32_t*)(w + L.off_offs);
  e.mp_part = (uint32_t*)(w + L.off_mp);
  e.part = (float*)(w + L.off_part);
  e.lb_agg = (unsigned long long*)(w + L.off_agg);
  e.lb_inc = (unsigned long long*)(w + L.off_inc);
  e.lb_flag = (unsigned*)(w + L.off_flag);
  e.tile_excl = (unsigned long long*)(w + L.off_excl);
  e.seg_c = (double*)(w + L.off_wq);
  e.seg_rho = (double*)(w + L.off_seg_rho);
  e.seg_E = (double*)(w + L.off_seg_E);
  e.tile_S = (double*)(w + L.off_tile_S);
  e.tile_m = (float*)(w + L.off_tile_m);
  e.seg_anc = (int*)(w + L.off_seg_anc);
  // the epoch kernel's systematic resampler marks whole-segment runs there
  e.anc_seg = (cfg->resampler == PF_RESAMPLE_SYSTEMATIC && !(cfg->flags & PF_FLAG_KERNEL_CHAIN)) ? 1 : 0;
  e.mlp = (const float*)(w + L.off_mlp);
  e.sat_dbg = (float*)(w + L.off_satdbg);
  eng->obs_rows = (ObsRow*)(w + L.off_obsrows);
  eng->desc_dev = (FilterDesc*)(w + L.off_desc);
  eng->ctrl_dev = (FilterCtrl*)(w + L.off_ctrl);
  e.desc = eng->desc_dev;
  e.ctrl = eng->ctrl_dev;
  e.tile_filter = (const int*)(w + L.off_tf);
  e.queue = (unsigned*)(w + L.off_queue);
  eng->bar = e.queue + 2 * Q_COUNT;
  e.err = (unsigned*)(w + L.off_err);
  e.obs = w + L.off_obs;
  e.obs_slot_bytes = L.obs_slot_bytes;
  e.spin_limit = 1ull << 24;
  e.p_total = L.P;
  e.obs_slots = cfg->obs_slots;
  e.n_filters = cfg->n_filters;
  e.max_sats = cfg->max_sats;
  e.resampler = cfg->resampler;
  e.mego_iters = cfg->megopolis_iters;
  e.lw_mode = cfg->lw_mode;
  e.sys_offset = cfg->sys_offset;
  e.flags = cfg->flags;
  e.ess_threshold = (float)cfg->ess_threshold;
  e.lookback_poison = 0;
  eng->export_buf = (double*)(w + L.off_export);

  auto fail = [&](int st) {
    pfe_destroy(eng);
    return st;
  };
  int dev = 0;
  if (check_cuda(cudaGetDevice(&dev), "cudaGetDevice") != PF_OK) return fail(PF_ECUDA);
  if (check_cuda(cudaDeviceGetAttribute(&eng->sm_count, cudaDevAttrMultiProcessorCount, dev), "sm count") != PF_OK)
    return fail(PF_ECUDA);
  int st = PF_OK;
  if (cfg->n_clk == 1) st = occupancy(k_step<1, PF_WEIGHT_GAUSSIAN>, eng->sm_count, &eng->resident[Q_STEP]);
  else if (cfg->n_clk == 2) st = occupancy(k_step<2, PF_WEIGHT_GAUSSIAN>, eng->sm_count, &eng->resident[Q_STEP]);
  else if (cfg->n_clk == 3) st = occupancy(k_step<3, PF_WEIGHT_GAUSSIAN>, eng->sm_count, &eng->resident[Q_STEP]);
  else st = occupancy(k_step<4, PF_WEIGHT_GAUSSIAN>, eng->sm_count, &eng->resident[Q_STEP]);
  if (st != PF_OK) return fail(st);
  if ((st = occupancy(k_scan, eng->sm_count, &eng->resident[Q_SCAN])) != PF_OK) return fail(st);
  if ((st = occupancy(k_offs, eng->sm_count, &eng->resident[Q_OFFS])) != PF_OK) return fail(st);
  if ((st = occupancy(k_merge, eng->sm_count, &eng->resident[Q_MERGE])) != PF_OK) return fail(st);
  if ((st = occupancy(k_mego, eng->sm_count, &eng->resident[Q_MEGO])) != PF_OK) return fail(st);
  if ((st = prepare_epoch_kernel(eng)) != PF_OK) return fail(st);
  if ((st = occupancy(k_init<7>, eng->sm_count, &eng->resident[Q_INIT])) != PF_OK) return fail(st);
  if ((st = occupancy(k_estimate<7>, eng->sm_count, &eng->resident[Q_EST])) != PF_OK) return fail(st);
  if ((st = occupancy(k_export<7>, eng->sm_count, &eng->resident[Q_EXPORT])) != PF_OK) return fail(st);

  for (int i = 0; i < 2; ++i) {
    if (pf_injected_alloc_failure()) {
      set_err(PF_ENOMEM, "pinned staging allocation failed (injected by pf_test_fail_alloc)");
      return fail(PF_ENOMEM);
    }
    if (check_cuda(cudaHostAlloc((void**)&eng->pinned[i], L.obs_slot_bytes, cudaHostAllocDefault), "pinned staging") != PF_OK)
      return fail(PF_ENOMEM);
    if (check_cuda(cudaEventCreateWithFlags(&eng->pin_ev[i], cudaEventDisableTiming), "event") != PF_OK)
      return fail(PF_ECUDA);
  }
  eng->ctrl_span = (L.off_err - L.off_ctrl) + sizeof(unsigned) * 4;
  if (pf_injected_alloc_failure()) {
    set_err(PF_ENOMEM, "pinned control-block allocation failed (injected by pf_test_fail_alloc)");
    return fail(PF_ENOMEM);
  }
  if (check_cuda(cudaHostAlloc((void**)&eng->ctrl_host, eng->ctrl_span, cudaHostAllocDefault), "pinned ctrl") != PF_OK)
    return fail(PF_ENOMEM);
  eng->err_host = (unsigned*)((unsigned char*)eng->ctrl_host + (L.off_err - L.off_ctrl));

  // Device tables and zeroed control blocks.
  std::vector<FilterCtrl> hc(cfg->n_filters);
  memset(hc.data(), 0, sizeof(FilterCtrl) * hc.size());
  for (auto& c : hc) {
    c.lw_zero = 1;
    c.rs_seq = 1;
  }
  if (check_cuda(cudaMemsetAsync(w + L.off_flag, 0, (size_t)L.T * 4, eng->stream), "memset flags") != PF_OK ||
      check_cuda(cudaMemsetAsync(w + L.off_queue, 0, sizeof(unsigned) * (2 * Q_COUNT + kBarWords),
                                 eng->stream), "memset queue") != PF_OK ||
      check_cuda(cudaMemsetAsync(w + L.off_err, 0, sizeof(unsigned) * 4, eng->stream), "memset err") != PF_OK ||
      check_cuda(cudaMemsetAsync(w + L.off_seg_anc, 0xFF, (size_t)L.T * kSubTiles * 4, eng->stream),
                 "memset segment markers") != PF_OK ||
      check_cuda(cudaMemsetAsync(w + L.off_obs, 0, L.obs_slot_bytes * cfg->obs_slots, eng->stream), "memset obs") != PF_OK ||
      check_cuda(cudaMemsetAsync(w + L.off_state0, 0, (size_t)L.D * L.P * 4, eng->stream), "memset state") != PF_OK ||
      check_cuda(cudaMemsetAsync(w + L.off_lw, 0, (size_t)L.P * 4, eng->stream), "memset lw") != PF_OK)
    return fail(PF_ECUDA);
  if (check_cuda(cudaMemcpyAsync(eng->desc_dev, eng->hdesc.data(), sizeof(FilterDesc) * cfg->n_filters,
                                 cudaMemcpyHostToDevice, eng->stream), "desc upload") != PF_OK ||
      check_cuda(cudaMemcpyAsync(eng->ctrl_dev, hc.data(), sizeof(FilterCtrl) * cfg->n_filters,
                                 cudaMemcpyHostToDevice, eng->stream), "ctrl upload") != PF_OK ||
      check_cuda(cudaMemcpyAsync((void*)e.tile_filter, eng->tile_filter.data(), sizeof(int) * L.T,
                                 cudaMemcpyHostToDevice, eng->stream), "tile table upload") != PF_OK ||
      check_cuda(cudaStreamSynchronize(eng->stream), "create sync") != PF_OK)
    return fail(PF_ECUDA);
  *out = eng;
  return PF_OK;
}

int pfe_destroy(pf_engine_t* eng) {
  if (!eng) return PF_OK;
  if (eng->stream) cudaStreamSynchronize(eng->stream);
  if (eng->gexec) cudaGraphExecDestroy(eng->gexec);
  if (eng->graph) cudaGraphDestroy(eng->graph);
  for (int i = 0; i < 2; ++i) {
    if (eng->pinned[i]) cudaFreeHost(eng->pinned[i]);
    if (eng->pin_ev[i]) cudaEventDestroy(eng->pin_ev[i]);
  }
  for (int i = 0; i < 2; ++i) {
    if (eng->io_exec[i]) cudaGraphExecDestroy(eng->io_exec[i]);
    if (eng->io_graph[i]) cudaGraphDestroy(eng->io_graph[i]);
  }
  if (eng->ctrl_host) cudaFreeHost(eng->ctrl_host);
  for (cudaEvent_t e : eng->tev) cudaEventDestroy(e);
  delete eng;
  return PF_OK;
}

int pfe_set_stream(pf_engine_t* eng, void* stream) {
  clear_err();
  if (!eng) return set_err(PF_EINVAL, "null engine");
  eng->stream = (cudaStream_t)stream;
  return PF_OK;
}

int pfe_set_epoch_ctas_per_sm(pf_engine_t* eng, int ctas_per_sm, int* resident_per_sm) {
  clear_err();
  if (!eng) return set_err(PF_EINVAL, "null engine");
  const int per_sm = eng->sm_count > 0 ? eng->epoch_resident / eng->sm_count : 0;
  if (resident_per_sm) *resident_per_sm = per_sm;
  if (ctas_per_sm < 0 || ctas_per_sm > per_sm)
    return set_err(PF_EINVAL, "ctas_per_sm must be 0 (all resident) .. %d", per_sm);
  eng->epoch_cap = ctas_per_sm == 0 ? 0 : ctas_per_sm * eng->sm_count;
  return PF_OK;
}

int pfe_set_filter_params(pf_engine_t* eng, int filter, const pf_filter_params_t* params) {
  clear_err();
  int s = check_filter(eng, filter);
  if (s != PF_OK) return s;
  if (!params) return set_err(PF_EINVAL, "null params");
  if (params->n_particles != eng->params[filter].n_particles)
    return set_err(PF_EINVAL, "n_particles cannot change after pfe_create");
  pf_engine_config_t one = eng->cfg;
  one.n_filters = 1;
  if ((s = validate_config(&one, params)) != PF_OK) return s;
  eng->params[filter] = *params;
  fill_desc(eng, filter);
  CK(cudaMemcpyAsync(eng->desc_dev + filter, &eng->hdesc[filter], sizeof(FilterDesc), cudaMemcpyHostToDevice,
                     eng->stream));
  CK(cudaStreamSynchronize(eng->stream));
  return PF_OK;
}

int pfe_initialize(pf_engine_t* eng, int filter, const double anchor_ecef[3], const double* clk0,
                   double spread_pos, double spread_clk) {
  clear_err();
  int s = check_filter(eng, filter);
  if (s != PF_OK) return s;
  if (!anchor_ecef) return set_err(PF_EINVAL, "null anchor");
  for (int i = 0; i < 3; ++i)
    if (!isfinite(anchor_ecef[i])) return set_err(PF_EINVAL, "anchor must be finite");
  if (!(spread_pos >= 0.0) || !(spread_clk >= 0.0) || !isfinite(spread_pos) || !isfinite(spread_clk))
    return set_err(PF_EINVAL, "spreads must be finite and >= 0");
  FilterDesc& d = eng->hdesc[filter];
  enu_rotation(anchor_ecef, d.rot);
  CK(cudaMemcpyAsync(eng->desc_dev + filter, &d, sizeof(FilterDesc), cudaMemcpyHostToDevice, eng->stream));
  // The control block goes through the pinned mirror so the copy is truly
  // asynchronous-safe.
  CK(cudaStreamSynchronize(eng->stream));
  FilterCtrl c;
  memset(&c, 0, sizeof(c));
  CK(cudaMemcpy(&c, eng->ctrl_dev + filter, sizeof(FilterCtrl), cudaMemcpyDeviceToHost));
  const unsigned rs_seq = c.rs_seq;
  memset(&c, 0, sizeof(c));
  for (int i = 0; i < 3; ++i) c.anchor[i] = anchor_ecef[i];
  for (int k = 0; k < eng->cfg.n_clk; ++k) {
    double v = clk0 ? clk0[k] : 0.0;
    if (!isfinite(v)) return set_err(PF_EINVAL, "clock anchor must be finite");
    c.clk_anchor[k] = v;
  }
  c.lw_zero = 1;
  c.rs_seq = rs_seq + 1u;
  c.initialized = 1;
  eng->ctrl_host[filter] = c;
  CK(cudaMemcpyAsync(eng->ctrl_dev + filter, &eng->ctrl_host[filter], sizeof(FilterCtrl), cudaMemcpyHostToDevice,
                     eng->stream));
  const int g = grid_for(eng, Q_INIT, d.n_tiles);
  switch (eng->D) {
    case 4: k_init<4><<<g, kThreads, 0, eng->stream>>>(eng->dev, d.tile_begin, d.n_tiles, (float)spread_pos, (float)spread_clk); break;
    case 5: k_init<5><<<g, kThreads, 0, eng->stream>>>(eng->dev, d.tile_begin, d.n_tiles, (float)spread_pos, (float)spread_clk); break;
    case 6: k_init<6><<<g, kThreads, 0, eng->stream>>>(eng->dev, d.tile_begin, d.n_tiles, (float)spread_pos, (float)spread_clk); break;
    default: k_init<7><<<g, kThreads, 0, eng->stream>>>(eng->dev, d.tile_begin, d.n_tiles, (float)spread_pos, (float)spread_clk); break;
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(eng->stream));
  eng->initialized[filter] = 1;
  return PF_OK;
}

int pfe_get_frame(pf_engine_t* eng, int filter, double rot[9], double anchor_ecef[3]) {
  clear_err();
  int s = check_filter(eng, filter);
  if (s != PF_OK) return s;
  if (rot) memcpy(rot, eng->hdesc[filter].rot, sizeof(double) * 9);
  if (anchor_ecef) {
    if ((s = read_ctrl(eng)) != PF_OK) return s;
    memcpy(anchor_ecef, eng->ctrl_host[filter].anchor, sizeof(double) * 3);
  }
  return PF_OK;
}

int pfe_obs_slot_bytes(pf_engine_t* eng, size_t* bytes) {
  clear_err();
  if (!eng || !bytes) return set_err(PF_EINVAL, "null argument");
  *bytes = eng->obs_slot_bytes;
  return PF_OK;
}

}  // extern "C"

namespace {

// Checks of one epoch's records before they are staged (pfe_upload_obs,
// pfe_step_io).
int validate_obs(pf_engine* eng, const pf_filter_epoch_t* fe, const pf_sat_t* sats, int n_sats_total) {
  const int F = eng->cfg.n_filters;
  const int cap = F * eng->cfg.max_sats;
  if (n_sats_total < 0 || n_sats_total > cap) return set_err(PF_ECAP, "n_sats_total %d above capacity %d", n_sats_total, cap);
  if (n_sats_total > 0 && !sats) return set_err(PF_EINVAL, "null sats");
  for (int f = 0; f < F; ++f) {
    const pf_filter_epoch_t& r = fe[f];
    if (r.n_sat < 0 || r.n_sat > eng->cfg.max_sats)
      return set_err(PF_ECAP, "filter %d: n_sat %d above max_sats %d", f, r.n_sat, eng->cfg.max_sats);
    if (r.sat_offset < 0 || r.sat_offset + r.n_sat > n_sats_total)
      return set_err(PF_EINVAL, "filter %d: satellite range out of bounds", f);
    for (int i = 0; i < 3; ++i)
      if (!isfinite(r.disp[i])) return set_err(PF_EINVAL, "filter %d: displacement must be finite", f);
    if ((r.flags & PF_EP_WEIGHT)) {
      for (int k = 0; k < r.n_sat; ++k) {
        const pf_sat_t& sv = sats[r.sat_offset + k];
        if (!isfinite(sv.x) || !isfinite(sv.y) || !isfinite(sv.z) || !isfinite(sv.pr) || !isfinite(sv.w) || sv.w < 0)
          return set_err(PF_EINVAL, "filter %d: satellite %d has non-finite position/pseudorange/weight", f, k);
        if (sv.clk < 0 || sv.clk >= eng->cfg.n_clk)
          return set_err(PF_EINVAL, "filter %d: satellite %d clock index %d out of range", f, k, sv.clk);
      }
    }
  }
  return PF_OK;
}

}  // namespace

extern "C" {

int pfe_upload_obs(pf_engine_t* eng, int slot, const pf_filter_epoch_t* fe, const pf_sat_t* sats,
                   int n_sats_total) {
  clear_err();
  if (!eng || !fe) return set_err(PF_EINVAL, "null argument");
  if (slot < 0 || slot >= eng->cfg.obs_slots) return set_err(PF_EINVAL, "slot %d out of range", slot);
  const int F = eng->cfg.n_filters;
  int vs = validate_obs(eng, fe, sats, n_sats_total);
  if (vs != PF_OK) return vs;
  const int b = eng->pin_cur;
  eng->pin_cur ^= 1;
  CK(cudaEventSynchronize(eng->pin_ev[b]));
  unsigned char* h = eng->pinned[b];
  const size_t fe_bytes = sizeof(pf_filter_epoch_t) * F;
  memcpy(h, fe, fe_bytes);
  if (n_sats_total > 0) memcpy(h + fe_bytes, sats, sizeof(pf_sat_t) * n_sats_total);
  const size_t bytes = fe_bytes + sizeof(pf_sat_t) * (size_t)n_sats_total;
  CK(cudaMemcpyAsync((void*)(eng->dev.obs + (size_t)slot * eng->obs_slot_bytes), h, bytes, cudaMemcpyHostToDevice,
                     eng->stream));
  CK(cudaEventRecord(eng->pin_ev[b], eng->stream));
  return PF_OK;
}

int pfe_step(pf_engine_t* eng) {
  clear_err();
  if (!eng) return set_err(PF_EINVAL, "null engine");
  for (int f = 0; f < eng->cfg.n_filters; ++f)
    if (!eng->initialized[f]) return set_err(PF_ENOTINIT, "filter %d not initialized", f);
  if (eng->cfg.weight_mode == PF_WEIGHT_MIXTURE && !eng->mlp_set)
    return set_err(PF_ENOTINIT, "mixture likelihood: network parameters not set (pfe_set_mlp)");
  int n = 1;
  cudaEvent_t* ev = nullptr;
  if (eng->t_slots > 0) {
    ev = &eng->tev[kTimingEvents * (size_t)eng->t_next];
    eng->t_next = (eng->t_next + 1) % eng->t_slots;
    eng->t_pending = std::min(eng->t_pending + 1, eng->t_slots);
    CK(cudaEventRecord(ev[0], eng->stream));
  }
  if (!use_chain(eng)) {
    int s = launch_epoch(eng, 0, eng->T);
    if (s != PF_OK) return s;
    // one event after the single kernel: every extra event record on the
    // stream adds microseconds to the measured step
    if (ev) CK(cudaEventRecord(ev[1], eng->stream));
    eng->last_launches = 1;
    return PF_OK;
  }
  int s = launch_step(eng, 0, eng->T);
  if (s != PF_OK) return s;
  if (ev) CK(cudaEventRecord(ev[1], eng->stream));
  s = launch_resample(eng, 0, eng->T, &n, (ev && eng->t_detailed) ? ev + 2 : nullptr);
  if (s != PF_OK) return s;
  if (ev && !eng->t_detailed) CK(cudaEventRecord(ev[kTimingEvents - 1], eng->stream));
  eng->last_launches = n;
  return PF_OK;
}

int pfe_read_timing_kernels(pf_engine_t* eng, float* out, int max_entries, int* count) {
  clear_err();
  if (!eng || !out || !count) return set_err(PF_EINVAL, "null argument");
  const int n = std::min((int)(eng->t_kernel_ms.size() / (kTimingEvents - 1)), max_entries);
  memcpy(out, eng->t_kernel_ms.data(), sizeof(float) * (size_t)n * (kTimingEvents - 1));
  *count = n;
  return PF_OK;
}

int pfe_enable_timing(pf_engine_t* eng, int slots, int detailed) {
  clear_err();
  if (!eng) return set_err(PF_EINVAL, "null engine");
  eng->t_detailed = detailed ? 1 : 0;
  if (slots < 0) return set_err(PF_EINVAL, "slots must be >= 0");
  if (eng->gexec || eng->graph) return set_err(PF_EINVAL, "timing applies to eager steps, not captured graphs");
  CK(cudaStreamSynchronize(eng->stream));
  for (cudaEvent_t e : eng->tev) cudaEventDestroy(e);
  eng->tev.clear();
  eng->t_slots = 0;
  eng->t_next = 0;
  eng->t_pending = 0;
  if (slots == 0) return PF_OK;
  eng->tev.resize(kTimingEvents * (size_t)slots, nullptr);
  for (auto& e : eng->tev) CK(cudaEventCreate(&e));
  eng->t_slots = slots;
  return PF_OK;
}

int pfe_read_timing(pf_engine_t* eng, float* step_kernel_ms, float* whole_step_ms, int max_entries,
                    int* count) {
  clear_err();
  if (!eng || !count) return set_err(PF_EINVAL, "null argument");
  *count = 0;
  if (eng->t_slots == 0) return set_err(PF_EINVAL, "timing is not enabled");
  CK(cudaStreamSynchronize(eng->stream));
  const int n = std::min(eng->t_pending, max_entries);
  eng->t_kernel_ms.assign((size_t)n * (kTimingEvents - 1), 0.f);
  const int first = (eng->t_next - eng->t_pending + eng->t_slots) % eng->t_slots;
  for (int i = 0; i < n; ++i) {
    const cudaEvent_t* ev = &eng->tev[kTimingEvents * (size_t)((first + i) % eng->t_slots)];
    float a = 0.f, b = 0.f;
    CK(cudaEventElapsedTime(&a, ev[0], ev[1]));
    if (use_chain(eng)) CK(cudaEventElapsedTime(&b, ev[0], ev[kTimingEvents - 1]));
    else b = a;  // the epoch kernel is the whole step
    if (step_kernel_ms) step_kernel_ms[i] = a;
    if (whole_step_ms) whole_step_ms[i] = b;
    for (int k = 0; k < kTimingEvents - 1; ++k) {
      float m = 0.f;
      if ((eng->t_detailed && use_chain(eng)) || k == 0) CK(cudaEventElapsedTime(&m, ev[k], ev[k + 1]));
      eng->t_kernel_ms[(size_t)i * (kTimingEvents - 1) + k] = m;
    }
    if (!eng->t_detailed && use_chain(eng)) eng->t_kernel_ms[(size_t)i * (kTimingEvents - 1) + 1] = b - a;
  }
  *count = n;
  eng->t_pending = 0;
  return PF_OK;
}

int pfe_step_per_filter(pf_engine_t* eng) {
  clear_err();
  if (!eng) return set_err(PF_EINVAL, "null engine");
  int n = 0;
  for (int f = 0; f < eng->cfg.n_filters; ++f) {
    if (!eng->initialized[f]) return set_err(PF_ENOTINIT, "filter %d not initialized", f);
    const FilterDesc& d = eng->hdesc[f];
    if (!use_chain(eng)) {
      int s = launch_epoch(eng, d.tile_begin, d.n_tiles);
      if (s != PF_OK) return s;
      ++n;
      continue;
    }
    int s = launch_step(eng, d.tile_begin, d.n_tiles);
    if (s != PF_OK) return s;
    ++n;
    s = launch_resample(eng, d.tile_begin, d.n_tiles, &n);
    if (s != PF_OK) return s;
  }
  eng->last_launches = n;
  return PF_OK;
}

int pfe_graph_capture(pf_engine_t* eng, int per_filter) {
  clear_err();
  if (!eng) return set_err(PF_EINVAL, "null engine");
  if (!eng->stream) return set_err(PF_EINVAL, "graph capture needs a non-default stream (pfe_set_stream)");
  if (eng->gexec) {
    cudaGraphExecDestroy(eng->gexec);
    eng->gexec = nullptr;
  }
  if (eng->graph) {
    cudaGraphDestroy(eng->graph);
    eng->graph = nullptr;
  }
  CK(cudaStreamBeginCapture(eng->stream, cudaStreamCaptureModeThreadLocal));
  const int saved_slots = eng->t_slots;  // no timing events inside a graph
  eng->t_slots = 0;
  int s = per_filter ? pfe_step_per_filter(eng) : pfe_step(eng);
  eng->t_slots = saved_slots;
  cudaGraph_t g = nullptr;
  cudaError_t ce = cudaStreamEndCapture(eng->stream, &g);
  if (s != PF_OK) {
    if (g) cudaGraphDestroy(g);
    return s;
  }
  CK(ce);
  eng->graph = g;
  CK(cudaGraphInstantiate(&eng->gexec, g, 0));
  return PF_OK;
}

int pfe_graph_launch(pf_engine_t* eng, int n_epochs) {
  clear_err();
  if (!eng || !eng->gexec) return set_err(PF_EINVAL, "no captured graph");
  for (int i = 0; i < n_epochs; ++i) CK(cudaGraphLaunch(eng->gexec, eng->stream));
  return PF_OK;
}

}  // extern "C"

namespace {

void fill_results(pf_engine* eng, pf_filter_result_t* out) {
  for (int f = 0; f < eng->cfg.n_filters; ++f) {
    const FilterCtrl& c = eng->ctrl_host[f];
    pf_filter_result_t& r = out[f];
    memset(&r, 0, sizeof(r));
    for (int i = 0; i < 3; ++i) r.est_ecef[i] = c.est_ecef[i];
    for (int k = 0; k < PF_MAX_CLK; ++k) r.est_clk[k] = c.est_clk[k];
    for (int i = 0; i < 6; ++i) r.cov_enu[i] = c.cov[i];
    r.ess = c.ess;
    r.sum_w = c.sum_w;
    r.max_lw = c.max_lw;
    r.resampled = c.resample_flag;
    r.epoch = c.epoch;
    r.initialized = eng->initialized[f];
  }
}

// Everything the epoch launch of a step-io graph depends on: the kernel's
// parameter block, the kernel chosen, the grid and its shared memory.
std::vector<unsigned char> io_key(pf_engine* eng) {
  struct Launch {
    EpochKernel fn;
    unsigned* bar;
    int T, resident, cap;
    size_t smem;
  } x;
  memset(&x, 0, sizeof(x));
  x.fn = epoch_kernel(eng);
  x.bar = eng->bar;
  x.T = eng->T;
  x.resident = eng->epoch_resident;
  x.cap = eng->epoch_cap;
  x.smem = eng->epoch_smem;
  std::vector<unsigned char> k(sizeof(EngineDev) + sizeof(Launch));
  memcpy(k.data(), &eng->dev, sizeof(EngineDev));
  memcpy(k.data() + sizeof(EngineDev), &x, sizeof(Launch));
  return k;
}

// (Re)capture staging buffer b's graph: upload copy of `bytes`, the epoch
// kernel, one copy of the control blocks and the error word back.
int io_capture(pf_engine* eng, int b, size_t bytes) {
  if (eng->io_exec[b]) cudaGraphExecDestroy(eng->io_exec[b]);
  if (eng->io_graph[b]) cudaGraphDestroy(eng->io_graph[b]);
  eng->io_exec[b] = nullptr;
  eng->io_graph[b] = nullptr;
  eng->io_h2d[b] = nullptr;
  eng->io_key[b].clear();
  CK(cudaStreamBeginCapture(eng->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t ce = cudaMemcpyAsync((void*)eng->dev.obs, eng->pinned[b], bytes, cudaMemcpyHostToDevice, eng->stream);
  int s = ce == cudaSuccess ? launch_epoch(eng, 0, eng->T) : set_err(PF_ECUDA, "capture upload: %s", cudaGetErrorString(ce));
  if (s == PF_OK) {
    ce = cudaMemcpyAsync(eng->ctrl_host, eng->ctrl_dev, eng->ctrl_span, cudaMemcpyDeviceToHost, eng->stream);
    if (ce != cudaSuccess) s = set_err(PF_ECUDA, "capture result copy: %s", cudaGetErrorString(ce));
  }
  cudaGraph_t g = nullptr;
  ce = cudaStreamEndCapture(eng->stream, &g);
  if (s != PF_OK) {
    if (g) cudaGraphDestroy(g);
    return s;
  }
  CK(ce);
  eng->io_graph[b] = g;
  size_t n = 0;
  CK(cudaGraphGetNodes(g, nullptr, &n));
  std::vector<cudaGraphNode_t> nodes(n);
  CK(cudaGraphGetNodes(g, nodes.data(), &n));
  for (cudaGraphNode_t nd : nodes) {
    cudaGraphNodeType t;
    CK(cudaGraphNodeGetType(nd, &t));
    if (t != cudaGraphNodeTypeMemcpy) continue;
    cudaMemcpy3DParms mp;
    CK(cudaGraphMemcpyNodeGetParams(nd, &mp));
    if (mp.kind == cudaMemcpyHostToDevice) eng->io_h2d[b] = nd;
  }
  if (!eng->io_h2d[b]) return set_err(PF_ECUDA, "step-io graph: upload node not found");
  CK(cudaGraphInstantiate(&eng->io_exec[b], g, 0));
  eng->io_h2d_bytes[b] = bytes;
  eng->io_key[b] = io_key(eng);
  return PF_OK;
}

}  // namespace

extern "C" {

int pfe_read_results(pf_engine_t* eng, pf_filter_result_t* out) {
  clear_err();
  if (!eng || !out) return set_err(PF_EINVAL, "null argument");
  int s = read_ctrl(eng);
  if (s != PF_OK) return s;
  fill_results(eng, out);
  return PF_OK;
}

int pfe_step_io(pf_engine_t* eng, const pf_filter_epoch_t* fe, const pf_sat_t* sats, int n_sats_total,
                pf_filter_result_t* out) {
  clear_err();
  if (!eng || !fe || !out) return set_err(PF_EINVAL, "null argument");
  if (eng->cfg.obs_slots != 1) return set_err(PF_EINVAL, "pfe_step_io needs an engine with obs_slots == 1");
  if (use_chain(eng) || eng->t_slots > 0 || !eng->stream) {
    // kernel chain, timed steps or the legacy stream: separate calls
    int s = pfe_upload_obs(eng, 0, fe, sats, n_sats_total);
    if (s != PF_OK) return s;
    if ((s = pfe_step(eng)) != PF_OK) return s;
    return pfe_read_results(eng, out);
  }
  int s = validate_obs(eng, fe, sats, n_sats_total);
  if (s != PF_OK) return s;
  for (int f = 0; f < eng->cfg.n_filters; ++f)
    if (!eng->initialized[f]) return set_err(PF_ENOTINIT, "filter %d not initialized", f);
  if (eng->cfg.weight_mode == PF_WEIGHT_MIXTURE && !eng->mlp_set)
    return set_err(PF_ENOTINIT, "mixture likelihood: network parameters not set (pfe_set_mlp)");
  const int b = eng->pin_cur;
  eng->pin_cur ^= 1;
  CK(cudaEventSynchronize(eng->pin_ev[b]));
  unsigned char* h = eng->pinned[b];
  const size_t fe_bytes = sizeof(pf_filter_epoch_t) * eng->cfg.n_filters;
  memcpy(h, fe, fe_bytes);
  if (n_sats_total > 0) memcpy(h + fe_bytes, sats, sizeof(pf_sat_t) * n_sats_total);
  const size_t bytes = fe_bytes + sizeof(pf_sat_t) * (size_t)n_sats_total;
  if (!eng->io_exec[b] || eng->io_key[b] != io_key(eng)) {
    if ((s = io_capture(eng, b, bytes)) != PF_OK) return s;
  } else if (bytes != eng->io_h2d_bytes[b]) {
    CK(cudaGraphExecMemcpyNodeSetParams1D(eng->io_exec[b], eng->io_h2d[b], (void*)eng->dev.obs, h, bytes,
                                          cudaMemcpyHostToDevice));
    eng->io_h2d_bytes[b] = bytes;
  }
  CK(cudaGraphLaunch(eng->io_exec[b], eng->stream));
  CK(cudaStreamSynchronize(eng->stream));
  eng->last_launches = 1;
  if ((s = err_status(*eng->err_host)) != PF_OK) return s;
  fill_results(eng, out);
  return PF_OK;
}

int pfe_result_bytes(pf_engine_t* eng, size_t* bytes) {
  clear_err();
  if (!eng || !bytes) return set_err(PF_EINVAL, "null argument");
  *bytes = sizeof(FilterCtrl) * (size_t)eng->cfg.n_filters;
  return PF_OK;
}

// One pass of k_estimate over filter f's current particles and weights;
// leaves api_est / api_m2 in the host copy of the control block.
static int run_estimate(pf_engine_t* eng, int filter) {
  int s = check_filter(eng, filter);
  if (s != PF_OK) return s;
  if (!eng->initialized[filter]) return set_err(PF_ENOTINIT, "filter %d not initialized", filter);
  const FilterDesc& d = eng->hdesc[filter];
  const int g = grid_for(eng, Q_EST, d.n_tiles);
  switch (eng->D) {
    case 4: k_estimate<4><<<g, kThreads, 0, eng->stream>>>(eng->dev, d.tile_begin, d.n_tiles); break;
    case 5: k_estimate<5><<<g, kThreads, 0, eng->stream>>>(eng->dev, d.tile_begin, d.n_tiles); break;
    case 6: k_estimate<6><<<g, kThreads, 0, eng->stream>>>(eng->dev, d.tile_begin, d.n_tiles); break;
    default: k_estimate<7><<<g, kThreads, 0, eng->stream>>>(eng->dev, d.tile_begin, d.n_tiles); break;
  }
  CK(cudaGetLastError());
  return read_ctrl(eng);
}

int pfe_estimate(pf_engine_t* eng, int filter, double* out) {
  clear_err();
  if (!out) return set_err(PF_EINVAL, "null out");
  int s = run_estimate(eng, filter);
  if (s != PF_OK) return s;
  for (int i = 0; i < eng->D; ++i) out[i] = eng->ctrl_host[filter].api_est[i];
  return PF_OK;
}

int pfe_current_ess(pf_engine_t* eng, int filter, double* out) {
  clear_err();
  if (!out) return set_err(PF_EINVAL, "null out");
  int s = run_estimate(eng, filter);
  if (s != PF_OK) return s;
  *out = eng->ctrl_host[filter].api_est[7];
  return PF_OK;
}

int pfe_position_spread(pf_engine_t* eng, int filter, const double* center_ecef, double* out) {
  clear_err();
  if (!out) return set_err(PF_EINVAL, "null out");
  if (center_ecef)
    for (int i = 0; i < 3; ++i)
      if (!isfinite(center_ecef[i])) return set_err(PF_EINVAL, "center must be finite");
  int s = run_estimate(eng, filter);
  if (s != PF_OK) return s;
  const FilterCtrl& c = eng->ctrl_host[filter];
  const double* rot = eng->hdesc[filter].rot;
  // local mean m and local centre q (rows of rot are E, N, U in ECEF)
  const double* ctr = center_ecef ? center_ecef : c.api_est;
  double m[3], q[3];
  for (int r = 0; r < 3; ++r) {
    m[r] = q[r] = 0.0;
    for (int i = 0; i < 3; ++i) {
      m[r] += rot[3 * r + i] * (c.api_est[i] - c.anchor[i]);
      q[r] += rot[3 * r + i] * (ctr[i] - c.anchor[i]);
    }
  }
  // E|x - q|^2 = E|x|^2 - 2 q.m + |q|^2 (second moments about the anchor)
  const double ex2 = c.api_m2[0] + c.api_m2[3] + c.api_m2[5];
  const double v = ex2 - 2.0 * (q[0] * m[0] + q[1] * m[1] + q[2] * m[2]) + q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
  *out = sqrt(v > 0.0 ? v : 0.0);
  return PF_OK;
}

int pfe_get_ess(pf_engine_t* eng, int filter, double* out) {
  clear_err();
  int s = check_filter(eng, filter);
  if (s != PF_OK) return s;
  if (!out) return set_err(PF_EINVAL, "null out");
  if (!eng->initialized[filter]) return set_err(PF_ENOTINIT, "filter %d not initialized", filter);
  if ((s = read_ctrl(eng)) != PF_OK) return s;
  const FilterCtrl& c = eng->ctrl_host[filter];
  *out = c.lw_zero ? (double)eng->hdesc[filter].n : c.ess;
  return PF_OK;
}

int pfe_get_particles(pf_engine_t* eng, int filter, double* out_host) {
  clear_err();
  int s = check_filter(eng, filter);
  if (s != PF_OK) return s;
  if (!out_host) return set_err(PF_EINVAL, "null out");
  if (!eng->initialized[filter]) return set_err(PF_ENOTINIT, "filter %d not initialized", filter);
  const FilterDesc& d = eng->hdesc[filter];
  const int g = grid_for(eng, Q_EXPORT, d.n_tiles);
  switch (eng->D) {
    case 4: k_export<4><<<g, kThreads, 0, eng->stream>>>(eng->dev, d.tile_begin, d.n_tiles, eng->export_buf); break;
    case 5: k_export<5><<<g, kThreads, 0, eng->stream>>>(eng->dev, d.tile_begin, d.n_tiles, eng->export_buf); break;
    case 6: k_export<6><<<g, kThreads, 0, eng->stream>>>(eng->dev, d.tile_begin, d.n_tiles, eng->export_buf); break;
    default: k_export<7><<<g, kThreads, 0, eng->stream>>>(eng->dev, d.tile_begin, d.n_tiles, eng->export_buf); break;
  }
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out_host, eng->export_buf, sizeof(double) * (size_t)d.n * eng->D, cudaMemcpyDeviceToHost,
                     eng->stream));
  return sync_and_check(eng);
}

int pfe_get_anchor(pf_engine_t* eng, int filter, double anchor_ecef[3], double clk_anchor[PF_MAX_CLK],
                   float shift[8]) {
  clear_err();
  int s = check_filter(eng, filter);
  if (s != PF_OK) return s;
  if ((s = read_ctrl(eng)) != PF_OK) return s;
  const FilterCtrl& c = eng->ctrl_host[filter];
  if (anchor_ecef) memcpy(anchor_ecef, c.anchor, sizeof(double) * 3);
  if (clk_anchor) memcpy(clk_anchor, c.clk_anchor, sizeof(double) * PF_MAX_CLK);
  if (shift) memcpy(shift, c.shift, sizeof(float) * 8);
  return PF_OK;
}

int pfe_get_state_f32(pf_engine_t* eng, int filter, float* out_state, float* out_lw, int raw) {
  clear_err();
  int s = check_filter(eng, filter);
  if (s != PF_OK) return s;
  if ((s = read_ctrl(eng)) != PF_OK) return s;
  const FilterCtrl& c = eng->ctrl_host[filter];
  int n, tb, nt;
  long long base;
  filter_dims(eng, filter, &n, &base, &tb, &nt);
  const float* src = c.parity ? eng->dev.state1 : eng->dev.state0;
  const bool gather = c.resample_flag && !raw;
  std::vector<int> anc;
  if (gather) {
    anc.resize(n);
    if ((s = read_ancestors(eng, filter, anc.data())) != PF_OK) return s;
  }
  if (out_state) {
    std::vector<float> tmp(n);
    for (int dd = 0; dd < eng->D; ++dd) {
      CK(cudaMemcpy(tmp.data(), src + (size_t)dd * eng->P + base, sizeof(float) * n, cudaMemcpyDeviceToHost));
      float* o = out_state + (size_t)dd * n;
      if (gather)
        for (int k = 0; k < n; ++k) o[k] = tmp[anc[k]];
      else
        memcpy(o, tmp.data(), sizeof(float) * n);
    }
  }
  if (out_lw) {
    if (c.lw_zero && !raw)
      memset(out_lw, 0, sizeof(float) * n);
    else
      CK(cudaMemcpy(out_lw, eng->dev.lw + base, sizeof(float) * n, cudaMemcpyDeviceToHost));
  }
  return PF_OK;
}

int pfe_set_state_f32(pf_engine_t* eng, int filter, const float* state, const float* lw) {
  clear_err();
  int s = check_filter(eng, filter);
  if (s != PF_OK) return s;
  if (!state) return set_err(PF_EINVAL, "null state");
  if (!eng->initialized[filter]) return set_err(PF_ENOTINIT, "filter %d not initialized", filter);
  if ((s = read_ctrl(eng)) != PF_OK) return s;
  FilterCtrl& c = eng->ctrl_host[filter];
  int n, tb, nt;
  long long base;
  filter_dims(eng, filter, &n, &base, &tb, &nt);
  float* dst = c.parity ? eng->dev.state1 : eng->dev.state0;
  for (int dd = 0; dd < eng->D; ++dd)
    CK(cudaMemcpy(dst + (size_t)dd * eng->P + base, state + (size_t)dd * n, sizeof(float) * n,
                  cudaMemcpyHostToDevice));
  if (lw) {
    for (int k = 0; k < n; ++k)
      if (isnan(lw[k]) || lw[k] == INFINITY) return set_err(PF_EINVAL, "log-weights must be finite or -inf");
    CK(cudaMemcpy(eng->dev.lw + base, lw, sizeof(float) * n, cudaMemcpyHostToDevice));
  }
  c.resample_flag = 0;
  c.lw_zero = lw ? 0 : 1;
  for (int d = 0; d < 8; ++d) c.shift[d] = 0.f;
  CK(cudaMemcpy(eng->ctrl_dev + filter, &c, sizeof(FilterCtrl), cudaMemcpyHostToDevice));
  return PF_OK;
}

// Checkpoint of one filter: a header, the local frame fixed at initialize
// (ECEF -> E/N/U rotation), the control block and the particle arrays the
// next step reads (the current state buffer, the log-weights and the last
// resample's ancestors).  The Philox counter is the control block's
// step counter, so a restored filter draws the same numbers.
namespace {
struct CkptHeader {
  uint32_t magic;      // 'PFCK'
  uint32_t version;
  int32_t D, n;
  uint32_t key0, key1;  // the filter's Philox key (its seed)
  uint32_t ctrl_bytes, pad;
};
constexpr uint32_t kCkptMagic = 0x4b434650u;  // "PFCK" little-endian
constexpr uint32_t kCkptVersion = 1u;
size_t ckpt_bytes(const pf_engine* eng, int n) {
  return sizeof(CkptHeader) + sizeof(double) * 9 + sizeof(FilterCtrl) +
         (size_t)n * (sizeof(float) * (size_t)(eng->D + 1) + sizeof(int));
}
}  // namespace

int pfe_checkpoint_bytes(pf_engine_t* eng, int filter, size_t* bytes) {
  clear_err();
  int s = check_filter(eng, filter);
  if (s != PF_OK) return s;
  if (!bytes) return set_err(PF_EINVAL, "null bytes");
  *bytes = ckpt_bytes(eng, eng->hdesc[filter].n);
  return PF_OK;
}

int pfe_checkpoint_save(pf_engine_t* eng, int filter, void* host_buf, size_t bytes) {
  clear_err();
  int s = check_filter(eng, filter);
  if (s != PF_OK) return s;
  if (!host_buf) return set_err(PF_EINVAL, "null buffer");
  if (!eng->initialized[filter]) return set_err(PF_ENOTINIT, "filter %d not initialized", filter);
  int n, tb, nt;
  long long base;
  filter_dims(eng, filter, &n, &base, &tb, &nt);
  if (bytes < ckpt_bytes(eng, n))
    return set_err(PF_ENOMEM, "checkpoint buffer too small (%zu < %zu bytes)", bytes, ckpt_bytes(eng, n));
  if ((s = read_ctrl(eng)) != PF_OK) return s;
  const FilterCtrl& c = eng->ctrl_host[filter];
  unsigned char* o = (unsigned char*)host_buf;
  CkptHeader h{kCkptMagic, kCkptVersion, eng->D, n, eng->hdesc[filter].key0, eng->hdesc[filter].key1,
               (uint32_t)sizeof(FilterCtrl), 0u};
  memcpy(o, &h, sizeof(h));
  o += sizeof(h);
  memcpy(o, eng->hdesc[filter].rot, sizeof(double) * 9);
  o += sizeof(double) * 9;
  memcpy(o, &c, sizeof(FilterCtrl));
  o += sizeof(FilterCtrl);
  const float* src = c.parity ? eng->dev.state1 : eng->dev.state0;
  for (int dd = 0; dd < eng->D; ++dd) {
    CK(cudaMemcpy(o, src + (size_t)dd * eng->P + base, sizeof(float) * n, cudaMemcpyDeviceToHost));
    o += sizeof(float) * n;
  }
  CK(cudaMemcpy(o, eng->dev.lw + base, sizeof(float) * n, cudaMemcpyDeviceToHost));
  o += sizeof(float) * n;
  std::vector<int> anc(n);
  if ((s = read_ancestors(eng, filter, anc.data())) != PF_OK) return s;
  memcpy(o, anc.data(), sizeof(int) * n);
  return PF_OK;
}

int pfe_checkpoint_load(pf_engine_t* eng, int filter, const void* host_buf, size_t bytes) {
  clear_err();
  int s = check_filter(eng, filter);
  if (s != PF_OK) return s;
  if (!host_buf) return set_err(PF_EINVAL, "null buffer");
  int n, tb, nt;
  long long base;
  filter_dims(eng, filter, &n, &base, &tb, &nt);
  if (bytes < sizeof(CkptHeader)) return set_err(PF_EINVAL, "checkpoint too short");
  CkptHeader h;
  memcpy(&h, host_buf, sizeof(h));
  if (h.magic != kCkptMagic || h.version != kCkptVersion)
    return set_err(PF_EINVAL, "not a checkpoint of this library (magic 0x%08x, version %u)", h.magic, h.version);
  if (h.D != eng->D || h.n != n || h.ctrl_bytes != sizeof(FilterCtrl))
    return set_err(PF_EINVAL, "checkpoint of D=%d, N=%d does not fit filter %d (D=%d, N=%d)", h.D, h.n, filter,
                   eng->D, n);
  if (h.key0 != eng->hdesc[filter].key0 || h.key1 != eng->hdesc[filter].key1)
    return set_err(PF_EINVAL, "checkpoint was taken with another seed than filter %d's", filter);
  if (bytes < ckpt_bytes(eng, n)) return set_err(PF_EINVAL, "checkpoint truncated");
  if ((s = sync_and_check(eng)) != PF_OK) return s;
  const unsigned char* in = (const unsigned char*)host_buf + sizeof(h);
  FilterDesc& d = eng->hdesc[filter];
  memcpy(d.rot, in, sizeof(double) * 9);
  in += sizeof(double) * 9;
  CK(cudaMemcpy(eng->desc_dev + filter, &d, sizeof(FilterDesc), cudaMemcpyHostToDevice));
  FilterCtrl c;
  memcpy(&c, in, sizeof(FilterCtrl));
  in += sizeof(FilterCtrl);
  float* dst = c.parity ? eng->dev.state1 : eng->dev.state0;
  for (int dd = 0; dd < eng->D; ++dd) {
    CK(cudaMemcpy(dst + (size_t)dd * eng->P + base, in, sizeof(float) * n, cudaMemcpyHostToDevice));
    in += sizeof(float) * n;
  }
  CK(cudaMemcpy(eng->dev.lw + base, in, sizeof(float) * n, cudaMemcpyHostToDevice));
  in += sizeof(float) * n;
  for (int k = 0; k < n; ++k) {  // the next gather indexes the state with these
    int a;
    memcpy(&a, in + sizeof(int) * (size_t)k, sizeof(int));
    if (a < 0 || a >= n) return set_err(PF_EINVAL, "checkpoint ancestor %d of slot %d out of range [0, %d)", a, k, n);
  }
  CK(cudaMemcpy(eng->dev.anc + base, in, sizeof(int) * n, cudaMemcpyHostToDevice));
  if ((s = clear_segment_markers(eng, filter)) != PF_OK) return s;
  c.ticket = 0u;
  c.est_ticket = 0u;
  eng->ctrl_host[filter] = c;
  CK(cudaMemcpy(eng->ctrl_dev + filter, &c, sizeof(FilterCtrl), cudaMemcpyHostToDevice));
  eng->initialized[filter] = 1;
  return PF_OK;
}

int pfe_get_ancestors(pf_engine_t* eng, int filter, int* out_host) {
  clear_err();
  int s = check_filter(eng, filter);
  if (s != PF_OK) return s;
  if (!out_host) return set_err(PF_EINVAL, "null out");
  if ((s = sync_and_check(eng)) != PF_OK) return s;
  return read_ancestors(eng, filter, out_host);
}

int pfe_get_resample_info(pf_engine_t* eng, int filter, uint32_t* u32, uint64_t* wq_total, float* max_lw) {
  clear_err();
  int s = check_filter(eng, filter);
  if (s != PF_OK) return s;
  if ((s = read_ctrl(eng)) != PF_OK) return s;
  const FilterCtrl& c = eng->ctrl_host[filter];
  if (u32) *u32 = c.sys_u;
  if (wq_total) *wq_total = c.wq_total;
  if (max_lw) *max_lw = c.max_lw;
  return PF_OK;
}

int pfe_error_word(pf_engine_t* eng, unsigned* word) {
  clear_err();
  if (!eng || !word) return set_err(PF_EINVAL, "null argument");
  CK(cudaStreamSynchronize(eng->stream));
  CK(cudaMemcpy(word, eng->dev.err, sizeof(unsigned), cudaMemcpyDeviceToHost));
  return PF_OK;
}

int pfe_set_likelihood(pf_engine_t* eng, const pf_likelihood_t* lik) {
  clear_err();
  if (!eng || !lik) return set_err(PF_EINVAL, "null argument");
  if (eng->cfg.weight_mode != PF_WEIGHT_GENERIC) return set_err(PF_EINVAL, "engine is not in generic mode");
  switch (lik->type) {
    case PF_LIK_GAUSSIAN: break;
    case PF_LIK_STUDENT_T:
      if (!(lik->nu > 0.0) || !isfinite(lik->nu)) return set_err(PF_EINVAL, "Student's t needs nu > 0");
      break;
    case PF_LIK_HUBER:
      if (!(lik->huber_k > 0.0) || !isfinite(lik->huber_k)) return set_err(PF_EINVAL, "Huber needs k > 0");
      break;
    case PF_LIK_GMM:
      if (!(lik->w_los > 0.0 && lik->w_los < 1.0)) return set_err(PF_EINVAL, "GMM needs 0 < w_los < 1");
      if (!(lik->sigma_nlos > 0.0) || !isfinite(lik->sigma_nlos) || !isfinite(lik->mu_nlos))
        return set_err(PF_EINVAL, "GMM needs a finite mu_nlos and sigma_nlos > 0");
      break;
    default: return set_err(PF_EINVAL, "unknown likelihood type %d", lik->type);
  }
  if (!(lik->gate_m >= 0.0) || !isfinite(lik->gate_m)) return set_err(PF_EINVAL, "gate_m must be finite and >= 0");
  eng->dev.lk_type = lik->type;
  eng->dev.lk_nu = (float)lik->nu;
  eng->dev.lk_huber_k = (float)lik->huber_k;
  eng->dev.lk_w_los = (float)lik->w_los;
  eng->dev.lk_mu_nlos = (float)lik->mu_nlos;
  eng->dev.lk_sigma_nlos = (float)lik->sigma_nlos;
  eng->dev.lk_gate_m = (float)lik->gate_m;
  return PF_OK;
}

int pfe_shift(pf_engine_t* eng, int filter, const double dpos_ecef[3], const double* dclk) {
  clear_err();
  int s = check_filter(eng, filter);
  if (s != PF_OK) return s;
  if (!dpos_ecef) return set_err(PF_EINVAL, "null displacement");
  for (int i = 0; i < 3; ++i)
    if (!isfinite(dpos_ecef[i])) return set_err(PF_EINVAL, "displacement not finite");
  if ((s = read_ctrl(eng)) != PF_OK) return s;
  FilterCtrl c = eng->ctrl_host[filter];
  for (int i = 0; i < 3; ++i) c.anchor[i] += dpos_ecef[i];
  if (dclk)
    for (int k = 0; k < eng->cfg.n_clk; ++k) {
      if (!isfinite(dclk[k])) return set_err(PF_EINVAL, "clock shift not finite");
      c.clk_anchor[k] += dclk[k];
    }
  CK(cudaMemcpyAsync(eng->ctrl_dev + filter, &c, sizeof(c), cudaMemcpyHostToDevice, eng->stream));
  CK(cudaStreamSynchronize(eng->stream));
  eng->ctrl_host[filter] = c;
  return PF_OK;
}

int pfe_add_position_term(pf_engine_t* eng, int filter, const double* refs_ecef, const double* log_pi, int K,
                          double sigma) {
  clear_err();
  int s = check_filter(eng, filter);
  if (s != PF_OK) return s;
  if (!eng->initialized[filter]) return set_err(PF_ENOTINIT, "filter %d not initialized", filter);
  if (!refs_ecef || K < 1 || K > kMaxPosRefs) return set_err(PF_EINVAL, "need 1..%d references", kMaxPosRefs);
  if (!(sigma > 0.0) || !isfinite(sigma)) return set_err(PF_EINVAL, "sigma must be > 0");
  if ((s = read_ctrl(eng)) != PF_OK) return s;
  const FilterCtrl& c = eng->ctrl_host[filter];
  const FilterDesc& d = eng->hdesc[filter];
  PosTerm pt;
  memset(&pt, 0, sizeof(pt));
  pt.K = K;
  pt.inv_2s2 = (float)(0.5 / (sigma * sigma));
  for (int j = 0; j < K; ++j) {
    double v[3];
    for (int i = 0; i < 3; ++i) {
      if (!isfinite(refs_ecef[3 * j + i])) return set_err(PF_EINVAL, "reference not finite");
      v[i] = refs_ecef[3 * j + i] - c.anchor[i];
    }
    for (int r = 0; r < 3; ++r) pt.ref[j][r] = (float)(d.rot[3 * r] * v[0] + d.rot[3 * r + 1] * v[1] + d.rot[3 * r + 2] * v[2]);
    pt.logpi[j] = (float)(log_pi ? log_pi[j] : -log((double)K));
  }
  const int g = std::max(1, std::min(eng->sm_count * 4, (d.n + kTile - 1) / kTile));
  switch (eng->D) {
    case 4: k_position_term<4><<<g, kThreads, 0, eng->stream>>>(eng->dev, filter, pt); break;
    case 5: k_position_term<5><<<g, kThreads, 0, eng->stream>>>(eng->dev, filter, pt); break;
    case 6: k_position_term<6><<<g, kThreads, 0, eng->stream>>>(eng->dev, filter, pt); break;
    default: k_position_term<7><<<g, kThreads, 0, eng->stream>>>(eng->dev, filter, pt); break;
  }
  CK(cudaGetLastError());
  // the weights are explicit now
  const int zero = 0;
  CK(cudaMemcpyAsync(reinterpret_cast<char*>(eng->ctrl_dev + filter) + offsetof(FilterCtrl, lw_zero), &zero,
                     sizeof(int), cudaMemcpyHostToDevice, eng->stream));
  CK(cudaStreamSynchronize(eng->stream));
  return PF_OK;
}

int pfe_add_obs_term(pf_engine_t* eng, int filter, int kind, const pf_obs_row_t* rows, int n_rows, double sigma,
                     double gate, double huber_k, int accumulate) {
  clear_err();
  int s = check_filter(eng, filter);
  if (s != PF_OK) return s;
  if (!eng->initialized[filter]) return set_err(PF_ENOTINIT, "filter %d not initialized", filter);
  if (kind < PF_OBS_DD_PSEUDORANGE || kind > PF_OBS_DD_CARRIER_AFV) return set_err(PF_EINVAL, "unknown kind %d", kind);
  if (n_rows < 0 || n_rows > kMaxObsRows) return set_err(PF_ECAP, "need 0..%d rows", kMaxObsRows);
  if (n_rows > 0 && !rows) return set_err(PF_EINVAL, "null rows");
  if (!(sigma > 0.0) || !isfinite(sigma)) return set_err(PF_EINVAL, "sigma must be > 0");
  if (!(gate >= 0.0) || !isfinite(gate)) return set_err(PF_EINVAL, "gate must be finite and >= 0");
  if (kind == PF_OBS_CARRIER_AFV && gate > 0.0) return set_err(PF_EINVAL, "the undifferenced carrier term has no gate");
  if (!(huber_k >= 0.0) || !isfinite(huber_k)) return set_err(PF_EINVAL, "huber_k must be finite and >= 0");
  if ((s = read_ctrl(eng)) != PF_OK) return s;
  const FilterCtrl& c = eng->ctrl_host[filter];
  const FilterDesc& d = eng->hdesc[filter];
  std::vector<ObsRow> host((size_t)std::max(n_rows, 1));
  const bool dd = kind != PF_OBS_CARRIER_AFV;
  for (int i = 0; i < n_rows; ++i) {
    const pf_obs_row_t& r = rows[i];
    bool ok = isfinite(r.obs) && isfinite(r.weight);
    for (int j = 0; j < 3; ++j) ok = ok && isfinite(r.sat_k[j]) && (!dd || isfinite(r.sat_ref[j]));
    if (dd) ok = ok && isfinite(r.base_k) && isfinite(r.base_ref);
    if (!ok) return set_err(PF_EINVAL, "row %d not finite", i);
    const bool carrier = kind != PF_OBS_DD_PSEUDORANGE;
    if (carrier && !(r.wavelength > 0.0 && isfinite(r.wavelength)))
      return set_err(PF_EINVAL, "row %d: wavelength must be > 0", i);
    ObsRow& o = host[i];
    memset(&o, 0, sizeof(o));
    double vk[3], vr[3];
    for (int j = 0; j < 3; ++j) {
      vk[j] = r.sat_k[j] - c.anchor[j];
      vr[j] = dd ? r.sat_ref[j] - c.anchor[j] : 0.0;
    }
    for (int q = 0; q < 3; ++q) {
      o.sk[q] = d.rot[3 * q] * vk[0] + d.rot[3 * q + 1] * vk[1] + d.rot[3 * q + 2] * vk[2];
      o.sr[q] = d.rot[3 * q] * vr[0] + d.rot[3 * q + 1] * vr[1] + d.rot[3 * q + 2] * vr[2];
    }
    o.w = r.weight;
    o.inv_wl = carrier ? 1.0 / r.wavelength : 1.0;
    if (kind == PF_OBS_DD_PSEUDORANGE)
      o.c = r.obs + r.base_k - r.base_ref;
    else if (kind == PF_OBS_CARRIER_AFV)
      o.c = r.obs - c.clk_anchor[0] * o.inv_wl;
    else
      o.c = r.obs + (r.base_k - r.base_ref) * o.inv_wl;
  }
  if (n_rows == 0 && accumulate) return PF_OK;
  ObsBlock b;
  memset(&b, 0, sizeof(b));
  b.n = n_rows;
  b.kind = kind;
  b.accumulate = accumulate ? 1 : 0;
  b.gate_min = std::min(n_rows, 3);
  b.inv_sigma2 = 1.0 / (sigma * sigma);
  b.inv_sigma = 1.0 / sigma;
  b.gate = gate;
  b.huber_k = huber_k;
  if (n_rows > 0)
    CK(cudaMemcpyAsync(eng->obs_rows, host.data(), sizeof(ObsRow) * n_rows, cudaMemcpyHostToDevice, eng->stream));
  const int g = std::max(1, std::min(eng->sm_count * 4, (d.n + kTile - 1) / kTile));
  switch (eng->D) {
    case 4: k_obs_term<4><<<g, kThreads, 0, eng->stream>>>(eng->dev, filter, b, eng->obs_rows); break;
    case 5: k_obs_term<5><<<g, kThreads, 0, eng->stream>>>(eng->dev, filter, b, eng->obs_rows); break;
    case 6: k_obs_term<6><<<g, kThreads, 0, eng->stream>>>(eng->dev, filter, b, eng->obs_rows); break;
    default: k_obs_term<7><<<g, kThreads, 0, eng->stream>>>(eng->dev, filter, b, eng->obs_rows); break;
  }
  CK(cudaGetLastError());
  const int zero = 0;
  CK(cudaMemcpyAsync(reinterpret_cast<char*>(eng->ctrl_dev + filter) + offsetof(FilterCtrl, lw_zero), &zero,
                     sizeof(int), cudaMemcpyHostToDevice, eng->stream));
  CK(cudaStreamSynchronize(eng->stream));
  return PF_OK;
}

static int vel_check(pf_engine_t* eng, int filter, pf_vel_state_t* vs) {
  int s = check_filter(eng, filter);
  if (s != PF_OK) return s;
  if (!vs || !vs->buf) return set_err(PF_EINVAL, "null velocity state");
  if (vs->sel != 0 && vs->sel != 1) return set_err(PF_EINVAL, "velocity state: sel must be 0 or 1");
  if (!eng->initialized[filter]) return set_err(PF_ENOTINIT, "filter %d not initialized", filter);
  return PF_OK;
}

static int vel_grid(pf_engine_t* eng, int n, int per_thread) {
  return std::max(1, std::min(eng->sm_count * 8, (n + kThreads * per_thread - 1) / (kThreads * per_thread)));
}

int pfe_vel_init(pf_engine_t* eng, int filter, pf_vel_state_t* vs, const double v0_ecef[3], double spread_vel,
                 double init_sigma, unsigned step) {
  clear_err();
  int s = vel_check(eng, filter, vs);
  if (s != PF_OK) return s;
  if (!v0_ecef) return set_err(PF_EINVAL, "null v0");
  for (int i = 0; i < 3; ++i)
    if (!isfinite(v0_ecef[i])) return set_err(PF_EINVAL, "v0 not finite");
  if (!(spread_vel >= 0.0) || !isfinite(spread_vel) || !isfinite(init_sigma))
    return set_err(PF_EINVAL, "spread_vel must be finite and >= 0");
  if ((s = read_ctrl(eng)) != PF_OK) return s;
  const int n = eng->hdesc[filter].n;
  k_vel_init<<<vel_grid(eng, n, 1), kThreads, 0, eng->stream>>>(eng->dev, filter, vs->buf, v0_ecef[0], v0_ecef[1],
                                                                  v0_ecef[2], spread_vel, init_sigma * init_sigma, step);
  CK(cudaGetLastError());
  vs->sel = 0;
  vs->seq = eng->ctrl_host[filter].rs_seq;
  return sync_and_check(eng);
}

int pfe_vel_follow(pf_engine_t* eng, int filter, pf_vel_state_t* vs) {
  clear_err();
  int s = vel_check(eng, filter, vs);
  if (s != PF_OK) return s;
  if ((s = read_ctrl(eng)) != PF_OK) return s;
  const FilterCtrl& c = eng->ctrl_host[filter];
  if (!c.resample_flag || c.rs_seq == vs->seq) return PF_OK;
  const int n = eng->hdesc[filter].n;
  const double* in = vs->buf + (size_t)vs->sel * kVelComp * n;
  double* out = vs->buf + (size_t)(vs->sel ^ 1) * kVelComp * n;
  k_vel_gather<<<vel_grid(eng, n, 1), kThreads, 0, eng->stream>>>(eng->dev, filter, in, out);
  CK(cudaGetLastError());
  vs->sel ^= 1;
  vs->seq = c.rs_seq;
  return sync_and_check(eng);
}

int pfe_vel_predict(pf_engine_t* eng, int filter, pf_vel_state_t* vs, const double guide_ecef[3], double dt,
                    double sigma_pos, double sigma_vel, double alpha, int kf, double q, unsigned step) {
  clear_err();
  int s = pfe_vel_follow(eng, filter, vs);
  if (s != PF_OK) return s;
  if (!guide_ecef) return set_err(PF_EINVAL, "null guide velocity");
  for (int i = 0; i < 3; ++i)
    if (!isfinite(guide_ecef[i])) return set_err(PF_EINVAL, "guide velocity not finite");
  if (!isfinite(dt) || !isfinite(sigma_pos) || !isfinite(sigma_vel) || !isfinite(alpha) || !isfinite(q) ||
      sigma_pos < 0.0 || sigma_vel < 0.0)
    return set_err(PF_EINVAL, "predict parameters must be finite, sigmas >= 0");
  FilterCtrl c = eng->ctrl_host[filter];  // read by the follow above
  const FilterDesc& d = eng->hdesc[filter];
  VelPredict vp;
  memset(&vp, 0, sizeof(vp));
  for (int i = 0; i < 3; ++i) vp.guide[i] = guide_ecef[i];
  for (int i = 0; i < 9; ++i) vp.rot[i] = d.rot[i];
  vp.dt = dt;
  vp.sigma_pos = sigma_pos;
  vp.sigma_vel = sigma_vel;
  vp.alpha = alpha;
  vp.q = q;
  vp.kf = kf ? 1 : 0;
  vp.step = step;
  double* vb = vs->buf + (size_t)vs->sel * kVelComp * d.n;
  const int g = vel_grid(eng, d.n, 4);
  switch (eng->D) {
    case 4: k_vel_predict<4><<<g, kThreads, 0, eng->stream>>>(eng->dev, filter, vb, vp); break;
    case 5: k_vel_predict<5><<<g, kThreads, 0, eng->stream>>>(eng->dev, filter, vb, vp); break;
    case 6: k_vel_predict<6><<<g, kThreads, 0, eng->stream>>>(eng->dev, filter, vb, vp); break;
    default: k_vel_predict<7><<<g, kThreads, 0, eng->stream>>>(eng->dev, filter, vb, vp); break;
  }
  CK(cudaGetLastError());
  // the particles now sit, gathered, in the other buffer
  c.parity ^= 1;
  c.resample_flag = 0;
  CK(cudaMemcpyAsync(eng->ctrl_dev + filter, &c, sizeof(c), cudaMemcpyHostToDevice, eng->stream));
  CK(cudaStreamSynchronize(eng->stream));
  eng->ctrl_host[filter] = c;
  return sync_and_check(eng);
}

int pfe_vel_doppler(pf_engine_t* eng, int filter, pf_vel_state_t* vs, const pf_doppler_row_t* rows, int n_rows,
                    double wavelength, double sigma_mps, double gain, double max_update, int kf) {
  clear_err();
  int s = pfe_vel_follow(eng, filter, vs);
  if (s != PF_OK) return s;
  if (n_rows < 1 || n_rows > kMaxDopplerRows || !rows) return set_err(PF_ECAP, "need 1..%d rows", kMaxDopplerRows);
  if (!(wavelength > 0.0) || !isfinite(wavelength) || !(sigma_mps > 0.0) || !isfinite(sigma_mps) || !isfinite(gain) ||
      !isfinite(max_update))
    return set_err(PF_EINVAL, "wavelength and sigma must be > 0, gain and cap finite");
  for (int i = 0; i < n_rows; ++i) {
    bool ok = isfinite(rows[i].doppler_hz) && isfinite(rows[i].weight);
    for (int k = 0; k < 3; ++k) ok = ok && isfinite(rows[i].sat[k]) && isfinite(rows[i].sat_vel[k]);
    if (!ok) return set_err(PF_EINVAL, "row %d not finite", i);
  }
  static_assert(sizeof(DopplerRow) == sizeof(pf_doppler_row_t), "row layout");
  // the rows ride in the observation-term scratch (128 x 80 bytes)
  static_assert(sizeof(DopplerRow) * kMaxDopplerRows <= sizeof(ObsRow) * kMaxObsRows, "scratch size");
  CK(cudaMemcpyAsync(eng->obs_rows, rows, sizeof(DopplerRow) * n_rows, cudaMemcpyHostToDevice, eng->stream));
  DopplerArgs a;
  memset(&a, 0, sizeof(a));
  a.n_sat = n_rows;
  a.kf = kf ? 1 : 0;
  a.wavelength = wavelength;
  a.sigma = sigma_mps;
  a.gain = gain;
  a.max_update = max_update;
  const FilterDesc& d = eng->hdesc[filter];
  double* vb = vs->buf + (size_t)vs->sel * kVelComp * d.n;
  const DopplerRow* dr = reinterpret_cast<const DopplerRow*>(eng->obs_rows);
  const int g = vel_grid(eng, d.n, 4);
  switch (eng->D) {
    case 4: k_doppler<4><<<g, kThreads, 0, eng->stream>>>(eng->dev, filter, vb, dr, a); break;
    case 5: k_doppler<5><<<g, kThreads, 0, eng->stream>>>(eng->dev, filter, vb, dr, a); break;
    case 6: k_doppler<6><<<g, kThreads, 0, eng->stream>>>(eng->dev, filter, vb, dr, a); break;
    default: k_doppler<7><<<g, kThreads, 0, eng->stream>>>(eng->dev, filter, vb, dr, a); break;
  }
  CK(cudaGetLastError());
  const int zero = 0;
  CK(cudaMemcpyAsync(reinterpret_cast<char*>(eng->ctrl_dev + filter) + offsetof(FilterCtrl, lw_zero), &zero,
                     sizeof(int), cudaMemcpyHostToDevice, eng->stream));
  return sync_and_check(eng);
}

static int mesh_dev(const pf_mesh_t* mesh, MeshDev& m) {
  if (!mesh) return set_err(PF_EINVAL, "null mesh");
  if (mesh->n_nodes < 0 || mesh->n_tris < 0 || (mesh->n_nodes > 0 && (!mesh->nodes || !mesh->tris)))
    return set_err(PF_EINVAL, "mesh: bad node or triangle arrays");
  if (mesh->n_nodes > std::max(1, mesh->n_tris)) return set_err(PF_EINVAL, "mesh: more nodes than the builder makes");
  memset(&m, 0, sizeof(m));
  m.nodes = static_cast<const float4*>(mesh->nodes);
  m.tris = static_cast<const float4*>(mesh->tris);
  m.n_nodes = mesh->n_nodes;
  m.n_tris = mesh->n_tris;
  for (int i = 0; i < 3; ++i) m.origin[i] = mesh->origin[i];
  for (int i = 0; i < 9; ++i) m.rot[i] = mesh->rot[i];
  return PF_OK;
}

int pf_mesh_build(const double* tris_ecef, int n_tri, float* nodes_out, float* tris_out, int* n_nodes,
                  double origin[3], double rot[9]) {
  clear_err();
  if (n_tri < 0 || (n_tri > 0 && (!tris_ecef || !nodes_out || !tris_out)) || !n_nodes || !origin || !rot)
    return set_err(PF_EINVAL, "null argument");
  if (n_tri >= (1 << 28)) return set_err(PF_ECAP, "at most 2^28 - 1 triangles");
  double o[3] = {0.0, 0.0, 0.0};
  for (int i = 0; i < n_tri * 9; ++i) {
    if (!isfinite(tris_ecef[i])) return set_err(PF_EINVAL, "triangle coordinate %d not finite", i);
    o[i % 3] += tris_ecef[i];
  }
  if (n_tri > 0)
    for (int a = 0; a < 3; ++a) o[a] /= 3.0 * n_tri;
  double R[9];
  enu_rotation(o, R);
  std::vector<double> tm((size_t)n_tri * 9);
  for (int i = 0; i < n_tri * 3; ++i) {
    const double v[3] = {tris_ecef[3 * (size_t)i] - o[0], tris_ecef[3 * (size_t)i + 1] - o[1],
                         tris_ecef[3 * (size_t)i + 2] - o[2]};
    for (int r = 0; r < 3; ++r) tm[3 * (size_t)i + r] = R[3 * r] * v[0] + R[3 * r + 1] * v[1] + R[3 * r + 2] * v[2];
  }
  HostBvh h;
  build_bvh(tm, n_tri, h);
  if (h.n_nodes > std::max(1, n_tri)) return set_err(PF_ECUDA, "internal: node count above n");
  if (h.n_nodes) memcpy(nodes_out, h.nodes.data(), sizeof(float) * h.nodes.size());
  if (n_tri) memcpy(tris_out, h.tris.data(), sizeof(float) * h.tris.size());
  *n_nodes = h.n_nodes;
  for (int a = 0; a < 3; ++a) origin[a] = o[a];
  for (int a = 0; a < 9; ++a) rot[a] = R[a];
  return PF_OK;
}

int pf_mesh_los(const pf_mesh_t* mesh, const double* d_rx, const double* d_sat, int n_rx, int n_sat,
                unsigned char* d_los_out, void* stream) {
  clear_err();
  MeshDev m;
  int s = mesh_dev(mesh, m);
  if (s != PF_OK) return s;
  if (n_rx < 0 || n_sat < 0) return set_err(PF_EINVAL, "negative sizes");
  const long long total = (long long)n_rx * n_sat;
  if (total == 0) return PF_OK;
  if (!d_rx || !d_sat || !d_los_out) return set_err(PF_EINVAL, "null argument");
  int dev = 0, sms = 148;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int g = (int)std::max(1LL, std::min((long long)sms * 8, (total + kThreads - 1) / kThreads));
  k_bvh_los<<<g, kThreads, 0, (cudaStream_t)stream>>>(m, d_rx, d_sat, n_rx, n_sat, d_los_out);
  CK(cudaGetLastError());
  return PF_OK;
}

int pfe_add_3d_term(pf_engine_t* eng, int filter, const pf_mesh_t* mesh, const double* sats, int n_sat,
                    double sigma_los, double sigma_nlos, double nlos_bias, double p_blocked, double p_clear,
                    int accumulate) {
  clear_err();
  int s = check_filter(eng, filter);
  if (s != PF_OK) return s;
  if (!eng->initialized[filter]) return set_err(PF_ENOTINIT, "filter %d not initialized", filter);
  MeshDev m;
  if ((s = mesh_dev(mesh, m)) != PF_OK) return s;
  if (n_sat < 1 || n_sat > kMax3dSats || !sats) return set_err(PF_ECAP, "need 1..%d satellites", kMax3dSats);
  for (int i = 0; i < 5 * n_sat; ++i)
    if (!isfinite(sats[i])) return set_err(PF_EINVAL, "satellite value %d not finite", i);
  if (!(sigma_los > 0.0) || !(sigma_nlos > 0.0) || !isfinite(sigma_los) || !isfinite(sigma_nlos) ||
      !isfinite(nlos_bias) || !isfinite(p_blocked) || !isfinite(p_clear))
    return set_err(PF_EINVAL, "sigmas must be > 0 and all parameters finite");
  static_assert(sizeof(Sat3d) * kMax3dSats <= sizeof(ObsRow) * kMaxObsRows, "scratch size");
  CK(cudaMemcpyAsync(eng->obs_rows, sats, sizeof(Sat3d) * n_sat, cudaMemcpyHostToDevice, eng->stream));
  Weight3dArgs a;
  memset(&a, 0, sizeof(a));
  a.n_sat = n_sat;
  a.accumulate = accumulate ? 1 : 0;
  a.inv_s2_los = 1.0 / (sigma_los * sigma_los);
  a.inv_s2_nlos = 1.0 / (sigma_nlos * sigma_nlos);
  a.nlos_bias = nlos_bias;
  a.p_blocked = p_blocked;
  a.p_clear = p_clear;
  const FilterDesc& d = eng->hdesc[filter];
  const Sat3d* sv = reinterpret_cast<const Sat3d*>(eng->obs_rows);
  const int g = std::max(1, std::min(eng->sm_count * 16, (d.n + kThreads - 1) / kThreads));
  switch (eng->D) {
    case 4: k_weight_3d<4><<<g, kThreads, 0, eng->stream>>>(eng->dev, filter, m, sv, a); break;
    case 5: k_weight_3d<5><<<g, kThreads, 0, eng->stream>>>(eng->dev, filter, m, sv, a); break;
    case 6: k_weight_3d<6><<<g, kThreads, 0, eng->stream>>>(eng->dev, filter, m, sv, a); break;
    default: k_weight_3d<7><<<g, kThreads, 0, eng->stream>>>(eng->dev, filter, m, sv, a); break;
  }
  CK(cudaGetLastError());
  const int zero = 0;
  CK(cudaMemcpyAsync(reinterpret_cast<char*>(eng->ctrl_dev + filter) + offsetof(FilterCtrl, lw_zero), &zero,
                     sizeof(int), cudaMemcpyHostToDevice, eng->stream));
  return sync_and_check(eng);
}

int pfe_set_mlp(pf_engine_t* eng, const float* params) {
  clear_err();
  if (!eng || !params) return set_err(PF_EINVAL, "null argument");
  if (eng->cfg.weight_mode != PF_WEIGHT_MIXTURE) return set_err(PF_EINVAL, "engine is not in mixture mode");
  for (int i = 0; i < kMlpParams; ++i)
    if (!isfinite(params[i])) return set_err(PF_EINVAL, "network parameter %d is not finite", i);
  CK(cudaMemcpyAsync((void*)eng->dev.mlp, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice, eng->stream));
  CK(cudaStreamSynchronize(eng->stream));
  eng->mlp_set = true;
  return PF_OK;
}

int pfe_get_sat_debug(pf_engine_t* eng, int filter, float* out, int max_sats, int* n_sat) {
  clear_err();
  if (!eng || !out || !n_sat) return set_err(PF_EINVAL, "null argument");
  if (eng->cfg.weight_mode != PF_WEIGHT_MIXTURE) return set_err(PF_EINVAL, "engine is not in mixture mode");
  if (filter < 0 || filter >= eng->cfg.n_filters) return set_err(PF_EINVAL, "bad filter index");
  CK(cudaStreamSynchronize(eng->stream));
  FilterCtrl c;
  CK(cudaMemcpy(&c, eng->ctrl_dev + filter, sizeof(c), cudaMemcpyDeviceToHost));
  const unsigned ep = c.epoch == 0 ? 0 : c.epoch - 1;
  const pf_filter_epoch_t* fe_dev = reinterpret_cast<const pf_filter_epoch_t*>(
      eng->dev.obs + (size_t)(ep % (unsigned)eng->cfg.obs_slots) * eng->dev.obs_slot_bytes) + filter;
  pf_filter_epoch_t fe;
  CK(cudaMemcpy(&fe, fe_dev, sizeof(fe), cudaMemcpyDeviceToHost));
  const int ns = std::max(0, std::min(std::min(fe.n_sat, eng->cfg.max_sats), max_sats));
  CK(cudaMemcpy(out, eng->dev.sat_dbg + (size_t)filter * eng->cfg.max_sats * kSatDbg, sizeof(float) * ns * kSatDbg,
                cudaMemcpyDeviceToHost));
  *n_sat = ns;
  return PF_OK;
}

int pfe_set_spin_limit(pf_engine_t* eng, unsigned long long limit) {
  clear_err();
  if (!eng) return set_err(PF_EINVAL, "null engine");
  eng->dev.spin_limit = limit ? limit : (1ull << 24);
  return PF_OK;
}

int pfe_last_launch_count(pf_engine_t* eng, int* count) {
  clear_err();
  if (!eng || !count) return set_err(PF_EINVAL, "null argument");
  *count = eng->last_launches;
  return PF_OK;
}

// Test hook: make the next look-back wait for a tag that is never published
// (on != 0), so its bounded spin runs out and sets the error word; clears
// the error word when switched off.
int pfe_test_poison_lookback(pf_engine_t* eng, int on) {
  clear_err();
  if (!eng) return set_err(PF_EINVAL, "null engine");
  eng->dev.lookback_poison = on ? 1 : 0;
  if (!on) {
    CK(cudaStreamSynchronize(eng->stream));
    CK(cudaMemset(eng->dev.err, 0, sizeof(unsigned)));
    // timed-out barriers leave their generation and arrival count behind: start clean
    CK(cudaMemset(eng->bar, 0, sizeof(unsigned) * kBarWords));
  }
  return PF_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Internal hook for the stateless API: systematic ancestors of one FP64
// log-weight vector (maximum at *d_max on the device), with the engine's
// look-back scan and merge-path kernels.
namespace pfb {

struct SysScratch {
  FilterDesc* desc;
  FilterCtrl* ctrl;
  int* tf;
  uint32_t* offs;
  uint32_t* mp;
  unsigned long long *agg, *inc, *excl;
  unsigned* flag;
  unsigned* queue;
  size_t bytes;
};

// One layout for both the size query and the carve.
static SysScratch carve_sys_scratch(unsigned char* w, int n) {
  const int T = (n + PF_TILE - 1) / PF_TILE;
  size_t o = 0;
  auto take = [&](size_t b) {
    unsigned char* p = w + o;
    o = align_up(o + b, 256);
    return p;
  };
  SysScratch s;
  s.desc = (FilterDesc*)take(sizeof(FilterDesc));
  s.ctrl = (FilterCtrl*)take(sizeof(FilterCtrl));
  s.tf = (int*)take((size_t)T * 4);
  s.offs = (uint32_t*)take(align_up((size_t)n, 4) * 4);
  s.mp = (uint32_t*)take((size_t)T * 4);
  s.agg = (unsigned long long*)take((size_t)T * 8);
  s.inc = (unsigned long long*)take((size_t)T * 8);
  s.excl = (unsigned long long*)take((size_t)T * 8);
  s.flag = (unsigned*)take((size_t)T * 4);
  s.queue = (unsigned*)take(sizeof(unsigned) * 2 * Q_COUNT + 16);
  s.bytes = o;
  return s;
}

size_t systematic_scratch_bytes(int n) { return carve_sys_scratch(nullptr, n).bytes; }

int systematic_ancestors(const double* d_lw64, const double* d_max, int n, uint32_t u, int* d_anc,
                         void* d_scratch, cudaStream_t st) {
  const int T = (n + PF_TILE - 1) / PF_TILE;
  SysScratch sc = carve_sys_scratch((unsigned char*)d_scratch, n);
  FilterDesc* desc = sc.desc;
  FilterCtrl* ctrl = sc.ctrl;
  int* tf = sc.tf;
  uint32_t* offs = sc.offs;
  uint32_t* mp = sc.mp;
  unsigned long long* agg = sc.agg;
  unsigned long long* inc = sc.inc;
  unsigned long long* excl = sc.excl;
  unsigned* flag = sc.flag;
  unsigned* queue = sc.queue;
  unsigned* err = queue + 2 * Q_COUNT;

  FilterDesc hd;
  memset(&hd, 0, sizeof(hd));
  hd.n = n;
  hd.tile_begin = 0;
  hd.n_tiles = T;
  hd.K = quant_exponent(n);
  hd.p_off = 0;
  FilterCtrl hc;
  memset(&hc, 0, sizeof(hc));
  hc.resample_flag = 1;
  hc.rs_seq = 1;
  hc.max_lw = 0.0f;
  hc.sys_u = u;
  std::vector<int> htf(T, 0);
  CK(cudaMemcpyAsync(desc, &hd, sizeof(hd), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctrl, &hc, sizeof(hc), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(tf, htf.data(), sizeof(int) * T, cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(flag, 0, (size_t)T * 4, st));
  CK(cudaMemsetAsync(queue, 0, sizeof(unsigned) * 2 * Q_COUNT + 16, st));

  EngineDev e;
  memset(&e, 0, sizeof(e));
  e.desc = desc;
  e.ctrl = ctrl;
  e.tile_filter = tf;
  e.lw = nullptr;
  e.lw64 = d_lw64;
  e.lw64_max = d_max;
  e.anc = d_anc;
  e.offs = offs;
  e.mp_part = mp;
  e.lb_agg = agg;
  e.lb_inc = inc;
  e.lb_flag = flag;
  e.tile_excl = excl;
  e.queue = queue;
  e.err = err;
  e.spin_limit = 1ull << 24;
  e.n_filters = 1;
  e.resampler = PF_RESAMPLE_SYSTEMATIC;
  int dev = 0, sms = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  int r_scan = 0, r_offs = 0, r_merge = 0;
  int s;
  if ((s = occupancy(k_scan, sms, &r_scan)) != PF_OK) return s;
  if ((s = occupancy(k_offs, sms, &r_offs)) != PF_OK) return s;
  if ((s = occupancy(k_merge, sms, &r_merge)) != PF_OK) return s;
  k_scan<<<std::min(T, r_scan), kThreads, 0, st>>>(e, 0, T);
  k_offs<<<std::min(T, r_offs), kThreads, 0, st>>>(e, 0, T);
  k_merge<<<std::min(T, r_merge), kThreads, 0, st>>>(e, 0, T);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(st));
  unsigned hw = 0;
  CK(cudaMemcpy(&hw, err, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (hw & ERR_LOOKBACK_TIMEOUT) return set_err(PF_ETIMEOUT, "device look-back spin limit reached");
  if (hw) return set_err(PF_EINVAL, "systematic resampling: invalid weights (error word 0x%x)", hw);
  return PF_OK;
}

}  // namespace pfb
