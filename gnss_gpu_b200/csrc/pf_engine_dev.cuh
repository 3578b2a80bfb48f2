// pf_engine_dev.cuh -- device data structures of the resident engine.
#pragma once
#include <stdint.h>
#include "../../include/gnss_pf_b200.h"
#include "pf_common.cuh"

namespace pfb {

constexpr int kThreads = 256;        // threads per CTA of the tile kernels
constexpr int kPerThread = 4;        // particles per thread (one float4)
constexpr int kTile = kThreads * kPerThread;
static_assert(kTile == PF_TILE, "tile size mismatch");
constexpr int kMergeDiag = 2 * kTile;  // merge-path diagonals per tile
constexpr int kPartStride = 16;        // floats per tile partial
constexpr int kWarpTile = 32 * kPerThread;      // particles per warp segment (epoch kernel)
constexpr int kSubTiles = kTile / kWarpTile;    // warp segments per tile
constexpr int kLightRun = 128;                  // epoch kernel: longest offspring run written by one lane
constexpr int kBarCount = 4;                    // epoch kernel: arrival counter in the barrier block
constexpr int kBarWords = 8;                    // epoch kernel: words of the barrier block
constexpr int kMaxEpochGrid = 2048;             // epoch kernel: most CTAs of one launch
constexpr int kMaxD = 3 + PF_MAX_CLK;

// Work-queue slots (two words each: next tile, exit ticket).
enum QueueSlot : int {
  Q_STEP = 0, Q_SCAN = 1, Q_OFFS = 2, Q_MERGE = 3, Q_MEGO = 4,
  Q_INIT = 5, Q_EST = 6, Q_EXPORT = 7, Q_COUNT = 8
};

// Error word bits.
enum : unsigned {
  ERR_LOOKBACK_TIMEOUT = 1u, ERR_BAD_WEIGHTS = 2u, ERR_SAT_CAP = 4u, ERR_BARRIER_TIMEOUT = 8u, ERR_INTERNAL_CAP = 16u,
  ERR_BOUNDS = 32u
};

// Checked build (-DPF_CHECKED, libgnsspf_b200_checked.so): indexes that come
// from data (ancestors, offspring ends, segment markers, satellite offsets) are
// tested before use; a bad one sets ERR_BOUNDS in the error word and the
// access is skipped or clamped, so the host reports the fault as an error
// instead of the device faulting.  The release build clamps the same indexes
// silently (or relies on invariants of the layout) and never sets the bit.
#ifdef PF_CHECKED
#define PF_BOUNDS_OK(e, cond) ((cond) ? true : (atomicOr((e).err, ERR_BOUNDS), false))
#else
#define PF_BOUNDS_OK(e, cond) true
#endif

struct FilterDesc {
  int n;
  int tile_begin;
  int n_tiles;
  int K;                  // quantisation exponent (quant_exponent(n))
  long long p_off;        // element offset of particle 0, multiple of 4
  uint32_t key0, key1;    // Philox key (filter seed)
  float sigma[8];         // predict noise per state component
  float sigma_pr;
  float inv_sigma_pr;
  float wscale;           // -0.5 / sigma_pr^2
  float huber_k;
  uint32_t sys_ref_u;     // (seed % 1e6)/(1e6 N) as a 32-bit slot fraction
  int filter_id;
  double rot[9];          // ECEF -> local (rows E, N, U)
};

struct FilterCtrl {
  double anchor[3];       // ECEF origin of the stored offsets
  double clk_anchor[PF_MAX_CLK];
  double est_ecef[3];     // fused weighted mean of the last step
  double est_clk[PF_MAX_CLK];
  double cov[6];
  double ess;
  double sum_w;
  double api_est[8];      // output of the on-demand estimate kernel
  double api_m2[6];       // its weighted second moments E[x_i x_j] of the local offsets
  unsigned long long wq_total;
  float shift[8];         // pending re-centring, applied by the next predict
  float max_lw;
  uint32_t sys_u;
  uint32_t sys_u_cur;     // systematic offset of the running step (written before its first grid barrier)
  int sys_q_cur;          // the running step builds the systematic CDF (written before its first grid barrier)
  int eflags_cur;         // the running step's epoch flags and epoch (written before its first grid
  unsigned epoch_cur;     // barrier; the owner advances `epoch` meanwhile)
  unsigned epoch;
  unsigned ticket;
  unsigned est_ticket;
  unsigned rs_seq;        // resample sequence number (look-back tag)
  int resample_flag;      // resampled in the last step: next read gathers
  int lw_zero;            // log-weights read as zero
  int parity;             // which state buffer is current
  int initialized;
};

struct EngineDev {
  const FilterDesc* desc;
  FilterCtrl* ctrl;
  const int* tile_filter;
  float* state0;
  float* state1;
  float* lw;
  int* anc;
  uint32_t* offs;
  uint32_t* mp_part;
  float* part;
  unsigned long long* lb_agg;
  unsigned long long* lb_inc;
  unsigned* lb_flag;
  unsigned long long* tile_excl;
  // tiled integer CDF of the systematic resampler (written in the step's
  // first phase; every value an integer below 2^53, held exactly as a
  // double): per particle the inclusive prefix c_i of its quantised weight
  // inside its 128-particle warp segment; per segment the scale rho_s =
  // e^(wm_s - tm_t) to the tile maximum and the exclusive prefix E_s of the
  // rescaled segment sums inside the tile; per tile their sum S_t and the
  // tile maximum tm_t
  double* seg_c;
  double* seg_rho;
  double* seg_E;
  double* tile_S;
  float* tile_m;
  // Systematic resampling in the epoch kernel: one word per 128-slot
  // segment of the ancestor array (kSubTiles per tile, at the filter's
  // tile_begin), >= 0 when every slot of the segment has that ancestor (the
  // slots themselves are then not written), -1 when the slots hold theirs.
  int* seg_anc;
  int anc_seg;               // 1: readers of the ancestors consult seg_anc first
  const float* mlp;          // mixture mode: network parameters (FP32)
  int lk_type;               // generic mode: pf_likelihood_type_t and its parameters
  float lk_nu, lk_huber_k, lk_w_los, lk_mu_nlos, lk_sigma_nlos, lk_gate_m;
  float* sat_dbg;            // mixture mode: per filter and satellite, features and outputs
  unsigned* queue;
  unsigned* err;
  const unsigned char* obs;
  unsigned long long obs_slot_bytes;
  unsigned long long spin_limit;
  long long p_total;      // stride between state components
  int obs_slots;
  int n_filters;
  int max_sats;
  int resampler;
  int mego_iters;
  int lw_mode;
  int sys_offset;
  unsigned flags;
  float ess_threshold;
  int lookback_poison;    // test hook: wait for a tag nobody publishes
  const double* lw64;     // stateless API: FP64 log-weights (else null)
  const double* lw64_max; // device pointer to their maximum
};

}  // namespace pfb
