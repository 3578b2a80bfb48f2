/*
 * gnss_pf_b200.h -- C ABI of the B200 (sm_100a) GNSS particle-filter step.
 *
 * Two groups of entry points live in libgnsspf_b200.so:
 *
 *  1. The stateless host-array functions `pf_*`.  Each one replaces the
 *     function of the same name that the reference binds through pybind11
 *     (include/gnss_gpu/particle_filter.h:15-64 of rsasaki0109/gnss_gpu,
 *     bound in python/gnss_gpu/_particle_filter_bindings.cpp:10-145).  They take
 *     caller-owned FP64 host arrays in the reference's SoA layout (px, py, pz,
 *     pcb) and keep the reference's argument order and meaning.  They differ in
 *     two visible ways: they return a status code instead of throwing, and the
 *     random streams come from this library's Philox4x32-10 keyed by
 *     (seed, particle, step) instead of cuRAND's, so draws are not bit-equal to
 *     the reference's (only equal in distribution).
 *
 *  2. The device-resident engine `pfe_*`: FP32 ENU offsets about an FP64
 *     anchor, one or many independent filters advanced by fused kernels,
 *     ESS-conditional resampling decided on the device, CUDA-graph capture.
 *     The Python `ParticleFilter` drop-in (gnss_gpu_b200/particle_filter.py)
 *     runs on this group.
 *
 * Every function returns a pf_status_t; the message of the last failure on the
 * calling thread is available from pf_last_error().  No function aborts or
 * throws across the ABI.
 */
#ifndef GNSS_PF_B200_H
#define GNSS_PF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PF_ABI_VERSION 2

typedef enum {
  PF_OK = 0,
  PF_EINVAL = 1,    /* bad size, NaN/Inf input, sigma <= 0, bad enum      */
  PF_ENOTINIT = 2,  /* engine filter used before pfe_initialize            */
  PF_ECUDA = 3,     /* CUDA runtime error (message in pf_last_error)       */
  PF_ETIMEOUT = 4,  /* a bounded device spin-wait gave up                  */
  PF_ECAP = 5,      /* n_sat above the configured capacity                 */
  PF_ENOMEM = 6     /* workspace too small / host allocation failed        */
} pf_status_t;

/* Message of the last failing call on this thread ("" if none). */
const char* pf_last_error(void);
int pf_abi_version(void);

/* ------------------------------------------------------------------------
 * 1. Stateless host-array API (drop-in for the reference's _gnss_gpu_pf).
 * All arrays are host memory, FP64, length n_particles unless stated.
 * Calls are synchronous: on return the outputs are in host memory.
 * ---------------------------------------------------------------------- */

/* Replaces gnss_gpu::pf_initialize (include/gnss_gpu/particle_filter.h:15-19;
 * kernel src/particle_filter/predict.cu:7-21). */
int pf_initialize(double* px, double* py, double* pz, double* pcb,
                  double init_x, double init_y, double init_z, double init_cb,
                  double spread_pos, double spread_cb,
                  int n_particles, unsigned long long seed);

/* Replaces gnss_gpu::pf_predict (particle_filter.h:21-26; predict.cu:23-38).
 * vx, vy, vz point to one element each (the velocity broadcast to every
 * particle, predict.cu:33-37). */
int pf_predict(double* px, double* py, double* pz, double* pcb,
               const double* vx, const double* vy, const double* vz,
               double dt, double sigma_pos, double sigma_cb,
               int n_particles, unsigned long long seed, int step);

/* Replaces gnss_gpu::pf_weight (particle_filter.h:28-35; weight.cu:13-57).
 * Overwrites log_weights (weight.cu:56).  sat_ecef is [n_sat*3]. */
int pf_weight(const double* px, const double* py, const double* pz,
              const double* pcb, const double* sat_ecef,
              const double* pseudoranges, const double* weights_sat,
              double* log_weights, int n_particles, int n_sat,
              double sigma_pr);

/* Replaces gnss_gpu::pf_compute_ess (particle_filter.h:37-38;
 * weight.cu:61-160).  The reference returns the ESS; here it is written to
 * *ess_out. */
int pf_compute_ess(const double* log_weights, int n_particles,
                   double* ess_out);

/* No counterpart in the reference.  ESS of log-weights already in device
 * memory, for callers that cannot allocate device memory (real-time loops
 * that must not allocate after start-up, or applications whose device memory
 * is owned by another allocator).  d_log_weights and d_ess_out
 * are caller-owned device pointers; the work is queued on `stream` (a
 * cudaStream_t, NULL = legacy) and *d_ess_out is valid once that stream
 * reaches this point.  The function allocates nothing: its scratch is one
 * fixed device array in the library, held by every GPU that loads the
 * library until the process exits.  Limits: n_particles <=
 * PF_NOALLOC_MAX_PARTICLES (larger -> PF_ECAP); all calls share that array,
 * so calls that overlap on the GPU race and must be serialised; the first
 * call on a device looks up the array's address and should come before any
 * stream capture. */
#define PF_NOALLOC_MAX_PARTICLES (1 << 22)
int pf_compute_ess_noalloc(const double* d_log_weights, int n_particles,
                           double* d_ess_out, void* stream);

/* Replaces gnss_gpu::pf_resample_systematic (particle_filter.h:40-44;
 * resampling.cu:60-168).  Keeps the reference's offset
 * u0 = (seed % 1e6) / (1e6 * N) (resampling.cu:152) and its lower-bound
 * predicate cdf[i] < (u0 + k) / N (resampling.cu:69-77), evaluated exactly
 * on an integer CDF of quantised weights. */
int pf_resample_systematic(double* px, double* py, double* pz, double* pcb,
                           const double* log_weights, int n_particles,
                           unsigned long long seed);

/* Replaces gnss_gpu::pf_resample_megopolis (particle_filter.h:46-51;
 * resampling.cu:175-272).  Keeps the reference's chain: per iteration a
 * per-particle offset j = (k + 1 + floor(U (N-1))) mod N, acceptance against
 * the slot's own log-weight, double-buffered copy. */
int pf_resample_megopolis(double* px, double* py, double* pz, double* pcb,
                          const double* log_weights, int n_particles,
                          int n_iterations, unsigned long long seed);

/* Replaces gnss_gpu::pf_estimate (particle_filter.h:53-58;
 * weight.cu:163-220,264-328).  result is [4] = (x, y, z, cb). */
int pf_estimate(const double* px, const double* py, const double* pz,
                const double* pcb, const double* log_weights, double* result,
                int n_particles);

/* Replaces gnss_gpu::pf_get_particles (particle_filter.h:60-64;
 * weight.cu:331-368).  output is [n_particles*4] interleaved. */
int pf_get_particles(const double* px, const double* py, const double* pz,
                     const double* pcb, double* output, int n_particles);

/* ------------------------------------------------------------------------
 * 2. Device-resident engine.
 * No reference counterpart as a C ABI; it is the B200 implementation behind
 * python/gnss_gpu/particle_filter.py:10-222 (ParticleFilter) and the batched
 * many-filter step.
 * ---------------------------------------------------------------------- */

#define PF_MAX_CLK 4        /* clock states per filter (one per constellation) */
#define PF_MAX_SATS 64      /* satellites per filter per epoch                 */
#define PF_TILE 1024        /* particles per work tile                          */

typedef enum { PF_RESAMPLE_SYSTEMATIC = 0, PF_RESAMPLE_MEGOPOLIS = 1 } pf_resampler_t;
typedef enum {
  PF_WEIGHT_GAUSSIAN = 0,
  PF_WEIGHT_HUBER = 1,
  PF_WEIGHT_MIXTURE = 2, /* learned LOS/NLOS mixture (pfe_set_mlp), Huber fallback;
                            epoch-kernel path only */
  PF_WEIGHT_GENERIC = 3  /* the device filter's likelihoods (pfe_set_likelihood);
                            epoch-kernel path only */
} pf_weight_mode_t;

/* Likelihood of PF_WEIGHT_GENERIC engines (pf_device.cu:189-276,373-436). */
typedef enum {
  PF_LIK_GAUSSIAN = 0,
  PF_LIK_STUDENT_T = 1,  /* nu > 0 */
  PF_LIK_HUBER = 2,      /* huber_k > 0 */
  PF_LIK_GMM = 3         /* w_los, mu_nlos, sigma_nlos */
} pf_likelihood_type_t;

typedef struct {
  int type;              /* pf_likelihood_type_t                              */
  int pad_;
  double nu;             /* Student's t degrees of freedom                    */
  double huber_k;        /* Huber threshold in sigmas                         */
  double w_los;          /* GMM: weight of the LOS component, in (0, 1)       */
  double mu_nlos;        /* GMM: mean of the NLOS component, m                */
  double sigma_nlos;     /* GMM: std of the NLOS component, m                 */
  double gate_m;         /* > 0: per-particle NLOS gate on |residual|, m      */
} pf_likelihood_t;

/* Differenced and carrier-phase observation terms (pfe_add_obs_term). */
typedef enum {
  PF_OBS_DD_PSEUDORANGE = 0,  /* pf_device.cu:282-368 (m)                    */
  PF_OBS_CARRIER_AFV = 1,     /* pf_device.cu:439-494 (cycles; uses clock 0)  */
  PF_OBS_DD_CARRIER_AFV = 2   /* pf_device.cu:496-604 (cycles)                */
} pf_obs_kind_t;

typedef struct {
  double sat_k[3];    /* ECEF m: the satellite, or satellite k of a DD pair     */
  double sat_ref[3];  /* ECEF m: the pair's reference satellite (DD kinds)      */
  double obs;         /* DD pseudorange (m) / carrier phase / DD carrier (cycles) */
  double base_k;      /* base-station range to sat_k, m (DD kinds)              */
  double base_ref;    /* base-station range to sat_ref, m (DD kinds)            */
  double weight;      /* row weight                                             */
  double wavelength;  /* m (carrier kinds)                                      */
} pf_obs_row_t;
#define PF_MAX_OBS_ROWS 128

/* Per-particle velocity states (pfe_vel_*): caller-owned device memory of
 * 2 x 12 x n doubles (n = the filter's particles): two buffers, component c
 * of particle j at buf[c * n + j] with c = 0..2 the ECEF velocity (m/s) and
 * 3..11 its 3x3 covariance row-major.  `sel` is the buffer holding the
 * current states and `seq` the resample already followed; both are kept by
 * the calls (initialise by pfe_vel_init). */
typedef struct {
  double* buf;
  int sel;
  unsigned seq;
} pf_vel_state_t;

/* One Doppler observation (pfe_vel_doppler). */
typedef struct {
  double sat[3];      /* satellite ECEF position, m      */
  double sat_vel[3];  /* satellite ECEF velocity, m/s    */
  double doppler_hz;  /* range rate = -doppler * lambda  */
  double weight;
} pf_doppler_row_t;
#define PF_MAX_DOPPLER_ROWS 64

/* A triangle mesh with its bounding-volume hierarchy on the device
 * (pf_mesh_build fills the host side; the caller copies nodes and tris to
 * device memory and sets the pointers).  nodes: n_nodes x 16 floats (each
 * the boxes of two children); tris: n_tris x 12 floats; coordinates in the mesh frame: East/North/Up at
 * `origin` (ECEF, m), rot the ECEF -> mesh rotation (rows E, N, U). */
typedef struct {
  const void* nodes;
  const void* tris;
  int n_nodes;
  int n_tris;
  double origin[3];
  double rot[9];
} pf_mesh_t;

typedef enum { PF_LW_OVERWRITE = 0, PF_LW_ACCUMULATE = 1 } pf_lw_mode_t;
typedef enum {
  PF_SYS_OFFSET_RANDOM = 0,    /* Philox draw per filter and epoch            */
  PF_SYS_OFFSET_REFERENCE = 1  /* (seed % 1e6) / (1e6 N), resampling.cu:152  */
} pf_sys_offset_t;

/* Engine flags. */
#define PF_FLAG_COVARIANCE 1u  /* fused 3x3 position covariance in the step   */
#define PF_FLAG_RECENTER 2u    /* re-anchor each filter at its weighted mean  */
#define PF_FLAG_KERNEL_CHAIN 4u /* one kernel per phase instead of the single
                                   cooperative epoch kernel (comparison path) */

typedef struct {
  int n_filters;
  int n_clk;             /* 1..PF_MAX_CLK; state dimension D = 3 + n_clk     */
  int resampler;         /* pf_resampler_t                                    */
  int megopolis_iters;   /* iterations of the Megopolis chain                 */
  int weight_mode;       /* pf_weight_mode_t                                  */
  int lw_mode;           /* pf_lw_mode_t                                      */
  int sys_offset;        /* pf_sys_offset_t                                   */
  int max_sats;          /* capacity per filter per epoch, <= PF_MAX_SATS    */
  int obs_slots;         /* resident epoch-input blocks (ring)                */
  unsigned flags;        /* PF_FLAG_*                                         */
  double ess_threshold;  /* resample when ESS < threshold * N                 */
  double huber_k;        /* Huber threshold in sigmas (PF_WEIGHT_HUBER)       */
} pf_engine_config_t;

typedef struct {
  int n_particles;
  int pad_;
  unsigned long long seed;
  double sigma_pos[3];   /* predict noise per local axis (E, N, U), m         */
  double sigma_clk;      /* predict noise of every clock state, m             */
  double sigma_pr;       /* pseudorange sigma of the likelihood, m            */
} pf_filter_params_t;

/* Per-filter, per-epoch input record. */
#define PF_EP_PREDICT 1        /* apply displacement + noise               */
#define PF_EP_WEIGHT 2         /* evaluate the likelihood (else keep lw)   */
#define PF_EP_FORCE_RESAMPLE 4 /* resample regardless of ESS               */
#define PF_EP_NO_RESAMPLE 8    /* never resample this epoch                */
#define PF_EP_RESAMPLE_CHECK 16 /* without PF_EP_WEIGHT: still test the ESS of
                                   the current weights and resample if needed */
typedef struct {
  double disp[3];        /* displacement in the filter's local E/N/U frame, m */
  int n_sat;
  int sat_offset;        /* index of the first pf_sat_t of this filter        */
  int flags;             /* PF_EP_*                                           */
  int pad_;
} pf_filter_epoch_t;

typedef struct {
  double x, y, z;        /* satellite ECEF, m                                 */
  double pr;             /* pseudorange, m                                    */
  double w;              /* per-satellite weight (1/sigma^2 scale), >= 0      */
  int clk;               /* clock state index, 0..n_clk-1                     */
  float cn0;             /* C/N0, dB-Hz (PF_WEIGHT_MIXTURE features)          */
  float blocked;         /* 1 if a ray trace at the prior mean says NLOS, else 0 */
  int pad_;
} pf_sat_t;

typedef struct {
  double est_ecef[3];    /* fused weighted mean (pre-resample), ECEF          */
  double est_clk[PF_MAX_CLK];
  double cov_enu[6];     /* xx, xy, xz, yy, yz, zz of the local frame         */
  double ess;
  double sum_w;          /* sum of exp(lw - max_lw)                           */
  float max_lw;
  int resampled;         /* resampling ran in the last epoch                  */
  unsigned epoch;        /* completed steps of this filter                    */
  int initialized;
} pf_filter_result_t;

typedef struct pf_engine pf_engine_t;

/* Bytes of device workspace pfe_create needs for this configuration. */
int pfe_workspace_bytes(const pf_engine_config_t* cfg,
                        const pf_filter_params_t* filters, size_t* bytes);

/* Create an engine on the current CUDA device.  dev_workspace is caller-owned
 * device memory of at least pfe_workspace_bytes (e.g. a torch uint8 tensor);
 * it must outlive the engine.  stream is a cudaStream_t (NULL = legacy). */
int pfe_create(const pf_engine_config_t* cfg,
               const pf_filter_params_t* filters, void* dev_workspace,
               size_t workspace_bytes, void* stream, pf_engine_t** out);
int pfe_destroy(pf_engine_t* eng);
int pfe_set_stream(pf_engine_t* eng, void* stream);
/* Tuning knob of the cooperative epoch kernel: launch at most ctas_per_sm
 * CTAs per SM (0 = every CTA that fits, the default).  *resident_per_sm
 * (optional) receives how many fit.  No counterpart in the reference. */
int pfe_set_epoch_ctas_per_sm(pf_engine_t* eng, int ctas_per_sm, int* resident_per_sm);
int pfe_set_filter_params(pf_engine_t* eng, int filter,
                          const pf_filter_params_t* params);

/* Scatter N(0, spread) offsets about anchor_ecef / clk0 (n_clk values). */
int pfe_initialize(pf_engine_t* eng, int filter, const double anchor_ecef[3],
                   const double* clk0, double spread_pos, double spread_clk);

/* ECEF -> local frame rotation of a filter (row-major 3x3, rows E, N, U). */
int pfe_get_frame(pf_engine_t* eng, int filter, double rot[9],
                  double anchor_ecef[3]);

/* Copy one epoch's inputs (n_filters records + sats) from host memory into
 * resident ring slot `slot` (async on the engine stream; the host buffers
 * are staged, so they may be reused on return). */
int pfe_upload_obs(pf_engine_t* eng, int slot, const pf_filter_epoch_t* fe,
                   const pf_sat_t* sats, int n_sats_total);
/* Bytes of one resident input slot. */
int pfe_obs_slot_bytes(pf_engine_t* eng, size_t* bytes);

/* One epoch for every filter: fused predict+weight+estimate, then the
 * configured resampler where the device decided to resample.  The input
 * block is ring slot (epoch % obs_slots). */
int pfe_step(pf_engine_t* eng);
/* The same kernels launched once per filter (comparison path). */
int pfe_step_per_filter(pf_engine_t* eng);
/* One epoch from host memory to host memory, the call of a real-time
 * caller: pfe_upload_obs into slot 0, pfe_step, pfe_read_results into
 * out[n_filters] (synchronises).  Needs obs_slots == 1. */
int pfe_step_io(pf_engine_t* eng, const pf_filter_epoch_t* fe, const pf_sat_t* sats, int n_sats_total,
                pf_filter_result_t* out);

/* Capture one epoch (pfe_step, or pfe_step_per_filter if per_filter != 0)
 * into a CUDA graph; pfe_graph_launch replays it n_epochs times. */
int pfe_graph_capture(pf_engine_t* eng, int per_filter);
int pfe_graph_launch(pf_engine_t* eng, int n_epochs);

/* Copy per-filter results to host (synchronises the engine stream). */
int pfe_read_results(pf_engine_t* eng, pf_filter_result_t* out);
/* Bytes pfe_read_results copies from the device. */
int pfe_result_bytes(pf_engine_t* eng, size_t* bytes);

/* Weighted mean over the current particle set with the current log-weights
 * (zero after a resample), as the reference's pf_estimate.  out is
 * [3 + n_clk] in ECEF / m.  Synchronous. */
int pfe_estimate(pf_engine_t* eng, int filter, double* out);
/* ESS of the log-weights of the last step (N after a resample): no kernel,
 * one control-block read.  Synchronous. */
int pfe_get_ess(pf_engine_t* eng, int filter, double* out);
/* ESS of the current log-weights, recomputed on the device (one estimate
 * pass): also right after pfe_add_position_term / pfe_set_state_f32
 * (pf_device.cu:1722 pf_device_ess).  Synchronous. */
int pfe_current_ess(pf_engine_t* eng, int filter, double* out);
/* Weighted RMS distance (m) of the current particles from center_ecef (null:
 * from their weighted mean), from one device pass over the particles
 * (pf_device.cu:1764 pf_device_position_spread).  Synchronous. */
int pfe_position_spread(pf_engine_t* eng, int filter, const double* center_ecef, double* out);
/* Export particles as FP64 ECEF rows [N][3 + n_clk] into host memory. */
int pfe_get_particles(pf_engine_t* eng, int filter, double* out_host);
/* Local-frame FP32 state [D][N] and FP32 log-weights of a filter.
 * raw == 0: the current particle set (gathered through the last resample's
 * ancestors) and the current log-weights (zeros after a resample).
 * raw != 0: the state buffer and log-weight array exactly as the last step
 * wrote them (before the resample gather). */
int pfe_get_state_f32(pf_engine_t* eng, int filter, float* out_host_DxN,
                      float* out_lw_host, int raw);
/* Committed anchor (ECEF), clock anchors [PF_MAX_CLK] and the pending
 * re-centring shift [8] that the next step subtracts. */
int pfe_get_anchor(pf_engine_t* eng, int filter, double anchor_ecef[3],
                   double clk_anchor[PF_MAX_CLK], float shift[8]);
/* Replace a filter's state: offsets [D][N] (FP32, local frame about the
 * committed anchor; the pending shift is cleared), lw (may be NULL = zeros;
 * finite or -inf, PF_EINVAL for NaN / +inf).  Used for checkpoint/restore,
 * ParticleFilterDevice.set_particle_states / set_log_weights and tests. */
int pfe_set_state_f32(pf_engine_t* eng, int filter, const float* state_DxN,
                      const float* lw_or_null);
/* Checkpoint and resume of one filter.  The checkpoint holds the filter's
 * local frame (the ECEF -> E/N/U rotation fixed at pfe_initialize), its
 * control block (FP64 anchor and clock anchors, pending re-centring shift,
 * the step counter that keys the Philox draws, state-buffer parity,
 * resample and log-weight flags, systematic offset, last estimate) and the
 * particle arrays the next step reads: the current FP32 offsets [D][N], the
 * log-weights [N] and the last resample's ancestors [N].  Loading it into a
 * filter of an engine created with the same configuration, particle count
 * and seed continues the filter bit for bit.  Replaces, for one filter, the
 * reference's pf_device_get/set_particle_states and get/set_log_weights
 * (include/gnss_gpu/pf_device.h:211-222), which carry the particles and
 * weights but not the anchor or the random-number position.
 * pfe_checkpoint_bytes gives the buffer size; save returns PF_ENOMEM for a
 * smaller buffer, PF_ENOTINIT for a filter never initialized; load returns
 * PF_EINVAL for a foreign, truncated or mismatched (D, N, seed) buffer or
 * an ancestor outside [0, N).
 * Velocity states, observation terms and the network of the learned
 * likelihood are not part of it. */
int pfe_checkpoint_bytes(pf_engine_t* eng, int filter, size_t* bytes);
int pfe_checkpoint_save(pf_engine_t* eng, int filter, void* host_buf, size_t bytes);
int pfe_checkpoint_load(pf_engine_t* eng, int filter, const void* host_buf, size_t bytes);
/* Ancestor indices written by the last resample (host copy, N ints). */
int pfe_get_ancestors(pf_engine_t* eng, int filter, int* out_host);
/* Systematic offset (u32 fraction of a slot) and quantised weight total
 * used by the last systematic resample. */
int pfe_get_resample_info(pf_engine_t* eng, int filter, uint32_t* u32,
                          uint64_t* wq_total, float* max_lw);
/* Test hook: make the library's nth next host or device allocation fail
 * (pinned staging of pfe_create, the stateless functions' workspace) as if
 * memory were exhausted: the call returns PF_ENOMEM, frees what it had
 * allocated, and later calls work again.  0 switches it off.  The
 * reference has no counterpart (its CUDA_CHECK throws on any CUDA error). */
int pf_test_fail_alloc(int nth);
/* Device error word (0 = fine); non-zero after a bounded spin gave up. */
int pfe_error_word(pf_engine_t* eng, unsigned* word);
/* Test hook: spin limit of the decoupled look-back (0 = default). */
int pfe_set_spin_limit(pf_engine_t* eng, unsigned long long limit);
/* Test hook: on != 0 makes the device waits (the look-back of the kernel
 * chain, the grid barriers of the epoch kernel) wait for a value that is
 * never published, so their bounded spins run out and set the error word
 * (no hang); on == 0 restores normal operation and clears the error word
 * and the barrier state. */
int pfe_test_poison_lookback(pf_engine_t* eng, int on);
/* Kernels launched by the last pfe_step / pfe_step_per_filter. */
int pfe_last_launch_count(pf_engine_t* eng, int* count);

/* Device timing of eager steps: with slots > 0, each pfe_step records CUDA
 * events on the engine stream before the fused step kernel, after it, and
 * after the last resampling kernel, into a ring of `slots` entries
 * (slots == 0 switches timing off).  detailed != 0 also records an event
 * after every resampling kernel; that serialises the kernels (no
 * programmatic overlap), so use it for breakdowns, not for throughput.
 * pfe_read_timing synchronises and returns, for the steps since the last
 * read (at most `slots`), the fused step kernel's duration and the whole
 * step's duration in milliseconds. */
int pfe_enable_timing(pf_engine_t* eng, int slots, int detailed);
int pfe_read_timing(pf_engine_t* eng, float* step_kernel_ms, float* whole_step_ms,
                    int max_entries, int* count);
/* Per-kernel durations (ms) of the steps returned by the last
 * pfe_read_timing: 4 per step -- fused step kernel, then the three
 * resampling kernels (look-back scan, offspring ends, merge path; for
 * Megopolis the chain kernel then two zeros).  Without detailed timing the
 * second entry holds all resampling kernels together and the rest are 0. */
int pfe_read_timing_kernels(pf_engine_t* eng, float* out_4_per_step,
                            int max_entries, int* count);

/* Likelihood of a PF_WEIGHT_GENERIC engine for the following steps. */
int pfe_set_likelihood(pf_engine_t* eng, const pf_likelihood_t* lik);
/* Moves every particle of filter f by dpos_ecef (m) and its clock states by
 * dclk[0..n_clk-1] (m; may be null): an O(1) change of the filter's anchor
 * (pf_device.cu:902-921). */
int pfe_shift(pf_engine_t* eng, int filter, const double dpos_ecef[3], const double* dclk);
/* Adds to the log-weights of filter f the position term
 *   log sum_j pi_j exp(-|p - ref_j|^2 / (2 sigma^2))   (1 <= K <= 64
 * references; log_pi may be null for equal pi_j = 1/K, and entries of -inf
 * drop a reference; K = 1 is
 * pf_device.cu:889-900) over the current particles (gathered through the
 * last resample, if any).  The filter's statistics (estimate, ESS) follow at
 * its next step; a step with flags PF_EP_RESAMPLE_CHECK (or 0) and no
 * satellites recomputes them and resamples if needed. */
int pfe_add_position_term(pf_engine_t* eng, int filter, const double* refs_ecef, const double* log_pi,
                          int K, double sigma);
/* One pass over filter f's current particles (gathered through the last
 * resample, if any) evaluating n_rows (0..PF_MAX_OBS_ROWS) observation rows
 * of one kind in FP64: per row -w r^2 / (2 sigma^2), or with huber_k > 0
 * the Huber cost -w rho_k(|r| / sigma); for the DD kinds gate > 0 drops rows
 * with |r| > gate unless fewer than min(n_rows, 3) would remain (gate must
 * be 0 for PF_OBS_CARRIER_AFV).  accumulate != 0 adds the sum to the
 * current log-weights (the reference's carrier kernels), 0 overwrites them
 * (its DD pseudorange kernel).  Statistics follow as for
 * pfe_add_position_term. */
int pfe_add_obs_term(pf_engine_t* eng, int filter, int kind, const pf_obs_row_t* rows, int n_rows,
                     double sigma, double gate, double huber_k, int accumulate);

/* Velocity states of filter f (pf_device.cu:67-100): v = v0 (+ spread_vel
 * N(0, 1) per axis when > 0), covariance init_sigma^2 I, in buffer 0.
 * `step` keys the random draws. */
int pfe_vel_init(pf_engine_t* eng, int filter, pf_vel_state_t* vs, const double v0_ecef[3], double spread_vel,
                 double init_sigma, unsigned step);
/* Follows the filter's last resample (gathers the states through its
 * ancestors) unless already followed.  Call after every step that may
 * resample, before the next one. */
int pfe_vel_follow(pf_engine_t* eng, int filter, pf_vel_state_t* vs);
/* Velocity predict (pf_device.cu:106-187): v = (1 - alpha) v + alpha guide
 * (+ sigma_vel noise unless kf), positions += v dt + noise, the noise
 * N(0, sigma_pos^2 I + dt^2 P_v) when kf != 0 (and P_v += q dt I), else
 * N(0, sigma_pos^2 I).  Clocks are not moved: the next pfe_step (flags
 * PF_EP_PREDICT, zero displacement) adds their noise.  Follows a pending
 * resample first; materialises the particles' gather. */
int pfe_vel_predict(pf_engine_t* eng, int filter, pf_vel_state_t* vs, const double guide_ecef[3], double dt,
                    double sigma_pos, double sigma_vel, double alpha, int kf, double q, unsigned step);
/* Doppler likelihood over the current particles and their velocities,
 * added to the log-weights: kf == 0 is pf_device.cu:610-748 (clock drift
 * per particle, then a blend of gain toward the particle's WLS velocity,
 * capped at max_update m/s when > 0); kf != 0 is pf_device.cu:750-887
 * (sequential velocity Kalman update, innovation likelihood).  1..64 rows. */
int pfe_vel_doppler(pf_engine_t* eng, int filter, pf_vel_state_t* vs, const pf_doppler_row_t* rows, int n_rows,
                    double wavelength, double sigma_mps, double gain, double max_update, int kf);

/* Builds the hierarchy of n_tri triangles (ECEF, m; n_tri x 9 doubles:
 * v0, v1, v2; fewer than 2^28) into host arrays: nodes_out (capacity
 * max(1, n_tri) x 16 floats),
 * tris_out (n_tri x 12 floats), the node count, the mesh frame's origin and
 * rotation (python/gnss_gpu/bvh.py BVHAccelerator, src/raytrace/bvh.cu). */
int pf_mesh_build(const double* tris_ecef, int n_tri, float* nodes_out, float* tris_out, int* n_nodes,
                  double origin[3], double rot[9]);
/* Stateless building-aware likelihood of FP64 host particle arrays, the
 * reference's _gnss_gpu_pf3d.pf_weight_3d (weight_3d.cu:182-253; px..pcb
 * n_particles each, sat_ecef n_sat x 3, triangles n_tri x 9 ECEF):
 * log_weights[i] = sum over satellites of the LOS/NLOS mixture term. */
int pf_weight_3d(const double* px, const double* py, const double* pz, const double* pcb, const double* sat_ecef,
                 const double* pseudoranges, const double* weights_sat, const double* triangles, int n_tri,
                 double* log_weights, int n_particles, int n_sat, double sigma_los, double sigma_nlos,
                 double nlos_bias, double blocked_nlos_prob, double clear_nlos_prob);
/* Line of sight of n_rx x n_sat rays, receiver rx[i] (device, n_rx x 3
 * doubles) to satellite sat[i][s] (device, n_rx x n_sat x 3 doubles):
 * los_out (device, n_rx x n_sat bytes) 1 when clear, 0 when blocked or not
 * finite.  Asynchronous on `stream` (BVHAccelerator.check_los_batch). */
int pf_mesh_los(const pf_mesh_t* mesh, const double* d_rx, const double* d_sat, int n_rx, int n_sat,
                unsigned char* d_los_out, void* stream);
/* Building-aware pseudorange likelihood over filter f's current particles
 * (weight_3d.cu:86-177, weight_3d_bvh.cu): per satellite (sats: n_sat x 5
 * doubles x, y, z, pseudorange, weight; 1..64) a ray through the mesh;
 * blocked rays use the NLOS prior p_blocked, clear ones p_clear, in the
 * mixture of N(r; 0, sigma_los) and N(r'; 0, sigma_nlos) with r' = r -
 * nlos_bias for r > 0.  accumulate != 0 adds to the log-weights, 0
 * overwrites them (the reference).  Statistics follow as for
 * pfe_add_position_term. */
int pfe_add_3d_term(pf_engine_t* eng, int filter, const pf_mesh_t* mesh, const double* sats, int n_sat,
                    double sigma_los, double sigma_nlos, double nlos_bias, double p_blocked, double p_clear,
                    int accumulate);

/* Network parameters of PF_WEIGHT_MIXTURE (host array of
 * pf_mlp_param_count() floats, copied to the engine).  Required before the
 * first step of a mixture engine. */
int pfe_set_mlp(pf_engine_t* eng, const float* params);
/* Per satellite of filter f's last weighted epoch (in upload order), 16
 * floats: the 12 network features, p_nlos, mu, likelihood mode (0 mixture,
 * 1 Huber fallback, 2 unused) and the residual against the prior mean.
 * *n_sat receives the satellite count.  Mixture engines only. */
int pfe_get_sat_debug(pf_engine_t* eng, int filter, float* out, int max_sats, int* n_sat);

/* ------------------------------------------------------------------------
 * Learned NLOS likelihood: a per-satellite network 12 -> 64 -> 64 -> 2
 * (ReLU; BF16 operands, FP32 accumulation on the tensor cores) giving the
 * NLOS probability p = sigmoid(o0) and the NLOS bias mean mu = 20 m *
 * softplus(o1).  No counterpart in the reference (its mixture likelihood,
 * pf_device.cu:373-436, takes fixed mixture parameters).  Parameters are an
 * FP32 array of pf_mlp_param_count() floats:
 *   W1t[64][16] b1[64] W2t[64][64] b2[64] W3t[2][64] b3[2]  (Wt[out][in]).
 * Inputs are n rows of 12 FP32 features; labels n rows of (nlos in {0,1},
 * bias in m).  Every pointer is device memory; calls are asynchronous on
 * `stream`.  Loss: mean over rows of BCE(p, nlos) + nlos ((mu - bias)/20)^2.
 */
int pf_mlp_param_count(void);
size_t pf_mlp_scratch_bytes(void);
/* Gradient of the mean loss (d_grad, param_count floats) and the loss. */
int pf_mlp_grad(const float* d_x, const float* d_y, int n, const float* d_params,
                float* d_grad, float* d_loss, void* d_scratch, size_t scratch_bytes,
                void* stream);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8, step >= 1) on d_params with
 * moments d_m, d_v over the batch. */
int pf_mlp_adam_step(const float* d_x, const float* d_y, int n, float* d_params,
                     float* d_m, float* d_v, int step, float lr, float* d_loss,
                     void* d_scratch, size_t scratch_bytes, void* stream);
/* (p_nlos, mu) per row into d_out (2 floats per row). */
int pf_mlp_forward(const float* d_x, int n, const float* d_params, float* d_out,
                   void* stream);

/* ------------------------------------------------------------------------
 * Input formation: satellite positions and clocks from broadcast records,
 * and the Sagnac-corrected geometric range.
 * ---------------------------------------------------------------------- */

/* Kepler broadcast record in the reference's EphemerisParams layout
 * (include/gnss_gpu/ephemeris.h:6-29; 21 doubles, int week, 176 bytes, as
 * packed by python/gnss_gpu/ephemeris.py:135-171).  toe / toc are seconds
 * of week of the record's own time scale; tgd is the group delay the clock
 * correction subtracts. */
typedef struct {
  double sqrt_a, e, i0, omega0, omega, M0, delta_n, omega_dot, idot;
  double cuc, cus, crc, crs, cic, cis;
  double toe, af0, af1, af2, toc, tgd;
  int week;
  int pad_;
} pf_ephemeris_t;

/* GLONASS broadcast state (python/gnss_gpu/orbit_glonass.py:38-62): toe in
 * seconds of week of the UTC-aligned scale, PZ-90 ECEF position (m),
 * velocity (m/s), luni-solar acceleration (m/s^2), clock bias tau_n (s) and
 * relative frequency bias gamma_n; clock = -tau_n + gamma_n (t - toe). */
typedef struct {
  double toe;
  double pos[3], vel[3], acc[3];
  double tau_n, gamma_n;
} pf_glonass_state_t;

/* One broadcast record of any system: system is the RINEX letter ('G', 'E',
 * 'J', 'C' use the Kepler orbit with that system's constants and time scale
 * (ephemeris.py:36-64; BeiDou receive time is GPST - 14 s), 'R' the GLONASS
 * integrator (GPST - 18 s); other letters use the GPS constants). */
typedef struct {
  int system;
  int pad_;
  union {
    pf_ephemeris_t kepler;
    pf_glonass_state_t glonass;
  } u;
} pf_broadcast_t;

/* Replaces gnss_gpu::compute_satellite_position (include/gnss_gpu/
 * ephemeris.h:31-36; src/ephemeris/ephemeris.cu:24-104,186-212): GPS
 * constants, host arrays: params[n_sat], sat_pos[n_sat*3], sat_clk[n_sat]. */
int pf_sat_positions(const pf_ephemeris_t* params, double gps_time, double* sat_pos, double* sat_clk,
                     int n_sat);
/* Replaces gnss_gpu::compute_satellite_position_batch (ephemeris.h:38-46;
 * ephemeris.cu:106-180,214-246): the same records at n_epoch times,
 * sat_pos[n_epoch*n_sat*3], sat_clk[n_epoch*n_sat]. */
int pf_sat_positions_batch(const pf_ephemeris_t* params, const double* gps_times, double* sat_pos,
                           double* sat_clk, int n_epoch, int n_sat);
/* Multi-system batch in one launch, all pointers device memory, asynchronous
 * on `stream`: output [e][s] comes from d_recs[d_rec_index[e*n_sat+s]] (from
 * d_recs[s] when d_rec_index is NULL; an index outside [0, n_recs) gives NaN)
 * at GPST second of week d_times[e].  d_pos (n_epoch*n_sat*3) or d_clk
 * (n_epoch*n_sat) may be NULL.  glo_step is the GLONASS RK4 step in seconds
 * (<= 0: 60 s, the reference's default, orbit_glonass.py:36).  Each call
 * takes up to 64 MB of scratch (the shared GLONASS states) from the
 * library's own stream-ordered memory pool on the current device; the pool
 * keeps that memory until the process exits. */
int pf_broadcast_orbits(const pf_broadcast_t* d_recs, int n_recs, const int* d_rec_index, const double* d_times,
                        int n_epoch, int n_sat, double glo_step, double* d_pos, double* d_clk, void* stream);
/* Sagnac rotation and geometric range (python/gnss_gpu/range_model.py:12-40)
 * for receivers d_rx (n_epoch*3) and satellites d_sat (n_epoch*n_sat*3),
 * device memory, asynchronous on `stream`: d_sat_rot (n_epoch*n_sat*3) and
 * d_range (n_epoch*n_sat), either may be NULL. */
int pf_sagnac(const double* d_rx, const double* d_sat, int n_epoch, int n_sat, double* d_sat_rot,
              double* d_range, void* stream);

/* Replaces gnss_gpu::ecef_to_lla (src/utils/coordinates.cu:29-51): WGS84
 * latitude / longitude (rad) and height (m) of n ECEF points, host arrays,
 * Bowring's closed form.  Used by the NMEA writer (ecef_to_nmea). */
int pf_ecef_to_lla(const double* ecef_x, const double* ecef_y, const double* ecef_z, double* lat, double* lon,
                   double* alt, int n);

/* Line of sight through a box city (the learned likelihood's simulator
 * cities: an n x n grid of cells of side `cell`, at most one axis-aligned
 * box per cell; no counterpart in the reference, whose 3D path uses meshes).
 * Device arrays: d_occ [n*n] (cell (ix, iy) at ix*n + iy), d_box [n*n*4]
 * (x0, x1, y0, y1 in the city's local E/N, m), d_height [n*n]; rays from
 * d_p [n_ray*3] (local E/N/U) along unit directions d_dir [n_ray*3] with
 * positive up component; at most `steps` cells per ray; d_blocked [n_ray]
 * 1 when a building is hit.  Asynchronous on `stream`. */
int pf_city_los(const unsigned char* d_occ, const double* d_box, const double* d_height, int n, double cell,
                double hmax, int steps, const double* d_p, const double* d_dir, int n_ray, unsigned char* d_blocked,
                void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GNSS_PF_B200_H */
