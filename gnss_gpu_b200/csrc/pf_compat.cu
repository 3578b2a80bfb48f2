// pf_compat.cu -- the stateless host-array API (pf_*), one function per
// entry of the reference's _gnss_gpu_pf module
// (python/gnss_gpu/_particle_filter_bindings.cpp:10-145 ->
//  include/gnss_gpu/particle_filter.h:15-64).
//
// Each call copies the caller's FP64 host arrays to the device, runs FP64
// kernels with the reference's arithmetic, and copies the results back, as
// the reference does (predict.cu:70-113, weight.cu:222-368,
// resampling.cu:85-272).  Unlike the reference it keeps one grow-only device
// workspace per device instead of cudaMalloc/cudaFree on every call, frees
// everything it uses, and finishes its reductions on the device.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "pf_bvh.cuh"
#include "pf_city.cuh"
#include "pf_common.cuh"
#include "pf_orbit.cuh"
#include "pf_status.h"

namespace pfb {
size_t systematic_scratch_bytes(int n);
int systematic_ancestors(const double* d_lw64, const double* d_max, int n, uint32_t u, int* d_anc,
                         void* d_scratch, cudaStream_t st);
}  // namespace pfb

using namespace pfb;

namespace {

constexpr int kB = 256;  // threads per block of the stateless kernels

struct Workspace {
  void* buf = nullptr;
  size_t bytes = 0;
  cudaStream_t stream = nullptr;
};

std::mutex g_mu;
std::vector<Workspace> g_ws;  // indexed by device


inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

int cuda_status(cudaError_t e, const char* what) {
  if (e != cudaSuccess) return set_err(PF_ECUDA, "%s: %s", what, cudaGetErrorString(e));
  return PF_OK;
}

#define CK(call)                                  \
  do {                                            \
    int _s = cuda_status((call), #call);          \
    if (_s != PF_OK) return _s;                   \
  } while (0)

// Grow-only workspace of the current device (caller holds g_mu).
int workspace(size_t bytes, Workspace** out) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if ((int)g_ws.size() <= dev) g_ws.resize(dev + 1);
  Workspace& w = g_ws[dev];
  if (!w.stream) CK(cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking));
  if (w.bytes < bytes) {
    if (w.buf) CK(cudaFree(w.buf));
    w.buf = nullptr;
    w.bytes = 0;
    size_t want = align_up(bytes, 1 << 20);
    if (pf_injected_alloc_failure())
      return set_err(PF_ENOMEM, "workspace allocation of %zu bytes failed (injected by pf_test_fail_alloc)", want);
    const cudaError_t e = cudaMalloc(&w.buf, want);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      w.buf = nullptr;
      return set_err(e == cudaErrorMemoryAllocation ? PF_ENOMEM : PF_ECUDA, "workspace allocation of %zu bytes: %s",
                     want, cudaGetErrorString(e));
    }
    w.bytes = want;
  }
  *out = &w;
  return PF_OK;
}

// Stream-ordered scratch of the asynchronous entry points: the library's own
// memory pool per device, which keeps freed memory (release threshold
// unlimited), so a call does not wait on the driver for fresh memory and the
// caller's default pool is left as it is.
std::vector<cudaMemPool_t> g_pools;  // indexed by device

int scratch_pool(cudaMemPool_t* out) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_mu);
  if ((int)g_pools.size() <= dev) g_pools.resize(dev + 1, nullptr);
  if (!g_pools[dev]) {
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    CK(cudaMemPoolCreate(&pool, &props));
    unsigned long long keep = ~0ull;
    CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    g_pools[dev] = pool;
  }
  *out = g_pools[dev];
  return PF_OK;
}

struct Carve {
  unsigned char* base;
  size_t off = 0;
  template <typename T>
  T* take(size_t count) {
    T* p = (T*)(base + off);
    off = align_up(off + count * sizeof(T), 256);
    return p;
  }
};

inline int grid_of(int n) { return (n + kB - 1) / kB; }

// --------------------------------------------------------------- kernels
// Building-aware likelihood of FP64 particle arrays (weight_3d.cu:86-177):
// one thread per particle, a ray per satellite through the mesh hierarchy.
__global__ void c_weight_3d(const double* px, const double* py, const double* pz, const double* pcb,
                            pfb::MeshDev m, const pfb::Sat3d* sats, pfb::Weight3dArgs a, double* lw, int n) {
  __shared__ pfb::Sat3d s_sat[pfb::kMax3dSats];
  for (int i = threadIdx.x; i < a.n_sat; i += blockDim.x) s_sat[i] = sats[i];
  __syncthreads();
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const double p[3] = {px[j], py[j], pz[j]};
  const float3 o = pfb::mesh_origin(m, p);
  double acc = 0.0;
  for (int s = 0; s < a.n_sat; ++s) {
    const pfb::Sat3d& sv = s_sat[s];
    const double v[3] = {sv.sat[0] - p[0], sv.sat[1] - p[1], sv.sat[2] - p[2]};
    const double L = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const bool blocked = pfb::bvh_blocked(m, o, pfb::mesh_dir(m, v, L), (float)L);
    const double r = sv.pr - (L + pcb[j]);
    const double los = -0.5 * sv.w * r * r * a.inv_s2_los;
    const double rn = r > 0.0 ? r - a.nlos_bias : r;
    const double nlos = -0.5 * sv.w * rn * rn * a.inv_s2_nlos;
    acc += pfb::mix_loglik(los, nlos, blocked ? a.p_blocked : a.p_clear);
  }
  lw[j] = acc;
}

__global__ void c_init(double* px, double* py, double* pz, double* pcb, double ix, double iy,
                       double iz, double icb, double sp, double scb, int n, uint32_t k0,
                       uint32_t k1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  U4 r = philox10(U4{(uint32_t)i, 0u, TAG_COMPAT_INIT, 0u}, k0, k1);
  double2 a = box_muller_f64(r.x, r.y), b = box_muller_f64(r.z, r.w);
  px[i] = ix + a.x * sp;
  py[i] = iy + a.y * sp;
  pz[i] = iz + b.x * sp;
  pcb[i] = icb + b.y * scb;
}

__global__ void c_predict(double* px, double* py, double* pz, double* pcb, double vx, double vy,
                          double vz, double dt, double sp, double scb, int n, uint32_t k0,
                          uint32_t k1, uint32_t step) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  U4 r = philox10(U4{(uint32_t)i, step, TAG_COMPAT_PREDICT, 0u}, k0, k1);
  double2 a = box_muller_f64(r.x, r.y), b = box_muller_f64(r.z, r.w);
  px[i] += vx * dt + a.x * sp;
  py[i] += vy * dt + a.y * sp;
  pz[i] += vz * dt + b.x * sp;
  pcb[i] += b.y * scb;
}

// weight.cu:13-57: Gaussian pseudorange log-likelihood, overwriting lw.
__global__ void c_weight(const double* px, const double* py, const double* pz, const double* pcb,
                         const double* sat, const double* pr, const double* ws, double* lw, int n,
                         int n_sat, double sigma_pr) {
  extern __shared__ double s[];
  double* s_sat = s;
  double* s_pr = s + 3 * n_sat;
  double* s_ws = s + 4 * n_sat;
  for (int k = threadIdx.x; k < n_sat; k += blockDim.x) {
    s_sat[3 * k] = sat[3 * k];
    s_sat[3 * k + 1] = sat[3 * k + 1];
    s_sat[3 * k + 2] = sat[3 * k + 2];
    s_pr[k] = pr[k];
    s_ws[k] = ws[k];
  }
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x = px[i], y = py[i], z = pz[i], cb = pcb[i];
  const double inv_s2 = 1.0 / (sigma_pr * sigma_pr);
  double acc = 0.0;
  for (int k = 0; k < n_sat; ++k) {
    const double dx = x - s_sat[3 * k], dy = y - s_sat[3 * k + 1], dz = z - s_sat[3 * k + 2];
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    const double res = s_pr[k] - (r + cb);
    acc += -0.5 * s_ws[k] * res * res * inv_s2;
  }
  lw[i] = acc;
}

// Max-shifted sums of one block: max, sum w, sum w^2, sum w x (4 arrays);
// the last block merges all block rows (weight.cu:61-160,163-328, with the
// host merge moved onto the device).  out: [0..3] weighted mean, [4] sum w,
// [5] sum w^2, [6] ESS, [7] max log-weight.
__global__ void c_stats(const double* lw, const double* px, const double* py, const double* pz,
                        const double* pcb, int n, double* rows, unsigned* ticket, double* out) {
  __shared__ double s_v[kB];
  __shared__ double s_r[7][kB / 32];
  __shared__ bool s_last;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool ok = i < n;
  const double l = ok ? lw[i] : -INFINITY;
  // block max
  double m = l;
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) s_v[threadIdx.x >> 5] = m;
  __syncthreads();
  double bm = s_v[0];
  for (int w = 1; w < kB / 32; ++w) bm = fmax(bm, s_v[w]);
  double v[6] = {0, 0, 0, 0, 0, 0};
  if (ok && bm > -INFINITY) {
    const double w = exp(l - bm);
    v[0] = w;
    v[1] = w * w;
    if (px) {
      v[2] = w * px[i];
      v[3] = w * py[i];
      v[4] = w * pz[i];
      v[5] = w * pcb[i];
    }
  }
  for (int k = 0; k < 6; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 6; ++k) s_r[k][threadIdx.x >> 5] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    double* row = rows + (size_t)blockIdx.x * 8;
    row[0] = bm;
    for (int k = 0; k < 6; ++k) {
      double t = 0;
      for (int w = 0; w < kB / 32; ++w) t += s_r[k][w];
      row[1 + k] = t;
    }
    __threadfence();
    s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  const int nb = gridDim.x;
  double gm = -INFINITY;
  for (int b = threadIdx.x; b < nb; b += kB) gm = fmax(gm, __ldcg(rows + (size_t)b * 8));
  for (int o = 16; o > 0; o >>= 1) gm = fmax(gm, __shfl_xor_sync(0xffffffffu, gm, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) s_v[threadIdx.x >> 5] = gm;
  __syncthreads();
  gm = s_v[0];
  for (int w = 1; w < kB / 32; ++w) gm = fmax(gm, s_v[w]);
  double a[6] = {0, 0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nb; b += kB) {
    const double* row = rows + (size_t)b * 8;
    const double rm = __ldcg(row);
    if (!(rm > -INFINITY)) continue;
    const double c = exp(rm - gm);
    a[0] += __ldcg(row + 1) * c;
    a[1] += __ldcg(row + 2) * c * c;
    for (int k = 2; k < 6; ++k) a[k] += __ldcg(row + 1 + k) * c;
  }
  for (int k = 0; k < 6; ++k)
    for (int o = 16; o > 0; o >>= 1) a[k] += __shfl_xor_sync(0xffffffffu, a[k], o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 6; ++k) s_r[k][threadIdx.x >> 5] = a[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    double t[6];
    for (int k = 0; k < 6; ++k) {
      t[k] = 0;
      for (int w = 0; w < kB / 32; ++w) t[k] += s_r[k][w];
    }
    out[0] = t[2] / t[0];
    out[1] = t[3] / t[0];
    out[2] = t[4] / t[0];
    out[3] = t[5] / t[0];
    out[4] = t[0];
    out[5] = t[1];
    out[6] = (t[0] * t[0]) / t[1];
    out[7] = gm;
    *ticket = 0u;
  }
}

__global__ void c_gather4(const double* ix, const double* iy, const double* iz, const double* icb,
                          double* ox, double* oy, double* oz, double* ocb, const int* anc, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int a = anc[k];
  ox[k] = ix[a];
  oy[k] = iy[a];
  oz[k] = iz[a];
  ocb[k] = icb[a];
}

__global__ void c_iota(int* a, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) a[k] = k;
}

// resampling.cu:175-219: one Megopolis iteration of the reference chain on
// ancestor indices.  Slot k proposes j = (k + 1 + floor(U (N-1))) mod N and
// copies the previous iteration's occupant of j with probability
// min(1, exp(lw[j] - lw[k])).
__device__ __forceinline__ double u53(uint32_t a, uint32_t b) {
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

__global__ void c_mego_iter(const double* lw, const int* src, int* dst, int n, uint32_t k0,
                            uint32_t k1, uint32_t iter) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  U4 r = philox10(U4{(uint32_t)k, iter, TAG_COMPAT_MEGO, 0u}, k0, k1);
  const double U1 = u53(r.x, r.y), U2 = u53(r.z, r.w);
  const long long off = (long long)(U1 * (double)(n - 1)) + 1;
  const int j = (int)(((long long)k + off) % n);
  const double alpha = fmin(1.0, exp(lw[j] - lw[k]));
  dst[k] = (U2 < alpha) ? src[j] : src[k];
}

__global__ void c_interleave(const double* px, const double* py, const double* pz, const double* pcb,
                             double* out, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  out[4 * (size_t)k] = px[k];
  out[4 * (size_t)k + 1] = py[k];
  out[4 * (size_t)k + 2] = pz[k];
  out[4 * (size_t)k + 3] = pcb[k];
}

int check_n(int n) {
  if (n <= 0) return set_err(PF_EINVAL, "n_particles must be > 0 (got %d)", n);
  return PF_OK;
}

int finish(Workspace* w) {
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(w->stream));
  return PF_OK;
}

uint32_t sys_u_reference(unsigned long long seed, int n) {
  double u0 = (double)(seed % 1000000ull) / (1000000.0 * (double)n);
  double v = floor(u0 * 4294967296.0);
  return (uint32_t)(v < 0 ? 0 : (v > 4294967295.0 ? 4294967295.0 : v));
}

}  // namespace

extern "C" {

int pf_initialize(double* px, double* py, double* pz, double* pcb, double init_x, double init_y,
                  double init_z, double init_cb, double spread_pos, double spread_cb, int n_particles,
                  unsigned long long seed) {
  clear_err();
  int s = check_n(n_particles);
  if (s != PF_OK) return s;
  if (!px || !py || !pz || !pcb) return set_err(PF_EINVAL, "null particle array");
  std::lock_guard<std::mutex> lk(g_mu);
  const size_t nb = (size_t)n_particles * 8;
  Workspace* w;
  if ((s = workspace(4 * align_up(nb, 256), &w)) != PF_OK) return s;
  Carve c{(unsigned char*)w->buf};
  double *dx = c.take<double>(n_particles), *dy = c.take<double>(n_particles),
         *dz = c.take<double>(n_particles), *dcb = c.take<double>(n_particles);
  c_init<<<grid_of(n_particles), kB, 0, w->stream>>>(dx, dy, dz, dcb, init_x, init_y, init_z, init_cb,
                                                     spread_pos, spread_cb, n_particles,
                                                     (uint32_t)seed, (uint32_t)(seed >> 32));
  CK(cudaMemcpyAsync(px, dx, nb, cudaMemcpyDeviceToHost, w->stream));
  CK(cudaMemcpyAsync(py, dy, nb, cudaMemcpyDeviceToHost, w->stream));
  CK(cudaMemcpyAsync(pz, dz, nb, cudaMemcpyDeviceToHost, w->stream));
  CK(cudaMemcpyAsync(pcb, dcb, nb, cudaMemcpyDeviceToHost, w->stream));
  return finish(w);
}

int pf_predict(double* px, double* py, double* pz, double* pcb, const double* vx, const double* vy,
               const double* vz, double dt, double sigma_pos, double sigma_cb, int n_particles,
               unsigned long long seed, int step) {
  clear_err();
  int s = check_n(n_particles);
  if (s != PF_OK) return s;
  if (!px || !py || !pz || !pcb || !vx || !vy || !vz) return set_err(PF_EINVAL, "null array");
  std::lock_guard<std::mutex> lk(g_mu);
  const size_t nb = (size_t)n_particles * 8;
  Workspace* w;
  if ((s = workspace(4 * align_up(nb, 256), &w)) != PF_OK) return s;
  Carve c{(unsigned char*)w->buf};
  double *dx = c.take<double>(n_particles), *dy = c.take<double>(n_particles),
         *dz = c.take<double>(n_particles), *dcb = c.take<double>(n_particles);
  CK(cudaMemcpyAsync(dx, px, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dy, py, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dz, pz, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dcb, pcb, nb, cudaMemcpyHostToDevice, w->stream));
  c_predict<<<grid_of(n_particles), kB, 0, w->stream>>>(dx, dy, dz, dcb, vx[0], vy[0], vz[0], dt, sigma_pos,
                                                        sigma_cb, n_particles, (uint32_t)seed,
                                                        (uint32_t)(seed >> 32), (uint32_t)step);
  CK(cudaMemcpyAsync(px, dx, nb, cudaMemcpyDeviceToHost, w->stream));
  CK(cudaMemcpyAsync(py, dy, nb, cudaMemcpyDeviceToHost, w->stream));
  CK(cudaMemcpyAsync(pz, dz, nb, cudaMemcpyDeviceToHost, w->stream));
  CK(cudaMemcpyAsync(pcb, dcb, nb, cudaMemcpyDeviceToHost, w->stream));
  return finish(w);
}

int pf_weight(const double* px, const double* py, const double* pz, const double* pcb,
              const double* sat_ecef, const double* pseudoranges, const double* weights_sat,
              double* log_weights, int n_particles, int n_sat, double sigma_pr) {
  clear_err();
  int s = check_n(n_particles);
  if (s != PF_OK) return s;
  if (n_sat <= 0) return set_err(PF_EINVAL, "n_sat must be > 0 (got %d)", n_sat);
  if (n_sat > 1024) return set_err(PF_ECAP, "n_sat %d above the 1024 satellites staged in shared memory", n_sat);
  if (!px || !py || !pz || !pcb || !sat_ecef || !pseudoranges || !weights_sat || !log_weights)
    return set_err(PF_EINVAL, "null array");
  if (!(sigma_pr > 0.0) || !isfinite(sigma_pr)) return set_err(PF_EINVAL, "sigma_pr must be finite and > 0");
  std::lock_guard<std::mutex> lk(g_mu);
  const size_t nb = (size_t)n_particles * 8;
  Workspace* w;
  if ((s = workspace(5 * align_up(nb, 256) + align_up((size_t)n_sat * 40, 256) * 2, &w)) != PF_OK) return s;
  Carve c{(unsigned char*)w->buf};
  double *dx = c.take<double>(n_particles), *dy = c.take<double>(n_particles),
         *dz = c.take<double>(n_particles), *dcb = c.take<double>(n_particles),
         *dlw = c.take<double>(n_particles);
  double *dsat = c.take<double>(3 * (size_t)n_sat), *dpr = c.take<double>(n_sat), *dws = c.take<double>(n_sat);
  CK(cudaMemcpyAsync(dx, px, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dy, py, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dz, pz, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dcb, pcb, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dsat, sat_ecef, (size_t)n_sat * 24, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dpr, pseudoranges, (size_t)n_sat * 8, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dws, weights_sat, (size_t)n_sat * 8, cudaMemcpyHostToDevice, w->stream));
  c_weight<<<grid_of(n_particles), kB, (size_t)n_sat * 40, w->stream>>>(dx, dy, dz, dcb, dsat, dpr, dws, dlw,
                                                                        n_particles, n_sat, sigma_pr);
  CK(cudaMemcpyAsync(log_weights, dlw, nb, cudaMemcpyDeviceToHost, w->stream));
  return finish(w);
}

int pf_compute_ess(const double* log_weights, int n_particles, double* ess_out) {
  clear_err();
  int s = check_n(n_particles);
  if (s != PF_OK) return s;
  if (!log_weights || !ess_out) return set_err(PF_EINVAL, "null array");
  std::lock_guard<std::mutex> lk(g_mu);
  const size_t nb = (size_t)n_particles * 8;
  const int g = grid_of(n_particles);
  Workspace* w;
  if ((s = workspace(align_up(nb, 256) + align_up((size_t)g * 64, 256) + 512, &w)) != PF_OK) return s;
  Carve c{(unsigned char*)w->buf};
  double* dlw = c.take<double>(n_particles);
  double* rows = c.take<double>((size_t)g * 8);
  double* out = c.take<double>(8);
  unsigned* ticket = c.take<unsigned>(4);
  CK(cudaMemcpyAsync(dlw, log_weights, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemsetAsync(ticket, 0, 16, w->stream));
  c_stats<<<g, kB, 0, w->stream>>>(dlw, nullptr, nullptr, nullptr, nullptr, n_particles, rows, ticket, out);
  double h[8];
  CK(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, w->stream));
  if ((s = finish(w)) != PF_OK) return s;
  *ess_out = h[6];
  return PF_OK;
}

int pf_estimate(const double* px, const double* py, const double* pz, const double* pcb,
                const double* log_weights, double* result, int n_particles) {
  clear_err();
  int s = check_n(n_particles);
  if (s != PF_OK) return s;
  if (!px || !py || !pz || !pcb || !log_weights || !result) return set_err(PF_EINVAL, "null array");
  std::lock_guard<std::mutex> lk(g_mu);
  const size_t nb = (size_t)n_particles * 8;
  const int g = grid_of(n_particles);
  Workspace* w;
  if ((s = workspace(5 * align_up(nb, 256) + align_up((size_t)g * 64, 256) + 512, &w)) != PF_OK) return s;
  Carve c{(unsigned char*)w->buf};
  double *dx = c.take<double>(n_particles), *dy = c.take<double>(n_particles),
         *dz = c.take<double>(n_particles), *dcb = c.take<double>(n_particles),
         *dlw = c.take<double>(n_particles);
  double* rows = c.take<double>((size_t)g * 8);
  double* out = c.take<double>(8);
  unsigned* ticket = c.take<unsigned>(4);
  CK(cudaMemcpyAsync(dx, px, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dy, py, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dz, pz, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dcb, pcb, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dlw, log_weights, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemsetAsync(ticket, 0, 16, w->stream));
  c_stats<<<g, kB, 0, w->stream>>>(dlw, dx, dy, dz, dcb, n_particles, rows, ticket, out);
  double h[8];
  CK(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, w->stream));
  if ((s = finish(w)) != PF_OK) return s;
  for (int i = 0; i < 4; ++i) result[i] = h[i];
  return PF_OK;
}

int pf_get_particles(const double* px, const double* py, const double* pz, const double* pcb,
                     double* output, int n_particles) {
  clear_err();
  int s = check_n(n_particles);
  if (s != PF_OK) return s;
  if (!px || !py || !pz || !pcb || !output) return set_err(PF_EINVAL, "null array");
  std::lock_guard<std::mutex> lk(g_mu);
  const size_t nb = (size_t)n_particles * 8;
  Workspace* w;
  if ((s = workspace(8 * align_up(nb, 256), &w)) != PF_OK) return s;
  Carve c{(unsigned char*)w->buf};
  double *dx = c.take<double>(n_particles), *dy = c.take<double>(n_particles),
         *dz = c.take<double>(n_particles), *dcb = c.take<double>(n_particles),
         *dout = c.take<double>(4 * (size_t)n_particles);
  CK(cudaMemcpyAsync(dx, px, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dy, py, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dz, pz, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dcb, pcb, nb, cudaMemcpyHostToDevice, w->stream));
  c_interleave<<<grid_of(n_particles), kB, 0, w->stream>>>(dx, dy, dz, dcb, dout, n_particles);
  CK(cudaMemcpyAsync(output, dout, 4 * nb, cudaMemcpyDeviceToHost, w->stream));
  return finish(w);
}

int pf_resample_systematic(double* px, double* py, double* pz, double* pcb, const double* log_weights,
                           int n_particles, unsigned long long seed) {
  clear_err();
  int s = check_n(n_particles);
  if (s != PF_OK) return s;
  if (!px || !py || !pz || !pcb || !log_weights) return set_err(PF_EINVAL, "null array");
  std::lock_guard<std::mutex> lk(g_mu);
  const int n = n_particles;
  const size_t nb = (size_t)n * 8;
  const int g = grid_of(n);
  const size_t need = 9 * align_up(nb, 256) + align_up((size_t)n * 4, 256) +
                      align_up((size_t)g * 64, 256) + 512 + pfb::systematic_scratch_bytes(n) + 256;
  Workspace* w;
  if ((s = workspace(need, &w)) != PF_OK) return s;
  Carve c{(unsigned char*)w->buf};
  double *ix = c.take<double>(n), *iy = c.take<double>(n), *iz = c.take<double>(n), *icb = c.take<double>(n);
  double *ox = c.take<double>(n), *oy = c.take<double>(n), *oz = c.take<double>(n), *ocb = c.take<double>(n);
  double* dlw = c.take<double>(n);
  int* anc = c.take<int>(n);
  double* rows = c.take<double>((size_t)g * 8);
  double* out = c.take<double>(8);
  unsigned* ticket = c.take<unsigned>(4);
  unsigned char* scratch = c.take<unsigned char>(pfb::systematic_scratch_bytes(n));
  CK(cudaMemcpyAsync(ix, px, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(iy, py, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(iz, pz, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(icb, pcb, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dlw, log_weights, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemsetAsync(ticket, 0, 16, w->stream));
  c_stats<<<g, kB, 0, w->stream>>>(dlw, nullptr, nullptr, nullptr, nullptr, n, rows, ticket, out);
  CK(cudaGetLastError());
  if ((s = pfb::systematic_ancestors(dlw, out + 7, n, sys_u_reference(seed, n), anc, scratch, w->stream)) != PF_OK)
    return s;
  c_gather4<<<g, kB, 0, w->stream>>>(ix, iy, iz, icb, ox, oy, oz, ocb, anc, n);
  CK(cudaMemcpyAsync(px, ox, nb, cudaMemcpyDeviceToHost, w->stream));
  CK(cudaMemcpyAsync(py, oy, nb, cudaMemcpyDeviceToHost, w->stream));
  CK(cudaMemcpyAsync(pz, oz, nb, cudaMemcpyDeviceToHost, w->stream));
  CK(cudaMemcpyAsync(pcb, ocb, nb, cudaMemcpyDeviceToHost, w->stream));
  return finish(w);
}

int pf_resample_megopolis(double* px, double* py, double* pz, double* pcb, const double* log_weights,
                          int n_particles, int n_iterations, unsigned long long seed) {
  clear_err();
  int s = check_n(n_particles);
  if (s != PF_OK) return s;
  if (n_iterations < 0) return set_err(PF_EINVAL, "n_iterations must be >= 0");
  if (!px || !py || !pz || !pcb || !log_weights) return set_err(PF_EINVAL, "null array");
  std::lock_guard<std::mutex> lk(g_mu);
  const int n = n_particles;
  const size_t nb = (size_t)n * 8;
  const int g = grid_of(n);
  Workspace* w;
  if ((s = workspace(9 * align_up(nb, 256) + 2 * align_up((size_t)n * 4, 256), &w)) != PF_OK) return s;
  Carve c{(unsigned char*)w->buf};
  double *ix = c.take<double>(n), *iy = c.take<double>(n), *iz = c.take<double>(n), *icb = c.take<double>(n);
  double *ox = c.take<double>(n), *oy = c.take<double>(n), *oz = c.take<double>(n), *ocb = c.take<double>(n);
  double* dlw = c.take<double>(n);
  int* a0 = c.take<int>(n);
  int* a1 = c.take<int>(n);
  CK(cudaMemcpyAsync(ix, px, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(iy, py, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(iz, pz, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(icb, pcb, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dlw, log_weights, nb, cudaMemcpyHostToDevice, w->stream));
  c_iota<<<g, kB, 0, w->stream>>>(a0, n);
  int* src = a0;
  int* dst = a1;
  for (int it = 0; it < n_iterations; ++it) {
    c_mego_iter<<<g, kB, 0, w->stream>>>(dlw, src, dst, n, (uint32_t)seed, (uint32_t)(seed >> 32), (uint32_t)it);
    int* t = src;
    src = dst;
    dst = t;
  }
  c_gather4<<<g, kB, 0, w->stream>>>(ix, iy, iz, icb, ox, oy, oz, ocb, src, n);
  CK(cudaMemcpyAsync(px, ox, nb, cudaMemcpyDeviceToHost, w->stream));
  CK(cudaMemcpyAsync(py, oy, nb, cudaMemcpyDeviceToHost, w->stream));
  CK(cudaMemcpyAsync(pz, oz, nb, cudaMemcpyDeviceToHost, w->stream));
  CK(cudaMemcpyAsync(pcb, ocb, nb, cudaMemcpyDeviceToHost, w->stream));
  return finish(w);
}

int pf_weight_3d(const double* px, const double* py, const double* pz, const double* pcb, const double* sat_ecef,
                 const double* pseudoranges, const double* weights_sat, const double* triangles, int n_tri,
                 double* log_weights, int n_particles, int n_sat, double sigma_los, double sigma_nlos,
                 double nlos_bias, double blocked_nlos_prob, double clear_nlos_prob) {
  clear_err();
  int s = check_n(n_particles);
  if (s != PF_OK) return s;
  if (n_sat <= 0 || n_sat > pfb::kMax3dSats) return set_err(PF_ECAP, "need 1..%d satellites", pfb::kMax3dSats);
  if (n_tri < 0 || (n_tri > 0 && !triangles)) return set_err(PF_EINVAL, "bad triangles");
  if (!px || !py || !pz || !pcb || !sat_ecef || !pseudoranges || !weights_sat || !log_weights)
    return set_err(PF_EINVAL, "null array");
  if (!(sigma_los > 0.0) || !(sigma_nlos > 0.0) || !isfinite(sigma_los) || !isfinite(sigma_nlos) ||
      !isfinite(nlos_bias) || !isfinite(blocked_nlos_prob) || !isfinite(clear_nlos_prob))
    return set_err(PF_EINVAL, "sigmas must be > 0 and all parameters finite");
  std::vector<float> nodes((size_t)std::max(1, n_tri) * 16), tris((size_t)std::max(1, n_tri) * 12);
  int n_nodes = 0;
  double origin[3], rot[9];
  if ((s = pf_mesh_build(triangles, n_tri, nodes.data(), tris.data(), &n_nodes, origin, rot)) != PF_OK) return s;
  std::vector<pfb::Sat3d> sv(n_sat);
  for (int i = 0; i < n_sat; ++i) {
    for (int k = 0; k < 3; ++k) sv[i].sat[k] = sat_ecef[3 * i + k];
    sv[i].pr = pseudoranges[i];
    sv[i].w = weights_sat[i];
  }
  std::lock_guard<std::mutex> lk(g_mu);
  const size_t nb = (size_t)n_particles * 8;
  const size_t nodes_b = sizeof(float) * nodes.size(), tris_b = sizeof(float) * tris.size();
  Workspace* w;
  if ((s = workspace(5 * align_up(nb, 256) + align_up(sizeof(pfb::Sat3d) * n_sat, 256) + align_up(nodes_b, 256) +
                         align_up(tris_b, 256),
                     &w)) != PF_OK)
    return s;
  Carve c{(unsigned char*)w->buf};
  double *dx = c.take<double>(n_particles), *dy = c.take<double>(n_particles),
         *dz = c.take<double>(n_particles), *dcb = c.take<double>(n_particles),
         *dlw = c.take<double>(n_particles);
  pfb::Sat3d* dsat = c.take<pfb::Sat3d>(n_sat);
  float* dnodes = c.take<float>(nodes.size());
  float* dtris = c.take<float>(tris.size());
  CK(cudaMemcpyAsync(dx, px, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dy, py, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dz, pz, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dcb, pcb, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dsat, sv.data(), sizeof(pfb::Sat3d) * n_sat, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dnodes, nodes.data(), nodes_b, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dtris, tris.data(), tris_b, cudaMemcpyHostToDevice, w->stream));
  pfb::MeshDev m;
  memset(&m, 0, sizeof(m));
  m.nodes = reinterpret_cast<const float4*>(dnodes);
  m.tris = reinterpret_cast<const float4*>(dtris);
  m.n_nodes = n_nodes;
  m.n_tris = n_tri;
  for (int k = 0; k < 3; ++k) m.origin[k] = origin[k];
  for (int k = 0; k < 9; ++k) m.rot[k] = rot[k];
  pfb::Weight3dArgs a;
  memset(&a, 0, sizeof(a));
  a.n_sat = n_sat;
  a.inv_s2_los = 1.0 / (sigma_los * sigma_los);
  a.inv_s2_nlos = 1.0 / (sigma_nlos * sigma_nlos);
  a.nlos_bias = nlos_bias;
  a.p_blocked = blocked_nlos_prob;
  a.p_clear = clear_nlos_prob;
  c_weight_3d<<<grid_of(n_particles), kB, 0, w->stream>>>(dx, dy, dz, dcb, m, dsat, a, dlw, n_particles);
  CK(cudaMemcpyAsync(log_weights, dlw, nb, cudaMemcpyDeviceToHost, w->stream));
  return finish(w);
}

// ------------------------------------------------------- input formation
int pf_sat_positions_batch(const pf_ephemeris_t* params, const double* gps_times, double* sat_pos,
                           double* sat_clk, int n_epoch, int n_sat) {
  clear_err();
  if (n_sat < 0 || n_epoch < 0) return set_err(PF_EINVAL, "n_sat and n_epoch must be >= 0");
  if ((long long)n_epoch * n_sat > (1ll << 30)) return set_err(PF_EINVAL, "n_epoch * n_sat above 2^30");
  if (n_sat == 0 || n_epoch == 0) return PF_OK;
  if (!params || !gps_times || !sat_pos || !sat_clk) return set_err(PF_EINVAL, "null array");
  int s;
  std::lock_guard<std::mutex> lk(g_mu);
  const size_t ne = (size_t)n_epoch * n_sat;
  Workspace* w;
  if ((s = workspace(align_up(sizeof(pf_ephemeris_t) * n_sat, 256) + align_up(8 * (size_t)n_epoch, 256) +
                         align_up(24 * ne, 256) + align_up(8 * ne, 256),
                     &w)) != PF_OK)
    return s;
  Carve c{(unsigned char*)w->buf};
  pf_ephemeris_t* dp = c.take<pf_ephemeris_t>(n_sat);
  double* dt = c.take<double>(n_epoch);
  double* dpos = c.take<double>(3 * ne);
  double* dclk = c.take<double>(ne);
  CK(cudaMemcpyAsync(dp, params, sizeof(pf_ephemeris_t) * n_sat, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dt, gps_times, 8 * (size_t)n_epoch, cudaMemcpyHostToDevice, w->stream));
  k_sat_pos_gps<<<(unsigned)((ne + kB - 1) / kB), kB, 0, w->stream>>>(dp, dt, n_epoch, n_sat, dpos, dclk);
  CK(cudaMemcpyAsync(sat_pos, dpos, 24 * ne, cudaMemcpyDeviceToHost, w->stream));
  CK(cudaMemcpyAsync(sat_clk, dclk, 8 * ne, cudaMemcpyDeviceToHost, w->stream));
  return finish(w);
}

int pf_sat_positions(const pf_ephemeris_t* params, double gps_time, double* sat_pos, double* sat_clk,
                     int n_sat) {
  return pf_sat_positions_batch(params, &gps_time, sat_pos, sat_clk, 1, n_sat);
}

int pf_broadcast_orbits(const pf_broadcast_t* d_recs, int n_recs, const int* d_rec_index, const double* d_times,
                        int n_epoch, int n_sat, double glo_step, double* d_pos, double* d_clk, void* stream) {
  clear_err();
  if (n_sat < 0 || n_epoch < 0 || n_recs < 0) return set_err(PF_EINVAL, "sizes must be >= 0");
  if ((long long)n_epoch * n_sat > (1ll << 30)) return set_err(PF_EINVAL, "n_epoch * n_sat above 2^30");
  if (n_sat == 0 || n_epoch == 0) return PF_OK;
  if (!d_times || (n_recs > 0 && !d_recs)) return set_err(PF_EINVAL, "null array");
  if (!d_rec_index && n_recs < n_sat) return set_err(PF_EINVAL, "without an index, n_recs must be >= n_sat");
  if (!isfinite(glo_step) || glo_step <= 0.0) glo_step = kGloStep;
  if (glo_step < 1.0) return set_err(PF_EINVAL, "glo_step below 1 s");
  const long ne = (long)n_epoch * n_sat;
  cudaStream_t st = (cudaStream_t)stream;
  const unsigned grid = (unsigned)((ne + kB - 1) / kB);
  // GLONASS state table: the epochs of a record share its states at whole
  // steps from toe, so they are integrated once per (record, direction)
  int kc = 0;
  if (n_recs > 0) {
    const size_t per_state = (size_t)2 * n_recs * 6 * sizeof(double);
    kc = (int)std::min<size_t>(kGloTable, kGloTableBytes / per_state);
    if (kc < 4) kc = 0;  // too many records for the scratch: walk from toe
  }
  if (kc == 0) {
    k_broadcast_orbits<<<grid, kB, 0, st>>>(d_recs, n_recs, d_rec_index, d_times, n_epoch, n_sat, glo_step,
                                            nullptr, 0, d_pos, d_clk, nullptr);
    CK(cudaGetLastError());
    return PF_OK;
  }
  const size_t kmax_bytes = align_up(sizeof(int) * 2 * (size_t)n_recs, 256);
  const size_t tbl_bytes = (size_t)2 * n_recs * kc * 6 * sizeof(double);
  unsigned char* scratch = nullptr;
  cudaMemPool_t pool = nullptr;
  int ps = scratch_pool(&pool);
  if (ps != PF_OK) return ps;
  CK(cudaMallocFromPoolAsync((void**)&scratch, kmax_bytes + tbl_bytes, pool, st));
  int* kmax = (int*)scratch;
  double* tbl = (double*)(scratch + kmax_bytes);
  cudaError_t ce = cudaMemsetAsync(kmax, 0, kmax_bytes, st);
  if (ce == cudaSuccess) {
    k_glo_need<<<grid, kB, 0, st>>>(d_recs, n_recs, d_rec_index, d_times, n_epoch, n_sat, glo_step, kc, kmax);
    k_glo_table<<<(unsigned)((2 * n_recs + 127) / 128), 128, 0, st>>>(d_recs, n_recs, glo_step, kmax, kc, tbl);
    k_broadcast_orbits<<<grid, kB, 0, st>>>(d_recs, n_recs, d_rec_index, d_times, n_epoch, n_sat, glo_step, tbl,
                                            kc, d_pos, d_clk, nullptr);
    ce = cudaGetLastError();
  }
  const cudaError_t fe = cudaFreeAsync(scratch, st);
  CK(ce);
  CK(fe);
  return PF_OK;
}

int pf_sagnac(const double* d_rx, const double* d_sat, int n_epoch, int n_sat, double* d_sat_rot,
              double* d_range, void* stream) {
  clear_err();
  if (n_sat < 0 || n_epoch < 0) return set_err(PF_EINVAL, "sizes must be >= 0");
  if ((long long)n_epoch * n_sat > (1ll << 30)) return set_err(PF_EINVAL, "n_epoch * n_sat above 2^30");
  if (n_sat == 0 || n_epoch == 0) return PF_OK;
  if (!d_rx || !d_sat) return set_err(PF_EINVAL, "null array");
  const long ne = (long)n_epoch * n_sat;
  k_sagnac<<<(unsigned)((ne + kB - 1) / kB), kB, 0, (cudaStream_t)stream>>>(d_rx, d_sat, n_epoch, n_sat,
                                                                           d_sat_rot, d_range);
  CK(cudaGetLastError());
  return PF_OK;
}

int pf_ecef_to_lla(const double* ecef_x, const double* ecef_y, const double* ecef_z, double* lat, double* lon,
                   double* alt, int n) {
  clear_err();
  if (n < 0) return set_err(PF_EINVAL, "n must be >= 0");
  if (n == 0) return PF_OK;
  if (!ecef_x || !ecef_y || !ecef_z || !lat || !lon || !alt) return set_err(PF_EINVAL, "null array");
  int s;
  std::lock_guard<std::mutex> lk(g_mu);
  const size_t nb = (size_t)n * 8;
  Workspace* w;
  if ((s = workspace(6 * align_up(nb, 256), &w)) != PF_OK) return s;
  Carve c{(unsigned char*)w->buf};
  double *dx = c.take<double>(n), *dy = c.take<double>(n), *dz = c.take<double>(n);
  double *dla = c.take<double>(n), *dlo = c.take<double>(n), *dal = c.take<double>(n);
  CK(cudaMemcpyAsync(dx, ecef_x, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dy, ecef_y, nb, cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(dz, ecef_z, nb, cudaMemcpyHostToDevice, w->stream));
  k_ecef_to_lla<<<grid_of(n), kB, 0, w->stream>>>(dx, dy, dz, dla, dlo, dal, n);
  CK(cudaMemcpyAsync(lat, dla, nb, cudaMemcpyDeviceToHost, w->stream));
  CK(cudaMemcpyAsync(lon, dlo, nb, cudaMemcpyDeviceToHost, w->stream));
  CK(cudaMemcpyAsync(alt, dal, nb, cudaMemcpyDeviceToHost, w->stream));
  return finish(w);
}

int pf_city_los(const unsigned char* d_occ, const double* d_box, const double* d_height, int n, double cell,
                double hmax, int steps, const double* d_p, const double* d_dir, int n_ray, unsigned char* d_blocked,
                void* stream) {
  clear_err();
  if (n_ray < 0 || n < 0 || steps < 0) return set_err(PF_EINVAL, "sizes must be >= 0");
  if (n_ray == 0) return PF_OK;
  if (!d_p || !d_dir || !d_blocked || (n > 0 && (!d_occ || !d_box || !d_height)))
    return set_err(PF_EINVAL, "null array");
  if (!(cell > 0.0) || !isfinite(cell) || !isfinite(hmax)) return set_err(PF_EINVAL, "cell must be > 0, hmax finite");
  if ((long long)n * n > (1ll << 28)) return set_err(PF_EINVAL, "city grid above 2^28 cells");
  pfb::CityDev c;
  c.occ = d_occ;
  c.box = d_box;
  c.height = d_height;
  c.n = n;
  c.cell = cell;
  c.hmax = hmax;
  c.steps = steps;
  k_city_los<<<grid_of(n_ray), kB, 0, (cudaStream_t)stream>>>(c, d_p, d_dir, n_ray, d_blocked);
  CK(cudaGetLastError());
  return PF_OK;
}

}  // extern "C"
