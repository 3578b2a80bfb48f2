// pf_noalloc.cu -- ESS of device-resident log-weights with no allocation.
//
// Some callers cannot call cudaMalloc: real-time loops such as a receiver
// node that must not allocate (and risk a stall) after start-up, and host
// applications whose device memory is all handed to another allocator, where
// a cudaMalloc of ours could fail or fragment their arena.
// pf_compute_ess_noalloc
// serves them: the caller passes its own device input and output, and the
// per-block partial sums live in a fixed file-scope device array instead of
// an allocated workspace.
//
// Limits and sharing:
//  * at most PF_NOALLOC_MAX_PARTICLES (2^22) log-weights per call: the
//    array holds one 32-byte row per 256 particles, 512 KiB in all; larger
//    calls are rejected with PF_ECAP;
//  * every GPU that loads the library holds the array until the process
//    exits;
//  * all calls share the array and it keeps the last call's contents: the
//    ticket that must start at zero is cleared by every call, and calls that
//    overlap on the GPU (other streams, other threads) race on the array --
//    serialise them;
//  * the first call on a device resolves the array's device address with
//    cudaGetSymbolAddress; make that first call before any stream capture.
#include <cuda_runtime.h>
#include <math.h>

#include <mutex>

#include "pf_status.h"

namespace {

constexpr int kB = 256;
constexpr int kMaxBlocks = PF_NOALLOC_MAX_PARTICLES / kB;
constexpr int kRowDoubles = 4;  // block max, sum w, sum w^2, pad
constexpr size_t kScratchBytes = (size_t)kMaxBlocks * kRowDoubles * sizeof(double) + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {nullptr};

// One-time per device: the device address of the array.  In host code the
// array's name is only a host-side stand-in, never a device address.
int scratch_for_current_device(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_err(PF_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return set_err(PF_EINVAL, "device index %d not supported", dev);
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return set_err(PF_ECUDA, "cudaGetSymbolAddress of the ESS scratch: %s", cudaGetErrorString(e));
    g_scratch_ptr[dev] = p;
  }
  *out = (unsigned char*)g_scratch_ptr[dev];
  return PF_OK;
}

// Block rows of (max, sum exp(lw - max), sum exp(2 (lw - max))); the last
// block (ticket) merges the rows with max-shift corrections and writes the
// ESS, then resets the ticket.  Same arithmetic as the reference's
// compute_ess_kernel + host merge (weight.cu:61-160), merged on the device.
__global__ void k_ess_noalloc(const double* __restrict__ lw, int n, unsigned char* scratch,
                              double* __restrict__ ess_out) {
  double* rows = reinterpret_cast<double*>(scratch + 256);
  unsigned* ticket = reinterpret_cast<unsigned*>(scratch);
  __shared__ double s_v[kB / 32];
  __shared__ double s_a[2][kB / 32];
  __shared__ bool s_last;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double l = i < n ? lw[i] : -INFINITY;
  double m = l;
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) s_v[threadIdx.x >> 5] = m;
  __syncthreads();
  double bm = s_v[0];
  for (int w = 1; w < kB / 32; ++w) bm = fmax(bm, s_v[w]);
  double w1 = 0.0, w2 = 0.0;
  if (i < n && bm > -INFINITY) {
    const double w = exp(l - bm);
    w1 = w;
    w2 = w * w;
  }
  for (int o = 16; o > 0; o >>= 1) {
    w1 += __shfl_xor_sync(0xffffffffu, w1, o);
    w2 += __shfl_xor_sync(0xffffffffu, w2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    s_a[0][threadIdx.x >> 5] = w1;
    s_a[1][threadIdx.x >> 5] = w2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t1 = 0.0, t2 = 0.0;
    for (int w = 0; w < kB / 32; ++w) {
      t1 += s_a[0][w];
      t2 += s_a[1][w];
    }
    double* row = rows + (size_t)blockIdx.x * kRowDoubles;
    row[0] = bm;
    row[1] = t1;
    row[2] = t2;
    __threadfence();
    s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double gm = -INFINITY;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += kB) gm = fmax(gm, __ldcg(rows + (size_t)b * kRowDoubles));
  for (int o = 16; o > 0; o >>= 1) gm = fmax(gm, __shfl_xor_sync(0xffffffffu, gm, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) s_v[threadIdx.x >> 5] = gm;
  __syncthreads();
  gm = s_v[0];
  for (int w = 1; w < kB / 32; ++w) gm = fmax(gm, s_v[w]);
  double a1 = 0.0, a2 = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += kB) {
    const double* row = rows + (size_t)b * kRowDoubles;
    const double rm = __ldcg(row);
    if (!(rm > -INFINITY)) continue;
    const double c = exp(rm - gm);
    a1 += __ldcg(row + 1) * c;
    a2 += __ldcg(row + 2) * c * c;
  }
  for (int o = 16; o > 0; o >>= 1) {
    a1 += __shfl_xor_sync(0xffffffffu, a1, o);
    a2 += __shfl_xor_sync(0xffffffffu, a2, o);
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    s_a[0][threadIdx.x >> 5] = a1;
    s_a[1][threadIdx.x >> 5] = a2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t1 = 0.0, t2 = 0.0;
    for (int w = 0; w < kB / 32; ++w) {
      t1 += s_a[0][w];
      t2 += s_a[1][w];
    }
    *ess_out = (t1 * t1) / t2;
    *ticket = 0u;
  }
}

}  // namespace

extern "C" int pf_compute_ess_noalloc(const double* d_log_weights, int n_particles, double* d_ess_out,
                                      void* stream) {
  clear_err();
  if (!d_log_weights || !d_ess_out) return set_err(PF_EINVAL, "null device pointer");
  if (n_particles <= 0) return set_err(PF_EINVAL, "n_particles must be > 0 (got %d)", n_particles);
  if (n_particles > PF_NOALLOC_MAX_PARTICLES)
    return set_err(PF_ECAP, "n_particles %d exceeds the no-allocation limit of %d", n_particles,
                   PF_NOALLOC_MAX_PARTICLES);
  unsigned char* scratch = nullptr;
  int s = scratch_for_current_device(&scratch);
  if (s != PF_OK) return s;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(unsigned), st);  // the ticket starts at zero
  if (e != cudaSuccess) return set_err(PF_ECUDA, "clearing the ticket: %s", cudaGetErrorString(e));
  const int grid = (n_particles + kB - 1) / kB;
  k_ess_noalloc<<<grid, kB, 0, st>>>(d_log_weights, n_particles, scratch, d_ess_out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(PF_ECUDA, "k_ess_noalloc launch: %s", cudaGetErrorString(e));
  return PF_OK;
}
