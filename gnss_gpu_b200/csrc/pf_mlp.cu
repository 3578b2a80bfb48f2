// pf_mlp.cu -- training and inference kernels of the per-satellite NLOS
// network (pf_mlp.cuh), on the tensor cores with BF16 operands and FP32
// accumulation.
//
// Loss per sample (label nlos in {0, 1}, bias b in metres):
//   L = BCE(sigmoid(o0), nlos) + nlos * ((mu - b) / 20 m)^2,  mu = 20 m softplus(o1)
// averaged over the batch.
//
// k_mlp_grad: each CTA takes rounds of 128 rows (8 warps x 16); per round a
// warp runs the forward pass and the backward pass of its rows on the tensor
// cores (dO -> dH2 = dO W3 masked by ReLU' -> dH1 = dH2 W2^T masked), stages
// activations and gradients in shared memory as BF16, and the CTA then forms
// the weight gradients dW = G^T H over the round's 128 rows, again as MMAs,
// accumulated across rounds in registers.  Per-CTA partial gradients go to a
// scratch array and k_mlp_reduce sums them in a fixed order (deterministic),
// then applies Adam or returns the gradient.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>

#include "pf_mlp.cuh"
#include "pf_status.h"

namespace pfb {

constexpr int kMlpThreads = 256;
constexpr int kRows = 128;  // rows per CTA round

struct GradSmem {
  MlpSmem w;
  float x[kRows * kMlpIn];          // inputs, FP32, cols 12..15 zero
  __nv_bfloat16 h1[kRows * kMlpH];  // activations after ReLU
  __nv_bfloat16 h2[kRows * kMlpH];
  __nv_bfloat16 g1[kRows * kMlpH];  // dL/d(pre-activation) of layer 1
  __nv_bfloat16 g2[kRows * kMlpH];  // of layer 2
  __nv_bfloat16 go[kRows * 16];     // dL/do (cols 0, 1), zero padded
  float loss[kMlpThreads / 32];
};

// Store a BF16 A fragment (k-tile q) of rows [r0, r0+16) into a row-major
// [rows][64] BF16 array.
__device__ __forceinline__ void store_frag(__nv_bfloat16* dst, int r0, int q, int lane, const uint32_t (&a)[4]) {
  const int g = lane >> 2, t = lane & 3;
  *reinterpret_cast<uint32_t*>(dst + (size_t)(r0 + g) * kMlpH + 16 * q + 2 * t) = a[0];
  *reinterpret_cast<uint32_t*>(dst + (size_t)(r0 + g + 8) * kMlpH + 16 * q + 2 * t) = a[1];
  *reinterpret_cast<uint32_t*>(dst + (size_t)(r0 + g) * kMlpH + 16 * q + 8 + 2 * t) = a[2];
  *reinterpret_cast<uint32_t*>(dst + (size_t)(r0 + g + 8) * kMlpH + 16 * q + 8 + 2 * t) = a[3];
}

__device__ __forceinline__ uint32_t pack_raw(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}
__device__ __forceinline__ float bf(uint32_t v, int hi) {
  return __bfloat162float(__ushort_as_bfloat16((unsigned short)(hi ? (v >> 16) : (v & 0xFFFFu))));
}

// A fragment of the transposed operand: A[m][k] = src[k][m] for the tile of
// rows m in [16 mt, 16 mt + 16) and k in [16 kt, 16 kt + 16); src is
// [kRows][ld] BF16 (zero where m >= valid_m).
template <int LD>
__device__ __forceinline__ void a_frag_t(const __nv_bfloat16* src, int mt, int kt, int lane, uint32_t (&a)[4]) {
  const int g = lane >> 2, t = lane & 3;
  const int m0 = 16 * mt + g, k0 = 16 * kt + 2 * t;
  a[0] = pack_raw(src[(size_t)k0 * LD + m0], src[(size_t)(k0 + 1) * LD + m0]);
  a[1] = pack_raw(src[(size_t)k0 * LD + m0 + 8], src[(size_t)(k0 + 1) * LD + m0 + 8]);
  a[2] = pack_raw(src[(size_t)(k0 + 8) * LD + m0], src[(size_t)(k0 + 9) * LD + m0]);
  a[3] = pack_raw(src[(size_t)(k0 + 8) * LD + m0 + 8], src[(size_t)(k0 + 9) * LD + m0 + 8]);
}
// B fragment B[k][n] = src[k][n], src [kRows][LD] BF16.
template <int LD>
__device__ __forceinline__ void b_frag_rows(const __nv_bfloat16* src, int kt, int nt, int lane, uint32_t& b0, uint32_t& b1) {
  const int g = lane >> 2, t = lane & 3;
  const int n = 8 * nt + g, k0 = 16 * kt + 2 * t;
  b0 = pack_raw(src[(size_t)k0 * LD + n], src[(size_t)(k0 + 1) * LD + n]);
  b1 = pack_raw(src[(size_t)(k0 + 8) * LD + n], src[(size_t)(k0 + 9) * LD + n]);
}

__global__ void __launch_bounds__(kMlpThreads, 1)
    k_mlp_grad(const float* __restrict__ X, const float* __restrict__ Y, int n, const float* __restrict__ prm,
               float inv_n, float* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  GradSmem& S = *reinterpret_cast<GradSmem*>(smem_raw);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  mlp_stage(prm, S.w, kMlpThreads);

  float acc2[4][4], acc1[4], acc3[4];  // dW2t (4 m-tiles of n-tile warp), dW1t block, dW3t n-tile warp
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    acc1[i] = 0.f;
    acc3[i] = 0.f;
#pragma unroll
    for (int j = 0; j < 4; ++j) acc2[i][j] = 0.f;
  }
  float bacc = 0.f;  // bias gradient owned by this thread (b1: 0..63, b2: 64..127, b3: 128..129)
  float lsum = 0.f;

  for (int base = blockIdx.x * kRows; base < n; base += gridDim.x * kRows) {
    __syncthreads();  // previous round's shared data consumed; weights staged
    for (int i = threadIdx.x; i < kRows * kMlpIn; i += kMlpThreads) {
      const int r = i / kMlpIn, c = i % kMlpIn;
      S.x[i] = (base + r < n && c < kMlpFeat) ? X[(size_t)(base + r) * kMlpFeat + c] : 0.f;
    }
    __syncthreads();
    const int r0 = warp * 16;
    MlpTile T;
    mlp_forward_tile(S.x + r0 * kMlpIn, S.w, lane, T);
    // loss and dL/do for rows r0 + g and r0 + g + 8 (lanes with t == 0)
    float d0[2] = {0.f, 0.f}, d1[2] = {0.f, 0.f};
    if (t == 0) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int row = base + r0 + g + 8 * h;
        if (row < n) {
          const float o0 = T.o[2 * h], o1 = T.o[2 * h + 1];
          const float y = Y[2 * (size_t)row], b = Y[2 * (size_t)row + 1];
          const float p = sigmoidf_(o0);
          const float mu = kMuScale * softplusf(o1);
          const float e = (mu - b) / kMuScale;
          // BCE from the logit, stable for large |o0|
          const float bce = fmaxf(o0, 0.f) - o0 * y + log1pf(expf(-fabsf(o0)));
          lsum += bce + y * e * e;
          d0[h] = (p - y) * inv_n;
          d1[h] = y * 2.f * e * sigmoidf_(o1) * inv_n;  // d(e^2)/d(o1) = 2 e * softplus'(o1)
        }
      }
    }
    // dO as an A fragment (cols 0, 1 only) and into shared memory
    uint32_t ad[4];
    ad[0] = pack_bf16(d0[0], d1[0]);
    ad[1] = pack_bf16(d0[1], d1[1]);
    ad[2] = 0u;
    ad[3] = 0u;
    if (t != 0) ad[0] = ad[1] = 0u;
    {
      uint32_t* gr = reinterpret_cast<uint32_t*>(S.go + (size_t)(r0 + g) * 16 + 2 * t);
      uint32_t* gr8 = reinterpret_cast<uint32_t*>(S.go + (size_t)(r0 + g + 8) * 16 + 2 * t);
      gr[0] = ad[0];
      gr8[0] = ad[1];
      *reinterpret_cast<uint32_t*>(S.go + (size_t)(r0 + g) * 16 + 8 + 2 * t) = 0u;
      *reinterpret_cast<uint32_t*>(S.go + (size_t)(r0 + g + 8) * 16 + 8 + 2 * t) = 0u;
    }
    // dH2 = dO W3 (B[k = out][n = hidden] = W3t[out][hidden], zero for out >= 2), masked by ReLU'(H2)
    uint32_t gh2[4][4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      float c[2][4];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int nn = 8 * (2 * q + h) + g;
        const uint32_t b0 = (t == 0) ? pack_raw(S.w.w3t[nn], S.w.w3t[kMlpH + nn]) : 0u;
#pragma unroll
        for (int i = 0; i < 4; ++i) c[h][i] = 0.f;
        mma_bf16(c[h], ad, b0, 0u);
      }
      // mask: the same lane holds H2 at the same (row, col) in fragment q
      gh2[q][0] = pack_bf16(bf(T.h2[q][0], 0) > 0.f ? c[0][0] : 0.f, bf(T.h2[q][0], 1) > 0.f ? c[0][1] : 0.f);
      gh2[q][1] = pack_bf16(bf(T.h2[q][1], 0) > 0.f ? c[0][2] : 0.f, bf(T.h2[q][1], 1) > 0.f ? c[0][3] : 0.f);
      gh2[q][2] = pack_bf16(bf(T.h2[q][2], 0) > 0.f ? c[1][0] : 0.f, bf(T.h2[q][2], 1) > 0.f ? c[1][1] : 0.f);
      gh2[q][3] = pack_bf16(bf(T.h2[q][3], 0) > 0.f ? c[1][2] : 0.f, bf(T.h2[q][3], 1) > 0.f ? c[1][3] : 0.f);
    }
    // dH1 = dH2 W2^T (B[k = out2][n = in2] = W2t[out2][in2]), masked by ReLU'(H1)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      float c[2][4];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int nn = 8 * (2 * q + h) + g;
#pragma unroll
        for (int i = 0; i < 4; ++i) c[h][i] = 0.f;
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
          const int k0 = 16 * kt + 2 * t;
          const uint32_t b0 = pack_raw(S.w.w2t[(size_t)k0 * kMlpH + nn], S.w.w2t[(size_t)(k0 + 1) * kMlpH + nn]);
          const uint32_t b1 = pack_raw(S.w.w2t[(size_t)(k0 + 8) * kMlpH + nn], S.w.w2t[(size_t)(k0 + 9) * kMlpH + nn]);
          mma_bf16(c[h], gh2[kt], b0, b1);
        }
      }
      uint32_t gq[4];
      gq[0] = pack_bf16(bf(T.h1[q][0], 0) > 0.f ? c[0][0] : 0.f, bf(T.h1[q][0], 1) > 0.f ? c[0][1] : 0.f);
      gq[1] = pack_bf16(bf(T.h1[q][1], 0) > 0.f ? c[0][2] : 0.f, bf(T.h1[q][1], 1) > 0.f ? c[0][3] : 0.f);
      gq[2] = pack_bf16(bf(T.h1[q][2], 0) > 0.f ? c[1][0] : 0.f, bf(T.h1[q][2], 1) > 0.f ? c[1][1] : 0.f);
      gq[3] = pack_bf16(bf(T.h1[q][3], 0) > 0.f ? c[1][2] : 0.f, bf(T.h1[q][3], 1) > 0.f ? c[1][3] : 0.f);
      store_frag(S.g1, r0, q, lane, gq);
      store_frag(S.g2, r0, q, lane, gh2[q]);
      store_frag(S.h1, r0, q, lane, T.h1[q]);
      store_frag(S.h2, r0, q, lane, T.h2[q]);
    }
    __syncthreads();
    // weight gradients over the round: dW2t[out][in] = sum_s g2[s][out] h1[s][in]
#pragma unroll
    for (int kt = 0; kt < kRows / 16; ++kt) {
      uint32_t b0, b1;
      b_frag_rows<kMlpH>(S.h1, kt, warp, lane, b0, b1);
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        uint32_t a[4];
        a_frag_t<kMlpH>(S.g2, mt, kt, lane, a);
        mma_bf16(acc2[mt], a, b0, b1);
      }
      // dW1t[out][in] = sum_s g1[s][out] x[s][in]: warp -> (mt = warp / 2, nt = warp % 2)
      {
        uint32_t a[4];
        a_frag_t<kMlpH>(S.g1, warp >> 1, kt, lane, a);
        const int nn = 8 * (warp & 1) + g, k0 = 16 * kt + 2 * t;
        const uint32_t xb0 = pack_bf16(S.x[(size_t)k0 * kMlpIn + nn], S.x[(size_t)(k0 + 1) * kMlpIn + nn]);
        const uint32_t xb1 = pack_bf16(S.x[(size_t)(k0 + 8) * kMlpIn + nn], S.x[(size_t)(k0 + 9) * kMlpIn + nn]);
        mma_bf16(acc1, a, xb0, xb1);
      }
      // dW3t[out][hid] = sum_s go[s][out] h2[s][hid]: rows out 0, 1 of the m-tile
      {
        uint32_t a[4];
        a_frag_t<16>(S.go, 0, kt, lane, a);
        uint32_t hb0, hb1;
        b_frag_rows<kMlpH>(S.h2, kt, warp, lane, hb0, hb1);
        mma_bf16(acc3, a, hb0, hb1);
      }
    }
    // bias gradients: column sums
    if (threadIdx.x < kMlpH) {
      for (int r = 0; r < kRows; ++r) bacc += __bfloat162float(S.g1[(size_t)r * kMlpH + threadIdx.x]);
    } else if (threadIdx.x < 2 * kMlpH) {
      for (int r = 0; r < kRows; ++r) bacc += __bfloat162float(S.g2[(size_t)r * kMlpH + threadIdx.x - kMlpH]);
    } else if (threadIdx.x < 2 * kMlpH + kMlpOut) {
      for (int r = 0; r < kRows; ++r) bacc += __bfloat162float(S.go[(size_t)r * 16 + threadIdx.x - 2 * kMlpH]);
    }
  }
  // per-CTA partial gradient
  float* P = partial + (size_t)blockIdx.x * (kMlpParams + 1);
#pragma unroll
  for (int mt = 0; mt < 4; ++mt) {
    const int o = 16 * mt + g, i = 8 * warp + 2 * t;
    P[kOffW2 + o * kMlpH + i] = acc2[mt][0];
    P[kOffW2 + o * kMlpH + i + 1] = acc2[mt][1];
    P[kOffW2 + (o + 8) * kMlpH + i] = acc2[mt][2];
    P[kOffW2 + (o + 8) * kMlpH + i + 1] = acc2[mt][3];
  }
  {
    const int o = 16 * (warp >> 1) + g, i = 8 * (warp & 1) + 2 * t;
    P[kOffW1 + o * kMlpIn + i] = acc1[0];
    P[kOffW1 + o * kMlpIn + i + 1] = acc1[1];
    P[kOffW1 + (o + 8) * kMlpIn + i] = acc1[2];
    P[kOffW1 + (o + 8) * kMlpIn + i + 1] = acc1[3];
  }
  if (g < kMlpOut) {
    const int i = 8 * warp + 2 * t;
    P[kOffW3 + g * kMlpH + i] = acc3[0];
    P[kOffW3 + g * kMlpH + i + 1] = acc3[1];
  }
  if (threadIdx.x < kMlpH) P[kOffB1 + threadIdx.x] = bacc;
  else if (threadIdx.x < 2 * kMlpH) P[kOffB2 + threadIdx.x - kMlpH] = bacc;
  else if (threadIdx.x < 2 * kMlpH + kMlpOut) P[kOffB3 + threadIdx.x - 2 * kMlpH] = bacc;
  // loss sum (lanes with t == 0 hold row losses)
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if (lane == 0) S.loss[warp] = lsum;
  __syncthreads();
  if (threadIdx.x == 0) {
    float s = 0.f;
    for (int w = 0; w < kMlpThreads / 32; ++w) s += S.loss[w];
    P[kMlpParams] = s;
  }
}

// Sum of the per-CTA partials in CTA order; then either the gradient
// (grad != nullptr) or one Adam step on prm (m, v moments, step >= 1).
__global__ void k_mlp_reduce(const float* __restrict__ partial, int nblk, float* grad, float* prm, float* m, float* v,
                             int step, float lr, float inv_n, float* loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > kMlpParams) return;
  float s = 0.f;
  for (int b = 0; b < nblk; ++b) s += partial[(size_t)b * (kMlpParams + 1) + i];
  if (i == kMlpParams) {
    if (loss) *loss = s * inv_n;
    return;
  }
  if (grad) grad[i] = s;
  if (prm) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float mi = b1 * m[i] + (1.f - b1) * s;
    const float vi = b2 * v[i] + (1.f - b2) * s * s;
    m[i] = mi;
    v[i] = vi;
    const float mh = mi / (1.f - powf(b1, (float)step)), vh = vi / (1.f - powf(b2, (float)step));
    prm[i] -= lr * mh / (sqrtf(vh) + eps);
  }
}

// Inference: (p_nlos, mu) per row.
__global__ void __launch_bounds__(kMlpThreads) k_mlp_forward(const float* __restrict__ X, int n,
                                                              const float* __restrict__ prm, float* __restrict__ out) {
  __shared__ MlpSmem W;
  __shared__ float xs[kRows * kMlpIn];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  mlp_stage(prm, W, kMlpThreads);
  for (int base = blockIdx.x * kRows; base < n; base += gridDim.x * kRows) {
    __syncthreads();
    for (int i = threadIdx.x; i < kRows * kMlpIn; i += kMlpThreads) {
      const int r = i / kMlpIn, c = i % kMlpIn;
      xs[i] = (base + r < n && c < kMlpFeat) ? X[(size_t)(base + r) * kMlpFeat + c] : 0.f;
    }
    __syncthreads();
    MlpTile T;
    mlp_forward_tile(xs + warp * 16 * kMlpIn, W, lane, T);
    if (t == 0) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int row = base + warp * 16 + g + 8 * h;
        if (row < n) {
          out[2 * (size_t)row] = sigmoidf_(T.o[2 * h]);
          out[2 * (size_t)row + 1] = kMuScale * softplusf(T.o[2 * h + 1]);
        }
      }
    }
  }
}

constexpr int kGradBlocks = 64;

}  // namespace pfb

using namespace pfb;

extern "C" {

int pf_mlp_param_count(void) { return kMlpParams; }

size_t pf_mlp_scratch_bytes(void) { return (size_t)kGradBlocks * (kMlpParams + 1) * sizeof(float); }

static int grad_launch(const float* d_x, const float* d_y, int n, const float* d_params, float* d_scratch,
                       int* nblk_out, cudaStream_t st) {
  const int nblk = std::min(kGradBlocks, (n + kRows - 1) / kRows);
  const size_t smem = sizeof(GradSmem);
  cudaError_t e = cudaFuncSetAttribute((const void*)k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return set_err(PF_ECUDA, "mlp grad attribute: %s", cudaGetErrorString(e));
  k_mlp_grad<<<nblk, kMlpThreads, smem, st>>>(d_x, d_y, n, d_params, 1.0f / (float)n, d_scratch);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(PF_ECUDA, "mlp grad launch: %s", cudaGetErrorString(e));
  *nblk_out = nblk;
  return PF_OK;
}

int pf_mlp_grad(const float* d_x, const float* d_y, int n, const float* d_params, float* d_grad, float* d_loss,
                void* d_scratch, size_t scratch_bytes, void* stream) {
  clear_err();
  if (!d_x || !d_y || !d_params || !d_grad || !d_scratch) return set_err(PF_EINVAL, "null pointer");
  if (n <= 0) return set_err(PF_EINVAL, "n must be > 0");
  if (scratch_bytes < pf_mlp_scratch_bytes()) return set_err(PF_EINVAL, "scratch too small");
  cudaStream_t st = (cudaStream_t)stream;
  int nblk = 0, s;
  if ((s = grad_launch(d_x, d_y, n, d_params, (float*)d_scratch, &nblk, st)) != PF_OK) return s;
  k_mlp_reduce<<<(kMlpParams + 256) / 256, 256, 0, st>>>((const float*)d_scratch, nblk, d_grad, nullptr, nullptr,
                                                          nullptr, 0, 0.f, 1.0f / (float)n, d_loss);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PF_OK : set_err(PF_ECUDA, "mlp reduce: %s", cudaGetErrorString(e));
}

int pf_mlp_adam_step(const float* d_x, const float* d_y, int n, float* d_params, float* d_m, float* d_v, int step,
                     float lr, float* d_loss, void* d_scratch, size_t scratch_bytes, void* stream) {
  clear_err();
  if (!d_x || !d_y || !d_params || !d_m || !d_v || !d_scratch) return set_err(PF_EINVAL, "null pointer");
  if (n <= 0 || step < 1 || !(lr > 0.f)) return set_err(PF_EINVAL, "bad n, step or lr");
  if (scratch_bytes < pf_mlp_scratch_bytes()) return set_err(PF_EINVAL, "scratch too small");
  cudaStream_t st = (cudaStream_t)stream;
  int nblk = 0, s;
  if ((s = grad_launch(d_x, d_y, n, d_params, (float*)d_scratch, &nblk, st)) != PF_OK) return s;
  k_mlp_reduce<<<(kMlpParams + 256) / 256, 256, 0, st>>>((const float*)d_scratch, nblk, nullptr, d_params, d_m, d_v,
                                                          step, lr, 1.0f / (float)n, d_loss);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PF_OK : set_err(PF_ECUDA, "mlp adam: %s", cudaGetErrorString(e));
}

int pf_mlp_forward(const float* d_x, int n, const float* d_params, float* d_out, void* stream) {
  clear_err();
  if (!d_x || !d_params || !d_out) return set_err(PF_EINVAL, "null pointer");
  if (n <= 0) return set_err(PF_EINVAL, "n must be > 0");
  const int nblk = std::min(1024, (n + kRows - 1) / kRows);
  k_mlp_forward<<<nblk, kMlpThreads, 0, (cudaStream_t)stream>>>(d_x, n, d_params, d_out);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PF_OK : set_err(PF_ECUDA, "mlp forward: %s", cudaGetErrorString(e));
}

}  // extern "C"
