// pf_mlp.cuh -- the per-satellite NLOS network: 12 -> 64 -> 64 -> 2 with
// ReLU, BF16 operands and FP32 accumulation on the tensor cores
// (mma.sync m16n8k16, one warp per 16 rows).
//
// Outputs per satellite: o0 -> p_nlos = sigmoid(o0), o1 -> mu = 20 m *
// softplus(o1), the mean of the NLOS bias.  Inputs are the 12 features of
// mlp_features() (padded with zeros to 16).
//
// Parameters (FP32 master copy, kMlpParams floats) in the order
//   W1t[64][16] b1[64] W2t[64][64] b2[64] W3t[2][64] b3[2]
// where Wt[out][in] is the transposed weight (column-major B operand).
//
// Why mma.sync and not tcgen05: the network is evaluated per (filter,
// satellite) -- at most 64 rows per filter and epoch inside the epoch
// kernel, 128 rows per CTA round in training.  A tcgen05 MMA is 128 rows
// wide with its accumulator in TMEM; for these shapes the TMEM allocation,
// descriptor set-up and round trip would cost more than the math, which is
// a few hundred register-operand MMAs per CTA.
#pragma once
#include <stdint.h>
#include <cuda_bf16.h>

namespace pfb {

constexpr int kMlpIn = 16;    // padded input width (12 features used)
constexpr int kMlpFeat = 12;
constexpr int kMlpH = 64;
constexpr int kMlpOut = 2;
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpH * kMlpIn;
constexpr int kOffW2 = kOffB1 + kMlpH;
constexpr int kOffB2 = kOffW2 + kMlpH * kMlpH;
constexpr int kOffW3 = kOffB2 + kMlpH;
constexpr int kOffB3 = kOffW3 + kMlpOut * kMlpH;
constexpr int kMlpParams = kOffB3 + kMlpOut;  // 5378
constexpr float kMuScale = 20.0f;             // metres per unit of softplus(o1)

// Two floats -> one register of two BF16 (round to nearest even); the
// first argument goes to the low half.
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}
__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// D = A(16x16, row) * B(16x8, col) + C, BF16 in, FP32 accumulate.
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Weights of one layer as BF16 in shared memory, Wt[out][in] (in
// contiguous).  The B fragment of k-tile kt, n-tile nt for lane (g, t):
// b0 = (Wt[n][k], Wt[n][k+1]) with n = 8 nt + g, k = 16 kt + 2t; b1 at k + 8.
template <int IN>
__device__ __forceinline__ void b_frag(const __nv_bfloat16* wt, int kt, int nt, int lane, uint32_t& b0, uint32_t& b1) {
  const int g = lane >> 2, t = lane & 3;
  const __nv_bfloat16* row = wt + (size_t)(8 * nt + g) * IN + 16 * kt + 2 * t;
  b0 = *reinterpret_cast<const uint32_t*>(row);
  b1 = *reinterpret_cast<const uint32_t*>(row + 8);
}

// Network weights staged in shared memory.
struct MlpSmem {
  __nv_bfloat16 w1t[kMlpH * kMlpIn];
  __nv_bfloat16 w2t[kMlpH * kMlpH];
  __nv_bfloat16 w3t[8 * kMlpH];  // rows 2..7 zero
  float b1[kMlpH];
  float b2[kMlpH];
  float b3[kMlpOut];
};

// All threads of the CTA: FP32 master parameters -> BF16 shared copy.
__device__ __forceinline__ void mlp_stage(const float* __restrict__ prm, MlpSmem& s, int nthreads) {
  for (int i = threadIdx.x; i < kMlpH * kMlpIn; i += nthreads) s.w1t[i] = __float2bfloat16_rn(prm[kOffW1 + i]);
  for (int i = threadIdx.x; i < kMlpH * kMlpH; i += nthreads) s.w2t[i] = __float2bfloat16_rn(prm[kOffW2 + i]);
  for (int i = threadIdx.x; i < 8 * kMlpH; i += nthreads)
    s.w3t[i] = __float2bfloat16_rn(i < kMlpOut * kMlpH ? prm[kOffW3 + i] : 0.0f);
  for (int i = threadIdx.x; i < kMlpH; i += nthreads) {
    s.b1[i] = prm[kOffB1 + i];
    s.b2[i] = prm[kOffB2 + i];
  }
  if (threadIdx.x < kMlpOut) s.b3[threadIdx.x] = prm[kOffB3 + threadIdx.x];
}

// Forward pass of one warp over 16 rows.  x: the warp's input rows in FP32
// (row stride kMlpIn).  Keeps the hidden activations (after ReLU, as the
// BF16 A fragments the next layer used: the C fragment of n-tiles 2q, 2q+1
// is the A fragment of k-tile q) and the output tile, whose cols 0, 1 (o0,
// o1) of rows g and g + 8 sit in the lanes with t == 0.
struct MlpTile {
  uint32_t h1[4][4];  // A fragments of H1 (k-tiles 0..3)
  uint32_t h2[4][4];  // A fragments of H2
  float o[4];         // C fragment of the output tile (cols 0, 1 are o0, o1)
};

// One hidden layer for a pair of n-tiles (2q, 2q+1): c = bias + A * W, then
// ReLU; returns the BF16 A fragment of k-tile q of the next layer.
template <int IN, int KT>
__device__ __forceinline__ void hidden_pair(const uint32_t (&a)[KT][4], const __nv_bfloat16* wt, const float* bias,
                                            int q, int lane, uint32_t (&out)[4]) {
  const int t = lane & 3;
  float c0[4], c1[4];
  {
    const float u0 = bias[16 * q + 2 * t], u1 = bias[16 * q + 2 * t + 1];
    c0[0] = u0; c0[1] = u1; c0[2] = u0; c0[3] = u1;
    const float v0 = bias[16 * q + 8 + 2 * t], v1 = bias[16 * q + 8 + 2 * t + 1];
    c1[0] = v0; c1[1] = v1; c1[2] = v0; c1[3] = v1;
  }
#pragma unroll
  for (int kt = 0; kt < KT; ++kt) {
    uint32_t b0, b1;
    b_frag<IN>(wt, kt, 2 * q, lane, b0, b1);
    mma_bf16(c0, a[kt], b0, b1);
    b_frag<IN>(wt, kt, 2 * q + 1, lane, b0, b1);
    mma_bf16(c1, a[kt], b0, b1);
  }
  out[0] = pack_bf16(fmaxf(c0[0], 0.f), fmaxf(c0[1], 0.f));
  out[1] = pack_bf16(fmaxf(c0[2], 0.f), fmaxf(c0[3], 0.f));
  out[2] = pack_bf16(fmaxf(c1[0], 0.f), fmaxf(c1[1], 0.f));
  out[3] = pack_bf16(fmaxf(c1[2], 0.f), fmaxf(c1[3], 0.f));
}

__device__ __forceinline__ void mlp_forward_tile(const float* x, const MlpSmem& s, int lane, MlpTile& T) {
  const int g = lane >> 2, t = lane & 3;
  uint32_t a[1][4];
  a[0][0] = pack_bf16(x[g * kMlpIn + 2 * t], x[g * kMlpIn + 2 * t + 1]);
  a[0][1] = pack_bf16(x[(g + 8) * kMlpIn + 2 * t], x[(g + 8) * kMlpIn + 2 * t + 1]);
  a[0][2] = pack_bf16(x[g * kMlpIn + 2 * t + 8], x[g * kMlpIn + 2 * t + 9]);
  a[0][3] = pack_bf16(x[(g + 8) * kMlpIn + 2 * t + 8], x[(g + 8) * kMlpIn + 2 * t + 9]);
#pragma unroll
  for (int q = 0; q < 4; ++q) hidden_pair<kMlpIn, 1>(a, s.w1t, s.b1, q, lane, T.h1[q]);
#pragma unroll
  for (int q = 0; q < 4; ++q) hidden_pair<kMlpH, 4>(T.h1, s.w2t, s.b2, q, lane, T.h2[q]);
  // layer 3: one n-tile, outputs in cols 0, 1 (rows 2..7 of W3t are zero)
  const float bo0 = (t == 0) ? s.b3[0] : 0.0f, bo1 = (t == 0) ? s.b3[1] : 0.0f;
  T.o[0] = bo0; T.o[1] = bo1; T.o[2] = bo0; T.o[3] = bo1;
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
    uint32_t b0, b1;
    b_frag<kMlpH>(s.w3t, kt, 0, lane, b0, b1);
    mma_bf16(T.o, T.h2[kt], b0, b1);
  }
}

__device__ __forceinline__ float softplusf(float x) { return x > 20.0f ? x : log1pf(expf(x)); }
__device__ __forceinline__ float sigmoidf_(float x) { return 1.0f / (1.0f + expf(-x)); }

}  // namespace pfb
