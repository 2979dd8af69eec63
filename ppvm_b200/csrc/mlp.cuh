// mlp.cuh — the term-priority network of learned truncation: 8 -> 64 -> 64 -> 1, GELU,
// BF16 weights and activations on the tensor cores (mma.sync m16n8k16, FP32 accumulate).
//
// A warp evaluates 16 terms at a time.  Layer 1 multiplies the 16 x 16 feature tile (8
// features, zero padded) by W1^T; the FP32 accumulator fragments of one layer are re-packed
// in registers as the BF16 A fragments of the next (n-tiles 2k and 2k+1 of a 16 x 8 output
// are exactly k-slice k of the next layer's 16 x 16 A operand), so activations never leave
// the registers; layer 3 (64 -> 1) is a quad-shuffle dot product.
//
// Parameters (FP32 master copy, flat): W1[64][8], b1[64], W2[64][64], b2[64], w3[64], b3.
// The device copy used by the kernels: W1 as BF16 [64][16] (k padded), W2 as BF16 [64][64]
// ([out][in]) and its transpose W2T [in][out] (for the backward pass), b1, b2, w3, b3 FP32.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace ppvm {

constexpr int kMlpIn = 8;
constexpr int kMlpK1 = 16;
constexpr int kMlpH = 64;
constexpr int kMlpParams = kMlpH * kMlpIn + kMlpH + kMlpH * kMlpH + kMlpH + kMlpH + 1;  // 4801
// offsets in the flat FP32 parameter vector
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kMlpH * kMlpIn, kOffW2 = kOffB1 + kMlpH,
              kOffB2 = kOffW2 + kMlpH * kMlpH, kOffW3 = kOffB2 + kMlpH, kOffB3 = kOffW3 + kMlpH;

// Device weights (what k_adam writes after every step).
struct MlpWeights {
  __nv_bfloat16 w1[kMlpH * kMlpK1];
  __nv_bfloat16 w2[kMlpH * kMlpH];
  __nv_bfloat16 w2t[kMlpH * kMlpH];
  float b1[kMlpH], b2[kMlpH], w3[kMlpH];
  float b3;
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// GELU (erf form) and its derivative.
__device__ __forceinline__ float gelu_f(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.3989422804014327f * expf(-0.5f * x * x);
}

// Per-warp activations of a 16-row tile, in accumulator-fragment layout: tile j covers
// output columns 8j..8j+7; element e of thread (g = lane/4, t = lane%4) is row g + 8*(e/2),
// column 8j + 2t + (e%2).
struct MlpTile {
  float z1[8][4], z2[8][4];  // pre-activations (kept for the backward pass)
  float h2[8][4];            // layer-2 activations
  float y[2];                // outputs of rows g and g+8 (valid in every lane of the quad)
};

// A fragment (16 x 16, row-major) from a BF16 tile in shared memory with row stride ld.
__device__ __forceinline__ void load_a(uint32_t (&a)[4], const __nv_bfloat16* s, int ld, int k0) {
  const int g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
  a[0] = *reinterpret_cast<const uint32_t*>(s + g * ld + k0 + 2 * t);
  a[1] = *reinterpret_cast<const uint32_t*>(s + (g + 8) * ld + k0 + 2 * t);
  a[2] = *reinterpret_cast<const uint32_t*>(s + g * ld + k0 + 2 * t + 8);
  a[3] = *reinterpret_cast<const uint32_t*>(s + (g + 8) * ld + k0 + 2 * t + 8);
}

// Forward pass of one warp over a 16-row feature tile X (BF16, [16][16] in shared memory).
// W: the weights in shared memory.
__device__ __forceinline__ void mlp_forward(const __nv_bfloat16* X, const MlpWeights& W, MlpTile& T) {
  const int g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
  uint32_t a[4];
  load_a(a, X, kMlpK1, 0);
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const float bl = W.b1[8 * j + 2 * t], bh = W.b1[8 * j + 2 * t + 1];
    T.z1[j][0] = bl;
    T.z1[j][1] = bh;
    T.z1[j][2] = bl;
    T.z1[j][3] = bh;
    const __nv_bfloat16* wr = W.w1 + (8 * j + g) * kMlpK1;
    mma_bf16(T.z1[j], a, *reinterpret_cast<const uint32_t*>(wr + 2 * t),
             *reinterpret_cast<const uint32_t*>(wr + 2 * t + 8));
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const float bl = W.b2[8 * j + 2 * t], bh = W.b2[8 * j + 2 * t + 1];
    T.z2[j][0] = bl;
    T.z2[j][1] = bh;
    T.z2[j][2] = bl;
    T.z2[j][3] = bh;
  }
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    uint32_t h[4];
    h[0] = pack_bf16(gelu_f(T.z1[2 * kk][0]), gelu_f(T.z1[2 * kk][1]));
    h[1] = pack_bf16(gelu_f(T.z1[2 * kk][2]), gelu_f(T.z1[2 * kk][3]));
    h[2] = pack_bf16(gelu_f(T.z1[2 * kk + 1][0]), gelu_f(T.z1[2 * kk + 1][1]));
    h[3] = pack_bf16(gelu_f(T.z1[2 * kk + 1][2]), gelu_f(T.z1[2 * kk + 1][3]));
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const __nv_bfloat16* wr = W.w2 + (8 * j + g) * kMlpH + 16 * kk;
      mma_bf16(T.z2[j], h, *reinterpret_cast<const uint32_t*>(wr + 2 * t),
               *reinterpret_cast<const uint32_t*>(wr + 2 * t + 8));
    }
  }
  float p0 = 0.f, p1 = 0.f;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const float wl = W.w3[8 * j + 2 * t], wh = W.w3[8 * j + 2 * t + 1];
#pragma unroll
    for (int e = 0; e < 4; ++e) T.h2[j][e] = gelu_f(T.z2[j][e]);
    p0 += T.h2[j][0] * wl + T.h2[j][1] * wh;
    p1 += T.h2[j][2] * wl + T.h2[j][3] * wh;
  }
  p0 += __shfl_xor_sync(0xffffffffu, p0, 1);
  p0 += __shfl_xor_sync(0xffffffffu, p0, 2);
  p1 += __shfl_xor_sync(0xffffffffu, p1, 1);
  p1 += __shfl_xor_sync(0xffffffffu, p1, 2);
  T.y[0] = p0 + W.b3;
  T.y[1] = p1 + W.b3;
}

// Term features of learned truncation on an L x L lattice (qubit r*L + c), 8 values:
//   weight/16, (log10|c| + 6)/6, layers_left/8, #X/8, #Y/8, #Z/8,
//   nearest-neighbour bonds inside the support/8, weight*layers_left/64 (the support's
//   overlap with the remaining RX layers, which act on every qubit).
template <int W>
__device__ __forceinline__ void term_features(const uint64_t (&x)[W], const uint64_t (&z)[W], double c, int L,
                                              int layers_left, float (&f)[kMlpIn]) {
  int nx = 0, ny = 0, nz = 0, bonds = 0;
#pragma unroll
  for (int w = 0; w < W; ++w) {
    nx += __popcll(x[w] & ~z[w]);
    ny += __popcll(x[w] & z[w]);
    nz += __popcll(~x[w] & z[w]);
  }
  const int wt = nx + ny + nz;
#pragma unroll
  for (int w = 0; w < W; ++w) {
    uint64_t m = x[w] | z[w];
    while (m) {
      const int q = w * 64 + __ffsll((long long)m) - 1;
      m &= m - 1;
      const int col = L > 0 ? q % L : 0;
      const int r = q + 1, d = q + L;
      if (L > 0 && col + 1 < L && r < 64 * W && (((x[r >> 6] | z[r >> 6]) >> (r & 63)) & 1ull)) ++bonds;
      if (L > 0 && d < 64 * W && (((x[d >> 6] | z[d >> 6]) >> (d & 63)) & 1ull)) ++bonds;
    }
  }
  const double a = fabs(c);
  const float lg = a > 0.0 ? (float)log10(a) : -30.0f;
  f[0] = wt * (1.0f / 16);
  f[1] = (lg + 6.0f) * (1.0f / 6);
  f[2] = layers_left * (1.0f / 8);
  f[3] = nx * (1.0f / 8);
  f[4] = ny * (1.0f / 8);
  f[5] = nz * (1.0f / 8);
  f[6] = bonds * (1.0f / 8);
  f[7] = wt * layers_left * (1.0f / 64);
}

// Order-preserving map of a float score to u32 (larger score -> larger key).
__device__ __forceinline__ uint32_t score_key(float s) {
  const uint32_t b = __float_as_uint(s);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

}  // namespace ppvm
