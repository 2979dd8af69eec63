// learned.cu — the term-priority network of learned truncation: parameters, training
// (forward, backward and Adam as hand-written kernels, BF16 tensor cores with FP32
// accumulation) and batch prediction.  The network scores a term by the predicted
// log10 |contribution| of the term to <O> at the end of the circuit; ppvm_truncate_budget
// (engine.cu) uses the score as the priority of a term-budget truncation.
//
// No counterpart in the reference: ppvm truncates by |coefficient| and Pauli weight only
// (crates/ppvm-pauli-sum/src/strategy.rs:12-170).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ppvm_cuda.h"
#include "mlp.cuh"

namespace ppvm {
void set_last_error(const std::string& msg);
}

using namespace ppvm;

struct ppvm_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  float* params = nullptr;  // FP32 master copy (flat)
  float* m = nullptr;       // Adam moments
  float* v = nullptr;
  float* grads = nullptr;
  float* loss = nullptr;    // [0] = sum of squared errors of the last pass
  float* slabs = nullptr;   // [kMaxTrainBlocks][kSlab]: per-block gradient partials + loss
  MlpWeights* w = nullptr;  // packed device weights
  int step = 0;
  float* d_feats = nullptr;  // training / prediction inputs (grown on demand)
  float* d_tgt = nullptr;
  uint32_t* d_order = nullptr;
  float* d_out = nullptr;
  size_t data_cap = 0;
};

namespace ppvm {
const MlpWeights* mlp_device_weights(const ppvm_mlp* m) { return m ? m->w : nullptr; }
int mlp_device(const ppvm_mlp* m) { return m ? m->device : -1; }
}  // namespace ppvm

namespace {

constexpr int kTrainWarps = 4;
constexpr int kMaxTrainBlocks = 296;
constexpr int kSlab = (kMlpParams + 1 + 3) & ~3;  // the parameters' gradients, then the block's loss

ppvm_status mfail(ppvm_status s, const std::string& msg) {
  ppvm::set_last_error(msg);
  return s;
}

#define MCUDA(expr)                                                                          \
  do {                                                                                       \
    cudaError_t e_ = (expr);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return mfail(e_ == cudaErrorMemoryAllocation ? PPVM_ECAPACITY : PPVM_ECUDA,            \
                   std::string(#expr) + ": " + cudaGetErrorString(e_));                      \
  } while (0)

#define MTRY(expr)                \
  do {                            \
    ppvm_status s_ = (expr);      \
    if (s_ != PPVM_OK) return s_; \
  } while (0)

// FP32 master parameters -> packed BF16/FP32 device weights.
__global__ void k_mlp_pack(const float* p, MlpWeights* w) {
  for (int i = threadIdx.x; i < kMlpH * kMlpK1; i += blockDim.x) {
    const int n = i / kMlpK1, k = i % kMlpK1;
    w->w1[i] = __float2bfloat16_rn(k < kMlpIn ? p[kOffW1 + n * kMlpIn + k] : 0.0f);
  }
  for (int i = threadIdx.x; i < kMlpH * kMlpH; i += blockDim.x) {
    const int n = i / kMlpH, k = i % kMlpH;
    const __nv_bfloat16 b = __float2bfloat16_rn(p[kOffW2 + i]);
    w->w2[i] = b;
    w->w2t[k * kMlpH + n] = b;
  }
  for (int i = threadIdx.x; i < kMlpH; i += blockDim.x) {
    w->b1[i] = p[kOffB1 + i];
    w->b2[i] = p[kOffB2 + i];
    w->w3[i] = p[kOffW3 + i];
  }
  if (threadIdx.x == 0) w->b3 = p[kOffB3];
}

// Adam on the flat parameter vector, one thread per parameter: the minibatch gradient (the
// training blocks' slabs summed in block order), the update, and the parameter's own packed
// copies written (W1's zero padding is set once by k_mlp_pack), so no thread waits for another.
__global__ void __launch_bounds__(256) k_mlp_adam(float* p, float* m, float* v, const float* slabs, int nslabs,
                                                  float* loss, MlpWeights* w, float lr_t, float b1, float b2,
                                                  float eps) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > kMlpParams) return;
  float gi = 0.0f;  // the minibatch gradient: slabs summed in block order
  for (int b = 0; b < nslabs; ++b) gi += slabs[(size_t)b * kSlab + i];
  if (i == kMlpParams) {  // the loss slot
    *loss += gi;
    return;
  }
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float pi = p[i] - lr_t * mi / (sqrtf(vi) + eps);
  p[i] = pi;
  if (i < kOffB1) {
    const int n = (i - kOffW1) / kMlpIn, k = (i - kOffW1) % kMlpIn;
    w->w1[n * kMlpK1 + k] = __float2bfloat16_rn(pi);
  } else if (i < kOffW2) {
    w->b1[i - kOffB1] = pi;
  } else if (i < kOffB2) {
    const int n = (i - kOffW2) / kMlpH, k = (i - kOffW2) % kMlpH;
    const __nv_bfloat16 b = __float2bfloat16_rn(pi);
    w->w2[n * kMlpH + k] = b;
    w->w2t[k * kMlpH + n] = b;
  } else if (i < kOffW3) {
    w->b2[i - kOffB2] = pi;
  } else if (i < kOffB3) {
    w->w3[i - kOffW3] = pi;
  } else {
    w->b3 = pi;
  }
}

// Stages the features of rows [r0, r0+16) of the sample list into a BF16 [16][16] tile.
__device__ __forceinline__ void stage_features(__nv_bfloat16* sX, const float* feats, const uint32_t* order,
                                               unsigned long long r0, unsigned long long rend) {
  const int lane = threadIdx.x & 31;
  for (int e = lane; e < 16 * kMlpK1; e += 32) {
    const int r = e / kMlpK1, k = e % kMlpK1;
    float v = 0.0f;
    const unsigned long long row = r0 + r;
    if (k < kMlpIn && row < rend) {
      const unsigned long long s = order ? order[row] : row;
      v = feats[s * kMlpIn + k];
    }
    sX[e] = __float2bfloat16_rn(v);
  }
  __syncwarp();
}

__device__ __forceinline__ uint32_t pack2(const __nv_bfloat16 lo, const __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// Sums a per-thread column partial over the 8 row groups of the warp (lanes with equal t)
// and adds it to the CTA gradient: cols 8j + 2t, 8j + 2t + 1 of vector `off`.
__device__ __forceinline__ void add_cols(float* sG, int off, int j, float lo, float hi) {
  lo += __shfl_xor_sync(0xffffffffu, lo, 4);
  lo += __shfl_xor_sync(0xffffffffu, lo, 8);
  lo += __shfl_xor_sync(0xffffffffu, lo, 16);
  hi += __shfl_xor_sync(0xffffffffu, hi, 4);
  hi += __shfl_xor_sync(0xffffffffu, hi, 8);
  hi += __shfl_xor_sync(0xffffffffu, hi, 16);
  const int lane = threadIdx.x & 31;
  if (lane < 4) {  // the warp's own gradient copy: each entry always written by the same lane
    sG[off + 8 * j + 2 * lane] += lo;
    sG[off + 8 * j + 2 * lane + 1] += hi;
  }
}

// Forward + backward over samples order[start .. start+count) of (feats, targets): squared
// error loss scaled by inv_n.  Deterministic: every warp accumulates into its own gradient copy
// (each entry always updated by the same lane), the block sums its warps' copies in a fixed
// order into its slab (slabs[blockIdx.x]: gradients, then the loss), and the consumer sums the
// slabs in block order.
__global__ void __launch_bounds__(kTrainWarps * 32)
k_mlp_train(const MlpWeights* Wg, const float* feats, const float* targets, const uint32_t* order,
            unsigned long long start, unsigned long long count, float inv_n, float* slabs) {
  extern __shared__ __align__(16) unsigned char smem[];
  MlpWeights& W = *reinterpret_cast<MlpWeights*>(smem);
  float* sG0 = reinterpret_cast<float*>(smem + sizeof(MlpWeights));  // kTrainWarps copies of kSlab
  __nv_bfloat16* sX0 = reinterpret_cast<__nv_bfloat16*>(sG0 + kTrainWarps * kSlab);
  __shared__ float s_loss[kTrainWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  __nv_bfloat16* sX = sX0 + warp * (16 * kMlpK1 + 2 * 16 * kMlpH);
  float* sG = sG0 + warp * kSlab;
  __nv_bfloat16* sD = sX + 16 * kMlpK1;  // [16][64]: dZ2, later dZ1
  __nv_bfloat16* sH = sD + 16 * kMlpH;   // [16][64]: H1
  {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(Wg);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&W);
    for (int i = threadIdx.x; i < (int)(sizeof(MlpWeights) / 4); i += blockDim.x) dst[i] = src[i];
    for (int i = threadIdx.x; i < kTrainWarps * kSlab; i += blockDim.x) sG0[i] = 0.0f;
  }
  __syncthreads();
  float lsum = 0.0f;
  const unsigned long long end = start + count;
  const unsigned long long ntiles = (count + 15) / 16;
  for (unsigned long long tile = (unsigned long long)blockIdx.x * kTrainWarps + warp; tile < ntiles;
       tile += (unsigned long long)gridDim.x * kTrainWarps) {
    const unsigned long long r0 = start + tile * 16;
    stage_features(sX, feats, order, r0, end);
    MlpTile T;
    mlp_forward(sX, W, T);
    // output error of rows g and g+8
    float dy[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const unsigned long long row = r0 + g + 8 * h;
      float d = 0.0f;
      if (row < end) {
        const float tg = targets[order ? order[row] : row];
        const float e = T.y[h] - tg;
        if (t == 0) lsum += e * e;
        d = 2.0f * e * inv_n;
      }
      dy[h] = d;
    }
    // layer 3: dW3 = sum dy h2, db3 = sum dy; layer-2 pre-activation gradient dZ2
    float dz2[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      add_cols(sG, kOffW3, j, dy[0] * T.h2[j][0] + dy[1] * T.h2[j][2], dy[0] * T.h2[j][1] + dy[1] * T.h2[j][3]);
      const float wl = W.w3[8 * j + 2 * t], wh = W.w3[8 * j + 2 * t + 1];
      dz2[j][0] = dy[0] * wl * gelu_grad(T.z2[j][0]);
      dz2[j][1] = dy[0] * wh * gelu_grad(T.z2[j][1]);
      dz2[j][2] = dy[1] * wl * gelu_grad(T.z2[j][2]);
      dz2[j][3] = dy[1] * wh * gelu_grad(T.z2[j][3]);
      add_cols(sG, kOffB2, j, dz2[j][0] + dz2[j][2], dz2[j][1] + dz2[j][3]);
    }
    {
      float s = (t == 0) ? dy[0] + dy[1] : 0.0f;
#pragma unroll
      for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) sG[kOffB3] += s;
    }
    // stage dZ2 and H1 (BF16, row-major [16][64]) for the weight gradient of layer 2
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c = 8 * j + 2 * t;
      sD[g * kMlpH + c] = __float2bfloat16_rn(dz2[j][0]);
      sD[g * kMlpH + c + 1] = __float2bfloat16_rn(dz2[j][1]);
      sD[(g + 8) * kMlpH + c] = __float2bfloat16_rn(dz2[j][2]);
      sD[(g + 8) * kMlpH + c + 1] = __float2bfloat16_rn(dz2[j][3]);
      sH[g * kMlpH + c] = __float2bfloat16_rn(gelu_f(T.z1[j][0]));
      sH[g * kMlpH + c + 1] = __float2bfloat16_rn(gelu_f(T.z1[j][1]));
      sH[(g + 8) * kMlpH + c] = __float2bfloat16_rn(gelu_f(T.z1[j][2]));
      sH[(g + 8) * kMlpH + c + 1] = __float2bfloat16_rn(gelu_f(T.z1[j][3]));
    }
    __syncwarp();
    // dW2[n][k] += sum_r dZ2[r][n] H1[r][k]: A = dZ2^T (64 x 16), B = H1 (16 x 64)
#pragma unroll 1
    for (int mt = 0; mt < 4; ++mt) {
      uint32_t a[4];
      const int n0 = 16 * mt + g;
      a[0] = pack2(sD[(2 * t) * kMlpH + n0], sD[(2 * t + 1) * kMlpH + n0]);
      a[1] = pack2(sD[(2 * t) * kMlpH + n0 + 8], sD[(2 * t + 1) * kMlpH + n0 + 8]);
      a[2] = pack2(sD[(2 * t + 8) * kMlpH + n0], sD[(2 * t + 9) * kMlpH + n0]);
      a[3] = pack2(sD[(2 * t + 8) * kMlpH + n0 + 8], sD[(2 * t + 9) * kMlpH + n0 + 8]);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int k0 = 8 * j + g;
        const uint32_t b0 = pack2(sH[(2 * t) * kMlpH + k0], sH[(2 * t + 1) * kMlpH + k0]);
        const uint32_t b1 = pack2(sH[(2 * t + 8) * kMlpH + k0], sH[(2 * t + 9) * kMlpH + k0]);
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        mma_bf16(acc, a, b0, b1);
        const int col = 8 * j + 2 * t;
        sG[kOffW2 + n0 * kMlpH + col] += acc[0];
        sG[kOffW2 + n0 * kMlpH + col + 1] += acc[1];
        sG[kOffW2 + (n0 + 8) * kMlpH + col] += acc[2];
        sG[kOffW2 + (n0 + 8) * kMlpH + col + 1] += acc[3];
      }
    }
    // dH1 = dZ2 W2 (A from the dZ2 fragments, B = W2T), dZ1 = dH1 * gelu'(Z1)
    float dz1[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) dz1[j][e] = 0.0f;
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      uint32_t a[4];
      a[0] = pack_bf16(dz2[2 * kk][0], dz2[2 * kk][1]);
      a[1] = pack_bf16(dz2[2 * kk][2], dz2[2 * kk][3]);
      a[2] = pack_bf16(dz2[2 * kk + 1][0], dz2[2 * kk + 1][1]);
      a[3] = pack_bf16(dz2[2 * kk + 1][2], dz2[2 * kk + 1][3]);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const __nv_bfloat16* wr = W.w2t + (8 * j + g) * kMlpH + 16 * kk;
        mma_bf16(dz1[j], a, *reinterpret_cast<const uint32_t*>(wr + 2 * t),
                 *reinterpret_cast<const uint32_t*>(wr + 2 * t + 8));
      }
    }
    __syncwarp();  // every lane has read sD before it is overwritten with dZ1
#pragma unroll
    for (int j = 0; j < 8; ++j) {
#pragma unroll
      for (int e = 0; e < 4; ++e) dz1[j][e] *= gelu_grad(T.z1[j][e]);
      add_cols(sG, kOffB1, j, dz1[j][0] + dz1[j][2], dz1[j][1] + dz1[j][3]);
      const int c = 8 * j + 2 * t;
      sD[g * kMlpH + c] = __float2bfloat16_rn(dz1[j][0]);
      sD[g * kMlpH + c + 1] = __float2bfloat16_rn(dz1[j][1]);
      sD[(g + 8) * kMlpH + c] = __float2bfloat16_rn(dz1[j][2]);
      sD[(g + 8) * kMlpH + c + 1] = __float2bfloat16_rn(dz1[j][3]);
    }
    __syncwarp();
    // dW1[n][k] += sum_r dZ1[r][n] X[r][k]: A = dZ1^T (64 x 16), B = X (16 x 8 real columns)
#pragma unroll 1
    for (int mt = 0; mt < 4; ++mt) {
      uint32_t a[4];
      const int n0 = 16 * mt + g;
      a[0] = pack2(sD[(2 * t) * kMlpH + n0], sD[(2 * t + 1) * kMlpH + n0]);
      a[1] = pack2(sD[(2 * t) * kMlpH + n0 + 8], sD[(2 * t + 1) * kMlpH + n0 + 8]);
      a[2] = pack2(sD[(2 * t + 8) * kMlpH + n0], sD[(2 * t + 9) * kMlpH + n0]);
      a[3] = pack2(sD[(2 * t + 8) * kMlpH + n0 + 8], sD[(2 * t + 9) * kMlpH + n0 + 8]);
      const uint32_t b0 = pack2(sX[(2 * t) * kMlpK1 + g], sX[(2 * t + 1) * kMlpK1 + g]);
      const uint32_t b1 = pack2(sX[(2 * t + 8) * kMlpK1 + g], sX[(2 * t + 9) * kMlpK1 + g]);
      float acc[4] = {0.f, 0.f, 0.f, 0.f};
      mma_bf16(acc, a, b0, b1);
      sG[kOffW1 + n0 * kMlpIn + 2 * t] += acc[0];
      sG[kOffW1 + n0 * kMlpIn + 2 * t + 1] += acc[1];
      sG[kOffW1 + (n0 + 8) * kMlpIn + 2 * t] += acc[2];
      sG[kOffW1 + (n0 + 8) * kMlpIn + 2 * t + 1] += acc[3];
    }
    __syncwarp();  // sX, sD and sH are rewritten by the next tile
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if (lane == 0) s_loss[warp] = lsum;
  __syncthreads();
  float* slab = slabs + (size_t)blockIdx.x * kSlab;
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) {
    float v = sG0[i];
#pragma unroll
    for (int w = 1; w < kTrainWarps; ++w) v += sG0[w * kSlab + i];
    slab[i] = v;
  }
  if (threadIdx.x == 0) {
    float l = s_loss[0];
    for (int w = 1; w < kTrainWarps; ++w) l += s_loss[w];
    slab[kMlpParams] = l;
  }
}

// Sums the slabs of k_mlp_train's blocks in block order: the gradient (one thread per
// parameter), and the loss into *loss (thread kMlpParams).
__global__ void __launch_bounds__(256) k_mlp_reduce(const float* slabs, int nslabs, float* grads, float* loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > kMlpParams) return;
  float v = 0.0f;
  for (int b = 0; b < nslabs; ++b) v += slabs[(size_t)b * kSlab + i];
  if (i < kMlpParams) grads[i] = v;
  else *loss += v;
}

// Scores of n feature rows (one warp per 16 rows).
__global__ void __launch_bounds__(128) k_mlp_predict(const MlpWeights* Wg, const float* feats, unsigned long long n,
                                                     float* out) {
  __shared__ MlpWeights W;
  __shared__ __nv_bfloat16 sX[4][16 * kMlpK1];
  {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(Wg);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&W);
    for (int i = threadIdx.x; i < (int)(sizeof(MlpWeights) / 4); i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const unsigned long long ntiles = (n + 15) / 16;
  for (unsigned long long tile = (unsigned long long)blockIdx.x * 4 + warp; tile < ntiles;
       tile += (unsigned long long)gridDim.x * 4) {
    stage_features(sX[warp], feats, nullptr, tile * 16, n);
    MlpTile T;
    mlp_forward(sX[warp], W, T);
    if (t == 0) {
      if (tile * 16 + g < n) out[tile * 16 + g] = T.y[0];
      if (tile * 16 + g + 8 < n) out[tile * 16 + g + 8] = T.y[1];
    }
    __syncwarp();
  }
}

size_t train_smem() {
  return sizeof(MlpWeights) + sizeof(float) * kTrainWarps * kSlab +
         sizeof(__nv_bfloat16) * kTrainWarps * (16 * kMlpK1 + 2 * 16 * kMlpH);
}

ppvm_status ensure_data(ppvm_mlp* m, size_t n) {
  if (n <= m->data_cap) return PPVM_OK;
  cudaFree(m->d_feats);
  cudaFree(m->d_tgt);
  cudaFree(m->d_order);
  cudaFree(m->d_out);
  m->d_feats = nullptr;
  m->d_tgt = nullptr;
  m->d_order = nullptr;
  m->d_out = nullptr;
  m->data_cap = 0;
  MCUDA(cudaMalloc(&m->d_feats, sizeof(float) * kMlpIn * n));
  MCUDA(cudaMalloc(&m->d_tgt, sizeof(float) * n));
  MCUDA(cudaMalloc(&m->d_order, sizeof(uint32_t) * n));
  MCUDA(cudaMalloc(&m->d_out, sizeof(float) * n));
  m->data_cap = n;
  return PPVM_OK;
}

// Forward + backward of one minibatch into the slabs; *nslabs = the number of slabs written.
ppvm_status launch_train(ppvm_mlp* m, bool use_order, unsigned long long start, unsigned long long count, float inv_n,
                         int* nslabs) {
  static unsigned long long attr = 0;
  if (!((attr >> m->device) & 1ull)) {
    MCUDA(cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)train_smem()));
    attr |= 1ull << m->device;
  }
  const unsigned long long tiles = (count + 15) / 16;
  const unsigned grid = (unsigned)std::max<unsigned long long>(
      1, std::min<unsigned long long>((tiles + kTrainWarps - 1) / kTrainWarps, kMaxTrainBlocks));
  k_mlp_train<<<grid, kTrainWarps * 32, train_smem(), m->stream>>>(m->w, m->d_feats, m->d_tgt,
                                                                   use_order ? m->d_order : nullptr, start, count,
                                                                   inv_n, m->slabs);
  MCUDA(cudaGetLastError());
  *nslabs = (int)grid;
  return PPVM_OK;
}

uint64_t splitmix(uint64_t& s) {
  s += 0x9E3779B97F4A7C15ull;
  uint64_t z = s;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

extern "C" {

ppvm_status ppvm_mlp_destroy(ppvm_mlp* m) {
  if (!m) return PPVM_OK;
  cudaSetDevice(m->device);
  if (m->stream) cudaStreamSynchronize(m->stream);
  cudaFree(m->params);
  cudaFree(m->m);
  cudaFree(m->v);
  cudaFree(m->grads);
  cudaFree(m->loss);
  cudaFree(m->slabs);
  cudaFree(m->w);
  cudaFree(m->d_feats);
  cudaFree(m->d_tgt);
  cudaFree(m->d_order);
  cudaFree(m->d_out);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
  return PPVM_OK;
}

ppvm_status ppvm_mlp_set_params(ppvm_mlp* m, const float* params, size_t n) {
  if (!m || !params || n != (size_t)kMlpParams) return mfail(PPVM_EINVAL, "need the 4801 network parameters");
  MCUDA(cudaSetDevice(m->device));
  MCUDA(cudaMemcpyAsync(m->params, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice, m->stream));
  MCUDA(cudaMemsetAsync(m->m, 0, sizeof(float) * kMlpParams, m->stream));
  MCUDA(cudaMemsetAsync(m->v, 0, sizeof(float) * kMlpParams, m->stream));
  k_mlp_pack<<<1, 256, 0, m->stream>>>(m->params, m->w);
  MCUDA(cudaGetLastError());
  MCUDA(cudaStreamSynchronize(m->stream));
  m->step = 0;
  return PPVM_OK;
}

ppvm_status ppvm_mlp_get_params(const ppvm_mlp* m, float* params, size_t n) {
  if (!m || !params || n != (size_t)kMlpParams) return mfail(PPVM_EINVAL, "need room for 4801 parameters");
  MCUDA(cudaSetDevice(m->device));
  MCUDA(cudaMemcpyAsync(params, m->params, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost, m->stream));
  MCUDA(cudaStreamSynchronize(m->stream));
  return PPVM_OK;
}

ppvm_status ppvm_mlp_create(ppvm_mlp** out, uint64_t seed, int device) {
  if (!out) return mfail(PPVM_EINVAL, "null out pointer");
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) return mfail(PPVM_ENODEV, std::string("no CUDA device: ") + cudaGetErrorString(e));
  if (device < 0 || device >= count) return mfail(PPVM_EINVAL, "device ordinal out of range");
  MCUDA(cudaSetDevice(device));
  ppvm_mlp* m = new ppvm_mlp();
  m->device = device;
  if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&m->params, sizeof(float) * kMlpParams) != cudaSuccess ||
      cudaMalloc(&m->m, sizeof(float) * kMlpParams) != cudaSuccess ||
      cudaMalloc(&m->v, sizeof(float) * kMlpParams) != cudaSuccess ||
      cudaMalloc(&m->grads, sizeof(float) * kMlpParams) != cudaSuccess ||
      cudaMalloc(&m->loss, sizeof(float)) != cudaSuccess || cudaMalloc(&m->w, sizeof(MlpWeights)) != cudaSuccess ||
      cudaMalloc(&m->slabs, sizeof(float) * kSlab * kMaxTrainBlocks) != cudaSuccess) {
    ppvm_mlp_destroy(m);
    return mfail(PPVM_ECAPACITY, "device allocation failed");
  }
  // uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights, zero biases (seeded splitmix64)
  std::vector<float> p(kMlpParams, 0.0f);
  uint64_t s = seed;
  auto u = [&](float a) { return (float)(((splitmix(s) >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0) * a; };
  for (int i = 0; i < kMlpH * kMlpIn; ++i) p[kOffW1 + i] = u(1.0f / std::sqrt((float)kMlpIn));
  for (int i = 0; i < kMlpH * kMlpH; ++i) p[kOffW2 + i] = u(1.0f / std::sqrt((float)kMlpH));
  for (int i = 0; i < kMlpH; ++i) p[kOffW3 + i] = u(1.0f / std::sqrt((float)kMlpH));
  ppvm_status st = ppvm_mlp_set_params(m, p.data(), p.size());
  if (st != PPVM_OK) {
    ppvm_mlp_destroy(m);
    return st;
  }
  *out = m;
  return PPVM_OK;
}

ppvm_status ppvm_mlp_grad(ppvm_mlp* m, const float* feats, const float* targets, size_t n, float* grads, float* loss) {
  if (!m || !feats || !targets || !grads || n == 0) return mfail(PPVM_EINVAL, "bad argument");
  MCUDA(cudaSetDevice(m->device));
  MTRY(ensure_data(m, n));
  MCUDA(cudaMemcpyAsync(m->d_feats, feats, sizeof(float) * kMlpIn * n, cudaMemcpyHostToDevice, m->stream));
  MCUDA(cudaMemcpyAsync(m->d_tgt, targets, sizeof(float) * n, cudaMemcpyHostToDevice, m->stream));
  MCUDA(cudaMemsetAsync(m->loss, 0, sizeof(float), m->stream));
  int nslabs = 0;
  MTRY(launch_train(m, false, 0, n, 1.0f / (float)n, &nslabs));
  k_mlp_reduce<<<(kMlpParams + 1 + 255) / 256, 256, 0, m->stream>>>(m->slabs, nslabs, m->grads, m->loss);
  MCUDA(cudaGetLastError());
  MCUDA(cudaMemcpyAsync(grads, m->grads, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost, m->stream));
  float ls = 0.f;
  MCUDA(cudaMemcpyAsync(&ls, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
  MCUDA(cudaStreamSynchronize(m->stream));
  if (loss) *loss = ls / (float)n;
  return PPVM_OK;
}

ppvm_status ppvm_mlp_train(ppvm_mlp* m, const float* feats, const float* targets, size_t n, int epochs, int batch,
                           float lr, uint64_t seed, float* last_epoch_loss) {
  if (!m || !feats || !targets || n == 0 || epochs <= 0 || batch <= 0 || !(lr > 0.0f))
    return mfail(PPVM_EINVAL, "bad argument");
  if (n >= 0xFFFFFFFFull) return mfail(PPVM_EINVAL, "too many samples");
  MCUDA(cudaSetDevice(m->device));
  MTRY(ensure_data(m, n));
  MCUDA(cudaMemcpyAsync(m->d_feats, feats, sizeof(float) * kMlpIn * n, cudaMemcpyHostToDevice, m->stream));
  MCUDA(cudaMemcpyAsync(m->d_tgt, targets, sizeof(float) * n, cudaMemcpyHostToDevice, m->stream));
  std::vector<uint32_t> order(n);
  uint64_t s = seed;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  float ls = 0.f;
  for (int ep = 0; ep < epochs; ++ep) {
    for (size_t i = 0; i < n; ++i) order[i] = (uint32_t)i;
    for (size_t i = n - 1; i > 0; --i) std::swap(order[i], order[splitmix(s) % (i + 1)]);  // Fisher-Yates
    MCUDA(cudaMemcpyAsync(m->d_order, order.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, m->stream));
    MCUDA(cudaMemsetAsync(m->loss, 0, sizeof(float), m->stream));
    for (size_t st = 0; st < n; st += (size_t)batch) {
      const size_t cnt = std::min<size_t>((size_t)batch, n - st);
      int nslabs = 0;
      MTRY(launch_train(m, true, st, cnt, 1.0f / (float)cnt, &nslabs));
      ++m->step;
      const float lr_t = lr * std::sqrt(1.0f - std::pow(b2, (float)m->step)) / (1.0f - std::pow(b1, (float)m->step));
      k_mlp_adam<<<(kMlpParams + 1 + 255) / 256, 256, 0, m->stream>>>(m->params, m->m, m->v, m->slabs, nslabs,
                                                                       m->loss, m->w, lr_t, b1, b2, eps);
      MCUDA(cudaGetLastError());
    }
    MCUDA(cudaMemcpyAsync(&ls, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    MCUDA(cudaStreamSynchronize(m->stream));  // the host order buffer is rewritten next epoch
  }
  if (last_epoch_loss) *last_epoch_loss = ls / (float)n;
  return PPVM_OK;
}

ppvm_status ppvm_mlp_predict(ppvm_mlp* m, const float* feats, size_t n, float* out) {
  if (!m || !feats || !out) return mfail(PPVM_EINVAL, "null argument");
  if (n == 0) return PPVM_OK;
  MCUDA(cudaSetDevice(m->device));
  MTRY(ensure_data(m, n));
  MCUDA(cudaMemcpyAsync(m->d_feats, feats, sizeof(float) * kMlpIn * n, cudaMemcpyHostToDevice, m->stream));
  const unsigned grid = (unsigned)std::max<size_t>(1, std::min<size_t>((n + 63) / 64, 1184));
  k_mlp_predict<<<grid, 128, 0, m->stream>>>(m->w, m->d_feats, n, m->d_out);
  MCUDA(cudaGetLastError());
  MCUDA(cudaMemcpyAsync(out, m->d_out, sizeof(float) * n, cudaMemcpyDeviceToHost, m->stream));
  MCUDA(cudaStreamSynchronize(m->stream));
  return PPVM_OK;
}

}  // extern "C"
