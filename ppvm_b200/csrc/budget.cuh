// budget.cuh — term-budget truncation: keep the B terms of highest priority.
//
// Priority keys are 32-bit and order-preserving: the high word of |c| as an IEEE double
// (plain truncation by magnitude) or the score of the term-priority network (learned
// truncation, mlp.cuh), computed in one pass (k_score).  The B-th largest key is found by
// an MSD radix select that never leaves the device (k_sel_init, then per digit k_sel_hist +
// k_sel_pick; digit width 8 or 11 bits), and k_budget_compact keeps, in place and in order,
// every term above that key plus the first terms equal to it, so exactly B survive and the
// result does not depend on thread timing.
#pragma once

#include "kernels.cuh"
#include "mlp.cuh"

namespace ppvm {

struct SelState {
  unsigned long long rank;  // keys still to keep among those matching the prefix
  uint32_t prefix, mask;    // fixed high digits of the threshold key
  int all;                  // N <= budget: keep everything
  int pad;
};

template <int W>
__global__ void __launch_bounds__(256) k_features(Planes P, const Ctrl* ctrl, int L, int layers_left, float* out) {
  const unsigned long long N = ld_volatile(&ctrl->n);
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    uint64_t x[W], z[W];
    load_key<W>(P, i, x, z);
    float f[kMlpIn];
    term_features<W>(x, z, P.c[i], L, layers_left, f);
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) out[i * kMlpIn + k] = f[k];
  }
}

// Priority key of every live term: plain (Wg == nullptr) or the network's score.
template <int W>
__global__ void __launch_bounds__(128) k_score(Planes P, const Ctrl* ctrl, const MlpWeights* Wg, int L,
                                               int layers_left, uint32_t* keys) {
  __shared__ MlpWeights Ws;
  __shared__ __nv_bfloat16 sX[4][16 * kMlpK1];
  const unsigned long long N = ld_volatile(&ctrl->n);
  if (!Wg) {
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (unsigned long long)gridDim.x * blockDim.x)
      keys[i] = (uint32_t)((unsigned long long)__double_as_longlong(fabs(P.c[i])) >> 32);
    return;
  }
  {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(Wg);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&Ws);
    for (int i = threadIdx.x; i < (int)(sizeof(MlpWeights) / 4); i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const unsigned long long ntiles = (N + 15) / 16;
  __nv_bfloat16* X = sX[warp];
  for (unsigned long long tile = (unsigned long long)blockIdx.x * 4 + warp; tile < ntiles;
       tile += (unsigned long long)gridDim.x * 4) {
    if (lane < 16) {
      const unsigned long long i = tile * 16 + lane;
      float f[kMlpIn];
      if (i < N) {
        uint64_t x[W], z[W];
        load_key<W>(P, i, x, z);
        term_features<W>(x, z, P.c[i], L, layers_left, f);
      } else {
#pragma unroll
        for (int k = 0; k < kMlpIn; ++k) f[k] = 0.0f;
      }
#pragma unroll
      for (int k = 0; k < kMlpK1; ++k) X[lane * kMlpK1 + k] = __float2bfloat16_rn(k < kMlpIn ? f[k] : 0.0f);
    }
    __syncwarp();
    MlpTile T;
    mlp_forward(X, Ws, T);
    if (t == 0) {
      if (tile * 16 + g < N) keys[tile * 16 + g] = score_key(T.y[0]);
      if (tile * 16 + g + 8 < N) keys[tile * 16 + g + 8] = score_key(T.y[1]);
    }
    __syncwarp();
  }
}

static __global__ void k_sel_init(const Ctrl* ctrl, unsigned long long budget, SelState* st) {
  const unsigned long long N = ctrl->n;
  st->all = (N <= budget) ? 1 : 0;
  st->rank = budget;
  st->prefix = 0;
  st->mask = 0;
}

template <int BITS>
__global__ void __launch_bounds__(256) k_sel_hist(const Ctrl* ctrl, const uint32_t* keys, const SelState* st,
                                                  int shift, unsigned* hist) {
  constexpr int NB = 1 << BITS;
  __shared__ unsigned sh[NB];
  if (st->all) return;
  const uint32_t prefix = st->prefix, mask = st->mask;
  for (int b = threadIdx.x; b < NB; b += blockDim.x) sh[b] = 0;
  __syncthreads();
  const unsigned long long N = ld_volatile(&ctrl->n);
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t k = keys[i];
    if ((k & mask) == prefix) atomicAdd(&sh[(k >> shift) & (NB - 1)], 1u);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < NB; b += blockDim.x)
    if (sh[b]) atomicAdd(&hist[b], sh[b]);
}

// Fixes the next digit of the threshold key; clears the histogram for the next pass.
template <int BITS>
__global__ void k_sel_pick(SelState* st, int shift, unsigned* hist) {
  constexpr int NB = 1 << BITS;
  if (threadIdx.x == 0 && !st->all) {
    unsigned long long above = 0;
    for (int b = NB - 1; b >= 0; --b) {
      const unsigned long long h = hist[b];
      if (above + h >= st->rank) {
        st->prefix |= (uint32_t)b << shift;
        st->mask |= (uint32_t)(NB - 1) << shift;
        st->rank -= above;
        break;
      }
      above += h;
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < NB; b += blockDim.x) hist[b] = 0;
}

// Keeps every term whose key is above the threshold and the first `rank` terms equal to it,
// in place and in order (a tile's reads finish before its writes; writes never pass reads).
template <int W, int BLOCK, int ITEMS>
__global__ void __launch_bounds__(BLOCK)
k_budget_compact(Planes P, Ctrl* ctrl, const uint32_t* keys, const SelState* st, unsigned long long* ts_gt,
                 unsigned ep_gt, unsigned long long* ts_eq, unsigned ep_eq) {
  __shared__ unsigned s_tile;
  __shared__ unsigned long long s_slot;
  __shared__ unsigned s_gt[ITEMS * (BLOCK / 32) + 1];
  __shared__ unsigned s_eq[ITEMS * (BLOCK / 32) + 1];
  if (ld_volatile_int(&ctrl->err) || st->all) return;
  const uint32_t T = st->prefix;
  const unsigned long long R = st->rank;
  const unsigned long long N = ld_volatile(&ctrl->n);
  constexpr unsigned long long TILE = (unsigned long long)BLOCK * ITEMS;
  const unsigned long long ntiles = (N + TILE - 1) / TILE;
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  constexpr int NW = BLOCK / 32;
  for (;;) {
    const unsigned tile = next_tile(&ctrl->tickets[2], &s_tile);
    if (tile >= ntiles) break;
    const unsigned long long base = (unsigned long long)tile * TILE;
    uint64_t kx[ITEMS][W], kz[ITEMS][W];
    double kc[ITEMS];
    unsigned gt_b[ITEMS], eq_b[ITEMS];
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const unsigned long long i = base + (unsigned long long)k * BLOCK + threadIdx.x;
      bool gt = false, eq = false;
      if (i < N) {
        load_key<W>(P, i, kx[k], kz[k]);
        kc[k] = P.c[i];
        const uint32_t key = keys[i];
        gt = key > T;
        eq = key == T;
      }
      gt_b[k] = __ballot_sync(kFull, gt);
      eq_b[k] = __ballot_sync(kFull, eq);
    }
    const unsigned agt = tile_ranks<BLOCK, ITEMS>(gt_b, s_gt);
    const unsigned aeq = tile_ranks<BLOCK, ITEMS>(eq_b, s_eq);
    const unsigned long long xgt = lookback(ts_gt, tile, agt, ep_gt, ctrl, 0, &s_slot);
    const unsigned long long xeq = lookback(ts_eq, tile, aeq, ep_eq, ctrl, 0, &s_slot);
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const bool gt = (gt_b[k] >> lane) & 1u, eq = (eq_b[k] >> lane) & 1u;
      if (!gt && !eq) continue;
      const unsigned long long gt_before = xgt + s_gt[k * NW + warp] + __popc(gt_b[k] & lt);
      const unsigned long long eq_before = xeq + s_eq[k * NW + warp] + __popc(eq_b[k] & lt);
      if (eq && eq_before >= R) continue;
      const unsigned long long pos = gt_before + (eq_before < R ? eq_before : R);
      store_key<W>(P, pos, kx[k], kz[k]);
      P.c[pos] = kc[k];
    }
    if (tile == ntiles - 1 && threadIdx.x == 0) {
      const unsigned long long teq = xeq + aeq;
      ctrl->n_s = xgt + agt + (teq < R ? teq : R);
    }
  }
}

static __global__ void k_commit_budget(Ctrl* ctrl, const SelState* st) {
  for (int t = 0; t < 4; ++t) ctrl->tickets[t] = 0;
  if (ctrl->err || st->all) return;
  ctrl->n = ctrl->n_s;
}

}  // namespace ppvm
