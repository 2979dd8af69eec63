// shard.cuh — moving a sum's terms between the ranks that share it (hash-owner sharding).
//
// A sum spread over P ranks keeps every key on exactly one rank.  A merge (a rotation, a
// fused run, amplitude damping) combines only keys that differ in the step's flip bits: a
// rotation by generator G merges K with K ^ G, a fused RX run merges the members of a group,
// which differ only in x bits on the run's qubits.  So before such a step every rank sends
// each term to owner(K) = hash(K with the step's flip bits cleared) mod P.  Keys that can
// merge then share an owner, and the step runs on every rank alone with the single-sum
// kernels (a merge adds at most two contributions, so the result is the same IEEE value on
// any rank).  Cliffords, diagonal noise and truncation need no exchange.
//
// Kernels (one 1024-term tile per block, tiles in index order; the live count N comes from
// the host, which sizes the grid and the tables from it):
//   k_shard_hist     per tile and owner: how many terms (part-major: [owner][tile])
//   k_shard_scan     exclusive scan of that table: each (owner, tile)'s first output row
//   k_shard_scatter  every term to its row, owners in order and, within an owner, terms in
//                    index order (a stable partition), as (2W+1)-word rows: x[W], z[W], c
//   k_shard_append   rows received from the other ranks appended to the sum
#pragma once

#include "kernels.cuh"

namespace ppvm {

constexpr int kShardBlock = 1024;   // terms per tile
constexpr int kShardMaxParts = 32;  // ranks a sum can be spread over (one scan warp each)

// Owner of term i: the hash of its key with the flip bits (mx, mz) cleared.
template <int W>
__device__ __forceinline__ unsigned shard_owner(const uint64_t (&x)[W], const uint64_t (&z)[W], const Gen& m,
                                                unsigned nparts) {
  uint64_t kx[W], kz[W];
#pragma unroll
  for (int w = 0; w < W; ++w) {
    kx[w] = x[w] & ~m.gx[w];
    kz[w] = z[w] & ~m.gz[w];
  }
  return (unsigned)((hash_key<W>(kx, kz) >> 40) % nparts);
}

// The term's owner (nparts for a thread past the end), its rank among the tile's terms of
// that owner, and in s_tot[p] every owner's count in the tile.  s_cnt: kShardMaxParts * 32.
template <int W>
__device__ __forceinline__ unsigned shard_rank(const Planes& P, unsigned long long i, unsigned long long N,
                                               const Gen& m, unsigned nparts, unsigned* s_cnt, unsigned* s_tot,
                                               uint64_t (&x)[W], uint64_t (&z)[W], unsigned& rank) {
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (unsigned t = threadIdx.x; t < kShardMaxParts * 32; t += blockDim.x) s_cnt[t] = 0;
  unsigned own = nparts;
  if (i < N) {
    load_key<W>(P, i, x, z);
    own = shard_owner<W>(x, z, m, nparts);
  }
  const unsigned same = __match_any_sync(kFull, own);
  const unsigned in_warp = __popc(same & ((1u << lane) - 1u));
  __syncthreads();
  if (own < nparts && in_warp == 0) s_cnt[own * 32 + warp] = __popc(same);
  __syncthreads();
  // warp p scans owner p's counts over the tile's 32 warps (lane = warp index)
  if (warp < nparts) {
    const unsigned c = s_cnt[warp * 32 + lane];
    unsigned v = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t = __shfl_up_sync(kFull, v, o);
      if (lane >= (unsigned)o) v += t;
    }
    s_cnt[warp * 32 + lane] = v - c;
    if (lane == 31) s_tot[warp] = v;
  }
  __syncthreads();
  rank = own < nparts ? s_cnt[own * 32 + warp] + in_warp : 0u;
  return own;
}

template <int W>
__global__ void __launch_bounds__(kShardBlock)
k_shard_hist(Planes P, unsigned long long N, Gen m, unsigned nparts, unsigned long long* hist) {
  __shared__ unsigned s_cnt[kShardMaxParts * 32], s_tot[kShardMaxParts];
  const unsigned long long ntiles = (N + kShardBlock - 1) / kShardBlock;  // = gridDim.x
  const unsigned long long i = (unsigned long long)blockIdx.x * kShardBlock + threadIdx.x;
  uint64_t x[W], z[W];
  unsigned rank;
  shard_rank<W>(P, i, N, m, nparts, s_cnt, s_tot, x, z, rank);
  if (threadIdx.x < nparts) hist[(unsigned long long)threadIdx.x * ntiles + blockIdx.x] = s_tot[threadIdx.x];
}

// One block: exclusive scan of the M = nparts * ntiles entries in place; first[p] = the first
// row of owner p (first[nparts] = N).
__global__ void __launch_bounds__(1024)
k_shard_scan(unsigned long long* hist, unsigned long long ntiles, unsigned nparts, unsigned long long* first) {
  __shared__ unsigned long long s_w[32];
  const unsigned long long M = ntiles * nparts;
  const unsigned long long per = (M + blockDim.x - 1) / blockDim.x;
  const unsigned long long a = (unsigned long long)threadIdx.x * per, b = min(M, a + per);
  unsigned long long local = 0;
  for (unsigned long long e = a; e < b; ++e) local += hist[e];
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long v = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long t = __shfl_up_sync(kFull, v, o);
    if (lane >= (unsigned)o) v += t;
  }
  if (lane == 31) s_w[warp] = v;
  __syncthreads();
  if (warp == 0) {
    const unsigned long long c = s_w[lane];
    unsigned long long u = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long t = __shfl_up_sync(kFull, u, o);
      if (lane >= (unsigned)o) u += t;
    }
    s_w[lane] = u - c;
  }
  __syncthreads();
  unsigned long long run = s_w[warp] + v - local;
  for (unsigned long long e = a; e < b; ++e) {
    const unsigned long long t = hist[e];
    hist[e] = run;
    if (e % ntiles == 0) first[e / ntiles] = run;
    run += t;
  }
  if (threadIdx.x == blockDim.x - 1) first[nparts] = run;  // the last thread's run ends at M's total
}

template <int W>
__global__ void __launch_bounds__(kShardBlock)
k_shard_scatter(Planes P, unsigned long long N, Gen m, unsigned nparts, const unsigned long long* offs,
                uint64_t* rows) {
  __shared__ unsigned s_cnt[kShardMaxParts * 32], s_tot[kShardMaxParts];
  const unsigned long long ntiles = (N + kShardBlock - 1) / kShardBlock;  // = gridDim.x
  const unsigned long long i = (unsigned long long)blockIdx.x * kShardBlock + threadIdx.x;
  uint64_t x[W], z[W];
  unsigned rank;
  const unsigned own = shard_rank<W>(P, i, N, m, nparts, s_cnt, s_tot, x, z, rank);
  if (own >= nparts) return;
  const unsigned long long r = offs[(unsigned long long)own * ntiles + blockIdx.x] + rank;
  uint64_t* row = rows + r * (2 * W + 1);
#pragma unroll
  for (int w = 0; w < W; ++w) {
    row[w] = x[w];
    row[W + w] = z[w];
  }
  row[2 * W] = (uint64_t)__double_as_longlong(P.c[i]);
}

// Appends k rows at [n0, n0 + k) and sets the live count.
template <int W>
__global__ void k_shard_append(Planes P, Ctrl* ctrl, const uint64_t* rows, unsigned long long k,
                               unsigned long long n0) {
  for (unsigned long long r = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; r < k;
       r += (unsigned long long)gridDim.x * blockDim.x) {
    const uint64_t* row = rows + r * (2 * W + 1);
    uint64_t x[W], z[W];
#pragma unroll
    for (int w = 0; w < W; ++w) {
      x[w] = row[w];
      z[w] = row[W + w];
    }
    store_key<W>(P, n0 + r, x, z);
    P.c[n0 + r] = __longlong_as_double((long long)row[2 * W]);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) ctrl->n = n0 + k;
}

}  // namespace ppvm
