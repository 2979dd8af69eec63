// noise.cuh — amplitude damping (crates/ppvm-pauli-sum/src/sum/noise.rs:132-163).
//
// The Heisenberg adjoint of amplitude damping on qubit q maps
//   I -> I,   X -> sqrt(1-g) X,   Y -> sqrt(1-g) Y,   Z -> (1-g) Z + g I,
// through map_insert (data.rs:204-226): a Z term (parent) is scaled in place and its child,
// the same word with I on q and coefficient v * g, is merged with `+=` into an existing term
// or appended after all terms, in parent order.  Unlike a rotation's child, this child can
// only land on a term with I on q, which is not a parent itself, so every key still receives
// at most two contributions and the result is bit-identical to the reference's.
//
//   k_rot_scan<..., DAMP>  parents (Z on q) in index order: s_idx, s_rec (key + coefficient)
//   k_damp_index           the parents' child keys into an epoch-tagged hash table
//   k_damp_probe           every term with I on q looks its own key up (a hit is the partner
//                          of that child); X and Y terms are scaled by sqrt(1-g) here
//   k_damp_apply           parents scaled by (1-g); each child merged into its partner or
//                          appended at N + (its rank among the unpartnered), in parent order
//   k_commit_damp          publishes the live count
//
// The capacity check (N + parents <= capacity) runs in k_damp_probe before any coefficient
// changes, so a replay after growth starts from unmodified terms.
#pragma once

#include "kernels.cuh"

namespace ppvm {

template <int W>
__device__ __forceinline__ void damp_child_key(const uint64_t* s_rec, unsigned long long s, const Gen& g,
                                               uint64_t (&x)[W], uint64_t (&z)[W], double& c) {
  load_rec<W>(s_rec, s, x, z, c);
#pragma unroll
  for (int w = 0; w < W; ++w) z[w] ^= g.gz[w];  // the parent has z = 1 on q: clear it
}

template <int W>
__global__ void __launch_bounds__(256)
k_damp_index(Ctrl* ctrl, Gen g, const uint64_t* s_rec, unsigned long long* table, unsigned long long table_cap,
             unsigned tepoch, int op) {
  pdl_wait();
  if (ld_volatile_int(&ctrl->err)) return;
  const unsigned long long ns = ld_volatile(&ctrl->n_s);
  if (ns == 0) return;
  unsigned long long tsize = next_pow2_ull(ns * 2 < 1024 ? 1024 : ns * 2);
  if (tsize > table_cap) tsize = table_cap;
  const unsigned long long mask = tsize - 1;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long s = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; s < ns; s += stride) {
    uint64_t x[W], z[W];
    double c;
    damp_child_key<W>(s_rec, s, g, x, z, c);
    const uint64_t h = hash_key<W>(x, z);
    const unsigned long long mine = make_slot(tepoch, (unsigned)(h >> 48) & 0xFFFFu, (unsigned)s);
    unsigned long long slot = h & mask;
    unsigned long long probes = 0;
    while (true) {  // child keys are distinct: take the first slot of an older epoch
      const unsigned long long cur = ld_volatile(&table[slot]);
      if (slot_epoch(cur) != (tepoch & 0xFFFFu)) {
        if (atomicCAS(&table[slot], cur, mine) == cur) break;
        continue;
      }
      slot = (slot + 1) & mask;
      if (++probes > tsize) {
        set_err(ctrl, kErrProbe, op);
        break;
      }
    }
  }
}

template <int W>
__global__ void __launch_bounds__(256)
k_damp_probe(Planes P, Ctrl* ctrl, Gen g, unsigned qw, const uint64_t* s_rec, uint32_t* partner,
             const unsigned long long* table, unsigned long long table_cap, unsigned tepoch, double sxy, int op) {
  pdl_wait();
  if (ld_volatile_int(&ctrl->err)) return;
  const unsigned long long N = ld_volatile(&ctrl->n);
  const unsigned long long ns = ld_volatile(&ctrl->n_s);
  if (N + ns > P.cap) {  // every child could be new: grow before anything changes
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      ctrl->cap_needed = N + ns;
      set_err(ctrl, kErrCapacity, op);
    }
    return;
  }
  unsigned long long tsize = next_pow2_ull(ns * 2 < 1024 ? 1024 : ns * 2);
  if (tsize > table_cap) tsize = table_cap;
  const unsigned long long mask = tsize - 1;
  const uint64_t bit = g.gz[qw];
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
    const uint64_t xq = P.x[(unsigned long long)qw * P.cap + i] & bit;
    if (xq) {  // X or Y on q
      P.c[i] = __dmul_rn(P.c[i], sxy);
      continue;
    }
    if (ns == 0 || (P.z[(unsigned long long)qw * P.cap + i] & bit)) continue;  // Z: a parent
    uint64_t x[W], z[W];
    load_key<W>(P, i, x, z);
    const uint64_t h = hash_key<W>(x, z);
    const unsigned tag = (unsigned)(h >> 48) & 0xFFFFu;
    unsigned long long slot = h & mask;
    for (unsigned long long probes = 0; probes <= tsize; ++probes) {
      const unsigned long long cur = ld_volatile(&table[slot]);
      if (slot_epoch(cur) != (tepoch & 0xFFFFu)) break;  // not a child key
      if (slot_tag(cur) == tag) {
        const unsigned s = slot_idx(cur);
        uint64_t cx[W], cz[W];
        double c;
        damp_child_key<W>(s_rec, s, g, cx, cz, c);
        bool eq = true;
#pragma unroll
        for (int w = 0; w < W; ++w) eq &= (cx[w] == x[w]) & (cz[w] == z[w]);
        if (eq) {
          partner[s] = (uint32_t)i;
          atomicAdd(&ctrl->n_pairs, 1ull);
          break;
        }
      }
      slot = (slot + 1) & mask;
    }
  }
}

template <int W, int BLOCK, int ITEMS>
__global__ void __launch_bounds__(BLOCK)
k_damp_apply(Planes P, Ctrl* ctrl, Gen g, double om, double gm, const uint32_t* s_idx, const uint64_t* s_rec,
             const uint32_t* partner, unsigned long long* ts, unsigned epoch, int op) {
  pdl_wait();
  __shared__ unsigned s_tile;
  __shared__ unsigned long long s_slot;
  __shared__ unsigned s_base[ITEMS * (BLOCK / 32) + 1];
  if (ld_volatile_int(&ctrl->err)) return;
  const unsigned long long N = ld_volatile(&ctrl->n);
  const unsigned long long ns = ld_volatile(&ctrl->n_s);
  if (ns == 0) return;
  constexpr unsigned long long TILE = (unsigned long long)BLOCK * ITEMS;
  const unsigned long long ntiles = (ns + TILE - 1) / TILE;
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = BLOCK / 32;
  for (;;) {
    const unsigned tile = next_tile(&ctrl->tickets[1], &s_tile);
    if (tile >= ntiles) break;
    const unsigned long long base = (unsigned long long)tile * TILE;
    unsigned ballots[ITEMS];
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const unsigned long long s = base + (unsigned long long)k * BLOCK + threadIdx.x;
      bool child = false;
      if (s < ns) {
        uint64_t x[W], z[W];
        double c;
        load_rec<W>(s_rec, s, x, z, c);
        P.c[s_idx[s]] = __dmul_rn(c, om);
        const uint32_t j = partner[s];
        if (j != kNone) {
          P.c[j] = __dadd_rn(P.c[j], __dmul_rn(c, gm));  // the partner is no parent: one writer
        } else {
          child = true;
        }
      }
      ballots[k] = __ballot_sync(kFull, child);
    }
    const unsigned agg = tile_ranks<BLOCK, ITEMS>(ballots, s_base);
    const unsigned long long excl = lookback(ts, tile, agg, epoch, ctrl, op, &s_slot);
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      if ((ballots[k] >> lane) & 1u) {
        const unsigned long long s = base + (unsigned long long)k * BLOCK + threadIdx.x;
        const unsigned long long r =
            N + excl + s_base[k * NW + warp] + __popc(ballots[k] & ((1u << lane) - 1u));
        uint64_t x[W], z[W];
        double c;
        damp_child_key<W>(s_rec, s, g, x, z, c);
        store_key<W>(P, r, x, z);
        P.c[r] = __dmul_rn(c, gm);
      }
    }
  }
}

// Publishes the live count after amplitude damping and resets the tile tickets (one thread).
static __global__ void k_commit_damp(Ctrl* ctrl, int op, OpLog* log) {
  pdl_wait();
  for (int t = 0; t < 4; ++t) ctrl->tickets[t] = 0;
  if (ctrl->err) return;
  const unsigned long long nchild = ctrl->n_s - ctrl->n_pairs;
  log[op].n_new = nchild;
  ctrl->n = ctrl->n + nchild;
  log[op].n_out = ctrl->n;
}

}  // namespace ppvm
