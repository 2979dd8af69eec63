// kernels.cuh — the hot-path kernels of the Pauli-propagation engine (sm_100a).
//
// Rotation exp(-i theta/2 G) on a sum held in SoA planes, reference semantics of
// PauliSum::map_insert (crates/ppvm-pauli-sum/src/sum/data.rs:204-226):
//   k_rot_scan   ordered compaction of the anticommuting terms into a dense record buffer
//   k_rot_pair   partner search: each record inserts min(K, K^G) into an epoch-tagged table;
//                the second of a pair to arrive links both (a child K^G can only collide with
//                its partner term, so every key receives at most two contributions)
//   k_rot_apply  parent <- c*cos (+ partner's c*(eps*sin)); partnerless parents append their
//                child in parent order, so the term order stays the reference's IndexMap order
//   k_commit     publishes the new live count and resets the tile tickets
// Clifford runs (sum/clifford.rs) and diagonal noise (sum/noise.rs) are one in-place pass
// (k_clifford); truncation (data.rs:275-311, strategy.rs) is an in-place stable compaction.
#pragma once

#include "common.cuh"

namespace ppvm {

constexpr unsigned kNone = 0xFFFFFFFFu;

template <int W>
__device__ __forceinline__ void load_key(const Planes& P, unsigned long long i, uint64_t (&x)[W],
                                         uint64_t (&z)[W]) {
#pragma unroll
  for (int w = 0; w < W; ++w) {
    x[w] = P.x[(unsigned long long)w * P.cap + i];
    z[w] = P.z[(unsigned long long)w * P.cap + i];
  }
}
template <int W>
__device__ __forceinline__ void store_key(const Planes& P, unsigned long long i,
                                          const uint64_t (&x)[W], const uint64_t (&z)[W]) {
#pragma unroll
  for (int w = 0; w < W; ++w) {
    P.x[(unsigned long long)w * P.cap + i] = x[w];
    P.z[(unsigned long long)w * P.cap + i] = z[w];
  }
}
// Dense record of an anticommuting term: [x0..x(W-1), z0..z(W-1), coeff bits].
template <int W>
__device__ __forceinline__ void load_rec(const uint64_t* rec, unsigned long long s, uint64_t (&x)[W],
                                         uint64_t (&z)[W], double& c) {
  const uint64_t* r = rec + s * (2 * W + 1);
#pragma unroll
  for (int w = 0; w < W; ++w) x[w] = r[w];
#pragma unroll
  for (int w = 0; w < W; ++w) z[w] = r[W + w];
  c = __longlong_as_double((long long)r[2 * W]);
}

// The generator as it acts on the term with X words x: on a lossy sum (g.lw != 0) it skips
// the term's lost qubits, which is the reference's loss fallback of rotate_2
// (crates/ppvm-pauli-sum/src/sum/rot2.rs:26-33) extended to any support: a lost qubit has
// x = z = 0, so the anticommutation test and the sign are those of the full generator and only
// the child's bits differ.
template <int W>
__device__ __forceinline__ void gen_on(const Gen& g, const uint64_t (&x)[W], uint64_t (&gx)[W],
                                       uint64_t (&gz)[W]) {
#pragma unroll
  for (int w = 0; w < W; ++w) {
    uint64_t lost = 0;
#pragma unroll
    for (int v = 0; v < W; ++v)
      if (g.lw && v == w + (int)g.lw) lost = x[v];
    gx[w] = g.gx[w] & ~lost;
    gz[w] = g.gz[w] & ~lost;
  }
}

template <int W>
struct ItemsFor {
  // terms per thread of a look-back tile: small enough that a sum of 10^5..10^6 terms
  // spreads over a few tiles per SM (a 256-thread tile holds 256 * ITEMS terms)
  static constexpr int value = W <= 2 ? 4 : (W <= 4 ? 2 : 1);
};

// ---------------------------------------------------------------------------------------
// k_rot_scan: flags anticommuting terms, writes their index and record in index order.
// With DAMP the flagged terms are those with Z (x = 0, z = 1) on the qubit of g.gz instead:
// the parents of amplitude damping.
// ---------------------------------------------------------------------------------------
template <int W, int BLOCK, int ITEMS, bool DAMP = false>
__global__ void __launch_bounds__(BLOCK)
k_rot_scan(Planes P, Ctrl* ctrl, Gen g, unsigned xmask, unsigned zmask, uint32_t* s_idx, uint64_t* s_rec,
           uint32_t* partner, unsigned long long* ts, unsigned epoch, int op, OpLog* log) {
  pdl_wait();
  __shared__ unsigned s_tile;
  __shared__ unsigned long long s_slot;
  __shared__ unsigned s_base[ITEMS * (BLOCK / 32) + 1];
  if (ld_volatile_int(&ctrl->err)) return;
  const unsigned long long N = ld_volatile(&ctrl->n);
  constexpr unsigned long long TILE = (unsigned long long)BLOCK * ITEMS;
  const unsigned long long ntiles = (N + TILE - 1) / TILE;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    log[op].n_in = N;
    ctrl->n_pairs = 0;
    if (N == 0) {
      ctrl->n_s = 0;
      log[op].n_s = 0;
    }
  }
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = BLOCK / 32;
  for (;;) {
    const unsigned tile = next_tile(&ctrl->tickets[0], &s_tile);
    if (tile >= ntiles) break;
    const unsigned long long base = (unsigned long long)tile * TILE;
    unsigned ballots[ITEMS];
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const unsigned long long i = base + (unsigned long long)k * BLOCK + threadIdx.x;
      bool a = false;
      if (i < N) {
        uint64_t acc = 0;
        if constexpr (DAMP) {
#pragma unroll
          for (int w = 0; w < W; ++w)
            if ((zmask >> w) & 1u)
              acc |= P.z[(unsigned long long)w * P.cap + i] & ~P.x[(unsigned long long)w * P.cap + i] & g.gz[w];
          a = acc != 0;
        } else {
#pragma unroll
          for (int w = 0; w < W; ++w) {
            if ((xmask >> w) & 1u) acc ^= P.x[(unsigned long long)w * P.cap + i] & g.gz[w];
            if ((zmask >> w) & 1u) acc ^= P.z[(unsigned long long)w * P.cap + i] & g.gx[w];
          }
          a = __popcll(acc) & 1;
        }
      }
      ballots[k] = __ballot_sync(kFull, a);
    }
    const unsigned agg = tile_ranks<BLOCK, ITEMS>(ballots, s_base);
    const unsigned long long excl = lookback(ts, tile, agg, epoch, ctrl, op, &s_slot);
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      if ((ballots[k] >> lane) & 1u) {
        const unsigned long long i = base + (unsigned long long)k * BLOCK + threadIdx.x;
        const unsigned long long r =
            excl + s_base[k * NW + warp] + __popc(ballots[k] & ((1u << lane) - 1u));
        s_idx[r] = (uint32_t)i;
        partner[r] = kNone;
        uint64_t* rec = s_rec + r * (2 * W + 1);
#pragma unroll
        for (int w = 0; w < W; ++w) rec[w] = P.x[(unsigned long long)w * P.cap + i];
#pragma unroll
        for (int w = 0; w < W; ++w) rec[W + w] = P.z[(unsigned long long)w * P.cap + i];
        rec[2 * W] = (uint64_t)__double_as_longlong(P.c[i]);
      }
    }
    if (tile == ntiles - 1 && threadIdx.x == 0) {
      ctrl->n_s = excl + agg;
      log[op].n_s = excl + agg;
    }
  }
}

// ---------------------------------------------------------------------------------------
// k_rot_pair: finds, for each anticommuting term, whether its partner K^G is also present.
// ---------------------------------------------------------------------------------------
template <int W>
__global__ void __launch_bounds__(256)
k_rot_pair(Ctrl* ctrl, Gen g, const uint64_t* s_rec, uint32_t* partner,
           unsigned long long* table, unsigned long long table_cap, unsigned tepoch, int op) {
  pdl_wait();
  if (ld_volatile_int(&ctrl->err)) return;
  const unsigned long long ns = ld_volatile(&ctrl->n_s);
  if (ns == 0) return;
  unsigned long long tsize = next_pow2_ull(ns * 2 < 1024 ? 1024 : ns * 2);
  if (tsize > table_cap) tsize = table_cap;
  const unsigned long long mask = tsize - 1;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long s = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; s < ns;
       s += stride) {
    uint64_t x[W], z[W], px[W], pz[W], ex[W], ez[W];
    double c;
    load_rec<W>(s_rec, s, x, z, c);
    gen_on<W>(g, x, ex, ez);
#pragma unroll
    for (int w = 0; w < W; ++w) {
      px[w] = x[w] ^ ex[w];
      pz[w] = z[w] ^ ez[w];
    }
    const bool use_p = key_less<W>(px, pz, x, z);
    uint64_t rx[W], rz[W];
#pragma unroll
    for (int w = 0; w < W; ++w) {
      rx[w] = use_p ? px[w] : x[w];
      rz[w] = use_p ? pz[w] : z[w];
    }
    const uint64_t h = hash_key<W>(rx, rz);
    const unsigned tag = (unsigned)(h >> 48) & 0xFFFFu;
    const unsigned long long mine = make_slot(tepoch, tag, (unsigned)s);
    unsigned long long slot = h & mask;
    unsigned long long probes = 0;
    while (true) {
      unsigned long long cur = ld_volatile(&table[slot]);
      if (slot_epoch(cur) != (tepoch & 0xFFFFu)) {
        const unsigned long long prev = atomicCAS(&table[slot], cur, mine);
        if (prev == cur) break;  // inserted; the partner (if any) will find us
        continue;                // slot was taken meanwhile: examine it again
      }
      if (slot_tag(cur) == tag) {
        const unsigned j = slot_idx(cur);
        uint64_t jx[W], jz[W];
        double jc;
        load_rec<W>(s_rec, j, jx, jz, jc);
        // j is our partner iff its key is exactly K ^ G
        bool eq = true;
#pragma unroll
        for (int w = 0; w < W; ++w) eq &= (jx[w] == px[w]) & (jz[w] == pz[w]);
        if (eq) {
          partner[s] = j;
          partner[j] = (uint32_t)s;
          atomicAdd(&ctrl->n_pairs, 1ull);
          break;
        }
      }
      slot = (slot + 1) & mask;
      if (++probes > tsize) {
        set_err(ctrl, kErrProbe, op);
        break;
      }
    }
  }
}

// ---------------------------------------------------------------------------------------
// k_rot_apply: new coefficients of anticommuting parents; children appended in order.
// ---------------------------------------------------------------------------------------
template <int W, int BLOCK, int ITEMS>
__global__ void __launch_bounds__(BLOCK)
k_rot_apply(Planes P, Ctrl* ctrl, Gen g, double sn, double cs, const uint32_t* s_idx,
            const uint64_t* s_rec, const uint32_t* partner, unsigned long long* ts,
            unsigned epoch, int op, OpLog* log) {
  pdl_wait();
  __shared__ unsigned s_tile;
  __shared__ unsigned long long s_slot;
  __shared__ unsigned s_base[ITEMS * (BLOCK / 32) + 1];
  if (ld_volatile_int(&ctrl->err)) return;
  const unsigned long long N = ld_volatile(&ctrl->n);
  const unsigned long long ns = ld_volatile(&ctrl->n_s);
  const unsigned long long np = ld_volatile(&ctrl->n_pairs);
  const unsigned long long nchild = ns - 2 * np;
  if (N + nchild > P.cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      ctrl->cap_needed = N + nchild;
      set_err(ctrl, kErrCapacity, op);
    }
    return;
  }
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
        const uint32_t j = partner[s];
        double nc;
        if (j != kNone) {
          uint64_t jx[W], jz[W];
          double jc;
          load_rec<W>(s_rec, j, jx, jz, jc);
          const double eps_j = rot_sign<W>(g, jx, jz);
          nc = __dadd_rn(__dmul_rn(c, cs), __dmul_rn(jc, eps_j * sn));
        } else {
          nc = __dmul_rn(c, cs);
          child = true;
        }
        P.c[s_idx[s]] = nc;
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
        load_rec<W>(s_rec, s, x, z, c);
        const double eps = rot_sign<W>(g, x, z);
        uint64_t ex[W], ez[W];
        gen_on<W>(g, x, ex, ez);
#pragma unroll
        for (int w = 0; w < W; ++w) {
          x[w] ^= ex[w];
          z[w] ^= ez[w];
        }
        store_key<W>(P, r, x, z);
        P.c[r] = __dmul_rn(c, eps * sn);
      }
    }
  }
}

// Publishes the live count after a rotation and resets the tile tickets (one thread).
static __global__ void k_commit_rot(Ctrl* ctrl, int op, OpLog* log) {
  pdl_wait();
  for (int t = 0; t < 4; ++t) ctrl->tickets[t] = 0;
  if (ctrl->err) return;
  const unsigned long long nchild = ctrl->n_s - 2 * ctrl->n_pairs;
  log[op].n_new = nchild;
  ctrl->n = ctrl->n + nchild;
  log[op].n_out = ctrl->n;
}

// ---------------------------------------------------------------------------------------
// Truncation: keep iff !(|c| < thr) and weight <= maxw (CombinedStrategy order does not
// matter for the kept set).  Dropped terms whose key is preserved are collected in order
// and re-appended after the kept ones (data.rs:283-310).  In place: a tile publishes its
// aggregate only after loading all of its terms, and writes go to positions <= its reads.
// ---------------------------------------------------------------------------------------
template <int W>
__device__ __forceinline__ bool preserved(const uint64_t (&x)[W], const uint64_t (&z)[W],
                                          const uint64_t* pres_keys, const int* pres_table,
                                          unsigned pres_mask) {
  unsigned long long slot = hash_key<W>(x, z) & pres_mask;
  for (unsigned probe = 0; probe <= pres_mask; ++probe) {
    const int j = pres_table[slot];
    if (j < 0) return false;
    const uint64_t* k = pres_keys + (unsigned long long)j * 2 * W;
    bool eq = true;
#pragma unroll
    for (int w = 0; w < W; ++w) eq &= (k[w] == x[w]) & (k[W + w] == z[w]);
    if (eq) return true;
    slot = (slot + 1) & pres_mask;
  }
  return false;
}

template <int W, int BLOCK, int ITEMS>
__global__ void __launch_bounds__(BLOCK)
k_truncate(Planes P, Ctrl* ctrl, double thr, unsigned long long maxw, const uint64_t* pres_keys,
           const int* pres_table, unsigned pres_mask, int npres, uint64_t* side,
           unsigned long long* ts, unsigned epoch, int op, OpLog* log, unsigned long long maxlw, unsigned lw) {
  pdl_wait();
  __shared__ unsigned s_tile;
  __shared__ unsigned long long s_slot;
  __shared__ unsigned s_base[ITEMS * (BLOCK / 32) + 1];
  __shared__ unsigned s_base2[ITEMS * (BLOCK / 32) + 1];
  if (ld_volatile_int(&ctrl->err)) return;
  const unsigned long long N = ld_volatile(&ctrl->n);
  constexpr unsigned long long TILE = (unsigned long long)BLOCK * ITEMS;
  const unsigned long long ntiles = (N + TILE - 1) / TILE;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    log[op].n_in = N;
    if (N == 0) {
      ctrl->n_s = 0;
      ctrl->n_side = 0;
    }
  }
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = BLOCK / 32;
  const bool wcap = maxw != ~0ull;
  for (;;) {
    const unsigned tile = next_tile(&ctrl->tickets[2], &s_tile);
    if (tile >= ntiles) break;
    const unsigned long long base = (unsigned long long)tile * TILE;
    uint64_t kx[ITEMS][W], kz[ITEMS][W];
    double kc[ITEMS];
    unsigned keep_b[ITEMS], side_b[ITEMS];
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const unsigned long long i = base + (unsigned long long)k * BLOCK + threadIdx.x;
      bool keep = false, sd = false;
      if (i < N) {
        load_key<W>(P, i, kx[k], kz[k]);
        kc[k] = P.c[i];
        keep = !(fabs(kc[k]) < thr);
        if (wcap) keep = keep && (weight<W>(kx[k], kz[k]) <= maxw);
        if (lw && maxlw != ~0ull) {  // MaxLossWeight: lost qubits, the X plane's upper words
          unsigned lost = 0;
#pragma unroll
          for (int w = 0; w < W; ++w)
            if (w >= (int)lw) lost += __popcll(kx[k][w]);
          keep = keep && lost <= maxlw;
        }
        if (!keep && npres > 0) sd = preserved<W>(kx[k], kz[k], pres_keys, pres_table, pres_mask);
      }
      keep_b[k] = __ballot_sync(kFull, keep);
      side_b[k] = __ballot_sync(kFull, sd);
    }
    const unsigned agg = tile_ranks<BLOCK, ITEMS>(keep_b, s_base);
    const unsigned agg2 = npres > 0 ? tile_ranks<BLOCK, ITEMS>(side_b, s_base2) : 0u;
    const unsigned long long packed = (unsigned long long)agg | ((unsigned long long)agg2 << 32);
    const unsigned long long excl = lookback(ts, tile, packed, epoch, ctrl, op, &s_slot);
    const unsigned long long kexcl = excl & 0xFFFFFFFFull, sexcl = excl >> 32;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const unsigned lt = (1u << lane) - 1u;
      if ((keep_b[k] >> lane) & 1u) {
        const unsigned long long r = kexcl + s_base[k * NW + warp] + __popc(keep_b[k] & lt);
        store_key<W>(P, r, kx[k], kz[k]);
        P.c[r] = kc[k];
      }
      if ((side_b[k] >> lane) & 1u) {
        const unsigned long long r = sexcl + s_base2[k * NW + warp] + __popc(side_b[k] & lt);
        uint64_t* rec = side + r * (2 * W + 1);
#pragma unroll
        for (int w = 0; w < W; ++w) {
          rec[w] = kx[k][w];
          rec[W + w] = kz[k][w];
        }
        rec[2 * W] = (uint64_t)__double_as_longlong(kc[k]);
      }
    }
    if (tile == ntiles - 1 && threadIdx.x == 0) {
      ctrl->n_s = kexcl + agg;
      ctrl->n_side = sexcl + agg2;
    }
  }
}

// Appends the preserved-but-dropped terms after the kept ones and publishes the count.
template <int W>
__global__ void k_commit_truncate(Planes P, Ctrl* ctrl, const uint64_t* side, int op, OpLog* log) {
  pdl_wait();
  if (threadIdx.x == 0 && blockIdx.x == 0)
    for (int t = 0; t < 4; ++t) ctrl->tickets[t] = 0;
  if (ld_volatile_int(&ctrl->err)) return;
  const unsigned long long kept = ctrl->n_s, nside = ctrl->n_side;
  for (unsigned long long j = threadIdx.x; j < nside; j += blockDim.x) {
    uint64_t x[W], z[W];
    double c;
    load_rec<W>(side, j, x, z, c);
    store_key<W>(P, kept + j, x, z);
    P.c[kept + j] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    ctrl->n = kept + nside;
    log[op].n_out = kept + nside;
    log[op].n_s = ctrl->n_s;
  }
}

// ---------------------------------------------------------------------------------------
// Clifford runs and diagonal channels: one in-place pass applying a list of local ops.
// ---------------------------------------------------------------------------------------
enum CliffCode : uint32_t {
  C_X = 0, C_Y, C_Z, C_H, C_S, C_SDAG, C_SQX, C_SQXDAG, C_SQY, C_SQYDAG,
  C_CNOT, C_CZ, C_CY,
  C_PAULI_ERROR, C_DEP1, C_DEP2,
  C_ROTC,  // Clifford-angle rotation on 1-2 qubits: axis bits in ax/az, sign of sin in f0
  C_PERR2  // two-qubit Pauli error: factor table f0 (16 doubles each) of the launch's tables
};

struct DevOp {
  uint32_t code;
  uint16_t w0, b0, w1, b1;
  uint16_t ax, az;  // bit0: qubit0, bit1: qubit1 (axis of C_ROTC)
  uint16_t two;
  uint16_t lw;      // lossy sums: first loss word of the X plane (two-qubit ops skip lost qubits)
  double f0, f1, f2;
};

constexpr int kMaxOpsPerLaunch = 256;
constexpr int kCliffBlock = 128;

template <int W, int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_clifford(Planes P, Ctrl* ctrl, const DevOp* ops, int nops, int op0, OpLog* log,
           const double* __restrict__ perr2) {
  pdl_wait();
  __shared__ DevOp s_ops[kMaxOpsPerLaunch];
  __shared__ uint64_t s_x[W][BLOCK];
  __shared__ uint64_t s_z[W][BLOCK];
  if (ld_volatile_int(&ctrl->err)) return;
  for (int o = threadIdx.x; o < nops; o += BLOCK) s_ops[o] = ops[o];
  __syncthreads();
  const unsigned long long N = ld_volatile(&ctrl->n);
  if (blockIdx.x == 0 && threadIdx.x == 0 && log) {
    for (int o = 0; o < nops; ++o) {
      log[op0 + o].n_in = N;
      log[op0 + o].n_s = N;
      log[op0 + o].n_new = 0;
      log[op0 + o].n_out = N;
    }
  }
  const unsigned t = threadIdx.x;
  for (unsigned long long i = (unsigned long long)blockIdx.x * BLOCK + t; i < N;
       i += (unsigned long long)gridDim.x * BLOCK) {
#pragma unroll
    for (int w = 0; w < W; ++w) {
      s_x[w][t] = P.x[(unsigned long long)w * P.cap + i];
      s_z[w][t] = P.z[(unsigned long long)w * P.cap + i];
    }
    double c = P.c[i];
    bool neg = false;
    for (int o = 0; o < nops; ++o) {
      const DevOp& d = s_ops[o];
      const uint64_t m0 = 1ull << d.b0, m1 = 1ull << d.b1;
      uint64_t x0w = s_x[d.w0][t], z0w = s_z[d.w0][t];
      const bool x0 = x0w & m0, z0 = z0w & m0;
      // lossy sums: which of the op's qubits are lost.  One-qubit ops need no test (a lost
      // qubit has x = z = 0, which every one-qubit rule leaves alone); two-qubit Cliffords,
      // depolarize2 and the two-qubit Pauli error skip the term (phase/clifford.rs:77,92,168;
      // noise.rs:98-102,122); a Clifford-angle rotation acts on the qubits that are not lost.
      bool l0 = false, l1 = false;
      if (d.lw) {
        const bool skip2 = d.code == C_CNOT || d.code == C_CZ || d.code == C_CY || d.code == C_DEP2 ||
                           d.code == C_PERR2;
        l0 = s_x[d.lw + d.w0][t] & m0;
        l1 = (skip2 || (d.code == C_ROTC && d.two)) ? (bool)(s_x[d.lw + d.w1][t] & m1) : false;
        if ((l0 || l1) && skip2) continue;
      }
      switch (d.code) {
        case C_X: neg ^= z0; break;
        case C_Y: neg ^= x0 ^ z0; break;
        case C_Z: neg ^= x0; break;
        case C_H:
          neg ^= x0 & z0;
          s_x[d.w0][t] = (x0w & ~m0) | (z0 ? m0 : 0);
          s_z[d.w0][t] = (z0w & ~m0) | (x0 ? m0 : 0);
          break;
        case C_S: neg ^= x0 & !z0; s_z[d.w0][t] = z0w ^ (x0 ? m0 : 0); break;
        case C_SDAG: neg ^= x0 & z0; s_z[d.w0][t] = z0w ^ (x0 ? m0 : 0); break;
        case C_SQX: neg ^= x0 & z0; s_x[d.w0][t] = x0w ^ (z0 ? m0 : 0); break;
        case C_SQXDAG: neg ^= !x0 & z0; s_x[d.w0][t] = x0w ^ (z0 ? m0 : 0); break;
        case C_SQY:
          neg ^= !x0 & z0;
          s_x[d.w0][t] = (x0w & ~m0) | (z0 ? m0 : 0);
          s_z[d.w0][t] = (z0w & ~m0) | (x0 ? m0 : 0);
          break;
        case C_SQYDAG:
          neg ^= x0 & !z0;
          s_x[d.w0][t] = (x0w & ~m0) | (z0 ? m0 : 0);
          s_z[d.w0][t] = (z0w & ~m0) | (x0 ? m0 : 0);
          break;
        case C_CNOT: case C_CZ: case C_CY: {
          const bool xc = x0, zc = z0;
          const bool xt = s_x[d.w1][t] & m1, zt = s_z[d.w1][t] & m1;
          bool nzc = zc, nxt = xt, nzt = zt;
          if (d.code == C_CNOT) {
            neg ^= xc & zt & (xt == zc);
            nzc = zc ^ zt;
            nxt = xt ^ xc;
          } else if (d.code == C_CZ) {
            neg ^= xc & xt & (zc ^ zt);
            nzc = zc ^ xt;
            nzt = zt ^ xc;
          } else {
            neg ^= xc & (xt ^ zt) & !(zc ^ zt);
            nzc = zc ^ xt ^ zt;
            nxt = xt ^ xc;
            nzt = zt ^ xc;
          }
          s_z[d.w0][t] = (s_z[d.w0][t] & ~m0) | (nzc ? m0 : 0);
          s_x[d.w1][t] = (s_x[d.w1][t] & ~m1) | (nxt ? m1 : 0);
          s_z[d.w1][t] = (s_z[d.w1][t] & ~m1) | (nzt ? m1 : 0);
          break;
        }
        case C_PAULI_ERROR: {
          const int code = (int)x0 | ((int)z0 << 1);
          if (code == 1) c = __dmul_rn(c, d.f0);
          else if (code == 2) c = __dmul_rn(c, d.f1);
          else if (code == 3) c = __dmul_rn(c, d.f2);
          break;
        }
        case C_DEP1: if (x0 | z0) c = __dmul_rn(c, d.f0); break;
        case C_PERR2: {  // factor of (P_q0, P_q1), code x | z << 1 on each qubit
          const bool x1 = s_x[d.w1][t] & m1, z1 = s_z[d.w1][t] & m1;
          const int code = ((int)x0 | ((int)z0 << 1)) << 2 | (int)x1 | ((int)z1 << 1);
          if (code) c = __dmul_rn(c, perr2[16 * (int)d.f0 + code]);
          break;
        }
        case C_DEP2: {
          const bool x1 = s_x[d.w1][t] & m1, z1 = s_z[d.w1][t] & m1;
          if (x0 | z0 | x1 | z1) c = __dmul_rn(c, d.f0);
          break;
        }
        case C_ROTC: {
          const bool ax0 = (d.ax & 1) && !l0, az0 = (d.az & 1) && !l0;
          bool x1 = false, z1 = false, ax1 = false, az1 = false;
          if (d.two) {
            x1 = s_x[d.w1][t] & m1;
            z1 = s_z[d.w1][t] & m1;
            ax1 = ((d.ax >> 1) & 1) && !l1;
            az1 = ((d.az >> 1) & 1) && !l1;
          }
          const bool anti = ((x0 & az0) ^ (z0 & ax0)) ^ ((x1 & az1) ^ (z1 & ax1));
          if (!anti) break;
          // phase of G*P per qubit (see rot_sign)
          auto g1 = [](bool gx, bool gz, bool px, bool pz) -> int {
            if (gx & !gz) return (px & pz) ? 1 : ((!px & pz) ? -1 : 0);
            if (gx & gz) return (!px & pz) ? 1 : ((px & !pz) ? -1 : 0);
            if (!gx & gz) return (px & !pz) ? 1 : ((px & pz) ? -1 : 0);
            return 0;
          };
          const int e = g1(ax0, az0, x0, z0) + g1(ax1, az1, x1, z1);
          const double eps = (((e + 1) & 3) == 0) ? 1.0 : -1.0;
          neg ^= (eps * d.f0) < 0.0;
          if (ax0) s_x[d.w0][t] ^= m0;
          if (az0) s_z[d.w0][t] ^= m0;
          if (d.two) {
            if (ax1) s_x[d.w1][t] ^= m1;
            if (az1) s_z[d.w1][t] ^= m1;
          }
          break;
        }
        default: break;
      }
    }
#pragma unroll
    for (int w = 0; w < W; ++w) {
      P.x[(unsigned long long)w * P.cap + i] = s_x[w][t];
      P.z[(unsigned long long)w * P.cap + i] = s_z[w][t];
    }
    P.c[i] = neg ? -c : c;
  }
}

// ---------------------------------------------------------------------------------------
// Reductions (deterministic: fixed element->thread map and fixed trees).
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ double block_sum(double v, double* s_red) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = __dadd_rn(v, __shfl_down_sync(kFull, v, o));
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) s_red[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    for (unsigned w = 0; w < blockDim.x / 32; ++w) r = __dadd_rn(r, s_red[w]);
  }
  __syncthreads();
  return r;
}

// Sum of coefficients of words without X bits: trace("Z?*") = overlap_with_zero.
template <int W>
__global__ void __launch_bounds__(256) k_owz(Planes P, const Ctrl* ctrl, double* partials) {
  pdl_wait();
  __shared__ double s_red[8];
  const unsigned long long N = ld_volatile(&ctrl->n);
  double acc = 0.0;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    uint64_t any = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) any |= P.x[(unsigned long long)w * P.cap + i];
    if (any == 0) acc = __dadd_rn(acc, P.c[i]);
  }
  const double b = block_sum(acc, s_red);
  if (threadIdx.x == 0) partials[blockIdx.x] = b;
}

static __global__ void k_sum_partials(const double* partials, int n, Ctrl* ctrl) {
  pdl_wait();
  __shared__ double s_red[8];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc = __dadd_rn(acc, partials[i]);
  const double b = block_sum(acc, s_red);
  if (threadIdx.x == 0) ctrl->sum = b;
}

// PauliPattern matcher (crates/ppvm-pauli-word/src/pattern/contains.rs:120-151).
struct PatItem {
  uint32_t kind;    // 0 = Position, 1 = Star, 2 = Repeat
  uint32_t accept;  // bit c set if Pauli code c (0=I 1=X 2=Z 3=Y) is accepted
  uint64_t arg;
};

template <int W>
__device__ __forceinline__ unsigned pauli_code(const uint64_t (&x)[W], const uint64_t (&z)[W],
                                               unsigned q) {
  uint64_t xw = 0, zw = 0;
#pragma unroll
  for (int w = 0; w < W; ++w)
    if ((int)(q >> 6) == w) {
      xw = x[w];
      zw = z[w];
    }
  return (unsigned)((xw >> (q & 63)) & 1u) | ((unsigned)((zw >> (q & 63)) & 1u) << 1);
}

// Pattern code of qubit q: pauli_code, or 4 for a lost qubit of a lossy sum (lw: first loss
// word of the X plane, 0 for a plain sum).  No pattern item accepts 4 (accept masks have four
// bits): L matches no Pauli pattern (crates/ppvm-pauli-word/src/pattern/contains.rs:25-41).
template <int W>
__device__ __forceinline__ unsigned pat_code(const uint64_t (&x)[W], const uint64_t (&z)[W], unsigned lw,
                                             unsigned q) {
  if (lw) {
    uint64_t l = 0;
#pragma unroll
    for (int w = 0; w < W; ++w)
      if ((int)(lw + (q >> 6)) == w) l = x[w];
    if ((l >> (q & 63)) & 1u) return 4u;
  }
  return pauli_code<W>(x, z, q);
}

template <int W>
__device__ bool pattern_match(const PatItem* items, int nitems, unsigned n, const uint64_t (&x)[W],
                              const uint64_t (&z)[W], unsigned lw) {
  unsigned pos = 0;
  for (int it = 0; it < nitems; ++it) {
    const PatItem p = items[it];
    if (p.kind == 0) {
      bool next = false;
      while (pos < n) {
        const unsigned q = pos++;
        const unsigned c = pat_code<W>(x, z, lw, q);
        if (q == p.arg) {
          next = (p.accept >> c) & 1u;
          break;
        }
        if (c == 0) continue;
        break;
      }
      if (!next) return false;
    } else if (p.kind == 1) {
      while (pos < n && ((p.accept >> pat_code<W>(x, z, lw, pos)) & 1u)) ++pos;
    } else {
      unsigned long long matched = 0;
      bool done = false;
      while (pos < n) {
        if ((p.accept >> pat_code<W>(x, z, lw, pos)) & 1u) {
          ++pos;
          if (++matched == p.arg) {
            done = true;
            break;
          }
        } else {
          if (matched < p.arg) return false;
          done = true;
          break;
        }
      }
      if (!done && matched != p.arg) return false;
    }
  }
  for (; pos < n; ++pos)
    if (pat_code<W>(x, z, lw, pos) != 0) return false;
  return true;
}

template <int W>
__global__ void __launch_bounds__(256)
k_trace(Planes P, const Ctrl* ctrl, const PatItem* items, int nitems, unsigned nq, double* partials,
        unsigned lw) {
  __shared__ double s_red[8];
  const unsigned long long N = ld_volatile(&ctrl->n);
  double acc = 0.0;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    uint64_t x[W], z[W];
    load_key<W>(P, i, x, z);
    if (pattern_match<W>(items, nitems, nq, x, z, lw)) acc = __dadd_rn(acc, P.c[i]);
  }
  const double b = block_sum(acc, s_red);
  if (threadIdx.x == 0) partials[blockIdx.x] = b;
}

template <int W>
__global__ void __launch_bounds__(256) k_weights(Planes P, const Ctrl* ctrl, uint32_t* out) {
  const unsigned long long N = ld_volatile(&ctrl->n);
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    uint64_t x[W], z[W];
    load_key<W>(P, i, x, z);
    out[i] = weight<W>(x, z);
  }
}

// ---------------------------------------------------------------------------------------
// Key index (cold paths: construction `+=`, overlap, equality).  table slot -> term index.
// ---------------------------------------------------------------------------------------
template <int W>
__device__ __forceinline__ void index_insert(const Planes& P, unsigned long long i,
                                             unsigned long long* table, unsigned long long mask,
                                             unsigned tepoch, Ctrl* ctrl) {
  uint64_t x[W], z[W];
  load_key<W>(P, i, x, z);
  const uint64_t h = hash_key<W>(x, z);
  const unsigned long long mine = make_slot(tepoch, (unsigned)(h >> 48), (unsigned)i);
  unsigned long long slot = h & mask;
  for (unsigned long long probe = 0; probe <= mask; ++probe) {
    const unsigned long long cur = ld_volatile(&table[slot]);
    if (slot_epoch(cur) != (tepoch & 0xFFFFu)) {
      const unsigned long long prev = atomicCAS(&table[slot], cur, mine);
      if (prev == cur) return;
      continue;
    }
    slot = (slot + 1) & mask;
  }
  set_err(ctrl, kErrProbe, -1);
}

template <int W>
__device__ __forceinline__ long long index_find(const Planes& P, const uint64_t (&x)[W],
                                                const uint64_t (&z)[W], const unsigned long long* table,
                                                unsigned long long mask, unsigned tepoch) {
  const uint64_t h = hash_key<W>(x, z);
  const unsigned tag = (unsigned)(h >> 48) & 0xFFFFu;
  unsigned long long slot = h & mask;
  for (unsigned long long probe = 0; probe <= mask; ++probe) {
    const unsigned long long cur = table[slot];
    if (slot_epoch(cur) != (tepoch & 0xFFFFu)) return -1;
    if (slot_tag(cur) == tag) {
      uint64_t jx[W], jz[W];
      load_key<W>(P, slot_idx(cur), jx, jz);
      bool eq = true;
#pragma unroll
      for (int w = 0; w < W; ++w) eq &= (jx[w] == x[w]) & (jz[w] == z[w]);
      if (eq) return slot_idx(cur);
    }
    slot = (slot + 1) & mask;
  }
  return -1;
}

template <int W>
__global__ void __launch_bounds__(256)
k_build_index(Planes P, Ctrl* ctrl, unsigned long long* table, unsigned long long mask, unsigned tepoch) {
  const unsigned long long N = ld_volatile(&ctrl->n);
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (unsigned long long)gridDim.x * blockDim.x)
    index_insert<W>(P, i, table, mask, tepoch, ctrl);
}

// `ps += (word, c)` for k new terms, strictly in order (one thread): existing key -> c += v,
// new key -> append (crates/ppvm-traits/src/map/hashmap.rs:40-44).
template <int W>
__global__ void k_add_terms_seq(Planes P, Ctrl* ctrl, const uint64_t* nx, const uint64_t* nz,
                                const double* nc, unsigned long long k, unsigned long long* table,
                                unsigned long long mask, unsigned tepoch) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  unsigned long long N = ctrl->n;
  for (unsigned long long t = 0; t < k; ++t) {
    uint64_t x[W], z[W];
#pragma unroll
    for (int w = 0; w < W; ++w) {
      x[w] = nx[t * W + w];
      z[w] = nz[t * W + w];
    }
    const long long j = index_find<W>(P, x, z, table, mask, tepoch);
    if (j >= 0) {
      P.c[j] = __dadd_rn(P.c[j], nc[t]);
    } else {
      if (N >= P.cap) {
        set_err(ctrl, kErrCapacity, -1);
        return;
      }
      store_key<W>(P, N, x, z);
      P.c[N] = nc[t];
      index_insert<W>(P, N, table, mask, tepoch, ctrl);
      ++N;
    }
  }
  ctrl->n = N;
}

// sum over b's terms of b[k] * a[k] (a indexed by `table`), per-block partials.
template <int W>
__global__ void __launch_bounds__(256)
k_overlap(Planes A, Planes B, const Ctrl* bctrl, const unsigned long long* table,
          unsigned long long mask, unsigned tepoch, double* partials, unsigned long long* mismatch) {
  __shared__ double s_red[8];
  const unsigned long long NB = ld_volatile(&bctrl->n);
  double acc = 0.0;
  unsigned long long miss = 0;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < NB;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    uint64_t x[W], z[W];
    load_key<W>(B, i, x, z);
    const long long j = index_find<W>(A, x, z, table, mask, tepoch);
    const double bv = B.c[i];
    if (j >= 0) {
      acc = __dadd_rn(acc, __dmul_rn(bv, A.c[j]));
      if (!(A.c[j] == bv)) ++miss;
    } else {
      acc = __dadd_rn(acc, __dmul_rn(bv, 0.0));
      ++miss;
    }
  }
  const double b = block_sum(acc, s_red);
  if (threadIdx.x == 0) partials[blockIdx.x] = b;
  if (miss) atomicAdd(mismatch, miss);
}

}  // namespace ppvm
