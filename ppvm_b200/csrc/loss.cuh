// loss.cuh — the loss channels of lossy sums (crates/ppvm-pauli-sum/src/sum/noise.rs:165-275).
//
// A lossy sum over n qubits keeps W = 2 * Wr words per plane (Wr = ceil(n/64)): the X plane's
// words [Wr, 2Wr) hold the loss bits, the Z plane's upper words stay zero, and a lost qubit has
// x = z = 0 in the lower words.  So L matches no Pauli, weights count it, and every gate of the
// plain engine that touches only its qubits' X/Z bits treats it as the reference does.
//
// The three channels of the reference, per term (v: its coefficient before the channel):
//   loss_channel(q, p)        L on q: child (q -> I, v*p), term kept;  else: v *= 1 - p
//   reset_loss_channel(q)     L on q: v *= 0;  I or Z on q: child (q -> L, v);  X, Y: nothing
//   correlated_loss_channel   (L,L): children (I,L) v*p2, (L,I) v*p2, (I,I) v*p0, term kept;
//     (a, b; p[3])            one lost: child with the lost qubit -> I, v*p1; v *= 1 - p2;
//                             none lost: v *= 1 - 2 p1 - p0
// The first two go through map_insert (data.rs:204-226): children are merged one at a time
// in parent order into the map (`+=`, new keys appended).  The third goes through
// map_insert_multiple (data.rs:227-248): children are summed per key in generation order
// into a fresh map, and consume (data.rs:180-189) then merges the smaller of (children, data)
// into the larger, whose order the result keeps.
//
// A child key can have up to three parents (reset: the I and Z terms; correlated (I,I): the
// (L,L), (I,L) and (L,I) terms), all of which differ from it only on the channel's qubits.
// So every output is computed by pulling: each output key enumerates its possible parents,
// finds them in an index of the sum, orders them by (parent index, child slot) — the order in
// which the reference generates children — and folds their contributions as the reference
// merges them.  One pass writes the whole output to the alternate planes:
//   k_loss_index   key index of the sum (slot -> term); zeroes the counters
//   k_loss_count   new keys (children absent from the sum, counted at their first parent) and
//                  distinct child keys (correlated channel: which map consume keeps)
//   k_loss_emit    capacity check, then every term at its place with its new coefficient and
//                  every new key after them, both in the reference's order (decoupled
//                  look-back); with the correlated channel and more distinct child keys than
//                  terms, the child keys first in generation order, then the other terms.
//                  The last block publishes the count and the op log.
#pragma once

#include "kernels.cuh"

namespace ppvm {

enum LossMode : int { kLossChannel = 0, kResetLoss = 1, kCorrelatedLoss = 2 };

struct LossOp {
  int mode;
  uint32_t qa, qb;  // qubits (qb = qa for the one-qubit channels)
  uint32_t lw;      // first loss word of the X plane (= Wr)
  double p0, p1, p2;
  double keep1;     // loss: 1 - p;  correlated: 1 - p2 (one lost qubit)
  double keep0;     // correlated: 1 - 2 p1 - p0 (no lost qubit)
};

// Pauli code of qubit q in a lossy key: 0 I, 1 X, 2 Z, 3 Y, 4 L.  Indexes stay static so the
// key stays in registers.
template <int W>
__device__ __forceinline__ int loss_code(const uint64_t (&x)[W], const uint64_t (&z)[W], unsigned lw, uint32_t q) {
  const unsigned w = q >> 6;
  const uint64_t m = 1ull << (q & 63);
  uint64_t xw = 0, zw = 0, lwd = 0;
#pragma unroll
  for (int i = 0; i < W; ++i) {
    if (i == (int)w) {
      xw = x[i];
      zw = z[i];
    }
    if (i == (int)(lw + w)) lwd = x[i];
  }
  if (lwd & m) return 4;
  return (int)((xw & m) != 0) | ((int)((zw & m) != 0) << 1);
}

template <int W>
__device__ __forceinline__ void loss_set(uint64_t (&x)[W], uint64_t (&z)[W], unsigned lw, uint32_t q, int code) {
  const unsigned w = q >> 6;
  const uint64_t m = 1ull << (q & 63);
#pragma unroll
  for (int i = 0; i < W; ++i) {
    if (i == (int)w) {
      x[i] = (code == 1 || code == 3) ? (x[i] | m) : (x[i] & ~m);
      z[i] = (code == 2 || code == 3) ? (z[i] | m) : (z[i] & ~m);
    }
    if (i == (int)(lw + w)) x[i] = code == 4 ? (x[i] | m) : (x[i] & ~m);
  }
}

// The possible parents of a key whose codes on (qa, qb) are (ca, cb): their codes, the slot of
// the key among each parent's children, and the factor on the parent's coefficient.  Returns
// how many (0..3).
__device__ __forceinline__ int loss_parents(const LossOp& op, int ca, int cb, int (&pa)[3], int (&pb)[3],
                                            int (&slot)[3], double (&f)[3]) {
  if (op.mode == kLossChannel) {
    if (ca != 0) return 0;
    pa[0] = 4, pb[0] = cb, slot[0] = 0, f[0] = op.p0;
    return 1;
  }
  if (op.mode == kResetLoss) {
    if (ca != 4) return 0;
    pa[0] = 0, pb[0] = cb, slot[0] = 0, f[0] = 1.0;  // the child keeps v: v * 1.0 is v exactly
    pa[1] = 2, pb[1] = cb, slot[1] = 0, f[1] = 1.0;
    return 2;
  }
  if (ca == 0 && cb == 4) {
    pa[0] = 4, pb[0] = 4, slot[0] = 0, f[0] = op.p2;
    return 1;
  }
  if (ca == 4 && cb == 0) {
    pa[0] = 4, pb[0] = 4, slot[0] = 1, f[0] = op.p2;
    return 1;
  }
  if (ca == 0 && cb == 0) {
    pa[0] = 4, pb[0] = 4, slot[0] = 2, f[0] = op.p0;
    pa[1] = 0, pb[1] = 4, slot[1] = 0, f[1] = op.p1;
    pa[2] = 4, pb[2] = 0, slot[2] = 0, f[2] = op.p1;
    return 3;
  }
  if (cb == 0 && ca >= 1 && ca <= 3) {
    pa[0] = ca, pb[0] = 4, slot[0] = 0, f[0] = op.p1;
    return 1;
  }
  if (ca == 0 && cb >= 1 && cb <= 3) {
    pa[0] = 4, pb[0] = cb, slot[0] = 0, f[0] = op.p1;
    return 1;
  }
  return 0;
}

// The codes on (qa, qb) of child `slot` of a term with codes (ca, cb); false if it has none.
__device__ __forceinline__ bool loss_child(const LossOp& op, int ca, int cb, int slot, int& na, int& nb) {
  na = ca, nb = cb;
  if (op.mode == kLossChannel) {
    if (slot != 0 || ca != 4) return false;
    na = 0;
    return true;
  }
  if (op.mode == kResetLoss) {
    if (slot != 0 || !(ca == 0 || ca == 2)) return false;
    na = 4;
    return true;
  }
  if (ca == 4 && cb == 4) {
    if (slot == 0) na = 0, nb = 4;
    else if (slot == 1) na = 4, nb = 0;
    else na = 0, nb = 0;
    return true;
  }
  if (slot != 0) return false;
  if (cb == 4) {
    nb = 0;
    return true;
  }
  if (ca == 4) {
    na = 0;
    return true;
  }
  return false;
}

// The coefficient of an existing term after the channel's own scaling.
__device__ __forceinline__ double loss_own(const LossOp& op, int ca, int cb, double v) {
  if (op.mode == kLossChannel) return ca == 4 ? v : __dmul_rn(v, op.keep1);
  if (op.mode == kResetLoss) return ca == 4 ? __dmul_rn(v, 0.0) : v;
  if (ca == 4 && cb == 4) return v;
  if (ca == 4 || cb == 4) return __dmul_rn(v, op.keep1);
  return __dmul_rn(v, op.keep0);
}

struct LossFound {
  int n;
  long long idx[3];
  int slot[3];
  double val[3];  // the child's contribution: parent coefficient * factor
};

// Finds the existing parents of key (x, z), sorted by (index, slot).
template <int W>
__device__ __forceinline__ void loss_find_parents(const LossOp& op, const Planes& P, const uint64_t (&x)[W],
                                                  const uint64_t (&z)[W], const unsigned long long* table,
                                                  unsigned long long mask, unsigned tepoch, LossFound& F) {
  const int ca = loss_code<W>(x, z, op.lw, op.qa);
  const int cb = op.mode == kCorrelatedLoss ? loss_code<W>(x, z, op.lw, op.qb) : 0;
  int pa[3], pb[3], sl[3];
  double f[3];
  const int np = loss_parents(op, ca, cb, pa, pb, sl, f);
  F.n = 0;
  for (int k = 0; k < np; ++k) {
    uint64_t px[W], pz[W];
#pragma unroll
    for (int w = 0; w < W; ++w) px[w] = x[w], pz[w] = z[w];
    loss_set<W>(px, pz, op.lw, op.qa, pa[k]);
    if (op.mode == kCorrelatedLoss) loss_set<W>(px, pz, op.lw, op.qb, pb[k]);
    const long long j = index_find<W>(P, px, pz, table, mask, tepoch);
    if (j < 0) continue;
    int at = F.n++;  // insertion sort by (index, slot)
    while (at > 0 && (F.idx[at - 1] > j || (F.idx[at - 1] == j && F.slot[at - 1] > sl[k]))) {
      F.idx[at] = F.idx[at - 1];
      F.slot[at] = F.slot[at - 1];
      F.val[at] = F.val[at - 1];
      --at;
    }
    F.idx[at] = j;
    F.slot[at] = sl[k];
    F.val[at] = __dmul_rn(P.c[j], f[k]);
  }
}

// The key's coefficient after the channel.  own: its scaled coefficient if it is a term of
// the sum (has_own).  map_insert (loss, reset): own, then each child added in order;
// map_insert_multiple (correlated): the children summed in order, then added to own.
__device__ __forceinline__ double loss_fold(const LossOp& op, bool has_own, double own, const LossFound& F) {
  if (op.mode != kCorrelatedLoss) {
    double acc = has_own ? own : F.val[0];
    for (int k = has_own ? 0 : 1; k < F.n; ++k) acc = __dadd_rn(acc, F.val[k]);
    return acc;
  }
  if (F.n == 0) return own;
  double s = F.val[0];
  for (int k = 1; k < F.n; ++k) s = __dadd_rn(s, F.val[k]);
  return has_own ? __dadd_rn(own, s) : s;
}

// Per term i: the child keys it generates first (first[s]), and which of those are new.
template <int W>
__device__ __forceinline__ int loss_children(const LossOp& op, const Planes& P, unsigned long long i,
                                             const uint64_t (&x)[W], const uint64_t (&z)[W],
                                             const unsigned long long* table, unsigned long long mask,
                                             unsigned tepoch, bool (&first)[3], bool (&isnew)[3]) {
  const int ca = loss_code<W>(x, z, op.lw, op.qa);
  const int cb = op.mode == kCorrelatedLoss ? loss_code<W>(x, z, op.lw, op.qb) : 0;
  const int S = op.mode == kCorrelatedLoss ? 3 : 1;
  int nfirst = 0;
  for (int s = 0; s < 3; ++s) {
    first[s] = false;
    isnew[s] = false;
    int na, nb;
    if (s >= S || !loss_child(op, ca, cb, s, na, nb)) continue;
    uint64_t cx[W], cz[W];
#pragma unroll
    for (int w = 0; w < W; ++w) cx[w] = x[w], cz[w] = z[w];
    loss_set<W>(cx, cz, op.lw, op.qa, na);
    if (op.mode == kCorrelatedLoss) loss_set<W>(cx, cz, op.lw, op.qb, nb);
    LossFound F;
    loss_find_parents<W>(op, P, cx, cz, table, mask, tepoch, F);
    // this term is among the child's parents; it generates the child first when no parent
    // comes before (index, slot) = (i, s)
    if (F.n > 0 && F.idx[0] == (long long)i && F.slot[0] == s) {
      first[s] = true;
      ++nfirst;
      isnew[s] = index_find<W>(P, cx, cz, table, mask, tepoch) < 0;
    }
  }
  return nfirst;
}

template <int W>
__global__ void __launch_bounds__(256)
k_loss_index(Planes P, Ctrl* ctrl, unsigned long long* table, unsigned long long mask, unsigned tepoch, int op,
             OpLog* log) {
  pdl_wait();
  if (ld_volatile_int(&ctrl->err)) return;
  const unsigned long long N = ld_volatile(&ctrl->n);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctrl->n_s = 0;      // new keys
    ctrl->n_pairs = 0;  // distinct child keys
    log[op].n_in = N;
  }
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (unsigned long long)gridDim.x * blockDim.x)
    index_insert<W>(P, i, table, mask, tepoch, ctrl);
}

// k_loss_count and k_loss_emit are compiled once per channel (M = op.mode): with the mode a
// constant, each keeps only its channel's children and parents, and far fewer registers.
template <int W, int M>
__global__ void __launch_bounds__(256)
k_loss_count(Planes P, Ctrl* ctrl, LossOp op_in, const unsigned long long* table, unsigned long long mask,
             unsigned tepoch) {
  pdl_wait();
  LossOp op = op_in;
  op.mode = M;
  __shared__ unsigned long long s_new, s_aux;
  if (ld_volatile_int(&ctrl->err)) return;
  if (threadIdx.x == 0) s_new = s_aux = 0;
  __syncthreads();
  const unsigned long long N = ld_volatile(&ctrl->n);
  unsigned long long nn = 0, na = 0;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    uint64_t x[W], z[W];
    load_key<W>(P, i, x, z);
    if constexpr (M == kLossChannel) {
      // a lost qubit's term is the only parent of its child (the qubit as I): the child is new
      // when that key is absent
      if (loss_code<W>(x, z, op.lw, op.qa) == 4) {
        loss_set<W>(x, z, op.lw, op.qa, 0);
        nn += index_find<W>(P, x, z, table, mask, tepoch) < 0;
      }
    } else {
      bool first[3], isnew[3];
      na += loss_children<W>(op, P, i, x, z, table, mask, tepoch, first, isnew);
      nn += (unsigned)isnew[0] + (unsigned)isnew[1] + (unsigned)isnew[2];
    }
  }
  if (nn) atomicAdd(&s_new, nn);
  if (na) atomicAdd(&s_aux, na);
  __syncthreads();
  if (threadIdx.x == 0) {
    if (s_new) atomicAdd(&ctrl->n_s, s_new);
    if (s_aux) atomicAdd(&ctrl->n_pairs, s_aux);
  }
}

// Exclusive prefix of v over the block's threads (in thread order) and the block total.
template <int BLOCK>
__device__ __forceinline__ unsigned block_excl(unsigned v, unsigned* s_w, unsigned& total) {
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned t = __shfl_up_sync(kFull, inc, o);
    if (lane >= (unsigned)o) inc += t;
  }
  __syncthreads();
  if (lane == 31) s_w[warp] = inc;
  __syncthreads();
  unsigned base = 0;
  total = 0;
#pragma unroll
  for (int w = 0; w < BLOCK / 32; ++w) {
    const unsigned t = s_w[w];
    if (w < (int)warp) base += t;
    total += t;
  }
  return base + inc - v;
}

template <int W, int BLOCK, int M>
__global__ void __launch_bounds__(BLOCK)
k_loss_emit(Planes P, Planes O, Ctrl* ctrl, LossOp op_in, const unsigned long long* table, unsigned long long mask,
            unsigned tepoch, unsigned long long* ts, unsigned long long* ts2, unsigned epoch, unsigned epoch2,
            int opi, OpLog* log) {
  pdl_wait();
  LossOp op = op_in;
  op.mode = M;
  __shared__ unsigned s_tile;
  __shared__ unsigned long long s_slot;
  __shared__ unsigned s_w[BLOCK / 32];
  if (ld_volatile_int(&ctrl->err)) return;
  const unsigned long long N = ld_volatile(&ctrl->n);
  const unsigned long long n_new = ld_volatile(&ctrl->n_s);
  const unsigned long long n_aux = ld_volatile(&ctrl->n_pairs);
  if (N + n_new > O.cap) {  // nothing has been written: grow and replay from this op
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      ctrl->cap_needed = N + n_new;
      set_err(ctrl, kErrCapacity, opi);
    }
    return;
  }
  // consume keeps the order of the larger map: the child keys' when they outnumber the terms
  const bool aux_first = op.mode == kCorrelatedLoss && n_aux > N;
  const unsigned long long ntiles = (N + BLOCK - 1) / BLOCK;
  if constexpr (M == kLossChannel) {
    // per term one index lookup: a term with L on qa keeps v and, when the key with I there is
    // absent, makes it as a new key with v * p (appended in parent order); a term with I on
    // qa takes v * (1 - p) plus p times the coefficient of the key with L there, if present;
    // X, Y, Z take v * (1 - p)
    for (;;) {
      const unsigned tile = next_tile(&ctrl->tickets[0], &s_tile);
      if (tile >= ntiles) break;
      const unsigned long long i = (unsigned long long)tile * BLOCK + threadIdx.x;
      uint64_t x[W], z[W];
      bool isnew = false;
      double v = 0.0, own = 0.0;
      if (i < N) {
        load_key<W>(P, i, x, z);
        v = P.c[i];
        const int ca = loss_code<W>(x, z, op.lw, op.qa);
        if (ca == 4 || ca == 0) {
          uint64_t kx[W], kz[W];
#pragma unroll
          for (int w = 0; w < W; ++w) kx[w] = x[w], kz[w] = z[w];
          loss_set<W>(kx, kz, op.lw, op.qa, ca == 4 ? 0 : 4);
          const long long j = index_find<W>(P, kx, kz, table, mask, tepoch);
          if (ca == 4) {
            own = v;
            isnew = j < 0;
          } else {
            own = __dmul_rn(v, op.keep1);
            if (j >= 0) own = __dadd_rn(own, __dmul_rn(P.c[j], op.p0));
          }
        } else {
          own = __dmul_rn(v, op.keep1);
        }
      }
      unsigned t1;
      const unsigned e1 = block_excl<BLOCK>(isnew ? 1u : 0u, s_w, t1);
      const unsigned long long x1 = lookback(ts, tile, t1, epoch, ctrl, opi, &s_slot);
      if (i < N) {
        store_key<W>(O, i, x, z);
        O.c[i] = own;
        if (isnew) {
          const unsigned long long r = N + x1 + e1;
          loss_set<W>(x, z, op.lw, op.qa, 0);
          store_key<W>(O, r, x, z);
          O.c[r] = __dmul_rn(v, op.p0);
        }
      }
    }
  } else
  for (;;) {
    const unsigned tile = next_tile(&ctrl->tickets[0], &s_tile);
    if (tile >= ntiles) break;
    const unsigned long long i = (unsigned long long)tile * BLOCK + threadIdx.x;
    uint64_t x[W], z[W];
    bool first[3] = {false, false, false}, isnew[3] = {false, false, false};
    bool rest = false;  // aux_first: a term that is no child key (goes after the child keys)
    double own = 0.0;
    if (i < N) {
      load_key<W>(P, i, x, z);
      loss_children<W>(op, P, i, x, z, table, mask, tepoch, first, isnew);
      const int ca = loss_code<W>(x, z, op.lw, op.qa);
      const int cb = op.mode == kCorrelatedLoss ? loss_code<W>(x, z, op.lw, op.qb) : 0;
      own = loss_own(op, ca, cb, P.c[i]);
      if (aux_first) {
        LossFound F;
        loss_find_parents<W>(op, P, x, z, table, mask, tepoch, F);
        rest = F.n == 0;
      }
    }
    // stream 1: new keys (or, aux_first, every first-generated child key); stream 2: rest
    unsigned c1 = 0;
    for (int s = 0; s < 3; ++s) c1 += aux_first ? (unsigned)first[s] : (unsigned)isnew[s];
    unsigned t1, t2;
    const unsigned e1 = block_excl<BLOCK>(c1, s_w, t1);
    const unsigned long long x1 = lookback(ts, tile, t1, epoch, ctrl, opi, &s_slot);
    unsigned long long x2 = 0;
    unsigned e2 = 0;
    if (aux_first) {
      e2 = block_excl<BLOCK>(rest ? 1u : 0u, s_w, t2);
      x2 = lookback(ts2, tile, t2, epoch2, ctrl, opi, &s_slot);
    }
    if (i < N) {
      if (!aux_first || rest) {  // the term itself, with its coefficient after the channel
        LossFound F;
        loss_find_parents<W>(op, P, x, z, table, mask, tepoch, F);
        const unsigned long long r = aux_first ? n_aux + x2 + e2 : i;
        store_key<W>(O, r, x, z);
        O.c[r] = loss_fold(op, true, own, F);
      }
      unsigned long long r = (aux_first ? 0ull : N) + x1 + e1;
      const int ca = loss_code<W>(x, z, op.lw, op.qa);
      const int cb = op.mode == kCorrelatedLoss ? loss_code<W>(x, z, op.lw, op.qb) : 0;
      for (int s = 0; s < 3; ++s) {
        if (!(aux_first ? first[s] : isnew[s])) continue;
        int na, nb;
        loss_child(op, ca, cb, s, na, nb);
        uint64_t cx[W], cz[W];
#pragma unroll
        for (int w = 0; w < W; ++w) cx[w] = x[w], cz[w] = z[w];
        loss_set<W>(cx, cz, op.lw, op.qa, na);
        if (op.mode == kCorrelatedLoss) loss_set<W>(cx, cz, op.lw, op.qb, nb);
        LossFound F;
        loss_find_parents<W>(op, P, cx, cz, table, mask, tepoch, F);
        const long long j = isnew[s] ? -1 : index_find<W>(P, cx, cz, table, mask, tepoch);
        double cown = 0.0;
        if (j >= 0) {
          const int ja = loss_code<W>(cx, cz, op.lw, op.qa);
          const int jb = op.mode == kCorrelatedLoss ? loss_code<W>(cx, cz, op.lw, op.qb) : 0;
          cown = loss_own(op, ja, jb, P.c[j]);
        }
        store_key<W>(O, r, cx, cz);
        O.c[r] = loss_fold(op, j >= 0, cown, F);
        ++r;
      }
    }
  }
  if (last_block_done(&ctrl->done) && threadIdx.x == 0) {
    for (int t = 0; t < 4; ++t) ctrl->tickets[t] = 0;
    if (ld_volatile_int(&ctrl->err)) return;
    log[opi].n_s = N;
    log[opi].n_new = n_new;
    log[opi].n_out = N + n_new;
    ctrl->n = N + n_new;
  }
}

}  // namespace ppvm
