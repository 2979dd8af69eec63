// runs.cuh — fused runs of single-qubit X-type or Z-type rotations.
//
// A run is a sequence of RX rotations on distinct qubits (or of RZ rotations on distinct
// qubits) with no other op in between, optionally ending in TRUNCATE.  During such a run a
// term's Z plane (RX) or X plane (RZ) never changes: it is the invariant plane v.  Gate j on
// qubit q acts on a term iff v has bit q, and then only flips bit q of the other plane f.
// So the terms sharing (v, f with the bits M = v & Q cleared) — Q the run's qubits — form a
// group that evolves on its own: its members are the 2^|M| words f0 | pdep(c, M), c in
// [0, 2^|M|).  The reference processes the run gate by gate over the whole map
// (PauliSum::map_insert per gate, crates/ppvm-pauli-sum/src/sum/data.rs:204-226); here each
// group is loaded once, the gates of the run are applied in the same order with the same
// arithmetic as a butterfly over coordinates c in shared memory (existence tracked
// separately from the coefficient, as a map entry exists even with coefficient 0), and the
// truncation that ends the run is applied before anything is written back.  The term set
// and every coefficient are identical to the reference's; only the output order differs
// (untouched terms in order, then groups by their first member, members by coordinate).
//
// Kernels, in order: k_run_classify (group keys into a hash table, members counted; terms
// outside every group compacted to the output with the truncation), k_run_order
// (deterministic group numbering by first member, member offsets), k_run_scatter (member
// lists), k_run_groups (butterfly + truncation + ordered write; its last block publishes the
// counts and the op log).
#pragma once

#include "kernels.cuh"

namespace ppvm {

constexpr int kRunMaxK = 10;       // groups up to 2^10 coordinates in shared memory
constexpr int kRunMaxGates = 256;  // gates per fused run
constexpr int kRunWarps = 4;       // warps of a k_run_groups block
constexpr int kRunTileGroups = 16; // groups per look-back tile of k_run_groups (at most 32)
constexpr unsigned long long kRunTileMinGroups = 8192;  // fewer groups: one look-back per group
constexpr unsigned long long kRunLogScratchBit = 1ull << 63;  // in the op log of a run's first gate
constexpr int kErrFallback = 4;    // device error: a group exceeds kRunMaxK; rerun per gate

struct RunDesc {
  uint32_t cls;   // 0: RX run (v = z plane, f = x plane); 1: RZ run (v = x, f = z)
  uint32_t L;     // gates
  uint64_t Q[kMaxW];
  uint32_t q[kRunMaxGates];
  double sn[kRunMaxGates];
  double cs[kRunMaxGates];
};

struct RunScratch {
  uint32_t* gslot;     // per term: group slot (kNone = untouched)
  uint32_t* grp_min;   // per table slot: smallest member index
  uint32_t* grp_cnt;   // per table slot: member count
  uint32_t* grp_ord;   // per table slot: group ordinal
  uint32_t* g_start;   // per group
  uint32_t* g_cnt;
  uint32_t* g_rep;
  uint32_t* g_fill;
  uint32_t* mcoord;    // per member, in group order: its coordinate index (bits of f at M)
  double* mcoef;       // per member, in group order: its coefficient
  uint64_t* gkey;      // per group: v[W] then f outside the coordinates, f0[W]
  unsigned long long* created;  // per gate of the run: children created
};

template <int W>
__device__ __forceinline__ void split_planes(uint32_t cls, const uint64_t (&x)[W], const uint64_t (&z)[W],
                                             uint64_t (&v)[W], uint64_t (&f)[W]) {
#pragma unroll
  for (int w = 0; w < W; ++w) {
    v[w] = cls == 0 ? z[w] : x[w];
    f[w] = cls == 0 ? x[w] : z[w];
  }
}

// ---------------------------------------------------------------------------------------
// Classifies every term and, in the same pass, writes the terms the run does not touch
// (no qubit of the run in the invariant plane) to the front of the output planes, in index
// order, with the run's TRUNCATE applied to them (tile ranks + decoupled look-back).  Touched
// terms join their group in the hash table.
template <int W, int BLOCK, int ITEMS>
__global__ void __launch_bounds__(BLOCK)
k_run_classify(Planes P, Planes O, Ctrl* ctrl, const RunDesc* rd, RunScratch R, unsigned long long* table,
               unsigned long long tmask, unsigned tepoch, int trunc, double thr, unsigned long long maxw,
               unsigned long long* ts, unsigned epoch, int op) {
  pdl_wait();
  __shared__ unsigned s_tile;
  __shared__ unsigned long long s_slot;
  __shared__ unsigned s_base[ITEMS * (BLOCK / 32) + 1];
  __shared__ int s_err;
  __shared__ uint16_t s_gidx[64 * W];  // qubit -> its gate's index in the run
  if (threadIdx.x == 0) s_err = ld_volatile_int(&ctrl->err);
  for (unsigned j = threadIdx.x; j < rd->L; j += BLOCK) s_gidx[rd->q[j]] = (uint16_t)j;
  __syncthreads();
  if (s_err) return;
  const unsigned long long N = ld_volatile(&ctrl->n);
  constexpr unsigned long long TILE = (unsigned long long)BLOCK * ITEMS;
  const unsigned long long ntiles = (N + TILE - 1) / TILE;
  if (blockIdx.x == 0 && threadIdx.x == 0 && N == 0) ctrl->n_s = 0;
  const uint32_t cls = rd->cls;
  uint64_t Q[W];
#pragma unroll
  for (int w = 0; w < W; ++w) Q[w] = rd->Q[w];
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = BLOCK / 32;
  const bool wcap = maxw != ~0ull;
  for (;;) {
    const unsigned tile = next_tile(&ctrl->tickets[1], &s_tile);
    if (tile >= ntiles) break;
    const unsigned long long base = (unsigned long long)tile * TILE;
    uint64_t kx[ITEMS][W], kz[ITEMS][W];
    double kc[ITEMS];
    unsigned bal[ITEMS];
    unsigned fb = 0;  // fallback: the largest gate cut among this thread's wide terms
#pragma unroll
    for (int it = 0; it < ITEMS; ++it) {
      const unsigned long long i = base + (unsigned long long)it * BLOCK + threadIdx.x;
      bool keep = false;
      if (i < N) {
        uint64_t v[W], f[W], M[W];
        load_key<W>(P, i, kx[it], kz[it]);
        split_planes<W>(cls, kx[it], kz[it], v, f);
        unsigned k = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) {
          M[w] = v[w] & Q[w];
          k += __popcll(M[w]);
          f[w] &= ~M[w];
        }
        if (k == 0) {  // untouched by the run
          R.gslot[i] = kNone;
          kc[it] = P.c[i];
          keep = true;
          if (trunc) {
            keep = !(fabs(kc[it]) < thr);
            if (wcap) keep = keep && (weight<W>(kx[it], kz[it]) <= maxw);
          }
        } else if (k > (unsigned)kRunMaxK) {
          // v is invariant through the run, so this term and all its descendants keep these
          // k coordinates: the run from gate p on, p = 1 + the gate index of the term's
          // (k - kRunMaxK)-th coordinate in gate order, holds at most kRunMaxK of them.  The
          // host runs the gates before the largest such p one at a time and fuses the rest.
          unsigned hi[kRunMaxK + 1];  // the kRunMaxK+1 largest gate indices, descending
          unsigned nhi = 0;
#pragma unroll
          for (int w = 0; w < W; ++w) {
            uint64_t m = M[w];
            while (m) {
              unsigned gi = s_gidx[w * 64 + (__ffsll((long long)m) - 1)];
              m &= m - 1;
              if (nhi == kRunMaxK + 1 && gi <= hi[kRunMaxK]) continue;
              unsigned r = nhi < kRunMaxK + 1 ? nhi++ : kRunMaxK;
              while (r > 0 && hi[r - 1] < gi) {
                hi[r] = hi[r - 1];
                --r;
              }
              hi[r] = gi;
            }
          }
          fb = max(fb, hi[kRunMaxK] + 1u);  // reported once per warp below
          R.gslot[i] = kNone;
        } else {
          const uint64_t h = hash_key<W>(v, f);
          const unsigned tag = (unsigned)(h >> 48) & 0xFFFFu;
          const unsigned long long mine = make_slot(tepoch, tag, (unsigned)i);
          unsigned long long slot = h & tmask;
          unsigned long long probes = 0;
          while (true) {
            const unsigned long long cur = ld_volatile(&table[slot]);
            if (slot_epoch(cur) != (tepoch & 0xFFFFu)) {
              const unsigned long long prev = atomicCAS(&table[slot], cur, mine);
              if (prev != cur) continue;
              break;  // new group
            }
            if (slot_tag(cur) == tag) {
              uint64_t jx[W], jz[W], jv[W], jf[W];
              load_key<W>(P, slot_idx(cur), jx, jz);
              split_planes<W>(cls, jx, jz, jv, jf);
              bool eq = true;
#pragma unroll
              for (int w = 0; w < W; ++w) eq &= (jv[w] == v[w]) & ((jf[w] & ~M[w]) == f[w]);
              if (eq) break;  // same group
            }
            slot = (slot + 1) & tmask;
            if (++probes > tmask) {
              set_err(ctrl, kErrProbe, op);
              break;
            }
          }
          R.gslot[i] = (uint32_t)slot;
          atomicMin(&R.grp_min[slot], (uint32_t)i);
          atomicAdd(&R.grp_cnt[slot], 1u);
        }
      }
      bal[it] = __ballot_sync(kFull, keep);
    }
    // terms with more than kRunMaxK coordinates: one report per warp instead of one atomic on
    // the same two words per term (a wide run has millions of such terms)
    fb = __reduce_max_sync(kFull, fb);
    if (fb && lane == 0) {
      if (ld_volatile(&ctrl->fb_cut) < fb) atomicMax(&ctrl->fb_cut, (unsigned long long)fb);
      if (!ld_volatile_int(&ctrl->err)) set_err(ctrl, kErrFallback, op);
    }
    const unsigned agg = tile_ranks<BLOCK, ITEMS>(bal, s_base);
    const unsigned long long excl = lookback(ts, tile, agg, epoch, ctrl, op, &s_slot);
#pragma unroll
    for (int it = 0; it < ITEMS; ++it)
      if ((bal[it] >> lane) & 1u) {
        const unsigned long long r = excl + s_base[it * NW + warp] + __popc(bal[it] & ((1u << lane) - 1u));
        store_key<W>(O, r, kx[it], kz[it]);
        O.c[r] = kc[it];
      }
    if (tile == ntiles - 1 && threadIdx.x == 0) ctrl->n_s = excl + agg;
  }
}

// Numbers the groups by their smallest member (index order) and lays out member lists.
// While the sum holds fewer than 2^21 terms (every block reads the same N), both running
// counts travel in one look-back value, groups in the low 21 bits and members in the next 21:
// one chain per tile instead of two.
constexpr int kOrderPackBits = 21;
template <int BLOCK, int ITEMS>
__global__ void __launch_bounds__(BLOCK)
k_run_order(Ctrl* ctrl, RunScratch R, unsigned long long* ts_a, unsigned long long* ts_b, unsigned ep_a,
            unsigned ep_b, int op) {
  pdl_wait();
  __shared__ unsigned s_tile;
  __shared__ unsigned long long s_slot;
  __shared__ unsigned s_base[ITEMS * (BLOCK / 32) + 1];
  __shared__ unsigned long long s_cnt[BLOCK];
  if (ld_volatile_int(&ctrl->err)) return;
  const unsigned long long N = ld_volatile(&ctrl->n);
  constexpr unsigned long long TILE = (unsigned long long)BLOCK * ITEMS;
  const unsigned long long ntiles = (N + TILE - 1) / TILE;
  if (blockIdx.x == 0 && threadIdx.x == 0 && N == 0) {
    ctrl->n_pairs = 0;   // groups
    ctrl->n_side = 0;    // members
  }
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = BLOCK / 32;
  for (;;) {
    const unsigned tile = next_tile(&ctrl->tickets[0], &s_tile);
    if (tile >= ntiles) break;
    const unsigned long long base = (unsigned long long)tile * TILE;
    unsigned ballots[ITEMS];
    unsigned cnts[ITEMS];
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const unsigned long long i = base + (unsigned long long)k * BLOCK + threadIdx.x;
      bool rep = false;
      cnts[k] = 0;
      if (i < N) {
        const uint32_t s = R.gslot[i];
        if (s != kNone) {
          const uint32_t first = R.grp_min[s], cnt = R.grp_cnt[s];  // both loads in flight at once
          if (first == (uint32_t)i) {
            rep = true;
            cnts[k] = cnt;
          }
        }
      }
      ballots[k] = __ballot_sync(kFull, rep);
    }
    const unsigned agg = tile_ranks<BLOCK, ITEMS>(ballots, s_base);
    // member-count prefix in index order: per item k, warp-level scan, then across (k, warp)
    // The per-(k,warp) sums are small; a second rank table over counts is built in s_cnt.
    unsigned long long item_pre[ITEMS];
    unsigned long long warp_tot[ITEMS];
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      unsigned long long v = cnts[k];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long t = __shfl_up_sync(kFull, v, o);
        if (lane >= (unsigned)o) v += t;
      }
      item_pre[k] = v - cnts[k];
      warp_tot[k] = __shfl_sync(kFull, v, 31);
    }
    // s_cnt[k*NW + warp] = warp totals; exclusive scan by thread 0 (ITEMS*NW <= 64 entries)
    __syncthreads();
    if (lane == 0) {
#pragma unroll
      for (int k = 0; k < ITEMS; ++k) s_cnt[k * NW + warp] = warp_tot[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long run = 0;
      for (int e = 0; e < ITEMS * NW; ++e) {
        const unsigned long long t = s_cnt[e];
        s_cnt[e] = run;
        run += t;
      }
      s_cnt[ITEMS * NW] = run;
    }
    __syncthreads();
    const unsigned long long agg_cnt = s_cnt[ITEMS * NW];
    unsigned long long excl, excl_cnt;
    if (N < (1ull << kOrderPackBits)) {
      const unsigned long long both =
          lookback(ts_a, tile, (unsigned long long)agg | (agg_cnt << kOrderPackBits), ep_a, ctrl, op, &s_slot);
      excl = both & ((1ull << kOrderPackBits) - 1);
      excl_cnt = both >> kOrderPackBits;
    } else {
      excl = lookback(ts_a, tile, agg, ep_a, ctrl, op, &s_slot);
      excl_cnt = lookback(ts_b, tile, agg_cnt, ep_b, ctrl, op, &s_slot);
    }
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      if ((ballots[k] >> lane) & 1u) {
        const unsigned long long i = base + (unsigned long long)k * BLOCK + threadIdx.x;
        const unsigned long long ord = excl + s_base[k * NW + warp] + __popc(ballots[k] & ((1u << lane) - 1u));
        const unsigned long long start = excl_cnt + s_cnt[k * NW + warp] + item_pre[k];
        const uint32_t s = R.gslot[i];
        R.grp_ord[s] = (uint32_t)ord;
        R.g_start[ord] = (uint32_t)start;
        R.g_cnt[ord] = cnts[k];
        R.g_rep[ord] = (uint32_t)i;
        R.g_fill[ord] = 0;
      }
    }
    if (tile == ntiles - 1 && threadIdx.x == 0) {
      ctrl->n_pairs = excl + agg;        // groups
      ctrl->n_side = excl_cnt + agg_cnt; // members (touched terms)
    }
  }
}

// Lays out each group's members contiguously, as (coordinate index, coefficient) records,
// and the group's key (from its representative), so k_run_groups reads one span per group
// instead of gathering members by index.  A member's coordinate index has bit t set when f
// has a 1 at the t-th lowest qubit of M = v & Q (the order k_run_groups uses).  Also hands
// the group table back clean: grp_min and grp_cnt were last read by k_run_order, so every
// member resets its slot (same values from every member), and the next run needs no
// clearing pass.  After a device error the host clears both arrays instead.
template <int W>
__global__ void __launch_bounds__(256) k_run_scatter(Planes P, Ctrl* ctrl, const RunDesc* rd, RunScratch R) {
  pdl_wait();
  if (ld_volatile_int(&ctrl->err)) return;
  const unsigned long long N = ld_volatile(&ctrl->n);
  const uint32_t cls = rd->cls;
  uint64_t Q[W];
#pragma unroll
  for (int w = 0; w < W; ++w) Q[w] = rd->Q[w];
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t s = R.gslot[i];
    if (s == kNone) continue;
    uint64_t x[W], z[W], v[W], f[W];
    load_key<W>(P, i, x, z);  // the term's own data: in flight with the group lookups below
    const double coef = P.c[i];
    const uint32_t o = R.grp_ord[s];
    const uint32_t pos = R.g_start[o] + atomicAdd(&R.g_fill[o], 1u);
    split_planes<W>(cls, x, z, v, f);
    unsigned c = 0, t = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) {
      uint64_t m = v[w] & Q[w];
      while (m) {
        const int b = __ffsll((long long)m) - 1;
        c |= (unsigned)((f[w] >> b) & 1ull) << t;
        ++t;
        m &= m - 1;
      }
    }
    R.mcoord[pos] = c;
    R.mcoef[pos] = coef;
    if (R.g_rep[o] == (uint32_t)i) {
      uint64_t* gk = R.gkey + (unsigned long long)o * 2 * W;
#pragma unroll
      for (int w = 0; w < W; ++w) {
        gk[w] = v[w];
        gk[W + w] = f[w] & ~(v[w] & Q[w]);
      }
    }
    R.grp_min[s] = kNone;
    R.grp_cnt[s] = 0u;
  }
}

// Publishes the count after the run and fills the op log of its gates (and its TRUNCATE):
// one warp of the last block of k_run_groups.  Gate j's live count is n0 plus the children
// the gates before it created (an exclusive scan of the created counts, 8 gates per lane).
__device__ __forceinline__ void run_commit(Ctrl* ctrl, RunScratch R, int op0, int L, int trunc_op, OpLog* log,
                                           bool scratch, unsigned long long cap) {
  const unsigned lane = threadIdx.x & 31;
  if (ld_volatile_int(&ctrl->err)) {
    if (lane < 4) ctrl->tickets[lane] = 0;
    return;
  }
  constexpr int PER = kRunMaxGates / 32;
  unsigned long long made[PER], tot = 0;
#pragma unroll
  for (int e = 0; e < PER; ++e) {
    const int j = (int)lane * PER + e;
    made[e] = j < L ? ld_volatile(&R.created[j]) : 0ull;
    tot += made[e];
  }
  unsigned long long incl = tot;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long t = __shfl_up_sync(kFull, incl, o);
    if (lane >= (unsigned)o) incl += t;
  }
  const unsigned long long total = __shfl_sync(kFull, incl, 31);
  const unsigned long long n0 = ld_volatile(&ctrl->n);
  unsigned long long run = n0 + incl - tot;
#pragma unroll
  for (int e = 0; e < PER; ++e) {
    const int j = (int)lane * PER + e;
    if (j < L) {
      log[op0 + j].n_in = run;
      run += made[e];
      log[op0 + j].n_new = made[e];
      log[op0 + j].n_out = run;
      log[op0 + j].n_s = 0;
      R.created[j] = 0;  // clean for the next run
    }
  }
  __syncwarp();
  if (lane == 0) {
    const unsigned long long ngroups = ld_volatile(&ctrl->n_pairs);
    const unsigned long long nun = ld_volatile(&ctrl->n_s);
    for (int t = 0; t < 4; ++t) ctrl->tickets[t] = 0;
    // scratch mode: the counter holds every group output; they reach O in k_run_place
    const unsigned long long cap_needed = scratch ? nun + ld_volatile(&ctrl->scr_top) : ld_volatile(&ctrl->cap_needed);
    if (scratch) {
      ctrl->scr_top = 0;
      if (cap_needed > cap) {
        ctrl->cap_needed = cap_needed;
        set_err(ctrl, kErrCapacity, op0);
        return;
      }
    }
    // touched terms (profiling bytes); bit 63 says the run took scratch mode
    log[op0].n_s = ld_volatile(&ctrl->n_side) | (scratch ? kRunLogScratchBit : 0ull);
    if (L > 1) log[op0 + L - 1].n_s = (ngroups == 0) ? 0 : cap_needed - nun;  // group outputs
    const unsigned long long out = (ngroups == 0) ? nun : cap_needed;
    if (trunc_op >= 0) {
      log[trunc_op].n_in = n0 + total;
      log[trunc_op].n_out = out;
    }
    ctrl->n = out;
  }
}

// A group of a fused run as one warp holds it: key, coordinate qubits (ascending), whether
// its weight passes the cap.  Its coefficients and existence bits live in the warp's
// shared-memory slots, its coordinate bits in gate order in the warp's order array.
template <int W>
struct RunGroup {
  uint64_t v[W], f0[W];
  uint16_t pos[kRunMaxK];
  unsigned k;
  bool wok;
};

// Loads group g into the warp's slots: key, coordinates, their gate order, members.
template <int W>
__device__ __forceinline__ void group_load(RunGroup<W>& G, unsigned long long g, const RunDesc* rd,
                                           const RunScratch& R, const uint16_t* s_gidx, uint8_t* ord, double* coef,
                                           unsigned* ex, bool wcap, unsigned long long maxw) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t start = R.g_start[g], cnt = R.g_cnt[g];  // loaded beside the group key
  uint64_t M[W];
  G.k = 0;
  {
    const uint64_t* gk = R.gkey + g * 2 * W;
#pragma unroll
    for (int w = 0; w < W; ++w) {
      G.v[w] = gk[w];
      G.f0[w] = gk[W + w];
      M[w] = G.v[w] & rd->Q[w];
    }
#pragma unroll
    for (int w = 0; w < W; ++w) {
      uint64_t m = M[w];
      while (m) {
        const int b = __ffsll((long long)m) - 1;
        G.pos[G.k++] = (uint16_t)(w * 64 + b);
        m &= m - 1;
      }
    }
  }
  {  // coordinate bits sorted by the position of their gate in the run (distinct): lane t
     // takes bit t, its rank is the number of bits whose gate comes earlier
    unsigned key = 0xFFFFu;
    for (unsigned t = 0; t < G.k; ++t)
      if (t == lane) key = s_gidx[G.pos[t]];
    unsigned rank = 0;
    for (unsigned t = 0; t < G.k; ++t) rank += __shfl_sync(kFull, key, t) < key;
    if (lane < G.k) ord[rank] = (uint8_t)lane;
  }
  G.wok = true;
  if (wcap) {
    unsigned wt = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) wt += __popcll(G.v[w] | G.f0[w]);
    G.wok = wt <= maxw;  // M is inside v, so every member has this weight
  }
  const unsigned size = 1u << G.k;
  for (unsigned e = lane; e < (size + 31) / 32; e += 32) ex[e] = 0u;
  __syncwarp();
  for (uint32_t m = lane; m < cnt; m += 32) {
    const unsigned c = R.mcoord[start + m];
    coef[c] = R.mcoef[start + m];
    atomicOr(&ex[c >> 5], 1u << (c & 31));
  }
  __syncwarp();
}

// The gates of the run in order over the group's slots; children created per gate go to
// s_created when it is given.  eps of a member with bit t = b:
//   RX: eps = b ? -1 : +1   (crates/ppvm-pauli-sum/src/sum/rot1.rs:73)
//   RZ: eps = b ? +1 : -1   (rot1.rs:124)
template <int W>
__device__ __forceinline__ void group_butterfly(const RunGroup<W>& G, uint32_t cls, const uint8_t* ord,
                                                const uint16_t* s_gidx, const double* s_cs, const double* s_sn,
                                                double* coef, unsigned* ex, unsigned long long* s_created) {
  const unsigned lane = threadIdx.x & 31;
  const unsigned size = 1u << G.k;
  const double eps_a = cls == 0 ? 1.0 : -1.0, eps_b = -eps_a;
  for (unsigned r = 0; r < G.k; ++r) {
    const unsigned t = ord[r];
    const unsigned j = s_gidx[G.pos[t]];
    const unsigned bit = 1u << t;
    const double cs = s_cs[j], sn = s_sn[j];
    unsigned made = 0;
    for (unsigned p = lane; p < size / 2; p += 32) {
      const unsigned a = ((p >> t) << (t + 1)) | (p & (bit - 1));
      const unsigned b = a | bit;
      const bool ea = (ex[a >> 5] >> (a & 31)) & 1u, eb = (ex[b >> 5] >> (b & 31)) & 1u;
      if (ea && eb) {
        const double ca = coef[a], cb = coef[b];
        coef[a] = __dadd_rn(__dmul_rn(ca, cs), __dmul_rn(cb, eps_b * sn));
        coef[b] = __dadd_rn(__dmul_rn(cb, cs), __dmul_rn(ca, eps_a * sn));
      } else if (ea) {
        const double ca = coef[a];
        coef[a] = __dmul_rn(ca, cs);
        coef[b] = __dmul_rn(ca, eps_a * sn);
        atomicOr(&ex[b >> 5], 1u << (b & 31));
        ++made;
      } else if (eb) {
        const double cb = coef[b];
        coef[b] = __dmul_rn(cb, cs);
        coef[a] = __dmul_rn(cb, eps_b * sn);
        atomicOr(&ex[a >> 5], 1u << (a & 31));
        ++made;
      }
    }
    __syncwarp();
    if (s_created) {
#pragma unroll
      for (int o = 16; o; o >>= 1) made += __shfl_down_sync(kFull, made, o);
      if (lane == 0 && made) atomicAdd(&s_created[j], (unsigned long long)made);
    }
  }
}

// Survivors of the group (existing slots that pass the run's TRUNCATE), on every lane.
template <int W>
__device__ __forceinline__ unsigned group_count(const RunGroup<W>& G, const double* coef, const unsigned* ex,
                                                int trunc, double thr) {
  const unsigned lane = threadIdx.x & 31;
  const unsigned size = 1u << G.k;
  unsigned mine = 0;
  for (unsigned c = lane; c < size; c += 32) {
    const bool e = (ex[c >> 5] >> (c & 31)) & 1u;
    bool keep = e;
    if (trunc && e) keep = G.wok && !(fabs(coef[c]) < thr);
    mine += keep;
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) mine += __shfl_down_sync(kFull, mine, o);
  return __shfl_sync(kFull, mine, 0);
}

// Writes the group's survivors, in coordinate order, to D from index out on.
template <int W>
__device__ __forceinline__ void group_write(const RunGroup<W>& G, Planes D, unsigned long long out, uint32_t cls,
                                            const double* coef, const unsigned* ex, int trunc, double thr) {
  const unsigned lane = threadIdx.x & 31;
  const unsigned size = 1u << G.k;
  for (unsigned c0 = 0; c0 < size; c0 += 32) {
    const unsigned c = c0 + lane;
    bool keep = false;
    if (c < size) {
      keep = (ex[c >> 5] >> (c & 31)) & 1u;
      if (trunc && keep) keep = G.wok && !(fabs(coef[c]) < thr);
    }
    const unsigned bal = __ballot_sync(kFull, keep);
    if (keep) {
      const unsigned long long r = out + __popc(bal & ((1u << lane) - 1u));
      if (r < D.cap) {
        uint64_t f[W], x[W], z[W];
#pragma unroll
        for (int w = 0; w < W; ++w) f[w] = G.f0[w];
        for (unsigned t = 0; t < G.k; ++t)
          if ((c >> t) & 1u) {
            const unsigned q = G.pos[t];
#pragma unroll
            for (int w = 0; w < W; ++w)
              if (w == (int)(q >> 6)) f[w] |= 1ull << (q & 63);
          }
#pragma unroll
        for (int w = 0; w < W; ++w) {
          x[w] = cls == 0 ? f[w] : G.v[w];
          z[w] = cls == 0 ? G.v[w] : f[w];
        }
        store_key<W>(D, r, x, z);
        D.c[r] = coef[c];
      }
    }
    out += __popc(bal);
  }
}

// ---- lane mode: one group per lane ------------------------------------------------------
constexpr int kRunLaneK = 3;  // groups of up to 3 coordinates (8 slots) run on one lane

// A small group on one lane: its slots in registers (slot c at coef[c], existence bit c of
// ex), its key and coordinate qubits, the gates of its coordinates in run order.
template <int W>
struct LaneGroup {
  uint64_t v[W], f0[W];
  uint16_t pos[kRunLaneK];  // qubit of coordinate bit t (ascending)
  uint8_t ord[kRunLaneK];   // coordinate bits in gate order
  unsigned k;
  bool wok;
  double coef[1 << kRunLaneK];
  unsigned ex;
};

// Loads group g's key on this lane: v, f0, its coordinates; false when it has more than
// kRunLaneK coordinates (the warp runs it instead).
template <int W>
__device__ __forceinline__ bool lane_key(LaneGroup<W>& G, unsigned long long g, const RunDesc* rd,
                                         const RunScratch& R, const uint16_t* s_gidx, bool wcap,
                                         unsigned long long maxw) {
  const uint64_t* gk = R.gkey + g * 2 * W;
  unsigned k = 0;
#pragma unroll
  for (int w = 0; w < W; ++w) {
    G.v[w] = gk[w];
    G.f0[w] = gk[W + w];
    k += __popcll(G.v[w] & rd->Q[w]);
  }
  G.k = k;
  if (k > (unsigned)kRunLaneK) return false;
  unsigned t = 0;
#pragma unroll
  for (int w = 0; w < W; ++w) {
    uint64_t m = G.v[w] & rd->Q[w];
    while (m) {
      const int b = __ffsll((long long)m) - 1;
      m &= m - 1;
      if (t < (unsigned)kRunLaneK) G.pos[t] = (uint16_t)(w * 64 + b);
      ++t;
    }
  }
  // coordinate bits by gate position (insertion sort of at most 3)
  for (unsigned a = 0; a < k; ++a) G.ord[a] = (uint8_t)a;
  for (unsigned a = 1; a < k; ++a)
    for (unsigned b = a; b > 0 && s_gidx[G.pos[G.ord[b - 1]]] > s_gidx[G.pos[G.ord[b]]]; --b) {
      const uint8_t tmp = G.ord[b - 1];
      G.ord[b - 1] = G.ord[b];
      G.ord[b] = tmp;
    }
  G.wok = true;
  if (wcap) {
    unsigned wt = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) wt += __popcll(G.v[w] | G.f0[w]);
    G.wok = wt <= maxw;
  }
  return true;
}

// The members and the butterfly of a small group on its lane, the same arithmetic in the same
// gate order as group_butterfly; children made per gate go to s_created.
template <int W>
__device__ __forceinline__ void lane_run(LaneGroup<W>& G, unsigned long long g, uint32_t cls, const RunScratch& R,
                                         const uint16_t* s_gidx, const double* s_cs, const double* s_sn,
                                         unsigned long long* s_created) {
  constexpr int SZ = 1 << kRunLaneK;
  const uint32_t start = R.g_start[g], cnt = R.g_cnt[g];
  G.ex = 0;
#pragma unroll
  for (int c = 0; c < SZ; ++c) G.coef[c] = 0.0;
  for (uint32_t m = 0; m < cnt; ++m) {
    const unsigned c = R.mcoord[start + m];
    const double v = R.mcoef[start + m];
#pragma unroll
    for (int e = 0; e < SZ; ++e)
      if (e == (int)c) G.coef[e] = v;
    G.ex |= 1u << c;
  }
  const double eps_a = cls == 0 ? 1.0 : -1.0, eps_b = -eps_a;
  for (unsigned r = 0; r < G.k; ++r) {
    const unsigned t = G.ord[r];
    const unsigned j = s_gidx[G.pos[t]];
    const unsigned bit = 1u << t;
    const double cs = s_cs[j], sn = s_sn[j];
    unsigned made = 0;
#pragma unroll
    for (int a = 0; a < SZ; ++a) {
      if ((a & (int)bit) || a >= (1 << G.k)) continue;
      const int b = a | (int)bit;
      double ca = 0.0, cb = 0.0;
#pragma unroll
      for (int e = 0; e < SZ; ++e) {  // registers only: slots picked by compile-time index
        if (e == a) ca = G.coef[e];
        if (e == b) cb = G.coef[e];
      }
      const bool ea = (G.ex >> a) & 1u, eb = (G.ex >> b) & 1u;
      double na = ca, nb = cb;
      if (ea && eb) {
        na = __dadd_rn(__dmul_rn(ca, cs), __dmul_rn(cb, eps_b * sn));
        nb = __dadd_rn(__dmul_rn(cb, cs), __dmul_rn(ca, eps_a * sn));
      } else if (ea) {
        na = __dmul_rn(ca, cs);
        nb = __dmul_rn(ca, eps_a * sn);
        G.ex |= 1u << b;
        ++made;
      } else if (eb) {
        nb = __dmul_rn(cb, cs);
        na = __dmul_rn(cb, eps_b * sn);
        G.ex |= 1u << a;
        ++made;
      }
#pragma unroll
      for (int e = 0; e < SZ; ++e) {
        if (e == a) G.coef[e] = na;
        if (e == b) G.coef[e] = nb;
      }
    }
    if (made) atomicAdd(&s_created[j], (unsigned long long)made);
  }
}

// Whether slot c of a small group is written (it exists and passes the run's TRUNCATE).
template <int W>
__device__ __forceinline__ bool lane_keep(const LaneGroup<W>& G, int c, int trunc, double thr) {
  if (!((G.ex >> c) & 1u)) return false;
  if (!trunc) return true;
  double v = 0.0;
#pragma unroll
  for (int e = 0; e < (1 << kRunLaneK); ++e)
    if (e == c) v = G.coef[e];
  return G.wok && !(fabs(v) < thr);
}

// Writes a small group's survivors, in coordinate order, to D from index out on.
template <int W>
__device__ __forceinline__ void lane_write(const LaneGroup<W>& G, Planes D, unsigned long long out, uint32_t cls,
                                           int trunc, double thr) {
#pragma unroll
  for (int c = 0; c < (1 << kRunLaneK); ++c) {
    if (c >= (1 << G.k) || !lane_keep<W>(G, c, trunc, thr)) continue;
    if (out < D.cap) {
      uint64_t f[W], x[W], z[W];
#pragma unroll
      for (int w = 0; w < W; ++w) f[w] = G.f0[w];
      for (unsigned t = 0; t < G.k; ++t)
        if ((c >> t) & 1) {
          const unsigned q = G.pos[t];
#pragma unroll
          for (int w = 0; w < W; ++w)
            if (w == (int)(q >> 6)) f[w] |= 1ull << (q & 63);
        }
#pragma unroll
      for (int w = 0; w < W; ++w) {
        x[w] = cls == 0 ? f[w] : G.v[w];
        z[w] = cls == 0 ? G.v[w] : f[w];
      }
      store_key<W>(D, out, x, z);
      D.c[out] = G.coef[c];
    }
    ++out;
  }
}

// Whether a run's groups go one per lane: forced (tile_mode 3), or chosen for many groups of
// mostly one member.  Lane mode places its 32-group tiles by look-back, never in scratch
// mode, so k_run_place makes the same decision to stand aside.
__device__ __forceinline__ bool run_lanes(unsigned long long ngroups, unsigned long long members, unsigned tile_mode) {
  return tile_mode == 3 || (tile_mode == 0 && ngroups >= kRunTileMinGroups && 2 * members < 3 * ngroups);
}

// The groups of a run, in one of four modes chosen per launch (the same in every block):
// - one group per lane (at least kRunTileMinGroups groups of fewer than 1.5 members on
//   average; placed by look-back at any group count): see the lane-mode branch;
// - one group per warp, taken by ticket (groups of several members): the warp runs the
//   butterfly, counts the survivors, finds the group's output offset by a warp look-back over
//   the lower-numbered groups, and writes;
// - tiles of kRunTileGroups groups per block (tile_mode 1 only; lane mode replaced it in the
//   automatic choice): warp w takes the tile's groups w,
//   w + kRunWarps, ...; the warps run every butterfly and count, a block scan orders the
//   counts, one decoupled look-back places the tile after all lower tiles, and the warps then
//   write, each warp's last group straight from its slots and the others after running their
//   butterflies again (the same arithmetic in the same order, so the same coefficients).  One
//   look-back per tile instead of per group; the second butterfly costs less than the
//   look-backs it saves only when the butterflies are short;
// - scratch mode (many groups, when not in lane mode): one group per warp, its survivors
//   written at once to the scratch planes S wherever a counter puts them; k_run_place then
//   moves every group's block to its place in O.
// Every mode writes the same terms in the same order: groups by number, members by
// coordinate.
template <int W>
__global__ void __launch_bounds__(kRunWarps * 32)
k_run_groups(Planes O, Planes S, Ctrl* ctrl, const RunDesc* rd, RunScratch R, int trunc, double thr,
             unsigned long long maxw, unsigned long long* ts, unsigned epoch, int op, int trunc_op, OpLog* log,
             unsigned long long scratch_min, unsigned tile_mode) {
  pdl_wait();
  constexpr int SZ = 1 << kRunMaxK;
  constexpr int GT = kRunTileGroups;
  __shared__ double s_coef[kRunWarps][SZ];
  __shared__ unsigned s_ex[kRunWarps][SZ / 32];
  __shared__ unsigned long long s_created[kRunMaxGates];
  __shared__ double s_cs[kRunMaxGates], s_sn[kRunMaxGates];
  __shared__ uint16_t s_gidx[64 * W];               // qubit -> its gate's index in the run
  __shared__ uint8_t s_ord[kRunWarps][kRunMaxK];    // a group's coordinate bits in gate order
  __shared__ unsigned s_cnt[GT], s_off[GT + 1];
  __shared__ unsigned s_tile;
  __shared__ unsigned long long s_slot;
  __shared__ int s_err;
  if (threadIdx.x == 0) s_err = ld_volatile_int(&ctrl->err);
  const uint32_t L = rd->L;
  for (unsigned j = threadIdx.x; j < L; j += blockDim.x) {
    s_created[j] = 0;
    s_cs[j] = rd->cs[j];
    s_sn[j] = rd->sn[j];
    s_gidx[rd->q[j]] = (uint16_t)j;  // the qubits of a run are distinct
  }
  __syncthreads();
  if (s_err) return;
  const unsigned long long ngroups = ld_volatile(&ctrl->n_pairs);
  const unsigned long long ubase = ld_volatile(&ctrl->n_s);  // untouched survivors go first
  const unsigned long long members = ld_volatile(&ctrl->n_side);
  const bool lanes = run_lanes(ngroups, members, tile_mode);  // the same in every block
  const bool scratch = !lanes && ngroups >= scratch_min;
  const uint32_t cls = rd->cls;
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool wcap = maxw != ~0ull;
  double* coef = s_coef[warp];
  unsigned* ex = s_ex[warp];
  uint8_t* ord = s_ord[warp];
  const bool tiled = !lanes && !scratch && tile_mode == 1;
  if (lanes) {
    // lane mode: a warp takes 32 consecutive groups by one ticket.  A group of at most
    // kRunLaneK coordinates runs on its lane alone; a larger one is run by the whole warp.
    // One warp scan and one look-back place the 32 groups, and
    // the warp runs its large groups again to write them.
    const unsigned long long ntiles = (ngroups + 31) / 32;
    for (;;) {
      unsigned long long t = 0;
      if (lane == 0) t = atomicAdd(&ctrl->tickets[2], 1ull);
      t = __shfl_sync(kFull, t, 0);
      if (t >= ntiles) break;
      const unsigned long long g = t * 32 + lane;
      const bool valid = g < ngroups;
      LaneGroup<W> LG;
      bool small = false;
      unsigned mine = 0;
      if (valid) {
        small = lane_key<W>(LG, g, rd, R, s_gidx, wcap, maxw);
        if (small) {
          lane_run<W>(LG, g, cls, R, s_gidx, s_cs, s_sn, s_created);
#pragma unroll
          for (int c = 0; c < (1 << kRunLaneK); ++c)
            if (c < (1 << LG.k)) mine += lane_keep<W>(LG, c, trunc, thr);
        }
      }
      const unsigned big = __ballot_sync(kFull, valid && !small);
      for (unsigned bb = big; bb; bb &= bb - 1) {
        const unsigned l = (unsigned)(__ffs(bb) - 1);
        RunGroup<W> G;
        group_load<W>(G, t * 32 + l, rd, R, s_gidx, ord, coef, ex, wcap, maxw);
        group_butterfly<W>(G, cls, ord, s_gidx, s_cs, s_sn, coef, ex, s_created);
        const unsigned m = group_count<W>(G, coef, ex, trunc, thr);
        if (lane == l) mine = m;
        __syncwarp();
      }
      unsigned incl = mine;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned v = __shfl_up_sync(kFull, incl, o);
        if (lane >= (unsigned)o) incl += v;
      }
      const unsigned total = __shfl_sync(kFull, incl, 31);
      const unsigned pre = incl - mine;
      const unsigned long long base = ubase + warp_lookback(ts, t, total, epoch, ctrl, op);
      const Planes D = O;
      if (valid && small) lane_write<W>(LG, D, base + pre, cls, trunc, thr);
      for (unsigned bb = big; bb; bb &= bb - 1) {
        const unsigned l = (unsigned)(__ffs(bb) - 1);
        const unsigned long long at = base + __shfl_sync(kFull, pre, l);
        __syncwarp();
        RunGroup<W> G;
        group_load<W>(G, t * 32 + l, rd, R, s_gidx, ord, coef, ex, wcap, maxw);
        group_butterfly<W>(G, cls, ord, s_gidx, s_cs, s_sn, coef, ex, nullptr);
        group_write<W>(G, D, at, cls, coef, ex, trunc, thr);
      }
      if (t == ntiles - 1 && lane == 0) {
        ctrl->cap_needed = base + total;
        if (base + total > O.cap) set_err(ctrl, kErrCapacity, op);
      }
      __syncwarp();
    }
  } else
  if (!tiled) {
    for (;;) {
      unsigned long long g = 0;
      if (lane == 0) g = atomicAdd(&ctrl->tickets[2], 1ull);
      g = __shfl_sync(kFull, g, 0);
      if (g >= ngroups) break;
      RunGroup<W> G;
      group_load<W>(G, g, rd, R, s_gidx, ord, coef, ex, wcap, maxw);
      group_butterfly<W>(G, cls, ord, s_gidx, s_cs, s_sn, coef, ex, s_created);
      const unsigned mine = group_count<W>(G, coef, ex, trunc, thr);
      if (scratch) {
        unsigned long long b = 0;
        if (lane == 0) {
          b = atomicAdd(&ctrl->scr_top, (unsigned long long)mine);
          R.g_rep[g] = (uint32_t)(b < 0xFFFFFFFFull ? b : 0xFFFFFFFFull);  // scratch offset (< capacity < 2^32)
          R.g_fill[g] = mine;                                                // survivors
        }
        group_write<W>(G, S, __shfl_sync(kFull, b, 0), cls, coef, ex, trunc, thr);
      } else {
        const unsigned long long excl = warp_lookback(ts, g, mine, epoch, ctrl, op);
        group_write<W>(G, O, ubase + excl, cls, coef, ex, trunc, thr);
        if (g == ngroups - 1 && lane == 0) {
          ctrl->cap_needed = ubase + excl + mine;
          if (ubase + excl + mine > O.cap) set_err(ctrl, kErrCapacity, op);
        }
      }
      __syncwarp();  // the slots and the order array are rewritten by the warp's next group
    }
  } else {
    const unsigned long long ntiles = (ngroups + GT - 1) / GT;
    for (;;) {
      const unsigned tile = next_tile(&ctrl->tickets[2], &s_tile);
      if (tile >= ntiles) break;
      const unsigned long long g0 = (unsigned long long)tile * GT;
      const unsigned ng = (unsigned)min((unsigned long long)GT, ngroups - g0);
      RunGroup<W> G;
      unsigned last = GT;  // this warp's last group of the tile (its slots stay loaded)
      for (unsigned j = warp; j < ng; j += kRunWarps) {
        group_load<W>(G, g0 + j, rd, R, s_gidx, ord, coef, ex, wcap, maxw);
        group_butterfly<W>(G, cls, ord, s_gidx, s_cs, s_sn, coef, ex, s_created);
        const unsigned mine = group_count<W>(G, coef, ex, trunc, thr);
        if (lane == 0) s_cnt[j] = mine;
        last = j;
        __syncwarp();  // the slots and the order array are rewritten by the warp's next group
      }
      __syncthreads();
      if (warp == 0) {  // exclusive scan of the tile's counts (GT <= 32)
        const unsigned c = lane < ng ? s_cnt[lane] : 0u;
        unsigned v = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const unsigned t = __shfl_up_sync(kFull, v, o);
          if (lane >= (unsigned)o) v += t;
        }
        if (lane < GT) s_off[lane] = v - c;
        if (lane == 31) s_off[GT] = v;
      }
      __syncthreads();
      const unsigned long long total = s_off[GT];
      const unsigned long long excl = lookback(ts, tile, total, epoch, ctrl, op, &s_slot);
      const unsigned long long out0 = ubase + excl;
      if (last < GT) {  // a warp without a group in a short last tile writes nothing
        group_write<W>(G, O, out0 + s_off[last], cls, coef, ex, trunc, thr);
        for (unsigned j = warp; j < last; j += kRunWarps) {
          __syncwarp();
          group_load<W>(G, g0 + j, rd, R, s_gidx, ord, coef, ex, wcap, maxw);
          group_butterfly<W>(G, cls, ord, s_gidx, s_cs, s_sn, coef, ex, nullptr);
          group_write<W>(G, O, out0 + s_off[j], cls, coef, ex, trunc, thr);
        }
      }
      __syncwarp();
      if (tile == ntiles - 1 && threadIdx.x == 0) {
        ctrl->cap_needed = out0 + total;
        if (out0 + total > O.cap) set_err(ctrl, kErrCapacity, op);
      }
    }
  }
  __syncthreads();
  for (unsigned j = threadIdx.x; j < L; j += blockDim.x)
    if (s_created[j]) atomicAdd(&R.created[j], s_created[j]);
  if (last_block_done(&ctrl->done) && warp == 0) run_commit(ctrl, R, op, (int)L, trunc_op, log, scratch, O.cap);
}

// Scratch mode of a fused run (many groups): k_run_groups left each group's survivors in a
// contiguous block of the scratch planes S, at R.g_rep[g] (R.g_fill[g] of them).  Groups are
// taken in tiles of BLOCK * ITEMS, in group order: one decoupled look-back per tile gives the
// tile's output offset, a block scan the offsets of its groups, and the block's warps then
// copy whole blocks (one term per lane) to O.  The result is the look-back mode's, term for
// term, at one look-back per tile instead of one per group.
template <int W, int BLOCK, int ITEMS>
__global__ void __launch_bounds__(BLOCK)
k_run_place(Planes S, Planes O, Ctrl* ctrl, RunScratch R, unsigned long long scratch_min, unsigned long long* ts,
            unsigned epoch, int op, unsigned tile_mode) {
  pdl_wait();
  constexpr int NW = BLOCK / 32;
  constexpr int TILE = BLOCK * ITEMS;
  __shared__ unsigned s_tile;
  __shared__ unsigned long long s_slot;
  __shared__ unsigned s_wsum[ITEMS * NW + 1];
  __shared__ uint32_t s_src[TILE], s_cnt[TILE];
  __shared__ unsigned long long s_dst[TILE];
  __shared__ int s_skip;
  if (threadIdx.x == 0) {
    const unsigned long long ng = ld_volatile(&ctrl->n_pairs);
    s_skip = ld_volatile_int(&ctrl->err) || ng == 0 || ng < scratch_min ||
             run_lanes(ng, ld_volatile(&ctrl->n_side), tile_mode);
  }
  __syncthreads();
  if (s_skip) return;  // the same in every block (look-back mode, or an earlier error)
  const unsigned long long ngroups = ld_volatile(&ctrl->n_pairs), ubase = ld_volatile(&ctrl->n_s);
  const unsigned long long ntiles = (ngroups + TILE - 1) / TILE;
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (;;) {
    const unsigned tile = next_tile(&ctrl->tickets[0], &s_tile);
    if (tile >= ntiles) break;
    const unsigned long long base = (unsigned long long)tile * TILE;
    unsigned cnt[ITEMS], pre[ITEMS];
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const unsigned long long gi = base + (unsigned long long)k * BLOCK + threadIdx.x;
      cnt[k] = gi < ngroups ? R.g_fill[gi] : 0u;
      unsigned v = cnt[k];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(kFull, v, o);
        if (lane >= (unsigned)o) v += t;
      }
      pre[k] = v - cnt[k];
      if (lane == 31) s_wsum[k * NW + warp] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {  // group order inside the tile: item k, then warp, then lane
      unsigned run = 0;
      for (int e = 0; e < ITEMS * NW; ++e) {
        const unsigned t = s_wsum[e];
        s_wsum[e] = run;
        run += t;
      }
      s_wsum[ITEMS * NW] = run;
    }
    __syncthreads();
    const unsigned long long excl = lookback(ts, tile, s_wsum[ITEMS * NW], epoch, ctrl, op, &s_slot);
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const unsigned long long gi = base + (unsigned long long)k * BLOCK + threadIdx.x;
      const int q = k * BLOCK + threadIdx.x;
      s_cnt[q] = cnt[k];
      s_src[q] = gi < ngroups ? R.g_rep[gi] : 0u;
      s_dst[q] = ubase + excl + s_wsum[k * NW + warp] + pre[k];
    }
    __syncthreads();
    for (int q = warp; q < TILE; q += NW) {  // one group per warp, one term per lane
      const unsigned n = s_cnt[q];
      const unsigned long long src = s_src[q], dst = s_dst[q];
      for (unsigned e = lane; e < n; e += 32) {
        const unsigned long long a = src + e, b = dst + e;
        if (a < S.cap && b < O.cap) {  // the commit checked that everything fits
#pragma unroll
          for (int w = 0; w < W; ++w) {
            O.x[(unsigned long long)w * O.cap + b] = S.x[(unsigned long long)w * S.cap + a];
            O.z[(unsigned long long)w * O.cap + b] = S.z[(unsigned long long)w * S.cap + a];
          }
          O.c[b] = S.c[a];
        }
      }
    }
    __syncthreads();  // the tile arrays are rewritten by the block's next tile
  }
  if (last_block_done(&ctrl->done) && threadIdx.x == 0) ctrl->tickets[0] = 0;
}

}  // namespace ppvm
