// batch.cu — many independent PauliSums advanced together: one CTA per sum.
//
// A batch holds K sums (instances) of up to 64*W qubits, each with its own gate list,
// truncation strategy and term capacity.  All instances live in one device pool; an
// instance table gives each one its region (offset table).  k_batch runs one Trotter layer
// of every instance per launch (a layer ends at every second TRUNCATE of the instance's
// list): CTA b interprets instance b's ops in order, entirely inside the CTA, so the only
// synchronisation is __syncthreads.  A batch that runs again unchanged replays its layer
// launches as CUDA graphs.
//
// Inputs: each op is an 8-byte record (header word + index into its instance's parameter
// table), so a list of 10^6 gates is 8 MB; the op records, layer ends, parameter tables and
// initial terms of all instances travel in one copy from a pinned staging buffer into one
// device block, and the pool and that block come from the library's buffer cache.  A batch
// built from host circuits therefore costs little more than its kernels.
//
// Per op, with reference semantics (crates/ppvm-pauli-sum/src/sum/data.rs:204-311):
//   rotation   scan (anticommuting terms, in order) -> pair (partner K^G through an
//              epoch-tagged table) -> apply (parent c*cos + partner's c*(eps*sin); the
//              partnerless append their child c*(eps*sin) at the end, in parent order)
//   Clifford / noise   in place, consecutive ops fused per term
//   TRUNCATE   stable in-place compaction (|c| < thr or weight > cap dropped)
// Term order therefore stays the reference's IndexMap order, and every coefficient is the
// same IEEE result, so each instance equals a PauliSum run on its own.  A rotation that
// would overflow its instance's capacity stops before writing anything; the host grows that
// instance's region and resumes from the failing op.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "../../include/ppvm_cuda.h"
#include "tableau.cuh"

namespace ppvm {
void set_last_error(const std::string& msg);
// The per-device buffer cache of the sums (engine.cu): buffers handed back once their
// stream is idle are reused by later batches and sums without cudaMalloc/cudaFree.
cudaError_t cache_malloc(void** out, size_t bytes);
void cache_free(void* p);
}

using namespace ppvm;

namespace {

enum BKind : uint32_t { B_ROT = 0, B_LOCAL = 1, B_TRUNC = 2 };

// One op of an instance's list in 8 bytes: a header word and the index of its first value in
// the instance's parameter table.  Header: kind:2 | code:5 | two:1 | ax:2 | az:2 | q0:10 |
// q1:10 (one-qubit ops repeat q0 in q1).  Parameters: rotation sin, cos of theta (host libm,
// as the reference's f64::sin_cos); Pauli error its three factors; depolarising channels
// their factor; Clifford-angle rotation the sign of sin.  Consecutive ops with the same
// values share one entry, so a Trotter list stores a few values per layer.
struct alignas(8) BOp {
  uint32_t h;
  uint32_t param;
};

constexpr uint32_t bop_header(uint32_t kind, uint32_t code, bool two, uint32_t ax, uint32_t az, uint32_t q0,
                              uint32_t q1) {
  return kind | code << 2 | (uint32_t)two << 7 | ax << 8 | az << 10 | q0 << 12 | q1 << 22;
}
__device__ __forceinline__ uint32_t bop_kind(uint32_t h) { return h & 3u; }

// The op as the per-op kernels' DevOp (loss word 0: batch instances hold plain words).
__device__ __forceinline__ DevOp bop_decode(const BOp o, const double* __restrict__ P) {
  DevOp d;
  const uint32_t h = o.h;
  d.code = (h >> 2) & 31u;
  d.two = (uint16_t)((h >> 7) & 1u);
  d.ax = (uint16_t)((h >> 8) & 3u);
  d.az = (uint16_t)((h >> 10) & 3u);
  const uint32_t q0 = (h >> 12) & 1023u, q1 = h >> 22;
  d.w0 = (uint16_t)(q0 >> 6);
  d.b0 = (uint16_t)(q0 & 63u);
  d.w1 = (uint16_t)(q1 >> 6);
  d.b1 = (uint16_t)(q1 & 63u);
  d.lw = 0;
  d.f0 = d.f1 = d.f2 = 0.0;
  if (bop_kind(h) == B_LOCAL && d.code >= C_PAULI_ERROR) {
    d.f0 = P[o.param];
    if (d.code == C_PAULI_ERROR) {
      d.f1 = P[o.param + 1];
      d.f2 = P[o.param + 2];
    }
  }
  return d;
}

struct BInst {
  unsigned long long off;    // region offset in the pool (u64 words)
  unsigned long long cap;    // term capacity of the region
  unsigned long long n;      // live terms
  unsigned long long tsize;  // pair-table slots (power of two)
  unsigned long long tgu;    // term-gate updates so far
  unsigned long long need;   // terms needed at a failing op
  double thr;
  unsigned long long maxw;
  unsigned long long param_off;  // first value of the instance's parameter table
  unsigned long long init_off;   // its initial terms in the input block (u64 words)
  uint32_t op_begin, op_end, pc, layer_off, n_layers, epoch;
  int err;
  int pad;
};

constexpr unsigned kBNone = 0xFFFFFFFFu;

__host__ __device__ inline unsigned long long region_words(int W, unsigned long long cap, unsigned long long tsize) {
  return (unsigned long long)(2 * W + 3) * cap + tsize;
}

template <int W>
struct Region {
  uint64_t* x;
  uint64_t* z;
  double* c;
  double* rc;      // coefficients of the anticommuting terms, before the op
  uint32_t* sidx;  // index of anticommuting term r
  uint32_t* part;  // its partner record, or kBNone
  unsigned long long* table;
  unsigned long long cap, tsize;
};

// The region layout from its first word b (in the pool, or in shared memory).
template <int W>
__device__ __forceinline__ Region<W> region_at(uint64_t* b, unsigned long long cap, unsigned long long tsize) {
  Region<W> r;
  r.cap = cap;
  r.tsize = tsize;
  r.x = b;
  r.z = b + (size_t)W * cap;
  r.c = reinterpret_cast<double*>(b + (size_t)2 * W * cap);
  r.rc = reinterpret_cast<double*>(b + (size_t)(2 * W + 1) * cap);
  r.sidx = reinterpret_cast<uint32_t*>(b + (size_t)(2 * W + 2) * cap);
  r.part = r.sidx + cap;
  r.table = reinterpret_cast<unsigned long long*>(b + (size_t)(2 * W + 3) * cap);
  return r;
}
template <int W>
__device__ __forceinline__ Region<W> region_of(uint64_t* pool, const BInst& I) {
  return region_at<W>(pool + I.off, I.cap, I.tsize);
}

template <int W>
__device__ __forceinline__ void rload(const Region<W>& R, unsigned long long i, uint64_t (&x)[W], uint64_t (&z)[W]) {
#pragma unroll
  for (int w = 0; w < W; ++w) {
    x[w] = R.x[(size_t)w * R.cap + i];
    z[w] = R.z[(size_t)w * R.cap + i];
  }
}
template <int W>
__device__ __forceinline__ void rstore(const Region<W>& R, unsigned long long i, const uint64_t (&x)[W],
                                       const uint64_t (&z)[W]) {
#pragma unroll
  for (int w = 0; w < W; ++w) {
    R.x[(size_t)w * R.cap + i] = x[w];
    R.z[(size_t)w * R.cap + i] = z[w];
  }
}
// word w of a W-word array without dynamic register indexing
template <int W>
__device__ __forceinline__ uint64_t wsel(const uint64_t (&a)[W], unsigned w) {
  uint64_t v = 0;
#pragma unroll
  for (int k = 0; k < W; ++k) v = (k == (int)w) ? a[k] : v;
  return v;
}
template <int W>
__device__ __forceinline__ void wflip(uint64_t (&a)[W], unsigned w, uint64_t m) {
#pragma unroll
  for (int k = 0; k < W; ++k)
    if (k == (int)w) a[k] ^= m;
}
template <int W>
__device__ __forceinline__ void wset(uint64_t (&a)[W], unsigned w, unsigned b, bool v) {
#pragma unroll
  for (int k = 0; k < W; ++k)
    if (k == (int)w) a[k] = (a[k] & ~(1ull << b)) | ((uint64_t)v << b);
}

// Rotation on at most two qubits with axes (ax, az) (bit 0: q0, bit 1: q1).  For a word with
// bits (x0, z0) at q0 and (x1, z1) at q1: whether it anticommutes, and eps of its child
// (+1 exactly when the anticommuting qubit's single-qubit phase in G*P is -1, as rot_sign).
struct RotBits {
  bool anti;
  bool eps_plus;
};
__device__ __forceinline__ RotBits rot_bits(const DevOp& d, bool x0, bool z0, bool x1, bool z1) {
  const bool ax0 = d.ax & 1, az0 = d.az & 1, ax1 = d.two && (d.ax & 2), az1 = d.two && (d.az & 2);
  RotBits r;
  r.anti = ((x0 & az0) ^ (z0 & ax0)) ^ ((x1 & az1) ^ (z1 & ax1));
  const bool m0 = (ax0 & !az0 & !x0 & z0) | (ax0 & az0 & x0 & !z0) | (!ax0 & az0 & x0 & z0);
  const bool m1 = (ax1 & !az1 & !x1 & z1) | (ax1 & az1 & x1 & !z1) | (!ax1 & az1 & x1 & z1);
  r.eps_plus = m0 | m1;
  return r;
}

template <int W>
__device__ __forceinline__ void op_bits(const DevOp& d, const uint64_t (&x)[W], const uint64_t (&z)[W], bool& x0,
                                        bool& z0, bool& x1, bool& z1) {
  x0 = (wsel<W>(x, d.w0) >> d.b0) & 1ull;
  z0 = (wsel<W>(z, d.w0) >> d.b0) & 1ull;
  x1 = (wsel<W>(x, d.w1) >> d.b1) & 1ull;
  z1 = (wsel<W>(z, d.w1) >> d.b1) & 1ull;
}

template <int W>
__device__ __forceinline__ void flip_gen(const DevOp& d, uint64_t (&x)[W], uint64_t (&z)[W]) {
  if (d.ax & 1) wflip<W>(x, d.w0, 1ull << d.b0);
  if (d.az & 1) wflip<W>(z, d.w0, 1ull << d.b0);
  if (d.two) {
    if (d.ax & 2) wflip<W>(x, d.w1, 1ull << d.b1);
    if (d.az & 2) wflip<W>(z, d.w1, 1ull << d.b1);
  }
}

// Bits of term i at the op's qubits, read from the planes (two words at most).
template <int W>
__device__ __forceinline__ void term_bits(const Region<W>& R, const DevOp& d, unsigned long long i, bool& x0,
                                          bool& z0, bool& x1, bool& z1) {
  x0 = (R.x[(size_t)d.w0 * R.cap + i] >> d.b0) & 1ull;
  z0 = (R.z[(size_t)d.w0 * R.cap + i] >> d.b0) & 1ull;
  x1 = z1 = false;
  if (d.two) {
    x1 = (R.x[(size_t)d.w1 * R.cap + i] >> d.b1) & 1ull;
    z1 = (R.z[(size_t)d.w1 * R.cap + i] >> d.b1) & 1ull;
  }
}

// One local op (Clifford, Clifford-angle rotation or diagonal noise) on a word, the rules of
// the per-op pass (crates/ppvm-pauli-sum/src/sum/clifford.rs:37-221, sum/noise.rs:17-129).
template <int W>
__device__ __forceinline__ void local_op(const DevOp& d, uint64_t (&x)[W], uint64_t (&z)[W], double& c, bool& neg) {
  bool x0, z0, x1, z1;
  op_bits<W>(d, x, z, x0, z0, x1, z1);
  switch (d.code) {
    case C_PAULI_ERROR: {
      const int k = (int)x0 | ((int)z0 << 1);
      if (k == 1) c = __dmul_rn(c, d.f0);
      else if (k == 2) c = __dmul_rn(c, d.f1);
      else if (k == 3) c = __dmul_rn(c, d.f2);
      return;
    }
    case C_DEP1:
      if (x0 | z0) c = __dmul_rn(c, d.f0);
      return;
    case C_DEP2:
      if (x0 | z0 | x1 | z1) c = __dmul_rn(c, d.f0);
      return;
    default: break;
  }
  const bool two = d.code == C_CNOT || d.code == C_CZ || d.code == C_CY || (d.code == C_ROTC && d.two);
  if (!two) x1 = z1 = false;
  cliff_rule<bool>(d, x0, z0, x1, z1, neg);
  wset<W>(x, d.w0, d.b0, x0);
  wset<W>(z, d.w0, d.b0, z0);
  if (two) {
    wset<W>(x, d.w1, d.b1, x1);
    wset<W>(z, d.w1, d.b1, z1);
  }
}

// Sums of two counts over the block in one pass (three barriers instead of six).
template <int BLOCK>
__device__ __forceinline__ void block_sum2_u64(unsigned long long& a, unsigned long long& b,
                                               unsigned long long* s_red) {
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    a += __shfl_down_sync(kFull, a, o);
    b += __shfl_down_sync(kFull, b, o);
  }
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) {
    s_red[warp] = a;
    s_red[BLOCK / 32 + warp] = b;
  }
  __syncthreads();
  unsigned long long ta = 0, tb = 0;
#pragma unroll
  for (int w = 0; w < BLOCK / 32; ++w) {
    ta += s_red[w];
    tb += s_red[BLOCK / 32 + w];
  }
  __syncthreads();
  a = ta;
  b = tb;
}

// One layer (or, with layer < 0, everything left) of every instance; CTA b = instance b.
template <int W, int BLOCK, int ITEMS>
__global__ void __launch_bounds__(BLOCK)
k_batch(BInst* insts, const BOp* __restrict__ ops, const uint32_t* __restrict__ layer_ends,
        const double* __restrict__ params, int layer, uint64_t* pool, unsigned long long resident_bytes) {
  constexpr int NW = BLOCK / 32;
  constexpr unsigned long long TILE = (unsigned long long)BLOCK * ITEMS;
  __shared__ unsigned s_base[ITEMS * NW + 1];
  __shared__ unsigned long long s_red[2 * NW];
  extern __shared__ __align__(16) uint64_t s_region[];  // resident_bytes of dynamic shared memory
  BInst& I = insts[blockIdx.x];
  if (I.err) return;
  const unsigned end = (layer < 0 || (unsigned)layer >= I.n_layers)
                           ? I.op_end
                           : min(I.op_end, layer_ends[I.layer_off + (unsigned)layer]);
  unsigned pc = I.pc;
  if (pc >= end) return;
  // An instance whose whole region fits in the launch's dynamic shared memory runs there: its
  // live terms are copied in, its pair table starts empty (a zero slot holds no epoch), and
  // the terms go back to the pool at the end.  The op loop is the same code either way (R's
  // arrays are generic pointers).  A region that does not fit runs from the pool.
  const bool resident = 8ull * region_words(W, I.cap, I.tsize) <= resident_bytes;
  const Region<W> R = resident ? region_at<W>(s_region, I.cap, I.tsize) : region_of<W>(pool, I);
  if (resident) {
    const Region<W> G = region_of<W>(pool, I);
    const unsigned long long n0 = I.n;
    for (unsigned long long i = threadIdx.x; i < n0; i += BLOCK) {
#pragma unroll
      for (int w = 0; w < W; ++w) {
        R.x[(size_t)w * R.cap + i] = G.x[(size_t)w * G.cap + i];
        R.z[(size_t)w * R.cap + i] = G.z[(size_t)w * G.cap + i];
      }
      R.c[i] = G.c[i];
    }
    for (unsigned long long t = threadIdx.x; t < R.tsize; t += BLOCK) R.table[t] = 0ull;
    __syncthreads();
  }
  const double* __restrict__ P = params + I.param_off;
  const double thr = I.thr;
  const unsigned long long maxw = I.maxw;
  const bool wcap = maxw != ~0ull;
  unsigned long long N = I.n, tgu = 0;
  unsigned epoch = I.epoch;
  int err = 0;
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  while (pc < end) {
    const BOp op = ops[pc];
    const uint32_t kind = bop_kind(op.h);
    if (kind == B_TRUNC) {
      // stable in-place compaction: a tile's reads finish (inside tile_ranks) before its
      // writes, and every write goes to a position at or below the word it came from
      unsigned long long kept = 0;
      for (unsigned long long base = 0; base < N; base += TILE) {
        uint64_t kx[ITEMS][W], kz[ITEMS][W];
        double kc[ITEMS];
        unsigned bal[ITEMS];
#pragma unroll
        for (int k = 0; k < ITEMS; ++k) {
          const unsigned long long i = base + (unsigned long long)k * BLOCK + threadIdx.x;
          bool keep = false;
          if (i < N) {
            rload<W>(R, i, kx[k], kz[k]);
            kc[k] = R.c[i];
            keep = !(fabs(kc[k]) < thr);
            if (wcap) keep = keep && (weight<W>(kx[k], kz[k]) <= maxw);
          }
          bal[k] = __ballot_sync(kFull, keep);
        }
        const unsigned agg = tile_ranks<BLOCK, ITEMS>(bal, s_base);
#pragma unroll
        for (int k = 0; k < ITEMS; ++k)
          if ((bal[k] >> lane) & 1u) {
            const unsigned long long r = kept + s_base[k * NW + warp] + __popc(bal[k] & lt);
            rstore<W>(R, r, kx[k], kz[k]);
            R.c[r] = kc[k];
          }
        kept += agg;
        __syncthreads();
      }
      N = kept;
      ++pc;
      continue;
    }
    if (kind == B_LOCAL) {
      unsigned j = pc;
      while (j < end && bop_kind(ops[j].h) == B_LOCAL) ++j;
      for (unsigned long long i = threadIdx.x; i < N; i += BLOCK) {
        uint64_t x[W], z[W];
        rload<W>(R, i, x, z);
        double c = R.c[i];
        bool neg = false;
        for (unsigned o = pc; o < j; ++o) local_op<W>(bop_decode(ops[o], P), x, z, c, neg);
        rstore<W>(R, i, x, z);
        R.c[i] = neg ? -c : c;
      }
      tgu += N * (unsigned long long)(j - pc);
      pc = j;
      __syncthreads();
      continue;
    }
    // ---- rotation exp(-i theta/2 G), G on op.d's one or two qubits ----
    const DevOp d = bop_decode(op, P);
    const double sn = P[op.param], cs = P[op.param + 1];
    if (++epoch >= 0xFFFFu) {  // pair-table epochs wrapped: clear the table once
      for (unsigned long long t = threadIdx.x; t < R.tsize; t += BLOCK) R.table[t] = 0ull;
      __syncthreads();
      epoch = 1;
    }
    // scan: anticommuting terms, in order
    unsigned long long S = 0;
    for (unsigned long long base = 0; base < N; base += TILE) {
      unsigned bal[ITEMS];
#pragma unroll
      for (int k = 0; k < ITEMS; ++k) {
        const unsigned long long i = base + (unsigned long long)k * BLOCK + threadIdx.x;
        bool a = false;
        if (i < N) {
          bool x0, z0, x1, z1;
          term_bits<W>(R, d, i, x0, z0, x1, z1);
          a = rot_bits(d, x0, z0, x1, z1).anti;
        }
        bal[k] = __ballot_sync(kFull, a);
      }
      const unsigned agg = tile_ranks<BLOCK, ITEMS>(bal, s_base);
#pragma unroll
      for (int k = 0; k < ITEMS; ++k)
        if ((bal[k] >> lane) & 1u) {
          const unsigned long long i = base + (unsigned long long)k * BLOCK + threadIdx.x;
          const unsigned long long r = S + s_base[k * NW + warp] + __popc(bal[k] & lt);
          R.sidx[r] = (uint32_t)i;
          R.part[r] = kBNone;
          R.rc[r] = R.c[i];
        }
      S += agg;
      __syncthreads();
    }
    // pair: the record of K and the record of K^G (if both exist) meet at min(K, K^G)
    unsigned long long mine = 0;
    const unsigned long long mask = R.tsize - 1;
    for (unsigned long long r = threadIdx.x; r < S; r += BLOCK) {
      uint64_t x[W], z[W], px[W], pz[W];
      rload<W>(R, R.sidx[r], x, z);
#pragma unroll
      for (int w = 0; w < W; ++w) {
        px[w] = x[w];
        pz[w] = z[w];
      }
      flip_gen<W>(d, px, pz);
      const bool use_p = key_less<W>(px, pz, x, z);
      uint64_t kx[W], kz[W];
#pragma unroll
      for (int w = 0; w < W; ++w) {
        kx[w] = use_p ? px[w] : x[w];
        kz[w] = use_p ? pz[w] : z[w];
      }
      const uint64_t h = hash_key<W>(kx, kz);
      const unsigned tag = (unsigned)(h >> 48) & 0xFFFFu;
      const unsigned long long me = make_slot(epoch, tag, (unsigned)r);
      unsigned long long slot = h & mask, probes = 0;
      while (true) {
        const unsigned long long cur = ld_volatile(&R.table[slot]);
        if (slot_epoch(cur) != (epoch & 0xFFFFu)) {
          if (atomicCAS(&R.table[slot], cur, me) == cur) break;
          continue;
        }
        if (slot_tag(cur) == tag) {
          const unsigned j = slot_idx(cur);
          uint64_t jx[W], jz[W];
          rload<W>(R, R.sidx[j], jx, jz);
          bool eq = true;
#pragma unroll
          for (int w = 0; w < W; ++w) eq &= (jx[w] == px[w]) & (jz[w] == pz[w]);
          if (eq) {
            R.part[r] = j;
            R.part[j] = (uint32_t)r;
            ++mine;
            break;
          }
        }
        slot = (slot + 1) & mask;
        if (++probes > mask) {
          err = kErrProbe;  // cannot happen with tsize >= 2 * cap; reported, not trapped
          break;
        }
      }
    }
    unsigned long long pairs = mine, perr = (unsigned long long)err;
    block_sum2_u64<BLOCK>(pairs, perr, s_red);
    if (perr) {
      err = kErrProbe;
      break;
    }
    const unsigned long long children = S - 2 * pairs;
    if (N + children > R.cap) {
      if (threadIdx.x == 0) I.need = N + children;
      err = kErrCapacity;
      break;
    }
    // apply: parents in place, partnerless children appended in parent order
    unsigned long long C = 0;
    for (unsigned long long base = 0; base < S; base += TILE) {
      unsigned bal[ITEMS];
#pragma unroll
      for (int k = 0; k < ITEMS; ++k) {
        const unsigned long long r = base + (unsigned long long)k * BLOCK + threadIdx.x;
        bool child = false;
        if (r < S) {
          const uint32_t i = R.sidx[r], j = R.part[r];
          const double c = R.rc[r];
          double nc;
          if (j != kBNone) {
            // the partner's key is K^G: its eps from this term's bits with G's bits flipped
            bool x0, z0, x1, z1;
            term_bits<W>(R, d, i, x0, z0, x1, z1);
            x0 ^= (bool)(d.ax & 1);
            z0 ^= (bool)(d.az & 1);
            if (d.two) {
              x1 ^= (bool)(d.ax & 2);
              z1 ^= (bool)(d.az & 2);
            }
            const double eps_j = rot_bits(d, x0, z0, x1, z1).eps_plus ? 1.0 : -1.0;
            nc = __dadd_rn(__dmul_rn(c, cs), __dmul_rn(R.rc[j], eps_j * sn));
          } else {
            nc = __dmul_rn(c, cs);
            child = true;
          }
          R.c[i] = nc;
        }
        bal[k] = __ballot_sync(kFull, child);
      }
      const unsigned agg = tile_ranks<BLOCK, ITEMS>(bal, s_base);
#pragma unroll
      for (int k = 0; k < ITEMS; ++k)
        if ((bal[k] >> lane) & 1u) {
          const unsigned long long r = base + (unsigned long long)k * BLOCK + threadIdx.x;
          const unsigned long long pos = N + C + s_base[k * NW + warp] + __popc(bal[k] & lt);
          uint64_t x[W], z[W];
          rload<W>(R, R.sidx[r], x, z);
          bool x0, z0, x1, z1;
          op_bits<W>(d, x, z, x0, z0, x1, z1);
          if (!d.two) x1 = z1 = false;
          const double eps = rot_bits(d, x0, z0, x1, z1).eps_plus ? 1.0 : -1.0;
          flip_gen<W>(d, x, z);
          rstore<W>(R, pos, x, z);
          R.c[pos] = __dmul_rn(R.rc[r], eps * sn);
        }
      C += agg;
      __syncthreads();
    }
    tgu += N;
    N += C;
    ++pc;
  }
  __syncthreads();
  if (resident) {  // the terms back to the pool (a failed op wrote nothing)
    const Region<W> G = region_of<W>(pool, I);
    for (unsigned long long i = threadIdx.x; i < N; i += BLOCK) {
#pragma unroll
      for (int w = 0; w < W; ++w) {
        G.x[(size_t)w * G.cap + i] = R.x[(size_t)w * R.cap + i];
        G.z[(size_t)w * G.cap + i] = R.z[(size_t)w * R.cap + i];
      }
      G.c[i] = R.c[i];
    }
  }
  if (threadIdx.x == 0) {
    I.n = N;
    I.pc = pc;
    I.tgu += tgu;
    I.epoch = epoch;
    if (err) I.err = err;
  }
}

// overlap_with_zero of every instance: CTA b sums instance b's coefficients of words
// without X bits, in a fixed order (thread-strided partial sums, then a fixed tree).
template <int W>
__global__ void __launch_bounds__(256) k_batch_owz(const BInst* insts, uint64_t* pool, double* out) {
  __shared__ double s_red[8];
  const BInst& I = insts[blockIdx.x];
  const Region<W> R = region_of<W>(pool, I);
  double acc = 0.0;
  for (unsigned long long i = threadIdx.x; i < I.n; i += blockDim.x) {
    uint64_t any = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) any |= R.x[(size_t)w * R.cap + i];
    if (any == 0) acc = __dadd_rn(acc, R.c[i]);
  }
  const double b = block_sum(acc, s_red);
  if (threadIdx.x == 0) out[blockIdx.x] = b;
}

// Loads initial terms (packed per instance: x[k][W], z[k][W], c[k] at init_off) into regions.
template <int W>
__global__ void k_batch_load(const BInst* insts, const uint64_t* src, uint64_t* pool) {
  const BInst& I = insts[blockIdx.x];
  const Region<W> R = region_of<W>(pool, I);
  const uint64_t* s = src + I.init_off;
  const unsigned long long k = I.n;
  for (unsigned long long i = threadIdx.x; i < k; i += blockDim.x) {
#pragma unroll
    for (int w = 0; w < W; ++w) {
      R.x[(size_t)w * R.cap + i] = s[i * W + w];
      R.z[(size_t)w * R.cap + i] = s[k * W + i * W + w];
    }
    R.c[i] = __longlong_as_double((long long)s[2 * k * W + i]);
  }
}

// Moves every instance's live terms from the old layout to the new one (capacity growth).
template <int W>
__global__ void k_batch_relocate(const BInst* old_i, const BInst* new_i, uint64_t* old_pool, uint64_t* new_pool) {
  const Region<W> A = region_of<W>(old_pool, old_i[blockIdx.x]);
  const Region<W> B = region_of<W>(new_pool, new_i[blockIdx.x]);
  const unsigned long long n = old_i[blockIdx.x].n;
  for (unsigned long long i = threadIdx.x; i < n; i += blockDim.x) {
#pragma unroll
    for (int w = 0; w < W; ++w) {
      B.x[(size_t)w * B.cap + i] = A.x[(size_t)w * A.cap + i];
      B.z[(size_t)w * B.cap + i] = A.z[(size_t)w * A.cap + i];
    }
    B.c[i] = A.c[i];
  }
}

ppvm_status bfail(ppvm_status s, const std::string& msg) {
  ppvm::set_last_error(msg);
  return s;
}

// Page-locked staging for the batches' input uploads: one buffer per process, grown on
// demand and kept, so that an upload is a memcpy into pinned memory and one DMA copy (no
// pageable copy through the driver's bounce buffer, no fresh pages to fault in).  An upload
// holds the lock until its copy has completed.
struct Staging {
  std::mutex mu;
  void* p = nullptr;
  size_t cap = 0;
};
Staging& staging() {
  static Staging s;
  return s;
}

#define BCUDA(expr)                                                                          \
  do {                                                                                       \
    cudaError_t e_ = (expr);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return bfail(e_ == cudaErrorMemoryAllocation ? PPVM_ECAPACITY : PPVM_ECUDA,            \
                   std::string(#expr) + ": " + cudaGetErrorString(e_));                      \
  } while (0)

#define BTRY(expr)                \
  do {                            \
    ppvm_status s_ = (expr);      \
    if (s_ != PPVM_OK) return s_; \
  } while (0)

unsigned long long pow2_at_least(unsigned long long v) {
  unsigned long long p = 1;
  while (p < v) p <<= 1;
  return p;
}

}  // namespace

struct ppvm_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  int W = 1;
  uint32_t flags = 0;
  size_t ninst = 0;
  std::vector<uint32_t> nq;
  std::vector<double> thr;
  std::vector<uint64_t> maxw;
  // initial terms per instance (instance words: ceil(n/64) per plane)
  std::vector<std::vector<uint64_t>> ix, iz;
  std::vector<std::vector<double>> ic;
  std::vector<std::vector<BOp>> ops;
  std::vector<std::vector<double>> params;   // parameter table of each instance's ops
  std::vector<std::vector<uint32_t>> lends;  // op index just past each layer's closing TRUNCATE
  std::vector<unsigned long long> cap;       // region capacities (kept across runs)
  // launch configuration (autotuned)
  int block = 256, items = 4, tfac = 2;
  // device state.  The inputs (op records, layer ends, parameters, initial terms) sit in one
  // device block, uploaded by one copy whenever a setter changed them.
  BInst* d_inst = nullptr;
  BInst* h_inst = nullptr;  // pinned mirror
  void* d_input = nullptr;
  size_t input_bytes = 0;   // capacity of d_input
  BOp* d_ops = nullptr;
  uint32_t* d_lends = nullptr;
  double* d_params = nullptr;
  uint64_t* d_init = nullptr;
  uint64_t* pool = nullptr;
  size_t pool_words = 0;
  unsigned long long resident_bytes = 0;  // dynamic shared memory per CTA for resident instances
  double* d_out = nullptr;
  bool inputs_dirty = true;
  bool layout_dirty = true;
  std::vector<cudaGraphExec_t> graphs;
  int graph_cfg[3] = {0, 0, 0};
  uint32_t max_layers = 0;
  bool ran = false;
  unsigned long long xfer_h2d = 0, xfer_d2h = 0;  // bytes copied host<->device since creation
};

namespace {

void drop_graphs(ppvm_batch* b) {
  for (auto g : b->graphs)
    if (g) cudaGraphExecDestroy(g);
  b->graphs.clear();
}

int words_of(uint32_t n) { return (int)((n + 63) / 64); }

// Batch plane width: 1, 2, 4 or 8 words.
int batch_words(uint32_t n_max) {
  const int w = words_of(n_max);
  return w <= 1 ? 1 : w <= 2 ? 2 : w <= 4 ? 4 : 8;
}

template <int W, int BLOCK, int ITEMS>
cudaError_t launch_layer(ppvm_batch* b, int layer) {
  const size_t dyn = (size_t)b->resident_bytes;
  if (dyn > 48 * 1024) {
    const cudaError_t e =
        cudaFuncSetAttribute(k_batch<W, BLOCK, ITEMS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    if (e != cudaSuccess) return e;
  }
  k_batch<W, BLOCK, ITEMS><<<(unsigned)b->ninst, BLOCK, dyn, b->stream>>>(b->d_inst, b->d_ops, b->d_lends,
                                                                           b->d_params, layer, b->pool, dyn);
  return cudaGetLastError();
}

template <int W>
cudaError_t launch_layer_w(ppvm_batch* b, int layer) {
  const int k = (b->block == 128 ? 0 : b->block == 256 ? 1 : 2) * 2 + (b->items == 2 ? 0 : 1);
  switch (k) {
    case 0: return launch_layer<W, 128, 2>(b, layer);
    case 1: return launch_layer<W, 128, 4>(b, layer);
    case 2: return launch_layer<W, 256, 2>(b, layer);
    case 3: return launch_layer<W, 256, 4>(b, layer);
    case 4: return launch_layer<W, 512, 2>(b, layer);
    default: return launch_layer<W, 512, 4>(b, layer);
  }
}

cudaError_t launch_any(ppvm_batch* b, int layer) {
  switch (b->W) {
    case 1: return launch_layer_w<1>(b, layer);
    case 2: return launch_layer_w<2>(b, layer);
    case 4: return launch_layer_w<4>(b, layer);
    default: return launch_layer_w<8>(b, layer);
  }
}

template <int W>
void launch_relocate(ppvm_batch* b, const BInst* d_old, uint64_t* old_pool, uint64_t* new_pool) {
  k_batch_relocate<W><<<(unsigned)b->ninst, 256, 0, b->stream>>>(d_old, b->d_inst, old_pool, new_pool);
}
template <int W>
void launch_load(ppvm_batch* b) {
  k_batch_load<W><<<(unsigned)b->ninst, 256, 0, b->stream>>>(b->d_inst, b->d_init, b->pool);
}
template <int W>
void launch_owz(ppvm_batch* b) {
  k_batch_owz<W><<<(unsigned)b->ninst, 256, 0, b->stream>>>(b->d_inst, b->pool, b->d_out);
}
#define BDISPATCH(W_, FN, ...)          \
  switch (W_) {                         \
    case 1: FN<1>(__VA_ARGS__); break;  \
    case 2: FN<2>(__VA_ARGS__); break;  \
    case 4: FN<4>(__VA_ARGS__); break;  \
    default: FN<8>(__VA_ARGS__); break; \
  }

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// Uploads what the setters changed: every instance's op records, layer ends (rebased to the
// concatenated op list), parameter table and initial terms (packed x[k][W], z[k][W], c[k]),
// written into the pinned staging buffer and copied to the device input block at once.
ppvm_status upload_inputs(ppvm_batch* b) {
  if (!b->inputs_dirty) return PPVM_OK;
  const int W = b->W;
  size_t nops = 0, nle = 0, npar = 0, ninit = 0;
  for (size_t i = 0; i < b->ninst; ++i) {
    nops += b->ops[i].size();
    nle += b->lends[i].size();
    npar += b->params[i].size();
    ninit += (size_t)(2 * W + 1) * b->ic[i].size();
  }
  if (nops >= 0xFFFFFFF0ull || nle >= 0xFFFFFFF0ull) return bfail(PPVM_ECAPACITY, "batch op list too long");
  const size_t o_ops = 0, o_le = align256(sizeof(BOp) * nops), o_par = o_le + align256(sizeof(uint32_t) * nle),
               o_init = o_par + align256(sizeof(double) * npar),
               total = std::max<size_t>(o_init + align256(sizeof(uint64_t) * ninit), 256);
  BCUDA(cudaStreamSynchronize(b->stream));  // the previous block may still be read
  if (total > b->input_bytes) {
    ppvm::cache_free(b->d_input);
    b->d_input = nullptr;
    b->input_bytes = 0;
    BCUDA(ppvm::cache_malloc(&b->d_input, total));
    b->input_bytes = total;
  }
  Staging& st = staging();
  std::lock_guard<std::mutex> lk(st.mu);
  if (st.cap < total) {
    if (st.p) cudaFreeHost(st.p);
    st.p = nullptr;
    st.cap = 0;
    const size_t want = std::max(total, (size_t)(1u << 20));
    BCUDA(cudaMallocHost(&st.p, want));
    st.cap = want;
  }
  char* h = static_cast<char*>(st.p);
  BOp* h_ops = reinterpret_cast<BOp*>(h + o_ops);
  uint32_t* h_le = reinterpret_cast<uint32_t*>(h + o_le);
  double* h_par = reinterpret_cast<double*>(h + o_par);
  uint64_t* h_init = reinterpret_cast<uint64_t*>(h + o_init);
  size_t at_op = 0, at_le = 0, at_par = 0, at_init = 0;
  b->max_layers = 0;
  for (size_t i = 0; i < b->ninst; ++i) {
    BInst& I = b->h_inst[i];
    const auto& ops = b->ops[i];
    I.op_begin = (uint32_t)at_op;
    I.layer_off = (uint32_t)at_le;
    I.n_layers = (uint32_t)b->lends[i].size();
    I.param_off = at_par;
    I.init_off = at_init;
    if (!ops.empty()) std::memcpy(h_ops + at_op, ops.data(), sizeof(BOp) * ops.size());
    for (uint32_t e : b->lends[i]) h_le[at_le++] = I.op_begin + e;
    at_op += ops.size();
    I.op_end = (uint32_t)at_op;
    if (!b->params[i].empty()) std::memcpy(h_par + at_par, b->params[i].data(), sizeof(double) * b->params[i].size());
    at_par += b->params[i].size();
    const int wi = words_of(b->nq[i]);
    const size_t k = b->ic[i].size();
    uint64_t* s = h_init + at_init;
    std::memset(s, 0, sizeof(uint64_t) * 2 * W * k);
    for (size_t t = 0; t < k; ++t)
      for (int w = 0; w < wi; ++w) {
        s[t * W + w] = b->ix[i][t * wi + w];
        s[k * W + t * W + w] = b->iz[i][t * wi + w];
      }
    if (k) std::memcpy(s + 2 * k * W, b->ic[i].data(), sizeof(double) * k);
    at_init += (size_t)(2 * W + 1) * k;
    b->max_layers = std::max(b->max_layers, I.n_layers);
  }
  char* d = static_cast<char*>(b->d_input);
  b->d_ops = reinterpret_cast<BOp*>(d + o_ops);
  b->d_lends = reinterpret_cast<uint32_t*>(d + o_le);
  b->d_params = reinterpret_cast<double*>(d + o_par);
  b->d_init = reinterpret_cast<uint64_t*>(d + o_init);
  BCUDA(cudaMemcpyAsync(b->d_input, st.p, total, cudaMemcpyHostToDevice, b->stream));
  BCUDA(cudaStreamSynchronize(b->stream));  // the staging buffer is free again
  b->xfer_h2d += total;
  b->inputs_dirty = false;
  drop_graphs(b);
  return PPVM_OK;
}

// Dynamic shared memory per CTA for resident instances: the largest region, when every
// instance's region fits within what each CTA can hold while all of them stay resident
// together (ceil(instances / SMs) CTAs per SM, 2 KB per CTA left to static shared memory and
// the system); otherwise none.  A batch where only some instances fit runs all of them from
// the pool: the shared memory taken by the small ones would shrink the L1 cache that the
// large ones, which set the batch's time, read through.
ppvm_status choose_resident(ppvm_batch* b) {
  static const bool never = [] {  // PPVM_BATCH_RESIDENT=never: every instance from the pool
    const char* e = std::getenv("PPVM_BATCH_RESIDENT");
    return e && std::strcmp(e, "never") == 0;
  }();
  b->resident_bytes = 0;
  if (never) return PPVM_OK;
  int nsm = 0, per_sm_bytes = 0, optin = 0;
  BCUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device));
  BCUDA(cudaDeviceGetAttribute(&per_sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, b->device));
  BCUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device));
  const unsigned long long per_sm = (b->ninst + nsm - 1) / std::max(nsm, 1);
  const unsigned long long share = (unsigned long long)per_sm_bytes / std::max<unsigned long long>(per_sm, 1);
  unsigned long long budget = std::min<unsigned long long>((unsigned long long)optin, share);
  budget = budget > 2048 ? ((budget - 2048) & ~15ull) : 0;
  unsigned long long need = 0;
  for (size_t i = 0; i < b->ninst; ++i)
    need = std::max<unsigned long long>(need, 8ull * region_words(b->W, b->h_inst[i].cap, b->h_inst[i].tsize));
  if (need <= budget) b->resident_bytes = need;
  return PPVM_OK;
}

// Lays the pool out for the current capacities.  With keep, live terms move over.
ppvm_status layout(ppvm_batch* b, bool keep) {
  std::vector<BInst> old(b->h_inst, b->h_inst + b->ninst);
  unsigned long long words = 0;
  for (size_t i = 0; i < b->ninst; ++i) {
    BInst& I = b->h_inst[i];
    I.cap = b->cap[i];
    I.tsize = pow2_at_least(std::max<unsigned long long>((unsigned long long)b->tfac * I.cap, 64));
    I.off = words;
    words += region_words(b->W, I.cap, I.tsize);
    words = (words + 31) & ~31ull;  // 256-byte aligned regions
    I.epoch = 0;
  }
  const size_t bytes = sizeof(uint64_t) * std::max<unsigned long long>(words, 1);
  BTRY(choose_resident(b));
  BCUDA(cudaStreamSynchronize(b->stream));
  void* np = nullptr;
  BCUDA(ppvm::cache_malloc(&np, bytes));
  // zeroed: pair-table slots of an earlier user must not carry a live epoch
  cudaError_t e = cudaMemsetAsync(np, 0, bytes, b->stream);
  void* d_old = nullptr;
  if (e == cudaSuccess && keep && b->pool) {
    e = ppvm::cache_malloc(&d_old, sizeof(BInst) * b->ninst);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_old, old.data(), sizeof(BInst) * b->ninst, cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(b->d_inst, b->h_inst, sizeof(BInst) * b->ninst, cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess) {
      b->xfer_h2d += 2 * sizeof(BInst) * b->ninst;
      BDISPATCH(b->W, launch_relocate, b, static_cast<BInst*>(d_old), b->pool, static_cast<uint64_t*>(np));
      e = cudaGetLastError();
    }
  }
  const cudaError_t se = cudaStreamSynchronize(b->stream);
  if (e == cudaSuccess) e = se;
  ppvm::cache_free(d_old);
  if (e != cudaSuccess) {
    if (se == cudaSuccess) ppvm::cache_free(np);
    return bfail(e == cudaErrorMemoryAllocation ? PPVM_ECAPACITY : PPVM_ECUDA,
                 std::string("batch layout: ") + cudaGetErrorString(e));
  }
  ppvm::cache_free(b->pool);
  b->pool = static_cast<uint64_t*>(np);
  b->pool_words = words;
  b->layout_dirty = false;
  drop_graphs(b);
  return PPVM_OK;
}

// Resets every instance to its initial terms (resident in the input block, scattered into
// the regions by a kernel).
ppvm_status load_initial(ppvm_batch* b) {
  for (size_t i = 0; i < b->ninst; ++i) {
    BInst& I = b->h_inst[i];
    I.n = b->ic[i].size();
    I.pc = I.op_begin;
    I.tgu = 0;
    I.need = 0;
    I.err = 0;
    I.thr = b->thr[i];
    I.maxw = b->maxw[i];
  }
  BCUDA(cudaMemcpyAsync(b->d_inst, b->h_inst, sizeof(BInst) * b->ninst, cudaMemcpyHostToDevice, b->stream));
  b->xfer_h2d += sizeof(BInst) * b->ninst;
  BDISPATCH(b->W, launch_load, b);
  BCUDA(cudaGetLastError());
  return PPVM_OK;
}

// One CUDA graph per layer (layer index max_layers runs whatever follows the last boundary).
ppvm_status ensure_graphs(ppvm_batch* b) {
  const int cfg[3] = {b->block, b->items, b->W};
  if (b->graphs.size() == (size_t)b->max_layers + 1 && std::equal(cfg, cfg + 3, b->graph_cfg)) return PPVM_OK;
  drop_graphs(b);
  for (uint32_t L = 0; L <= b->max_layers; ++L) {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    BCUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const cudaError_t le = launch_any(b, (int)L);
    const cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
    if (le != cudaSuccess || ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return bfail(PPVM_ECUDA, std::string("layer graph capture failed: ") +
                                   cudaGetErrorString(le != cudaSuccess ? le : ce));
    }
    const cudaError_t ie = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return bfail(PPVM_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
    b->graphs.push_back(ge);
  }
  std::copy(cfg, cfg + 3, b->graph_cfg);
  return PPVM_OK;
}

// After a launch sequence: grows the regions of instances that ran out of capacity.
// Returns the first layer to relaunch through *first (UINT32_MAX when nothing failed).
ppvm_status grow_failed(ppvm_batch* b, uint32_t* first) {
  *first = 0xFFFFFFFFu;
  bool grow = false;
  for (size_t i = 0; i < b->ninst; ++i) {
    BInst& I = b->h_inst[i];
    if (!I.err) continue;
    if (I.err != kErrCapacity)
      return bfail(PPVM_ECUDA, "batch instance " + std::to_string(i) + ": device error " + std::to_string(I.err));
    b->cap[i] = std::max<unsigned long long>(2 * b->cap[i], I.need + I.need / 2 + 64);
    if (b->cap[i] >= 0xFFFFFFF0ull) return bfail(PPVM_ECAPACITY, "batch instance capacity limit (2^32) exceeded");
    I.err = 0;
    grow = true;
    uint32_t L = 0;  // the layer holding the failing op
    while (L < I.n_layers && b->lends[i][L] <= I.pc - I.op_begin) ++L;
    *first = std::min(*first, L);
  }
  if (grow) BTRY(layout(b, true));
  return PPVM_OK;
}

ppvm_status run_all(ppvm_batch* b, bool use_graphs, bool persistent) {
  BCUDA(cudaSetDevice(b->device));
  BTRY(upload_inputs(b));
  if (b->layout_dirty || !b->pool) BTRY(layout(b, false));
  BTRY(load_initial(b));
  uint32_t first = 0;
  for (int attempt = 0; attempt < 64; ++attempt) {
    if (persistent) {
      BCUDA(launch_any(b, -1));
    } else {
      if (use_graphs) BTRY(ensure_graphs(b));
      for (uint32_t L = first; L <= b->max_layers; ++L) {
        if (use_graphs) BCUDA(cudaGraphLaunch(b->graphs[L], b->stream));
        else BCUDA(launch_any(b, (int)L));
      }
    }
    BCUDA(cudaMemcpyAsync(b->h_inst, b->d_inst, sizeof(BInst) * b->ninst, cudaMemcpyDeviceToHost, b->stream));
    BCUDA(cudaStreamSynchronize(b->stream));
    b->xfer_d2h += sizeof(BInst) * b->ninst;
    BTRY(grow_failed(b, &first));
    if (first == 0xFFFFFFFFu) {
      b->ran = true;
      return PPVM_OK;
    }
  }
  return bfail(PPVM_ECAPACITY, "batch capacity growth did not converge");
}

}  // namespace

namespace {

// One instance's gate list as op records, parameter table and layer ends.  Runs on any host
// thread: a failure is returned with its message instead of being recorded.
struct Packed {
  std::vector<BOp> out;
  std::vector<double> par;
  std::vector<uint32_t> le;
  ppvm_status st = PPVM_OK;
  const char* msg = nullptr;
  ppvm_status fail(ppvm_status s, const char* m) {
    st = s;
    msg = m;
    return s;
  }
};

ppvm_status pack_ops(uint32_t n, uint32_t flags, const ppvm_op* ops, size_t n_ops, Packed& pk) {
  const double half_pi = 1.5707963267948966;
  std::vector<BOp>& out = pk.out;
  std::vector<double>& par = pk.par;
  std::vector<uint32_t>& le = pk.le;
  out.clear();
  par.clear();
  le.clear();
  out.reserve(n_ops);
  int truncs = 0;
  SinCosMemo trig;
  // consecutive ops with the same values (bit for bit) share one parameter entry
  double last[3] = {0.0, 0.0, 0.0};
  int last_k = 0;
  uint32_t last_at = 0;
  auto put = [&](const double* v, int k) -> uint32_t {
    if (last_k == k && std::memcmp(last, v, sizeof(double) * k) == 0) return last_at;
    last_at = (uint32_t)par.size();
    par.insert(par.end(), v, v + k);
    std::memcpy(last, v, sizeof(double) * k);
    last_k = k;
    return last_at;
  };
  for (size_t i = 0; i < n_ops; ++i) {
    const ppvm_op& op = ops[i];
    if (op.flags != 0 || op.code >= PPVM_OP_COUNT_) return pk.fail(PPVM_EINVAL, "bad op code or flags");
    if (op.code == PPVM_OP_LOSS_CHANNEL || op.code == PPVM_OP_RESET_LOSS_CHANNEL ||
        op.code == PPVM_OP_CORRELATED_LOSS_CHANNEL)
      return pk.fail(PPVM_EINVAL, "batched instances hold plain words: loss channels need a lossy PauliSum");
    if (op.code == PPVM_OP_TRUNCATE) {
      out.push_back(BOp{bop_header(B_TRUNC, 0, false, 0, 0, 0, 0), 0u});
      if (++truncs % 2 == 0) le.push_back((uint32_t)out.size());
      continue;
    }
    const bool two = op.code == PPVM_OP_CNOT || op.code == PPVM_OP_CZ || op.code == PPVM_OP_CY ||
                     op.code == PPVM_OP_RXX || op.code == PPVM_OP_RYY || op.code == PPVM_OP_RZZ ||
                     op.code == PPVM_OP_DEPOLARIZE2;
    if (op.q0 >= n || (two && (op.q1 >= n || op.q1 == op.q0)))
      return pk.fail(PPVM_EINVAL, "qubit index out of range (or a two-qubit op on one qubit)");
    const uint32_t q0 = op.q0, q1 = two ? op.q1 : op.q0;
    const bool rot = op.code >= PPVM_OP_RX && op.code <= PPVM_OP_RZZ;
    if (rot) {
      const bool gx = op.code == PPVM_OP_RX || op.code == PPVM_OP_RY || op.code == PPVM_OP_RXX || op.code == PPVM_OP_RYY;
      const bool gz = op.code == PPVM_OP_RZ || op.code == PPVM_OP_RY || op.code == PPVM_OP_RZZ || op.code == PPVM_OP_RYY;
      const uint32_t ax = (gx ? 1u : 0u) | ((gx && two) ? 2u : 0u);
      const uint32_t az = (gz ? 1u : 0u) | ((gz && two) ? 2u : 0u);
      if ((flags & PPVM_FLAG_CLIFFORD_ANGLES) && (op.theta == half_pi || op.theta == -half_pi)) {
        const double sign = op.theta > 0 ? 1.0 : -1.0;
        out.push_back(BOp{bop_header(B_LOCAL, C_ROTC, two, ax, az, q0, q1), put(&sign, 1)});
      } else {
        double sc[2];
        trig.get(op.theta, sc[0], sc[1]);
        out.push_back(BOp{bop_header(B_ROT, 0, two, ax, az, q0, q1), put(sc, 2)});
      }
      continue;
    }
    uint32_t code = 0;
    double f[3] = {0.0, 0.0, 0.0};
    int nf = 0;
    switch (op.code) {
      case PPVM_OP_X: code = C_X; break;
      case PPVM_OP_Y: code = C_Y; break;
      case PPVM_OP_Z: code = C_Z; break;
      case PPVM_OP_H: code = C_H; break;
      case PPVM_OP_S: code = C_S; break;
      case PPVM_OP_S_DAG: code = C_SDAG; break;
      case PPVM_OP_SQRT_X: code = C_SQX; break;
      case PPVM_OP_SQRT_X_DAG: code = C_SQXDAG; break;
      case PPVM_OP_SQRT_Y: code = C_SQY; break;
      case PPVM_OP_SQRT_Y_DAG: code = C_SQYDAG; break;
      case PPVM_OP_CNOT: code = C_CNOT; break;
      case PPVM_OP_CZ: code = C_CZ; break;
      case PPVM_OP_CY: code = C_CY; break;
      case PPVM_OP_PAULI_ERROR: {  // noise.rs:17-37, factors as the per-op pass computes them
        code = C_PAULI_ERROR;
        const double one = 1.0;
        f[0] = one - op.p[1] * 2.0 - op.p[2] * 2.0;
        f[1] = one - op.p[0] * 2.0 - op.p[1] * 2.0;
        f[2] = one - op.p[0] * 2.0 - op.p[2] * 2.0;
        nf = 3;
        break;
      }
      case PPVM_OP_DEPOLARIZE1: code = C_DEP1; f[0] = 1.0 - op.theta * (4.0 / 3.0); nf = 1; break;
      case PPVM_OP_DEPOLARIZE2: code = C_DEP2; f[0] = 1.0 - op.theta * (16.0 / 15.0); nf = 1; break;
      default: return pk.fail(PPVM_EINVAL, "unsupported op in a batch");
    }
    out.push_back(BOp{bop_header(B_LOCAL, code, two, 0, 0, q0, q1), nf ? put(f, nf) : 0u});
  }
  if (par.size() >= 0xFFFFFFF0ull) return pk.fail(PPVM_ECAPACITY, "batch parameter table too long");
  return PPVM_OK;
}

}  // namespace

namespace ppvm {
void release_batch_staging() {
  Staging& st = staging();
  std::lock_guard<std::mutex> lk(st.mu);
  if (st.p) cudaFreeHost(st.p);
  st.p = nullptr;
  st.cap = 0;
}
}  // namespace ppvm

extern "C" {

ppvm_status ppvm_batch_destroy(ppvm_batch* b) {
  if (!b) return PPVM_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graphs(b);
  ppvm::cache_free(b->d_inst);
  cudaFreeHost(b->h_inst);
  ppvm::cache_free(b->d_input);
  ppvm::cache_free(b->pool);
  ppvm::cache_free(b->d_out);
  if (b->stream && b->own_stream) cudaStreamDestroy(b->stream);
  delete b;
  return PPVM_OK;
}

ppvm_status ppvm_batch_create(ppvm_batch** out, size_t n_inst, const uint32_t* n_qubits, const double* min_abs_coeff,
                              const uint64_t* max_weight, uint32_t flags, int device) {
  if (!out) return bfail(PPVM_EINVAL, "null out pointer");
  *out = nullptr;
  if (n_inst == 0 || n_inst > 65535 || !n_qubits || !min_abs_coeff || !max_weight)
    return bfail(PPVM_EINVAL, "need 1..65535 instances and their n_qubits, min_abs_coeff, max_weight");
  uint32_t nmax = 0;
  for (size_t i = 0; i < n_inst; ++i) {
    if (n_qubits[i] == 0 || n_qubits[i] > 512) return bfail(PPVM_EINVAL, "n_qubits must be in [1, 512]");
    nmax = std::max(nmax, n_qubits[i]);
  }
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) return bfail(PPVM_ENODEV, std::string("no CUDA device: ") + cudaGetErrorString(e));
  if (device < 0 || device >= count) return bfail(PPVM_EINVAL, "device ordinal out of range");
  BCUDA(cudaSetDevice(device));
  ppvm_batch* b = new ppvm_batch();
  b->device = device;
  b->flags = flags;
  b->ninst = n_inst;
  b->W = batch_words(nmax);
  b->nq.assign(n_qubits, n_qubits + n_inst);
  b->thr.assign(min_abs_coeff, min_abs_coeff + n_inst);
  b->maxw.assign(max_weight, max_weight + n_inst);
  b->ix.resize(n_inst);
  b->iz.resize(n_inst);
  b->ic.resize(n_inst);
  b->ops.resize(n_inst);
  b->params.resize(n_inst);
  b->lends.resize(n_inst);
  b->cap.assign(n_inst, 256);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      ppvm::cache_malloc((void**)&b->d_inst, sizeof(BInst) * n_inst) != cudaSuccess ||
      cudaMallocHost(&b->h_inst, sizeof(BInst) * n_inst) != cudaSuccess ||
      ppvm::cache_malloc((void**)&b->d_out, sizeof(double) * n_inst) != cudaSuccess) {
    ppvm_batch_destroy(b);
    return bfail(PPVM_ECAPACITY, "device allocation failed");
  }
  std::memset(b->h_inst, 0, sizeof(BInst) * n_inst);
  *out = b;
  return PPVM_OK;
}

ppvm_status ppvm_batch_set_stream(ppvm_batch* b, void* cuda_stream) {
  if (!b) return bfail(PPVM_EINVAL, "null batch");
  BCUDA(cudaSetDevice(b->device));
  BCUDA(cudaStreamSynchronize(b->stream));
  if (b->own_stream) cudaStreamDestroy(b->stream);
  if (cuda_stream) {
    b->stream = (cudaStream_t)cuda_stream;
    b->own_stream = false;
  } else {
    BCUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    b->own_stream = true;
  }
  drop_graphs(b);
  return PPVM_OK;
}

ppvm_status ppvm_batch_add_terms(ppvm_batch* b, size_t inst, const uint64_t* x, const uint64_t* z, const double* c,
                                 size_t k) {
  if (!b || inst >= b->ninst) return bfail(PPVM_EINVAL, "bad batch or instance index");
  if (k && (!x || !z || !c)) return bfail(PPVM_EINVAL, "null term arrays");
  const int wi = words_of(b->nq[inst]);
  const int tail = (int)(b->nq[inst] % 64);
  auto& X = b->ix[inst];
  auto& Z = b->iz[inst];
  auto& Cc = b->ic[inst];
  for (size_t t = 0; t < k; ++t) {
    if (tail && ((x[t * wi + wi - 1] | z[t * wi + wi - 1]) >> tail))
      return bfail(PPVM_EINVAL, "word has bits set at or above n_qubits");
    // `+=` into an insertion-ordered map (crates/ppvm-pauli-sum/src/sum/ops.rs:140-151)
    size_t j = 0;
    const size_t have = Cc.size();
    for (; j < have; ++j) {
      bool eq = true;
      for (int w = 0; w < wi && eq; ++w) eq = X[j * wi + w] == x[t * wi + w] && Z[j * wi + w] == z[t * wi + w];
      if (eq) break;
    }
    if (j < have) {
      Cc[j] += c[t];
    } else {
      X.insert(X.end(), x + t * wi, x + (t + 1) * wi);
      Z.insert(Z.end(), z + t * wi, z + (t + 1) * wi);
      Cc.push_back(c[t]);
    }
  }
  const unsigned long long want = 2 * Cc.size() + 64;
  if (want > b->cap[inst]) {
    b->cap[inst] = want;
    b->layout_dirty = true;
  }
  b->inputs_dirty = true;
  return PPVM_OK;
}

ppvm_status ppvm_batch_set_ops(ppvm_batch* b, size_t inst, const ppvm_op* ops, size_t n_ops) {
  if (!b || inst >= b->ninst) return bfail(PPVM_EINVAL, "bad batch or instance index");
  if (n_ops && !ops) return bfail(PPVM_EINVAL, "null op list");
  Packed pk;
  if (pack_ops(b->nq[inst], b->flags, ops, n_ops, pk) != PPVM_OK) return bfail(pk.st, pk.msg);
  b->ops[inst] = std::move(pk.out);
  b->params[inst] = std::move(pk.par);
  b->lends[inst] = std::move(pk.le);
  b->inputs_dirty = true;
  return PPVM_OK;
}

ppvm_status ppvm_batch_set_ops_all(ppvm_batch* b, const ppvm_op* const* ops, const size_t* n_ops) {
  if (!b || !ops || !n_ops) return bfail(PPVM_EINVAL, "null argument");
  for (size_t i = 0; i < b->ninst; ++i)
    if (n_ops[i] && !ops[i]) return bfail(PPVM_EINVAL, "null op list of instance " + std::to_string(i));
  std::vector<Packed> pk(b->ninst);
  size_t total = 0;
  for (size_t i = 0; i < b->ninst; ++i) total += n_ops[i];
  // host threads over instances, each packing whole lists (about 10^5 ops per thread at least)
  const size_t hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nt = std::min({hw, (size_t)16, b->ninst, total / 100000 + 1});
  std::atomic<size_t> next{0};
  auto work = [&] {
    for (size_t i; (i = next.fetch_add(1)) < b->ninst;) pack_ops(b->nq[i], b->flags, ops[i], n_ops[i], pk[i]);
  };
  std::vector<std::thread> th;
  for (size_t t = 1; t < nt; ++t) th.emplace_back(work);
  work();
  for (auto& t : th) t.join();
  for (size_t i = 0; i < b->ninst; ++i)  // nothing changes unless every list is valid
    if (pk[i].st != PPVM_OK) return bfail(pk[i].st, "instance " + std::to_string(i) + ": " + pk[i].msg);
  for (size_t i = 0; i < b->ninst; ++i) {
    b->ops[i] = std::move(pk[i].out);
    b->params[i] = std::move(pk[i].par);
    b->lends[i] = std::move(pk[i].le);
  }
  b->inputs_dirty = true;
  return PPVM_OK;
}

ppvm_status ppvm_batch_reserve(ppvm_batch* b, const uint64_t* caps) {
  if (!b || !caps) return bfail(PPVM_EINVAL, "null argument");
  for (size_t i = 0; i < b->ninst; ++i) {
    if (caps[i] >= 0xFFFFFFF0ull) return bfail(PPVM_EINVAL, "capacity limit (2^32) exceeded");
    if (caps[i] > b->cap[i]) {
      b->cap[i] = caps[i];
      b->layout_dirty = true;
    }
  }
  return PPVM_OK;
}

ppvm_status ppvm_batch_get_capacity(const ppvm_batch* b, uint64_t* caps) {
  if (!b || !caps) return bfail(PPVM_EINVAL, "null argument");
  for (size_t i = 0; i < b->ninst; ++i) caps[i] = b->cap[i];
  return PPVM_OK;
}

ppvm_status ppvm_batch_set_config(ppvm_batch* b, int block, int items, int table_factor) {
  if (!b) return bfail(PPVM_EINVAL, "null batch");
  if ((block != 128 && block != 256 && block != 512) || (items != 2 && items != 4) ||
      (table_factor != 2 && table_factor != 4))
    return bfail(PPVM_EINVAL, "block in {128, 256, 512}, items in {2, 4}, table_factor in {2, 4}");
  if (table_factor != b->tfac) b->layout_dirty = true;
  b->block = block;
  b->items = items;
  b->tfac = table_factor;
  return PPVM_OK;
}

ppvm_status ppvm_batch_get_config(const ppvm_batch* b, int* block, int* items, int* table_factor) {
  if (!b || !block || !items || !table_factor) return bfail(PPVM_EINVAL, "null argument");
  *block = b->block;
  *items = b->items;
  *table_factor = b->tfac;
  return PPVM_OK;
}

ppvm_status ppvm_batch_run(ppvm_batch* b) {
  if (!b) return bfail(PPVM_EINVAL, "null batch");
  // Layer graphs pay off from the second run of an unchanged batch on.  A batch's first run
  // (and the first after new ops or a new layout) launches the layers directly, which saves
  // capturing and instantiating one graph per layer for a batch that runs once.
  const bool reuse = b->ran && !b->inputs_dirty && !b->layout_dirty;
  return run_all(b, reuse, false);
}

ppvm_status ppvm_batch_run_persistent(ppvm_batch* b) {
  if (!b) return bfail(PPVM_EINVAL, "null batch");
  return run_all(b, false, true);
}

ppvm_status ppvm_batch_autotune(ppvm_batch* b, int* block, int* items, int* table_factor, double* best_ms) {
  if (!b) return bfail(PPVM_EINVAL, "null batch");
  BCUDA(cudaSetDevice(b->device));
  BTRY(run_all(b, true, false));  // sizes every region to its peak first
  const int blocks[3] = {128, 256, 512}, its[2] = {2, 4}, tfs[2] = {2, 4};
  double best = 1e300;
  int bb = b->block, bi = b->items, bt = b->tfac;
  cudaEvent_t e0, e1;
  BCUDA(cudaEventCreate(&e0));
  BCUDA(cudaEventCreate(&e1));
  for (int tf : tfs)
    for (int bl : blocks)
      for (int it : its) {
        BTRY(ppvm_batch_set_config(b, bl, it, tf));
        BTRY(run_all(b, true, false));  // warm: graphs captured, layout fixed
        BCUDA(cudaEventRecord(e0, b->stream));
        BTRY(run_all(b, true, false));
        BCUDA(cudaEventRecord(e1, b->stream));
        BCUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        BCUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) {
          best = ms;
          bb = bl;
          bi = it;
          bt = tf;
        }
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  BTRY(ppvm_batch_set_config(b, bb, bi, bt));
  BTRY(run_all(b, true, false));
  if (block) *block = bb;
  if (items) *items = bi;
  if (table_factor) *table_factor = bt;
  if (best_ms) *best_ms = best;
  return PPVM_OK;
}

ppvm_status ppvm_batch_overlap_with_zero(ppvm_batch* b, double* out) {
  if (!b || !out) return bfail(PPVM_EINVAL, "null argument");
  if (!b->ran) return bfail(PPVM_EINVAL, "run the batch first");
  BCUDA(cudaSetDevice(b->device));
  BDISPATCH(b->W, launch_owz, b);
  BCUDA(cudaGetLastError());
  BCUDA(cudaMemcpyAsync(out, b->d_out, sizeof(double) * b->ninst, cudaMemcpyDeviceToHost, b->stream));
  BCUDA(cudaStreamSynchronize(b->stream));
  b->xfer_d2h += sizeof(double) * b->ninst;
  return PPVM_OK;
}

ppvm_status ppvm_batch_transfer_counters(const ppvm_batch* b, uint64_t* h2d_bytes, uint64_t* d2h_bytes) {
  if (!b || !h2d_bytes || !d2h_bytes) return bfail(PPVM_EINVAL, "null argument");
  *h2d_bytes = b->xfer_h2d;
  *d2h_bytes = b->xfer_d2h;
  return PPVM_OK;
}

ppvm_status ppvm_batch_len(const ppvm_batch* b, size_t inst, size_t* out) {
  if (!b || !out || inst >= b->ninst) return bfail(PPVM_EINVAL, "bad argument");
  *out = b->ran ? (size_t)b->h_inst[inst].n : b->ic[inst].size();
  return PPVM_OK;
}

ppvm_status ppvm_batch_term_gate_updates(const ppvm_batch* b, uint64_t* per_inst, uint64_t* total) {
  if (!b) return bfail(PPVM_EINVAL, "null batch");
  uint64_t t = 0;
  for (size_t i = 0; i < b->ninst; ++i) {
    const uint64_t v = b->ran ? b->h_inst[i].tgu : 0;
    if (per_inst) per_inst[i] = v;
    t += v;
  }
  if (total) *total = t;
  return PPVM_OK;
}

ppvm_status ppvm_batch_export_terms(ppvm_batch* b, size_t inst, uint64_t* x, uint64_t* z, double* c, size_t cap,
                                    size_t* n_out) {
  if (!b || !n_out || inst >= b->ninst) return bfail(PPVM_EINVAL, "bad argument");
  if (!b->ran) return bfail(PPVM_EINVAL, "run the batch first");
  const BInst& I = b->h_inst[inst];
  const size_t n = std::min<size_t>(cap, I.n);
  *n_out = n;
  if (n == 0) return PPVM_OK;
  if (!x || !z || !c) return bfail(PPVM_EINVAL, "null output arrays");
  BCUDA(cudaSetDevice(b->device));
  const int W = b->W, wi = words_of(b->nq[inst]);
  std::vector<uint64_t> buf((size_t)(2 * W) * n);
  const uint64_t* base = b->pool + I.off;
  for (int w = 0; w < 2 * W; ++w)
    BCUDA(cudaMemcpyAsync(buf.data() + (size_t)w * n, base + (size_t)w * I.cap, sizeof(uint64_t) * n,
                          cudaMemcpyDeviceToHost, b->stream));
  BCUDA(cudaMemcpyAsync(c, base + (size_t)2 * W * I.cap, sizeof(double) * n, cudaMemcpyDeviceToHost, b->stream));
  BCUDA(cudaStreamSynchronize(b->stream));
  for (size_t i = 0; i < n; ++i)
    for (int w = 0; w < wi; ++w) {
      x[i * wi + w] = buf[(size_t)w * n + i];
      z[i * wi + w] = buf[(size_t)(W + w) * n + i];
    }
  return PPVM_OK;
}

}  // extern "C"
