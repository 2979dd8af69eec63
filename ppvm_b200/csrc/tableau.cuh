// tableau.cuh — a run of Clifford gates applied as one composed map (Clifford tableau).
//
// Every Clifford gate of the reference (sum/clifford.rs:37-221, with the sign tables of
// crates/ppvm-pauli-word/src/phase/clifford.rs:72-182) maps a Pauli word P to +-P', and that
// map is conjugation by a unitary, so it respects products: f(A B) = f(A) f(B).  The map of a
// whole run, f = f_L o ... o f_1, is therefore fixed by the images of the 2n generators X_q,
// Z_q.  The host composes those images once per run (64 generators per machine word, gates in
// run order, with the same per-gate rules the per-op kernel uses), and k_tableau maps each
// term with one product over its non-identity qubits instead of L gate steps:
//
//   P = i^{|x&z|} X^x Z^z  ->  i^{|x&z|} prod_{q in x} f(X_q) prod_{q in z} f(Z_q)
//
// with images stored as i^ph X^a Z^b and X^u Z^v X^a Z^b = (-1)^{|v&a|} X^{u^a} Z^{v^b}.  A
// sign flip is the only change to a coefficient, so the result is bit-identical to applying
// the gates one by one.  The truncation that ends the run (if any) is fused: survivors are
// written, in order, to the alternate planes (stable compaction with decoupled look-back).
#pragma once

#include "kernels.cuh"

namespace ppvm {

constexpr int kTabMinOps = 8;          // shorter Clifford runs use the per-op pass
constexpr int kTabBlock = 256;
constexpr size_t kTabMaxSmem = 160 * 1024;

// ---- per-gate rules over "bit vectors" B: bool (one word) or uint64_t (64 words at once) ----
__host__ __device__ __forceinline__ bool bnot(int b) { return !b; }  // bool operands promote to int
__host__ __device__ __forceinline__ uint64_t bnot(uint64_t b) { return ~b; }
template <class B>
__host__ __device__ __forceinline__ B bconst(bool v);
template <>
__host__ __device__ __forceinline__ bool bconst<bool>(bool v) { return v; }
template <>
__host__ __device__ __forceinline__ uint64_t bconst<uint64_t>(bool v) { return v ? ~0ull : 0ull; }

// Applies the Clifford op d to the bits of its qubit(s): (x0, z0) on q0, (x1, z1) on q1, and
// toggles neg where the word's sign flips.  The rules are those of k_clifford.  Returns false
// (and changes nothing) for the diagonal noise ops, which are not Clifford maps.
template <class B>
__host__ __device__ inline bool cliff_rule(const DevOp& d, B& x0, B& z0, B& x1, B& z1, B& neg) {
  switch (d.code) {
    case C_X: neg ^= z0; break;
    case C_Y: neg ^= x0 ^ z0; break;
    case C_Z: neg ^= x0; break;
    case C_H: { neg ^= x0 & z0; const B t = x0; x0 = z0; z0 = t; break; }
    case C_S: neg ^= x0 & bnot(z0); z0 ^= x0; break;
    case C_SDAG: neg ^= x0 & z0; z0 ^= x0; break;
    case C_SQX: neg ^= x0 & z0; x0 ^= z0; break;
    case C_SQXDAG: neg ^= bnot(x0) & z0; x0 ^= z0; break;
    case C_SQY: { neg ^= bnot(x0) & z0; const B t = x0; x0 = z0; z0 = t; break; }
    case C_SQYDAG: { neg ^= x0 & bnot(z0); const B t = x0; x0 = z0; z0 = t; break; }
    case C_CNOT: {  // q0 control, q1 target
      const B xc = x0, zc = z0, xt = x1, zt = z1;
      neg ^= xc & zt & bnot(xt ^ zc);
      z0 = zc ^ zt;
      x1 = xt ^ xc;
      break;
    }
    case C_CZ: {
      const B xc = x0, zc = z0, xt = x1, zt = z1;
      neg ^= xc & xt & (zc ^ zt);
      z0 = zc ^ xt;
      z1 = zt ^ xc;
      break;
    }
    case C_CY: {
      const B xc = x0, zc = z0, xt = x1, zt = z1;
      neg ^= xc & (xt ^ zt) & bnot(zc ^ zt);
      z0 = zc ^ xt ^ zt;
      x1 = xt ^ xc;
      z1 = zt ^ xc;
      break;
    }
    case C_ROTC: {
      // exp(-i theta/2 G) at theta = +-pi/2: anticommuting P -> (eps * sign(theta)) (P xor G).
      // eps = +1 exactly when the one anticommuting qubit has single-qubit phase -1 in G*P
      // (G_q = X: P_q = Z; G_q = Y: P_q = X; G_q = Z: P_q = Y), the rule of rot_sign.
      const bool two = d.two != 0;
      const B ax0 = bconst<B>(d.ax & 1), az0 = bconst<B>(d.az & 1);
      const B ax1 = bconst<B>(two && ((d.ax >> 1) & 1)), az1 = bconst<B>(two && ((d.az >> 1) & 1));
      const B anti = (x0 & az0) ^ (z0 & ax0) ^ (x1 & az1) ^ (z1 & ax1);
      const B m0 = (ax0 & bnot(az0) & bnot(x0) & z0) | (ax0 & az0 & x0 & bnot(z0)) |
                   (bnot(ax0) & az0 & x0 & z0);
      const B m1 = (ax1 & bnot(az1) & bnot(x1) & z1) | (ax1 & az1 & x1 & bnot(z1)) |
                   (bnot(ax1) & az1 & x1 & z1);
      const B eps_plus = m0 | m1;
      neg ^= anti & (d.f0 > 0.0 ? bnot(eps_plus) : eps_plus);
      x0 ^= anti & ax0;
      z0 ^= anti & az0;
      x1 ^= anti & ax1;
      z1 ^= anti & az1;
      break;
    }
    default: return false;
  }
  return true;
}

__host__ __device__ inline bool is_cliff_code(uint32_t code) {
  return code <= C_CY || code == C_ROTC;
}

// ---- device side --------------------------------------------------------------------------
struct TabParams {
  uint64_t T[kMaxW];    // touched qubits (support of the run)
  uint64_t Tx[kMaxW];   // touched qubits whose X_q image is not X_q itself
  uint64_t Tz[kMaxW];   // touched qubits whose Z_q image is not Z_q itself
  uint32_t pre[kMaxW];  // touched qubits in words < w (rank prefix)
  uint32_t nrows;       // 2 * touched: row 2r = image of X_q, 2r+1 = image of Z_q (r = rank of q)
};

// Maps the word (x, z) through the composed run: (ox, oz) receives the image word, and the
// return value e is the sign's phase, image = i^e * (Hermitian word): e = 0 or 2 (sign -1);
// an odd e would mean a broken table.  rows/ph: the image table (shared memory).
//
// Generators whose image is themselves are left out of the product: bits outside Tx (X) and
// Tz (Z) stay as they are.  The product takes the X images before the Z images, so a kept
// Z_q passes the X images; it anticommutes only with the image of X_q (images keep the
// commutation of their generators), which contributes a sign where x_q = z_q = 1, q in Tx
// and not in Tz.
template <int W>
__device__ __forceinline__ unsigned tab_map(const uint64_t* rows, const uint8_t* ph, const TabParams& tp,
                                            const uint64_t (&x)[W], const uint64_t (&z)[W], uint64_t (&ox)[W],
                                            uint64_t (&oz)[W]) {
  unsigned p = 0;
  uint64_t m[2 * W];
#pragma unroll
  for (int w = 0; w < W; ++w) {
    p += __popcll(x[w] & z[w]) + 2u * __popcll(x[w] & z[w] & tp.Tx[w] & ~tp.Tz[w]);
    ox[w] = x[w] & ~tp.Tx[w];
    oz[w] = z[w] & ~tp.Tz[w];
    m[w] = x[w] & tp.Tx[w];
    m[W + w] = z[w] & tp.Tz[w];
  }
#pragma unroll
  for (int s = 0; s < 2; ++s) {
#pragma unroll
    for (int w = 0; w < W; ++w) {
      uint64_t mk = m[s * W + w];
      while (mk) {
        const int b = __ffsll((long long)mk) - 1;
        mk &= mk - 1;
        const unsigned row = 2u * (tp.pre[w] + __popcll(tp.T[w] & ((1ull << b) - 1ull))) + (unsigned)s;
        const uint64_t* e = rows + (size_t)row * 2 * W;
        unsigned t = 0;
#pragma unroll
        for (int ww = 0; ww < W; ++ww) {
          const uint64_t a = e[ww];
          t += __popcll(oz[ww] & a);
          ox[ww] ^= a;
          oz[ww] ^= e[W + ww];
        }
        p += ph[row] + 2u * t;
      }
    }
  }
  unsigned hw = 0;
#pragma unroll
  for (int w = 0; w < W; ++w) hw += __popcll(ox[w] & oz[w]);
  return (p - hw) & 3u;
}

// ---- chunk tables (one machine word, n <= 64) ----------------------------------------------
// tab_map costs one image per moved bit, up to 128 for a heavy 64-qubit term.  With one word
// the block can instead tabulate, for each 4-qubit chunk c, the images of all 256 sub-words
// X^{x_c} Z^{z_c} (16 tables, 64 KB of shared memory), and a term maps with 16 lookups
// whatever its weight.  The chunks' factors act on disjoint qubits and commute, so
//   X^x Z^z = prod_c X^{x_c} Z^{z_c}   and   f(X^x Z^z) = prod_c f(X^{x_c} Z^{z_c})
// exactly, phases included: the image is the one tab_map computes.  A warp takes the tables
// when one of its terms has more than chunk_min moved bits.
constexpr int kTabChunks = 16;                 // 4 qubits each
constexpr int kTabChunkEntries = 256;          // index: x nibble | z nibble << 4
constexpr size_t kTabChunkSmem = (size_t)kTabChunks * kTabChunkEntries * (2 * sizeof(uint64_t) + 1);
constexpr int kTabChunkMinBits = 12;           // per warp: tables above this many moved bits
constexpr unsigned long long kTabChunkMinTerms = 1ull << 15;  // host: build them from here on
constexpr int kTabChunkMinMoved = 32;          // host: and when the run moves this many generators

// The image of X_q (s = 0) or Z_q (s = 1) multiplied onto i^p X^u Z^v from the right.
__device__ __forceinline__ void tab_mul_gen(const uint64_t* rows, const uint8_t* ph, uint64_t T, int q, int s,
                                            uint64_t& u, uint64_t& v, unsigned& p) {
  uint64_t a, b;
  unsigned e;
  if ((T >> q) & 1ull) {
    const unsigned row = 2u * (unsigned)__popcll(T & ((1ull << q) - 1ull)) + (unsigned)s;
    a = rows[2 * row];
    b = rows[2 * row + 1];
    e = ph[row];
  } else {  // untouched qubit: the generator itself
    a = s ? 0ull : 1ull << q;
    b = s ? 1ull << q : 0ull;
    e = 0;
  }
  p += e + 2u * (unsigned)__popcll(v & a);
  u ^= a;
  v ^= b;
}

// Fills the 16 chunk tables: thread (c, x nibble) forms f(X^{x_c}), then walks the 16 z nibbles
// in Gray-code order, one image product per entry.  Dropping Z_q again multiplies by f(Z_q),
// which is exact: the Z images commute and each squares to the identity.
__device__ inline void tab_build_chunks(const uint64_t* rows, const uint8_t* ph, uint64_t T, uint64_t* tab,
                                        uint8_t* tph) {
  for (unsigned t = threadIdx.x; t < (unsigned)kTabChunks * 16u; t += blockDim.x) {
    const int c = (int)(t >> 4);
    const unsigned xv = t & 15u;
    uint64_t u = 0, v = 0;
    unsigned p = 0;
    for (int j = 0; j < 4; ++j)
      if ((xv >> j) & 1u) tab_mul_gen(rows, ph, T, 4 * c + j, 0, u, v, p);
    unsigned idx = (unsigned)c * kTabChunkEntries + xv;
    tab[2 * idx] = u;
    tab[2 * idx + 1] = v;
    tph[idx] = (uint8_t)(p & 3u);
    unsigned g = 0;
    for (unsigned k = 1; k < 16; ++k) {
      const int j = __ffs((int)k) - 1;
      g ^= 1u << j;
      tab_mul_gen(rows, ph, T, 4 * c + j, 1, u, v, p);
      idx = (unsigned)c * kTabChunkEntries + (xv | (g << 4));
      tab[2 * idx] = u;
      tab[2 * idx + 1] = v;
      tph[idx] = (uint8_t)(p & 3u);
    }
  }
}

// tab_map for one word through the chunk tables; same contract.
__device__ __forceinline__ unsigned tab_map_chunks(const uint64_t* tab, const uint8_t* tph, uint64_t x, uint64_t z,
                                                   uint64_t& ox, uint64_t& oz) {
  unsigned p = (unsigned)__popcll(x & z);
  uint64_t u = 0, v = 0;
  const ulonglong2* t2 = reinterpret_cast<const ulonglong2*>(tab);
#pragma unroll
  for (int c = 0; c < kTabChunks; ++c) {
    const unsigned idx = (unsigned)c * kTabChunkEntries + (unsigned)((x >> (4 * c)) & 15ull) +
                         ((unsigned)((z >> (4 * c)) & 15ull) << 4);
    const ulonglong2 e = t2[idx];
    p += tph[idx] + 2u * (unsigned)__popcll(v & e.x);
    u ^= e.x;
    v ^= e.y;
  }
  ox = u;
  oz = v;
  return (p - (unsigned)__popcll(u & v)) & 3u;
}

// Maps every live term through the run; with trunc, drops what the strategy drops.  Survivors
// go to O in input order; the last block to finish publishes their count (and the log of the
// fused TRUNCATE, trunc_op).  chunk_min >= 0 (one word only): the block builds the chunk
// tables, and a warp maps through them when one of its terms has more than chunk_min moved
// bits.  Dynamic shared memory: [chunk tables][rows][chunk phases][row phases], the chunk
// parts only with chunk_min >= 0.
template <int W, int BLOCK, int ITEMS>
__global__ void __launch_bounds__(BLOCK)
k_tableau(Planes P, Planes O, Ctrl* ctrl, TabParams tp, const uint64_t* __restrict__ g_rows,
          const uint8_t* __restrict__ g_ph, int trunc, double thr, unsigned long long maxw,
          unsigned long long* ts, unsigned epoch, int op0, int nops, int trunc_op, OpLog* log, int chunk_min) {
  pdl_wait();
  extern __shared__ __align__(16) uint64_t s_dyn[];
  __shared__ unsigned s_tile;
  __shared__ unsigned long long s_slot;
  __shared__ unsigned s_base[ITEMS * (BLOCK / 32) + 1];
  __shared__ int s_err;
  const bool chunked = W == 1 && chunk_min >= 0;
  uint64_t* s_tab = s_dyn;
  uint64_t* s_rows = s_dyn + (chunked ? (size_t)kTabChunks * kTabChunkEntries * 2 : 0);
  uint8_t* s_tph = reinterpret_cast<uint8_t*>(s_rows + (size_t)tp.nrows * 2 * W);
  uint8_t* s_ph = s_tph + (chunked ? kTabChunks * kTabChunkEntries : 0);
  if (threadIdx.x == 0) s_err = ld_volatile_int(&ctrl->err);
  for (unsigned i = threadIdx.x; i < tp.nrows * 2 * W; i += BLOCK) s_rows[i] = g_rows[i];
  for (unsigned i = threadIdx.x; i < tp.nrows; i += BLOCK) s_ph[i] = g_ph[i];
  __syncthreads();
  if (s_err) return;
  if constexpr (W == 1) {
    if (chunked) {
      tab_build_chunks(s_rows, s_ph, tp.T[0], s_tab, s_tph);
      __syncthreads();
    }
  }
  const unsigned long long N = ld_volatile(&ctrl->n);
  constexpr unsigned long long TILE = (unsigned long long)BLOCK * ITEMS;
  const unsigned long long ntiles = (N + TILE - 1) / TILE;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    for (int o = 0; o < nops; ++o) {
      log[op0 + o].n_in = N;
      log[op0 + o].n_s = N;
      log[op0 + o].n_new = 0;
      log[op0 + o].n_out = N;
    }
    if (N == 0) ctrl->n_s = 0;
  }
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = BLOCK / 32;
  const bool wcap = maxw != ~0ull;
  for (;;) {
    const unsigned tile = next_tile(&ctrl->tickets[3], &s_tile);
    if (tile >= ntiles) break;
    const unsigned long long base = (unsigned long long)tile * TILE;
    uint64_t ox[ITEMS][W], oz[ITEMS][W];
    double oc[ITEMS];
    unsigned keep_b[ITEMS];
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const unsigned long long i = base + (unsigned long long)k * BLOCK + threadIdx.x;
      bool keep = false;
      uint64_t x[W], z[W];
#pragma unroll
      for (int w = 0; w < W; ++w) x[w] = z[w] = 0ull;
      if (i < N) load_key<W>(P, i, x, z);
      [[maybe_unused]] bool use_tables = false;
      if constexpr (W == 1) {
        if (chunked) {  // warp-uniform: every lane of the block reaches each item
          const int moved = __popcll(x[0] & tp.Tx[0]) + __popcll(z[0] & tp.Tz[0]);
          use_tables = __any_sync(kFull, moved > chunk_min);
        }
      }
      if (i < N) {
        const double c = P.c[i];
        unsigned e;
        if constexpr (W == 1) {
          e = use_tables ? tab_map_chunks(s_tab, s_tph, x[0], z[0], ox[k][0], oz[k][0])
                         : tab_map<W>(s_rows, s_ph, tp, x, z, ox[k], oz[k]);
        } else {
          e = tab_map<W>(s_rows, s_ph, tp, x, z, ox[k], oz[k]);
        }
        if (e & 1u) set_err(ctrl, kErrProbe, op0);  // not a Hermitian image: internal error
        oc[k] = (e == 2u) ? -c : c;
        keep = true;
        if (trunc) {
          keep = !(fabs(c) < thr);
          if (wcap) keep = keep && (weight<W>(ox[k], oz[k]) <= maxw);
        }
      }
      keep_b[k] = __ballot_sync(kFull, keep);
    }
    const unsigned agg = tile_ranks<BLOCK, ITEMS>(keep_b, s_base);
    const unsigned long long excl = lookback(ts, tile, agg, epoch, ctrl, op0, &s_slot);
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      if ((keep_b[k] >> lane) & 1u) {
        const unsigned long long r = excl + s_base[k * NW + warp] + __popc(keep_b[k] & ((1u << lane) - 1u));
        store_key<W>(O, r, ox[k], oz[k]);
        O.c[r] = oc[k];
      }
    }
    if (tile == ntiles - 1 && threadIdx.x == 0) ctrl->n_s = excl + agg;
  }
  if (last_block_done(&ctrl->done) && threadIdx.x == 0) {
    for (int t = 0; t < 4; ++t) ctrl->tickets[t] = 0;
    if (ld_volatile_int(&ctrl->err)) return;
    const unsigned long long n_out = N == 0 ? 0ull : ld_volatile(&ctrl->n_s);
    if (trunc_op >= 0) {
      log[trunc_op].n_in = N;
      log[trunc_op].n_s = n_out;
      log[trunc_op].n_new = 0;
      log[trunc_op].n_out = n_out;
    }
    ctrl->n = n_out;
  }
}

}  // namespace ppvm
