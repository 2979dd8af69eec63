// common.cuh — device-side building blocks of the Pauli-propagation engine.
//
// Term storage is structure-of-arrays: for a sum of capacity `cap`, X plane word w of
// term i lives at x[w * cap + i], Z plane likewise, coefficient at c[i].  W = ceil(n/64).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

namespace ppvm {

// Host: sin and cos of a gate angle, recomputed only when the angle's bit pattern changes
// (gate lists repeat a few angles many times).  The values are the libm results either way;
// comparing bits, not values, keeps -0.0 and +0.0 apart, as their sines differ in sign.
struct SinCosMemo {
  uint64_t bits = 0x7FF8DEADBEEF0001ull;  // a NaN pattern no caller passes
  double sn = 0.0, cs = 0.0;
  void get(double theta, double& s, double& c) {
    uint64_t b;
    std::memcpy(&b, &theta, sizeof(b));
    if (b != bits) {
      bits = b;
      sn = std::sin(theta);
      cs = std::cos(theta);
    }
    s = sn;
    c = cs;
  }
};

constexpr int kMaxW = 8;  // up to 512 qubits
constexpr unsigned kFull = 0xffffffffu;

// Error codes written to Ctrl::err by device code (first writer wins).
enum DevErr : int { kOk = 0, kErrCapacity = 1, kErrTimeout = 2, kErrProbe = 3 };

// Per-stream control block in device memory.
struct Ctrl {
  unsigned long long n;        // live terms
  unsigned long long n_s;      // anticommuting terms of the current rotation
  unsigned long long n_pairs;  // partner pairs found among them
  unsigned long long n_side;   // truncation: dropped-but-preserved terms
  unsigned long long tickets[4];
  int err;
  int err_op;
  double sum;                  // result slot of reductions
  unsigned long long umax;     // result slot of max reductions
  unsigned long long cap_needed;
  unsigned long long fb_cut;   // fused-run fallback: gates at the head of the run to apply one at a time, 0 = none
  unsigned long long done;     // blocks of the current launch that finished (last_block_done)
  unsigned long long scr_top;  // fused run in scratch mode: group outputs placed in the scratch so far
  unsigned spin_limit;         // polls a look-back waits before it gives up; 0 = kSpinLimit
  unsigned reserved;
};

// Per-op counters recorded for the term-gate-updates metric and the roofline bytes.
struct OpLog {
  unsigned long long n_in;   // live terms entering the op
  unsigned long long n_s;    // touched terms (anticommuting for rotations)
  unsigned long long n_new;  // children appended (rotations)
  unsigned long long n_out;  // live terms after the op
};

struct Planes {
  uint64_t* x;
  uint64_t* z;
  double* c;
  unsigned long long cap;
};

// A Pauli generator (rotation axis) as X/Z plane masks.  lw: for a lossy sum, the first loss
// word of the X plane (the generator then acts only on qubits that are not lost); 0 otherwise.
struct Gen {
  uint64_t gx[kMaxW];
  uint64_t gz[kMaxW];
  uint32_t lw;
  uint32_t reserved;
};

// ---- memory ordering helpers (decoupled look-back) ----------------------------------
__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_volatile(const unsigned long long* p) {
  return *reinterpret_cast<const volatile unsigned long long*>(p);
}
__device__ __forceinline__ int ld_volatile_int(const int* p) {
  return *reinterpret_cast<const volatile int*>(p);
}

// Waits until the grids this one depends on in its stream have completed and their writes
// are visible.  Kernels of the single-sum engine start with it, so the host may launch them
// with programmatic stream serialization: the launch overlaps the previous kernel's run.
// Without such a launch it returns at once.
__device__ __forceinline__ void pdl_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  // Let the next kernel of the stream be launched now: it is scheduled only once every block
  // of this grid has started, and its blocks wait in their own pdl_wait() for this grid.
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// True (in every thread) in the last block of the grid to call it: by then every block's
// writes made before its call are visible.  Blocks never wait on each other.  The last block
// resets the counter for the next launch; after a device error the host resets it.
__device__ __forceinline__ bool last_block_done(unsigned long long* counter) {
  __shared__ bool s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned long long prev = atomicAdd(counter, 1ull);
    s_last = prev == (unsigned long long)gridDim.x * gridDim.y * gridDim.z - 1;
    if (s_last) *counter = 0;
  }
  __syncthreads();
  if (s_last) __threadfence();
  return s_last;
}

__device__ __forceinline__ void set_err(Ctrl* ctrl, int code, int op) {
  if (atomicCAS(&ctrl->err, 0, code) == 0) ctrl->err_op = op;
}

// ---- decoupled look-back ---------------------------------------------------------------
// Tile state word: [epoch:20][flag:2][value:42].  flag 1 = aggregate, 2 = inclusive prefix.
constexpr int kValueBits = 42;
constexpr unsigned long long kValueMask = (1ull << kValueBits) - 1;
constexpr unsigned kSpinLimit = 1u << 22;

// The poll bound of a look-back: the control block's spin_limit, or kSpinLimit when it is 0.
__device__ __forceinline__ unsigned spin_limit_of(const Ctrl* ctrl) {
  const unsigned v = ctrl->spin_limit;
  return v ? v : kSpinLimit;
}

__device__ __forceinline__ unsigned long long pack_state(unsigned epoch, unsigned flag,
                                                          unsigned long long v) {
  return ((unsigned long long)(epoch & 0xFFFFFu) << 44) | ((unsigned long long)flag << 42) |
         (v & kValueMask);
}

// Exclusive prefix of tile `tile` given its aggregate.  All threads of the block call it;
// warp 0 publishes and looks back.  Every wait is bounded; on timeout the error flag is set
// and a (wrong) prefix is returned so that the kernel ends.  That prefix is the sum of the
// non-negative aggregates read before the wait gave up, never more than the true prefix, so
// every output offset derived from it stays at or below its true value: writes stay inside
// the buffers sized for the true outputs.
static __device__ unsigned long long lookback(unsigned long long* ts, unsigned tile,
                                       unsigned long long agg, unsigned epoch, Ctrl* ctrl,
                                       int op, unsigned long long* s_slot) {
  if (threadIdx.x < 32) {
    const unsigned lane = threadIdx.x;
    unsigned long long excl = 0;
    if (tile == 0) {
      if (lane == 0) st_release(&ts[0], pack_state(epoch, 2, agg));
    } else {
      if (lane == 0) st_release(&ts[tile], pack_state(epoch, 1, agg));
      long long pred = (long long)tile - 1 - (long long)lane;
      unsigned spins = 0;
      const unsigned lim = spin_limit_of(ctrl);
      const unsigned ep = epoch & 0xFFFFFu;
      while (true) {
        unsigned flag;
        unsigned long long val;
        while (true) {
          if (pred >= 0) {
            unsigned long long st = ld_acquire(&ts[pred]);
            flag = ((unsigned)(st >> 44) == ep) ? (unsigned)((st >> 42) & 3ull) : 0u;
            val = st & kValueMask;
          } else {
            flag = 2;
            val = 0;
          }
          if (__all_sync(kFull, flag != 0)) break;
          if (++spins > lim) {
            if (lane == 0) set_err(ctrl, kErrTimeout, op);
            flag = 2;
            val = 0;
            break;
          }
          __nanosleep(64);
        }
        const unsigned pmask = __ballot_sync(kFull, flag == 2);
        const unsigned first = pmask ? (unsigned)(__ffs(pmask) - 1) : 32u;
        unsigned long long contrib = (lane <= first) ? val : 0ull;
#pragma unroll
        for (int o = 16; o; o >>= 1) contrib += __shfl_down_sync(kFull, contrib, o);
        excl += __shfl_sync(kFull, contrib, 0);
        if (pmask) break;
        pred -= 32;
      }
      if (lane == 0) st_release(&ts[tile], pack_state(epoch, 2, excl + agg));
    }
    if (lane == 0) *s_slot = excl;
  }
  __syncthreads();
  unsigned long long r = *s_slot;
  __syncthreads();
  return r;
}

// Exclusive prefix of tile `tile` for a tile owned by one warp (all 32 lanes call it): the
// warp publishes its aggregate, looks back over its predecessors 32 at a time, then
// publishes its inclusive prefix.  Bounded like lookback(); no block barrier.
__device__ __forceinline__ unsigned long long warp_lookback(unsigned long long* ts, unsigned long long tile,
                                                            unsigned long long agg, unsigned epoch, Ctrl* ctrl,
                                                            int op) {
  const unsigned lane = threadIdx.x & 31;
  const unsigned ep = epoch & 0xFFFFFu;
  unsigned long long excl = 0;
  if (tile == 0) {
    if (lane == 0) st_release(&ts[0], pack_state(epoch, 2, agg));
    __syncwarp();
    return 0;
  }
  if (lane == 0) st_release(&ts[tile], pack_state(epoch, 1, agg));
  long long pred = (long long)tile - 1 - (long long)lane;
  unsigned spins = 0;
  const unsigned lim = spin_limit_of(ctrl);
  while (true) {
    unsigned flag;
    unsigned long long val;
    while (true) {
      if (pred >= 0) {
        const unsigned long long st = ld_acquire(&ts[pred]);
        flag = ((unsigned)(st >> 44) == ep) ? (unsigned)((st >> 42) & 3ull) : 0u;
        val = st & kValueMask;
      } else {
        flag = 2;
        val = 0;
      }
      if (__all_sync(kFull, flag != 0)) break;
      if (++spins > lim) {
        if (lane == 0) set_err(ctrl, kErrTimeout, op);
        flag = 2;
        val = 0;
        break;
      }
      __nanosleep(32);
    }
    const unsigned pmask = __ballot_sync(kFull, flag == 2);
    const unsigned first = pmask ? (unsigned)(__ffs(pmask) - 1) : 32u;
    unsigned long long contrib = (lane <= first) ? val : 0ull;
#pragma unroll
    for (int o = 16; o; o >>= 1) contrib += __shfl_down_sync(kFull, contrib, o);
    excl += __shfl_sync(kFull, contrib, 0);
    if (pmask) break;
    pred -= 32;
  }
  if (lane == 0) st_release(&ts[tile], pack_state(epoch, 2, excl + agg));
  __syncwarp();
  return excl;
}

// Takes the next tile ticket (all threads get the same value).
__device__ __forceinline__ unsigned next_tile(unsigned long long* counter, unsigned* s_tile) {
  if (threadIdx.x == 0) *s_tile = (unsigned)atomicAdd(counter, 1ull);
  __syncthreads();
  unsigned t = *s_tile;
  __syncthreads();
  return t;
}

// Block-wide ordered ranks for a [ITEMS][BLOCK] tile of flags in index order
// i = k*BLOCK + tid.  ballots[k] holds the warp ballot of item k.  Writes per-(k,warp)
// exclusive bases into s_base and returns the tile aggregate (all threads).
template <int BLOCK, int ITEMS>
__device__ unsigned tile_ranks(const unsigned (&ballots)[ITEMS], unsigned* s_base) {
  constexpr int NW = BLOCK / 32;
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) s_base[k * NW + warp] = __popc(ballots[k]);
  }
  __syncthreads();
  constexpr int M = ITEMS * NW;  // <= 64 entries, scanned by warp 0
  if (threadIdx.x < 32) {
    constexpr int PER = (M + 31) / 32;
    unsigned v[PER];
    unsigned local = 0;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      int idx = lane * PER + j;
      v[j] = idx < M ? s_base[idx] : 0u;
      local += v[j];
    }
    unsigned incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      unsigned t = __shfl_up_sync(kFull, incl, o);
      if (lane >= (unsigned)o) incl += t;
    }
    unsigned run = incl - local;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      int idx = lane * PER + j;
      if (idx < M) s_base[idx] = run;
      run += v[j];
    }
    if (lane == 31) s_base[M] = incl;
  }
  __syncthreads();
  unsigned total = s_base[M];
  return total;
}

// ---- Pauli arithmetic --------------------------------------------------------------------
__device__ __forceinline__ uint64_t mix64(uint64_t v) {
  v ^= v >> 30;
  v *= 0xbf58476d1ce4e5b9ull;
  v ^= v >> 27;
  v *= 0x94d049bb133111ebull;
  v ^= v >> 31;
  return v;
}

template <int W>
__device__ __forceinline__ uint64_t hash_key(const uint64_t (&x)[W], const uint64_t (&z)[W]) {
  uint64_t h = 0x9E3779B97F4A7C15ull;
#pragma unroll
  for (int w = 0; w < W; ++w) h = mix64(h ^ x[w]) + 0x632BE59BD9B4E019ull;
#pragma unroll
  for (int w = 0; w < W; ++w) h = mix64(h ^ z[w]) + 0x632BE59BD9B4E019ull;
  return h;
}

template <int W>
__device__ __forceinline__ bool anticommutes(const Gen& g, const uint64_t (&x)[W],
                                             const uint64_t (&z)[W]) {
  uint64_t acc = 0;
#pragma unroll
  for (int w = 0; w < W; ++w) acc ^= (x[w] & g.gz[w]) ^ (z[w] & g.gx[w]);
  return __popcll(acc) & 1;
}

// Sign s in {+1,-1} with i*G*P = s * (G xor P) for anticommuting P: G*P = i^e (G xor P),
// e = sum over qubits of the single-qubit product phase (X*Y=iZ, Y*Z=iX, Z*X=iY and
// the reverse products with -i).  Returns -1 when (e + 1) = 2 mod 4.
template <int W>
__device__ __forceinline__ double rot_sign(const Gen& g, const uint64_t (&x)[W],
                                           const uint64_t (&z)[W]) {
  int e = 0;
#pragma unroll
  for (int w = 0; w < W; ++w) {
    const uint64_t x1 = g.gx[w], z1 = g.gz[w], x2 = x[w], z2 = z[w];
    const uint64_t gX = x1 & ~z1, gY = x1 & z1, gZ = ~x1 & z1;
    const uint64_t pX = x2 & ~z2, pY = x2 & z2, pZ = ~x2 & z2;
    e += __popcll(gX & pY) - __popcll(gX & pZ);
    e += __popcll(gY & pZ) - __popcll(gY & pX);
    e += __popcll(gZ & pX) - __popcll(gZ & pY);
  }
  return (((e + 1) & 3) == 0) ? 1.0 : -1.0;
}

template <int W>
__device__ __forceinline__ unsigned weight(const uint64_t (&x)[W], const uint64_t (&z)[W]) {
  unsigned t = 0;
#pragma unroll
  for (int w = 0; w < W; ++w) t += __popcll(x[w] | z[w]);
  return t;
}

// Lexicographic "a < b" over (x words high..low, z words high..low).
template <int W>
__device__ __forceinline__ bool key_less(const uint64_t (&ax)[W], const uint64_t (&az)[W],
                                         const uint64_t (&bx)[W], const uint64_t (&bz)[W]) {
#pragma unroll
  for (int w = W - 1; w >= 0; --w)
    if (ax[w] != bx[w]) return ax[w] < bx[w];
#pragma unroll
  for (int w = W - 1; w >= 0; --w)
    if (az[w] != bz[w]) return az[w] < bz[w];
  return false;
}

// ---- epoch-tagged open-addressing slots: [epoch:16][tag:16][index:32] -----------------------
__device__ __forceinline__ unsigned long long make_slot(unsigned epoch, unsigned tag, unsigned idx) {
  return ((unsigned long long)(epoch & 0xFFFFu) << 48) | ((unsigned long long)(tag & 0xFFFFu) << 32) |
         (unsigned long long)idx;
}
__device__ __forceinline__ unsigned slot_epoch(unsigned long long s) { return (unsigned)(s >> 48); }
__device__ __forceinline__ unsigned slot_tag(unsigned long long s) { return (unsigned)(s >> 32) & 0xFFFFu; }
__device__ __forceinline__ unsigned slot_idx(unsigned long long s) { return (unsigned)s; }

__device__ __forceinline__ unsigned long long next_pow2_ull(unsigned long long v) {
  unsigned long long p = 1;
  while (p < v) p <<= 1;
  return p;
}

}  // namespace ppvm
