// engine.cu — host side of the C ABI declared in include/ppvm_cuda.h.
//
// A ppvm_sum owns SoA term planes on one device plus the scratch the rotation pipeline
// needs, and one CUDA stream.  Each API call lowers its gates to a list of ops, enqueues
// the kernels of kernels.cuh for the whole list without host round trips (every kernel
// reads live counts from the device control block), then synchronises once and checks the
// device error word.  A rotation that would overflow the term capacity stops before it
// modifies anything; the call then grows the storage and replays from that op.

#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <set>
#include <unordered_map>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ppvm_cuda.h"
#include "runs.cuh"
#include "tableau.cuh"
#include "budget.cuh"
#include "loss.cuh"
#include "noise.cuh"
#include "shard.cuh"

using namespace ppvm;

namespace {

thread_local std::string g_err;

ppvm_status fail(ppvm_status s, const std::string& msg) {
  g_err = msg;
  return s;
}

#define CUDA_TRY(expr)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (expr);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(e_ == cudaErrorMemoryAllocation ? PPVM_ECAPACITY : PPVM_ECUDA,         \
                  std::string(#expr) + ": " + cudaGetErrorString(e_));                   \
  } while (0)

// Calls that read a sum's terms refuse a sum that an earlier failure left unusable (its
// planes and live count may be partial): they return the same status as the ops do.
#define REQUIRE_USABLE(s)                                                                \
  do {                                                                                   \
    if ((s)->poisoned) return fail(PPVM_ECUDA, "sum is in an error state from an earlier failure"); \
  } while (0)

#define PPVM_TRY(expr)                  \
  do {                                  \
    ppvm_status s_ = (expr);            \
    if (s_ != PPVM_OK) return s_;       \
  } while (0)

constexpr int kScanBlock = 256;
constexpr int kPairBlock = 256;
constexpr int kRedBlock = 256;
constexpr int kMaxPreserve = 1023;
const double kHalfPi = 1.5707963267948966;

// host mirror of the device hash (common.cuh) for the preserve-set table
uint64_t h_mix64(uint64_t v) {
  v ^= v >> 30;
  v *= 0xbf58476d1ce4e5b9ull;
  v ^= v >> 27;
  v *= 0x94d049bb133111ebull;
  v ^= v >> 31;
  return v;
}
uint64_t h_hash_key(const uint64_t* x, const uint64_t* z, int W) {
  uint64_t h = 0x9E3779B97F4A7C15ull;
  for (int w = 0; w < W; ++w) h = h_mix64(h ^ x[w]) + 0x632BE59BD9B4E019ull;
  for (int w = 0; w < W; ++w) h = h_mix64(h ^ z[w]) + 0x632BE59BD9B4E019ull;
  return h;
}

int g_sm_count = 0;

struct ProfLaunch {
  int family;
  int op;
  int nops;  // ops covered (Clifford runs)
  int aux;   // fused TRUNCATE op of a tableau pass, else -1
  uint64_t bytes;  // algorithmic bytes of a launch outside the op list (op < 0), else unused
  cudaEvent_t a, b;
};

enum Family {
  F_SCAN = 0, F_PAIR, F_APPLY, F_COMMIT, F_CLIFF, F_TRUNC, F_READ,
  F_RUN_CLASSIFY, F_RUN_ORDER, F_RUN_SCATTER, F_RUN_GROUPS, F_RUN_PLACE, F_TABLEAU, F_LOSS, F_COUNT
};
const char* kFamilyNames[F_COUNT] = {"rot_scan", "rot_pair", "rot_apply", "rot_commit",
                                     "clifford", "truncate", "readout",
                                     "run_classify", "run_order", "run_scatter", "run_groups", "run_place",
                                     "tableau", "loss"};

// One pinned host chunk and its device twin: per-call uploads (op descriptors, run
// descriptors, tableaux) are packed here and copied with truly asynchronous copies.
struct StageChunk {
  uint8_t* h = nullptr;
  uint8_t* d = nullptr;
  size_t cap = 0;
  size_t used = 0;
};

}  // namespace

namespace ppvm {
// Lets other translation units of the library set the text of ppvm_last_error_string().
void set_last_error(const std::string& msg) { g_err = msg; }
// The term-priority network's device weights and device (learned.cu).
const MlpWeights* mlp_device_weights(const ppvm_mlp* m);
int mlp_device(const ppvm_mlp* m);
}  // namespace ppvm

struct ppvm_sum {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  uint32_t n = 0;
  int W = 1;                   // words per plane (a lossy sum: 2 * wr, the loss bits in X's upper half)
  int wr = 1;                  // words of the qubits' X/Z bits: ceil(n/64)
  bool lossy = false;          // PPVM_FLAG_LOSSY
  double thr = 1e-10;
  uint64_t maxw = UINT64_MAX;
  uint64_t maxlw = UINT64_MAX;  // MaxLossWeight of a lossy sum's strategy
  uint32_t flags = 0;
  unsigned long long cap = 0;
  unsigned long long n_host = 0;  // live count at the last synchronisation
  unsigned long long n_ub = 0;    // upper bound of the live count (sizes grids)

  uint64_t* planes = nullptr;  // x[W*cap] z[W*cap] c[cap]
  uint64_t* alt = nullptr;     // second plane buffer: fused runs write here, then swap
  uint64_t* scr = nullptr;     // fused runs in scratch mode: group outputs before placement (cap terms)
  RunScratch R = {};
  unsigned long long* tstate2 = nullptr;
  std::vector<int> swaps;      // op indices of fused runs enqueued in the current attempt
  std::map<size_t, int> run_cap;   // run start -> most gates a fused run there may take; -L: L gates per gate
  std::map<size_t, int> run_len;   // run start -> gates of the fused run enqueued there (this attempt)
  uint32_t* s_idx = nullptr;
  uint64_t* s_rec = nullptr;
  uint32_t* partner = nullptr;
  unsigned long long* table = nullptr;
  unsigned long long table_cap = 0;
  unsigned long long run_slots_used = 0;  // group-table slots the fused runs since the last clean state hashed into
  unsigned long long* tstate = nullptr;
  unsigned long long tstate_cap = 0;
  unsigned long long scr_cap = 0;  // capacity scr was allocated for
  uint64_t* side = nullptr;
  Ctrl* d_ctrl = nullptr;
  Ctrl* h_ctrl = nullptr;
  OpLog* d_log = nullptr;
  OpLog* h_log = nullptr;
  size_t log_cap = 0;
  size_t last_nops = 0;
  PatItem* d_pat = nullptr;
  double* d_partials = nullptr;
  unsigned long long* d_counter = nullptr;
  SelState* d_sel = nullptr;   // radix select state of budget truncation
  unsigned* d_hist = nullptr;  // its digit histogram (2^11 bins, kept zero between uses)
  uint64_t* d_pres_keys = nullptr;
  std::vector<double> perr2_host;    // factor tables of the internal two-qubit Pauli error ops
  const double* d_perr2 = nullptr;   // their staged copy for the current attempt
  int* d_pres_table = nullptr;
  unsigned pres_mask = 0;
  int npres = 0;
  std::vector<uint64_t> h_pres;

  unsigned tile_epoch = 0;
  unsigned table_epoch = 0;
  bool poisoned = false;

  std::vector<StageChunk> stage;  // upload arena, reset at the start of every submission
  size_t stage_cur = 0;
  unsigned long long xfer_h2d = 0, xfer_d2h = 0;  // bytes copied host<->device since creation
  unsigned long long launch_count = 0;            // kernels launched since creation

  bool prof = false;
  std::vector<ProfLaunch> prof_pending;
  std::vector<cudaEvent_t> event_pool;  // reused profiling events
  double prof_ms[F_COUNT] = {};
  uint64_t prof_launches[F_COUNT] = {};
  uint64_t prof_bytes[F_COUNT] = {};

  Planes view_of(uint64_t* base) const {
    Planes p;
    p.x = base;
    p.z = base + (size_t)W * cap;
    p.c = reinterpret_cast<double*>(base + (size_t)2 * W * cap);
    p.cap = cap;
    return p;
  }
  Planes planes_view() const { return view_of(planes); }
  Planes alt_view() const { return view_of(alt); }
  unsigned next_tile_epoch() {
    if (++tile_epoch >= 0xFFFFFu) {
      cudaMemsetAsync(tstate, 0, tstate_cap * sizeof(unsigned long long), stream);
      cudaMemsetAsync(tstate2, 0, tstate_cap * sizeof(unsigned long long), stream);
      tile_epoch = 1;
    }
    return tile_epoch;
  }
  unsigned next_table_epoch() {
    if (++table_epoch >= 0xFFFFu) {
      cudaMemsetAsync(table, 0, table_cap * sizeof(unsigned long long), stream);
      table_epoch = 1;
    }
    return table_epoch;
  }
};

namespace {

// ---- caching pool for the large per-sum buffers -----------------------------------------------
// Term planes and scratch are taken from, and given back to, a per-device free list instead of
// cudaMalloc/cudaFree on every sum: creating sums of the same size again (a user's loop over
// circuits, the term-budget runs of learned truncation) then allocates nothing and does not
// synchronise the device.  Buffers are handed back only when their sum's stream is idle.
// ppvm_release_cached_memory() returns the cached memory to the driver.
std::mutex g_pool_mu;
std::multimap<size_t, void*> g_pool_free[64];
std::unordered_map<void*, std::pair<int, size_t>> g_pool_live;

void pool_release_device(int dev) {  // caller holds g_pool_mu; dev is current
  for (auto& kv : g_pool_free[dev]) cudaFree(kv.second);
  g_pool_free[dev].clear();
}

// Where a pool allocation is made, for the allocation-failure test hook below.
enum AllocSite : unsigned { kAllocCreate = 0, kAllocGrowth = 1, kAllocRunScratch = 2 };

// Test hook: PPVM_TEST_FAIL_ALLOC names allocation sites ("growth": storage growth of a live
// sum; "run-scratch": the fused runs' scratch planes; comma-separated) whose pool
// allocations fail as if the device had no memory left, without calling cudaMalloc.  Read
// once per process; the failure-handling tests set it in a child process.
bool alloc_fails(AllocSite site) {
  static const unsigned mask = [] {
    unsigned m = 0;
    const char* e = std::getenv("PPVM_TEST_FAIL_ALLOC");
    if (e) {
      const std::string v(e);
      if (v.find("growth") != std::string::npos) m |= 1u << kAllocGrowth;
      if (v.find("run-scratch") != std::string::npos) m |= 1u << kAllocRunScratch;
    }
    return m;
  }();
  return (mask >> site) & 1u;
}

cudaError_t pool_malloc(void** out, size_t bytes, AllocSite site = kAllocCreate) {
  if (alloc_fails(site)) return cudaErrorMemoryAllocation;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaMalloc(out, bytes);
  const size_t want = (bytes + ((1u << 20) - 1)) & ~(size_t)((1u << 20) - 1);  // 1 MiB granules
  std::lock_guard<std::mutex> lk(g_pool_mu);
  auto it = g_pool_free[dev].lower_bound(want);
  if (it != g_pool_free[dev].end() && it->first <= want + want / 2) {
    *out = it->second;
    g_pool_live[it->second] = {dev, it->first};
    g_pool_free[dev].erase(it);
    return cudaSuccess;
  }
  e = cudaMalloc(out, want);
  if (e == cudaErrorMemoryAllocation) {  // give the cache back and try once more
    cudaGetLastError();
    pool_release_device(dev);
    e = cudaMalloc(out, want);
  }
  if (e == cudaSuccess) g_pool_live[*out] = {dev, want};
  return e;
}

void pool_free(void* p) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  auto it = g_pool_live.find(p);
  if (it == g_pool_live.end()) {
    cudaFree(p);
    return;
  }
  g_pool_free[it->second.first].emplace(it->second.second, p);
  g_pool_live.erase(it);
}

void destroy_now(ppvm_sum* s);                 // frees a sum and everything it holds
ppvm_sum* take_cached(int device, int W);      // a cached sum of that device and width, or null

// Fused runs with at least this many groups take scratch mode (k_run_place).  Below it the
// per-group look-back is cheaper than the extra placement pass.  PPVM_RUN_SCRATCH_MIN_GROUPS
// overrides it (the tests set it low, so that small sums take the scratch path too).
unsigned long long run_scratch_min_groups() {
  static const unsigned long long v = [] {
    const char* e = std::getenv("PPVM_RUN_SCRATCH_MIN_GROUPS");
    if (e && *e) {
      char* end = nullptr;
      const unsigned long long x = std::strtoull(e, &end, 10);
      if (end && *end == 0) return std::max<unsigned long long>(x, 1);
    }
    return 1ull << 18;
  }();
  return v;
}

// The group mode of k_run_groups: 0 chosen per run (many single-member groups: one group per
// lane; otherwise one group per warp), 1 tiles of groups per block, 2 one group per warp, 3 one
// group per lane.  PPVM_RUN_GROUP_MODE=tiled|warp|lanes forces one; the tests run the
// fused-run cases in each.
unsigned run_tile_mode() {
  static const unsigned v = [] {
    const char* e = std::getenv("PPVM_RUN_GROUP_MODE");
    if (e && std::strcmp(e, "tiled") == 0) return 1u;
    if (e && std::strcmp(e, "warp") == 0) return 2u;
    if (e && std::strcmp(e, "lanes") == 0) return 3u;
    return 0u;
  }();
  return v;
}

// Chunk tables of the composed Clifford pass (one-word sums): 0 = by size and moved
// generators, 1 = always (every warp with a moved bit takes them), 2 = never.
// PPVM_TABLEAU_CHUNKS=always|never forces one; the tests run the tableau cases in each.
unsigned tableau_chunk_mode() {
  static const unsigned v = [] {
    const char* e = std::getenv("PPVM_TABLEAU_CHUNKS");
    if (e && std::strcmp(e, "always") == 0) return 1u;
    if (e && std::strcmp(e, "never") == 0) return 2u;
    return 0u;
  }();
  return v;
}

// Polls a look-back waits for its predecessors before it gives up with PPVM_ETIMEOUT.  0 (the
// default) leaves the device's bound of 2^22 polls; PPVM_SPIN_LIMIT overrides it, read once
// per process (the timeout test sets a few polls, so that a multi-tile look-back gives up).
unsigned spin_limit_setting() {
  static const unsigned v = [] {
    const char* e = std::getenv("PPVM_SPIN_LIMIT");
    if (e && *e) {
      char* end = nullptr;
      const unsigned long long x = std::strtoull(e, &end, 10);
      if (end && *end == 0) return (unsigned)std::min<unsigned long long>(x, 0xFFFFFFFFull);
    }
    return 0u;
  }();
  return v;
}

// The control block of a new or reused sum: all zero but the look-back poll bound.
ppvm_status init_ctrl(ppvm_sum* s, unsigned long long n) {
  std::memset(s->h_ctrl, 0, sizeof(Ctrl));
  s->h_ctrl->n = n;
  s->h_ctrl->spin_limit = spin_limit_setting();
  CUDA_TRY(cudaMemcpyAsync(s->d_ctrl, s->h_ctrl, sizeof(Ctrl), cudaMemcpyHostToDevice, s->stream));
  return PPVM_OK;
}

unsigned long long next_pow2(unsigned long long v) {
  unsigned long long p = 1;
  while (p < v) p <<= 1;
  return p;
}

ppvm_status ensure_device(int dev) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0)
    return fail(PPVM_ENODEV, std::string("no CUDA device: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= count) return fail(PPVM_EINVAL, "device ordinal out of range");
  CUDA_TRY(cudaSetDevice(dev));
  if (g_sm_count == 0) CUDA_TRY(cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev));
  return PPVM_OK;
}

// Words handed in by a caller: bits at or above n_qubits clear; on a lossy sum the Z plane's
// upper words clear and a lost qubit without X or Z bits (it is L, not X, Y or Z).
ppvm_status check_words(const ppvm_sum* s, const uint64_t* x, const uint64_t* z, size_t k) {
  const int W = s->W, wr = s->wr;
  const int tail = (int)(s->n % 64);
  const uint64_t top = tail ? ~((1ull << tail) - 1) : 0ull;
  for (size_t i = 0; i < k; ++i) {
    const uint64_t* xi = x + i * W;
    const uint64_t* zi = z + i * W;
    if ((xi[wr - 1] | zi[wr - 1]) & top) return fail(PPVM_EINVAL, "word has bits set at or above n_qubits");
    if (!s->lossy) continue;
    if (xi[W - 1] & top) return fail(PPVM_EINVAL, "word has loss bits set at or above n_qubits");
    for (int w = 0; w < wr; ++w) {
      if (zi[wr + w]) return fail(PPVM_EINVAL, "a lossy word's Z plane has bits in its loss half");
      if (xi[wr + w] & (xi[w] | zi[w]))
        return fail(PPVM_EINVAL, "a lost qubit cannot also carry X or Z (LossyPauliWord::get panics)");
    }
  }
  return PPVM_OK;
}

void free_scratch(ppvm_sum* s) {
  pool_free(s->alt);
  pool_free(s->scr);
  s->scr = nullptr;
  pool_free(s->tstate2);
  uint32_t* run_arrays[] = {s->R.gslot, s->R.grp_min, s->R.grp_cnt, s->R.grp_ord, s->R.g_start,
                            s->R.g_cnt, s->R.g_rep, s->R.g_fill, s->R.mcoord};
  for (uint32_t* p : run_arrays) pool_free(p);
  pool_free(s->R.created);
  s->R = RunScratch{};
  s->alt = nullptr;
  s->tstate2 = nullptr;
  pool_free(s->s_idx);
  pool_free(s->s_rec);
  pool_free(s->partner);
  pool_free(s->table);
  pool_free(s->tstate);
  s->s_idx = nullptr;
  s->s_rec = nullptr;
  s->partner = nullptr;
  s->table = nullptr;
  s->tstate = nullptr;
}

// The fused-run group tables in their clean state (grp_min all ones, counts zero) over their
// first `slots` entries: the whole table after allocation, and after a failed attempt only
// the part its runs hashed into (a handle's table can be far larger than the sum it holds).
ppvm_status clear_run_tables(ppvm_sum* s, unsigned long long slots) {
  slots = std::min<unsigned long long>(slots, s->table_cap);
  if (slots) {
    CUDA_TRY(cudaMemsetAsync(s->R.grp_min, 0xFF, sizeof(uint32_t) * slots, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->R.grp_cnt, 0, sizeof(uint32_t) * slots, s->stream));
  }
  CUDA_TRY(cudaMemsetAsync(s->R.created, 0, sizeof(unsigned long long) * kRunMaxGates, s->stream));
  s->run_slots_used = 0;
  return PPVM_OK;
}

// (Re)allocates term storage of capacity new_cap, keeping the first n_host terms.
ppvm_status grow(ppvm_sum* s, unsigned long long new_cap) {
  if (new_cap >= 0xFFFFFFF0ull) return fail(PPVM_ECAPACITY, "term capacity limit (2^32) exceeded");
  const int W = s->W;
  const AllocSite site = s->planes ? kAllocGrowth : kAllocCreate;
  uint64_t* np = nullptr;
  CUDA_TRY(pool_malloc((void**)&np, sizeof(uint64_t) * (size_t)(2 * W + 1) * new_cap, site));
  if (s->planes) {
    for (int w = 0; w < 2 * W + 1; ++w)
      CUDA_TRY(cudaMemcpyAsync(np + (size_t)w * new_cap, s->planes + (size_t)w * s->cap,
                               sizeof(uint64_t) * s->n_host, cudaMemcpyDeviceToDevice, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    pool_free(s->planes);
  }
  s->planes = np;
  s->cap = new_cap;
  free_scratch(s);
  CUDA_TRY(pool_malloc((void**)&s->s_idx, sizeof(uint32_t) * new_cap, site));
  CUDA_TRY(pool_malloc((void**)&s->partner, sizeof(uint32_t) * new_cap, site));
  CUDA_TRY(pool_malloc((void**)&s->s_rec, sizeof(uint64_t) * (size_t)(2 * W + 1) * new_cap, site));
  s->table_cap = next_pow2(std::max<unsigned long long>(2 * new_cap, 1024));
  CUDA_TRY(pool_malloc((void**)&s->table, sizeof(unsigned long long) * s->table_cap, site));
  CUDA_TRY(cudaMemsetAsync(s->table, 0, sizeof(unsigned long long) * s->table_cap, s->stream));
  s->table_epoch = 0;
  // one tile-state word per look-back tile: the smallest tile is k_run_groups' kRunWarps groups
  s->tstate_cap = new_cap + 64;  // one tile-state word per group of a fused run at most
  CUDA_TRY(pool_malloc((void**)&s->tstate, sizeof(unsigned long long) * s->tstate_cap, site));
  CUDA_TRY(cudaMemsetAsync(s->tstate, 0, sizeof(unsigned long long) * s->tstate_cap, s->stream));
  CUDA_TRY(pool_malloc((void**)&s->tstate2, sizeof(unsigned long long) * s->tstate_cap, site));
  CUDA_TRY(cudaMemsetAsync(s->tstate2, 0, sizeof(unsigned long long) * s->tstate_cap, s->stream));
  s->tile_epoch = 0;
  CUDA_TRY(pool_malloc((void**)&s->alt, sizeof(uint64_t) * (size_t)(2 * W + 1) * new_cap, site));
  CUDA_TRY(pool_malloc((void**)&s->R.gslot, sizeof(uint32_t) * new_cap, site));
  CUDA_TRY(pool_malloc((void**)&s->R.grp_min, sizeof(uint32_t) * s->table_cap, site));
  CUDA_TRY(pool_malloc((void**)&s->R.grp_cnt, sizeof(uint32_t) * s->table_cap, site));
  CUDA_TRY(pool_malloc((void**)&s->R.grp_ord, sizeof(uint32_t) * s->table_cap, site));
  CUDA_TRY(pool_malloc((void**)&s->R.g_start, sizeof(uint32_t) * new_cap, site));
  CUDA_TRY(pool_malloc((void**)&s->R.g_cnt, sizeof(uint32_t) * new_cap, site));
  CUDA_TRY(pool_malloc((void**)&s->R.g_rep, sizeof(uint32_t) * new_cap, site));
  CUDA_TRY(pool_malloc((void**)&s->R.g_fill, sizeof(uint32_t) * new_cap, site));
  CUDA_TRY(pool_malloc((void**)&s->R.mcoord, sizeof(uint32_t) * new_cap, site));
  // member coefficients and group keys live in the rotation records, unused during a run
  s->R.mcoef = reinterpret_cast<double*>(s->s_rec);
  s->R.gkey = s->s_rec + new_cap;  // 2W words per group, at most new_cap groups
  CUDA_TRY(pool_malloc((void**)&s->R.created, sizeof(unsigned long long) * kRunMaxGates, site));
  return clear_run_tables(s, s->table_cap);
}

ppvm_status ensure_log(ppvm_sum* s, size_t nops) {
  if (nops <= s->log_cap) return PPVM_OK;
  size_t cap = std::max<size_t>(nops, 2 * s->log_cap);
  cudaFree(s->d_log);
  cudaFreeHost(s->h_log);
  s->d_log = nullptr;
  s->h_log = nullptr;
  CUDA_TRY(cudaMalloc(&s->d_log, sizeof(OpLog) * cap));
  CUDA_TRY(cudaMallocHost(&s->h_log, sizeof(OpLog) * cap));
  s->log_cap = cap;
  return PPVM_OK;
}

// Copies `bytes` from src into the upload arena and enqueues its copy to the device on the
// sum's stream; *dptr receives the device address.  The arena's contents stay valid until the
// next stage_reset, which callers issue only after the stream has been synchronised.
ppvm_status stage_put(ppvm_sum* s, const void* src, size_t bytes, const void** dptr) {
  const size_t need = std::max<size_t>((bytes + 255) & ~size_t(255), 256);
  while (s->stage_cur < s->stage.size() && s->stage[s->stage_cur].cap - s->stage[s->stage_cur].used < need)
    ++s->stage_cur;
  if (s->stage_cur == s->stage.size()) {
    StageChunk ch;
    ch.cap = std::max<size_t>(need, (size_t)1 << 20);
    CUDA_TRY(cudaMallocHost(&ch.h, ch.cap));
    if (cudaMalloc(&ch.d, ch.cap) != cudaSuccess) {
      cudaFreeHost(ch.h);
      return fail(PPVM_ECAPACITY, "device allocation of the upload arena failed");
    }
    s->stage.push_back(ch);
  }
  StageChunk& ch = s->stage[s->stage_cur];
  std::memcpy(ch.h + ch.used, src, bytes);
  CUDA_TRY(cudaMemcpyAsync(ch.d + ch.used, ch.h + ch.used, bytes, cudaMemcpyHostToDevice, s->stream));
  *dptr = ch.d + ch.used;
  ch.used += need;
  s->xfer_h2d += bytes;
  return PPVM_OK;
}

void stage_reset(ppvm_sum* s) {
  for (auto& ch : s->stage) ch.used = 0;
  s->stage_cur = 0;
}

// Kernel launch with programmatic stream serialization: the kernel may be launched while
// the previous kernel of the stream finishes, and waits for it in pdl_wait() (every kernel
// launched this way starts with it).  PPVM_PDL=0 in the environment turns it off.
bool pdl_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("PPVM_PDL");
    return !(e && e[0] == '0');
  }();
  return on;
}

template <typename... KArgs, typename... Args>
void launch(void (*kern)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t st, Args... args) {
  if (!pdl_enabled()) {
    kern<<<grid, block, smem, st>>>(args...);
    return;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kern, args...);
}

unsigned grid_for(unsigned long long work, unsigned long long per_block, int max_per_sm) {
  unsigned long long g = (work + per_block - 1) / per_block;
  const unsigned long long cap = (unsigned long long)g_sm_count * max_per_sm;
  if (g > cap) g = cap;
  if (g == 0) g = 1;
  return (unsigned)g;
}

// ---- profiling ------------------------------------------------------------------------------
struct ProfScope {
  ppvm_sum* s;
  ProfLaunch L;
  bool on;
  ProfScope(ppvm_sum* sum, int family, int op, int nops, int aux = -1) : s(sum), on(sum->prof) {
    ++s->launch_count;
    if (!on) return;
    L.family = family;
    L.op = op;
    L.nops = nops;
    L.aux = aux;
    L.bytes = 0;
    L.a = take();
    L.b = take();
    cudaEventRecord(L.a, s->stream);
  }
  ~ProfScope() {
    if (!on) return;
    cudaEventRecord(L.b, s->stream);
    s->prof_pending.push_back(L);
  }
  cudaEvent_t take() {
    if (s->event_pool.empty()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      return e;
    }
    cudaEvent_t e = s->event_pool.back();
    s->event_pool.pop_back();
    return e;
  }
};

// Algorithmic bytes of one launch, from the op log: the bytes the launch must move at least
// (B = 16W + 8 per term: X and Z planes and the coefficient), the numerator of its roofline.
uint64_t launch_bytes(const ppvm_sum* s, const ProfLaunch& L, const std::vector<int>& test_words) {
  const uint64_t B = 16ull * s->W + 8;
  const OpLog& g = s->h_log[L.op];
  switch (L.family) {
    case F_SCAN: {
      const int tw = (L.op < (int)test_words.size()) ? test_words[L.op] : 1;
      return g.n_in * 8ull * tw + g.n_s * (B + B + 8);  // test words + gather + record/idx/partner
    }
    case F_PAIR: return g.n_s * B * 2;                 // own record + partner record
    case F_APPLY: return g.n_s * (B + 8) + g.n_new * B;  // records, coeff writes, children
    case F_CLIFF: return 2ull * g.n_in * B;
    case F_TRUNC: return g.n_in * B + g.n_out * B;
    case F_RUN_CLASSIFY: return g.n_in * B + g.n_in * 4;       // every term read once, group slots
    case F_TABLEAU: {  // every term read once, survivors written once
      const uint64_t out = L.aux >= 0 ? s->h_log[L.aux].n_out : g.n_in;
      return g.n_in * B + out * B;
    }
    case F_RUN_GROUPS: {                                       // members read, group outputs written
      const OpLog& last = s->h_log[L.op + std::max(L.nops, 1) - 1];
      return (g.n_s & ~kRunLogScratchBit) * B + (L.nops > 1 ? last.n_s : 0) * B;
    }
    case F_LOSS: return g.n_in * B + g.n_out * B;  // every term read once, every output written once
    case F_RUN_PLACE: {  // scratch mode: group outputs read from the scratch, written to their place
      if (!(g.n_s & kRunLogScratchBit)) return 0;  // look-back mode: the kernel returned at once
      const OpLog& last = s->h_log[L.op + std::max(L.nops, 1) - 1];
      return 2ull * (L.nops > 1 ? last.n_s : 0) * B;
    }
    default: return 0;
  }
}

void prof_collect(ppvm_sum* s, const std::vector<int>& test_words) {
  for (auto& L : s->prof_pending) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, L.a, L.b);
    s->prof_ms[L.family] += ms;
    s->prof_launches[L.family] += 1;
    if (L.op >= 0 && (size_t)L.op < s->log_cap) s->prof_bytes[L.family] += launch_bytes(s, L, test_words);
    else if (L.op < 0) s->prof_bytes[L.family] += L.bytes;
    s->event_pool.push_back(L.a);
    s->event_pool.push_back(L.b);
  }
  s->prof_pending.clear();
}

// ---- op lowering ----------------------------------------------------------------------------
// Internal op code, never accepted in a public gate list: TwoQubitPauliError on (q0, q1) with
// the factor table at perr2_host[16 * theta]; made only by ppvm_two_qubit_pauli_error.
constexpr uint32_t kOpPauliError2 = 0x100;

bool is_clifford_angle(const ppvm_sum* s, double th) {
  return (s->flags & PPVM_FLAG_CLIFFORD_ANGLES) && (th == kHalfPi || th == -kHalfPi);
}

// Whether op runs in the fused elementwise pass.
bool is_local(const ppvm_sum* s, const ppvm_op& op) {
  switch (op.code) {
    case PPVM_OP_RX: case PPVM_OP_RY: case PPVM_OP_RZ:
    case PPVM_OP_RXX: case PPVM_OP_RYY: case PPVM_OP_RZZ:
      return is_clifford_angle(s, op.theta);
    case PPVM_OP_TRUNCATE: case PPVM_OP_AMPLITUDE_DAMPING: return false;
    case PPVM_OP_LOSS_CHANNEL: case PPVM_OP_RESET_LOSS_CHANNEL: case PPVM_OP_CORRELATED_LOSS_CHANNEL: return false;
    case kOpPauliError2: return true;
    default: return op.code < PPVM_OP_COUNT_;
  }
}

ppvm_status validate(const ppvm_sum* s, const ppvm_op& op) {
  if (op.code >= PPVM_OP_COUNT_) return fail(PPVM_EINVAL, "unknown op code");
  if (op.code == PPVM_OP_TRUNCATE) return PPVM_OK;
  if (op.q0 >= s->n) return fail(PPVM_EINVAL, "qubit index out of range");
  const bool loss_op = op.code == PPVM_OP_LOSS_CHANNEL || op.code == PPVM_OP_RESET_LOSS_CHANNEL ||
                       op.code == PPVM_OP_CORRELATED_LOSS_CHANNEL;
  if (loss_op && !s->lossy) return fail(PPVM_EINVAL, "loss channels need a lossy sum (PPVM_FLAG_LOSSY)");
  const bool two = op.code == PPVM_OP_CNOT || op.code == PPVM_OP_CZ || op.code == PPVM_OP_CY ||
                   op.code == PPVM_OP_RXX || op.code == PPVM_OP_RYY || op.code == PPVM_OP_RZZ ||
                   op.code == PPVM_OP_DEPOLARIZE2 || op.code == PPVM_OP_CORRELATED_LOSS_CHANNEL;
  if (two && (op.q1 >= s->n || op.q1 == op.q0))
    return fail(PPVM_EINVAL, "two-qubit op needs two distinct qubits in range");
  return PPVM_OK;
}

DevOp to_devop(const ppvm_op& op) {
  DevOp d;
  std::memset(&d, 0, sizeof(d));
  d.w0 = (uint16_t)(op.q0 >> 6);
  d.b0 = (uint16_t)(op.q0 & 63);
  d.w1 = (uint16_t)(op.q1 >> 6);
  d.b1 = (uint16_t)(op.q1 & 63);
  switch (op.code) {
    case PPVM_OP_X: d.code = C_X; break;
    case PPVM_OP_Y: d.code = C_Y; break;
    case PPVM_OP_Z: d.code = C_Z; break;
    case PPVM_OP_H: d.code = C_H; break;
    case PPVM_OP_S: d.code = C_S; break;
    case PPVM_OP_S_DAG: d.code = C_SDAG; break;
    case PPVM_OP_SQRT_X: d.code = C_SQX; break;
    case PPVM_OP_SQRT_X_DAG: d.code = C_SQXDAG; break;
    case PPVM_OP_SQRT_Y: d.code = C_SQY; break;
    case PPVM_OP_SQRT_Y_DAG: d.code = C_SQYDAG; break;
    case PPVM_OP_CNOT: d.code = C_CNOT; break;
    case PPVM_OP_CZ: d.code = C_CZ; break;
    case PPVM_OP_CY: d.code = C_CY; break;
    case PPVM_OP_PAULI_ERROR: {  // noise.rs:17-37: factors computed as the reference does
      d.code = C_PAULI_ERROR;
      const double one = 1.0;
      d.f0 = one - op.p[1] * 2.0 - op.p[2] * 2.0;  // X
      d.f1 = one - op.p[0] * 2.0 - op.p[1] * 2.0;  // Z
      d.f2 = one - op.p[0] * 2.0 - op.p[2] * 2.0;  // Y
      break;
    }
    case PPVM_OP_DEPOLARIZE1: d.code = C_DEP1; d.f0 = 1.0 - op.theta * (4.0 / 3.0); break;
    case PPVM_OP_DEPOLARIZE2: d.code = C_DEP2; d.f0 = 1.0 - op.theta * (16.0 / 15.0); break;
    case kOpPauliError2: d.code = C_PERR2; d.f0 = op.theta; break;  // theta: factor table index
    default: {  // Clifford-angle rotation
      d.code = C_ROTC;
      const bool gx = op.code == PPVM_OP_RX || op.code == PPVM_OP_RY || op.code == PPVM_OP_RXX ||
                      op.code == PPVM_OP_RYY;
      const bool gz = op.code == PPVM_OP_RZ || op.code == PPVM_OP_RY || op.code == PPVM_OP_RZZ ||
                      op.code == PPVM_OP_RYY;
      d.two = (op.code == PPVM_OP_RXX || op.code == PPVM_OP_RYY || op.code == PPVM_OP_RZZ) ? 1 : 0;
      d.ax = (uint16_t)((gx ? 1 : 0) | ((gx && d.two) ? 2 : 0));
      d.az = (uint16_t)((gz ? 1 : 0) | ((gz && d.two) ? 2 : 0));
      d.f0 = op.theta > 0 ? 1.0 : -1.0;
      break;
    }
  }
  return d;
}

void gen_from_op(const ppvm_sum* s, const ppvm_op& op, Gen& g) {
  std::memset(&g, 0, sizeof(g));
  auto set = [&](uint32_t q, bool x, bool z) {
    if (x) g.gx[q >> 6] |= 1ull << (q & 63);
    if (z) g.gz[q >> 6] |= 1ull << (q & 63);
  };
  switch (op.code) {
    case PPVM_OP_RX: set(op.q0, true, false); break;
    case PPVM_OP_RY: set(op.q0, true, true); break;
    case PPVM_OP_RZ: set(op.q0, false, true); break;
    case PPVM_OP_RXX: set(op.q0, true, false); set(op.q1, true, false); break;
    case PPVM_OP_RYY: set(op.q0, true, true); set(op.q1, true, true); break;
    case PPVM_OP_RZZ: set(op.q0, false, true); set(op.q1, false, true); break;
    default: break;
  }
  g.lw = s->lossy ? (uint32_t)s->wr : 0u;
}

// ---- Clifford tableau of a run (host) ------------------------------------------------------------
struct HostTableau {
  TabParams tp;
  std::vector<uint32_t> tq;    // touched qubits, ascending (rank order)
  std::vector<uint64_t> rows;  // per row: a[W] (X plane), b[W] (Z plane) of the image
  std::vector<uint8_t> ph;     // image = i^ph X^a Z^b
  std::vector<uint8_t> sign;   // image = (-1)^sign * (Hermitian word a, b)
};

bool devop_two(const DevOp& d) {
  return d.code == C_CNOT || d.code == C_CZ || d.code == C_CY || (d.code == C_ROTC && d.two);
}

// Images of X_q and Z_q (q touched by the run) under the Clifford ops d[0..L), applied in
// order with cliff_rule to 64 generators per word (column form: one bit per generator).
void compose_tableau(int W, const DevOp* d, int L, HostTableau& t) {
  std::memset(&t.tp, 0, sizeof(t.tp));
  for (int i = 0; i < L; ++i) {
    t.tp.T[d[i].w0] |= 1ull << d[i].b0;
    if (devop_two(d[i])) t.tp.T[d[i].w1] |= 1ull << d[i].b1;
  }
  t.tq.clear();
  std::vector<int> rank((size_t)64 * W, -1);
  for (int w = 0; w < W; ++w) {
    t.tp.pre[w] = (uint32_t)t.tq.size();
    for (int b = 0; b < 64; ++b)
      if ((t.tp.T[w] >> b) & 1ull) {
        rank[(size_t)w * 64 + b] = (int)t.tq.size();
        t.tq.push_back((uint32_t)(w * 64 + b));
      }
  }
  const int nt = (int)t.tq.size(), R = 2 * nt, RW = (R + 63) / 64;
  t.tp.nrows = (uint32_t)R;
  std::vector<uint64_t> cx((size_t)nt * RW, 0), cz((size_t)nt * RW, 0), sg(RW, 0);
  for (int r = 0; r < nt; ++r) {
    cx[(size_t)r * RW + (2 * r) / 64] |= 1ull << ((2 * r) % 64);
    cz[(size_t)r * RW + (2 * r + 1) / 64] |= 1ull << ((2 * r + 1) % 64);
  }
  for (int i = 0; i < L; ++i) {
    const int r0 = rank[(size_t)d[i].w0 * 64 + d[i].b0];
    const int r1 = devop_two(d[i]) ? rank[(size_t)d[i].w1 * 64 + d[i].b1] : -1;
    for (int j = 0; j < RW; ++j) {
      uint64_t x0 = cx[(size_t)r0 * RW + j], z0 = cz[(size_t)r0 * RW + j];
      uint64_t x1 = r1 >= 0 ? cx[(size_t)r1 * RW + j] : 0ull, z1 = r1 >= 0 ? cz[(size_t)r1 * RW + j] : 0ull;
      uint64_t ng = sg[j];
      cliff_rule<uint64_t>(d[i], x0, z0, x1, z1, ng);
      cx[(size_t)r0 * RW + j] = x0;
      cz[(size_t)r0 * RW + j] = z0;
      if (r1 >= 0) {
        cx[(size_t)r1 * RW + j] = x1;
        cz[(size_t)r1 * RW + j] = z1;
      }
      sg[j] = ng;
    }
  }
  t.rows.assign((size_t)R * 2 * W, 0);
  for (int c = 0; c < nt; ++c) {
    const uint32_t q = t.tq[c];
    for (int j = 0; j < RW; ++j) {
      for (int pl = 0; pl < 2; ++pl) {
        uint64_t m = (pl == 0 ? cx : cz)[(size_t)c * RW + j];
        while (m) {
          const int row = j * 64 + __builtin_ctzll(m);
          m &= m - 1;
          t.rows[(size_t)row * 2 * W + (size_t)pl * W + (q >> 6)] |= 1ull << (q & 63);
        }
      }
    }
  }
  t.ph.assign(R, 0);
  t.sign.assign(R, 0);
  for (int row = 0; row < R; ++row) {
    const uint64_t* e = &t.rows[(size_t)row * 2 * W];
    unsigned p = 0;
    for (int w = 0; w < W; ++w) p += (unsigned)__builtin_popcountll(e[w] & e[W + w]);
    const bool neg = (sg[row / 64] >> (row % 64)) & 1ull;
    t.sign[row] = neg ? 1 : 0;
    t.ph[row] = (uint8_t)((p + (neg ? 2u : 0u)) & 3u);
  }
  // generators whose image is themselves (same word, phase 0) stay out of the kernel's product
  for (int c = 0; c < nt; ++c) {
    const uint32_t q = t.tq[c];
    for (int pl = 0; pl < 2; ++pl) {
      const int row = 2 * c + pl;
      const uint64_t* e = &t.rows[(size_t)row * 2 * W];
      bool self = t.ph[row] == 0;
      for (int w = 0; w < W && self; ++w) {
        const uint64_t bit = (w == (int)(q >> 6)) ? 1ull << (q & 63) : 0ull;
        self = e[w] == (pl == 0 ? bit : 0ull) && e[W + w] == (pl == 1 ? bit : 0ull);
      }
      if (!self) (pl == 0 ? t.tp.Tx : t.tp.Tz)[q >> 6] |= 1ull << (q & 63);
    }
  }
}

// ---- kernel enqueue (templated on W) ------------------------------------------------------------
template <int W>
struct K {
  static constexpr int ITEMS = ItemsFor<W>::value;
  static constexpr unsigned long long TILE = (unsigned long long)kScanBlock * ITEMS;

  static void rotation(ppvm_sum* s, const Gen& g, double theta, int op) {
    const Planes P = s->planes_view();
    unsigned xmask = 0, zmask = 0;
    for (int w = 0; w < W; ++w) {
      if (g.gz[w]) xmask |= 1u << w;
      if (g.gx[w]) zmask |= 1u << w;
    }
    const double sn = std::sin(theta), cs = std::cos(theta);
    const unsigned long long nub = std::max<unsigned long long>(s->n_ub, 1);
    {
      ProfScope ps(s, F_SCAN, op, 1);
      launch(k_rot_scan<W, kScanBlock, ITEMS>, grid_for(nub, TILE, 8), kScanBlock, 0, s->stream,
          P, s->d_ctrl, g, xmask, zmask, s->s_idx, s->s_rec, s->partner, s->tstate,
          s->next_tile_epoch(), op, s->d_log);
    }
    {
      ProfScope ps(s, F_PAIR, op, 1);
      launch(k_rot_pair<W>, grid_for(nub, kPairBlock, 8), kPairBlock, 0, s->stream,
          s->d_ctrl, g, s->s_rec, s->partner, s->table, s->table_cap, s->next_table_epoch(), op);
    }
    {
      ProfScope ps(s, F_APPLY, op, 1);
      launch(k_rot_apply<W, kScanBlock, ITEMS>, grid_for(nub, TILE, 8), kScanBlock, 0, s->stream,
          P, s->d_ctrl, g, sn, cs, s->s_idx, s->s_rec, s->partner, s->tstate, s->next_tile_epoch(),
          op, s->d_log);
    }
    {
      ProfScope ps(s, F_COMMIT, op, 1);
      launch(k_commit_rot, 1, 1, 0, s->stream, s->d_ctrl, op, s->d_log);
    }
    s->n_ub = std::min<unsigned long long>(s->cap, 2 * s->n_ub);
  }

  // AmplitudeDamping::amplitude_damping (noise.rs:132-163) on qubit q: see noise.cuh.
  static void damping(ppvm_sum* s, uint32_t q, double gamma, int op) {
    const Planes P = s->planes_view();
    Gen g;
    std::memset(&g, 0, sizeof(g));
    g.gz[q >> 6] = 1ull << (q & 63);
    const unsigned qmask = 1u << (q >> 6);
    const double om = 1.0 - gamma;    // T::Coeff::from(1.0) - gamma
    const double sxy = std::sqrt(om);  // (1 - gamma).sqrt()
    const unsigned long long nub = std::max<unsigned long long>(s->n_ub, 1);
    {
      ProfScope ps(s, F_SCAN, op, 1);
      launch(k_rot_scan<W, kScanBlock, ITEMS, true>, grid_for(nub, TILE, 8), kScanBlock, 0, s->stream,
          P, s->d_ctrl, g, 0u, qmask, s->s_idx, s->s_rec, s->partner, s->tstate,
          s->next_tile_epoch(), op, s->d_log);
    }
    const unsigned tep = s->next_table_epoch();
    {
      ProfScope ps(s, F_PAIR, op, 1);
      launch(k_damp_index<W>, grid_for(nub, kPairBlock, 8), kPairBlock, 0, s->stream,
          s->d_ctrl, g, s->s_rec, s->table, s->table_cap, tep, op);
      launch(k_damp_probe<W>, grid_for(nub, kPairBlock, 8), kPairBlock, 0, s->stream,
          P, s->d_ctrl, g, q >> 6, s->s_rec, s->partner, s->table, s->table_cap, tep, sxy, op);
    }
    {
      ProfScope ps(s, F_APPLY, op, 1);
      launch(k_damp_apply<W, kScanBlock, ITEMS>, grid_for(nub, TILE, 8), kScanBlock, 0, s->stream,
          P, s->d_ctrl, g, om, gamma, s->s_idx, s->s_rec, s->partner, s->tstate, s->next_tile_epoch(), op);
    }
    {
      ProfScope ps(s, F_COMMIT, op, 1);
      launch(k_commit_damp, 1, 1, 0, s->stream, s->d_ctrl, op, s->d_log);
    }
    s->n_ub = std::min<unsigned long long>(s->cap, 2 * s->n_ub);
  }

  // LossChannel / ResetLossChannel / CorrelatedLossChannel (noise.rs:165-275) on a lossy sum:
  // see loss.cuh.  Writes the whole output into the alternate planes, then swaps.
  static void loss(ppvm_sum* s, const ppvm_op& o, int op) {
    const Planes P = s->planes_view(), O = s->alt_view();
    const unsigned long long nub = std::max<unsigned long long>(s->n_ub, 1);
    unsigned long long tsize = next_pow2(std::max<unsigned long long>(2 * nub, 1024));
    if (tsize > s->table_cap) tsize = s->table_cap;
    LossOp lo;
    std::memset(&lo, 0, sizeof(lo));
    lo.mode = o.code == PPVM_OP_LOSS_CHANNEL ? kLossChannel
              : o.code == PPVM_OP_RESET_LOSS_CHANNEL ? kResetLoss : kCorrelatedLoss;
    lo.qa = o.q0;
    lo.qb = lo.mode == kCorrelatedLoss ? o.q1 : o.q0;
    lo.lw = (uint32_t)s->wr;
    if (lo.mode == kLossChannel) {
      lo.p0 = o.theta;
      lo.keep1 = 1.0 - o.theta;  // T::Coeff::from(1.0) - p
    } else if (lo.mode == kCorrelatedLoss) {
      lo.p0 = o.p[0];
      lo.p1 = o.p[1];
      lo.p2 = o.p[2];
      lo.keep1 = 1.0 - o.p[2];
      lo.keep0 = 1.0 - o.p[1] * 2.0 - o.p[0];
    }
    const unsigned tep = s->next_table_epoch();
    {
      ProfScope ps(s, F_LOSS, op, 1);
      launch(k_loss_index<W>, grid_for(nub, 256, 8), 256, 0, s->stream, P, s->d_ctrl, s->table, tsize - 1, tep,
             op, s->d_log);
      const unsigned e1 = s->next_tile_epoch(), e2 = s->next_tile_epoch();
      auto count_emit = [&](auto count_k, auto emit_k) {
        launch(count_k, grid_for(nub, 256, 8), 256, 0, s->stream, P, s->d_ctrl, lo, s->table, tsize - 1, tep);
        launch(emit_k, grid_for(nub, 256, 8), 256, 0, s->stream, P, O, s->d_ctrl, lo, s->table, tsize - 1, tep,
               s->tstate, s->tstate2, e1, e2, op, s->d_log);
      };
      if (lo.mode == kLossChannel)
        count_emit(k_loss_count<W, kLossChannel>, k_loss_emit<W, 256, kLossChannel>);
      else if (lo.mode == kResetLoss)
        count_emit(k_loss_count<W, kResetLoss>, k_loss_emit<W, 256, kResetLoss>);
      else
        count_emit(k_loss_count<W, kCorrelatedLoss>, k_loss_emit<W, 256, kCorrelatedLoss>);
    }
    std::swap(s->planes, s->alt);
    s->swaps.push_back(op);
    s->n_ub = std::min<unsigned long long>(s->cap, s->n_ub * (lo.mode == kCorrelatedLoss ? 4 : 2));
  }

  static void clifford(ppvm_sum* s, const DevOp* ops_dev, int nops, int op0) {
    const Planes P = s->planes_view();
    ProfScope ps(s, F_CLIFF, op0, nops);
    launch(k_clifford<W, kCliffBlock>, grid_for(std::max<unsigned long long>(s->n_ub, 1), kCliffBlock, 16),
           kCliffBlock, 0, s->stream, P, s->d_ctrl, ops_dev, nops, op0, s->d_log, s->d_perr2);
  }

  static void truncate(ppvm_sum* s, int op) {
    const Planes P = s->planes_view();
    {
      ProfScope ps(s, F_TRUNC, op, 1);
      launch(k_truncate<W, kScanBlock, ITEMS>, grid_for(std::max<unsigned long long>(s->n_ub, 1), TILE, 8),
             kScanBlock, 0, s->stream,
          P, s->d_ctrl, s->thr, s->maxw, s->d_pres_keys, s->d_pres_table, s->pres_mask, s->npres,
          s->side, s->tstate, s->next_tile_epoch(), op, s->d_log, s->maxlw, s->lossy ? (unsigned)s->wr : 0u);
    }
    ProfScope ps2(s, F_COMMIT, op, 1);
    launch(k_commit_truncate<W>, 1, 256, 0, s->stream, P, s->d_ctrl, s->side, op, s->d_log);
  }

  // Fused run of single-qubit RX (cls 0) or RZ (cls 1) rotations, ops[op0..op0+L), optionally
  // followed by its TRUNCATE (trunc_op >= 0).  Writes into the alternate planes, then swaps.
  static ppvm_status run(ppvm_sum* s, const RunDesc& rd, int op0, int L, int trunc_op) {
    const Planes P = s->planes_view(), O = s->alt_view();
    const unsigned long long nub = std::max<unsigned long long>(s->n_ub, 1);
    unsigned long long tsize = next_pow2(std::max<unsigned long long>(2 * nub, 1024));
    if (tsize > s->table_cap) tsize = s->table_cap;
    s->run_slots_used = std::max(s->run_slots_used, tsize);
    const void* d_rd_v = nullptr;
    PPVM_TRY(stage_put(s, &rd, sizeof(RunDesc), &d_rd_v));
    const RunDesc* d_rd = static_cast<const RunDesc*>(d_rd_v);
    // grp_min, grp_cnt and created are clean here: k_run_scatter and the last block of
    // k_run_groups reset what a run used, grow() clears them on allocation and run_list()
    // after a device error
    const int trunc = trunc_op >= 0 ? 1 : 0;
    {
      ProfScope ps(s, F_RUN_CLASSIFY, op0, L);
      const unsigned tep = s->next_table_epoch();
      launch(k_run_classify<W, kScanBlock, ITEMS>, grid_for(nub, TILE, 8), kScanBlock, 0, s->stream, P, O,
             s->d_ctrl, d_rd, s->R, s->table, tsize - 1, tep, trunc, s->thr, s->maxw, s->tstate,
             s->next_tile_epoch(), op0);
    }
    {
      ProfScope ps(s, F_RUN_ORDER, op0, L);
      const unsigned ea = s->next_tile_epoch(), eb = s->next_tile_epoch();
      launch(k_run_order<kScanBlock, 2>, grid_for(nub, kScanBlock * 2, 8), kScanBlock, 0, s->stream,
          s->d_ctrl, s->R, s->tstate, s->tstate2, ea, eb, op0);
    }
    {
      ProfScope ps(s, F_RUN_SCATTER, op0, L);
      launch(k_run_scatter<W>, grid_for(nub, 256, 8), 256, 0, s->stream, P, s->d_ctrl, d_rd, s->R);
    }
    // Many groups: scratch mode (group outputs placed by k_run_place, one look-back per tile
    // of groups instead of one per group).  ngroups <= live terms <= nub, so below the
    // threshold the device takes look-back mode and k_run_place is not needed.
    // Scratch offsets are 32-bit (RunScratch::g_rep): scratch mode needs cap < 2^32, which
    // grow() guarantees by refusing capacities from 0xFFFFFFF0 up.
    const unsigned long long smin = run_scratch_min_groups();
    bool allow = nub >= smin && s->cap < 0xFFFFFFFFull;
    if (allow && (!s->scr || s->scr_cap != s->cap)) {
      pool_free(s->scr);
      s->scr = nullptr;
      s->scr_cap = 0;
      if (pool_malloc((void**)&s->scr, sizeof(uint64_t) * (size_t)(2 * s->W + 1) * s->cap, kAllocRunScratch) !=
          cudaSuccess) {
        // no room for the scratch planes: this run takes look-back mode, which needs none
        // (same output, slower on many groups); a later run tries the allocation again
        cudaGetLastError();
        s->scr = nullptr;
        allow = false;
      } else {
        s->scr_cap = s->cap;
      }
    }
    const Planes S = allow ? s->view_of(s->scr) : O;
    const unsigned long long scratch_min = allow ? smin : ~0ull;
    {
      ProfScope ps(s, F_RUN_GROUPS, op0, L);
      // no more blocks than fit on the GPU at once: warps take groups by ticket, so blocks
      // beyond that would only queue on the ticket counter
      static int resident = 0;  // blocks per SM (the same on every B200)
      if (!resident) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, k_run_groups<W>, kRunWarps * 32, 0) !=
                cudaSuccess || resident < 1)
          resident = 1;
      }
      launch(k_run_groups<W>, grid_for(nub, kRunWarps, std::min(resident, 8)), kRunWarps * 32, 0, s->stream,
          O, S, s->d_ctrl, d_rd, s->R, trunc, s->thr, s->maxw, s->tstate, s->next_tile_epoch(), op0,
          trunc_op, s->d_log, scratch_min, run_tile_mode());  // its last block publishes the counts and the op log
    }
    if (allow) {
      ProfScope ps(s, F_RUN_PLACE, op0, L);
      launch(k_run_place<W, 256, 2>, grid_for(nub, 512, 4), 256, 0, s->stream,
          S, O, s->d_ctrl, s->R, scratch_min, s->tstate, s->next_tile_epoch(), op0, run_tile_mode());
    }
    std::swap(s->planes, s->alt);
    s->swaps.push_back(op0);
    const int grow_bits = std::min(L, kRunMaxK);
    s->n_ub = std::min<unsigned long long>(s->cap, s->n_ub << grow_bits);
    return PPVM_OK;
  }

  // A composed Clifford run ops[op0..op0+nops), optionally with its TRUNCATE (trunc_op >= 0):
  // one pass from the planes into the alternate planes, then a swap.
  static ppvm_status tableau(ppvm_sum* s, const HostTableau& t, int op0, int nops, int trunc_op) {
    const Planes P = s->planes_view(), O = s->alt_view();
    const void* d_rows = nullptr;
    const void* d_ph = nullptr;
    PPVM_TRY(stage_put(s, t.rows.data(), t.rows.size() * sizeof(uint64_t), &d_rows));
    PPVM_TRY(stage_put(s, t.ph.data(), t.ph.size(), &d_ph));
    const unsigned long long nub = std::max<unsigned long long>(s->n_ub, 1);
    // one-word sums of many terms through a run that moves many generators: chunk tables
    int chunk_min = -1;
    if constexpr (W == 1) {
      const unsigned mode = tableau_chunk_mode();
      const int moved = __builtin_popcountll(t.tp.Tx[0]) + __builtin_popcountll(t.tp.Tz[0]);
      if (mode == 1 && moved > 0) chunk_min = 0;
      else if (mode == 0 && nub >= kTabChunkMinTerms && moved >= kTabChunkMinMoved) chunk_min = kTabChunkMinBits;
    }
    const size_t smem = t.rows.size() * sizeof(uint64_t) + t.ph.size() + (chunk_min >= 0 ? kTabChunkSmem : 0);
    if (smem > kTabMaxSmem) return fail(PPVM_EINVAL, "internal: tableau exceeds shared memory");
    static unsigned long long attr_set = 0;  // one bit per device
    if (!((attr_set >> s->device) & 1ull)) {
      CUDA_TRY(cudaFuncSetAttribute(k_tableau<W, kTabBlock, ITEMS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kTabMaxSmem));
      attr_set |= 1ull << s->device;
    }
    // blocks per SM: with the tables, as many as 227 KB of shared memory hold (3)
    const int bps = chunk_min >= 0 ? (int)std::max<size_t>(1, std::min<size_t>(4, (227 * 1024) / (smem + 2048)))
                                   : (int)std::max<size_t>(1, std::min<size_t>(4, (200 * 1024) / (smem + 4096)));
    {
      ProfScope ps(s, F_TABLEAU, op0, nops, trunc_op);
      launch(k_tableau<W, kTabBlock, ITEMS>, grid_for(nub, (unsigned long long)kTabBlock * ITEMS, bps), kTabBlock, smem, s->stream,
          P, O, s->d_ctrl, t.tp, static_cast<const uint64_t*>(d_rows), static_cast<const uint8_t*>(d_ph),
          trunc_op >= 0 ? 1 : 0, s->thr, s->maxw, s->tstate, s->next_tile_epoch(), op0, nops, trunc_op,
          s->d_log, chunk_min);  // its last block publishes the count
    }
    std::swap(s->planes, s->alt);
    s->swaps.push_back(op0);
    return PPVM_OK;
  }

  // Term-budget truncation: priority keys, radix select of the budget-th largest, compaction.
  static void budget(ppvm_sum* s, unsigned long long B, const MlpWeights* mw, int L, int layers_left, int bits) {
    const Planes P = s->planes_view();
    uint32_t* keys = s->s_idx;  // cap entries, free outside the rotation pipeline
    const unsigned long long nub = std::max<unsigned long long>(s->n_host, 1);
    k_score<W><<<grid_for(nub, 128, 8), 128, 0, s->stream>>>(P, s->d_ctrl, mw, L, layers_left, keys);
    k_sel_init<<<1, 1, 0, s->stream>>>(s->d_ctrl, B, s->d_sel);
    if (bits == 11) {
      for (int shift : {21, 10, 0}) {
        k_sel_hist<11><<<grid_for(nub, 256, 4), 256, 0, s->stream>>>(s->d_ctrl, keys, s->d_sel, shift, s->d_hist);
        k_sel_pick<11><<<1, 256, 0, s->stream>>>(s->d_sel, shift, s->d_hist);
      }
    } else {
      for (int shift : {24, 16, 8, 0}) {
        k_sel_hist<8><<<grid_for(nub, 256, 4), 256, 0, s->stream>>>(s->d_ctrl, keys, s->d_sel, shift, s->d_hist);
        k_sel_pick<8><<<1, 256, 0, s->stream>>>(s->d_sel, shift, s->d_hist);
      }
    }
    const unsigned ea = s->next_tile_epoch(), eb = s->next_tile_epoch();
    k_budget_compact<W, kScanBlock, ITEMS><<<grid_for(nub, TILE, 8), kScanBlock, 0, s->stream>>>(
        P, s->d_ctrl, keys, s->d_sel, s->tstate, ea, s->tstate2, eb);
    k_commit_budget<<<1, 1, 0, s->stream>>>(s->d_ctrl, s->d_sel);
    s->launch_count += 3 + 2 * (bits == 11 ? 3 : 4) + 1;
  }
  static void features(ppvm_sum* s, int L, int layers_left, float* out) {
    k_features<W><<<grid_for(std::max<unsigned long long>(s->n_host, 1), 256, 8), 256, 0, s->stream>>>(
        s->planes_view(), s->d_ctrl, L, layers_left, out);
  }

  static void owz(ppvm_sum* s, int nblocks) {
    ProfScope ps(s, F_READ, -1, 1);
    ps.L.bytes = s->n_host * (8ull * W + 8);  // every term's X words and coefficient
    s->launch_count += 1;                     // k_sum_partials (ProfScope counts k_owz)
    k_owz<W><<<nblocks, kRedBlock, 0, s->stream>>>(s->planes_view(), s->d_ctrl, s->d_partials);
    k_sum_partials<<<1, kRedBlock, 0, s->stream>>>(s->d_partials, nblocks, s->d_ctrl);
  }
  static void trace(ppvm_sum* s, int nblocks, int nitems) {
    k_trace<W><<<nblocks, kRedBlock, 0, s->stream>>>(s->planes_view(), s->d_ctrl, s->d_pat, nitems,
                                                     s->n, s->d_partials, s->lossy ? (unsigned)s->wr : 0u);
    k_sum_partials<<<1, kRedBlock, 0, s->stream>>>(s->d_partials, nblocks, s->d_ctrl);
  }
  static void weights(ppvm_sum* s, uint32_t* out) {
    k_weights<W><<<grid_for(std::max<unsigned long long>(s->n_host, 1), kRedBlock, 8), kRedBlock, 0,
                   s->stream>>>(s->planes_view(), s->d_ctrl, out);
  }
  static void build_index(ppvm_sum* s, unsigned long long mask, unsigned ep) {
    k_build_index<W><<<grid_for(std::max<unsigned long long>(s->n_host, 1), kRedBlock, 8), kRedBlock, 0,
                       s->stream>>>(s->planes_view(), s->d_ctrl, s->table, mask, ep);
  }
  static void add_seq(ppvm_sum* s, const uint64_t* nx, const uint64_t* nz, const double* nc,
                      unsigned long long k, unsigned long long mask, unsigned ep) {
    k_add_terms_seq<W><<<1, 1, 0, s->stream>>>(s->planes_view(), s->d_ctrl, nx, nz, nc, k, s->table,
                                                mask, ep);
  }
  // hash-owner sharding: stable partition of the terms by owner into caller rows; append
  static void shard_export(ppvm_sum* s, const Gen& m, unsigned nparts, unsigned long long ntiles,
                           unsigned long long* hist, unsigned long long* first, uint64_t* rows) {
    const Planes P = s->planes_view();
    const unsigned long long N = s->n_host;
    k_shard_hist<W><<<(unsigned)ntiles, kShardBlock, 0, s->stream>>>(P, N, m, nparts, hist);
    k_shard_scan<<<1, 1024, 0, s->stream>>>(hist, ntiles, nparts, first);
    k_shard_scatter<W><<<(unsigned)ntiles, kShardBlock, 0, s->stream>>>(P, N, m, nparts, hist, rows);
    k_shard_append<W><<<1, 32, 0, s->stream>>>(P, s->d_ctrl, nullptr, 0ull, 0ull);  // the sum is now empty
    s->launch_count += 4;
  }
  static void shard_append(ppvm_sum* s, const uint64_t* rows, unsigned long long k) {
    k_shard_append<W><<<(unsigned)grid_for(k, 256, 8), 256, 0, s->stream>>>(s->planes_view(), s->d_ctrl, rows, k,
                                                                          s->n_host);
    s->launch_count += 1;
  }
  static void overlap(ppvm_sum* a, ppvm_sum* b, unsigned long long mask, unsigned ep, int nblocks,
                      unsigned long long* mismatch) {
    k_overlap<W><<<nblocks, kRedBlock, 0, a->stream>>>(a->planes_view(), b->planes_view(), b->d_ctrl,
                                                       a->table, mask, ep, a->d_partials, mismatch);
    k_sum_partials<<<1, kRedBlock, 0, a->stream>>>(a->d_partials, nblocks, a->d_ctrl);
  }
};

#define DISPATCH_W(W_, CALL)                 \
  switch (W_) {                              \
    case 1: K<1>::CALL; break;               \
    case 2: K<2>::CALL; break;               \
    case 3: K<3>::CALL; break;               \
    case 4: K<4>::CALL; break;               \
    case 5: K<5>::CALL; break;               \
    case 6: K<6>::CALL; break;               \
    case 7: K<7>::CALL; break;               \
    default: K<8>::CALL; break;              \
  }

#define DISPATCH_W_RET(W_, CALL)                   \
  switch (W_) {                                    \
    case 1: return K<1>::CALL;                     \
    case 2: return K<2>::CALL;                     \
    case 3: return K<3>::CALL;                     \
    case 4: return K<4>::CALL;                     \
    case 5: return K<5>::CALL;                     \
    case 6: return K<6>::CALL;                     \
    case 7: return K<7>::CALL;                     \
    default: return K<8>::CALL;                    \
  }

ppvm_status enqueue_run(ppvm_sum* s, const RunDesc& rd, int op0, int L, int trunc_op) {
  DISPATCH_W_RET(s->W, run(s, rd, op0, L, trunc_op));
}

ppvm_status enqueue_tableau(ppvm_sum* s, const HostTableau& t, int op0, int nops, int trunc_op) {
  DISPATCH_W_RET(s->W, tableau(s, t, op0, nops, trunc_op));
}

int test_words_of(int W, const Gen& g) {
  int n = 0;
  for (int w = 0; w < W; ++w) n += (g.gz[w] != 0) + (g.gx[w] != 0);
  return n;
}

// Reads the control block and the op log back; synchronises.
ppvm_status sync_state(ppvm_sum* s, size_t nops) {
  CUDA_TRY(cudaMemcpyAsync(s->h_ctrl, s->d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s->stream));
  if (nops) CUDA_TRY(cudaMemcpyAsync(s->h_log, s->d_log, sizeof(OpLog) * nops, cudaMemcpyDeviceToHost, s->stream));
  s->xfer_d2h += sizeof(Ctrl) + sizeof(OpLog) * nops;
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  return PPVM_OK;
}

ppvm_status clear_err(ppvm_sum* s) {
  Ctrl c = *s->h_ctrl;
  c.err = 0;
  c.err_op = 0;
  c.fb_cut = 0;
  c.done = 0;  // blocks that returned early on the error never counted
  c.scr_top = 0;
  for (int t = 0; t < 4; ++t) c.tickets[t] = 0;
  CUDA_TRY(cudaMemcpyAsync(s->d_ctrl, &c, sizeof(Ctrl), cudaMemcpyHostToDevice, s->stream));
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  s->xfer_h2d += sizeof(Ctrl);
  return PPVM_OK;
}

// Whether a local op can join a composed Clifford (tableau) pass: a Clifford map applied to
// every term alike.  On a lossy sum a two-qubit gate leaves terms with a lost qubit alone, so
// its map depends on the term: those ops take the per-op pass.
bool tab_ok(const ppvm_sum* s, const DevOp& d) {
  if (!is_cliff_code(d.code)) return false;
  if (!s->lossy) return true;
  return !(d.code == C_CNOT || d.code == C_CZ || d.code == C_CY || (d.code == C_ROTC && d.two));
}

// Enqueues ops[start..n) (gate-list indices start..n).  Generators of explicit Pauli rotations
// come from `gens` when ops[i].flags == 1 (index in q0).
ppvm_status enqueue(ppvm_sum* s, const ppvm_op* ops, size_t n_ops, size_t start,
                    const std::vector<Gen>& gens, std::vector<int>& test_words) {
  std::vector<DevOp> run;  // pending local ops (Cliffords, Clifford-angle rotations, noise)
  int run_start = -1;
  SinCosMemo trig;          // the fused runs' gate angles
  size_t per_gate_end = 0;  // ops before this index take the per-gate path (a wide run)
  s->d_perr2 = nullptr;
  if (!s->perr2_host.empty()) {
    const void* d = nullptr;
    PPVM_TRY(stage_put(s, s->perr2_host.data(), sizeof(double) * s->perr2_host.size(), &d));
    s->d_perr2 = static_cast<const double*>(d);
  }
  // in-place per-op pass over run[a, b)
  auto per_op = [&](size_t a, size_t b) -> ppvm_status {
    size_t off = a;
    while (off < b) {
      const int cnt = (int)std::min<size_t>(kMaxOpsPerLaunch, b - off);
      const void* d_ops = nullptr;
      PPVM_TRY(stage_put(s, run.data() + off, sizeof(DevOp) * cnt, &d_ops));
      DISPATCH_W(s->W, clifford(s, static_cast<const DevOp*>(d_ops), cnt, run_start + (int)off));
      off += cnt;
    }
    return PPVM_OK;
  };
  // Enqueues the pending local ops.  Stretches of at least kTabMinOps Clifford ops become one
  // tableau pass; the rest (noise ops, short stretches) take the per-op pass.  A TRUNCATE at
  // trunc_op that directly follows the ops is fused into a final tableau pass when the sum
  // has no preserve strings (*fused is then set).
  auto flush = [&](int trunc_op, bool* fused) -> ppvm_status {
    if (fused) *fused = false;
    size_t a = 0, pend = 0;  // run[pend, a) waits for the per-op pass
    while (a < run.size()) {
      size_t b = a;
      while (b < run.size() && tab_ok(s, run[b])) ++b;
      if (b - a >= (size_t)kTabMinOps) {
        PPVM_TRY(per_op(pend, a));
        const int t_op =
            (b == run.size() && trunc_op >= 0 && s->npres == 0 && s->maxlw == UINT64_MAX) ? trunc_op : -1;
        HostTableau tab;
        compose_tableau(s->W, run.data() + a, (int)(b - a), tab);
        PPVM_TRY(enqueue_tableau(s, tab, run_start + (int)a, (int)(b - a), t_op));
        if (t_op >= 0 && fused) *fused = true;
        pend = a = b;
      } else {
        a = (b == a) ? a + 1 : b;
      }
    }
    PPVM_TRY(per_op(pend, run.size()));
    run.clear();
    run_start = -1;
    return PPVM_OK;
  };
  for (size_t i = start; i < n_ops; ++i) {
    const ppvm_op& op = ops[i];
    if (op.flags == 1) {  // explicit generator
      PPVM_TRY(flush(-1, nullptr));
      const Gen& g = gens[op.q0];
      test_words[i] = test_words_of(s->W, g);
      bool cliff = is_clifford_angle(s, op.theta);
      if (cliff) {
        return fail(PPVM_EINVAL, "internal: explicit Clifford-angle generators are lowered earlier");
      }
      DISPATCH_W(s->W, rotation(s, g, op.theta, (int)i));
      continue;
    }
    if (op.code == PPVM_OP_TRUNCATE) {
      bool fused = false;
      PPVM_TRY(flush((int)i, &fused));
      if (!fused) DISPATCH_W(s->W, truncate(s, (int)i));
      continue;
    }
    if (op.code == PPVM_OP_AMPLITUDE_DAMPING) {
      PPVM_TRY(flush(-1, nullptr));
      DISPATCH_W(s->W, damping(s, op.q0, op.theta, (int)i));
      continue;
    }
    if (op.code == PPVM_OP_LOSS_CHANNEL || op.code == PPVM_OP_RESET_LOSS_CHANNEL ||
        op.code == PPVM_OP_CORRELATED_LOSS_CHANNEL) {
      PPVM_TRY(flush(-1, nullptr));
      DISPATCH_W(s->W, loss(s, op, (int)i));
      continue;
    }
    if (is_local(s, op)) {
      if (run.empty()) run_start = (int)i;
      DevOp d = to_devop(op);
      d.lw = s->lossy ? (uint16_t)s->wr : (uint16_t)0;
      run.push_back(d);
      continue;
    }
    // fused run of single-qubit RX (or RZ) rotations on distinct qubits.  Not on a lossy sum:
    // its correlated loss channel sums up to three children per key in the reference's term
    // order, which a fused run (same terms, another order) would change in the last bit.
    const auto cap_it = s->run_cap.find(i);
    int max_gates = cap_it == s->run_cap.end() ? kRunMaxGates : cap_it->second;
    if (max_gates < 0) {  // the run starting here goes gate by gate: -max_gates gates
      per_gate_end = i + (size_t)(-max_gates);
      max_gates = 0;
    }
    const bool fusable = (op.code == PPVM_OP_RX || op.code == PPVM_OP_RZ) &&
                         !(s->flags & PPVM_FLAG_EXACT_ORDER) && !s->lossy && s->npres == 0 && max_gates >= 2 &&
                         i >= per_gate_end;
    if (fusable) {
      RunDesc rd;
      std::memset(&rd, 0, sizeof(rd));
      rd.cls = op.code == PPVM_OP_RX ? 0 : 1;
      size_t j = i;
      while (j < n_ops && (int)(j - i) < max_gates) {
        const ppvm_op& o = ops[j];
        if (o.flags != 0 || o.code != op.code || is_clifford_angle(s, o.theta)) break;
        if ((rd.Q[o.q0 >> 6] >> (o.q0 & 63)) & 1ull) break;  // qubit repeats: end the run
        rd.Q[o.q0 >> 6] |= 1ull << (o.q0 & 63);
        rd.q[rd.L] = o.q0;
        trig.get(o.theta, rd.sn[rd.L], rd.cs[rd.L]);
        ++rd.L;
        ++j;
      }
      if (rd.L >= 2) {
        PPVM_TRY(flush(-1, nullptr));
        const int trunc_op =
            (j < n_ops && ops[j].code == PPVM_OP_TRUNCATE && ops[j].flags == 0 && s->maxlw == UINT64_MAX) ? (int)j
                                                                                                      : -1;
        PPVM_TRY(enqueue_run(s, rd, (int)i, (int)rd.L, trunc_op));
        s->run_len[i] = (int)rd.L;
        i = trunc_op >= 0 ? j : j - 1;  // the loop's ++i moves past the run (and its TRUNCATE)
        continue;
      }
    }
    PPVM_TRY(flush(-1, nullptr));
    Gen g;
    gen_from_op(s, op, g);
    test_words[i] = test_words_of(s->W, g);
    DISPATCH_W(s->W, rotation(s, g, op.theta, (int)i));
  }
  PPVM_TRY(flush(-1, nullptr));
  CUDA_TRY(cudaGetLastError());
  return PPVM_OK;
}

// Runs a validated op list with capacity growth and replay.
ppvm_status run_list(ppvm_sum* s, const ppvm_op* ops, size_t n_ops, const std::vector<Gen>& gens) {
  if (s->poisoned) return fail(PPVM_ECUDA, "sum is in an error state from an earlier failure");
  PPVM_TRY(ensure_device(s->device));
  PPVM_TRY(ensure_log(s, std::max<size_t>(n_ops, 1)));
  std::vector<int> test_words(n_ops, 0);
  size_t start = 0;
  s->run_cap.clear();
  // every failed attempt grows the capacity or cuts a run, so the loop ends; the bound only
  // turns a logic error into a status
  const size_t max_attempts = 64 + 8 * n_ops;
  for (size_t attempt = 0; attempt < max_attempts; ++attempt) {
    s->swaps.clear();
    s->run_len.clear();
    stage_reset(s);  // the stream is idle here: every earlier upload has completed
    PPVM_TRY(enqueue(s, ops, n_ops, start, gens, test_words));
    PPVM_TRY(sync_state(s, n_ops));
    const Ctrl& c = *s->h_ctrl;
    s->n_host = c.n;
    if (c.err == kOk) {
      s->n_ub = s->n_host;
      s->last_nops = n_ops;
      if (s->prof) prof_collect(s, test_words);
      return PPVM_OK;
    }
    if (s->prof) prof_collect(s, test_words);
    PPVM_TRY(clear_run_tables(s, s->run_slots_used));  // a run stopped part-way leaves its slots set
    // fused runs at or after the failing op did not run: give their buffers back
    for (int op0 : s->swaps)
      if (op0 >= c.err_op) std::swap(s->planes, s->alt);
    if (c.err == kErrFallback && c.err_op >= 0 && (size_t)c.err_op >= start) {
      // a group of the run starting at err_op has more than kRunMaxK coordinates.  A
      // group's coordinates are fixed for the whole run (the plane the gates leave alone
      // holds them), so k_run_classify reports the number p of leading gates after which
      // every term, and every descendant, has at most kRunMaxK coordinates left.  Replay
      // with those p gates one at a time and the rest as one fused run, which then fits.
      start = (size_t)c.err_op;
      const auto len = s->run_len.find(start);
      const int L = len == s->run_len.end() ? 1 : len->second;
      const int p = c.fb_cut ? (int)std::min<unsigned long long>(c.fb_cut, (unsigned long long)L) : L;
      s->run_cap[start] = -p;
      PPVM_TRY(clear_err(s));
      s->n_ub = s->n_host;
      continue;
    }
    if (c.err == kErrCapacity && c.err_op >= 0 && (size_t)c.err_op >= start) {
      const unsigned long long need = c.cap_needed;
      start = (size_t)c.err_op;
      PPVM_TRY(clear_err(s));
      unsigned long long nc = std::max<unsigned long long>(2 * s->cap, need + need / 2 + 1024);
      if (nc >= 0xFFFFFFF0ull) nc = std::max<unsigned long long>(need, 0xFFFFFFF0ull - 1);
      ppvm_status st = grow(s, nc);
      if (st != PPVM_OK) {
        s->poisoned = true;
        return st;
      }
      s->n_ub = s->n_host;
      continue;
    }
    s->poisoned = true;
    if (c.err == kErrTimeout) return fail(PPVM_ETIMEOUT, "device wait timed out (op " + std::to_string(c.err_op) + ")");
    return fail(PPVM_ECUDA, "device error " + std::to_string(c.err) + " at op " + std::to_string(c.err_op));
  }
  s->poisoned = true;
  return fail(PPVM_ECAPACITY, "capacity growth did not converge");
}

ppvm_status run_gate(ppvm_sum* s, uint32_t code, const uint32_t* t, size_t k, bool pairs, double theta,
                     const double* p, int truncate) {
  if (!s) return fail(PPVM_EINVAL, "null sum");
  if (k && !t) return fail(PPVM_EINVAL, "null target list");
  if (pairs && (k % 2)) return fail(PPVM_EINVAL, "two-qubit operations require an even number of targets");
  std::vector<ppvm_op> ops;
  const size_t step = pairs ? 2 : 1;
  for (size_t i = 0; i < k; i += step) {
    ppvm_op op;
    std::memset(&op, 0, sizeof(op));
    op.code = code;
    op.q0 = t[i];
    op.q1 = pairs ? t[i + 1] : 0;
    op.theta = theta;
    if (p) for (int j = 0; j < 3; ++j) op.p[j] = p[j];
    PPVM_TRY(validate(s, op));
    ops.push_back(op);
  }
  if (truncate) {
    ppvm_op op;
    std::memset(&op, 0, sizeof(op));
    op.code = PPVM_OP_TRUNCATE;
    ops.push_back(op);
  }
  if (ops.empty()) return PPVM_OK;
  return run_list(s, ops.data(), ops.size(), {});
}

ppvm_status do_reduce_owz(ppvm_sum* s, double* out) {
  const int nb = (int)grid_for(std::max<unsigned long long>(s->n_host, 1), kRedBlock * 4, 2);
  DISPATCH_W(s->W, owz(s, nb));
  CUDA_TRY(cudaGetLastError());
  PPVM_TRY(sync_state(s, 0));
  if (s->prof) prof_collect(s, {});
  *out = s->h_ctrl->sum;
  return PPVM_OK;
}

// PauliPattern grammar (crates/ppvm-pauli-word/src/pattern/parse.rs:32-127) -> PatItems.
// Accept bits: 1 = I, 2 = X, 4 = Z, 8 = Y; '_' accepts only I, as the reference matcher does.
bool parse_pattern(const char* text, std::vector<PatItem>& out) {
  std::string in(text);
  size_t b = in.find_first_not_of(" \t\n\r"), e = in.find_last_not_of(" \t\n\r");
  in = (b == std::string::npos) ? std::string() : in.substr(b, e - b + 1);
  auto bit = [](char c) -> unsigned { return c == 'X' ? 2u : c == 'Z' ? 4u : c == 'Y' ? 8u : 0u; };
  size_t i = 0;
  while (i < in.size()) {
    const char c = in[i++];
    unsigned acc;
    if (c == '[') {
      unsigned set = 0;
      while (i < in.size()) {  // an unclosed '[' ends at the end of the text, as in parse.rs
        const char d = in[i];
        if (d == ']') {
          ++i;
          break;
        }
        if (!bit(d)) return false;
        set |= bit(d);
        ++i;
      }
      if (!set) return false;
      acc = set;
    } else if (c == '_') {
      acc = 1u;
    } else if (bit(c)) {
      acc = bit(c);
    } else {
      return false;
    }
    if (i < in.size() && in[i] == '?') {
      ++i;
      acc |= 1u;
    }
    PatItem it;
    it.accept = acc;
    it.arg = 0;
    if (i < in.size() && in[i] == '*') {
      ++i;
      it.kind = 1;
    } else if (i < in.size() && in[i] == '{') {
      ++i;
      std::string num;
      while (i < in.size() && isdigit((unsigned char)in[i])) num.push_back(in[i++]);
      if (i >= in.size() || in[i] != '}' || num.empty()) return false;
      ++i;
      it.kind = 2;
      it.arg = std::stoull(num);
    } else if (i < in.size() && isdigit((unsigned char)in[i])) {
      std::string num;
      while (i < in.size() && isdigit((unsigned char)in[i])) num.push_back(in[i++]);
      it.kind = 0;
      it.arg = std::stoull(num);
    } else {
      return false;
    }
    out.push_back(it);
  }
  return true;
}

// Builds the sum's key index (table slot -> term) for the cold lookup paths.
ppvm_status build_index(ppvm_sum* s, unsigned long long expected, unsigned long long* mask_out,
                        unsigned* epoch_out) {
  unsigned long long tsize = next_pow2(std::max<unsigned long long>(2 * expected, 1024));
  if (tsize > s->table_cap) return fail(PPVM_ECAPACITY, "index table too small");
  const unsigned ep = s->next_table_epoch();
  DISPATCH_W(s->W, build_index(s, tsize - 1, ep));
  *mask_out = tsize - 1;
  *epoch_out = ep;
  return PPVM_OK;
}

}  // namespace

// =============================================================================================
extern "C" {

const char* ppvm_last_error_string(void) { return g_err.c_str(); }
const char* ppvm_version(void) { return "ppvm_b200 0.1 (sm_100a)"; }

ppvm_status ppvm_sum_create2(ppvm_sum** out, uint32_t n_qubits, double min_abs_coeff, uint64_t max_weight,
                             size_t capacity_hint, uint32_t flags, int device) {
  if (!out) return fail(PPVM_EINVAL, "null out pointer");
  *out = nullptr;
  if (n_qubits == 0 || n_qubits > 64 * kMaxW)
    return fail(PPVM_EINVAL, "n_qubits must be in [1, 512]");
  const bool lossy = (flags & PPVM_FLAG_LOSSY) != 0;
  if (lossy && n_qubits > 32 * kMaxW) return fail(PPVM_EINVAL, "a lossy sum holds at most 256 qubits");
  PPVM_TRY(ensure_device(device));
  const int wr = (int)((n_qubits + 63) / 64);
  const int W = lossy ? 2 * wr : wr;  // a lossy sum keeps its loss bits in the X plane's upper words
  if (ppvm_sum* c = take_cached(device, W)) {  // a cached handle: reset its state
    c->n = n_qubits;
    c->wr = wr;
    c->lossy = lossy;
    c->thr = min_abs_coeff;
    c->maxw = max_weight;
    c->maxlw = UINT64_MAX;
    c->flags = flags;
    c->n_host = c->n_ub = 0;
    c->poisoned = false;
    c->swaps.clear();
    c->run_cap.clear();
    c->run_len.clear();
    c->npres = 0;
    c->h_pres.clear();
    c->prof = false;
    for (int f = 0; f < F_COUNT; ++f) c->prof_ms[f] = 0, c->prof_launches[f] = 0, c->prof_bytes[f] = 0;
    c->launch_count = c->xfer_h2d = c->xfer_d2h = 0;
    c->last_nops = 0;
    ppvm_status st = init_ctrl(c, 0);
    if (st == PPVM_OK && c->cap < std::max<size_t>(capacity_hint, 4096))
      st = grow(c, std::max<size_t>(capacity_hint, 4096));
    if (st == PPVM_OK && cudaStreamSynchronize(c->stream) != cudaSuccess) st = fail(PPVM_ECUDA, "sync failed");
    if (st != PPVM_OK) {
      destroy_now(c);
      return st;
    }
    *out = c;
    return PPVM_OK;
  }
  ppvm_sum* s = new ppvm_sum();
  s->device = device;
  s->n = n_qubits;
  s->W = W;
  s->wr = wr;
  s->lossy = lossy;
  s->thr = min_abs_coeff;
  s->maxw = max_weight;
  s->flags = flags;
  auto bail = [&](ppvm_status st) {
    destroy_now(s);
    return st;
  };
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(PPVM_ECUDA, "cudaStreamCreate failed"));
  if (cudaMalloc(&s->d_ctrl, sizeof(Ctrl)) != cudaSuccess ||
      cudaMallocHost(&s->h_ctrl, sizeof(Ctrl)) != cudaSuccess ||
      cudaMalloc(&s->d_partials, sizeof(double) * 8192) != cudaSuccess ||
      cudaMalloc(&s->d_counter, sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&s->d_sel, sizeof(SelState)) != cudaSuccess ||
      cudaMalloc(&s->d_hist, sizeof(unsigned) * 2048) != cudaSuccess ||
      cudaMalloc(&s->side, sizeof(uint64_t) * (2 * s->W + 1) * (kMaxPreserve + 1)) != cudaSuccess)
    return bail(fail(PPVM_ECAPACITY, "device allocation failed"));
  if (cudaMemsetAsync(s->d_hist, 0, sizeof(unsigned) * 2048, s->stream) != cudaSuccess)
    return bail(fail(PPVM_ECUDA, "memset failed"));
  ppvm_status st = init_ctrl(s, 0);
  if (st != PPVM_OK) return bail(st);
  st = grow(s, std::max<size_t>(capacity_hint, 4096));
  if (st != PPVM_OK) return bail(st);
  st = ensure_log(s, 64);
  if (st != PPVM_OK) return bail(st);
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return bail(fail(PPVM_ECUDA, "sync failed"));
  *out = s;
  return PPVM_OK;
}

ppvm_status ppvm_sum_create(ppvm_sum** out, uint32_t n_qubits, double min_abs_coeff, uint64_t max_weight,
                            size_t capacity_hint) {
  return ppvm_sum_create2(out, n_qubits, min_abs_coeff, max_weight, capacity_hint, 0, 0);
}

}  // extern "C"

namespace {
// Destroyed sums that own their stream go to a small per-process cache and are handed out
// again by ppvm_sum_create2 for the same device and plane width, with every buffer, the
// stream and the upload arena still allocated: creating a sum then costs no allocation.
std::vector<ppvm_sum*> g_sum_cache;  // guarded by g_pool_mu
constexpr size_t kSumCacheMax = 8;

void destroy_now(ppvm_sum* s) {
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (auto& L : s->prof_pending) {
    cudaEventDestroy(L.a);
    cudaEventDestroy(L.b);
  }
  for (cudaEvent_t e : s->event_pool) cudaEventDestroy(e);
  for (auto& ch : s->stage) {
    cudaFreeHost(ch.h);
    cudaFree(ch.d);
  }
  pool_free(s->planes);
  free_scratch(s);
  cudaFree(s->side);
  cudaFree(s->d_ctrl);
  cudaFreeHost(s->h_ctrl);
  cudaFree(s->d_log);
  cudaFreeHost(s->h_log);
  cudaFree(s->d_pat);
  cudaFree(s->d_partials);
  cudaFree(s->d_counter);
  cudaFree(s->d_sel);
  cudaFree(s->d_hist);
  cudaFree(s->d_pres_keys);
  cudaFree(s->d_pres_table);
  if (s->stream && s->own_stream) cudaStreamDestroy(s->stream);
  delete s;
}

ppvm_sum* take_cached(int device, int W) {
  // the largest cached capacity: a new sum then rarely grows (growth replays ops)
  std::lock_guard<std::mutex> lk(g_pool_mu);
  long best = -1;
  for (size_t i = 0; i < g_sum_cache.size(); ++i)
    if (g_sum_cache[i]->device == device && g_sum_cache[i]->W == W &&
        (best < 0 || g_sum_cache[i]->cap > g_sum_cache[(size_t)best]->cap))
      best = (long)i;
  if (best < 0) return nullptr;
  ppvm_sum* s = g_sum_cache[(size_t)best];
  g_sum_cache.erase(g_sum_cache.begin() + best);
  return s;
}
}  // namespace

namespace ppvm {
// The buffer cache for the other translation units (batch.cu): same rules as for the sums,
// a buffer goes back only when the stream that used it is idle.
cudaError_t cache_malloc(void** out, size_t bytes) { return pool_malloc(out, bytes); }
void cache_free(void* p) { pool_free(p); }
void release_batch_staging();  // batch.cu: frees the pinned staging buffer of the uploads
}  // namespace ppvm

extern "C" {

ppvm_status ppvm_sum_destroy(ppvm_sum* s) {
  if (!s) return PPVM_OK;
  cudaSetDevice(s->device);
  const bool idle = !s->stream || cudaStreamSynchronize(s->stream) == cudaSuccess;
  if (idle && !s->poisoned && !s->own_stream) {  // give a cached handle a stream of its own
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess) {
      s->stream = st;
      s->own_stream = true;
    }
  }
  if (idle && !s->poisoned && s->own_stream) {
    for (auto& L : s->prof_pending) {
      s->event_pool.push_back(L.a);
      s->event_pool.push_back(L.b);
    }
    s->prof_pending.clear();
    cudaFree(s->d_pat);
    cudaFree(s->d_pres_keys);
    cudaFree(s->d_pres_table);
    s->d_pat = nullptr;
    s->d_pres_keys = nullptr;
    s->d_pres_table = nullptr;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (g_sum_cache.size() < kSumCacheMax) {
      g_sum_cache.push_back(s);
      return PPVM_OK;
    }
  }
  destroy_now(s);
  return PPVM_OK;
}

ppvm_status ppvm_sum_set_stream(ppvm_sum* s, void* cuda_stream) {
  if (!s) return fail(PPVM_EINVAL, "null sum");
  CUDA_TRY(cudaSetDevice(s->device));
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  if (s->own_stream) cudaStreamDestroy(s->stream);
  if (cuda_stream) {
    s->stream = (cudaStream_t)cuda_stream;
    s->own_stream = false;
  } else {
    CUDA_TRY(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    s->own_stream = true;
  }
  return PPVM_OK;
}

ppvm_status ppvm_sum_clone(const ppvm_sum* src, ppvm_sum** out) {
  if (!src || !out) return fail(PPVM_EINVAL, "null argument");
  REQUIRE_USABLE(src);
  ppvm_sum* d = nullptr;
  PPVM_TRY(ppvm_sum_create2(&d, src->n, src->thr, src->maxw, std::max<unsigned long long>(src->cap, 4096),
                            src->flags, src->device));
  ppvm_sum* s = const_cast<ppvm_sum*>(src);
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  for (int w = 0; w < 2 * src->W + 1; ++w)
    CUDA_TRY(cudaMemcpyAsync(d->planes + (size_t)w * d->cap, src->planes + (size_t)w * src->cap,
                             sizeof(uint64_t) * src->n_host, cudaMemcpyDeviceToDevice, d->stream));
  d->n_host = src->n_host;
  d->n_ub = src->n_host;
  d->maxlw = src->maxlw;
  PPVM_TRY(init_ctrl(d, src->n_host));
  if (src->npres) {
    std::vector<uint64_t> x, z;
    for (int j = 0; j < src->npres; ++j)
      for (int w = 0; w < src->W; ++w) {
        x.push_back(src->h_pres[(size_t)j * 2 * src->W + w]);
        z.push_back(src->h_pres[(size_t)j * 2 * src->W + src->W + w]);
      }
    PPVM_TRY(ppvm_sum_set_preserve(d, x.data(), z.data(), src->npres));
  }
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  *out = d;
  return PPVM_OK;
}

ppvm_status ppvm_len(const ppvm_sum* s, size_t* out) {
  if (!s || !out) return fail(PPVM_EINVAL, "null argument");
  *out = (size_t)s->n_host;
  return PPVM_OK;
}

ppvm_status ppvm_sum_add_terms(ppvm_sum* s, const uint64_t* x, const uint64_t* z, const double* c, size_t k) {
  if (!s) return fail(PPVM_EINVAL, "null sum");
  if (k == 0) return PPVM_OK;
  if (!x || !z || !c) return fail(PPVM_EINVAL, "null term arrays");
  if (s->poisoned) return fail(PPVM_ECUDA, "sum is in an error state from an earlier failure");
  const int W = s->W;
  PPVM_TRY(check_words(s, x, z, k));
  PPVM_TRY(ensure_device(s->device));
  if (s->n_host + k > s->cap) PPVM_TRY(grow(s, std::max<unsigned long long>(2 * s->cap, s->n_host + k + 1024)));
  // the new terms go up through the pinned upload arena (the stream is idle between calls)
  std::vector<uint64_t> packed((size_t)(2 * W + 1) * k);
  std::memcpy(packed.data(), x, sizeof(uint64_t) * W * k);
  std::memcpy(packed.data() + (size_t)W * k, z, sizeof(uint64_t) * W * k);
  std::memcpy(packed.data() + (size_t)2 * W * k, c, sizeof(double) * k);
  stage_reset(s);
  const void* d_packed = nullptr;
  PPVM_TRY(stage_put(s, packed.data(), sizeof(uint64_t) * packed.size(), &d_packed));
  const uint64_t* dx = static_cast<const uint64_t*>(d_packed);
  const uint64_t* dz = dx + (size_t)W * k;
  const double* dc = reinterpret_cast<const double*>(dx + (size_t)2 * W * k);
  unsigned long long mask;
  unsigned ep;
  ppvm_status st = build_index(s, s->n_host + k, &mask, &ep);
  if (st == PPVM_OK) {
    DISPATCH_W(W, add_seq(s, dx, dz, dc, k, mask, ep));
    st = sync_state(s, 0);
  }
  PPVM_TRY(st);
  if (s->h_ctrl->err) {
    s->poisoned = true;
    return fail(PPVM_ECUDA, "device error while adding terms");
  }
  s->n_host = s->h_ctrl->n;
  s->n_ub = s->n_host;
  return PPVM_OK;
}

ppvm_status ppvm_sum_shard_export(ppvm_sum* s, const uint64_t* mask_x, const uint64_t* mask_z, uint32_t n_parts,
                                  void* d_rows, size_t rows_cap, uint64_t* counts) {
  if (!s || !mask_x || !mask_z || !counts) return fail(PPVM_EINVAL, "null argument");
  if (n_parts < 1 || n_parts > (uint32_t)kShardMaxParts)
    return fail(PPVM_EINVAL, "n_parts must be in [1, " + std::to_string(kShardMaxParts) + "]");
  REQUIRE_USABLE(s);
  PPVM_TRY(ensure_device(s->device));
  const unsigned long long N = s->n_host;
  for (uint32_t p = 0; p < n_parts; ++p) counts[p] = 0;
  if (N == 0) return PPVM_OK;
  if (!d_rows) return fail(PPVM_EINVAL, "null row buffer");
  if (rows_cap < N) return fail(PPVM_EINVAL, "row buffer holds fewer rows than the sum has terms");
  Gen m;
  std::memset(&m, 0, sizeof(m));
  for (int w = 0; w < s->W; ++w) {
    m.gx[w] = mask_x[w];
    m.gz[w] = mask_z[w];
  }
  const unsigned long long ntiles = (N + kShardBlock - 1) / kShardBlock;
  unsigned long long* hist = nullptr;
  CUDA_TRY(pool_malloc((void**)&hist, sizeof(unsigned long long) * (ntiles * n_parts + n_parts + 1)));
  unsigned long long* first = hist + ntiles * n_parts;
  DISPATCH_W(s->W, shard_export(s, m, n_parts, ntiles, hist, first, static_cast<uint64_t*>(d_rows)));
  std::vector<unsigned long long> h_first(n_parts + 1);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h_first.data(), first, sizeof(unsigned long long) * (n_parts + 1), cudaMemcpyDeviceToHost,
                        s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  pool_free(hist);
  if (e != cudaSuccess) {
    s->poisoned = true;
    return fail(PPVM_ECUDA, std::string("shard export: ") + cudaGetErrorString(e));
  }
  for (uint32_t p = 0; p < n_parts; ++p) counts[p] = h_first[p + 1] - h_first[p];
  s->xfer_d2h += sizeof(unsigned long long) * (n_parts + 1);
  s->n_host = 0;
  s->n_ub = 0;
  return PPVM_OK;
}

ppvm_status ppvm_sum_shard_append(ppvm_sum* s, const void* d_rows, size_t k) {
  if (!s) return fail(PPVM_EINVAL, "null sum");
  REQUIRE_USABLE(s);
  if (k == 0) return PPVM_OK;
  if (!d_rows) return fail(PPVM_EINVAL, "null row buffer");
  PPVM_TRY(ensure_device(s->device));
  if (s->n_host + k > s->cap) PPVM_TRY(grow(s, std::max<unsigned long long>(2 * s->cap, s->n_host + k + 1024)));
  DISPATCH_W(s->W, shard_append(s, static_cast<const uint64_t*>(d_rows), k));
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);  // the caller may free the rows on return
  if (e != cudaSuccess) {
    s->poisoned = true;
    return fail(PPVM_ECUDA, std::string("shard append: ") + cudaGetErrorString(e));
  }
  s->n_host += k;
  s->n_ub = s->n_host;
  return PPVM_OK;
}

ppvm_status ppvm_sum_add_string(ppvm_sum* s, const char* word, double c) {
  if (!s || !word) return fail(PPVM_EINVAL, "null argument");
  std::vector<uint64_t> x(s->W, 0), z(s->W, 0);
  uint32_t q = 0;
  for (const char* p = word; *p; ++p) {
    const char ch = *p;
    if (ch == '_') continue;
    if (q >= s->n) return fail(PPVM_EINVAL, "word longer than n_qubits");
    const uint64_t b = 1ull << (q & 63);
    if (ch == 'X') x[q >> 6] |= b;
    else if (ch == 'Z') z[q >> 6] |= b;
    else if (ch == 'Y') { x[q >> 6] |= b; z[q >> 6] |= b; }
    else if (ch == 'L' && s->lossy) x[s->wr + (q >> 6)] |= b;
    else if (ch != 'I') return fail(PPVM_EINVAL, std::string("Invalid Pauli character: ") + ch);
    ++q;
  }
  if (q != s->n) return fail(PPVM_EINVAL, "word length differs from n_qubits");
  return ppvm_sum_add_terms(s, x.data(), z.data(), &c, 1);
}

ppvm_status ppvm_sum_set_preserve(ppvm_sum* s, const uint64_t* x, const uint64_t* z, size_t k) {
  if (!s) return fail(PPVM_EINVAL, "null sum");
  if (k > (size_t)kMaxPreserve) return fail(PPVM_EINVAL, "at most 1023 preserve strings are supported");
  if (k && (!x || !z)) return fail(PPVM_EINVAL, "null preserve arrays");
  PPVM_TRY(ensure_device(s->device));
  const int W = s->W;
  cudaFree(s->d_pres_keys);
  cudaFree(s->d_pres_table);
  s->d_pres_keys = nullptr;
  s->d_pres_table = nullptr;
  s->npres = 0;
  s->h_pres.clear();
  if (k == 0) return PPVM_OK;
  // de-duplicate (a HashSet in the reference builder, data.rs:75-77)
  std::vector<uint64_t> keys;
  for (size_t i = 0; i < k; ++i) {
    bool dup = false;
    for (size_t j = 0; j < keys.size() / (2 * W) && !dup; ++j) {
      bool eq = true;
      for (int w = 0; w < W; ++w) eq &= keys[j * 2 * W + w] == x[i * W + w] && keys[j * 2 * W + W + w] == z[i * W + w];
      dup = eq;
    }
    if (dup) continue;
    for (int w = 0; w < W; ++w) keys.push_back(x[i * W + w]);
    for (int w = 0; w < W; ++w) keys.push_back(z[i * W + w]);
  }
  const int np = (int)(keys.size() / (2 * W));
  const unsigned tsize = 2048;
  std::vector<int> table(tsize, -1);
  for (int j = 0; j < np; ++j) {
    unsigned slot = (unsigned)(h_hash_key(&keys[(size_t)j * 2 * W], &keys[(size_t)j * 2 * W + W], W) & (tsize - 1));
    while (table[slot] >= 0) slot = (slot + 1) & (tsize - 1);
    table[slot] = j;
  }
  CUDA_TRY(cudaMalloc(&s->d_pres_keys, sizeof(uint64_t) * keys.size()));
  CUDA_TRY(cudaMalloc(&s->d_pres_table, sizeof(int) * tsize));
  CUDA_TRY(cudaMemcpyAsync(s->d_pres_keys, keys.data(), sizeof(uint64_t) * keys.size(), cudaMemcpyHostToDevice, s->stream));
  CUDA_TRY(cudaMemcpyAsync(s->d_pres_table, table.data(), sizeof(int) * tsize, cudaMemcpyHostToDevice, s->stream));
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  s->pres_mask = tsize - 1;
  s->npres = np;
  s->h_pres = keys;
  return PPVM_OK;
}

ppvm_status ppvm_export_terms(const ppvm_sum* cs, uint64_t* x, uint64_t* z, double* c, size_t cap, size_t* n_out) {
  if (!cs || !n_out) return fail(PPVM_EINVAL, "null argument");
  REQUIRE_USABLE(cs);
  ppvm_sum* s = const_cast<ppvm_sum*>(cs);
  PPVM_TRY(ensure_device(s->device));
  const size_t n = std::min<size_t>(cap, s->n_host);
  *n_out = n;
  if (n == 0) return PPVM_OK;
  if (!x || !z || !c) return fail(PPVM_EINVAL, "null output arrays");
  const int W = s->W;
  std::vector<uint64_t> buf((size_t)(2 * W) * n);
  for (int w = 0; w < 2 * W; ++w)
    CUDA_TRY(cudaMemcpyAsync(buf.data() + (size_t)w * n, s->planes + (size_t)w * s->cap, sizeof(uint64_t) * n,
                             cudaMemcpyDeviceToHost, s->stream));
  CUDA_TRY(cudaMemcpyAsync(c, s->planes + (size_t)2 * W * s->cap, sizeof(double) * n, cudaMemcpyDeviceToHost,
                           s->stream));
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  for (size_t i = 0; i < n; ++i)
    for (int w = 0; w < W; ++w) {
      x[i * W + w] = buf[(size_t)w * n + i];
      z[i * W + w] = buf[(size_t)(W + w) * n + i];
    }
  return PPVM_OK;
}

ppvm_status ppvm_weights(const ppvm_sum* cs, uint32_t* w, size_t cap, size_t* n_out) {
  if (!cs || !n_out) return fail(PPVM_EINVAL, "null argument");
  REQUIRE_USABLE(cs);
  ppvm_sum* s = const_cast<ppvm_sum*>(cs);
  PPVM_TRY(ensure_device(s->device));
  const size_t n = std::min<size_t>(cap, s->n_host);
  *n_out = n;
  if (n == 0) return PPVM_OK;
  if (!w) return fail(PPVM_EINVAL, "null output array");
  uint32_t* d = reinterpret_cast<uint32_t*>(s->s_idx);  // scratch, cap entries
  DISPATCH_W(s->W, weights(s, d));
  CUDA_TRY(cudaMemcpyAsync(w, d, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s->stream));
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  return PPVM_OK;
}

ppvm_status ppvm_current_max_weight(const ppvm_sum* s, uint64_t* out) {
  if (!s || !out) return fail(PPVM_EINVAL, "null argument");
  std::vector<uint32_t> w(s->n_host);
  size_t n = 0;
  PPVM_TRY(ppvm_weights(s, w.data(), w.size(), &n));
  uint64_t m = 0;
  for (size_t i = 0; i < n; ++i) m = std::max<uint64_t>(m, w[i]);
  *out = m;
  return PPVM_OK;
}

#define GATE1(name, CODE)                                                                     \
  ppvm_status name(ppvm_sum* s, const uint32_t* t, size_t k, int truncate) {                  \
    return run_gate(s, CODE, t, k, false, 0.0, nullptr, truncate);                            \
  }
#define GATE2(name, CODE)                                                                     \
  ppvm_status name(ppvm_sum* s, const uint32_t* t, size_t k, int truncate) {                  \
    return run_gate(s, CODE, t, k, true, 0.0, nullptr, truncate);                             \
  }
#define ROT1(name, CODE)                                                                      \
  ppvm_status name(ppvm_sum* s, const uint32_t* t, size_t k, double theta, int truncate) {    \
    return run_gate(s, CODE, t, k, false, theta, nullptr, truncate);                          \
  }
#define ROT2(name, CODE)                                                                      \
  ppvm_status name(ppvm_sum* s, const uint32_t* t, size_t k, double theta, int truncate) {    \
    return run_gate(s, CODE, t, k, true, theta, nullptr, truncate);                           \
  }

GATE1(ppvm_x, PPVM_OP_X)
GATE1(ppvm_y, PPVM_OP_Y)
GATE1(ppvm_z, PPVM_OP_Z)
GATE1(ppvm_h, PPVM_OP_H)
GATE1(ppvm_s, PPVM_OP_S)
GATE1(ppvm_s_dag, PPVM_OP_S_DAG)
GATE1(ppvm_sqrt_x, PPVM_OP_SQRT_X)
GATE1(ppvm_sqrt_x_dag, PPVM_OP_SQRT_X_DAG)
GATE1(ppvm_sqrt_y, PPVM_OP_SQRT_Y)
GATE1(ppvm_sqrt_y_dag, PPVM_OP_SQRT_Y_DAG)
GATE2(ppvm_cnot, PPVM_OP_CNOT)
GATE2(ppvm_cz, PPVM_OP_CZ)
GATE2(ppvm_cy, PPVM_OP_CY)
ROT1(ppvm_rx, PPVM_OP_RX)
ROT1(ppvm_ry, PPVM_OP_RY)
ROT1(ppvm_rz, PPVM_OP_RZ)
ROT2(ppvm_rxx, PPVM_OP_RXX)
ROT2(ppvm_ryy, PPVM_OP_RYY)
ROT2(ppvm_rzz, PPVM_OP_RZZ)

ppvm_status ppvm_r(ppvm_sum* s, uint32_t q, double axis_angle, double theta, int truncate) {
  if (!s) return fail(PPVM_EINVAL, "null sum");
  ppvm_op ops[4];
  std::memset(ops, 0, sizeof(ops));
  ops[0].code = PPVM_OP_RZ; ops[0].q0 = q; ops[0].theta = axis_angle;
  ops[1].code = PPVM_OP_RX; ops[1].q0 = q; ops[1].theta = theta;
  ops[2].code = PPVM_OP_RZ; ops[2].q0 = q; ops[2].theta = -axis_angle;
  ops[3].code = PPVM_OP_TRUNCATE;
  for (int i = 0; i < 3; ++i) PPVM_TRY(validate(s, ops[i]));
  return run_list(s, ops, truncate ? 4 : 3, {});
}

ppvm_status ppvm_pauli_error(ppvm_sum* s, const uint32_t* t, size_t k, const double p[3], int truncate) {
  if (!p) return fail(PPVM_EINVAL, "null probabilities");
  return run_gate(s, PPVM_OP_PAULI_ERROR, t, k, false, 0.0, p, truncate);
}
ppvm_status ppvm_depolarize1(ppvm_sum* s, const uint32_t* t, size_t k, double p, int truncate) {
  return run_gate(s, PPVM_OP_DEPOLARIZE1, t, k, false, p, nullptr, truncate);
}
ppvm_status ppvm_depolarize2(ppvm_sum* s, const uint32_t* t, size_t k, double p, int truncate) {
  return run_gate(s, PPVM_OP_DEPOLARIZE2, t, k, true, p, nullptr, truncate);
}

// Loss channels of lossy sums (noise.rs:165-275), one call per target list like the other
// channels: the reference's Python binding applies each to one qubit (or pair) and truncates.
ppvm_status ppvm_loss_channel(ppvm_sum* s, const uint32_t* t, size_t k, double p, int truncate) {
  return run_gate(s, PPVM_OP_LOSS_CHANNEL, t, k, false, p, nullptr, truncate);
}
ppvm_status ppvm_reset_loss_channel(ppvm_sum* s, const uint32_t* t, size_t k, int truncate) {
  return run_gate(s, PPVM_OP_RESET_LOSS_CHANNEL, t, k, false, 0.0, nullptr, truncate);
}
ppvm_status ppvm_correlated_loss_channel(ppvm_sum* s, const uint32_t* t, size_t k, const double p[3],
                                         int truncate) {
  if (!p) return fail(PPVM_EINVAL, "null probabilities");
  return run_gate(s, PPVM_OP_CORRELATED_LOSS_CHANNEL, t, k, true, 0.0, p, truncate);
}
ppvm_status ppvm_sum_set_max_loss_weight(ppvm_sum* s, uint64_t max_loss_weight) {
  if (!s) return fail(PPVM_EINVAL, "null sum");
  if (!s->lossy && max_loss_weight != UINT64_MAX)
    return fail(PPVM_EINVAL, "a loss-weight cap needs a lossy sum (PPVM_FLAG_LOSSY)");
  s->maxlw = max_loss_weight;
  return PPVM_OK;
}

// The factor of each (P_a, P_b), code x | z << 1 per qubit, is 1 - 2 p[i1] - ... - 2 p[i8] over
// the eight two-qubit Paulis that anticommute with it, subtracted in the order the reference
// writes them (noise.rs:50-99; the order fixes the rounding).  p indices name IX IY IZ XI XX
// XY XZ YI YX YY YZ ZI ZX ZY ZZ.
static void perr2_factors(const double p[15], double f[16]) {
  static const int8_t kOrder[16][8] = {
      {0},                              // II: unchanged
      {1, 10, 13, 14, 2, 5, 6, 9},      // IX
      {0, 1, 12, 13, 4, 5, 8, 9},       // IZ
      {0, 10, 12, 14, 2, 4, 6, 8},      // IY
      {10, 11, 12, 13, 14, 7, 8, 9},    // XI
      {1, 11, 12, 2, 5, 6, 7, 8},       // XX
      {0, 1, 10, 11, 14, 4, 5, 7},      // XZ
      {0, 11, 13, 2, 4, 6, 7, 9},       // XY
      {10, 3, 4, 5, 6, 7, 8, 9},        // ZI
      {1, 13, 14, 2, 3, 4, 7, 8},       // ZX
      {0, 1, 10, 12, 13, 3, 6, 7},      // ZZ
      {0, 12, 14, 2, 3, 5, 7, 9},       // ZY
      {11, 12, 13, 14, 3, 4, 5, 6},     // YI
      {1, 10, 11, 12, 2, 3, 4, 9},      // YX
      {0, 1, 11, 14, 3, 6, 8, 9},       // YZ
      {0, 10, 11, 13, 2, 3, 5, 8}};     // YY
  f[0] = 1.0;
  for (int code = 1; code < 16; ++code) {
    double acc = 1.0;
    for (int t = 0; t < 8; ++t) acc = acc - p[kOrder[code][t]] * 2.0;
    f[code] = acc;
  }
}

ppvm_status ppvm_two_qubit_pauli_error(ppvm_sum* s, const uint32_t* t, size_t k, const double p[15],
                                       int truncate) {
  if (!s) return fail(PPVM_EINVAL, "null sum");
  if (!p || (k && !t)) return fail(PPVM_EINVAL, "null argument");
  if (k % 2) return fail(PPVM_EINVAL, "two-qubit operations require an even number of targets");
  std::vector<ppvm_op> ops;
  for (size_t i = 0; i < k; i += 2) {
    if (t[i] >= s->n || t[i + 1] >= s->n || t[i] == t[i + 1])
      return fail(PPVM_EINVAL, "two-qubit op needs two distinct qubits in range");
    ppvm_op op;
    std::memset(&op, 0, sizeof(op));
    op.code = kOpPauliError2;
    op.q0 = t[i];
    op.q1 = t[i + 1];
    op.theta = 0.0;  // every pair of the call uses table 0
    ops.push_back(op);
  }
  if (truncate) {
    ppvm_op op;
    std::memset(&op, 0, sizeof(op));
    op.code = PPVM_OP_TRUNCATE;
    ops.push_back(op);
  }
  if (ops.empty()) return PPVM_OK;
  s->perr2_host.assign(16, 0.0);
  perr2_factors(p, s->perr2_host.data());
  const ppvm_status st = run_list(s, ops.data(), ops.size(), {});
  s->perr2_host.clear();
  return st;
}

ppvm_status ppvm_amplitude_damping(ppvm_sum* s, uint32_t q, double gamma, int truncate) {
  return run_gate(s, PPVM_OP_AMPLITUDE_DAMPING, &q, 1, false, gamma, nullptr, truncate);
}

ppvm_status ppvm_pauli_rotation(ppvm_sum* s, const uint64_t* gx, const uint64_t* gz, double theta, int truncate) {
  if (!s || !gx || !gz) return fail(PPVM_EINVAL, "null argument");
  const int W = s->W, wr = s->wr;
  const int tail = (int)(s->n % 64);
  if (tail && ((gx[wr - 1] | gz[wr - 1]) >> tail)) return fail(PPVM_EINVAL, "generator has bits at or above n_qubits");
  for (int w = wr; w < W; ++w)
    if (gx[w] | gz[w]) return fail(PPVM_EINVAL, "a generator has no loss bits (the upper words must be 0)");
  bool any = false;
  for (int w = 0; w < W; ++w) any |= (gx[w] | gz[w]) != 0;
  std::vector<Gen> gens(1);
  std::memset(&gens[0], 0, sizeof(Gen));
  for (int w = 0; w < W; ++w) {
    gens[0].gx[w] = gx[w];
    gens[0].gz[w] = gz[w];
  }
  gens[0].lw = s->lossy ? (uint32_t)wr : 0u;
  std::vector<ppvm_op> ops;
  if (any) {
    if (is_clifford_angle(s, theta)) {
      // Clifford-angle generic rotation: run it through the rotation pipeline with cos = 0
      // is not equivalent (the parent would remain with coefficient 0); lower to ops when the
      // support is 1-2 qubits, else reject.
      std::vector<uint32_t> sup;
      for (uint32_t q = 0; q < s->n; ++q)
        if (((gx[q >> 6] | gz[q >> 6]) >> (q & 63)) & 1) sup.push_back(q);
      if (sup.size() > 2) return fail(PPVM_EINVAL, "Clifford-angle mode supports generic rotations on <= 2 qubits");
      auto axis = [&](uint32_t q) { return (int)((gx[q >> 6] >> (q & 63)) & 1) | ((int)((gz[q >> 6] >> (q & 63)) & 1) << 1); };
      ppvm_op op;
      std::memset(&op, 0, sizeof(op));
      op.theta = theta;
      op.q0 = sup[0];
      if (sup.size() == 1) {
        const int a = axis(sup[0]);
        op.code = a == 1 ? PPVM_OP_RX : a == 2 ? PPVM_OP_RZ : PPVM_OP_RY;
      } else {
        const int a = axis(sup[0]), b = axis(sup[1]);
        if (a != b) return fail(PPVM_EINVAL, "Clifford-angle mode supports XX, YY, ZZ two-qubit generators");
        op.q1 = sup[1];
        op.code = a == 1 ? PPVM_OP_RXX : a == 2 ? PPVM_OP_RZZ : PPVM_OP_RYY;
      }
      ops.push_back(op);
    } else {
      ppvm_op op;
      std::memset(&op, 0, sizeof(op));
      op.code = PPVM_OP_RX;  // placeholder code; flags = 1 selects gens[q0]
      op.flags = 1;
      op.q0 = 0;
      op.theta = theta;
      ops.push_back(op);
    }
  }
  if (truncate) {
    ppvm_op op;
    std::memset(&op, 0, sizeof(op));
    op.code = PPVM_OP_TRUNCATE;
    ops.push_back(op);
  }
  if (ops.empty()) return PPVM_OK;
  return run_list(s, ops.data(), ops.size(), gens);
}

ppvm_status ppvm_truncate(ppvm_sum* s) {
  if (!s) return fail(PPVM_EINVAL, "null sum");
  ppvm_op op;
  std::memset(&op, 0, sizeof(op));
  op.code = PPVM_OP_TRUNCATE;
  return run_list(s, &op, 1, {});
}

ppvm_status ppvm_gate_list_run(ppvm_sum* s, const ppvm_op* ops, size_t n_ops) {
  if (!s) return fail(PPVM_EINVAL, "null sum");
  if (n_ops && !ops) return fail(PPVM_EINVAL, "null op list");
  for (size_t i = 0; i < n_ops; ++i) {
    if (ops[i].flags != 0) return fail(PPVM_EINVAL, "op flags must be 0");
    PPVM_TRY(validate(s, ops[i]));
  }
  if (n_ops == 0) return PPVM_OK;
  return run_list(s, ops, n_ops, {});
}

ppvm_status ppvm_last_run_live_counts(const ppvm_sum* s, uint64_t* counts, size_t cap, size_t* n_out) {
  if (!s || !n_out) return fail(PPVM_EINVAL, "null argument");
  *n_out = s->last_nops;
  const size_t n = std::min(cap, s->last_nops);
  if (n && !counts) return fail(PPVM_EINVAL, "null output");
  for (size_t i = 0; i < n; ++i) counts[i] = s->h_log[i].n_in;
  return PPVM_OK;
}

ppvm_status ppvm_overlap_with_zero(ppvm_sum* s, double* out) {
  if (!s || !out) return fail(PPVM_EINVAL, "null argument");
  REQUIRE_USABLE(s);
  PPVM_TRY(ensure_device(s->device));
  return do_reduce_owz(s, out);
}

ppvm_status ppvm_expectation(ppvm_sum* s, double* out) { return ppvm_overlap_with_zero(s, out); }

ppvm_status ppvm_trace(ppvm_sum* s, const char* pattern, double* out) {
  if (!s || !pattern || !out) return fail(PPVM_EINVAL, "null argument");
  REQUIRE_USABLE(s);
  std::vector<PatItem> items;
  if (!parse_pattern(pattern, items)) return fail(PPVM_EINVAL, std::string("bad Pauli pattern: ") + pattern);
  PPVM_TRY(ensure_device(s->device));
  if (items.size() == 1 && items[0].kind == 1 && items[0].accept == (1u | 4u))  // "Z?*"
    return do_reduce_owz(s, out);
  cudaFree(s->d_pat);
  s->d_pat = nullptr;
  CUDA_TRY(cudaMalloc(&s->d_pat, sizeof(PatItem) * std::max<size_t>(items.size(), 1)));
  if (!items.empty())
    CUDA_TRY(cudaMemcpyAsync(s->d_pat, items.data(), sizeof(PatItem) * items.size(), cudaMemcpyHostToDevice, s->stream));
  const int nb = (int)grid_for(std::max<unsigned long long>(s->n_host, 1), kRedBlock * 4, 2);
  DISPATCH_W(s->W, trace(s, nb, (int)items.size()));
  CUDA_TRY(cudaGetLastError());
  PPVM_TRY(sync_state(s, 0));
  *out = s->h_ctrl->sum;
  return PPVM_OK;
}

ppvm_status ppvm_overlap(ppvm_sum* a, ppvm_sum* b, double* out) {
  if (!a || !b || !out) return fail(PPVM_EINVAL, "null argument");
  REQUIRE_USABLE(a);
  REQUIRE_USABLE(b);
  if (a->n != b->n) return fail(PPVM_EINVAL, "sums have different qubit counts");
  if (a->device != b->device) return fail(PPVM_EINVAL, "sums live on different devices");
  PPVM_TRY(ensure_device(a->device));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  unsigned long long mask;
  unsigned ep;
  PPVM_TRY(build_index(a, a->n_host, &mask, &ep));
  CUDA_TRY(cudaMemsetAsync(a->d_counter, 0, sizeof(unsigned long long), a->stream));
  const int nb = (int)grid_for(std::max<unsigned long long>(b->n_host, 1), kRedBlock * 4, 2);
  DISPATCH_W(a->W, overlap(a, b, mask, ep, nb, a->d_counter));
  CUDA_TRY(cudaGetLastError());
  PPVM_TRY(sync_state(a, 0));
  *out = a->h_ctrl->sum;
  return PPVM_OK;
}

ppvm_status ppvm_equal(const ppvm_sum* ca, const ppvm_sum* cb, int* out) {
  if (!ca || !cb || !out) return fail(PPVM_EINVAL, "null argument");
  REQUIRE_USABLE(ca);
  REQUIRE_USABLE(cb);
  ppvm_sum* a = const_cast<ppvm_sum*>(ca);
  ppvm_sum* b = const_cast<ppvm_sum*>(cb);
  *out = 0;
  if (a->n != b->n || a->n_host != b->n_host) return PPVM_OK;
  if (a->n_host == 0) {
    *out = 1;
    return PPVM_OK;
  }
  PPVM_TRY(ensure_device(a->device));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  unsigned long long mask;
  unsigned ep;
  PPVM_TRY(build_index(a, a->n_host, &mask, &ep));
  CUDA_TRY(cudaMemsetAsync(a->d_counter, 0, sizeof(unsigned long long), a->stream));
  const int nb = (int)grid_for(std::max<unsigned long long>(b->n_host, 1), kRedBlock * 4, 2);
  DISPATCH_W(a->W, overlap(a, b, mask, ep, nb, a->d_counter));
  unsigned long long miss = 1;
  CUDA_TRY(cudaMemcpyAsync(&miss, a->d_counter, sizeof(miss), cudaMemcpyDeviceToHost, a->stream));
  CUDA_TRY(cudaStreamSynchronize(a->stream));
  *out = miss == 0 ? 1 : 0;
  return PPVM_OK;
}

ppvm_status ppvm_clifford_tableau(uint32_t n_qubits, const ppvm_op* ops, size_t n_ops, uint64_t* img_x,
                                  uint64_t* img_z, uint8_t* sign) {
  if (n_qubits == 0 || n_qubits > 64 * kMaxW) return fail(PPVM_EINVAL, "n_qubits must be in [1, 512]");
  if ((n_ops && !ops) || !img_x || !img_z || !sign) return fail(PPVM_EINVAL, "null argument");
  ppvm_sum probe;  // validation only: qubit range and Clifford-angle rule
  probe.n = n_qubits;
  probe.flags = PPVM_FLAG_CLIFFORD_ANGLES;
  std::vector<DevOp> d;
  for (size_t i = 0; i < n_ops; ++i) {
    PPVM_TRY(validate(&probe, ops[i]));
    if (!is_local(&probe, ops[i]) || ops[i].flags != 0)
      return fail(PPVM_EINVAL, "ppvm_clifford_tableau takes Clifford ops and rotations at +-pi/2 only");
    d.push_back(to_devop(ops[i]));
    if (!is_cliff_code(d.back().code)) return fail(PPVM_EINVAL, "noise channels are not Clifford maps");
  }
  const int W = (int)((n_qubits + 63) / 64);
  for (uint32_t q = 0; q < n_qubits; ++q)
    for (int p = 0; p < 2; ++p) {
      const size_t row = 2 * (size_t)q + p;
      for (int w = 0; w < W; ++w) img_x[row * W + w] = img_z[row * W + w] = 0;
      (p == 0 ? img_x : img_z)[row * W + (q >> 6)] = 1ull << (q & 63);
      sign[row] = 0;
    }
  if (d.empty()) return PPVM_OK;
  HostTableau t;
  compose_tableau(W, d.data(), (int)d.size(), t);
  for (size_t c = 0; c < t.tq.size(); ++c)
    for (int p = 0; p < 2; ++p) {
      const size_t row = 2 * (size_t)t.tq[c] + p, trow = 2 * c + p;
      for (int w = 0; w < W; ++w) {
        img_x[row * W + w] = t.rows[trow * 2 * W + w];
        img_z[row * W + w] = t.rows[trow * 2 * W + W + w];
      }
      sign[row] = t.sign[trow];
    }
  return PPVM_OK;
}

ppvm_status ppvm_transfer_counters(const ppvm_sum* s, uint64_t* h2d_bytes, uint64_t* d2h_bytes) {
  if (!s || !h2d_bytes || !d2h_bytes) return fail(PPVM_EINVAL, "null argument");
  *h2d_bytes = s->xfer_h2d;
  *d2h_bytes = s->xfer_d2h;
  return PPVM_OK;
}

ppvm_status ppvm_launch_count(const ppvm_sum* s, uint64_t* out) {
  if (!s || !out) return fail(PPVM_EINVAL, "null argument");
  *out = s->launch_count;
  return PPVM_OK;
}

ppvm_status ppvm_term_features(ppvm_sum* s, uint32_t lattice_l, uint32_t layers_left, float* out, size_t cap,
                               size_t* n_out) {
  if (!s || !n_out) return fail(PPVM_EINVAL, "null argument");
  REQUIRE_USABLE(s);
  if (lattice_l > 0 && (uint64_t)lattice_l * lattice_l > s->n) return fail(PPVM_EINVAL, "lattice larger than the sum");
  PPVM_TRY(ensure_device(s->device));
  const size_t n = std::min<size_t>(cap, s->n_host);
  *n_out = n;
  if (n == 0) return PPVM_OK;
  if (!out) return fail(PPVM_EINVAL, "null output");
  float* d = nullptr;
  CUDA_TRY(cudaMalloc(&d, sizeof(float) * kMlpIn * std::max<unsigned long long>(s->n_host, 1)));
  DISPATCH_W(s->W, features(s, (int)lattice_l, (int)layers_left, d));
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, sizeof(float) * kMlpIn * n, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  cudaFree(d);
  if (e != cudaSuccess) return fail(PPVM_ECUDA, std::string("term features: ") + cudaGetErrorString(e));
  s->xfer_d2h += sizeof(float) * kMlpIn * n;
  return PPVM_OK;
}

ppvm_status ppvm_truncate_budget(ppvm_sum* s, uint64_t budget, const ppvm_mlp* mlp, uint32_t lattice_l,
                                 uint32_t layers_left, int digit_bits) {
  if (!s) return fail(PPVM_EINVAL, "null sum");
  if (digit_bits == 0) digit_bits = 8;
  if (digit_bits != 8 && digit_bits != 11) return fail(PPVM_EINVAL, "digit_bits must be 8 or 11");
  if (lattice_l > 0 && (uint64_t)lattice_l * lattice_l > s->n) return fail(PPVM_EINVAL, "lattice larger than the sum");
  if (s->poisoned) return fail(PPVM_ECUDA, "sum is in an error state from an earlier failure");
  PPVM_TRY(ensure_device(s->device));
  const MlpWeights* mw = nullptr;
  if (mlp) {
    if (mlp_device(mlp) != s->device) return fail(PPVM_EINVAL, "network and sum live on different devices");
    mw = mlp_device_weights(mlp);
  }
  if (s->n_host <= budget) return PPVM_OK;
  DISPATCH_W(s->W, budget(s, budget, mw, (int)lattice_l, (int)layers_left, digit_bits));
  CUDA_TRY(cudaGetLastError());
  PPVM_TRY(sync_state(s, 0));
  if (s->h_ctrl->err) {
    s->poisoned = true;
    return fail(PPVM_ECUDA, "device error in budget truncation");
  }
  s->n_host = s->h_ctrl->n;
  s->n_ub = s->n_host;
  return PPVM_OK;
}

ppvm_status ppvm_release_cached_memory(void) {
  int cur = 0;
  cudaGetDevice(&cur);
  std::vector<ppvm_sum*> handles;
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    handles.swap(g_sum_cache);
  }
  for (ppvm_sum* h : handles) destroy_now(h);  // their buffers go back to the pool first
  ppvm::release_batch_staging();
  std::lock_guard<std::mutex> lk(g_pool_mu);
  for (int d = 0; d < 64; ++d) {
    if (g_pool_free[d].empty()) continue;
    if (cudaSetDevice(d) == cudaSuccess) pool_release_device(d);
  }
  cudaSetDevice(cur);
  return PPVM_OK;
}

ppvm_status ppvm_profile_enable(ppvm_sum* s, int on) {
  if (!s) return fail(PPVM_EINVAL, "null sum");
  s->prof = on != 0;
  if (on) {
    for (int f = 0; f < F_COUNT; ++f) {
      s->prof_ms[f] = 0;
      s->prof_launches[f] = 0;
      s->prof_bytes[f] = 0;
    }
  }
  return PPVM_OK;
}

ppvm_status ppvm_profile_read(ppvm_sum* s, char* names, size_t names_cap, double* ms, uint64_t* launches,
                              uint64_t* bytes, size_t cap, size_t* n_out) {
  if (!s || !n_out) return fail(PPVM_EINVAL, "null argument");
  *n_out = F_COUNT;
  std::string all;
  for (int f = 0; f < F_COUNT; ++f) {
    all += kFamilyNames[f];
    all.push_back('\0');
  }
  if (names && names_cap) std::memcpy(names, all.data(), std::min(names_cap, all.size()));
  for (size_t f = 0; f < std::min<size_t>(cap, F_COUNT); ++f) {
    if (ms) ms[f] = s->prof_ms[f];
    if (launches) launches[f] = s->prof_launches[f];
    if (bytes) bytes[f] = s->prof_bytes[f];
  }
  return PPVM_OK;
}

}  // extern "C"
