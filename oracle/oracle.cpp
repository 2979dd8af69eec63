// oracle/oracle.cpp — TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement of the reference's PauliSum hot path (QuEraComputing/ppvm,
// crate `ppvm-pauli-sum`).  It is the checker the GPU engine is compared against and
// the CPU baseline that bench.py times.  Nothing in the product (ppvm_b200/) links,
// loads or calls it.
//
// Two map configurations of the reference are restated, behind the same gate code:
//  * IndexMap + FxHash, single-threaded: the configuration the Python binding uses
//    (crates/ppvm-python-native/src/interface.rs:414).  Term order is the reference's
//    insertion order; every parity test compares against this one.
//  * DashMap + FxHash with rayon (crates/ppvm-pauli-sum/src/config/dashmap.rs,
//    crates/ppvm-traits/src/map/dashmap.rs): the reference's multi-threaded
//    configuration, restated with a pool of host threads.  Same terms and coefficients (a merged key
//    takes at most two contributions per gate, so the sum does not depend on order);
//    term order is per-shard.  bench.py's reference arm times it on every host core.
//
// The reference is Rust and cannot be compiled in this environment (no cargo/rustc),
// so this file restates it.  It is pinned by the reference's own golden values and
// truth tables (tests/test_oracle_golden.py): crates/ppvm-pauli-sum/tests/trotter.rs:104,
// tests/cnot.rs:27, tests/ghz.rs, src/sum/rot1.rs:186-310, src/sum/rot2.rs:266-350,
// crates/ppvm-pauli-word/src/phase/clifford.rs:184-374, tests/strategy.rs,
// tests/truncation_semantics.rs, tests/preserve.rs, and an independent numpy
// state-vector check of Heisenberg propagation.
//
// Semantics restated (file:line in the reference):
//  * storage: a map word -> f64.  IndexMap: new keys append; `+=` on an existing key
//    modifies in place (crates/ppvm-traits/src/map/hashmap.rs:40-44); `retain` keeps
//    order (hashmap.rs:242-258 -> IndexMap::retain).
//  * rotations: map_insert (crates/ppvm-pauli-sum/src/sum/data.rs:204-226): every
//    anticommuting parent is scaled in place by cos and its child (word, v*(eps*sin)) is
//    pushed to a scratch Vec in iteration order; then the scratch is merged with `+=`,
//    one key after the other.
//  * Cliffords: scale (in place, data.rs:192-197) for X/Y/Z; map_add (data.rs:255-265,
//    hashmap.rs:46-54): aux cleared, every entry mapped into aux, data and aux swapped.
//  * truncate: data.rs:275-311 with CombinedStrategy(CoefficientThreshold, MaxPauliWeight)
//    (crates/ppvm-pauli-sum/src/strategy.rs:12-30, 73-90, 125-134).
//  * trace: fold in iteration order (hashmap.rs:108-127) with the PauliPattern matcher
//    (crates/ppvm-pauli-word/src/pattern/parse.rs:32-127, contains.rs:19-151).
//
// Build: `make -C oracle` (g++ -O2 -ffp-contract=off -pthread); the library is
// oracle/_build/liboracle.so.

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "../include/ppvm_cuda.h"

namespace {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;

inline uint64_t rotl(uint64_t v, int r) { return (v << r) | (v >> (64 - r)); }

// FxHash-style word hash (the reference hashes the raw storage bytes with FxHasher,
// crates/ppvm-pauli-word/src/word/data.rs:184-200).  Only speed and the DashMap shard a
// key lives in depend on it.
inline uint64_t fx_hash(const uint64_t* k, int nw) {
  uint64_t h = 0;
  for (int i = 0; i < nw; ++i) h = (rotl(h, 5) ^ k[i]) * 0x517cc1b727220a95ull;
  return h ^ (h >> 32);
}

inline uint64_t table_cap_for(size_t entries) {
  uint64_t cap = 16;
  while (cap < 2 * (uint64_t)entries + 2) cap <<= 1;
  return cap;
}

// Word geometry and the strategy, shared by both map configurations.  A key is the X
// plane's W words followed by the Z plane's W words; a lossy word (LossyPauliWord,
// crates/ppvm-pauli-word/src/loss/data.rs:33-44) adds its loss plane's W words.  A lost qubit
// (Pauli::L) has x = z = 0 and l = 1 (data.rs:218-230).
struct Words {
  uint32_t n = 0;
  int W = 1;  // words per plane
  double thr = 1e-10;
  uint64_t maxw = UINT64_MAX;
  uint64_t maxlw = UINT64_MAX;  // MaxLossWeight (strategy.rs:145-180)
  bool clifford_angles = false;
  bool lossy = false;
  std::vector<uint64_t> preserve;  // flat [j][kw()]

  int kw() const { return (lossy ? 3 : 2) * W; }
  size_t kb() const { return sizeof(uint64_t) * kw(); }
  bool get_x(const uint64_t* k, uint32_t q) const { return (k[q >> 6] >> (q & 63)) & 1u; }
  bool get_z(const uint64_t* k, uint32_t q) const { return (k[W + (q >> 6)] >> (q & 63)) & 1u; }
  bool get_l(const uint64_t* k, uint32_t q) const {
    return lossy && ((k[2 * W + (q >> 6)] >> (q & 63)) & 1u);
  }
  static void set_bit(uint64_t* w, uint32_t q, bool b) {
    uint64_t m = 1ull << (q & 63);
    if (b) w[q >> 6] |= m; else w[q >> 6] &= ~m;
  }
  void set_x(uint64_t* k, uint32_t q, bool b) const { set_bit(k, q, b); }
  void set_z(uint64_t* k, uint32_t q, bool b) const { set_bit(k + W, q, b); }
  void set_l(uint64_t* k, uint32_t q, bool b) const { set_bit(k + 2 * W, q, b); }
  // Pauli::I/X/Z/Y/L on qubit q: the reference's `k.set(q, pauli)` (data.rs:255-283)
  void set_code(uint64_t* k, uint32_t q, int code) const {  // 0 I, 1 X, 2 Z, 3 Y, 4 L
    set_x(k, q, code == 1 || code == 3);
    set_z(k, q, code == 2 || code == 3);
    if (lossy) set_l(k, q, code == 4);
  }
  int code(const uint64_t* k, uint32_t q) const {
    return get_l(k, q) ? 4 : ((int)get_x(k, q) | ((int)get_z(k, q) << 1));
  }
  // weight counts lost qubits too; loss_weight only those (loss/data.rs:132-200)
  uint64_t weight(const uint64_t* k) const {
    uint64_t t = 0;
    for (int w = 0; w < W; ++w) t += __builtin_popcountll(k[w] | k[W + w] | (lossy ? k[2 * W + w] : 0));
    return t;
  }
  uint64_t loss_weight(const uint64_t* k) const {
    uint64_t t = 0;
    if (lossy)
      for (int w = 0; w < W; ++w) t += __builtin_popcountll(k[2 * W + w]);
    return t;
  }
  // "Z?*" matches only words with no X bit and no lost qubit
  bool zero_overlap_word(const uint64_t* k) const {
    for (int w = 0; w < W; ++w)
      if (k[w] | (lossy ? k[2 * W + w] : 0)) return false;
    return true;
  }
};

// ---- IndexMap configuration -------------------------------------------------------------
struct IndexStore : Words {
  std::vector<uint64_t> keys;  // [i][2W]: x words then z words
  std::vector<double> vals;
  std::vector<uint32_t> table;  // open addressing, slot -> entry index
  uint64_t mask = 0;
  std::vector<uint64_t> scratch_keys;
  std::vector<double> scratch_vals;
  // aux map of map_add: kept from gate to gate, as the reference's aux.clear() keeps it
  std::vector<uint64_t> aux_keys;
  std::vector<double> aux_vals;
  std::vector<uint32_t> aux_table;
  uint64_t aux_mask = 0;

  void init() { rebuild_index(); }
  size_t len() const { return vals.size(); }
  const uint64_t* key(size_t i) const { return &keys[i * kw()]; }
  uint64_t* key(size_t i) { return &keys[i * kw()]; }

  void reserve_index(size_t expected) {  // empty table sized for `expected` entries
    uint64_t cap = table_cap_for(expected);
    table.assign(cap, kEmpty);
    mask = cap - 1;
  }
  void rebuild_index() {
    reserve_index(len());
    for (size_t i = 0; i < len(); ++i) {
      uint64_t s = fx_hash(key(i), kw()) & mask;
      while (table[s] != kEmpty) s = (s + 1) & mask;
      table[s] = (uint32_t)i;
    }
  }
  long find(const uint64_t* k) const {
    if (table.empty()) return -1;
    uint64_t s = fx_hash(k, kw()) & mask;
    while (table[s] != kEmpty) {
      if (std::memcmp(key(table[s]), k, kb()) == 0) return table[s];
      s = (s + 1) & mask;
    }
    return -1;
  }
  bool get(const uint64_t* k, double& v) const {
    long i = find(k);
    if (i < 0) return false;
    v = vals[i];
    return true;
  }
  // IndexMap entry(key).and_modify(|v| *v += value).or_insert(value)
  void add_assign(const uint64_t* k, double v) {
    long i = find(k);
    if (i >= 0) {
      vals[i] += v;
      return;
    }
    if (table.empty() || 2 * (len() + 1) + 2 > table.size()) {
      keys.insert(keys.end(), k, k + kw());
      vals.push_back(v);
      rebuild_index();
      return;
    }
    size_t idx = len();
    keys.insert(keys.end(), k, k + kw());
    vals.push_back(v);
    uint64_t s = fx_hash(k, kw()) & mask;
    while (table[s] != kEmpty) s = (s + 1) & mask;
    table[s] = (uint32_t)idx;
  }
  template <class F>
  void retain(F keep) {  // stable, like IndexMap::retain
    size_t o = 0;
    for (size_t i = 0; i < len(); ++i) {
      if (keep(key(i), vals[i])) {
        if (o != i) {
          std::memcpy(key(o), key(i), kb());
          vals[o] = vals[i];
        }
        ++o;
      }
    }
    keys.resize(o * kw());
    vals.resize(o);
    rebuild_index();
  }
  // map_insert (data.rs:204-226): f(child_key, &v, child_value) -> has child.
  template <class F>
  void map_insert(F f) {
    scratch_keys.clear();
    scratch_vals.clear();
    std::vector<uint64_t> ck(kw());
    size_t n0 = len();
    for (size_t i = 0; i < n0; ++i) {
      double cv;
      std::memcpy(ck.data(), key(i), kb());
      if (f(ck.data(), vals[i], cv)) {
        scratch_keys.insert(scratch_keys.end(), ck.begin(), ck.end());
        scratch_vals.push_back(cv);
      }
    }
    for (size_t j = 0; j < scratch_vals.size(); ++j) add_assign(&scratch_keys[j * kw()], scratch_vals[j]);
  }
  // map_add (data.rs:255-265, hashmap.rs:46-54): `aux.clear()`, every entry mapped and
  // `+=`-inserted into aux in iteration order, then data and aux swap.  Clearing costs a
  // pass over aux's index, as the reference's table clear does.
  template <class F>
  void map_add(F f) {
    aux_keys.clear();
    aux_vals.clear();
    uint64_t cap = table_cap_for(len());
    if (aux_table.size() < cap) aux_table.assign(cap, kEmpty);
    else std::fill(aux_table.begin(), aux_table.end(), kEmpty);
    aux_mask = aux_table.size() - 1;
    std::vector<uint64_t> nk(kw());
    for (size_t i = 0; i < len(); ++i) {
      std::memcpy(nk.data(), key(i), kb());
      double v = vals[i];
      f(nk.data(), v);
      uint64_t s = fx_hash(nk.data(), kw()) & aux_mask;
      bool merged = false;
      while (aux_table[s] != kEmpty) {
        if (std::memcmp(&aux_keys[(size_t)aux_table[s] * kw()], nk.data(), kb()) == 0) {
          aux_vals[aux_table[s]] += v;
          merged = true;
          break;
        }
        s = (s + 1) & aux_mask;
      }
      if (!merged) {
        aux_table[s] = (uint32_t)aux_vals.size();
        aux_keys.insert(aux_keys.end(), nk.begin(), nk.end());
        aux_vals.push_back(v);
      }
    }
    keys.swap(aux_keys);
    vals.swap(aux_vals);
    table.swap(aux_table);
    std::swap(mask, aux_mask);
  }
  template <class F>
  void scale(F f) {
    for (size_t i = 0; i < len(); ++i) f(key(i), vals[i]);
  }
  template <class F>
  void for_each(F f) const {  // iteration order
    for (size_t i = 0; i < len(); ++i) f(key(i), vals[i]);
  }
  double overlap_with_zero() const {  // trace("Z?*"): fold in order over X-free words
    double acc = 0.0;
    for (size_t i = 0; i < len(); ++i)
      if (zero_overlap_word(key(i))) acc += vals[i];
    return acc;
  }
  // map_insert_multiple (data.rs:227-248): aux cleared; every parent's children `+=`-inserted
  // into aux in iteration order (hashmap.rs:181-194); then consume (data.rs:180-189): the
  // larger map takes the smaller one's entries with `+=` (hashmap.rs:302-308), in the smaller
  // one's order, and ends up as the data map.  f(key, &v, out_keys, out_vals) appends children.
  template <class F>
  void map_insert_multiple(F f) {
    aux_keys.clear();
    aux_vals.clear();
    std::vector<uint32_t> atab(table_cap_for(len()), kEmpty);
    uint64_t amask = atab.size() - 1;
    auto aux_find = [&](const uint64_t* k) -> long {
      uint64_t s = fx_hash(k, kw()) & amask;
      while (atab[s] != kEmpty) {
        if (std::memcmp(&aux_keys[(size_t)atab[s] * kw()], k, kb()) == 0) return atab[s];
        s = (s + 1) & amask;
      }
      return -1;
    };
    auto aux_add = [&](const uint64_t* k, double v) {
      long j = aux_find(k);
      if (j >= 0) {
        aux_vals[j] += v;
        return;
      }
      aux_keys.insert(aux_keys.end(), k, k + kw());
      aux_vals.push_back(v);
      if (2 * aux_vals.size() + 2 > atab.size()) {
        atab.assign(table_cap_for(aux_vals.size()), kEmpty);
        amask = atab.size() - 1;
        for (size_t i = 0; i < aux_vals.size(); ++i) {
          uint64_t s = fx_hash(&aux_keys[i * kw()], kw()) & amask;
          while (atab[s] != kEmpty) s = (s + 1) & amask;
          atab[s] = (uint32_t)i;
        }
        return;
      }
      uint64_t s = fx_hash(k, kw()) & amask;
      while (atab[s] != kEmpty) s = (s + 1) & amask;
      atab[s] = (uint32_t)(aux_vals.size() - 1);
    };
    std::vector<uint64_t> ck;
    std::vector<double> cv;
    for (size_t i = 0; i < len(); ++i) {
      ck.clear();
      cv.clear();
      f(key(i), vals[i], ck, cv);
      for (size_t j = 0; j < cv.size(); ++j) aux_add(&ck[j * kw()], cv[j]);
    }
    if (aux_vals.size() > len()) {  // aux.consume(data); swap
      for (size_t i = 0; i < len(); ++i) aux_add(key(i), vals[i]);
      keys.swap(aux_keys);
      vals.swap(aux_vals);
      rebuild_index();
    } else {  // data.consume(aux)
      const size_t na = aux_vals.size();
      for (size_t j = 0; j < na; ++j) add_assign(&aux_keys[j * kw()], aux_vals[j]);
    }
  }
};

// A fixed pool of host threads for the DashMap configuration's parallel loops (rayon's
// global pool in the reference).  parallel_for(count, f) runs f(0..count) over the
// pool's threads and the caller, items handed out one at a time, and returns when all
// are done.
class Pool {
 public:
  explicit Pool(int threads) {
    for (int i = 1; i < threads; ++i) workers_.emplace_back([this] { loop(); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    start_.notify_all();
    for (auto& t : workers_) t.join();
  }
  template <class F>
  void parallel_for(long count, F f) {
    std::function<void(long)> job = f;
    if (workers_.empty() || count <= 1) {
      for (long i = 0; i < count; ++i) job(i);
      return;
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      job_ = &job;
      total_ = count;
      next_.store(0);
      pending_ = (int)workers_.size();
      ++epoch_;
    }
    start_.notify_all();
    drain(job);
    std::unique_lock<std::mutex> lk(mu_);
    done_.wait(lk, [&] { return pending_ == 0; });
    job_ = nullptr;
  }

 private:
  void drain(const std::function<void(long)>& job) {
    for (long i; (i = next_.fetch_add(1)) < total_;) job(i);
  }
  void loop() {
    uint64_t seen = 0;
    for (;;) {
      const std::function<void(long)>* job;
      {
        std::unique_lock<std::mutex> lk(mu_);
        start_.wait(lk, [&] { return stop_ || epoch_ != seen; });
        if (stop_) return;
        seen = epoch_;
        job = job_;
      }
      drain(*job);
      std::lock_guard<std::mutex> lk(mu_);
      if (--pending_ == 0) done_.notify_one();
    }
  }
  std::vector<std::thread> workers_;
  std::mutex mu_;
  std::condition_variable start_, done_;
  const std::function<void(long)>* job_ = nullptr;
  long total_ = 0;
  std::atomic<long> next_{0};
  int pending_ = 0;
  uint64_t epoch_ = 0;
  bool stop_ = false;
};


// ---- DashMap configuration ----------------------------------------------------------------
// DashMap keeps 4 x (hardware threads) shards, rounded up to a power of two; a key lives
// in the shard its hash selects, and each shard is a lock-guarded hash map.  The rayon
// operations of crates/ppvm-traits/src/map/dashmap.rs run over the shards in parallel:
// scale (par_iter_mut, :194-210), map_add_assign (par_iter, each output inserted under
// its shard's lock, :46-55), map_insert_vec (par_extend of the parents' children in shard
// order, :158-166) and trace (par_iter filter + sum, :96-113).  `retain` walks the shards
// one after another (DashMap::retain, :222-227), and PauliSum::map_insert merges the
// scratch Vec one key at a time (data.rs:221-223), so truncation and the child merge of a
// rotation stay serial, as in the reference.
struct ShardStore : Words {
  // Each shard on cache lines of its own, as DashMap pads its shards: two threads that fill
  // different shards then never write the same line.
  struct alignas(128) Shard {
    std::vector<uint64_t> keys;
    std::vector<double> vals;
    std::vector<uint32_t> table;
    uint64_t mask = 0;
  };
  int threads = 1;
  int shard_bits = 0;
  std::vector<Shard> data, aux;
  struct alignas(128) Lock {
    std::atomic<uint32_t> held{0};
  };
  std::unique_ptr<Lock[]> locks;  // one per shard of the map being filled
  std::unique_ptr<Pool> pool;
  std::vector<std::vector<uint64_t>> child_keys;    // per shard: the rotation's children
  std::vector<std::vector<double>> child_vals;

  ShardStore() = default;
  ShardStore(const ShardStore& o)
      : Words(o), threads(o.threads), shard_bits(o.shard_bits), data(o.data), aux(o.aux),
        child_keys(o.child_keys), child_vals(o.child_vals) {
    make_locks();
    pool.reset(new Pool(threads));
  }

  size_t shards() const { return data.size(); }
  void make_locks() {
    locks.reset(new Lock[shards()]);
  }
  void init() {
    if (threads < 1) threads = 1;
    size_t s = 1;
    while (s < 4 * (size_t)threads) s <<= 1;
    shard_bits = 0;
    while ((1ull << shard_bits) < s) ++shard_bits;
    data.assign(s, Shard());
    aux.assign(s, Shard());
    for (auto& sh : data) reset(sh, 0);
    for (auto& sh : aux) reset(sh, 0);
    child_keys.assign(s, {});
    child_vals.assign(s, {});
    make_locks();
    pool.reset(new Pool(threads));
  }
  // bits 40.. of the hash pick the shard, the low bits the slot inside it
  size_t shard_of(uint64_t h) const { return (size_t)(h >> 40) & (shards() - 1); }
  void reset(Shard& sh, size_t expected) {
    uint64_t cap = table_cap_for(expected);
    if (sh.table.size() < cap) sh.table.assign(cap, kEmpty);
    else std::fill(sh.table.begin(), sh.table.end(), kEmpty);
    sh.mask = sh.table.size() - 1;
    sh.keys.clear();
    sh.vals.clear();
  }
  void reindex(Shard& sh) const {
    uint64_t cap = table_cap_for(sh.vals.size());
    sh.table.assign(cap, kEmpty);
    sh.mask = cap - 1;
    for (size_t i = 0; i < sh.vals.size(); ++i) {
      uint64_t s = fx_hash(&sh.keys[i * kw()], kw()) & sh.mask;
      while (sh.table[s] != kEmpty) s = (s + 1) & sh.mask;
      sh.table[s] = (uint32_t)i;
    }
  }
  long find_in(const Shard& sh, const uint64_t* k, uint64_t h) const {
    uint64_t s = h & sh.mask;
    while (sh.table[s] != kEmpty) {
      if (std::memcmp(&sh.keys[(size_t)sh.table[s] * kw()], k, kb()) == 0) return sh.table[s];
      s = (s + 1) & sh.mask;
    }
    return -1;
  }
  // entry(key).and_modify(+=).or_insert into one shard (the caller holds its lock)
  void insert_in(Shard& sh, const uint64_t* k, double v, uint64_t h) const {
    long i = find_in(sh, k, h);
    if (i >= 0) {
      sh.vals[i] += v;
      return;
    }
    sh.keys.insert(sh.keys.end(), k, k + kw());
    sh.vals.push_back(v);
    if (2 * sh.vals.size() + 2 > sh.table.size()) {
      reindex(sh);
      return;
    }
    uint64_t s = h & sh.mask;
    while (sh.table[s] != kEmpty) s = (s + 1) & sh.mask;
    sh.table[s] = (uint32_t)(sh.vals.size() - 1);
  }

  size_t len() const {
    size_t t = 0;
    for (const auto& sh : data) t += sh.vals.size();
    return t;
  }
  bool get(const uint64_t* k, double& v) const {
    uint64_t h = fx_hash(k, kw());
    const Shard& sh = data[shard_of(h)];
    long i = find_in(sh, k, h);
    if (i < 0) return false;
    v = sh.vals[i];
    return true;
  }
  void add_assign(const uint64_t* k, double v) {  // single caller: the shard lock is free
    uint64_t h = fx_hash(k, kw());
    insert_in(data[shard_of(h)], k, v, h);
  }
  template <class F>
  void retain(F keep) {  // shard after shard (DashMap::retain)
    for (auto& sh : data) {
      size_t o = 0;
      for (size_t i = 0; i < sh.vals.size(); ++i) {
        if (keep(&sh.keys[i * kw()], sh.vals[i])) {
          if (o != i) {
            std::memcpy(&sh.keys[o * kw()], &sh.keys[i * kw()], kb());
            sh.vals[o] = sh.vals[i];
          }
          ++o;
        }
      }
      sh.keys.resize(o * kw());
      sh.vals.resize(o);
      reindex(sh);
    }
  }
  template <class F>
  void map_insert(F f) {
    const long S = (long)shards();
    pool->parallel_for(S, [&](long s) {
      Shard& sh = data[s];
      auto& ok = child_keys[s];
      auto& ov = child_vals[s];
      ok.clear();
      ov.clear();
      std::vector<uint64_t> ck(kw());
      const size_t n0 = sh.vals.size();
      for (size_t i = 0; i < n0; ++i) {
        double cv;
        std::memcpy(ck.data(), &sh.keys[i * kw()], kb());
        if (f(ck.data(), sh.vals[i], cv)) {
          ok.insert(ok.end(), ck.begin(), ck.end());
          ov.push_back(cv);
        }
      }
    });
    for (long s = 0; s < S; ++s)  // the scratch Vec, merged one key after the other
      for (size_t j = 0; j < child_vals[s].size(); ++j) add_assign(&child_keys[s][j * kw()], child_vals[s][j]);
  }
  template <class F>
  void map_add(F f) {
    const long S = (long)shards();
    size_t expect = len() / shards() + 1;
    for (auto& sh : aux) reset(sh, expect);  // aux.clear(): capacity kept
    pool->parallel_for(S, [&](long s) {
      const Shard& sh = data[s];
      std::vector<uint64_t> nk(kw());
      for (size_t i = 0; i < sh.vals.size(); ++i) {
        std::memcpy(nk.data(), &sh.keys[i * kw()], kb());
        double v = sh.vals[i];
        f(nk.data(), v);
        uint64_t h = fx_hash(nk.data(), kw());
        size_t d = shard_of(h);
        uint32_t z = 0;
        while (!locks[d].held.compare_exchange_weak(z, 1u, std::memory_order_acquire)) z = 0;
        insert_in(aux[d], nk.data(), v, h);
        locks[d].held.store(0u, std::memory_order_release);
      }
    });
    data.swap(aux);
  }
  template <class F>
  void scale(F f) {
    const long S = (long)shards();
    pool->parallel_for(S, [&](long s) {
      Shard& sh = data[s];
      for (size_t i = 0; i < sh.vals.size(); ++i) f(&sh.keys[i * kw()], sh.vals[i]);
    });
  }
  template <class F>
  void for_each(F f) const {
    for (const auto& sh : data)
      for (size_t i = 0; i < sh.vals.size(); ++i) f(&sh.keys[i * kw()], sh.vals[i]);
  }
  double overlap_with_zero() const {  // per-shard partial sums, added in shard order
    const long S = (long)shards();
    std::vector<double> part(S, 0.0);
    pool->parallel_for(S, [&](long s) {
      const Shard& sh = data[s];
      double acc = 0.0;
      for (size_t i = 0; i < sh.vals.size(); ++i)
        if (zero_overlap_word(&sh.keys[i * kw()])) acc += sh.vals[i];
      part[s] = acc;
    });
    double acc = 0.0;
    for (long s = 0; s < S; ++s) acc += part[s];
    return acc;
  }
};

// ---- gates, noise and truncation over either map ------------------------------------------
template <class M>
struct Sum : M {
  using M::W;
  using M::get_x;
  using M::get_z;
  using M::set_x;
  using M::set_z;

  // ---- Clifford gates (crates/ppvm-pauli-sum/src/sum/clifford.rs) ------------------
  // A gate on a lost qubit leaves the word alone (clifford.rs:42-199 check get_lbit first).
  using M::get_l;
  void g_x(uint32_t q) { this->scale([&](const uint64_t* k, double& v) { if (!get_l(k, q) && get_z(k, q)) v *= -1.0; }); }
  void g_y(uint32_t q) { this->scale([&](const uint64_t* k, double& v) { if (!get_l(k, q) && (get_x(k, q) ^ get_z(k, q))) v *= -1.0; }); }
  void g_z(uint32_t q) { this->scale([&](const uint64_t* k, double& v) { if (!get_l(k, q) && get_x(k, q)) v *= -1.0; }); }
  // single-qubit map_add gates: mode selects the bit map and the sign rule.
  enum Single { H, S, SDAG, SQX, SQXDAG, SQY, SQYDAG };
  void g_single(Single g, uint32_t q) {
    this->map_add([&](uint64_t* k, double& v) {
      if (get_l(k, q)) return;
      bool x = get_x(k, q), z = get_z(k, q);
      bool neg = false;
      switch (g) {
        case H: set_x(k, q, z); set_z(k, q, x); neg = x & z; break;             // clifford.rs:69-87
        case S: set_z(k, q, x ^ z); neg = x & !z; break;                       // :90-107
        case SDAG: set_z(k, q, x ^ z); neg = x & z; break;                     // :115-132
        case SQX: set_x(k, q, x ^ z); neg = x & z; break;                      // :135-152
        case SQXDAG: set_x(k, q, x ^ z); neg = !x & z; break;                  // :176-193
        case SQY: set_x(k, q, z); set_z(k, q, x); neg = !x & z; break;         // :155-173
        case SQYDAG: set_x(k, q, z); set_z(k, q, x); neg = x & !z; break;      // :196-214
      }
      if (neg) v = -v;
    });
  }
  // two-qubit map_word! gates via PhasedPauliWord (crates/ppvm-pauli-word/src/phase/clifford.rs:72-100,168-182)
  enum Two { CNOT, CZ, CY };
  void g_two(Two g, uint32_t c, uint32_t t) {
    this->map_add([&](uint64_t* k, double& v) {
      if (get_l(k, c) || get_l(k, t)) return;  // phase/clifford.rs:77,92,168
      bool xc = get_x(k, c), zc = get_z(k, c), xt = get_x(k, t), zt = get_z(k, t);
      bool neg = false;
      switch (g) {
        case CNOT:
          neg = xc & zt & (xt == zc);
          set_z(k, c, zt ^ zc); set_x(k, t, xc ^ xt);  // traits/clifford.rs:142-151
          break;
        case CZ:
          neg = xc & xt & (zc ^ zt);
          set_z(k, c, zc ^ xt); set_z(k, t, zt ^ xc);  // traits/clifford.rs:154-165
          break;
        case CY:
          neg = xc & (xt ^ zt) & !(zc ^ zt);
          set_z(k, c, zc ^ xt ^ zt); set_x(k, t, xt ^ xc); set_z(k, t, zt ^ xc);  // :328-341
          break;
      }
      if (neg) v = -v;
    });
  }

  // ---- rotations (crates/ppvm-pauli-sum/src/sum/rot1.rs:55-128, rot2.rs:63-184) -----
  // Each closure mirrors the reference fast path: parent *= cos; child = v * (eps * sin).
  void r_x(uint32_t q, double s, double co) {
    this->map_insert([&](uint64_t* k, double& v, double& cv) {
      if (get_l(k, q) || !get_z(k, q)) return false;  // rot1.rs:60
      bool xb = get_x(k, q);
      double coeff = v;
      v *= co;
      set_x(k, q, !xb);
      double eps = xb ? -1.0 : 1.0;
      cv = coeff * (eps * s);
      return true;
    });
  }
  void r_y(uint32_t q, double s, double co) {
    this->map_insert([&](uint64_t* k, double& v, double& cv) {
      if (get_l(k, q)) return false;  // rot1.rs:85
      bool xb = get_x(k, q), zb = get_z(k, q);
      if (xb == zb) return false;
      double coeff = v;
      v *= co;
      set_x(k, q, !xb); set_z(k, q, !zb);
      double eps = zb ? -1.0 : 1.0;
      cv = coeff * (eps * s);
      return true;
    });
  }
  void r_z(uint32_t q, double s, double co) {
    this->map_insert([&](uint64_t* k, double& v, double& cv) {
      if (get_l(k, q)) return false;  // rot1.rs:111
      bool xb = get_x(k, q);
      if (!xb) return false;
      bool zb = get_z(k, q);
      double coeff = v;
      v *= co;
      set_z(k, q, !zb);
      double eps = zb ? 1.0 : -1.0;
      cv = coeff * (eps * s);
      return true;
    });
  }
  // rotate_1 closure (rot1.rs:9-42) on qubit q about axis (ax, az): the loss fallback of the
  // two-qubit rotations (rot2.rs:28-33, 70-75, 109-114, 149-154).  Levi-Civita sign of the
  // axis times the qubit's Pauli, as rot_sign computes it for a one-qubit generator.
  bool rot1_closure(uint64_t* k, double& v, double& cv, uint32_t q, bool ax, bool az, double s, double co) const {
    if (get_l(k, q)) return false;
    const bool x = get_x(k, q), z = get_z(k, q);
    if (!((x & az) ^ (z & ax))) return false;
    std::vector<uint64_t> gx(W, 0), gz(W, 0);
    if (ax) gx[q >> 6] |= 1ull << (q & 63);
    if (az) gz[q >> 6] |= 1ull << (q & 63);
    const double eps = (double)rot_sign(gx.data(), gz.data(), k);
    double coeff = v;
    v *= co;
    set_x(k, q, x ^ ax);
    set_z(k, q, z ^ az);
    cv = coeff * (eps * s);
    return true;
  }
  void r_zz(uint32_t a, uint32_t b, double s, double co) {
    this->map_insert([&](uint64_t* k, double& v, double& cv) {
      if (get_l(k, a)) return rot1_closure(k, v, cv, b, false, true, s, co);
      if (get_l(k, b)) return rot1_closure(k, v, cv, a, false, true, s, co);
      bool xa = get_x(k, a), xb = get_x(k, b);
      if (xa == xb) return false;
      bool za = get_z(k, a), zb = get_z(k, b);
      bool zanti = xa ? za : zb;
      double eps = zanti ? 1.0 : -1.0;
      double coeff = v;
      v *= co;
      set_z(k, a, !za); set_z(k, b, !zb);
      cv = coeff * (eps * s);
      return true;
    });
  }
  void r_xx(uint32_t a, uint32_t b, double s, double co) {
    this->map_insert([&](uint64_t* k, double& v, double& cv) {
      if (get_l(k, a)) return rot1_closure(k, v, cv, b, true, false, s, co);
      if (get_l(k, b)) return rot1_closure(k, v, cv, a, true, false, s, co);
      bool za = get_z(k, a), zb = get_z(k, b);
      if (za == zb) return false;
      bool xa = get_x(k, a), xb = get_x(k, b);
      bool xanti = za ? xa : xb;
      double eps = xanti ? -1.0 : 1.0;
      double coeff = v;
      v *= co;
      set_x(k, a, !xa); set_x(k, b, !xb);
      cv = coeff * (eps * s);
      return true;
    });
  }
  void r_yy(uint32_t a, uint32_t b, double s, double co) {
    this->map_insert([&](uint64_t* k, double& v, double& cv) {
      if (get_l(k, a)) return rot1_closure(k, v, cv, b, true, true, s, co);
      if (get_l(k, b)) return rot1_closure(k, v, cv, a, true, true, s, co);
      bool xa = get_x(k, a), za = get_z(k, a), xb = get_x(k, b), zb = get_z(k, b);
      bool pa = xa ^ za, pb = xb ^ zb;
      if (pa == pb) return false;
      bool xanti = pa ? xa : xb;
      double eps = xanti ? 1.0 : -1.0;
      double coeff = v;
      v *= co;
      set_x(k, a, !xa); set_z(k, a, !za); set_x(k, b, !xb); set_z(k, b, !zb);
      cv = coeff * (eps * s);
      return true;
    });
  }
  // Sign of i*G*P for anticommuting P (G, P as X/Z planes): G*P = i^e (G xor P),
  // e summed per qubit with the Aaronson-Gottesman g function.  Returns +1 or -1.
  int rot_sign(const uint64_t* gx, const uint64_t* gz, const uint64_t* k) const {
    int e = 0;
    for (int w = 0; w < W; ++w) {
      uint64_t x1 = gx[w], z1 = gz[w], x2 = k[w], z2 = k[W + w];
      // G=X (x1 & ~z1): g = z2*(2*x2-1)  -> +1 on Y, -1 on Z
      // G=Y (x1 & z1):  g = z2 - x2      -> +1 on Z, -1 on X
      // G=Z (~x1 & z1): g = x2*(1-2*z2)  -> +1 on X, -1 on Y
      uint64_t gX = x1 & ~z1, gY = x1 & z1, gZ = ~x1 & z1;
      uint64_t pX = x2 & ~z2, pY = x2 & z2, pZ = ~x2 & z2;
      e += __builtin_popcountll(gX & pY) - __builtin_popcountll(gX & pZ);
      e += __builtin_popcountll(gY & pZ) - __builtin_popcountll(gY & pX);
      e += __builtin_popcountll(gZ & pX) - __builtin_popcountll(gZ & pY);
    }
    int t = ((e + 1) % 4 + 4) % 4;  // i^(e+1) is real for odd e
    return t == 0 ? 1 : -1;
  }
  bool anticommutes(const uint64_t* gx, const uint64_t* gz, const uint64_t* k) const {
    int par = 0;
    for (int w = 0; w < W; ++w)
      par ^= __builtin_parityll((k[w] & gz[w]) ^ (k[W + w] & gx[w]));
    return par;
  }
  // Generic exp(-i theta/2 G): rotate_1 / rotate_2 generalised to any support.  On a lossy
  // word the generator acts only on qubits that are not lost, which is the reference's loss
  // fallback of rotate_2 (rot2.rs:26-33) extended to any support.
  void r_pauli(const uint64_t* gx, const uint64_t* gz, double s, double co) {
    this->map_insert([&](uint64_t* k, double& v, double& cv) {
      std::vector<uint64_t> ex(gx, gx + W), ez(gz, gz + W);
      if (this->lossy)
        for (int w = 0; w < W; ++w) { ex[w] &= ~k[2 * W + w]; ez[w] &= ~k[2 * W + w]; }
      if (!anticommutes(ex.data(), ez.data(), k)) return false;
      double eps = (double)rot_sign(ex.data(), ez.data(), k);
      double coeff = v;
      v *= co;
      for (int w = 0; w < W; ++w) { k[w] ^= ex[w]; k[W + w] ^= ez[w]; }
      cv = coeff * (eps * s);
      return true;
    });
  }
  // Clifford-angle rotation (theta = +-pi/2 with cos taken as exactly 0): anticommuting
  // P -> sign * (iGP), a bijection on words.  Tests pin it against the reference's
  // Clifford compositions (e.g. RZZ(-pi/2) == CZ, S_DAG, S_DAG).
  void r_pauli_clifford(const uint64_t* gx, const uint64_t* gz, double sin_sign) {
    this->map_add([&](uint64_t* k, double& v) {
      std::vector<uint64_t> ex(gx, gx + W), ez(gz, gz + W);
      if (this->lossy)
        for (int w = 0; w < W; ++w) { ex[w] &= ~k[2 * W + w]; ez[w] &= ~k[2 * W + w]; }
      if (!anticommutes(ex.data(), ez.data(), k)) return;
      double eps = (double)rot_sign(ex.data(), ez.data(), k);
      for (int w = 0; w < W; ++w) { k[w] ^= ex[w]; k[W + w] ^= ez[w]; }
      v = v * (eps * sin_sign);
    });
  }

  // ---- noise (crates/ppvm-pauli-sum/src/sum/noise.rs) --------------------------------
  void pauli_error(uint32_t q, const double p[3]) {  // noise.rs:17-37
    double one = 1.0;
    double xf = one - p[1] * 2.0 - p[2] * 2.0;
    double zf = one - p[0] * 2.0 - p[1] * 2.0;
    double yf = one - p[0] * 2.0 - p[2] * 2.0;
    this->scale([&](const uint64_t* k, double& v) {
      if (get_l(k, q)) return;  // noise.rs:25
      int code = (int)get_x(k, q) | ((int)get_z(k, q) << 1);
      if (code == 1) v *= xf; else if (code == 2) v *= zf; else if (code == 3) v *= yf;
    });
  }
  void depolarize1(uint32_t q, double p) {  // noise.rs:107-116
    double f = 1.0 - p * (4.0 / 3.0);
    this->scale([&](const uint64_t* k, double& v) { if (!get_l(k, q) && (get_x(k, q) | get_z(k, q))) v *= f; });
  }
  void depolarize2(uint32_t a, uint32_t b, double p) {  // noise.rs:119-129
    double f = 1.0 - p * (16.0 / 15.0);
    this->scale([&](const uint64_t* k, double& v) {
      if (get_l(k, a) || get_l(k, b)) return;  // noise.rs:122
      if (get_x(k, a) | get_z(k, a) | get_x(k, b) | get_z(k, b)) v *= f;
    });
  }

  // two_qubit_pauli_error (noise.rs:39-105).  A term with Paulis (Pa, Pb) on the pair is
  // scaled by acc = 1 - 2 p[i1] - 2 p[i2] - ... - 2 p[i8] over the eight two-qubit Paulis that
  // anticommute with it, subtracted in the reference's index order (the order fixes the
  // rounding).  Rows by (code a, code b), code = x | z << 1 (I 0, X 1, Z 2, Y 3); p indices
  // name IX IY IZ XI XX XY XZ YI YX YY YZ ZI ZX ZY ZZ in that order.
  void two_qubit_pauli_error(uint32_t a, uint32_t b, const double p[15]) {
    static const int8_t kIdx[4][4][8] = {
        {{-1}, {1, 10, 13, 14, 2, 5, 6, 9}, {0, 1, 12, 13, 4, 5, 8, 9}, {0, 10, 12, 14, 2, 4, 6, 8}},
        {{10, 11, 12, 13, 14, 7, 8, 9}, {1, 11, 12, 2, 5, 6, 7, 8}, {0, 1, 10, 11, 14, 4, 5, 7},
         {0, 11, 13, 2, 4, 6, 7, 9}},
        {{10, 3, 4, 5, 6, 7, 8, 9}, {1, 13, 14, 2, 3, 4, 7, 8}, {0, 1, 10, 12, 13, 3, 6, 7},
         {0, 12, 14, 2, 3, 5, 7, 9}},
        {{11, 12, 13, 14, 3, 4, 5, 6}, {1, 10, 11, 12, 2, 3, 4, 9}, {0, 1, 11, 14, 3, 6, 8, 9},
         {0, 10, 11, 13, 2, 3, 5, 8}}};
    double f[4][4];
    for (int ca = 0; ca < 4; ++ca)
      for (int cb = 0; cb < 4; ++cb) {
        double acc = 1.0;
        if (ca | cb)
          for (int t = 0; t < 8; ++t) acc = acc - p[kIdx[ca][cb][t]] * 2.0;
        f[ca][cb] = acc;
      }
    this->scale([&](const uint64_t* k, double& v) {
      if (get_l(k, a) || get_l(k, b)) return;  // a lost qubit: no channel (noise.rs:98-102)
      const int ca = (int)get_x(k, a) | ((int)get_z(k, a) << 1);
      const int cb = (int)get_x(k, b) | ((int)get_z(k, b) << 1);
      if (ca | cb) v *= f[ca][cb];
    });
  }
  // amplitude_damping (noise.rs:132-163): I unchanged; X, Y scaled by sqrt(1 - gamma); Z
  // scaled by (1 - gamma) with the child (Z -> I on q, v * gamma) collected by map_insert.
  void amplitude_damping(uint32_t q, double gamma) {
    const double om = 1.0 - gamma;
    const double sxy = std::sqrt(om);
    this->map_insert([&](uint64_t* ck, double& v, double& cv) {
      if (get_l(ck, q)) return false;  // noise.rs:138 (L like I)
      if (get_x(ck, q)) {
        v *= sxy;
        return false;
      }
      if (!get_z(ck, q)) return false;
      cv = v * gamma;
      set_z(ck, q, false);
      v *= om;
      return true;
    });
  }

  // ---- loss channels (crates/ppvm-pauli-sum/src/sum/noise.rs:165-275) -----------------
  // loss_channel (noise.rs:165-181): L on q -> child with I on q, v * p (parent unchanged);
  // I, X, Y, Z on q: v *= 1 - p.
  void loss_channel(uint32_t q, double p) {
    this->map_insert([&](uint64_t* ck, double& v, double& cv) {
      if (this->code(ck, q) == 4) {
        cv = v * p;
        this->set_code(ck, q, 0);
        return true;
      }
      v *= 1.0 - p;
      return false;
    });
  }
  // correlated_loss_channel (noise.rs:184-243) through map_insert_multiple.
  void correlated_loss_channel(uint32_t a, uint32_t b, const double p[3]) {
    const int kw = this->kw();
    this->map_insert_multiple([&](const uint64_t* k, double& v, std::vector<uint64_t>& ok,
                                  std::vector<double>& ov) {
      const int ca = this->code(k, a), cb = this->code(k, b);
      auto child = [&](int na, int nb, double val) {
        const size_t o = ok.size();
        ok.insert(ok.end(), k, k + kw);
        this->set_code(&ok[o], a, na);
        this->set_code(&ok[o], b, nb);
        ov.push_back(val);
      };
      if (ca == 4 && cb == 4) {  // both lost: (I,L), (L,I) with p[2]; (I,I) with p[0]
        const double v_il = v * p[2];
        child(0, 4, v_il);
        child(4, 0, v_il);
        child(0, 0, v * p[0]);
      } else if (cb == 4) {  // qubit 1 lost
        const double nv = v * p[1];
        v *= 1.0 - p[2];
        child(ca, 0, nv);
      } else if (ca == 4) {  // qubit 0 lost
        const double nv = v * p[1];
        v *= 1.0 - p[2];
        child(0, cb, nv);
      } else {
        v *= 1.0 - p[1] * 2.0 - p[0];
      }
    });
  }
  // reset_loss_channel (noise.rs:245-275): L on q -> v *= 0.0; I or Z -> child with L on q
  // (same coefficient); X, Y unchanged.
  void reset_loss_channel(uint32_t q) {
    this->map_insert([&](uint64_t* ck, double& v, double& cv) {
      const int c = this->code(ck, q);
      if (c == 4) {
        v *= 0.0;
        return false;
      }
      if (c == 0 || c == 2) {
        cv = v;
        this->set_code(ck, q, 4);
        return true;
      }
      return false;
    });
  }

  // ---- truncation (data.rs:275-311, strategy.rs) -------------------------------------
  void strategy() {
    double t = this->thr;
    this->retain([&](const uint64_t*, double v) { return !(std::fabs(v) < t); });  // strategy.rs:125-134
    if (this->maxw != UINT64_MAX) {  // strategy.rs:86-90
      uint64_t mw = this->maxw;
      this->retain([&](const uint64_t* k, double) { return this->weight(k) <= mw; });
    }
    if (this->lossy && this->maxlw != UINT64_MAX) {  // MaxLossWeight (strategy.rs:165-180)
      uint64_t ml = this->maxlw;
      this->retain([&](const uint64_t* k, double) { return this->loss_weight(k) <= ml; });
    }
  }
  bool is_preserved(const uint64_t* k) const {
    const int kw = this->kw();
    size_t np = this->preserve.size() / kw;
    for (size_t j = 0; j < np; ++j)
      if (std::memcmp(&this->preserve[j * kw], k, this->kb()) == 0) return true;
    return false;
  }
  void truncate() {
    if (this->preserve.empty()) { strategy(); return; }
    const int kw = this->kw();
    std::vector<uint64_t> sk;
    std::vector<double> sv;
    this->for_each([&](const uint64_t* k, double v) {
      if (is_preserved(k)) { sk.insert(sk.end(), k, k + kw); sv.push_back(v); }
    });
    strategy();
    double dummy;
    for (size_t j = 0; j < sv.size(); ++j)
      if (!this->get(&sk[j * kw], dummy)) this->add_assign(&sk[j * kw], sv[j]);
  }
};

// ---- PauliPattern (crates/ppvm-pauli-word/src/pattern) ---------------------------------
// Pauli codes: 0=I 1=X 2=Z 3=Y (x | z<<1).  OpPattern -> accepted set as a 4-bit mask.
// Note: the reference's AnyPauliOrIdentity ('_') accepts only I (contains.rs:38).
struct PatItem { int kind; unsigned accept; size_t arg; };  // kind 0=Position 1=Star 2=Repeat
struct Pattern {
  std::vector<PatItem> items;
  bool ok = true;
};
Pattern parse_pattern(const char* s) {  // parse.rs:32-127
  Pattern P;
  std::string in(s);
  size_t b = in.find_first_not_of(" \t\n\r"), e = in.find_last_not_of(" \t\n\r");
  in = (b == std::string::npos) ? std::string() : in.substr(b, e - b + 1);
  size_t i = 0;
  auto bitof = [](char c) -> unsigned { return c == 'X' ? 2u : c == 'Z' ? 4u : c == 'Y' ? 8u : 0u; };
  while (i < in.size()) {
    char c = in[i++];
    unsigned acc = 0;
    if (c == '[') {
      unsigned set = 0;
      int cnt = 0;
      while (i < in.size()) {
        char d = in[i];
        if (d == ']') { ++i; break; }
        if (d == 'X' || d == 'Y' || d == 'Z') {
          if (!(set & bitof(d))) ++cnt;
          set |= bitof(d); ++i;
        } else { P.ok = false; return P; }
      }
      if (cnt == 0 || cnt > 3) { P.ok = false; return P; }
      acc = set;
    } else if (c == '_') {
      acc = 1u;  // AnyPauliOrIdentity: contains only I in the reference matcher
    } else if (c == 'X' || c == 'Y' || c == 'Z') {
      acc = bitof(c);
    } else { P.ok = false; return P; }
    if (i < in.size() && in[i] == '?') { ++i; acc |= 1u; }  // add_identity
    if (i < in.size() && in[i] == '*') { ++i; P.items.push_back({1, acc, 0}); }
    else if (i < in.size() && in[i] == '{') {
      ++i;
      std::string num;
      while (i < in.size() && isdigit((unsigned char)in[i])) num.push_back(in[i++]);
      if (i < in.size() && in[i] == '}') ++i;
      else { P.ok = false; return P; }
      if (num.empty()) { P.ok = false; return P; }
      P.items.push_back({2, acc, (size_t)std::stoull(num)});
    } else if (i < in.size() && isdigit((unsigned char)in[i])) {
      std::string num;
      while (i < in.size() && isdigit((unsigned char)in[i])) num.push_back(in[i++]);
      P.items.push_back({0, acc, (size_t)std::stoull(num)});
    } else { P.ok = false; return P; }
  }
  return P;
}
// contains.rs:120-151 (match_position :44-66, match_star :68-84, match_repeat :86-116)
bool pattern_contains(const Pattern& P, const Words& S, const uint64_t* k) {
  uint32_t pos = 0, n = S.n;
  auto code = [&](uint32_t q) { return (unsigned)S.code(k, q); };  // 4 = L: no item accepts it
  auto accepts = [](unsigned acc, unsigned c) { return c < 4 && ((acc >> c) & 1u); };
  for (const PatItem& it : P.items) {
    if (it.kind == 0) {
      bool next = false;
      while (pos < n) {
        uint32_t q = pos++;
        unsigned c = code(q);
        if (q == it.arg) { if (accepts(it.accept, c)) { next = true; } break; }
        if (c == 0) continue;
        break;
      }
      if (!next) return false;
    } else if (it.kind == 1) {
      while (pos < n && accepts(it.accept, code(pos))) ++pos;
    } else {
      size_t matched = 0;
      bool done = false;
      while (pos < n) {
        if (accepts(it.accept, code(pos))) {
          ++pos;
          if (++matched == it.arg) { done = true; break; }
        } else {
          if (matched < it.arg) return false;
          done = true;
          break;
        }
      }
      if (!done && matched != it.arg) return false;
    }
  }
  for (; pos < n; ++pos) if (code(pos) != 0) return false;
  return true;
}

bool qok(const Words* s, uint32_t q) { return q < s->n; }

template <class M>
int run_op(Sum<M>* s, const ppvm_op& op) {
  using SumT = Sum<M>;
  const double HALF_PI = 1.5707963267948966;
  auto two_ok = [&]() { return qok(s, op.q0) && qok(s, op.q1) && op.q0 != op.q1; };
  auto is_cliff_angle = [&](double th) { return s->clifford_angles && (th == HALF_PI || th == -HALF_PI); };
  std::vector<uint64_t> gx(s->W, 0), gz(s->W, 0);
  auto setg = [&](uint32_t q, bool x, bool z) {
    if (x) gx[q >> 6] |= 1ull << (q & 63);
    if (z) gz[q >> 6] |= 1ull << (q & 63);
  };
  switch (op.code) {
    case PPVM_OP_X: if (!qok(s, op.q0)) return 1; s->g_x(op.q0); return 0;
    case PPVM_OP_Y: if (!qok(s, op.q0)) return 1; s->g_y(op.q0); return 0;
    case PPVM_OP_Z: if (!qok(s, op.q0)) return 1; s->g_z(op.q0); return 0;
    case PPVM_OP_H: if (!qok(s, op.q0)) return 1; s->g_single(SumT::H, op.q0); return 0;
    case PPVM_OP_S: if (!qok(s, op.q0)) return 1; s->g_single(SumT::S, op.q0); return 0;
    case PPVM_OP_S_DAG: if (!qok(s, op.q0)) return 1; s->g_single(SumT::SDAG, op.q0); return 0;
    case PPVM_OP_SQRT_X: if (!qok(s, op.q0)) return 1; s->g_single(SumT::SQX, op.q0); return 0;
    case PPVM_OP_SQRT_X_DAG: if (!qok(s, op.q0)) return 1; s->g_single(SumT::SQXDAG, op.q0); return 0;
    case PPVM_OP_SQRT_Y: if (!qok(s, op.q0)) return 1; s->g_single(SumT::SQY, op.q0); return 0;
    case PPVM_OP_SQRT_Y_DAG: if (!qok(s, op.q0)) return 1; s->g_single(SumT::SQYDAG, op.q0); return 0;
    case PPVM_OP_CNOT: if (!two_ok()) return 1; s->g_two(SumT::CNOT, op.q0, op.q1); return 0;
    case PPVM_OP_CZ: if (!two_ok()) return 1; s->g_two(SumT::CZ, op.q0, op.q1); return 0;
    case PPVM_OP_CY: if (!two_ok()) return 1; s->g_two(SumT::CY, op.q0, op.q1); return 0;
    case PPVM_OP_RX: case PPVM_OP_RY: case PPVM_OP_RZ: {
      if (!qok(s, op.q0)) return 1;
      bool gxb = op.code != PPVM_OP_RZ, gzb = op.code != PPVM_OP_RX;
      if (is_cliff_angle(op.theta)) {
        setg(op.q0, gxb, gzb);
        s->r_pauli_clifford(gx.data(), gz.data(), op.theta > 0 ? 1.0 : -1.0);
        return 0;
      }
      double sn = std::sin(op.theta), cs = std::cos(op.theta);
      if (op.code == PPVM_OP_RX) s->r_x(op.q0, sn, cs);
      else if (op.code == PPVM_OP_RY) s->r_y(op.q0, sn, cs);
      else s->r_z(op.q0, sn, cs);
      return 0;
    }
    case PPVM_OP_RXX: case PPVM_OP_RYY: case PPVM_OP_RZZ: {
      if (!two_ok()) return 1;
      bool gxb = op.code != PPVM_OP_RZZ, gzb = op.code != PPVM_OP_RXX;
      if (is_cliff_angle(op.theta)) {
        setg(op.q0, gxb, gzb); setg(op.q1, gxb, gzb);
        s->r_pauli_clifford(gx.data(), gz.data(), op.theta > 0 ? 1.0 : -1.0);
        return 0;
      }
      double sn = std::sin(op.theta), cs = std::cos(op.theta);
      if (op.code == PPVM_OP_RXX) s->r_xx(op.q0, op.q1, sn, cs);
      else if (op.code == PPVM_OP_RYY) s->r_yy(op.q0, op.q1, sn, cs);
      else s->r_zz(op.q0, op.q1, sn, cs);
      return 0;
    }
    case PPVM_OP_PAULI_ERROR: if (!qok(s, op.q0)) return 1; s->pauli_error(op.q0, op.p); return 0;
    case PPVM_OP_DEPOLARIZE1: if (!qok(s, op.q0)) return 1; s->depolarize1(op.q0, op.theta); return 0;
    case PPVM_OP_DEPOLARIZE2: if (!two_ok()) return 1; s->depolarize2(op.q0, op.q1, op.theta); return 0;
    case PPVM_OP_TRUNCATE: s->truncate(); return 0;
    case PPVM_OP_AMPLITUDE_DAMPING: if (!qok(s, op.q0)) return 1; s->amplitude_damping(op.q0, op.theta); return 0;
    case PPVM_OP_LOSS_CHANNEL: if (!qok(s, op.q0)) return 1; s->loss_channel(op.q0, op.theta); return 0;
    case PPVM_OP_RESET_LOSS_CHANNEL:  // defined for lossy words only (noise.rs:245-252)
      if (!qok(s, op.q0) || !s->lossy) return 1;
      s->reset_loss_channel(op.q0);
      return 0;
    case PPVM_OP_CORRELATED_LOSS_CHANNEL:
      if (!two_ok()) return 1;
      // The DashMap configuration inserts a parent's children with a plain `insert`
      // from several threads at once (crates/ppvm-traits/src/map/dashmap.rs:168-183): the
      // value of a key with several children depends on thread timing, so it is not restated.
      if constexpr (std::is_same<M, ShardStore>::value) return 1;
      else s->correlated_loss_channel(op.q0, op.q1, op.p);
      return 0;
    default: return 1;
  }
}

// One handle type for both configurations: the C functions below dispatch on it.
struct Handle {
  virtual ~Handle() = default;
  virtual Handle* clone() const = 0;
  virtual Words& words() = 0;
  virtual size_t len() const = 0;
  virtual void add_assign(const uint64_t* k, double v) = 0;
  virtual int run(const ppvm_op& op) = 0;
  virtual void two_qubit_pauli_error(uint32_t a, uint32_t b, const double* p) = 0;
  virtual void truncate() = 0;
  virtual void rotation(const uint64_t* gx, const uint64_t* gz, double theta) = 0;
  virtual double overlap_with_zero() const = 0;
  virtual void each(const std::function<void(const uint64_t*, double)>& f) const = 0;
  virtual bool get(const uint64_t* k, double& v) const = 0;
};

template <class M>
struct HandleT : Handle {
  Sum<M> s;
  Handle* clone() const override { return new HandleT(*this); }
  Words& words() override { return s; }
  size_t len() const override { return s.len(); }
  void add_assign(const uint64_t* k, double v) override { s.add_assign(k, v); }
  int run(const ppvm_op& op) override { return run_op(&s, op); }
  void two_qubit_pauli_error(uint32_t a, uint32_t b, const double* p) override { s.two_qubit_pauli_error(a, b, p); }
  void truncate() override { s.truncate(); }
  void rotation(const uint64_t* gx, const uint64_t* gz, double theta) override {
    const double HALF_PI = 1.5707963267948966;
    if (s.clifford_angles && (theta == HALF_PI || theta == -HALF_PI)) {
      s.r_pauli_clifford(gx, gz, theta > 0 ? 1.0 : -1.0);
      return;
    }
    s.r_pauli(gx, gz, std::sin(theta), std::cos(theta));
  }
  double overlap_with_zero() const override { return s.overlap_with_zero(); }
  void each(const std::function<void(const uint64_t*, double)>& f) const override { s.for_each(f); }
  bool get(const uint64_t* k, double& v) const override { return s.get(k, v); }
};

template <class M>
Handle* make_handle(uint32_t n, double thr, uint64_t maxw, uint32_t flags, int threads) {
  auto* h = new HandleT<M>();
  Sum<M>& s = h->s;
  s.n = n;
  s.W = (int)((n + 63) / 64);
  s.thr = thr;
  s.maxw = maxw;
  s.clifford_angles = (flags & PPVM_FLAG_CLIFFORD_ANGLES) != 0;
  s.lossy = (flags & PPVM_FLAG_LOSSY) != 0;
  if constexpr (std::is_same<M, ShardStore>::value) s.threads = threads;
  s.init();
  return h;
}

}  // namespace

extern "C" {

// Words cross this interface in the engine's layout: W = ceil(n/64) words per plane, or for
// a lossy sum 2W, the X plane's upper W words holding the loss bits and the Z plane's upper W
// words zero (include/ppvm_cuda.h, PPVM_FLAG_LOSSY).  These convert to and from a key.
static int api_words(const Words& s) { return s.lossy ? 2 * s.W : s.W; }
static void key_from_api(const Words& s, const uint64_t* x, const uint64_t* z, uint64_t* key) {
  for (int w = 0; w < s.W; ++w) {
    key[w] = x[w];
    key[s.W + w] = z[w];
    if (s.lossy) key[2 * s.W + w] = x[s.W + w];
  }
}
static void key_to_api(const Words& s, const uint64_t* key, uint64_t* x, uint64_t* z) {
  for (int w = 0; w < s.W; ++w) {
    x[w] = key[w];
    z[w] = key[s.W + w];
    if (s.lossy) {
      x[s.W + w] = key[2 * s.W + w];
      z[s.W + w] = 0;
    }
  }
}

void* oracle_create(uint32_t n, double thr, uint64_t maxw, uint32_t flags) {
  if (n == 0 || ((flags & PPVM_FLAG_LOSSY) && n > 256)) return nullptr;
  return make_handle<IndexStore>(n, thr, maxw, flags, 1);
}
// The DashMap configuration on `threads` threads (0: every hardware thread).
void* oracle_create_sharded(uint32_t n, double thr, uint64_t maxw, uint32_t flags, int threads) {
  if (n == 0) return nullptr;
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  return make_handle<ShardStore>(n, thr, maxw, flags, threads);
}
void oracle_destroy(void* h) { delete (Handle*)h; }
void* oracle_clone(void* h) { return ((Handle*)h)->clone(); }
int oracle_words(void* h) { return api_words(((Handle*)h)->words()); }
// MaxLossWeight of a lossy sum's strategy (UINT64_MAX: off).
void oracle_set_max_loss_weight(void* h, uint64_t maxlw) { ((Handle*)h)->words().maxlw = maxlw; }
size_t oracle_len(void* h) { return ((Handle*)h)->len(); }

// x, z term-major [k][W]
int oracle_add_terms(void* h, const uint64_t* x, const uint64_t* z, const double* c, size_t k) {
  Handle* s = (Handle*)h;
  const Words& ws = s->words();
  const int A = api_words(ws);
  std::vector<uint64_t> key(ws.kw());
  for (size_t i = 0; i < k; ++i) {
    key_from_api(ws, x + i * A, z + i * A, key.data());
    s->add_assign(key.data(), c[i]);
  }
  return 0;
}
// two_qubit_pauli_error_many: pairs (flat, k_flat even) in order, then the strategy if asked.
int oracle_two_qubit_pauli_error(void* h, const uint32_t* pairs, size_t k_flat, const double* p,
                                 int truncate) {
  Handle* s = (Handle*)h;
  const uint32_t n = s->words().n;
  if (k_flat % 2) return 1;
  for (size_t i = 0; i < k_flat; i += 2)
    if (pairs[i] >= n || pairs[i + 1] >= n || pairs[i] == pairs[i + 1]) return 1;
  for (size_t i = 0; i < k_flat; i += 2) s->two_qubit_pauli_error(pairs[i], pairs[i + 1], p);
  if (truncate) s->truncate();
  return 0;
}
int oracle_set_preserve(void* h, const uint64_t* x, const uint64_t* z, size_t k) {
  Words& s = ((Handle*)h)->words();
  const int A = api_words(s);
  s.preserve.assign(k * s.kw(), 0);
  for (size_t i = 0; i < k; ++i) key_from_api(s, x + i * A, z + i * A, &s.preserve[i * s.kw()]);
  return 0;
}
// Runs ops in order; records the live count entering each op into counts (may be NULL).
int oracle_run_ops(void* h, const ppvm_op* ops, size_t n_ops, uint64_t* counts) {
  Handle* s = (Handle*)h;
  for (size_t i = 0; i < n_ops; ++i) {
    if (counts) counts[i] = s->len();
    if (s->run(ops[i]) != 0) return (int)(i + 1);
  }
  return 0;
}
int oracle_pauli_rotation(void* h, const uint64_t* gx, const uint64_t* gz, double theta) {
  ((Handle*)h)->rotation(gx, gz, theta);
  return 0;
}
double oracle_overlap_with_zero(void* h) { return ((Handle*)h)->overlap_with_zero(); }
int oracle_trace(void* h, const char* pattern, double* out) {
  Handle* s = (Handle*)h;
  Pattern P = parse_pattern(pattern);
  if (!P.ok) return 1;
  double acc = 0.0;
  const Words& w = s->words();
  s->each([&](const uint64_t* k, double v) {
    if (pattern_contains(P, w, k)) acc += v;
  });
  *out = acc;
  return 0;
}
// PauliSum::overlap (sum/trace.rs:31-37): other.iter().map(|(k,v)| v * self[k]).sum()
double oracle_overlap(void* a, void* b) {
  Handle* A = (Handle*)a;
  Handle* B = (Handle*)b;
  double acc = 0.0;
  B->each([&](const uint64_t* k, double v) {
    double av;
    acc += v * (A->get(k, av) ? av : 0.0);
  });
  return acc;
}
size_t oracle_export(void* h, uint64_t* x, uint64_t* z, double* c, size_t cap) {
  Handle* s = (Handle*)h;
  const Words& ws = s->words();
  const int A = api_words(ws);
  size_t i = 0;
  s->each([&](const uint64_t* k, double v) {
    if (i >= cap) return;
    key_to_api(ws, k, x + i * A, z + i * A);
    c[i] = v;
    ++i;
  });
  return i;
}

}  // extern "C"
