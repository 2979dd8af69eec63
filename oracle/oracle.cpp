// oracle/oracle.cpp — TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement of the reference's PauliSum hot path (QuEraComputing/ppvm,
// crate `ppvm-pauli-sum` with the IndexMap + FxHash config that the Python binding
// uses, crates/ppvm-python-native/src/interface.rs:414).  It is the checker the GPU
// engine is compared against and the CPU baseline that bench.py times.  Nothing in
// the product (ppvm_b200/) links, loads or calls it.
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
//  * storage: an insertion-ordered map word -> f64 (IndexMap).  New keys append;
//    `+=` on an existing key modifies in place (crates/ppvm-traits/src/map/hashmap.rs:40-44);
//    `retain` keeps order (hashmap.rs:242-258 -> IndexMap::retain).
//  * rotations: map_insert (crates/ppvm-pauli-sum/src/sum/data.rs:204-226): every
//    anticommuting parent is scaled in place by cos and its child (word, v*(eps*sin)) is
//    pushed to a scratch Vec in iteration order; then the scratch is merged with `+=`.
//  * Cliffords: scale (in place, data.rs:192-197) for X/Y/Z; map_add (data.rs:255-265,
//    hashmap.rs:46-54) — a full rebuild into the aux map in iteration order — for the rest.
//  * truncate: data.rs:275-311 with CombinedStrategy(CoefficientThreshold, MaxPauliWeight)
//    (crates/ppvm-pauli-sum/src/strategy.rs:12-30, 73-90, 125-134).
//  * trace: fold in iteration order (hashmap.rs:108-127) with the PauliPattern matcher
//    (crates/ppvm-pauli-word/src/pattern/parse.rs:32-127, contains.rs:19-151).
//
// Build: `make -C oracle` (g++ -O2 -ffp-contract=off); the library is
// oracle/_build/liboracle.so.

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../include/ppvm_cuda.h"

namespace {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;

inline uint64_t rotl(uint64_t v, int r) { return (v << r) | (v >> (64 - r)); }

// FxHash-style word hash (the reference hashes the raw storage bytes with FxHasher,
// crates/ppvm-pauli-word/src/word/data.rs:184-200).  Only speed depends on it.
inline uint64_t fx_hash(const uint64_t* k, int nw) {
  uint64_t h = 0;
  for (int i = 0; i < nw; ++i) h = (rotl(h, 5) ^ k[i]) * 0x517cc1b727220a95ull;
  return h ^ (h >> 32);
}

struct Pattern;

struct OSum {
  uint32_t n = 0;
  int W = 1;  // words per plane
  double thr = 1e-10;
  uint64_t maxw = UINT64_MAX;
  bool clifford_angles = false;
  std::vector<uint64_t> keys;  // [i][2W]: x words then z words
  std::vector<double> vals;
  std::vector<uint32_t> table;  // open addressing, slot -> entry index
  uint64_t mask = 0;
  std::vector<uint64_t> preserve;  // flat [j][2W]
  std::vector<uint64_t> scratch_keys;
  std::vector<double> scratch_vals;

  size_t len() const { return vals.size(); }
  const uint64_t* key(size_t i) const { return &keys[i * 2 * W]; }
  uint64_t* key(size_t i) { return &keys[i * 2 * W]; }

  void reserve_index(size_t expected) {  // empty table sized for `expected` entries
    uint64_t cap = 16;
    while (cap < 2 * (uint64_t)expected + 2) cap <<= 1;
    table.assign(cap, kEmpty);
    mask = cap - 1;
  }
  void rebuild_index() {
    reserve_index(len());
    for (size_t i = 0; i < len(); ++i) {
      uint64_t s = fx_hash(key(i), 2 * W) & mask;
      while (table[s] != kEmpty) s = (s + 1) & mask;
      table[s] = (uint32_t)i;
    }
  }
  long find(const uint64_t* k) const {
    if (table.empty()) return -1;
    uint64_t s = fx_hash(k, 2 * W) & mask;
    while (table[s] != kEmpty) {
      if (std::memcmp(key(table[s]), k, sizeof(uint64_t) * 2 * W) == 0) return table[s];
      s = (s + 1) & mask;
    }
    return -1;
  }
  // IndexMap entry(key).and_modify(|v| *v += value).or_insert(value)
  void add_assign(const uint64_t* k, double v) {
    long i = find(k);
    if (i >= 0) {
      vals[i] += v;
      return;
    }
    if (table.empty() || 2 * (len() + 1) + 2 > table.size()) {
      keys.insert(keys.end(), k, k + 2 * W);
      vals.push_back(v);
      rebuild_index();
      return;
    }
    size_t idx = len();
    keys.insert(keys.end(), k, k + 2 * W);
    vals.push_back(v);
    uint64_t s = fx_hash(k, 2 * W) & mask;
    while (table[s] != kEmpty) s = (s + 1) & mask;
    table[s] = (uint32_t)idx;
  }
  template <class F>
  void retain(F keep) {  // stable, like IndexMap::retain
    size_t o = 0;
    for (size_t i = 0; i < len(); ++i) {
      if (keep(key(i), vals[i])) {
        if (o != i) {
          std::memcpy(key(o), key(i), sizeof(uint64_t) * 2 * W);
          vals[o] = vals[i];
        }
        ++o;
      }
    }
    keys.resize(o * 2 * W);
    vals.resize(o);
    rebuild_index();
  }
  bool get_x(const uint64_t* k, uint32_t q) const { return (k[q >> 6] >> (q & 63)) & 1u; }
  bool get_z(const uint64_t* k, uint32_t q) const { return (k[W + (q >> 6)] >> (q & 63)) & 1u; }
  static void set_bit(uint64_t* w, uint32_t q, bool b) {
    uint64_t m = 1ull << (q & 63);
    if (b) w[q >> 6] |= m; else w[q >> 6] &= ~m;
  }
  void set_x(uint64_t* k, uint32_t q, bool b) const { set_bit(k, q, b); }
  void set_z(uint64_t* k, uint32_t q, bool b) const { set_bit(k + W, q, b); }
  uint64_t weight(const uint64_t* k) const {
    uint64_t t = 0;
    for (int w = 0; w < W; ++w) t += __builtin_popcountll(k[w] | k[W + w]);
    return t;
  }

  // map_insert (data.rs:204-226): f(key, &v, child_key) -> has child, child value.
  template <class F>
  void map_insert(F f) {
    scratch_keys.clear();
    scratch_vals.clear();
    std::vector<uint64_t> ck(2 * W);
    size_t n0 = len();
    for (size_t i = 0; i < n0; ++i) {
      double cv;
      std::memcpy(ck.data(), key(i), sizeof(uint64_t) * 2 * W);
      if (f(ck.data(), vals[i], cv)) {
        scratch_keys.insert(scratch_keys.end(), ck.begin(), ck.end());
        scratch_vals.push_back(cv);
      }
    }
    for (size_t j = 0; j < scratch_vals.size(); ++j) add_assign(&scratch_keys[j * 2 * W], scratch_vals[j]);
  }
  // map_add (data.rs:255-265): rebuild into a fresh map in iteration order.
  template <class F>
  void map_add(F f) {
    OSum aux;
    aux.n = n; aux.W = W;
    aux.keys.reserve(keys.size());
    aux.vals.reserve(vals.size());
    aux.reserve_index(len());  // aux keeps its capacity across gates (aux.clear())
    std::vector<uint64_t> nk(2 * W);
    for (size_t i = 0; i < len(); ++i) {
      std::memcpy(nk.data(), key(i), sizeof(uint64_t) * 2 * W);
      double v = vals[i];
      f(nk.data(), v);
      aux.add_assign(nk.data(), v);
    }
    keys.swap(aux.keys);
    vals.swap(aux.vals);
    table.swap(aux.table);
    mask = aux.mask;
  }
  template <class F>
  void scale(F f) {
    for (size_t i = 0; i < len(); ++i) f(key(i), vals[i]);
  }

  // ---- Clifford gates (crates/ppvm-pauli-sum/src/sum/clifford.rs) ------------------
  void g_x(uint32_t q) { scale([&](const uint64_t* k, double& v) { if (get_z(k, q)) v *= -1.0; }); }
  void g_y(uint32_t q) { scale([&](const uint64_t* k, double& v) { if (get_x(k, q) ^ get_z(k, q)) v *= -1.0; }); }
  void g_z(uint32_t q) { scale([&](const uint64_t* k, double& v) { if (get_x(k, q)) v *= -1.0; }); }
  // single-qubit map_add gates: mode selects the bit map and the sign rule.
  enum Single { H, S, SDAG, SQX, SQXDAG, SQY, SQYDAG };
  void g_single(Single g, uint32_t q) {
    map_add([&](uint64_t* k, double& v) {
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
    map_add([&](uint64_t* k, double& v) {
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
    map_insert([&](uint64_t* k, double& v, double& cv) {
      if (!get_z(k, q)) return false;
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
    map_insert([&](uint64_t* k, double& v, double& cv) {
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
    map_insert([&](uint64_t* k, double& v, double& cv) {
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
  void r_zz(uint32_t a, uint32_t b, double s, double co) {
    map_insert([&](uint64_t* k, double& v, double& cv) {
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
    map_insert([&](uint64_t* k, double& v, double& cv) {
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
    map_insert([&](uint64_t* k, double& v, double& cv) {
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
  // Generic exp(-i theta/2 G): rotate_1 / rotate_2 generalised to any support.
  void r_pauli(const uint64_t* gx, const uint64_t* gz, double s, double co) {
    map_insert([&](uint64_t* k, double& v, double& cv) {
      if (!anticommutes(gx, gz, k)) return false;
      double eps = (double)rot_sign(gx, gz, k);
      double coeff = v;
      v *= co;
      for (int w = 0; w < W; ++w) { k[w] ^= gx[w]; k[W + w] ^= gz[w]; }
      cv = coeff * (eps * s);
      return true;
    });
  }
  // Clifford-angle rotation (theta = +-pi/2 with cos taken as exactly 0): anticommuting
  // P -> sign * (iGP), a bijection on words.  Tests pin it against the reference's
  // Clifford compositions (e.g. RZZ(-pi/2) == CZ, S_DAG, S_DAG).
  void r_pauli_clifford(const uint64_t* gx, const uint64_t* gz, double sin_sign) {
    map_add([&](uint64_t* k, double& v) {
      if (!anticommutes(gx, gz, k)) return;
      double eps = (double)rot_sign(gx, gz, k);
      for (int w = 0; w < W; ++w) { k[w] ^= gx[w]; k[W + w] ^= gz[w]; }
      v = v * (eps * sin_sign);
    });
  }

  // ---- noise (crates/ppvm-pauli-sum/src/sum/noise.rs) --------------------------------
  void pauli_error(uint32_t q, const double p[3]) {  // noise.rs:17-37
    double one = 1.0;
    double xf = one - p[1] * 2.0 - p[2] * 2.0;
    double zf = one - p[0] * 2.0 - p[1] * 2.0;
    double yf = one - p[0] * 2.0 - p[2] * 2.0;
    scale([&](const uint64_t* k, double& v) {
      int code = (int)get_x(k, q) | ((int)get_z(k, q) << 1);
      if (code == 1) v *= xf; else if (code == 2) v *= zf; else if (code == 3) v *= yf;
    });
  }
  void depolarize1(uint32_t q, double p) {  // noise.rs:107-116
    double f = 1.0 - p * (4.0 / 3.0);
    scale([&](const uint64_t* k, double& v) { if (get_x(k, q) | get_z(k, q)) v *= f; });
  }
  void depolarize2(uint32_t a, uint32_t b, double p) {  // noise.rs:119-129
    double f = 1.0 - p * (16.0 / 15.0);
    scale([&](const uint64_t* k, double& v) {
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
    scale([&](const uint64_t* k, double& v) {
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
    map_insert([&](uint64_t* ck, double& v, double& cv) {
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

  // ---- truncation (data.rs:275-311, strategy.rs) -------------------------------------
  void strategy() {
    double t = thr;
    retain([&](const uint64_t*, double v) { return !(std::fabs(v) < t); });  // strategy.rs:125-134
    if (maxw != UINT64_MAX) {  // strategy.rs:86-90
      uint64_t mw = maxw;
      retain([&](const uint64_t* k, double) { return weight(k) <= mw; });
    }
  }
  bool is_preserved(const uint64_t* k) const {
    size_t np = preserve.size() / (2 * W);
    for (size_t j = 0; j < np; ++j)
      if (std::memcmp(&preserve[j * 2 * W], k, sizeof(uint64_t) * 2 * W) == 0) return true;
    return false;
  }
  void truncate() {
    if (preserve.empty()) { strategy(); return; }
    std::vector<uint64_t> sk;
    std::vector<double> sv;
    for (size_t i = 0; i < len(); ++i)
      if (is_preserved(key(i))) { sk.insert(sk.end(), key(i), key(i) + 2 * W); sv.push_back(vals[i]); }
    strategy();
    for (size_t j = 0; j < sv.size(); ++j)
      if (find(&sk[j * 2 * W]) < 0) add_assign(&sk[j * 2 * W], sv[j]);
  }

  double overlap_with_zero() const {  // trace("Z?*"): fold in order over X-free words
    double acc = 0.0;
    for (size_t i = 0; i < len(); ++i) {
      const uint64_t* k = key(i);
      bool xfree = true;
      for (int w = 0; w < W; ++w) xfree &= (k[w] == 0);
      if (xfree) acc += vals[i];
    }
    return acc;
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
bool pattern_contains(const Pattern& P, const OSum& S, const uint64_t* k) {
  uint32_t pos = 0, n = S.n;
  auto code = [&](uint32_t q) { return (unsigned)S.get_x(k, q) | ((unsigned)S.get_z(k, q) << 1); };
  auto accepts = [](unsigned acc, unsigned c) { return (acc >> (c == 0 ? 0 : c == 1 ? 1 : c == 2 ? 2 : 3)) & 1u; };
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

thread_local std::string g_err;

bool qok(const OSum* s, uint32_t q) { return q < s->n; }

int run_op(OSum* s, const ppvm_op& op) {
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
    case PPVM_OP_H: if (!qok(s, op.q0)) return 1; s->g_single(OSum::H, op.q0); return 0;
    case PPVM_OP_S: if (!qok(s, op.q0)) return 1; s->g_single(OSum::S, op.q0); return 0;
    case PPVM_OP_S_DAG: if (!qok(s, op.q0)) return 1; s->g_single(OSum::SDAG, op.q0); return 0;
    case PPVM_OP_SQRT_X: if (!qok(s, op.q0)) return 1; s->g_single(OSum::SQX, op.q0); return 0;
    case PPVM_OP_SQRT_X_DAG: if (!qok(s, op.q0)) return 1; s->g_single(OSum::SQXDAG, op.q0); return 0;
    case PPVM_OP_SQRT_Y: if (!qok(s, op.q0)) return 1; s->g_single(OSum::SQY, op.q0); return 0;
    case PPVM_OP_SQRT_Y_DAG: if (!qok(s, op.q0)) return 1; s->g_single(OSum::SQYDAG, op.q0); return 0;
    case PPVM_OP_CNOT: if (!two_ok()) return 1; s->g_two(OSum::CNOT, op.q0, op.q1); return 0;
    case PPVM_OP_CZ: if (!two_ok()) return 1; s->g_two(OSum::CZ, op.q0, op.q1); return 0;
    case PPVM_OP_CY: if (!two_ok()) return 1; s->g_two(OSum::CY, op.q0, op.q1); return 0;
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
    default: return 1;
  }
}

}  // namespace

extern "C" {

void* oracle_create(uint32_t n, double thr, uint64_t maxw, uint32_t flags) {
  if (n == 0) return nullptr;
  OSum* s = new OSum();
  s->n = n;
  s->W = (int)((n + 63) / 64);
  s->thr = thr;
  s->maxw = maxw;
  s->clifford_angles = (flags & PPVM_FLAG_CLIFFORD_ANGLES) != 0;
  s->rebuild_index();
  return s;
}
void oracle_destroy(void* h) { delete (OSum*)h; }
void* oracle_clone(void* h) { return new OSum(*(OSum*)h); }
int oracle_words(void* h) { return ((OSum*)h)->W; }
size_t oracle_len(void* h) { return ((OSum*)h)->len(); }

// x, z term-major [k][W]
int oracle_add_terms(void* h, const uint64_t* x, const uint64_t* z, const double* c, size_t k) {
  OSum* s = (OSum*)h;
  std::vector<uint64_t> key(2 * s->W);
  for (size_t i = 0; i < k; ++i) {
    for (int w = 0; w < s->W; ++w) { key[w] = x[i * s->W + w]; key[s->W + w] = z[i * s->W + w]; }
    s->add_assign(key.data(), c[i]);
  }
  return 0;
}
// two_qubit_pauli_error_many: pairs (flat, k_flat even) in order, then the strategy if asked.
int oracle_two_qubit_pauli_error(void* h, const uint32_t* pairs, size_t k_flat, const double* p,
                                 int truncate) {
  OSum* s = (OSum*)h;
  if (k_flat % 2) return 1;
  for (size_t i = 0; i < k_flat; i += 2)
    if (pairs[i] >= s->n || pairs[i + 1] >= s->n || pairs[i] == pairs[i + 1]) return 1;
  for (size_t i = 0; i < k_flat; i += 2) s->two_qubit_pauli_error(pairs[i], pairs[i + 1], p);
  if (truncate) s->truncate();
  return 0;
}
int oracle_set_preserve(void* h, const uint64_t* x, const uint64_t* z, size_t k) {
  OSum* s = (OSum*)h;
  s->preserve.clear();
  for (size_t i = 0; i < k; ++i) {
    for (int w = 0; w < s->W; ++w) s->preserve.push_back(x[i * s->W + w]);
    for (int w = 0; w < s->W; ++w) s->preserve.push_back(z[i * s->W + w]);
  }
  return 0;
}
// Runs ops in order; records the live count entering each op into counts (may be NULL).
int oracle_run_ops(void* h, const ppvm_op* ops, size_t n_ops, uint64_t* counts) {
  OSum* s = (OSum*)h;
  for (size_t i = 0; i < n_ops; ++i) {
    if (counts) counts[i] = s->len();
    if (run_op(s, ops[i]) != 0) return (int)(i + 1);
  }
  return 0;
}
int oracle_pauli_rotation(void* h, const uint64_t* gx, const uint64_t* gz, double theta) {
  OSum* s = (OSum*)h;
  const double HALF_PI = 1.5707963267948966;
  if (s->clifford_angles && (theta == HALF_PI || theta == -HALF_PI)) {
    s->r_pauli_clifford(gx, gz, theta > 0 ? 1.0 : -1.0);
    return 0;
  }
  s->r_pauli(gx, gz, std::sin(theta), std::cos(theta));
  return 0;
}
double oracle_overlap_with_zero(void* h) { return ((OSum*)h)->overlap_with_zero(); }
int oracle_trace(void* h, const char* pattern, double* out) {
  OSum* s = (OSum*)h;
  Pattern P = parse_pattern(pattern);
  if (!P.ok) return 1;
  double acc = 0.0;
  for (size_t i = 0; i < s->len(); ++i)
    if (pattern_contains(P, *s, s->key(i))) acc += s->vals[i];
  *out = acc;
  return 0;
}
// PauliSum::overlap (sum/trace.rs:31-37): other.iter().map(|(k,v)| v * self[k]).sum()
double oracle_overlap(void* a, void* b) {
  OSum* A = (OSum*)a;
  OSum* B = (OSum*)b;
  double acc = 0.0;
  for (size_t i = 0; i < B->len(); ++i) {
    long j = A->find(B->key(i));
    acc += B->vals[i] * (j >= 0 ? A->vals[j] : 0.0);
  }
  return acc;
}
size_t oracle_export(void* h, uint64_t* x, uint64_t* z, double* c, size_t cap) {
  OSum* s = (OSum*)h;
  size_t n = s->len() < cap ? s->len() : cap;
  for (size_t i = 0; i < n; ++i) {
    const uint64_t* k = s->key(i);
    for (int w = 0; w < s->W; ++w) { x[i * s->W + w] = k[w]; z[i * s->W + w] = k[s->W + w]; }
    c[i] = s->vals[i];
  }
  return n;
}

}  // extern "C"
