/*
 * ppvm_cuda.h — C ABI of the B200 Pauli-propagation engine.
 *
 * This is the drop-in boundary for the Heisenberg-picture PauliSum hot path of
 * QuEraComputing/ppvm.  Every entry point below names the reference interface it
 * replaces (paths are relative to the ppvm repository).  The reference binds this
 * path through PyO3 (`crates/ppvm-python-native/src/interface.rs`); a Rust crate
 * or a Python ctypes shim binds these symbols instead.
 *
 * Conventions
 *  - A Pauli word over n qubits is two bit planes of W = ceil(n/64) u64 words:
 *    qubit q is bit (q % 64) of word (q / 64) of the X plane and of the Z plane.
 *    I=(0,0) X=(1,0) Z=(0,1) Y=(1,1), as `PauliWord` stores it
 *    (`crates/ppvm-pauli-word/src/word/data.rs:43-52`, Lsb0 bit order).
 *  - Host arrays of words are term-major: x[k*W + w].  Bits at or above n must be 0.
 *  - Coefficients are IEEE binary64.
 *  - Every call returns a ppvm_status; no call aborts the process.  The text of the
 *    last error on the calling thread is available from ppvm_last_error_string().
 *  - A handle owns its device buffers and one CUDA stream.  Calls on one handle
 *    are serialised by the caller (the reference's `&mut self`); different handles
 *    may be driven from different threads.
 *  - Gate calls with `truncate != 0` run the handle's truncation strategy once
 *    after the whole target list, as the PyO3 binding does
 *    (`interface.rs:156-310`: `<gate>_many(targets)` then `truncate()`).
 */
#ifndef PPVM_CUDA_H
#define PPVM_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ppvm_status {
  PPVM_OK = 0,
  PPVM_EINVAL = 1,    /* bad argument (odd pair list, qubit out of range, ...) */
  PPVM_ECAPACITY = 2, /* device memory exhausted / size limit exceeded */
  PPVM_ECUDA = 3,     /* a CUDA runtime call failed */
  PPVM_ETIMEOUT = 4,  /* a bounded device-side wait gave up */
  PPVM_ENODEV = 5     /* no usable CUDA device */
} ppvm_status;

typedef struct ppvm_sum ppvm_sum; /* opaque */

/* Operation codes of a gate list (ppvm_gate_list_run). */
typedef enum ppvm_opcode {
  PPVM_OP_X = 0, PPVM_OP_Y, PPVM_OP_Z, PPVM_OP_H, PPVM_OP_S, PPVM_OP_S_DAG,
  PPVM_OP_SQRT_X, PPVM_OP_SQRT_X_DAG, PPVM_OP_SQRT_Y, PPVM_OP_SQRT_Y_DAG,
  PPVM_OP_CNOT, PPVM_OP_CZ, PPVM_OP_CY,                  /* q0 = control, q1 = target */
  PPVM_OP_RX, PPVM_OP_RY, PPVM_OP_RZ,                    /* angle in theta */
  PPVM_OP_RXX, PPVM_OP_RYY, PPVM_OP_RZZ,                 /* q0, q1, theta */
  PPVM_OP_PAULI_ERROR,                                   /* q0, p[0..2] = (px, py, pz) */
  PPVM_OP_DEPOLARIZE1,                                   /* q0, theta = p */
  PPVM_OP_DEPOLARIZE2,                                   /* q0, q1, theta = p */
  PPVM_OP_TRUNCATE,                                      /* run the strategy */
  PPVM_OP_AMPLITUDE_DAMPING,                             /* q0, theta = gamma */
  PPVM_OP_LOSS_CHANNEL,                                  /* q0, theta = p (lossy sums) */
  PPVM_OP_RESET_LOSS_CHANNEL,                            /* q0 (lossy sums only) */
  PPVM_OP_CORRELATED_LOSS_CHANNEL,                       /* q0, q1, p[0..2] (lossy sums) */
  PPVM_OP_COUNT_
} ppvm_opcode;

typedef struct ppvm_op {
  uint32_t code;  /* ppvm_opcode */
  uint32_t q0;
  uint32_t q1;
  uint32_t flags; /* reserved, 0 */
  double theta;
  double p[3];
} ppvm_op;

/* Sum creation options (bit flags for ppvm_sum_create2). */
#define PPVM_FLAG_CLIFFORD_ANGLES 1u /* treat Pauli rotations at theta = +-pi/2 as the
                                        Clifford they equal (cos = 0, sin = +-1 exactly) */
#define PPVM_FLAG_EXACT_ORDER 2u     /* keep the reference's term order (IndexMap insertion
                                        order) through every op: disables fused rotation runs,
                                        which reorder terms (same terms, same coefficients) */
#define PPVM_FLAG_LOSSY 4u           /* lossy words (LossyPauliWord): each qubit may also be lost
                                        (L); at most 256 qubits.  Words of a lossy sum are passed
                                        with 2*ceil(n/64) u64 per plane: the X plane's upper half
                                        holds the loss bits (qubit q at bit q%64 of word
                                        ceil(n/64) + q/64), the Z plane's upper half is zero, and a
                                        lost qubit has x = z = 0 in the lower halves.  A lossy sum
                                        keeps the reference's term order through every op (as
                                        with PPVM_FLAG_EXACT_ORDER): the correlated loss channel
                                        adds up to three children per key in that order */

/* ---- lifetime ------------------------------------------------------------------ */

/* PauliSum::builder().n_qubits(n).strategy(CombinedStrategy(CoefficientThreshold(min_abs_coeff),
 * MaxPauliWeight(max_weight))).capacity(..).build()  (crates/ppvm-pauli-sum/src/sum/data.rs:65-91,
 * strategy built as in crates/ppvm-python-native/src/interface.rs:51-57,78-98).
 * max_weight = UINT64_MAX disables the weight cap (crates/ppvm-pauli-sum/src/strategy.rs:86-88).
 * capacity_hint = initial term capacity (0 = a small default); storage grows on demand. */
ppvm_status ppvm_sum_create(ppvm_sum** out, uint32_t n_qubits, double min_abs_coeff,
                            uint64_t max_weight, size_t capacity_hint);
/* As ppvm_sum_create, plus option flags (PPVM_FLAG_*) and a device ordinal. */
ppvm_status ppvm_sum_create2(ppvm_sum** out, uint32_t n_qubits, double min_abs_coeff,
                             uint64_t max_weight, size_t capacity_hint, uint32_t flags,
                             int device);
/* Drop (data.rs:40 `PauliSum` owns both maps). NULL is accepted. */
ppvm_status ppvm_sum_destroy(ppvm_sum* sum);
/* Clone (data.rs:40 derive(Clone); interface.rs:373-375 __copy__): device-to-device copy. */
ppvm_status ppvm_sum_clone(const ppvm_sum* src, ppvm_sum** out);
/* Bind the handle to a caller-owned cudaStream_t (NULL = the handle's own stream). */
ppvm_status ppvm_sum_set_stream(ppvm_sum* sum, void* cuda_stream);

/* ---- terms --------------------------------------------------------------------- */

/* `ps += (word, c)` for each of k terms, in order (crates/ppvm-pauli-sum/src/sum/ops.rs:140-151
 * -> IndexMap entry().and_modify(+=).or_insert, crates/ppvm-traits/src/map/hashmap.rs:40-44). */
ppvm_status ppvm_sum_add_terms(ppvm_sum* sum, const uint64_t* x, const uint64_t* z,
                               const double* c, size_t k);
/* Same for one Pauli string "IXYZ..." of length n ('_' skipped as in word/data.rs:332-377). */
ppvm_status ppvm_sum_add_string(ppvm_sum* sum, const char* word, double c);
/* preserve_strings of the builder (data.rs:75-77, restore logic data.rs:283-310). */
ppvm_status ppvm_sum_set_preserve(ppvm_sum* sum, const uint64_t* x, const uint64_t* z, size_t k);

/* ---- one sum spread over several ranks (hash-owner sharding) ---------------------- */
/* No counterpart in the reference, which keeps a sum in one process.  A sum is split over
 * n_parts ranks, every key on one rank.  Before a step that merges keys differing in the
 * bits (mask_x, mask_z) (a rotation: its generator's bits; a fused RX run: the run's qubits
 * in the X plane; RZ: in the Z plane), every rank calls ppvm_sum_shard_export: its terms go,
 * as rows of 2W+1 u64 (x[W], z[W], the coefficient's bits) into the DEVICE buffer d_rows
 * (room for at least len() rows), grouped by owner p = hash(key with the mask bits cleared)
 * mod n_parts, owners in order and terms in their order within an owner; counts[p] gets each
 * owner's row count, and the sum is left empty.  The caller exchanges the rows between the
 * ranks (an all-to-all) and gives each rank the rows it owns with ppvm_sum_shard_append,
 * which appends them without merging: keys never repeat across ranks.  Every key that the
 * step can merge then lives on one rank, and the step runs on each rank alone.  n_parts is at
 * most 32; mask_x and mask_z hold the sum's W words each.  Both calls synchronise the sum's
 * stream before they return. */
ppvm_status ppvm_sum_shard_export(ppvm_sum* sum, const uint64_t* mask_x, const uint64_t* mask_z,
                                  uint32_t n_parts, void* d_rows, size_t rows_cap, uint64_t* counts);
ppvm_status ppvm_sum_shard_append(ppvm_sum* sum, const void* d_rows, size_t k);

/* len() (data.rs:165-167; interface.rs:389-391). */
ppvm_status ppvm_len(const ppvm_sum* sum, size_t* out);
/* terms() (interface.rs:393-395): copies up to cap terms in the sum's iteration order. */
ppvm_status ppvm_export_terms(const ppvm_sum* sum, uint64_t* x, uint64_t* z, double* c,
                              size_t cap, size_t* n_out);
/* weights() / current_max_weight() (interface.rs:397-403; PauliWord::weight, word/data.rs:150-182). */
ppvm_status ppvm_weights(const ppvm_sum* sum, uint32_t* w, size_t cap, size_t* n_out);
ppvm_status ppvm_current_max_weight(const ppvm_sum* sum, uint64_t* out);
/* __eq__ (data.rs:345-352): same n_qubits and same key->value map (order-free). */
ppvm_status ppvm_equal(const ppvm_sum* a, const ppvm_sum* b, int* out);

/* ---- Clifford gates (crates/ppvm-pauli-sum/src/sum/clifford.rs:37-221) ----------- */
/* Single-qubit: targets[k]; CliffordBatch `*_many` loops (crates/ppvm-traits/src/traits/clifford.rs:175-258). */
ppvm_status ppvm_x(ppvm_sum* sum, const uint32_t* targets, size_t k, int truncate);
ppvm_status ppvm_y(ppvm_sum* sum, const uint32_t* targets, size_t k, int truncate);
ppvm_status ppvm_z(ppvm_sum* sum, const uint32_t* targets, size_t k, int truncate);
ppvm_status ppvm_h(ppvm_sum* sum, const uint32_t* targets, size_t k, int truncate);
ppvm_status ppvm_s(ppvm_sum* sum, const uint32_t* targets, size_t k, int truncate);
ppvm_status ppvm_s_dag(ppvm_sum* sum, const uint32_t* targets, size_t k, int truncate);
ppvm_status ppvm_sqrt_x(ppvm_sum* sum, const uint32_t* targets, size_t k, int truncate);
ppvm_status ppvm_sqrt_x_dag(ppvm_sum* sum, const uint32_t* targets, size_t k, int truncate);
ppvm_status ppvm_sqrt_y(ppvm_sum* sum, const uint32_t* targets, size_t k, int truncate);
ppvm_status ppvm_sqrt_y_dag(ppvm_sum* sum, const uint32_t* targets, size_t k, int truncate);
/* Two-qubit: flat (control, target) pairs; odd k_flat -> PPVM_EINVAL
 * (crates/ppvm-python-native/src/lib.rs:12-22 flat_pairs). */
ppvm_status ppvm_cnot(ppvm_sum* sum, const uint32_t* pairs_flat, size_t k_flat, int truncate);
ppvm_status ppvm_cz(ppvm_sum* sum, const uint32_t* pairs_flat, size_t k_flat, int truncate);
ppvm_status ppvm_cy(ppvm_sum* sum, const uint32_t* pairs_flat, size_t k_flat, int truncate);

/* ---- rotations (crates/ppvm-pauli-sum/src/sum/rot1.rs:44-143, rot2.rs:12-184) ----- */
ppvm_status ppvm_rx(ppvm_sum* sum, const uint32_t* targets, size_t k, double theta, int truncate);
ppvm_status ppvm_ry(ppvm_sum* sum, const uint32_t* targets, size_t k, double theta, int truncate);
ppvm_status ppvm_rz(ppvm_sum* sum, const uint32_t* targets, size_t k, double theta, int truncate);
/* RotXY::r = rz(phi); rx(theta); rz(-phi) (rot1.rs:131-143; interface.rs:281-285). */
ppvm_status ppvm_r(ppvm_sum* sum, uint32_t q, double axis_angle, double theta, int truncate);
ppvm_status ppvm_rxx(ppvm_sum* sum, const uint32_t* pairs_flat, size_t k_flat, double theta, int truncate);
ppvm_status ppvm_ryy(ppvm_sum* sum, const uint32_t* pairs_flat, size_t k_flat, double theta, int truncate);
ppvm_status ppvm_rzz(ppvm_sum* sum, const uint32_t* pairs_flat, size_t k_flat, double theta, int truncate);
/* Generic Pauli rotation exp(-i theta/2 G), G given by its X/Z planes (W words each).
 * Generalises RotationOne::rotate_1 (rot1.rs:49-52) and RotationTwo::rotate_2 (rot2.rs:17-60)
 * to any support: commuting P is unchanged; anticommuting P -> cos(theta) P + sin(theta) iGP. */
ppvm_status ppvm_pauli_rotation(ppvm_sum* sum, const uint64_t* gx, const uint64_t* gz,
                                double theta, int truncate);

/* ---- noise channels (crates/ppvm-pauli-sum/src/sum/noise.rs) ------------------------ */
/* PauliError::pauli_error (noise.rs:17-37), p = (px, py, pz); pauli_error_many loops. */
ppvm_status ppvm_pauli_error(ppvm_sum* sum, const uint32_t* targets, size_t k, const double p[3],
                             int truncate);
/* Depolarizing::depolarize1 / depolarize2 (noise.rs:107-129). */
ppvm_status ppvm_depolarize1(ppvm_sum* sum, const uint32_t* targets, size_t k, double p, int truncate);
ppvm_status ppvm_depolarize2(ppvm_sum* sum, const uint32_t* pairs_flat, size_t k_flat, double p,
                             int truncate);
/* Lossy sums (PPVM_FLAG_LOSSY) only; PPVM_EINVAL on a plain sum.
 * LossChannel::loss_channel (crates/ppvm-pauli-sum/src/sum/noise.rs:165-181; Python binding
 * crates/ppvm-python-native/src/interface.rs:18-24) on each target: L -> keeps, plus I with p;
 * I, X, Y, Z -> (1 - p). */
ppvm_status ppvm_loss_channel(ppvm_sum* sum, const uint32_t* targets, size_t k, double p, int truncate);
/* ResetLossChannel::reset_loss_channel (noise.rs:245-275; interface.rs:40-46) on each target:
 * L -> 0; I, Z -> keeps, plus L with the same coefficient; X, Y unchanged. */
ppvm_status ppvm_reset_loss_channel(ppvm_sum* sum, const uint32_t* targets, size_t k, int truncate);
/* CorrelatedLossChannel::correlated_loss_channel (noise.rs:184-243; interface.rs:26-38) on each
 * pair (a, b) of pairs_flat (even length, else PPVM_EINVAL), p = {p0, p1, p2} as the reference
 * documents them (both lost together, one lost, the second lost after the first). */
ppvm_status ppvm_correlated_loss_channel(ppvm_sum* sum, const uint32_t* pairs_flat, size_t k_flat,
                                         const double p[3], int truncate);
/* MaxLossWeight (crates/ppvm-pauli-sum/src/strategy.rs:145-180) of a lossy sum's strategy, run
 * after the coefficient threshold and the weight cap, as the Python binding's lossy tiers
 * combine them (interface.rs:58-66).  UINT64_MAX (the default) turns it off. */
ppvm_status ppvm_sum_set_max_loss_weight(ppvm_sum* sum, uint64_t max_loss_weight);
/* TwoQubitPauliError::two_qubit_pauli_error (noise.rs:39-105), applied pair by pair
 * (two_qubit_pauli_error_many, crates/ppvm-traits/src/traits/noise.rs:77-81).  p[0..15) are
 * the probabilities of IX IY IZ XI XX XY XZ YI YX YY YZ ZI ZX ZY ZZ, first letter on the
 * pair's first qubit; a term is scaled by 1 - 2 * (sum of the p of the Paulis that
 * anticommute with it on the pair).  Odd k_flat: PPVM_EINVAL. */
ppvm_status ppvm_two_qubit_pauli_error(ppvm_sum* sum, const uint32_t* pairs_flat, size_t k_flat,
                                       const double p[15], int truncate);
/* AmplitudeDamping::amplitude_damping (noise.rs:132-163) on qubit q, Heisenberg adjoint:
 * Z -> (1 - gamma) Z + gamma I, X/Y -> sqrt(1 - gamma) X/Y, I -> I.  The I child merges
 * into an existing term with `+=` or is appended in parent order, as map_insert does. */
ppvm_status ppvm_amplitude_damping(ppvm_sum* sum, uint32_t q, double gamma, int truncate);

/* ---- truncation, readout ---------------------------------------------------------- */
/* PauliSum::truncate (data.rs:275-311) with CombinedStrategy(CoefficientThreshold, MaxPauliWeight)
 * (crates/ppvm-pauli-sum/src/strategy.rs:12-30,73-90,125-134). */
ppvm_status ppvm_truncate(ppvm_sum* sum);
/* overlap_with_zero() = trace("Z?*") (interface.rs:122-130): sum of c over words without X bits. */
ppvm_status ppvm_overlap_with_zero(ppvm_sum* sum, double* out);
/* <0..0| O |0..0> of the propagated observable; the same quantity as overlap_with_zero. */
ppvm_status ppvm_expectation(ppvm_sum* sum, double* out);
/* trace(pattern) (interface.rs:122-126) for the PauliPattern grammar of
 * crates/ppvm-pauli-word/src/pattern/parse.rs:32-127, matched as pattern/contains.rs:120-151. */
ppvm_status ppvm_trace(ppvm_sum* sum, const char* pattern, double* out);
/* PauliSum::overlap (crates/ppvm-pauli-sum/src/sum/trace.rs:31-37): sum_k a[k] * b[k]. */
ppvm_status ppvm_overlap(ppvm_sum* a, ppvm_sum* b, double* out);

/* overlap_with_zero for terms the caller already holds in device memory, for callers that
 * cannot let a library allocate device memory: frameworks whose own pool owns the GPU's
 * memory, or latency-critical loops where cudaMalloc/cudaFree would stall the device.
 * No counterpart in the reference; it computes what ppvm_overlap_with_zero computes.
 *   d_x      X plane words, word w of term i at d_x[w * x_stride + i] (x_stride >= n_terms)
 *   n_words  words per plane, 1..8 (up to 512 qubits)
 *   d_c      n_terms coefficients;  d_out  one double, written with the sum
 *   cuda_stream  stream the work is queued on (NULL: the default stream); asynchronous
 * Allocates nothing: its working memory is a fixed 32 KiB array compiled into the library,
 * held on every GPU that loads the library until the process exits.  Limit: n_terms <=
 * 16,777,216 (one partial sum per 4096 terms); larger inputs return PPVM_EINVAL.  Every
 * call looks up that array's device address on the current device (a lookup that allocates
 * nothing); the first call on a device may also load the library's device code, so make
 * that first call before any stream capture.  All calls on a device share the array: calls
 * whose kernels overlap on the GPU (unordered streams) race and may return wrong sums. */
ppvm_status ppvm_overlap_with_zero_noalloc(const uint64_t* d_x, size_t x_stride, uint32_t n_words,
                                           const double* d_c, size_t n_terms, double* d_out,
                                           void* cuda_stream);

/* ---- fused gate lists ---------------------------------------------------------------- */
/* Runs ops[0..n_ops) in order; PPVM_OP_TRUNCATE marks where the strategy runs.  Consecutive
 * Clifford ops are fused into one device pass.  Equivalent to calling the per-gate
 * functions above with truncate = 0 plus ppvm_truncate at each TRUNCATE op. */
ppvm_status ppvm_gate_list_run(ppvm_sum* sum, const ppvm_op* ops, size_t n_ops);
/* Number of live terms entering each op of the last ppvm_gate_list_run (the numerator of
 * the term-gate-updates metric); cap entries are written, n_out = n_ops of that run. */
ppvm_status ppvm_last_run_live_counts(const ppvm_sum* sum, uint64_t* counts, size_t cap,
                                      size_t* n_out);
/* The composed map of a list of Clifford ops (X..CY, and rotations at theta = +-pi/2 taken
 * as the Clifford they equal), as a gate list applies it to a sum's terms: row 2q is the
 * image of X_q, row 2q+1 the image of Z_q, as W-word X/Z planes (img_x[row*W + w],
 * img_z[row*W + w]) and a sign (image = (-1)^sign[row] * word).  2*n_qubits rows.  Host
 * only; no device is needed.  No per-call counterpart in the reference: the reference maps
 * the terms gate by gate (`crates/ppvm-pauli-sum/src/sum/clifford.rs:37-221`); this is the
 * map that ppvm_gate_list_run applies in one pass to runs of kTabMinOps (8) or more
 * Clifford ops. */
ppvm_status ppvm_clifford_tableau(uint32_t n_qubits, const ppvm_op* ops, size_t n_ops,
                                  uint64_t* img_x, uint64_t* img_z, uint8_t* sign);
/* Bytes this handle has copied host->device and device->host since it was created
 * (terms, op and run descriptors, tableaux, control blocks, op logs, results). */
ppvm_status ppvm_transfer_counters(const ppvm_sum* sum, uint64_t* h2d_bytes, uint64_t* d2h_bytes);
/* Kernels this handle has launched since it was created (all families, readouts included). */
ppvm_status ppvm_launch_count(const ppvm_sum* sum, uint64_t* out);

/* ---- term-budget and learned truncation ---------------------------------------------- */
/* No counterpart in the reference, which truncates by |coefficient| and Pauli weight only
 * (`crates/ppvm-pauli-sum/src/strategy.rs:12-170`).  A term-budget truncation keeps the
 * `budget` terms of highest priority (exactly budget when the sum is larger), in order.
 * Priority is |c| (mlp = NULL) or the score of a term-priority network: a BF16 tensor-core
 * MLP 8 -> 64 -> 64 -> 1 (GELU) over per-term features, trained to predict
 * log10 |contribution of the term to <O>|.  Features, for a sum on an L x L lattice (qubit
 * r*L + c) with `layers_left` layers still to apply: weight/16, (log10|c| + 6)/6,
 * layers_left/8, #X/8, #Y/8, #Z/8, nearest-neighbour bonds inside the support/8,
 * weight*layers_left/64.  digit_bits (8 or 11; 0 = 8) is the radix-select digit width. */
typedef struct ppvm_mlp ppvm_mlp; /* opaque */
ppvm_status ppvm_truncate_budget(ppvm_sum* sum, uint64_t budget, const ppvm_mlp* mlp,
                                 uint32_t lattice_l, uint32_t layers_left, int digit_bits);
/* Features of the current terms, in iteration order: out[i*8 + k], up to cap rows. */
ppvm_status ppvm_term_features(ppvm_sum* sum, uint32_t lattice_l, uint32_t layers_left, float* out,
                               size_t cap, size_t* n_out);
/* The network: 4801 FP32 parameters (W1[64][8], b1[64], W2[64][64], b2[64], w3[64], b3),
 * seeded uniform initialisation.  Training runs on the device: per minibatch one
 * forward+backward kernel (squared error on the targets) and one Adam step (beta 0.9,
 * 0.999); samples are shuffled every epoch with a seeded permutation.  ppvm_mlp_grad
 * returns the gradient of the mean squared error over all n samples without updating. */
ppvm_status ppvm_mlp_create(ppvm_mlp** out, uint64_t seed, int device);
ppvm_status ppvm_mlp_destroy(ppvm_mlp* mlp);
ppvm_status ppvm_mlp_set_params(ppvm_mlp* mlp, const float* params, size_t n);
ppvm_status ppvm_mlp_get_params(const ppvm_mlp* mlp, float* params, size_t n);
ppvm_status ppvm_mlp_train(ppvm_mlp* mlp, const float* feats, const float* targets, size_t n, int epochs,
                           int batch, float lr, uint64_t seed, float* last_epoch_loss);
ppvm_status ppvm_mlp_grad(ppvm_mlp* mlp, const float* feats, const float* targets, size_t n, float* grads,
                          float* loss);
ppvm_status ppvm_mlp_predict(ppvm_mlp* mlp, const float* feats, size_t n, float* out);

/* ---- batches of independent sums ----------------------------------------------------- */
/* Many independent PauliSums (instances), each with its own qubit count, truncation
 * strategy, initial terms and gate list, advanced together on one GPU: one CTA per
 * instance, one launch per Trotter layer (a layer ends at every second TRUNCATE of an
 * instance's list).  Each instance's result equals a ppvm_sum run of the same list with
 * PPVM_FLAG_EXACT_ORDER: same terms in the same order, same coefficients.  The reference runs such sets one PauliSum at a time
 * (its benches loop over circuits, `crates/ppvm-pauli-sum/benches/trotter.rs:28-44`); there
 * is no batch object in the reference.  Supported ops: Cliffords, rotations, Pauli-error and
 * depolarising channels, TRUNCATE (no amplitude damping or loss channels, no explicit
 * generators or preserve strings); set_ops refuses the others with PPVM_EINVAL.  Instances
 * have up to 512 qubits. */
typedef struct ppvm_batch ppvm_batch; /* opaque */
ppvm_status ppvm_batch_create(ppvm_batch** out, size_t n_inst, const uint32_t* n_qubits,
                              const double* min_abs_coeff, const uint64_t* max_weight,
                              uint32_t flags, int device);
ppvm_status ppvm_batch_destroy(ppvm_batch* batch);
ppvm_status ppvm_batch_set_stream(ppvm_batch* batch, void* cuda_stream);
/* Initial terms of instance `inst` (ceil(n/64) words per plane), merged with += in order. */
ppvm_status ppvm_batch_add_terms(ppvm_batch* batch, size_t inst, const uint64_t* x,
                                 const uint64_t* z, const double* c, size_t k);
/* Gate list of instance `inst` (as ppvm_gate_list_run takes it). */
ppvm_status ppvm_batch_set_ops(ppvm_batch* batch, size_t inst, const ppvm_op* ops, size_t n_ops);
/* Gate lists of every instance at once (ops[i], n_ops[i] for instance i; n_inst of each),
 * packed by several host threads.  All or nothing: on a bad list no instance changes and the
 * error names the first failing instance. */
ppvm_status ppvm_batch_set_ops_all(ppvm_batch* batch, const ppvm_op* const* ops, const size_t* n_ops);
/* Runs every instance from its initial terms through its whole list.  Inputs changed by
 * the setters since the last run (8-byte op records, parameter tables, initial terms) go to
 * the device in one copy from a pinned staging buffer; the first run of a batch launches the
 * layers directly, later runs of the unchanged batch replay them as CUDA graphs. */
ppvm_status ppvm_batch_run(ppvm_batch* batch);
/* The same in one launch: each CTA runs its instance's whole list. */
ppvm_status ppvm_batch_run_persistent(ppvm_batch* batch);
/* Term capacity per instance (n_inst values): reserve raises capacities before a run (a
 * caller that knows the peak sizes avoids the growth replays of a first run); get reads the
 * current ones (after a run: at least each instance's peak). */
ppvm_status ppvm_batch_reserve(ppvm_batch* batch, const uint64_t* caps);
ppvm_status ppvm_batch_get_capacity(const ppvm_batch* batch, uint64_t* caps);
/* Launch configuration: CTA size (128, 256, 512), items per thread (2, 4) and pair-table
 * slots per term of capacity (2, 4).  ppvm_batch_autotune times every combination on this
 * batch (a full run each) and keeps the fastest; best_ms = its run time. */
ppvm_status ppvm_batch_set_config(ppvm_batch* batch, int block, int items, int table_factor);
ppvm_status ppvm_batch_get_config(const ppvm_batch* batch, int* block, int* items, int* table_factor);
ppvm_status ppvm_batch_autotune(ppvm_batch* batch, int* block, int* items, int* table_factor,
                                double* best_ms);
/* Readouts after a run: overlap_with_zero of every instance (n_inst doubles), live terms,
 * terms of one instance (its own word count per plane), term-gate updates (per instance
 * and total; NULL skips either). */
ppvm_status ppvm_batch_overlap_with_zero(ppvm_batch* batch, double* out);
ppvm_status ppvm_batch_len(const ppvm_batch* batch, size_t inst, size_t* out);
ppvm_status ppvm_batch_export_terms(ppvm_batch* batch, size_t inst, uint64_t* x, uint64_t* z,
                                    double* c, size_t cap, size_t* n_out);
ppvm_status ppvm_batch_term_gate_updates(const ppvm_batch* batch, uint64_t* per_inst, uint64_t* total);
/* Bytes this batch has copied host->device and device->host since it was created. */
ppvm_status ppvm_batch_transfer_counters(const ppvm_batch* batch, uint64_t* h2d_bytes, uint64_t* d2h_bytes);

/* ---- memory -------------------------------------------------------------------------- */
/* The large buffers of a sum (term planes, scratch) and of a batch (term pool, input block)
 * come from a per-device cache: a destroyed or grown sum or batch gives them back to the
 * cache, and later ones reuse them without cudaMalloc/cudaFree (which synchronise the
 * device).  This call returns every cached buffer to the driver, and frees the pinned host
 * buffer that stages the batches' uploads.  No counterpart in the reference (Rust's
 * allocator plays this part). */
ppvm_status ppvm_release_cached_memory(void);

/* ---- diagnostics ------------------------------------------------------------------- */
/* Thread-local text of the last failing call ("" if none). */
const char* ppvm_last_error_string(void);
/* Device time per kernel family, accumulated while profiling is on (CUDA events on the
 * handle's stream).  names: NUL-separated list written to `names` (cap bytes). */
ppvm_status ppvm_profile_enable(ppvm_sum* sum, int on);
ppvm_status ppvm_profile_read(ppvm_sum* sum, char* names, size_t names_cap, double* ms,
                              uint64_t* launches, uint64_t* bytes, size_t cap, size_t* n_out);
/* Library version string. */
const char* ppvm_version(void);

#ifdef __cplusplus
}
#endif
#endif /* PPVM_CUDA_H */
