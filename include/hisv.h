/*
 * hisv.h — C ABI of the B200-native hierarchical state-vector simulator.
 *
 * This is the drop-in boundary for the hot path of pnnl/hisvsim: the per-part
 * gather -> apply -> scatter update of a state vector (execute.hpp,
 * state_vector.hpp, loop.hpp, basic_gates.hpp) and the qubit redistribution
 * (svsim-mpi.hpp, mpi_redistributer.hpp).  The reference exposes that path to
 * Python through the pybind11 module `svsimulator_py_wrapper`
 * (py_wrapper.cpp:15-177); the pybind11 module shipped in hisvsim_b200/ binds
 * the same names onto the functions declared here.  Every entry point below
 * names the reference interface it replaces.
 *
 * Conventions
 *  - Plain C types only: pointers, sizes, fixed-width integers, doubles.  A
 *    CUDA stream is passed as `void*` (NULL = the library's own stream).
 *  - Every call returns HS_OK (0) or a negative HS_E* code and never aborts;
 *    hs_last_error() gives a one-line message for the calling thread.
 *    (The reference asserts / calls exit(); types.hpp:34-37,
 *    state_vector.hpp:194-196.)
 *  - Amplitudes are stored slot-ordered, interleaved (re, im): complex128
 *    (16 B) for HS_DTYPE_C128 and complex64 (8 B) for HS_DTYPE_C64.
 *  - Qubit q lives in slot qubit_to_slot[q]; amplitude index bit s is slot s
 *    (state_vector.hpp:41-119 keeps the same qubit<->slot permutation).
 *  - Calls are stream-ordered; functions that return host values synchronise.
 */
#ifndef HISV_H_
#define HISV_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define HS_OK 0
#define HS_E_INVALID (-1)     /* bad argument (qubit index, size, type ...) */
#define HS_E_NOMEM (-2)       /* device or host allocation failed          */
#define HS_E_CUDA (-3)        /* a CUDA runtime call failed                */
#define HS_E_UNSUPPORTED (-4) /* valid request outside what is built       */
#define HS_E_TIMEOUT (-5)     /* a bounded device-side wait expired        */
#define HS_E_NODEVICE (-6)    /* no CUDA device visible                     */

/* ---- amplitude types ----------------------------------------------------- */
#define HS_DTYPE_C128 0 /* std::complex<double>, the reference's Type (types.hpp:27) */
#define HS_DTYPE_C64 1  /* complex64, the precision form                           */

/* ---- gate types: same numbering as SvSim::GateType (basic_gates.hpp:12-44) */
enum hs_gate_type {
  HS_GATE_INVALID = 0,
  HS_GATE_ALLOC = 1,
  HS_GATE_FREE = 2,
  HS_GATE_I = 3,
  HS_GATE_X = 4,
  HS_GATE_Y = 5,
  HS_GATE_Z = 6,
  HS_GATE_H = 7,
  HS_GATE_S = 8,
  HS_GATE_T = 9,
  HS_GATE_RX = 10,
  HS_GATE_RY = 11,
  HS_GATE_RZ = 12,
  HS_GATE_RI = 13,
  HS_GATE_R1 = 14,
  HS_GATE_RXFRAC = 15,
  HS_GATE_RYFRAC = 16,
  HS_GATE_RZFRAC = 17,
  HS_GATE_RIFRAC = 18,
  HS_GATE_R1FRAC = 19,
  HS_GATE_SWAP = 20,
  HS_GATE_C1 = 21,
  HS_GATE_C2 = 22,
  HS_GATE_U1 = 23,
  HS_GATE_U2 = 24,
  HS_GATE_U3 = 25,
  HS_GATE_RXX = 26,
  HS_GATE_RYY = 27,
  HS_GATE_RZZ = 28,
  HS_GATE_TDG = 29,
  HS_GATE_SDG = 30
};

#define HS_MAX_CONTROLS 5 /* MAX_CONTROL_QUBITS, types.hpp:8 */
#define HS_MAX_TARGETS 5  /* MAX_TARGET_QUBITS, types.hpp:9  */

/*
 * One bound gate: the C form of SvSim::BoundGate (state_vector.hpp:1332-1379)
 * = an AggregateGateFactory (basic_gates.hpp:1779) + controls + targets.
 * `params` holds the constructor's complex arguments in order as (re, im)
 * pairs: theta (1-param gates), phi, lambda (U2), theta, phi, lambda (U3),
 * c00..c11 (C1), c00..c33 (C2).  Frac gates use frac_num / frac_pow
 * (AggregateGate_Frac, basic_gates.hpp:1678).  sizeof == 320.
 */
typedef struct hs_gate {
  int32_t type; /* enum hs_gate_type */
  int32_t num_controls;
  int32_t num_targets;
  int32_t controls[HS_MAX_CONTROLS];
  int32_t targets[HS_MAX_TARGETS];
  uint32_t frac_num;
  uint32_t frac_pow;
  int32_t reserved;
  double params[32];
} hs_gate;

typedef struct hs_state hs_state;

/* ---- library ------------------------------------------------------------ */
const char* hs_last_error(void);
int hs_version(void);
/* Number of CUDA devices visible (0 on a host without a GPU). */
int hs_device_count(int* count);
/* Select the device used by this thread's subsequent calls (one process per
 * GPU: rank r calls hs_device_set(local_rank)). */
int hs_device_set(int device);
int hs_device_synchronize(void);

/* ---- device timing (CUDA events on the caller's stream) ------------------- */
int hs_event_create(void** ev);
int hs_event_record(void* ev, void* stream);
int hs_event_elapsed_ms(void* start, void* stop, float* ms); /* waits for stop */
int hs_event_destroy(void* ev);

/* ---- state vector: StateVector (state_vector.hpp:41-1076) ------------------ */

/* StateVector(n, numa) (py_wrapper.cpp:143, state_vector.hpp:60-119): a
 * device-resident 2^n state initialised to |0...0>, identity slot map. */
int hs_state_create(int num_qubits, int dtype, hs_state** out);
int hs_state_destroy(hs_state* st);
int hs_state_num_qubits(const hs_state* st, int* n);
int hs_state_dtype(const hs_state* st, int* dtype);
/* Device pointer of the slot-ordered amplitude array (for zero-copy users). */
int hs_state_device_ptr(const hs_state* st, void** dptr);
/* qubit_to_slot_ / slot_to_qubit_ (state_vector.hpp:146-150,250-265). */
int hs_state_qubit_to_slot(const hs_state* st, int32_t* q2s /* [n] */);
/* Set |x> (x in qubit order), identity slot map. */
int hs_state_set_basis(hs_state* st, uint64_t x, void* stream);
/* Copy `count` amplitudes starting at slot-ordered index `first`.
 * `host` holds interleaved (re,im) of the state's dtype. */
int hs_state_copy_to_host(hs_state* st, void* host, uint64_t first, uint64_t count,
                          void* stream);
int hs_state_copy_from_host(hs_state* st, const void* host, uint64_t first,
                            uint64_t count, void* stream);
/* Permute slots back to the identity map (qubit q in slot q) with K2 passes. */
int hs_state_canonicalize(hs_state* st, void* stream);
/* Convert between dtypes (c128 -> c64 rounding, c64 -> c128 widening); the two
 * states must have the same qubit count; dst takes src's slot map. */
int hs_state_convert(const hs_state* src, hs_state* dst, void* stream);

/* ---- plain form (complex128 / complex64 state, per-gate arithmetic) -------- */

/* BoundGate::apply (state_vector.hpp:1349 -> apply 402-510): one gate, one
 * sweep over the state. */
int hs_gate_apply(hs_state* st, const hs_gate* gate, void* stream);

/* gather_and_execute_on (execute.hpp:171; live semantics of
 * gather_and_execute_on_multi, execute.hpp:318-470): one part — every gate of
 * `gates` applied in order inside one K1 launch that stages each 2^m tile of
 * the state on chip and writes it back once.  The stored amplitudes are exact
 * after the call; hs_part_run_carry (below) is the same with the rotations'
 * pending factors kept for the next part. */
int hs_part_run(hs_state* st, const hs_gate* gates, int num_gates, void* stream);

/* Several parts back to back (the loop of execute_qasm_parts,
 * qasm_assembler_standalone.py:1784-2018); part i is
 * gates[part_offsets[i] .. part_offsets[i+1]).  One or more K1 passes per
 * part; the phases that the factored one-qubit rotations leave pending are
 * carried from part to part and applied by the last pass, so the state after
 * the call is the reference's (to rounding) while the states between parts
 * are not observable. */
int hs_parts_run(hs_state* st, const hs_gate* gates, const int32_t* part_offsets,
                 int num_parts, void* stream);

/* hs_parts_run with every part planned first and then launched back to back,
 * part_ms[p] = device time of part p (CUDA events between consecutive parts;
 * synchronises).  The harvest of part timings for the cost model. */
int hs_parts_run_timed(hs_state* st, const hs_gate* gates, const int32_t* part_offsets,
                       int num_parts, float* part_ms, void* stream);

/* Deferred factors between part calls (no counterpart in the reference).
 * hs_part_run leaves the stored amplitudes exact after every call, so each
 * call applies the phase / scale factors its one-qubit rotations leave
 * pending (one op at the end of the part).  A caller that runs parts one call
 * at a time (the reference's gather_and_execute_on loop) can keep them
 * pending instead: hs_part_run_carry applies a part with the pending factors
 * of `fr` carried in and out, as hs_parts_run does between its parts, and
 * hs_frames_flush applies whatever is pending (one pass over the state, none
 * when nothing is).  While factors are pending the true state is the stored
 * amplitudes times them: flush before any other entry point reads or writes
 * the state.  The factors belong to qubits, so qubit permutations
 * (hs_permute_bits, hs_gather_qubits) may come in between. */
typedef struct hs_frames hs_frames;
int hs_frames_create(int num_qubits, hs_frames** out);
int hs_frames_destroy(hs_frames* fr);
/* *pending = 1 while any factor is pending */
int hs_frames_pending(const hs_frames* fr, int* pending);
int hs_part_run_carry(hs_state* st, hs_frames* fr, const hs_gate* gates, int num_gates,
                      void* stream);
int hs_frames_flush(hs_state* st, hs_frames* fr, void* stream);

/* Host-only: plan one part (identity slot map) without touching a device and
 * report stats[0..5] = {passes, register groups, ops, dense ops, diagonal
 * ops, tile bits}.  Used by the cost model and by tests of the planner. */
int hs_plan_stats(int num_qubits, int dtype, const hs_gate* gates, int num_gates,
                  int32_t* stats);

/* Tile-size override for K1 (0 = automatic).  Returns the previous value. */
int hs_set_tile_qubits(int m);
/* Amplitudes per thread of K1 passes: 2^r with r = 4 (default; complex128
 * tiles of 2^10 in CTAs of 64 threads, or 2^11 in CTAs of 128) or 3 (CTAs
 * twice as wide, register groups of three qubits).  Returns the previous
 * value. */
int hs_set_k1_reg_bits(int r);

/* ---- precision form (complex64 state, fused unitaries on the tensor cores) --
 * No counterpart in the reference: each part (<= 6 qubits) becomes one 64x64
 * unitary composed in FP64 (K5), applied to a complex64 state by K4 as a real
 * 128x128 GEMM on the tcgen05 tensor cores with split-BF16 operands and FP32
 * accumulation, up to two unitaries per state pass.  Parts have the meaning of
 * gather_and_execute_on's gate lists (execute.hpp:171). */
#define HS_FUSED_BF16X3 0 /* Ah*Bh + Ah*Bl + Al*Bh: ~2^-16 relative per product */
#define HS_FUSED_BF16X1 1 /* one BF16 product (fast, ~2^-8) */
int hs_fused_parts_run(hs_state* st, const hs_gate* gates, const int32_t* part_offsets,
                       int num_parts, int precision, void* stream);
/* Apply one given 64x64 unitary (row-major, interleaved re/im doubles; local
 * index bit j = qubits[j]) to a complex64 state with K4: the form of
 * gather_and_execute_on for a part whose unitary the caller already has. */
int hs_fused_apply(hs_state* st, const double* u, const int32_t* qubits, int precision,
                   void* stream);
/* K4 kernel for one unitary per pass: 2 = bulk-loaded (default: a loader
 * warp streams tiles into a shared-memory ring with bulk copies, four deep
 * for tiles of up to 2^12 amplitudes, two deep for 2^13; producer, MMA and
 * epilogue warps hand tiles over through mbarriers; passes that do not fit
 * its shape run variant 1), 1 = warp-specialised (producers load tiles
 * straight from HBM), 0 = direct (CTA-wide barriers between load / MMA /
 * drain).  Returns the previous choice. */
int hs_set_k4_variant(int variant);
/* Shape of the fused passes: unitaries applied per state pass and tile bits,
 * 1 with 10..13 (default 1, 13) or 2 with 10..12.  Returns the previous
 * shape as ops * 100 + bits. */
int hs_set_fused_shape(int max_ops_per_pass, int tile_bits);
/* K5 alone, for checking: the FP64 unitaries of the parts on an n-qubit
 * register with identity slot map.  out_u: num_parts x 64 x 64 complex128
 * (row-major, row = output basis index); out_qubits: num_parts x 6, the qubit
 * of each local bit (bit j = j-th lowest slot; parts smaller than six qubits
 * are padded with the lowest other qubits). */
int hs_fused_compose(int num_qubits, const hs_gate* gates, const int32_t* part_offsets,
                     int num_parts, double* out_u, int32_t* out_qubits);
/* out = {Re<a|b>, Im<a|b>, max|a-b|, <b|b>} in FP64 for states of any two
 * precisions (slot maps are brought to the identity first): the fidelity
 * |<a|b>|^2 / (<a|a><b|b>) and max amplitude error of the precision form. */
int hs_compare(hs_state* a, hs_state* b, double out[4]);
/* Same as hs_compare with b given as 2^n host amplitudes in qubit order (of
 * dtype bdtype), streamed through the device in 2^26-amplitude chunks: for
 * comparisons whose two states do not fit in HBM together. */
int hs_compare_host(hs_state* a, const void* host_b, int bdtype, double out[4]);

/* ---- redistribution (svsim-mpi.hpp:123-173, mpi_redistributer.hpp:100-344) */

/* In-place bit-swap pass (K2): exchange slot bits pairs[2i] <-> pairs[2i+1]
 * for all i (disjoint pairs).  Updates the slot map. */
int hs_permute_bits(hs_state* st, const int32_t* pairs, int num_pairs, void* stream);

/* SvSimMPI::gather_qubits semantics on one device (svsim-mpi.hpp:123-173 with
 * gather_slots, mpi_redistributer.hpp:265-344): slots holding the qubits in
 * `proc_qubits` become the top `num` slots (in current slot order) and all
 * other qubits keep their relative order below them.  Done as at most two
 * in-place involution passes of K2. */
int hs_gather_qubits(hs_state* st, const int32_t* proc_qubits, int num, void* stream);

/* ---- bounds-checked build (no counterpart in the reference) -----------------
 * libhisv_bounds.so is this library compiled with index checks at every
 * global and shared-memory access of the part (K1), bit-swap (K2), fused
 * (K4) and batch (K6) kernels; a failed check skips the access and sets the
 * kernel's bit (1 = K1, 2 = K2, 4 = K4, 8 = K6).  flags: the bits set since
 * the last reset (synchronises the device).  The normal build returns
 * HS_E_UNSUPPORTED. */
int hs_bounds_status(uint32_t* flags, int reset);

/* ---- FP64 reductions (K3) ------------------------------------------------- */

/* sum |a|^2 (is_normalized, state_vector.hpp:63-72) */
int hs_norm2(hs_state* st, double* out);
/* <a|b> = sum conj(a_i) b_i over qubit-aligned amplitudes (b is brought to
 * a's slot map first if the maps differ). */
int hs_inner(hs_state* a, hs_state* b, double out[2]);
/* max_i |a_i - b_i| (state_equal / operator==, state_vector.hpp:1003-1072). */
int hs_max_abs_diff(hs_state* a, hs_state* b, double* out);
/* sum |a|^2 like hs_norm2, but allocating no device memory (no counterpart in
 * the reference).  For callers that may not let the library call cudaMalloc /
 * cudaFree: hosts that give all device memory to their own pool, or loops that
 * must not incur the synchronisation those calls can cause.  Partial sums live
 * in a fixed 1 MiB array in the library's device image, so states of at most
 * 2^33 amplitudes are accepted (HS_E_UNSUPPORTED beyond).  The first call on a
 * device looks the array's address up (make it before any stream capture);
 * calls share the array, so calls that overlap on the GPU race.  Synchronises
 * `stream` before returning. */
int hs_norm2_noalloc(hs_state* st, double* out, void* stream);
/* probability(qubit, value) (state_vector.hpp:897-923), race-free. */
int hs_probability(hs_state* st, int qubit, int value, double* out);
/* <Z_i Z_j> for num_pairs qubit pairs. */
int hs_expect_zz(hs_state* st, const int32_t* pairs, int num_pairs, double* out);
/* measure(qubits, num_samples) (state_vector.hpp:925-981) with a seeded
 * generator: out[s*nq + j] = value of qubits[j] in sample s. */
int hs_measure(hs_state* st, const int32_t* qubits, int num_qubits,
               uint32_t num_samples, uint64_t seed, int32_t* out);

/* Projection (StateVector::project, state_vector.hpp:829-894): the part of
 * the state with qubits[i] = values[i] (values NULL: all 0) as a NEW state
 * over the remaining qubits, renumbered 0.. in increasing order.  norm_mode
 * 0 divides by sqrt(p), 1 divides by p as the reference does, 2 leaves it
 * unnormalised (the reference's renormalize=false); p <= 1e-12 is left as is.
 * *prob_out = p = the squared norm of the projected part (may be NULL). */
int hs_project(hs_state* st, const int32_t* qubits, const int32_t* values, int count,
               int norm_mode, hs_state** out, double* prob_out, void* stream);

/* Measured FP64 FMA throughput of this device (TFLOP/s, 2 flops per FMA):
 * the compute roofline of the complex128 part kernel. */
int hs_fp64_peak(double* tflops);

/* ---- batching form (no counterpart in the reference) -----------------------
 * Many QAOA MaxCut circuits of different qubit counts (parameter sweeps), all
 * advanced by one persistent launch (K6) replayed as a captured CUDA graph:
 * |+>^n, then p rounds of RZZ(gamma_r) on every edge and RX(2 beta_r) on every
 * qubit (the reference's RZZ/RX, basic_gates.hpp:341-363,1235-1313), complex64
 * states, and <H_C> = sum_E (1 - <Z_a Z_b>)/2 per instance accumulated in FP64.
 * edges: pairs, instance i uses pairs [edge_offsets[i], edge_offsets[i+1]);
 * gammas / betas: num_instances x p. */
typedef struct hs_batch hs_batch;
int hs_batch_create_qaoa(int num_instances, const int32_t* num_qubits,
                         const int32_t* edge_offsets, const int32_t* edges, int p,
                         const double* gammas, const double* betas, hs_batch** out);
/* New angles for the next run (the captured graph is reused). */
int hs_batch_set_params(hs_batch* b, const double* gammas, const double* betas);
/* Tile cap (6..12 qubits per pass; a cap of 12 runs CTAs of 256 threads) and
 * persistent CTAs per SM (clamped to what fits on an SM). */
int hs_batch_configure(hs_batch* b, int tile_cap, int ctas_per_sm);
/* Tiles per work item (a dequeued chunk of one step of one instance). */
int hs_batch_set_chunk(hs_batch* b, int tiles_per_item);
/* Lowest qubits (2 or 3) kept in the tile of every pass after the first:
 * 32- or 64-byte contiguous runs against one more new qubit per pass. */
int hs_batch_set_low_keep(hs_batch* b, int low);
/* Autotuner: times every (tile cap, CTAs per SM) candidate on the whole batch
 * and keeps the best, then refines the tile cap per qubit count (largest
 * states first), keeping a change only when the batch gets >= 1% faster. */
int hs_batch_tune(hs_batch* b, int32_t* best_cap, int32_t* best_ctas, double* best_ms);
/* The tile cap in force for every instance (num_instances entries). */
int hs_batch_tile_caps(hs_batch* b, int32_t* caps);
/* One whole run (graph launch, synchronised): expect_out[i] = <H_C> of
 * instance i; *ms = device time of the run between CUDA events on the
 * batch's stream, read-back of the results included (may be NULL). */
int hs_batch_run(hs_batch* b, double* expect_out, double* ms);
/* Failure detection of the persistent launch.  A work item waits (bounded)
 * until every chunk of the previous step of its instance is done; after
 * `polls` polls (~0.1 us apart; default 2^24) it gives up, the launch ends
 * early and hs_batch_run returns HS_E_TIMEOUT, leaving the device usable.
 * hs_batch_set_wait_limit sets that bound. */
int hs_batch_set_wait_limit(hs_batch* b, uint32_t polls);
/* Test hook for the above: block = 1 makes the wait of step `step` (>= 1) of
 * `instance` unreachable (its need count exceeds what the previous step can
 * complete), block = 0 restores the planned count.  No counterpart in the
 * reference. */
int hs_batch_block_step(hs_batch* b, int instance, int step, int block);
/* {work items, steps, bytes moved per run, tile cap, CTAs per SM, tiles per
 * item, lowest qubits kept in later passes' tiles, threads per CTA} */
int hs_batch_stats(hs_batch* b, int64_t* stats);
/* Complex64 amplitudes of one instance (qubit order) into host memory. */
int hs_batch_state(hs_batch* b, int instance, void* host_out);
int hs_batch_destroy(hs_batch* b);

/* ---- learned cost model (no counterpart in the reference) -------------------
 * A small MLP (in_dim -> 64 -> 64 -> 64 -> 1, ReLU, FP32) that predicts the
 * log run time of a part from its features; trained on part timings the
 * simulator measures.  Forward, backward and Adam are the library's own K7
 * kernels.  Arrays are host memory, x row-major n x in_dim.  Parameters are
 * one flat array: W1 (64 x in_dim, row-major, W[out][in]) b1 W2 b2 W3 b3 W4 b4. */
typedef struct hs_mlp hs_mlp;
int hs_mlp_create(int in_dim, uint64_t seed, hs_mlp** out);
int hs_mlp_num_params(const hs_mlp* m);
int hs_mlp_get_params(hs_mlp* m, float* host);
/* Sets the parameters and resets the Adam moments. */
int hs_mlp_set_params(hs_mlp* m, const float* host);
int hs_mlp_predict(hs_mlp* m, const float* x, int n, float* y_out);
/* Gradient of the mean squared error (1/n) sum (f(x_i) - y_i)^2 with respect
 * to every parameter, and that loss. */
int hs_mlp_gradients(hs_mlp* m, const float* x, const float* y, int n, float* grad_out,
                     float* loss_out);
/* Minibatch Adam (beta 0.9 / 0.999, eps 1e-8) on the mean squared error,
 * seeded shuffles; epoch_loss (epochs entries, may be NULL) gets each epoch's
 * mean squared error. */
int hs_mlp_train(hs_mlp* m, const float* x, const float* y, int n, int epochs, int batch,
                 float lr, uint64_t seed, float* epoch_loss);
int hs_mlp_destroy(hs_mlp* m);

/* Features of parts for the cost model (host only, no GPU): 43 floats per
 * part = {n/32, part qubits/12, gates/32, non-diagonal target qubits/12,
 * qubits at slot >= 10 /12, max slot/n, min non-diagonal target slot/n,
 * fraction of multi-qubit gates, controlled gates/32, the K1 planner's
 * passes/4, register groups/16, ops/64, dense ops/64, diagonal ops/64, tile
 * bits/12, then the count/16 of each gate type I..SDG}.  Parts are gate index
 * lists: part p = part_gates[part_offsets[p] .. part_offsets[p+1]). */
int hs_num_part_features(void);
int hs_part_features(int num_qubits, int dtype, const hs_gate* gates, int num_gates,
                     const int32_t* part_gates, const int32_t* part_offsets, int num_parts,
                     float* feats);
/* Every contiguous segment order[i..i+len) with at most max_qubits qubits and
 * max_len gates (a segment of a topological order is a valid acyclic part),
 * with its features; *count = number of segments (an error if above capacity). */
int hs_order_segments(int num_qubits, int dtype, const hs_gate* gates, int num_gates,
                      const int32_t* order, int max_qubits, int max_len, int capacity,
                      int32_t* seg_start, int32_t* seg_len, float* feats, int32_t* count);

/* ---- timers (py_wrapper.cpp:163-169) -------------------------------------- */
/* Accumulated device time of K1/K2 launches in microseconds, and the number of
 * gates / state passes issued since the last reset. */
int hs_counters(long long* apply_us, long long* gate_count, long long* pass_count);
int hs_counters_reset(void);
/* Bytes of kernel parameters (gate programs) sent with K1/K2 launches since
 * the last counter reset: the host-to-device traffic of a circuit. */
int hs_launch_bytes(long long* bytes);
/* Enable (1) or disable (0) device-time accounting for hs_counters; returns the
 * previous setting. */
int hs_set_timing(int on);

#ifdef __cplusplus
}
#endif

#endif /* HISV_H_ */
