// Internal declarations shared by the host code and the kernels of libhisv.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <complex>
#include <string>
#include <vector>

#include "hisv.h"

namespace hisv {

using cplx = std::complex<double>;

// ---- errors ---------------------------------------------------------------
int set_error(int code, const char* fmt, ...);
#define HS_CUDA(call)                                                              \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess)                                                         \
      return ::hisv::set_error(HS_E_CUDA, "%s: %s (%s:%d)", #call,                 \
                               cudaGetErrorString(e_), __FILE__, __LINE__);        \
  } while (0)
#define HS_TRY(expr)            \
  do {                          \
    int rc_ = (expr);           \
    if (rc_ != HS_OK) return rc_; \
  } while (0)

// ---- gate lowering (gatemath.cpp) ------------------------------------------
// A gate lowered to its matrix on 1 or 2 targets, in the reference's index
// convention: for 2 targets, local index i = 2*b(target0) + b(target1)
// (basic_gates.hpp:992-1004).  Controls are kept as qubits.
struct LoweredGate {
  int nt = 1;                 // 0 = identity (dropped), 1 or 2
  int targets[2] = {0, 0};    // qubits
  int nc = 0;
  int controls[HS_MAX_CONTROLS] = {0, 0, 0, 0, 0};
  cplx m[16];                 // row-major 2x2 or 4x4
};
// Returns HS_OK or HS_E_INVALID (message set) for gates the reference rejects.
int lower_gate(const hs_gate& g, int num_qubits, LoweredGate* out);

// ---- K1 part program --------------------------------------------------------
constexpr int kRegBits = 4;        // amplitudes per thread = 2^kRegBits
constexpr int kMaxTileBits = 13;   // 2^13 complex128 = 128 KiB of shared memory
constexpr int kMaxOps = 128;
constexpr int kMaxCoef = 640;      // complex coefficients (double2)
constexpr int kMaxGroups = 48;
constexpr int kMaxRuns = 16;
constexpr int kMaxFlush = 64;      // thread / outer entries of the frame flushes of a program
constexpr int kMaxRounds = 128;

// What an op does (planner statistics and the features of the learned form).
enum OpKind : uint8_t {
  OP1_ROT = 0,    // uncontrolled one-qubit rotation RY RZ as shears (K1 codes zy / y)
  OP1_DENSE = 1,  // general 2x2, uncontrolled or controlled
  OP2_DENSE = 4,  // 4x4
  OP2_SWAP = 5,   // swap |01>,|10>
  // diagonal ops: targets anywhere (register, thread or outer bits)
  OPD_PHASE = 8,  // multiply by c0 where every bit of the mask is 1
  OPD_NEG = 9,    // negate where every bit of the mask is 1
  OPD_DIAG = 10,  // multiply by c[b0 | b1 << 1] where the control mask holds
  OPD_FLUSH = 11, // multiply by G * prod over listed thread/outer bits b set of r_b
};

// K1 dispatch codes (one dense range).  j = register position of the
// target, M = register mask.
//   rotation RY(theta) RZ(beta) on register bit j:   kc_zy + j
//   rotation RY(theta) alone:                        kc_y + j
//   general 2x2, uncontrolled:                       kc_d1 + j
//   general 2x2, controlled:                         kc_c1 + j
//   sign flip, register mask M:                      kc_neg + M   (M = 0: whole thread, deferred)
//   phase c0, register mask M:                       kc_ph + M
//   general diagonal:                                kc_diag
//   4x4 uncontrolled / controlled / swap, register pair p: kc_d2 / kc_c2 / kc_sw + p
//   frame flush:                                     kc_flush
enum K1Code : uint8_t {
  kc_zy = 0,
  kc_y = 4,
  kc_d1 = 8,
  kc_c1 = 12,
  kc_neg = 16,
  kc_ph = 32,
  kc_diag = 48,
  kc_d2 = 49,
  kc_c2 = 55,
  kc_sw = 61,
  kc_flush = 67,
  kc_count = 68,
};
enum TargetWhere : uint8_t { TW_NONE = 0, TW_REG = 1, TW_THR = 2, TW_OUT = 3 };

struct DevOp {
  uint8_t kind;               // OpKind
  uint8_t code;               // K1Code
  uint8_t ja, jb;             // register positions of non-diagonal targets (ja < jb)
  uint8_t t0w, t0p, t1w, t1p;  // diagonal targets: where (TargetWhere) and position
  uint16_t coef;              // first coefficient (index into PartProgram::coef)
  uint16_t creg;              // control/mask bits that are register bits (element space)
  uint32_t cthr;              // control/mask bits that are thread bits (tile-index space)
  uint64_t couter;            // control/mask bits outside the tile (global index space)
  uint16_t fl_first, fl_n;    // flush: entries [fl_first, fl_first + fl_n) of flw/flp
  uint32_t form;              // rotation: shear form (RoundDesc), else 0
};
static_assert(sizeof(DevOp) == 32, "DevOp layout");

struct Runs {  // bit-run deposit: out |= ((x >> src) & (2^len - 1)) << dst
  uint8_t n;
  uint8_t src[kMaxRuns];
  uint8_t len[kMaxRuns];
  uint8_t dst[kMaxRuns];
};

// A round of a register group, packed in one 64-bit word (read with a single
// load): at most one rotation per register bit j, applied in the order
// j = 0, 1, ..., then ops[others[first_other .. first_other + num_other)).
//   bits  0- 3  rotation on register bit j has a phase part
//   bits  4-11  num_other
//   bits 12-19  first_other
//   bits 20+11j rotation on register bit j: bits 0-8 coefficient pair p
//               (coef[2p], coef[2p+1]; p = 0: no rotation), bits 9-10 its
//               shear form: 0 three shears, 1 without the third, 2 without
//               the first
// The planner packs a group's ops into rounds without changing their order
// where they do not commute.
using RoundDesc = uint64_t;
inline RoundDesc round_pack(uint32_t zmask, uint32_t first_other, uint32_t num_other,
                            const uint32_t pair[4], const uint32_t form[4]) {
  uint64_t w = uint64_t(zmask & 15u) | uint64_t(num_other & 255u) << 4 |
               uint64_t(first_other & 255u) << 12;
  for (int j = 0; j < 4; ++j)
    w |= uint64_t((pair[j] & 511u) | (form[j] & 3u) << 9) << (20 + 11 * j);
  return w;
}

struct GroupDesc {
  uint8_t reg_tbit[kRegBits];  // tile bit held by register bit j
  uint32_t dx[kRegBits];       // shared-memory byte-offset change of setting register bit j
  uint16_t first_op, num_ops;  // every op of the group (rotations included), in order
  uint16_t first_round, num_rounds;
  Runs thr;                    // thread index -> tile index
};

struct PartProgram {
  int32_t n;           // qubits (slots) of the state
  int32_t m;           // tile bits
  int32_t ngroups;
  int32_t nops;
  int32_t ncoef;
  int32_t rbits;       // register bits of every group (amplitudes per thread = 2^rbits)
  uint64_t ntiles;     // 2^(n-m)
  Runs tile;           // tile index -> global index
  Runs outer;          // tile number -> global index
  uint8_t tile_slot[16];  // global slot of tile bit b
  // shared-memory layout of the tile: 16-byte slot s (tile index >> SH, SH =
  // 1 for complex64) sits at slot s ^ (XOR over the set bits k of s of
  // fold[k]); fold[k] < 8 only moves a slot within its 128-byte row.  The
  // planner picks fold per program so that the lanes of every register
  // group's shared-memory accesses hit distinct banks.
  uint8_t fold[16];
  int32_t nfl;         // used entries of flw / flp
  uint8_t flw[kMaxFlush], flp[kMaxFlush];  // flush entries: where (TW_THR / TW_OUT), position
  int32_t nrounds, nothers;
  GroupDesc groups[kMaxGroups];
  DevOp ops[kMaxOps];            // per group: rotations and others in program order
  uint8_t others[kMaxOps];       // per round: indices into ops of its non-rotation ops
  RoundDesc rounds[kMaxRounds];
  // per round: up to four sign flips applied right after its rotations,
  // 16 bits each from bit 0 (0 = none): bits 0-3 register mask M (the
  // elements whose register bits cover M), bits 4-5 condition (0 none, 1 a
  // thread tile bit, 2 an outer slot), bits 6-11 its position
  uint64_t signs[kMaxRounds];
  double2 coef[kMaxCoef];
};
static_assert(sizeof(PartProgram) <= 32000, "kernel parameter space");
static_assert(kMaxOps <= 256 && kMaxCoef <= 1024, "round packing: 8-bit op indices, 9-bit coefficient pairs");

// Pending diagonal of a state under planning: the true state is
// G * (prod_q diag(1, r[q]) on qubit q) * (the stored amplitudes).  Uncontrolled
// one-qubit gates are applied as rotations in factored form, and the phases
// and scale factors they leave are carried here instead of being applied
// (they commute with every diagonal gate and are absorbed by the next
// one-qubit gate on the same qubit); a flush applies them.
struct Frames {
  std::vector<cplx> r;   // per qubit
  cplx G{1.0, 0.0};
  void reset(int n) {
    r.assign(n, cplx(1.0, 0.0));
    G = cplx(1.0, 0.0);
  }
  bool identity() const;
};

// Build the K1 programs for a sequence of lowered gates on a state whose
// qubit q sits in slot q2s[q].  `fr` carries the pending diagonal in and out;
// with `flush` the last program applies it (fr becomes the identity).  Long
// parts produce several programs (each one state pass).  Returns HS_OK or an
// error.
int plan_gates(int n, const std::vector<int>& q2s, const std::vector<LoweredGate>& gates,
               Frames* fr, bool flush, int tile_bits_hint, int dtype,
               std::vector<PartProgram>* programs);
// one self-contained part: fresh frames, flushed at the end
int plan_part(int n, const std::vector<int>& q2s, const std::vector<LoweredGate>& gates,
              int tile_bits_hint, int dtype, std::vector<PartProgram>* programs);
int current_tile_hint();  // hs_set_tile_qubits' value
// register bits per thread of K1 programs (hs_set_k1_reg_bits: 4 = 16
// amplitudes (default), 3 = 8 amplitudes)
int k1_reg_bits(int dtype);
// tiles go to 2^12 amplitudes (one 64 KiB buffer per CTA for complex128);
// complex128 with 8 amplitudes per thread stops at 2^11 (256 threads)
inline int max_tile_bits(int dtype) {
  return dtype == HS_DTYPE_C64 ? 12 : (k1_reg_bits(dtype) >= 4 ? 12 : 11);
}

// ---- K2 bit-swap program ----------------------------------------------------
struct PermProgram {
  int32_t n;
  int32_t m;            // tile bits (low run + low-high partners)
  uint64_t ntiles;      // tiles of the tile space (before orbit pairing)
  Runs tile;            // tile index -> global index (source layout)
  Runs outer;           // tile number -> global index
  uint32_t tile_swap_src;   // in tile-index space: bit pairs swapped inside a tile
  uint8_t ntswap;
  uint8_t tsa[32], tsb[32]; // tile-bit pairs swapped inside the tile
  uint64_t hh_mask_a, hh_mask_b;  // disjoint high-high pairs (global bits)
  uint8_t nhh;
  uint8_t hha[32], hhb[32];
};

// ---- precision form: fused 64x64 unitaries (kernels_fused.cu) ----------------
constexpr int kFusedBits = 6;   // qubits per fused unitary
constexpr int kFusedDim = 64;
constexpr int kFusedMaxOps = 2;  // fused unitaries applied per state pass
constexpr int kFusedABytes = 2 * 128 * 128 * 2;  // BF16 hi + lo of the real 128x128 form

// one gate of a part in the part's local bits (local bit j = j-th lowest slot)
struct FusedGate {
  int32_t nt;         // 1 or 2
  int32_t t0, t1;     // local target bits
  int32_t cmask;      // local control bits
  double2 m[16];      // 2x2 (m[0..3]) or 4x4, reference index i = 2*b(t0) + b(t1)
};

struct FusedPass {
  int32_t n, m;
  uint64_t ntiles;
  Runs tile, outer;
  int32_t nops;
  int32_t precision;                // 0: 3 BF16 products, 1: one product
  int32_t part[kFusedMaxOps];       // index of the part's A operand
  uint8_t pbits[kFusedMaxOps][kFusedBits];  // tile bit of local bit j
};

int launch_compose(const FusedGate* d_gates, const int32_t* d_offs, int nparts, double2* d_u,
                   void* d_a, cudaStream_t s);
int launch_fused(void* amp, const FusedPass& P, const void* d_a, int* d_err, cudaStream_t s);
// row-major 64 x 64 unitaries (nparts of them) -> A operands (real form, BF16 hi/lo)
int launch_pack(const double2* d_u, int nparts, void* d_a, cudaStream_t s);
int set_k4_variant(int v);  // one unitary per pass: 0 direct, 1 warp-specialised
int reduce_compare(const void* a, int adtype, const void* b, int bdtype, int n, double out[4],
                   cudaStream_t s);
int reduce_compare_count(const void* a, int adtype, const void* b, int bdtype, uint64_t count,
                         double out[4], cudaStream_t s);

// ---- batching form (kernels_batch.cu, batch_api.cpp) -------------------------
constexpr int kBatchMaxQubits = 30;
constexpr int kBatchMaxEdges = 64;
constexpr int kBatchMaxRounds = 8;
constexpr int kBatchMaxPasses = 4;   // passes per round
constexpr int kBatchMaxSteps = 32;   // passes over an instance's state, all rounds
constexpr int kBatchMaxVisits = 5;   // register-group visits per pass
// 16 amplitudes per thread: CTAs of 128 threads take tiles of up to 2^11,
// CTAs of 256 threads tiles of up to 2^12
constexpr int kBatchMaxTileBits = 12;

// one pass over an instance's state: the tile bits, register groups of 4
// tile bits, and the group visits in order.  A visit loads its group's
// amplitudes into registers, applies RX of round ra to the register bits in
// rx_a, then (ph) the cost phase of round rb, then RX of round rb to the bits
// in rx_b.  A pass that ends round r and starts round r+1 visits its groups
// forward with round r's RX, applies the phase in the last group, and visits
// them backward with round r+1's RX.
struct BatchPass {
  int32_t m;                 // tile bits
  int32_t ngroups;           // register groups (<= 3)
  int32_t nvisits;           // group visits (<= kBatchMaxVisits)
  uint32_t cut_off;          // byte offset of this pass's cut table (phase passes)
  Runs tile, outer;
  uint8_t tile_slot[16];
  uint8_t group_bits[3][4];  // tile bits in registers per group (4 each)
  uint8_t visit_group[kBatchMaxVisits];
  uint8_t rx_a[kBatchMaxVisits];  // bit j set: register bit j gets RX of round ra
  uint8_t ph[kBatchMaxVisits];    // 1: then the cost phase of round rb
  uint8_t rx_b[kBatchMaxVisits];  // bit j set: then RX of round rb
  uint8_t ra, rb;
  uint8_t phase;             // 1: a visit applies the cost phase
  int8_t tbit[kBatchMaxQubits];   // tile bit of qubit q, -1 outside the tile
  uint8_t pad[5];
};

struct BatchInstance {
  float2* amp;
  int32_t n, nedges, p, nsteps;
  uint8_t edge_a[kBatchMaxEdges], edge_b[kBatchMaxEdges];
  BatchPass pass[kBatchMaxSteps];
  uint64_t step_base;        // index of this instance's first counter
  // cut tables of the phase passes (2^m entries each: cut of the edges with
  // both ends in the pass's tile); pass 0's comes first (tile = qubits [0, m))
  const uint8_t* cut;
};

struct BatchParams {         // per instance per round (updated for sweeps)
  float2 rx[kBatchMaxRounds][2];        // cos(beta), -i sin(beta) as (c, s)
  float2 phase[kBatchMaxRounds][kBatchMaxEdges + 1];  // e^{i gamma/2 (2c - |E|)} for cut c
};

struct BatchItem {           // one (instance, step): its tiles in chunks, one work item per chunk
  uint64_t first;            // global index of the first chunk
  int32_t inst, step;
  uint32_t ntiles, chunk;    // tiles of the step, tiles per chunk
  uint32_t need;             // chunks of the previous step of this instance
};

// d_limit: the polls a dependency wait makes before it gives up (device memory)
int launch_batch(const BatchInstance* d_inst, const BatchParams* d_par, const BatchItem* d_items,
                 int nitems_groups, uint64_t total_items, uint32_t* d_counters,
                 unsigned long long* d_head, int* d_err, const uint32_t* d_limit, int grid,
                 int threads, cudaStream_t s);
constexpr uint32_t kBatchDefaultWaitLimit = 1u << 24;
int batch_max_ctas_per_sm(int threads);  // occupancy limit of the persistent kernel
int launch_batch_init(const BatchInstance* d_inst, int ninst, cudaStream_t s);
int launch_batch_expect(const BatchInstance* d_inst, int ninst, int max_n, double* d_partial,
                        double* d_out, cudaStream_t s);

// ---- launchers (kernels_*.cu) ----------------------------------------------
int launch_part(void* amp, int dtype, const PartProgram& prog, cudaStream_t s);
int launch_permute(void* amp, int dtype, int n, const int32_t* pairs, int npairs,
                   cudaStream_t s);
int reduce_norm2(const void* amp, int dtype, int n, double* out, cudaStream_t s);
int reduce_inner(const void* a, const void* b, int dtype, int n, double out[2],
                 cudaStream_t s);
int reduce_maxdiff(const void* a, const void* b, int dtype, int n, double* out,
                   cudaStream_t s);
int reduce_prob0(const void* amp, int dtype, int n, int slot, double* out, cudaStream_t s);
int reduce_zz(const void* amp, int dtype, int n, const int32_t* slot_pairs, int npairs,
              double* out, cudaStream_t s);
int reduce_chunks(const void* amp, int dtype, int n, int chunk_bits, double* host_out,
                  cudaStream_t s);
int set_basis_kernel(void* amp, int dtype, int n, uint64_t index, cudaStream_t s);
// out[j] = in[offset | deposit(j, old_slots)] for j < 2^out_bits
int project_kernel(const void* in, void* out, int dtype, int out_bits, const int* old_slots,
                   uint64_t offset, cudaStream_t s);
int scale_kernel(void* amp, int dtype, int n, double f, cudaStream_t s);
int fp64_probe(double* tflops);
int convert_kernel(const void* src, int sdtype, void* dst, int ddtype, uint64_t count,
                   cudaStream_t s);

// ---- per-device launch facts ---------------------------------------------------
// SM count of the current device (looked up once per device).
int device_sms();
// Raise the dynamic shared-memory limit of kernel `func` to 227 KiB on the
// current device, once per (device, kernel); thread-safe.
int smem_optin(const void* func);

// ---- counters ---------------------------------------------------------------
void count_pass(long long gates);
// device-time accounting (hs_set_timing): brackets launches with CUDA events
struct TimedRegion {
  cudaStream_t s;
  cudaEvent_t a = nullptr, b = nullptr;
  explicit TimedRegion(cudaStream_t s_);
  ~TimedRegion();
};

inline size_t amp_bytes(int dtype) { return dtype == HS_DTYPE_C64 ? 8 : 16; }

// ---- learned cost model (kernels_mlp.cu, mlp_api.cpp) -------------------------
// in -> 64 -> 64 -> 64 -> 1, ReLU, FP32.  Flat parameter layout (row-major,
// W[out][in]): W1 b1 W2 b2 W3 b3 W4 b4.
constexpr int kMlpHidden = 64;
constexpr int kMlpMaxIn = 64;
constexpr int kMlpSamples = 64;  // samples per block iteration
inline int mlp_num_params(int in) {
  const int H = kMlpHidden;
  return H * in + H + 2 * (H * H + H) + H + 1;
}
int launch_mlp_forward(const float* params, int in, const float* x, int n, float* out,
                       cudaStream_t s);
// per-block gradient partials of loss = sum_i scale/2 * (f(x_i) - y_i)^2 over the
// rows idx[0..n) (idx may be null: rows 0..n); partial: nblk x P, loss_partial: nblk
int launch_mlp_backward(const float* params, int in, const float* x, const float* y,
                        const int32_t* idx, int n, float scale, float* partial,
                        float* loss_partial, int nblk, cudaStream_t s);
int launch_mlp_reduce(const float* partial, const float* loss_partial, int nblk, int P,
                      float* grad, float* loss, cudaStream_t s);
int launch_mlp_adam(float* params, const float* grad, float* m, float* v, int P, float lr,
                    float beta1, float beta2, float eps, int step, cudaStream_t s);

}  // namespace hisv

// pending factors carried between hs_part_run_carry calls
struct hs_frames {
  int n = 0;
  hisv::Frames fr;
};

struct hs_state {
  int n = 0;
  int dtype = HS_DTYPE_C128;
  void* amp = nullptr;  // device, slot-ordered
  std::vector<int> q2s, s2q;
};
