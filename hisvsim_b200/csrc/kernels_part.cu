// K1: the part kernel.  One CTA holds one 2^m-amplitude tile of the state at a
// time (grid-stride over the 2^(n-m) tiles); every gate of the part is applied
// to the tile on chip and the tile is written back once.
//
// Replaces the per-part gather -> execute_on -> scatter of
// gather_and_execute_on_multi (execute.hpp:318-470) and the OpenMP loop nest
// that drives it (loop.hpp:468-962, state_vector.hpp:310-342).
//
// Layout on chip: thread t of the CTA holds E = 2^R amplitudes v[e]; the tile
// index of v[e] is deposit(t -> the group's thread bits) | deposit(e -> the
// group's register bits).  A gate targets register bits only, so it runs on
// registers with compile-time indices.  Between groups the tile goes through
// shared memory (XOR-swizzled 16-byte slots) to re-assign the register bits.
// The first group loads straight from global memory and the last group stores
// straight to it.
#include "internal.h"

namespace hisv {
namespace {

template <typename V>
struct Scalar;
template <>
struct Scalar<double2> {
  using T = double;
};
template <>
struct Scalar<float2> {
  using T = float;
};

template <typename V>
__device__ __forceinline__ V mk(typename Scalar<V>::T x, typename Scalar<V>::T y) {
  V r;
  r.x = x;
  r.y = y;
  return r;
}

// c * a + d * b with complex operands (coefficients in double, cast to T)
template <typename V>
__device__ __forceinline__ V cmac2(double2 c, V a, double2 d, V b) {
  using T = typename Scalar<V>::T;
  const T cr = T(c.x), ci = T(c.y), dr = T(d.x), di = T(d.y);
  T re = cr * a.x;
  re = fma(-ci, a.y, re);
  re = fma(dr, b.x, re);
  re = fma(-di, b.y, re);
  T im = cr * a.y;
  im = fma(ci, a.x, im);
  im = fma(dr, b.y, im);
  im = fma(di, b.x, im);
  return mk<V>(re, im);
}

template <typename V>
__device__ __forceinline__ V cmul(double2 c, V a) {
  using T = typename Scalar<V>::T;
  const T cr = T(c.x), ci = T(c.y);
  return mk<V>(fma(-ci, a.y, cr * a.x), fma(ci, a.x, cr * a.y));
}

__device__ __forceinline__ uint64_t deposit(uint64_t x, const Runs& r) {
  uint64_t out = 0;
  for (int i = 0; i < r.n; ++i)
    out |= ((x >> r.src[i]) & ((1ull << r.len[i]) - 1ull)) << r.dst[i];
  return out;
}

// shared-memory slot of tile index i: XOR the 16-byte slot within a 128-byte
// row with a fold of the higher bits, so that lanes differing in any three
// bits with distinct residues mod 3 hit distinct bank groups
__device__ __forceinline__ uint32_t swz(uint32_t i) {
  return i ^ (((i >> 3) ^ (i >> 6) ^ (i >> 9) ^ (i >> 12)) & 7u);
}

// ---- gate bodies on registers ------------------------------------------------

template <int R, int J, typename V>
__device__ __forceinline__ void apply1(V (&v)[1 << R], const DevOp& op, const double2* coef,
                                       bool thr_ok) {
  constexpr int E = 1 << R;
  const uint32_t creg = op.creg;
#pragma unroll
  for (int p = 0; p < E / 2; ++p) {
    const int e0 = ((p >> J) << (J + 1)) | (p & ((1 << J) - 1));
    const int e1 = e0 | (1 << J);
    if (!thr_ok || ((uint32_t(e0) & creg) != creg)) continue;
    V a = v[e0], b = v[e1];
    switch (op.kind) {
      case OP1_DENSE:
        v[e0] = cmac2(coef[0], a, coef[1], b);
        v[e1] = cmac2(coef[2], a, coef[3], b);
        break;
      case OP1_DIAG:
        v[e0] = cmul(coef[0], a);
        v[e1] = cmul(coef[1], b);
        break;
      case OP1_PHASE:
        v[e1] = cmul(coef[0], b);
        break;
      case OP1_NEG:
        v[e1] = mk<V>(-b.x, -b.y);
        break;
      case OP1_X:
        v[e0] = b;
        v[e1] = a;
        break;
      case OP1_H: {
        using T = typename Scalar<V>::T;
        const T s = T(0.707106781186547524401);
        v[e0] = mk<V>(s * (a.x + b.x), s * (a.y + b.y));
        v[e1] = mk<V>(s * (a.x - b.x), s * (a.y - b.y));
        break;
      }
      case OP1_Y:  // [[0,-i],[i,0]]
        v[e0] = mk<V>(b.y, -b.x);
        v[e1] = mk<V>(-a.y, a.x);
        break;
      default:
        break;
    }
  }
}

template <int R, int JA, int JB, typename V>
__device__ __forceinline__ void apply2(V (&v)[1 << R], const DevOp& op, const double2* coef,
                                       bool thr_ok) {
  constexpr int E = 1 << R;
  const uint32_t creg = op.creg;
#pragma unroll
  for (int p = 0; p < E / 4; ++p) {
    // insert zero bits at JA (< JB) and JB
    int x = ((p >> JA) << (JA + 1)) | (p & ((1 << JA) - 1));
    x = ((x >> JB) << (JB + 1)) | (x & ((1 << JB) - 1));
    const int e[4] = {x, x | (1 << JA), x | (1 << JB), x | (1 << JA) | (1 << JB)};
    if (!thr_ok || ((uint32_t(x) & creg) != creg)) continue;
    if (op.kind == OP2_SWAP) {
      V t = v[e[1]];
      v[e[1]] = v[e[2]];
      v[e[2]] = t;
    } else if (op.kind == OP2_DIAG) {
#pragma unroll
      for (int k = 0; k < 4; ++k) v[e[k]] = cmul(coef[k], v[e[k]]);
    } else {
      V a[4] = {v[e[0]], v[e[1]], v[e[2]], v[e[3]]};
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        V t0 = cmac2(coef[4 * r], a[0], coef[4 * r + 1], a[1]);
        V t1 = cmac2(coef[4 * r + 2], a[2], coef[4 * r + 3], a[3]);
        v[e[r]] = mk<V>(t0.x + t1.x, t0.y + t1.y);
      }
    }
  }
}

template <int R, typename V>
__device__ __forceinline__ void apply_op(V (&v)[1 << R], const DevOp& op, const double2* coef,
                                         bool thr_ok) {
  if (op.kind < OP2_DENSE) {
    switch (op.ja) {
      case 0: apply1<R, 0>(v, op, coef, thr_ok); break;
      case 1: if constexpr (R > 1) apply1<R, 1>(v, op, coef, thr_ok); break;
      case 2: if constexpr (R > 2) apply1<R, 2>(v, op, coef, thr_ok); break;
      case 3: if constexpr (R > 3) apply1<R, 3>(v, op, coef, thr_ok); break;
      default: break;
    }
  } else if constexpr (R >= 2) {
    const int key = op.ja * 4 + op.jb;
    switch (key) {
      case 1: apply2<R, 0, 1>(v, op, coef, thr_ok); break;
      case 2: if constexpr (R > 2) apply2<R, 0, 2>(v, op, coef, thr_ok); break;
      case 3: if constexpr (R > 3) apply2<R, 0, 3>(v, op, coef, thr_ok); break;
      case 6: if constexpr (R > 2) apply2<R, 1, 2>(v, op, coef, thr_ok); break;
      case 7: if constexpr (R > 3) apply2<R, 1, 3>(v, op, coef, thr_ok); break;
      case 11: if constexpr (R > 3) apply2<R, 2, 3>(v, op, coef, thr_ok); break;
      default: break;
    }
  }
}

}  // namespace

namespace {

template <int R, typename V>
__global__ void __launch_bounds__(512, 1)
    k1_part(V* __restrict__ sv, const __grid_constant__ PartProgram P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* sm = reinterpret_cast<V*>(smem_raw);
  constexpr int E = 1 << R;
  const uint32_t t = threadIdx.x;
  V v[E];

  // global offsets of this thread's elements for the first and the last group
  const GroupDesc& g0 = P.groups[0];
  const GroupDesc& gl = P.groups[P.ngroups - 1];
  const uint64_t gthr0 = deposit(deposit(t, g0.thr), P.tile);
  const uint64_t gthrl = deposit(deposit(t, gl.thr), P.tile);
  uint64_t greg0[R], gregl[R];
#pragma unroll
  for (int j = 0; j < R; ++j) {
    greg0[j] = deposit(1ull << g0.reg_tbit[j], P.tile);
    gregl[j] = deposit(1ull << gl.reg_tbit[j], P.tile);
  }

  for (uint64_t tile = blockIdx.x; tile < P.ntiles; tile += gridDim.x) {
    const uint64_t gbase = deposit(tile, P.outer);
    for (int g = 0; g < P.ngroups; ++g) {
      const GroupDesc& G = P.groups[g];
      const uint32_t thr = uint32_t(deposit(t, G.thr));
      if (g == 0) {
        const V* src = sv + gbase + gthr0;
#pragma unroll
        for (int e = 0; e < E; ++e) {
          uint64_t off = 0;
#pragma unroll
          for (int j = 0; j < R; ++j)
            if ((e >> j) & 1) off += greg0[j];
          v[e] = __ldcs(src + off);
        }
      } else {
        uint32_t rb[R];
#pragma unroll
        for (int j = 0; j < R; ++j) rb[j] = 1u << G.reg_tbit[j];
#pragma unroll
        for (int e = 0; e < E; ++e) {
          uint32_t idx = thr;
#pragma unroll
          for (int j = 0; j < R; ++j)
            if ((e >> j) & 1) idx |= rb[j];
          v[e] = sm[swz(idx)];
        }
        __syncthreads();  // every read of this exchange precedes the next write
      }
      for (int o = G.first_op; o < G.first_op + G.num_ops; ++o) {
        const DevOp op = P.ops[o];
        const bool thr_ok = ((thr & op.cthr) == op.cthr) && ((gbase & op.couter) == op.couter);
        apply_op<R>(v, op, P.coef + op.coef, thr_ok);
      }
      if (g == P.ngroups - 1) {
        V* dst = sv + gbase + gthrl;
#pragma unroll
        for (int e = 0; e < E; ++e) {
          uint64_t off = 0;
#pragma unroll
          for (int j = 0; j < R; ++j)
            if ((e >> j) & 1) off += gregl[j];
          __stcs(dst + off, v[e]);
        }
      } else {
        uint32_t rb[R];
#pragma unroll
        for (int j = 0; j < R; ++j) rb[j] = 1u << G.reg_tbit[j];
#pragma unroll
        for (int e = 0; e < E; ++e) {
          uint32_t idx = thr;
#pragma unroll
          for (int j = 0; j < R; ++j)
            if ((e >> j) & 1) idx |= rb[j];
          sm[swz(idx)] = v[e];
        }
        __syncthreads();  // the whole tile is in shared memory
      }
    }
  }
}

struct LaunchCfg {
  int threads;
  size_t smem;
  int grid;
};

int g_num_sms = 0;

template <int R, typename V>
int launch_k1(V* sv, const PartProgram& P, cudaStream_t s) {
  static bool attr_set[64] = {false};
  int dev = 0;
  HS_CUDA(cudaGetDevice(&dev));
  if (!attr_set[dev & 63]) {
    HS_CUDA(cudaFuncSetAttribute(k1_part<R, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(sizeof(V)) << kMaxTileBits));
    attr_set[dev & 63] = true;
  }
  if (g_num_sms == 0) HS_CUDA(cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev));
  const int threads = 1 << (P.m - R);
  const size_t smem = P.ngroups > 1 ? (sizeof(V) << P.m) : 0;
  int per_sm = 0;
  HS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k1_part<R, V>, threads, smem));
  if (per_sm < 1) return set_error(HS_E_UNSUPPORTED, "K1 tile does not fit an SM (m=%d)", P.m);
  const uint64_t want = uint64_t(g_num_sms) * uint64_t(per_sm);
  const int grid = int(P.ntiles < want ? P.ntiles : want);
  k1_part<R, V><<<grid, threads, smem, s>>>(sv, P);
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}

}  // namespace

int launch_part(void* amp, int dtype, const PartProgram& P, cudaStream_t s) {
  if (P.ngroups < 1 || P.nops < 1) return HS_OK;
  const int R = P.m < kRegBits ? P.m : kRegBits;
  if (dtype == HS_DTYPE_C128) {
    double2* a = static_cast<double2*>(amp);
    switch (R) {
      case 1: return launch_k1<1>(a, P, s);
      case 2: return launch_k1<2>(a, P, s);
      case 3: return launch_k1<3>(a, P, s);
      default: return launch_k1<4>(a, P, s);
    }
  }
  float2* a = static_cast<float2*>(amp);
  switch (R) {
    case 1: return launch_k1<1>(a, P, s);
    case 2: return launch_k1<2>(a, P, s);
    case 3: return launch_k1<3>(a, P, s);
    default: return launch_k1<4>(a, P, s);
  }
}

}  // namespace hisv
