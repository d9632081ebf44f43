// K7: the learned cost model's network, forward, backward and Adam, in FP32.
// One block handles 64 samples at a time with the whole parameter set, the
// activations of its samples and its gradient accumulators in shared memory
// (about 160 KB); gradients leave as per-block partials that a second kernel
// sums in a fixed order, so training is deterministic.
#include "internal.h"

namespace hisv {
namespace {

constexpr int H = kMlpHidden;
constexpr int SB = kMlpSamples;
constexpr int LDH = H + 1;  // odd row strides: no shared-memory bank conflicts
constexpr int kThreads = 256;

struct Offs {  // flat parameter offsets (global layout)
  int w1, b1, w2, b2, w3, b3, w4, b4, P;
  __host__ __device__ explicit Offs(int in) {
    w1 = 0;
    b1 = w1 + H * in;
    w2 = b1 + H;
    b2 = w2 + H * H;
    w3 = b2 + H;
    b3 = w3 + H * H;
    w4 = b3 + H;
    b4 = w4 + H;
    P = b4 + 1;
  }
};

// shared-memory image of the parameters: weight rows padded to odd strides
struct SParams {
  float *w1, *b1, *w2, *b2, *w3, *b3, *w4, *b4;
  int ld1;
};

__device__ float* carve(float*& p, int n) {
  float* r = p;
  p += n;
  return r;
}

__device__ SParams load_params(const float* __restrict__ g, int in, float*& sm) {
  const Offs o(in);
  SParams s;
  s.ld1 = in + 1;
  s.w1 = carve(sm, H * s.ld1);
  s.b1 = carve(sm, H);
  s.w2 = carve(sm, H * LDH);
  s.b2 = carve(sm, H);
  s.w3 = carve(sm, H * LDH);
  s.b3 = carve(sm, H);
  s.w4 = carve(sm, H);
  s.b4 = carve(sm, 4);
  for (int i = threadIdx.x; i < H * in; i += kThreads) s.w1[(i / in) * s.ld1 + i % in] = g[o.w1 + i];
  for (int i = threadIdx.x; i < H * H; i += kThreads) {
    s.w2[(i / H) * LDH + i % H] = g[o.w2 + i];
    s.w3[(i / H) * LDH + i % H] = g[o.w3 + i];
  }
  for (int i = threadIdx.x; i < H; i += kThreads) {
    s.b1[i] = g[o.b1 + i];
    s.b2[i] = g[o.b2 + i];
    s.b3[i] = g[o.b3 + i];
    s.w4[i] = g[o.w4 + i];
  }
  if (threadIdx.x == 0) s.b4[0] = g[o.b4];
  return s;
}

// out[s][j] = relu(sum_k W[j][k] in[s][k] + b[j]); thread: sample t/4,
// neurons (t%4) + 4i
__device__ __forceinline__ void dense_relu(const float* W, int ldw, const float* b, const float* in,
                                           int ldi, int K, float* out) {
  const int s = threadIdx.x >> 2, j0 = threadIdx.x & 3;
  float acc[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) acc[i] = b[j0 + 4 * i];
  for (int k = 0; k < K; ++k) {
    const float x = in[s * ldi + k];
#pragma unroll
    for (int i = 0; i < 16; ++i) acc[i] = fmaf(W[(j0 + 4 * i) * ldw + k], x, acc[i]);
  }
#pragma unroll
  for (int i = 0; i < 16; ++i) out[s * LDH + j0 + 4 * i] = fmaxf(acc[i], 0.f);
}

// f[s] = w4 . h3[s] + b4 (4 threads per sample, fixed-order shuffle sum)
__device__ __forceinline__ float head(const SParams& P, const float* h3) {
  const int s = threadIdx.x >> 2, j0 = threadIdx.x & 3;
  float a = 0.f;
#pragma unroll
  for (int i = 0; i < 16; ++i) a = fmaf(P.w4[j0 + 4 * i], h3[s * LDH + j0 + 4 * i], a);
  a += __shfl_xor_sync(0xffffffffu, a, 1);
  a += __shfl_xor_sync(0xffffffffu, a, 2);
  return a + P.b4[0];
}

// rows [0, ns) of x (through idx) into sx[s][k], zero rows beyond
__device__ void load_x(const float* __restrict__ x, int in, const int32_t* __restrict__ idx,
                       int first, int ns, float* sx) {
  const int ldx = in + 1;
  for (int i = threadIdx.x; i < SB * in; i += kThreads) {
    const int s = i / in, k = i % in;
    float v = 0.f;
    if (s < ns) {
      const int64_t row = idx ? int64_t(idx[first + s]) : int64_t(first + s);
      v = x[row * in + k];
    }
    sx[s * ldx + k] = v;
  }
}

__global__ void __launch_bounds__(kThreads) k7_forward(const float* __restrict__ params, int in,
                                                       const float* __restrict__ x, int n,
                                                       float* __restrict__ out) {
  extern __shared__ __align__(16) float smem[];
  float* sm = smem;
  const SParams P = load_params(params, in, sm);
  float* sx = carve(sm, SB * (in + 1));
  float* h1 = carve(sm, SB * LDH);
  float* h2 = carve(sm, SB * LDH);
  for (int first = blockIdx.x * SB; first < n; first += gridDim.x * SB) {
    const int ns = min(SB, n - first);
    __syncthreads();
    load_x(x, in, nullptr, first, ns, sx);
    __syncthreads();
    dense_relu(P.w1, P.ld1, P.b1, sx, in + 1, in, h1);
    __syncthreads();
    dense_relu(P.w2, LDH, P.b2, h1, LDH, H, h2);
    __syncthreads();
    dense_relu(P.w3, LDH, P.b3, h2, LDH, H, h1);
    __syncthreads();
    const float f = head(P, h1);
    const int s = threadIdx.x >> 2;
    if ((threadIdx.x & 3) == 0 && s < ns) out[first + s] = f;
  }
}

// gW[j][k] += sum_s dz[s][j] in[s][k], gb[j] += sum_s dz[s][j]
// (thread: row j = t/4, columns (t%4) + 4i)
__device__ __forceinline__ void grad_weights(const float* dz, const float* in, int ldi, int K,
                                             float* gW, float* gb) {
  const int j = threadIdx.x >> 2, k0 = threadIdx.x & 3;
  float acc[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) acc[i] = 0.f;
  float ab = 0.f;
  for (int s = 0; s < SB; ++s) {
    const float d = dz[s * LDH + j];
    ab += d;
#pragma unroll
    for (int i = 0; i < 16; ++i)
      if (k0 + 4 * i < K) acc[i] = fmaf(d, in[s * ldi + k0 + 4 * i], acc[i]);
  }
#pragma unroll
  for (int i = 0; i < 16; ++i)
    if (k0 + 4 * i < K) gW[j * K + k0 + 4 * i] += acc[i];
  if (k0 == 0) gb[j] += ab;
}

// in place: h[s][k] <- (sum_j dz[s][j] W[j][k]) * (h[s][k] > 0)
__device__ __forceinline__ void back_relu(const float* dz, const float* W, float* h) {
  const int s = threadIdx.x >> 2, k0 = threadIdx.x & 3;
  float acc[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) acc[i] = 0.f;
  for (int j = 0; j < H; ++j) {
    const float d = dz[s * LDH + j];
#pragma unroll
    for (int i = 0; i < 16; ++i) acc[i] = fmaf(d, W[j * LDH + k0 + 4 * i], acc[i]);
  }
  __syncthreads();  // every thread has read dz before anyone overwrites h (dz may alias)
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    float* hp = &h[s * LDH + k0 + 4 * i];
    *hp = *hp > 0.f ? acc[i] : 0.f;
  }
}

__global__ void __launch_bounds__(kThreads)
    k7_backward(const float* __restrict__ params, int in, const float* __restrict__ x,
                const float* __restrict__ y, const int32_t* __restrict__ idx, int n, float scale,
                float* __restrict__ partial, float* __restrict__ loss_partial) {
  extern __shared__ __align__(16) float smem[];
  float* sm = smem;
  const SParams P = load_params(params, in, sm);
  const Offs o(in);
  float* sx = carve(sm, SB * (in + 1));
  float* h1 = carve(sm, SB * LDH);
  float* h2 = carve(sm, SB * LDH);
  float* h3 = carve(sm, SB * LDH);
  float* sg = carve(sm, (o.P + 3) & ~3);
  float* sl = carve(sm, kThreads / 32);
  for (int i = threadIdx.x; i < o.P; i += kThreads) sg[i] = 0.f;
  float loss = 0.f;
  for (int first = blockIdx.x * SB; first < n; first += gridDim.x * SB) {
    const int ns = min(SB, n - first);
    __syncthreads();
    load_x(x, in, idx, first, ns, sx);
    __syncthreads();
    dense_relu(P.w1, P.ld1, P.b1, sx, in + 1, in, h1);
    __syncthreads();
    dense_relu(P.w2, LDH, P.b2, h1, LDH, H, h2);
    __syncthreads();
    dense_relu(P.w3, LDH, P.b3, h2, LDH, H, h3);
    __syncthreads();
    const int s = threadIdx.x >> 2, k0 = threadIdx.x & 3;
    const float f = head(P, h3);
    float d = 0.f;
    if (s < ns) {
      const int64_t row = idx ? int64_t(idx[first + s]) : int64_t(first + s);
      const float r = f - y[row];
      d = scale * r;
      if (k0 == 0) loss += r * r;
    }
    // head gradients: gw4[k] = sum_s d_s h3[s][k], gb4 = sum_s d_s
    // dz3 = d_s w4[k] (h3 > 0), in place over h3 once h3 is consumed
    {
      // d of sample s lives in the 4 threads of s; stage it in h2's spare column
      if (k0 == 0) h2[s * LDH + H] = d;
    }
    __syncthreads();
    if (threadIdx.x < H) {
      float a = 0.f;
      for (int q = 0; q < SB; ++q) a = fmaf(h2[q * LDH + H], h3[q * LDH + threadIdx.x], a);
      sg[o.w4 + threadIdx.x] += a;
    } else if (threadIdx.x == H) {
      float a = 0.f;
      for (int q = 0; q < SB; ++q) a += h2[q * LDH + H];
      sg[o.b4] += a;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      float* hp = &h3[s * LDH + k0 + 4 * i];
      *hp = *hp > 0.f ? d * P.w4[k0 + 4 * i] : 0.f;
    }
    __syncthreads();
    grad_weights(h3, h2, LDH, H, sg + o.w3, sg + o.b3);
    __syncthreads();
    back_relu(h3, P.w3, h2);  // dz2 over h2
    __syncthreads();
    grad_weights(h2, h1, LDH, H, sg + o.w2, sg + o.b2);
    __syncthreads();
    back_relu(h2, P.w2, h1);  // dz1 over h1
    __syncthreads();
    grad_weights(h1, sx, in + 1, in, sg + o.w1, sg + o.b1);
  }
  // block loss: fixed-order warp sums, then warps in order
  for (int off = 16; off > 0; off >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, off);
  if ((threadIdx.x & 31) == 0) sl[threadIdx.x >> 5] = loss;
  __syncthreads();
  for (int i = threadIdx.x; i < o.P; i += kThreads) partial[size_t(blockIdx.x) * o.P + i] = sg[i];
  if (threadIdx.x == 0) {
    float a = 0.f;
    for (int w = 0; w < kThreads / 32; ++w) a += sl[w];
    loss_partial[blockIdx.x] = a;
  }
}

__global__ void k7_reduce(const float* __restrict__ partial, const float* __restrict__ loss_partial,
                          int nblk, int P, float* __restrict__ grad, float* __restrict__ loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < P) {
    float a = 0.f;
    for (int b = 0; b < nblk; ++b) a += partial[size_t(b) * P + i];
    grad[i] = a;
  }
  if (i == 0 && loss) {
    float a = 0.f;
    for (int b = 0; b < nblk; ++b) a += loss_partial[b];
    *loss = a;
  }
}

__global__ void k7_adam(float* __restrict__ params, const float* __restrict__ grad,
                        float* __restrict__ m, float* __restrict__ v, int P, float lr, float b1,
                        float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  const float g = grad[i];
  const float mi = b1 * m[i] + (1.f - b1) * g;
  const float vi = b2 * v[i] + (1.f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  params[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

size_t smem_forward(int in) {
  return sizeof(float) * size_t(H * (in + 1) + 3 * H + 2 * H * LDH + H + 4 + SB * (in + 1) +
                                 2 * SB * LDH);
}
size_t smem_backward(int in) {
  const Offs o(in);
  return smem_forward(in) + sizeof(float) * size_t(SB * LDH + ((o.P + 3) & ~3) + kThreads / 32);
}

}  // namespace

int launch_mlp_forward(const float* params, int in, const float* x, int n, float* out,
                       cudaStream_t s) {
  if (in < 1 || in > kMlpMaxIn) return set_error(HS_E_INVALID, "input width %d", in);
  if (n <= 0) return HS_OK;
  const size_t sm = smem_forward(in);
  HS_CUDA(cudaFuncSetAttribute(k7_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
  int dev = 0, sms = 148;
  HS_CUDA(cudaGetDevice(&dev));
  HS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int grid = std::min((n + SB - 1) / SB, sms);
  k7_forward<<<grid, kThreads, sm, s>>>(params, in, x, n, out);
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}

int launch_mlp_backward(const float* params, int in, const float* x, const float* y,
                        const int32_t* idx, int n, float scale, float* partial,
                        float* loss_partial, int nblk, cudaStream_t s) {
  if (in < 1 || in > kMlpMaxIn) return set_error(HS_E_INVALID, "input width %d", in);
  const size_t sm = smem_backward(in);
  HS_CUDA(cudaFuncSetAttribute(k7_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
  k7_backward<<<nblk, kThreads, sm, s>>>(params, in, x, y, idx, n, scale, partial, loss_partial);
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}

int launch_mlp_reduce(const float* partial, const float* loss_partial, int nblk, int P,
                      float* grad, float* loss, cudaStream_t s) {
  k7_reduce<<<(P + 255) / 256, 256, 0, s>>>(partial, loss_partial, nblk, P, grad, loss);
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}

int launch_mlp_adam(float* params, const float* grad, float* m, float* v, int P, float lr,
                    float beta1, float beta2, float eps, int step, cudaStream_t s) {
  const float c1 = 1.f - std::pow(beta1, float(step));
  const float c2 = 1.f - std::pow(beta2, float(step));
  k7_adam<<<(P + 255) / 256, 256, 0, s>>>(params, grad, m, v, P, lr, beta1, beta2, eps, c1, c2);
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}

}  // namespace hisv
