// Host side of the learned cost model (hs_mlp_*): parameter storage on the
// device, seeded initialisation, inference, one-shot gradients, and the
// minibatch Adam training loop driving the K7 kernels.
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.h"

using namespace hisv;

struct hs_mlp {
  int in = 0, P = 0, sms = 148;
  float* d_params = nullptr;
  float* d_m = nullptr;
  float* d_v = nullptr;
  float* d_grad = nullptr;
  float* d_partial = nullptr;  // sms x P
  float* d_lpart = nullptr;    // sms
  int step = 0;                // Adam steps taken
};

namespace {

// splitmix64: a small seeded generator, identical on every platform
struct Rng {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
  }
  double uniform() { return double(next() >> 11) * (1.0 / 9007199254740992.0); }
};

template <class T>
struct DevBuf {  // scratch device buffer freed on scope exit
  T* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

int blocks_for(const hs_mlp* m, int n) {
  const int b = (n + kMlpSamples - 1) / kMlpSamples;
  return b < 1 ? 1 : (b > m->sms ? m->sms : b);
}

}  // namespace

extern "C" {

int hs_mlp_create(int in_dim, uint64_t seed, hs_mlp** out) {
  if (!out) return set_error(HS_E_INVALID, "null output");
  *out = nullptr;
  if (in_dim < 1 || in_dim > kMlpMaxIn)
    return set_error(HS_E_INVALID, "input width %d outside 1..%d", in_dim, kMlpMaxIn);
  int dev = 0, ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_error(HS_E_NODEVICE, "no CUDA device");
  }
  auto* m = new hs_mlp;
  m->in = in_dim;
  m->P = mlp_num_params(in_dim);
  auto fail = [&](int rc) {
    hs_mlp_destroy(m);
    return rc;
  };
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&m->sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return fail(set_error(HS_E_CUDA, "device query"));
  const size_t pb = sizeof(float) * size_t(m->P);
  if (cudaMalloc(&m->d_params, pb) != cudaSuccess || cudaMalloc(&m->d_m, pb) != cudaSuccess ||
      cudaMalloc(&m->d_v, pb) != cudaSuccess || cudaMalloc(&m->d_grad, pb) != cudaSuccess ||
      cudaMalloc(&m->d_partial, pb * size_t(m->sms)) != cudaSuccess ||
      cudaMalloc(&m->d_lpart, sizeof(float) * size_t(m->sms)) != cudaSuccess) {
    cudaGetLastError();
    return fail(set_error(HS_E_NOMEM, "model buffers"));
  }
  // He-uniform weights (bound sqrt(6 / fan_in)), zero biases
  std::vector<float> p(m->P, 0.f);
  Rng r{seed};
  const int H = kMlpHidden;
  auto fill = [&](int off, int count, int fan_in) {
    const double a = std::sqrt(6.0 / fan_in);
    for (int i = 0; i < count; ++i) p[off + i] = float((2.0 * r.uniform() - 1.0) * a);
  };
  int off = 0;
  fill(off, H * in_dim, in_dim);
  off += H * in_dim + H;
  fill(off, H * H, H);
  off += H * H + H;
  fill(off, H * H, H);
  off += H * H + H;
  fill(off, H, H);
  int rc = hs_mlp_set_params(m, p.data());
  if (rc != HS_OK) return fail(rc);
  *out = m;
  return HS_OK;
}

int hs_mlp_num_params(const hs_mlp* m) { return m ? m->P : set_error(HS_E_INVALID, "null model"); }

int hs_mlp_get_params(hs_mlp* m, float* host) {
  if (!m || !host) return set_error(HS_E_INVALID, "null argument");
  HS_CUDA(cudaMemcpy(host, m->d_params, sizeof(float) * size_t(m->P), cudaMemcpyDeviceToHost));
  return HS_OK;
}

int hs_mlp_set_params(hs_mlp* m, const float* host) {
  if (!m || !host) return set_error(HS_E_INVALID, "null argument");
  const size_t pb = sizeof(float) * size_t(m->P);
  HS_CUDA(cudaMemcpy(m->d_params, host, pb, cudaMemcpyHostToDevice));
  HS_CUDA(cudaMemset(m->d_m, 0, pb));
  HS_CUDA(cudaMemset(m->d_v, 0, pb));
  m->step = 0;
  return HS_OK;
}

int hs_mlp_predict(hs_mlp* m, const float* x, int n, float* y_out) {
  if (!m || (n > 0 && (!x || !y_out)) || n < 0) return set_error(HS_E_INVALID, "bad arguments");
  if (n == 0) return HS_OK;
  DevBuf<float> dx, dy;
  HS_CUDA(cudaMalloc(&dx.p, sizeof(float) * size_t(n) * m->in));
  HS_CUDA(cudaMalloc(&dy.p, sizeof(float) * size_t(n)));
  HS_CUDA(cudaMemcpy(dx.p, x, sizeof(float) * size_t(n) * m->in, cudaMemcpyHostToDevice));
  HS_TRY(launch_mlp_forward(m->d_params, m->in, dx.p, n, dy.p, nullptr));
  HS_CUDA(cudaMemcpy(y_out, dy.p, sizeof(float) * size_t(n), cudaMemcpyDeviceToHost));
  return HS_OK;
}

int hs_mlp_gradients(hs_mlp* m, const float* x, const float* y, int n, float* grad_out,
                     float* loss_out) {
  if (!m || !x || !y || n < 1) return set_error(HS_E_INVALID, "bad arguments");
  DevBuf<float> dx, dy, dl;
  HS_CUDA(cudaMalloc(&dx.p, sizeof(float) * size_t(n) * m->in));
  HS_CUDA(cudaMalloc(&dy.p, sizeof(float) * size_t(n)));
  HS_CUDA(cudaMalloc(&dl.p, sizeof(float)));
  HS_CUDA(cudaMemcpy(dx.p, x, sizeof(float) * size_t(n) * m->in, cudaMemcpyHostToDevice));
  HS_CUDA(cudaMemcpy(dy.p, y, sizeof(float) * size_t(n), cudaMemcpyHostToDevice));
  const int nblk = blocks_for(m, n);
  HS_TRY(launch_mlp_backward(m->d_params, m->in, dx.p, dy.p, nullptr, n, 2.f / float(n),
                             m->d_partial, m->d_lpart, nblk, nullptr));
  HS_TRY(launch_mlp_reduce(m->d_partial, m->d_lpart, nblk, m->P, m->d_grad, dl.p, nullptr));
  if (grad_out)
    HS_CUDA(cudaMemcpy(grad_out, m->d_grad, sizeof(float) * size_t(m->P), cudaMemcpyDeviceToHost));
  if (loss_out) {
    float l = 0.f;
    HS_CUDA(cudaMemcpy(&l, dl.p, sizeof(float), cudaMemcpyDeviceToHost));
    *loss_out = l / float(n);
  }
  return HS_OK;
}

int hs_mlp_train(hs_mlp* m, const float* x, const float* y, int n, int epochs, int batch,
                 float lr, uint64_t seed, float* epoch_loss) {
  if (!m || !x || !y || n < 1 || epochs < 0 || batch < 1 || !(lr > 0.f))
    return set_error(HS_E_INVALID, "bad arguments");
  DevBuf<float> dx, dy, dl;
  DevBuf<int32_t> didx;
  const int steps_per_epoch = (n + batch - 1) / batch;
  HS_CUDA(cudaMalloc(&dx.p, sizeof(float) * size_t(n) * m->in));
  HS_CUDA(cudaMalloc(&dy.p, sizeof(float) * size_t(n)));
  HS_CUDA(cudaMalloc(&didx.p, sizeof(int32_t) * size_t(n)));
  HS_CUDA(cudaMalloc(&dl.p, sizeof(float) * size_t(steps_per_epoch)));
  HS_CUDA(cudaMemcpy(dx.p, x, sizeof(float) * size_t(n) * m->in, cudaMemcpyHostToDevice));
  HS_CUDA(cudaMemcpy(dy.p, y, sizeof(float) * size_t(n), cudaMemcpyHostToDevice));
  std::vector<int32_t> perm(n);
  std::vector<float> losses(steps_per_epoch);
  Rng r{seed};
  for (int e = 0; e < epochs; ++e) {
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int i = n - 1; i > 0; --i) std::swap(perm[i], perm[int(r.next() % uint64_t(i + 1))]);
    HS_CUDA(cudaMemcpy(didx.p, perm.data(), sizeof(int32_t) * size_t(n), cudaMemcpyHostToDevice));
    for (int st = 0; st < steps_per_epoch; ++st) {
      const int b0 = st * batch, nb = std::min(batch, n - b0);
      const int nblk = blocks_for(m, nb);
      HS_TRY(launch_mlp_backward(m->d_params, m->in, dx.p, dy.p, didx.p + b0, nb, 2.f / float(nb),
                                 m->d_partial, m->d_lpart, nblk, nullptr));
      HS_TRY(launch_mlp_reduce(m->d_partial, m->d_lpart, nblk, m->P, m->d_grad, dl.p + st,
                               nullptr));
      HS_TRY(launch_mlp_adam(m->d_params, m->d_grad, m->d_m, m->d_v, m->P, lr, 0.9f, 0.999f,
                             1e-8f, ++m->step, nullptr));
    }
    if (epoch_loss) {
      HS_CUDA(cudaMemcpy(losses.data(), dl.p, sizeof(float) * size_t(steps_per_epoch),
                         cudaMemcpyDeviceToHost));
      double s = 0;
      for (float l : losses) s += l;
      epoch_loss[e] = float(s / n);  // mean squared error over the epoch
    }
  }
  HS_CUDA(cudaDeviceSynchronize());
  return HS_OK;
}

int hs_mlp_destroy(hs_mlp* m) {
  if (!m) return HS_OK;
  for (float* p : {m->d_params, m->d_m, m->d_v, m->d_grad, m->d_partial, m->d_lpart})
    if (p) cudaFree(p);
  delete m;
  return HS_OK;
}

}  // extern "C"
