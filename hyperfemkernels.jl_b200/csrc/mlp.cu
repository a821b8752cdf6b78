// The learned correction's network as a standalone object (hfk_mlp_*): creation with a seeded
// Glorot initialisation, weights in and out, forward pass, gradient and Adam training, all on the
// GPU with the kernels of kern_mlp.cuh (BF16 weights, FP32 accumulation). Its use inside the
// p-multigrid cycle (features, the correction and its energy-optimal step) lives with the cycle.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <memory>
#include <vector>

#include "engine.h"
#include "hfk_internal.h"
#include "kern_mlp.cuh"

using namespace hfk;

namespace {
uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

void mlp_upload(hfk_mlp* m, const float* w_host) {
  m->w.upload(w_host, MLP_NPARAM, m->stream);
  m->wb.resize(MLP_NPARAM);
  mlp_to_bf16_kernel<<<vec_grid(MLP_NPARAM), 256, 0, m->stream>>>(MLP_NPARAM, m->w.p, m->wb.p);
  HFK_CUDA(cudaGetLastError());
}

void mlp_grad_dev(hfk_mlp* m, const float* feats, const float* targets, int64_t n, float* grad, float* loss) {
  static PerDeviceLimit attr;
  raise_smem_limit(mlp_grad_kernel, mlp_grad_smem_bytes(), attr);
  HFK_CUDA(cudaMemsetAsync(grad, 0, MLP_NPARAM * sizeof(float), m->stream));
  HFK_CUDA(cudaMemsetAsync(loss, 0, sizeof(float), m->stream));
  const int64_t chunks = (n + MLP_CHUNK - 1) / MLP_CHUNK;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(chunks, (int64_t)sm_count() * 2));
  mlp_grad_kernel<<<grid, 128, mlp_grad_smem_bytes(), m->stream>>>(n, m->wb.p, feats, targets,
                                                                   1.0f / (float)std::max<int64_t>(n, 1), grad, loss);
  HFK_CUDA(cudaGetLastError());
}
}  // namespace

extern "C" {

int hfk_mlp_create(hfk_mlp** out, uint64_t seed) {
  HFK_API_BEGIN
  HFK_REQUIRE(out, HFK_ERR_ARG, "null output handle");
  auto m = std::make_unique<hfk_mlp>();
  HFK_CUDA(cudaStreamCreate(&m->stream));
  // uniform Glorot initialisation from a seeded generator; biases zero
  std::vector<float> w(MLP_NPARAM, 0.f);
  uint64_t s = seed;
  auto fill = [&](int off, int fan_out, int fan_in) {
    const double lim = std::sqrt(6.0 / (fan_in + fan_out));
    for (int i = 0; i < fan_out * fan_in; ++i) {
      const double u = (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0);
      w[off + i] = (float)((2 * u - 1) * lim);
    }
  };
  fill(MLP_OW1, MLP_W, MLP_IN);
  fill(MLP_OW2, MLP_W, MLP_W);
  fill(MLP_OW3, MLP_OUT, MLP_W);
  for (int i = 0; i < MLP_NW3; ++i) w[MLP_OW3 + i] *= 0.1f;  // start close to the plain cycle
  mlp_upload(m.get(), w.data());
  m->m1.resize(MLP_NPARAM);
  m->m2.resize(MLP_NPARAM);
  m->grad.resize(MLP_NPARAM);
  m->loss.resize(1);
  m->m1.zero(m->stream);
  m->m2.zero(m->stream);
  HFK_CUDA(cudaStreamSynchronize(m->stream));
  *out = m.release();
  HFK_API_END
}

int hfk_mlp_destroy(hfk_mlp* m) {
  HFK_API_BEGIN
  if (m) {
    cudaStreamSynchronize(m->stream);
    cudaStreamDestroy(m->stream);
    delete m;
  }
  HFK_API_END
}

int hfk_mlp_num_params(void) { return MLP_NPARAM; }

int hfk_mlp_get_weights(hfk_mlp* m, float* w) {
  HFK_API_BEGIN
  HFK_REQUIRE(m && w, HFK_ERR_ARG, "null argument");
  HFK_CUDA(cudaMemcpyAsync(w, m->w.p, MLP_NPARAM * sizeof(float), cudaMemcpyDefault, m->stream));
  HFK_CUDA(cudaStreamSynchronize(m->stream));
  HFK_API_END
}

int hfk_mlp_set_weights(hfk_mlp* m, const float* w) {
  HFK_API_BEGIN
  HFK_REQUIRE(m && w, HFK_ERR_ARG, "null argument");
  std::vector<float> h(MLP_NPARAM);
  HFK_CUDA(cudaMemcpy(h.data(), w, MLP_NPARAM * sizeof(float), cudaMemcpyDefault));
  mlp_upload(m, h.data());
  m->m1.zero(m->stream);
  m->m2.zero(m->stream);
  m->steps = 0;
  HFK_CUDA(cudaStreamSynchronize(m->stream));
  HFK_API_END
}

int hfk_mlp_forward(hfk_mlp* m, const float* feats, int64_t n, float* out) {
  HFK_API_BEGIN
  HFK_REQUIRE(m && feats && out && n >= 0, HFK_ERR_ARG, "invalid argument");
  HFK_REQUIRE(is_device_ptr(feats) && is_device_ptr(out), HFK_ERR_ARG, "features and outputs must be device pointers");
  HFK_CUDA(cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(MLP_NPARAM * sizeof(float))));
  if (n) mlp_forward_kernel<<<vec_grid(n, 128), 128, MLP_NPARAM * sizeof(float), m->stream>>>(n, m->wb.p, feats, out);
  HFK_CUDA(cudaGetLastError());
  HFK_CUDA(cudaStreamSynchronize(m->stream));
  HFK_API_END
}

int hfk_mlp_grad(hfk_mlp* m, const float* feats, const float* targets, int64_t n, float* grad, float* loss) {
  HFK_API_BEGIN
  HFK_REQUIRE(m && feats && targets && grad && loss && n > 0, HFK_ERR_ARG, "invalid argument");
  HFK_REQUIRE(is_device_ptr(feats) && is_device_ptr(targets), HFK_ERR_ARG, "samples must be device pointers");
  mlp_grad_dev(m, feats, targets, n, m->grad.p, m->loss.p);
  HFK_CUDA(cudaMemcpyAsync(grad, m->grad.p, MLP_NPARAM * sizeof(float), cudaMemcpyDefault, m->stream));
  HFK_CUDA(cudaMemcpyAsync(loss, m->loss.p, sizeof(float), cudaMemcpyDefault, m->stream));
  HFK_CUDA(cudaStreamSynchronize(m->stream));
  HFK_API_END
}

int hfk_mlp_train(hfk_mlp* m, const float* feats, const float* targets, int64_t n, int steps, int64_t batch, float lr,
                  float* last_loss) {
  HFK_API_BEGIN
  HFK_REQUIRE(m && feats && targets && n > 0 && steps >= 0 && batch > 0 && lr > 0, HFK_ERR_ARG, "invalid argument");
  HFK_REQUIRE(is_device_ptr(feats) && is_device_ptr(targets), HFK_ERR_ARG, "samples must be device pointers");
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  int64_t start = 0;
  for (int it = 0; it < steps; ++it) {
    const int64_t nb = std::min(batch, n - start);
    mlp_grad_dev(m, feats + start * MLP_IN, targets + start * MLP_OUT, nb, m->grad.p, m->loss.p);
    m->steps++;
    const float c1 = 1.f - std::pow(b1, (float)m->steps), c2 = 1.f - std::pow(b2, (float)m->steps);
    mlp_adam_kernel<<<vec_grid(MLP_NPARAM), 256, 0, m->stream>>>(MLP_NPARAM, m->w.p, m->wb.p, m->grad.p, m->m1.p,
                                                                  m->m2.p, lr, b1, b2, eps, c1, c2);
    HFK_CUDA(cudaGetLastError());
    start += nb;
    if (start >= n) start = 0;
  }
  if (last_loss) HFK_CUDA(cudaMemcpyAsync(last_loss, m->loss.p, sizeof(float), cudaMemcpyDefault, m->stream));
  HFK_CUDA(cudaStreamSynchronize(m->stream));
  HFK_API_END
}


}  // extern "C"
