// Per-node MLP for the learned correction inside the p-multigrid V-cycle (no counterpart in the
// reference). 3 layers: NIN -> 64 -> 64 -> 3, tanh activations, BF16 weights (the copy the forward
// pass reads), FP32 master weights, FP32 accumulation. One sample = one mesh node (its 3 dofs).
//
// Features of node n (NIN = 16, zero-padded): the residual entering the correction s_n (3), its
// block-Jacobi preconditioned value (B_n^-1 s)_n (3), the residual entering the V-cycle r_n (3), the
// V-cycle output y_n (3), log lambda, log mu; each vector group scaled by its RMS over the nodes
// (scales passed in, so the network sees O(1) inputs). Target: the remaining error e_n = (A^-1 s)_n
// in the scale of the cycle's output y (what the cycle left undone, relative to what it did: for the
// smooth modes that the coarse solve reduces only in part, e is close to a local multiple of y).
#pragma once
#include <cuda_bf16.h>

#include "hfk_internal.h"

namespace hfk {

constexpr int MLP_IN = 16, MLP_W = 64, MLP_OUT = 3;
constexpr int MLP_NW1 = MLP_W * MLP_IN, MLP_NB1 = MLP_W, MLP_NW2 = MLP_W * MLP_W, MLP_NB2 = MLP_W;
constexpr int MLP_NW3 = MLP_OUT * MLP_W, MLP_NB3 = MLP_OUT;
// parameter offsets in one flat vector: W1 (row-major [out][in]), b1, W2, b2, W3, b3
constexpr int MLP_OW1 = 0, MLP_OB1 = MLP_OW1 + MLP_NW1, MLP_OW2 = MLP_OB1 + MLP_NB1, MLP_OB2 = MLP_OW2 + MLP_NW2;
constexpr int MLP_OW3 = MLP_OB2 + MLP_NB2, MLP_OB3 = MLP_OW3 + MLP_NW3, MLP_NPARAM = MLP_OB3 + MLP_NB3;

// BF16 weights to FP32 in shared memory (every block)
__device__ __forceinline__ void mlp_load_weights(const __nv_bfloat16* wb, float* ws) {
  for (int i = threadIdx.x; i < MLP_NPARAM; i += blockDim.x) ws[i] = __bfloat162float(wb[i]);
  __syncthreads();
}

// forward of one sample; a1/a2 receive the activations when non-null (training)
__device__ __forceinline__ void mlp_forward_one(const float* ws, const float* x, float* out, float* a1, float* a2) {
  float h1[MLP_W];
#pragma unroll 4
  for (int j = 0; j < MLP_W; ++j) {
    float s = ws[MLP_OB1 + j];
#pragma unroll
    for (int i = 0; i < MLP_IN; ++i) s += ws[MLP_OW1 + j * MLP_IN + i] * x[i];
    h1[j] = tanhf(s);
    if (a1) a1[j] = h1[j];
  }
  float o0 = ws[MLP_OB3], o1 = ws[MLP_OB3 + 1], o2 = ws[MLP_OB3 + 2];
#pragma unroll 2
  for (int j = 0; j < MLP_W; ++j) {
    float s = ws[MLP_OB2 + j];
#pragma unroll 16
    for (int i = 0; i < MLP_W; ++i) s += ws[MLP_OW2 + j * MLP_W + i] * h1[i];
    const float h = tanhf(s);
    if (a2) a2[j] = h;
    o0 += ws[MLP_OW3 + j] * h;
    o1 += ws[MLP_OW3 + MLP_W + j] * h;
    o2 += ws[MLP_OW3 + 2 * MLP_W + j] * h;
  }
  out[0] = o0;
  out[1] = o1;
  out[2] = o2;
}

// inference: out (n x 3) = MLP(feats (n x 16))
static __global__ void __launch_bounds__(128) mlp_forward_kernel(int64_t n, const __nv_bfloat16* wb, const float* feats,
                                                          float* out) {
  extern __shared__ float mlp_ws[];
  float* ws = mlp_ws;
  mlp_load_weights(wb, ws);
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
    float x[MLP_IN];
#pragma unroll
    for (int i = 0; i < MLP_IN; ++i) x[i] = feats[s * MLP_IN + i];
    mlp_forward_one(ws, x, out + s * MLP_OUT, nullptr, nullptr);
  }
}

// Training: forward + backward of a chunk of samples per block, squared-error loss
// L = sum_s |out_s - t_s|^2 / count. Per block, the activations of its chunk are kept in
// shared memory and the weight gradients summed over the chunk there (no atomics per sample);
// one atomicAdd per parameter and block into the FP32 gradient vector.
constexpr int MLP_CHUNK = 64;

static __global__ void __launch_bounds__(128) mlp_grad_kernel(int64_t n, const __nv_bfloat16* wb, const float* feats,
                                                       const float* targets, float inv_count, float* grad,
                                                       float* loss) {
  extern __shared__ float mlp_sm[];
  float* ws = mlp_sm;                            // NPARAM
  float* X = ws + MLP_NPARAM;                    // CHUNK x IN
  float* A1 = X + MLP_CHUNK * MLP_IN;            // CHUNK x W
  float* A2 = A1 + MLP_CHUNK * MLP_W;            // CHUNK x W
  float* D2 = A2 + MLP_CHUNK * MLP_W;            // CHUNK x W   (dL/dz2)
  float* D1 = D2 + MLP_CHUNK * MLP_W;            // CHUNK x W   (dL/dz1)
  float* D3 = D1 + MLP_CHUNK * MLP_W;            // CHUNK x OUT (dL/dout)
  float* G = D3 + MLP_CHUNK * MLP_OUT;           // NPARAM gradient of the block
  mlp_load_weights(wb, ws);
  for (int i = threadIdx.x; i < MLP_NPARAM; i += blockDim.x) G[i] = 0.f;
  float lsum = 0.f;
  for (int64_t c0 = (int64_t)blockIdx.x * MLP_CHUNK; c0 < n; c0 += (int64_t)gridDim.x * MLP_CHUNK) {
    const int cn = (int)(n - c0 < MLP_CHUNK ? n - c0 : MLP_CHUNK);
    __syncthreads();
    // forward + output error (one thread per sample)
    for (int s = threadIdx.x; s < MLP_CHUNK; s += blockDim.x) {
      float x[MLP_IN], o[MLP_OUT];
      if (s < cn) {
#pragma unroll
        for (int i = 0; i < MLP_IN; ++i) x[i] = feats[(c0 + s) * MLP_IN + i];
        mlp_forward_one(ws, x, o, A1 + s * MLP_W, A2 + s * MLP_W);
        for (int k = 0; k < MLP_OUT; ++k) {
          const float e = o[k] - targets[(c0 + s) * MLP_OUT + k];
          lsum += e * e;
          D3[s * MLP_OUT + k] = 2.f * e * inv_count;
        }
      } else {
#pragma unroll
        for (int i = 0; i < MLP_IN; ++i) x[i] = 0.f;
        for (int j = 0; j < MLP_W; ++j) A1[s * MLP_W + j] = A2[s * MLP_W + j] = 0.f;
        for (int k = 0; k < MLP_OUT; ++k) D3[s * MLP_OUT + k] = 0.f;
      }
      for (int i = 0; i < MLP_IN; ++i) X[s * MLP_IN + i] = x[i];
    }
    __syncthreads();
    // dz2 = (W3^T d3) * (1 - a2^2)
    for (int e = threadIdx.x; e < MLP_CHUNK * MLP_W; e += blockDim.x) {
      const int s = e / MLP_W, j = e % MLP_W;
      float g = 0.f;
      for (int k = 0; k < MLP_OUT; ++k) g += ws[MLP_OW3 + k * MLP_W + j] * D3[s * MLP_OUT + k];
      const float a = A2[s * MLP_W + j];
      D2[e] = g * (1.f - a * a);
    }
    __syncthreads();
    // dz1 = (W2^T dz2) * (1 - a1^2)
    for (int e = threadIdx.x; e < MLP_CHUNK * MLP_W; e += blockDim.x) {
      const int s = e / MLP_W, i = e % MLP_W;
      float g = 0.f;
      for (int j = 0; j < MLP_W; ++j) g += ws[MLP_OW2 + j * MLP_W + i] * D2[s * MLP_W + j];
      const float a = A1[s * MLP_W + i];
      D1[e] = g * (1.f - a * a);
    }
    __syncthreads();
    // parameter gradients summed over the chunk (each thread owns parameters)
    for (int p = threadIdx.x; p < MLP_NPARAM; p += blockDim.x) {
      float g = 0.f;
      if (p < MLP_OB1) {
        const int j = p / MLP_IN, i = p % MLP_IN;
        for (int s = 0; s < MLP_CHUNK; ++s) g += D1[s * MLP_W + j] * X[s * MLP_IN + i];
      } else if (p < MLP_OW2) {
        const int j = p - MLP_OB1;
        for (int s = 0; s < MLP_CHUNK; ++s) g += D1[s * MLP_W + j];
      } else if (p < MLP_OB2) {
        const int j = (p - MLP_OW2) / MLP_W, i = (p - MLP_OW2) % MLP_W;
        for (int s = 0; s < MLP_CHUNK; ++s) g += D2[s * MLP_W + j] * A1[s * MLP_W + i];
      } else if (p < MLP_OW3) {
        const int j = p - MLP_OB2;
        for (int s = 0; s < MLP_CHUNK; ++s) g += D2[s * MLP_W + j];
      } else if (p < MLP_OB3) {
        const int k = (p - MLP_OW3) / MLP_W, j = (p - MLP_OW3) % MLP_W;
        for (int s = 0; s < MLP_CHUNK; ++s) g += D3[s * MLP_OUT + k] * A2[s * MLP_W + j];
      } else {
        const int k = p - MLP_OB3;
        for (int s = 0; s < MLP_CHUNK; ++s) g += D3[s * MLP_OUT + k];
      }
      G[p] += g;
    }
  }
  __syncthreads();
  for (int p = threadIdx.x; p < MLP_NPARAM; p += blockDim.x) atomicAdd(&grad[p], G[p]);
  // loss: block reduction then one atomic
  __shared__ float red[32];
  float v = lsum;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    atomicAdd(loss, t * inv_count);
  }
}

constexpr size_t mlp_grad_smem_bytes() {
  return sizeof(float) * ((size_t)2 * MLP_NPARAM + MLP_CHUNK * MLP_IN + 4 * MLP_CHUNK * MLP_W + MLP_CHUNK * MLP_OUT);
}

// Adam on the FP32 master weights, then the BF16 copy the forward pass reads
static __global__ void mlp_adam_kernel(int np, float* w, __nv_bfloat16* wb, const float* g, float* m1, float* m2, float lr,
                                float b1, float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    m1[i] = b1 * m1[i] + (1.f - b1) * gi;
    m2[i] = b2 * m2[i] + (1.f - b2) * gi * gi;
    const float mh = m1[i] / c1, vh = m2[i] / c2;
    w[i] -= lr * mh / (sqrtf(vh) + eps);
    wb[i] = __float2bfloat16(w[i]);
  }
}

static __global__ void mlp_to_bf16_kernel(int np, const float* w, __nv_bfloat16* wb) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) wb[i] = __float2bfloat16(w[i]);
}

// ---- features and the correction on the free dofs, per nodal block ----------------------------
// feats[b] = [s/ss, (Binv s)/sm, r/sr, y/sy, log lam, log mu, 0, 0]; the dofs of block b = bdofs[3b..]
// Per-segment scales: scales[seg * sstride + j], j = 0..3 the root mean squares of s, Binv s, r, y;
// loglm[2 seg], loglm[2 seg + 1] = log lambda, log mu of the segment (one segment: segb null).
static __global__ void mlp_features_kernel(int nb, const int32_t* dofs, const int32_t* segb, const double* Binv,
                                    const double* s, const double* r, const double* y, const double* scales,
                                    int sstride, const float* loglm, float* feats) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    const int sg = segb ? segb[b] : 0;
    const double* sc = scales + (size_t)sg * sstride;
    const float is = sc[0] > 0 ? 1.f / (float)sc[0] : 0.f;
    const float im = sc[1] > 0 ? 1.f / (float)sc[1] : 0.f;
    const float ir = sc[2] > 0 ? 1.f / (float)sc[2] : 0.f;
    const float iy = sc[3] > 0 ? 1.f / (float)sc[3] : 0.f;
    const int d0 = dofs[3 * b], d1 = dofs[3 * b + 1], d2 = dofs[3 * b + 2];
    const double sv[3] = {d0 ? s[d0 - 1] : 0.0, d1 ? s[d1 - 1] : 0.0, d2 ? s[d2 - 1] : 0.0};
    const double* M = Binv + 9 * (size_t)b;
    float* f = feats + (size_t)b * MLP_IN;
    const int dd[3] = {d0, d1, d2};
    for (int i = 0; i < 3; ++i) {
      const double ms = M[i] * sv[0] + M[i + 3] * sv[1] + M[i + 6] * sv[2];
      f[i] = (float)sv[i] * is;
      f[3 + i] = dd[i] ? (float)ms * im : 0.f;
      f[6 + i] = dd[i] ? (float)r[dd[i] - 1] * ir : 0.f;
      f[9 + i] = dd[i] ? (float)y[dd[i] - 1] * iy : 0.f;
    }
    f[12] = loglm[2 * sg];
    f[13] = loglm[2 * sg + 1];
    f[14] = 0.f;
    f[15] = 0.f;
  }
}
static __global__ void mlp_scatter_kernel(int nb, const int32_t* dofs, const int32_t* segb, const float* out,
                                   const double* scales, int sstride, double* delta) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    const double sc = scales[(size_t)(segb ? segb[b] : 0) * sstride + 3];
    for (int i = 0; i < 3; ++i) {
      const int d = dofs[3 * b + i];
      if (d) delta[d - 1] = (double)out[(size_t)b * MLP_OUT + i] * sc;
    }
  }
}
static __global__ void mlp_targets_kernel(int nb, const int32_t* dofs, const int32_t* segb, const double* e,
                                   const double* scales, int sstride, float* t) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    const double s1 = scales[(size_t)(segb ? segb[b] : 0) * sstride + 3];
    const double sc = s1 > 0 ? 1.0 / s1 : 0.0;
    for (int i = 0; i < 3; ++i) {
      const int d = dofs[3 * b + i];
      t[(size_t)b * MLP_OUT + i] = d ? (float)(e[d - 1] * sc) : 0.f;
    }
  }
}
// y += omega delta per segment, omega = (delta . s) / (delta . A delta) when both are positive, else 0:
// the step along delta that minimises the energy (A-norm) error of y, the norm the outer CG
// minimises (a residual-norm test would reject any prediction with small high-frequency noise).
// c = nrm + seg * stride: c[0] = delta . s, c[1] = delta . A delta.
__device__ __forceinline__ double mlp_step(const double* c) { return (c[0] > 0 && c[1] > 0) ? c[0] / c[1] : 0.0; }
static __global__ void mlp_accept_kernel(int64_t n, const int32_t* seg, const double* nrm, int stride, const double* delta,
                                  double* y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double w = mlp_step(nrm + (size_t)(seg ? seg[i] : 0) * stride);
    if (w > 0) y[i] += w * delta[i];
  }
}
// one CTA: *accepted += the number of segments with a positive step
static __global__ void mlp_accept_count_kernel(int nseg, const double* nrm, int stride, int* accepted) {
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  int mine = 0;
  for (int s = threadIdx.x; s < nseg; s += blockDim.x) mine += mlp_step(nrm + (size_t)s * stride) > 0;
  atomicAdd(&cnt, mine);
  __syncthreads();
  if (threadIdx.x == 0) *accepted += cnt;
}

}  // namespace hfk
