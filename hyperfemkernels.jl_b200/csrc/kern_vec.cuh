// Vector-level kernels: reductions, nodal blocks (extraction, inversion, application), the fused
// Chebyshev steps, transfers between levels, dense coarse solve. All memory-bound: grid-stride
// loops sized to the SM count, coalesced along the free-dof vectors.
#pragma once
#include "hfk_internal.h"
#include "pointwise.cuh"

namespace hfk {

// ---- deterministic two-stage reductions ------------------------------------------------------
constexpr int RED_BLOCKS = 592;  // 4 x 148 SMs
constexpr int RED_THREADS = 256;

template <typename R>
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void block_sum_store(double v, double* out) {
  __shared__ double ws[32];
  v = warp_sum<double>(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) ws[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < (blockDim.x >> 5) ? ws[lane] : 0.0;
    v = warp_sum<double>(v);
    if (lane == 0) *out = v;
  }
  __syncthreads();
}

// partial[k * gridDim.x + block] for up to 3 dot products x_k . y_k
template <typename R>
__global__ void dots_kernel(int64_t n, int k, const R* a0, const R* b0, const R* a1, const R* b1, const R* a2,
                            const R* b2, double* partial) {
  double s0 = 0, s1 = 0, s2 = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    s0 += (double)a0[i] * (double)b0[i];
    if (k > 1) s1 += (double)a1[i] * (double)b1[i];
    if (k > 2) s2 += (double)a2[i] * (double)b2[i];
  }
  block_sum_store(s0, partial + blockIdx.x);
  if (k > 1) block_sum_store(s1, partial + gridDim.x + blockIdx.x);
  if (k > 2) block_sum_store(s2, partial + 2 * gridDim.x + blockIdx.x);
}

static __global__ void finish_sums_kernel(int nparts, int k, const double* partial, double* out) {
  for (int j = 0; j < k; ++j) {
    double s = 0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) s += partial[j * nparts + i];
    block_sum_store(s, out + j);
  }
}

// ---- elementwise ----------------------------------------------------------------------------
template <typename R>
__global__ void fill_kernel(int64_t n, R v, R* x) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) x[i] = v;
}
template <typename A, typename B>
__global__ void convert_kernel(int64_t n, const A* x, B* y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) y[i] = (B)x[i];
}
// y = a x + b y
template <typename R>
__global__ void axpby_kernel(int64_t n, R a, const R* x, R b, R* y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) y[i] = a * x[i] + b * y[i];
}
// z = a x + b y
// x *= a
static __global__ void scale_kernel(int64_t n, double a, double* x) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) x[i] *= a;
}
template <typename R>
__global__ void axpbyz_kernel(int64_t n, R a, const R* x, R b, const R* y, R* z) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) z[i] = a * x[i] + b * y[i];
}
// CG update: x += alpha p; rold = r; r -= alpha q
static __global__ void cg_update_kernel(int64_t n, double alpha, const double* p, const double* q, double* x, double* r,
                                 double* rold) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double ri = r[i];
    if (rold) rold[i] = ri;
    x[i] += alpha * p[i];
    r[i] = ri - alpha * q[i];
  }
}

// ---- nodal blocks ---------------------------------------------------------------------------
// B_blk[ci,cj] += sum_q sum_{K,K'} dN^[n,K,q] Dh_q[(ci,K),(cj,K')] dN^[n,K',q] over the nodes of the
// cells of one colour (blocks_from_tangents!, src/preconditioners.jl:250-280, with the tangent
// pulled back once per point as in the assembly kernel).
struct BlockIO {
  const double* u;
  const double* dvals;
  const double* dNt;       // (nn, 3, np) tensor order
  const int32_t* block_of; // (nn, ncells)
  double* B;               // (9, nblocks)
  int np, nn;
  int atomic;              // 1: atomicAdd into B (all cells in one launch)
};

static __global__ void __launch_bounds__(256) blocks_kernel(CellData cd, BlockIO io) {
  extern __shared__ __align__(16) double sm[];
  const int np = io.np, nn = io.nn, ndl = 3 * nn;
  double* xl = sm;               // ndl
  double* Hs = xl + ndl;         // 9 np
  double* iJs = Hs + 9 * np;     // 9 np
  double* dVs = iJs + 9 * np;    // np
  double* Dh = dVs + np;         // 81 np
  const int li = blockIdx.x;
  if (li >= cd.ncells_list) return;
  const int cell = cd.cells ? cd.cells[li] : li;
  const int32_t* gid = cd.ids + (size_t)cell * ndl;
  for (int j = threadIdx.x; j < ndl; j += blockDim.x) {
    const int32_t id = gid[j];
    xl[j] = id > 0 ? io.u[id - 1] : (id < 0 ? io.dvals[-id - 1] : 0.0);
  }
  __syncthreads();
  const double* A = io.dNt;
  for (int q = threadIdx.x; q < np; q += blockDim.x) {
    double G[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int n = 0; n < nn; ++n) {
      const double a0 = A[n + nn * (3 * q)], a1 = A[n + nn * (1 + 3 * q)], a2 = A[n + nn * (2 + 3 * q)];
      for (int c = 0; c < 3; ++c) {
        const double x = xl[c * nn + n];
        G[c][0] += x * a0;
        G[c][1] += x * a1;
        G[c][2] += x * a2;
      }
    }
    double Jt[9], iJ[9], det;
    if (cd.affine[cell]) {
      for (int i = 0; i < 9; ++i) iJ[i] = cd.geo[(size_t)cell * 10 + i];
      det = cd.geo[(size_t)cell * 10 + 9];
    } else {
      point_jacobian_dev(cd, cell, q, Jt);
      det = det3(Jt);
      inv3(Jt, det, iJ);
      det = fabs(det);
    }
    for (int c = 0; c < 3; ++c)
      for (int J = 0; J < 3; ++J) Hs[q * 9 + c + 3 * J] = iJ[J] * G[c][0] + iJ[J + 3] * G[c][1] + iJ[J + 6] * G[c][2];
    for (int i = 0; i < 9; ++i) iJs[q * 9 + i] = iJ[i];
    dVs[q] = cd.w[q] * det;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < np * 9; e += blockDim.x) {
    const int q = e / 9, ck = e % 9, c = ck / 3, k = ck % 3;
    double Tb[9];  // T[(c,J),(k,L)] at Tb[J + 3 L]
    law_tangent_block(cd.law, cd.lam_of(cell), cd.mu_of(cell), Hs + q * 9, c, k, Tb);
    const double* iJ = iJs + q * 9;
    double X[3][3];
    for (int J = 0; J < 3; ++J)
      for (int Kp = 0; Kp < 3; ++Kp) {
        double s = 0;
        for (int L = 0; L < 3; ++L) s += Tb[J + 3 * L] * iJ[L + 3 * Kp];
        X[J][Kp] = s;
      }
    for (int K = 0; K < 3; ++K)
      for (int Kp = 0; Kp < 3; ++Kp) {
        double s = 0;
        for (int J = 0; J < 3; ++J) s += iJ[J + 3 * K] * X[J][Kp];
        Dh[q * 81 + (c * 3 + K) + 9 * (k * 3 + Kp)] = dVs[q] * s;
      }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nn * 9; e += blockDim.x) {
    const int n = e / 9, ck = e % 9, ci = ck / 3, cj = ck % 3;
    const int blk = io.block_of[n + (size_t)nn * cell];
    if (blk == 0) continue;
    double s = 0;
    for (int q = 0; q < np; ++q) {
      const double a0 = A[n + nn * (3 * q)], a1 = A[n + nn * (1 + 3 * q)], a2 = A[n + nn * (2 + 3 * q)];
      const double* D = Dh + q * 81 + ci * 3 + 9 * (cj * 3);
      s += a0 * (D[0] * a0 + D[9] * a1 + D[18] * a2) + a1 * (D[1] * a0 + D[10] * a1 + D[19] * a2) +
           a2 * (D[2] * a0 + D[11] * a1 + D[20] * a2);
    }
    if (io.atomic) atomicAdd(&io.B[(size_t)(blk - 1) * 9 + ci + 3 * cj], s);
    else io.B[(size_t)(blk - 1) * 9 + ci + 3 * cj] += s;
  }
}

// The same blocks sum-factorised, for tensor-product cells (Q nodes, P points per direction, Q <= P).
// With a_K(n, q) = d phi_n / d xi_K (q), a product of 1D factors, a_K a_K' is the product over the
// directions d of u_e(n_d, q_d), e = [d == K] + [d == K'] (u_0 = N^2, u_1 = N dN, u_2 = dN^2); the
// nine (K, K') pairs fall in six patterns of exponents (K = K' = 0, 1, 2; {0,1}, {0,2}, {1,2}). Per
// point, the tangent block of (ci, cj) pulled back to the reference gradients gives six pattern
// sums F; three 1D sweeps contract each of the 54 fields over the points, and the node's block
// entry is the sum over its six patterns: O(54 (Q P^2 + Q^2 P + Q^3) P) per cell instead of
// O(9 Q^3 P^3) for the dense form.
template <int Q, int P>
__global__ void __launch_bounds__(256) blocks_tp_kernel(CellData cd, Tab1D<double> tab, BlockIO io) {
  constexpr int NN = Q * Q * Q, NP = P * P * P, NF = 54, T1N = Q * P * P, T2N = Q * Q * P;
  static_assert(Q <= P, "the sweeps reuse the field regions: Q <= P");
  extern __shared__ __align__(16) double sm[];
  double* xl = sm;            // 3 NN
  double* Hs = xl + 3 * NN;   // 9 NP
  double* iJs = Hs + 9 * NP;  // 9 NP
  double* dVs = iJs + 9 * NP; // NP
  double* F = dVs + NP;       // NF NP; then the y-sweep output (NF T2N)
  double* T1 = F + NF * NP;   // NF T1N; then the z-sweep output (NF NN)
  const int li = blockIdx.x;
  if (li >= cd.ncells_list) return;
  const int cell = cd.cells ? cd.cells[li] : li;
  const int32_t* gid = cd.ids + (size_t)cell * 3 * NN;
  for (int j = threadIdx.x; j < 3 * NN; j += blockDim.x) {
    const int32_t id = gid[j];
    xl[j] = id > 0 ? io.u[id - 1] : (id < 0 ? io.dvals[-id - 1] : 0.0);
  }
  __syncthreads();
  const double* A = io.dNt;
  // physical gradients H per point: with few points per cell the reference gradients are spread one
  // (point, component, direction) per thread (measured faster for Q2), else one point per thread
  constexpr bool SPREAD = 9 * NP <= 512;
  auto point_geometry = [&](int q, double* iJ, double& det) {
    double Jt[9];
    if (cd.affine[cell]) {
      for (int i = 0; i < 9; ++i) iJ[i] = cd.geo[(size_t)cell * 10 + i];
      det = cd.geo[(size_t)cell * 10 + 9];
    } else {
      point_jacobian_dev(cd, cell, q, Jt);
      det = det3(Jt);
      inv3(Jt, det, iJ);
      det = fabs(det);
    }
  };
  if constexpr (SPREAD) {
    double* Gs = F;  // 9 NP, in the field region (free until the tangent phase)
    for (int e = threadIdx.x; e < NP * 9; e += blockDim.x) {
      const int q = e / 9, cK = e % 9, c = cK / 3, K = cK % 3;
      const double* a = A + NN * (K + 3 * q);
      const double* x = xl + c * NN;
      double g = 0;
      for (int n = 0; n < NN; ++n) g += x[n] * a[n];
      Gs[e] = g;
    }
    for (int q = threadIdx.x; q < NP; q += blockDim.x) {
      double iJ[9], det;
      point_geometry(q, iJ, det);
      for (int i = 0; i < 9; ++i) iJs[q * 9 + i] = iJ[i];
      dVs[q] = cd.w[q] * det;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < NP * 9; e += blockDim.x) {  // H[q][c + 3 J] = sum_K iJ[J + 3 K] G[q][c][K]
      const int q = e / 9, cJ = e % 9, c = cJ % 3, J = cJ / 3;
      const double* iJ = iJs + q * 9;
      const double* G = Gs + q * 9 + c * 3;
      Hs[q * 9 + c + 3 * J] = iJ[J] * G[0] + iJ[J + 3] * G[1] + iJ[J + 6] * G[2];
    }
  } else {
    for (int q = threadIdx.x; q < NP; q += blockDim.x) {
      double G[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int n = 0; n < NN; ++n) {
        const double a0 = A[n + NN * (3 * q)], a1 = A[n + NN * (1 + 3 * q)], a2 = A[n + NN * (2 + 3 * q)];
        for (int c = 0; c < 3; ++c) {
          const double x = xl[c * NN + n];
          G[c][0] += x * a0;
          G[c][1] += x * a1;
          G[c][2] += x * a2;
        }
      }
      double iJ[9], det;
      point_geometry(q, iJ, det);
      for (int c = 0; c < 3; ++c)
        for (int J = 0; J < 3; ++J) Hs[q * 9 + c + 3 * J] = iJ[J] * G[c][0] + iJ[J + 3] * G[c][1] + iJ[J + 6] * G[c][2];
      for (int i = 0; i < 9; ++i) iJs[q * 9 + i] = iJ[i];
      dVs[q] = cd.w[q] * det;
    }
  }
  __syncthreads();
  // per point and component pair: D[K][K'] = dV sum_{J,L} iJ[J + 3K] T[(ci,J),(cj,L)] iJ[L + 3K'],
  // folded into the six pattern sums
  for (int e = threadIdx.x; e < NP * 9; e += blockDim.x) {
    const int q = e / 9, cc = e % 9, ci = cc / 3, cj = cc % 3;
    double Tb[9];
    law_tangent_block(cd.law, cd.lam_of(cell), cd.mu_of(cell), Hs + q * 9, ci, cj, Tb);
    const double* iJ = iJs + q * 9;
    double X[3][3], D[3][3];
    for (int J = 0; J < 3; ++J)
      for (int Kp = 0; Kp < 3; ++Kp) X[J][Kp] = Tb[J] * iJ[3 * Kp] + Tb[J + 3] * iJ[1 + 3 * Kp] + Tb[J + 6] * iJ[2 + 3 * Kp];
    for (int K = 0; K < 3; ++K)
      for (int Kp = 0; Kp < 3; ++Kp)
        D[K][Kp] = dVs[q] * (iJ[3 * K] * X[0][Kp] + iJ[1 + 3 * K] * X[1][Kp] + iJ[2 + 3 * K] * X[2][Kp]);
    double* f = F + (size_t)cc * 6 * NP + q;
    f[0 * NP] = D[0][0];
    f[1 * NP] = D[1][1];
    f[2 * NP] = D[2][2];
    f[3 * NP] = D[0][1] + D[1][0];
    f[4 * NP] = D[0][2] + D[2][0];
    f[5 * NP] = D[1][2] + D[2][1];
  }
  __syncthreads();
  auto ex = [](int pat, int d) {
    // pattern -> (ex, ey, ez): 0:(2,0,0) 1:(0,2,0) 2:(0,0,2) 3:(1,1,0) 4:(1,0,1) 5:(0,1,1)
    const int t[6][3] = {{2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
    return t[pat][d];
  };
  auto u = [&](int e, int n, int q) {
    const double a = tab.N1[q * Q + n], b = tab.dN1[q * Q + n];
    return e == 0 ? a * a : (e == 1 ? a * b : b * b);
  };
  for (int e = threadIdx.x; e < NF * T1N; e += blockDim.x) {  // x: [f][q3][q2][n1]
    const int f = e / T1N, r = e - f * T1N, n1 = r % Q, q23 = r / Q, ei = ex(f % 6, 0);
    const double* src = F + (size_t)f * NP + P * q23;
    double acc = 0;
#pragma unroll
    for (int q1 = 0; q1 < P; ++q1) acc += u(ei, n1, q1) * src[q1];
    T1[(size_t)f * T1N + n1 + Q * q23] = acc;
  }
  __syncthreads();
  double* T2 = F;
  for (int e = threadIdx.x; e < NF * T2N; e += blockDim.x) {  // y: [f][q3][n2][n1]
    const int f = e / T2N, r = e - f * T2N, n1 = r % Q, n2 = (r / Q) % Q, q3 = r / (Q * Q), ei = ex(f % 6, 1);
    const double* src = T1 + (size_t)f * T1N + n1 + Q * P * q3;
    double acc = 0;
#pragma unroll
    for (int q2 = 0; q2 < P; ++q2) acc += u(ei, n2, q2) * src[Q * q2];
    T2[(size_t)f * T2N + n1 + Q * n2 + Q * Q * q3] = acc;
  }
  __syncthreads();
  double* S = T1;
  for (int e = threadIdx.x; e < NF * NN; e += blockDim.x) {  // z: [f][n3][n2][n1]
    const int f = e / NN, n = e - f * NN, n12 = n % (Q * Q), n3 = n / (Q * Q), ei = ex(f % 6, 2);
    const double* src = T2 + (size_t)f * T2N + n12;
    double acc = 0;
#pragma unroll
    for (int q3 = 0; q3 < P; ++q3) acc += u(ei, n3, q3) * src[Q * Q * q3];
    S[(size_t)f * NN + n] = acc;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 9 * NN; e += blockDim.x) {
    const int cc = e / NN, n = e - cc * NN, ci = cc / 3, cj = cc % 3;
    const int blk = io.block_of[n + (size_t)NN * cell];
    if (blk == 0) continue;
    double v = 0;
#pragma unroll
    for (int pat = 0; pat < 6; ++pat) v += S[(size_t)(cc * 6 + pat) * NN + n];
    if (io.atomic) atomicAdd(&io.B[(size_t)(blk - 1) * 9 + ci + 3 * cj], v);
    else io.B[(size_t)(blk - 1) * 9 + ci + 3 * cj] += v;
  }
}

template <int Q, int P>
constexpr size_t blocks_tp_smem() {
  return ((size_t)3 * Q * Q * Q + 19 * P * P * P + 54 * P * P * P + 54 * Q * P * P) * sizeof(double);
}

// _invert_blocks! (src/preconditioners.jl:312-327): fixed components -> identity rows/columns
static __global__ void invert_blocks_kernel(int nb, const int32_t* dofs, const double* B, double* Binv, float* Binv32,
                                     int* bad) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    double M[9];
    bool fin = true;
    for (int j = 0; j < 3; ++j)
      for (int i = 0; i < 3; ++i) {
        const bool fixed = dofs[3 * b + i] == 0 || dofs[3 * b + j] == 0;
        M[i + 3 * j] = fixed ? (i == j ? 1.0 : 0.0) : B[9 * (size_t)b + i + 3 * j];
        fin &= isfinite(M[i + 3 * j]);
      }
    double Mi[9];
    if (fin) {
      inv3(M, det3(M), Mi);
      for (int i = 0; i < 9; ++i) fin &= isfinite(Mi[i]);
    } else {
      for (int i = 0; i < 9; ++i) Mi[i] = M[i];
    }
    if (!fin) atomicOr(bad, 1);
    for (int i = 0; i < 9; ++i) {
      Binv[9 * (size_t)b + i] = Mi[i];
      if (Binv32) Binv32[9 * (size_t)b + i] = (float)Mi[i];
    }
  }
}

// y[dofs] = Binv r[dofs] (ldiv!, src/preconditioners.jl:329-344)
template <typename R>
__global__ void blocks_apply_kernel(int nb, const int32_t* dofs, const R* Binv, const R* r, R* y) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    const int d0 = dofs[3 * b], d1 = dofs[3 * b + 1], d2 = dofs[3 * b + 2];
    const R r0 = d0 ? r[d0 - 1] : R(0), r1 = d1 ? r[d1 - 1] : R(0), r2 = d2 ? r[d2 - 1] : R(0);
    const R* M = Binv + 9 * (size_t)b;
    if (d0) y[d0 - 1] = M[0] * r0 + M[3] * r1 + M[6] * r2;
    if (d1) y[d1 - 1] = M[1] * r0 + M[4] * r1 + M[7] * r2;
    if (d2) y[d2 - 1] = M[2] * r0 + M[5] * r1 + M[8] * r2;
  }
}

// ---- Chebyshev (smooth!, src/smoothers.jl:116-146), fused per nodal block ----------------------
// start: r = rhs (zero guess) or r = rhs - Ax (z holds Ax); d = Binv r / theta; x = d or x += d
template <typename R>
__global__ void cheb_start_kernel(int nb, const int32_t* dofs, const R* Binv, const R* rhs, const R* Ax, R* r, R* d,
                                  R* x, R inv_theta, int zero_guess) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    int dd[3] = {dofs[3 * b], dofs[3 * b + 1], dofs[3 * b + 2]};
    R rr[3];
    for (int i = 0; i < 3; ++i) {
      rr[i] = 0;
      if (dd[i]) {
        R v = rhs[dd[i] - 1];
        if (!zero_guess) v -= Ax[dd[i] - 1];
        r[dd[i] - 1] = v;
        rr[i] = v;
      }
    }
    const R* M = Binv + 9 * (size_t)b;
    for (int i = 0; i < 3; ++i) {
      if (!dd[i]) continue;
      const R z = M[i] * rr[0] + M[i + 3] * rr[1] + M[i + 6] * rr[2];
      const R di = z * inv_theta;
      d[dd[i] - 1] = di;
      x[dd[i] - 1] = zero_guess ? di : x[dd[i] - 1] + di;
    }
  }
}
// step: r -= z (z = A d); if more: d = c1 d + c2 Binv r; x += d
template <typename R>
__global__ void cheb_step_kernel(int nb, const int32_t* dofs, const R* Binv, const R* z, R* r, R* d, R* x, R c1, R c2,
                                 int update_d) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    int dd[3] = {dofs[3 * b], dofs[3 * b + 1], dofs[3 * b + 2]};
    R rr[3];
    for (int i = 0; i < 3; ++i) {
      rr[i] = 0;
      if (dd[i]) {
        const R v = r[dd[i] - 1] - z[dd[i] - 1];
        r[dd[i] - 1] = v;
        rr[i] = v;
      }
    }
    if (!update_d) continue;
    const R* M = Binv + 9 * (size_t)b;
    for (int i = 0; i < 3; ++i) {
      if (!dd[i]) continue;
      const R zz = M[i] * rr[0] + M[i + 3] * rr[1] + M[i + 6] * rr[2];
      const R dn = c1 * d[dd[i] - 1] + c2 * zz;
      d[dd[i] - 1] = dn;
      x[dd[i] - 1] += dn;
    }
  }
}

// The same two steps with the coefficients read from device memory (coef = [1/theta, c1_1, c2_1,
// c1_2, c2_2, ...], written by the host at every update), so that a V-cycle captured once in a CUDA
// graph stays valid when the smoothing interval changes. With segments (segb non-null) block b
// reads the coefficients of its segment, coef + segb[b] * cstride.
template <typename R>
__global__ void cheb_start_dev_kernel(int nb, const int32_t* dofs, const R* Binv, const R* rhs, const R* Ax, R* r,
                                      R* d, R* x, const double* coef, const int32_t* segb, int cstride, int zero_guess) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    const R inv_theta = (R)coef[(segb ? (size_t)segb[b] * cstride : 0)];
    int dd[3] = {dofs[3 * b], dofs[3 * b + 1], dofs[3 * b + 2]};
    R rr[3];
    for (int i = 0; i < 3; ++i) {
      rr[i] = 0;
      if (dd[i]) {
        R v = rhs[dd[i] - 1];
        if (!zero_guess) v -= Ax[dd[i] - 1];
        r[dd[i] - 1] = v;
        rr[i] = v;
      }
    }
    const R* M = Binv + 9 * (size_t)b;
    for (int i = 0; i < 3; ++i) {
      if (!dd[i]) continue;
      const R di = (M[i] * rr[0] + M[i + 3] * rr[1] + M[i + 6] * rr[2]) * inv_theta;
      d[dd[i] - 1] = di;
      x[dd[i] - 1] = zero_guess ? di : x[dd[i] - 1] + di;
    }
  }
}
template <typename R>
__global__ void cheb_step_dev_kernel(int nb, const int32_t* dofs, const R* Binv, const R* z, R* r, R* d, R* x,
                                     const double* coef, const int32_t* segb, int cstride, int step, int update_d) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    const double* cb = coef + (segb ? (size_t)segb[b] * cstride : 0);
    const R c1 = update_d ? (R)cb[2 * step - 1] : R(0), c2 = update_d ? (R)cb[2 * step] : R(0);
    int dd[3] = {dofs[3 * b], dofs[3 * b + 1], dofs[3 * b + 2]};
    R rr[3];
    for (int i = 0; i < 3; ++i) {
      rr[i] = 0;
      if (dd[i]) {
        const R v = r[dd[i] - 1] - z[dd[i] - 1];
        r[dd[i] - 1] = v;
        rr[i] = v;
      }
    }
    if (!update_d) continue;
    const R* M = Binv + 9 * (size_t)b;
    for (int i = 0; i < 3; ++i) {
      if (!dd[i]) continue;
      const R dn = c1 * d[dd[i] - 1] + c2 * (M[i] * rr[0] + M[i + 3] * rr[1] + M[i + 6] * rr[2]);
      d[dd[i] - 1] = dn;
      x[dd[i] - 1] += dn;
    }
  }
}

// ---- Arnoldi without host synchronisation: scalars stay on the device -----------------------
// y += sign * (*alpha) * x
// *s = sqrt(*s)
// y = x / *s (0 when *s is 0: the breakdown is decided on the host from the Hessenberg matrix)

// ---- transfers (src/transfers.jl) ------------------------------------------------------------
struct XferData {
  const int32_t* ids_f;   // (3 NF, ncells) fine level, tensor order
  const int32_t* ids_c;   // (3 NC, ncells) coarse level
  const double* E;        // (NF, NC) column-major, tensor orders
  const double* Einj;     // (NC, NF)
  const int32_t* mult;    // per fine free dof
  const int32_t* cells;   // colour list or nullptr
  int ncells_list, NF, NC;
};

// prolongate_cells! (src/transfers.jl:179-193): fine value = E * coarse local values, inserted
template <typename R>
__global__ void prolongate_kernel(XferData t, const R* xc, R* yf) {
  const int per = 3 * t.NF;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)t.ncells_list * per;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int li = (int)(e / per), j = (int)(e % per);
    const int cell = t.cells ? t.cells[li] : li;
    const int32_t idf = t.ids_f[(size_t)cell * per + j];
    if (idf <= 0) continue;
    const int comp = j / t.NF, f = j % t.NF;
    const int32_t* ic = t.ids_c + (size_t)cell * 3 * t.NC + comp * t.NC;
    double s = 0;
    for (int c = 0; c < t.NC; ++c) {
      const double w = t.E[f + (size_t)t.NF * c];
      const int32_t id = ic[c];
      if (w != 0.0 && id > 0) s += w * (double)xc[id - 1];
    }
    yf[idf - 1] = (R)s;
  }
}

// restrict_cells! (src/transfers.jl:195-213): E^T (yf / multiplicity), scatter-add (coloured)
template <typename R>
__global__ void restrict_kernel(XferData t, const R* yf, R* yc) {
  const int per = 3 * t.NC;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)t.ncells_list * per;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int li = (int)(e / per), j = (int)(e % per);
    const int cell = t.cells ? t.cells[li] : li;
    const int32_t idc = t.ids_c[(size_t)cell * per + j];
    if (idc <= 0) continue;
    const int comp = j / t.NC, c = j % t.NC;
    const int32_t* iff = t.ids_f + (size_t)cell * 3 * t.NF + comp * t.NF;
    double s = 0;
    for (int f = 0; f < t.NF; ++f) {
      const double w = t.E[f + (size_t)t.NF * c];
      const int32_t id = iff[f];
      if (w != 0.0 && id > 0) s += w * ((double)yf[id - 1] / t.mult[id - 1]);
    }
    yc[idc - 1] += (R)s;
  }
}

// Sum-factorised transfers for tensor-product pairs of levels: the cell interpolation matrix is
// E = E1 (x) E1 (x) E1 (fine node i = i1 + nf (i2 + nf i3), coarse node b likewise), so the cell
// products of prolongate_cells! / restrict_cells! run as three 1D contractions per component
// instead of one dense NF x NC product. One warp per cell; the warp's shared-memory slab holds the
// cell's values and the two intermediate contractions.
struct XferTP {
  int nf = 0, nc = 0;            // 1D node counts of the fine and coarse levels
  double e1[MAXQ * MAXQ] = {};   // e1[i * nc + b] = E1[i][b]
  const double* invmult = nullptr;  // 1 / multiplicity per fine free dof (exact: 1, 2, 4, 8 cells)
};

__host__ __device__ inline int xfer_tp_slab(int nf, int nc) {  // doubles of one warp's slab
  return 3 * (nf * nf * nf + nf * nf * nc + nf * nc * nc);
}

// restrict_cells! (src/transfers.jl:195-213), sum-factorised: E^T (yf / multiplicity) per cell,
// added into yc atomically (atomic = 1) or by plain read-modify-write (one colour per launch)
template <typename R>
__global__ void restrict_tp_kernel(XferData t, XferTP tp, int atomic, const R* __restrict__ yf, R* yc) {
  extern __shared__ double xsm[];
  const int wpb = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int li = blockIdx.x * wpb + warp;
  if (li >= t.ncells_list) return;
  const int cell = t.cells ? t.cells[li] : li;
  const int nf = tp.nf, nc = tp.nc, NF = nf * nf * nf, NC = nc * nc * nc;
  double* u = xsm + (size_t)warp * xfer_tp_slab(nf, nc);  // [comp][i3][i2][i1]
  double* a = u + 3 * NF;                                 // [comp][i3][i2][b1]
  double* b = a + 3 * nf * nf * nc;                       // [comp][i3][b2][b1]
  const int32_t* iff = t.ids_f + (size_t)cell * 3 * NF;
  for (int q = lane; q < 3 * NF; q += 32) {
    const int32_t id = iff[q];
    u[q] = id > 0 ? (double)yf[id - 1] * tp.invmult[id - 1] : 0.0;
  }
  __syncwarp();
  for (int q = lane; q < 3 * nf * nf * nc; q += 32) {
    const int b1 = q % nc, r = q / nc;
    double s = 0;
    for (int i = 0; i < nf; ++i) s += tp.e1[i * nc + b1] * u[r * nf + i];
    a[q] = s;
  }
  __syncwarp();
  for (int q = lane; q < 3 * nf * nc * nc; q += 32) {
    const int b1 = q % nc, b2 = (q / nc) % nc, r = q / (nc * nc);
    double s = 0;
    for (int j = 0; j < nf; ++j) s += tp.e1[j * nc + b2] * a[(r * nf + j) * nc + b1];
    b[q] = s;
  }
  __syncwarp();
  const int32_t* ic = t.ids_c + (size_t)cell * 3 * NC;
  for (int q = lane; q < 3 * NC; q += 32) {
    const int32_t idc = ic[q];
    if (idc <= 0) continue;
    const int b12 = q % (nc * nc), r = q / (nc * nc), b3 = r % nc, comp = r / nc;
    double s = 0;
    for (int k = 0; k < nf; ++k) s += tp.e1[k * nc + b3] * b[(comp * nf + k) * nc * nc + b12];
    if (atomic) atomicAdd(yc + idc - 1, (R)s);
    else yc[idc - 1] += (R)s;
  }
}

// prolongate_cells! (src/transfers.jl:179-193), sum-factorised: fine values = E x coarse local
// values, written (cells sharing a fine dof write the same value)
template <typename R>
__global__ void prolongate_tp_kernel(XferData t, XferTP tp, const R* __restrict__ xc, R* yf) {
  extern __shared__ double xsm[];
  const int wpb = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int li = blockIdx.x * wpb + warp;
  if (li >= t.ncells_list) return;
  const int cell = t.cells ? t.cells[li] : li;
  const int nf = tp.nf, nc = tp.nc, NF = nf * nf * nf, NC = nc * nc * nc;
  double* v = xsm + (size_t)warp * xfer_tp_slab(nf, nc);  // [comp][b3][b2][b1]
  double* b = v + 3 * NC;                                 // [comp][i3][b2][b1]
  double* a = b + 3 * nf * nc * nc;                       // [comp][i3][i2][b1]
  const int32_t* ic = t.ids_c + (size_t)cell * 3 * NC;
  for (int q = lane; q < 3 * NC; q += 32) {
    const int32_t id = ic[q];
    v[q] = id > 0 ? (double)xc[id - 1] : 0.0;
  }
  __syncwarp();
  for (int q = lane; q < 3 * nf * nc * nc; q += 32) {
    const int b12 = q % (nc * nc), r = q / (nc * nc), k = r % nf, comp = r / nf;
    double s = 0;
    for (int b3 = 0; b3 < nc; ++b3) s += tp.e1[k * nc + b3] * v[(comp * nc + b3) * nc * nc + b12];
    b[q] = s;
  }
  __syncwarp();
  for (int q = lane; q < 3 * nf * nf * nc; q += 32) {
    const int b1 = q % nc, j = (q / nc) % nf, r = q / (nc * nf);
    double s = 0;
    for (int b2 = 0; b2 < nc; ++b2) s += tp.e1[j * nc + b2] * b[(r * nc + b2) * nc + b1];
    a[q] = s;
  }
  __syncwarp();
  const int32_t* iff = t.ids_f + (size_t)cell * 3 * NF;
  for (int q = lane; q < 3 * NF; q += 32) {
    const int32_t idf = iff[q];
    if (idf <= 0) continue;
    const int i = q % nf, r = q / nf;
    double s = 0;
    for (int b1 = 0; b1 < nc; ++b1) s += tp.e1[i * nc + b1] * a[r * nc + b1];
    yf[idf - 1] = (R)s;
  }
}

// inject_field! (src/transfers.jl:295-313)
static __global__ void inject_kernel(XferData t, int ncells, const double* xf, const double* df, double* xc, double* dc) {
  const int per = 3 * t.NC;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)ncells * per;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int cell = (int)(e / per), j = (int)(e % per);
    const int comp = j / t.NC, c = j % t.NC;
    const int32_t* iff = t.ids_f + (size_t)cell * 3 * t.NF + comp * t.NF;
    double v = 0;
    for (int f = 0; f < t.NF; ++f) {
      const double w = t.Einj[c + (size_t)t.NC * f];
      if (w == 0.0) continue;
      const int32_t id = iff[f];
      v += w * (id > 0 ? xf[id - 1] : df[-id - 1]);
    }
    const int32_t idc = t.ids_c[(size_t)cell * per + j];
    if (idc > 0) xc[idc - 1] = v;
    else if (idc < 0) dc[-idc - 1] = v;
  }
}

// ---- dense coarse solve -----------------------------------------------------------------------
// CSC (1-based) -> dense column-major n x n
static __global__ void csc_to_dense_kernel(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval,
                                    double* A) {
  for (int64_t c = blockIdx.x; c < n; c += gridDim.x)
    for (int64_t k = colptr[c] - 1 + threadIdx.x; k < colptr[c + 1] - 1; k += blockDim.x)
      A[(rowval[k] - 1) + n * c] = nzval[k];
}
}  // namespace hfk
