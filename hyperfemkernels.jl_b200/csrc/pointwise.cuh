// Pointwise laws and 3x3 geometry helpers (device).
//
// Conventions: a 3x3 matrix is column-major, M[i + 3*j]. H[c + 3*J] = du_c/dx_J (Gridap's
// grad(u)', so F = I + H). The laws are the pointwise functions the reference's codegen emits for
// the SVK form of test/common.jl:1-8 (README.md:61-67) and for the linear-elastic stress of
// test/solvers/test_pmultigrid.jl:9 (sigma = lambda tr(G) I + mu (G + G')).
#pragma once
#include "hfk_internal.h"

namespace hfk {

__host__ __device__ inline double det3(const double* A) {
  return A[0] * (A[4] * A[8] - A[7] * A[5]) - A[3] * (A[1] * A[8] - A[7] * A[2]) + A[6] * (A[1] * A[5] - A[4] * A[2]);
}

__host__ __device__ inline void inv3(const double* A, double d, double* B) {
  const double id = 1.0 / d;
  B[0] = (A[4] * A[8] - A[7] * A[5]) * id;
  B[3] = -(A[3] * A[8] - A[6] * A[5]) * id;
  B[6] = (A[3] * A[7] - A[6] * A[4]) * id;
  B[1] = -(A[1] * A[8] - A[7] * A[2]) * id;
  B[4] = (A[0] * A[8] - A[6] * A[2]) * id;
  B[7] = -(A[0] * A[7] - A[6] * A[1]) * id;
  B[2] = (A[1] * A[5] - A[4] * A[2]) * id;
  B[5] = -(A[0] * A[5] - A[3] * A[2]) * id;
  B[8] = (A[0] * A[4] - A[3] * A[1]) * id;
}

// Jt[K + 3i] = sum_n dM[n, K, q] x[n, i] (point_jacobian, src/assembly.jl:1073-1081), trilinear map
__device__ inline void point_jacobian_dev(const CellData& cd, int cell, int q, double* Jt) {
#pragma unroll
  for (int i = 0; i < 9; ++i) Jt[i] = 0.0;
  const double* X = cd.coords + (size_t)cell * 24;
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    const double x0 = X[3 * n], x1 = X[3 * n + 1], x2 = X[3 * n + 2];
#pragma unroll
    for (int K = 0; K < 3; ++K) {
      const double g = cd.dMt[n + 8 * (K + 3 * q)];
      Jt[K] += g * x0;
      Jt[K + 3] += g * x1;
      Jt[K + 6] += g * x2;
    }
  }
}

// H[c + 3J] = sum_K iJ[J + 3K] G[f0 + c][K]: physical gradient from reference gradients
template <typename R, int NF>
__device__ __forceinline__ void phys_grad(const R* iJ, const R (&G)[NF][3], int f0, R* H) {
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int J = 0; J < 3; ++J) H[c + 3 * J] = iJ[J] * G[f0 + c][0] + iJ[J + 3] * G[f0 + c][1] + iJ[J + 6] * G[f0 + c][2];
}

// out[c][K] = dV sum_J iJ[J + 3K] M[c + 3J]: slot coefficients pulled back to the reference
// gradients (slot_coefs, src/kernels.jl:323-338)
template <typename R>
__device__ __forceinline__ void pull_back(const R* iJ, const R* M, R dV, R (&out)[3][3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int K = 0; K < 3; ++K)
      out[c][K] = dV * (iJ[3 * K] * M[c] + iJ[1 + 3 * K] * M[c + 3] + iJ[2 + 3 * K] * M[c + 6]);
}

// First Piola stress P(F), F = I + H
template <typename R>
__device__ __forceinline__ void law_stress(int law, R lam, R mu, const R* H, R* Pm) {
  if (law == HFK_LAW_LINEAR_ELASTIC) {
    const R tr = H[0] + H[4] + H[8];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int J = 0; J < 3; ++J) Pm[c + 3 * J] = (c == J ? lam * tr : R(0)) + mu * (H[c + 3 * J] + H[J + 3 * c]);
    return;
  }
  R F[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) F[i] = H[i];
  F[0] += R(1);
  F[4] += R(1);
  F[8] += R(1);
  // S = lam tr(E) I + 2 mu E, E = (F'F - I)/2 -> S = lam tr(E) I + mu (C - I)
  R C[9];
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int J = 0; J < 3; ++J) C[I + 3 * J] = F[3 * I] * F[3 * J] + F[1 + 3 * I] * F[1 + 3 * J] + F[2 + 3 * I] * F[2 + 3 * J];
  const R trE = R(0.5) * (C[0] + C[4] + C[8] - R(3));
  R S[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) S[i] = mu * C[i];
  S[0] += lam * trE - mu;
  S[4] += lam * trE - mu;
  S[8] += lam * trE - mu;
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int J = 0; J < 3; ++J) Pm[c + 3 * J] = F[c] * S[3 * J] + F[c + 3] * S[1 + 3 * J] + F[c + 6] * S[2 + 3 * J];
}

// Directional derivative dP = (dP/dF)[Hd] at the deformation gradient F (stored per point)
// SVK: dP = Hd S + F (lam tr(F'Hd) I + mu (Hd'F + F'Hd))
template <typename R>
__device__ __forceinline__ void law_dstress_F(int law, R lam, R mu, const R* F, const R* Hd, R* dP) {
  if (law == HFK_LAW_LINEAR_ELASTIC) {
    law_stress<R>(law, lam, mu, Hd, dP);
    return;
  }
  R C[9], M[9];
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int J = 0; J < 3; ++J) {
      C[I + 3 * J] = F[3 * I] * F[3 * J] + F[1 + 3 * I] * F[1 + 3 * J] + F[2 + 3 * I] * F[2 + 3 * J];
      M[I + 3 * J] = F[3 * I] * Hd[3 * J] + F[1 + 3 * I] * Hd[1 + 3 * J] + F[2 + 3 * I] * Hd[2 + 3 * J];
    }
  const R trE = R(0.5) * (C[0] + C[4] + C[8] - R(3));
  const R trM = M[0] + M[4] + M[8];
  R S[9], W[9];
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int J = 0; J < 3; ++J) {
      S[I + 3 * J] = mu * C[I + 3 * J] + (I == J ? lam * trE - mu : R(0));
      W[I + 3 * J] = mu * (M[I + 3 * J] + M[J + 3 * I]) + (I == J ? lam * trM : R(0));
    }
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int J = 0; J < 3; ++J)
      dP[c + 3 * J] = Hd[c] * S[3 * J] + Hd[c + 3] * S[1 + 3 * J] + Hd[c + 6] * S[2 + 3 * J] + F[c] * W[3 * J] +
                      F[c + 3] * W[1 + 3 * J] + F[c + 6] * W[2 + 3 * J];
}

// Full tangent T[(c*3+J) + 9*(k*3+L)] = dP[c,J]/dF[k,L] (point_tangent, src/factorforms.jl:316-322)
// SVK: delta_ck S[L,J] + lam F[c,J] F[k,L] + mu F[c,L] F[k,J] + mu (F F')[c,k] delta_JL
// Stored energy density of a law at H = grad u (H[c + 3J] = d u_c / d x_J): SVK
// Ψ = μ E:E + λ/2 (tr E)², E = (FᵀF - I)/2; linear elasticity the same with E = sym(H)
__device__ inline double law_energy(int law, double lam, double mu, const double* H) {
  double E[9];
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int J = 0; J < 3; ++J) {
      double e = 0.5 * (H[I + 3 * J] + H[J + 3 * I]);
      if (law != HFK_LAW_LINEAR_ELASTIC) e += 0.5 * (H[3 * I] * H[3 * J] + H[1 + 3 * I] * H[1 + 3 * J] + H[2 + 3 * I] * H[2 + 3 * J]);
      E[I + 3 * J] = e;
    }
  double ee = 0;
#pragma unroll
  for (int i = 0; i < 9; ++i) ee += E[i] * E[i];
  const double tr = E[0] + E[4] + E[8];
  return mu * ee + 0.5 * lam * tr * tr;
}

// One 3x3 block of the tangent: Tb[J + 3 L] = T[(c,J),(k,L)] (the same closed forms as
// law_tangent, for callers that need the (c, k) block only: no 81-entry array per thread)
__device__ inline void law_tangent_block(int law, double lam, double mu, const double* H, int c, int k, double* Tb) {
  if (law == HFK_LAW_LINEAR_ELASTIC) {
#pragma unroll
    for (int J = 0; J < 3; ++J)
#pragma unroll
      for (int L = 0; L < 3; ++L)
        Tb[J + 3 * L] = lam * (c == J) * (k == L) + mu * ((c == k) * (J == L) + (c == L) * (J == k));
    return;
  }
  double F[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) F[i] = H[i] + ((i % 4) == 0 ? 1.0 : 0.0);
  double Fc[3], Fk[3];  // rows c and k of F
#pragma unroll
  for (int J = 0; J < 3; ++J) {
    Fc[J] = c == 0 ? F[3 * J] : (c == 1 ? F[1 + 3 * J] : F[2 + 3 * J]);
    Fk[J] = k == 0 ? F[3 * J] : (k == 1 ? F[1 + 3 * J] : F[2 + 3 * J]);
  }
  double C[9];
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int J = 0; J < 3; ++J) C[I + 3 * J] = F[3 * I] * F[3 * J] + F[1 + 3 * I] * F[1 + 3 * J] + F[2 + 3 * I] * F[2 + 3 * J];
  const double trE = 0.5 * (C[0] + C[4] + C[8] - 3.0);
  const double ffck = Fc[0] * Fk[0] + Fc[1] * Fk[1] + Fc[2] * Fk[2];
#pragma unroll
  for (int J = 0; J < 3; ++J)
#pragma unroll
    for (int L = 0; L < 3; ++L) {
      const double S = mu * C[L + 3 * J] + (L == J ? lam * trE - mu : 0.0);
      Tb[J + 3 * L] = (c == k ? S : 0.0) + lam * Fc[J] * Fk[L] + mu * Fc[L] * Fk[J] + (J == L ? mu * ffck : 0.0);
    }
}

__device__ inline void law_tangent(int law, double lam, double mu, const double* H, double* T) {
  if (law == HFK_LAW_LINEAR_ELASTIC) {
    for (int c = 0; c < 3; ++c)
      for (int J = 0; J < 3; ++J)
        for (int k = 0; k < 3; ++k)
          for (int L = 0; L < 3; ++L)
            T[(c * 3 + J) + 9 * (k * 3 + L)] = lam * (c == J) * (k == L) + mu * ((c == k) * (J == L) + (c == L) * (J == k));
    return;
  }
  double F[9];
  for (int i = 0; i < 9; ++i) F[i] = H[i];
  F[0] += 1;
  F[4] += 1;
  F[8] += 1;
  double C[9], FF[9];
  for (int I = 0; I < 3; ++I)
    for (int J = 0; J < 3; ++J) {
      C[I + 3 * J] = F[3 * I] * F[3 * J] + F[1 + 3 * I] * F[1 + 3 * J] + F[2 + 3 * I] * F[2 + 3 * J];
      FF[I + 3 * J] = F[I] * F[J] + F[I + 3] * F[J + 3] + F[I + 6] * F[J + 6];
    }
  const double trE = 0.5 * (C[0] + C[4] + C[8] - 3.0);
  double S[9];
  for (int I = 0; I < 3; ++I)
    for (int J = 0; J < 3; ++J) S[I + 3 * J] = mu * C[I + 3 * J] + (I == J ? lam * trE - mu : 0.0);
  for (int c = 0; c < 3; ++c)
    for (int J = 0; J < 3; ++J)
      for (int k = 0; k < 3; ++k)
        for (int L = 0; L < 3; ++L)
          T[(c * 3 + J) + 9 * (k * 3 + L)] = (c == k ? S[L + 3 * J] : 0.0) + lam * F[c + 3 * J] * F[k + 3 * L] +
                                             mu * F[c + 3 * L] * F[k + 3 * J] + (J == L ? mu * FF[c + 3 * k] : 0.0);
}

}  // namespace hfk
