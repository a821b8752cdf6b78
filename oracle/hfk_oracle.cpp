// CPU oracle: a C++17/OpenMP restatement of HyperFEMKernels' hot-path algorithms.
//
// TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA engine and the timed CPU
// baseline ("CPU restatement of the reference algorithm"). Nothing in the product links it.
//
// Parity status: the reference (Julia + Gridap) cannot run without Julia, which is absent, and ships
// no golden vectors (its tests compare against a live Gridap). The restatement is pinned by the
// reference's own known-answer and property tests, restated in tests/ (partition of unity,
// exact affine gradients, tensor-product == dense tables, matrix-free == assembled,
// colouring conflict-freedom, coarse = P^T A P, Chebyshev damping closed form, ...), plus an
// independent finite-difference check of the tangent. Parity vs Gridap: unpinned.
//
// Layouts are Julia's column-major ones (the reference's arrays as a `ccall` would pass them):
//   ids    (ndl, ncells) int32, ldof = c*nn + n, >0 free id (1-based), <0 Dirichlet (-id)
//   Nt     (nn, np)         dNt (nn, 3, np)        dMt (ng, 3, np)        w (np)
//   xq     (3, np)          coords (3, ng, ncells)
// Every function cites the reference file:line it restates.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int D = 3;
constexpr int NS = 9;  // gradient slots of a 3-component field: s = c*3 + J

struct Problem {
  int ncells, nn, np, ng, ndl;
  int64_t nfree, ndir;
  std::vector<double> Nt, dNt, dMt, w, xq, coords;
  std::vector<int32_t> ids;
  int law;  // 1 = St Venant-Kirchhoff, 2 = linear elasticity
  double lam, mu, body[3];
  // geometry once per affine cell (GeoTable.cellaff, src/tables.jl:128-156; cell_geometry, src/assembly.jl:1100-1107)
  std::vector<uint8_t> affine;
  std::vector<double> cellJt;  // 9 per cell (at point 1)
  // colours
  std::vector<std::vector<int32_t>> colors;
  // pattern
  std::vector<int64_t> colptr, rowval;
  std::vector<int32_t> nzpos;
  // matrix-free data (GroupData, src/matrixfree.jl:14-23)
  std::vector<double> T, iJt, dV;
  // tensor-product table (TPTable, src/tensorproduct.jl:13-91)
  int Q = 0, P = 0;
  std::vector<double> N1, dN1;  // P x Q column-major: N1[a + P*i]
  std::vector<int> nodeperm, pointperm;
  // nodal blocks (FieldBlocks, src/preconditioners.jl:123-130)
  int nblocks = 0;
  std::vector<int32_t> block_of;  // nn x ncells
  std::vector<int32_t> bdofs;     // 3 x nblocks
  std::vector<double> B, Binv;    // 9 x nblocks
};

inline int nthreads_or(int n) {
#ifdef _OPENMP
  return n > 0 ? n : omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

// ---- small 3x3 helpers (column-major: M[i + 3*j]) ----------------------------------------
inline double det3(const double* A) {
  return A[0] * (A[4] * A[8] - A[7] * A[5]) - A[3] * (A[1] * A[8] - A[7] * A[2]) +
         A[6] * (A[1] * A[5] - A[4] * A[2]);
}
inline void inv3(const double* A, double* B) {
  double d = det3(A);
  double id = 1.0 / d;
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

// Jt[K, i] = sum_n dM[n, K, q] x[n, i]  (point_jacobian, src/assembly.jl:1073-1081)
void point_jacobian(const Problem& p, int q, int cell, double* Jt) {
  for (int i = 0; i < 9; ++i) Jt[i] = 0.0;
  const double* X = &p.coords[(size_t)cell * 3 * p.ng];
  for (int n = 0; n < p.ng; ++n)
    for (int K = 0; K < 3; ++K) {
      double g = p.dMt[n + p.ng * (K + 3 * q)];
      for (int i = 0; i < 3; ++i) Jt[K + 3 * i] += g * X[i + 3 * n];
    }
}

// (dV, iJt) at point q (point_geometry with CellGeometry, src/assembly.jl:1083-1111)
void point_geometry(const Problem& p, int q, int cell, double& dV, double* iJt) {
  double Jt[9];
  if (p.affine[cell]) {
    std::memcpy(Jt, &p.cellJt[9 * (size_t)cell], sizeof Jt);
  } else {
    point_jacobian(p, q, cell, Jt);
  }
  dV = p.w[q] * std::fabs(det3(Jt));
  inv3(Jt, iJt);
}

// affine_cells (src/tables.jl:128-156): every node satisfies x_n - x_1 = (xi_n - xi_1) . Jt
void compute_affine(Problem& p) {
  p.affine.assign(p.ncells, 0);
  p.cellJt.assign(9 * (size_t)p.ncells, 0.0);
  if (p.ng != 8) return;
  const double eps = 2.220446049250313e-16;
  for (int cell = 0; cell < p.ncells; ++cell) {
    double Jt[9];
    point_jacobian(p, 0, cell, Jt);
    std::memcpy(&p.cellJt[9 * (size_t)cell], Jt, sizeof Jt);
    const double* X = &p.coords[(size_t)cell * 3 * p.ng];
    double h = 0.0;
    for (int n = 1; n < 8; ++n) {
      double s = 0;
      for (int i = 0; i < 3; ++i) s += (X[i + 3 * n] - X[i]) * (X[i + 3 * n] - X[i]);
      h = std::max(h, std::sqrt(s));
    }
    bool ok = true;
    for (int n = 1; n < 8; ++n) {
      double xi[3] = {double(n & 1), double((n >> 1) & 1), double((n >> 2) & 1)};
      double e2 = 0, nx = 0;
      for (int i = 0; i < 3; ++i) {
        double pr = 0;
        for (int K = 0; K < 3; ++K) pr += xi[K] * Jt[K + 3 * i];
        double r = X[i + 3 * n] - X[i] - pr;
        e2 += r * r;
        nx += X[i + 3 * n] * X[i + 3 * n];
      }
      ok &= std::sqrt(e2) <= 1e-13 * h + 8 * eps * std::sqrt(nx);
    }
    p.affine[cell] = ok;
  }
}

// ---- the pointwise laws ------------------------------------------------------------------
// F[c, J] = delta + du_c/dx_J  (Gridap's F = I + grad(u)'), column-major F[c + 3J].
// SVK: P = F S, S = lam tr(E) I + 2 mu E, E = (F^T F - I)/2 (test/common.jl:1-8, README.md:61-67).
void law_stress(const Problem& p, const double* F, double* Pout) {
  if (p.law == 2) {  // sigma = lam tr(H) I + mu (H + H^T), H = F - I
    double tr = F[0] + F[4] + F[8] - 3.0;
    for (int J = 0; J < 3; ++J)
      for (int c = 0; c < 3; ++c) {
        double hcj = F[c + 3 * J] - (c == J ? 1.0 : 0.0);
        double hjc = F[J + 3 * c] - (c == J ? 1.0 : 0.0);
        Pout[c + 3 * J] = (c == J ? p.lam * tr : 0.0) + p.mu * (hcj + hjc);
      }
    return;
  }
  double E[9], S[9];
  for (int I = 0; I < 3; ++I)
    for (int J = 0; J < 3; ++J) {
      double s = 0;
      for (int a = 0; a < 3; ++a) s += F[a + 3 * I] * F[a + 3 * J];
      E[I + 3 * J] = 0.5 * (s - (I == J ? 1.0 : 0.0));
    }
  double tr = E[0] + E[4] + E[8];
  for (int i = 0; i < 9; ++i) S[i] = 2 * p.mu * E[i];
  S[0] += p.lam * tr;
  S[4] += p.lam * tr;
  S[8] += p.lam * tr;
  for (int c = 0; c < 3; ++c)
    for (int J = 0; J < 3; ++J) {
      double s = 0;
      for (int M = 0; M < 3; ++M) s += F[c + 3 * M] * S[M + 3 * J];
      Pout[c + 3 * J] = s;
    }
}

// T[(c,J),(k,L)] = dP[c,J]/dF[k,L], slot s = c*3 + J, T[sv + 9*su]: the exact tangent that the
// factorised form evaluates with dual numbers (point_tangent, src/factorforms.jl:316-322).
// SVK: delta_ck S[L,J] + lam F[c,J] F[k,L] + mu F[c,L] F[k,J] + mu (F F^T)[c,k] delta_JL.
void law_tangent(const Problem& p, const double* F, double* T) {
  if (p.law == 2) {
    for (int c = 0; c < 3; ++c)
      for (int J = 0; J < 3; ++J)
        for (int k = 0; k < 3; ++k)
          for (int L = 0; L < 3; ++L)
            T[(c * 3 + J) + 9 * (k * 3 + L)] = p.lam * (c == J) * (k == L) + p.mu * ((c == k) * (J == L) + (c == L) * (J == k));
    return;
  }
  double E[9], S[9], FF[9];
  for (int I = 0; I < 3; ++I)
    for (int J = 0; J < 3; ++J) {
      double s = 0, t = 0;
      for (int a = 0; a < 3; ++a) {
        s += F[a + 3 * I] * F[a + 3 * J];
        t += F[I + 3 * a] * F[J + 3 * a];
      }
      E[I + 3 * J] = 0.5 * (s - (I == J ? 1.0 : 0.0));
      FF[I + 3 * J] = t;
    }
  double tr = E[0] + E[4] + E[8];
  for (int i = 0; i < 9; ++i) S[i] = 2 * p.mu * E[i];
  S[0] += p.lam * tr;
  S[4] += p.lam * tr;
  S[8] += p.lam * tr;
  for (int c = 0; c < 3; ++c)
    for (int J = 0; J < 3; ++J)
      for (int k = 0; k < 3; ++k)
        for (int L = 0; L < 3; ++L) {
          double v = (c == k ? S[L + 3 * J] : 0.0) + p.lam * F[c + 3 * J] * F[k + 3 * L] +
                     p.mu * F[c + 3 * L] * F[k + 3 * J] + (J == L ? p.mu * FF[c + 3 * k] : 0.0);
          T[(c * 3 + J) + 9 * (k * 3 + L)] = v;
        }
}

// gather_cell! (src/assembly.jl:1060-1070)
void gather_cell(const Problem& p, const double* x, const double* dvals, int cell, double* xl) {
  const int32_t* id = &p.ids[(size_t)cell * p.ndl];
  for (int j = 0; j < p.ndl; ++j) {
    int32_t v = id[j];
    xl[j] = v > 0 ? x[v - 1] : (v < 0 ? dvals[-v - 1] : 0.0);
  }
}

// F at point q from local values: G^[c,K] = sum_n x_{n,c} dN[n,K,q]; grad u[J,c] = sum_K iJt[J,K] G^[c,K]
// (field_point_values, src/kernels.jl:210-232)
void point_F(const Problem& p, const double* xl, int q, const double* iJt, double* F) {
  double G[9] = {0};
  for (int n = 0; n < p.nn; ++n)
    for (int K = 0; K < 3; ++K) {
      double d = p.dNt[n + p.nn * (K + 3 * q)];
      for (int c = 0; c < 3; ++c) G[c + 3 * K] += xl[c * p.nn + n] * d;
    }
  for (int c = 0; c < 3; ++c)
    for (int J = 0; J < 3; ++J) {
      double s = 0;
      for (int K = 0; K < 3; ++K) s += iJt[J + 3 * K] * G[c + 3 * K];
      F[c + 3 * J] = s + (c == J ? 1.0 : 0.0);
    }
}

// element_residual_mm! (src/assembly.jl:1219-1241) + residual_coefs! (src/kernels.jl:340-356)
// + residual_products! (src/assembly.jl:1249-1270)
void element_residual(const Problem& p, const double* xl, int cell, double* re, std::vector<double>& C) {
  const int nn = p.nn, np = p.np;
  C.assign((size_t)np * 4 * 3, 0.0);  // rows (q, jj): jj 0 = value, 1..3 = reference gradients
  for (int q = 0; q < np; ++q) {
    double dV, iJt[9], F[9], Pq[9];
    point_geometry(p, q, cell, dV, iJt);
    point_F(p, xl, q, iJt, F);
    law_stress(p, F, Pq);
    for (int c = 0; c < 3; ++c) {
      C[(q * 4 + 0) + (size_t)np * 4 * c] = -dV * p.body[c];
      for (int K = 0; K < 3; ++K) {
        double s = 0;
        for (int J = 0; J < 3; ++J) s += iJt[J + 3 * K] * Pq[c + 3 * J];
        C[(q * 4 + 1 + K) + (size_t)np * 4 * c] = dV * s;
      }
    }
  }
  for (int c = 0; c < 3; ++c)
    for (int n = 0; n < nn; ++n) {
      double s = 0;
      for (int q = 0; q < np; ++q) {
        s += p.Nt[n + nn * q] * C[(q * 4) + (size_t)np * 4 * c];
        for (int K = 0; K < 3; ++K) s += p.dNt[n + nn * (K + 3 * q)] * C[(q * 4 + 1 + K) + (size_t)np * 4 * c];
      }
      re[c * nn + n] = s;
    }
}

// gemm_add! (src/kernels.jl:640-690): C[m, n] += sum_r A[m, r] B[r, n], m < M, n < N, r < R, with
// MB x NB tiles of C held in registers over the whole r loop: 8 x 4 tiles, then 4/2/1-row and
// 1-column remainders. Each entry is summed over r in order, then added to C once.
template <int MB, int NB>
inline void gemm_tile(double* __restrict__ C, int ldc, const double* __restrict__ A, int lda,
                      const double* __restrict__ B, int ldb, int R) {
  if constexpr (MB % 4 == 0) {
    typedef double v4 __attribute__((vector_size(32)));
    constexpr int MV = MB / 4;
    v4 acc[NB][MV];
#pragma GCC unroll 8
    for (int j = 0; j < NB; ++j)
#pragma GCC unroll 8
      for (int i = 0; i < MV; ++i) acc[j][i] = v4{0, 0, 0, 0};
    for (int r = 0; r < R; ++r) {
      const double* a = A + (size_t)lda * r;
      v4 av[MV];
#pragma GCC unroll 8
      for (int i = 0; i < MV; ++i) __builtin_memcpy(&av[i], a + 4 * i, sizeof(v4));
#pragma GCC unroll 8
      for (int j = 0; j < NB; ++j) {
        const double b = B[r + (size_t)ldb * j];
#pragma GCC unroll 8
        for (int i = 0; i < MV; ++i) acc[j][i] += av[i] * b;
      }
    }
    for (int j = 0; j < NB; ++j)
      for (int i = 0; i < MV; ++i)
        for (int l = 0; l < 4; ++l) C[4 * i + l + (size_t)ldc * j] += acc[j][i][l];
  } else {
    double acc[NB][MB] = {};
    for (int r = 0; r < R; ++r) {
      const double* a = A + (size_t)lda * r;
#pragma GCC unroll 8
      for (int j = 0; j < NB; ++j) {
        const double b = B[r + (size_t)ldb * j];
#pragma GCC unroll 8
        for (int i = 0; i < MB; ++i) acc[j][i] += a[i] * b;
      }
    }
    for (int j = 0; j < NB; ++j)
      for (int i = 0; i < MB; ++i) C[i + (size_t)ldc * j] += acc[j][i];
  }
}

template <int NB>
inline void gemm_cols(double* C, int ldc, const double* A, int lda, const double* B, int ldb, int M, int R) {
  int m0 = 0;
  for (; m0 + 8 <= M; m0 += 8) gemm_tile<8, NB>(C + m0, ldc, A + m0, lda, B, ldb, R);
  int rem = M - m0;
  if (rem >= 4) { gemm_tile<4, NB>(C + m0, ldc, A + m0, lda, B, ldb, R); m0 += 4; rem -= 4; }
  if (rem >= 2) { gemm_tile<2, NB>(C + m0, ldc, A + m0, lda, B, ldb, R); m0 += 2; rem -= 2; }
  if (rem >= 1) gemm_tile<1, NB>(C + m0, ldc, A + m0, lda, B, ldb, R);
}

inline void gemm_add(double* C, int ldc, const double* A, int lda, const double* B, int ldb, int M, int N, int R) {
  int n0 = 0;
  for (; n0 + 4 <= N; n0 += 4) gemm_cols<4>(C + (size_t)ldc * n0, ldc, A, lda, B + (size_t)ldb * n0, ldb, M, R);
  for (; n0 < N; ++n0) gemm_cols<1>(C + (size_t)ldc * n0, ldc, A, lda, B + (size_t)ldb * n0, ldb, M, R);
}

// element_jacobian_mm! (src/assembly.jl:1316-1342): point blocks of POINT_BLOCK points,
// B[(ql,jj), n] = W[n, jj] (store_test_weights!), G[m, (ql,jj), k, c] = dV sum_ll T W[m, ll]
// (store_trial_block!), KeT[(m,k), (n,c)] += sum_r G B (block_products!/gemm_add!, src/kernels.jl:615-705).
void element_jacobian(const Problem& p, const double* xl, int cell, double* KeT, int point_block,
                      std::vector<double>& W, std::vector<double>& Bb, std::vector<double>& Gb) {
  const int nn = p.nn, np = p.np, ndl = p.ndl;
  std::fill(KeT, KeT + (size_t)ndl * ndl, 0.0);
  const int qb = point_block <= 0 ? np : std::min(point_block, np);
  W.assign((size_t)nn * 3, 0.0);
  Bb.assign((size_t)qb * 3 * nn, 0.0);     // (ql*3 + jj) + qb*3*n
  Gb.assign((size_t)nn * qb * 3 * 9, 0.0);  // m + nn*((ql*3+jj) + qb*3*(k + 3c))
  for (int q0 = 0; q0 < np; q0 += qb) {
    int nq = std::min(qb, np - q0);
    for (int ql = 0; ql < nq; ++ql) {
      int q = q0 + ql;
      double dV, iJt[9], F[9], T[81];
      point_geometry(p, q, cell, dV, iJt);
      // physical gradient weights W[n, J] (point_weights!, src/kernels.jl:142-157)
      for (int J = 0; J < 3; ++J)
        for (int n = 0; n < nn; ++n) {
          double s = 0;
          for (int K = 0; K < 3; ++K) s += iJt[J + 3 * K] * p.dNt[n + nn * (K + 3 * q)];
          W[n + nn * J] = s;
        }
      point_F(p, xl, q, iJt, F);
      law_tangent(p, F, T);
      for (int n = 0; n < nn; ++n)
        for (int jj = 0; jj < 3; ++jj) Bb[(ql * 3 + jj) + (size_t)qb * 3 * n] = W[n + nn * jj];
      const double* __restrict__ W0 = W.data();
      const double* __restrict__ W1 = W0 + nn;
      const double* __restrict__ W2 = W0 + 2 * nn;
      for (int c = 0; c < 3; ++c)
        for (int k = 0; k < 3; ++k)
          for (int jj = 0; jj < 3; ++jj) {
            const double z0 = dV * T[(c * 3 + jj) + 9 * (k * 3 + 0)];
            const double z1 = dV * T[(c * 3 + jj) + 9 * (k * 3 + 1)];
            const double z2 = dV * T[(c * 3 + jj) + 9 * (k * 3 + 2)];
            double* __restrict__ g = &Gb[(size_t)nn * ((ql * 3 + jj) + (size_t)qb * 3 * (k + 3 * c))];
            for (int m = 0; m < nn; ++m) g[m] = z0 * W0[m] + z1 * W1[m] + z2 * W2[m];
          }
    }
    const int R = nq * 3;
    for (int c = 0; c < 3; ++c)
      for (int k = 0; k < 3; ++k)
        if (getenv("SKIPG")==nullptr) gemm_add(&KeT[(size_t)k * nn + (size_t)ndl * c * nn], ndl, &Gb[(size_t)nn * qb * 3 * (k + 3 * c)], nn,
                 Bb.data(), qb * 3, nn, nn, R);
  }
}

// ---- tensor-product kernels (src/tensorproduct.jl) -------------------------------------------
void tp_interpolate(const Problem& p, const double* u, double* out /* np x 4 */, double* tmp) {
  const int Q = p.Q, P = p.P;
  const double* N1 = p.N1.data();
  const double* dN1 = p.dN1.data();
  const int ld = 2 * P * P;  // tmp rows
  auto T = [&](int r, int c) -> double& { return tmp[r + (size_t)ld * c]; };
  for (int k = 0; k < Q; ++k)
    for (int j = 0; j < Q; ++j)
      for (int a = 0; a < P; ++a) {
        double s = 0, ds = 0;
        for (int i = 0; i < Q; ++i) {
          double v = u[i + Q * j + Q * Q * k];
          s += N1[a + P * i] * v;
          ds += dN1[a + P * i] * v;
        }
        int c = j + k * Q;
        T(a, c) = s;
        T(a + P, c) = ds;
      }
  const int o2 = 2 * Q * Q;
  for (int k = 0; k < Q; ++k)
    for (int b = 0; b < P; ++b)
      for (int a = 0; a < P; ++a) {
        double v = 0, g1 = 0, g2 = 0;
        for (int j = 0; j < Q; ++j) {
          int c = j + k * Q;
          v += N1[b + P * j] * T(a, c);
          g1 += N1[b + P * j] * T(a + P, c);
          g2 += dN1[b + P * j] * T(a, c);
        }
        int r = a + b * P;
        T(r, o2 + k) = v;
        T(r, o2 + Q + k) = g1;
        T(r, o2 + 2 * Q + k) = g2;
      }
  for (int c = 0; c < P; ++c)
    for (int b = 0; b < P; ++b)
      for (int a = 0; a < P; ++a) {
        int r = a + b * P;
        double v = 0, g1 = 0, g2 = 0, g3 = 0;
        for (int k = 0; k < Q; ++k) {
          v += N1[c + P * k] * T(r, o2 + k);
          g1 += N1[c + P * k] * T(r, o2 + Q + k);
          g2 += N1[c + P * k] * T(r, o2 + 2 * Q + k);
          g3 += dN1[c + P * k] * T(r, o2 + k);
        }
        int pl = r + c * P * P;
        out[pl * 4 + 0] = v;
        out[pl * 4 + 1] = g1;
        out[pl * 4 + 2] = g2;
        out[pl * 4 + 3] = g3;
      }
}

void tp_contract(const Problem& p, const double* coef /* np x 4 */, double* r, double* tmp) {
  const int Q = p.Q, P = p.P;
  const double* N1 = p.N1.data();
  const double* dN1 = p.dN1.data();
  const int ld = 2 * P * P;
  auto T = [&](int rr, int c) -> double& { return tmp[rr + (size_t)ld * c]; };
  const int o2 = 2 * Q * Q;
  for (int k = 0; k < Q; ++k)
    for (int b = 0; b < P; ++b)
      for (int a = 0; a < P; ++a) {
        int r2 = a + b * P;
        double t0 = 0, t1 = 0, t2 = 0;
        for (int c = 0; c < P; ++c) {
          int pl = r2 + c * P * P;
          t0 += N1[c + P * k] * coef[pl * 4 + 0] + dN1[c + P * k] * coef[pl * 4 + 3];
          t1 += N1[c + P * k] * coef[pl * 4 + 1];
          t2 += N1[c + P * k] * coef[pl * 4 + 2];
        }
        T(r2, o2 + k) = t0;
        T(r2, o2 + Q + k) = t1;
        T(r2, o2 + 2 * Q + k) = t2;
      }
  for (int k = 0; k < Q; ++k)
    for (int j = 0; j < Q; ++j)
      for (int a = 0; a < P; ++a) {
        double s0 = 0, s1 = 0;
        for (int b = 0; b < P; ++b) {
          int r2 = a + b * P;
          s0 += N1[b + P * j] * T(r2, o2 + k) + dN1[b + P * j] * T(r2, o2 + 2 * Q + k);
          s1 += N1[b + P * j] * T(r2, o2 + Q + k);
        }
        int c = j + k * Q;
        T(a, c) = s0;
        T(a + P, c) = s1;
      }
  for (int k = 0; k < Q; ++k)
    for (int j = 0; j < Q; ++j)
      for (int i = 0; i < Q; ++i) {
        int c = j + k * Q;
        double s = 0;
        for (int a = 0; a < P; ++a) s += N1[a + P * i] * T(a, c) + dN1[a + P * i] * T(a + P, c);
        r[i + Q * j + Q * Q * k] = s;
      }
}

void lagrange1d(int Q, double xi, double* N, double* dN) {
  std::vector<double> xs(Q);
  if (Q == 1) xs[0] = 0.5;
  else
    for (int i = 0; i < Q; ++i) xs[i] = double(i) / (Q - 1);
  for (int i = 0; i < Q; ++i) {
    double v = 1;
    for (int j = 0; j < Q; ++j)
      if (j != i) v *= (xi - xs[j]) / (xs[i] - xs[j]);
    N[i] = v;
    double d = 0;
    for (int m = 0; m < Q; ++m) {
      if (m == i) continue;
      double t = 1.0 / (xs[i] - xs[m]);
      for (int j = 0; j < Q; ++j)
        if (j != i && j != m) t *= (xi - xs[j]) / (xs[i] - xs[j]);
      d += t;
    }
    dN[i] = d;
  }
}

// TPTable (src/tensorproduct.jl:55-91): 1D tables and permutations found numerically
bool build_tp(Problem& p) {
  int Q = (int)std::lround(std::cbrt((double)p.nn));
  int P = (int)std::lround(std::cbrt((double)p.np));
  if (Q * Q * Q != p.nn || P * P * P != p.np) return false;
  std::vector<double> xs;
  for (int q = 0; q < p.np; ++q) xs.push_back(std::round(p.xq[3 * q] * 1e12) / 1e12);
  std::sort(xs.begin(), xs.end());
  xs.erase(std::unique(xs.begin(), xs.end()), xs.end());
  if ((int)xs.size() != P) return false;
  p.Q = Q;
  p.P = P;
  p.N1.assign(P * Q, 0);
  p.dN1.assign(P * Q, 0);
  std::vector<double> n1(Q), dn1(Q);
  for (int a = 0; a < P; ++a) {
    // evaluated at the unrounded coordinate (the reference evaluates at the 12-digit-rounded one,
    // src/tensorproduct.jl:64-71, a ~1e-12 perturbation of the sum-factorised path)
    double xa = xs[a];
    for (int q = 0; q < p.np; ++q)
      if (std::round(p.xq[3 * q] * 1e12) / 1e12 == xs[a]) {
        xa = p.xq[3 * q];
        break;
      }
    lagrange1d(Q, xa, n1.data(), dn1.data());
    for (int i = 0; i < Q; ++i) {
      p.N1[a + P * i] = n1[i];
      p.dN1[a + P * i] = dn1[i];
    }
  }
  p.pointperm.assign(p.np, -1);
  for (int lin = 0; lin < p.np; ++lin) {
    int t[3] = {lin % P, (lin / P) % P, lin / (P * P)};
    for (int q = 0; q < p.np; ++q) {
      bool ok = true;
      for (int d = 0; d < 3; ++d) ok &= std::fabs(p.xq[d + 3 * q] - xs[t[d]]) <= 1e-10;
      if (ok) {
        p.pointperm[lin] = q;
        break;
      }
    }
    if (p.pointperm[lin] < 0) return false;
  }
  p.nodeperm.assign(p.nn, -1);
  std::vector<char> used(p.nn, 0);
  for (int lin = 0; lin < p.nn; ++lin) {
    int ii[3] = {lin % Q, (lin / Q) % Q, lin / (Q * Q)};
    for (int n = 0; n < p.nn; ++n) {
      if (used[n]) continue;
      bool ok = true;
      for (int pl = 0; pl < p.np && ok; ++pl) {
        int aa[3] = {pl % P, (pl / P) % P, pl / (P * P)};
        double v = 1;
        for (int d = 0; d < 3; ++d) v *= p.N1[aa[d] + P * ii[d]];
        ok = std::fabs(p.Nt[n + p.nn * p.pointperm[pl]] - v) <= 1e-7;
      }
      if (ok) {
        used[n] = 1;
        p.nodeperm[lin] = n;
        break;
      }
    }
    if (p.nodeperm[lin] < 0) return false;
  }
  return true;
}

}  // namespace

extern "C" {

void* o_create(int ncells, int nn, int np, int ng, const double* xq, const double* w, const double* Nt,
               const double* dNt, const double* dMt, const double* coords, const int32_t* ids, int64_t nfree,
               int64_t ndir, int law, const double* params, int nparams) {
  auto* p = new Problem();
  p->ncells = ncells;
  p->nn = nn;
  p->np = np;
  p->ng = ng;
  p->ndl = 3 * nn;
  p->nfree = nfree;
  p->ndir = ndir;
  p->xq.assign(xq, xq + 3 * np);
  p->w.assign(w, w + np);
  p->Nt.assign(Nt, Nt + (size_t)nn * np);
  p->dNt.assign(dNt, dNt + (size_t)nn * 3 * np);
  p->dMt.assign(dMt, dMt + (size_t)ng * 3 * np);
  p->coords.assign(coords, coords + (size_t)3 * ng * ncells);
  p->ids.assign(ids, ids + (size_t)p->ndl * ncells);
  p->law = law;
  p->lam = nparams > 0 ? params[0] : 0;
  p->mu = nparams > 1 ? params[1] : 0;
  for (int c = 0; c < 3; ++c) p->body[c] = nparams > 2 + c ? params[2 + c] : 0;
  compute_affine(*p);
  build_tp(*p);
  return p;
}

void o_free(void* h) { delete (Problem*)h; }

int o_has_tp(void* h) { return ((Problem*)h)->Q > 0; }
int o_affine_count(void* h) {
  auto& p = *(Problem*)h;
  int s = 0;
  for (auto a : p.affine) s += a;
  return s;
}
void o_set_params(void* h, const double* params, int nparams) {
  auto& p = *(Problem*)h;
  p.lam = nparams > 0 ? params[0] : 0;
  p.mu = nparams > 1 ? params[1] : 0;
  for (int c = 0; c < 3; ++c) p.body[c] = nparams > 2 + c ? params[2 + c] : 0;
}

// color_cells (src/coloring.jl:4-28): greedy first fit over cells, 128-bit masks of free test rows
int o_color(void* h, int32_t* color_out) {
  auto& p = *(Problem*)h;
  std::vector<unsigned __int128> masks(p.nfree + 1, 0);
  std::vector<int> color(p.ncells);
  int ncol = 0;
  for (int cell = 0; cell < p.ncells; ++cell) {
    unsigned __int128 used = 0;
    const int32_t* id = &p.ids[(size_t)cell * p.ndl];
    for (int j = 0; j < p.ndl; ++j)
      if (id[j] > 0) used |= masks[id[j]];
    int c = 0;
    while (c < 128 && ((used >> c) & 1)) ++c;  // trailing_ones
    if (c >= 128) return -1;
    color[cell] = c;
    unsigned __int128 bit = (unsigned __int128)1 << c;
    for (int j = 0; j < p.ndl; ++j)
      if (id[j] > 0) masks[id[j]] |= bit;
    ncol = std::max(ncol, c + 1);
  }
  p.colors.assign(ncol, {});
  for (int cell = 0; cell < p.ncells; ++cell) p.colors[color[cell]].push_back(cell);
  for (int cell = 0; cell < p.ncells; ++cell) color_out[cell] = color[cell] + 1;
  return ncol;
}

// sparsity (src/assembly.jl:773-818) with full_keys! and cell_positions! (:864-880)
int64_t o_pattern(void* h) {
  auto& p = *(Problem*)h;
  std::vector<uint64_t> keys;
  keys.reserve((size_t)p.ncells * p.ndl * p.ndl);
  for (int cell = 0; cell < p.ncells; ++cell) {
    const int32_t* id = &p.ids[(size_t)cell * p.ndl];
    for (int jj = 0; jj < p.ndl; ++jj) {
      int32_t c = id[jj];
      if (c <= 0) continue;
      for (int ii = 0; ii < p.ndl; ++ii) {
        int32_t r = id[ii];
        if (r > 0) keys.push_back(((uint64_t)c << 32) | (uint64_t)r);
      }
    }
  }
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  p.colptr.assign(p.nfree + 1, 0);
  p.rowval.resize(keys.size());
  std::vector<int64_t> cnt(p.nfree + 1, 0);
  for (size_t k = 0; k < keys.size(); ++k) {
    cnt[keys[k] >> 32] += 1;
    p.rowval[k] = (int64_t)(keys[k] & 0xffffffffu);
  }
  p.colptr[0] = 1;
  for (int64_t c = 1; c <= p.nfree; ++c) p.colptr[c] = p.colptr[c - 1] + cnt[c];
  p.nzpos.assign((size_t)p.ndl * p.ndl * p.ncells, 0);
#pragma omp parallel for schedule(static)
  for (int cell = 0; cell < p.ncells; ++cell) {
    const int32_t* id = &p.ids[(size_t)cell * p.ndl];
    for (int jj = 0; jj < p.ndl; ++jj) {
      int32_t c = id[jj];
      if (c <= 0) continue;
      int64_t lo = p.colptr[c - 1] - 1, hi = p.colptr[c] - 1;  // 0-based [lo, hi)
      for (int ii = 0; ii < p.ndl; ++ii) {
        int32_t r = id[ii];
        if (r <= 0) continue;
        auto it = std::lower_bound(p.rowval.begin() + lo, p.rowval.begin() + hi, (int64_t)r);
        p.nzpos[ii + (size_t)jj * p.ndl + (size_t)p.ndl * p.ndl * cell] = (int32_t)(it - p.rowval.begin()) + 1;
      }
    }
  }
  return (int64_t)keys.size();
}

void o_pattern_get(void* h, int64_t* colptr, int64_t* rowval, int32_t* nzpos) {
  auto& p = *(Problem*)h;
  if (colptr) std::memcpy(colptr, p.colptr.data(), sizeof(int64_t) * p.colptr.size());
  if (rowval) std::memcpy(rowval, p.rowval.data(), sizeof(int64_t) * p.rowval.size());
  if (nzpos) std::memcpy(nzpos, p.nzpos.data(), sizeof(int32_t) * p.nzpos.size());
}

void o_element_residual(void* h, const double* x, const double* dvals, int cell, double* re) {
  auto& p = *(Problem*)h;
  std::vector<double> xl(p.ndl), C;
  gather_cell(p, x, dvals, cell, xl.data());
  element_residual(p, xl.data(), cell, re, C);
}

void o_element_jacobian(void* h, const double* x, const double* dvals, int cell, int point_block, double* KeT) {
  auto& p = *(Problem*)h;
  std::vector<double> xl(p.ndl), W, Bb, Gb;
  gather_cell(p, x, dvals, cell, xl.data());
  element_jacobian(p, xl.data(), cell, KeT, point_block, W, Bb, Gb);
}

// residual! (src/assembly.jl:909-916) through run_cells!/cells! (:1413-1505): colour by colour,
// cells of a colour in parallel, scatter_residual! (:1390-1399)
void o_residual(void* h, const double* x, const double* dvals, double* b, int nthreads) {
  auto& p = *(Problem*)h;
  std::fill(b, b + p.nfree, 0.0);
  int nt = nthreads_or(nthreads);
  for (auto& color : p.colors) {
#pragma omp parallel num_threads(nt)
    {
      std::vector<double> xl(p.ndl), re(p.ndl), C;
#pragma omp for schedule(dynamic, 4)
      for (size_t i = 0; i < color.size(); ++i) {
        int cell = color[i];
        gather_cell(p, x, dvals, cell, xl.data());
        element_residual(p, xl.data(), cell, re.data(), C);
        const int32_t* id = &p.ids[(size_t)cell * p.ndl];
        for (int j = 0; j < p.ndl; ++j)
          if (id[j] > 0) b[id[j] - 1] += re[j];
      }
    }
  }
}

// jacobian! (src/assembly.jl:918-927): zero-fill, colour loop, scatter_jacobian! (:1402-1408)
void o_jacobian(void* h, const double* x, const double* dvals, double* nzval, int nthreads, int point_block) {
  auto& p = *(Problem*)h;
  std::fill(nzval, nzval + p.rowval.size(), 0.0);
  int nt = nthreads_or(nthreads);
  const int ndl = p.ndl;
  for (auto& color : p.colors) {
#pragma omp parallel num_threads(nt)
    {
      std::vector<double> xl(ndl), KeT((size_t)ndl * ndl), W, Bb, Gb;
#pragma omp for schedule(dynamic, 1)
      for (size_t i = 0; i < color.size(); ++i) {
        int cell = color[i];
        gather_cell(p, x, dvals, cell, xl.data());
        element_jacobian(p, xl.data(), cell, KeT.data(), point_block, W, Bb, Gb);
        const int32_t* pos = &p.nzpos[(size_t)ndl * ndl * cell];
        for (int jj = 0; jj < ndl; ++jj)
          for (int ii = 0; ii < ndl; ++ii) {
            int32_t ps = pos[ii + ndl * jj];
            if (ps > 0) nzval[ps - 1] += KeT[jj + (size_t)ndl * ii];
          }
      }
    }
  }
}

// prepare! / prepare_cells! (src/matrixfree.jl:140-228): T, iJt, dV per point
void o_mf_prepare(void* h, const double* x, const double* dvals, int nthreads) {
  auto& p = *(Problem*)h;
  p.T.assign((size_t)81 * p.np * p.ncells, 0.0);
  p.iJt.assign((size_t)9 * p.np * p.ncells, 0.0);
  p.dV.assign((size_t)p.np * p.ncells, 0.0);
  int nt = nthreads_or(nthreads);
#pragma omp parallel num_threads(nt)
  {
    std::vector<double> xl(p.ndl);
#pragma omp for schedule(static)
    for (int cell = 0; cell < p.ncells; ++cell) {
      gather_cell(p, x, dvals, cell, xl.data());
      for (int q = 0; q < p.np; ++q) {
        double dV, iJt[9], F[9];
        point_geometry(p, q, cell, dV, iJt);
        point_F(p, xl.data(), q, iJt, F);
        size_t pq = (size_t)q + (size_t)p.np * cell;
        law_tangent(p, F, &p.T[81 * pq]);
        std::memcpy(&p.iJt[9 * pq], iJt, sizeof iJt);
        p.dV[pq] = dV;
      }
    }
  }
}

void o_mf_get(void* h, double* T, double* iJt, double* dV) {
  auto& p = *(Problem*)h;
  if (T) std::memcpy(T, p.T.data(), sizeof(double) * p.T.size());
  if (iJt) std::memcpy(iJt, p.iJt.data(), sizeof(double) * p.iJt.size());
  if (dV) std::memcpy(dV, p.dV.data(), sizeof(double) * p.dV.size());
}

// mul! / apply_cells! with interpolate_slots!/contract_slots! on the tensor-product path
// (src/matrixfree.jl:246-260, :341-424, :496-520)
int o_mf_apply(void* h, const double* dx, double* y, int nthreads) {
  auto& p = *(Problem*)h;
  if (p.Q == 0 || p.T.empty()) return -1;
  std::fill(y, y + p.nfree, 0.0);
  int nt = nthreads_or(nthreads);
  const int nn = p.nn, np = p.np, ndl = p.ndl, Q = p.Q, P = p.P;
  for (auto& color : p.colors) {
#pragma omp parallel num_threads(nt)
    {
      std::vector<double> xl(ndl), re(ndl), uc(nn), pts(4 * (size_t)np), su(9 * (size_t)np), sv(9 * (size_t)np),
          coef(4 * (size_t)np), rc(nn), tmp((size_t)2 * P * P * (2 * Q * Q + 3 * Q));
#pragma omp for schedule(dynamic, 4)
      for (size_t ci = 0; ci < color.size(); ++ci) {
        int cell = color[ci];
        const int32_t* id = &p.ids[(size_t)cell * ndl];
        for (int j = 0; j < ndl; ++j) xl[j] = id[j] > 0 ? dx[id[j] - 1] : 0.0;
        for (int c = 0; c < 3; ++c) {
          for (int n = 0; n < nn; ++n) uc[n] = xl[c * nn + p.nodeperm[n]];
          tp_interpolate(p, uc.data(), pts.data(), tmp.data());
          for (int pl = 0; pl < np; ++pl) {
            int q = p.pointperm[pl];
            const double* iJ = &p.iJt[9 * ((size_t)q + (size_t)np * cell)];
            for (int J = 0; J < 3; ++J) {
              double s = 0;
              for (int K = 0; K < 3; ++K) s += iJ[J + 3 * K] * pts[pl * 4 + 1 + K];
              su[(c * 3 + J) + 9 * q] = s;
            }
          }
        }
        for (int q = 0; q < np; ++q) {
          const double* Tq = &p.T[81 * ((size_t)q + (size_t)np * cell)];
          double dVq = p.dV[(size_t)q + (size_t)np * cell];
          for (int i = 0; i < 9; ++i) {
            double s = 0;
            for (int j = 0; j < 9; ++j) s += Tq[i + 9 * j] * su[j + 9 * q];
            sv[i + 9 * q] = s * dVq;
          }
        }
        std::fill(re.begin(), re.end(), 0.0);
        for (int c = 0; c < 3; ++c) {
          for (int pl = 0; pl < np; ++pl) {
            int q = p.pointperm[pl];
            const double* iJ = &p.iJt[9 * ((size_t)q + (size_t)np * cell)];
            coef[pl * 4 + 0] = 0.0;
            for (int K = 0; K < 3; ++K) {
              double s = 0;
              for (int J = 0; J < 3; ++J) s += sv[(c * 3 + J) + 9 * q] * iJ[J + 3 * K];
              coef[pl * 4 + 1 + K] = s;
            }
          }
          tp_contract(p, coef.data(), rc.data(), tmp.data());
          for (int n = 0; n < nn; ++n) re[c * nn + p.nodeperm[n]] += rc[n];
        }
        for (int j = 0; j < ndl; ++j)
          if (id[j] > 0) y[id[j] - 1] += re[j];
      }
    }
  }
  return 0;
}

// BlockJacobi: field_blocks (src/preconditioners.jl:151-173), blocks_from_tangents!
// (:250-280), _invert_blocks! (:312-327); returns the number of blocks
int o_blocks(void* h, int nthreads) {
  auto& p = *(Problem*)h;
  if (p.T.empty()) return -1;
  (void)nthreads;
  const int nn = p.nn;
  if (p.block_of.empty()) {
    p.block_of.assign((size_t)nn * p.ncells, 0);
    std::map<std::array<int32_t, 3>, int32_t> keys;
    p.bdofs.clear();
    for (int cell = 0; cell < p.ncells; ++cell)
      for (int n = 0; n < nn; ++n) {
        std::array<int32_t, 3> key;
        bool anyfree = false;
        for (int c = 0; c < 3; ++c) {
          key[c] = p.ids[(size_t)cell * p.ndl + c * nn + n];
          anyfree |= key[c] > 0;
        }
        if (!anyfree) continue;
        auto it = keys.find(key);
        int32_t blk;
        if (it == keys.end()) {
          for (int c = 0; c < 3; ++c) p.bdofs.push_back(key[c] > 0 ? key[c] : 0);
          blk = (int32_t)keys.size() + 1;
          keys.emplace(key, blk);
        } else {
          blk = it->second;
        }
        p.block_of[n + (size_t)nn * cell] = blk;
      }
    p.nblocks = (int)keys.size();
  }
  p.B.assign(9 * (size_t)p.nblocks, 0.0);
  p.Binv.assign(9 * (size_t)p.nblocks, 0.0);
  std::vector<double> W((size_t)nn * 3);
  for (auto& color : p.colors)
    for (int cell : color)
      for (int q = 0; q < p.np; ++q) {
        size_t pq = (size_t)q + (size_t)p.np * cell;
        const double* iJ = &p.iJt[9 * pq];
        const double* Tq = &p.T[81 * pq];
        for (int J = 0; J < 3; ++J)
          for (int n = 0; n < nn; ++n) {
            double s = 0;
            for (int K = 0; K < 3; ++K) s += iJ[J + 3 * K] * p.dNt[n + nn * (K + 3 * q)];
            W[n + nn * J] = s;
          }
        double dVq = p.dV[pq];
        for (int n = 0; n < nn; ++n) {
          int blk = p.block_of[n + (size_t)nn * cell];
          if (blk == 0) continue;
          for (int cj = 0; cj < 3; ++cj)
            for (int ci = 0; ci < 3; ++ci) {
              double s = 0;
              for (int b = 0; b < 3; ++b) {
                double wu = W[n + nn * b];
                for (int a = 0; a < 3; ++a) s += W[n + nn * a] * Tq[(ci * 3 + a) + 9 * (cj * 3 + b)] * wu;
              }
              p.B[ci + 3 * cj + 9 * (size_t)(blk - 1)] += dVq * s;
            }
        }
      }
  for (int blk = 0; blk < p.nblocks; ++blk) {
    double M[9];
    bool fin = true;
    for (int j = 0; j < 3; ++j)
      for (int i = 0; i < 3; ++i) {
        bool fixed = p.bdofs[i + 3 * blk] == 0 || p.bdofs[j + 3 * blk] == 0;
        M[i + 3 * j] = fixed ? (i == j ? 1.0 : 0.0) : p.B[i + 3 * j + 9 * (size_t)blk];
        fin &= std::isfinite(M[i + 3 * j]);
      }
    if (fin) inv3(M, &p.Binv[9 * (size_t)blk]);
    else std::memcpy(&p.Binv[9 * (size_t)blk], M, sizeof M);
  }
  return p.nblocks;
}

void o_blocks_get(void* h, int32_t* dofs, double* B, double* Binv) {
  auto& p = *(Problem*)h;
  if (dofs) std::memcpy(dofs, p.bdofs.data(), sizeof(int32_t) * p.bdofs.size());
  if (B) std::memcpy(B, p.B.data(), sizeof(double) * p.B.size());
  if (Binv) std::memcpy(Binv, p.Binv.data(), sizeof(double) * p.Binv.size());
}

// ldiv!(y, BlockJacobiState, r) (src/preconditioners.jl:329-344); rows of Dirichlet components untouched
void o_blocks_apply(void* h, const double* r, double* y) {
  auto& p = *(Problem*)h;
#pragma omp parallel for schedule(static)
  for (int blk = 0; blk < p.nblocks; ++blk)
    for (int i = 0; i < 3; ++i) {
      int id = p.bdofs[i + 3 * blk];
      if (id == 0) continue;
      double s = 0;
      for (int j = 0; j < 3; ++j) {
        int jd = p.bdofs[j + 3 * blk];
        if (jd != 0) s += p.Binv[i + 3 * j + 9 * (size_t)blk] * r[jd - 1];
      }
      y[id - 1] = s;
    }
}

void o_point_law(int law, const double* params, const double* F, double* Pout, double* T) {
  Problem p;
  p.law = law;
  p.lam = params[0];
  p.mu = params[1];
  if (Pout) law_stress(p, F, Pout);
  if (T) law_tangent(p, F, T);
}

// ---- transfers (src/transfers.jl) ------------------------------------------------------------
struct Transfer {
  int ncells, NF, NC;
  int64_t nf, nc;
  std::vector<double> E, Einj;  // NF x NC, NC x NF (column-major)
  std::vector<int32_t> ids_f, ids_c;
  std::vector<int32_t> mult;
};

void* o_transfer_create(int ncells, int NF, int NC, const double* E, const double* Einj, const int32_t* ids_f,
                        const int32_t* ids_c, int64_t nf, int64_t nc) {
  auto* t = new Transfer();
  t->ncells = ncells;
  t->NF = NF;
  t->NC = NC;
  t->nf = nf;
  t->nc = nc;
  t->E.assign(E, E + (size_t)NF * NC);
  t->Einj.assign(Einj, Einj + (size_t)NF * NC);
  t->ids_f.assign(ids_f, ids_f + (size_t)3 * NF * ncells);
  t->ids_c.assign(ids_c, ids_c + (size_t)3 * NC * ncells);
  t->mult.assign(nf, 0);
  for (size_t k = 0; k < t->ids_f.size(); ++k)
    if (t->ids_f[k] > 0) t->mult[t->ids_f[k] - 1] += 1;
  return t;
}
void o_transfer_free(void* h) { delete (Transfer*)h; }

// prolongate! (src/transfers.jl:238-245, prolongate_cells! :179-193): insertion of E xl
void o_prolongate(void* h, const double* xc, double* yf) {
  auto& t = *(Transfer*)h;
  std::fill(yf, yf + t.nf, 0.0);
  std::vector<double> xl(3 * t.NC), yl(3 * t.NF);
  for (int cell = 0; cell < t.ncells; ++cell) {
    const int32_t* ic = &t.ids_c[(size_t)3 * t.NC * cell];
    const int32_t* iff = &t.ids_f[(size_t)3 * t.NF * cell];
    for (int j = 0; j < 3 * t.NC; ++j) xl[j] = ic[j] > 0 ? xc[ic[j] - 1] : 0.0;
    for (int comp = 0; comp < 3; ++comp)
      for (int f = 0; f < t.NF; ++f) {
        double s = 0;
        for (int c = 0; c < t.NC; ++c) s += t.E[f + (size_t)t.NF * c] * xl[comp * t.NC + c];
        yl[comp * t.NF + f] = s;
      }
    for (int j = 0; j < 3 * t.NF; ++j)
      if (iff[j] > 0) yf[iff[j] - 1] = yl[j];
  }
}

// restrict! (src/transfers.jl:252-259, restrict_cells! :195-213): E^T of yf / multiplicity, scatter-add
void o_restrict(void* h, const double* yf, double* yc) {
  auto& t = *(Transfer*)h;
  std::fill(yc, yc + t.nc, 0.0);
  std::vector<double> xl(3 * t.NC), yl(3 * t.NF);
  for (int cell = 0; cell < t.ncells; ++cell) {
    const int32_t* ic = &t.ids_c[(size_t)3 * t.NC * cell];
    const int32_t* iff = &t.ids_f[(size_t)3 * t.NF * cell];
    for (int j = 0; j < 3 * t.NF; ++j) yl[j] = iff[j] > 0 ? yf[iff[j] - 1] / t.mult[iff[j] - 1] : 0.0;
    for (int comp = 0; comp < 3; ++comp)
      for (int c = 0; c < t.NC; ++c) {
        double s = 0;
        for (int f = 0; f < t.NF; ++f) s += t.E[f + (size_t)t.NF * c] * yl[comp * t.NF + f];
        xl[comp * t.NC + c] = s;
      }
    for (int j = 0; j < 3 * t.NC; ++j)
      if (ic[j] > 0) yc[ic[j] - 1] += xl[j];
  }
}

// inject! (src/transfers.jl:285-313)
void o_inject(void* h, const double* xf, const double* df, double* xc, double* dc) {
  auto& t = *(Transfer*)h;
  for (int cell = 0; cell < t.ncells; ++cell) {
    const int32_t* ic = &t.ids_c[(size_t)3 * t.NC * cell];
    const int32_t* iff = &t.ids_f[(size_t)3 * t.NF * cell];
    for (int comp = 0; comp < 3; ++comp)
      for (int c = 0; c < t.NC; ++c) {
        double v = 0;
        for (int f = 0; f < t.NF; ++f) {
          double w = t.Einj[c + (size_t)t.NC * f];
          if (w == 0.0) continue;
          int32_t idf = iff[comp * t.NF + f];
          v += w * (idf > 0 ? xf[idf - 1] : df[-idf - 1]);
        }
        int32_t idc = ic[comp * t.NC + c];
        if (idc > 0) xc[idc - 1] = v;
        else if (idc < 0) dc[-idc - 1] = v;
      }
  }
}

// KernelFunctional (src/functionals.jl:10-27) for the recognised laws: kind 0 = the stored energy
// Σ_cells Σ_q Ψ(F) dV (reduce = :sum; SVK Ψ = μ E:E + λ/2 (tr E)², linear elasticity
// Ψ = μ ε:ε + λ/2 (tr ε)²), kind 1 = min over the points of det F (reduce = :min, unweighted)
double o_functional(void* h, const double* x, const double* dvals, int kind) {
  auto& p = *(Problem*)h;
  double total = kind == 0 ? 0.0 : INFINITY;
  std::vector<double> xl(p.ndl);
  for (int cell = 0; cell < p.ncells; ++cell) {
    gather_cell(p, x, dvals, cell, xl.data());
    for (int q = 0; q < p.np; ++q) {
      double dV, iJt[9], F[9];
      point_geometry(p, q, cell, dV, iJt);
      point_F(p, xl.data(), q, iJt, F);
      if (kind == 1) {
        const double d = F[0] * (F[4] * F[8] - F[7] * F[5]) - F[3] * (F[1] * F[8] - F[7] * F[2]) +
                         F[6] * (F[1] * F[5] - F[4] * F[2]);
        total = std::min(total, d);
        continue;
      }
      double E[9];
      for (int I = 0; I < 3; ++I)
        for (int J = 0; J < 3; ++J) {
          if (p.law == 2) {
            E[I + 3 * J] = 0.5 * (F[I + 3 * J] + F[J + 3 * I]) - (I == J ? 1.0 : 0.0);
          } else {
            double s = 0;
            for (int a = 0; a < 3; ++a) s += F[a + 3 * I] * F[a + 3 * J];
            E[I + 3 * J] = 0.5 * (s - (I == J ? 1.0 : 0.0));
          }
        }
      double ee = 0;
      for (int i = 0; i < 9; ++i) ee += E[i] * E[i];
      const double tr = E[0] + E[4] + E[8];
      total += dV * (p.mu * ee + 0.5 * p.lam * tr * tr);
    }
  }
  return total;
}

int o_max_threads() { return nthreads_or(0); }

}  // extern "C"
