// Sum-factorised cell kernels: residual, matrix-free Jacobian product (tangent recomputed from the
// state, or read from stored per-point tangents) for a 3-component Lagrangian field on hexahedra.
//
// Mapping: a warp holds CPW = 32 / M^2 cells (M = max(P, Q)); the M^2 lanes of a cell own the
// tensor lines of each sum-factorisation sweep (x lines (j,k), then y lines (a,k), then z lines
// (a,b)), so every sweep reads each input once and writes P (or 3P) outputs from registers. Lane
// (a,b) then owns the P points (a,b,c) for the pointwise law. Cells of one colour share no free
// dof, so the scatter is a plain read-modify-write (colour-by-colour launches), or an atomicAdd
// when one launch covers all cells.
//
// Reference: tp_interpolate!/tp_contract! (src/tensorproduct.jl:125-224), apply_cells!
// (src/matrixfree.jl:341-396), element_residual_mm! (src/assembly.jl:1219-1241); the tangent of
// SVK is the exact derivative the factorised form evaluates (src/factorforms.jl:316-322).
#pragma once
#include "hfk_internal.h"
#include "pointwise.cuh"

namespace hfk {

enum CellMode { MODE_RESIDUAL = 0, MODE_JV = 1, MODE_JV_STORED = 2 };

template <int Q, int P>
struct TPShape {
  static constexpr int NN = Q * Q * Q;
  static constexpr int NP = P * P * P;
  static constexpr int M = P > Q ? P : Q;
  static constexpr int TPC = M * M;        // lanes per cell
  static constexpr int CPW = 32 / TPC;     // cells per warp
  static_assert(CPW >= 1, "a cell must fit in a warp (max(P,Q) <= 5)");
};

// shared-memory layout of one cell (in units of R), see the phase comments in the kernel
template <int Q, int P, int MODE>
struct CellSmem {
  using S = TPShape<Q, P>;
  static constexpr int NF = MODE == MODE_JV ? 6 : 3;            // gathered fields
  static constexpr int XL = NF * S::NN;                          // local values
  static constexpr int XR = (6 * P * Q * Q > 12 * S::NP - XL ? 6 * P * Q * Q : 12 * S::NP - XL);  // x-sweep / y-contraction
  static constexpr int YR0 = NF * 3 * Q * P * P;
  static constexpr int YR = YR0 > 9 * Q * P * P ? YR0 : 9 * Q * P * P;                      // y-sweep / z-contraction
  static constexpr int VALS = XL + XR + YR;                      // R elements
};

// bytes of one cell's shared region, rounded up to 16 so that every region starts aligned
template <int Q, int P, int MODE, typename R>
__host__ __device__ constexpr size_t cell_region_bytes() {
  return (((size_t)CellSmem<Q, P, MODE>::VALS * sizeof(R) + (size_t)3 * TPShape<Q, P>::NN * sizeof(int32_t)) + 15) /
         16 * 16;
}

template <typename R>
struct CellIO {
  const R* u;       // state free values (MODE_RESIDUAL, MODE_JV)
  const R* dvals;   // state Dirichlet values
  const R* dx;      // increment (MODE_JV, MODE_JV_STORED)
  R* y;             // output (scatter-add)
  const double* T;  // stored tangents (cell*81 + i)*NP + q
  const double* iJtq;
  const double* dVq;
  int atomic;       // 1: atomicAdd scatter (all cells in one launch)
};

template <int Q, int P, int MODE, typename R>
__global__ void __launch_bounds__(128) cell_kernel(CellData cd, Tab1D<R> tab, CellIO<R> io) {
  using S = TPShape<Q, P>;
  using L = CellSmem<Q, P, MODE>;
  constexpr int NN = S::NN, NP = S::NP, TPC = S::TPC, CPW = S::CPW;
  constexpr int NDL = 3 * NN;
  constexpr int NF = L::NF;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  const int slot = lane / TPC;        // cell slot in the warp
  const bool active = slot < CPW;     // lanes past CPW * TPC idle (every phase is guarded by t)
  const int t = active ? lane - slot * TPC : (1 << 20);  // lane within the cell
  // per-cell regions
  const int cell_index_base = (blockIdx.x * nwarps + warp) * CPW;
  const size_t per_cell_bytes = cell_region_bytes<Q, P, MODE, R>();
  unsigned char* base = smem_raw + (size_t)(warp * CPW + (active ? slot : 0)) * per_cell_bytes;
  R* xl = reinterpret_cast<R*>(base);     // [NF][NN]
  R* xr = xl + L::XL;                     // x-sweep out [2][P][Q][Q], later y-contraction out [3][2][P][Q][Q]
  R* yr = xr + L::XR;                     // y-sweep out [NF][3][Q][P*P], later z-contraction out [3][3][Q][P*P]
  R* rh = xl;                             // pointwise coefficients [3][4][P][P*P] (aliases xl + xr)
  int32_t* sid = reinterpret_cast<int32_t*>(yr + L::YR);

  const int list_index = cell_index_base + (active ? slot : 0);
  const bool has_cell = active && list_index < cd.ncells_list;
  const int cell = has_cell ? (cd.cells ? cd.cells[list_index] : list_index) : 0;

  // ---- gather (gather_cell!, src/assembly.jl:1060-1070; dx: zero at Dirichlet dofs) -------
  if (has_cell) {
    const int32_t* gid = cd.ids + (size_t)cell * NDL;
    for (int j = t; j < NDL; j += TPC) {
      int32_t id = gid[j];
      sid[j] = id;
      if (MODE == MODE_RESIDUAL || MODE == MODE_JV)
        xl[j] = id > 0 ? io.u[id - 1] : (id < 0 ? io.dvals[-id - 1] : R(0));
      if (MODE == MODE_JV) xl[NDL + j] = id > 0 ? io.dx[id - 1] : R(0);
      if (MODE == MODE_JV_STORED) xl[j] = id > 0 ? io.dx[id - 1] : R(0);
    }
  }
  __syncwarp();

  // ---- interpolation sweeps per field (tp_interpolate! 3D, reference gradients only) ---------
#pragma unroll 1
  for (int f = 0; f < NF; ++f) {
    const R* uf = xl + f * NN;
    if (t < Q * Q) {  // x lines (j, k)
      const int j = t % Q, k = t / Q;
      R v[Q];
#pragma unroll
      for (int i = 0; i < Q; ++i) v[i] = uf[i + Q * j + Q * Q * k];
#pragma unroll
      for (int a = 0; a < P; ++a) {
        R s = 0, ds = 0;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
          s += tab.N1[a * Q + i] * v[i];
          ds += tab.dN1[a * Q + i] * v[i];
        }
        xr[a + P * (j + Q * k)] = s;
        xr[P * Q * Q + a + P * (j + Q * k)] = ds;
      }
    }
    __syncwarp();
    if (t < P * Q) {  // y lines (a, k): C = N1.(N1 u), D = dN1.(N1 u), E = N1.(dN1 u)
      const int a = t % P, k = t / P;
      R va[Q], vb[Q];
#pragma unroll
      for (int j = 0; j < Q; ++j) {
        va[j] = xr[a + P * (j + Q * k)];
        vb[j] = xr[P * Q * Q + a + P * (j + Q * k)];
      }
#pragma unroll
      for (int b = 0; b < P; ++b) {
        R c0 = 0, d0 = 0, e0 = 0;
#pragma unroll
        for (int j = 0; j < Q; ++j) {
          c0 += tab.N1[b * Q + j] * va[j];
          d0 += tab.dN1[b * Q + j] * va[j];
          e0 += tab.N1[b * Q + j] * vb[j];
        }
        const int ab = a + P * b;
        yr[((f * 3 + 0) * Q + k) * P * P + ab] = c0;
        yr[((f * 3 + 1) * Q + k) * P * P + ab] = d0;
        yr[((f * 3 + 2) * Q + k) * P * P + ab] = e0;
      }
    }
    __syncwarp();
  }

  // ---- pointwise phase: lane (a, b) owns the points (a, b, c) ------------------------------
  // affine cells: one inverse Jacobian per cell (cell_geometry, src/assembly.jl:1100-1107)
  double iJc[9], detc = 0;
  bool aff = false;
  if (has_cell && MODE != MODE_JV_STORED) {
    aff = cd.affine[cell];
    if (aff) {
#pragma unroll
      for (int i = 0; i < 9; ++i) iJc[i] = cd.geo[(size_t)cell * 10 + i];
      detc = cd.geo[(size_t)cell * 10 + 9];
    }
  }
  if (has_cell && t < P * P) {
    const int ab = t;
#pragma unroll 1
    for (int c = 0; c < P; ++c) {
      const int q = ab + P * P * c;
      // z sweep of every field at this point: reference gradients G[f][K]
      R G[NF][3];
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        R g1 = 0, g2 = 0, g3 = 0;
#pragma unroll
        for (int k = 0; k < Q; ++k) {
          const R cv = yr[((f * 3 + 0) * Q + k) * P * P + ab];
          const R dv = yr[((f * 3 + 1) * Q + k) * P * P + ab];
          const R ev = yr[((f * 3 + 2) * Q + k) * P * P + ab];
          const R n = tab.N1[c * Q + k], dn = tab.dN1[c * Q + k];
          g1 += n * ev;
          g2 += n * dv;
          g3 += dn * cv;
        }
        G[f][0] = g1;
        G[f][1] = g2;
        G[f][2] = g3;
      }
      // geometry at the point
      R iJ[9], dV;
      if (MODE == MODE_JV_STORED) {
#pragma unroll
        for (int i = 0; i < 9; ++i) iJ[i] = (R)io.iJtq[((size_t)cell * 9 + i) * NP + q];
        dV = (R)io.dVq[(size_t)cell * NP + q];
      } else if (aff) {
#pragma unroll
        for (int i = 0; i < 9; ++i) iJ[i] = (R)iJc[i];
        dV = (R)(cd.w[q] * detc);
      } else {
        double Jt[9], iJd[9];
        point_jacobian_dev(cd, cell, q, Jt);
        const double det = det3(Jt);
        inv3(Jt, det, iJd);
#pragma unroll
        for (int i = 0; i < 9; ++i) iJ[i] = (R)iJd[i];
        dV = (R)(cd.w[q] * fabs(det));
      }
      R out[3][3];   // R^[comp][K] = dV sum_J iJt[J,K] P[comp,J]
      R outv[3];     // value coefficients (body force of the residual)
      if (MODE == MODE_RESIDUAL) {
        R H[9];
        phys_grad<R>(iJ, G, 0, H);
        R Pm[9];
        law_stress<R>(cd.law, (R)cd.lam, (R)cd.mu, H, Pm);
        pull_back<R>(iJ, Pm, dV, out);
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) outv[cc] = -dV * (R)cd.body[cc];
      } else if (MODE == MODE_JV) {
        R H[9], Hd[9], dP[9];
        phys_grad<R>(iJ, G, 0, H);
        phys_grad<R>(iJ, G, 3, Hd);
        law_dstress<R>(cd.law, (R)cd.lam, (R)cd.mu, H, Hd, dP);
        pull_back<R>(iJ, dP, dV, out);
      } else {
        // stored tangent: su = physical gradients of dx, sv = dV T su (apply_cells!, src/matrixfree.jl:367-375)
        R Hd[9], sv[9];
        phys_grad<R>(iJ, G, 0, Hd);
        const double* Tq = io.T + (size_t)cell * 81 * NP + q;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
          R s = 0;
#pragma unroll
          for (int j = 0; j < 9; ++j) s += (R)Tq[(size_t)(i + 9 * j) * NP] * Hd[(j / 3) + 3 * (j % 3)];
          sv[(i / 3) + 3 * (i % 3)] = s;
        }
        pull_back<R>(iJ, sv, dV, out);
      }
      // store coefficients of this point (rh aliases xl/xr, whose last reads precede the last sync)
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
#pragma unroll
        for (int K = 0; K < 3; ++K) rh[((cc * 4 + 1 + K) * P + c) * P * P + ab] = out[cc][K];
        rh[((cc * 4 + 0) * P + c) * P * P + ab] = MODE == MODE_RESIDUAL ? outv[cc] : R(0);
      }
    }
  }
  __syncwarp();

  // ---- contraction (tp_contract! 3D): z, then y, then x ------------------------------------
  if (t < P * P) {  // z lines (a, b) -> t0, t1, t2 [k]
    const int ab = t;
#pragma unroll 1
    for (int cc = 0; cc < 3; ++cc) {
#pragma unroll
      for (int k = 0; k < Q; ++k) {
        R t0 = 0, t1 = 0, t2 = 0;
#pragma unroll
        for (int c = 0; c < P; ++c) {
          const R n = tab.N1[c * Q + k], dn = tab.dN1[c * Q + k];
          t0 += n * rh[((cc * 4 + 0) * P + c) * P * P + ab] + dn * rh[((cc * 4 + 3) * P + c) * P * P + ab];
          t1 += n * rh[((cc * 4 + 1) * P + c) * P * P + ab];
          t2 += n * rh[((cc * 4 + 2) * P + c) * P * P + ab];
        }
        yr[((cc * 3 + 0) * Q + k) * P * P + ab] = t0;
        yr[((cc * 3 + 1) * Q + k) * P * P + ab] = t1;
        yr[((cc * 3 + 2) * Q + k) * P * P + ab] = t2;
      }
    }
  }
  __syncwarp();
  if (t < P * Q) {  // y lines (a, k) -> s0, s1 [j]
    const int a = t % P, k = t / P;
#pragma unroll 1
    for (int cc = 0; cc < 3; ++cc) {
      R v0[P], v1[P], v2[P];
#pragma unroll
      for (int b = 0; b < P; ++b) {
        v0[b] = yr[((cc * 3 + 0) * Q + k) * P * P + a + P * b];
        v1[b] = yr[((cc * 3 + 1) * Q + k) * P * P + a + P * b];
        v2[b] = yr[((cc * 3 + 2) * Q + k) * P * P + a + P * b];
      }
#pragma unroll
      for (int j = 0; j < Q; ++j) {
        R s0 = 0, s1 = 0;
#pragma unroll
        for (int b = 0; b < P; ++b) {
          s0 += tab.N1[b * Q + j] * v0[b] + tab.dN1[b * Q + j] * v2[b];
          s1 += tab.N1[b * Q + j] * v1[b];
        }
        xr[(cc * 2 + 0) * P * Q * Q + a + P * (j + Q * k)] = s0;
        xr[(cc * 2 + 1) * P * Q * Q + a + P * (j + Q * k)] = s1;
      }
    }
  }
  __syncwarp();
  if (has_cell && t < Q * Q) {  // x lines (j, k) -> r[i], scatter of free test rows
    const int j = t % Q, k = t / Q;
#pragma unroll 1
    for (int cc = 0; cc < 3; ++cc) {
      R v0[P], v1[P];
#pragma unroll
      for (int a = 0; a < P; ++a) {
        v0[a] = xr[(cc * 2 + 0) * P * Q * Q + a + P * (j + Q * k)];
        v1[a] = xr[(cc * 2 + 1) * P * Q * Q + a + P * (j + Q * k)];
      }
#pragma unroll
      for (int i = 0; i < Q; ++i) {
        R s = 0;
#pragma unroll
        for (int a = 0; a < P; ++a) s += tab.N1[a * Q + i] * v0[a] + tab.dN1[a * Q + i] * v1[a];
        const int32_t id = sid[cc * NN + i + Q * j + Q * Q * k];
        if (id > 0) {
          if (io.atomic) atomicAdd(&io.y[id - 1], s);
          else io.y[id - 1] += s;
        }
      }
    }
  }
}

template <int Q, int P, int MODE, typename R>
constexpr size_t cell_smem_bytes(int warps) {
  return (size_t)warps * TPShape<Q, P>::CPW * cell_region_bytes<Q, P, MODE, R>();
}

}  // namespace hfk
