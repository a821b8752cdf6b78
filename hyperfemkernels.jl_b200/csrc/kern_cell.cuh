// Sum-factorised cell kernels for a 3-component Lagrangian field on hexahedra:
//   MODE_RESIDUAL  residual of the law at the state u (gathers u)
//   MODE_PREP_F    deformation gradient F = I + grad u at every point, stored (gathers u)
//   MODE_ENERGY    the stored energy Σ Ψ(F) dV and min det F of the cells (gathers u; per-warp partials)
//   MODE_JV        J(u) dx with the tangent re-evaluated from the stored F (gathers dx)
//   MODE_JV_STORED J(u) dx with the reference's stored per-point tangents T, inv(Jt), dV
//
// Mapping: a warp holds CPW = 32 / M^2 cells (M = max(P, Q)); the M^2 lanes of a cell own the
// tensor lines of each sum-factorisation sweep (x lines (j,k), y lines (a,k), z lines (a,b)), so
// every sweep reads each input once and writes P (or 3P) outputs from registers. Lane (a,b) owns
// the P points (a,b,c): it loads its z column of the y-sweep into registers and writes the point
// coefficients back in place (each lane only touches addresses of its own column), which keeps
// the shared footprint of a cell small (occupancy). Cells of one colour share no free dof, so the
// scatter is a plain read-modify-write (colour-by-colour launches), or atomicAdd in one launch.
//
// Reference: tp_interpolate!/tp_contract! (src/tensorproduct.jl:125-224), apply_cells!
// (src/matrixfree.jl:341-396), element_residual_mm! (src/assembly.jl:1219-1241); the SVK tangent
// is the exact derivative the factorised form evaluates (src/factorforms.jl:316-322).
#pragma once
#include "hfk_internal.h"
#include "pointwise.cuh"

namespace hfk {

enum CellMode { MODE_RESIDUAL = 0, MODE_JV = 1, MODE_JV_STORED = 2, MODE_PREP_F = 3, MODE_ENERGY = 4 };

template <int Q, int P>
struct TPShape {
  static constexpr int NN = Q * Q * Q;
  static constexpr int NP = P * P * P;
  static constexpr int M = P > Q ? P : Q;
  static constexpr int TPC = M * M;     // lanes per cell
  static constexpr int CPW = 32 / TPC;  // cells per warp
  static_assert(CPW >= 1, "a cell must fit in a warp (max(P,Q) <= 5)");
  static_assert(3 * Q <= 4 * P, "the in-place z contraction needs 3Q <= 4P");
};

constexpr int cmax(int a, int b) { return a > b ? a : b; }

// Shared layout of one cell, in units of R:
//   YR  [rows][P*P]: y-sweep out (3 fields x 3 kinds x Q rows), then the point coefficients in
//       place (3 comps x 4 slots x P rows), then the z-contraction out (3 comps x 3 kinds x Q rows)
//   xl  [3][NN] local values;  XS [2][P*Q*Q] x-sweep out
//   the y-contraction out (3 comps x 2 x P*Q*Q) uses the tail: YR rows past 9Q, then xl and XS
template <int Q, int P>
struct CellSmem {
  static constexpr int NN = Q * Q * Q, NP = P * P * P;
  static constexpr int YR = cmax(9 * Q * P * P, 12 * NP);
  static constexpr int XL = 3 * NN;
  static constexpr int XS0 = 2 * P * Q * Q;
  static constexpr int TAIL0 = YR - 9 * Q * P * P + XL + XS0;
  static constexpr int XS = TAIL0 >= 6 * P * Q * Q ? XS0 : XS0 + (6 * P * Q * Q - TAIL0);
  static constexpr int VALS = YR + XL + XS;
};

// Bytes of one cell's shared region. With several cells per warp the region stride is padded to
// TPC * sizeof(R) modulo 128 bytes, so the lanes of consecutive cells (each reading TPC consecutive
// words) fall on consecutive banks instead of the same ones.
template <int Q, int P, typename R>
__host__ __device__ constexpr size_t cell_region_bytes() {
  size_t raw = (size_t)CellSmem<Q, P>::VALS * sizeof(R) + (size_t)3 * TPShape<Q, P>::NN * sizeof(int32_t);
  raw = (raw + sizeof(R) - 1) / sizeof(R) * sizeof(R);
  if (TPShape<Q, P>::CPW > 1) {
    const size_t target = ((size_t)TPShape<Q, P>::TPC * sizeof(R)) % 128;
    while (raw % 128 != target) raw += sizeof(R);
  }
  return raw;
}

// resident CTAs per SM the register allocation of a mode targets (measured on B200 with the atomic
// scatter: the stored formulation prefers 2, the recompute product 3 (no spills) over 4; the FP32
// recompute product 6 (80 registers, 24 warps per SM: 0.40 -> 0.30 ms on Q2 64^3), where FP64 at
// 4 or 5 spills and loses)
template <int MODE, typename R>
constexpr int cell_min_blocks() {
  return MODE == MODE_JV_STORED ? 2 : (MODE == MODE_JV && sizeof(R) == 4 ? 6 : 3);
}

template <typename R>
struct CellIO {
  const R* u;       // state free values (MODE_RESIDUAL, MODE_PREP_F)
  const R* dvals;   // state Dirichlet values
  const R* dx;      // increment (MODE_JV, MODE_JV_STORED)
  R* y;             // output (scatter-add)
  const R* Fq;      // stored F (MODE_JV): (cell*9 + i)*NP + q
  R* Fout;          // MODE_PREP_F output, same layout
  const double* T;  // stored tangents (cell*81 + i)*NP + q
  const double* iJtq;
  const double* dVq;
  int atomic;       // 1: atomicAdd scatter (all cells in one launch)
  double* red;      // MODE_ENERGY: per warp of the grid, (Σ Ψ dV, min det F)
};

template <int Q, int P, int MODE, typename R>
__global__ void __launch_bounds__(128, cell_min_blocks<MODE, R>()) cell_kernel(CellData cd, Tab1D<R> tab, CellIO<R> io) {
  using S = TPShape<Q, P>;
  using L = CellSmem<Q, P>;
  constexpr int NN = S::NN, NP = S::NP, TPC = S::TPC, CPW = S::CPW;
  constexpr int NDL = 3 * NN;
  constexpr int PP = P * P;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  const int slot = lane / TPC;
  const bool active = slot < CPW;  // lanes past CPW * TPC idle: every phase is guarded by t
  const int t = active ? lane - slot * TPC : (1 << 20);
  unsigned char* base = smem_raw + (size_t)(warp * CPW + (active ? slot : 0)) * cell_region_bytes<Q, P, R>();
  R* yr = reinterpret_cast<R*>(base);
  R* xl = yr + L::YR;
  R* xs = xl + L::XL;
  R* tail = yr + 9 * Q * PP;  // y-contraction out (contiguous over the YR tail, xl, xs)
  int32_t* sid = reinterpret_cast<int32_t*>(yr + L::VALS);

  const int list_index = (blockIdx.x * nwarps + warp) * CPW + (active ? slot : 0);
  const int cell = active && list_index < cd.ncells_list ? (cd.cells ? cd.cells[list_index] : list_index) : 0;
  const bool has_cell = active && list_index < cd.ncells_list && !cd.skipped(cell);
  if (__all_sync(0xffffffffu, !has_cell)) {  // a warp without work (only __syncwarp below)
    if (MODE == MODE_ENERGY && lane == 0) {
      io.red[2 * ((size_t)blockIdx.x * nwarps + warp)] = 0.0;
      io.red[2 * ((size_t)blockIdx.x * nwarps + warp) + 1] = INFINITY;
    }
    return;
  }
  const R lam_c = (R)cd.lam_of(cell), mu_c = (R)cd.mu_of(cell);

  // ---- gather (gather_cell!, src/assembly.jl:1060-1070; increments are zero at Dirichlet dofs) ----
  if (has_cell) {
    const int32_t* gid = cd.ids + (size_t)cell * NDL;
#pragma unroll 3
    for (int j = t; j < NDL; j += TPC) {
      const int32_t id = gid[j];
      sid[j] = id;
      if (MODE == MODE_RESIDUAL || MODE == MODE_PREP_F || MODE == MODE_ENERGY)
        xl[j] = id > 0 ? io.u[id - 1] : (id < 0 ? io.dvals[-id - 1] : R(0));
      else
        xl[j] = id > 0 ? io.dx[id - 1] : R(0);
    }
  }
  // geometry of an affine cell (cell_geometry, src/assembly.jl:1100-1107), loaded early
  bool aff = false;
  if (has_cell && MODE != MODE_JV_STORED) aff = cd.affine[cell];
  __syncwarp();

  // ---- interpolation sweeps (tp_interpolate! 3D, reference gradients only) ------------------
#pragma unroll 1
  for (int f = 0; f < 3; ++f) {
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
        xs[a + P * (j + Q * k)] = s;
        xs[P * Q * Q + a + P * (j + Q * k)] = ds;
      }
    }
    __syncwarp();
    if (t < P * Q) {  // y lines (a, k): C = N1.(N1 u), D = dN1.(N1 u), E = N1.(dN1 u)
      const int a = t % P, k = t / P;
      R va[Q], vb[Q];
#pragma unroll
      for (int j = 0; j < Q; ++j) {
        va[j] = xs[a + P * (j + Q * k)];
        vb[j] = xs[P * Q * Q + a + P * (j + Q * k)];
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
        yr[((f * 3 + 0) * Q + k) * PP + ab] = c0;
        yr[((f * 3 + 1) * Q + k) * PP + ab] = d0;
        yr[((f * 3 + 2) * Q + k) * PP + ab] = e0;
      }
    }
    __syncwarp();
  }

  // ---- pointwise phase: lane (a, b) owns the points (a, b, c) --------------------------------
  double esum = 0.0, dmin = INFINITY;  // MODE_ENERGY
  if (t < PP) {
    const int ab = t;
    R yc[3][3][Q];  // this lane's column of the y-sweep: [field][kind][k]
#pragma unroll
    for (int f = 0; f < 3; ++f)
#pragma unroll
      for (int kind = 0; kind < 3; ++kind)
#pragma unroll
        for (int k = 0; k < Q; ++k) yc[f][kind][k] = yr[((f * 3 + kind) * Q + k) * PP + ab];
#pragma unroll 1
    for (int c = 0; c < P; ++c) {
      const int q = ab + PP * c;
      R G[3][3];  // z sweep: reference gradients G[f][K]
#pragma unroll
      for (int f = 0; f < 3; ++f) {
        R g1 = 0, g2 = 0, g3 = 0;
#pragma unroll
        for (int k = 0; k < Q; ++k) {
          const R n = tab.N1[c * Q + k], dn = tab.dN1[c * Q + k];
          g1 += n * yc[f][2][k];
          g2 += n * yc[f][1][k];
          g3 += dn * yc[f][0][k];
        }
        G[f][0] = g1;
        G[f][1] = g2;
        G[f][2] = g3;
      }
      R iJ[9], dV = 0;
      if (MODE == MODE_JV_STORED) {
        if (has_cell) {
#pragma unroll
          for (int i = 0; i < 9; ++i) iJ[i] = (R)io.iJtq[((size_t)cell * 9 + i) * NP + q];
          dV = (R)io.dVq[(size_t)cell * NP + q];
        } else {
#pragma unroll
          for (int i = 0; i < 9; ++i) iJ[i] = 0;
        }
      } else if (aff || !has_cell) {
        // the cell's inverse Jacobian read per point (an L1 hit shared by the cell's lanes)
        const double* gc = cd.geo + (size_t)(has_cell ? cell : 0) * 10;
#pragma unroll
        for (int i = 0; i < 9; ++i) iJ[i] = has_cell ? (R)__ldg(gc + i) : R(0);
        dV = has_cell ? (R)(cd.w[q] * __ldg(gc + 9)) : R(0);
      } else {
        double Jt[9], iJd[9];
        point_jacobian_dev(cd, cell, q, Jt);
        const double det = det3(Jt);
        inv3(Jt, det, iJd);
#pragma unroll
        for (int i = 0; i < 9; ++i) iJ[i] = (R)iJd[i];
        dV = (R)(cd.w[q] * fabs(det));
      }
      R H[9];
      phys_grad<R, 3>(iJ, G, 0, H);
      if (MODE == MODE_PREP_F) {
        if (has_cell) {
#pragma unroll
          for (int i = 0; i < 9; ++i) io.Fout[((size_t)cell * 9 + i) * NP + q] = H[i] + ((i % 4) == 0 ? R(1) : R(0));
        }
        continue;
      }
      if (MODE == MODE_ENERGY) {
        if (has_cell) {
          double Hd[9], Fd[9];
#pragma unroll
          for (int i = 0; i < 9; ++i) {
            Hd[i] = (double)H[i];
            Fd[i] = Hd[i] + ((i % 4) == 0 ? 1.0 : 0.0);
          }
          esum += (double)dV * law_energy(cd.law, (double)lam_c, (double)mu_c, Hd);
          dmin = fmin(dmin, det3(Fd));
        }
        continue;
      }
      R out[3][3];
      R outv[3] = {0, 0, 0};
      if (MODE == MODE_RESIDUAL) {
        R Pm[9];
        law_stress<R>(cd.law, lam_c, mu_c, H, Pm);
        pull_back<R>(iJ, Pm, dV, out);
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) outv[cc] = -dV * (R)cd.body[cc];
      } else if (MODE == MODE_JV) {
        R Fm[9], dP[9];
        if (has_cell) {
#pragma unroll
          for (int i = 0; i < 9; ++i) Fm[i] = io.Fq[((size_t)cell * 9 + i) * NP + q];
        } else {
#pragma unroll
          for (int i = 0; i < 9; ++i) Fm[i] = (i % 4) == 0 ? R(1) : R(0);
        }
        law_dstress_F<R>(cd.law, lam_c, mu_c, Fm, H, dP);
        pull_back<R>(iJ, dP, dV, out);
      } else {
        // stored tangent: sv = dV T su (apply_cells!, src/matrixfree.jl:367-375)
        R sv[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) {
          R s = 0;
          if (has_cell) {
            const double* Tq = io.T + (size_t)cell * 81 * NP + q;
#pragma unroll
            for (int j = 0; j < 9; ++j) s += (R)Tq[(size_t)(i + 9 * j) * NP] * H[(j / 3) + 3 * (j % 3)];
          }
          sv[(i / 3) + 3 * (i % 3)] = s;
        }
        pull_back<R>(iJ, sv, dV, out);
      }
      // point coefficients written in place into this lane's own column of YR
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
        yr[((cc * 4 + 0) * P + c) * PP + ab] = outv[cc];
#pragma unroll
        for (int K = 0; K < 3; ++K) yr[((cc * 4 + 1 + K) * P + c) * PP + ab] = out[cc][K];
      }
    }
  }
  if (MODE == MODE_PREP_F) return;
  if (MODE == MODE_ENERGY) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      esum += __shfl_down_sync(0xffffffffu, esum, o);
      dmin = fmin(dmin, __shfl_down_sync(0xffffffffu, dmin, o));
    }
    if (lane == 0) {
      io.red[2 * ((size_t)blockIdx.x * nwarps + warp)] = esum;
      io.red[2 * ((size_t)blockIdx.x * nwarps + warp) + 1] = dmin;
    }
    return;
  }
  __syncwarp();

  // ---- contraction (tp_contract! 3D): z (in place, per lane column), y, x -------------------
  if (t < PP) {
    const int ab = t;
#pragma unroll 1
    for (int cc = 0; cc < 3; ++cc) {
      // the z-contraction rows of cc overlap only coefficient rows of cc or of earlier components
      R rv[4][P];
#pragma unroll
      for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int c = 0; c < P; ++c) rv[s][c] = yr[((cc * 4 + s) * P + c) * PP + ab];
#pragma unroll
      for (int k = 0; k < Q; ++k) {
        R t0 = 0, t1 = 0, t2 = 0;
#pragma unroll
        for (int c = 0; c < P; ++c) {
          const R n = tab.N1[c * Q + k], dn = tab.dN1[c * Q + k];
          t0 += n * rv[0][c] + dn * rv[3][c];
          t1 += n * rv[1][c];
          t2 += n * rv[2][c];
        }
        yr[((cc * 3 + 0) * Q + k) * PP + ab] = t0;
        yr[((cc * 3 + 1) * Q + k) * PP + ab] = t1;
        yr[((cc * 3 + 2) * Q + k) * PP + ab] = t2;
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
        v0[b] = yr[((cc * 3 + 0) * Q + k) * PP + a + P * b];
        v1[b] = yr[((cc * 3 + 1) * Q + k) * PP + a + P * b];
        v2[b] = yr[((cc * 3 + 2) * Q + k) * PP + a + P * b];
      }
#pragma unroll
      for (int j = 0; j < Q; ++j) {
        R s0 = 0, s1 = 0;
#pragma unroll
        for (int b = 0; b < P; ++b) {
          s0 += tab.N1[b * Q + j] * v0[b] + tab.dN1[b * Q + j] * v2[b];
          s1 += tab.N1[b * Q + j] * v1[b];
        }
        tail[(cc * 2 + 0) * P * Q * Q + a + P * (j + Q * k)] = s0;
        tail[(cc * 2 + 1) * P * Q * Q + a + P * (j + Q * k)] = s1;
      }
    }
  }
  __syncwarp();
  if (has_cell && t < Q * Q) {  // x lines (j, k) -> r[i]; scatter of the free test rows
    const int j = t % Q, k = t / Q;
    R r[3][Q];
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) {
      R v0[P], v1[P];
#pragma unroll
      for (int a = 0; a < P; ++a) {
        v0[a] = tail[(cc * 2 + 0) * P * Q * Q + a + P * (j + Q * k)];
        v1[a] = tail[(cc * 2 + 1) * P * Q * Q + a + P * (j + Q * k)];
      }
#pragma unroll
      for (int i = 0; i < Q; ++i) {
        R s = 0;
#pragma unroll
        for (int a = 0; a < P; ++a) s += tab.N1[a * Q + i] * v0[a] + tab.dN1[a * Q + i] * v1[a];
        r[cc][i] = s;
      }
    }
    if (io.atomic) {
#pragma unroll
      for (int cc = 0; cc < 3; ++cc)
#pragma unroll
        for (int i = 0; i < Q; ++i) {
          const int32_t id = sid[cc * NN + i + Q * j + Q * Q * k];
          if (id > 0) atomicAdd(&io.y[id - 1], r[cc][i]);
        }
    } else {
      R old[3][Q];
#pragma unroll
      for (int cc = 0; cc < 3; ++cc)
#pragma unroll
        for (int i = 0; i < Q; ++i) {
          const int32_t id = sid[cc * NN + i + Q * j + Q * Q * k];
          old[cc][i] = id > 0 ? io.y[id - 1] : R(0);
        }
#pragma unroll
      for (int cc = 0; cc < 3; ++cc)
#pragma unroll
        for (int i = 0; i < Q; ++i) {
          const int32_t id = sid[cc * NN + i + Q * j + Q * Q * k];
          if (id > 0) io.y[id - 1] = old[cc][i] + r[cc][i];
        }
    }
  }
}

template <int Q, int P, typename R>
constexpr size_t cell_smem_bytes(int warps) {
  return (size_t)warps * TPShape<Q, P>::CPW * cell_region_bytes<Q, P, R>();
}

}  // namespace hfk
