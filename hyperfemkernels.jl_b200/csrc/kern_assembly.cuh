// Fused element Jacobian + scatter into the CSC nonzeros.
//
// Per point the tangent is pulled back to the reference gradients once,
//   Dh_q[(c,K),(k,K')] = dV sum_{J,L} iJt[J,K] T[(c,J),(k,L)] iJt[L,K'],
// so that the element matrix
//   K[(n,c),(m,k)] = sum_q sum_{K,K'} dN^[n,K,q] Dh_q[(c,K),(k,K')] dN^[m,K',q]
// only reads the reference tables (shared by all cells). For 27-node cells it is formed as the
// reference forms it (element_jacobian_mm!, src/assembly.jl:1316-1342): per test component c,
// G_c[(q,K),(m,k)] = sum_K' Dh[(c,K),(k,K')] dN^[m,K',q], then K_c = A^T G_c with A = dN^ as an
// (np*3) x nn matrix. Three kernels:
//   jacobian_kernel_sym27 (the default for the symmetric tangents of the recognised laws): the
//     blocks k >= c only, on the FP64 FMA pipe, with a sum-factorised contraction when the tables
//     are tensor products; persistent CTAs;
//   jacobian_kernel_g (27-node cells, any tangent; selectable for the symmetric ones): K_c on the
//     FP64 tensor cores (mma.sync m8n8k4), one CTA per cell;
//   jacobian_kernel_direct (8-node cells): one thread per element entry, one CTA per cell.
// All cells in one launch, or the cells of one colour per launch. The entries are added at their
// precomputed positions (scatter_jacobian!, src/assembly.jl:1402-1408) by reductions.
#pragma once
#include "hfk_internal.h"
#include "kern_async.cuh"
#include "pointwise.cuh"

namespace hfk {

struct AsmIO {
  const double* u;
  const double* dvals;
  const double* dNt;      // (nn, 3, np) tensor order
  const int32_t* nzpos;   // (ndl*ndl, ncells) 1-based
  double* nzval;
  int np;
  int ldg;                // shared row stride of G_c[r][mk] (27-node cells, >= 3 nn)
};

// Row stride of G_c in the 27-node kernel when it fits: at least the 88 columns of the padded
// product, with zeros past column 81, and 4 modulo 16 doubles, so that the 4 x 8 elements of a B
// fragment (k rows apart by the stride, columns adjacent) fall on distinct 8-byte bank pairs within
// each half-warp and two per pair over the warp: two wavefronts, the minimum for 32 doubles
constexpr int ASM_LDG_PADDED = 100;

// Phase 1 (shared by both variants): per point, physical gradient of u, geometry, pulled-back
// tangent Dh[q][(c*3+K) + 9*(k*3+K')] in shared memory.
template <int NN>
__device__ void asm_point_phase(const CellData& cd, const AsmIO& io, int cell, const double* A, const double* xl,
                                double* Hs, double* iJs, double* dVs, double* Dh) {
  const int np = io.np;
  // per point: H, iJt, dV
  for (int q = threadIdx.x; q < np; q += blockDim.x) {
    double G[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int n = 0; n < NN; ++n) {
      const double a0 = A[n + NN * (0 + 3 * q)], a1 = A[n + NN * (1 + 3 * q)], a2 = A[n + NN * (2 + 3 * q)];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double x = xl[c * NN + n];
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
  // per (point, c, k): the 3x3 block of Dh
  for (int e = threadIdx.x; e < np * 9; e += blockDim.x) {
    const int q = e / 9, ck = e % 9, c = ck / 3, k = ck % 3;
    double Tb[9];  // T[(c,J),(k,L)] at Tb[J + 3 L]
    law_tangent_block(cd.law, cd.lam_of(cell), cd.mu_of(cell), Hs + q * 9, c, k, Tb);
    const double* iJ = iJs + q * 9;
    const double dV = dVs[q];
    // X[J][K'] = sum_L T[(c,J),(k,L)] iJ[L + 3K']
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
        Dh[q * 81 + (c * 3 + K) + 9 * (k * 3 + Kp)] = dV * s;
      }
  }
  __syncthreads();
}

// One element-matrix entry added at its precomputed position (scatter_jacobian!,
// src/assembly.jl:1402-1408). The add is a reduction whose result is not read: the thread does not
// wait for the nonzero to arrive from memory, as a load-add-store would. Launched colour by colour,
// no two adds of a launch meet the same nonzero (cells of one colour share no free test dof, the
// entries of one cell have distinct positions), so the colours add in a fixed order and the sums
// are deterministic; launched over all cells at once, neighbouring cells' adds meet in L2.
__device__ __forceinline__ void scatter_add(double* nzval, int32_t p, double v) {
  if (p > 0) atomicAdd(nzval + (p - 1), v);
}

// FP64 tensor-core product of an 8x4 and a 4x8 tile (mma.sync m8n8k4, PTX ISA "Matrix Fragments for
// mma.m8n8k4 with .f64"): lane l holds a = A[l/4][l%4], b = B[l%4][l/4] and the accumulators
// d[i] = D[l/4][2(l%4) + i].
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// One test component c of the 27-node kernel (below): G_c in shared memory, then K_c = A^T G_c on the
// FP64 tensor cores and the scatter. C is a template parameter so that the first column tile
// (TMIN, under SYM) is a constant: the tile loops and their bounds resolve at compile time.
template <int NN, bool PADDED, bool SYM, int C>
__device__ __forceinline__ void asm_component(const AsmIO& io, const int32_t* pos, const double* A, const double* Dh,
                                              double* G) {
  constexpr int NDL = 3 * NN;
  constexpr int MT = (NN + 7) / 8, NT = (NDL + 7) / 8;  // 8-row bands of K_c, 8-column tiles
  constexpr int MK0 = SYM ? C * NN : 0;                 // first column of K_c that is formed
  constexpr int TMIN = MK0 / 8;                         // first column tile that reaches it
  constexpr int TPW = (NT - TMIN + 1) / 2;              // column tiles per warp (two warps per band)
  constexpr int RG = 256 / NDL;                         // thread groups of G_c's construction
  const int np = io.np, ldg = io.ldg;
  const int R = 3 * np, ksteps = (R + 3) / 4;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int band = warp % MT, tile0 = warp / MT;
  const int fr = lane >> 2, fc = lane & 3;  // fragment row / column of this lane
  // G_c[r = q*3 + K][mk = k*NN + m] = sum_K' Dh_q[(c,K),(k,K')] dN^[m,K',q]: thread (g, mk) fills
  // column mk for the points q = g, g + RG, ...; a point's three values of A serve its three rows.
  // Only the columns of the tiles the products read are formed (from the first tile's start; the
  // few of its columns below MK0 are computed, but their entries are not scattered).
  if (threadIdx.x < RG * NDL) {
    const int g = threadIdx.x / NDL, mk = threadIdx.x - g * NDL;
    const int k = mk / NN, m = mk - k * NN;
    if (mk >= TMIN * 8)
      for (int q = g; q < np; q += RG) {
        const double a0 = A[m + NN * (3 * q)], a1 = A[m + NN * (3 * q + 1)], a2 = A[m + NN * (3 * q + 2)];
        const double* D = Dh + q * 81 + C * 3 + 27 * k;
#pragma unroll
        for (int K = 0; K < 3; ++K) G[(3 * q + K) * ldg + mk] = D[K] * a0 + D[K + 9] * a1 + D[K + 18] * a2;
      }
  }
  __syncthreads();
  // this lane's output entries: rows n = band*8 + fr, columns mk = tile*8 + 2 fc + i; positions
  // loaded first (their latency overlaps the products); under SYM also the transposed entry's
  const int n = band * 8 + fr;
  int32_t pp[TPW][2], pt[TPW][2];
  double acc[2][TPW][2];  // even and odd k-steps: two independent chains of tensor-core steps
#pragma unroll
  for (int j = 0; j < TPW; ++j) {
    const int tile = TMIN + tile0 + 2 * j;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int mk = tile * 8 + 2 * fc + i;
      const bool own = tile < NT && n < NN && mk < NDL && mk >= MK0;
      pp[j][i] = own ? __ldg(pos + (C * NN + n) + NDL * mk) : 0;
      pt[j][i] = (SYM && own && mk >= MK0 + NN) ? __ldg(pos + mk + NDL * (C * NN + n)) : 0;
      acc[0][j][i] = acc[1][j][i] = 0.0;
    }
  }
  // fragment elements past the matrices' edges are zeros: a lane whose element lies outside
  // loads a valid address and selects zero, so the warp stays converged for mma.sync
  const bool na = n < NN;
  auto kstep = [&](int ks, double (&ac)[TPW][2]) {
    const int r = ks * 4 + fc;  // k index of this lane's A^T and B fragment elements
    const bool ra = na && r < R;
    double a = A[ra ? n + NN * r : 0];
    a = ra ? a : 0.0;
    const double* Gr = G + r * ldg + fr;
#pragma unroll
    for (int j = 0; j < TPW; ++j) {
      const int tile = TMIN + tile0 + 2 * j;
      if (tile < NT) {  // uniform over the warp
        double b;
        if (PADDED) {
          b = Gr[tile * 8];
        } else {
          const bool rb = r < R && tile * 8 + fr < NDL;
          b = G[rb ? r * ldg + tile * 8 + fr : 0];
          b = rb ? b : 0.0;
        }
        dmma_8x8x4(ac[j][0], ac[j][1], a, b);
      }
    }
  };
  for (int ks = 0; ks < ksteps; ks += 2) {
    kstep(ks, acc[0]);
    if (ks + 1 < ksteps) kstep(ks + 1, acc[1]);  // uniform over the block
  }
#pragma unroll
  for (int j = 0; j < TPW; ++j)
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const double v = acc[0][j][i] + acc[1][j][i];
      scatter_add(io.nzval, pp[j][i], v);
      if (SYM) scatter_add(io.nzval, pt[j][i], v);
    }
  __syncthreads();
}

// 27-node cells (Q2): G_c in shared memory, K_c = A^T G_c on the FP64 tensor cores. Eight warps:
// warp w takes the 8-row band w % 4 of K_c (rows n, 27 padded to 32) and every other 8-column tile
// (columns mk, 81 padded to 88) from w / 4; the k dimension (r = 3 np) runs in steps of 4, padded
// with zeros. A warp loads one fragment of A^T per k-step and reuses it for its five or six tiles.
// PADDED: G_c has the row stride ASM_LDG_PADDED and zeros past its last row and column, so the B
// fragments load without bounds selects; otherwise (large np) the stride is 81 and they select.
// SYM: the tangent has the major symmetry T[(c,J),(k,L)] = T[(k,L),(c,J)] (every hyperelastic law:
// SVK, linear elasticity), so K[(n,c),(m,k)] = K[(m,k),(n,c)]: only the blocks k >= c are formed
// (the column tiles that reach columns k*NN + m >= c*NN: 24 of 33 tiles, and the G_c columns of
// those tiles), and each entry of a block k > c is added at its own position and at its transpose's.
template <int NN, bool PADDED, bool SYM>
__global__ void __launch_bounds__(256) jacobian_kernel_g(CellData cd, AsmIO io) {
  constexpr int NDL = 3 * NN;
  constexpr int MT = (NN + 7) / 8, NT = (NDL + 7) / 8;
  static_assert(MT == 4, "eight warps: four row bands x two column-tile sets");
  extern __shared__ __align__(16) double sm[];
  const int np = io.np, ldg = io.ldg;
  const int R = 3 * np, ksteps = (R + 3) / 4;
  double* A = sm;                       // NN * R
  double* xl = A + (size_t)NN * R;      // NDL
  double* Hs = xl + NDL;                // 9 np
  double* iJs = Hs + 9 * np;            // 9 np
  double* dVs = iJs + 9 * np;           // np
  double* Dh = dVs + np;                // 81 np
  double* G = Dh + 81 * np;             // 4 ksteps x ldg
  const int li = blockIdx.x;
  if (li >= cd.ncells_list) return;
  const int cell = cd.cells ? cd.cells[li] : li;
  const int32_t* gid = cd.ids + (size_t)cell * NDL;
  for (int i = threadIdx.x; i < NN * R; i += blockDim.x) A[i] = io.dNt[i];
  for (int j = threadIdx.x; j < NDL; j += blockDim.x) {
    const int32_t id = gid[j];
    xl[j] = id > 0 ? io.u[id - 1] : (id < 0 ? io.dvals[-id - 1] : 0.0);
  }
  if (PADDED) {  // the padding of G_c: columns NDL..NT*8-1 of every row, and the rows past R
    constexpr int W = NT * 8 - NDL;
    for (int i = threadIdx.x; i < R * W; i += blockDim.x) G[(i / W) * ldg + NDL + i % W] = 0.0;
    for (int i = threadIdx.x; i < (4 * ksteps - R) * NT * 8; i += blockDim.x)
      G[(R + i / (NT * 8)) * ldg + i % (NT * 8)] = 0.0;
  }
  __syncthreads();
  asm_point_phase<NN>(cd, io, cell, A, xl, Hs, iJs, dVs, Dh);
  const int32_t* pos = io.nzpos + (size_t)NDL * NDL * cell;
  asm_component<NN, PADDED, SYM, 0>(io, pos, A, Dh, G);
  asm_component<NN, PADDED, SYM, 1>(io, pos, A, Dh, G);
  asm_component<NN, PADDED, SYM, 2>(io, pos, A, Dh, G);
}

// ---- symmetric tangents on 27-node cells: the element blocks on the FP64 FMA pipe --------------
// The recognised laws have the major symmetry T[(c,J),(k,L)] = T[(k,L),(c,J)], so the element
// matrix is symmetric and the blocks k >= c determine it. Their columns form one index j in [0, 162):
// pair p = 0..5 for (c, k) = (0,0) (0,1) (0,2) (1,1) (1,2) (2,2) and j = 27 p + m. The matrix of
// all six blocks, K_sym[n][j] = sum_r A^T[n][r] G[r][j] with G[(q,K)][j] = G_c[(q,K)][(k,m)], is
// one 27 x 162 x 3np product: 243 threads each hold a 3-row x 6-column tile of it in registers and,
// per k-step, read 3 values of A (9 distinct addresses per warp) and 6 of G (in 16-byte pairs,
// about 5 distinct column groups per warp) for 18 FMAs. G is built QC points at a time so that
// three CTAs share an SM; a thread builds three columns (m, m + 9, m + 18) of one pair and point
// from the pair's 3 x 3 block held in registers. The CTAs are persistent: each loads the reference
// tables once and then takes cell after cell. Against the tensor-core kernel above this forms
// 27 x 162 instead of 32 x 192 entries per k-step, on the FP64 FMA pipe, whose measured rate on
// B200 is above the FP64 MMA's.
#ifndef HFK_ASM_SYM27_QC
#define HFK_ASM_SYM27_QC 9  // points per G chunk (73 KB of shared memory per CTA at 27 points: 3 CTAs per SM)
#endif
#ifndef HFK_ASM_SYM27_MINB
#define HFK_ASM_SYM27_MINB 3  // CTAs per SM the register budget is sized for
#endif
#ifndef HFK_ASM_SYM27_MINB_TP
#define HFK_ASM_SYM27_MINB_TP 2  // the same for the tensor-product contraction (27 results per thread)
#endif
constexpr int ASM_SYM27_QC = HFK_ASM_SYM27_QC, ASM_SYM27_MINB = HFK_ASM_SYM27_MINB;
constexpr int ASM_SYM27_MINB_TP = HFK_ASM_SYM27_MINB_TP;
constexpr int SYM27_COLS = 162;
constexpr int SYM27_LDG = 164;  // row stride of the G chunk: even, so each row starts on 16 bytes
constexpr int SYM27_LDK = 29;   // column stride of the staged element blocks

// (c, k) of pair p and the first combined column of component c
__device__ __forceinline__ void sym27_pair(int p, int& c, int& k) {
  c = p < 3 ? 0 : (p < 5 ? 1 : 2);
  k = p < 3 ? p : (p < 5 ? p - 2 : 2);
}

// staged per cell after the doubles: its positions (81 x 81 from the 16-byte boundary at or below
// the first: at most 1641 pieces of 16 bytes) and the dof ids of this cell and the next
constexpr int SYM27_POS_INTS = 6568, SYM27_IDS_INTS = 84;
__host__ __device__ inline size_t sym27_g_offset(int np) { return ((size_t)181 * np + 91 + 1) & ~(size_t)1; }
inline size_t sym27_smem_bytes(int np, int qc) {
  return (sym27_g_offset(np) + (size_t)3 * qc * SYM27_LDG) * sizeof(double) +
         (SYM27_POS_INTS + 2 * SYM27_IDS_INTS) * sizeof(int32_t);
}


// the staged element blocks (162 columns of stride SYM27_LDK) fit over Dh and the G chunk
// (Dh starts 100 np + 91 doubles in; from there to the end: 81 np + the chunk, at least)
inline bool sym27_fits(int np, int qc) { return (size_t)81 * np + 3 * qc * SYM27_LDG >= (size_t)SYM27_COLS * SYM27_LDK; }

// TP: the cell's tables are the tensor product of the 1D tables tab (3 nodes and 3 Gauss points per
// direction, points in chunks of QC = 9, one z-layer each): the product is then a sum-factorised
// contraction per column (x and y within a chunk, z accumulated over the chunks), 729 FMAs per
// column instead of 2187, one thread per column with its 27 results in registers, reading only its
// own column of G.
template <bool TP, int QC, int MINB>
__global__ void __launch_bounds__(256, MINB) jacobian_kernel_sym27(CellData cd, AsmIO io, Tab1D<double> tab) {
  constexpr int NN = 27, NDL = 81, NT = 256;
  extern __shared__ __align__(16) double sm[];
  __shared__ int s_affine;
  const int np = io.np, R = 3 * np;
  double* A = sm;                       // (NN, 3, np): A[m + NN * (K + 3q)]
  double* xl = A + NN * R;              // NDL
  double* gs = xl + NDL;                // 10: the cell's affine geometry (iJt, |det|)
  double* Gq = gs + 10;                 // 9 np: reference gradient of u, Gq[q*9 + c*3 + K]
  double* iJs = Gq + 9 * np;            // 9 np
  double* dVs = iJs + 9 * np;           // np
  double* Dh = dVs + np;                // 81 np (the blocks k >= c)
  double* G = sm + sym27_g_offset(np);  // 3 QC rows x SYM27_LDG
  int32_t* posS = reinterpret_cast<int32_t*>(G + 3 * QC * SYM27_LDG);  // 16-byte aligned (even offsets)
  int32_t* idsS = posS + SYM27_POS_INTS;                                // two buffers of SYM27_IDS_INTS
  const int t = threadIdx.x;
  // the reference tables, once per CTA (four loads in flight per thread)
  {
    const int n = NN * R;
    int i = t;
    for (; i + 3 * NT < n; i += 4 * NT) {
      const double v0 = __ldg(io.dNt + i), v1 = __ldg(io.dNt + i + NT), v2 = __ldg(io.dNt + i + 2 * NT),
                   v3 = __ldg(io.dNt + i + 3 * NT);
      A[i] = v0;
      A[i + NT] = v1;
      A[i + 2 * NT] = v2;
      A[i + 3 * NT] = v3;
    }
    for (; i < n; i += NT) A[i] = __ldg(io.dNt + i);
  }
  static_assert(!TP || QC == 9, "the tensor-product contraction takes one z-layer of 3 x 3 points per chunk");
  const bool prod = t < 243;
  const int ig = t % 9, jg = t / 9;  // dense product tile: rows 3 ig .. 3 ig + 2, columns 6 jg .. 6 jg + 5
  // tensor-product contraction: column jt, 21 per warp so that every scheduler gets two warps
  const int jt = (t >> 5) * 21 + (t & 31);
  const bool tcol = (t & 31) < 21 && jt < SYM27_COLS;
  if (blockIdx.x < cd.ncells_list && t < NDL) {  // the first cell's dof ids
    const int cell0 = cd.cells ? cd.cells[blockIdx.x] : blockIdx.x;
    cp_async4(idsS + t, cd.ids + (size_t)cell0 * NDL + t);
  }
  cp_async_commit();
  int buf = 0;
  for (int li = blockIdx.x; li < cd.ncells_list; li += gridDim.x, buf ^= 1) {
    const int cell = cd.cells ? cd.cells[li] : li;
    cp_async_wait_all();
    __syncthreads();  // this cell's ids have arrived; the previous cell's scatter has read its positions
    // staged asynchronously while this cell is computed: the next cell's ids and this cell's positions
    const int lnext = li + gridDim.x;
    if (lnext < cd.ncells_list && t < NDL) {
      const int cn = cd.cells ? cd.cells[lnext] : lnext;
      cp_async4(idsS + SYM27_IDS_INTS * (buf ^ 1) + t, cd.ids + (size_t)cn * NDL + t);
    }
    const size_t pa = reinterpret_cast<size_t>(io.nzpos + (size_t)NDL * NDL * cell);
    const int pofs = (int)((pa & 15) >> 2);
    {
      const char* src = reinterpret_cast<const char*>(pa & ~(size_t)15);
      const int npiece = (int)(((pa & 15) + NDL * NDL * sizeof(int32_t) + 15) >> 4);
      for (int i = t; i < npiece; i += NT) cp_async16(posS + 4 * i, src + 16 * (size_t)i);
    }
    cp_async_commit();
    // the cell's values, its affine geometry and flag (the previous cell's readers of these are
    // behind at least three barriers)
    if (t < NDL) {
      const int32_t id = idsS[SYM27_IDS_INTS * buf + t];
      xl[t] = id > 0 ? io.u[id - 1] : (id < 0 ? io.dvals[-id - 1] : 0.0);
    } else if (t >= 96 && t < 106) {
      gs[t - 96] = cd.geo[(size_t)cell * 10 + (t - 96)];
    } else if (t == 128) {
      s_affine = cd.affine[cell];
    }
    __syncthreads();
    // reference gradient of u per point and component (one thread per entry), geometry per point
    for (int e = t; e < 9 * np; e += NT) {
      const int q = e / 9, cK = e - 9 * q, c = cK / 3, K = cK - 3 * c;
      const double* a = A + NN * (K + 3 * q);
      const double* x = xl + c * NN;
      double s0 = 0, s1 = 0, s2 = 0;
#pragma unroll
      for (int n = 0; n < NN; n += 3) {
        s0 += x[n] * a[n];
        s1 += x[n + 1] * a[n + 1];
        s2 += x[n + 2] * a[n + 2];
      }
      Gq[e] = s0 + s1 + s2;
    }
    const bool aff = s_affine != 0;
    for (int q = t; q < np; q += NT) {
      double Jt[9], iJ[9], det;
      if (aff) {
        for (int i = 0; i < 9; ++i) iJ[i] = gs[i];
        det = gs[9];
      } else {
        point_jacobian_dev(cd, cell, q, Jt);
        det = det3(Jt);
        inv3(Jt, det, iJ);
        det = fabs(det);
      }
      for (int i = 0; i < 9; ++i) iJs[q * 9 + i] = iJ[i];
      dVs[q] = cd.w[q] * det;
    }
    __syncthreads();
    // per (point, pair): the pulled-back tangent block Dh_q[(c,K),(k,K')]
    for (int e = t; e < 6 * np; e += NT) {
      const int q = e / 6;
      int c, k;
      sym27_pair(e - 6 * q, c, k);
      const double* iJ = iJs + q * 9;
      const double* g = Gq + q * 9;
      double H[9];  // H[c' + 3J] = sum_K iJ[J + 3K] Gq[c'][K]
#pragma unroll
      for (int cc = 0; cc < 3; ++cc)
#pragma unroll
        for (int J = 0; J < 3; ++J)
          H[cc + 3 * J] = iJ[J] * g[cc * 3] + iJ[J + 3] * g[cc * 3 + 1] + iJ[J + 6] * g[cc * 3 + 2];
      double Tb[9];
      law_tangent_block(cd.law, cd.lam_of(cell), cd.mu_of(cell), H, c, k, Tb);
      double X[3][3];
#pragma unroll
      for (int J = 0; J < 3; ++J)
#pragma unroll
        for (int Kp = 0; Kp < 3; ++Kp)
          X[J][Kp] = Tb[J] * iJ[3 * Kp] + Tb[J + 3] * iJ[1 + 3 * Kp] + Tb[J + 6] * iJ[2 + 3 * Kp];
      const double dV = dVs[q];
#pragma unroll
      for (int K = 0; K < 3; ++K)
#pragma unroll
        for (int Kp = 0; Kp < 3; ++Kp)
          Dh[q * 81 + (c * 3 + K) + 9 * (k * 3 + Kp)] =
              dV * (iJ[3 * K] * X[0][Kp] + iJ[1 + 3 * K] * X[1][Kp] + iJ[2 + 3 * K] * X[2][Kp]);
    }
    __syncthreads();
    double acc[3][6];  // dense product
    double out[27];    // tensor-product contraction: column jt of the element blocks
#pragma unroll
    for (int s = 0; s < 3; ++s)
#pragma unroll
      for (int h = 0; h < 6; ++h) acc[s][h] = 0.0;
#pragma unroll
    for (int i = 0; i < 27; ++i) out[i] = 0.0;
    for (int q0 = 0; q0 < np; q0 += QC) {
      const int nq = min(QC, np - q0);
      // G rows 3 (q - q0) + K, columns 27 p + m: sum_K' Dh_q[(c,K),(k,K')] dN^[m,K',q]; a thread
      // takes one point and pair and the nodes m = mg, mg + 9, mg + 18
      for (int e = t; e < nq * 54; e += NT) {
        const int mg = e % 9, rest = e / 9, pr = rest % 6, qq = rest / 6;
        int c, k;
        sym27_pair(pr, c, k);
        const int q = q0 + qq;
        const double* D = Dh + q * 81 + c * 3 + 27 * k;  // D[K + 9 K'] = Dh_q[(c,K),(k,K')]
        const double* a = A + mg + NN * 3 * q;
        double av[3][3];  // av[i][K'] = dN^[mg + 9 i, K', q]
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int Kp = 0; Kp < 3; ++Kp) av[i][Kp] = a[9 * i + NN * Kp];
        double* g = G + 3 * qq * SYM27_LDG + 27 * pr + mg;
#pragma unroll
        for (int K = 0; K < 3; ++K) {
          const double d0 = D[K], d1 = D[K + 9], d2 = D[K + 18];
#pragma unroll
          for (int i = 0; i < 3; ++i) g[K * SYM27_LDG + 9 * i] = d0 * av[i][0] + d1 * av[i][1] + d2 * av[i][2];
        }
      }
      __syncthreads();
      if (TP && tcol) {
        // out[n1 + 3 n2 + 9 n3] += sum_K sum_{q1,q2} Tx(n1,q1) Ty(n2,q2) Tz(n3,q3) G[(q,K)][jt], with T
        // the derivative table in direction K and the basis table in the others (T(n, q) = N1[3q + n])
        const int q3 = q0 / 9;
#pragma unroll
        for (int K = 0; K < 3; ++K) {
          const double* Tx = K == 0 ? tab.dN1 : tab.N1;
          const double* Ty = K == 1 ? tab.dN1 : tab.N1;
          const double* Tz = K == 2 ? tab.dN1 : tab.N1;
          double g[9];  // g[q1 + 3 q2]
#pragma unroll
          for (int i = 0; i < 9; ++i) g[i] = G[(3 * i + K) * SYM27_LDG + jt];
          double sx[9];  // sx[n1 + 3 q2]
#pragma unroll
          for (int q2 = 0; q2 < 3; ++q2)
#pragma unroll
            for (int n1 = 0; n1 < 3; ++n1)
              sx[n1 + 3 * q2] = Tx[n1] * g[3 * q2] + Tx[3 + n1] * g[1 + 3 * q2] + Tx[6 + n1] * g[2 + 3 * q2];
#pragma unroll
          for (int n2 = 0; n2 < 3; ++n2)
#pragma unroll
            for (int n1 = 0; n1 < 3; ++n1) {
              const double u = Ty[n2] * sx[n1] + Ty[3 + n2] * sx[n1 + 3] + Ty[6 + n2] * sx[n1 + 6];
#pragma unroll
              for (int n3 = 0; n3 < 3; ++n3) out[n1 + 3 * n2 + 9 * n3] += Tz[3 * q3 + n3] * u;
            }
        }
      }
      if (!TP && prod) {
        const double* Ar = A + 3 * ig + NN * 3 * q0;
        const double* Gr = G + 6 * jg;
#pragma unroll 3
        for (int rr = 0; rr < 3 * nq; ++rr) {
          const double a[3] = {Ar[0], Ar[1], Ar[2]};
          const double2 b01 = *reinterpret_cast<const double2*>(Gr);
          const double2 b23 = *reinterpret_cast<const double2*>(Gr + 2);
          const double2 b45 = *reinterpret_cast<const double2*>(Gr + 4);
          const double b[6] = {b01.x, b01.y, b23.x, b23.y, b45.x, b45.y};
#pragma unroll
          for (int s = 0; s < 3; ++s)
#pragma unroll
            for (int h = 0; h < 6; ++h) acc[s][h] += a[s] * b[h];
          Ar += NN;
          Gr += SYM27_LDG;
        }
      }
      __syncthreads();
    }
    // the element blocks into shared memory, over Dh and the G chunk (both dead now), column by
    // column: Kt[j * SYM27_LDK + n] (odd stride: both scatter loops below read it without conflicts)
    double* Kt = Dh;
    if (TP && tcol)
#pragma unroll
      for (int n = 0; n < 27; ++n) Kt[jt * SYM27_LDK + n] = out[n];
    if (!TP && prod)
#pragma unroll
      for (int h = 0; h < 6; ++h)
#pragma unroll
        for (int s = 0; s < 3; ++s) Kt[(6 * jg + h) * SYM27_LDK + 3 * ig + s] = acc[s][h];
    cp_async_wait_all();  // the positions
    __syncthreads();
    // scatter: entry (n, c) x (m, k) at its position, n fastest (27 consecutive positions of one
    // CSC column per 27 threads); then the blocks k > c at the transposed positions, m fastest
    const int32_t* pos = posS + pofs;
#pragma unroll 4
    for (int e = t; e < NN * SYM27_COLS; e += NT) {
      const int j = e / NN, n = e - NN * j, pr = j / NN, m = j - NN * pr;
      int c, k;
      sym27_pair(pr, c, k);
      scatter_add(io.nzval, pos[(c * NN + n) + NDL * (k * NN + m)], Kt[j * SYM27_LDK + n]);
    }
#pragma unroll 4
    for (int e = t; e < NN * NN * 3; e += NT) {
      const int m = e % NN, rest = e / NN, n = rest % NN, b = rest / NN;
      const int pr = b == 0 ? 1 : (b == 1 ? 2 : 4);  // (0,1) (0,2) (1,2)
      int c, k;
      sym27_pair(pr, c, k);
      scatter_add(io.nzval, pos[(k * NN + m) + NDL * (c * NN + n)], Kt[(NN * pr + m) * SYM27_LDK + n]);
    }
  }
}

// Small cells (Q1, any number of points): one thread per element entry
template <int NN>
__global__ void __launch_bounds__(256) jacobian_kernel_direct(CellData cd, AsmIO io) {
  constexpr int NDL = 3 * NN;
  extern __shared__ __align__(16) double sm[];
  const int np = io.np;
  double* A = sm;
  double* xl = A + NN * 3 * np;
  double* Hs = xl + NDL;
  double* iJs = Hs + 9 * np;
  double* dVs = iJs + 9 * np;
  double* Dh = dVs + np;
  const int li = blockIdx.x;
  if (li >= cd.ncells_list) return;
  const int cell = cd.cells ? cd.cells[li] : li;
  const int32_t* gid = cd.ids + (size_t)cell * NDL;
  for (int i = threadIdx.x; i < NN * 3 * np; i += blockDim.x) A[i] = io.dNt[i];
  for (int j = threadIdx.x; j < NDL; j += blockDim.x) {
    const int32_t id = gid[j];
    xl[j] = id > 0 ? io.u[id - 1] : (id < 0 ? io.dvals[-id - 1] : 0.0);
  }
  __syncthreads();
  asm_point_phase<NN>(cd, io, cell, A, xl, Hs, iJs, dVs, Dh);
  const int32_t* pos = io.nzpos + (size_t)NDL * NDL * cell;
  for (int e = threadIdx.x; e < NDL * NDL; e += blockDim.x) {
    const int ii = e % NDL, jj = e / NDL;
    const int c = ii / NN, n = ii % NN, k = jj / NN, m = jj % NN;
    const int32_t pe = __ldg(pos + ii + NDL * jj);  // loaded first: its latency overlaps the sum
    double acc = 0;
    for (int q = 0; q < np; ++q) {
      const double* D = Dh + q * 81;
      double an[3], am[3];
      for (int K = 0; K < 3; ++K) {
        an[K] = A[n + NN * (K + 3 * q)];
        am[K] = A[m + NN * (K + 3 * q)];
      }
      for (int K = 0; K < 3; ++K) {
        const double* Dk = D + (c * 3 + K) + 9 * (k * 3);
        acc += an[K] * (Dk[0] * am[0] + Dk[9] * am[1] + Dk[18] * am[2]);
      }
    }
    scatter_add(io.nzval, pe, acc);
  }
}

// with_g: G_c with row stride ldg and the rows of the padded k dimension (3 np rounded up to 4)
inline size_t asm_smem_bytes(int nn, int np, bool with_g, int ldg) {
  size_t v = (size_t)nn * 3 * np + 3 * nn + 9 * np + 9 * np + np + 81 * np;
  if (with_g) v += (size_t)((3 * np + 3) / 4 * 4) * ldg;
  return v * sizeof(double);
}

}  // namespace hfk
