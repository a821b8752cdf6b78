// Cholesky factorisation of the assembled coarse level in band storage, and the triangular tile
// solves that turn the factor into the block triangular solves' D^-1 L tiles (kern_band.cuh).
//
// The coarse p = 1 level is solved directly in the reference (Gridap's LU of the assembled matrix,
// src/pmultigrid.jl:97-98, :206-211). Its matrix is symmetric positive definite and banded in the
// node-major numbering (lower bandwidth b ~ 3 (n_x n_y + n_x + 1) dofs), and a Cholesky factor keeps
// the band, so only the band is stored and factored: CB_T x CB_T tiles (i, j) with j <= i <= j + W,
// W = ceil(b / CB_T), block column after block column, each tile column-major. Rows past n are
// padded with the identity. Memory is (n / CB_T) (W + 1) CB_T^2 doubles, about n (b + CB_T), instead
// of n^2: a Q1 32^3 coarse level (101 277 dofs, b = 3 369) takes 2.9 GB.
//
// Right-looking blocked factorisation, two launches per block column k:
//   panel k:  the update of block column k by block column k - 1, then tile (k, k) <- chol(A_kk)
//             (every CTA of the launch updates and factors it in shared memory; CTA 0 stores it),
//             tile (k + q, k) <- A_{k+q,k} L_kk^-T (CTA q >= 1);
//   update k: tile (i, j) -= L_ik L_jk^T for k + 1 < j <= i <= k + W (one CTA per tile), on a
//             second stream, where it overlaps panel k + 1.
// A pivot that is not positive and finite records the block column (1-based) in *info (the first
// one wins) and is replaced by 1 so that the remaining work stays finite; the host rejects the
// factor.
#pragma once
#include <cstdint>

namespace hfk {

constexpr int CB_T = 64;         // tile size of the band storage
constexpr int CB_THREADS = 256;  // threads per CTA of the factorisation kernels
constexpr int CB_LD = CB_T + 1;  // padded leading dimension of a tile in shared memory
constexpr int CB_LDU = CB_T + 4;  // the same for the trailing update's tiles: the 8 x 4 fragments of
                                  // each half-warp fall on distinct banks

// offset (in doubles) of tile (i, j), j <= i <= j + W, in the band storage
__host__ __device__ inline size_t band_tile_offset(int i, int j, int W) {
  return ((size_t)j * (W + 1) + (size_t)(i - j)) * (size_t)(CB_T * CB_T);
}

// The lower triangle of the CSC matrix (colptr, rowval 1-based, Julia's) into the zeroed band
// storage, and the identity on the padding rows n .. nbt CB_T - 1.
static __global__ void band_fill_kernel(int64_t n, int nbt, int W, const int64_t* __restrict__ colptr,
                                        const int64_t* __restrict__ rowval, const double* __restrict__ nzval,
                                        double* __restrict__ Lb) {
  const int64_t npad = (int64_t)nbt * CB_T;
  for (int64_t c = blockIdx.x; c < npad; c += gridDim.x) {
    if (c >= n) {
      if (threadIdx.x == 0) {
        const int j = (int)(c / CB_T), jj = (int)(c % CB_T);
        Lb[band_tile_offset(j, j, W) + jj + (size_t)CB_T * jj] = 1.0;
      }
      continue;
    }
    const int j = (int)(c / CB_T), jj = (int)(c % CB_T);
    for (int64_t k = colptr[c] - 1 + threadIdx.x; k < colptr[c + 1] - 1; k += blockDim.x) {
      const int64_t r = rowval[k] - 1;
      if (r < c) continue;
      const int i = (int)(r / CB_T), ii = (int)(r % CB_T);
      if (i - j <= W) Lb[band_tile_offset(i, j, W) + ii + (size_t)CB_T * jj] = nzval[k];
    }
  }
}

// A CB_T x CB_T tile between global memory (contiguous, column-major) and shared memory (leading
// dimension CB_LD), by NT threads: 16-byte global accesses, the loop unrolled so that every
// thread's loads are in flight together (the tiles are read on the factorisation's critical path).
template <int NT, int LD = CB_LD>
__device__ __forceinline__ void tile_to_shared(double* S, const double* __restrict__ G, int tid) {
  constexpr int N2 = CB_T * CB_T / 2;
  static_assert(N2 % NT == 0, "whole pairs per thread");
  double2 v[N2 / NT];
#pragma unroll
  for (int k = 0; k < N2 / NT; ++k) v[k] = reinterpret_cast<const double2*>(G)[tid + NT * k];
#pragma unroll
  for (int k = 0; k < N2 / NT; ++k) {
    const int e = 2 * (tid + NT * k), r = e % CB_T, c = e / CB_T;  // r even: r + 1 in the same column
    S[r + LD * c] = v[k].x;
    S[r + 1 + LD * c] = v[k].y;
  }
}
template <int NT, bool LOWER>
__device__ __forceinline__ void tile_to_global(double* __restrict__ G, const double* S, int tid) {
  constexpr int N2 = CB_T * CB_T / 2;
#pragma unroll 8
  for (int k = 0; k < N2 / NT; ++k) {
    const int e = 2 * (tid + NT * k), r = e % CB_T, c = e / CB_T;
    double2 v;
    v.x = (!LOWER || r >= c) ? S[r + CB_LD * c] : 0.0;
    v.y = (!LOWER || r + 1 >= c) ? S[r + 1 + CB_LD * c] : 0.0;
    reinterpret_cast<double2*>(G)[tid + NT * k] = v;
  }
}

// S -= Li Lj^T for CB_T x CB_T tiles in shared memory (leading dimension CB_LD), by 128 threads on
// the FP64 tensor cores (mma.sync m8n8k4): warp w the rows 16 w .. 16 w + 15 (two 8-row bands), all
// eight 8-column tiles; lane l holds fragment entries (row l / 4, k l % 4) and accumulator entries
// (row l / 4, columns 2 (l % 4), + 1). lower: only the lower triangle of S is written.
__device__ __forceinline__ void tile_sub_prod128(double* S, const double* Li, const double* Lj, int tid, bool lower) {
  const int warp = tid >> 5, lane = tid & 31, fr = lane >> 2, fc = lane & 3;
  double acc[2][8][2];
#pragma unroll
  for (int rb = 0; rb < 2; ++rb)
#pragma unroll
    for (int t = 0; t < 8; ++t) acc[rb][t][0] = acc[rb][t][1] = 0.0;
#pragma unroll 2
  for (int m = 0; m < CB_T; m += 4) {
    double a[2];
#pragma unroll
    for (int rb = 0; rb < 2; ++rb) a[rb] = Li[(16 * warp + 8 * rb + fr) + CB_LD * (m + fc)];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      const double b = Lj[(8 * t + fr) + CB_LD * (m + fc)];
#pragma unroll
      for (int rb = 0; rb < 2; ++rb)
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                     : "+d"(acc[rb][t][0]), "+d"(acc[rb][t][1])
                     : "d"(a[rb]), "d"(b));
    }
  }
  // S is neither Li nor Lj: its entries are written without waiting for the other warps
#pragma unroll
  for (int rb = 0; rb < 2; ++rb)
#pragma unroll
    for (int t = 0; t < 8; ++t)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = 16 * warp + 8 * rb + fr, c = 8 * t + 2 * fc + h;
        if (!lower || r >= c) S[r + CB_LD * c] -= acc[rb][t][h];
      }
}

constexpr int CB_PANEL_THREADS = 128;
constexpr int CB_PB = 16;  // columns per block of the panel

// S[r][c] -= sum_{j < 16} P[r][p0 + j] Q[c][p0 + j] for r0 <= r < CB_T, t0 <= c < CB_T (r0 and t0
// multiples of 8; tiles in shared memory, leading dimension CB_LD), by 128 threads on the FP64 tensor
// cores: the 8 x 8 output tiles round-robin over the 4 warps, 4 MMAs each. lower: tiles above the
// diagonal skipped, diagonal tiles written below it only. S's columns t0.. never overlap the read
// columns p0 .. p0 + 15.
__device__ __forceinline__ void panel_rank16_dmma(double* S, const double* P, const double* Q, int p0, int r0, int t0,
                                                  int tid, bool lower) {
  const int warp = tid >> 5, lane = tid & 31, fr = lane >> 2, fc = lane & 3;
  const int nr = (CB_T - r0) / 8, nt = nr * ((CB_T - t0) / 8);
  for (int e = warp; e < nt; e += CB_PANEL_THREADS / 32) {
    const int tr = e % nr, tc = e / nr;
    const int rb = r0 + 8 * tr, cb = t0 + 8 * tc;
    if (lower && rb + 7 < cb) continue;  // above the diagonal (uniform over the warp)
    double d0 = 0.0, d1 = 0.0;
#pragma unroll
    for (int j = 0; j < CB_PB; j += 4) {
      const double a = P[(rb + fr) + CB_LD * (p0 + j + fc)];
      const double b = Q[(cb + fr) + CB_LD * (p0 + j + fc)];
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                   : "+d"(d0), "+d"(d1)
                   : "d"(a), "d"(b));
    }
    const int r = rb + fr, c = cb + 2 * fc;
    if (!lower || r >= c) S[r + CB_LD * c] -= d0;
    if (!lower || r >= c + 1) S[r + CB_LD * (c + 1)] -= d1;
  }
}

// Panel k, blocked by 16 columns, the tile in shared memory (CB_PANEL_THREADS threads). Per block of
// 16 columns: (1) one warp factors the 16 x 16 diagonal block, row i in lane i's registers, the
// pivots and multipliers passed by shuffles (no barrier inside: the chain of dependent pivots is
// the critical path of the whole factorisation, so it runs at warp latency, with one reciprocal
// square root per pivot); (2) the rows below are solved against it, one thread per row; (3) the
// trailing lower triangle takes the block's rank-16 update. Every CTA of the launch factors the
// tile (no CTA waits for another); CTA 0 stores it. CTA q >= 1 then solves X L_kk^T = A_{k+q,k} by
// the same blocks: a block of 16 columns of X, then the update of X's later columns.
// A pivot that is not positive and finite records k + 1 in *info and is replaced by 1.

// fuse: block column k first takes its update by block column k - 1 (the tiles (k + q, k) -= L_{k+q,k-1}
// L_{k,k-1}^T, the diagonal one by every CTA, as it factors it), so that no separate launch sits
// between two panels on the factorisation's critical path; four tiles of shared memory then.
static __global__ void __launch_bounds__(CB_PANEL_THREADS) band_panel_kernel(int nbt, int W, int k, double* Lb,
                                                                             int* info, int fuse) {
  extern __shared__ __align__(16) double cbs[];
  double* A = cbs;                 // the diagonal tile, becoming L_kk (column-major, leading dimension CB_LD)
  double* X = cbs + CB_T * CB_LD;  // the panel tile below (CTA q >= 1)
  double* Ld = X + CB_T * CB_LD;   // fuse: L_{k,k-1}
  double* Lq = Ld + CB_T * CB_LD;  // fuse: L_{k+q,k-1}
  __shared__ double s_inv[CB_T];   // reciprocals of L_kk's diagonal
  __shared__ int s_bad;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, q = blockIdx.x;
  double* Akk = Lb + band_tile_offset(k, k, W);
  double* Aik = Lb + band_tile_offset(k + q, k, W);
  const bool fz = fuse && k > 0 && W >= 1;
  const bool fq = fz && q >= 1 && q + 1 <= W;  // tile (k + q, k - 1) lies in the band
  tile_to_shared<CB_PANEL_THREADS>(A, Akk, tid);
  if (q >= 1) tile_to_shared<CB_PANEL_THREADS>(X, Aik, tid);
  if (fz) tile_to_shared<CB_PANEL_THREADS>(Ld, Lb + band_tile_offset(k, k - 1, W), tid);
  if (fq) tile_to_shared<CB_PANEL_THREADS>(Lq, Lb + band_tile_offset(k + q, k - 1, W), tid);
  if (tid == 0) s_bad = 0;
  __syncthreads();
  if (fz) {
    tile_sub_prod128(A, Ld, Ld, tid, true);
    if (fq) tile_sub_prod128(X, Lq, Ld, tid, false);
    __syncthreads();
  }
#pragma unroll 1
  for (int p0 = 0; p0 < CB_T; p0 += CB_PB) {
    // (1) the diagonal block, by warp 0
    if (warp == 0) {
      const int i = lane & (CB_PB - 1);
      double b[CB_PB];
#pragma unroll
      for (int c = 0; c < CB_PB; ++c) b[c] = c <= i ? A[(p0 + i) + CB_LD * (p0 + c)] : 0.0;
      bool ok = true;
#pragma unroll
      for (int c = 0; c < CB_PB; ++c) {
        const double piv = __shfl_sync(0xffffffffu, b[c], c);
        const bool good = piv > 0.0 && piv < INFINITY;  // NaN fails both comparisons
        ok = ok && good;
        const double pv = good ? piv : 1.0;
        const double iv = rsqrt(pv);
        const double l = i > c ? b[c] * iv : (i == c ? pv * iv : 0.0);
        b[c] = l;
        if (lane == 0) s_inv[p0 + c] = iv;
        // a constant trip count with a predicate (not s2 = c + 1 ..): the loops unroll completely
        // and b stays in registers
#pragma unroll
        for (int s2 = 0; s2 < CB_PB; ++s2) {
          if (s2 > c) {
            const double ls = __shfl_sync(0xffffffffu, l, s2);
            if (i >= s2) b[s2] = fma(-l, ls, b[s2]);
          }
        }
      }
      if (lane < CB_PB) {
#pragma unroll
        for (int c = 0; c < CB_PB; ++c)
          if (c <= i) A[(p0 + i) + CB_LD * (p0 + c)] = b[c];
      }
      if (!ok && lane == 0) s_bad = 1;
    }
    __syncthreads();
    // (2) the rows below the block: x L_pp^T = a, one thread per row
    const int r = p0 + CB_PB + tid;
    if (r < CB_T) {
      double x[CB_PB];
#pragma unroll
      for (int c = 0; c < CB_PB; ++c) x[c] = A[r + CB_LD * (p0 + c)];
#pragma unroll
      for (int c = 0; c < CB_PB; ++c) {
        const double v = x[c] * s_inv[p0 + c];
        x[c] = v;
#pragma unroll
        for (int s2 = 0; s2 < CB_PB; ++s2)
          if (s2 > c) x[s2] = fma(-v, A[(p0 + s2) + CB_LD * (p0 + c)], x[s2]);
      }
#pragma unroll
      for (int c = 0; c < CB_PB; ++c) A[r + CB_LD * (p0 + c)] = x[c];
    }
    __syncthreads();
    // (3) rank-16 update of the trailing lower triangle (FP64 tensor cores)
    const int t0 = p0 + CB_PB;
    if (t0 < CB_T) panel_rank16_dmma(A, A, A, p0, t0, t0, tid, true);
    __syncthreads();
  }
  if (q == 0) {
    if (s_bad && tid == 0) atomicCAS(info, 0, k + 1);
    tile_to_global<CB_PANEL_THREADS, true>(Akk, A, tid);
    return;
  }
#pragma unroll 1
  for (int p0 = 0; p0 < CB_T; p0 += CB_PB) {
    // the block of 16 columns of X: row r solves x L_pp^T = a
    if (tid < CB_T) {
      double x[CB_PB];
#pragma unroll
      for (int c = 0; c < CB_PB; ++c) x[c] = X[tid + CB_LD * (p0 + c)];
#pragma unroll
      for (int c = 0; c < CB_PB; ++c) {
        const double v = x[c] * s_inv[p0 + c];
        x[c] = v;
#pragma unroll
        for (int s2 = 0; s2 < CB_PB; ++s2)
          if (s2 > c) x[s2] = fma(-v, A[(p0 + s2) + CB_LD * (p0 + c)], x[s2]);
      }
#pragma unroll
      for (int c = 0; c < CB_PB; ++c) X[tid + CB_LD * (p0 + c)] = x[c];
    }
    __syncthreads();
    // the later columns of X: X[r][s] -= sum_c X[r][p0 + c] L[s][p0 + c] (FP64 tensor cores)
    const int t0 = p0 + CB_PB;
    if (t0 < CB_T) panel_rank16_dmma(X, X, A, p0, 0, t0, tid, false);
    __syncthreads();
  }
  tile_to_global<CB_PANEL_THREADS, false>(Aik, X, tid);
}

// Update k: tile (i, j) -= L_ik L_jk^T for the m (m + 1) / 2 tiles k < j <= i <= k + m (m = min(W,
// nbt - 1 - k)); CTA b takes the b-th tile in the order (i, j) = (k+1, k+1), (k+2, k+1), (k+2, k+2),
// ... part = 2 takes only the tiles j >= k + 2 (in the same order over that smaller triangle; block
// column k + 1 is updated inside the next panel launch), 0 all. Each warp forms 8 rows of the
// product on the FP64 tensor cores. On a diagonal tile only the lower triangle is written. Dynamic
// shared memory: two tiles of leading dimension CB_LDU.
static __global__ void __launch_bounds__(CB_THREADS) band_update_kernel(int nbt, int W, int k, double* Lb, int part) {
  extern __shared__ __align__(16) double cbs[];
  double* Li = cbs;
  double* Lj = cbs + CB_T * CB_LDU;
  const int tid = threadIdx.x;
  // b -> (ii, jj), jj <= ii: ii (ii + 1) / 2 <= b < (ii + 1) (ii + 2) / 2
  const int b = blockIdx.x;
  int ii = (int)((sqrt(8.0 * b + 1.0) - 1.0) * 0.5);
  while ((ii + 1) * (ii + 2) / 2 <= b) ++ii;
  while (ii * (ii + 1) / 2 > b) --ii;
  int jj = b - ii * (ii + 1) / 2;
  if (part == 2) {
    ++ii;
    ++jj;
  }
  const int i = k + 1 + ii, j = k + 1 + jj;
  const double* Lik = Lb + band_tile_offset(i, k, W);
  const double* Ljk = Lb + band_tile_offset(j, k, W);
  tile_to_shared<CB_THREADS, CB_LDU>(Li, Lik, tid);
  tile_to_shared<CB_THREADS, CB_LDU>(Lj, Ljk, tid);
  __syncthreads();
  // L_ik L_jk^T on the FP64 tensor cores (mma.sync m8n8k4): warp w the rows 8w .. 8w + 7, all eight
  // 8-column tiles; per k-step of 4 one fragment of L_ik and eight of L_jk (the same index pattern:
  // lane l holds entry (8 t + l / 4, m + l % 4) of its tile)
  const int warp = tid >> 5, lane = tid & 31, fr = lane >> 2, fc = lane & 3;
  double acc[8][2];
#pragma unroll
  for (int t = 0; t < 8; ++t) acc[t][0] = acc[t][1] = 0.0;
#pragma unroll 4
  for (int m = 0; m < CB_T; m += 4) {
    const double a = Li[(8 * warp + fr) + CB_LDU * (m + fc)];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      const double b = Lj[(8 * t + fr) + CB_LDU * (m + fc)];
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                   : "+d"(acc[t][0]), "+d"(acc[t][1])
                   : "d"(a), "d"(b));
    }
  }
  double* Aij = Lb + band_tile_offset(i, j, W);
  const int r = 8 * warp + fr;
#pragma unroll
  for (int t = 0; t < 8; ++t)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int c = 8 * t + 2 * fc + h;
      if (i != j || r >= c) Aij[r + (size_t)CB_T * c] -= acc[t][h];
    }
}

// Entry (r, c), r >= c, of the band factor (zero outside the band)
__device__ inline double band_entry(const double* Lb, int W, int64_t r, int64_t c) {
  const int i = (int)(r / CB_T), j = (int)(c / CB_T);
  if (i - j > W || r < c) return 0.0;
  return Lb[band_tile_offset(i, j, W) + (r % CB_T) + (size_t)CB_T * (c % CB_T)];
}

// x <- D_hh^-1 x for one half (rows r0 .. r0 + H - 1) of a column, D_hh the half's diagonal block
// of the triangular D in shared memory (column-major, leading dimension BS): forward (lower) or
// backward (upper) substitution, right-looking, the column half in registers.
template <int BS, int H>
__device__ __forceinline__ void trsm_half(double (&x)[H], const double* Ds, const double* dinv, int r0, bool upper) {
  if (!upper) {
#pragma unroll
    for (int c = 0; c < H; ++c) {
      const double v = x[c] * dinv[r0 + c];
      x[c] = v;
#pragma unroll
      for (int s2 = c + 1; s2 < H; ++s2) x[s2] = fma(-v, Ds[(r0 + s2) + BS * (r0 + c)], x[s2]);
    }
  } else {
#pragma unroll
    for (int c = H - 1; c >= 0; --c) {
      const double v = x[c] * dinv[r0 + c];
      x[c] = v;
#pragma unroll
      for (int s2 = 0; s2 < c; ++s2) x[s2] = fma(-v, Ds[(r0 + s2) + BS * (r0 + c)], x[s2]);
    }
  }
}

// In place X <- D^-1 X for every tile of the block triangular solves (kern_band.cuh layout: 2 nb
// steps of wt + 1 tiles of BS x BS, diag holding D of each step: lower for the forward direction,
// upper for the backward one). One CTA per tile, D in shared memory, two threads per column of the
// tile, one per half of it, the half in registers: the half that comes first (top for forward,
// bottom for backward) is solved with its diagonal block and published in shared memory, then the
// other half subtracts its coupling to it and is solved with its own diagonal block. The reads of D
// are uniform over each warp (both halves of a warp's columns run the same instruction stream).
template <int BS>
static __global__ void __launch_bounds__(2 * BS) tile_trsm_kernel(int nb, int wt, const double* __restrict__ diag,
                                                                   double* __restrict__ tiles) {
  constexpr int H = BS / 2;
  extern __shared__ __align__(16) double trs[];
  double* Ds = trs;               // BS x BS, column-major
  double* Xs = trs + BS * BS;     // H x BS: the first half solved, Xs[m * BS + j]
  double* dinv = Xs + H * BS;     // BS reciprocals of the diagonal
  const int64_t tt = (int64_t)BS * BS;
  const int64_t tile = blockIdx.x;  // d * nb * (wt + 1) + s * (wt + 1) + t
  const int64_t ds = tile / (wt + 1);
  const bool upper = ds / nb != 0;
  const double* Dk = diag + ds * tt;
  double* X = tiles + tile * tt;
  const int tid = threadIdx.x;
  for (int e = tid; e < BS * BS; e += blockDim.x) Ds[e] = Dk[e];
  for (int e = tid; e < BS; e += blockDim.x) dinv[e] = 1.0 / Dk[e + (int64_t)BS * e];
  __syncthreads();
  const int j = tid % BS, h = tid / BS;
  const int first = upper ? 1 : 0;
  const int r0 = h * H;
  double x[H];
  if (h == first) {
#pragma unroll
    for (int i = 0; i < H; ++i) x[i] = X[(r0 + i) + (int64_t)BS * j];
    trsm_half<BS, H>(x, Ds, dinv, r0, upper);
#pragma unroll
    for (int i = 0; i < H; ++i) {
      Xs[i * BS + j] = x[i];
      X[(r0 + i) + (int64_t)BS * j] = x[i];
    }
  }
  __syncthreads();
  if (h != first) {
    const int m0 = first * H;
#pragma unroll
    for (int i = 0; i < H; ++i) x[i] = X[(r0 + i) + (int64_t)BS * j];
    for (int m = 0; m < H; ++m) {
      const double xm = Xs[m * BS + j];
#pragma unroll
      for (int i = 0; i < H; ++i) x[i] = fma(-Ds[(r0 + i) + BS * (m0 + m)], xm, x[i]);
    }
    trsm_half<BS, H>(x, Ds, dinv, r0, upper);
#pragma unroll
    for (int i = 0; i < H; ++i) X[(r0 + i) + (int64_t)BS * j] = x[i];
  }
}

}  // namespace hfk
