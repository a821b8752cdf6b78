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
//   panel k:  tile (k, k) <- chol(A_kk) (every CTA of the launch factors it in shared memory; CTA 0
//             stores it), tile (k + q, k) <- A_{k+q,k} L_kk^-T (CTA q >= 1);
//   update k: tile (i, j) -= L_ik L_jk^T for k < j <= i <= k + W (one CTA per tile).
// A pivot that is not positive and finite records the block column (1-based) in *info (the first
// one wins) and is replaced by 1 so that the remaining work stays finite; the host rejects the
// factor.
#pragma once
#include <cstdint>

namespace hfk {

constexpr int CB_T = 64;         // tile size of the band storage
constexpr int CB_THREADS = 256;  // threads per CTA of the factorisation kernels
constexpr int CB_LD = CB_T + 1;  // padded leading dimension of a tile in shared memory

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

// Cholesky factor of the CB_T x CB_T tile in shared memory D (column-major, leading dimension
// CB_LD, lower triangle used), in place, unblocked and right-looking: per column, the pivot's
// square root, the column scaled below it, the trailing lower triangle updated by the column's
// outer product. Returns (uniform over the CTA) whether every pivot was positive and finite.
__device__ inline bool tile_cholesky(double* D) {
  const int tid = threadIdx.x;
  bool ok = true;
  for (int c = 0; c < CB_T; ++c) {
    __syncthreads();  // the previous column's trailing update is complete
    const double piv = D[c + CB_LD * c];
    const bool good = piv > 0.0 && piv < INFINITY;  // NaN fails both comparisons
    ok = ok && good;
    const double d = sqrt(good ? piv : 1.0);
    const double inv = 1.0 / d;
    for (int r = c + 1 + tid; r < CB_T; r += blockDim.x) D[r + CB_LD * c] *= inv;
    __syncthreads();
    // the diagonal entry is written here: the trailing update below never reads it
    if (tid == 0) D[c + CB_LD * c] = d;
    // trailing update: thread (r, s group) over the columns s = c+1+g, c+1+g+G, ... and row r >= s
    constexpr int G = CB_THREADS / CB_T;
    const int r = tid % CB_T;
    const double lr = r > c ? D[r + CB_LD * c] : 0.0;
    for (int s = c + 1 + tid / CB_T; s < CB_T; s += G)
      if (r >= s) D[r + CB_LD * s] -= lr * D[s + CB_LD * c];
  }
  __syncthreads();
  return ok;
}

// Panel k: CTA 0 stores chol(A_kk); CTA q >= 1 solves X L_kk^T = A_{k+q,k} for the tile below.
// Dynamic shared memory: two tiles of CB_T x CB_LD doubles.
static __global__ void __launch_bounds__(CB_THREADS) band_panel_kernel(int nbt, int W, int k, double* Lb, int* info) {
  extern __shared__ __align__(16) double cbs[];
  double* D = cbs;                  // L_kk
  double* X = cbs + CB_T * CB_LD;   // the panel tile
  const int tid = threadIdx.x, q = blockIdx.x;
  double* Akk = Lb + band_tile_offset(k, k, W);
  for (int e = tid; e < CB_T * CB_T; e += blockDim.x) D[(e % CB_T) + CB_LD * (e / CB_T)] = Akk[e];
  __syncthreads();
  const bool ok = tile_cholesky(D);
  if (q == 0) {
    if (!ok && tid == 0) atomicCAS(info, 0, k + 1);
    for (int e = tid; e < CB_T * CB_T; e += blockDim.x) {
      const int r = e % CB_T, c = e / CB_T;
      Akk[e] = r >= c ? D[r + CB_LD * c] : 0.0;
    }
    return;
  }
  const int i = k + q;
  double* Aik = Lb + band_tile_offset(i, k, W);
  for (int e = tid; e < CB_T * CB_T; e += blockDim.x) X[(e % CB_T) + CB_LD * (e / CB_T)] = Aik[e];
  __syncthreads();
  // row r of X: X[r][c] = (A[r][c] - sum_{m<c} X[r][m] L[c][m]) / L[c][c], in place; four threads per
  // row (h = 0..3) each sum the columns m = h, h + 4, ... and combine by shuffles within the warp
  const int r = tid >> 2, h = tid & 3;
  for (int c = 0; c < CB_T; ++c) {
    double part = 0.0;
    for (int m = h; m < c; m += 4) part += X[r + CB_LD * m] * D[c + CB_LD * m];
    part += __shfl_xor_sync(0xffffffffu, part, 1);
    part += __shfl_xor_sync(0xffffffffu, part, 2);
    const double v = (X[r + CB_LD * c] - part) / D[c + CB_LD * c];
    __syncwarp();
    if (h == 0) X[r + CB_LD * c] = v;
    __syncwarp();
  }
  __syncthreads();
  for (int e = tid; e < CB_T * CB_T; e += blockDim.x) Aik[e] = X[(e % CB_T) + CB_LD * (e / CB_T)];
}

// Update k: tile (i, j) -= L_ik L_jk^T for the m (m + 1) / 2 tiles k < j <= i <= k + m (m = min(W,
// nbt - 1 - k)); CTA b takes the b-th tile in the order (i, j) = (k+1, k+1), (k+2, k+1), (k+2, k+2),
// ... Each thread forms a 4 x 4 block of the product (rows tr + 16 a, columns ts + 16 b). On a
// diagonal tile only the lower triangle is written. Dynamic shared memory: two tiles.
static __global__ void __launch_bounds__(CB_THREADS) band_update_kernel(int nbt, int W, int k, double* Lb) {
  extern __shared__ __align__(16) double cbs[];
  double* Li = cbs;
  double* Lj = cbs + CB_T * CB_LD;
  const int tid = threadIdx.x;
  // b -> (ii, jj), jj <= ii: ii (ii + 1) / 2 <= b < (ii + 1) (ii + 2) / 2
  const int b = blockIdx.x;
  int ii = (int)((sqrt(8.0 * b + 1.0) - 1.0) * 0.5);
  while ((ii + 1) * (ii + 2) / 2 <= b) ++ii;
  while (ii * (ii + 1) / 2 > b) --ii;
  const int jj = b - ii * (ii + 1) / 2;
  const int i = k + 1 + ii, j = k + 1 + jj;
  const double* Lik = Lb + band_tile_offset(i, k, W);
  const double* Ljk = Lb + band_tile_offset(j, k, W);
  for (int e = tid; e < CB_T * CB_T; e += blockDim.x) {
    Li[(e % CB_T) + CB_LD * (e / CB_T)] = Lik[e];
    Lj[(e % CB_T) + CB_LD * (e / CB_T)] = Ljk[e];
  }
  __syncthreads();
  const int tr = tid % 16, ts = tid / 16;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[a][c] = 0.0;
  for (int m = 0; m < CB_T; ++m) {
    double x[4], y[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      x[a] = Li[tr + 16 * a + CB_LD * m];
      y[a] = Lj[ts + 16 * a + CB_LD * m];
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][c] = fma(x[a], y[c], acc[a][c]);
  }
  double* Aij = Lb + band_tile_offset(i, j, W);
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int r = tr + 16 * a, s = ts + 16 * c;
      if (i != j || r >= s) Aij[r + (size_t)CB_T * s] -= acc[a][c];
    }
}

// Entry (r, c), r >= c, of the band factor (zero outside the band)
__device__ inline double band_entry(const double* Lb, int W, int64_t r, int64_t c) {
  const int i = (int)(r / CB_T), j = (int)(c / CB_T);
  if (i - j > W || r < c) return 0.0;
  return Lb[band_tile_offset(i, j, W) + (r % CB_T) + (size_t)CB_T * (c % CB_T)];
}

// In place X <- D^-1 X for every tile of the block triangular solves (kern_band.cuh layout: 2 nb
// steps of wt + 1 tiles of BS x BS, diag holding D of each step: lower for the forward direction,
// upper for the backward one). One CTA per tile, one thread per column of the tile: forward
// (d = 0) or backward (d = 1) substitution down its column, the column in shared memory and the
// triangular block read with warp-uniform loads.
template <int BS>
static __global__ void __launch_bounds__(BS) tile_trsm_kernel(int nb, int wt, const double* __restrict__ diag,
                                                               double* __restrict__ tiles) {
  extern __shared__ __align__(16) double xs[];  // BS x BS: xs[m * BS + j] = column j's entry m
  const int64_t tt = (int64_t)BS * BS;
  const int64_t tile = blockIdx.x;  // d * nb * (wt + 1) + s * (wt + 1) + t
  const int64_t ds = tile / (wt + 1);
  const int d = (int)(ds / nb);
  const double* Dk = diag + ds * tt;
  double* X = tiles + tile * tt;
  const int j = threadIdx.x;
  for (int m = 0; m < BS; ++m) xs[m * BS + j] = X[m + (int64_t)BS * j];
  if (d == 0) {
    for (int r = 0; r < BS; ++r) {
      double s = xs[r * BS + j];
      for (int m = 0; m < r; ++m) s -= Dk[r + (int64_t)BS * m] * xs[m * BS + j];
      xs[r * BS + j] = s / Dk[r + (int64_t)BS * r];
    }
  } else {
    for (int r = BS - 1; r >= 0; --r) {
      double s = xs[r * BS + j];
      for (int m = r + 1; m < BS; ++m) s -= Dk[r + (int64_t)BS * m] * xs[m * BS + j];
      xs[r * BS + j] = s / Dk[r + (int64_t)BS * r];
    }
  }
  for (int m = 0; m < BS; ++m) X[m + (int64_t)BS * j] = xs[m * BS + j];
}

}  // namespace hfk
