// Banded block triangular solves of the coarse level's Cholesky factor (A = L L^T, lower bandwidth b).
//
// The coarse solve of the p-multigrid cycle (the reference's LU solve of the assembled p = 1 level,
// src/pmultigrid.jl:97-98) applies A^-1 = L^-T L^-1 once per V-cycle. Both triangular solves run
// over blocks of BS_T rows in sequence (forward: blocks 0, 1, ...; backward: the last block first).
// With G_{k,j} = D_k^-1 L_{k,j} (D_k the diagonal block of block row k) precomputed at every
// factorisation, the block of step s is
//     y_k = D_k^-1 in_k - sum_{j in the band} G_{k,j} y_j
// so a step reads its dependencies' outputs only through dense BS_T x BS_T tiles and no step
// carries a triangular substitution. One launch per direction: CTAs take steps in the order they
// start (a ticket counter), add the tile of a dependency as soon as that dependency's block is
// published (a step's last dependency is the only one on the critical path) and publish their own.
// The output is filled with a sentinel bit pattern before the launch and a block is published by
// writing its values: a reader polls the very words it needs, so the critical path between two
// steps is one store and one load through L2 (no fence, no flag). A CTA waits only for steps with
// smaller tickets, which belong to CTAs already running, so the launch progresses whatever the
// number of resident CTAs. Every wait is bounded: on expiry the CTA records the failure in the error
// word, skips its remaining tiles and still publishes its block (zeros), so that every CTA of the
// launch returns; the host reads the error word after the cycle.
#pragma once
#include <cstdint>

#include "kern_chol.cuh"

namespace hfk {

constexpr int BS_T = 128;                  // rows per block (one CTA per block)
constexpr int BS_THREADS = 512;            // 4 threads per row, each over 32 columns of a tile
constexpr int BS_H = BS_THREADS / BS_T;
constexpr int BS_J = BS_T / BS_H;
constexpr int BS_SPIN_LIMIT = 1 << 22;     // polls of a dependency before the wait gives up (default)

// Tiles of both directions from the factor's band (kern_chol.cuh storage, lower block bandwidth W
// in CB_T tiles; zeros outside the band). Direction d (0 forward on L, 1 backward on L^T), step s
// (block k = s, or nb - 1 - s backward) has wt + 1 tiles of BS_T x BS_T, column-major: tile t < wt
// multiplies the output of step s - wt + t (zero when that step does not exist), tile wt is the
// identity (it becomes D_k^-1 after the tile triangular solves). diag receives D_k (lower,
// forward) or D_k^T (upper, backward), with unit diagonal on rows past n.
static __global__ void band_tiles_kernel(int64_t n, int nb, int wt, const double* __restrict__ Lb, int W,
                                         double* __restrict__ tiles, double* __restrict__ diag) {
  const int64_t tt = (int64_t)BS_T * BS_T;
  const int64_t ntile = (int64_t)2 * nb * (wt + 1);
  const int64_t total = ntile * tt + (int64_t)2 * nb * tt;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    if (e < ntile * tt) {
      const int64_t tile = e / tt;
      const int ij = (int)(e - tile * tt);
      const int i = ij % BS_T, j = ij / BS_T;
      const int t = (int)(tile % (wt + 1));
      const int64_t ds = tile / (wt + 1);
      const int d = (int)(ds / nb), s = (int)(ds % nb);
      double v = 0.0;
      if (t == wt) {
        v = i == j ? 1.0 : 0.0;
      } else {
        const int sd = s - wt + t;
        if (sd >= 0) {
          const int64_t k = d ? nb - 1 - s : s, kb = d ? nb - 1 - sd : sd;
          // forward: L[k T + i, kb T + j] (kb < k); backward: L^T[k T + i, kb T + j] = L[kb T + j, k T + i]
          const int64_t r = d ? kb * BS_T + j : k * BS_T + i;
          const int64_t c = d ? k * BS_T + i : kb * BS_T + j;
          if (r < n && c < n) v = band_entry(Lb, W, r, c);
        }
      }
      tiles[e] = v;
    } else {
      const int64_t q = e - ntile * tt;
      const int64_t ds = q / tt;
      const int ij = (int)(q - ds * tt);
      const int i = ij % BS_T, j = ij / BS_T;
      const int d = (int)(ds / nb), s = (int)(ds % nb);
      const int64_t k = d ? nb - 1 - s : s;
      double v = 0.0;
      if (d ? j >= i : i >= j) {
        const int64_t r = k * BS_T + (i > j ? i : j), c = k * BS_T + (i > j ? j : i);
        v = r < n ? band_entry(Lb, W, r, c) : (i == j ? 1.0 : 0.0);
      }
      diag[q] = v;
    }
  }
}

// p[0 .. n) = v (a launch, so that it can sit inside a captured stream)
static __global__ void fill_int_kernel(int n, int* p, int v) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = v;
}

// the bit pattern the outputs are filled with before a launch (a negative NaN with every payload
// bit set; NaNs computed on the GPU are canonical)
constexpr unsigned long long BS_SENTINEL = 0xffffffffffffffffull;

__device__ __forceinline__ unsigned long long bs_load_relaxed_u64(const double* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void bs_store_relaxed_u64(double* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// One direction of the solve: out_k = tile_wt(s) in_k - sum_t tile_t(s) out_{step s - wt + t}.
// ticket: zeroed before the launch, out: filled with BS_SENTINEL before the launch. err: set to 1 when a
// wait ran out (after spin_limit polls of one value). Launched with nb CTAs of BS_THREADS threads.
static __global__ void __launch_bounds__(BS_THREADS, 1)
    band_solve_kernel(int64_t n, int nb, int wt, int backward, const double* __restrict__ tiles,
                      const double* __restrict__ in, double* out, int* ticket, int* err, int spin_limit) {
  __shared__ int s_step;
  __shared__ double yb[BS_T];
  __shared__ double part[BS_H][BS_T];
  const int tid = threadIdx.x, i = tid % BS_T, h = tid / BS_T;
  if (tid == 0) s_step = atomicAdd(ticket, 1);
  __syncthreads();
  const int s = s_step;
  if (s >= nb) return;  // the grid has nb CTAs: never taken
  const int64_t k = backward ? nb - 1 - s : s;
  const int64_t tt = (int64_t)BS_T * BS_T;
  const double* ts = tiles + (int64_t)s * (wt + 1) * tt;
  const int j0 = h * BS_J;
  // D_k^-1 in_k
  if (tid < BS_T) {
    const int64_t r = k * BS_T + tid;
    yb[tid] = r < n ? in[r] : 0.0;
  }
  __syncthreads();
  double acc = 0.0;
  {
    const double* tw = ts + (int64_t)wt * tt + i + (int64_t)BS_T * j0;
#pragma unroll
    for (int jj = 0; jj < BS_J; ++jj) acc = fma(tw[(int64_t)BS_T * jj], yb[j0 + jj], acc);
  }
  // the dependencies in step order; the next tile's values are loaded before its flag is polled
  const int t0 = wt - s > 0 ? wt - s : 0;
  double reg[BS_J];
  bool failed = false;  // uniform over the CTA
  if (t0 < wt) {
    const double* tp = ts + (int64_t)t0 * tt + i + (int64_t)BS_T * j0;
#pragma unroll
    for (int jj = 0; jj < BS_J; ++jj) reg[jj] = tp[(int64_t)BS_T * jj];
  }
  for (int t = t0; t < wt; ++t) {
    const int sd = s - wt + t;
    __syncthreads();  // yb is rewritten below
    // the dependency's block, each value polled until it is no longer the sentinel
    int fail = 0;
    if (tid < BS_T) {
      const int64_t r = (int64_t)(backward ? nb - 1 - sd : sd) * BS_T + tid;
      double v = 0.0;
      if (r < n) {
        int polls = 0;
        for (;;) {
          const unsigned long long bits = bs_load_relaxed_u64(out + r);
          if (bits != BS_SENTINEL) {
            v = __longlong_as_double((long long)bits);
            break;
          }
          if (++polls > spin_limit || ((polls & 1023) == 0 && *((volatile int*)err))) {
            atomicExch(err, 1);
            fail = 1;
            break;
          }
          __nanosleep(20);
        }
      }
      yb[tid] = v;
    }
    failed = __syncthreads_or(fail) != 0;
    if (failed) break;
#pragma unroll
    for (int jj = 0; jj < BS_J; ++jj) acc = fma(-reg[jj], yb[j0 + jj], acc);
    if (t + 1 < wt) {
      const double* tp = ts + (int64_t)(t + 1) * tt + i + (int64_t)BS_T * j0;
#pragma unroll
      for (int jj = 0; jj < BS_J; ++jj) reg[jj] = tp[(int64_t)BS_T * jj];
    }
  }
  part[h][i] = acc;
  __syncthreads();
  if (tid < BS_T) {
    double v = part[0][tid];
#pragma unroll
    for (int q = 1; q < BS_H; ++q) v += part[q][tid];
    const int64_t r = k * BS_T + tid;
    // published value by value: a successor polls these very words (a value that reached the
    // sentinel's bit pattern would have to be a NaN that arithmetic on the GPU never produces)
    if (r < n) bs_store_relaxed_u64(out + r, (unsigned long long)__double_as_longlong(failed ? 0.0 : v));
  }
}

}  // namespace hfk
