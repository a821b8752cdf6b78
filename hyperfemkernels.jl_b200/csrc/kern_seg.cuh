// Segmented vector kernels: many independent problems held in one handle (a disjoint union of
// meshes). Every launch covers all problems at once; what differs per problem (a "segment": a
// contiguous range of free dofs) is read from small per-segment scalar arrays:
//  - reductions are computed per segment, in a fixed order (deterministic): the dofs are cut into
//    chunks of at most SEG_CHUNK entries that never straddle a segment, one CTA per chunk, then
//    one CTA per segment sums its chunks;
//  - the Krylov scalars (alpha, beta), the convergence flags and the Chebyshev coefficients are
//    per segment, indexed through seg_of_dof / seg_of_block.
// The reference solves one problem per operator; the batched path follows its per-problem
// algorithms (MatrixFreeSolver.solve!, src/solvers.jl:111-159; eigenvalue_bounds,
// src/preconditioners.jl:374-389) segment by segment. A problem with one segment goes through
// the same kernels with null segment maps.
#pragma once
#include "kern_vec.cuh"

namespace hfk {

constexpr int SEG_CHUNK = 8192;
// per-segment scalars of a Krylov solve: sc[s * SEG_NS + slot]
constexpr int SEG_NS = 16;
enum SegSlot { S_BB = 0, S_RR, S_RZ, S_PQ, S_ALPHA, S_BETA, S_TOL, S_ZR, S_ZROLD, S_RR0 };
// per-segment flags: fl[s * SEG_NF + flag]
constexpr int SEG_NF = 4;
enum SegFlag { F_ACTIVE = 0, F_CONV, F_INDEF, F_ITERS };

__device__ __forceinline__ int seg_at(const int32_t* of, int64_t i) { return of ? of[i] : 0; }

// partial[3 * chunk + j]: the chunk's share of up to three dot products
template <typename R>
__global__ void __launch_bounds__(RED_THREADS) seg_dots_kernel(int k, const int64_t* lo, const int64_t* hi, const R* a0,
                                                               const R* b0, const R* a1, const R* b1, const R* a2,
                                                               const R* b2, double* partial) {
  const int it = blockIdx.x;
  const int64_t l = lo[it], h = hi[it];
  double s0 = 0, s1 = 0, s2 = 0;
  for (int64_t i = l + threadIdx.x; i < h; i += blockDim.x) {
    s0 += (double)a0[i] * (double)b0[i];
    if (k > 1) s1 += (double)a1[i] * (double)b1[i];
    if (k > 2) s2 += (double)a2[i] * (double)b2[i];
  }
  block_sum_store(s0, partial + 3 * (size_t)it);
  if (k > 1) block_sum_store(s1, partial + 3 * (size_t)it + 1);
  if (k > 2) block_sum_store(s2, partial + 3 * (size_t)it + 2);
}

// out[s * stride + j] = sum over the chunks of segment s (one CTA per segment)
static __global__ void __launch_bounds__(RED_THREADS) seg_finish_kernel(int k, const int32_t* first, const double* partial,
                                                                 double* out, int stride) {
  const int s = blockIdx.x;
  const int f = first[s], e = first[s + 1];
  for (int j = 0; j < k; ++j) {
    double v = 0;
    for (int it = f + threadIdx.x; it < e; it += blockDim.x) v += partial[3 * (size_t)it + j];
    block_sum_store(v, out + (size_t)s * stride + j);
  }
}

// ---- several inner products at once (classical Gram-Schmidt of the Arnoldi estimate) ---------
constexpr int SEG_MDOTS = 16;  // vectors per multi-dot launch

// partial[it * SEG_MDOTS + j] = sum over chunk it of V_j[i] w[i], j < k <= SEG_MDOTS (V_j = V + j ldv)
static __global__ void __launch_bounds__(RED_THREADS) seg_mdots_kernel(int k, const int64_t* lo, const int64_t* hi,
                                                                const double* V, int64_t ldv, const double* w,
                                                                double* partial) {
  const int it = blockIdx.x;
  const int64_t l = lo[it], h = hi[it];
  double s[SEG_MDOTS];
#pragma unroll
  for (int j = 0; j < SEG_MDOTS; ++j) s[j] = 0;
  for (int64_t i = l + threadIdx.x; i < h; i += blockDim.x) {
    const double wi = w[i];
#pragma unroll
    for (int j = 0; j < SEG_MDOTS; ++j)
      if (j < k) s[j] += V[(size_t)j * ldv + i] * wi;
  }
#pragma unroll
  for (int j = 0; j < SEG_MDOTS; ++j)
    if (j < k) block_sum_store(s[j], partial + (size_t)it * SEG_MDOTS + j);
}

// out[s * stride + j] = sum over the chunks of segment s, j < k (one CTA per segment)
static __global__ void __launch_bounds__(RED_THREADS) seg_mfinish_kernel(int k, const int32_t* first, const double* partial,
                                                                  double* out, int stride) {
  const int s = blockIdx.x;
  const int f = first[s], e = first[s + 1];
  for (int j = 0; j < k; ++j) {
    double v = 0;
    for (int it = f + threadIdx.x; it < e; it += blockDim.x) v += partial[(size_t)it * SEG_MDOTS + j];
    block_sum_store(v, out + (size_t)s * stride + j);
  }
}

// y[i] -= sum_{j<k} c[seg(i) * stride + j] V_j[i]
static __global__ void seg_maxpy_kernel(int64_t n, const int32_t* seg, int k, const double* c, int stride, const double* V,
                                 int64_t ldv, double* y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double* cs = c + (size_t)seg_at(seg, i) * stride;
    double acc = 0;
    for (int j = 0; j < k; ++j) acc += cs[j] * V[(size_t)j * ldv + i];
    y[i] -= acc;
  }
}

// dst[s * stride + j] += src[s * stride + j], j < k, every segment s
static __global__ void seg_add_kernel(int ns, int k, const double* src, double* dst, int stride) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ns * k; e += gridDim.x * blockDim.x) {
    const int s = e / k, j = e - s * k;
    dst[(size_t)s * stride + j] += src[(size_t)s * stride + j];
  }
}

// y[i] += sign * a[seg(i) * stride] x[i]
static __global__ void seg_axpy_kernel(int64_t n, const int32_t* seg, const double* a, int stride, double sign,
                                const double* x, double* y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] += sign * a[(size_t)seg_at(seg, i) * stride] * x[i];
}

// y[i] = x[i] / s[seg(i) * stride] (0 where the scale is 0)
static __global__ void seg_scale_kernel(int64_t n, const int32_t* seg, const double* s, int stride, const double* x,
                                 double* y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = s[(size_t)seg_at(seg, i) * stride];
    y[i] = v != 0.0 ? x[i] / v : 0.0;
  }
}

// s[j * stride] = sqrt(max(s[j * stride], 0)) for every segment j (a rounding-negative square of a
// vanished vector, possible in the P^-1 inner product, is a breakdown, not a NaN)
static __global__ void seg_sqrt_kernel(int nseg, double* s, int stride) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nseg; j += gridDim.x * blockDim.x)
    s[(size_t)j * stride] = sqrt(fmax(s[(size_t)j * stride], 0.0));
}

// sc[out] = sc[den] > 0 ? sc[num] / sc[den] : 0 per segment; then sc[den] = sc[num] when `shift`
// (the fixed-count CG of the inexact coarse solve: alpha = rz / pq, beta = rz' / rz)
static __global__ void seg_ratio_kernel(int nseg, double* sc, int num, int den, int out, int shift) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x) {
    double* c = sc + (size_t)s * SEG_NS;
    const double d = c[den];
    c[out] = d > 0 ? c[num] / d : 0.0;
    if (shift) c[den] = c[num];
  }
}

// one CTA: count the active segments into *nactive
static __device__ void seg_count_active(int nseg, const int* fl, int* nactive) {
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  int mine = 0;
  for (int s = threadIdx.x; s < nseg; s += blockDim.x) mine += fl[(size_t)s * SEG_NF + F_ACTIVE];
  atomicAdd(&cnt, mine);
  __syncthreads();
  if (threadIdx.x == 0) *nactive = cnt;
}

// start of a solve: tol = atol + rtol ||b||; a segment is active while ||r|| > tol
static __global__ void seg_cg_init_kernel(int nseg, double* sc, int* fl, double rtol, double atol, int* nactive) {
  for (int s = threadIdx.x; s < nseg; s += blockDim.x) {
    double* c = sc + (size_t)s * SEG_NS;
    int* f = fl + (size_t)s * SEG_NF;
    c[S_TOL] = atol + rtol * sqrt(c[S_BB]);
    c[S_RR0] = c[S_RR];
    const bool act = sqrt(c[S_RR]) > c[S_TOL];
    f[F_ACTIVE] = act;
    f[F_CONV] = !act;
    f[F_INDEF] = 0;
    f[F_ITERS] = 0;
  }
  __syncthreads();
  seg_count_active(nseg, fl, nactive);
}

// alpha = rz / pq for the active segments; a non-positive curvature stops the segment as
// indefinite (src/solvers.jl:135-139); inactive segments get alpha = 0 (their iterates stay)
static __global__ void seg_cg_alpha_kernel(int nseg, double* sc, int* fl) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x) {
    double* c = sc + (size_t)s * SEG_NS;
    int* f = fl + (size_t)s * SEG_NF;
    double a = 0;
    if (f[F_ACTIVE]) {
      if (c[S_PQ] > 0) {
        a = c[S_RZ] / c[S_PQ];
        f[F_ITERS] += 1;
      } else {
        f[F_ACTIVE] = 0;
        f[F_INDEF] = 1;
      }
    }
    c[S_ALPHA] = a;
  }
}

// x += alpha p, r -= alpha q per segment (rold = r before the update, for the flexible beta)
static __global__ void seg_cg_update_kernel(int64_t n, const int32_t* seg, const double* sc, const double* p, const double* q,
                                     double* x, double* r, double* rold) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double a = sc[(size_t)seg_at(seg, i) * SEG_NS + S_ALPHA];
    const double ri = r[i];
    if (rold) rold[i] = ri;
    x[i] += a * p[i];
    r[i] = ri - a * q[i];
  }
}

// convergence test on the recursive residual; counts the segments still active
static __global__ void seg_cg_check_kernel(int nseg, const double* sc, int* fl, int* nactive) {
  for (int s = threadIdx.x; s < nseg; s += blockDim.x) {
    const double* c = sc + (size_t)s * SEG_NS;
    int* f = fl + (size_t)s * SEG_NF;
    if (f[F_ACTIVE] && sqrt(c[S_RR]) <= c[S_TOL]) {
      f[F_ACTIVE] = 0;
      f[F_CONV] = 1;
    }
  }
  __syncthreads();
  seg_count_active(nseg, fl, nactive);
}

// End of one iteration of the device-driven batched CG (the body of a CUDA graph while node): count
// the iteration and continue while a segment is active and the iteration limit is not reached.
static __global__ void seg_cg_loop_kernel(cudaGraphConditionalHandle h, const int* nactive, int* it, int maxiter) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    const int i = *it + 1;
    *it = i;
    cudaGraphSetConditional(h, (*nactive > 0 && i < maxiter) ? 1u : 0u);
  }
}
static __global__ void set_int_kernel(int* p, int v) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *p = v;
}

// beta per segment: Polak-Ribiere (flexible) (z.r - z.rold) / rz, else z.r / rz; rz <- z.r
static __global__ void seg_cg_beta_kernel(int nseg, double* sc, const int* fl, int flexible) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x) {
    double* c = sc + (size_t)s * SEG_NS;
    double b = 0;
    if (fl[(size_t)s * SEG_NF + F_ACTIVE] && c[S_RZ] != 0) b = (flexible ? c[S_ZR] - c[S_ZROLD] : c[S_ZR]) / c[S_RZ];
    c[S_BETA] = b;
    c[S_RZ] = c[S_ZR];
  }
}

// p = z + sc[slot] p per segment
static __global__ void seg_xpby_kernel(int64_t n, const int32_t* seg, const double* sc, int slot, const double* z, double* p) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = z[i] + sc[(size_t)seg_at(seg, i) * SEG_NS + slot] * p[i];
}

// the cell kernels' segment flags from a batched solve's flags (value = -1: set every flag to 1)
static __global__ void seg_mask_kernel(int nseg, const int* fl, int32_t* mask, int value) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x)
    mask[s] = value < 0 ? fl[(size_t)s * SEG_NF + F_ACTIVE] : value;
}

// x[i] *= f[seg(i)]
static __global__ void seg_mul_kernel(int64_t n, const int32_t* seg, const double* f, double* x) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] *= f[seg_at(seg, i)];
}

// v[s * stride + j] = sqrt(v[s * stride + j] / n_s) for j < k (root mean squares per segment)
static __global__ void seg_rms_kernel(int nseg, double* v, int stride, int k, const int64_t* off) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x) {
    const double ns = (double)(off[s + 1] - off[s]);
    for (int j = 0; j < k; ++j) {
      double* x = v + (size_t)s * stride + j;
      *x = ns > 0 ? sqrt(*x / ns) : 0.0;
    }
  }
}

}  // namespace hfk
