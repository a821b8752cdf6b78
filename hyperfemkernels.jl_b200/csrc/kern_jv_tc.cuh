// FP32 matrix-free Jacobian-vector product of Q2 cells (27 nodes, 27 Gauss points) with both
// contractions on the 5th-generation tensor cores (tcgen05.mma kind::tf32, FP32 accumulation in
// tensor memory).
//
// The reference evaluates the product cell by cell with sum factorisation (tp_interpolate! /
// tp_contract!, src/tensorproduct.jl:125-224, called from apply_cells!, src/matrixfree.jl:341-424).
// Here a CTA takes 128 cells (the MMA's M = 128 rows, one TMEM lane and one thread per cell) and
// applies the two contractions as dense GEMMs over the cells:
//   interpolation  G_c[cell, 3q + K] = sum_n U_c[cell, n] dN[n, K, q]      (K = 32 nodes, N = 96)
//   contraction    y_c[cell, n]      = sum_{q,K} C_c[cell, 3q + K] dN[n, K, q]  (K = 96, N = 32)
// U_c: the cell's increment of component c (gathered), C_c the pulled-back stress increment of the
// pointwise law (one thread per cell, FP32 on the CUDA cores, the same law code as the other
// products). The dense GEMMs do 3x the multiply-adds of the sum-factorised sweeps, on a pipe with
// far more throughput than the FP32 FMA pipe.
//
// Accuracy: TF32 keeps 10 mantissa bits, so every operand is split, x = hi + lo with hi = x rounded
// to TF32 and lo = x - hi (exact), and the products accumulate hi*hi + hi*lo + lo*hi (the 3xTF32
// scheme; the dropped lo*lo term is 2^-22 relative): the result has FP32 accuracy.
//
// Operands: U (A, shared memory, K-major, no swizzle), the reference-gradient tables (B, shared
// memory, prepared once per problem in the canonical layout), C (A of the contraction, tensor
// memory: the hi part written in place of the interpolation results it was computed from, the lo
// part staged). Tensor memory: 512 columns, interpolation at 0 / 96 / 192 (component c), the lo part
// of the component being contracted at 288, the products at 384 / 416 / 448. Every wait on the
// tensor cores' completion barrier is bounded: on expiry the CTA records the failure in the error
// word, skips the rest of its work, frees its tensor memory and returns.
#pragma once
#include <cstdint>
#include <cstring>

#include "hfk_internal.h"
#include "kern_cell.cuh"
#include "pointwise.cuh"

namespace hfk {

constexpr int TC_CELLS = 128;  // cells per CTA = MMA rows = TMEM lanes = threads
constexpr int TC_NN = 27;      // nodes of a Q2 cell
constexpr int TC_NP = 27;      // Gauss points
constexpr int TC_K1 = 32;      // interpolation K: the nodes, padded with zeros
constexpr int TC_N1 = 96;      // interpolation N: (point, direction) 3q + K, 81 padded to 96
constexpr int TC_K2 = TC_N1;   // contraction K
constexpr int TC_N2 = 32;      // contraction N: the nodes, padded
constexpr int TC_COL_LO = 3 * TC_N1;          // 288
constexpr int TC_COL_Y = TC_COL_LO + TC_K2;   // 384
constexpr int TC_TMEM_COLS = 512;
constexpr int TC_A_BYTES = TC_CELLS * TC_K1 * 4;  // 16 KB: one A operand (component, hi or lo)
constexpr int TC_B1_BYTES = TC_N1 * TC_K1 * 4;    // 12 KB
constexpr int TC_B2_BYTES = TC_N2 * TC_K2 * 4;    // 12 KB
constexpr int TC_OFF_B = 6 * TC_A_BYTES;          // tables after the six A operands (96 KB)
constexpr int TC_TAB_FLOATS = (2 * TC_B1_BYTES + 2 * TC_B2_BYTES) / 4;
constexpr int TC_OFF_BAR = TC_OFF_B + 4 * TC_TAB_FLOATS;
constexpr int TC_SMEM = TC_OFF_BAR + 16;
constexpr int TC_WAIT_LIMIT = 1 << 22;  // polls of the completion barrier before a CTA gives up
static_assert(2 * TC_K2 * TC_CELLS * 4 <= TC_OFF_B, "the lo staging of two components fits the A region");

// Byte offset of element (row, k) of a K-major operand with `rows` rows (a multiple of 8) in the
// canonical layout without swizzle: 8-row x 16-byte core matrices, row groups 128 bytes apart
// (the descriptor's stride byte offset), the 4-element K chunks (rows / 8) * 128 bytes apart (its
// leading byte offset).
__host__ __device__ inline uint32_t tc_kmajor_off(int row, int k, int rows) {
  return (uint32_t)(((k >> 2) * (rows >> 3) + (row >> 3)) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

// x rounded to TF32 (10 mantissa bits, to nearest, ties away from zero), as an FP32 bit pattern
__host__ __device__ inline float tf32_round(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  u = (u + 0x1000u) & 0xffffe000u;
  float r;
  memcpy(&r, &u, 4);
  return r;
}

// Shared-memory matrix descriptor (no swizzle): start address, leading and stride byte offsets in
// 16-byte units, descriptor version 1 (bits 46-47)
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3fffu) | ((uint64_t)((lbo >> 4) & 0x3fffu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3fffu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::tf32: FP32 accumulator, A and B TF32 and K-major, N / 8, M / 16
constexpr uint32_t tc_idesc(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t tc_smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// D (TMEM) (+)= A (shared) B (shared)
__device__ __forceinline__ void tc_mma_ss(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

// D (TMEM) (+)= A (TMEM) B (shared)
__device__ __forceinline__ void tc_mma_ts(uint32_t d, uint32_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d),
      "r"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

// the completion of every MMA issued so far by this thread arrives on the barrier
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_bar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// bounded wait for the barrier's phase `parity` to complete; false when the limit ran out
__device__ __forceinline__ bool tc_bar_wait(uint32_t bar, uint32_t parity, int limit) {
  for (int i = 0; i < limit; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    __nanosleep(64);
  }
  return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ float tc_ld1(uint32_t taddr) {
  uint32_t v;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(v) : "r"(taddr) : "memory");
  return __uint_as_float(v);
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_st1(uint32_t taddr, float v) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x1.b32 [%0], {%1};" ::"r"(taddr), "r"(__float_as_uint(v)) : "memory");
}
__device__ __forceinline__ void tc_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// The B operands of both GEMMs from the reference gradients dNt (nn, 3, np; tensor order), each
// split into TF32 hi and lo, in the canonical K-major layouts: [B1 hi | B1 lo | B2 hi | B2 lo].
// B1: N = 96 rows (3q + K), K = 32 (nodes); B2: N = 32 rows (nodes), K = 96 (3q + K). Zero padding.
static __global__ void tc_tables_kernel(const double* __restrict__ dNt, float* __restrict__ tabs) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < TC_N1 * TC_K1; e += gridDim.x * blockDim.x) {
    const int r = e % TC_N1, n = e / TC_N1;  // r = 3q + K
    const float v = (r < 3 * TC_NP && n < TC_NN) ? (float)dNt[n + TC_NN * r] : 0.0f;
    const float hi = tf32_round(v), lo = tf32_round(v - hi);
    const uint32_t o1 = tc_kmajor_off(r, n, TC_N1) / 4, o2 = tc_kmajor_off(n, r, TC_N2) / 4;
    tabs[o1] = hi;
    tabs[TC_B1_BYTES / 4 + o1] = lo;
    tabs[2 * (TC_B1_BYTES / 4) + o2] = hi;
    tabs[2 * (TC_B1_BYTES / 4) + TC_B2_BYTES / 4 + o2] = lo;
  }
}

// The product y += J(u) dx over the listed cells (all cells: cd.cells == nullptr), FP32, scatter by
// atomics. F is the prepared FP32 deformation gradient per point ((cell*9 + i)*27 + q).
static __global__ void __launch_bounds__(TC_CELLS, 1)
    jv_tc_kernel(CellData cd, const float* __restrict__ tabs, CellIO<float> io, int* err) {
  extern __shared__ __align__(1024) unsigned char tcs[];
  __shared__ uint32_t s_tmem;
  const int t = threadIdx.x, warp = t >> 5;
  const int li = blockIdx.x * TC_CELLS + t;
  const bool has = li < cd.ncells_list;
  const int cell = has ? (cd.cells ? cd.cells[li] : li) : 0;
  const bool live = has && !cd.skipped(cell);
  const uint32_t sb = tc_smem_addr(tcs);
  const uint32_t bar = sb + TC_OFF_BAR;
  // the tables (16-byte copies) and this cell's increment, split hi / lo, into the A operands
  {
    const int4* src = reinterpret_cast<const int4*>(tabs);
    int4* dst = reinterpret_cast<int4*>(tcs + TC_OFF_B);
    for (int e = t; e < TC_TAB_FLOATS / 4; e += TC_CELLS) dst[e] = src[e];
  }
  const int32_t* gid = cd.ids + (size_t)cell * (3 * TC_NN);
#pragma unroll
  for (int c = 0; c < 3; ++c)
    for (int n = 0; n < TC_K1; ++n) {
      float u = 0.0f;
      if (live && n < TC_NN) {
        const int32_t id = gid[c * TC_NN + n];
        u = id > 0 ? io.dx[id - 1] : 0.0f;
      }
      const float hi = tf32_round(u), lo = tf32_round(u - hi);
      const uint32_t o = tc_kmajor_off(t, n, TC_CELLS);
      *reinterpret_cast<float*>(tcs + (2 * c) * TC_A_BYTES + o) = hi;
      *reinterpret_cast<float*>(tcs + (2 * c + 1) * TC_A_BYTES + o) = lo;
    }
  if (t == 0) {
    tc_bar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_addr(&s_tmem)),
                 "r"(TC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_proxy_async();  // the operands written by the threads become visible to the tensor cores
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const uint32_t lanes = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's quarter of the lanes
  constexpr uint32_t ID1 = tc_idesc(TC_CELLS, TC_N1), ID2 = tc_idesc(TC_CELLS, TC_N2);
  constexpr uint32_t LBO_A = (TC_CELLS / 8) * 128, LBO_B1 = (TC_N1 / 8) * 128, LBO_B2 = (TC_N2 / 8) * 128;
  const uint32_t b1hi = sb + TC_OFF_B, b1lo = b1hi + TC_B1_BYTES;
  const uint32_t b2hi = b1lo + TC_B1_BYTES, b2lo = b2hi + TC_B2_BYTES;
  // ---- interpolation: G_c = U_c dN (3xTF32), one thread issues -----------------------------
  if (t == 0) {
    for (int c = 0; c < 3; ++c) {
      const uint32_t ahi = sb + (2 * c) * TC_A_BYTES, alo = ahi + TC_A_BYTES;
      for (int s = 0; s < TC_K1 / 8; ++s) {
        const uint64_t dah = tc_desc(ahi + s * 2 * LBO_A, LBO_A, 128), dal = tc_desc(alo + s * 2 * LBO_A, LBO_A, 128);
        const uint64_t dbh = tc_desc(b1hi + s * 2 * LBO_B1, LBO_B1, 128), dbl = tc_desc(b1lo + s * 2 * LBO_B1, LBO_B1, 128);
        const uint32_t d = tmem + c * TC_N1;
        tc_mma_ss(d, dah, dbh, ID1, s > 0 ? 1u : 0u);
        tc_mma_ss(d, dah, dbl, ID1, 1u);
        tc_mma_ss(d, dal, dbh, ID1, 1u);
      }
    }
    tc_commit(bar);
  }
  uint32_t pending = 0;  // the parity of a committed phase not yet seen complete (0xff: none)
  bool ok = tc_bar_wait(bar, 0, TC_WAIT_LIMIT);
  if (ok) pending = 0xffu;
  tc_fence_after();
  // ---- pointwise: per point, the 9 reference gradients from TMEM, the law, C back to TMEM -----
  float iJ[9], detv = 0.0f;
  if (live && cd.affine[cell]) {
    const double* gc = cd.geo + (size_t)cell * 10;
#pragma unroll
    for (int i = 0; i < 9; ++i) iJ[i] = (float)gc[i];
    detv = (float)gc[9];
  } else {
#pragma unroll
    for (int i = 0; i < 9; ++i) iJ[i] = 0.0f;
  }
  const float lam = live ? (float)cd.lam_of(cell) : 0.0f, mu = live ? (float)cd.mu_of(cell) : 0.0f;
  float* stage = reinterpret_cast<float*>(tcs);  // [2][TC_K2][TC_CELLS]: C_lo of components 1 and 2
  for (int q = 0; q < TC_NP; ++q) {
    float G[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int K = 0; K < 3; ++K) G[c][K] = tc_ld1(lanes + c * TC_N1 + 3 * q + K);
    tc_wait_ld();
    float out[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    if (live && ok) {
      float iJq[9], dV;
      if (cd.affine[cell]) {
#pragma unroll
        for (int i = 0; i < 9; ++i) iJq[i] = iJ[i];
        dV = (float)cd.w[q] * detv;
      } else {
        double Jt[9], iJd[9];
        point_jacobian_dev(cd, cell, q, Jt);
        const double det = det3(Jt);
        inv3(Jt, det, iJd);
#pragma unroll
        for (int i = 0; i < 9; ++i) iJq[i] = (float)iJd[i];
        dV = (float)(cd.w[q] * fabs(det));
      }
      float H[9], Fm[9], dP[9];
      phys_grad<float, 3>(iJq, G, 0, H);
#pragma unroll
      for (int i = 0; i < 9; ++i) Fm[i] = io.Fq[((size_t)cell * 9 + i) * TC_NP + q];
      law_dstress_F<float>(cd.law, lam, mu, Fm, H, dP);
      pull_back<float>(iJq, dP, dV, out);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int K = 0; K < 3; ++K) {
        const float v = out[c][K], hi = tf32_round(v), lo = tf32_round(v - hi);
        const int k = 3 * q + K;
        tc_st1(lanes + c * TC_N1 + k, hi);  // in place of the gradient it came from
        if (c == 0) tc_st1(lanes + TC_COL_LO + k, lo);
        else stage[((c - 1) * TC_K2 + k) * TC_CELLS + t] = lo;
      }
  }
  for (int k = 3 * TC_NP; k < TC_K2; ++k) {  // the padding of the contraction's K
    tc_st1(lanes + TC_COL_LO + k, 0.0f);
    stage[k * TC_CELLS + t] = 0.0f;
    stage[(TC_K2 + k) * TC_CELLS + t] = 0.0f;
  }
  tc_wait_st();
  tc_fence_before();
  ok = __syncthreads_and(ok) != 0;  // uniform from here on
  tc_fence_after();
  // ---- contraction: y_c = C_c dN^T; component 0 whole, the hi terms of 1 and 2 --------------
  if (t == 0 && ok) {
    for (int c = 0; c < 3; ++c)
      for (int s = 0; s < TC_K2 / 8; ++s) {
        const uint64_t dbh = tc_desc(b2hi + s * 2 * LBO_B2, LBO_B2, 128), dbl = tc_desc(b2lo + s * 2 * LBO_B2, LBO_B2, 128);
        const uint32_t d = tmem + TC_COL_Y + c * TC_N2, a = tmem + c * TC_N1 + 8 * s;
        tc_mma_ts(d, a, dbh, ID2, s > 0 ? 1u : 0u);
        tc_mma_ts(d, a, dbl, ID2, 1u);
        if (c == 0) tc_mma_ts(d, tmem + TC_COL_LO + 8 * s, dbh, ID2, 1u);
      }
    tc_commit(bar);
  }
  if (ok) {
    pending = 1;
    ok = tc_bar_wait(bar, 1, TC_WAIT_LIMIT);
    if (ok) pending = 0xffu;
  }
  // the lo terms of components 1 and 2, one after the other through the same TMEM columns
  for (int c = 1; c < 3; ++c) {
    ok = __syncthreads_and(ok) != 0;
    tc_fence_after();
    if (ok)
      for (int k = 0; k < TC_K2; ++k) tc_st1(lanes + TC_COL_LO + k, stage[((c - 1) * TC_K2 + k) * TC_CELLS + t]);
    tc_wait_st();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (t == 0 && ok) {
      for (int s = 0; s < TC_K2 / 8; ++s)
        tc_mma_ts(tmem + TC_COL_Y + c * TC_N2, tmem + TC_COL_LO + 8 * s, tc_desc(b2hi + s * 2 * LBO_B2, LBO_B2, 128),
                  ID2, 1u);
      tc_commit(bar);
    }
    if (ok) {
      pending = c == 1 ? 0u : 1u;
      ok = tc_bar_wait(bar, pending, TC_WAIT_LIMIT);
      if (ok) pending = 0xffu;
    }
  }
  ok = __syncthreads_and(ok) != 0;
  tc_fence_after();
  // ---- the products, scattered at the free dofs ---------------------------------------------
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float yv[TC_NN];
#pragma unroll
    for (int n = 0; n < TC_NN; ++n) yv[n] = tc_ld1(lanes + TC_COL_Y + c * TC_N2 + n);
    tc_wait_ld();
    if (live && ok) {
#pragma unroll
      for (int n = 0; n < TC_NN; ++n) {
        const int32_t id = gid[c * TC_NN + n];
        if (id > 0) atomicAdd(io.y + (id - 1), yv[n]);
      }
    }
  }
  if (!ok && t == 0) {
    atomicExch(err, 1);
    // the tensor memory is freed below: give the operations still in flight one more bounded wait
    if (pending != 0xffu) tc_bar_wait(bar, pending, TC_WAIT_LIMIT);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS));
  }
}

}  // namespace hfk
