// Internal definitions of the B200 engine (not part of the C ABI).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <map>
#include <vector>

#include "../../include/hfk.h"

namespace hfk {

// ---- error handling: every ABI entry point returns a status and records the message ----------
void set_error(const std::string& msg);
struct Error {
  int code;
  std::string msg;
};

#define HFK_CUDA(call)                                                                      \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      throw ::hfk::Error{HFK_ERR_CUDA, std::string("HyperFEMKernels: CUDA error: ") +       \
                                           cudaGetErrorString(e_) + " at " #call};          \
  } while (0)
#define HFK_REQUIRE(cond, code, msg)                                       \
  do {                                                                     \
    if (!(cond)) throw ::hfk::Error{code, std::string("HyperFEMKernels: ") + (msg)}; \
  } while (0)

// ABI entry points: body between HFK_API_BEGIN and HFK_API_END; errors become a status + message
#define HFK_API_BEGIN try {
#define HFK_API_END                                     \
  return HFK_OK;                                        \
  }                                                     \
  catch (const hfk::Error& e) {                         \
    hfk::set_error(e.msg);                              \
    return e.code;                                      \
  }                                                     \
  catch (const std::exception& e) {                     \
    hfk::set_error(std::string("HyperFEMKernels: ") + e.what()); \
    return HFK_ERR_INTERNAL;                            \
  }

// ---- a device buffer owned by a handle ---------------------------------------------------
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void resize(size_t m) {
    if (m == n && p) return;
    release();
    if (m) HFK_CUDA(cudaMalloc(&p, m * sizeof(T)));
    n = m;
  }
  void upload(const T* h, size_t m, cudaStream_t s) {
    resize(m);
    if (m) HFK_CUDA(cudaMemcpyAsync(p, h, m * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void zero(cudaStream_t s) {
    if (n) HFK_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
};

// max supported nodes / points per direction in the tensor-product kernels
constexpr int MAXQ = 6;

// 1D tables (tensor order), passed by value to kernels (constant bank, broadcast reads)
template <typename R>
struct Tab1D {
  R N1[MAXQ * MAXQ];   // N1[a * Q + i]: basis i at 1D point a
  R dN1[MAXQ * MAXQ];
  R w1[MAXQ];          // 1D weights (unused when the product weights are passed)
};

// Per-problem read-only data the cell kernels take (device pointers), passed by value.
struct CellData {
  const int32_t* ids;     // (ndl, ncells) cell-major, tensor node order, ldof = c*nn + n
  const int32_t* cells;   // list of cells (one colour) or nullptr for 0..ncells-1
  int ncells_list;
  int ncells;
  const double* geo;      // 10 per cell: iJt (column-major 3x3) and |det Jt| at the first point
  const uint8_t* affine;  // per cell
  const double* coords;   // (3, 8, ncells)
  const double* dMt;      // (8, 3, np) tensor point order
  const double* w;        // (np) tensor point order
  int law;                // HFK_LAW_*
  double lam, mu, body[3];
  const double* cell_lm;  // optional (2, ncells): lambda, mu per cell (batched problems), else lam, mu
  // batched problems: the cell kernels skip the cells of segments whose flag is 0 (problems that
  // have converged inside a batched solve; all flags are 1 outside one). nullptr: no masking.
  const int32_t* cell_seg;    // per cell its segment
  const int32_t* seg_active;  // per segment 1 = compute, 0 = skip
  __host__ __device__ double lam_of(int cell) const { return cell_lm ? cell_lm[2 * (size_t)cell] : lam; }
  __host__ __device__ double mu_of(int cell) const { return cell_lm ? cell_lm[2 * (size_t)cell + 1] : mu; }
  __host__ __device__ bool skipped(int cell) const { return seg_active && !seg_active[cell_seg[cell]]; }
};

// Work of the two-stage reductions (partial sums and the result)
struct Reducer {
  DBuf<double> partial, out;
  double host[3];
};

// Work vectors of the Krylov solve, kept with the operator between solves
struct CGWork {
  DBuf<double> b, x, r, z, p, q, rold;
  Reducer red;
  DBuf<double> sc;  // per-segment scalars of the batched solve
  DBuf<int> fl, cnt;
  DBuf<int> itd;  // the batched solve's iteration count, when its loop runs on the device
};

// Work of the restarted GMRES / FGMRES: the Krylov basis V ((restart + 1) n), the preconditioned
// basis Z (restart n for FGMRES, one vector for GMRES), a work vector and the projections (device),
// the multi-dot partial sums and the one reduction range {0, nitems}
struct GmresWork {
  DBuf<double> V, Z, w, h, part;
  DBuf<int32_t> all;
};

// State of a matrix-free level in a precision
template <typename R>
struct LevelState {
  DBuf<R> x, dvals;
};

}  // namespace hfk

// The opaque handles of the ABI
// the learned correction's network (hfk_mlp_*): FP32 master weights, their BF16 copy, Adam moments
struct hfk_mlp {
  hfk::DBuf<float> w, m1, m2, grad, loss;
  hfk::DBuf<__nv_bfloat16> wb;
  int64_t steps = 0;
  cudaStream_t stream = nullptr;
};

struct hfk_problem {
  int D = 3, nn = 0, nc = 3, np = 0, ng = 8, ndl = 0, ncells = 0;
  int Q = 0, P = 0;             // tensor-product structure (0 = none)
  int64_t nfree = 0, ndir = 0;
  int law = 0;
  double params[5] = {0, 0, 0, 0, 0};
  cudaStream_t stream = nullptr;      // launch stream (own_stream or the caller's)
  cudaStream_t own_stream = nullptr;
  int device = 0;
  // host copies of the construction data
  std::vector<int> nodeperm, pointperm;   // tensor index -> caller index
  std::vector<int32_t> h_ids;             // caller order
  std::vector<double> h_w;                // caller point order
  std::vector<double> h_N1, h_dN1;        // P x Q (a * Q + i)
  // device data (tensor order)
  hfk::DBuf<int32_t> ids;                 // (ndl, ncells)
  hfk::DBuf<double> geo, coords, dMt, w, Nt, dNt;  // Nt (nn, np), dNt (nn, 3, np) tensor order
  hfk::DBuf<uint8_t> affine;
  hfk::DBuf<double> cell_lm;              // per-cell lambda, mu (empty: the problem's parameters)
  // segments: independent problems held in one handle. Segment s owns the free dofs
  // [seg_off[s], seg_off[s+1]) and the cells [seg_cells[s], seg_cells[s+1]); reductions, Krylov
  // scalars, Chebyshev intervals and convergence are per segment. One segment by default.
  int nseg = 1;
  std::vector<int64_t> seg_off;           // nseg + 1
  std::vector<int32_t> seg_cells;         // nseg + 1 (empty: not given)
  std::vector<double> seg_lm;             // (2, nseg) lambda, mu per segment (empty: the problem's)
  hfk::DBuf<int32_t> seg_of_dof;          // per free dof (empty when nseg == 1)
  hfk::DBuf<int32_t> seg_of_block;        // per nodal block (empty when nseg == 1)
  hfk::DBuf<int64_t> item_lo, item_hi;    // segmented reductions: chunks of one segment's dofs
  hfk::DBuf<int32_t> item_first;          // nseg + 1: the first chunk of each segment
  hfk::DBuf<int64_t> seg_off_d;           // device copy of seg_off
  hfk::DBuf<double> seg_partial;          // per-chunk partial sums (3 per chunk)
  hfk::DBuf<int32_t> cell_seg;            // per cell its segment (nseg > 1 with cell ranges)
  hfk::DBuf<int32_t> seg_active_own;      // per segment: 1 = the cell kernels compute its cells
  int32_t* seg_active = nullptr;          // the flags the kernels read: own, or the working level's
  int nitems = 0;
  bool items_built = false;
  // colours
  int ncolors = 0;
  std::vector<int32_t> h_color_of;        // per cell, 1-based
  std::vector<int> color_start;           // ncolors + 1 offsets into cells_by_color
  hfk::DBuf<int32_t> cells_by_color;
  // sparsity pattern (CSC, 0-based int32 internally) and positions (tensor order, 1-based, 0 = none)
  int64_t nnz = 0;
  hfk::DBuf<int64_t> colptr;              // 1-based (Julia SparseMatrixCSC)
  hfk::DBuf<int64_t> rowval;
  hfk::DBuf<int32_t> nzpos;               // (ndl*ndl, ncells)
  hfk::DBuf<double> nzval;
  // current state (FP64)
  hfk::DBuf<double> x, dvals;
  bool prepared = false;
  int mf_mode = HFK_MF_RECOMPUTE;
  // deformation gradient per point (recompute formulation), FP64 and its FP32 copy
  hfk::DBuf<double> Fq;
  hfk::DBuf<float> Fq32;
  bool Fq32_valid = false;
  // stored tangents (reference formulation: T, iJt, dV per point)
  hfk::DBuf<double> T, iJtq, dVq;
  // nodal blocks
  int nblocks = 0;
  hfk::DBuf<int32_t> block_of;            // (nn, ncells) tensor order, 0 = none
  hfk::DBuf<int32_t> bdofs;               // (3, nblocks) 1-based, 0 = fixed
  hfk::DBuf<double> B, Binv;              // (9, nblocks)
  hfk::DBuf<float> Binv32;
  bool blocks_ok = false;
  // staging for host pointers
  hfk::DBuf<double> stage_in, stage_in2, stage_out;
  // hfk_mf_apply_many: two staging slots per direction, the copy-in and copy-out streams and their
  // events (fork, then per slot: copied in, product done, copied out), created on first use
  hfk::DBuf<double> many_in[2], many_out[2];
  cudaStream_t many_s[2] = {nullptr, nullptr};
  cudaEvent_t many_ev[7] = {};
  hfk::DBuf<int64_t> stage_l;
  hfk::DBuf<float> tmp32a, tmp32b;
  // hfk_jacobian into host memory: the cells in chunks; once a chunk has run, the prefix of the CSC
  // values that no later chunk touches is copied back on jc_copy while the next chunk is assembled
  hfk::DBuf<int32_t> jc_cells;            // 0 .. ncells - 1
  std::vector<int> jc_start;              // chunk boundaries (cells), nchunks + 1
  std::vector<int64_t> jc_done;           // per chunk: the CSC values complete once it has run
  cudaStream_t jc_copy = nullptr;
  std::vector<cudaEvent_t> jc_ev;
  // the tensor-core product: its B operands (once per problem) and the error word of its bounded waits
  hfk::DBuf<float> tc_tabs;
  hfk::DBuf<int> tc_err;
  // error flag for numerical checks
  hfk::DBuf<int> flag;
  // timing of the last kernel sequence (CUDA events)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // kernel timing (hfk_problem_set_timing): event pairs around the element-kernel launches
  bool ktiming = false;
  std::vector<cudaEvent_t> kev;
  size_t kev_used = 0;
  int launches = 0;
  int scatter = HFK_SCATTER_AUTO;
  int shape = 4;  // launch shape under an explicit scatter mode (warps per CTA, or a point-parallel shape)
  int asm_kernel = 0;  // assembled Jacobian of 27-node cells: 0 the default choice, 1 the FP64 tensor-core kernel
  hfk::DBuf<double> func_red;             // per-warp partials of the functionals
  std::map<int, std::pair<bool, int>> tuned;  // autotuned (atomic scatter, warps per CTA) per kernel mode
  bool no_tune = false;
  bool solve_graph = true;  // batched CG: after two host-driven iterations, the rest as one CUDA graph
                            // whose while node loops on the device  // set while a call that must not tune (allocation-free smoothing) runs
  hfk::CGWork cg;
  hfk::GmresWork gm;
};
