// C ABI of the B200 engine: construction (host C++), dispatch of the CUDA kernels, solver loops.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <memory>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include "devcache.h"
#include "engine.h"
#include "hfk_internal.h"
#include "kern_assembly.cuh"
#include "kern_q1.cuh"
#include "kern_band.cuh"
#include "kern_cell.cuh"
#include "kern_chol.cuh"
#include "kern_jvp.cuh"
#include "kern_mlp.cuh"
#include "kern_seg.cuh"
#include "kern_vec.cuh"


using namespace hfk;

namespace hfk {
thread_local std::string g_last_error;
void set_error(const std::string& m) { g_last_error = m; }
}  // namespace hfk

namespace {

// ---- 1D Lagrange basis on [0,1], equispaced nodes (lagrange1d, src/tensorproduct.jl:24-47) ----
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

// TPTable (src/tensorproduct.jl:55-91): 1D tables and the permutations tensor index -> caller index
bool detect_tp(hfk_problem* p, const double* xq, const double* Nt) {
  const int Q = (int)std::lround(std::cbrt((double)p->nn));
  const int P = (int)std::lround(std::cbrt((double)p->np));
  if (Q * Q * Q != p->nn || P * P * P != p->np || Q > MAXQ || P > MAXQ) return false;
  std::vector<double> xs;
  for (int q = 0; q < p->np; ++q) xs.push_back(std::round(xq[3 * q] * 1e12) / 1e12);
  std::sort(xs.begin(), xs.end());
  xs.erase(std::unique(xs.begin(), xs.end()), xs.end());
  if ((int)xs.size() != P) return false;
  for (int d = 1; d < 3; ++d) {
    std::vector<double> ys;
    for (int q = 0; q < p->np; ++q) ys.push_back(std::round(xq[d + 3 * q] * 1e12) / 1e12);
    std::sort(ys.begin(), ys.end());
    ys.erase(std::unique(ys.begin(), ys.end()), ys.end());
    if (ys.size() != xs.size()) return false;
    for (size_t i = 0; i < ys.size(); ++i)
      if (std::fabs(ys[i] - xs[i]) > 1e-10) return false;
  }
  p->h_N1.assign(P * Q, 0);
  p->h_dN1.assign(P * Q, 0);
  std::vector<double> n1(Q), dn1(Q);
  // the 1D basis is evaluated at the unrounded coordinate of each 1D point (the rounding only
  // identifies equal coordinates; evaluating at the rounded value would perturb the tables by ~1e-12)
  for (int a = 0; a < P; ++a) {
    double xa = xs[a];
    for (int q = 0; q < p->np; ++q)
      if (std::round(xq[3 * q] * 1e12) / 1e12 == xs[a]) {
        xa = xq[3 * q];
        break;
      }
    lagrange1d(Q, xa, n1.data(), dn1.data());
    for (int i = 0; i < Q; ++i) {
      p->h_N1[a * Q + i] = n1[i];
      p->h_dN1[a * Q + i] = dn1[i];
    }
  }
  p->pointperm.assign(p->np, -1);
  for (int lin = 0; lin < p->np; ++lin) {
    const int t[3] = {lin % P, (lin / P) % P, lin / (P * P)};
    for (int q = 0; q < p->np; ++q) {
      bool ok = true;
      for (int d = 0; d < 3; ++d) ok &= std::fabs(xq[d + 3 * q] - xs[t[d]]) <= 1e-10;
      if (ok) {
        p->pointperm[lin] = q;
        break;
      }
    }
    if (p->pointperm[lin] < 0) return false;
  }
  p->nodeperm.assign(p->nn, -1);
  std::vector<char> used(p->nn, 0);
  for (int lin = 0; lin < p->nn; ++lin) {
    const int ii[3] = {lin % Q, (lin / Q) % Q, lin / (Q * Q)};
    for (int n = 0; n < p->nn; ++n) {
      if (used[n]) continue;
      bool ok = true;
      for (int pl = 0; pl < p->np && ok; ++pl) {
        const int aa[3] = {pl % P, (pl / P) % P, pl / (P * P)};
        double v = 1;
        for (int d = 0; d < 3; ++d) v *= p->h_N1[aa[d] * Q + ii[d]];
        ok = std::fabs(Nt[n + (size_t)p->nn * p->pointperm[pl]] - v) <= 1e-7;
      }
      if (ok) {
        used[n] = 1;
        p->nodeperm[lin] = n;
        break;
      }
    }
    if (p->nodeperm[lin] < 0) return false;
  }
  p->Q = Q;
  p->P = P;
  return true;
}

template <typename R>
Tab1D<R> make_tab(const hfk_problem* p) {
  Tab1D<R> t;
  std::memset(&t, 0, sizeof t);
  for (int a = 0; a < p->P; ++a)
    for (int i = 0; i < p->Q; ++i) {
      t.N1[a * p->Q + i] = (R)p->h_N1[a * p->Q + i];
      t.dN1[a * p->Q + i] = (R)p->h_dN1[a * p->Q + i];
    }
  return t;
}

}  // namespace
CellData hfk::cell_data(const hfk_problem* p, const int32_t* cells, int ncells_list) {
  CellData cd;
  cd.ids = p->ids.p;
  cd.cells = cells;
  cd.ncells_list = ncells_list;
  cd.ncells = p->ncells;
  cd.geo = p->geo.p;
  cd.affine = p->affine.p;
  cd.coords = p->coords.p;
  cd.dMt = p->dMt.p;
  cd.w = p->w.p;
  cd.law = p->law;
  cd.lam = p->params[0];
  cd.mu = p->params[1];
  cd.cell_lm = p->cell_lm.p;
  const bool masked = p->seg_active && p->cell_seg.p;
  cd.cell_seg = masked ? p->cell_seg.p : nullptr;
  cd.seg_active = masked ? p->seg_active : nullptr;
  for (int c = 0; c < 3; ++c) cd.body[c] = p->params[2 + c];
  return cd;
}
namespace {

// ---- cell-kernel dispatch over (Q, P) ----------------------------------------------------------
template <int Q, int P, int MODE, typename R>
void launch_cell(hfk_problem* p, const int32_t* cells, int ncl, const CellIO<R>& io, int warps) {
  using S = TPShape<Q, P>;
  const size_t smem = cell_smem_bytes<Q, P, R>(warps);
  static PerDeviceLimit attr;
  raise_smem_limit(cell_kernel<Q, P, MODE, R>, smem, attr);
  const int per_cta = warps * S::CPW;
  const int grid = (ncl + per_cta - 1) / per_cta;
  if (grid == 0) return;
  cell_kernel<Q, P, MODE, R><<<grid, warps * 32, smem, p->stream>>>(cell_data(p, cells, ncl), make_tab<R>(p), io);
  check_launch(p);
}

// the point-parallel product (kern_jvp.cuh), NT threads per CTA
template <int Q, int P, typename R, int NT>
void launch_jvp(hfk_problem* p, const int32_t* cells, int ncl, const CellIO<R>& io) {
  using S = JvpShape<Q, P, NT>;
  const size_t smem = jvp_smem_bytes<Q, P, R, NT>();
  static PerDeviceLimit attr;
  raise_smem_limit(jvp_kernel<Q, P, R, NT>, smem, attr);
  const int grid = (ncl + S::C - 1) / S::C;
  if (grid == 0) return;
  jvp_kernel<Q, P, R, NT><<<grid, NT, smem, p->stream>>>(cell_data(p, cells, ncl), make_tab<R>(p), io);
  check_launch(p);
}

// Launch shapes: 2 or 4 = warps per CTA of the line-mapped kernel; SHAPE_PT_NARROW / SHAPE_PT_WIDE =
// the point-parallel product (matrix-free product only) with one cell per CTA or 256 threads
constexpr int SHAPE_PT_NARROW = 100, SHAPE_PT_WIDE = 108;
// SHAPE_TC: the FP32 product of Q2 cells with both contractions on the tensor cores (kern_jv_tc.cuh)
constexpr int SHAPE_TC = 120;
// SHAPE_Q1: the warp-synchronous product of Q1 cells with 2^3 Gauss points (kern_q1.cuh)
constexpr int SHAPE_Q1 = 130;

template <typename R>
void launch_q1(hfk_problem* p, const int32_t* cells, int ncl, const CellIO<R>& io) {
  const int grid = (ncl + Q1_THREADS / 8 - 1) / (Q1_THREADS / 8);
  if (grid == 0) return;
  q1_jv_kernel<R><<<grid, Q1_THREADS, 0, p->stream>>>(cell_data(p, cells, ncl), make_tab<R>(p), io);
  check_launch(p);
}

// whether the tensor-core product serves this problem and precision
template <int MODE, typename R>
bool tc_eligible(const hfk_problem* p) {
  return MODE == MODE_JV && std::is_same<R, float>::value && p->Q == 3 && p->P == 3;
}

template <int Q, int P, int MODE, typename R>
void launch_shape(hfk_problem* p, const int32_t* cells, int ncl, const CellIO<R>& io, int shape) {
  if constexpr (MODE == MODE_JV && Q == 3 && P == 3 && std::is_same<R, float>::value) {
    if (shape == SHAPE_TC) {
      launch_jv_tc(p, cells, ncl, io);
      return;
    }
  }
  if constexpr (MODE == MODE_JV && Q == 2 && P == 2) {
    if (shape == SHAPE_Q1) {
      launch_q1<R>(p, cells, ncl, io);
      return;
    }
  }
  if (MODE == MODE_JV && shape == SHAPE_PT_NARROW) launch_jvp<Q, P, R, jvp_narrow<P>()>(p, cells, ncl, io);
  else if (MODE == MODE_JV && shape == SHAPE_PT_WIDE) launch_jvp<Q, P, R, JVP_WIDE>(p, cells, ncl, io);
  else launch_cell<Q, P, MODE, R>(p, cells, ncl, io, shape >= SHAPE_PT_NARROW ? 4 : shape);  // SHAPE_TC/Q1 elsewhere: 4 warps
}

template <int MODE, typename R>
void dispatch_cell(hfk_problem* p, const int32_t* cells, int ncl, const CellIO<R>& io, int warps = 4) {
  const int key = p->Q * 10 + p->P;
  switch (key) {
#define HFK_CASE(Qv, Pv) \
  case Qv * 10 + Pv:     \
    launch_shape<Qv, Pv, MODE, R>(p, cells, ncl, io, warps); \
    return;
    HFK_CASE(2, 2)
    HFK_CASE(2, 3)
    HFK_CASE(2, 4)
    HFK_CASE(2, 5)
    HFK_CASE(3, 3)
    HFK_CASE(3, 4)
    HFK_CASE(3, 5)
    HFK_CASE(4, 4)
    HFK_CASE(4, 5)
    HFK_CASE(5, 5)
#undef HFK_CASE
    default:
      throw Error{HFK_ERR_UNSUPPORTED, "HyperFEMKernels: no sum-factorised kernel for Q=" + std::to_string(p->Q) +
                                           " P=" + std::to_string(p->P)};
  }
}

// Run a cell kernel colour by colour (deterministic scatter)
// Scatter policy: colour by colour (deterministic) unless the colours are too small to fill the
// GPU, then one launch over all cells with atomicAdd (an order-dependent last bit). A colour needs
// about 4 warps per SM to hide the gather latency.
}  // namespace
bool hfk::use_atomic_scatter(const hfk_problem* p) {
  // AUTO scatters with atomics: one launch instead of one per colour (no wave tails, no launch
  // gaps), and a fire-and-forget reduction in L2 instead of a dependent read of y before the
  // write (measured on B200, Q2 64^3 J*v: 0.55 ms against 0.75 ms by colour)
  return p->scatter != HFK_SCATTER_COLOURED;
}
namespace {

template <int MODE, typename R>
void run_cells_as(hfk_problem* p, CellIO<R> io, bool atomic, int warps) {
  ktimer_mark(p);
  if (atomic) {
    io.atomic = 1;
    dispatch_cell<MODE, R>(p, nullptr, p->ncells, io, warps);
  } else {
    io.atomic = 0;
    for (int c = 0; c < p->ncolors; ++c) {
      const int n = p->color_start[c + 1] - p->color_start[c];
      dispatch_cell<MODE, R>(p, p->cells_by_color.p + p->color_start[c], n, io, warps);
    }
  }
  ktimer_mark(p);
}

// Launch-shape autotuner (per problem, per kernel mode and precision, so per degree): on the first
// AUTO call the kernel runs with each candidate (atomic or colour-by-colour scatter, 2 or 4 warps
// per CTA of the line-mapped kernel and, for the matrix-free product, the point-parallel kernel of
// 8 warps), timed with CUDA events, and the fastest is kept. Outputs are zeroed before each
// candidate and once more before the real run. No tuning while the stream is being captured (the
// V-cycle is captured from its second application, when every kernel of it has run once) nor inside
// the allocation-free smoother (an untuned kernel runs with the atomic scatter and 4 warps there).
template <int MODE, typename R>
void run_cells(hfk_problem* p, CellIO<R> io) {
  if (p->scatter != HFK_SCATTER_AUTO) {
    run_cells_as<MODE, R>(p, io, p->scatter == HFK_SCATTER_ATOMIC, p->shape);
    return;
  }
  const int key = MODE * 2 + (sizeof(R) == sizeof(float) ? 1 : 0);
  auto it = p->tuned.find(key);
  if (it == p->tuned.end()) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    HFK_CUDA(cudaStreamIsCapturing(p->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone || !io.y || p->no_tune) {
      run_cells_as<MODE, R>(p, io, true, 4);
      return;
    }
    // (atomic, warps per CTA); the matrix-free product also tries the point-parallel kernel
    std::vector<std::pair<int, int>> cand = {{1, 4}, {1, 2}, {0, 4}, {0, 2}};
    // batched problems keep the line-mapped kernels (and the Q1 one): the tuning call has every
    // problem active, but most of a batched solve runs with converged problems masked, where the
    // per-warp exit of these kernels measured better (256 SVK Q2 problems: 22.3 s against 23.9 s
    // with the point-parallel product picked for the Q1 level)
    if (MODE == MODE_JV && p->nseg <= 1)
      for (int a : {1, 0})
        for (int sh : {SHAPE_PT_NARROW, SHAPE_PT_WIDE}) cand.push_back({a, sh});
    const bool tc = tc_eligible<MODE, R>(p) && p->nseg <= 1;
    if (tc) cand.push_back({1, SHAPE_TC});
    if (MODE == MODE_JV && p->Q == 2 && p->P == 2) {
      cand.push_back({1, SHAPE_Q1});
      cand.push_back({0, SHAPE_Q1});
    }
    const int ncand = (int)cand.size();
    cudaEvent_t e0, e1;
    HFK_CUDA(cudaEventCreate(&e0));
    HFK_CUDA(cudaEventCreate(&e1));
    float best = 0;
    int pick = 0;
    std::vector<R> ref, got;  // the tensor-core candidate is kept only if it agrees with the first one
    for (int c = 0; c < ncand; ++c) {
      float t = 1e30f;
      for (int rep = 0; rep < 2; ++rep) {
        HFK_CUDA(cudaMemsetAsync(io.y, 0, p->nfree * sizeof(R), p->stream));
        HFK_CUDA(cudaEventRecord(e0, p->stream));
        run_cells_as<MODE, R>(p, io, cand[c].first != 0, cand[c].second);
        HFK_CUDA(cudaEventRecord(e1, p->stream));
        HFK_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        HFK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        t = std::min(t, ms);
      }
      if (tc && (c == 0 || cand[c].second == SHAPE_TC)) {
        std::vector<R>& v = c == 0 ? ref : got;
        v.resize(p->nfree);
        HFK_CUDA(cudaMemcpyAsync(v.data(), io.y, p->nfree * sizeof(R), cudaMemcpyDeviceToHost, p->stream));
        HFK_CUDA(cudaStreamSynchronize(p->stream));
        if (c > 0) {
          int err = 0;
          HFK_CUDA(cudaMemcpy(&err, p->tc_err.p, sizeof(int), cudaMemcpyDeviceToHost));
          double dmax = 0, rmax = 0;
          for (int64_t i = 0; i < p->nfree; ++i) {
            dmax = std::max(dmax, (double)std::fabs((double)got[i] - (double)ref[i]));
            rmax = std::max(rmax, (double)std::fabs((double)ref[i]));
          }
          if (err || !(dmax <= 1e-5 * rmax)) t = 1e30f;  // not eligible
          if (err) HFK_CUDA(cudaMemset(p->tc_err.p, 0, sizeof(int)));
        }
      }
      if (c == 0 || t < best) {
        best = t;
        pick = c;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    it = p->tuned.emplace(key, std::make_pair(cand[pick].first != 0, cand[pick].second)).first;
    HFK_CUDA(cudaMemsetAsync(io.y, 0, p->nfree * sizeof(R), p->stream));
  }
  run_cells_as<MODE, R>(p, io, it->second.first, it->second.second);
}

// ---- colouring (color_cells, src/coloring.jl:4-28) --------------------------------------------
}  // namespace
void hfk::color_cells(hfk_problem* p) {
  std::vector<unsigned __int128> masks(p->nfree + 1, 0);
  p->h_color_of.assign(p->ncells, 0);
  int ncol = 0;
  for (int cell = 0; cell < p->ncells; ++cell) {
    const int32_t* id = &p->h_ids[(size_t)cell * p->ndl];
    unsigned __int128 used = 0;
    for (int j = 0; j < p->ndl; ++j)
      if (id[j] > 0) used |= masks[id[j]];
    int c = 0;
    while (c < 128 && ((used >> c) & 1)) ++c;
    HFK_REQUIRE(c < 128, HFK_ERR_ARG, "more than 128 colours needed");
    p->h_color_of[cell] = c + 1;
    const unsigned __int128 bit = (unsigned __int128)1 << c;
    for (int j = 0; j < p->ndl; ++j)
      if (id[j] > 0) masks[id[j]] |= bit;
    ncol = std::max(ncol, c + 1);
  }
  p->ncolors = ncol;
  p->color_start.assign(ncol + 1, 0);
  for (int cell = 0; cell < p->ncells; ++cell) p->color_start[p->h_color_of[cell]]++;
  for (int c = 0; c < ncol; ++c) p->color_start[c + 1] += p->color_start[c];
  std::vector<int32_t> order(p->ncells);
  std::vector<int> fill(p->color_start.begin(), p->color_start.end() - 1);
  for (int cell = 0; cell < p->ncells; ++cell) order[fill[p->h_color_of[cell] - 1]++] = cell;
  p->cells_by_color.upload(order.data(), order.size(), p->stream);
}
namespace {

// ---- affine cells and per-cell geometry (affine_cells, src/tables.jl:128-156) ------------------
void cell_geometry(hfk_problem* p, const double* coords, const double* dMt_caller) {
  std::vector<uint8_t> aff(p->ncells, 0);
  std::vector<double> geo((size_t)p->ncells * 10, 0.0);
  const double eps = 2.220446049250313e-16;
  for (int cell = 0; cell < p->ncells; ++cell) {
    const double* X = coords + (size_t)cell * 3 * p->ng;
    double Jt[9] = {0};
    for (int n = 0; n < p->ng; ++n)
      for (int K = 0; K < 3; ++K) {
        const double g = dMt_caller[n + p->ng * (K + 3 * 0)];
        for (int i = 0; i < 3; ++i) Jt[K + 3 * i] += g * X[i + 3 * n];
      }
    bool ok = p->ng == 8;
    if (ok) {
      double h = 0;
      for (int n = 1; n < 8; ++n) {
        double s = 0;
        for (int i = 0; i < 3; ++i) s += (X[i + 3 * n] - X[i]) * (X[i + 3 * n] - X[i]);
        h = std::max(h, std::sqrt(s));
      }
      for (int n = 1; n < 8; ++n) {
        const double xi[3] = {double(n & 1), double((n >> 1) & 1), double((n >> 2) & 1)};
        double e2 = 0, nx = 0;
        for (int i = 0; i < 3; ++i) {
          double pr = 0;
          for (int K = 0; K < 3; ++K) pr += xi[K] * Jt[K + 3 * i];
          const double r = X[i + 3 * n] - X[i] - pr;
          e2 += r * r;
          nx += X[i + 3 * n] * X[i + 3 * n];
        }
        ok &= std::sqrt(e2) <= 1e-13 * h + 8 * eps * std::sqrt(nx);
      }
    }
    aff[cell] = ok;
    const double d = det3(Jt);
    double iJ[9];
    inv3(Jt, d, iJ);
    for (int i = 0; i < 9; ++i) geo[(size_t)cell * 10 + i] = iJ[i];
    geo[(size_t)cell * 10 + 9] = std::fabs(d);
  }
  p->affine.upload(aff.data(), aff.size(), p->stream);
  p->geo.upload(geo.data(), geo.size(), p->stream);
}

void require_tp(hfk_problem* p) {
  HFK_REQUIRE(p->Q > 0, HFK_ERR_UNSUPPORTED,
              "the cells have no tensor-product structure (sum-factorised kernels need Q^3 nodes and P^3 Gauss points)");
}

void bind_state(hfk_problem* p, const double* x, const double* dvals) {
  const double* dx = dev_in(x, p->nfree, p->stage_in, p->stream);
  const double* dd = dev_in(dvals, p->ndir, p->stage_in2, p->stream);
  p->x.resize(p->nfree);
  p->dvals.resize(std::max<int64_t>(p->ndir, 1));
  if (p->nfree) HFK_CUDA(cudaMemcpyAsync(p->x.p, dx, p->nfree * sizeof(double), cudaMemcpyDeviceToDevice, p->stream));
  if (p->ndir) HFK_CUDA(cudaMemcpyAsync(p->dvals.p, dd, p->ndir * sizeof(double), cudaMemcpyDeviceToDevice, p->stream));
}

// ---- reductions -------------------------------------------------------------------------------

template <typename R>
void dots(hfk_problem* p, Reducer& red, int64_t n, int k, const R* a0, const R* b0, const R* a1 = nullptr,
          const R* b1 = nullptr, const R* a2 = nullptr, const R* b2 = nullptr, double* res = nullptr) {
  red.partial.resize((size_t)3 * RED_BLOCKS);
  red.out.resize(3);
  dots_kernel<R><<<RED_BLOCKS, RED_THREADS, 0, p->stream>>>(n, k, a0, b0, a1, b1, a2, b2, red.partial.p);
  check_launch(p);
  finish_sums_kernel<<<1, 1024, 0, p->stream>>>(RED_BLOCKS, k, red.partial.p, red.out.p);
  check_launch(p);
  HFK_CUDA(cudaMemcpyAsync(red.host, red.out.p, k * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  if (res)
    for (int i = 0; i < k; ++i) res[i] = red.host[i];
}

// ---- segments (independent problems in one handle) -------------------------------------------
// The chunks of the segmented reductions, built on first use (one segment: [0, nfree)).
void ensure_seg_items(hfk_problem* p) {
  if (p->items_built) return;
  if (p->seg_off.empty()) p->seg_off = {0, p->nfree};
  std::vector<int64_t> lo, hi;
  std::vector<int32_t> first(p->nseg + 1);
  for (int s = 0; s < p->nseg; ++s) {
    first[s] = (int32_t)lo.size();
    for (int64_t a = p->seg_off[s]; a < p->seg_off[s + 1]; a += SEG_CHUNK) {
      lo.push_back(a);
      hi.push_back(std::min<int64_t>(a + SEG_CHUNK, p->seg_off[s + 1]));
    }
  }
  first[p->nseg] = (int32_t)lo.size();
  p->nitems = (int)lo.size();
  if (lo.empty()) {
    lo.push_back(0);
    hi.push_back(0);
  }
  p->item_lo.upload(lo.data(), lo.size(), p->stream);
  p->item_hi.upload(hi.data(), hi.size(), p->stream);
  p->item_first.upload(first.data(), first.size(), p->stream);
  p->seg_off_d.upload(p->seg_off.data(), p->seg_off.size(), p->stream);
  p->seg_partial.resize((size_t)3 * std::max(p->nitems, 1));
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  p->items_built = true;
}

const int32_t* seg_dof_map(const hfk_problem* p) { return p->nseg > 1 ? p->seg_of_dof.p : nullptr; }
const int32_t* seg_block_map(const hfk_problem* p) { return p->nseg > 1 ? p->seg_of_block.p : nullptr; }

// Per-segment sums of up to three products a_j . b_j into out[s * stride + j] (device), sync-free
template <typename R>
void seg_dots(hfk_problem* p, int k, double* out, int stride, const R* a0, const R* b0, const R* a1 = nullptr,
              const R* b1 = nullptr, const R* a2 = nullptr, const R* b2 = nullptr) {
  ensure_seg_items(p);
  if (p->nitems) {
    seg_dots_kernel<R><<<p->nitems, RED_THREADS, 0, p->stream>>>(k, p->item_lo.p, p->item_hi.p, a0, b0, a1, b1, a2, b2,
                                                                  p->seg_partial.p);
    check_launch(p);
  }
  seg_finish_kernel<<<p->nseg, RED_THREADS, 0, p->stream>>>(k, p->item_first.p, p->seg_partial.p, out, stride);
  check_launch(p);
}

// segment of every nodal block (the segment of its first free dof)
void build_seg_of_block(hfk_problem* p, const std::vector<int32_t>& dofs) {
  if (p->nseg <= 1) return;
  std::vector<int32_t> sb(std::max(p->nblocks, 1), 0);
  for (int b = 0; b < p->nblocks; ++b) {
    int32_t d = 0;
    for (int c = 0; c < 3 && !d; ++c) d = dofs[3 * (size_t)b + c];
    const int64_t i = (int64_t)d - 1;
    sb[b] = (int32_t)(std::upper_bound(p->seg_off.begin(), p->seg_off.end(), i) - p->seg_off.begin()) - 1;
  }
  p->seg_of_block.upload(sb.data(), sb.size(), p->stream);
}

// ---- matrix-free products on device vectors ---------------------------------------------------
}  // namespace
void hfk::mf_apply_dev(hfk_problem* p, const double* dx, double* y) {
  HFK_REQUIRE(p->prepared, HFK_ERR_STATE, "the matrix-free Jacobian has not been prepared (call hfk_mf_prepare)");
  HFK_CUDA(cudaMemsetAsync(y, 0, p->nfree * sizeof(double), p->stream));
  CellIO<double> io{};
  io.dx = dx;
  io.y = y;
  if (p->mf_mode == HFK_MF_STORED) {
    io.T = p->T.p;
    io.iJtq = p->iJtq.p;
    io.dVq = p->dVq.p;
    run_cells<MODE_JV_STORED, double>(p, io);
  } else {
    io.Fq = p->Fq.p;
    run_cells<MODE_JV, double>(p, io);
  }
}
namespace {

// the FP32 copy of the stored deformation gradients (made on first use after a prepare)
void ensure_F32(hfk_problem* p) {
  if (p->Fq32_valid) return;
  HFK_REQUIRE(p->Fq.p, HFK_ERR_STATE, "the FP32 product needs a prepared tangent (recompute mode)");
  p->Fq32.resize(p->Fq.n);
  convert_kernel<double, float><<<vec_grid((int64_t)p->Fq.n), 256, 0, p->stream>>>((int64_t)p->Fq.n, p->Fq.p, p->Fq32.p);
  check_launch(p);
  p->Fq32_valid = true;
}

void mf_apply_dev32(hfk_problem* p, const float* dx, float* y) {
  HFK_REQUIRE(p->prepared, HFK_ERR_STATE, "the matrix-free Jacobian has not been prepared (call hfk_mf_prepare)");
  HFK_REQUIRE(p->mf_mode == HFK_MF_RECOMPUTE, HFK_ERR_STATE, "the FP32 product needs the recompute formulation");
  ensure_F32(p);
  HFK_CUDA(cudaMemsetAsync(y, 0, p->nfree * sizeof(float), p->stream));
  CellIO<float> io{};
  io.dx = dx;
  io.y = y;
  io.Fq = p->Fq32.p;
  run_cells<MODE_JV, float>(p, io);
}

// prepare in the recompute formulation: F = I + grad u at every point of every cell (from x, dvals)
void prepare_F(hfk_problem* p) {
  require_tp(p);
  p->Fq.resize((size_t)9 * p->np * p->ncells);
  CellIO<double> io{};
  io.u = p->x.p;
  io.dvals = p->dvals.p;
  io.Fout = p->Fq.p;
  dispatch_cell<MODE_PREP_F, double>(p, nullptr, p->ncells, io);
  p->Fq32_valid = false;
  p->mf_mode = HFK_MF_RECOMPUTE;
  p->prepared = true;
}

template <typename R>
void mf_apply_any(hfk_problem* p, const R* dx, R* y);
template <>
void mf_apply_any<double>(hfk_problem* p, const double* dx, double* y) {
  mf_apply_dev(p, dx, y);
}
template <>
void mf_apply_any<float>(hfk_problem* p, const float* dx, float* y) {
  mf_apply_dev32(p, dx, y);
}

// ---- stored tangents (prepare_cells!, src/matrixfree.jl:199-228) -------------------------------
__global__ void store_tangents_kernel(CellData cd, const double* u, const double* dvals, const double* dNt, int nn,
                                      int np, double* T, double* iJtq, double* dVq) {
  const int ndl = 3 * nn;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)cd.ncells * np;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int cell = (int)(e / np), q = (int)(e % np);
    const int32_t* gid = cd.ids + (size_t)cell * ndl;
    double G[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int c = 0; c < 3; ++c)
      for (int n = 0; n < nn; ++n) {
        const int32_t id = gid[c * nn + n];
        const double x = id > 0 ? u[id - 1] : (id < 0 ? dvals[-id - 1] : 0.0);
        for (int K = 0; K < 3; ++K) G[c][K] += x * dNt[n + nn * (K + 3 * q)];
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
    double H[9], Tq[81];
    for (int c = 0; c < 3; ++c)
      for (int J = 0; J < 3; ++J) H[c + 3 * J] = iJ[J] * G[c][0] + iJ[J + 3] * G[c][1] + iJ[J + 6] * G[c][2];
    law_tangent(cd.law, cd.lam_of(cell), cd.mu_of(cell), H, Tq);
    for (int i = 0; i < 81; ++i) T[((size_t)cell * 81 + i) * np + q] = Tq[i];
    for (int i = 0; i < 9; ++i) iJtq[((size_t)cell * 9 + i) * np + q] = iJ[i];
    dVq[(size_t)cell * np + q] = cd.w[q] * det;
  }
}

// ---- blocks -----------------------------------------------------------------------------------
void build_block_structure(hfk_problem* p) {
  // field_blocks (src/preconditioners.jl:151-173): one block per node key (its 3 test ids), numbered
  // in order of first appearance over cells and the caller's node order. A free dof belongs to one
  // node, so a node with a free dof is identified by its first free id: a direct-indexed table
  // (O(1) per node, no hashing) gives the same numbering as a map of the keys.
  std::vector<int32_t> block_by_first((size_t)p->nfree + 1, 0);
  std::vector<int32_t> dofs;
  std::vector<int32_t> block_of((size_t)p->nn * p->ncells, 0);  // tensor order
  std::vector<int> inv_node(p->nn);
  for (int lin = 0; lin < p->nn; ++lin) inv_node[p->nodeperm[lin]] = lin;
  int32_t nb = 0;
  for (int cell = 0; cell < p->ncells; ++cell)
    for (int n = 0; n < p->nn; ++n) {
      int32_t key[3], first = 0;
      for (int c = 0; c < 3; ++c) {
        key[c] = p->h_ids[(size_t)cell * p->ndl + c * p->nn + n];
        if (!first && key[c] > 0) first = key[c];
      }
      if (!first) continue;
      int32_t& blk = block_by_first[first];
      if (!blk) {
        for (int c = 0; c < 3; ++c) dofs.push_back(key[c] > 0 ? key[c] : 0);
        blk = ++nb;
      }
      block_of[inv_node[n] + (size_t)p->nn * cell] = blk;
    }
  p->nblocks = (int)nb;
  p->block_of.upload(block_of.data(), block_of.size(), p->stream);
  p->bdofs.upload(dofs.data(), dofs.size(), p->stream);
  build_seg_of_block(p, dofs);
  p->B.resize(9 * (size_t)std::max(p->nblocks, 1));
  p->Binv.resize(9 * (size_t)std::max(p->nblocks, 1));
  p->Binv32.resize(9 * (size_t)std::max(p->nblocks, 1));
}

void invert_blocks_and_check(hfk_problem* p, int* ok) {
  p->flag.resize(1);
  p->flag.zero(p->stream);
  invert_blocks_kernel<<<vec_grid(p->nblocks), 256, 0, p->stream>>>(p->nblocks, p->bdofs.p, p->B.p, p->Binv.p,
                                                                     p->Binv32.p, p->flag.p);
  check_launch(p);
  int bad = 0;
  HFK_CUDA(cudaMemcpyAsync(&bad, p->flag.p, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  p->blocks_ok = !bad;
  *ok = !bad;
}

// the sum-factorised block extraction (kern_vec.cuh) for tensor-product cells with Q <= P; false
// when the problem has no such shape (the dense kernel then runs)
template <int Q, int P>
void blocks_tp_launch(hfk_problem* p, BlockIO io) {
  const size_t smem = blocks_tp_smem<Q, P>();
  static PerDeviceLimit attr;
  raise_smem_limit(blocks_tp_kernel<Q, P>, smem, attr);
  const Tab1D<double> tab = make_tab<double>(p);
  if (use_atomic_scatter(p)) {
    io.atomic = 1;
    blocks_tp_kernel<Q, P><<<p->ncells, 256, smem, p->stream>>>(cell_data(p, nullptr, p->ncells), tab, io);
    check_launch(p);
  } else {
    for (int c = 0; c < p->ncolors; ++c) {
      const int n = p->color_start[c + 1] - p->color_start[c];
      if (!n) continue;
      blocks_tp_kernel<Q, P><<<n, 256, smem, p->stream>>>(cell_data(p, p->cells_by_color.p + p->color_start[c], n), tab,
                                                          io);
      check_launch(p);
    }
  }
}

bool blocks_tp_dev(hfk_problem* p, const BlockIO& io) {
  if (p->Q < 2 || p->P < p->Q || p->nn != p->Q * p->Q * p->Q || p->np != p->P * p->P * p->P) return false;
  switch (p->Q * 10 + p->P) {
#define HFK_BCASE(Qv, Pv)             \
  case Qv * 10 + Pv:                  \
    blocks_tp_launch<Qv, Pv>(p, io); \
    return true;
    HFK_BCASE(2, 2)
    HFK_BCASE(2, 3)
    HFK_BCASE(2, 4)
    HFK_BCASE(2, 5)
    HFK_BCASE(3, 3)
    HFK_BCASE(3, 4)
    HFK_BCASE(3, 5)
    HFK_BCASE(4, 4)
    HFK_BCASE(4, 5)
    HFK_BCASE(5, 5)
#undef HFK_BCASE
    default:
      return false;
  }
}

void blocks_update_dev(hfk_problem* p, int* ok) {
  HFK_REQUIRE(p->prepared, HFK_ERR_STATE, "blocks need a prepared tangent (call hfk_mf_prepare)");
  if (p->bdofs.n == 0 && p->nblocks == 0) build_block_structure(p);
  if (p->nblocks == 0) {
    *ok = 1;
    p->blocks_ok = true;
    return;
  }
  p->B.zero(p->stream);
  BlockIO io{p->x.p, p->dvals.p, p->dNt.p, p->block_of.p, p->B.p, p->np, p->nn, 0};
  if (blocks_tp_dev(p, io)) {
    invert_blocks_and_check(p, ok);
    return;
  }
  const size_t smem = ((size_t)3 * p->nn + 9 * p->np + 9 * p->np + p->np + 81 * p->np) * sizeof(double);
  static PerDeviceLimit attr;
  raise_smem_limit(blocks_kernel, smem, attr);
  if (use_atomic_scatter(p)) {  // one launch over all cells, atomic accumulation of the blocks
    io.atomic = 1;
    blocks_kernel<<<p->ncells, 256, smem, p->stream>>>(cell_data(p, nullptr, p->ncells), io);
    check_launch(p);
  } else {
    for (int c = 0; c < p->ncolors; ++c) {
      const int n = p->color_start[c + 1] - p->color_start[c];
      if (!n) continue;
      blocks_kernel<<<n, 256, smem, p->stream>>>(cell_data(p, p->cells_by_color.p + p->color_start[c], n), io);
      check_launch(p);
    }
  }
  invert_blocks_and_check(p, ok);
}

template <typename R>
const R* binv_of(hfk_problem* p);
template <>
const double* binv_of<double>(hfk_problem* p) {
  return p->Binv.p;
}
template <>
const float* binv_of<float>(hfk_problem* p) {
  return p->Binv32.p;
}

template <typename R>
void blocks_apply_dev(hfk_problem* p, const R* r, R* y) {
  HFK_REQUIRE(p->blocks_ok || p->nblocks == 0 || p->Binv.p, HFK_ERR_STATE, "blocks not built (call hfk_blocks_update)");
  if (!p->nblocks) return;
  blocks_apply_kernel<R><<<vec_grid(p->nblocks), 256, 0, p->stream>>>(p->nblocks, p->bdofs.p, binv_of<R>(p), r, y);
  check_launch(p);
}

// ---- Chebyshev on device vectors (smooth!, src/smoothers.jl:116-146) ----------------------------
template <typename R>
struct ChebWork {
  DBuf<R> r, z, d;
  void ensure(int64_t n) {
    r.resize(n);
    z.resize(n);
    d.resize(n);
  }
};

template <typename R>
void cheb_smooth_dev(hfk_problem* p, ChebWork<R>& w, double a, double b, int degree, const R* rhs, R* x, bool zero_guess,
                     R* residual) {
  const int64_t n = p->nfree;
  w.ensure(n);
  const double th = (b + a) / 2, de = (b - a) / 2, sg = th / de;
  if (!zero_guess) mf_apply_any<R>(p, x, w.z.p);
  cheb_start_kernel<R><<<vec_grid(p->nblocks), 256, 0, p->stream>>>(p->nblocks, p->bdofs.p, binv_of<R>(p), rhs, w.z.p,
                                                                    w.r.p, w.d.p, x, (R)(1.0 / th), zero_guess ? 1 : 0);
  check_launch(p);
  double rho = 1.0 / sg;
  for (int i = 1; i <= degree; ++i) {
    // x += d was applied by the previous kernel
    if (i == degree && !residual) break;
    mf_apply_any<R>(p, w.d.p, w.z.p);  // z = A d
    const bool last = i == degree;
    double c1 = 0, c2 = 0, rn = 0;
    if (!last) {
      rn = 1.0 / (2 * sg - rho);
      c1 = rn * rho;
      c2 = 2 * rn / de;
    }
    cheb_step_kernel<R><<<vec_grid(p->nblocks), 256, 0, p->stream>>>(p->nblocks, p->bdofs.p, binv_of<R>(p), w.z.p,
                                                                      w.r.p, w.d.p, x, (R)c1, (R)c2, last ? 0 : 1);
    check_launch(p);
    if (last) break;
    rho = rn;
  }
  if (residual) HFK_CUDA(cudaMemcpyAsync(residual, w.r.p, n * sizeof(R), cudaMemcpyDeviceToDevice, p->stream));
}

// The same smoothing with the coefficients read from device memory (`coef`, see
// cheb_start_dev_kernel): used by the V-cycle, which is captured once in a CUDA graph.
// With segments, coef holds one coefficient set per segment (stride 1 + 2 degree).
template <typename R>
void cheb_smooth_coef(hfk_problem* p, ChebWork<R>& w, const double* coef, int degree, const R* rhs, R* x,
                      bool zero_guess, R* residual) {
  const int64_t n = p->nfree;
  const int cstride = 1 + 2 * degree;
  const int32_t* segb = seg_block_map(p);
  w.ensure(n);
  if (!zero_guess) mf_apply_any<R>(p, x, w.z.p);
  cheb_start_dev_kernel<R><<<vec_grid(p->nblocks), 256, 0, p->stream>>>(p->nblocks, p->bdofs.p, binv_of<R>(p), rhs,
                                                                        w.z.p, w.r.p, w.d.p, x, coef, segb, cstride,
                                                                        zero_guess ? 1 : 0);
  check_launch(p);
  for (int i = 1; i <= degree; ++i) {
    if (i == degree && !residual) break;
    mf_apply_any<R>(p, w.d.p, w.z.p);
    const bool last = i == degree;
    cheb_step_dev_kernel<R><<<vec_grid(p->nblocks), 256, 0, p->stream>>>(p->nblocks, p->bdofs.p, binv_of<R>(p), w.z.p,
                                                                          w.r.p, w.d.p, x, coef, segb, cstride, i,
                                                                          last ? 0 : 1);
    check_launch(p);
    if (last) break;
  }
  if (residual) HFK_CUDA(cudaMemcpyAsync(residual, w.r.p, n * sizeof(R), cudaMemcpyDeviceToDevice, p->stream));
}

// Chebyshev coefficients of smooth! (src/smoothers.jl:116-146) on [a, b]: [1/theta, c1_1, c2_1, ...]
std::vector<double> chebyshev_coefficients(double a, double b, int degree) {
  const double th = (b + a) / 2, de = (b - a) / 2, sg = th / de;
  std::vector<double> c(1 + 2 * (size_t)degree, 0.0);
  c[0] = 1.0 / th;
  double rho = 1.0 / sg;
  for (int i = 1; i < degree; ++i) {
    const double rn = 1.0 / (2 * sg - rho);
    c[2 * i - 1] = rn * rho;
    c[2 * i] = 2 * rn / de;
    rho = rn;
  }
  return c;
}

// ---- small dense eigenvalues (Francis double-shift QR on a Hessenberg matrix) ---------------------
// The eigvals call of eigenvalue_bounds (src/preconditioners.jl:386); real and imaginary parts.
bool hessenberg_eigvals(int n, std::vector<double> H /* column-major n x n */, double* re, double* im) {
  auto h = [&](int i, int j) -> double& { return H[i + (size_t)n * j]; };
  const double eps = 2.220446049250313e-16;
  int hi = n - 1, iter = 0;
  while (hi >= 0) {
    if (hi == 0) {
      re[0] = h(0, 0);
      im[0] = 0;
      hi = -1;
      break;
    }
    int l = hi;
    while (l > 0) {
      const double s = std::fabs(h(l - 1, l - 1)) + std::fabs(h(l, l));
      if (std::fabs(h(l, l - 1)) <= eps * (s == 0 ? 1.0 : s)) {
        h(l, l - 1) = 0;
        break;
      }
      --l;
    }
    if (l == hi) {
      re[hi] = h(hi, hi);
      im[hi] = 0;
      --hi;
      iter = 0;
      continue;
    }
    if (l == hi - 1) {
      const double a = h(hi - 1, hi - 1), b = h(hi - 1, hi), c = h(hi, hi - 1), d = h(hi, hi);
      const double m = 0.5 * (a + d), disc = 0.25 * (a - d) * (a - d) + b * c;
      if (disc >= 0) {
        const double s = std::sqrt(disc);
        re[hi - 1] = m + s;
        re[hi] = m - s;
        im[hi - 1] = im[hi] = 0;
      } else {
        const double s = std::sqrt(-disc);
        re[hi - 1] = re[hi] = m;
        im[hi - 1] = s;
        im[hi] = -s;
      }
      hi -= 2;
      iter = 0;
      continue;
    }
    if (++iter > 200 * n) return false;
    // shifts: eigenvalues of the trailing 2x2 (exceptional shifts every 11 iterations)
    double s, t;
    if (iter % 11 == 0) {
      const double e = std::fabs(h(hi, hi - 1)) + std::fabs(h(hi - 1, hi - 2));
      s = 1.5 * e;
      t = e * e;
    } else {
      s = h(hi - 1, hi - 1) + h(hi, hi);
      t = h(hi - 1, hi - 1) * h(hi, hi) - h(hi - 1, hi) * h(hi, hi - 1);
    }
    double x = h(l, l) * h(l, l) + h(l, l + 1) * h(l + 1, l) - s * h(l, l) + t;
    double y = h(l + 1, l) * (h(l, l) + h(l + 1, l + 1) - s);
    double z = h(l + 1, l) * h(l + 2, l + 1);
    for (int k = l; k <= hi - 2; ++k) {
      // Householder reflector mapping (x, y, z) onto the first axis
      const double nrm = std::sqrt(x * x + y * y + z * z);
      if (nrm > 0) {
        const double alpha = x > 0 ? -nrm : nrm;
        double u0 = x - alpha, u1 = y, u2 = z;
        const double uu = u0 * u0 + u1 * u1 + u2 * u2;
        if (uu > 0) {
          const double f = 2.0 / uu;
          const int c0 = std::max(l, k - 1);
          for (int j = c0; j <= hi; ++j) {
            const double sdot = u0 * h(k, j) + u1 * h(k + 1, j) + u2 * h(k + 2, j);
            h(k, j) -= f * u0 * sdot;
            h(k + 1, j) -= f * u1 * sdot;
            h(k + 2, j) -= f * u2 * sdot;
          }
          const int r1 = std::min(k + 3, hi);
          for (int i = l; i <= r1; ++i) {
            const double sdot = u0 * h(i, k) + u1 * h(i, k + 1) + u2 * h(i, k + 2);
            h(i, k) -= f * u0 * sdot;
            h(i, k + 1) -= f * u1 * sdot;
            h(i, k + 2) -= f * u2 * sdot;
          }
        }
      }
      x = h(k + 1, k);
      y = h(k + 2, k);
      if (k < hi - 2) z = h(k + 3, k);
    }
    // final Givens rotation on rows/columns hi-1, hi
    {
      const double r = std::hypot(x, y);
      if (r > 0) {
        const double c = x / r, sn = y / r;
        const int k = hi - 1;
        for (int j = std::max(l, k - 1); j <= hi; ++j) {
          const double a = h(k, j), b = h(k + 1, j);
          h(k, j) = c * a + sn * b;
          h(k + 1, j) = -sn * a + c * b;
        }
        for (int i = l; i <= hi; ++i) {
          const double a = h(i, k), b = h(i, k + 1);
          h(i, k) = c * a + sn * b;
          h(i, k + 1) = -sn * a + c * b;
        }
      }
    }
  }
  return true;
}

struct EigWork {
  DBuf<double> V, Z, t, w, pw, Hd, h2, part;
};

// eigenvalue_bounds (src/preconditioners.jl:374-389) of every segment at once: k Arnoldi steps
// (classical Gram-Schmidt with one reorthogonalisation) on J P^-1 from the start vector with per-segment inner products, so that
// each segment builds its own Hessenberg matrix (a block-diagonal operator keeps the segments'
// Krylov spaces apart); breakdown truncation and Ritz values per segment on the host. One copy
// of the Hessenberg matrices to the host, no other synchronisation.
// pinner: orthogonalise in the P^-1 inner product <u, v> = u . P^-1 v instead of the Euclidean one
// (an option of this engine): J P^-1 is self-adjoint in it, so H is symmetric and its Ritz values
// lie inside the spectrum; the Euclidean process (the reference's) can give Ritz values outside the
// spectrum of a strongly non-normal J P^-1. Z = P^-1 V is kept beside V, so each step costs one
// more block application and one more update per basis vector.
void eig_bounds_dev(hfk_problem* p, EigWork& ew, int k, const double* start_dev, std::vector<double>& lmin,
                    std::vector<double>& lmax, bool pinner = false) {
  const int64_t n = p->nfree;
  const int ns = p->nseg;
  k = (int)std::max<int64_t>(1, std::min<int64_t>(k, n));
  const int ld = k + 1;
  const int hs = ld * (k + 1);  // per segment: H (ld x k) and one scratch column
  ew.V.resize((size_t)(k + 1) * n);
  ew.t.resize(n);
  ew.w.resize(n);
  ew.Hd.resize((size_t)hs * ns);
  ew.Hd.zero(p->stream);
  ew.h2.resize((size_t)hs * ns);
  ensure_seg_items(p);
  ew.part.resize((size_t)SEG_MDOTS * std::max(p->nitems, 1));
  double* Hd = ew.Hd.p;
  const int32_t* seg = seg_dof_map(p);
  const int sg = std::max(1, (ns + 255) / 256);
  double* nrm = Hd + (size_t)ld * k;  // scratch scalar past each Hessenberg matrix
  auto V = [&](int i) { return ew.V.p + (size_t)i * n; };
  auto Z = [&](int i) { return ew.Z.p + (size_t)i * n; };
  if (pinner) {
    ew.Z.resize((size_t)(k + 1) * n);
    ew.pw.resize(n);
    blocks_apply_dev<double>(p, start_dev, ew.t.p);
    seg_dots<double>(p, 1, nrm, hs, start_dev, ew.t.p);
  } else {
    seg_dots<double>(p, 1, nrm, hs, start_dev, start_dev);
  }
  seg_sqrt_kernel<<<sg, 256, 0, p->stream>>>(ns, nrm, hs);
  check_launch(p);
  seg_scale_kernel<<<vec_grid(n), 256, 0, p->stream>>>(n, seg, nrm, hs, start_dev, V(0));
  check_launch(p);
  if (pinner) {
    seg_scale_kernel<<<vec_grid(n), 256, 0, p->stream>>>(n, seg, nrm, hs, ew.t.p, Z(0));
    check_launch(p);
  }
  for (int j = 0; j < k; ++j) {
    if (pinner) {
      mf_apply_dev(p, Z(j), ew.w.p);
      blocks_apply_dev<double>(p, ew.w.p, ew.pw.p);
    } else {
      blocks_apply_dev<double>(p, V(j), ew.t.p);
      mf_apply_dev(p, ew.t.p, ew.w.p);
    }
    // classical Gram-Schmidt with one reorthogonalisation: h = B^T w, w -= V h (and pw -= Z h in
    // the P^-1 inner product, B = Z; else B = V), twice, the second pass's coefficients added to
    // the first's; one multi-dot and one multi-axpy launch per pass and 16 basis vectors
    for (int pass = 0; pass < 2; ++pass) {
      double* hc = pass == 0 ? Hd + (size_t)ld * j : ew.h2.p;  // per segment at stride hs
      for (int c0 = 0; c0 <= j; c0 += SEG_MDOTS) {
        const int kc = std::min(SEG_MDOTS, j + 1 - c0);
        if (p->nitems) {
          seg_mdots_kernel<<<p->nitems, RED_THREADS, 0, p->stream>>>(kc, p->item_lo.p, p->item_hi.p,
                                                                    pinner ? Z(c0) : V(c0), n, ew.w.p, ew.part.p);
          check_launch(p);
        }
        seg_mfinish_kernel<<<ns, RED_THREADS, 0, p->stream>>>(kc, p->item_first.p, ew.part.p, hc + c0, hs);
        check_launch(p);
      }
      for (int c0 = 0; c0 <= j; c0 += SEG_MDOTS) {
        const int kc = std::min(SEG_MDOTS, j + 1 - c0);
        seg_maxpy_kernel<<<vec_grid(n), 256, 0, p->stream>>>(n, seg, kc, hc + c0, hs, V(c0), n, ew.w.p);
        check_launch(p);
        if (pinner) {
          seg_maxpy_kernel<<<vec_grid(n), 256, 0, p->stream>>>(n, seg, kc, hc + c0, hs, Z(c0), n, ew.pw.p);
          check_launch(p);
        }
      }
    }
    seg_add_kernel<<<std::max(1, (ns * (j + 1) + 255) / 256), 256, 0, p->stream>>>(ns, j + 1, ew.h2.p,
                                                                                 Hd + (size_t)ld * j, hs);
    check_launch(p);
    double* hn = Hd + (j + 1) + (size_t)ld * j;
    seg_dots<double>(p, 1, hn, hs, ew.w.p, pinner ? ew.pw.p : ew.w.p);
    seg_sqrt_kernel<<<sg, 256, 0, p->stream>>>(ns, hn, hs);
    check_launch(p);
    seg_scale_kernel<<<vec_grid(n), 256, 0, p->stream>>>(n, seg, hn, hs, ew.w.p, V(j + 1));
    check_launch(p);
    if (pinner) {
      seg_scale_kernel<<<vec_grid(n), 256, 0, p->stream>>>(n, seg, hn, hs, ew.pw.p, Z(j + 1));
      check_launch(p);
    }
  }
  std::vector<double> Hall((size_t)hs * ns);
  HFK_CUDA(cudaMemcpyAsync(Hall.data(), Hd, sizeof(double) * Hall.size(), cudaMemcpyDeviceToHost, p->stream));
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  lmin.assign(ns, NAN);
  lmax.assign(ns, NAN);
  for (int s = 0; s < ns; ++s) {
    const double* H = Hall.data() + (size_t)hs * s;
    // breakdown truncation (src/preconditioners.jl:379-385)
    int jj = k;
    for (int i = 1; i < k; ++i) {
      double m = 0;
      for (int a = 0; a < i; ++a)
        for (int b = 0; b < i; ++b) m = std::max(m, std::fabs(H[a + (size_t)ld * b]));
      if (std::fabs(H[i + (size_t)ld * (i - 1)]) <= 1e-8 * std::max(1.0, m)) {
        jj = i;
        break;
      }
    }
    std::vector<double> Hs((size_t)jj * jj);
    for (int a = 0; a < jj; ++a)
      for (int b = 0; b < jj; ++b) Hs[a + (size_t)jj * b] = H[a + (size_t)ld * b];
    std::vector<double> re(jj), im(jj);
    if (!hessenberg_eigvals(jj, Hs, re.data(), im.data())) continue;
    lmin[s] = *std::min_element(re.begin(), re.end());
    lmax[s] = *std::max_element(re.begin(), re.end());
  }
}

// The fixed start vector of the eigenvalue estimate (src/smoothers.jl:68-71); with segments, each
// segment gets the vector of its own size (so that it sees the start of a problem solved alone).
void chebyshev_start_vector(const hfk_problem* p, std::vector<double>& v) {
  v.resize(p->nfree);
  const int ns = p->seg_off.empty() ? 1 : p->nseg;
  for (int sg = 0; sg < ns; ++sg) {
    const int64_t a = p->seg_off.empty() ? 0 : p->seg_off[sg], e = p->seg_off.empty() ? p->nfree : p->seg_off[sg + 1];
    double s = 0;
    for (int64_t i = a; i < e; ++i) {
      const double ii = (double)(i - a + 1);
      v[i] = std::sin(1.0 + 0.7 * ii) + 0.3 * std::cos(2.3 * ii);
      s += v[i] * v[i];
    }
    s = std::sqrt(s);
    for (int64_t i = a; i < e; ++i) v[i] /= s;
  }
}

// ---- GPU sparsity pattern (sparsity, src/assembly.jl:773-818; cell_positions!, :864-880) -----------
__global__ void pattern_keys_kernel(int ncells, int ndl, const int32_t* ids, uint64_t* keys, unsigned long long* count) {
  // one block per cell: keys (col << 32) | row of every free (row, col) pair
  const int cell = blockIdx.x;
  if (cell >= ncells) return;
  const int32_t* id = ids + (size_t)cell * ndl;
  __shared__ unsigned long long base;
  __shared__ int nfree_local;
  __shared__ int32_t fids[384];
  if (threadIdx.x == 0) {
    int c = 0;
    for (int j = 0; j < ndl; ++j)
      if (id[j] > 0) fids[c++] = id[j];
    nfree_local = c;
    base = atomicAdd(count, (unsigned long long)c * c);
  }
  __syncthreads();
  const int m = nfree_local;
  for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
    const int a = e % m, b = e / m;
    keys[base + e] = ((uint64_t)(uint32_t)fids[b] << 32) | (uint64_t)(uint32_t)fids[a];
  }
}

__global__ void pattern_csc_kernel(int64_t nnz, int64_t ncols, const uint64_t* keys, int64_t* rowval, int64_t* colptr) {
  // sorted unique keys: rowval, and colptr (1-based) at the first entry of every column; every
  // column is non-empty (the diagonal entry of a free dof is always a key)
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t key = keys[k];
    rowval[k] = (int64_t)(key & 0xffffffffu);
    const int64_t col = (int64_t)(key >> 32);
    if (k == 0 || (keys[k - 1] >> 32) != (uint64_t)col) colptr[col - 1] = k + 1;
    if (k == 0) colptr[ncols] = nnz + 1;
  }
}

__global__ void nzpos_kernel(int ncells, int ndl, const int32_t* ids, const int64_t* colptr, const int64_t* rowval,
                             int32_t* nzpos) {
  const int64_t per = (int64_t)ndl * ndl;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)ncells * per;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int cell = (int)(e / per);
    const int r = (int)(e % per), ii = r % ndl, jj = r / ndl;
    const int32_t* id = ids + (size_t)cell * ndl;
    const int32_t c = id[jj], rw = id[ii];
    int32_t pos = 0;
    if (c > 0 && rw > 0) {
      int64_t lo = colptr[c - 1] - 1, hi = colptr[c] - 1;
      const int64_t end = hi;
      while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (rowval[mid] < rw) lo = mid + 1;
        else hi = mid;
      }
      if (lo < end && rowval[lo] == rw) pos = (int32_t)(lo + 1);
    }
    nzpos[e] = pos;
  }
}

}  // namespace
void hfk::pattern_build_dev(hfk_problem* p) {
  if (p->nnz > 0) return;
  HFK_REQUIRE(p->ndl <= 384, HFK_ERR_UNSUPPORTED, "pattern construction supports up to 384 dofs per cell");
  // count keys
  std::vector<int64_t> nf_cell(p->ncells);
  size_t total = 0;
  for (int cell = 0; cell < p->ncells; ++cell) {
    int c = 0;
    for (int j = 0; j < p->ndl; ++j) c += p->h_ids[(size_t)cell * p->ndl + j] > 0;
    total += (size_t)c * c;
  }
  DBuf<uint64_t> keys, keys2;
  DBuf<unsigned long long> cnt;
  keys.resize(std::max<size_t>(total, 1));
  keys2.resize(std::max<size_t>(total, 1));
  cnt.resize(1);
  cnt.zero(p->stream);
  pattern_keys_kernel<<<p->ncells, 256, 0, p->stream>>>(p->ncells, p->ndl, p->ids.p, keys.p, cnt.p);
  check_launch(p);
  int end_bit = 32;
  while (end_bit < 64 && ((uint64_t)1 << (end_bit - 32)) <= (uint64_t)p->nfree) ++end_bit;
  size_t tmp_bytes = 0;
  HFK_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, keys.p, keys2.p, (int64_t)total, 0, end_bit, p->stream));
  DBuf<unsigned char> tmp;
  tmp.resize(tmp_bytes);
  HFK_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, tmp_bytes, keys.p, keys2.p, (int64_t)total, 0, end_bit, p->stream));
  DBuf<int64_t> nsel;
  nsel.resize(1);
  size_t tmp2 = 0;
  HFK_CUDA(cub::DeviceSelect::Unique(nullptr, tmp2, keys2.p, keys.p, nsel.p, (int64_t)total, p->stream));
  if (tmp2 > tmp.n) tmp.resize(tmp2);
  HFK_CUDA(cub::DeviceSelect::Unique(tmp.p, tmp2, keys2.p, keys.p, nsel.p, (int64_t)total, p->stream));
  int64_t nnz = 0;
  HFK_CUDA(cudaMemcpyAsync(&nnz, nsel.p, sizeof(int64_t), cudaMemcpyDeviceToHost, p->stream));
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  p->nnz = nnz;
  p->rowval.resize(std::max<int64_t>(nnz, 1));
  p->colptr.resize(p->nfree + 1);
  pattern_csc_kernel<<<vec_grid(nnz), 256, 0, p->stream>>>(nnz, p->nfree, keys.p, p->rowval.p, p->colptr.p);
  check_launch(p);
  // 16 bytes of slack: the assembly kernels copy a cell's positions in 16-byte pieces from the
  // 16-byte boundary below its first one, so the last cell's copy may reach 12 bytes past its end
  p->nzpos.resize((size_t)p->ndl * p->ndl * p->ncells + 4);
  nzpos_kernel<<<vec_grid((int64_t)p->ndl * p->ndl * p->ncells), 256, 0, p->stream>>>(p->ncells, p->ndl, p->ids.p,
                                                                                      p->colptr.p, p->rowval.p,
                                                                                      p->nzpos.p);
  check_launch(p);
  p->nzval.resize(std::max<int64_t>(nnz, 1));
  HFK_CUDA(cudaStreamSynchronize(p->stream));
}
namespace {

// after_chunk (atomic scatter only): the cells are launched in the chunks of jc_start, and
// after_chunk(k) runs (on the host, in launch order) right after chunk k's launch
void jacobian_dev(hfk_problem* p, const double* u, const double* dvals, double* nzval,
                  const std::function<void(int)>* after_chunk = nullptr) {
  pattern_build_dev(p);
  HFK_CUDA(cudaMemsetAsync(nzval, 0, p->nnz * sizeof(double), p->stream));
  const bool g = p->nn == 27;
  HFK_REQUIRE(p->nn == 27 || p->nn <= 8, HFK_ERR_UNSUPPORTED, "assembled Jacobians support 8- and 27-node cells");
  // 27-node cells: G_c padded (conflict-free, select-free tensor-core fragments) when it fits
  const bool padded = g && asm_smem_bytes(p->nn, p->np, true, ASM_LDG_PADDED) <= 227 * 1024;
  const int ldg = g ? (padded ? ASM_LDG_PADDED : 3 * p->nn) : 0;
  AsmIO io{u, dvals, p->dNt.p, p->nzpos.p, nzval, p->np, ldg};
  const size_t smem = asm_smem_bytes(p->nn, p->np, g, ldg);
  HFK_REQUIRE(smem <= 227 * 1024, HFK_ERR_UNSUPPORTED, "too many quadrature points for the assembly kernel");
  HFK_REQUIRE(g || p->nn == 8, HFK_ERR_UNSUPPORTED, "assembled Jacobians support 8- and 27-node cells");
  // the recognised laws are hyperelastic (symmetric tangent): only the element blocks k >= c are
  // formed; on 27-node cells by the FP64 FMA kernel when its shared memory fits, else on the FP64
  // tensor cores
  const bool sym = p->law == HFK_LAW_SVK || p->law == HFK_LAW_LINEAR_ELASTIC;
  const size_t smem_s = sym27_smem_bytes(p->np, ASM_SYM27_QC);
  const bool fma27 = g && sym && p->asm_kernel != 1 && smem_s <= 227 * 1024 && sym27_fits(p->np, ASM_SYM27_QC);
  auto kern_g = padded ? (sym ? jacobian_kernel_g<27, true, true> : jacobian_kernel_g<27, true, false>)
                       : (sym ? jacobian_kernel_g<27, false, true> : jacobian_kernel_g<27, false, false>);
  // on Q2 cells with 3^3 Gauss points the product is the sum-factorised contraction
  const bool tp27 = p->Q == 3 && p->P == 3 && ASM_SYM27_QC == 9;
  auto kern_s = tp27 ? jacobian_kernel_sym27<true, 9, ASM_SYM27_MINB_TP>
                     : jacobian_kernel_sym27<false, ASM_SYM27_QC, ASM_SYM27_MINB>;
  const Tab1D<double> tab = make_tab<double>(p);
  int grid_s = 0;  // the FMA kernel's persistent CTAs: as many as are resident at once
  if (fma27) {
    static PerDeviceLimit attr[2];
    raise_smem_limit(kern_s, smem_s, attr[tp27]);
    // resident CTAs per SM, per (device, variant, shared-memory size): the dense variant's size
    // depends on the number of points
    static std::mutex occ_mutex;
    static std::map<std::tuple<int, bool, size_t>, int> occ;
    int dev = 0;
    HFK_CUDA(cudaGetDevice(&dev));
    int per_sm = 0;
    {
      std::lock_guard<std::mutex> lock(occ_mutex);
      auto it = occ.find({dev, tp27, smem_s});
      if (it == occ.end()) {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern_s, 256, smem_s) != cudaSuccess) b = 1;
        it = occ.emplace(std::make_tuple(dev, tp27, smem_s), std::max(b, 1)).first;
      }
      per_sm = it->second;
    }
    grid_s = per_sm * sm_count();
  } else if (g) {
    static PerDeviceLimit attr[4];
    raise_smem_limit(kern_g, smem, attr[2 * padded + sym]);
  } else {
    static PerDeviceLimit attr;
    raise_smem_limit(jacobian_kernel_direct<8>, smem, attr);
  }
  auto launch = [&](const int32_t* cells, int n) {
    CellData cd = cell_data(p, cells, n);
    if (fma27) kern_s<<<std::min(n, grid_s), 256, smem_s, p->stream>>>(cd, io, tab);
    else if (g) kern_g<<<n, 256, smem, p->stream>>>(cd, io);
    else jacobian_kernel_direct<8><<<n, 256, smem, p->stream>>>(cd, io);
    check_launch(p);
  };
  // the atomic scatter (the default) assembles every cell in one launch: CTAs of neighbouring cells
  // may then add to the same nonzero, in an order that can change the last bit from run to run; by
  // colour (HFK_SCATTER_COLOURED) the adds of one nonzero come one launch after another, in colour
  // order, and the result is reproducible bit for bit
  ktimer_mark(p);
  if (use_atomic_scatter(p) && after_chunk) {
    for (size_t k = 0; k + 1 < p->jc_start.size(); ++k) {
      const int c0 = p->jc_start[k], n = p->jc_start[k + 1] - c0;
      if (n) launch(p->jc_cells.p + c0, n);
      (*after_chunk)((int)k);
    }
  } else if (use_atomic_scatter(p)) {
    if (p->ncells) launch(nullptr, p->ncells);
  } else {
    for (int c = 0; c < p->ncolors; ++c) {
      const int n = p->color_start[c + 1] - p->color_start[c];
      if (n) launch(p->cells_by_color.p + p->color_start[c], n);
    }
  }
  ktimer_mark(p);
}

// The chunks of the host-output assembly (once per problem): at least two full waves of CTAs each,
// at most 8; per chunk the CSC values that are complete once it has run: the columns below the
// smallest free dof any later chunk's cells touch (every cell of a later chunk adds only to the
// columns of its own dofs)
void jacobian_chunks(hfk_problem* p) {
  if (!p->jc_start.empty()) return;
  const int K = (int)std::max<int64_t>(1, std::min<int64_t>(8, p->ncells / (2 * (int64_t)sm_count() * 2)));
  p->jc_start.assign(K + 1, 0);
  for (int k = 0; k <= K; ++k) p->jc_start[k] = (int)((int64_t)p->ncells * k / K);
  std::vector<int32_t> all(p->ncells);
  for (int c = 0; c < p->ncells; ++c) all[c] = c;
  p->jc_cells.upload(all.data(), all.size(), p->stream);
  std::vector<int64_t> colptr(p->nfree + 1);
  HFK_CUDA(cudaMemcpyAsync(colptr.data(), p->colptr.p, colptr.size() * sizeof(int64_t), cudaMemcpyDeviceToHost,
                           p->stream));
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  // smallest free id (1-based) over the cells from chunk k on, for k = K-1 .. 1
  std::vector<int64_t> minid(K + 1, p->nfree + 1);
  for (int k = K - 1; k >= 0; --k) {
    int64_t m = minid[k + 1];
    for (int c = p->jc_start[k]; c < p->jc_start[k + 1]; ++c)
      for (int j = 0; j < p->ndl; ++j) {
        const int32_t id = p->h_ids[(size_t)c * p->ndl + j];
        if (id > 0) m = std::min<int64_t>(m, id);
      }
    minid[k] = m;
  }
  p->jc_done.assign(K, p->nnz);
  for (int k = 0; k + 1 < K; ++k) p->jc_done[k] = colptr[minid[k + 1] - 1] - 1;  // columns < minid - 1
  p->jc_done[K - 1] = p->nnz;
}

void residual_dev(hfk_problem* p, const double* u, const double* dvals, double* b) {
  require_tp(p);
  HFK_CUDA(cudaMemsetAsync(b, 0, p->nfree * sizeof(double), p->stream));
  CellIO<double> io{};
  io.u = u;
  io.dvals = dvals;
  io.y = b;
  run_cells<MODE_RESIDUAL, double>(p, io);
}

}  // namespace

// ---- functionals (KernelFunctional, src/functionals.jl:10-27) ----------------------------------
__global__ void functional_finish_kernel(int64_t nw, const double* red, double* out) {
  double s = 0, mn = INFINITY;
  for (int64_t i = threadIdx.x; i < nw; i += blockDim.x) {
    s += red[2 * i];
    mn = fmin(mn, red[2 * i + 1]);
  }
  __shared__ double ss[32], sm[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    ss[w] = s;
    sm[w] = mn;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = INFINITY;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
      a += ss[i];
      b = fmin(b, sm[i]);
    }
    out[0] = a;
    out[1] = b;
  }
}

// out[0] = Σ_cells Σ_q Ψ(F) dV, out[1] = min_q det F (device), at the state (u, dvals)
void functional_dev(hfk_problem* p, const double* u, const double* dvals, double* out) {
  require_tp(p);
  constexpr int WARPS = 4;
  const int m = std::max(p->Q, p->P);
  const int cpw = std::max(1, 32 / (m * m));
  const int64_t grid = ((int64_t)p->ncells + WARPS * cpw - 1) / (WARPS * cpw);
  const int64_t nw = grid * WARPS;
  p->func_red.resize((size_t)2 * nw);
  CellIO<double> io{};
  io.u = u;
  io.dvals = dvals;
  io.red = p->func_red.p;
  dispatch_cell<MODE_ENERGY, double>(p, nullptr, p->ncells, io, WARPS);
  functional_finish_kernel<<<1, 1024, 0, p->stream>>>(nw, p->func_red.p, out);
  check_launch(p);
}

// ---- transfers and p-multigrid handles ---------------------------------------------------------
struct hfk_transfer {
  hfk_problem* fine = nullptr;
  hfk_problem* coarse = nullptr;
  int NF = 0, NC = 0;
  DBuf<double> E, Einj;
  DBuf<int32_t> mult;
  // the transfer's colours: those of the fine level (cells sharing a coarse dof share a fine dof)
  // tensor-product pair of levels (E = E1 x E1 x E1): the sum-factorised kernels
  bool tp = false;
  XferTP tpd;
  DBuf<double> invmult;
};

namespace {
XferData xfer_data(hfk_transfer* t, const int32_t* cells, int ncl) {
  XferData d;
  d.ids_f = t->fine->ids.p;
  d.ids_c = t->coarse->ids.p;
  d.E = t->E.p;
  d.Einj = t->Einj.p;
  d.mult = t->mult.p;
  d.cells = cells;
  d.ncells_list = ncl;
  d.NF = t->NF;
  d.NC = t->NC;
  return d;
}

// warps per CTA of the sum-factorised transfer kernels and their dynamic shared memory
int xfer_tp_warps(const hfk_transfer* t) {
  return 4 * xfer_tp_slab(t->tpd.nf, t->tpd.nc) * (int)sizeof(double) <= 48 * 1024 ? 4 : 2;
}

template <typename R>
void prolongate_dev(hfk_transfer* t, const R* xc, R* yf) {
  hfk_problem* p = t->fine;
  HFK_CUDA(cudaMemsetAsync(yf, 0, p->nfree * sizeof(R), p->stream));
  if (t->tp) {
    const int w = xfer_tp_warps(t);
    prolongate_tp_kernel<R><<<(p->ncells + w - 1) / w, 32 * w, w * xfer_tp_slab(t->tpd.nf, t->tpd.nc) * sizeof(double),
                              p->stream>>>(xfer_data(t, nullptr, p->ncells), t->tpd, xc, yf);
    check_launch(p);
    return;
  }
  for (int c = 0; c < p->ncolors; ++c) {
    const int n = p->color_start[c + 1] - p->color_start[c];
    if (!n) continue;
    prolongate_kernel<R><<<vec_grid((int64_t)n * 3 * t->NF), 256, 0, p->stream>>>(
        xfer_data(t, p->cells_by_color.p + p->color_start[c], n), xc, yf);
    check_launch(p);
  }
}

template <typename R>
void restrict_dev(hfk_transfer* t, const R* yf, R* yc) {
  hfk_problem* p = t->fine;
  HFK_CUDA(cudaMemsetAsync(yc, 0, t->coarse->nfree * sizeof(R), p->stream));
  if (t->tp) {
    // one atomic launch, or colour by colour (reproducible sums) when the fine level scatters so
    const int w = xfer_tp_warps(t);
    const size_t sm = (size_t)w * xfer_tp_slab(t->tpd.nf, t->tpd.nc) * sizeof(double);
    if (p->scatter != HFK_SCATTER_COLOURED) {
      restrict_tp_kernel<R><<<(p->ncells + w - 1) / w, 32 * w, sm, p->stream>>>(xfer_data(t, nullptr, p->ncells),
                                                                                 t->tpd, 1, yf, yc);
      check_launch(p);
      return;
    }
    for (int c = 0; c < p->ncolors; ++c) {
      const int n = p->color_start[c + 1] - p->color_start[c];
      if (!n) continue;
      restrict_tp_kernel<R><<<(n + w - 1) / w, 32 * w, sm, p->stream>>>(
          xfer_data(t, p->cells_by_color.p + p->color_start[c], n), t->tpd, 0, yf, yc);
      check_launch(p);
    }
    return;
  }
  for (int c = 0; c < p->ncolors; ++c) {
    const int n = p->color_start[c + 1] - p->color_start[c];
    if (!n) continue;
    restrict_kernel<R><<<vec_grid((int64_t)n * 3 * t->NC), 256, 0, p->stream>>>(
        xfer_data(t, p->cells_by_color.p + p->color_start[c], n), yf, yc);
    check_launch(p);
  }
}

void inject_dev(hfk_transfer* t, const double* xf, const double* df, double* xc, double* dc) {
  hfk_problem* p = t->fine;
  inject_kernel<<<vec_grid((int64_t)p->ncells * 3 * t->NC), 256, 0, p->stream>>>(xfer_data(t, nullptr, p->ncells),
                                                                                 p->ncells, xf, df, xc, dc);
  check_launch(p);
}
}  // namespace

// The learned correction's network (FP32 master weights, BF16 copy, Adam moments)
template <typename R>
struct LevelWork {
  DBuf<R> b, x, r, e;
  ChebWork<R> cheb;
};

// coarse mode of a one-level block-Jacobi slot (not a public value of hfk_pmg_set_coarse)
constexpr int COARSE_BLOCKS = 2;

struct hfk_pmg {
  int L = 0;
  std::vector<hfk_problem*> lv;
  std::vector<hfk_transfer*> tr;
  int degree = 2;
  double range = 20, inflate = 1.1;
  int eig_iters = 10, coarse_every = 1, precision = HFK_FP64;
  std::vector<double> a, b, lmin, lmax;
  std::vector<char> lok;
  bool ok = false, built = false;
  // a failed update that met an indefinite tangent: on some smoothing level finite blocks and a
  // finite estimate with a non-positive Ritz value (preconditioner_indefinite, src/pmultigrid.jl:343;
  // smoother_indefinite, src/smoothers.jl:48)
  bool indefinite = false;
  int since = 0, nupdate = 0, nbuild = 0;
  int band = -1;  // lower bandwidth of the coarse level's pattern (computed once)
  std::vector<std::unique_ptr<LevelWork<double>>> w64;
  std::vector<std::unique_ptr<LevelWork<float>>> w32;
  // coarse: dense Cholesky factor (lower) of the assembled coarse tangent, or (HFK_COARSE_CG) a
  // fixed number of block-Jacobi CG steps per segment on the matrix-free coarse level
  int coarse_mode = HFK_COARSE_CHOLESKY, coarse_iters = 20;  // or COARSE_BLOCKS (a block-Jacobi slot)
  int eig_inner = HFK_EIG_EUCLIDEAN;  // inner product of the eigenvalue estimate
  DBuf<double> Lb, cb, cx;  // Lb: the coarse Cholesky factor in band storage (kern_chol.cuh)
  int cb_nbt = 0, cb_W = 0;  // its block rows and lower block bandwidth
  DBuf<int> cb_info;         // first block column with a bad pivot (1-based), 0 = none
  DBuf<double> ccg_r, ccg_z, ccg_p, ccg_q, ccg_sc;
  bool coarse_ok = false;
  std::vector<std::unique_ptr<EigWork>> ew;          // per level (no reallocation between levels)
  std::vector<std::vector<double>> seg_lmin, seg_lmax;  // per level, per segment
  std::vector<std::unique_ptr<DBuf<double>>> start;  // per level: the fixed Arnoldi start vector
  // banded factor: the block tiles of both triangular solves (kern_band.cuh), rebuilt with the
  // factor; bs_sync holds both directions' tickets, then the error word
  bool bs_on = false;
  int bs_nb = 0, bs_wt = 0;
  // the coarse build runs on a side stream while the smoothers are set up (enqueued by
  // coarse_factor_launch, collected by coarse_factor_finish)
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_c0 = nullptr, ev_c1 = nullptr, ev_p0 = nullptr, ev_p1 = nullptr;
  cudaStream_t cb_stream = nullptr;  // the factorisation's lookahead stream (the trailing updates)
  std::vector<cudaEvent_t> cb_ev;    // its two ordering events (panel done, update rest done)
  bool cf_pending = false;
  DBuf<double> bs_tiles, bs_diag, bs_y;
  DBuf<int> bs_sync;
  DBuf<double> top_r, top_y;
  double t_potrf = 0;  // time of the factorisations proper (ms)
  int bs_spin = BS_SPIN_LIMIT;  // polls before a wait of the block triangular solves gives up
  int bs_skip = 0;              // test knob: the next forward solve starts its tickets at 1
  // learned correction after each cycle (null = plain cycle) and its work buffers
  hfk_mlp* mlp = nullptr;
  DBuf<double> ml_s, ml_t, ml_q, ml_delta, ml_scal;  // ml_scal: 8 per segment
  DBuf<float> ml_feats, ml_out, ml_loglm;                    // ml_loglm: log lambda, log mu per segment
  DBuf<int> ml_accepted;
  int64_t ml_tried = 0;
  // Chebyshev coefficients per level on the device (rewritten at every update)
  std::vector<std::unique_ptr<DBuf<double>>> coef;
  // the V-cycle as a CUDA graph, captured on the second cycle and replayed until a level's law
  // parameters change (the coefficients and states it reads live in fixed device buffers)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  int cycles_since_update = 0;
  std::vector<double> graph_params;
  // statistics: times in ms (host wall clock for the update phases, CUDA events for the cycles)
  double t_update = 0, t_coarse = 0, t_blocks = 0, t_eig = 0, t_cycle = 0;
  int64_t ncycles = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool ev_pending = false;
};

namespace {

// every level launches on level 0's stream (which the caller may have changed since)
void pmg_bind_stream(hfk_pmg* m) {
  for (int l = 1; l < m->L; ++l) m->lv[l]->stream = m->lv[0]->stream;
}

__global__ void lower_bandwidth_kernel(int64_t n, const int64_t* colptr, const int64_t* rowval, int* band) {
  int mine = 0;
  for (int64_t c = blockIdx.x; c < n; c += gridDim.x)
    for (int64_t k = colptr[c] - 1 + threadIdx.x; k < colptr[c + 1] - 1; k += blockDim.x)
      mine = max(mine, (int)(rowval[k] - 1 - c));
  atomicMax(band, mine);
}

// The tiles of the block triangular solves (kern_band.cuh) from the band factor in m->Lb: the band
// of each block row and block column copied into BS_T x BS_T tiles, then every tile multiplied by
// the inverse of its step's diagonal block (tile_trsm_kernel; the identity tile becomes D^-1).
void band_prepare(hfk_pmg* m, int64_t n) {
  hfk_problem* c = m->lv[m->L - 1];
  const int nb = (int)((n + BS_T - 1) / BS_T);
  const int wt = std::min(nb - 1, (m->band + BS_T - 1) / BS_T);
  const size_t tt = (size_t)BS_T * BS_T;
  const size_t per = (size_t)(wt + 1) * tt;
  m->bs_tiles.resize((size_t)2 * nb * per);
  m->bs_diag.resize((size_t)2 * nb * tt);
  m->bs_y.resize(n);
  m->bs_sync.resize(3);  // the two directions' tickets, the error word
  if (m->bs_nb != nb || m->bs_wt != wt) {
    m->bs_sync.zero(c->stream);
    m->bs_nb = nb;
    m->bs_wt = wt;
  }
  const int64_t total = (int64_t)2 * nb * (wt + 2) * (int64_t)tt;
  band_tiles_kernel<<<(int)std::min<int64_t>((total + 255) / 256, (int64_t)sm_count() * 64), 256, 0, c->stream>>>(
      n, nb, wt, m->Lb.p, m->cb_W, m->bs_tiles.p, m->bs_diag.p);
  check_launch(c);
  const size_t smem = (tt + tt / 2 + BS_T) * sizeof(double);
  static PerDeviceLimit attr;
  raise_smem_limit(tile_trsm_kernel<BS_T>, smem, attr);
  tile_trsm_kernel<BS_T><<<2 * nb * (wt + 1), 2 * BS_T, smem, c->stream>>>(nb, wt, m->bs_diag.p, m->bs_tiles.p);
  check_launch(c);
}

// the error word of the block triangular solves: a wait between blocks that ran out (the cycle's
// coarse correction is then invalid)
void band_check(hfk_pmg* m) {
  if (!m->bs_on || !m->bs_sync.p) return;
  int e = 0;
  hfk_problem* c = m->lv[m->L - 1];
  int* word = m->bs_sync.p + 2;
  HFK_CUDA(cudaMemcpyAsync(&e, word, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  HFK_CUDA(cudaStreamSynchronize(c->stream));
  if (e) {
    HFK_CUDA(cudaMemsetAsync(word, 0, sizeof(int), c->stream));
    throw Error{HFK_ERR_INTERNAL, "HyperFEMKernels: a block of the coarse triangular solve timed out"};
  }
}

// Cholesky factor of the assembled coarse level (in place of the reference's LU, the matrix being
// symmetric positive definite), hand-written over band storage (kern_chol.cuh): the lower triangle
// of the assembled CSC matrix copied into CB_T x CB_T tiles of its band, then one panel launch and
// one trailing-update launch per block column, O(n b^2) work and O(n b) memory for the lower
// bandwidth b (a full lower triangle when the band is wide). Then the D^-1 L tiles of the cycle's
// block triangular solves.
void coarse_factor_launch(hfk_pmg* m) {
  hfk_problem* c = m->lv[m->L - 1];
  if (!m->ev_c0)
    for (cudaEvent_t* e : {&m->ev_fork, &m->ev_c0, &m->ev_c1, &m->ev_p0, &m->ev_p1}) HFK_CUDA(cudaEventCreate(e));
  HFK_CUDA(cudaEventRecord(m->ev_c0, c->stream));
  pattern_build_dev(c);
  jacobian_dev(c, c->x.p, c->dvals.p, c->nzval.p);
  const int64_t n = c->nfree;
  if (n == 0) {  // nothing to factor: the coarse solve is empty
    m->cb_info.resize(1);
    m->cb_info.zero(c->stream);
    HFK_CUDA(cudaEventRecord(m->ev_p0, c->stream));
    HFK_CUDA(cudaEventRecord(m->ev_p1, c->stream));
    HFK_CUDA(cudaEventRecord(m->ev_c1, c->stream));
    m->cf_pending = true;
    return;
  }
  if (m->band < 0) {  // the pattern's lower bandwidth, once
    DBuf<int> bd;
    bd.resize(1);
    bd.zero(c->stream);
    lower_bandwidth_kernel<<<(int)std::min<int64_t>(n, 4096), 128, 0, c->stream>>>(n, c->colptr.p, c->rowval.p, bd.p);
    check_launch(c);
    HFK_CUDA(cudaMemcpyAsync(&m->band, bd.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    HFK_CUDA(cudaStreamSynchronize(c->stream));
  }
  const int nbt = (int)((n + CB_T - 1) / CB_T);
  const int W = std::min(nbt - 1, (m->band + CB_T - 1) / CB_T);
  m->Lb.resize((size_t)nbt * (W + 1) * CB_T * CB_T);
  m->Lb.zero(c->stream);
  band_fill_kernel<<<(int)std::min<int64_t>((int64_t)nbt * CB_T, 65535), 128, 0, c->stream>>>(
      n, nbt, W, c->colptr.p, c->rowval.p, c->nzval.p, m->Lb.p);
  check_launch(c);
  m->cb_nbt = nbt;
  m->cb_W = W;
  m->cb_info.resize(1);
  m->cb_info.zero(c->stream);
  const size_t smem_p = (size_t)4 * CB_T * CB_LD * sizeof(double), smem = (size_t)2 * CB_T * CB_LDU * sizeof(double);
  static PerDeviceLimit attr_p, attr_u;
  raise_smem_limit(band_panel_kernel, smem_p, attr_p);
  raise_smem_limit(band_update_kernel, smem, attr_u);
  HFK_CUDA(cudaEventRecord(m->ev_p0, c->stream));
  // Lookahead: panel k + 1 applies the update of block column k + 1 by block column k itself (the
  // only tiles it needs), and the rest of that trailing update (block columns k + 2 ..) runs on a
  // second stream, where it overlaps panel k + 1. Block column k is last written by the rest of
  // update k - 2, so panel k waits for that (two alternating events); the rest of update k waits
  // for panel k and follows the rest of update k - 1 on its stream.
  if (!m->cb_stream) HFK_CUDA(cudaStreamCreateWithFlags(&m->cb_stream, cudaStreamNonBlocking));
  while ((int)m->cb_ev.size() < 3) {
    cudaEvent_t e;
    HFK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    m->cb_ev.push_back(e);
  }
  cudaEvent_t ev_pan = m->cb_ev[0], ev_rest[2] = {m->cb_ev[1], m->cb_ev[2]};
  bool rest_rec[2] = {false, false};
  HFK_CUDA(cudaEventRecord(ev_pan, c->stream));  // the band storage is filled
  HFK_CUDA(cudaStreamWaitEvent(m->cb_stream, ev_pan, 0));
  for (int k = 0; k < nbt; ++k) {
    const int mq = std::min(W, nbt - 1 - k);
    if (rest_rec[k % 2]) HFK_CUDA(cudaStreamWaitEvent(c->stream, ev_rest[k % 2], 0));  // the rest of update k - 2
    band_panel_kernel<<<mq + 1, CB_PANEL_THREADS, smem_p, c->stream>>>(nbt, W, k, m->Lb.p, m->cb_info.p, 1);
    check_launch(c);
    rest_rec[k % 2] = false;
    if (mq > 1) {
      HFK_CUDA(cudaEventRecord(ev_pan, c->stream));
      HFK_CUDA(cudaStreamWaitEvent(m->cb_stream, ev_pan, 0));
      band_update_kernel<<<(mq - 1) * mq / 2, CB_THREADS, smem, m->cb_stream>>>(nbt, W, k, m->Lb.p, 2);
      check_launch(c);
      HFK_CUDA(cudaEventRecord(ev_rest[k % 2], m->cb_stream));
      rest_rec[k % 2] = true;
    }
  }
  for (int i = 0; i < 2; ++i)
    if (rest_rec[i]) HFK_CUDA(cudaStreamWaitEvent(c->stream, ev_rest[i], 0));
  HFK_CUDA(cudaEventRecord(m->ev_p1, c->stream));
  // the block tiles of the cycle's triangular solves (used only if every pivot was positive)
  band_prepare(m, n);
  HFK_CUDA(cudaEventRecord(m->ev_c1, c->stream));
  m->cf_pending = true;
}

// waits for the coarse build (on the coarse level's stream, the side stream) and reads the pivots'
// status; Lb then holds the band of the Cholesky factor L (A = L L^T) and the cycle applies A^-1 by
// the two block triangular solves
void coarse_factor_finish(hfk_pmg* m) {
  if (!m->cf_pending) return;
  hfk_problem* c = m->lv[m->L - 1];
  m->cf_pending = false;
  int info = 0;
  HFK_CUDA(cudaMemcpyAsync(&info, m->cb_info.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  HFK_CUDA(cudaStreamSynchronize(c->stream));
  float ms = 0;
  HFK_CUDA(cudaEventElapsedTime(&ms, m->ev_p0, m->ev_p1));
  m->t_potrf += ms;
  HFK_CUDA(cudaEventElapsedTime(&ms, m->ev_c0, m->ev_c1));
  m->t_coarse += ms;
  m->coarse_ok = info == 0;
  m->bs_on = m->coarse_ok;
  if (m->coarse_ok) m->nbuild++;
}

// The coarse level's build on the side stream: forked from the level-0 stream once the coarse state
// is injected, joined (on the host) before the update returns. The guard also joins it when an
// exception leaves the update early, and gives the coarse level the shared stream back.
struct CoarseFork {
  hfk_pmg* m;
  bool active = false;
  explicit CoarseFork(hfk_pmg* mm) : m(mm) {}
  void fork() {
    hfk_problem* p0 = m->lv[0];
    if (!m->side) HFK_CUDA(cudaStreamCreateWithFlags(&m->side, cudaStreamNonBlocking));
    if (!m->ev_c0)
      for (cudaEvent_t* e : {&m->ev_fork, &m->ev_c0, &m->ev_c1, &m->ev_p0, &m->ev_p1}) HFK_CUDA(cudaEventCreate(e));
    HFK_CUDA(cudaEventRecord(m->ev_fork, p0->stream));
    HFK_CUDA(cudaStreamWaitEvent(m->side, m->ev_fork, 0));
    m->lv[m->L - 1]->stream = m->side;
    active = true;
  }
  void join() {
    if (!active) return;
    coarse_factor_finish(m);  // still on the side stream
    active = false;
    m->lv[m->L - 1]->stream = m->lv[0]->stream;
  }
  ~CoarseFork() {
    if (!active) return;
    cudaStreamSynchronize(m->side);
    m->cf_pending = false;
    m->lv[m->L - 1]->stream = m->lv[0]->stream;
  }
};

// the inexact coarse solve's set-up: the coarse level's blocks and work vectors
void coarse_cg_update(hfk_pmg* m) {
  hfk_problem* c = m->lv[m->L - 1];
  const int64_t n = c->nfree;
  int bok = 0;
  blocks_update_dev(c, &bok);
  ensure_seg_items(c);
  m->ccg_r.resize(n);
  m->ccg_z.resize(n);
  m->ccg_p.resize(n);
  m->ccg_q.resize(n);
  m->ccg_sc.resize((size_t)SEG_NS * c->nseg);
  m->ccg_sc.zero(c->stream);
  m->coarse_ok = bok != 0;
  if (m->coarse_ok) m->nbuild++;
}

// x = A^-1 b with the Cholesky factor: L y = b, L^T x = y, FP64, by the block triangular solves of
// kern_band.cuh (forward into bs_y, backward into x)
void coarse_solve(hfk_pmg* m, const double* b, double* x) {
  hfk_problem* c = m->lv[m->L - 1];
  const int64_t n = c->nfree;
  HFK_REQUIRE(m->bs_on, HFK_ERR_STATE, "the coarse factor is not available");
  if (n == 0) return;
  const int nb = m->bs_nb;
  int* sy = m->bs_sync.p;
  HFK_CUDA(cudaMemsetAsync(sy, 0, 2 * sizeof(int), c->stream));
  if (m->bs_skip) {  // test knob: step 0 of the forward solve is never taken, so step 1 waits in vain
    fill_int_kernel<<<1, 32, 0, c->stream>>>(1, sy, 1);
    check_launch(c);
    m->bs_skip = 0;
  }
  HFK_CUDA(cudaMemsetAsync(m->bs_y.p, 0xff, n * sizeof(double), c->stream));  // the sentinel
  HFK_CUDA(cudaMemsetAsync(x, 0xff, n * sizeof(double), c->stream));
  band_solve_kernel<<<nb, BS_THREADS, 0, c->stream>>>(n, nb, m->bs_wt, 0, m->bs_tiles.p, b, m->bs_y.p, sy, sy + 2,
                                                      m->bs_spin);
  check_launch(c);
  band_solve_kernel<<<nb, BS_THREADS, 0, c->stream>>>(n, nb, m->bs_wt, 1,
                                                      m->bs_tiles.p + (size_t)nb * (m->bs_wt + 1) * BS_T * BS_T,
                                                      m->bs_y.p, x, sy + 1, sy + 2, m->bs_spin);
  check_launch(c);
}

// x ~= A^-1 b on the coarse level by coarse_iters steps of block-Jacobi preconditioned CG per
// segment from x = 0, with every scalar on the device (capturable in the cycle's graph). The
// approximation varies with b, which the flexible outer CG tolerates. Used where a dense factor of
// the coarse level does not fit (many problems, or more coarse dofs than the dense solve takes).
void coarse_cg(hfk_pmg* m, const double* b, double* x) {
  hfk_problem* c = m->lv[m->L - 1];
  const int64_t n = c->nfree;
  const int ns = c->nseg;
  const int32_t* seg = seg_dof_map(c);
  const int sg = std::max(1, (ns + 255) / 256);
  double* sc = m->ccg_sc.p;
  double *r = m->ccg_r.p, *z = m->ccg_z.p, *pp = m->ccg_p.p, *q = m->ccg_q.p;
  cudaStream_t st = c->stream;
  HFK_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), st));
  HFK_CUDA(cudaMemcpyAsync(r, b, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  blocks_apply_dev<double>(c, r, z);
  HFK_CUDA(cudaMemcpyAsync(pp, z, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  seg_dots<double>(c, 1, sc + S_RZ, SEG_NS, r, z);
  for (int it = 0; it < m->coarse_iters; ++it) {
    mf_apply_dev(c, pp, q);
    seg_dots<double>(c, 1, sc + S_PQ, SEG_NS, pp, q);
    seg_ratio_kernel<<<sg, 256, 0, st>>>(ns, sc, S_RZ, S_PQ, S_ALPHA, 0);
    check_launch(c);
    seg_cg_update_kernel<<<vec_grid(n), 256, 0, st>>>(n, seg, sc, pp, q, x, r, nullptr);
    check_launch(c);
    if (it + 1 == m->coarse_iters) break;
    blocks_apply_dev<double>(c, r, z);
    seg_dots<double>(c, 1, sc + S_ZR, SEG_NS, z, r);
    seg_ratio_kernel<<<sg, 256, 0, st>>>(ns, sc, S_ZR, S_RZ, S_BETA, 1);
    check_launch(c);
    seg_xpby_kernel<<<vec_grid(n), 256, 0, st>>>(n, seg, sc, S_BETA, z, pp);
    check_launch(c);
  }
}

template <typename R>
LevelWork<R>& level_work(hfk_pmg* m, int l);
template <>
LevelWork<double>& level_work<double>(hfk_pmg* m, int l) {
  return *m->w64[l];
}
template <>
LevelWork<float>& level_work<float>(hfk_pmg* m, int l) {
  return *m->w32[l];
}

// vcycle! (src/pmultigrid.jl:316-329): rhs in level_work(l).b, solution into level_work(l).x
template <typename R>
void vcycle_dev(hfk_pmg* m, int l) {
  hfk_problem* p = m->lv[l];
  LevelWork<R>& w = level_work<R>(m, l);
  if (m->L == 1) {  // a one-level slot (hfk_slot_create, FP64): its solve is the whole application
    if constexpr (sizeof(R) == sizeof(double)) {
      if (m->coarse_mode == COARSE_BLOCKS) blocks_apply_dev<double>(p, w.b.p, w.x.p);
      else coarse_solve(m, w.b.p, w.x.p);
    }
    return;
  }
  // pre-smoothing from zero, with the residual for the restriction
  cheb_smooth_coef<R>(p, w.cheb, m->coef[l]->p, m->degree, w.b.p, w.x.p, true, w.r.p);
  if (l + 1 == m->L - 1) {
    hfk_problem* c = m->lv[l + 1];
    LevelWork<R>& wc = level_work<R>(m, l + 1);
    restrict_dev<R>(m->tr[l], w.r.p, wc.b.p);
    const double* bc;
    if (sizeof(R) == sizeof(double)) {
      bc = reinterpret_cast<const double*>(wc.b.p);
    } else {
      convert_kernel<R, double><<<vec_grid(c->nfree), 256, 0, p->stream>>>(c->nfree, wc.b.p, m->cb.p);
      check_launch(p);
      bc = m->cb.p;
    }
    if (m->coarse_mode == HFK_COARSE_CG) coarse_cg(m, bc, m->cx.p);
    else coarse_solve(m, bc, m->cx.p);
    convert_kernel<double, R><<<vec_grid(c->nfree), 256, 0, p->stream>>>(c->nfree, m->cx.p, wc.x.p);
    check_launch(p);
  } else {
    restrict_dev<R>(m->tr[l], w.r.p, level_work<R>(m, l + 1).b.p);
    vcycle_dev<R>(m, l + 1);
  }
  prolongate_dev<R>(m->tr[l], level_work<R>(m, l + 1).x.p, w.e.p);
  axpby_kernel<R><<<vec_grid(p->nfree), 256, 0, p->stream>>>(p->nfree, R(1), w.e.p, R(1), w.x.p);
  check_launch(p);
  // post-smoothing with the same polynomial (symmetric cycle)
  cheb_smooth_coef<R>(p, w.cheb, m->coef[l]->p, m->degree, w.b.p, w.x.p, false, nullptr);
}

void pmg_drop_graph(hfk_pmg* m) {
  if (m->graph_exec) cudaGraphExecDestroy(m->graph_exec);
  if (m->graph) cudaGraphDestroy(m->graph);
  m->graph_exec = nullptr;
  m->graph = nullptr;
  m->cycles_since_update = 0;
}

void pmg_collect_cycle_time(hfk_pmg* m) {
  if (!m->ev_pending) return;
  HFK_CUDA(cudaEventSynchronize(m->ev1));
  float ms = 0;
  HFK_CUDA(cudaEventElapsedTime(&ms, m->ev0, m->ev1));
  m->t_cycle += ms;
  m->ev_pending = false;
}

// one V-cycle from level_work(0).b into level_work(0).x, replayed from a CUDA graph once captured
void pmg_cycle_on_buffers(hfk_pmg* m) {
  hfk_problem* p0 = m->lv[0];
  cudaStream_t s = p0->stream;
  // inside a capture of the caller's (the device-driven batched solve) the cycle's kernels are
  // recorded into that graph directly
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  HFK_CUDA(cudaStreamIsCapturing(s, &cs));
  if (cs != cudaStreamCaptureStatusNone) {
    if (m->precision == HFK_FP32) vcycle_dev<float>(m, 0);
    else vcycle_dev<double>(m, 0);
    return;
  }
  // the legacy default stream cannot be captured (a caller that launches its own work there, such
  // as a partitioned solve ordering the engine with torch, gets the cycle uncaptured)
  if (!m->graph_exec && m->cycles_since_update >= 1 && s != cudaStreamLegacy) {
    // every buffer exists (the first cycle after the update ran uncaptured): capture the cycle
    HFK_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
      if (m->precision == HFK_FP32) vcycle_dev<float>(m, 0);
      else vcycle_dev<double>(m, 0);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(s, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    HFK_CUDA(cudaStreamEndCapture(s, &m->graph));
    HFK_CUDA(cudaGraphInstantiate(&m->graph_exec, m->graph, 0));
  }
  if (m->graph_exec) {
    HFK_CUDA(cudaGraphLaunch(m->graph_exec, s));
  } else if (m->precision == HFK_FP32) {
    vcycle_dev<float>(m, 0);
  } else {
    vcycle_dev<double>(m, 0);
  }
  m->cycles_since_update++;
}

// Features of the fine level for the residual r and the cycle output y: s = r - A y and, per
// segment at ml_scal + 8 seg, the scales [rms s, rms Binv s, rms r, rms y] and |s|^2 (slot 4).
// Returns the block count.
int mlp_prepare_features(hfk_pmg* m, const double* r, const double* y) {
  hfk_problem* p = m->lv[0];
  const int64_t n = p->nfree;
  const int nb = p->nblocks;
  const int ns = p->nseg;
  m->ml_s.resize(n);
  m->ml_t.resize(n);
  m->ml_q.resize(n);
  m->ml_scal.resize((size_t)8 * ns);
  m->ml_feats.resize((size_t)nb * MLP_IN);
  mf_apply_dev(p, y, m->ml_q.p);
  axpbyz_kernel<double><<<vec_grid(n), 256, 0, p->stream>>>(n, 1.0, r, -1.0, m->ml_q.p, m->ml_s.p);
  check_launch(p);
  blocks_apply_dev<double>(p, m->ml_s.p, m->ml_t.p);
  seg_dots<double>(p, 3, m->ml_scal.p, 8, m->ml_s.p, m->ml_s.p, m->ml_t.p, m->ml_t.p, r, r);
  seg_dots<double>(p, 2, m->ml_scal.p + 3, 8, y, y, m->ml_s.p, m->ml_s.p);
  ensure_seg_items(p);
  seg_rms_kernel<<<std::max(1, (ns + 255) / 256), 256, 0, p->stream>>>(ns, m->ml_scal.p, 8, 4, p->seg_off_d.p);
  check_launch(p);
  mlp_features_kernel<<<vec_grid(nb), 256, 0, p->stream>>>(nb, p->bdofs.p, seg_block_map(p), p->Binv.p, m->ml_s.p, r,
                                                            y, m->ml_scal.p, 8, m->ml_loglm.p, m->ml_feats.p);
  check_launch(p);
  return nb;
}

// y += omega delta, delta = MLP(features), with the per-segment step omega that minimises the energy
// error of y along delta (omega = 0, the plain cycle, where delta is not a descent direction)
void mlp_correct(hfk_pmg* m, const double* r, double* y) {
  hfk_problem* p = m->lv[0];
  const int64_t n = p->nfree;
  const int nb = mlp_prepare_features(m, r, y);
  m->ml_out.resize((size_t)nb * MLP_OUT);
  m->ml_delta.resize(n);
  static PerDeviceLimit attr;
  raise_smem_limit(mlp_forward_kernel, MLP_NPARAM * sizeof(float), attr);
  mlp_forward_kernel<<<vec_grid(nb, 128), 128, MLP_NPARAM * sizeof(float), p->stream>>>(nb, m->mlp->wb.p, m->ml_feats.p,
                                                                                       m->ml_out.p);
  check_launch(p);
  HFK_CUDA(cudaMemsetAsync(m->ml_delta.p, 0, n * sizeof(double), p->stream));
  mlp_scatter_kernel<<<vec_grid(nb), 256, 0, p->stream>>>(nb, p->bdofs.p, seg_block_map(p), m->ml_out.p, m->ml_scal.p,
                                                           8, m->ml_delta.p);
  check_launch(p);
  mf_apply_dev(p, m->ml_delta.p, m->ml_q.p);
  seg_dots<double>(p, 2, m->ml_scal.p + 5, 8, m->ml_delta.p, m->ml_s.p, m->ml_delta.p, m->ml_q.p);
  m->ml_accepted.resize(1);
  mlp_accept_kernel<<<vec_grid(n), 256, 0, p->stream>>>(n, seg_dof_map(p), m->ml_scal.p + 5, 8, m->ml_delta.p, y);
  check_launch(p);
  mlp_accept_count_kernel<<<1, 256, 0, p->stream>>>(p->nseg, m->ml_scal.p + 5, 8, m->ml_accepted.p);
  check_launch(p);
  m->ml_tried += p->nseg;
}

// ldiv!(y, PMultigridState, r) on device vectors
void pmg_apply_dev(hfk_pmg* m, const double* r, double* y) {
  hfk_problem* p0 = m->lv[0];
  const int64_t n = p0->nfree;
  if (!m->ok) {
    fill_kernel<double><<<vec_grid(n), 256, 0, p0->stream>>>(n, NAN, y);
    check_launch(p0);
    return;
  }
  // the cycle is timed with events, except while the stream is being captured (a graph body may
  // hold no event nodes)
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  HFK_CUDA(cudaStreamIsCapturing(p0->stream, &cs));
  const bool timed = cs == cudaStreamCaptureStatusNone;
  if (timed) {
    pmg_collect_cycle_time(m);
    if (!m->ev0) {
      HFK_CUDA(cudaEventCreate(&m->ev0));
      HFK_CUDA(cudaEventCreate(&m->ev1));
    }
    HFK_CUDA(cudaEventRecord(m->ev0, p0->stream));
  }
  if (m->precision == HFK_FP32) {
    LevelWork<float>& w = *m->w32[0];
    convert_kernel<double, float><<<vec_grid(n), 256, 0, p0->stream>>>(n, r, w.b.p);
    check_launch(p0);
    pmg_cycle_on_buffers(m);
    convert_kernel<float, double><<<vec_grid(n), 256, 0, p0->stream>>>(n, w.x.p, y);
    check_launch(p0);
  } else {
    LevelWork<double>& w = *m->w64[0];
    HFK_CUDA(cudaMemcpyAsync(w.b.p, r, n * sizeof(double), cudaMemcpyDeviceToDevice, p0->stream));
    pmg_cycle_on_buffers(m);
    HFK_CUDA(cudaMemcpyAsync(y, w.x.p, n * sizeof(double), cudaMemcpyDeviceToDevice, p0->stream));
  }
  if (m->mlp) mlp_correct(m, r, y);
  if (timed) {
    HFK_CUDA(cudaEventRecord(m->ev1, p0->stream));
    m->ev_pending = true;
  }
  m->ncycles++;
}

}  // namespace

// =================================================================================================
// ABI
// =================================================================================================
extern "C" {

const char* hfk_last_error(void) { return g_last_error.c_str(); }
int hfk_version(void) { return 100; }

int hfk_problem_create(hfk_problem** out, int nn, int np, int ng, int ncells, const double* xq, const double* w,
                       const double* Nt, const double* dNt, const double* dMt, const double* coords,
                       const int32_t* cell_dof_ids, int64_t nfree, int64_t ndir, int law, const double* params,
                       int nparams) {
  HFK_API_BEGIN
  HFK_REQUIRE(out, HFK_ERR_ARG, "null output handle");
  *out = nullptr;
  HFK_REQUIRE(nn > 0 && np > 0 && ncells > 0 && ng == 8, HFK_ERR_ARG, "invalid sizes (nn, np, ncells > 0; ng == 8)");
  HFK_REQUIRE(xq && w && Nt && dNt && dMt && coords && cell_dof_ids, HFK_ERR_ARG, "null input array");
  HFK_REQUIRE(law == HFK_LAW_SVK || law == HFK_LAW_LINEAR_ELASTIC, HFK_ERR_ARG, "unknown law");
  HFK_REQUIRE(nparams >= 2 && nparams <= 5 && params, HFK_ERR_ARG, "law parameters: lambda, mu[, body force x y z]");
  HFK_REQUIRE(nfree >= 0 && ndir >= 0 && nfree < (1ll << 31), HFK_ERR_ARG, "invalid dof counts");
  auto p = std::make_unique<hfk_problem>();
  p->nn = nn;
  p->np = np;
  p->ng = ng;
  p->ncells = ncells;
  p->ndl = 3 * nn;
  p->nfree = nfree;
  p->ndir = ndir;
  p->law = law;
  for (int i = 0; i < nparams; ++i) p->params[i] = params[i];
  HFK_CUDA(cudaGetDevice(&p->device));
  // a blocking stream: ordered with the legacy default stream, on which callers (torch) write inputs
  HFK_CUDA(cudaStreamCreate(&p->own_stream));
  p->stream = p->own_stream;
  // validate ids
  const size_t nids = (size_t)p->ndl * ncells;
  for (size_t k = 0; k < nids; ++k) {
    const int32_t id = cell_dof_ids[k];
    HFK_REQUIRE(id <= nfree && -(int64_t)id <= ndir, HFK_ERR_ARG, "cell dof id out of range");
  }
  p->h_ids.assign(cell_dof_ids, cell_dof_ids + nids);
  {
    std::vector<char> seen(nfree + 1, 0);
    for (size_t k = 0; k < nids; ++k)
      if (cell_dof_ids[k] > 0) seen[cell_dof_ids[k]] = 1;
    for (int64_t i = 1; i <= nfree; ++i) HFK_REQUIRE(seen[i], HFK_ERR_ARG, "a free dof belongs to no cell");
  }
  if (!detect_tp(p.get(), xq, Nt)) {
    p->Q = p->P = 0;
    p->nodeperm.resize(nn);
    p->pointperm.resize(np);
    for (int i = 0; i < nn; ++i) p->nodeperm[i] = i;
    for (int i = 0; i < np; ++i) p->pointperm[i] = i;
  }
  // tensor-order copies of the tables and ids
  std::vector<int32_t> ids_t(nids);
  for (int cell = 0; cell < ncells; ++cell)
    for (int c = 0; c < 3; ++c)
      for (int lin = 0; lin < nn; ++lin)
        ids_t[(size_t)cell * p->ndl + c * nn + lin] = cell_dof_ids[(size_t)cell * p->ndl + c * nn + p->nodeperm[lin]];
  std::vector<double> w_t(np), dMt_t((size_t)ng * 3 * np), Nt_t((size_t)nn * np), dNt_t((size_t)nn * 3 * np);
  for (int pl = 0; pl < np; ++pl) {
    const int q = p->pointperm[pl];
    w_t[pl] = w[q];
    for (int n = 0; n < ng; ++n)
      for (int K = 0; K < 3; ++K) dMt_t[n + ng * (K + 3 * pl)] = dMt[n + ng * (K + 3 * q)];
    for (int lin = 0; lin < nn; ++lin) {
      const int n = p->nodeperm[lin];
      Nt_t[lin + (size_t)nn * pl] = Nt[n + (size_t)nn * q];
      for (int K = 0; K < 3; ++K) dNt_t[lin + (size_t)nn * (K + 3 * pl)] = dNt[n + (size_t)nn * (K + 3 * q)];
    }
  }
  p->h_w = w_t;
  p->ids.upload(ids_t.data(), nids, p->stream);
  p->w.upload(w_t.data(), np, p->stream);
  p->dMt.upload(dMt_t.data(), dMt_t.size(), p->stream);
  p->Nt.upload(Nt_t.data(), Nt_t.size(), p->stream);
  p->dNt.upload(dNt_t.data(), dNt_t.size(), p->stream);
  p->coords.upload(coords, (size_t)3 * ng * ncells, p->stream);
  cell_geometry(p.get(), coords, dMt);
  color_cells(p.get());
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  *out = p.release();
  HFK_API_END
}

int hfk_problem_destroy(hfk_problem* p) {
  HFK_API_BEGIN
  if (!p) return HFK_OK;
  // only the handle's own stream is touched: `stream` may be a caller's or a hierarchy's stream, and
  // freeing device memory waits for the device anyway
  if (p->own_stream) {
    cudaStreamSynchronize(p->own_stream);
    cudaStreamDestroy(p->own_stream);
  }
  for (cudaStream_t s : p->many_s)
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  for (cudaEvent_t e : p->many_ev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : p->kev) cudaEventDestroy(e);
  if (p->jc_copy) {
    cudaStreamSynchronize(p->jc_copy);
    cudaStreamDestroy(p->jc_copy);
  }
  for (cudaEvent_t e : p->jc_ev) cudaEventDestroy(e);
  delete p;
  cudaGetLastError();  // a release reports nothing: leave no error behind for the next checked call
  HFK_API_END
}

int hfk_problem_set_params(hfk_problem* p, const double* params, int nparams) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && params && nparams >= 2 && nparams <= 5, HFK_ERR_ARG, "law parameters: lambda, mu[, body force x y z]");
  for (int i = 0; i < 5; ++i) p->params[i] = i < nparams ? params[i] : 0.0;
  HFK_API_END
}

int hfk_problem_set_stream(hfk_problem* p, void* stream) {
  HFK_API_BEGIN
  HFK_REQUIRE(p, HFK_ERR_ARG, "null handle");
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  p->stream = stream ? (cudaStream_t)stream : p->own_stream;
  HFK_API_END
}

int hfk_functional(hfk_problem* p, const double* x, const double* dvals, int kind, double* out) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && x && out && (dvals || p->ndir == 0), HFK_ERR_ARG, "null argument");
  HFK_REQUIRE(kind == HFK_FUNCTIONAL_ENERGY || kind == HFK_FUNCTIONAL_MIN_DETF, HFK_ERR_ARG,
              "functional kind must be HFK_FUNCTIONAL_ENERGY or HFK_FUNCTIONAL_MIN_DETF");
  const double* dx = dev_in(x, p->nfree, p->stage_in, p->stream);
  const double* dd = dvals ? dev_in(dvals, p->ndir, p->stage_in2, p->stream) : nullptr;
  DBuf<double> o;
  o.resize(2);
  functional_dev(p, dx, dd, o.p);
  double h[2];
  HFK_CUDA(cudaMemcpyAsync(h, o.p, sizeof h, cudaMemcpyDeviceToHost, p->stream));
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  *out = kind == HFK_FUNCTIONAL_ENERGY ? h[0] : h[1];
  HFK_API_END
}

int hfk_problem_tuning(hfk_problem* p, int mode, int precision, int* atomic, int* kernel, int* warps) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && atomic && kernel && warps && (precision == HFK_FP64 || precision == HFK_FP32), HFK_ERR_ARG,
              "invalid argument");
  const int internal = mode == 0 ? MODE_JV : (mode == 1 ? MODE_RESIDUAL : MODE_JV_STORED);
  auto it = p->tuned.find(internal * 2 + (precision == HFK_FP32 ? 1 : 0));
  *atomic = it == p->tuned.end() ? -1 : (int)it->second.first;
  const int shape = it == p->tuned.end() ? 0 : it->second.second;
  *kernel = shape == SHAPE_Q1 ? 3 : (shape == SHAPE_TC ? 2 : (shape >= SHAPE_PT_NARROW ? 1 : 0));
  *warps = shape == SHAPE_Q1 ? Q1_THREADS / 32
         : shape == SHAPE_TC ? JV_TC_WARPS
                             : (shape == SHAPE_PT_NARROW ? (p->P * p->P * p->P + 31) / 32
                                                         : (shape == SHAPE_PT_WIDE ? JVP_WIDE / 32 : shape));
  HFK_API_END
}

int hfk_problem_set_launch(hfk_problem* p, int kernel, int warps) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && kernel >= 0 && kernel <= 3, HFK_ERR_ARG,
              "kernel must be 0 (line-mapped), 1 (point-parallel), 2 (tensor cores) or 3 (Q1 warp-synchronous)");
  HFK_REQUIRE(kernel != 0 || warps == 2 || warps == 4, HFK_ERR_ARG, "the line-mapped kernels take 2 or 4 warps per CTA");
  HFK_REQUIRE(kernel != 1 || warps == 0 || warps == JVP_WIDE / 32, HFK_ERR_ARG,
              "the point-parallel product takes 0 (one cell per CTA) or 8 warps per CTA");
  HFK_REQUIRE(kernel != 2 || (p->Q == 3 && p->P == 3), HFK_ERR_UNSUPPORTED,
              "the tensor-core product serves Q2 cells with 3^3 Gauss points");
  HFK_REQUIRE(kernel != 3 || (p->Q == 2 && p->P == 2), HFK_ERR_UNSUPPORTED,
              "the warp-synchronous Q1 product serves Q1 cells with 2^3 Gauss points");
  p->shape = kernel == 0 ? warps
                         : (kernel == 2 ? SHAPE_TC
                                        : (kernel == 3 ? SHAPE_Q1 : (warps == 0 ? SHAPE_PT_NARROW : SHAPE_PT_WIDE)));
  HFK_API_END
}

int hfk_problem_set_solve_graph(hfk_problem* p, int on) {
  HFK_API_BEGIN
  HFK_REQUIRE(p, HFK_ERR_ARG, "null handle");
  p->solve_graph = on != 0;
  HFK_API_END
}

int hfk_problem_set_assembly_kernel(hfk_problem* p, int kernel) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && (kernel == 0 || kernel == 1), HFK_ERR_ARG,
              "kernel must be 0 (the default choice) or 1 (the FP64 tensor-core kernel)");
  p->asm_kernel = kernel;
  HFK_API_END
}

int hfk_problem_set_scatter(hfk_problem* p, int mode) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && (mode == HFK_SCATTER_AUTO || mode == HFK_SCATTER_COLOURED || mode == HFK_SCATTER_ATOMIC),
              HFK_ERR_ARG, "scatter mode must be HFK_SCATTER_AUTO, _COLOURED or _ATOMIC");
  p->scatter = mode;
  HFK_API_END
}

int hfk_problem_info(hfk_problem* p, int64_t* nfree, int* Q, int* P, int* ncolors, int64_t* nnz) {
  HFK_API_BEGIN
  HFK_REQUIRE(p, HFK_ERR_ARG, "null handle");
  if (nfree) *nfree = p->nfree;
  if (Q) *Q = p->Q;
  if (P) *P = p->P;
  if (ncolors) *ncolors = p->ncolors;
  if (nnz) *nnz = p->nnz;
  HFK_API_END
}

int hfk_launch_count(hfk_problem* p, int64_t* count) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && count, HFK_ERR_ARG, "null argument");
  *count = p->launches;
  HFK_API_END
}

int hfk_problem_device_errors(hfk_problem* p, int* errors) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && errors, HFK_ERR_ARG, "null argument");
  *errors = 0;
  if (p->tc_err.p) {
    HFK_CUDA(cudaMemcpyAsync(errors, p->tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    HFK_CUDA(cudaStreamSynchronize(p->stream));
    HFK_CUDA(cudaMemsetAsync(p->tc_err.p, 0, sizeof(int), p->stream));
  }
  HFK_API_END
}

int hfk_problem_set_timing(hfk_problem* p, int on) {
  HFK_API_BEGIN
  HFK_REQUIRE(p, HFK_ERR_ARG, "null argument");
  p->ktiming = on != 0;
  p->kev_used = 0;
  HFK_API_END
}

int hfk_problem_kernel_time(hfk_problem* p, double* ms, int64_t* count) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && ms && count, HFK_ERR_ARG, "null argument");
  double total = 0;
  if (p->kev_used) HFK_CUDA(cudaEventSynchronize(p->kev[p->kev_used - 1]));
  for (size_t i = 0; i + 1 < p->kev_used; i += 2) {
    float t = 0;
    HFK_CUDA(cudaEventElapsedTime(&t, p->kev[i], p->kev[i + 1]));
    total += t;
  }
  *ms = total;
  *count = (int64_t)(p->kev_used / 2);
  p->kev_used = 0;
  HFK_API_END
}

int hfk_colors(hfk_problem* p, int32_t* color_of_cell) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && color_of_cell, HFK_ERR_ARG, "null argument");
  std::memcpy(color_of_cell, p->h_color_of.data(), sizeof(int32_t) * p->ncells);
  HFK_API_END
}

int hfk_pattern_build(hfk_problem* p, int64_t* nnz) {
  HFK_API_BEGIN
  HFK_REQUIRE(p, HFK_ERR_ARG, "null handle");
  pattern_build_dev(p);
  if (nnz) *nnz = p->nnz;
  HFK_API_END
}

int hfk_pattern_get(hfk_problem* p, int64_t* colptr, int64_t* rowval) {
  HFK_API_BEGIN
  HFK_REQUIRE(p, HFK_ERR_ARG, "null handle");
  pattern_build_dev(p);
  if (colptr) {
    int64_t* d = dev_out(colptr, p->nfree + 1, p->stage_l);
    HFK_CUDA(cudaMemcpyAsync(d, p->colptr.p, (p->nfree + 1) * sizeof(int64_t), cudaMemcpyDeviceToDevice, p->stream));
    finish_out(colptr, d, p->nfree + 1, p->stream);
  }
  if (rowval) {
    int64_t* d = dev_out(rowval, p->nnz, p->stage_l);
    HFK_CUDA(cudaMemcpyAsync(d, p->rowval.p, p->nnz * sizeof(int64_t), cudaMemcpyDeviceToDevice, p->stream));
    finish_out(rowval, d, p->nnz, p->stream);
  }
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  HFK_API_END
}

int hfk_nonzero_positions(hfk_problem* p, int32_t* nzpos) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && nzpos, HFK_ERR_ARG, "null argument");
  pattern_build_dev(p);
  const size_t per = (size_t)p->ndl * p->ndl;
  std::vector<int32_t> h(per * p->ncells);
  HFK_CUDA(cudaMemcpyAsync(h.data(), p->nzpos.p, h.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, p->stream));
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  // tensor local order -> caller local order
  std::vector<int> loc(p->ndl);
  for (int c = 0; c < 3; ++c)
    for (int lin = 0; lin < p->nn; ++lin) loc[c * p->nn + lin] = c * p->nn + p->nodeperm[lin];
  for (int cell = 0; cell < p->ncells; ++cell)
    for (int jj = 0; jj < p->ndl; ++jj)
      for (int ii = 0; ii < p->ndl; ++ii)
        nzpos[(size_t)cell * per + loc[ii] + (size_t)p->ndl * loc[jj]] = h[(size_t)cell * per + ii + (size_t)p->ndl * jj];
  HFK_API_END
}

int hfk_residual(hfk_problem* p, const double* x, const double* dvals, double* b) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && x && b && (dvals || p->ndir == 0), HFK_ERR_ARG, "null argument");
  const double* dx = dev_in(x, p->nfree, p->stage_in, p->stream);
  const double* dd = dvals ? dev_in(dvals, p->ndir, p->stage_in2, p->stream) : nullptr;
  double* db = dev_out(b, p->nfree, p->stage_out);
  residual_dev(p, dx, dd, db);
  finish_out(b, db, p->nfree, p->stream);
  HFK_API_END
}

int hfk_jacobian(hfk_problem* p, const double* x, const double* dvals, double* nzval) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && x && nzval && (dvals || p->ndir == 0), HFK_ERR_ARG, "null argument");
  pattern_build_dev(p);
  const double* dx = dev_in(x, p->nfree, p->stage_in, p->stream);
  const double* dd = dvals ? dev_in(dvals, p->ndir, p->stage_in2, p->stream) : nullptr;
  double* dn = dev_out(nzval, p->nnz, p->stage_out);
  if (dn != nzval && use_atomic_scatter(p) && p->ncells > 0 && p->nnz > 0) {
    // host output: each chunk's finished prefix of the values travels to the host while the next
    // chunk is assembled (the copies on their own stream, ordered after the chunk by an event)
    jacobian_chunks(p);
    const int K = (int)p->jc_done.size();
    if (!p->jc_copy) HFK_CUDA(cudaStreamCreateWithFlags(&p->jc_copy, cudaStreamNonBlocking));
    while ((int)p->jc_ev.size() < K) {
      cudaEvent_t e;
      HFK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      p->jc_ev.push_back(e);
    }
    int64_t sent = 0;
    const std::function<void(int)> after = [&](int k) {
      HFK_CUDA(cudaEventRecord(p->jc_ev[k], p->stream));
      HFK_CUDA(cudaStreamWaitEvent(p->jc_copy, p->jc_ev[k], 0));
      const int64_t upto = p->jc_done[k];
      if (upto > sent) {
        HFK_CUDA(cudaMemcpyAsync(nzval + sent, dn + sent, (upto - sent) * sizeof(double), cudaMemcpyDeviceToHost,
                                 p->jc_copy));
        sent = upto;
      }
    };
    jacobian_dev(p, dx, dd, dn, &after);
    HFK_CUDA(cudaStreamSynchronize(p->jc_copy));
  } else {
    jacobian_dev(p, dx, dd, dn);
    finish_out(nzval, dn, p->nnz, p->stream);
  }
  HFK_API_END
}

int hfk_mf_prepare(hfk_problem* p, const double* x, const double* dvals, int mode) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && x && (dvals || p->ndir == 0), HFK_ERR_ARG, "null argument");
  HFK_REQUIRE(mode == HFK_MF_STORED || mode == HFK_MF_RECOMPUTE, HFK_ERR_ARG, "unknown matrix-free mode");
  require_tp(p);
  bind_state(p, x, dvals);
  p->mf_mode = mode;
  if (mode == HFK_MF_STORED) {
    const size_t npq = (size_t)p->np * p->ncells;
    p->T.resize(81 * npq);
    p->iJtq.resize(9 * npq);
    p->dVq.resize(npq);
    CellData cd = cell_data(p, nullptr, p->ncells);
    store_tangents_kernel<<<vec_grid((int64_t)npq), 256, 0, p->stream>>>(cd, p->x.p, p->dvals.p, p->dNt.p, p->nn,
                                                                          p->np, p->T.p, p->iJtq.p, p->dVq.p);
    check_launch(p);
    p->Fq.release();
    p->Fq32.release();
    p->Fq32_valid = false;
  } else {
    p->T.release();
    p->iJtq.release();
    p->dVq.release();
    prepare_F(p);
  }
  p->prepared = true;
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  HFK_API_END
}

int hfk_mf_apply(hfk_problem* p, const double* dx, double* y) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && dx && y, HFK_ERR_ARG, "null argument");
  const double* d = dev_in(dx, p->nfree, p->stage_in, p->stream);
  double* dy = dev_out(y, p->nfree, p->stage_out);
  mf_apply_dev(p, d, dy);
  finish_out(y, dy, p->nfree, p->stream);
  HFK_API_END
}

// A stream of products: H2D of vector i + 1 and D2H of vector i - 1 overlap the product of vector
// i (two staging slots per direction, a copy-in and a copy-out stream, the product on the problem's
// stream). Device pointers skip their copies. Returns when every output is written.
int hfk_mf_apply_many(hfk_problem* p, int count, const double* const* dx, double* const* y) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && count >= 0 && (count == 0 || (dx && y)), HFK_ERR_ARG, "null argument");
  for (int i = 0; i < count; ++i) HFK_REQUIRE(dx[i] && y[i], HFK_ERR_ARG, "null vector pointer");
  if (count == 0) return HFK_OK;
  const size_t n = p->nfree, bytes = n * sizeof(double);
  if (!p->many_s[0]) {
    for (cudaStream_t& s : p->many_s) HFK_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    for (cudaEvent_t& e : p->many_ev) HFK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  for (int b = 0; b < 2; ++b) {
    p->many_in[b].resize(std::max<size_t>(p->many_in[b].n, n));
    p->many_out[b].resize(std::max<size_t>(p->many_out[b].n, n));
  }
  cudaStream_t sin = p->many_s[0], sout = p->many_s[1], sc = p->stream;
  cudaEvent_t* ev = p->many_ev;  // 0 fork, 1+b copied in, 3+b product done, 5+b copied out
  // the copies start after the work the caller queued on the problem's stream
  HFK_CUDA(cudaEventRecord(ev[0], sc));
  HFK_CUDA(cudaStreamWaitEvent(sin, ev[0], 0));
  HFK_CUDA(cudaStreamWaitEvent(sout, ev[0], 0));
  for (int i = 0; i < count; ++i) {
    const int b = i & 1;
    const bool din = is_device_ptr(dx[i]), dout = is_device_ptr(y[i]);
    const double* d = dx[i];
    if (!din) {
      if (i >= 2) HFK_CUDA(cudaStreamWaitEvent(sin, ev[3 + b], 0));  // slot read by product i - 2
      HFK_CUDA(cudaMemcpyAsync(p->many_in[b].p, dx[i], bytes, cudaMemcpyHostToDevice, sin));
      HFK_CUDA(cudaEventRecord(ev[1 + b], sin));
      HFK_CUDA(cudaStreamWaitEvent(sc, ev[1 + b], 0));
      d = p->many_in[b].p;
    }
    double* o = y[i];
    if (!dout) {
      if (i >= 2) HFK_CUDA(cudaStreamWaitEvent(sc, ev[5 + b], 0));  // slot copied out by D2H i - 2
      o = p->many_out[b].p;
    }
    mf_apply_dev(p, d, o);
    HFK_CUDA(cudaEventRecord(ev[3 + b], sc));
    if (!dout) {
      HFK_CUDA(cudaStreamWaitEvent(sout, ev[3 + b], 0));
      HFK_CUDA(cudaMemcpyAsync(y[i], o, bytes, cudaMemcpyDeviceToHost, sout));
      HFK_CUDA(cudaEventRecord(ev[5 + b], sout));
    }
  }
  // later work on the problem's stream follows every copy; host outputs are complete on return
  HFK_CUDA(cudaEventRecord(ev[5], sout));
  HFK_CUDA(cudaStreamWaitEvent(sc, ev[5], 0));
  HFK_CUDA(cudaEventRecord(ev[1], sin));
  HFK_CUDA(cudaStreamWaitEvent(sc, ev[1], 0));
  HFK_CUDA(cudaStreamSynchronize(sc));
  HFK_API_END
}

int hfk_mf_apply_f32(hfk_problem* p, const float* dx, float* y) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && dx && y, HFK_ERR_ARG, "null argument");
  const float* d = dev_in(dx, p->nfree, p->tmp32a, p->stream);
  float* dy = dev_out(y, p->nfree, p->tmp32b);
  mf_apply_dev32(p, d, dy);
  finish_out(y, dy, p->nfree, p->stream);
  HFK_API_END
}

int hfk_blocks_update(hfk_problem* p, int* ok) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && ok, HFK_ERR_ARG, "null argument");
  blocks_update_dev(p, ok);
  HFK_API_END
}

int hfk_blocks_apply(hfk_problem* p, const double* r, double* y) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && r && y, HFK_ERR_ARG, "null argument");
  const double* d = dev_in(r, p->nfree, p->stage_in, p->stream);
  double* dy = dev_out(y, p->nfree, p->stage_out);
  if (dy != y) HFK_CUDA(cudaMemsetAsync(dy, 0, p->nfree * sizeof(double), p->stream));
  blocks_apply_dev<double>(p, d, dy);
  finish_out(y, dy, p->nfree, p->stream);
  HFK_API_END
}

int hfk_blocks_set(hfk_problem* p, const double* B, int* ok) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && B && ok, HFK_ERR_ARG, "null argument");
  HFK_REQUIRE(p->nblocks > 0, HFK_ERR_STATE, "blocks not numbered (call hfk_blocks_update first)");
  const size_t n = 9 * (size_t)p->nblocks;
  if (is_device_ptr(B))
    HFK_CUDA(cudaMemcpyAsync(p->B.p, B, n * sizeof(double), cudaMemcpyDeviceToDevice, p->stream));
  else
    HFK_CUDA(cudaMemcpyAsync(p->B.p, B, n * sizeof(double), cudaMemcpyHostToDevice, p->stream));
  invert_blocks_and_check(p, ok);
  HFK_API_END
}

int hfk_blocks_get(hfk_problem* p, int* nblocks, int32_t* dofs, double* B, double* Binv) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && nblocks, HFK_ERR_ARG, "null argument");
  *nblocks = p->nblocks;
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  if (dofs && p->nblocks)
    HFK_CUDA(cudaMemcpy(dofs, p->bdofs.p, sizeof(int32_t) * 3 * p->nblocks, cudaMemcpyDeviceToHost));
  if (B && p->nblocks) HFK_CUDA(cudaMemcpy(B, p->B.p, sizeof(double) * 9 * p->nblocks, cudaMemcpyDeviceToHost));
  if (Binv && p->nblocks) HFK_CUDA(cudaMemcpy(Binv, p->Binv.p, sizeof(double) * 9 * p->nblocks, cudaMemcpyDeviceToHost));
  HFK_API_END
}

int hfk_hessenberg_eigvals(int n, const double* H, double* re, double* im) {
  HFK_API_BEGIN
  HFK_REQUIRE(n > 0 && H && re && im, HFK_ERR_ARG, "null argument");
  std::vector<double> h(H, H + (size_t)n * n);
  HFK_REQUIRE(hessenberg_eigvals(n, h, re, im), HFK_ERR_NUMERIC, "QR iteration did not converge");
  HFK_API_END
}

int hfk_eigenvalue_bounds(hfk_problem* p, int k, const double* start, double* lmin, double* lmax) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && lmin && lmax && k >= 1, HFK_ERR_ARG, "invalid argument");
  HFK_REQUIRE(p->nblocks > 0 || p->blocks_ok, HFK_ERR_STATE, "blocks not built (call hfk_blocks_update)");
  std::vector<double> v;
  if (!start) {
    chebyshev_start_vector(p, v);
    start = v.data();
  }
  const double* d = dev_in(start, p->nfree, p->stage_in2, p->stream);
  EigWork ew;
  std::vector<double> lo, hi;
  eig_bounds_dev(p, ew, k, d, lo, hi);
  // a problem with several segments reports the extreme bounds over its segments
  *lmin = *std::min_element(lo.begin(), lo.end());
  *lmax = *std::max_element(hi.begin(), hi.end());
  for (size_t s = 0; s < lo.size(); ++s)
    if (!std::isfinite(lo[s]) || !std::isfinite(hi[s])) *lmin = *lmax = NAN;
  HFK_API_END
}

int hfk_chebyshev_smooth(hfk_problem* p, double a, double b, int degree, const double* rhs, double* x, int zero_guess,
                         double* residual) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && rhs && x && degree >= 1 && b > a, HFK_ERR_ARG, "invalid argument");
  const int64_t n = p->nfree;
  const double* drhs = dev_in(rhs, n, p->stage_in, p->stream);
  DBuf<double> xs, rs;
  double* dxp = x;
  if (!is_device_ptr(x)) {
    xs.resize(n);
    HFK_CUDA(cudaMemcpyAsync(xs.p, x, n * sizeof(double), cudaMemcpyHostToDevice, p->stream));
    dxp = xs.p;
  }
  double* dres = nullptr;
  if (residual) dres = dev_out(residual, n, p->stage_out);
  ChebWork<double> w;
  cheb_smooth_dev<double>(p, w, a, b, degree, drhs, dxp, zero_guess != 0, dres);
  finish_out(x, dxp, n, p->stream);
  if (residual) finish_out(residual, dres, n, p->stream);
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  HFK_API_END
}

int hfk_transfer_create(hfk_transfer** out, hfk_problem* fine, hfk_problem* coarse, const double* E, const double* Einj) {
  HFK_API_BEGIN
  HFK_REQUIRE(out && fine && coarse && E && Einj, HFK_ERR_ARG, "null argument");
  HFK_REQUIRE(fine->ncells == coarse->ncells, HFK_ERR_ARG, "the two levels live on different meshes");
  HFK_REQUIRE(fine->nn >= coarse->nn, HFK_ERR_ARG, "the coarse space has more nodes per cell than the fine one");
  auto t = std::make_unique<hfk_transfer>();
  t->fine = fine;
  t->coarse = coarse;
  t->NF = fine->nn;
  t->NC = coarse->nn;
  // tensor orders of both levels
  std::vector<double> Et((size_t)t->NF * t->NC), Eit((size_t)t->NF * t->NC);
  for (int f = 0; f < t->NF; ++f)
    for (int c = 0; c < t->NC; ++c) {
      const int fo = fine->nodeperm[f], co = coarse->nodeperm[c];
      Et[f + (size_t)t->NF * c] = E[fo + (size_t)t->NF * co];
      Eit[c + (size_t)t->NC * f] = Einj[co + (size_t)t->NC * fo];
    }
  // Dirichlet consistency (src/transfers.jl:98-120): a fine Dirichlet dof gets no weight from a free
  // coarse dof; a coarse Dirichlet dof interpolates only from fine Dirichlet dofs
  for (int cell = 0; cell < fine->ncells; ++cell)
    for (int comp = 0; comp < 3; ++comp) {
      for (int f = 0; f < t->NF; ++f) {
        if (fine->h_ids[(size_t)cell * fine->ndl + comp * t->NF + f] > 0) continue;
        for (int c = 0; c < t->NC; ++c)
          HFK_REQUIRE(!(E[f + (size_t)t->NF * c] != 0 && coarse->h_ids[(size_t)cell * coarse->ndl + comp * t->NC + c] > 0),
                      HFK_ERR_ARG,
                      "the two levels have different Dirichlet boundaries (a fine Dirichlet dof is interpolated from a "
                      "free coarse dof; use the same closed Dirichlet set on every level)");
      }
      for (int c = 0; c < t->NC; ++c) {
        if (coarse->h_ids[(size_t)cell * coarse->ndl + comp * t->NC + c] > 0) continue;
        for (int f = 0; f < t->NF; ++f)
          HFK_REQUIRE(!(Einj[c + (size_t)t->NC * f] != 0 && fine->h_ids[(size_t)cell * fine->ndl + comp * t->NF + f] > 0),
                      HFK_ERR_ARG,
                      "the two levels have different Dirichlet boundaries (a coarse Dirichlet dof is interpolated from "
                      "a free fine dof)");
      }
    }
  std::vector<int32_t> mult(std::max<int64_t>(fine->nfree, 1), 0);
  for (size_t k = 0; k < fine->h_ids.size(); ++k)
    if (fine->h_ids[k] > 0) mult[fine->h_ids[k] - 1] += 1;
  t->E.upload(Et.data(), Et.size(), fine->stream);
  t->Einj.upload(Eit.data(), Eit.size(), fine->stream);
  t->mult.upload(mult.data(), mult.size(), fine->stream);
  // a tensor-product pair: E1 from the first row of nodes, then every entry of E checked against
  // E1 x E1 x E1 (E1[0][0] = cbrt E[0][0])
  {
    const int nf = (int)std::lround(std::cbrt((double)t->NF)), nc = (int)std::lround(std::cbrt((double)t->NC));
    bool tp = nf * nf * nf == t->NF && nc * nc * nc == t->NC && nf <= MAXQ && nc <= MAXQ && Et[0] > 0;
    if (tp) {
      const double c0 = std::cbrt(Et[0]);
      double emax = 0;
      for (double v : Et) emax = std::max(emax, std::fabs(v));
      XferTP d;
      d.nf = nf;
      d.nc = nc;
      for (int i = 0; i < nf; ++i)
        for (int b = 0; b < nc; ++b) d.e1[i * nc + b] = Et[i + (size_t)t->NF * b] / (c0 * c0);
      for (int f = 0; f < t->NF && tp; ++f)
        for (int c = 0; c < t->NC; ++c) {
          const int i1 = f % nf, i2 = (f / nf) % nf, i3 = f / (nf * nf);
          const int b1 = c % nc, b2 = (c / nc) % nc, b3 = c / (nc * nc);
          const double k = d.e1[i1 * nc + b1] * d.e1[i2 * nc + b2] * d.e1[i3 * nc + b3];
          if (std::fabs(k - Et[f + (size_t)t->NF * c]) > 1e-13 * emax) {
            tp = false;
            break;
          }
        }
      if (tp) {
        std::vector<double> im(mult.size());
        for (size_t q = 0; q < mult.size(); ++q) im[q] = mult[q] > 0 ? 1.0 / mult[q] : 0.0;
        t->invmult.upload(im.data(), im.size(), fine->stream);
        d.invmult = t->invmult.p;
        t->tpd = d;
        t->tp = true;
      }
    }
  }
  HFK_CUDA(cudaStreamSynchronize(fine->stream));
  *out = t.release();
  HFK_API_END
}

int hfk_transfer_set_multiplicity(hfk_transfer* t, const int32_t* mult) {
  HFK_API_BEGIN
  HFK_REQUIRE(t && mult, HFK_ERR_ARG, "null argument");
  const int64_t n = t->fine->nfree;
  std::vector<int32_t> m(mult, mult + n);
  std::vector<int32_t> own(std::max<int64_t>(n, 1), 0);
  for (size_t k = 0; k < t->fine->h_ids.size(); ++k)
    if (t->fine->h_ids[k] > 0) own[t->fine->h_ids[k] - 1] += 1;
  for (int64_t q = 0; q < n; ++q)
    HFK_REQUIRE(m[q] >= own[q] && (m[q] > 0) == (own[q] > 0), HFK_ERR_ARG,
                "a multiplicity is below the number of this level's cells that share the dof");
  if (n) t->mult.upload(m.data(), m.size(), t->fine->stream);
  if (t->tp) {
    std::vector<double> im(std::max<int64_t>(n, 1), 0.0);
    for (int64_t q = 0; q < n; ++q) im[q] = m[q] > 0 ? 1.0 / m[q] : 0.0;
    t->invmult.upload(im.data(), im.size(), t->fine->stream);
    t->tpd.invmult = t->invmult.p;
  }
  HFK_CUDA(cudaStreamSynchronize(t->fine->stream));
  HFK_API_END
}

int hfk_transfer_destroy(hfk_transfer* t) {
  HFK_API_BEGIN
  delete t;
  HFK_API_END
}

int hfk_prolongate(hfk_transfer* t, const double* xc, double* yf) {
  HFK_API_BEGIN
  HFK_REQUIRE(t && xc && yf, HFK_ERR_ARG, "null argument");
  hfk_problem* p = t->fine;
  const double* d = dev_in(xc, t->coarse->nfree, p->stage_in, p->stream);
  double* dy = dev_out(yf, p->nfree, p->stage_out);
  prolongate_dev<double>(t, d, dy);
  finish_out(yf, dy, p->nfree, p->stream);
  HFK_API_END
}

int hfk_restrict(hfk_transfer* t, const double* yf, double* yc) {
  HFK_API_BEGIN
  HFK_REQUIRE(t && yc && yf, HFK_ERR_ARG, "null argument");
  hfk_problem* p = t->fine;
  const double* d = dev_in(yf, p->nfree, p->stage_in, p->stream);
  double* dy = dev_out(yc, t->coarse->nfree, p->stage_out);
  restrict_dev<double>(t, d, dy);
  finish_out(yc, dy, t->coarse->nfree, p->stream);
  HFK_API_END
}

int hfk_inject(hfk_transfer* t, const double* xf, const double* df, double* xc, double* dc) {
  HFK_API_BEGIN
  HFK_REQUIRE(t && xf && xc && (df || t->fine->ndir == 0) && (dc || t->coarse->ndir == 0), HFK_ERR_ARG, "null argument");
  hfk_problem* p = t->fine;
  hfk_problem* c = t->coarse;
  const double* d1 = dev_in(xf, p->nfree, p->stage_in, p->stream);
  const double* d2 = df ? dev_in(df, p->ndir, p->stage_in2, p->stream) : nullptr;
  DBuf<double> oc, od;
  double* dxc = dev_out(xc, c->nfree, oc);
  double* ddc = dc ? dev_out(dc, c->ndir, od) : nullptr;
  inject_dev(t, d1, d2, dxc, ddc);
  finish_out(xc, dxc, c->nfree, p->stream);
  if (dc) finish_out(dc, ddc, c->ndir, p->stream);
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  HFK_API_END
}

}  // extern "C"
namespace {
hfk_pmg* pmg_create_impl(int nlevels, hfk_problem* const* levels, hfk_transfer* const* transfers, int degree,
                         double range, double inflate, int eig_iters, int coarse_every, int precision) {
  HFK_REQUIRE(levels && (transfers || nlevels == 1), HFK_ERR_ARG, "null argument");
  HFK_REQUIRE(degree >= 1, HFK_ERR_ARG, "Chebyshev: degree must be >= 1");
  HFK_REQUIRE(range > 1, HFK_ERR_ARG, "Chebyshev: range must be > 1");
  HFK_REQUIRE(inflate >= 1, HFK_ERR_ARG, "Chebyshev: inflate must be >= 1");
  HFK_REQUIRE(eig_iters >= 2, HFK_ERR_ARG, "Chebyshev: eig_iters must be >= 2");
  HFK_REQUIRE(coarse_every >= 1, HFK_ERR_ARG, "PMultigrid: coarse_every must be >= 1");
  HFK_REQUIRE(precision == HFK_FP64 || precision == HFK_FP32, HFK_ERR_ARG, "precision must be HFK_FP64 or HFK_FP32");
  auto m = std::make_unique<hfk_pmg>();
  m->L = nlevels;
  for (int l = 0; l < nlevels; ++l) {
    HFK_REQUIRE(levels[l], HFK_ERR_ARG, "null level");
    m->lv.push_back(levels[l]);
  }
  for (int l = 1; l < nlevels; ++l)
    HFK_REQUIRE(levels[l]->nseg == levels[0]->nseg && levels[l]->seg_cells == levels[0]->seg_cells, HFK_ERR_ARG,
                "the levels hold different segments (set the same segments on every level before the hierarchy)");
  for (int l = 0; l < nlevels - 1; ++l) {
    HFK_REQUIRE(transfers[l] && transfers[l]->fine == levels[l] && transfers[l]->coarse == levels[l + 1], HFK_ERR_ARG,
                "transfers[l] must go from level l+1 to level l");
    m->tr.push_back(transfers[l]);
    require_tp(levels[l]);
  }
  // one stream for the whole hierarchy: the V-cycle moves data between levels; with batched
  // problems the levels also read the working level's segment flags
  for (int l = 1; l < nlevels; ++l) {
    HFK_CUDA(cudaStreamSynchronize(levels[l]->stream));
    levels[l]->stream = levels[0]->stream;
    if (levels[l]->seg_active && levels[0]->seg_active) levels[l]->seg_active = levels[0]->seg_active;
  }
  m->degree = degree;
  m->range = range;
  m->inflate = inflate;
  m->eig_iters = eig_iters;
  m->coarse_every = coarse_every;
  m->precision = precision;
  m->a.assign(nlevels, 0);
  m->b.assign(nlevels, 0);
  m->lmin.assign(nlevels, 0);
  m->seg_lmin.assign(nlevels, {});
  m->seg_lmax.assign(nlevels, {});
  m->lmax.assign(nlevels, 0);
  m->lok.assign(nlevels, 0);
  for (int l = 0; l < nlevels; ++l) {
    const int64_t n = levels[l]->nfree;
    if (precision == HFK_FP32) {
      auto w = std::make_unique<LevelWork<float>>();
      w->b.resize(n);
      w->x.resize(n);
      w->r.resize(n);
      w->e.resize(n);
      m->w32.push_back(std::move(w));
    } else {
      auto w = std::make_unique<LevelWork<double>>();
      w->b.resize(n);
      w->x.resize(n);
      w->r.resize(n);
      w->e.resize(n);
      m->w64.push_back(std::move(w));
    }
  }
  for (int l = 0; l < nlevels; ++l) {
    m->coef.push_back(std::make_unique<DBuf<double>>());
    m->coef.back()->resize((1 + 2 * (size_t)degree) * levels[l]->nseg);
    m->ew.push_back(std::make_unique<EigWork>());
    m->start.push_back(std::make_unique<DBuf<double>>());
  }
  const int64_t nc = levels[nlevels - 1]->nfree;
  m->cb.resize(nc);
  m->cx.resize(nc);
  return m.release();
}
}  // namespace
extern "C" {

int hfk_pmg_create(hfk_pmg** out, int nlevels, hfk_problem* const* levels, hfk_transfer* const* transfers, int degree,
                   double range, double inflate, int eig_iters, int coarse_every, int precision) {
  HFK_API_BEGIN
  HFK_REQUIRE(out && levels && transfers, HFK_ERR_ARG, "null argument");
  HFK_REQUIRE(nlevels >= 2, HFK_ERR_ARG, "PMultigrid needs at least two levels");
  *out = pmg_create_impl(nlevels, levels, transfers, degree, range, inflate, eig_iters, coarse_every, precision);
  HFK_API_END
}

int hfk_slot_create(hfk_pmg** out, hfk_problem* op, int kind, int every) {
  HFK_API_BEGIN
  HFK_REQUIRE(out && op, HFK_ERR_ARG, "null argument");
  HFK_REQUIRE(kind == HFK_SLOT_LAGGED_ASSEMBLED || kind == HFK_SLOT_BLOCK_JACOBI, HFK_ERR_ARG,
              "slot kind must be HFK_SLOT_LAGGED_ASSEMBLED or HFK_SLOT_BLOCK_JACOBI");
  HFK_REQUIRE(every >= 1, HFK_ERR_ARG, "LaggedAssembled: every must be >= 1");
  hfk_problem* lv[1] = {op};
  hfk_pmg* m = pmg_create_impl(1, lv, nullptr, 1, 20.0, 1.1, 10, kind == HFK_SLOT_BLOCK_JACOBI ? 1 : every, HFK_FP64);
  m->coarse_mode = kind == HFK_SLOT_BLOCK_JACOBI ? COARSE_BLOCKS : HFK_COARSE_CHOLESKY;
  *out = m;
  HFK_API_END
}

int hfk_pmg_destroy(hfk_pmg* m) {
  HFK_API_BEGIN
  if (m) {
    cudaStreamSynchronize(m->lv[0]->stream);
    // the coarser levels go back to their own streams and flags (levels must outlive their hierarchy)
    for (int l = 1; l < m->L; ++l) {
      m->lv[l]->stream = m->lv[l]->own_stream;
      if (m->lv[l]->seg_active) m->lv[l]->seg_active = m->lv[l]->seg_active_own.p;
    }
    if (m->side) {
      cudaStreamSynchronize(m->side);
      cudaStreamDestroy(m->side);
    }
    if (m->cb_stream) {
      cudaStreamSynchronize(m->cb_stream);
      cudaStreamDestroy(m->cb_stream);
    }
    for (cudaEvent_t e : m->cb_ev) cudaEventDestroy(e);
    for (cudaEvent_t e : {m->ev_fork, m->ev_c0, m->ev_c1, m->ev_p0, m->ev_p1})
      if (e) cudaEventDestroy(e);
    pmg_drop_graph(m);
    if (m->ev0) cudaEventDestroy(m->ev0);
    if (m->ev1) cudaEventDestroy(m->ev1);
  }
  delete m;
  cudaGetLastError();  // a release reports nothing: leave no error behind for the next checked call
  HFK_API_END
}

int hfk_pmg_update(hfk_pmg* m, const double* x, const double* dvals, int* ok) {
  HFK_API_BEGIN
  HFK_REQUIRE(m && x && ok, HFK_ERR_ARG, "null argument");
  pmg_bind_stream(m);
  pmg_collect_cycle_time(m);
  {
    // the captured cycle bakes in the levels' law parameters: capture again if they changed
    std::vector<double> prm;
    for (auto* lv : m->lv) prm.insert(prm.end(), lv->params, lv->params + 5);
    if (prm != m->graph_params) {
      pmg_drop_graph(m);
      m->graph_params = prm;
    }
  }
  const auto t_start = std::chrono::steady_clock::now();
  auto ms_since = [](std::chrono::steady_clock::time_point t) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
  };
  hfk_problem* p0 = m->lv[0];
  const bool f32 = m->precision == HFK_FP32;
  // level 0 state: the Newton's tangent (prepared in the recompute formulation)
  bind_state(p0, x, dvals);
  prepare_F(p0);
  // inject level by level and prepare (update_levels!, src/pmultigrid.jl:197-204)
  for (int l = 0; l + 1 < m->L; ++l) {
    hfk_problem* f = m->lv[l];
    hfk_problem* c = m->lv[l + 1];
    c->x.resize(c->nfree);
    c->dvals.resize(std::max<int64_t>(c->ndir, 1));
    inject_dev(m->tr[l], f->x.p, f->dvals.p, c->x.p, c->dvals.p);
    if (l + 1 < m->L - 1 || m->coarse_mode == HFK_COARSE_CG) {
      prepare_F(c);
    } else {
      c->prepared = true;  // the coarse level is assembled
    }
  }
  (void)f32;
  // coarse level (every coarse_every updates): the assembled factorisation starts now on the side
  // stream and overlaps the smoothers' set-up below
  m->since++;
  const bool rebuild = !m->built || m->since >= m->coarse_every;
  CoarseFork cfork(m);
  if (rebuild && m->coarse_mode == HFK_COARSE_CHOLESKY) {
    if (m->L > 1) cfork.fork();  // a one-level slot has nothing to overlap with
    coarse_factor_launch(m);
  }
  // smoothers: blocks and intervals (smoother_update!, src/smoothers.jl:86-107)
  bool all_ok = true, indef = false;
  for (int l = 0; l + 1 < m->L; ++l) {
    hfk_problem* p = m->lv[l];
    int bok = 0;
    auto tb = std::chrono::steady_clock::now();
    blocks_update_dev(p, &bok);
    m->t_blocks += ms_since(tb);
    if (!bok) {
      m->lok[l] = 0;
      all_ok = false;
      continue;
    }
    if (m->start[l]->n != (size_t)p->nfree) {
      std::vector<double> v;
      chebyshev_start_vector(p, v);
      m->start[l]->upload(v.data(), v.size(), p->stream);
    }
    auto te = std::chrono::steady_clock::now();
    std::vector<double>&lo = m->seg_lmin[l], &hi = m->seg_lmax[l];
    eig_bounds_dev(p, *m->ew[l], m->eig_iters, m->start[l]->p, lo, hi, m->eig_inner == HFK_EIG_PRECONDITIONED);
    m->t_eig += ms_since(te);
    // per segment: interval [b / range, b] with b = inflate * lmax (smoother_update!,
    // src/smoothers.jl:86-107) and its coefficients at coef + s * (1 + 2 degree)
    const int ns = p->nseg;
    std::vector<double> coefs;
    coefs.reserve((size_t)ns * (1 + 2 * m->degree));
    bool lok = true;
    m->lmin[l] = INFINITY;
    m->lmax[l] = -INFINITY;
    for (int sgi = 0; sgi < ns; ++sgi) {
      const bool ok_s = std::isfinite(hi[sgi]) && hi[sgi] > 0 && lo[sgi] > 0;
      lok &= ok_s;
      indef |= std::isfinite(hi[sgi]) && std::isfinite(lo[sgi]) && (lo[sgi] <= 0 || hi[sgi] <= 0);
      const double bs = ok_s ? m->inflate * hi[sgi] : 1.0;
      const std::vector<double> c = chebyshev_coefficients(bs / m->range, bs, m->degree);
      coefs.insert(coefs.end(), c.begin(), c.end());
      m->lmin[l] = std::min(m->lmin[l], lo[sgi]);
      m->lmax[l] = std::max(m->lmax[l], hi[sgi]);
    }
    if (!lok) m->lmin[l] = m->lmax[l] = NAN;
    m->lok[l] = lok;
    all_ok &= lok;
    m->b[l] = m->inflate * m->lmax[l];
    m->a[l] = m->b[l] / m->range;
    if (m->coef[l]->n != coefs.size()) pmg_drop_graph(m);  // the captured cycle holds the buffer's address
    m->coef[l]->upload(coefs.data(), coefs.size(), p->stream);
    if (f32) ensure_F32(p);
  }
  {
    // the network's material features: log lambda, log mu per segment of the working level
    std::vector<float> lg((size_t)2 * p0->nseg);
    for (int sgi = 0; sgi < p0->nseg; ++sgi) {
      const double la = p0->seg_lm.empty() ? p0->params[0] : p0->seg_lm[2 * (size_t)sgi];
      const double mu = p0->seg_lm.empty() ? p0->params[1] : p0->seg_lm[2 * (size_t)sgi + 1];
      lg[2 * sgi] = (float)std::log(std::max(la, 1e-300));
      lg[2 * sgi + 1] = (float)std::log(std::max(mu, 1e-300));
    }
    m->ml_loglm.upload(lg.data(), lg.size(), p0->stream);
  }
  if (rebuild) {
    if (m->coarse_mode == HFK_COARSE_CG) {
      auto tc = std::chrono::steady_clock::now();
      coarse_cg_update(m);
      HFK_CUDA(cudaStreamSynchronize(p0->stream));
      m->t_coarse += ms_since(tc);
    } else if (m->coarse_mode == COARSE_BLOCKS) {
      int bok = 0;
      auto tb = std::chrono::steady_clock::now();
      blocks_update_dev(p0, &bok);
      m->t_blocks += ms_since(tb);
      m->coarse_ok = bok != 0;
      if (m->coarse_ok) m->nbuild++;
    } else if (m->L > 1) {
      cfork.join();
    } else {
      coarse_factor_finish(m);
    }
    m->since = 0;
  }
  all_ok &= m->coarse_ok;
  m->ok = all_ok;
  m->indefinite = !all_ok && indef;
  m->built = true;
  m->nupdate++;
  *ok = all_ok;
  m->t_update += ms_since(t_start);
  HFK_API_END
}

int hfk_pmg_vcycle(hfk_pmg* m, const double* r, double* y) {
  HFK_API_BEGIN
  HFK_REQUIRE(m && r && y, HFK_ERR_ARG, "null argument");
  HFK_REQUIRE(m->built, HFK_ERR_STATE, "PMultigrid: call hfk_pmg_update first");
  pmg_bind_stream(m);
  hfk_problem* p0 = m->lv[0];
  const double* dr = dev_in(r, p0->nfree, m->top_r, p0->stream);
  double* dy = dev_out(y, p0->nfree, m->top_y);
  pmg_apply_dev(m, dr, dy);
  finish_out(y, dy, p0->nfree, p0->stream);
  HFK_CUDA(cudaStreamSynchronize(p0->stream));
  band_check(m);
  HFK_API_END
}

int hfk_pmg_stats(hfk_pmg* m, double* out) {
  HFK_API_BEGIN
  HFK_REQUIRE(m && out, HFK_ERR_ARG, "null argument");
  pmg_collect_cycle_time(m);
  out[0] = (double)m->nupdate;
  out[1] = (double)m->nbuild;
  out[2] = (double)m->ncycles;
  out[3] = m->t_update;
  out[4] = m->t_coarse;
  out[5] = m->t_blocks;
  out[6] = m->t_eig;
  out[7] = m->t_cycle;
  out[8] = m->t_potrf;
  HFK_API_END
}

int hfk_pmg_status(hfk_pmg* m, int* ok, int* indefinite) {
  HFK_API_BEGIN
  HFK_REQUIRE(m && ok && indefinite, HFK_ERR_ARG, "null argument");
  *ok = m->ok;
  *indefinite = m->indefinite;
  HFK_API_END
}

int hfk_pmg_level_info(hfk_pmg* m, int level, double* lmin, double* lmax, double* a, double* b) {
  HFK_API_BEGIN
  HFK_REQUIRE(m && level >= 0 && level < m->L, HFK_ERR_ARG, "invalid level");
  if (lmin) *lmin = m->lmin[level];
  if (lmax) *lmax = m->lmax[level];
  if (a) *a = m->a[level];
  if (b) *b = m->b[level];
  HFK_API_END
}

}  // extern "C"

namespace {
// MatrixFreeSolver.solve! (src/solvers.jl:111-159): FP64 (flexible) CG, true-residual stopping test
void solve_cg_dev(hfk_problem* op, hfk_pmg* prec, const double* b, double* x, double rtol, double atol, int maxiter,
                  int flexible, int* iters, int* converged, int* indefinite, double* relres) {
  HFK_REQUIRE(op && b && x && iters && converged, HFK_ERR_ARG, "null argument");
  HFK_REQUIRE(rtol >= 0 && rtol < 1, HFK_ERR_ARG, "the relative tolerance must be in [0, 1)");
  HFK_REQUIRE(atol >= 0 && maxiter > 0, HFK_ERR_ARG, "atol must be >= 0 and maxiter > 0");
  HFK_REQUIRE(op->prepared, HFK_ERR_STATE, "the operator has not been prepared");
  const int64_t n = op->nfree;
  if (prec) {
    HFK_REQUIRE(prec->lv[0] == op, HFK_ERR_ARG, "the preconditioner's working level is not this operator");
    pmg_bind_stream(prec);
  }
  cudaStream_t s = op->stream;
  *iters = 0;
  *converged = 0;
  if (indefinite) *indefinite = 0;
  if (relres) *relres = NAN;
  if (prec && !prec->ok) {  // src/solvers.jl:114-121: no iteration, a failed solve (indefinite or not)
    if (is_device_ptr(x)) HFK_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), s));
    else std::fill(x, x + n, 0.0);
    HFK_CUDA(cudaStreamSynchronize(s));
    if (indefinite) *indefinite = prec->indefinite;
    return;
  }
  hfk::CGWork& cw = op->cg;
  DBuf<double>&db = cw.b, &dx = cw.x, &r = cw.r, &z = cw.z, &pp = cw.p, &q = cw.q, &rold = cw.rold;
  const double* bd = dev_in(b, n, db, s);
  double* xd = x;
  if (!is_device_ptr(x)) {
    dx.resize(n);
    HFK_CUDA(cudaMemcpyAsync(dx.p, x, n * sizeof(double), cudaMemcpyHostToDevice, s));
    xd = dx.p;
  }
  r.resize(n);
  z.resize(n);
  pp.resize(n);
  q.resize(n);
  if (flexible) rold.resize(n);
  Reducer& red = cw.red;
  double res[3];
  // r = b - A x
  mf_apply_dev(op, xd, q.p);
  axpbyz_kernel<double><<<vec_grid(n), 256, 0, s>>>(n, 1.0, bd, -1.0, q.p, r.p);
  check_launch(op);
  dots<double>(op, red, n, 2, bd, bd, r.p, r.p, nullptr, nullptr, res);
  const double nb = std::sqrt(res[0]);
  const double tol = atol + rtol * nb;
  double rn = std::sqrt(res[1]);
  int it = 0;
  bool conv = rn <= tol;
  bool indef = false;
  auto apply_prec = [&](const double* in, double* outp) {
    if (prec) pmg_apply_dev(prec, in, outp);
    else HFK_CUDA(cudaMemcpyAsync(outp, in, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  };
  if (!conv) {
    apply_prec(r.p, z.p);
    HFK_CUDA(cudaMemcpyAsync(pp.p, z.p, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    dots<double>(op, red, n, 1, r.p, z.p, nullptr, nullptr, nullptr, nullptr, res);
    double rz = res[0];
    while (it < maxiter) {
      ++it;
      mf_apply_dev(op, pp.p, q.p);
      dots<double>(op, red, n, 1, pp.p, q.p, nullptr, nullptr, nullptr, nullptr, res);
      const double pq = res[0];
      if (!(pq > 0)) {
        indef = true;
        break;
      }
      const double alpha = rz / pq;
      cg_update_kernel<<<vec_grid(n), 256, 0, s>>>(n, alpha, pp.p, q.p, xd, r.p, flexible ? rold.p : nullptr);
      check_launch(op);
      dots<double>(op, red, n, 1, r.p, r.p, nullptr, nullptr, nullptr, nullptr, res);
      rn = std::sqrt(res[0]);
      if (rn <= tol) {
        conv = true;
        break;
      }
      apply_prec(r.p, z.p);
      double beta;
      if (flexible) {
        dots<double>(op, red, n, 2, z.p, r.p, z.p, rold.p, nullptr, nullptr, res);
        beta = (res[0] - res[1]) / rz;
        rz = res[0];
      } else {
        dots<double>(op, red, n, 1, z.p, r.p, nullptr, nullptr, nullptr, nullptr, res);
        beta = res[0] / rz;
        rz = res[0];
      }
      axpby_kernel<double><<<vec_grid(n), 256, 0, s>>>(n, 1.0, z.p, beta, pp.p);
      check_launch(op);
    }
  }
  // true residual check (src/solvers.jl:150-157)
  mf_apply_dev(op, xd, q.p);
  axpbyz_kernel<double><<<vec_grid(n), 256, 0, s>>>(n, 1.0, bd, -1.0, q.p, r.p);
  check_launch(op);
  dots<double>(op, red, n, 1, r.p, r.p, nullptr, nullptr, nullptr, nullptr, res);
  const double tr = std::sqrt(res[0]);
  if (relres) *relres = nb > 0 ? tr / nb : tr;
  // the recursive residual decides; a solve stopped without it is judged on the true residual
  conv = !indef && (conv || tr <= tol);
  finish_out(x, xd, n, s);
  *iters = it;
  *converged = conv;
  if (indefinite) *indefinite = indef;
}
// MatrixFreeSolver.solve! with krylov = :gmres / :fgmres (src/solvers.jl:128-131): restarted GMRES
// with right preconditioning (A N^-1 u = b, x = N^-1 u; Krylov.jl's gmres!/fgmres! with restart),
// every vector on the device. Each iteration: z = N^-1 v_j, w = A z, classical Gram-Schmidt with
// one reorthogonalisation (two passes of cuBLAS gemv: h = V^T w, w -= V h), v_{j+1} = w / ||w||;
// the Hessenberg matrix and its Givens rotations live on the host. The cycle ends when the
// residual estimate |g_{j+1}| meets atol + rtol ||b||, at `restart` iterations or at maxiter; then
// x += Z y (FGMRES, flexible != 0: the preconditioned basis kept, any preconditioner) or
// x += N^-1 (V y) (GMRES: one more preconditioner application, a fixed preconditioner), and the
// true residual decides convergence or a restart. x is the initial guess on input.
void solve_gmres_dev(hfk_problem* op, hfk_pmg* prec, const double* b, double* x, double rtol, double atol, int maxiter,
                     int restart, int flexible, int* iters, int* converged, double* relres) {
  HFK_REQUIRE(op && b && x && iters && converged, HFK_ERR_ARG, "null argument");
  HFK_REQUIRE(rtol >= 0 && rtol < 1, HFK_ERR_ARG, "the relative tolerance must be in [0, 1)");
  HFK_REQUIRE(atol >= 0 && maxiter > 0 && restart > 0, HFK_ERR_ARG, "atol must be >= 0, maxiter and restart > 0");
  HFK_REQUIRE(op->prepared, HFK_ERR_STATE, "the operator has not been prepared");
  const int64_t n = op->nfree;
  HFK_REQUIRE(n < ((int64_t)1 << 31), HFK_ERR_UNSUPPORTED, "GMRES supports fewer than 2^31 free dofs");
  if (prec) {
    HFK_REQUIRE(prec->lv[0] == op, HFK_ERR_ARG, "the preconditioner's working level is not this operator");
    pmg_bind_stream(prec);
  }
  cudaStream_t s = op->stream;
  *iters = 0;
  *converged = 0;
  if (relres) *relres = NAN;
  if (prec && !prec->ok) {  // src/solvers.jl:114-121: no iteration, a failed solve
    if (is_device_ptr(x)) HFK_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), s));
    else std::fill(x, x + n, 0.0);
    HFK_CUDA(cudaStreamSynchronize(s));
    return;
  }
  const int m = std::min(restart, maxiter);
  hfk::CGWork& cw = op->cg;
  hfk::GmresWork& gw = op->gm;
  const double* bd = dev_in(b, n, cw.b, s);
  double* xd = x;
  if (!is_device_ptr(x)) {
    cw.x.resize(n);
    HFK_CUDA(cudaMemcpyAsync(cw.x.p, x, n * sizeof(double), cudaMemcpyHostToDevice, s));
    xd = cw.x.p;
  }
  gw.V.resize((size_t)(m + 1) * n);
  gw.Z.resize((size_t)(flexible ? m : 1) * n);
  gw.w.resize(n);
  gw.h.resize(m + 1);
  // Gram-Schmidt and basis combinations on the engine's multi-dot / multi-axpy kernels, over the
  // whole vector (one range of reduction chunks for all segments)
  ensure_seg_items(op);
  gw.part.resize((size_t)std::max(op->nitems, 1) * SEG_MDOTS);
  const int32_t all[2] = {0, op->nitems};
  gw.all.upload(all, 2, s);
  auto gram_dots = [&](int k, const double* Vb, const double* w, double* h) {  // h = Vb[:, :k]^T w
    for (int c0 = 0; c0 < k; c0 += SEG_MDOTS) {
      const int kc = std::min(SEG_MDOTS, k - c0);
      if (op->nitems) {
        seg_mdots_kernel<<<op->nitems, RED_THREADS, 0, s>>>(kc, op->item_lo.p, op->item_hi.p, Vb + (size_t)c0 * n, n,
                                                             w, gw.part.p);
        check_launch(op);
      }
      seg_mfinish_kernel<<<1, RED_THREADS, 0, s>>>(kc, gw.all.p, gw.part.p, h + c0, 0);
      check_launch(op);
    }
  };
  auto basis_sub = [&](int k, const double* c, const double* Vb, double* y) {  // y -= Vb[:, :k] c
    seg_maxpy_kernel<<<vec_grid(n), 256, 0, s>>>(n, nullptr, k, c, 0, Vb, n, y);
    check_launch(op);
  };
  auto apply_prec = [&](const double* in, double* outp) {
    if (prec) pmg_apply_dev(prec, in, outp);
    else HFK_CUDA(cudaMemcpyAsync(outp, in, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  };
  Reducer& red = cw.red;
  double res[3];
  double* V = gw.V.p;
  // r0 = b - A x into V[:, 0]
  mf_apply_dev(op, xd, gw.w.p);
  axpbyz_kernel<double><<<vec_grid(n), 256, 0, s>>>(n, 1.0, bd, -1.0, gw.w.p, V);
  check_launch(op);
  dots<double>(op, red, n, 2, bd, bd, V, V, nullptr, nullptr, res);
  const double nb = std::sqrt(res[0]);
  const double tol = atol + rtol * nb;
  double beta = std::sqrt(res[1]);
  bool conv = beta <= tol;
  int it = 0;
  std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m), h1(m + 1), h2(m + 1);
  while (!conv && it < maxiter) {
    scale_kernel<<<vec_grid(n), 256, 0, s>>>(n, 1.0 / beta, V);
    check_launch(op);
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int jend = 0;
    for (int j = 0; j < m && it < maxiter; ++j) {
      double* vj = V + (size_t)j * n;
      double* vn = V + (size_t)(j + 1) * n;
      double* zj = gw.Z.p + (flexible ? (size_t)j * n : 0);
      apply_prec(vj, zj);
      mf_apply_dev(op, zj, vn);
      // classical Gram-Schmidt, twice
      for (int pass = 0; pass < 2; ++pass) {
        gram_dots(j + 1, V, vn, gw.h.p);
        basis_sub(j + 1, gw.h.p, V, vn);
        HFK_CUDA(cudaMemcpyAsync(pass ? h2.data() : h1.data(), gw.h.p, (j + 1) * sizeof(double),
                                 cudaMemcpyDeviceToHost, s));
      }
      dots<double>(op, red, n, 1, vn, vn, nullptr, nullptr, nullptr, nullptr, res);  // synchronises
      const double hn = std::sqrt(res[0]);
      double* Hj = H.data() + (size_t)j * (m + 1);
      for (int i = 0; i <= j; ++i) Hj[i] = h1[i] + h2[i];
      Hj[j + 1] = hn;
      for (int i = 0; i < j; ++i) {  // the previous rotations
        const double t = cs[i] * Hj[i] + sn[i] * Hj[i + 1];
        Hj[i + 1] = -sn[i] * Hj[i] + cs[i] * Hj[i + 1];
        Hj[i] = t;
      }
      const double rr = std::hypot(Hj[j], Hj[j + 1]);
      cs[j] = rr > 0 ? Hj[j] / rr : 1.0;
      sn[j] = rr > 0 ? Hj[j + 1] / rr : 0.0;
      Hj[j] = rr;
      Hj[j + 1] = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      ++it;
      jend = j + 1;
      if (std::fabs(g[j + 1]) <= tol || !(hn > 0) || !std::isfinite(hn)) break;  // estimate met, or breakdown
      scale_kernel<<<vec_grid(n), 256, 0, s>>>(n, 1.0 / hn, vn);
      check_launch(op);
    }
    // y = R^-1 g, then the update of x
    for (int i = jend - 1; i >= 0; --i) {
      double t = g[i];
      for (int k = i + 1; k < jend; ++k) t -= H[(size_t)k * (m + 1) + i] * y[k];
      const double d = H[(size_t)i * (m + 1) + i];
      y[i] = d != 0.0 ? t / d : 0.0;
    }
    for (int i = 0; i < jend; ++i) y[i] = -y[i];  // the multi-axpy subtracts
    HFK_CUDA(cudaMemcpyAsync(gw.h.p, y.data(), jend * sizeof(double), cudaMemcpyHostToDevice, s));
    if (flexible) {
      basis_sub(jend, gw.h.p, gw.Z.p, xd);
    } else {
      HFK_CUDA(cudaMemsetAsync(gw.w.p, 0, n * sizeof(double), s));
      basis_sub(jend, gw.h.p, V, gw.w.p);
      apply_prec(gw.w.p, gw.Z.p);
      axpby_kernel<double><<<vec_grid(n), 256, 0, s>>>(n, 1.0, gw.Z.p, 1.0, xd);
      check_launch(op);
    }
    // the true residual decides (and starts the next cycle)
    mf_apply_dev(op, xd, gw.w.p);
    axpbyz_kernel<double><<<vec_grid(n), 256, 0, s>>>(n, 1.0, bd, -1.0, gw.w.p, V);
    check_launch(op);
    dots<double>(op, red, n, 1, V, V, nullptr, nullptr, nullptr, nullptr, res);
    beta = std::sqrt(res[0]);
    conv = beta <= tol;
    if (!std::isfinite(beta)) break;
  }
  if (relres) *relres = nb > 0 ? beta / nb : beta;
  finish_out(x, xd, n, s);
  HFK_CUDA(cudaStreamSynchronize(s));
  *iters = it;
  *converged = conv;
}

// The remaining iterations of the batched CG as one CUDA graph: a while node whose body is one
// iteration (both halves, captured from the engine's own launches) and a last kernel that counts
// the iteration and sets the loop condition (a segment still active, the limit not reached). The
// host launches it once and waits. After the last check finds no active segment the body's second
// half still runs once; it changes only the direction and its scalars, which nothing reads after
// the loop. Returns the iteration count reached, or -1 (nothing launched) if the graph could not be
// built, in which case the caller continues on the host.
int seg_cg_device_loop(hfk_problem* op, const std::function<void()>& step_half,
                       const std::function<void()>& direction_half, hfk::CGWork& cw, int it0, int maxiter) {
  cudaStream_t s = op->stream;
  cw.itd.resize(1);
  set_int_kernel<<<1, 1, 0, s>>>(cw.itd.p, it0);
  check_launch(op);
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  bool built = false;
  if (cudaGraphCreate(&g, 0) == cudaSuccess) {
    cudaGraphConditionalHandle h;
    cudaGraphNodeParams np{};
    cudaGraphNode_t node;
    if (cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) == cudaSuccess) {
      np.type = cudaGraphNodeTypeConditional;
      np.conditional.handle = h;
      np.conditional.type = cudaGraphCondTypeWhile;
      np.conditional.size = 1;
      if (cudaGraphAddNode(&node, g, nullptr, 0, &np) == cudaSuccess &&
          cudaStreamBeginCaptureToGraph(s, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                        cudaStreamCaptureModeRelaxed) == cudaSuccess) {
        bool captured = true;
        try {
          step_half();
          direction_half();
          seg_cg_loop_kernel<<<1, 32, 0, s>>>(h, cw.cnt.p, cw.itd.p, maxiter);
          check_launch(op);
        } catch (...) {
          captured = false;
        }
        cudaGraph_t body = nullptr;
        captured = cudaStreamEndCapture(s, &body) == cudaSuccess && captured;
        built = captured && cudaGraphInstantiate(&ge, g, 0) == cudaSuccess;
      }
    }
  }
  if (!built) {
    cudaGetLastError();  // the failed build's error state, not a launch error
    if (ge) cudaGraphExecDestroy(ge);
    if (g) cudaGraphDestroy(g);
    return -1;
  }
  int reached = it0;
  const cudaError_t e = cudaGraphLaunch(ge, s);
  if (e == cudaSuccess) {
    HFK_CUDA(cudaMemcpyAsync(&reached, cw.itd.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    HFK_CUDA(cudaStreamSynchronize(s));
  }
  cudaGraphExecDestroy(ge);
  cudaGraphDestroy(g);
  HFK_CUDA(e);
  return reached;
}

// MatrixFreeSolver.solve! (src/solvers.jl:111-159) on every segment of op at once: one FP64
// (flexible) CG per segment with its own alpha, beta, tolerance atol + rtol ||b_s|| and stopping
// test; every product and preconditioner application covers all segments in one launch sequence.
// The scalars stay on the device; one flag count is read per iteration. A segment stops when it
// converges or meets non-positive curvature (indefinite); its iterate is then left unchanged.
void solve_cg_seg_dev(hfk_problem* op, hfk_pmg* prec, const double* b, double* x, double rtol, double atol, int maxiter,
                      int flexible, int* iters, int* converged, int* indefinite, double* relres, int* sweeps) {
  HFK_REQUIRE(op && b && x && iters && converged, HFK_ERR_ARG, "null argument");
  HFK_REQUIRE(rtol >= 0 && rtol < 1, HFK_ERR_ARG, "the relative tolerance must be in [0, 1)");
  HFK_REQUIRE(atol >= 0 && maxiter > 0, HFK_ERR_ARG, "atol must be >= 0 and maxiter > 0");
  HFK_REQUIRE(op->prepared, HFK_ERR_STATE, "the operator has not been prepared");
  const int64_t n = op->nfree;
  const int ns = op->nseg;
  if (prec) {
    HFK_REQUIRE(prec->lv[0] == op, HFK_ERR_ARG, "the preconditioner's working level is not this operator");
    pmg_bind_stream(prec);
  }
  cudaStream_t s = op->stream;
  for (int i = 0; i < ns; ++i) {
    iters[i] = 0;
    converged[i] = 0;
    if (indefinite) indefinite[i] = 0;
    if (relres) relres[i] = NAN;
  }
  if (sweeps) *sweeps = 0;
  if (prec && !prec->ok) {  // src/solvers.jl:114-121: no iteration, a failed solve
    if (is_device_ptr(x)) HFK_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), s));
    else std::fill(x, x + n, 0.0);
    HFK_CUDA(cudaStreamSynchronize(s));
    return;
  }
  ensure_seg_items(op);
  hfk::CGWork& cw = op->cg;
  DBuf<double>&db = cw.b, &dx = cw.x, &r = cw.r, &z = cw.z, &pp = cw.p, &q = cw.q, &rold = cw.rold;
  const double* bd = dev_in(b, n, db, s);
  double* xd = x;
  if (!is_device_ptr(x)) {
    dx.resize(n);
    HFK_CUDA(cudaMemcpyAsync(dx.p, x, n * sizeof(double), cudaMemcpyHostToDevice, s));
    xd = dx.p;
  }
  r.resize(n);
  z.resize(n);
  pp.resize(n);
  q.resize(n);
  if (flexible) rold.resize(n);
  cw.sc.resize((size_t)SEG_NS * ns);
  cw.fl.resize((size_t)SEG_NF * ns);
  cw.cnt.resize(1);
  double* sc = cw.sc.p;
  int* fl = cw.fl.p;
  const int32_t* seg = seg_dof_map(op);
  const int sg = std::max(1, (ns + 255) / 256);
  auto active_count = [&]() {
    int c = 0;
    HFK_CUDA(cudaMemcpyAsync(&c, cw.cnt.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    HFK_CUDA(cudaStreamSynchronize(s));
    return c;
  };
  // r = b - A x
  mf_apply_dev(op, xd, q.p);
  axpbyz_kernel<double><<<vec_grid(n), 256, 0, s>>>(n, 1.0, bd, -1.0, q.p, r.p);
  check_launch(op);
  seg_dots<double>(op, 2, sc + S_BB, SEG_NS, bd, bd, r.p, r.p);
  seg_cg_init_kernel<<<1, 256, 0, s>>>(ns, sc, fl, rtol, atol, cw.cnt.p);
  check_launch(op);
  // the cell kernels of every level skip the problems that are not active (the flags are shared
  // with the hierarchy's levels); every flag is set back to 1 when the solve ends
  int32_t* mask = op->seg_active;
  auto set_mask = [&](int value) {
    if (mask) seg_mask_kernel<<<sg, 256, 0, s>>>(ns, fl, mask, value);
  };
  struct MaskReset {
    std::function<void()> f;
    ~MaskReset() { f(); }
  } mask_reset{[&]() {
    if (mask) seg_mask_kernel<<<sg, 256, 0, s>>>(ns, fl, mask, 1);
  }};
  set_mask(-1);
  int nact = active_count();
  int it = 0;
  auto apply_prec = [&](const double* in, double* outp) {
    if (prec) pmg_apply_dev(prec, in, outp);
    else HFK_CUDA(cudaMemcpyAsync(outp, in, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  };
  // one iteration in two halves: the product, step and convergence check; then the preconditioner
  // and the new direction (skipped on the host when no segment is active any more)
  auto step_half = [&]() {
    mf_apply_dev(op, pp.p, q.p);
    seg_dots<double>(op, 1, sc + S_PQ, SEG_NS, pp.p, q.p);
    seg_cg_alpha_kernel<<<sg, 256, 0, s>>>(ns, sc, fl);
    check_launch(op);
    seg_cg_update_kernel<<<vec_grid(n), 256, 0, s>>>(n, seg, sc, pp.p, q.p, xd, r.p, flexible ? rold.p : nullptr);
    check_launch(op);
    seg_dots<double>(op, 1, sc + S_RR, SEG_NS, r.p, r.p);
    seg_cg_check_kernel<<<1, 256, 0, s>>>(ns, sc, fl, cw.cnt.p);
    check_launch(op);
    set_mask(-1);
  };
  auto direction_half = [&]() {
    apply_prec(r.p, z.p);
    if (flexible) seg_dots<double>(op, 2, sc + S_ZR, SEG_NS, z.p, r.p, z.p, rold.p);
    else seg_dots<double>(op, 1, sc + S_ZR, SEG_NS, z.p, r.p);
    seg_cg_beta_kernel<<<sg, 256, 0, s>>>(ns, sc, fl, flexible);
    check_launch(op);
    seg_xpby_kernel<<<vec_grid(n), 256, 0, s>>>(n, seg, sc, S_BETA, z.p, pp.p);
    check_launch(op);
  };
  bool device_loop = op->solve_graph && s != cudaStreamLegacy;
  if (nact > 0) {
    apply_prec(r.p, z.p);
    HFK_CUDA(cudaMemcpyAsync(pp.p, z.p, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    seg_dots<double>(op, 1, sc + S_RZ, SEG_NS, r.p, z.p);
    while (it < maxiter) {
      ++it;
      step_half();
      if (active_count() == 0) break;
      direction_half();
      // two host-driven iterations have created every buffer and tuned every launch shape: the
      // remaining iterations run as one graph launch, the loop itself on the device
      if (device_loop && it >= 2 && it < maxiter) {
        const int reached = seg_cg_device_loop(op, step_half, direction_half, cw, it, maxiter);
        if (reached >= 0) {
          // one cycle per body run; the capture itself counted one
          if (prec) prec->ncycles += reached - it - 1;
          it = reached;
          break;
        }
        device_loop = false;  // the graph could not be built: carry on from the host
      }
    }
  }
  // true residual check per segment (src/solvers.jl:150-157), on every problem
  set_mask(1);
  mf_apply_dev(op, xd, q.p);
  axpbyz_kernel<double><<<vec_grid(n), 256, 0, s>>>(n, 1.0, bd, -1.0, q.p, r.p);
  check_launch(op);
  seg_dots<double>(op, 1, sc + S_RR, SEG_NS, r.p, r.p);
  std::vector<double> hs((size_t)SEG_NS * ns);
  std::vector<int> hf((size_t)SEG_NF * ns);
  HFK_CUDA(cudaMemcpyAsync(hs.data(), sc, hs.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  HFK_CUDA(cudaMemcpyAsync(hf.data(), fl, hf.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
  finish_out(x, xd, n, s);
  HFK_CUDA(cudaStreamSynchronize(s));
  for (int i = 0; i < ns; ++i) {
    const double* c = hs.data() + (size_t)SEG_NS * i;
    const int* f = hf.data() + (size_t)SEG_NF * i;
    const double tr = std::sqrt(c[S_RR]), nb = std::sqrt(c[S_BB]);
    if (relres) relres[i] = nb > 0 ? tr / nb : tr;
    // the recursive residual decides; a solve stopped without it is judged on the true residual
    converged[i] = !f[F_INDEF] && (f[F_CONV] || tr <= c[S_TOL]);
    iters[i] = f[F_ITERS];
    if (indefinite) indefinite[i] = f[F_INDEF];
  }
  if (sweeps) *sweeps = it;
}
}  // namespace

extern "C" {
int hfk_solve_cg(hfk_problem* op, hfk_pmg* prec, const double* b, double* x, double rtol, double atol, int maxiter,
                 int flexible, int* iters, int* converged, int* indefinite, double* relres) {
  HFK_API_BEGIN
  solve_cg_dev(op, prec, b, x, rtol, atol, maxiter, flexible, iters, converged, indefinite, relres);
  if (prec) band_check(prec);
  HFK_API_END
}

int hfk_solve_gmres(hfk_problem* op, hfk_pmg* prec, const double* b, double* x, double rtol, double atol, int maxiter,
                    int restart, int flexible, int* iters, int* converged, double* relres) {
  HFK_API_BEGIN
  solve_gmres_dev(op, prec, b, x, rtol, atol, maxiter, restart, flexible, iters, converged, relres);
  if (prec) band_check(prec);
  HFK_API_END
}

int hfk_solve_cg_batched(hfk_problem* op, hfk_pmg* prec, const double* b, double* x, double rtol, double atol,
                         int maxiter, int flexible, int* iters, int* converged, int* indefinite, double* relres,
                         int* sweeps) {
  HFK_API_BEGIN
  solve_cg_seg_dev(op, prec, b, x, rtol, atol, maxiter, flexible, iters, converged, indefinite, relres, sweeps);
  if (prec) band_check(prec);
  HFK_API_END
}

int hfk_problem_set_segments(hfk_problem* p, int nseg, const int64_t* dof_off, const int32_t* cell_off,
                             const double* params) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && dof_off && nseg >= 1, HFK_ERR_ARG, "segments: null argument or nseg < 1");
  HFK_REQUIRE(dof_off[0] == 0 && dof_off[nseg] == p->nfree, HFK_ERR_ARG,
              "segments: dof offsets must start at 0 and end at the number of free dofs");
  for (int s = 0; s < nseg; ++s)
    HFK_REQUIRE(dof_off[s] <= dof_off[s + 1], HFK_ERR_ARG, "segments: dof offsets must be non-decreasing");
  HFK_REQUIRE(!params || cell_off, HFK_ERR_ARG, "segments: per-segment parameters need the cell ranges");
  if (cell_off) {
    HFK_REQUIRE(cell_off[0] == 0 && cell_off[nseg] == p->ncells, HFK_ERR_ARG,
                "segments: cell offsets must start at 0 and end at the number of cells");
    for (int s = 0; s < nseg; ++s) {
      HFK_REQUIRE(cell_off[s] <= cell_off[s + 1], HFK_ERR_ARG, "segments: cell offsets must be non-decreasing");
      // independence: the free dofs of a segment's cells lie in the segment's dof range
      for (int32_t c = cell_off[s]; c < cell_off[s + 1]; ++c)
        for (int j = 0; j < p->ndl; ++j) {
          const int32_t id = p->h_ids[(size_t)c * p->ndl + j];
          HFK_REQUIRE(id <= 0 || (id - 1 >= dof_off[s] && id - 1 < dof_off[s + 1]), HFK_ERR_ARG,
                      "segments: a cell of one segment holds a free dof of another (segments must be independent)");
        }
    }
  }
  if (params)
    for (int s = 0; s < 2 * nseg; ++s)
      HFK_REQUIRE(std::isfinite(params[s]), HFK_ERR_ARG, "segments: non-finite law parameter");
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  p->nseg = nseg;
  p->seg_off.assign(dof_off, dof_off + nseg + 1);
  if (cell_off) p->seg_cells.assign(cell_off, cell_off + nseg + 1);
  else p->seg_cells.clear();
  if (nseg > 1) {
    std::vector<int32_t> sd(std::max<int64_t>(p->nfree, 1), 0);
    for (int s = 0; s < nseg; ++s)
      for (int64_t i = dof_off[s]; i < dof_off[s + 1]; ++i) sd[i] = s;
    p->seg_of_dof.upload(sd.data(), sd.size(), p->stream);
    if (p->nblocks > 0) {
      std::vector<int32_t> dofs((size_t)3 * p->nblocks);
      HFK_CUDA(cudaMemcpy(dofs.data(), p->bdofs.p, dofs.size() * sizeof(int32_t), cudaMemcpyDeviceToHost));
      build_seg_of_block(p, dofs);
    }
  } else {
    p->seg_of_dof.release();
    p->seg_of_block.release();
  }
  if (nseg > 1 && cell_off) {
    std::vector<int32_t> cs(std::max(p->ncells, 1), 0);
    for (int s = 0; s < nseg; ++s)
      for (int32_t c = cell_off[s]; c < cell_off[s + 1]; ++c) cs[c] = s;
    p->cell_seg.upload(cs.data(), cs.size(), p->stream);
    std::vector<int32_t> ones(nseg, 1);
    p->seg_active_own.upload(ones.data(), ones.size(), p->stream);
    p->seg_active = p->seg_active_own.p;
  } else {
    p->cell_seg.release();
    p->seg_active_own.release();
    p->seg_active = nullptr;
  }
  if (params) {
    p->seg_lm.assign(params, params + 2 * (size_t)nseg);
    std::vector<double> lm((size_t)2 * std::max(p->ncells, 1), 0.0);
    for (int s = 0; s < nseg; ++s)
      for (int32_t c = cell_off[s]; c < cell_off[s + 1]; ++c) {
        lm[2 * (size_t)c] = params[2 * s];
        lm[2 * (size_t)c + 1] = params[2 * s + 1];
      }
    p->cell_lm.upload(lm.data(), lm.size(), p->stream);
  } else {
    p->seg_lm.clear();
  }
  p->items_built = false;
  ensure_seg_items(p);
  HFK_API_END
}

int hfk_problem_segments(hfk_problem* p, int* nseg) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && nseg, HFK_ERR_ARG, "null argument");
  *nseg = p->nseg;
  HFK_API_END
}

int hfk_problem_set_cell_params(hfk_problem* p, const double* lm) {
  HFK_API_BEGIN
  HFK_REQUIRE(p, HFK_ERR_ARG, "null handle");
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  if (!lm) {
    p->cell_lm.release();
  } else {
    HFK_REQUIRE(!is_device_ptr(lm), HFK_ERR_ARG, "per-cell parameters are read from host memory");
    for (size_t i = 0; i < 2 * (size_t)p->ncells; ++i)
      HFK_REQUIRE(std::isfinite(lm[i]), HFK_ERR_ARG, "non-finite per-cell law parameter");
    p->cell_lm.upload(lm, 2 * (size_t)p->ncells, p->stream);
    HFK_CUDA(cudaStreamSynchronize(p->stream));
  }
  HFK_API_END
}

int hfk_segment_dots(hfk_problem* p, const double* a, const double* b, double* out) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && a && b && out, HFK_ERR_ARG, "null argument");
  const double* da = dev_in(a, p->nfree, p->stage_in, p->stream);
  const double* db = dev_in(b, p->nfree, p->stage_in2, p->stream);
  DBuf<double> o;
  o.resize(p->nseg);
  seg_dots<double>(p, 1, o.p, 1, da, db);
  HFK_CUDA(cudaMemcpyAsync(out, o.p, p->nseg * sizeof(double), cudaMemcpyDefault, p->stream));
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  HFK_API_END
}

int hfk_segment_scale(hfk_problem* p, double* x, const double* f) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && x && f, HFK_ERR_ARG, "null argument");
  HFK_REQUIRE(is_device_ptr(x), HFK_ERR_ARG, "hfk_segment_scale scales a device vector");
  DBuf<double> d;
  d.upload(f, p->nseg, p->stream);
  seg_mul_kernel<<<vec_grid(p->nfree), 256, 0, p->stream>>>(p->nfree, seg_dof_map(p), d.p, x);
  check_launch(p);
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  HFK_API_END
}

int hfk_pmg_segment_bounds(hfk_pmg* m, int level, double* lmin, double* lmax) {
  HFK_API_BEGIN
  HFK_REQUIRE(m && level >= 0 && level < m->L && lmin && lmax, HFK_ERR_ARG, "invalid argument");
  const std::vector<double>&lo = m->seg_lmin[level], &hi = m->seg_lmax[level];
  for (int s = 0; s < m->lv[level]->nseg; ++s) {
    lmin[s] = s < (int)lo.size() ? lo[s] : NAN;
    lmax[s] = s < (int)hi.size() ? hi[s] : NAN;
  }
  HFK_API_END
}

int hfk_pmg_set_eig_inner(hfk_pmg* m, int mode) {
  HFK_API_BEGIN
  HFK_REQUIRE(m && (mode == HFK_EIG_EUCLIDEAN || mode == HFK_EIG_PRECONDITIONED), HFK_ERR_ARG,
              "eigenvalue estimate: mode must be HFK_EIG_EUCLIDEAN or HFK_EIG_PRECONDITIONED");
  m->eig_inner = mode;
  HFK_API_END
}

int hfk_pmg_set_coarse(hfk_pmg* m, int mode, int iters) {
  HFK_API_BEGIN
  HFK_REQUIRE(m && (mode == HFK_COARSE_CHOLESKY || mode == HFK_COARSE_CG), HFK_ERR_ARG,
              "coarse mode must be HFK_COARSE_CHOLESKY or HFK_COARSE_CG");
  HFK_REQUIRE(mode != HFK_COARSE_CG || iters >= 1, HFK_ERR_ARG, "the coarse CG needs at least one iteration");
  HFK_CUDA(cudaStreamSynchronize(m->lv[0]->stream));
  m->coarse_mode = mode;
  if (mode == HFK_COARSE_CG) m->coarse_iters = iters;
  pmg_drop_graph(m);
  // the hierarchy is rebuilt by the next update
  m->built = false;
  m->ok = false;
  HFK_API_END
}

int hfk_pmg_test_coarse_wait(hfk_pmg* m, int polls, int skip_first) {
  HFK_API_BEGIN
  HFK_REQUIRE(m && polls >= 0, HFK_ERR_ARG, "invalid argument");
  HFK_CUDA(cudaStreamSynchronize(m->lv[0]->stream));
  m->bs_spin = polls > 0 ? polls : BS_SPIN_LIMIT;
  m->bs_skip = skip_first != 0;
  pmg_drop_graph(m);  // the captured cycle holds the old limit; the next cycle runs uncaptured
  HFK_API_END
}

}  // extern "C"

// =================================================================================================
// Learned correction: the network, its training, and its place after the V-cycle
// =================================================================================================
extern "C" {

int hfk_pmg_set_mlp(hfk_pmg* m, hfk_mlp* net) {
  HFK_API_BEGIN
  HFK_REQUIRE(m, HFK_ERR_ARG, "null handle");
  m->mlp = net;
  m->ml_accepted.resize(1);
  m->ml_accepted.zero(m->lv[0]->stream);
  m->ml_tried = 0;
  HFK_CUDA(cudaStreamSynchronize(m->lv[0]->stream));
  HFK_API_END
}

int hfk_pmg_mlp_stats(hfk_pmg* m, int64_t* tried, int64_t* accepted) {
  HFK_API_BEGIN
  HFK_REQUIRE(m && tried && accepted, HFK_ERR_ARG, "null argument");
  int acc = 0;
  if (m->ml_accepted.p) {
    HFK_CUDA(cudaMemcpyAsync(&acc, m->ml_accepted.p, sizeof(int), cudaMemcpyDeviceToHost, m->lv[0]->stream));
    HFK_CUDA(cudaStreamSynchronize(m->lv[0]->stream));
  }
  *tried = m->ml_tried;
  *accepted = acc;
  HFK_API_END
}

int hfk_pmg_mlp_sample(hfk_pmg* m, const double* r, float* feats, float* targets, int* nsamples, double rtol) {
  HFK_API_BEGIN
  HFK_REQUIRE(m && r && feats && targets && nsamples && rtol > 0 && rtol < 1, HFK_ERR_ARG, "invalid argument");
  HFK_REQUIRE(m->built && m->ok, HFK_ERR_STATE, "PMultigrid: call hfk_pmg_update first (with a usable hierarchy)");
  HFK_REQUIRE(is_device_ptr(r) && is_device_ptr(feats) && is_device_ptr(targets), HFK_ERR_ARG,
              "hfk_pmg_mlp_sample takes device pointers");
  pmg_bind_stream(m);
  hfk_problem* p = m->lv[0];
  const int64_t n = p->nfree;
  DBuf<double> y, e;
  y.resize(n);
  e.resize(n);
  hfk_mlp* net = m->mlp;
  m->mlp = nullptr;  // plain cycle
  try {
    pmg_apply_dev(m, r, y.p);
    const int nb = mlp_prepare_features(m, r, y.p);
    // the remaining error e = A^-1 s, by an accurate solve preconditioned by the plain cycle
    HFK_CUDA(cudaMemsetAsync(e.p, 0, n * sizeof(double), p->stream));
    if (p->nseg > 1) {
      std::vector<int> its(p->nseg), conv(p->nseg);
      solve_cg_seg_dev(p, m, m->ml_s.p, e.p, rtol, 0.0, 500, 1, its.data(), conv.data(), nullptr, nullptr, nullptr);
      for (int c : conv) HFK_REQUIRE(c, HFK_ERR_NUMERIC, "the target solve of a training sample did not converge");
    } else {
      int its = 0, conv = 0, ind = 0;
      double rel = 0;
      solve_cg_dev(p, m, m->ml_s.p, e.p, rtol, 0.0, 500, 1, &its, &conv, &ind, &rel);
      HFK_REQUIRE(conv, HFK_ERR_NUMERIC, "the target solve of a training sample did not converge");
    }
    mlp_targets_kernel<<<vec_grid(nb), 256, 0, p->stream>>>(nb, p->bdofs.p, seg_block_map(p), e.p, m->ml_scal.p, 8,
                                                             targets);
    check_launch(p);
    HFK_CUDA(cudaMemcpyAsync(feats, m->ml_feats.p, (size_t)nb * MLP_IN * sizeof(float), cudaMemcpyDeviceToDevice,
                             p->stream));
    HFK_CUDA(cudaStreamSynchronize(p->stream));
    *nsamples = nb;
  } catch (...) {
    m->mlp = net;
    throw;
  }
  m->mlp = net;
  HFK_API_END
}

}  // extern "C"
