// C ABI of the Oseen-BDF step on Taylor-Hood P2-P1 tetrahedra: the handle, its set-up, and the
// dispatch of the fused element kernels (kern_oseen.cuh).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <memory>
#include <string>
#include <vector>

#include "engine.h"
#include "kern_oseen.cuh"

using namespace hfk;

// =================================================================================================
// Oseen–BDF step on Taylor–Hood P2–P1 tetrahedra (the reference's Oseen volume group,
// test/common.jl:164-228; assembly driver src/assembly.jl:909-927, :1413-1505)
// =================================================================================================
struct hfk_oseen {
  hfk_problem base;  // ids, colours, CSC pattern and positions (34 local dofs, the caller's order)
  int nq = 0;
  DBuf<double> w, N2, dN2, H2, N1, dN1, un, und, unm1, unm1d;
  double rho = 1, mu = 1e-3, dt = 1e-3;
  int bdf2 = 1;
  // outlet boundary group (0 facets: none)
  int nf = 0, nqf = 0;
  DBuf<int32_t> fcell, fface;
  DBuf<double> farea, fnormal, fw, fN;
  double Pc = 0.7, ZA = 2.3;
};

namespace {
OseenData oseen_data(hfk_oseen* o, const int32_t* cells, int n) {
  OseenData d;
  d.ids = o->base.ids.p;
  d.cells = cells;
  d.ncells_list = n;
  d.coords = o->base.coords.p;
  d.w = o->w.p;
  d.N2 = o->N2.p;
  d.dN2 = o->dN2.p;
  d.H2 = o->H2.p;
  d.N1 = o->N1.p;
  d.dN1 = o->dN1.p;
  d.un = o->un.p;
  d.und = o->und.p;
  d.unm1 = o->unm1.p;
  d.unm1d = o->unm1d.p;
  d.nq = o->nq;
  d.rho = o->rho;
  d.mu = o->mu;
  d.bdf2 = o->bdf2;
  d.c0 = o->bdf2 ? 1.5 / o->dt : 1.0 / o->dt;  // BDF coefficients (test/common.jl:183-185)
  d.c1 = o->bdf2 ? 2.0 / o->dt : 1.0 / o->dt;
  d.c2 = o->bdf2 ? 0.5 / o->dt : 0.0;
  return d;
}

void oseen_run(hfk_oseen* o, OseenIO io) {
  hfk_problem* p = &o->base;
  const size_t smem = (size_t)OseenSmem{o->nq}.total() * sizeof(double);
  static PerDeviceLimit attr;
  raise_smem_limit(oseen_kernel, smem, attr);
  if (use_atomic_scatter(p)) {
    io.atomic = 1;
    oseen_kernel<<<p->ncells, OS_THREADS, smem, p->stream>>>(oseen_data(o, nullptr, p->ncells), io);
    check_launch(p);
    return;
  }
  io.atomic = 0;
  for (int c = 0; c < p->ncolors; ++c) {
    const int n = p->color_start[c + 1] - p->color_start[c];
    if (!n) continue;
    oseen_kernel<<<n, OS_THREADS, smem, p->stream>>>(oseen_data(o, p->cells_by_color.p + p->color_start[c], n), io);
    check_launch(p);
  }
}

// the outlet boundary group after the volume terms (atomic scatter: its facets are few)
void oseen_run_outlet(hfk_oseen* o, OseenIO io) {
  if (!o->nf) return;
  hfk_problem* p = &o->base;
  OutletData fd{o->nf, o->nqf, o->fcell.p, o->fface.p, o->farea.p, o->fnormal.p, o->fw.p, o->fN.p, o->Pc, o->ZA};
  oseen_outlet_kernel<<<o->nf, 128, 0, p->stream>>>(oseen_data(o, nullptr, p->ncells), fd, io);
  check_launch(p);
}

void oseen_set_params(hfk_oseen* o, const double* params, int nparams) {
  HFK_REQUIRE(params && nparams == 4, HFK_ERR_ARG, "Oseen parameters: rho, mu, dt, bdf2 (0 or 1)");
  HFK_REQUIRE(params[0] > 0 && params[1] > 0 && params[2] > 0, HFK_ERR_ARG, "rho, mu and dt must be positive");
  o->rho = params[0];
  o->mu = params[1];
  o->dt = params[2];
  o->bdf2 = params[3] != 0;
}
}  // namespace

extern "C" {

int hfk_oseen_create(hfk_oseen** out, int ncells, int nq, const double* w, const double* N2, const double* dN2,
                     const double* H2, const double* N1, const double* dN1, const double* coords,
                     const int32_t* cell_dof_ids, int64_t nfree, int64_t ndir, const double* params, int nparams) {
  HFK_API_BEGIN
  HFK_REQUIRE(out, HFK_ERR_ARG, "null output handle");
  *out = nullptr;
  HFK_REQUIRE(ncells > 0 && nq > 0 && nq <= OS_MAXQ, HFK_ERR_ARG, "invalid sizes (ncells > 0, 0 < nq <= 64)");
  HFK_REQUIRE(w && N2 && dN2 && H2 && N1 && dN1 && coords && cell_dof_ids, HFK_ERR_ARG, "null input array");
  HFK_REQUIRE(nfree >= 0 && ndir >= 0 && nfree < (1ll << 31), HFK_ERR_ARG, "invalid dof counts");
  auto o = std::make_unique<hfk_oseen>();
  oseen_set_params(o.get(), params, nparams);
  hfk_problem* p = &o->base;
  p->ncells = ncells;
  p->ndl = OS_NDL;
  p->nn = OS_NDL;
  p->np = nq;
  p->nfree = nfree;
  p->ndir = ndir;
  HFK_CUDA(cudaGetDevice(&p->device));
  HFK_CUDA(cudaStreamCreate(&p->own_stream));
  p->stream = p->own_stream;
  const size_t nids = (size_t)OS_NDL * ncells;
  for (size_t k = 0; k < nids; ++k)
    HFK_REQUIRE(cell_dof_ids[k] <= nfree && -(int64_t)cell_dof_ids[k] <= ndir, HFK_ERR_ARG, "cell dof id out of range");
  p->h_ids.assign(cell_dof_ids, cell_dof_ids + nids);
  p->nodeperm.resize(OS_NDL);
  for (int i = 0; i < OS_NDL; ++i) p->nodeperm[i] = i;
  p->ids.upload(cell_dof_ids, nids, p->stream);
  p->coords.upload(coords, (size_t)12 * ncells, p->stream);
  o->nq = nq;
  o->w.upload(w, nq, p->stream);
  o->N2.upload(N2, (size_t)OS_NV * nq, p->stream);
  o->dN2.upload(dN2, (size_t)OS_NV * 3 * nq, p->stream);
  o->H2.upload(H2, (size_t)OS_NV * 9, p->stream);
  o->N1.upload(N1, (size_t)OS_NP * nq, p->stream);
  o->dN1.upload(dN1, (size_t)OS_NP * 3 * nq, p->stream);
  for (auto* b : {&o->un, &o->unm1}) {
    b->resize(std::max<int64_t>(nfree, 1));
    b->zero(p->stream);
  }
  for (auto* b : {&o->und, &o->unm1d}) {
    b->resize(std::max<int64_t>(ndir, 1));
    b->zero(p->stream);
  }
  color_cells(p);
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  *out = o.release();
  HFK_API_END
}

int hfk_oseen_destroy(hfk_oseen* o) {
  HFK_API_BEGIN
  if (!o) return HFK_OK;
  if (o->base.own_stream) {
    cudaStreamSynchronize(o->base.own_stream);
    cudaStreamDestroy(o->base.own_stream);
  }
  delete o;
  HFK_API_END
}

int hfk_oseen_set_params(hfk_oseen* o, const double* params, int nparams) {
  HFK_API_BEGIN
  HFK_REQUIRE(o, HFK_ERR_ARG, "null handle");
  oseen_set_params(o, params, nparams);
  HFK_API_END
}

int hfk_oseen_set_scatter(hfk_oseen* o, int mode) {
  HFK_API_BEGIN
  HFK_REQUIRE(o && (mode == HFK_SCATTER_AUTO || mode == HFK_SCATTER_COLOURED || mode == HFK_SCATTER_ATOMIC),
              HFK_ERR_ARG, "scatter mode must be HFK_SCATTER_AUTO, _COLOURED or _ATOMIC");
  o->base.scatter = mode;
  HFK_API_END
}

int hfk_oseen_set_history(hfk_oseen* o, const double* un, const double* und, const double* unm1, const double* unm1d) {
  HFK_API_BEGIN
  HFK_REQUIRE(o && un && unm1 && ((und && unm1d) || o->base.ndir == 0), HFK_ERR_ARG, "null argument");
  hfk_problem* p = &o->base;
  auto copy_in = [&](DBuf<double>& dst, const double* src, int64_t n) {
    if (n) HFK_CUDA(cudaMemcpyAsync(dst.p, src, n * sizeof(double), cudaMemcpyDefault, p->stream));
  };
  copy_in(o->un, un, p->nfree);
  copy_in(o->unm1, unm1, p->nfree);
  if (p->ndir) {
    copy_in(o->und, und, p->ndir);
    copy_in(o->unm1d, unm1d, p->ndir);
  }
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  HFK_API_END
}

int hfk_oseen_pattern(hfk_oseen* o, int64_t* nnz) {
  HFK_API_BEGIN
  HFK_REQUIRE(o && nnz, HFK_ERR_ARG, "null argument");
  pattern_build_dev(&o->base);
  *nnz = o->base.nnz;
  HFK_API_END
}

int hfk_oseen_pattern_get(hfk_oseen* o, int64_t* colptr, int64_t* rowval) {
  HFK_API_BEGIN
  HFK_REQUIRE(o, HFK_ERR_ARG, "null handle");
  hfk_problem* p = &o->base;
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

int hfk_oseen_residual(hfk_oseen* o, const double* x, const double* dvals, double* b) {
  HFK_API_BEGIN
  HFK_REQUIRE(o && x && b && (dvals || o->base.ndir == 0), HFK_ERR_ARG, "null argument");
  hfk_problem* p = &o->base;
  OseenIO io{};
  io.mode = 0;
  io.x = dev_in(x, p->nfree, p->stage_in, p->stream);
  io.dvals = dvals ? dev_in(dvals, p->ndir, p->stage_in2, p->stream) : nullptr;
  io.b = dev_out(b, p->nfree, p->stage_out);
  HFK_CUDA(cudaMemsetAsync(io.b, 0, p->nfree * sizeof(double), p->stream));
  oseen_run(o, io);
  oseen_run_outlet(o, io);
  finish_out(b, io.b, p->nfree, p->stream);
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  HFK_API_END
}

int hfk_oseen_jacobian(hfk_oseen* o, double* nzval) {
  HFK_API_BEGIN
  HFK_REQUIRE(o && nzval, HFK_ERR_ARG, "null argument");
  hfk_problem* p = &o->base;
  pattern_build_dev(p);
  OseenIO io{};
  io.mode = 1;
  io.nzpos = p->nzpos.p;
  io.nzval = is_device_ptr(nzval) ? nzval : p->nzval.p;
  HFK_CUDA(cudaMemsetAsync(io.nzval, 0, p->nnz * sizeof(double), p->stream));
  oseen_run(o, io);
  oseen_run_outlet(o, io);
  finish_out(nzval, io.nzval, p->nnz, p->stream);
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  HFK_API_END
}

int hfk_oseen_set_outlet(hfk_oseen* o, int nfacets, const int32_t* cells, const int32_t* faces, const double* areas,
                         const double* normals, int nq, const double* w, const double* N, double Pc, double ZA) {
  HFK_API_BEGIN
  HFK_REQUIRE(o && nfacets >= 0, HFK_ERR_ARG, "invalid argument");
  HFK_REQUIRE(nfacets == 0 || (cells && faces && areas && normals && w && N && nq > 0 && nq <= OS_MAXQF), HFK_ERR_ARG,
              "outlet facets: null array or 0 < nq <= 32 violated");
  hfk_problem* p = &o->base;
  for (int f = 0; f < nfacets; ++f)
    HFK_REQUIRE(cells[f] >= 0 && cells[f] < p->ncells && faces[f] >= 0 && faces[f] < 4, HFK_ERR_ARG,
                "outlet facet: cell or local face out of range");
  o->nf = nfacets;
  o->nqf = nq;
  o->Pc = Pc;
  o->ZA = ZA;
  if (nfacets) {
    o->fcell.upload(cells, nfacets, p->stream);
    o->fface.upload(faces, nfacets, p->stream);
    o->farea.upload(areas, nfacets, p->stream);
    o->fnormal.upload(normals, 3 * (size_t)nfacets, p->stream);
    o->fw.upload(w, nq, p->stream);
    o->fN.upload(N, (size_t)OS_NV * nq * 4, p->stream);
  }
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  HFK_API_END
}

int hfk_oseen_launch_count(hfk_oseen* o, int64_t* count) {
  HFK_API_BEGIN
  HFK_REQUIRE(o && count, HFK_ERR_ARG, "null argument");
  *count = o->base.launches;
  HFK_API_END
}

}  // extern "C"
