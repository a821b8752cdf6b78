// CPU oracle of the Oseen–BDF step on Taylor–Hood P2–P1 tetrahedra (TEST INFRASTRUCTURE: used by
// tests/ and bench.py's CPU baseline only, never by the product).
//
// Restates the volume terms of the reference's Oseen problem (test/common.jl:164-228,
// oseen_channel): a((u,p),(v,q)) and l((v,q)) with SUPG/PSPG/LSIC stabilisation, the τ formulas
// (:196-198), Ru (:199), the BDF2 coefficients (:183-187) and the elementwise Laplacian of uⁿ
// (:188-193; exact for P2 on affine cells). The integrands are evaluated literally, term by term,
// for every (test, trial) pair of basis functions with Gridap's tensor conventions
// ((∇u)[i,j] = ∂u_j/∂x_i, ∇u' its transpose, (∇u')·w = (w·∇)u): an independent restatement of what
// the GPU kernel computes in factorised form. Assembly follows the reference's colour-by-colour
// driver (src/assembly.jl:1413-1505) and its CSC pattern (src/assembly.jl:773-899).
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr int NV = 10, NP1 = 4, NDL = 34;

struct Oseen {
  int ncells = 0, nq = 0;
  int64_t nfree = 0, ndir = 0;
  std::vector<double> w, N2, dN2, H2, N1, dN1, coords;  // column-major as passed
  std::vector<int32_t> ids;                              // (34, ncells)
  double rho = 1, mu = 1e-3, dt = 1e-3;
  bool bdf2 = true;
  std::vector<double> un, und, unm1, unm1d;
  std::vector<std::vector<int32_t>> colors;
  std::vector<int64_t> colptr, rowval;
  std::vector<int32_t> nzpos;  // (34*34, ncells) 1-based, 0 = none
  // outlet boundary group (test/common.jl:194-210): facets, their cell, local face, area, normal
  int nf = 0, nqf = 0;
  std::vector<int32_t> fcell, fface;
  std::vector<double> farea, fnormal, fw, fN;  // fN (10, nqf, 4)
  double Pc = 0.7, ZA = 2.3;
};

double det3(const double* A) {  // column-major
  return A[0] * (A[4] * A[8] - A[7] * A[5]) - A[3] * (A[1] * A[8] - A[7] * A[2]) + A[6] * (A[1] * A[5] - A[4] * A[2]);
}

void inv3(const double* A, double* B) {
  const double d = det3(A);
  B[0] = (A[4] * A[8] - A[7] * A[5]) / d;
  B[3] = -(A[3] * A[8] - A[6] * A[5]) / d;
  B[6] = (A[3] * A[7] - A[6] * A[4]) / d;
  B[1] = -(A[1] * A[8] - A[7] * A[2]) / d;
  B[4] = (A[0] * A[8] - A[6] * A[2]) / d;
  B[7] = -(A[0] * A[7] - A[6] * A[1]) / d;
  B[2] = (A[1] * A[5] - A[4] * A[2]) / d;
  B[5] = -(A[0] * A[5] - A[3] * A[2]) / d;
  B[8] = (A[0] * A[4] - A[3] * A[1]) / d;
}

// one basis function of the multi-field space at a point: velocity u (3), its gradient
// Gu[i][j] = ∂u_j/∂x_i, pressure p and ∇p
struct Fn {
  double u[3] = {0, 0, 0}, Gu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, p = 0, gp[3] = {0, 0, 0};
};

struct PointData {
  double phi[NV], gphi[NV][3], psi[NP1], gpsi[NP1][3];
  double w[3], un[3], f[3], dV, taus, taup, taul;
};

struct CellGeo {
  double iJ[9];   // J^-1 column-major: iJ[K + 3c] = (J^-1)[K][c]
  double detJ, h, lap[NV];
};

CellGeo cell_geo(const Oseen& o, int cell) {
  CellGeo g;
  const double* X = &o.coords[(size_t)cell * 12];  // X[c + 3 v]
  double J[9];                                      // J[c + 3K] = x_{K+1,c} - x_{0,c}
  for (int K = 0; K < 3; ++K)
    for (int c = 0; c < 3; ++c) J[c + 3 * K] = X[c + 3 * (K + 1)] - X[c];
  g.detJ = det3(J);
  inv3(J, g.iJ);
  const double vol = std::fabs(g.detJ) / 6.0;
  g.h = std::cbrt(6.0 * std::sqrt(2.0) * vol);
  // Δφ_a = Σ_{K,K'} Ĥ_a[K,K'] Σ_c (J^-1)[K][c] (J^-1)[K'][c]
  for (int a = 0; a < NV; ++a) {
    double s = 0;
    for (int K = 0; K < 3; ++K)
      for (int Kp = 0; Kp < 3; ++Kp) {
        double G = 0;
        for (int c = 0; c < 3; ++c) G += g.iJ[K + 3 * c] * g.iJ[Kp + 3 * c];
        s += o.H2[a + NV * (K + 3 * Kp)] * G;
      }
    g.lap[a] = s;
  }
  return g;
}

double local_value(const Oseen& o, const std::vector<double>& free, const std::vector<double>& dir, int32_t id) {
  return id > 0 ? free[id - 1] : (id < 0 ? dir[-id - 1] : 0.0);
}

void point_data(const Oseen& o, int cell, const CellGeo& g, int q, PointData& P) {
  const int32_t* id = &o.ids[(size_t)cell * NDL];
  for (int a = 0; a < NV; ++a) {
    P.phi[a] = o.N2[a + NV * q];
    for (int c = 0; c < 3; ++c) {
      double s = 0;
      for (int K = 0; K < 3; ++K) s += g.iJ[K + 3 * c] * o.dN2[a + NV * (K + 3 * q)];
      P.gphi[a][c] = s;
    }
  }
  for (int a = 0; a < NP1; ++a) {
    P.psi[a] = o.N1[a + NP1 * q];
    for (int c = 0; c < 3; ++c) {
      double s = 0;
      for (int K = 0; K < 3; ++K) s += g.iJ[K + 3 * c] * o.dN1[a + NP1 * (K + 3 * q)];
      P.gpsi[a][c] = s;
    }
  }
  const double c1 = o.bdf2 ? 2.0 / o.dt : 1.0 / o.dt, c2 = o.bdf2 ? 0.5 / o.dt : 0.0;
  double nrm = 0;
  for (int c = 0; c < 3; ++c) {
    double un = 0, um = 0;
    for (int a = 0; a < NV; ++a) {
      un += P.phi[a] * local_value(o, o.un, o.und, id[c * NV + a]);
      um += P.phi[a] * local_value(o, o.unm1, o.unm1d, id[c * NV + a]);
    }
    P.un[c] = un;
    P.w[c] = o.bdf2 ? 2.0 * un - um : un;  // wadv (test/common.jl:186)
    P.f[c] = c1 * un - c2 * um;             // hist (:185)
    nrm += un * un;
  }
  nrm = std::sqrt(nrm);
  // τ (test/common.jl:196-198), evaluated at uⁿ and the cell size h
  P.taus = std::pow(std::pow(2 * nrm / g.h, 2) + 9 * std::pow(4 * o.mu / (o.rho * g.h * g.h), 2), -0.5);
  P.taup = P.taus / o.rho;
  P.taul = o.rho * nrm * g.h * 0.5;
  P.dV = o.w[q] * std::fabs(g.detJ);
}

// basis function k of the local dofs (0..29 velocity c*10 + n, 30..33 pressure)
Fn basis(const PointData& P, int k) {
  Fn F;
  if (k < 30) {
    const int c = k / NV, n = k % NV;
    F.u[c] = P.phi[n];
    for (int i = 0; i < 3; ++i) F.Gu[i][c] = P.gphi[n][i];  // ∂u_c/∂x_i
  } else {
    const int n = k - 30;
    F.p = P.psi[n];
    for (int i = 0; i < 3; ++i) F.gp[i] = P.gpsi[n][i];
  }
  return F;
}

// (∇u')·w = Σ_j ∂u_i/∂x_j w_j
void conv(const Fn& F, const double* w, double* out) {
  for (int i = 0; i < 3; ++i) out[i] = F.Gu[0][i] * w[0] + F.Gu[1][i] * w[1] + F.Gu[2][i] * w[2];
}

double div(const Fn& F) { return F.Gu[0][0] + F.Gu[1][1] + F.Gu[2][2]; }

// a((u,p),(v,q)) integrand at a point (test/common.jl:200-210)
double form_a(const Oseen& o, const PointData& P, const Fn& U, const Fn& Vt, double c) {
  double cu[3], cv[3], Ru[3];
  conv(U, P.w, cu);
  conv(Vt, P.w, cv);
  for (int i = 0; i < 3; ++i) Ru[i] = o.rho * c * U.u[i] + o.rho * cu[i];
  double uv = 0, eps = 0, adv = 0, supg = 0, supgp = 0, pspg = 0, pspgp = 0;
  for (int i = 0; i < 3; ++i) {
    uv += U.u[i] * Vt.u[i];
    adv += cu[i] * Vt.u[i];
    supg += cv[i] * Ru[i];
    supgp += cv[i] * U.gp[i];
    pspg += Vt.gp[i] * Ru[i];
    pspgp += Vt.gp[i] * U.gp[i];
    for (int j = 0; j < 3; ++j) {
      const double eu = 0.5 * (U.Gu[i][j] + U.Gu[j][i]), ev = 0.5 * (Vt.Gu[i][j] + Vt.Gu[j][i]);
      eps += eu * ev;
    }
  }
  return o.rho * c * uv + 2 * o.mu * eps + o.rho * adv - U.p * div(Vt) - Vt.p * div(U) + P.taus * supg +
         P.taus * supgp - P.taup * pspg - P.taup * pspgp + P.taul * div(Vt) * div(U);
}

// l((v,q)) integrand (test/common.jl:211-216); rk = ρ f + μ Δuⁿ
double form_l(const Oseen& o, const PointData& P, const Fn& Vt, const double* rk) {
  double cv[3];
  conv(Vt, P.w, cv);
  double fv = 0, s = 0, pp = 0;
  for (int i = 0; i < 3; ++i) {
    fv += P.f[i] * Vt.u[i];
    s += cv[i] * rk[i];
    pp += Vt.gp[i] * rk[i];
  }
  return o.rho * fv + P.taus * s - P.taup * pp;
}

// element matrix Ke[test + 34 trial] and load Fe[test]
void element(const Oseen& o, int cell, double* Ke, double* Fe) {
  std::fill(Ke, Ke + NDL * NDL, 0.0);
  std::fill(Fe, Fe + NDL, 0.0);
  const CellGeo g = cell_geo(o, cell);
  const int32_t* id = &o.ids[(size_t)cell * NDL];
  double lapn[3];
  for (int c = 0; c < 3; ++c) {
    double s = 0;
    for (int a = 0; a < NV; ++a) s += g.lap[a] * local_value(o, o.un, o.und, id[c * NV + a]);
    lapn[c] = s;
  }
  const double c0 = o.bdf2 ? 1.5 / o.dt : 1.0 / o.dt;
  PointData P;
  for (int q = 0; q < o.nq; ++q) {
    point_data(o, cell, g, q, P);
    double rk[3];
    for (int c = 0; c < 3; ++c) rk[c] = o.rho * P.f[c] + o.mu * lapn[c];
    Fn B[NDL];
    for (int k = 0; k < NDL; ++k) B[k] = basis(P, k);
    for (int te = 0; te < NDL; ++te) {
      Fe[te] += P.dV * form_l(o, P, B[te], rk);
      for (int tr = 0; tr < NDL; ++tr) Ke[te + NDL * tr] += P.dV * form_a(o, P, B[tr], B[te], c0);
    }
  }
}

// outlet facet f: Kf[test + 34 trial] and Ff over the velocity dofs of its cell (test/common.jl:
// -∫ρ negpart(w·n)(u·v) dΓ + ∫ ZA (u·n)(v·n) dΓ in a, -∫ Pc (v·n) dΓ in l; negpart(s) = (s - |s|)/2)
void facet_element(const Oseen& o, int f, double* Kf, double* Ff) {
  std::fill(Kf, Kf + NDL * NDL, 0.0);
  std::fill(Ff, Ff + NDL, 0.0);
  const int cell = o.fcell[f], lf = o.fface[f];
  const int32_t* id = &o.ids[(size_t)cell * NDL];
  const double* n = &o.fnormal[3 * (size_t)f];
  for (int q = 0; q < o.nqf; ++q) {
    const double* phi = &o.fN[NV * (q + o.nqf * lf)];
    double w[3];
    for (int c = 0; c < 3; ++c) {
      double u0 = 0, u1 = 0;
      for (int a = 0; a < NV; ++a) {
        u0 += phi[a] * local_value(o, o.un, o.und, id[c * NV + a]);
        u1 += phi[a] * local_value(o, o.unm1, o.unm1d, id[c * NV + a]);
      }
      w[c] = o.bdf2 ? 2.0 * u0 - u1 : u0;
    }
    const double wn = w[0] * n[0] + w[1] * n[1] + w[2] * n[2];
    const double neg = 0.5 * (wn - std::fabs(wn));
    const double dS = o.fw[q] * o.farea[f];
    for (int te = 0; te < 30; ++te) {
      double v[3] = {0, 0, 0};
      v[te / NV] = phi[te % NV];
      const double vn = v[0] * n[0] + v[1] * n[1] + v[2] * n[2];
      Ff[te] += dS * (-o.Pc * vn);
      for (int tr = 0; tr < 30; ++tr) {
        double u[3] = {0, 0, 0};
        u[tr / NV] = phi[tr % NV];
        const double un = u[0] * n[0] + u[1] * n[1] + u[2] * n[2];
        const double uv = u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
        Kf[te + NDL * tr] += dS * (-o.rho * neg * uv + o.ZA * un * vn);
      }
    }
  }
}

}  // namespace

extern "C" {

void o_oseen_set_outlet(void* h, int nf, const int32_t* cells, const int32_t* faces, const double* areas,
                        const double* normals, int nqf, const double* w, const double* N, double Pc, double ZA) {
  auto& o = *(Oseen*)h;
  o.nf = nf;
  o.nqf = nqf;
  o.fcell.assign(cells, cells + nf);
  o.fface.assign(faces, faces + nf);
  o.farea.assign(areas, areas + nf);
  o.fnormal.assign(normals, normals + 3 * (size_t)nf);
  o.fw.assign(w, w + nqf);
  o.fN.assign(N, N + (size_t)NV * nqf * 4);
  o.Pc = Pc;
  o.ZA = ZA;
}

void* o_oseen_create(int ncells, int nq, const double* w, const double* N2, const double* dN2, const double* H2,
                     const double* N1, const double* dN1, const double* coords, const int32_t* ids, int64_t nfree,
                     int64_t ndir, const double* params) {
  auto* o = new Oseen();
  o->ncells = ncells;
  o->nq = nq;
  o->nfree = nfree;
  o->ndir = ndir;
  o->w.assign(w, w + nq);
  o->N2.assign(N2, N2 + NV * nq);
  o->dN2.assign(dN2, dN2 + NV * 3 * nq);
  o->H2.assign(H2, H2 + NV * 9);
  o->N1.assign(N1, N1 + NP1 * nq);
  o->dN1.assign(dN1, dN1 + NP1 * 3 * nq);
  o->coords.assign(coords, coords + (size_t)12 * ncells);
  o->ids.assign(ids, ids + (size_t)NDL * ncells);
  o->rho = params[0];
  o->mu = params[1];
  o->dt = params[2];
  o->bdf2 = params[3] != 0;
  o->un.assign(nfree, 0.0);
  o->unm1.assign(nfree, 0.0);
  o->und.assign(ndir, 0.0);
  o->unm1d.assign(ndir, 0.0);
  // greedy colouring over the free dofs (src/coloring.jl:4-28)
  std::vector<unsigned __int128> masks(nfree + 1, 0);
  std::vector<int> color(ncells);
  int ncol = 0;
  for (int cell = 0; cell < ncells; ++cell) {
    unsigned __int128 used = 0;
    const int32_t* id = &o->ids[(size_t)cell * NDL];
    for (int j = 0; j < NDL; ++j)
      if (id[j] > 0) used |= masks[id[j]];
    int c = 0;
    while (c < 128 && ((used >> c) & 1)) ++c;
    if (c >= 128) {
      delete o;
      return nullptr;
    }
    color[cell] = c;
    for (int j = 0; j < NDL; ++j)
      if (id[j] > 0) masks[id[j]] |= (unsigned __int128)1 << c;
    ncol = std::max(ncol, c + 1);
  }
  o->colors.assign(ncol, {});
  for (int cell = 0; cell < ncells; ++cell) o->colors[color[cell]].push_back(cell);
  return o;
}

void o_oseen_free(void* h) { delete (Oseen*)h; }

void o_oseen_set_history(void* h, const double* un, const double* und, const double* unm1, const double* unm1d) {
  auto& o = *(Oseen*)h;
  o.un.assign(un, un + o.nfree);
  o.und.assign(und, und + o.ndir);
  o.unm1.assign(unm1, unm1 + o.nfree);
  o.unm1d.assign(unm1d, unm1d + o.ndir);
}

void o_oseen_element(void* h, int cell, double* Ke, double* Fe) { element(*(Oseen*)h, cell, Ke, Fe); }

int64_t o_oseen_pattern(void* h) {
  auto& o = *(Oseen*)h;
  std::vector<uint64_t> keys;
  for (int cell = 0; cell < o.ncells; ++cell) {
    const int32_t* id = &o.ids[(size_t)cell * NDL];
    for (int jj = 0; jj < NDL; ++jj)
      for (int ii = 0; ii < NDL; ++ii)
        if (id[jj] > 0 && id[ii] > 0) keys.push_back(((uint64_t)id[jj] << 32) | (uint64_t)id[ii]);
  }
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  o.colptr.assign(o.nfree + 1, 0);
  o.rowval.resize(keys.size());
  std::vector<int64_t> cnt(o.nfree + 1, 0);
  for (size_t k = 0; k < keys.size(); ++k) {
    cnt[keys[k] >> 32] += 1;
    o.rowval[k] = (int64_t)(keys[k] & 0xffffffffu);
  }
  o.colptr[0] = 1;
  for (int64_t c = 1; c <= o.nfree; ++c) o.colptr[c] = o.colptr[c - 1] + cnt[c];
  o.nzpos.assign((size_t)NDL * NDL * o.ncells, 0);
#pragma omp parallel for schedule(static)
  for (int cell = 0; cell < o.ncells; ++cell) {
    const int32_t* id = &o.ids[(size_t)cell * NDL];
    for (int jj = 0; jj < NDL; ++jj)
      for (int ii = 0; ii < NDL; ++ii) {
        if (id[jj] <= 0 || id[ii] <= 0) continue;
        const int64_t* b = o.rowval.data() + (o.colptr[id[jj] - 1] - 1);
        const int64_t* e = o.rowval.data() + (o.colptr[id[jj]] - 1);
        const int64_t* f = std::lower_bound(b, e, (int64_t)id[ii]);
        o.nzpos[(size_t)cell * NDL * NDL + ii + (size_t)NDL * jj] = (int32_t)(f - o.rowval.data() + 1);
      }
  }
  return (int64_t)keys.size();
}

void o_oseen_pattern_get(void* h, int64_t* colptr, int64_t* rowval, int32_t* nzpos) {
  auto& o = *(Oseen*)h;
  if (colptr) std::memcpy(colptr, o.colptr.data(), sizeof(int64_t) * o.colptr.size());
  if (rowval) std::memcpy(rowval, o.rowval.data(), sizeof(int64_t) * o.rowval.size());
  if (nzpos) std::memcpy(nzpos, o.nzpos.data(), sizeof(int32_t) * o.nzpos.size());
}

// residual r = a(x, ·) - l(·) at the free dofs (x: free values, dvals: Dirichlet values)
void o_oseen_residual(void* h, const double* x, const double* dvals, double* b, int nthreads) {
  auto& o = *(Oseen*)h;
  std::fill(b, b + o.nfree, 0.0);
  const int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
  for (auto& color : o.colors) {
#pragma omp parallel num_threads(nt)
    {
      std::vector<double> Ke(NDL * NDL), Fe(NDL);
#pragma omp for schedule(dynamic, 16)
      for (size_t ci = 0; ci < color.size(); ++ci) {
        const int cell = color[ci];
        element(o, cell, Ke.data(), Fe.data());
        const int32_t* id = &o.ids[(size_t)cell * NDL];
        double xl[NDL];
        for (int j = 0; j < NDL; ++j) xl[j] = id[j] > 0 ? x[id[j] - 1] : (id[j] < 0 ? dvals[-id[j] - 1] : 0.0);
        for (int i = 0; i < NDL; ++i) {
          if (id[i] <= 0) continue;
          double s = -Fe[i];
          for (int j = 0; j < NDL; ++j) s += Ke[i + NDL * j] * xl[j];
          b[id[i] - 1] += s;
        }
      }
    }
  }
  std::vector<double> Kf(NDL * NDL), Ff(NDL);
  for (int f = 0; f < o.nf; ++f) {  // outlet boundary group, serial (few facets)
    facet_element(o, f, Kf.data(), Ff.data());
    const int32_t* id = &o.ids[(size_t)o.fcell[f] * NDL];
    double xl[NDL];
    for (int j = 0; j < NDL; ++j) xl[j] = id[j] > 0 ? x[id[j] - 1] : (id[j] < 0 ? dvals[-id[j] - 1] : 0.0);
    for (int i = 0; i < NDL; ++i) {
      if (id[i] <= 0) continue;
      double s = -Ff[i];
      for (int j = 0; j < NDL; ++j) s += Kf[i + NDL * j] * xl[j];
      b[id[i] - 1] += s;
    }
  }
}

void o_oseen_jacobian(void* h, double* nzval, int nthreads) {
  auto& o = *(Oseen*)h;
  if (o.colptr.empty()) o_oseen_pattern(h);
  std::fill(nzval, nzval + o.rowval.size(), 0.0);
  const int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
  for (auto& color : o.colors) {
#pragma omp parallel num_threads(nt)
    {
      std::vector<double> Ke(NDL * NDL), Fe(NDL);
#pragma omp for schedule(dynamic, 16)
      for (size_t ci = 0; ci < color.size(); ++ci) {
        const int cell = color[ci];
        element(o, cell, Ke.data(), Fe.data());
        const int32_t* pos = &o.nzpos[(size_t)cell * NDL * NDL];
        for (int e = 0; e < NDL * NDL; ++e)
          if (pos[e] > 0) nzval[pos[e] - 1] += Ke[e];
      }
    }
  }
  std::vector<double> Kf(NDL * NDL), Ff(NDL);
  for (int f = 0; f < o.nf; ++f) {
    facet_element(o, f, Kf.data(), Ff.data());
    const int32_t* pos = &o.nzpos[(size_t)o.fcell[f] * NDL * NDL];
    for (int e = 0; e < NDL * NDL; ++e)
      if (pos[e] > 0) nzval[pos[e] - 1] += Kf[e];
  }
}

}  // extern "C"
