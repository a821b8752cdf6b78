// Oseen–BDF step on Taylor–Hood P2–P1 affine tetrahedra: fused element matrix / load vector with
// the scatter into the CSC nonzeros (Jacobian) or into the residual a(x, ·) - l(·).
//
// Volume terms of the reference's Oseen problem (test/common.jl:200-216): with velocity test
// v = φ_a e_i, trial u = φ_b e_j and pressures ψ,
//   K[(i,a),(j,b)] = δ_ij M_ab + Σ_q dV (μ ∂_jφ_a ∂_iφ_b + τl ∂_iφ_a ∂_jφ_b)
//   M_ab = Σ_q dV (ρ c0 φ_a φ_b + μ ∇φ_a·∇φ_b + ρ (w·∇φ_b) φ_a + τs (w·∇φ_a)(ρ c0 φ_b + ρ w·∇φ_b))
//   K[(i,a), p_b] = Σ_q dV (-ψ_b ∂_iφ_a + τs (w·∇φ_a) ∂_iψ_b)
//   K[q_a, (j,b)] = Σ_q dV (-ψ_a ∂_jφ_b - τp ∂_jψ_a (ρ c0 φ_b + ρ w·∇φ_b))
//   K[q_a, p_b]   = -Σ_q dV τp ∇ψ_a·∇ψ_b
//   F[(i,a)] = Σ_q dV (ρ f_i φ_a + τs (w·∇φ_a) rk_i),  F[q_a] = -Σ_q dV τp ∇ψ_a·rk,  rk = ρ f + μ Δuⁿ
// (2μ ε(u):ε(v) expands to μ δ_ij ∇φ_a·∇φ_b + μ ∂_jφ_a ∂_iφ_b), the τ of test/common.jl:196-198
// at uⁿ and h = (6√2 |K|)^(1/3), w = 2uⁿ - uⁿ⁻¹ and f = c1 uⁿ - c2 uⁿ⁻¹ under BDF2 (:183-187),
// Δuⁿ exact per cell (P2 on an affine cell). One CTA per cell: the point data are built once in
// shared memory (one thread per point). The Jacobian: one thread per basis pair, which forms every
// component entry of that pair in one pass over the points (the 9 entries of a velocity pair share
// their loads). The residual a(x, ·) - l(·) is formed matrix-free: the point values of u, ∇u, p,
// ∇p from x give per point the coefficients of φ_a, ∇φ_a and w·∇φ_a in each test row, then one
// thread per test function contracts them over the points (no element matrix).
#pragma once
#include "hfk_internal.h"
#include "kern_async.cuh"
#include "pointwise.cuh"

namespace hfk {

constexpr int OS_NV = 10, OS_NP = 4, OS_NDL = 34, OS_MAXQ = 64, OS_THREADS = 128;

struct OseenData {
  const int32_t* ids;     // (34, ncells)
  const int32_t* cells;   // list (one colour) or nullptr
  int ncells_list;
  const double* coords;   // (3, 4, ncells)
  const double* w;        // (nq)
  const double* N2;       // (10, nq)
  const double* dN2;      // (10, 3, nq)
  const double* H2;       // (10, 3, 3) reference Hessians
  const double* N1;       // (4, nq)
  const double* dN1;      // (4, 3, nq)
  const double* un;       // history, free values (trial space numbering)
  const double* und;      // history, Dirichlet values
  const double* unm1;
  const double* unm1d;
  int nq;
  double rho, mu, c0, c1, c2;
  int bdf2;
};

struct OseenIO {
  int mode;               // 0: residual into b, 1: Jacobian into nzval
  int atomic;
  const double* x;        // residual: free values
  const double* dvals;    // residual: Dirichlet values
  double* b;
  const int32_t* nzpos;   // (34*34, ncells) 1-based
  double* nzval;
};

// shared layout (doubles) for nq points
struct OseenSmem {
  int nq;
  __host__ __device__ int phi() const { return 0; }                   // [q][10]
  __host__ __device__ int gphi() const { return phi() + 10 * nq; }    // [q][10][3]
  __host__ __device__ int psi() const { return gphi() + 30 * nq; }    // [q][4]
  __host__ __device__ int wg() const { return psi() + 4 * nq; }       // [q][10]  w·∇φ
  __host__ __device__ int sup() const { return wg() + 10 * nq; }      // [q][10]  ρ c0 φ + ρ w·∇φ
  __host__ __device__ int rk() const { return sup() + 10 * nq; }      // [q][3]
  __host__ __device__ int f() const { return rk() + 3 * nq; }         // [q][3]
  __host__ __device__ int sc() const { return f() + 3 * nq; }         // [q][4]  dV, τs, τp, τl
  __host__ __device__ int cellv() const { return sc() + 4 * nq; }     // iJ 9, det, h, gpsi 12, lapn 3 (26)
  __host__ __device__ int loc() const { return cellv() + 32; }        // xl 34, unl 30, uml 30
  __host__ __device__ int rc() const { return loc() + 96; }           // [q][20] residual point coefficients
  __host__ __device__ int total() const { return rc() + 20 * nq; }
};

static __global__ void __launch_bounds__(OS_THREADS) oseen_kernel(OseenData d, OseenIO io) {
  extern __shared__ __align__(16) double osm[];
  __shared__ int32_t sid[OS_NDL];
  __shared__ __align__(16) int32_t spos[OS_NDL * OS_NDL];  // Jacobian: the cell's positions
  const OseenSmem L{d.nq};
  const int t = threadIdx.x;
  const int li = blockIdx.x;
  if (li >= d.ncells_list) return;
  const int cell = d.cells ? d.cells[li] : li;
  if (io.mode == 1) {  // the cell's 34 x 34 positions (4 624 bytes, 16-byte aligned blocks), in flight
                       // while the cell's data and point tables are computed
    const char* src = reinterpret_cast<const char*>(io.nzpos + (size_t)OS_NDL * OS_NDL * cell);
    for (int i = t; i < OS_NDL * OS_NDL * 4 / 16; i += blockDim.x) cp_async16(spos + 4 * i, src + 16 * i);
    cp_async_commit();
  }
  const int nq = d.nq;
  double* cv = osm + L.cellv();
  double* xl = osm + L.loc();
  double* unl = xl + OS_NDL;
  double* uml = unl + 30;
  // ---- gathers ----------------------------------------------------------------------------
  if (t < OS_NDL) {
    const int32_t id = d.ids[(size_t)cell * OS_NDL + t];
    sid[t] = id;
    if (io.mode == 0) xl[t] = id > 0 ? io.x[id - 1] : (id < 0 ? io.dvals[-id - 1] : 0.0);
    if (t < 30) {
      unl[t] = id > 0 ? d.un[id - 1] : (id < 0 ? d.und[-id - 1] : 0.0);
      uml[t] = id > 0 ? d.unm1[id - 1] : (id < 0 ? d.unm1d[-id - 1] : 0.0);
    }
  }
  // ---- cell geometry (affine): J[c + 3K] = x_{K+1,c} - x_{0,c}, its inverse, h -----------------
  if (t == 0) {
    const double* X = d.coords + (size_t)cell * 12;
    double J[9], iJ[9];
    for (int K = 0; K < 3; ++K)
      for (int c = 0; c < 3; ++c) J[c + 3 * K] = X[c + 3 * (K + 1)] - X[c];
    const double det = det3(J);
    inv3(J, det, iJ);  // iJ[K + 3c] = (J^-1)[K][c]
    for (int i = 0; i < 9; ++i) cv[i] = iJ[i];
    cv[9] = fabs(det);
    cv[10] = cbrt(6.0 * sqrt(2.0) * fabs(det) / 6.0);
  }
  __syncthreads();
  if (t < 12) {  // ∇ψ_a (constant): gpsi[a][c] = Σ_K dN1[a,K] (J^-1)[K][c]
    const int a = t / 3, c = t % 3;
    double s = 0;
    for (int K = 0; K < 3; ++K) s += cv[K + 3 * c] * d.dN1[a + OS_NP * (K + 0)];
    cv[11 + t] = s;
  } else if (t >= 32 && t < 35) {  // Δuⁿ_c = Σ_a uⁿ_{c,a} Σ_{K,K'} Ĥ_a[K,K'] (J^-1 J^-T)[K,K']
    const int c = t - 32;
    double G[9];
    for (int K = 0; K < 3; ++K)
      for (int Kp = 0; Kp < 3; ++Kp) G[K + 3 * Kp] = cv[K] * cv[Kp] + cv[K + 3] * cv[Kp + 3] + cv[K + 6] * cv[Kp + 6];
    double s = 0;
    for (int a = 0; a < OS_NV; ++a) {
      double la = 0;
      for (int e = 0; e < 9; ++e) la += d.H2[a + OS_NV * e] * G[e];
      s += la * unl[c * OS_NV + a];
    }
    cv[23 + c] = s;
  }
  __syncthreads();
  // ---- point data -------------------------------------------------------------------------
  // the basis values and physical gradients per (point, basis function): all threads
  for (int e = t; e < nq * OS_NV; e += blockDim.x) {
    const int q = e / OS_NV, a = e - OS_NV * q;
    osm[L.phi() + 10 * q + a] = d.N2[a + OS_NV * q];
    const double g0 = d.dN2[a + OS_NV * (3 * q)], g1 = d.dN2[a + OS_NV * (1 + 3 * q)], g2 = d.dN2[a + OS_NV * (2 + 3 * q)];
    double* gphi = osm + L.gphi() + 30 * q + a * 3;
#pragma unroll
    for (int c = 0; c < 3; ++c) gphi[c] = cv[3 * c] * g0 + cv[1 + 3 * c] * g1 + cv[2 + 3 * c] * g2;
    if (a < OS_NP) osm[L.psi() + 4 * q + a] = d.N1[a + OS_NP * q];
  }
  __syncthreads();
  for (int q = t; q < nq; q += blockDim.x) {
    double* phi = osm + L.phi() + 10 * q;
    double* gphi = osm + L.gphi() + 30 * q;
    double* psi = osm + L.psi() + 4 * q;
    double w[3], f[3], nrm = 0;
    for (int c = 0; c < 3; ++c) {
      double u0 = 0, u1 = 0;
      for (int a = 0; a < OS_NV; ++a) {
        u0 += phi[a] * unl[c * OS_NV + a];
        u1 += phi[a] * uml[c * OS_NV + a];
      }
      w[c] = d.bdf2 ? 2.0 * u0 - u1 : u0;
      f[c] = d.c1 * u0 - d.c2 * u1;
      nrm += u0 * u0;
    }
    nrm = sqrt(nrm);
    const double h = cv[10];
    const double a1 = 2.0 * nrm / h, a2 = 4.0 * d.mu / (d.rho * h * h);
    const double taus = 1.0 / sqrt(a1 * a1 + 9.0 * a2 * a2);
    double* sc = osm + L.sc() + 4 * q;
    sc[0] = d.w[q] * cv[9];
    sc[1] = taus;
    sc[2] = taus / d.rho;
    sc[3] = d.rho * nrm * h * 0.5;
    double* wg = osm + L.wg() + 10 * q;
    double* sup = osm + L.sup() + 10 * q;
    for (int a = 0; a < OS_NV; ++a) {
      wg[a] = w[0] * gphi[a * 3] + w[1] * gphi[a * 3 + 1] + w[2] * gphi[a * 3 + 2];
      sup[a] = d.rho * d.c0 * phi[a] + d.rho * wg[a];
    }
    for (int c = 0; c < 3; ++c) {
      osm[L.f() + 3 * q + c] = f[c];
      osm[L.rk() + 3 * q + c] = d.rho * f[c] + d.mu * cv[23 + c];
    }
    if (io.mode == 0) {
      // point values of x: u_i, G[k][i] = ∂_k u_i, p, ∇p (constant)
      double u[3], G[3][3], p = 0, gp[3] = {0, 0, 0};
      for (int i = 0; i < 3; ++i) {
        u[i] = 0;
        for (int k = 0; k < 3; ++k) G[k][i] = 0;
        for (int a = 0; a < OS_NV; ++a) {
          const double xa = xl[i * OS_NV + a];
          u[i] += phi[a] * xa;
          for (int k = 0; k < 3; ++k) G[k][i] += gphi[a * 3 + k] * xa;
        }
      }
      for (int a = 0; a < OS_NP; ++a) {
        const double xa = xl[30 + a];
        p += psi[a] * xa;
        for (int k = 0; k < 3; ++k) gp[k] += cv[11 + a * 3 + k] * xa;
      }
      const double divu = G[0][0] + G[1][1] + G[2][2];
      const double dV = sc[0];
      double* R = osm + L.rc() + 20 * q;
      // velocity row (i, a): Σ_q [φ_a R[i] + Σ_k ∂_kφ_a R[3 + 3i + k] + (w·∇φ_a) R[12 + i]]
      // pressure row a:     Σ_q [ψ_a R[15]] + ∇ψ_a · Σ_q R[16..18]
      for (int i = 0; i < 3; ++i) {
        const double conv = w[0] * G[0][i] + w[1] * G[1][i] + w[2] * G[2][i];  // ((∇u')·w)_i
        const double Ru = d.rho * d.c0 * u[i] + d.rho * conv;
        const double rk = osm[L.rk() + 3 * q + i];
        R[i] = dV * (d.rho * d.c0 * u[i] + d.rho * conv - d.rho * f[i]);
        for (int k = 0; k < 3; ++k)
          R[3 + 3 * i + k] = dV * (d.mu * (G[k][i] + G[i][k]) + (k == i ? sc[3] * divu - p : 0.0));
        R[12 + i] = dV * taus * (Ru + gp[i] - rk);
        R[16 + i] = -dV * sc[2] * (Ru + gp[i] - rk);
      }
      R[15] = -dV * divu;
    }
  }
  __syncthreads();
  if (io.mode == 0) {
    // ---- residual rows, scattered at the free test dofs ----------------------------------------
    if (t < OS_NDL) {
      const int32_t id = sid[t];
      double r = 0;
      if (t < 30) {
        const int i = t / OS_NV, a = t % OS_NV;
        for (int q = 0; q < nq; ++q) {
          const double* R = osm + L.rc() + 20 * q;
          const double* g = osm + L.gphi() + 30 * q + a * 3;
          r += osm[L.phi() + 10 * q + a] * R[i] + g[0] * R[3 + 3 * i] + g[1] * R[4 + 3 * i] + g[2] * R[5 + 3 * i] +
               osm[L.wg() + 10 * q + a] * R[12 + i];
        }
      } else {
        const int a = t - 30;
        double v0 = 0, v1 = 0, v2 = 0;
        for (int q = 0; q < nq; ++q) {
          const double* R = osm + L.rc() + 20 * q;
          r += osm[L.psi() + 4 * q + a] * R[15];
          v0 += R[16];
          v1 += R[17];
          v2 += R[18];
        }
        r += cv[11 + a * 3] * v0 + cv[12 + a * 3] * v1 + cv[13 + a * 3] * v2;
      }
      if (id > 0) {
        if (io.atomic) atomicAdd(&io.b[id - 1], r);
        else io.b[id - 1] += r;
      }
    }
    return;
  }
  // ---- Jacobian: one thread per basis pair --------------------------------------------------
  cp_async_wait_all();
  __syncthreads();  // every thread's pieces of the positions have arrived
  const double* gpsi = cv + 11;
  const int32_t* pos = spos;
  auto put = [&](int te, int tr, double v) {
    const int32_t ps = pos[te + OS_NDL * tr];
    if (ps > 0) {
      if (io.atomic) atomicAdd(&io.nzval[ps - 1], v);
      else io.nzval[ps - 1] += v;
    }
  };
  for (int item = t; item < 196; item += blockDim.x) {
    if (item < 100) {  // velocity pair (a, b): M_ab and the 9 component entries
      const int a = item % OS_NV, b = item / OS_NV;
      double M = 0, X[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int q = 0; q < nq; ++q) {
        const double* phi = osm + L.phi() + 10 * q;
        const double* ga = osm + L.gphi() + 30 * q + a * 3;
        const double* gb = osm + L.gphi() + 30 * q + b * 3;
        const double* sc = osm + L.sc() + 4 * q;
        const double dV = sc[0], mdv = d.mu * dV, ldv = sc[3] * dV;
        const double wga = osm[L.wg() + 10 * q + a], wgb = osm[L.wg() + 10 * q + b];
        const double gg = ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2];
        M += dV * (d.rho * d.c0 * phi[a] * phi[b] + d.mu * gg + d.rho * wgb * phi[a] +
                   sc[1] * wga * osm[L.sup() + 10 * q + b]);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) X[i][j] += mdv * ga[j] * gb[i] + ldv * ga[i] * gb[j];
      }
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) put(i * OS_NV + a, j * OS_NV + b, X[i][j] + (i == j ? M : 0.0));
    } else if (item < 140) {  // velocity test (., a), pressure trial b
      const int a = (item - 100) % OS_NV, b = (item - 100) / OS_NV;
      double V[3] = {0, 0, 0};
      for (int q = 0; q < nq; ++q) {
        const double* ga = osm + L.gphi() + 30 * q + a * 3;
        const double* sc = osm + L.sc() + 4 * q;
        const double psib = osm[L.psi() + 4 * q + b], wga = osm[L.wg() + 10 * q + a];
        for (int i = 0; i < 3; ++i) V[i] += sc[0] * (-psib * ga[i] + sc[1] * wga * gpsi[b * 3 + i]);
      }
      for (int i = 0; i < 3; ++i) put(i * OS_NV + a, 30 + b, V[i]);
    } else if (item < 180) {  // pressure test a, velocity trial (., b)
      const int b = (item - 140) % OS_NV, a = (item - 140) / OS_NV;
      double V[3] = {0, 0, 0};
      for (int q = 0; q < nq; ++q) {
        const double* gb = osm + L.gphi() + 30 * q + b * 3;
        const double* sc = osm + L.sc() + 4 * q;
        const double psia = osm[L.psi() + 4 * q + a], supb = osm[L.sup() + 10 * q + b];
        for (int j = 0; j < 3; ++j) V[j] += sc[0] * (-psia * gb[j] - sc[2] * gpsi[a * 3 + j] * supb);
      }
      for (int j = 0; j < 3; ++j) put(30 + a, j * OS_NV + b, V[j]);
    } else {  // pressure pair
      const int a = (item - 180) % OS_NP, b = (item - 180) / OS_NP;
      double s = 0;
      for (int q = 0; q < nq; ++q) s += osm[L.sc() + 4 * q] * osm[L.sc() + 4 * q + 2];
      put(30 + a, 30 + b,
          -s * (gpsi[a * 3] * gpsi[b * 3] + gpsi[a * 3 + 1] * gpsi[b * 3 + 1] + gpsi[a * 3 + 2] * gpsi[b * 3 + 2]));
    }
  }
}

// ---- the outlet boundary group (test/common.jl:194-210) ----------------------------------------
// -∫ ρ negpart(w·n)(u·v) dΓ + ∫ ZA (u·n)(v·n) dΓ in a, -∫ Pc (v·n) dΓ in l, negpart(s) = (s - |s|)/2,
// on the facets of one boundary part, each with its cell, local face, area and outward unit normal.
constexpr int OS_MAXQF = 32;

struct OutletData {
  int nf, nqf;
  const int32_t* cell;
  const int32_t* face;
  const double* area;
  const double* normal;  // (3, nf)
  const double* w;       // (nqf), sum 1
  const double* N;       // (10, nqf, 4): the cell's P2 values at the points of each local face
  double Pc, ZA;
};

static __global__ void __launch_bounds__(128) oseen_outlet_kernel(OseenData d, OutletData fd, OseenIO io) {
  __shared__ double phi[OS_MAXQF][OS_NV], c1[OS_MAXQF], c2[OS_MAXQF], dS[OS_MAXQF], uq[OS_MAXQF][3];
  __shared__ double unl[30], uml[30], xl[30];
  __shared__ int32_t sid[OS_NDL];
  const int f = blockIdx.x, t = threadIdx.x;
  if (f >= fd.nf) return;
  const int cell = fd.cell[f], lf = fd.face[f];
  const double n0 = fd.normal[3 * (size_t)f], n1 = fd.normal[3 * (size_t)f + 1], n2 = fd.normal[3 * (size_t)f + 2];
  if (t < OS_NDL) sid[t] = d.ids[(size_t)cell * OS_NDL + t];
  __syncthreads();
  if (t < 30) {
    const int32_t id = sid[t];
    unl[t] = id > 0 ? d.un[id - 1] : (id < 0 ? d.und[-id - 1] : 0.0);
    uml[t] = id > 0 ? d.unm1[id - 1] : (id < 0 ? d.unm1d[-id - 1] : 0.0);
    if (io.mode == 0) xl[t] = id > 0 ? io.x[id - 1] : (id < 0 ? io.dvals[-id - 1] : 0.0);
  }
  __syncthreads();
  for (int q = t; q < fd.nqf; q += blockDim.x) {
    double w[3], u[3];
    for (int a = 0; a < OS_NV; ++a) phi[q][a] = fd.N[a + OS_NV * (q + fd.nqf * lf)];
    for (int c = 0; c < 3; ++c) {
      double u0 = 0, u1 = 0, ux = 0;
      for (int a = 0; a < OS_NV; ++a) {
        u0 += phi[q][a] * unl[c * OS_NV + a];
        u1 += phi[q][a] * uml[c * OS_NV + a];
        if (io.mode == 0) ux += phi[q][a] * xl[c * OS_NV + a];
      }
      w[c] = d.bdf2 ? 2.0 * u0 - u1 : u0;
      u[c] = ux;
    }
    const double wn = w[0] * n0 + w[1] * n1 + w[2] * n2;
    dS[q] = fd.w[q] * fd.area[f];
    c1[q] = -d.rho * 0.5 * (wn - fabs(wn)) * dS[q];
    c2[q] = fd.ZA * dS[q];
    for (int c = 0; c < 3; ++c) uq[q][c] = u[c];
  }
  __syncthreads();
  const double nv[3] = {n0, n1, n2};
  if (io.mode == 0) {  // residual rows of the velocity test functions (i, a)
    if (t < 30) {
      const int i = t / OS_NV, a = t % OS_NV;
      double r = 0;
      for (int q = 0; q < fd.nqf; ++q) {
        const double un = uq[q][0] * n0 + uq[q][1] * n1 + uq[q][2] * n2;
        r += phi[q][a] * (c1[q] * uq[q][i] + c2[q] * un * nv[i] + dS[q] * fd.Pc * nv[i]);
      }
      const int32_t id = sid[t];
      if (id > 0) atomicAdd(&io.b[id - 1], r);
    }
    return;
  }
  if (t < OS_NV * OS_NV) {  // Jacobian: velocity pair (a, b), its 9 component entries
    const int a = t % OS_NV, b = t / OS_NV;
    double m1 = 0, m2 = 0;
    for (int q = 0; q < fd.nqf; ++q) {
      const double pp = phi[q][a] * phi[q][b];
      m1 += c1[q] * pp;
      m2 += c2[q] * pp;
    }
    const int32_t* pos = io.nzpos + (size_t)OS_NDL * OS_NDL * cell;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        const int32_t ps = pos[(i * OS_NV + a) + OS_NDL * (j * OS_NV + b)];
        if (ps > 0) atomicAdd(&io.nzval[ps - 1], (i == j ? m1 : 0.0) + nv[i] * nv[j] * m2);
      }
  }
}

}  // namespace hfk
