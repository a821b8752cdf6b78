"""Oseen–BDF step on Taylor–Hood P2–P1 tetrahedra: host side (mesh, spaces, tables, data).

Mirrors the volume part of the reference's Oseen test problem (``test/common.jl:164-228``,
``oseen_channel``): velocity P2 (3 components) and pressure P1, SUPG/PSPG/LSIC stabilisation with
the reference's τ definitions, BDF2 coefficients, the elementwise Laplacian of uⁿ in the
stabilisation right-hand side. What Gridap supplies there (the Kuhn split ``simplexify``, the
numbering, the reference bases, the quadrature) is built here: a cube of n³ hexahedra split into
6 tetrahedra each (all sharing the hexahedron's main diagonal), P2 nodes at vertices and edge
midpoints, multi-field numbering with all velocity dofs before the pressure dofs (Gridap's
consecutive ``MultiFieldFESpace`` blocks), a conical-product Gauss–Jacobi rule.

Boundary: x = 0 is the inlet (face interior, profile 16 y(1-y) z(1-z) eₓ), the four lateral faces
are walls (closed: with every box edge and vertex), x = 1 is a free outlet; the pressure is free —
the reference's tags (inlet = face 25, wall = vertices, edges and faces 21-24).
"""
from __future__ import annotations

import ctypes
import itertools

import numpy as np
import scipy.sparse as sp

from . import _lib
from ._lib import call, ptr

# local nodes of the P2 tetrahedron: 4 vertices, then the 6 edges in this order
EDGES = ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3))
NV, NP1, NQ2 = 10, 4, 34  # P2 nodes, P1 nodes, local dofs (3 * 10 + 4)


class TetMesh:
    """Unit cube of n³ hexahedra, each split into 6 tetrahedra along its main diagonal."""

    def __init__(self, n: int):
        self.n = n = int(n)
        g = np.linspace(0.0, 1.0, n + 1)
        X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
        self.vertices = np.stack([X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F")], axis=1)
        vid = lambda i, j, k: i + (n + 1) * (j + (n + 1) * k)
        ex, ey, ez = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
        ex, ey, ez = ex.ravel(order="F"), ey.ravel(order="F"), ez.ravel(order="F")
        tets = []
        for perm in itertools.permutations(range(3)):
            # path v0 -> v0 + e_perm0 -> + e_perm1 -> + e_perm2 = v7 (Kuhn simplex)
            steps = [np.zeros(3, dtype=int)]
            for a in perm:
                s = steps[-1].copy()
                s[a] = 1
                steps.append(s)
            tets.append(np.stack([vid(ex + s[0], ey + s[1], ez + s[2]) for s in steps], axis=1))
        # cells ordered hexahedron by hexahedron, 6 per hexahedron
        self.tets = np.stack(tets, axis=1).reshape(-1, 4).astype(np.int64)
        self.ncells = self.tets.shape[0]
        # (3, 4, ncells) column-major vertex coordinates
        self.coords = np.asfortranarray(self.vertices[self.tets].transpose(2, 1, 0))


# local faces of a tetrahedron: face f is opposite local vertex f
FACES = ((1, 2, 3), (0, 2, 3), (0, 1, 3), (0, 1, 2))
# reference vertices
REF_V = np.array([[0.0, 0, 0], [1.0, 0, 0], [0.0, 1, 0], [0.0, 0, 1]])


def tri_quadrature(m: int = 3):
    """Conical-product rule on the reference triangle (barycentric (s, t) in the unit simplex) with m²
    points, exact for degree 2m - 1 (m = 3: degree 5, the backflow term's measure); weights sum to 1
    (multiplied by the facet area)."""
    from scipy.special import roots_jacobi

    a, wa = roots_jacobi(m, 1, 0)
    b, wb = roots_jacobi(m, 0, 0)
    a, b = (a + 1) / 2, (b + 1) / 2
    wa, wb = wa / 4, wb / 2
    pts, ws = [], []
    for i in range(m):
        for j in range(m):
            pts.append((a[i], b[j] * (1 - a[i])))
            ws.append(wa[i] * wb[j] * 2)  # × 2: weights of the unit-area normalisation
    return np.array(pts), np.array(ws)


class OutletFacets:
    """The boundary facets of the outlet x = 1: per facet its cell, the local face, the area and the
    outward unit normal; and the P2 tables of the cell at the facet points for each local face."""

    def __init__(self, mesh: TetMesh, quad_m: int = 3):
        tets, X = mesh.tets, mesh.vertices
        on = np.isclose(X[:, 0], 1.0)
        cells, faces, areas, normals = [], [], [], []
        for f_id, (i, j, k) in enumerate(FACES):
            sel = np.nonzero(on[tets[:, i]] & on[tets[:, j]] & on[tets[:, k]])[0]
            for c in sel:
                P = X[tets[c, [i, j, k]]]
                nrm = np.cross(P[1] - P[0], P[2] - P[0])
                opp = X[tets[c, f_id]]
                if nrm @ (P[0] - opp) < 0:
                    nrm = -nrm
                cells.append(c)
                faces.append(f_id)
                areas.append(np.linalg.norm(nrm) / 2)
                normals.append(nrm / np.linalg.norm(nrm))
        order = np.argsort(cells, kind="stable")
        self.cells = np.array(cells, dtype=np.int32)[order]
        self.faces = np.array(faces, dtype=np.int32)[order]
        self.areas = np.array(areas)[order]
        self.normals = np.ascontiguousarray(np.array(normals)[order].T)  # (3, nfacets)
        self.nfacets = len(self.cells)
        st, self.w = tri_quadrature(quad_m)
        self.nq = len(self.w)
        # P2 values of the cell at the facet points, per local face: (10, nq, 4)
        N = np.zeros((NV, self.nq, 4))
        for f_id, vs in enumerate(FACES):
            V0, V1, V2 = REF_V[list(vs)]
            for q, (s_, t_) in enumerate(st):
                N[:, q, f_id] = p2_basis(V0 + s_ * (V1 - V0) + t_ * (V2 - V0))[0]
        self.N = np.asfortranarray(N)


def p2_basis(xi):
    """P2 basis values (10,) and reference gradients (10, 3) at xi (3,): vertices λ(2λ-1), edges 4λiλj."""
    lam = np.array([1.0 - xi[0] - xi[1] - xi[2], xi[0], xi[1], xi[2]])
    dlam = np.array([[-1.0, -1.0, -1.0], [1.0, 0, 0], [0, 1.0, 0], [0, 0, 1.0]])
    N = np.zeros(NV)
    dN = np.zeros((NV, 3))
    for i in range(4):
        N[i] = lam[i] * (2 * lam[i] - 1)
        dN[i] = (4 * lam[i] - 1) * dlam[i]
    for e, (i, j) in enumerate(EDGES):
        N[4 + e] = 4 * lam[i] * lam[j]
        dN[4 + e] = 4 * (lam[i] * dlam[j] + lam[j] * dlam[i])
    return N, dN


def p2_hessians():
    """Reference second derivatives of the P2 basis (constant): (10, 3, 3)."""
    dlam = np.array([[-1.0, -1.0, -1.0], [1.0, 0, 0], [0, 1.0, 0], [0, 0, 1.0]])
    H = np.zeros((NV, 3, 3))
    for i in range(4):
        H[i] = 4 * np.outer(dlam[i], dlam[i])
    for e, (i, j) in enumerate(EDGES):
        H[4 + e] = 4 * (np.outer(dlam[i], dlam[j]) + np.outer(dlam[j], dlam[i]))
    return H


def p1_basis(xi):
    N = np.array([1.0 - xi[0] - xi[1] - xi[2], xi[0], xi[1], xi[2]])
    dN = np.array([[-1.0, -1.0, -1.0], [1.0, 0, 0], [0, 1.0, 0], [0, 0, 1.0]])
    return N, dN


def tet_quadrature(m: int = 3):
    """Conical-product (Stroud) rule on the reference tetrahedron with m³ points: Gauss–Jacobi in the
    collapsed coordinates, exact for polynomials of degree 2m - 1 (m = 3: degree 5 >= the form's 4).
    Returns points (np, 3) and weights (np,) summing to 1/6."""
    from scipy.special import roots_jacobi

    a, wa = roots_jacobi(m, 2, 0)  # weight (1 - t)^2 on [-1, 1]
    b, wb = roots_jacobi(m, 1, 0)
    c, wc = roots_jacobi(m, 0, 0)
    a, b, c = (a + 1) / 2, (b + 1) / 2, (c + 1) / 2
    wa, wb, wc = wa / 8, wb / 4, wc / 2
    pts, ws = [], []
    for i in range(m):
        for j in range(m):
            for k in range(m):
                x = a[i]
                y = b[j] * (1 - a[i])
                z = c[k] * (1 - a[i]) * (1 - b[j])
                pts.append((x, y, z))
                ws.append(wa[i] * wb[j] * wc[k])
    return np.array(pts), np.array(ws)


class TaylorHoodSpace:
    """P2 velocity × P1 pressure on a ``TetMesh``, multi-field numbering (velocity block first).

    ``cell_dof_ids`` (34, ncells) Int32, local dof c*10 + n for the velocity component c at P2 node
    n, 30 + n for the pressure at vertex n; > 0 free (1-based), < 0 Dirichlet (1-based index into
    the Dirichlet values). Velocity dofs are node-major, component fastest.
    """

    def __init__(self, mesh: TetMesh):
        self.mesh = mesh
        n = mesh.n
        M = 2 * n + 1  # P2 nodes on the half-step lattice
        self.M = M
        tets = mesh.tets
        vert_ijk = np.stack([tets % (n + 1), (tets // (n + 1)) % (n + 1), tets // (n + 1) ** 2], axis=-1) * 2
        node_ijk = np.zeros((mesh.ncells, NV, 3), dtype=np.int64)
        node_ijk[:, :4] = vert_ijk
        for e, (i, j) in enumerate(EDGES):
            node_ijk[:, 4 + e] = (vert_ijk[:, i] + vert_ijk[:, j]) // 2
        gnode = node_ijk[..., 0] + M * (node_ijk[..., 1] + M * node_ijk[..., 2])  # (ncells, 10)
        self.nnodes = M ** 3
        gi, gj, gk = np.meshgrid(np.arange(M), np.arange(M), np.arange(M), indexing="ij")
        gi, gj, gk = gi.ravel(order="F"), gj.ravel(order="F"), gk.ravel(order="F")
        self.node_coords = np.stack([gi, gj, gk], axis=1) / (M - 1)
        wall = (gj == 0) | (gj == M - 1) | (gk == 0) | (gk == M - 1)
        inlet = (gi == 0) & ~wall
        fixed = wall | inlet
        dof_fixed = np.repeat(fixed, 3)
        nvel = 3 * self.nnodes
        nfree_u = int((~dof_fixed).sum())
        free_id = np.zeros(nvel, dtype=np.int64)
        dir_id = np.zeros(nvel, dtype=np.int64)
        free_id[~dof_fixed] = np.arange(1, nfree_u + 1)
        dir_id[dof_fixed] = np.arange(1, int(dof_fixed.sum()) + 1)
        gid_u = np.where(dof_fixed, -dir_id, free_id)
        # pressure: P1 on the vertices (the even lattice points), all free, after the velocity block
        self.nvert = (n + 1) ** 3
        self.nfree_u = nfree_u
        self.nfree = nfree_u + self.nvert
        self.ndir = int(dof_fixed.sum())
        ids = np.empty((mesh.ncells, NQ2), dtype=np.int64)
        for c in range(3):
            ids[:, c * NV:(c + 1) * NV] = gid_u[3 * gnode + c]
        ids[:, 30:34] = nfree_u + 1 + tets
        self.cell_dof_ids = np.asfortranarray(ids.T.astype(np.int32))
        self.cell_nodes = gnode
        # Dirichlet values: inlet profile along x, zero on the walls
        vals = np.zeros((self.nnodes, 3))
        y, z = self.node_coords[:, 1], self.node_coords[:, 2]
        vals[inlet, 0] = (16 * y * (1 - y) * z * (1 - z))[inlet]
        self.dirichlet_values = np.zeros(self.ndir)
        for c in range(3):
            m = dof_fixed[c::3]
            self.dirichlet_values[-gid_u[3 * np.nonzero(m)[0] + c] - 1] = vals[m, c]
        self.gid_u = gid_u
        self.ndof_total = nvel + self.nvert

    def interpolate_velocity(self, f):
        """Free and Dirichlet values of the P2 interpolant of the velocity f: x (m, 3) -> (m, 3)
        (the pressure entries of the free vector are 0)."""
        v = np.asarray(f(self.node_coords), dtype=float).reshape(self.nnodes, 3).ravel()
        free = np.zeros(self.nfree)
        dvals = np.zeros(self.ndir)
        g = self.gid_u
        free[g[g > 0] - 1] = v[g > 0]
        dvals[-g[g < 0] - 1] = v[g < 0]
        return free, dvals


def fourier_field(seed: int = 2, modes: int = 8, amplitude: float = 1.0, kmax: int = 2):
    """A seeded sum of ``modes`` divergence-free Fourier modes: a_m sin(2π k_m·x + φ_m) with
    a_m ⊥ k_m, |a_m| = amplitude."""
    rng = np.random.default_rng(seed)
    ks, amps, phs = [], [], []
    while len(ks) < modes:
        k = rng.integers(-kmax, kmax + 1, size=3)
        if not k.any():
            continue
        r = rng.standard_normal(3)
        a = r - (r @ k) / (k @ k) * k
        a = amplitude * a / np.linalg.norm(a)
        ks.append(k)
        amps.append(a)
        phs.append(rng.uniform(0, 2 * np.pi))
    ks, amps, phs = np.array(ks, float), np.array(amps), np.array(phs)

    def f(X):
        X = np.asarray(X, float)
        return np.sin(2 * np.pi * X @ ks.T + phs) @ amps

    return f


def tables(q_pts):
    """P2 values (10, nq), reference gradients (10, 3, nq), P1 values (4, nq) and gradients (4, 3, nq)
    at the points, column-major; P2 reference Hessians (10, 3, 3)."""
    nq = len(q_pts)
    N2 = np.zeros((NV, nq))
    dN2 = np.zeros((NV, 3, nq))
    N1 = np.zeros((NP1, nq))
    dN1 = np.zeros((NP1, 3, nq))
    for q, xi in enumerate(q_pts):
        N2[:, q], dN2[:, :, q] = p2_basis(xi)
        N1[:, q], dN1[:, :, q] = p1_basis(xi)
    return (np.asfortranarray(N2), np.asfortranarray(dN2), np.asfortranarray(N1), np.asfortranarray(dN1),
            np.asfortranarray(p2_hessians()))


class OseenParams:
    """ρ, μ, Δt and the BDF order of the step (``oseen_channel``'s c0, c1, c2)."""

    def __init__(self, rho=1.0, mu=1e-3, dt=1e-3, bdf2=True):
        self.rho, self.mu, self.dt, self.bdf2 = float(rho), float(mu), float(dt), bool(bdf2)

    def array(self):
        return np.array([self.rho, self.mu, self.dt, 1.0 if self.bdf2 else 0.0])


class OseenOperator:
    """The Oseen step as an operator over the engine (``hfk_oseen_*``): ``residual`` and the CSC
    ``jacobian`` of a(x, y) - l(y) (linear in x), with the reference's method names."""

    def __init__(self, space: TaylorHoodSpace, params: OseenParams, un, und, unm1=None, unm1d=None, quad_m: int = 3):
        self.space, self.params = space, params
        pts, w = tet_quadrature(quad_m)
        self.xq, self.w = pts, w
        N2, dN2, N1, dN1, H2 = tables(pts)
        self._keep = (N2, dN2, N1, dN1, H2)
        h = ctypes.c_void_p()
        prm = params.array()
        call("hfk_oseen_create", ctypes.byref(h), space.mesh.ncells, len(w), ptr(w), ptr(N2), ptr(dN2), ptr(H2), ptr(N1),
             ptr(dN1), ptr(space.mesh.coords), ptr(space.cell_dof_ids, np.int32), space.nfree, space.ndir, ptr(prm),
             len(prm))
        self.h = h
        self.set_history(un, und, un if unm1 is None else unm1, und if unm1d is None else unm1d)
        self._pattern = None

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            try:
                _lib.lib().hfk_oseen_destroy(h)
            except Exception:
                pass
            self.h = None

    def set_outlet(self, facets: "OutletFacets | None", Pc: float = 0.7, ZA: float = 2.3):
        """The outlet boundary group (backflow, Robin, Windkessel pressure; the reference's Pc and ZA)."""
        if facets is None:
            call("hfk_oseen_set_outlet", self.h, 0, None, None, None, None, 0, None, None, Pc, ZA)
            return
        self._outlet = facets
        call("hfk_oseen_set_outlet", self.h, facets.nfacets, ptr(facets.cells, np.int32), ptr(facets.faces, np.int32),
             ptr(np.ascontiguousarray(facets.areas)), ptr(np.asfortranarray(facets.normals)), facets.nq,
             ptr(np.ascontiguousarray(facets.w)), ptr(facets.N), Pc, ZA)

    def set_history(self, un, und, unm1, unm1d):
        """uⁿ and uⁿ⁻¹ (free and Dirichlet values of the trial space; pressure entries ignored)."""
        call("hfk_oseen_set_history", self.h, ptr(un), ptr(und), ptr(unm1), ptr(unm1d))

    def sparsity_pattern(self) -> sp.csc_matrix:
        if self._pattern is None:
            nnz = ctypes.c_int64()
            call("hfk_oseen_pattern", self.h, ctypes.byref(nnz))
            n = self.space.nfree
            colptr = np.zeros(n + 1, dtype=np.int64)
            rowval = np.zeros(nnz.value, dtype=np.int64)
            call("hfk_oseen_pattern_get", self.h, ptr(colptr, np.int64), ptr(rowval, np.int64))
            self._pattern = sp.csc_matrix((np.zeros(nnz.value), rowval - 1, colptr - 1), shape=(n, n))
        return self._pattern

    def residual(self, b, x, dvals=None):
        d = self.space.dirichlet_values if dvals is None else dvals
        call("hfk_oseen_residual", self.h, ptr(x), ptr(d), ptr(b))
        return b

    def jacobian_values(self, nzval):
        self.sparsity_pattern()
        call("hfk_oseen_jacobian", self.h, ptr(nzval))
        return nzval

    def jacobian(self):
        A = self.sparsity_pattern().copy()
        A.data = self.jacobian_values(np.zeros(A.nnz))
        return A

    def set_scatter(self, mode: str):
        m = {"auto": _lib.SCATTER_AUTO, "coloured": _lib.SCATTER_COLOURED, "atomic": _lib.SCATTER_ATOMIC}[mode]
        call("hfk_oseen_set_scatter", self.h, m)
