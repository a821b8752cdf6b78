"""Host-side finite-element spaces on Cartesian hexahedral meshes.

This module produces the arrays that the reference obtains from Gridap and hands to its kernels:

* cell -> dof ids as a dense ``ndl x ncells`` Int32 matrix, negative entries = Dirichlet dofs
  (the convention of ``cell_dof_matrix``, HyperFEMKernels ``src/tables.jl:329-342``), with the
  dofs of one component consecutive inside a cell (``ldof[n, c] = c*nn + n``, the CONTIG layout
  of ``FieldTable``, ``src/tables.jl:181-182``);
* reference tables ``Nt`` (nn x np) and ``dNt`` (nn x D x np) of the scalar nodal shape functions
  at the quadrature points (``FieldTable``, ``src/tables.jl:171-237``) and the geometry tables
  (``GeoTable``, ``src/tables.jl:42-106``): the Q1 map gradients ``dMt`` (ng x D x np), the
  weights and the vertex coordinates per cell;
* the 1D basis ``lagrange1d`` on [0, 1] with equispaced nodes (``src/tensorproduct.jl:24-47``).

Gridap itself is not available here, so the numbering is this module's own (lexicographic nodes,
x fastest; free dofs numbered node-major, component fastest). Everything downstream consumes the
ids and never re-derives them, so any other numbering (Gridap's) goes through the same code.
"""
from __future__ import annotations

import dataclasses
from typing import Callable, Sequence

import numpy as np


def lagrange1d(Q: int, xi: float):
    """Values and derivatives of the 1D Lagrange basis with Q equispaced nodes on [0, 1] at xi.

    Restates ``lagrange1d`` (HyperFEMKernels ``src/tensorproduct.jl:24-47``): Q == 1 is the
    constant on node 0.5; the derivative is the sum over the omitted factor.
    """
    xs = np.array([0.5]) if Q == 1 else np.linspace(0.0, 1.0, Q)
    N = np.zeros(Q)
    dN = np.zeros(Q)
    for i in range(Q):
        v = 1.0
        for j in range(Q):
            if j != i:
                v *= (xi - xs[j]) / (xs[i] - xs[j])
        N[i] = v
        d = 0.0
        for m in range(Q):
            if m == i:
                continue
            t = 1.0 / (xs[i] - xs[m])
            for j in range(Q):
                if j != i and j != m:
                    t *= (xi - xs[j]) / (xs[i] - xs[j])
            d += t
        dN[i] = d
    return N, dN


def gauss1d(P: int):
    """P-point Gauss-Legendre rule on [0, 1] (points ascending, weights summing to 1)."""
    x, w = np.polynomial.legendre.leggauss(P)
    return 0.5 * (x + 1.0), 0.5 * w


def points_for_degree(degree: int) -> int:
    """Gauss points per direction that integrate polynomials of ``degree`` exactly (Gridap's rule)."""
    return max(1, (degree + 2) // 2)


@dataclasses.dataclass
class Quadrature:
    """Tensor-product Gauss quadrature on the reference cube [0, 1]^3 (point index a + P*(b + P*c))."""

    P: int
    xq: np.ndarray  # 3 x np (column-major)
    w: np.ndarray  # np

    @classmethod
    def gauss(cls, degree: int) -> "Quadrature":
        P = points_for_degree(degree)
        x1, w1 = gauss1d(P)
        a, b, c = np.meshgrid(np.arange(P), np.arange(P), np.arange(P), indexing="ij")
        a, b, c = a.ravel(order="F"), b.ravel(order="F"), c.ravel(order="F")
        xq = np.stack([x1[a], x1[b], x1[c]], axis=1)
        w = w1[a] * w1[b] * w1[c]
        # xq as (D, np) column-major: the memory layout of a vector of Points
        return cls(P, np.asfortranarray(xq.T), np.ascontiguousarray(w))

    @property
    def np(self) -> int:
        return len(self.w)

    def points(self) -> np.ndarray:
        """Points as an (np, 3) array, one row per point."""
        return np.ascontiguousarray(self.xq.T)


def lagrange_tables(Q: int, xq: np.ndarray):
    """ND tables of the Q^3-node Lagrange element at the points ``xq`` (np x 3, row per point).

    Node index n = i + Q*(j + Q*k). Returns (Nt, dNt): Nt[n, q] and dNt[n, K, q] (reference
    gradients), the layout of ``FieldTable.Nt``/``dNt`` (``src/tables.jl:176-178``).
    """
    npt = xq.shape[0]
    nn = Q ** 3
    Nt = np.zeros((nn, npt))
    dNt = np.zeros((nn, 3, npt))
    for q in range(npt):
        v = [lagrange1d(Q, xq[q, d]) for d in range(3)]
        for k in range(Q):
            for j in range(Q):
                for i in range(Q):
                    n = i + Q * (j + Q * k)
                    Nt[n, q] = v[0][0][i] * v[1][0][j] * v[2][0][k]
                    dNt[n, 0, q] = v[0][1][i] * v[1][0][j] * v[2][0][k]
                    dNt[n, 1, q] = v[0][0][i] * v[1][1][j] * v[2][0][k]
                    dNt[n, 2, q] = v[0][0][i] * v[1][0][j] * v[2][1][k]
    return np.asfortranarray(Nt), np.asfortranarray(dNt)


FACES = ("x0", "x1", "y0", "y1", "z0", "z1")


@dataclasses.dataclass
class CartesianMesh:
    """Structured hexahedral mesh of the box ``domain`` with ``n = (nx, ny, nz)`` cells.

    Cells are numbered x fastest (Gridap's ``CartesianDiscreteModel`` order); each cell is the
    image of [0,1]^3 under its trilinear (Q1) map with vertices ordered a + 2b + 4c.
    ``perturb`` moves interior vertices by a seeded random fraction of the cell size, which
    makes the cells non-affine (used to test the per-point geometry path).
    """

    n: tuple
    domain: tuple = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    perturb: float = 0.0
    seed: int = 0

    def __post_init__(self):
        self.n = tuple(int(v) for v in self.n)
        nx, ny, nz = self.n
        x0, x1, y0, y1, z0, z1 = self.domain
        gx = np.linspace(x0, x1, nx + 1)
        gy = np.linspace(y0, y1, ny + 1)
        gz = np.linspace(z0, z1, nz + 1)
        X, Y, Z = np.meshgrid(gx, gy, gz, indexing="ij")
        verts = np.stack([X, Y, Z], axis=-1)  # (nx+1, ny+1, nz+1, 3)
        if self.perturb > 0:
            rng = np.random.default_rng(self.seed)
            h = np.array([(x1 - x0) / nx, (y1 - y0) / ny, (z1 - z0) / nz])
            d = rng.uniform(-1, 1, verts.shape) * h * self.perturb
            d[0, :, :, 0] = d[-1, :, :, 0] = 0
            d[:, 0, :, 1] = d[:, -1, :, 1] = 0
            d[:, :, 0, 2] = d[:, :, -1, 2] = 0
            verts = verts + d
        self.vertices = verts
        ex, ey, ez = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
        ex, ey, ez = ex.ravel(order="F"), ey.ravel(order="F"), ez.ravel(order="F")
        self.cell_ijk = np.stack([ex, ey, ez], axis=1)
        coords = np.empty((self.ncells, 8, 3))
        for v in range(8):
            a, b, c = v & 1, (v >> 1) & 1, (v >> 2) & 1
            coords[:, v, :] = verts[ex + a, ey + b, ez + c]
        self.vertex_coords = coords  # ncells x 8 x 3
        # (D, ng, ncells) column-major: the memory layout of ``GeoTable.coords`` (ng x ncells VectorValue{D})
        self.coords = np.asfortranarray(coords.transpose(2, 1, 0))

    @property
    def ncells(self) -> int:
        return self.n[0] * self.n[1] * self.n[2]

    def map_point(self, cell: int, xi: np.ndarray) -> np.ndarray:
        """Physical point of reference point xi (3,) in ``cell`` (trilinear map)."""
        N, _ = q1_shape(xi)
        return N @ self.vertex_coords[cell]


def q1_shape(xi: np.ndarray):
    """Trilinear shape functions (8,) and reference gradients (8, 3) at xi (vertex a + 2b + 4c)."""
    N = np.zeros(8)
    dN = np.zeros((8, 3))
    for v in range(8):
        a, b, c = v & 1, (v >> 1) & 1, (v >> 2) & 1
        fx = xi[0] if a else 1 - xi[0]
        fy = xi[1] if b else 1 - xi[1]
        fz = xi[2] if c else 1 - xi[2]
        gx = 1.0 if a else -1.0
        gy = 1.0 if b else -1.0
        gz = 1.0 if c else -1.0
        N[v] = fx * fy * fz
        dN[v] = (gx * fy * fz, fx * gy * fz, fx * fy * gz)
    return N, dN


def geometry_tables(xq: np.ndarray):
    """Q1 geometry reference gradients dMt[v, K, q] (8 x 3 x np), ``GeoTable.dM`` transposed."""
    npt = xq.shape[0]
    dMt = np.zeros((8, 3, npt))
    for q in range(npt):
        dMt[:, :, q] = q1_shape(xq[q])[1]
    return np.asfortranarray(dMt)


class VectorLagrangeSpace:
    """Vector-valued (3 components) Lagrangian space of order ``order`` on a ``CartesianMesh``.

    ``dirichlet`` lists the closed faces ("x0", "x1", ...; "boundary" = all six) on which every
    component is fixed; a face includes its edges and vertices (the closed Dirichlet set that
    the p-multigrid transfers need, HyperFEMKernels ``src/transfers.jl:188-207``).
    ``open_faces=True`` fixes only the faces' interiors, as Gridap's face tags do (the assembly
    benchmark's setting, ``test/solvers/test_transfers.jl:10-12``).
    ``g`` gives the Dirichlet values: a callable x (m x 3) -> (m x 3), or one callable per face
    in ``dirichlet`` order (later faces win on shared edges).
    """

    def __init__(self, mesh: CartesianMesh, order: int, dirichlet: Sequence[str] = ("x0", "x1"),
                 g=None, open_faces: bool = False):
        self.mesh = mesh
        self.order = p = int(order)
        self.Q = p + 1
        self.nn = self.Q ** 3
        self.nc = 3
        self.ndl = self.nn * self.nc
        nx, ny, nz = mesh.n
        self.NX, self.NY, self.NZ = p * nx + 1, p * ny + 1, p * nz + 1
        nnodes = self.NX * self.NY * self.NZ
        self.nnodes = nnodes
        if isinstance(dirichlet, str):
            dirichlet = FACES if dirichlet == "boundary" else (dirichlet,)
        self.dirichlet_faces = tuple(dirichlet)
        gi, gj, gk = np.meshgrid(np.arange(self.NX), np.arange(self.NY), np.arange(self.NZ), indexing="ij")
        gi, gj, gk = gi.ravel(order="F"), gj.ravel(order="F"), gk.ravel(order="F")
        self.node_lattice = np.stack([gi, gj, gk], axis=1)
        fixed = np.zeros(nnodes, dtype=bool)
        face_of = np.full(nnodes, -1)
        sel = {"x0": gi == 0, "x1": gi == self.NX - 1, "y0": gj == 0, "y1": gj == self.NY - 1,
               "z0": gk == 0, "z1": gk == self.NZ - 1}
        if open_faces:
            # Gridap's face tags: the interior of the face, without its edges and vertices
            inner = {"x": (gj > 0) & (gj < self.NY - 1) & (gk > 0) & (gk < self.NZ - 1),
                     "y": (gi > 0) & (gi < self.NX - 1) & (gk > 0) & (gk < self.NZ - 1),
                     "z": (gi > 0) & (gi < self.NX - 1) & (gj > 0) & (gj < self.NY - 1)}
            sel = {f: m & inner[f[0]] for f, m in sel.items()}
        for f_idx, f in enumerate(self.dirichlet_faces):
            if f not in sel:
                raise ValueError(f"HyperFEMKernels: unknown face {f!r}")
            fixed |= sel[f]
            face_of[sel[f]] = f_idx
        self.node_fixed = fixed
        self.node_face = face_of
        # dof numbering: node-major, component fastest; free and Dirichlet numbered separately
        dof_fixed = np.repeat(fixed, 3)
        free_id = np.zeros(3 * nnodes, dtype=np.int64)
        dir_id = np.zeros(3 * nnodes, dtype=np.int64)
        free_id[~dof_fixed] = np.arange(1, int((~dof_fixed).sum()) + 1)
        dir_id[dof_fixed] = np.arange(1, int(dof_fixed.sum()) + 1)
        gid = np.where(dof_fixed, -dir_id, free_id)  # signed id per global dof
        self.dof_signed = gid
        self.nfree = int((~dof_fixed).sum())
        self.ndir = int(dof_fixed.sum())
        # cell -> dof ids (ndl x ncells), ldof = c*nn + n, n = i + Q*(j + Q*k)
        Q = self.Q
        ijk = mesh.cell_ijk
        li, lj, lk = np.meshgrid(np.arange(Q), np.arange(Q), np.arange(Q), indexing="ij")
        li, lj, lk = li.ravel(order="F"), lj.ravel(order="F"), lk.ravel(order="F")
        gnode = ((ijk[:, 0:1] * p + li[None, :])
                 + self.NX * ((ijk[:, 1:2] * p + lj[None, :]) + self.NY * (ijk[:, 2:3] * p + lk[None, :])))
        self.cell_nodes = gnode  # ncells x nn
        ids = np.empty((mesh.ncells, 3, self.nn), dtype=np.int64)
        for c in range(3):
            ids[:, c, :] = gid[3 * gnode + c]
        # (ndl, ncells) column-major Int32: the memory layout of ``cell_dof_matrix``
        self.cell_dof_ids = np.asfortranarray(ids.reshape(mesh.ncells, self.ndl).T.astype(np.int32))
        # physical coordinates of the nodes
        self.node_coords = self._node_coordinates()
        self.g = g
        self.dirichlet_values = self.interpolate_dirichlet(g)

    # -- helpers ---------------------------------------------------------------------------
    def _node_coordinates(self) -> np.ndarray:
        """Physical coordinates of every global node (through the cell maps)."""
        m = self.mesh
        Q, p = self.Q, self.order
        xs = np.array([0.5]) if Q == 1 else np.linspace(0.0, 1.0, Q)
        out = np.zeros((self.nnodes, 3))
        li, lj, lk = np.meshgrid(np.arange(Q), np.arange(Q), np.arange(Q), indexing="ij")
        li, lj, lk = li.ravel(order="F"), lj.ravel(order="F"), lk.ravel(order="F")
        Nq = np.stack([q1_shape(np.array([xs[a], xs[b], xs[c]]))[0] for a, b, c in zip(li, lj, lk)])  # nn x 8
        X = np.einsum("nv,cvd->cnd", Nq, m.vertex_coords)  # ncells x nn x 3
        out[self.cell_nodes.ravel()] = X.reshape(-1, 3)
        return out

    def interpolate_dirichlet(self, g) -> np.ndarray:
        """Dirichlet values (ndir,) from ``g`` (see the class docstring); zeros when ``g`` is None."""
        vals = np.zeros(self.ndir)
        if g is None or self.ndir == 0:
            return vals
        fixed_nodes = np.nonzero(self.node_fixed)[0]
        x = self.node_coords[fixed_nodes]
        if callable(g):
            v = np.asarray(g(x), dtype=float).reshape(len(fixed_nodes), 3)
        else:
            v = np.zeros((len(fixed_nodes), 3))
            faces = self.node_face[fixed_nodes]
            for f_idx, gf in enumerate(g):
                sel = faces == f_idx
                if sel.any():
                    v[sel] = np.asarray(gf(x[sel]), dtype=float).reshape(int(sel.sum()), 3)
        for c in range(3):
            ids = -self.dof_signed[3 * fixed_nodes + c]
            vals[ids - 1] = v[:, c]
        return vals

    def interpolate(self, f: Callable) -> tuple:
        """Free and Dirichlet values of the nodal interpolation of f: x (m x 3) -> (m x 3)."""
        v = np.asarray(f(self.node_coords), dtype=float).reshape(self.nnodes, 3)
        flat = v.ravel()
        free = np.zeros(self.nfree)
        dvals = np.zeros(self.ndir)
        gid = self.dof_signed
        free[gid[gid > 0] - 1] = flat[gid > 0]
        dvals[-gid[gid < 0] - 1] = flat[gid < 0]
        return free, dvals

    def tables(self, quad: Quadrature):
        """(Nt, dNt) of this space at the points of ``quad``."""
        return lagrange_tables(self.Q, quad.points())


def transfer_matrices(Qf: int, Qc: int):
    """Embedding E (nf x nc) and nodal interpolation Einj (nc x nf) between nested Q elements.

    E[f, c] = coarse shape function c at fine node f; Einj[c, f] = fine shape function f at
    coarse node c (``TransferField``, HyperFEMKernels ``src/transfers.jl:57-97``), with entries
    within 1e-7 of 0 or 1 snapped (``src/transfers.jl:95-96``).
    """
    def nodes(Q):
        xs = np.array([0.5]) if Q == 1 else np.linspace(0.0, 1.0, Q)
        a, b, c = np.meshgrid(np.arange(Q), np.arange(Q), np.arange(Q), indexing="ij")
        return np.stack([xs[a.ravel(order="F")], xs[b.ravel(order="F")], xs[c.ravel(order="F")]], axis=1)

    fine_nodes, coarse_nodes = nodes(Qf), nodes(Qc)
    Ncf, _ = lagrange_tables(Qc, fine_nodes)  # nc x nf_points
    Nfc, _ = lagrange_tables(Qf, coarse_nodes)  # nf x nc_points
    E = np.asfortranarray(Ncf.T)
    Einj = np.asfortranarray(Nfc.T)

    def snap(a):
        a = np.array(a, order="F")
        a[np.abs(a) < 1e-7] = 0.0
        a[np.abs(a - 1.0) < 1e-7] = 1.0
        return a

    return snap(E), snap(Einj)
