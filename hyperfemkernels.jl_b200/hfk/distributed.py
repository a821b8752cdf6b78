"""Domain decomposition of one problem over ranks (one process per GPU).

The reference runs on one node's threads; partitioning a mesh over GPUs is this engine's own layer
around the same per-cell kernels. Two schemes, both built on a partition of the cells
(``cell_rank``; ``slab_partition`` cuts the mesh into layers of cells along z):

* **halo sum-exchange** (matrix-free products, residuals, block-Jacobi CG): every rank runs the cell
  kernels over its own cells into a local vector over the free dofs those cells touch; the dofs a
  rank shares with a neighbour then hold a partial sum, completed by ONE exchange with each
  neighbour (send the partial values of the shared dofs, add what arrives). Dot products count each
  dof once (on its owner, the lowest rank whose cells touch it) and are all-reduced.
* **owner computes** (assembly): every rank also takes the cells of its neighbours that touch a dof
  it owns (ghost cells), so the residual entries and the Jacobian rows of its owned dofs are
  complete without any exchange; the state on the ghost cells' dofs comes from their owners
  (``Halo.sync_``).

Communication goes through a ``comm`` object with ``exchange(sends)`` (point-to-point, one buffer per
neighbour, both directions) and ``allreduce_(tensor, op)``; ``TorchComm`` implements it with
``torch.distributed`` (NCCL between GPUs, gloo on CPU). Vectors are torch tensors (CUDA on the GPU
path); the per-cell work is the engine's kernels through a local ``KernelOperator``.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import call, ptr

_CUDA_STREAM_LEGACY = 1  # cudaStreamLegacy


def slab_partition(mesh, world: int) -> np.ndarray:
    """Rank of every cell when the mesh is cut into ``world`` layers of cells along z (balanced: the
    layer counts differ by at most one). Cells are numbered x fastest, so each rank's cells are one
    contiguous range and a rank touches at most two neighbours."""
    nz = mesh.n[2]
    if not 1 <= world <= nz:
        raise ValueError(f"HyperFEMKernels: cannot cut {nz} cell layers into {world} slabs")
    k = mesh.cell_ijk[:, 2]
    return ((k * world) // nz).astype(np.int32)


class _SubMesh:
    """The cells of a subdomain, as the kernels see a mesh (count and vertex coordinates)."""

    def __init__(self, mesh, cells):
        self.n = None
        self.ncells = len(cells)
        self.coords = np.asfortranarray(mesh.coords[:, :, cells])
        self.cell_ijk = mesh.cell_ijk[cells]


class SubSpace:
    """A subdomain's view of a ``VectorLagrangeSpace``: the same element, its cells only, free dofs
    numbered locally (1-based, in increasing global order), Dirichlet ids and values kept global."""

    def __init__(self, space, cells, free_global):
        self.parent = space
        self.order, self.Q, self.nn, self.nc, self.ndl = space.order, space.Q, space.nn, space.nc, space.ndl
        self.mesh = _SubMesh(space.mesh, cells)
        gid = space.cell_dof_ids[:, cells]
        loc = gid.astype(np.int64)
        pos = gid > 0
        loc[pos] = np.searchsorted(free_global, gid[pos].astype(np.int64) - 1) + 1
        self.cell_dof_ids = np.asfortranarray(loc.astype(np.int32))
        self.nfree = len(free_global)
        self.ndir = space.ndir
        self.dirichlet_values = space.dirichlet_values

    def tables(self, quad):
        return self.parent.tables(quad)


class Subdomain:
    """Rank ``rank``'s part of ``space`` under the cell partition ``cell_rank`` (rank per cell).

    ``ghost=False``: the rank's own cells (halo sum-exchange). ``ghost=True``: its own cells and every
    other cell that touches a dof it owns (owner computes).

    Attributes: ``cells`` (global cell indices), ``space`` (a ``SubSpace``), ``free_global`` (global
    0-based free index of every local dof), ``owned`` (bool per local dof), ``shared`` (per neighbour
    rank the local indices of the dofs both touch, in increasing global order: both sides list the
    same dofs in the same order), ``peer_owns`` (per neighbour, which of those it owns).
    """

    def __init__(self, space, cell_rank, rank: int, ghost: bool = False):
        cell_rank = np.asarray(cell_rank, dtype=np.int32)
        if cell_rank.shape != (space.mesh.ncells,):
            raise ValueError("HyperFEMKernels: cell_rank needs one rank per cell")
        self.world = world = int(cell_rank.max()) + 1
        if not 0 <= rank < world:
            raise ValueError(f"HyperFEMKernels: rank {rank} outside the partition's {world} ranks")
        self.rank, self.ghost = rank, ghost
        ids = space.cell_dof_ids
        nfree = space.nfree
        # per rank the free dofs its own cells touch; the owner of a dof is the lowest such rank
        touched = []
        for s in range(world):
            t = np.zeros(nfree, dtype=bool)
            g = ids[:, cell_rank == s]
            t[g[g > 0].astype(np.int64) - 1] = True
            touched.append(t)
        owner = np.full(nfree, world, dtype=np.int32)
        for s in range(world):
            owner[touched[s] & (owner == world)] = s
        if (owner == world).any():
            raise ValueError("HyperFEMKernels: a free dof is touched by no cell")
        self.owner_of = owner
        # Dirichlet dofs: the same rule (lowest rank whose cells reference them), for gathers
        downer = np.full(space.ndir, world, dtype=np.int32)
        for s in range(world):
            g = ids[:, cell_rank == s]
            t = np.zeros(space.ndir, dtype=bool)
            t[-g[g < 0].astype(np.int64) - 1] = True
            downer[t & (downer == world)] = s
        self.dir_owned = downer == rank
        if ghost:
            mine = owner == rank
            sel = ids > 0
            hit = np.zeros(ids.shape, dtype=bool)
            hit[sel] = mine[ids[sel].astype(np.int64) - 1]
            cells = np.nonzero(hit.any(axis=0) | (cell_rank == rank))[0]
            # what each rank holds in this scheme (its cells with their ghosts)
            holds = []
            for s in range(world):
                own_s = owner == s
                h = np.zeros(ids.shape, dtype=bool)
                h[sel] = own_s[ids[sel].astype(np.int64) - 1]
                cs = h.any(axis=0) | (cell_rank == s)
                t = np.zeros(nfree, dtype=bool)
                g = ids[:, cs]
                t[g[g > 0].astype(np.int64) - 1] = True
                holds.append(t)
        else:
            cells = np.nonzero(cell_rank == rank)[0]
            holds = touched
        self.cells = cells
        self.free_global = np.nonzero(holds[rank])[0].astype(np.int64)
        self.space = SubSpace(space, cells, self.free_global)
        self.owned = owner[self.free_global] == rank
        self.shared, self.peer_owns = {}, {}
        for s in range(world):
            if s == rank:
                continue
            both = np.nonzero(holds[rank] & holds[s])[0]
            if len(both):
                self.shared[s] = np.searchsorted(self.free_global, both)
                self.peer_owns[s] = owner[both] == s

    @property
    def nfree(self) -> int:
        return len(self.free_global)

    def restrict(self, x_global):
        """The local part of a global free-dof vector (numpy or torch)."""
        if isinstance(x_global, torch.Tensor):
            return x_global[torch.as_tensor(self.free_global, device=x_global.device)].contiguous()
        return np.ascontiguousarray(np.asarray(x_global)[self.free_global])

    def owned_global(self) -> np.ndarray:
        """Global 0-based free indices of the dofs this rank owns."""
        return self.free_global[self.owned]


class TorchComm:
    """Point-to-point exchange and all-reduce over a ``torch.distributed`` process group. Buffers live
    on ``device`` (the GPU for NCCL, the CPU for gloo); tensors on another device are moved."""

    def __init__(self, group=None, device=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
                else torch.device("cpu")
        self.device = torch.device(device)

    def exchange(self, sends: dict) -> dict:
        """Send ``sends[peer]`` to every peer and receive a buffer of the same shape from it."""
        dist = self.dist
        if not sends:
            return {}
        sends = {s: t.to(self.device).contiguous() for s, t in sends.items()}
        recvs = {s: torch.empty_like(t) for s, t in sends.items()}
        ops = []
        for s in sorted(sends):
            ops.append(dist.P2POp(dist.isend, sends[s], s, self.group))
            ops.append(dist.P2POp(dist.irecv, recvs[s], s, self.group))
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        return recvs

    def allreduce_(self, t: torch.Tensor, op: str = "sum") -> torch.Tensor:
        dist = self.dist
        red = {"sum": dist.ReduceOp.SUM, "min": dist.ReduceOp.MIN, "max": dist.ReduceOp.MAX}[op]
        buf = t.to(self.device)
        dist.all_reduce(buf, op=red, group=self.group)
        if buf is not t:
            t.copy_(buf)
        return t


class Halo:
    """The exchanges of one subdomain: sum of the shared dofs' partial values, owners' values to the
    copies, sum of shared nodal blocks, and owned-dof inner products."""

    def __init__(self, sub: Subdomain, comm):
        self.sub, self.comm = sub, comm
        self.peers = sorted(sub.shared)
        self._idx = {}
        self._w = {}

    def _index(self, device):
        key = str(device)
        if key not in self._idx:
            self._idx[key] = {s: torch.as_tensor(self.sub.shared[s], dtype=torch.int64, device=device)
                              for s in self.peers}
            self._idx[key + "own"] = {s: torch.as_tensor(self.sub.shared[s][self.sub.peer_owns[s]], dtype=torch.int64,
                                                         device=device) for s in self.peers}
            self._idx[key + "ownpos"] = {s: torch.as_tensor(np.nonzero(self.sub.peer_owns[s])[0], dtype=torch.int64,
                                                            device=device) for s in self.peers}
        return self._idx[key], self._idx[key + "own"], self._idx[key + "ownpos"]

    def sum_(self, y: torch.Tensor) -> torch.Tensor:
        """Complete the partial values of the shared dofs: every neighbour's partial sum is added (one
        exchange with each neighbour). With two ranks per shared dof (slabs) both copies end bitwise
        equal."""
        if not self.peers:
            return y
        idx, _, _ = self._index(y.device)
        recvs = self.comm.exchange({s: y.index_select(0, idx[s]) for s in self.peers})
        for s in self.peers:
            y.index_add_(0, idx[s], recvs[s].to(y.device))
        return y

    def sync_(self, x: torch.Tensor) -> torch.Tensor:
        """Give every copy of a shared dof its owner's value (one exchange with each neighbour)."""
        if not self.peers:
            return x
        idx, own, ownpos = self._index(x.device)
        recvs = self.comm.exchange({s: x.index_select(0, idx[s]) for s in self.peers})
        for s in self.peers:
            if len(own[s]):
                x.index_copy_(0, own[s], recvs[s].to(x.device).index_select(0, ownpos[s]))
        return x

    def sum_blocks(self, dofs: np.ndarray, B: torch.Tensor) -> torch.Tensor:
        """Sum the nodal blocks ``B`` (nblocks x 9) of the nodes shared with neighbours; ``dofs``
        (nblocks x 3) are the blocks' local 1-based dofs (0 = fixed component)."""
        if not self.peers:
            return B
        key = "blocks"
        if key not in self._w:
            first = np.where(dofs[:, 0] > 0, dofs[:, 0], np.where(dofs[:, 1] > 0, dofs[:, 1], dofs[:, 2]))
            glob = self.sub.free_global[first.astype(np.int64) - 1]
            per = {}
            for s in self.peers:
                shared_glob = self.sub.free_global[self.sub.shared[s]]
                hit = np.isin(glob, shared_glob)
                blk = np.nonzero(hit)[0]
                per[s] = blk[np.argsort(glob[blk], kind="stable")]
            self._w[key] = per
        per = self._w[key]
        idx = {s: torch.as_tensor(per[s], dtype=torch.int64, device=B.device) for s in self.peers}
        recvs = self.comm.exchange({s: B.index_select(0, idx[s]) for s in self.peers})
        for s in self.peers:
            B.index_add_(0, idx[s], recvs[s].to(B.device))
        return B

    def weights(self, device, dtype=torch.float64) -> torch.Tensor:
        key = (str(device), dtype)
        if key not in self._w:
            self._w[key] = torch.as_tensor(self.sub.owned, device=device).to(dtype)
        return self._w[key]

    def dots(self, pairs) -> list:
        """Global inner products of (a, b) pairs of consistent local vectors, one all-reduce."""
        w = self.weights(pairs[0][0].device, pairs[0][0].dtype)
        local = torch.stack([torch.dot(w * a, b) for a, b in pairs])
        self.comm.allreduce_(local, "sum")
        return [float(v) for v in local.cpu()]


class DistributedJacobian:
    """The matrix-free Jacobian of a partitioned problem (halo sum-exchange).

    ``mf`` is the ``MatrixFreeJacobian`` of a ``KernelOperator`` over ``sub.space`` (the engine's
    product); ``apply`` may replace it with any local product ``apply(y, dx)``. ``mul`` is the local
    product over the rank's cells followed by the halo sum, so its output is the global product's
    local part on every local dof.
    """

    def __init__(self, sub: Subdomain, comm, mf=None, apply=None):
        if (mf is None) == (apply is None):
            raise ValueError("HyperFEMKernels: give exactly one of mf and apply")
        self.sub, self.comm = sub, comm
        self.halo = Halo(sub, comm)
        self.mf = mf
        self._apply = apply
        if mf is not None and torch.cuda.is_available():
            # the engine's launches on torch's current stream, so that they are ordered with the
            # exchange's torch and NCCL work and with the other levels' launches; torch's default
            # stream is the legacy default stream (handle 0), passed as cudaStreamLegacy (handle 1)
            # because handle 0 selects the problem's own stream
            s = torch.cuda.current_stream().cuda_stream
            mf.op.problem.set_stream(s if s else _CUDA_STREAM_LEGACY)

    @property
    def nfree(self) -> int:
        return self.sub.nfree

    def prepare(self, x_local, dvals=None):
        """``prepare!`` at the local part of the (consistent) state."""
        if self.mf is None:
            raise RuntimeError("HyperFEMKernels: prepare needs the engine's MatrixFreeJacobian")
        self.mf.prepare(x_local, dvals)
        return self

    def mul(self, y: torch.Tensor, dx: torch.Tensor) -> torch.Tensor:
        if self.mf is not None:
            self.mf.mul(y, dx)
        else:
            self._apply(y, dx)
        return self.halo.sum_(y)

    def dot(self, a, b) -> float:
        return self.halo.dots([(a, b)])[0]


class DistributedBlockJacobi:
    """``BlockJacobi`` of a partitioned problem: every rank extracts the nodal blocks of its cells with
    the engine's kernels, the blocks of shared nodes are summed over the neighbours, and the engine
    inverts and applies them (``hfk_blocks_set``, ``hfk_blocks_apply``)."""

    def __init__(self, A: DistributedJacobian):
        if A.mf is None:
            raise ValueError("HyperFEMKernels: the block-Jacobi needs the engine's MatrixFreeJacobian")
        self.A = A
        self.ok = False
        self._dofs = None

    def update(self):
        h = self.A.mf.op.problem.h
        ok = ctypes.c_int()
        call("hfk_blocks_update", h, ctypes.byref(ok))
        nb = ctypes.c_int()
        call("hfk_blocks_get", h, ctypes.byref(nb), None, None, None)
        dofs = np.zeros(3 * nb.value, dtype=np.int32)
        B = np.zeros(9 * nb.value)
        call("hfk_blocks_get", h, ctypes.byref(nb), ptr(dofs, np.int32), ptr(B), None)
        self._dofs = dofs.reshape(nb.value, 3)
        Bt = torch.from_numpy(B.reshape(nb.value, 9))
        Bt = self.A.halo.sum_blocks(self._dofs, Bt)
        Bs = np.ascontiguousarray(Bt.cpu().numpy()).ravel()
        call("hfk_blocks_set", h, ptr(Bs), ctypes.byref(ok))
        flag = torch.tensor([float(ok.value)], dtype=torch.float64)
        self.A.comm.allreduce_(flag, "min")
        self.ok = bool(flag.item() > 0)
        return self

    def ldiv(self, y, r):
        call("hfk_blocks_apply", self.A.mf.op.problem.h, ptr(r), ptr(y))
        return y


def cg(A, b: torch.Tensor, prec=None, rtol: float = 1e-8, atol: float = 0.0, maxiter: int = 500, x0=None):
    """Preconditioned flexible CG over a partitioned problem: the engine's (or any) ``A.mul`` with its
    halo sum, ``prec(z, r)`` local (a block-Jacobi is, once its shared blocks are summed), and two
    all-reduces per iteration (p·Ap; then r·r, z·r and z·r_old together). Stops on
    ||r|| <= atol + rtol ||b|| like ``MatrixFreeSolver``'s CG (``src/solvers.jl:128-148``).
    Returns (x, iterations, converged, relative residual)."""
    halo = A.halo
    x = torch.zeros_like(b) if x0 is None else x0.clone()
    r = b.clone()
    if x0 is not None:
        Ax = torch.empty_like(b)
        A.mul(Ax, x)
        r -= Ax
    nb2, rr = halo.dots([(b, b), (r, r)])
    nb = nb2 ** 0.5
    tol = atol + rtol * nb
    if rr ** 0.5 <= tol:
        return x, 0, True, rr ** 0.5 / max(nb, 1e-300)
    z = torch.empty_like(b)
    if prec is not None:
        prec(z, r)
    else:
        z.copy_(r)
    p = z.clone()
    rz = halo.dots([(r, z)])[0]
    Ap = torch.empty_like(b)
    it = 0
    while it < maxiter:
        it += 1
        A.mul(Ap, p)
        pAp = halo.dots([(p, Ap)])[0]
        if not pAp > 0:
            return x, it, False, float("nan")
        alpha = rz / pAp
        x.add_(p, alpha=alpha)
        rn = r - alpha * Ap
        if prec is not None:
            prec(z, rn)
        else:
            z.copy_(rn)
        rr, rzn, zr_old = halo.dots([(rn, rn), (rn, z), (z, r)])
        if rr ** 0.5 <= tol:
            return x, it, True, rr ** 0.5 / nb
        beta = (rzn - zr_old) / rz
        p.mul_(beta).add_(z)
        r, rz = rn, rzn
    return x, it, False, rr ** 0.5 / nb


class OwnerAssembly:
    """Residual entries and Jacobian rows of the dofs a rank owns (owner computes: no exchange after the
    state is synchronised). ``op`` is a ``KernelOperator`` over ``sub.space`` of a ``ghost=True``
    subdomain."""

    def __init__(self, sub: Subdomain, op, comm=None):
        if not sub.ghost:
            raise ValueError("HyperFEMKernels: owner-computes assembly needs a subdomain with ghost cells")
        self.sub, self.op = sub, op
        self.halo = Halo(sub, comm) if comm is not None else None

    def residual(self, x_local):
        """(global free indices, values) of the owned residual entries."""
        b = np.zeros(self.sub.nfree)
        self.op.residual(b, np.ascontiguousarray(x_local, dtype=np.float64))
        return self.sub.owned_global(), b[self.sub.owned]

    def jacobian_rows(self, x_local):
        """The owned rows of the Jacobian as a CSR matrix (owned rows in increasing global order x all
        global free columns)."""
        import scipy.sparse as sp

        A = self.op.allocate_jacobian()
        self.op.jacobian(A, np.ascontiguousarray(x_local, dtype=np.float64))
        rows = A.tocsr()[np.nonzero(self.sub.owned)[0]]
        coo = rows.tocoo()
        nglob = self.sub.space.parent.nfree
        return sp.csr_matrix((coo.data, (coo.row, self.sub.free_global[coo.col])),
                             shape=(rows.shape[0], nglob))


def _global_multiplicity(space) -> np.ndarray:
    """Cells containing every free dof of ``space`` over the whole mesh (``cells_of``,
    ``src/transfers.jl:124-127``)."""
    ids = space.cell_dof_ids
    return np.bincount(ids[ids > 0].astype(np.int64) - 1, minlength=space.nfree).astype(np.int32)


class DistributedPMultigrid:
    """``PMultigrid`` (``src/pmultigrid.jl:256-338``) over a partitioned mesh.

    Every level is partitioned like the finest (the same ``cell_rank``), so a level's subdomain holds
    the same cells on every level and the transfers stay cell-local: prolongation of a consistent
    coarse vector is consistent as it is; the restriction divides by the multiplicity over the whole
    mesh (``hfk_transfer_set_multiplicity``) and its partial coarse sums are completed by the coarse
    level's halo sum. The smoothers are the reference's Chebyshev–block-Jacobi (``src/smoothers.jl:
    42-146``) over the halo-summed products and summed nodal blocks, with the Arnoldi estimate's inner
    products all-reduced and its start vector evaluated at the global dof numbers (the estimate of the
    single-domain problem). The coarsest level is solved directly (``coarse="cholesky"``: every rank
    holds the whole coarse level, assembled and factorised by the engine, and gathers the coarse
    right-hand side from the owners with one all-reduce) or by ``coarse_iters`` distributed
    block-Jacobi CG steps (``"cg"``: a variable preconditioner, use the flexible ``cg``).

    ``A`` is the finest level's ``DistributedJacobian``; ``spaces`` the global trial spaces of the
    coarser levels, finest first excluded.
    """

    def __init__(self, A: DistributedJacobian, spaces, cell_rank, smoother=None, coarse: str = "cholesky",
                 coarse_iters: int = 20):
        from .operator import KernelOperator, MatrixFreeJacobian
        from .solvers import Chebyshev, Prolongation

        if A.mf is None:
            raise ValueError("HyperFEMKernels: the p-multigrid needs the engine's MatrixFreeJacobian")
        if coarse not in ("cholesky", "cg"):
            raise ValueError("HyperFEMKernels: coarse must be 'cholesky' or 'cg'")
        if coarse_iters < 1:
            raise ValueError("HyperFEMKernels: coarse_iters must be ≥ 1")
        self.coarse = coarse
        self.smoother = smoother if smoother is not None else Chebyshev()
        if self.smoother.eig_inner != "euclidean":
            raise ValueError("HyperFEMKernels: the partitioned p-multigrid runs the Euclidean Arnoldi estimate")
        self.coarse_iters = int(coarse_iters)
        op = A.mf.op
        self.A = [A]
        for U in spaces:
            sub = Subdomain(U, cell_rank, A.sub.rank)
            lop = KernelOperator(op.res, op.jac, sub.space, jacobian="matrixfree")
            self.A.append(DistributedJacobian(sub, A.comm, mf=MatrixFreeJacobian(lop)))
        self.P = []
        for l in range(len(self.A) - 1):
            lf, lc = self.A[l], self.A[l + 1]
            t = Prolongation(lc.mf.op.problem, lf.mf.op.problem)
            glob = lf.sub.space.parent
            m = np.ascontiguousarray(_global_multiplicity(glob)[lf.sub.free_global])
            call("hfk_transfer_set_multiplicity", t.h, ptr(m, np.int32))
            self.P.append(t)
        self.blocks = [DistributedBlockJacobi(a) for a in self.A]
        self.bounds = [None] * (len(self.A) - 1)
        self.ok = False
        self._gmf = self._slot = None
        if coarse == "cholesky":
            # the whole coarse level on every rank: assembled and factorised by the engine's
            # LaggedAssembled slot (rebuilt at every update, as the reference's LU)
            gop = KernelOperator(op.res, op.jac, spaces[-1], jacobian="matrixfree")
            self._gmf = MatrixFreeJacobian(gop)
            if torch.cuda.is_available():
                s = torch.cuda.current_stream().cuda_stream
                gop.problem.set_stream(s if s else _CUDA_STREAM_LEGACY)
            c = self.A[-1].sub
            self._own_loc = np.nonzero(c.owned)[0]
            self._own_glob = c.owned_global()

    @property
    def levels(self) -> int:
        return len(self.A)

    def update(self):
        """``update_levels!`` + the smoothers' updates (``src/pmultigrid.jl:168-221``) at the state the
        finest level was prepared at."""
        fine = self.A[0].mf
        dev = torch.device("cuda", torch.cuda.current_device())
        x = fine.x if isinstance(fine.x, torch.Tensor) else torch.from_numpy(np.asarray(fine.x)).to(dev)
        d = fine.dvals if isinstance(fine.dvals, torch.Tensor) else torch.from_numpy(np.asarray(fine.dvals)).to(dev)
        for l, P in enumerate(self.P):
            c = self.A[l + 1]
            xc = torch.zeros(c.sub.nfree, dtype=torch.float64, device=dev)
            dc = torch.zeros(c.sub.space.ndir, dtype=torch.float64, device=dev)
            P.inject(xc, dc, x, d)
            c.prepare(xc, dc)
            x, d = xc, dc
        ok = True
        blocks = self.blocks if self.coarse == "cg" else self.blocks[:-1]
        for b in blocks:
            ok &= b.update().ok
        if self.coarse == "cholesky":
            from .solvers import LaggedAssembled, SlotState

            c = self.A[-1]
            xg = self._gather(x)
            dg = d * torch.as_tensor(c.sub.dir_owned, device=d.device).to(d.dtype)
            c.comm.allreduce_(dg, "sum")
            self._gmf.prepare(xg, dg)
            if self._slot is None:
                self._slot = SlotState(LaggedAssembled(every=1), self._gmf)
            else:
                self._slot.update(self._gmf)
            flag = torch.tensor([1.0 if self._slot.ok else 0.0], dtype=torch.float64)
            c.comm.allreduce_(flag, "min")
            ok &= bool(flag.item() > 0)
        for l in range(len(self.A) - 1):
            lo, hi = self._eig_bounds(l)
            self.bounds[l] = (lo, hi)
            ok &= bool(np.isfinite(hi) and hi > 0 and lo > 0)
        self.ok = ok
        return self

    def _eig_bounds(self, l: int):
        """Ritz bounds of J P⁻¹ after ``eig_iters`` Arnoldi steps (``src/preconditioners.jl:350-389``):
        classical Gram–Schmidt with one reorthogonalisation, each pass one all-reduce."""
        from .solvers import hessenberg_eigvals

        A, prec = self.A[l], self.blocks[l]
        k = min(self.smoother.eig_iters, A.sub.space.parent.nfree)
        dev = torch.device("cuda", torch.cuda.current_device())
        i = torch.from_numpy(A.sub.free_global.astype(np.float64) + 1.0).to(dev)
        v0 = torch.sin(1.0 + 0.7 * i) + 0.3 * torch.cos(2.3 * i)
        v0 /= A.halo.dots([(v0, v0)])[0] ** 0.5
        V = [v0]
        H = np.zeros((k + 1, k))
        z = torch.empty_like(v0)
        for j in range(k):
            prec.ldiv(z, V[j])
            w = torch.empty_like(v0)
            A.mul(w, z)
            for _ in range(2):
                h = A.halo.dots([(V[i], w) for i in range(j + 1)])
                for i in range(j + 1):
                    w.add_(V[i], alpha=-h[i])
                    H[i, j] += h[i]
            H[j + 1, j] = A.halo.dots([(w, w)])[0] ** 0.5
            if H[j + 1, j] == 0:
                break
            V.append(w / H[j + 1, j])
        jj = k
        for i in range(1, k):
            if abs(H[i, i - 1]) <= 1e-8 * max(1.0, np.max(np.abs(H[:i, :i]))):
                jj = i
                break
        ev = hessenberg_eigvals(np.asfortranarray(H[:jj, :jj])).real
        return float(ev.min()), float(ev.max())

    def _smooth(self, l: int, x, rhs, zero_guess: bool, want_residual: bool):
        """``smooth!`` (``src/smoothers.jl:116-146``) on level ``l``."""
        A, prec, c = self.A[l], self.blocks[l], self.smoother
        b = c.inflate * self.bounds[l][1]
        a = b / c.range
        th, de = (b + a) / 2, (b - a) / 2
        sg = th / de
        tmp = torch.empty_like(rhs)
        if zero_guess:
            x = torch.zeros_like(rhs)
            r = rhs.clone()
        else:
            A.mul(tmp, x)
            r = rhs - tmp
        z = torch.empty_like(rhs)
        prec.ldiv(z, r)
        rho = 1 / sg
        d = z / th
        for it in range(1, c.degree + 1):
            x.add_(d)
            if it == c.degree and not want_residual:
                break
            A.mul(tmp, d)
            r.sub_(tmp)
            if it == c.degree:
                break
            prec.ldiv(z, r)
            rn = 1 / (2 * sg - rho)
            d.mul_(rn * rho).add_(z, alpha=2 * rn / de)
            rho = rn
        return x, (r if want_residual else None)

    def _gather(self, v):
        """The whole coarse-level vector on every rank from the owners' entries (one all-reduce)."""
        c = self.A[-1]
        key = str(v.device)
        if getattr(self, "_gidx", (None,))[0] != key:
            self._gidx = (key, torch.as_tensor(self._own_loc, device=v.device),
                          torch.as_tensor(self._own_glob, device=v.device),
                          torch.as_tensor(c.sub.free_global, device=v.device))
        _, loc, glob, _ = self._gidx
        g = torch.zeros(c.sub.space.parent.nfree, dtype=v.dtype, device=v.device)
        g.index_copy_(0, glob, v.index_select(0, loc))
        c.comm.allreduce_(g, "sum")
        return g

    def _coarse(self, b):
        """The coarse solve: the replicated Cholesky on the gathered right-hand side, or
        ``coarse_iters`` block-Jacobi CG steps from zero (α and β 0 where their denominator is not
        positive)."""
        if self.coarse == "cholesky":
            bg = self._gather(b)
            yg = torch.zeros_like(bg)
            self._slot.ldiv(yg, bg)
            return yg.index_select(0, self._gidx[3])
        A, prec = self.A[-1], self.blocks[-1]
        x = torch.zeros_like(b)
        r = b.clone()
        z = torch.empty_like(b)
        prec.ldiv(z, r)
        p = z.clone()
        q = torch.empty_like(b)
        rz = A.halo.dots([(r, z)])[0]
        for it in range(self.coarse_iters):
            A.mul(q, p)
            pq = A.halo.dots([(p, q)])[0]
            a = rz / pq if pq > 0 else 0.0
            x.add_(p, alpha=a)
            r.add_(q, alpha=-a)
            if it + 1 == self.coarse_iters:
                break
            prec.ldiv(z, r)
            zr = A.halo.dots([(z, r)])[0]
            beta = zr / rz if rz > 0 else 0.0
            rz = zr
            p.mul_(beta).add_(z)
        return x

    def _vcycle(self, b, l: int):
        if l == len(self.A) - 1:
            return self._coarse(b)
        P, coarse = self.P[l], self.A[l + 1]
        x, r = self._smooth(l, None, b, zero_guess=True, want_residual=True)
        bc = torch.zeros(coarse.sub.nfree, dtype=b.dtype, device=b.device)
        P.restrict(bc, r)
        coarse.halo.sum_(bc)
        xc = self._vcycle(bc, l + 1)
        t = torch.empty_like(b)
        P.prolongate(t, xc)
        x.add_(t)
        x, _ = self._smooth(l, x, b, zero_guess=False, want_residual=False)
        return x

    def ldiv(self, y, r):
        """``ldiv!(y, PMultigridState, r)``: one V-cycle; NaN when the update failed
        (``src/pmultigrid.jl:331-335``)."""
        if not self.ok:
            y.fill_(float("nan"))
            return y
        y.copy_(self._vcycle(r, 0))
        return y


def newton_solve(A: DistributedJacobian, prec, g_full, loads, x0=None, *, rtol: float = 1e-8, atol: float = 0.0,
                 maxiter: int = 500, rtol_newton: float = 1e-8, atol_newton: float = 1e-12, max_newton: int = 20,
                 lift=None):
    """The load-stepped Newton loop of ``hfk.newton.newton_solve`` (HyperFEMKernels
    ``test/solvers/test_pmultigrid.jl:86-115``) over a partitioned problem.

    ``A`` is the finest level's ``DistributedJacobian`` (its ``KernelOperator`` computes the local
    residuals), ``prec`` a ``DistributedPMultigrid`` over ``A`` (or None). Per Newton iteration: the
    local residual completed by the halo sum, its norm all-reduced, ``prepare`` at the state, the
    preconditioner's update, then the flexible ``cg`` to ``atol + rtol ||b||``. ``g_full`` (global
    Dirichlet values at load factor 1), ``x0`` and ``lift`` are global vectors; the result is the
    rank's local part of the solution and the ``NewtonStats`` (the same on every rank).
    """
    import time

    from .newton import NewtonStats

    sub = A.sub
    op = A.mf.op
    dev = torch.device("cuda", torch.cuda.current_device())
    x = torch.zeros(sub.nfree, dtype=torch.float64, device=dev) if x0 is None else \
        torch.from_numpy(sub.restrict(np.asarray(x0, dtype=np.float64))).to(dev)
    b = torch.zeros(sub.nfree, dtype=torch.float64, device=dev)
    lift_l = None if lift is None else torch.from_numpy(sub.restrict(np.asarray(lift, dtype=np.float64))).to(dev)
    g_full = np.ascontiguousarray(g_full, dtype=np.float64)
    st = NewtonStats()
    prev = 0.0
    t0 = time.perf_counter()
    for lam in loads:
        dv = torch.from_numpy(lam * g_full).to(dev)
        if lift_l is not None:
            x.add_(lift_l, alpha=lam - prev)
        prev = lam
        st.load_steps += 1
        r0 = None
        for _ in range(max_newton):
            op.residual(b, x, dv)
            A.halo.sum_(b)
            rn = A.halo.dots([(b, b)])[0] ** 0.5
            st.residual_norms.append(rn)
            if r0 is None:
                r0 = rn
            if rn <= max(rtol_newton * r0, atol_newton):
                break
            A.prepare(x, dv)
            if prec is not None:
                prec.update()
            dx, its, conv, _ = cg(A, -b, prec.ldiv if prec is not None else None, rtol=rtol, atol=atol,
                                  maxiter=maxiter)
            st.krylov_iters.append(its)
            if not conv:
                st.converged = False
                break
            x.add_(dx)
            st.newton_iters += 1
        else:
            st.converged = False
        if not st.converged:
            break
    torch.cuda.synchronize()
    st.seconds = time.perf_counter() - t0
    return x, st
