"""Domain decomposition (``hfk.distributed``): partition properties, the halo sum-exchange product, the
block-Jacobi CG and the owner-computes assembly.

CPU tests run the ranks as gloo processes (world size 2) with the oracle as the local product; GPU
tests run two ranks as host threads on one GPU with the engine's kernels (only the host waits: the
threads exchange buffers through queues, no kernel waits on another) and compare with the
single-domain engine."""
import os
import queue
import socket
import threading

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from conftest import svk_space, svk_state as _state


# ---------------------------------------------------------------------------------------------------
# partition (host only)


@pytest.mark.parametrize("ghost", [False, True])
def test_subdomains_partition_properties(ghost):
    from hfk.distributed import Subdomain, slab_partition

    space = svk_space((3, 2, 6))
    world = 3
    cr = slab_partition(space.mesh, world)
    assert sorted(np.bincount(cr)) == [12, 12, 12]
    subs = [Subdomain(space, cr, r, ghost=ghost) for r in range(world)]
    # every free dof owned exactly once, every cell taken (ghosts may repeat cells)
    owned = np.concatenate([s.owned_global() for s in subs])
    assert np.array_equal(np.sort(owned), np.arange(space.nfree))
    assert set(np.concatenate([s.cells for s in subs]).tolist()) == set(range(space.mesh.ncells))
    if not ghost:
        assert sum(len(s.cells) for s in subs) == space.mesh.ncells
    for s in subs:
        # local ids map back to the global ids of the same cells
        loc = s.space.cell_dof_ids.astype(np.int64)
        glob = space.cell_dof_ids[:, s.cells].astype(np.int64)
        pos = loc > 0
        assert np.array_equal(s.free_global[loc[pos] - 1] + 1, glob[pos])
        assert np.array_equal(loc[~pos], glob[~pos])
        assert np.all(np.diff(s.free_global) > 0)
        for p, idx in s.shared.items():  # both sides list the same dofs in the same order
            other = subs[p]
            assert np.array_equal(s.free_global[idx], other.free_global[other.shared[s.rank]])
            assert np.array_equal(s.peer_owns[p], space_owner(subs, s.free_global[idx]) == p)
    # slabs: each rank has one or two neighbours
    assert [sorted(s.shared) for s in subs] == [[1], [0, 2], [1]]
    # every Dirichlet dof has exactly one owner, among the ranks whose cells reference it
    downed = np.stack([s.dir_owned for s in subs])
    assert np.array_equal(downed.sum(axis=0), np.ones(space.ndir))
    for s in subs:
        ids = s.space.cell_dof_ids
        refd = np.unique(-ids[ids < 0].astype(np.int64) - 1)
        assert set(np.nonzero(s.dir_owned)[0]) <= set(refd.tolist())


def test_whole_mesh_multiplicity_counts_cells_per_dof():
    """The restriction's multiplicity on a subdomain is the whole mesh's: the cells of every rank that
    contain the dof (a Q2 vertex dof inside the mesh lies in 8 cells, an edge midpoint in 4, a face
    midpoint in 2, a cell centre in 1)."""
    from hfk.distributed import Subdomain, _global_multiplicity, slab_partition

    space = svk_space((3, 3, 4), faces=("x0",))
    mult = _global_multiplicity(space)
    assert mult.shape == (space.nfree,) and mult.min() >= 1 and mult.max() == 8
    assert sorted(set(mult.tolist())) == [1, 2, 4, 8]
    cr = slab_partition(space.mesh, 2)
    for r in range(2):
        sub = Subdomain(space, cr, r)
        ids = sub.space.cell_dof_ids
        local = np.bincount(ids[ids > 0].astype(np.int64) - 1, minlength=sub.nfree)
        whole = mult[sub.free_global]
        assert np.all(whole >= local)
        # interface dofs see fewer cells locally than on the whole mesh, interior ones the same
        shared = np.zeros(sub.nfree, dtype=bool)
        for idx in sub.shared.values():
            shared[idx] = True
        assert np.all(whole[~shared] == local[~shared]) and np.all(whole[shared] > local[shared])


def space_owner(subs, glob):
    return subs[0].owner_of[glob]


def test_ghost_cells_complete_owned_rows():
    """Owner computes: every cell that touches an owned dof is held by the owner."""
    from hfk.distributed import Subdomain, slab_partition

    space = svk_space((2, 3, 5))
    cr = slab_partition(space.mesh, 2)
    for r in range(2):
        s = Subdomain(space, cr, r, ghost=True)
        mine = set(s.owned_global().tolist())
        ids = space.cell_dof_ids
        need = {c for c in range(space.mesh.ncells) if any(int(i) - 1 in mine for i in ids[:, c] if i > 0)}
        assert need <= set(s.cells.tolist())


def test_slab_partition_rejects_more_ranks_than_layers():
    from hfk.distributed import slab_partition

    space = svk_space((2, 2, 2))
    with pytest.raises(ValueError, match="HyperFEMKernels"):
        slab_partition(space.mesh, 3)


# ---------------------------------------------------------------------------------------------------
# gloo ranks on CPU, the oracle as each rank's local product


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _spawn(target, world, *args):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, q) + args) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return sorted(res, key=lambda t: t[0])


class _OracleBlocks:
    """Block-Jacobi from the oracle's local blocks, summed over the neighbours with the halo."""

    def __init__(self, orc, halo):
        import torch

        dofs, B, _ = orc.blocks()
        flat = torch.from_numpy(np.ascontiguousarray(B.transpose(0, 2, 1).reshape(-1, 9)))
        flat = halo.sum_blocks(dofs, flat).numpy()
        M = flat.reshape(-1, 3, 3).transpose(0, 2, 1).copy()
        for i in range(3):
            for j in range(3):
                fixed = (dofs[:, i] == 0) | (dofs[:, j] == 0)
                M[fixed, i, j] = 1.0 if i == j else 0.0
        self.Minv = np.linalg.inv(M)
        self.dofs = dofs

    def __call__(self, z, r):
        import torch

        rn = r.numpy()
        out = np.zeros_like(rn)
        d = self.dofs.astype(np.int64) - 1
        v = np.where(d >= 0, rn[np.maximum(d, 0)], 0.0)
        y = np.einsum("bij,bj->bi", self.Minv, v)
        for i in range(3):
            sel = d[:, i] >= 0
            out[d[sel, i]] = y[sel, i]
        z.copy_(torch.from_numpy(out))
        return z


def _dd_rank(rank, world, port, out):
    import torch
    import torch.distributed as dist

    import oracle as O
    from hfk.distributed import DistributedJacobian, Subdomain, TorchComm, cg, slab_partition
    from hfk.fespace import Quadrature

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        space = svk_space((2, 3, 4))
        quad = Quadrature.gauss(4)
        x = _state(space)
        d = space.dirichlet_values
        sub = Subdomain(space, slab_partition(space.mesh, world), rank)
        orc = O.OracleProblem(sub.space, quad)
        orc.mf_prepare(sub.restrict(x), d)
        comm = TorchComm()

        def apply(y, dx):
            y.copy_(torch.from_numpy(orc.mf_apply(dx.numpy())))
            return y

        A = DistributedJacobian(sub, comm, apply=apply)
        dx = np.random.default_rng(1).standard_normal(space.nfree)
        y = torch.zeros(sub.nfree, dtype=torch.float64)
        A.mul(y, torch.from_numpy(sub.restrict(dx)))
        # residual with the same halo sum
        res = torch.from_numpy(orc.residual(sub.restrict(x), d))
        A.halo.sum_(res)
        prec = _OracleBlocks(orc, A.halo)
        b = torch.from_numpy(sub.restrict(np.random.default_rng(2).standard_normal(space.nfree)))
        xs, it, conv, rel = cg(A, b, prec, rtol=1e-10, maxiter=400)
        # owners' values to the copies
        v = torch.from_numpy(sub.restrict(np.arange(space.nfree, dtype=np.float64)))
        v[~torch.from_numpy(sub.owned)] = -1.0
        A.halo.sync_(v)
        dist.barrier()
        out.put((rank, sub.free_global, y.numpy(), res.numpy(), xs.numpy(), it, conv, v.numpy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_product_residual_cg(world):
    # world 3: the middle slab exchanges with both neighbours in one batch of sends and receives
    import torch

    import oracle as O
    from hfk.distributed import DistributedJacobian, Subdomain, cg, slab_partition
    from hfk.fespace import Quadrature

    res = _spawn(_dd_rank, world)
    assert len(res) == world
    space = svk_space((2, 3, 4))
    quad = Quadrature.gauss(4)
    x = _state(space)
    d = space.dirichlet_values
    g = O.OracleProblem(space, quad)
    g.mf_prepare(x, d)
    dx = np.random.default_rng(1).standard_normal(space.nfree)
    y = g.mf_apply(dx)
    r = g.residual(x, d)
    b = np.random.default_rng(2).standard_normal(space.nfree)
    xd = spla.spsolve(g.jacobian(x, d).tocsc(), b)
    # the same CG on one rank (no neighbours) for the iteration count
    sub1 = Subdomain(space, slab_partition(space.mesh, 1), 0)

    class _NoComm:
        def exchange(self, sends):
            return {}

        def allreduce_(self, t, op="sum"):
            return t

    A1 = DistributedJacobian(sub1, _NoComm(), apply=lambda yy, v: yy.copy_(torch.from_numpy(g.mf_apply(v.numpy()))))
    _, it1, conv1, _ = cg(A1, torch.from_numpy(b), _OracleBlocks(g, A1.halo), rtol=1e-10, maxiter=400)
    assert conv1
    for rank, fg, yl, rl, xl, it, conv, v in res:
        assert np.linalg.norm(yl - y[fg]) <= 1e-12 * np.linalg.norm(y[fg])
        assert np.linalg.norm(rl - r[fg]) <= 1e-12 * np.linalg.norm(r[fg]) + 1e-16
        assert conv and abs(it - it1) <= 2
        assert np.linalg.norm(xl - xd[fg]) <= 1e-7 * np.linalg.norm(xd[fg])
        assert np.array_equal(v, fg.astype(np.float64))  # every copy holds its owner's value
    # neighbouring slabs' copies of an interface dof agree bitwise after the halo sum (two ranks per dof)
    for (_, f0, y0, *_), (_, f1, y1, *_) in zip(res[:-1], res[1:]):
        common, i0, i1 = np.intersect1d(f0, f1, return_indices=True)
        assert len(common) > 0 and np.array_equal(y0[i0], y1[i1])


class _OracleOp:
    """The oracle with ``KernelOperator``'s residual/jacobian interface (for the owner assembly)."""

    def __init__(self, space, quad):
        import oracle as O

        self.orc = O.OracleProblem(space, quad)
        self.d = space.dirichlet_values

    def residual(self, b, x):
        b[:] = self.orc.residual(x, self.d)
        return b

    def allocate_jacobian(self):
        import scipy.sparse as sp

        colptr, rowval = self.orc.pattern()
        n = self.orc.nfree
        return sp.csc_matrix((np.zeros(len(rowval)), rowval - 1, colptr - 1), shape=(n, n))

    def jacobian(self, A, x):
        A.data[:] = self.orc.jacobian_values(x, self.d)
        return A


def test_owner_assembly_rows_equal_global():
    import scipy.sparse as sp

    import oracle as O
    from hfk.distributed import OwnerAssembly, Subdomain, slab_partition
    from hfk.fespace import Quadrature

    space = svk_space((2, 2, 6))
    quad = Quadrature.gauss(4)
    x = _state(space)
    g = O.OracleProblem(space, quad)
    J = g.jacobian(x, space.dirichlet_values).tocsr()
    r = g.residual(x, space.dirichlet_values)
    cr = slab_partition(space.mesh, 3)
    rows, blocks, rvals = [], [], []
    for rank in range(3):
        sub = Subdomain(space, cr, rank, ghost=True)
        asm = OwnerAssembly(sub, _OracleOp(sub.space, quad))
        gi, rv = asm.residual(sub.restrict(x))
        rows.append(gi)
        rvals.append(rv)
        blocks.append(asm.jacobian_rows(sub.restrict(x)))
    order = np.concatenate(rows)
    assert np.array_equal(np.sort(order), np.arange(space.nfree))
    rr = np.zeros(space.nfree)
    rr[order] = np.concatenate(rvals)
    assert np.linalg.norm(rr - r) <= 1e-12 * np.linalg.norm(r)
    Jd = sp.vstack(blocks).tocsr()
    perm = sp.csr_matrix((np.ones(space.nfree), (order, np.arange(space.nfree))), shape=(space.nfree, space.nfree))
    D = (perm @ Jd - J)
    assert abs(D).max() <= 1e-12 * abs(J).max()


# ---------------------------------------------------------------------------------------------------
# GPU: two ranks as host threads on one GPU, the engine's kernels


class ThreadComm:
    """An in-process stand-in for a two-or-more-rank process group whose ranks are host threads.
    Buffers pass through queues; all CUDA work stays ordered on the device's default stream."""

    def __init__(self, world):
        self.world = world
        self.q = {(a, b): queue.Queue() for a in range(world) for b in range(world)}
        self.slots = [None] * world
        self.bar = threading.Barrier(world)

    def rank(self, r):
        c = self

        class _R:
            def exchange(self, sends):
                for s, t in sends.items():
                    c.q[(r, s)].put(t.clone())
                return {s: c.q[(s, r)].get(timeout=120) for s in sends}

            def allreduce_(self, t, op="sum"):
                c.slots[r] = t.detach().cpu().clone()
                c.bar.wait(timeout=120)
                v = np.stack([s.numpy() for s in c.slots])
                red = {"sum": v.sum(0), "min": v.min(0), "max": v.max(0)}[op]
                c.bar.wait(timeout=120)
                t.copy_(__import__("torch").from_numpy(red).to(t.device))
                return t

        return _R()


def _run_threads(world, fn):
    comm = ThreadComm(world)
    out, errs = [None] * world, []

    def run(r):
        try:
            out[r] = fn(r, comm.rank(r))
        except BaseException as e:  # reported after the join
            errs.append(e)
            comm.bar.abort()

    th = [threading.Thread(target=run, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=600)
    if errs:
        raise errs[0]
    return out


@pytest.mark.gpu
def test_gpu_two_subdomains_product_blocks_cg():
    import torch

    from hfk.distributed import DistributedBlockJacobi, DistributedJacobian, Subdomain, cg, slab_partition
    from hfk.forms import svk_jacobian, svk_residual
    from hfk.operator import KernelOperator, MatrixFreeJacobian

    space = svk_space((4, 4, 8))
    res_f, jac_f = svk_residual(), svk_jacobian()
    x = _state(space)
    d = space.dirichlet_values
    # single domain
    op = KernelOperator(res_f, jac_f, space, jacobian="matrixfree")
    mf = MatrixFreeJacobian(op)
    mf.prepare(x)
    dx = np.random.default_rng(1).standard_normal(space.nfree)
    y = np.zeros(space.nfree)
    mf.mul(y, dx)
    opa = KernelOperator(res_f, jac_f, space)
    J = opa.jacobian(opa.allocate_jacobian(), x)
    b = np.random.default_rng(2).standard_normal(space.nfree)
    xd = spla.spsolve(J.tocsc(), b)
    cr = slab_partition(space.mesh, 2)

    def rank_fn(rank, comm):
        sub = Subdomain(space, cr, rank)
        lop = KernelOperator(res_f, jac_f, sub.space, jacobian="matrixfree")
        A = DistributedJacobian(sub, comm, mf=MatrixFreeJacobian(lop))
        A.prepare(torch.from_numpy(sub.restrict(x)).cuda(), d)
        yl = torch.zeros(sub.nfree, dtype=torch.float64, device="cuda")
        A.mul(yl, torch.from_numpy(sub.restrict(dx)).cuda())
        P = DistributedBlockJacobi(A).update()
        bl = torch.from_numpy(sub.restrict(b)).cuda()
        xs, it, conv, rel = cg(A, bl, P.ldiv, rtol=1e-10, maxiter=1000)
        torch.cuda.synchronize()
        return sub.free_global, yl.cpu().numpy(), xs.cpu().numpy(), it, conv, P.ok, lop.problem.launches()

    out = _run_threads(2, rank_fn)
    for fg, yl, xl, it, conv, ok, launches in out:
        assert launches > 0  # the engine's kernels ran
        assert ok and conv
        assert np.linalg.norm(yl - y[fg]) <= 1e-12 * np.linalg.norm(y[fg])
        assert np.linalg.norm(xl - xd[fg]) <= 1e-7 * np.linalg.norm(xd[fg])
    assert out[0][3] == out[1][3]  # both ranks stop on the same (all-reduced) test


@pytest.mark.gpu
def test_gpu_owner_assembly_rows_equal_global():
    import scipy.sparse as sp

    from hfk.distributed import OwnerAssembly, Subdomain, slab_partition
    from hfk.forms import svk_jacobian, svk_residual
    from hfk.operator import KernelOperator

    space = svk_space((3, 2, 6))
    res_f, jac_f = svk_residual(), svk_jacobian()
    x = _state(space)
    op = KernelOperator(res_f, jac_f, space)
    J = op.jacobian(op.allocate_jacobian(), x).tocsr()
    r = op.residual(np.zeros(space.nfree), x)
    cr = slab_partition(space.mesh, 3)
    order, vals, blocks = [], [], []
    for rank in range(3):
        sub = Subdomain(space, cr, rank, ghost=True)
        asm = OwnerAssembly(sub, KernelOperator(res_f, jac_f, sub.space))
        gi, rv = asm.residual(sub.restrict(x))
        order.append(gi)
        vals.append(rv)
        blocks.append(asm.jacobian_rows(sub.restrict(x)))
    order = np.concatenate(order)
    rr = np.zeros(space.nfree)
    rr[order] = np.concatenate(vals)
    assert np.linalg.norm(rr - r) <= 1e-12 * np.linalg.norm(r)
    perm = sp.csr_matrix((np.ones(space.nfree), (order, np.arange(space.nfree))), shape=(space.nfree, space.nfree))
    D = perm @ sp.vstack(blocks).tocsr() - J
    assert abs(D).max() <= 1e-12 * abs(J).max()


@pytest.mark.gpu
@pytest.mark.parametrize("coarse", ["cholesky", "cg"])
@pytest.mark.parametrize("orders,n", [((2, 1), (3, 3, 6)), ((4, 2, 1), (2, 2, 4))])
def test_gpu_two_subdomains_pmultigrid_matches_oracle(orders, n, coarse):
    """The partitioned V-cycle (Chebyshev–block-Jacobi levels; the replicated direct coarse solve or
    block-Jacobi CG coarse steps) equals the oracle's single-domain V-cycle with the same coarse solve,
    and preconditions a CG solve to the direct solution."""
    import torch

    import oracle as O
    from hfk import forms
    from hfk.distributed import DistributedJacobian, DistributedPMultigrid, Subdomain, cg, slab_partition
    from hfk.fespace import CartesianMesh, Quadrature, VectorLagrangeSpace
    from hfk.operator import KernelOperator, MatrixFreeJacobian
    from hfk.solvers import Chebyshev

    m = CartesianMesh(n)
    g = lambda X: np.stack([0.01 * X[:, 0], -0.02 * X[:, 1] * X[:, 2], 0.005 + 0 * X[:, 0]], axis=1)
    Vs = [VectorLagrangeSpace(m, o, "boundary", g=g if l == 0 else None) for l, o in enumerate(orders)]
    deg = 2 * orders[0]
    body = (0.3, -0.2, 0.5)
    res_f, jac_f = forms.svk_residual(2.0, 1.0, deg, body), forms.svk_jacobian(2.0, 1.0, deg)
    from conftest import svk_state

    x = svk_state(Vs[0], amp=1e-3, disp=0.0)
    d = Vs[0].dirichlet_values
    iters = 8
    ref = O.OraclePMG(Vs, Quadrature.gauss(deg), O.LAW_SVK, (2.0, 1.0) + body, degree=2,
                      coarse="direct" if coarse == "cholesky" else "cg", coarse_iters=iters)
    ref.update(x, d)
    r = np.random.default_rng(2).standard_normal(Vs[0].nfree)
    yref = ref.ldiv(r)
    xd = spla.spsolve(ref.levels[0].jacobian(x, d).tocsc(), r)  # any order (the engine assembles Q1/Q2)
    _, it_ref, conv_ref, _ = O.pcg(ref.levels[0].mf_apply, r, ref.ldiv, rtol=1e-9, maxiter=200)
    assert conv_ref
    cr = slab_partition(m, 2)

    def rank_fn(rank, comm):
        sub = Subdomain(Vs[0], cr, rank)
        lop = KernelOperator(res_f, jac_f, sub.space, jacobian="matrixfree")
        A = DistributedJacobian(sub, comm, mf=MatrixFreeJacobian(lop))
        A.prepare(torch.from_numpy(sub.restrict(x)).cuda(), d)
        mg = DistributedPMultigrid(A, Vs[1:], cr, Chebyshev(degree=2), coarse=coarse, coarse_iters=iters).update()
        rl = torch.from_numpy(sub.restrict(r)).cuda()
        y = torch.zeros_like(rl)
        mg.ldiv(y, rl)
        xs, it, conv, _ = cg(A, rl, mg.ldiv, rtol=1e-9, maxiter=200)
        torch.cuda.synchronize()
        return sub.free_global, mg.ok, mg.bounds[0], y.cpu().numpy(), xs.cpu().numpy(), it, conv

    out = _run_threads(2, rank_fn)
    lmax_ref = ref.smoothers[0].lmax
    for fg, ok, (lo, hi), y, xs, it, conv in out:
        assert ok
        assert abs(hi - lmax_ref) <= 1e-9 * lmax_ref
        assert np.linalg.norm(y - yref[fg]) <= 1e-9 * np.linalg.norm(yref[fg])
        assert conv and abs(it - it_ref) <= 2
        assert np.linalg.norm(xs - xd[fg]) <= 1e-6 * np.linalg.norm(xd[fg])


@pytest.mark.gpu
def test_gpu_two_subdomains_newton_matches_single_domain():
    """The load-stepped Newton over two subdomains (partitioned p-multigrid under the flexible CG)
    follows the single-domain engine's Newton: the same Newton iterations, the same solution."""
    import torch

    from hfk import forms
    from hfk import solvers as S
    from hfk.distributed import DistributedJacobian, DistributedPMultigrid, Subdomain, newton_solve, slab_partition
    from hfk.fespace import CartesianMesh, VectorLagrangeSpace
    from hfk.newton import newton_solve as newton_single
    from hfk.operator import KernelOperator, MatrixFreeJacobian

    m = CartesianMesh((3, 3, 6))
    gfun = [lambda X: 0 * X, lambda X: np.tile([0.1, 0.0, 0.0], (len(X), 1))]
    Vs = [VectorLagrangeSpace(m, o, ("x0", "x1"), g=gfun if o == 2 else None) for o in (2, 1)]
    g_full = Vs[0].dirichlet_values.copy()
    res_f, jac_f = forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4)
    loads = [0.5, 1.0]
    op = KernelOperator(res_f, jac_f, Vs[0], jacobian="matrixfree")
    ls = S.MatrixFreeSolver(krylov="fcg", rtol=1e-10, preconditioner=S.PMultigrid(Vs, S.Chebyshev(degree=3)))
    x1, st1 = newton_single(op, ls, g_full, loads, rtol_newton=1e-10)
    x1 = x1.cpu().numpy()
    Vs[0].dirichlet_values = g_full.copy()
    cr = slab_partition(m, 2)

    def rank_fn(rank, comm):
        sub = Subdomain(Vs[0], cr, rank)
        lop = KernelOperator(res_f, jac_f, sub.space, jacobian="matrixfree")
        A = DistributedJacobian(sub, comm, mf=MatrixFreeJacobian(lop))
        A.prepare(torch.zeros(sub.nfree, dtype=torch.float64, device="cuda"), g_full)
        mg = DistributedPMultigrid(A, Vs[1:], cr, S.Chebyshev(degree=3))
        x, st = newton_solve(A, mg, g_full, loads, rtol=1e-10, rtol_newton=1e-10)
        return sub.free_global, x.cpu().numpy(), st

    out = _run_threads(2, rank_fn)
    for fg, x, st in out:
        assert st.converged and st.newton_iters == st1.newton_iters
        assert np.linalg.norm(x - x1[fg]) <= 1e-8 * np.linalg.norm(x1[fg])
