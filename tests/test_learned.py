"""The learned correction: the network's kernels against the CPU oracle, training on the GPU, and
the trained correction inside the p-multigrid (judged against the plain cycle)."""
import numpy as np
import pytest

from conftest import reldiff

import oracle as O

pytestmark = pytest.mark.gpu


def _data(n, seed=0):
    import torch

    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, 16)).astype(np.float32)
    T = (0.3 * X[:, :3] - 0.2 * X[:, 3:6] + 0.1 * np.tanh(X[:, 6:9])).astype(np.float32)
    return X, T, torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()


def test_mlp_forward_and_gradient_match_the_cpu_oracle():
    import torch
    from hfk.learned import MLP, num_params

    assert num_params() == 16 * 64 + 64 + 64 * 64 + 64 + 3 * 64 + 3
    net = MLP(seed=3)
    X, T, Xd, Td = _data(1000)
    w = net.weights()
    out = torch.zeros(1000, 3, dtype=torch.float32, device="cuda")
    net.forward(Xd, out)
    assert reldiff(out.cpu().numpy(), O.mlp_forward(w, X.astype(np.float64))) < 1e-5
    g, loss = net.grad(Xd, Td)
    go, lo = O.mlp_grad(w, X.astype(np.float64), T.astype(np.float64))
    assert abs(loss - lo) < 1e-5 * lo
    assert reldiff(g, go) < 1e-4
    # per block of parameters too (the small output layer must not hide in the global norm)
    for s, e in ((0, 1024), (1088, 5184), (5248, 5440), (5440, 5443)):
        assert reldiff(g[s:e], go[s:e]) < 1e-3


def test_mlp_training_on_the_gpu_reduces_the_loss():
    from hfk.learned import MLP

    net = MLP(seed=1)
    X, T, Xd, Td = _data(20000, seed=2)
    _, l0 = net.grad(Xd, Td)
    net.train(Xd, Td, steps=400, batch=2048, lr=3e-3)
    _, l1 = net.grad(Xd, Td)
    assert l1 < 0.1 * l0


def test_learned_correction_inside_the_pmg():
    import torch

    from hfk import forms
    from hfk import solvers as S
    from hfk.fespace import CartesianMesh, VectorLagrangeSpace
    from hfk.learned import MLP, attach, collect_samples, stats
    from hfk.operator import KernelOperator

    m = CartesianMesh((6, 6, 6))
    g = [lambda x: 0 * x, lambda x: np.tile([0.05, 0.0, 0.0], (len(x), 1))]
    Vs = [VectorLagrangeSpace(m, o, ("x0", "x1"), g=g if o == 2 else None) for o in (2, 1)]
    res, jac = forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4)
    op = KernelOperator(res, jac, Vs[0], jacobian="matrixfree")
    rng = np.random.default_rng(0)
    x = torch.from_numpy(rng.uniform(-1e-3, 1e-3, Vs[0].nfree)).cuda()
    mf = op.allocate_jacobian(x)
    op.jacobian(mf, x)
    ls = S.MatrixFreeSolver(krylov="fcg", rtol=1e-8, preconditioner=S.PMultigrid(Vs, S.Chebyshev(degree=2)))
    ns = S.numerical_setup(ls, mf)
    # training pairs from the plain cycle
    feats, targets = [], []
    for seed in range(3):
        b = torch.from_numpy(np.random.default_rng(10 + seed).standard_normal(Vs[0].nfree)).cuda()
        f, t = collect_samples(ns.prec, mf, b, cycles=3)
        feats.append(f)
        targets.append(t)
    feats, targets = torch.cat(feats), torch.cat(targets)
    perm = torch.randperm(feats.shape[0], device="cuda")
    feats, targets = feats[perm].contiguous(), targets[perm].contiguous()
    net = MLP(seed=0)
    _, l0 = net.grad(feats, targets)
    net.train(feats, targets, steps=600, batch=4096, lr=2e-3)
    _, l1 = net.grad(feats, targets)
    assert l1 < l0
    # solve a held-out right-hand side with and without the correction
    b = torch.from_numpy(np.random.default_rng(99).standard_normal(Vs[0].nfree)).cuda()
    its = {}
    for use in (False, True):
        attach(ns.prec, net if use else None)
        dx = torch.zeros_like(b)
        S.solve(dx, ns, b)
        assert S.linear_converged(ns)
        r = b - mf.mul(torch.zeros_like(b), dx)
        assert float(torch.linalg.norm(r)) <= 1e-8 * float(torch.linalg.norm(b)) * 1.01
        its[use] = S.linear_iterations(ns)
    st = stats(ns.prec)
    print(f"learned correction: loss {l0:.3e} -> {l1:.3e}; FCG iterations plain {its[False]}, learned {its[True]}; "
          f"accepted {st['accepted']}/{st['tried']}")
    assert st["tried"] > 0
    assert its[True] <= its[False] + 2


def test_trained_correction_lowers_the_error_of_a_cycle():
    # What the trained network gains over the method without it, per application of the V-cycle:
    # the energy-norm error left by one cycle on held-out right-hand sides b = A x* (exact error
    # known), plain cycle vs cycle + correction with an untrained network vs with the trained one.
    # The step along the prediction minimises the energy error, so no variant can be worse than the
    # plain cycle; training must add a clear margin over the untrained network.
    import torch

    from hfk import forms
    from hfk import solvers as S
    from hfk.fespace import CartesianMesh, VectorLagrangeSpace
    from hfk.learned import MLP, attach, collect_samples
    from hfk.operator import KernelOperator

    m = CartesianMesh((6, 6, 6))
    g = [lambda x: 0 * x, lambda x: np.tile([0.05, 0.0, 0.0], (len(x), 1))]
    Vs = [VectorLagrangeSpace(m, o, ("x0", "x1"), g=g if o == 2 else None) for o in (2, 1)]
    op = KernelOperator(forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4), Vs[0], jacobian="matrixfree")
    x = torch.from_numpy(np.random.default_rng(0).uniform(-1e-3, 1e-3, Vs[0].nfree)).cuda()
    mf = op.allocate_jacobian(x)
    op.jacobian(mf, x)
    st = S.PMultigridState(S.PMultigrid(Vs, S.Chebyshev(degree=2)), mf)
    assert st.ok
    feats, targets = [], []
    for seed in range(4):
        b = torch.from_numpy(np.random.default_rng(10 + seed).standard_normal(Vs[0].nfree)).cuda()
        f, t = collect_samples(st, mf, b, cycles=3)
        feats.append(f)
        targets.append(t)
    feats, targets = torch.cat(feats), torch.cat(targets)
    perm = torch.randperm(feats.shape[0], device="cuda", generator=torch.Generator("cuda").manual_seed(0))
    feats, targets = feats[perm].contiguous(), targets[perm].contiguous()
    trained = MLP(seed=0)
    trained.train(feats, targets, steps=800, batch=4096, lr=2e-3)
    untrained = MLP(seed=7)

    def energy(e):
        Ae = torch.zeros_like(e)
        mf.mul(Ae, e)
        return float(torch.dot(e, Ae)) ** 0.5

    ratios = {}
    for name, net in (("plain", None), ("untrained", untrained), ("trained", trained)):
        attach(st, net)
        rs = []
        for seed in range(100, 104):  # held out: not among the training right-hand sides
            xs = torch.from_numpy(np.random.default_rng(seed).standard_normal(Vs[0].nfree)).cuda()
            b = torch.zeros_like(xs)
            mf.mul(b, xs)
            y = torch.zeros_like(xs)
            st.ldiv(y, b)
            rs.append(energy(xs - y) / energy(xs))
        ratios[name] = float(np.mean(rs))
    attach(st, None)
    print("energy error left by one cycle (mean of 4 held-out right-hand sides): "
          + ", ".join(f"{k} {v:.4f}" for k, v in ratios.items()))
    assert ratios["untrained"] <= ratios["plain"] * (1 + 1e-12)
    assert ratios["trained"] <= ratios["plain"] * (1 + 1e-12)
    assert ratios["trained"] < ratios["untrained"]
    assert ratios["trained"] < 0.95 * ratios["plain"]
