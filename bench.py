"""Benchmark of the hot path: matrix-free SVK Jacobian-vector product, Q2 hexahedra on a 64^3 cube.

One step = one J(x)·dx over the whole mesh (6.34 M free dofs), FP64, tangent re-evaluated from the
state inside the product (sum factorisation). Inputs are resident in HBM for `value`; `e2e` runs the
same product through the public C ABI with pinned host buffers (dx copied in, y copied out every
step). Prints one JSON line (rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

`--impl reference` times the CPU restatement of the reference algorithm (the oracle: the
reference's stored-tangent matrix-free product, OpenMP over all host cores) on a bounded sample of
the same workload.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "hyperfemkernels.jl_b200"))

METRIC = "Q2 SVK Jacobian GDOF/s (matrix-free J*v, FP64)"
UNIT = "GDOF/s"
N_CELLS = 64
ORDER = 2
WORKLOAD = "MF Jacobian-vector product, SVK (lambda=2, mu=1), Q2 hexahedra, 64^3 unit cube, Gauss 3^3"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--n", type=int, default=N_CELLS, help="cells per direction")
    ap.add_argument("--no-extra", action="store_true", help="skip the secondary measurements")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--batch", action="store_true",
                    help="the batched workload instead: 256 SVK Q2 Newton solves (plain p-MG vs learned correction)")
    ap.add_argument("--batch-count", type=int, default=256)
    ap.add_argument("--batch-precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--oseen", type=int, default=0, metavar="N",
                    help="only the Oseen P2-P1 assembly on the N^3 tetrahedral cube (the secondary case; 0 = off)")
    ap.add_argument("--launch", default="auto", choices=["auto", "line2", "line4", "point"],
                    help="launch shape of the J*v (auto: the autotuner's; a fixed one for profiling, where the "
                         "profiler's overhead would skew the autotuner's timings)")
    ap.add_argument("--assembly", action="store_true",
                    help="only the Q2 SVK 20x10x10 residual + CSC Jacobian (the CPU-runnable configuration)")
    ap.add_argument("--vcycle", type=int, default=0, metavar="K",
                    help="only K V-cycles of the Q4 16^3 p-multigrid 4 -> 2 -> 1 (the Newton case's preconditioner)")
    return ap.parse_args()


def build_case(n, order=ORDER, seed=0):
    from hfk.fespace import CartesianMesh, VectorLagrangeSpace

    m = CartesianMesh((n, n, n))
    g = [lambda x: 0 * x, lambda x: np.tile([0.05, 0.0, 0.0], (len(x), 1))]
    V = VectorLagrangeSpace(m, order, ("x0", "x1"), g=g)
    rng = np.random.default_rng(seed)
    x, _ = V.interpolate(lambda p: np.stack([0.05 * p[:, 0], 0 * p[:, 0], 0 * p[:, 0]], axis=1))
    x = x + rng.uniform(-1e-3, 1e-3, V.nfree)
    dx = np.random.default_rng(seed + 1).standard_normal(V.nfree)
    return V, x, dx


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sms, maxs, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [s.strip() for s in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sms.append(float(f[1]))
                maxs.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sms:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sms), "sm_max_mhz": max(maxs), "reasons": sorted(reasons),
                "samples": len(sms)}


def jv_flops_per_cell(Q, P):
    """FP64 flops of one recompute J*v cell: 3 interpolations (the components of dx), 3
    contractions, the pointwise law (F is stored, not interpolated)."""
    interp = 2 * (2 * P * Q**3 + 3 * P**2 * Q**2 + 3 * P**3 * Q)  # x, y, z sweeps (FMA = 2)
    contract = 2 * (3 * P**3 * Q + 3 * P**2 * Q**2 + 2 * P * Q**3)
    pointwise = P**3 * (2 * (27 + 27 + 18 + 27 + 27 + 27 + 27) + 60)  # grads, F'F, F'Hd, Hd S, F W, pull-back
    return 3 * interp + 3 * contract + pointwise


def engine(args):
    import torch
    import torch.distributed as dist

    from hfk import _lib, forms
    from hfk.operator import KernelOperator, MatrixFreeJacobian

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    V, x, dx = build_case(args.n)
    op = KernelOperator(forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4), V, jacobian="matrixfree")
    stream = torch.cuda.current_stream()
    op.problem.set_stream(stream.cuda_stream)
    n = V.nfree
    dev = torch.device("cuda", local)
    xd = torch.from_numpy(x).to(dev)
    dd = torch.from_numpy(np.ascontiguousarray(V.dirichlet_values)).to(dev)
    dxd = torch.from_numpy(dx).to(dev)
    yd = torch.zeros(n, dtype=torch.float64, device=dev)
    if args.launch != "auto":
        op.problem.set_scatter("atomic")
        op.problem.set_launch("point" if args.launch == "point" else "line",
                              0 if args.launch == "point" else int(args.launch[-1]))
    mf = MatrixFreeJacobian(op, "recompute")
    mf.prepare(xd, dd)
    h = op.problem.h

    def step():
        _lib.call("hfk_mf_apply", h, _lib.ptr(dxd), _lib.ptr(yd))

    def timed(fn, steps, warm):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    # ---- headline: device-resident FP64 J*v ----
    step()
    torch.cuda.synchronize()
    l0 = op.problem.launches()
    with ClockSampler(local) as clk:
        ms = timed(step, args.steps, args.warmup)
    launches = (op.problem.launches() - l0) // (args.steps + args.warmup) * args.steps
    ms_step = ms / args.steps
    value = world * n / (ms_step * 1e-3) / 1e9
    clocks = clk.summary()

    # ---- e2e: host (pinned) buffers through the public ABI, H2D + D2H of every step's vector ----
    # a stream of K host vectors in one hfk_mf_apply_many call (the copies of one vector overlap the
    # product of the next), inputs and outputs cycling through a ring of pinned buffers
    ring = 4
    dxh = [torch.from_numpy(dx).pin_memory() for _ in range(ring)]
    yh = [torch.zeros(n, dtype=torch.float64).pin_memory() for _ in range(ring)]
    k_e2e = max(3, args.steps // 2)
    pin = (ctypes.c_void_p * k_e2e)(*[dxh[i % ring].data_ptr() for i in range(k_e2e)])
    pout = (ctypes.c_void_p * k_e2e)(*[yh[i % ring].data_ptr() for i in range(k_e2e)])

    def step_e2e_many():
        _lib.call("hfk_mf_apply_many", h, k_e2e, ctypes.cast(pin, ctypes.c_void_p), ctypes.cast(pout, ctypes.c_void_p))

    ms_e2e = timed(step_e2e_many, 1, 1) / k_e2e
    e2e_err = max(float(torch.linalg.norm(y.to(dev) - yd) / torch.linalg.norm(yd)) for y in yh[:min(ring, k_e2e)])

    def step_e2e():  # one vector per synchronous call: copy in, product, copy out
        _lib.call("hfk_mf_apply", h, _lib.ptr(dxh[0]), _lib.ptr(yh[0]))

    ms_single = timed(step_e2e, max(3, args.steps // 2), 2) / max(3, args.steps // 2)
    e2e = {"value": world * n / (ms_e2e * 1e-3) / 1e9, "unit": UNIT, "h2d_bytes_per_step": 8 * n,
           "d2h_bytes_per_step": 8 * n, "ms_per_step": ms_e2e,
           "mode": f"{k_e2e} host vectors per hfk_mf_apply_many call (pinned ring of {ring})",
           "rel_err_vs_device_resident": e2e_err,
           "single_call": {"value": world * n / (ms_single * 1e-3) / 1e9, "ms_per_step": ms_single}}

    # ---- roofline of the dominant kernel (colour launches of the J*v cell kernel) ----
    ncells = V.mesh.ncells
    # ids, dx read, y read+write, F per point (prepared deformation gradient), per-cell geometry
    alg_bytes = 4 * V.ndl * ncells + 8 * n * 3 + 72 * 27 * ncells + 81 * ncells
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        hbm, src = float(peaks["hbm_gbs"]), "measured"
    except Exception:
        hbm, src = 6650.0, "fallback"
    achieved = alg_bytes / (ms_step * 1e-3) / 1e9
    flops = jv_flops_per_cell(3, 3) * ncells
    # DRAM bytes (read + write) of one launch of this kernel and launch shape from an ncu capture of
    # the 48^3 case (110 592 cells: 302.7 MB + 22.5 MB), scaled by cells; the profile summary gives
    # the capture's command
    traffic = (302.712e6 + 22.487e6) * ncells / 110592 if ORDER == 2 else None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": traffic, "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, Q2 48^3 "
                "launch, scaled by cells", "peak_source": src, "bytes_per_launch": alg_bytes,
                "fp64_tflops": flops / (ms_step * 1e-3) / 1e12, "fp64_flops_per_launch": flops,
                "note": "recompute J*v is latency/FP64-issue bound; hbm frac uses the algorithmic bytes"}

    extra = {}
    if not args.no_extra and rank == 0:
        # reference formulation on the GPU: stored tangents (T, inv(Jt), dV per point)
        mfs = MatrixFreeJacobian(op, "stored")
        mfs.prepare(xd, dd)
        ms_s = timed(step, max(3, args.steps // 2), 2) / max(3, args.steps // 2)
        stored_bytes = 8 * 91 * 27 * ncells + 8 * n * 2 + 4 * V.ndl * ncells
        extra["jv_stored_fp64"] = {"gdofs": n / (ms_s * 1e-3) / 1e9, "ms": ms_s,
                                   "hbm_frac": stored_bytes / (ms_s * 1e-3) / 1e9 / hbm}
        mf.prepare(xd, dd)
        dx32 = dxd.float()
        y32 = torch.zeros(n, dtype=torch.float32, device=dev)

        def step32():
            _lib.call("hfk_mf_apply_f32", h, _lib.ptr(dx32, np.float32), _lib.ptr(y32, np.float32))

        ms32 = timed(step32, max(3, args.steps // 2), 2) / max(3, args.steps // 2)
        step()
        torch.cuda.synchronize()
        err32 = float(torch.linalg.norm(y32.double() - yd) / torch.linalg.norm(yd))
        extra["jv_recompute_fp32"] = {"gdofs": n / (ms32 * 1e-3) / 1e9, "ms": ms32, "rel_err_vs_fp64": err32}
        extra["autotuned_launch_shape"] = {k: op.problem.tuning(*k.split("_")) for k in ("jv_fp64", "jv_fp32")}
        extra.update(assembly_case(torch, dev, stream, timed))
        extra.update(jv_sizes_case(torch, dev, stream, timed))
        extra.update(oseen_case(torch, dev, stream, timed))
        extra.update(newton_case())

    cpu = cpu_baseline_sample() if rank == 0 and not args.no_cpu else None
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": WORKLOAD, "cells": ncells, "free_dofs_per_gpu": n, "order": ORDER,
                           "quadrature_points_per_cell": 27, "parallelism": f"replicas x{world}",
                           "l2": f"inputs larger than L2 ({alg_bytes / 1e6:.0f} MB read per step, L2 126 MB)",
                           "state": "u = 0.05 x e_x + U(-1e-3, 1e-3), dx ~ N(0,1), seeds 0/1"},
                "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks, "roofline": roofline,
                "cpu_baseline": cpu, "extra": extra}
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def jv_sizes_case(torch, dev, stream, timed, cases=((2, 48), (4, 48), (4, 64))):
    """Secondary: the other C1 sizes (Q2 48^3, Q4 48^3 and 64^3; Q4 with Gauss 5^3), FP64 and FP32
    recompute J*v, same law, state and increment as the headline."""
    from hfk import _lib, forms
    from hfk.operator import KernelOperator, MatrixFreeJacobian

    out = {}
    for order, n in cases:
        V, x, dx = build_case(n, order)
        deg = 2 * order
        op = KernelOperator(forms.svk_residual(2.0, 1.0, deg), forms.svk_jacobian(2.0, 1.0, deg), V,
                            jacobian="matrixfree")
        op.problem.set_stream(stream.cuda_stream)
        xd = torch.from_numpy(x).to(dev)
        dd = torch.from_numpy(np.ascontiguousarray(V.dirichlet_values)).to(dev)
        dxd = torch.from_numpy(dx).to(dev)
        yd = torch.zeros(V.nfree, dtype=torch.float64, device=dev)
        mf = MatrixFreeJacobian(op, "recompute")
        mf.prepare(xd, dd)
        h = op.problem.h
        steps = 20 if order == 4 else 50
        ms64 = timed(lambda: _lib.call("hfk_mf_apply", h, _lib.ptr(dxd), _lib.ptr(yd)), steps, 3) / steps
        dx32, y32 = dxd.float(), torch.zeros(V.nfree, dtype=torch.float32, device=dev)
        ms32 = timed(lambda: _lib.call("hfk_mf_apply_f32", h, _lib.ptr(dx32, np.float32), _lib.ptr(y32, np.float32)),
                     steps, 3) / steps
        err = float(torch.linalg.norm(y32.double() - yd) / torch.linalg.norm(yd))
        Q, P = order + 1, order + 1
        flops = jv_flops_per_cell(Q, P) * V.mesh.ncells
        out[f"jv_q{order}_{n}"] = {"free_dofs": V.nfree, "fp64_ms": ms64, "fp64_gdofs": V.nfree / (ms64 * 1e-3) / 1e9,
                                   "fp64_tflops": flops / (ms64 * 1e-3) / 1e12, "fp32_ms": ms32,
                                   "fp32_gdofs": V.nfree / (ms32 * 1e-3) / 1e9, "fp32_rel_err": err}
        del op, mf, xd, dxd, yd, dx32, y32
        torch.cuda.empty_cache()
    return out


def oseen_case(torch, dev, stream, timed, n=32, cpu_n=12):
    """Secondary (config 2): one FP64 residual and one CSC Jacobian of the Oseen-BDF2 step (volume terms
    and the outlet boundary group), Taylor-Hood P2-P1 on the 32^3 cube split into 196 608 tetrahedra
    (859 812 dofs), rho = 1, mu = 1e-3, dt = 1e-3,
    advection from a seeded sum of 8 divergence-free Fourier modes of amplitude 1 (u^n = u^(n-1));
    the CPU restatement (literal weak form, all host cores) timed on a 12^3 sample."""
    from hfk import _lib
    from hfk import oseen as OS

    m = OS.TetMesh(n)
    V = OS.TaylorHoodSpace(m)
    un, und = V.interpolate_velocity(OS.fourier_field(2))
    params = OS.OseenParams(rho=1.0, mu=1e-3, dt=1e-3, bdf2=True)
    op = OS.OseenOperator(V, params, un, und)
    op.set_outlet(OS.OutletFacets(m))  # the outlet boundary group (backflow, Robin, Windkessel)
    x = np.random.default_rng(0).standard_normal(V.nfree)
    A = op.sparsity_pattern()
    xd = torch.from_numpy(x).to(dev)
    dd = torch.from_numpy(np.ascontiguousarray(V.dirichlet_values)).to(dev)
    bd = torch.zeros(V.nfree, dtype=torch.float64, device=dev)
    nz = torch.zeros(A.nnz, dtype=torch.float64, device=dev)
    h = op.h
    ms_j = timed(lambda: _lib.call("hfk_oseen_jacobian", h, _lib.ptr(nz)), 10, 3) / 10
    ms_r = timed(lambda: _lib.call("hfk_oseen_residual", h, _lib.ptr(xd), _lib.ptr(dd), _lib.ptr(bd)), 10, 3) / 10
    # CPU restatement on a sample
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    ms_ = OS.TetMesh(cpu_n)
    Vs = OS.TaylorHoodSpace(ms_)
    uns, unds = Vs.interpolate_velocity(OS.fourier_field(2))
    orc = O.OracleOseen(Vs, params, uns, unds)
    orc.set_outlet(OS.OutletFacets(ms_))
    orc.pattern()
    xs = np.random.default_rng(0).standard_normal(Vs.nfree)
    t0 = time.perf_counter()
    orc.jacobian_values()
    tj = time.perf_counter() - t0
    t0 = time.perf_counter()
    orc.residual(xs, Vs.dirichlet_values)
    tr = time.perf_counter() - t0
    scale = m.ncells / ms_.ncells
    return {f"oseen_p2p1_tet_{n}": {"cells": m.ncells, "dofs": V.ndof_total, "free_dofs": V.nfree, "nnz": int(A.nnz),
                                  "jacobian_ms": ms_j, "residual_ms": ms_r,
                                  "jacobian_gdofs": V.nfree / (ms_j * 1e-3) / 1e9,
                                  "cpu_sample": f"oracle on {cpu_n}^3 ({ms_.ncells} cells), {O.lib().o_max_threads()} threads",
                                  "cpu_jacobian_ms_extrapolated": 1e3 * tj * scale,
                                  "cpu_residual_ms_extrapolated": 1e3 * tr * scale,
                                  "speedup_jacobian_vs_cpu": 1e3 * tj * scale / ms_j}}


def oseen_main(args):
    """The Oseen assembly alone (``--oseen N``), or the Q2 SVK 20x10x10 CSC assembly alone
    (``--assembly``), one JSON line: the cases for profiling their kernels."""
    import torch

    stream = torch.cuda.current_stream()

    def timed(fn, steps, warm):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    if args.assembly:
        out = assembly_case(torch, torch.device("cuda"), stream, timed)
    else:
        out = oseen_case(torch, torch.device("cuda"), stream, timed, n=args.oseen, cpu_n=min(args.oseen, 8))
    print(json.dumps(out))


def vcycle_main(args, n=16):
    """The p-multigrid V-cycle alone (``--vcycle K``): the Newton case's hierarchy (SVK Q4 -> Q2 -> Q1
    on the 16^3 cube, Chebyshev degree 4, assembled Q1 coarse level with its banded Cholesky) built
    once at a loaded state, then K cycles on a device vector, timed with CUDA events. One JSON line;
    the case for the cycle's launch list."""
    import torch

    from hfk import forms
    from hfk import solvers as S
    from hfk.fespace import CartesianMesh, VectorLagrangeSpace
    from hfk.operator import KernelOperator

    m = CartesianMesh((n, n, n))
    gfun = [lambda x: 0 * x, lambda x: np.tile([0.05, 0.0, 0.0], (len(x), 1))]
    Vs = [VectorLagrangeSpace(m, o, ("x0", "x1"), g=gfun if o == 4 else None) for o in (4, 2, 1)]
    op = KernelOperator(forms.svk_residual(2.0, 1.0, 8), forms.svk_jacobian(2.0, 1.0, 8), Vs[0], jacobian="matrixfree")
    x = np.zeros(Vs[0].nfree)
    mf = op.allocate_jacobian(x)
    mf.prepare(x, 0.1 * Vs[0].dirichlet_values)
    st = S.PMultigridState(S.PMultigrid(Vs, S.Chebyshev(degree=4)), mf)
    r = torch.randn(Vs[0].nfree, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(0))
    y = torch.zeros_like(r)
    stream = torch.cuda.current_stream()
    for _ in range(3):
        st.ldiv(y, r)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.vcycle):
        st.ldiv(y, r)
    e1.record(stream)
    torch.cuda.synchronize()
    print(json.dumps({"case": f"V-cycle SVK Q4 {n}^3 -> Q2 -> Q1", "free_dofs": Vs[0].nfree,
                      "coarse_free_dofs": Vs[2].nfree, "cycles": args.vcycle,
                      "ms_per_cycle": e0.elapsed_time(e1) / args.vcycle}))


def assembly_case(torch, dev, stream, timed):
    """Secondary: Q2 SVK 20x10x10 residual + CSC Jacobian (the reference's CPU-runnable case)."""
    from hfk import _lib, forms
    from hfk.fespace import CartesianMesh, VectorLagrangeSpace
    from hfk.operator import KernelOperator

    m = CartesianMesh((20, 10, 10))
    g = [lambda x: 0 * x, lambda x: np.tile([0.05, 0.0, 0.0], (len(x), 1))]
    V = VectorLagrangeSpace(m, 2, ("x0", "x1"), g=g, open_faces=True)  # Gridap face tags: 52 077 free dofs
    rng = np.random.default_rng(0)
    x, _ = V.interpolate(lambda p: np.stack([0.05 * p[:, 0], 0 * p[:, 0], 0 * p[:, 0]], axis=1))
    x = x + rng.uniform(-1e-3, 1e-3, V.nfree)
    op = KernelOperator(forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4), V)
    op.problem.set_stream(stream.cuda_stream)
    op.sparsity_pattern()
    nnz = op.sparsity_pattern().nnz
    xd = torch.from_numpy(x).to(dev)
    dd = torch.from_numpy(np.ascontiguousarray(V.dirichlet_values)).to(dev)
    nz = torch.zeros(nnz, dtype=torch.float64, device=dev)
    b = torch.zeros(V.nfree, dtype=torch.float64, device=dev)
    h = op.problem.h

    def jac():
        _lib.call("hfk_jacobian", h, _lib.ptr(xd), _lib.ptr(dd), _lib.ptr(nz))

    def res():
        _lib.call("hfk_residual", h, _lib.ptr(xd), _lib.ptr(dd), _lib.ptr(b))

    ms_j = timed(jac, 10, 3) / 10
    ms_r = timed(res, 10, 3) / 10
    # the bit-reproducible colour-by-colour scatter (HFK_SCATTER_COLOURED) for comparison
    op.problem.set_scatter("coloured")
    ms_jc = timed(jac, 10, 3) / 10
    nz_c = nz.clone()
    op.problem.set_scatter("auto")
    jac()
    # the same assembly by the CPU restatement of the reference algorithm (matrix-product element
    # Jacobian with point blocks of 12, colour loop, OpenMP on all host cores), best of 5
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from hfk.fespace import Quadrature

    orc = O.OracleProblem(V, Quadrature.gauss(4))
    orc.pattern()
    d = np.ascontiguousarray(V.dirichlet_values)
    orc.jacobian_values(x, d)
    tj, tr = [], []
    for _ in range(5):
        t0 = time.perf_counter()
        orc.jacobian_values(x, d)
        tj.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        orc.residual(x, d)
        tr.append(time.perf_counter() - t0)
    ref = orc.jacobian_values(x, d)
    got = nz.cpu().numpy()
    err = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    cpu_j, cpu_r = 1e3 * min(tj), 1e3 * min(tr)
    err_c = float(np.linalg.norm(nz_c.cpu().numpy() - ref) / np.linalg.norm(ref))
    return {"assembly_q2_20x10x10": {"free_dofs": V.nfree, "nnz": int(nnz), "jacobian_ms": ms_j, "residual_ms": ms_r,
                                     "jacobian_coloured_ms": ms_jc, "rel_err_coloured_vs_cpu": err_c,
                                     "jacobian_gdofs": V.nfree / (ms_j * 1e-3) / 1e9,
                                     "jacobian_qps": 27 * V.mesh.ncells / (ms_j * 1e-3),
                                     "cpu_jacobian_ms": cpu_j, "cpu_residual_ms": cpu_r,
                                     "cpu_cores": O.lib().o_max_threads(), "cpu_kind": "port",
                                     "speedup_jacobian_vs_cpu": cpu_j / ms_j,
                                     "speedup_residual_jacobian_vs_cpu": (cpu_j + cpu_r) / (ms_j + ms_r),
                                     "rel_err_vs_cpu": err}}


def newton_case(n=16, loads=(0.1, 0.325, 0.55, 0.775, 1.0)):
    """Secondary: matrix-free Newton on SVK Q4 16^3 (823 875 dofs), load factor 0.1-1.0 in 5 steps,
    flexible CG + p-multigrid 4 -> 2 -> 1 (Chebyshev degree 4, assembled Q1 coarse), every linear
    solve to 1e-8 relative; plain FP64 vs FP32 smoothers/products under the FP64 outer loop."""
    from hfk import forms
    from hfk import solvers as S
    from hfk.fespace import CartesianMesh, VectorLagrangeSpace
    from hfk.newton import newton_solve
    from hfk.operator import KernelOperator

    m = CartesianMesh((n, n, n))
    gfun = [lambda x: 0 * x, lambda x: np.tile([0.05, 0.0, 0.0], (len(x), 1))]
    Vs = [VectorLagrangeSpace(m, o, ("x0", "x1"), g=gfun if o == 4 else None) for o in (4, 2, 1)]
    g_full = Vs[0].dirichlet_values.copy()
    res, jac = forms.svk_residual(2.0, 1.0, 8), forms.svk_jacobian(2.0, 1.0, 8)
    out = {}
    for prec in ("fp64", "fp32"):
        op = KernelOperator(res, jac, Vs[0], jacobian="matrixfree")
        ls = S.MatrixFreeSolver(krylov="fcg", rtol=1e-8, maxiter=300,
                                preconditioner=S.PMultigrid(Vs, S.Chebyshev(degree=4), precision=prec))
        newton_solve(op, ls, g_full, loads[:1], rtol_newton=1e-8)  # warm-up (kernel attributes, handles)
        x, st = newton_solve(op, ls, g_full, loads, rtol_newton=1e-8)
        out[prec] = {"seconds": st.seconds, "newton_iters": st.newton_iters, "krylov_iters": st.krylov_iters,
                     "converged": st.converged, "final_residual": st.residual_norms[-1], "pmg": st.pmg,
                     "residual_norms": [float(f"{r:.3e}") for r in st.residual_norms]}
    # the reference guide's production setting: the coarse level rebuilt every third update
    # (PMultigrid(...; coarse_every = 3), docs/guide/README.md:256-261)
    for prec in ("fp64", "fp32"):
        op = KernelOperator(res, jac, Vs[0], jacobian="matrixfree")
        ls = S.MatrixFreeSolver(krylov="fcg", rtol=1e-8, maxiter=300,
                                preconditioner=S.PMultigrid(Vs, S.Chebyshev(degree=4), precision=prec, coarse_every=3))
        newton_solve(op, ls, g_full, loads[:1], rtol_newton=1e-8)
        x, st = newton_solve(op, ls, g_full, loads, rtol_newton=1e-8)
        out[f"{prec}_coarse_every3"] = {"seconds": st.seconds, "newton_iters": st.newton_iters,
                                        "krylov_iters": int(sum(st.krylov_iters)), "converged": st.converged,
                                        "final_residual": st.residual_norms[-1],
                                        "coarse_builds": st.pmg["coarse_builds"]}
    out["speedup_mixed_vs_fp64"] = out["fp64"]["seconds"] / out["fp32"]["seconds"]
    return {"newton_pmg_svk_q4_16": {"free_dofs": Vs[0].nfree, "levels": "Q4 -> Q2 -> Q1 (assembled, banded Cholesky)",
                                     "loads": list(loads), **out}}


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_baseline_sample(budget_s=15.0):
    """Oracle (CPU restatement, stored-tangent J*v as the reference) on a bounded sample: Q2 24^3."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from hfk.fespace import Quadrature

    nsub = 24
    V, x, dx = build_case(nsub)
    p = O.OracleProblem(V, Quadrature.gauss(4))
    p.mf_prepare(x, V.dirichlet_values)
    p.mf_apply(dx)
    t0 = time.perf_counter()
    k = 0
    while True:
        p.mf_apply(dx)
        k += 1
        if time.perf_counter() - t0 > budget_s or k >= 50:
            break
    t = (time.perf_counter() - t0) / k
    return {"value": V.nfree / t / 1e9, "unit": UNIT, "cores": O.lib().o_max_threads(), "kind": "port",
            "sample": f"Q2 {nsub}^3 ({V.nfree} free dofs), {k} stored-tangent J*v applies, OpenMP all host cores"}


def reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from hfk.fespace import Quadrature

    # bounded sample of the workload per step: Q2 24^3 (1/19 of the cells), the reference's formulation
    nsub = 24
    V, x, dx = build_case(nsub)
    p = O.OracleProblem(V, Quadrature.gauss(4))
    p.mf_prepare(x, V.dirichlet_values)
    for _ in range(max(1, args.warmup)):
        p.mf_apply(dx)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        p.mf_apply(dx)
    t = (time.perf_counter() - t0) / args.steps
    value = V.nfree / t / 1e9
    cores = O.lib().o_max_threads()
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample": f"Q2 {nsub}^3 per step"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"Q2 {nsub}^3 ({V.nfree} free dofs) stored-tangent J*v per step"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


BATCH_LOADS = (0.1, 0.325, 0.55, 0.775, 1.0)
# block-Jacobi CG steps of the batched coarse solve (measured on the 256 problems, FP64: 5 / 10 / 15
# / 20 / 40 steps -> 29.8 / 21.7 / 23.2 / 24.1 / 32.8 s; each step costs ~0.85 ms a cycle, and more
# steps barely lower the Krylov count of the slowest problem)
BATCH_COARSE_STEPS = 10


def _batch_setup(count, seed=4, rank=0, world=1):
    from hfk import batch as B

    problems = B.draw_batch(256, seed=seed)[:count]
    if world > 1:  # shard by problem: every rank solves its own subset, no data exchange
        problems = [problems[k] for k in B.shard_problems(problems, rank, world)]
    (U2, U1), g = B.cube_batch(problems)
    return problems, U2, U1, g, B.cube_lifting(U2)


def _batch_solver(U2, U1, precision):
    from hfk import solvers as S

    return S.MatrixFreeSolver(krylov="fcg", rtol=1e-8, maxiter=400,
                              preconditioner=S.PMultigrid([U2, U1], S.Chebyshev(degree=4), precision=precision,
                                                          coarse="cg", coarse_iters=BATCH_COARSE_STEPS))


def batch_cpu_sample(problems, budget_s=20.0):
    """The same per-problem Newton (lifting predictor, 5 load steps, FCG + p-MG Q2 -> Q1 with the
    10-step coarse CG, all to 1e-8) by the oracle on the host cores, on the smallest problems of
    the batch until ``budget_s`` is spent; returns seconds per free dof (to extrapolate)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from hfk import batch as B
    from hfk.fespace import Quadrature

    q = Quadrature.gauss(4)
    done, dofs, t_all = [], 0, 0.0
    for k in np.argsort([p.n for p in problems]):
        pb = problems[k]
        (U2, U1), g = B.cube_batch([pb])
        V2, V1 = U2.spaces[0], U1.spaces[0]
        lift = B.cube_lifting(U2)
        orc = O.OracleProblem(V2, q, O.LAW_SVK, (pb.lam, pb.mu))
        mg = O.OraclePMG([V2, V1], q, O.LAW_SVK, (pb.lam, pb.mu), degree=4, coarse="cg", coarse_iters=BATCH_COARSE_STEPS)
        x = np.zeros(V2.nfree)
        t0 = time.perf_counter()
        prev = 0.0
        for lam in BATCH_LOADS:
            d = lam * g
            x = x + (lam - prev) * lift
            prev = lam
            r0 = None
            for _ in range(20):
                r = orc.residual(x, d)
                rn = np.linalg.norm(r)
                r0 = rn if r0 is None else r0
                if rn <= max(1e-8 * r0, 1e-12):
                    break
                orc.mf_prepare(x, d)
                mg.update(x, d)
                dx, _, ok, _ = O.pcg(orc.mf_apply, -r, mg.ldiv, rtol=1e-8, maxiter=400)
                x = x + dx
        t_all += time.perf_counter() - t0
        dofs += V2.nfree
        done.append(int(pb.n))
        if t_all > budget_s:
            break
    return {"seconds_per_free_dof": t_all / dofs, "sample": f"{len(done)} problems n={done} ({dofs} free dofs), "
            f"{t_all:.1f} s", "cores": O.lib().o_max_threads(), "kind": "port"}


def batch_main(args):
    """Batched workload: ``--batch-count`` independent SVK Q2 Newton solves (n ~ U{8..24} cells per
    direction, lambda, mu log-uniform in [0.5, 20] x [0.2, 5], seed 4), x = 0 clamped, x = 1 moved
    0.05 along x in 5 load steps, every Newton and linear solve to 1e-8, all problems advanced by the
    same launches (one handle, per-problem scalars). First with the plain p-multigrid (Q2 -> Q1,
    Chebyshev 4, 10-step coarse CG), then with the learned correction trained on pairs from the
    plain cycle at seeded states of the converged solution."""
    import torch

    from hfk import batch as B
    from hfk import forms, learned
    from hfk.operator import KernelOperator

    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def max_over_ranks(v):
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    t0 = time.perf_counter()
    problems, U2, U1, g, lift = _batch_setup(args.batch_count, rank=rank, world=world)
    res, jac = forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4)
    op = KernelOperator(res, jac, U2, jacobian="matrixfree")
    t_setup = time.perf_counter() - t0
    # warm-up (kernel attributes, handles, first-touch allocations) on a two-problem batch
    p0, W2, W1, gw, lw = _batch_setup(2)
    opw = KernelOperator(res, jac, W2, jacobian="matrixfree")
    B.newton_solve_batched(opw, _batch_solver(W2, W1, args.batch_precision), gw, BATCH_LOADS[:1], lift=lw)
    del opw
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    if world > 1:
        torch.cuda.synchronize()
        dist.barrier()
    with clocks:
        x, st = B.newton_solve_batched(op, _batch_solver(U2, U1, args.batch_precision), g, BATCH_LOADS, lift=lift)
    st.seconds = max_over_ranks(st.seconds)
    plain = {"seconds": st.seconds, "newton_sweeps": st.newton_sweeps, "krylov_sweeps": int(sum(st.krylov_sweeps)),
             "newton_iters_mean": float(st.newton_iters.mean()), "krylov_iters_mean": float(st.krylov_iters.mean()),
             "krylov_iters_max": int(st.krylov_iters.max()), "converged": int(st.converged.sum()), "pmg": st.pmg}
    # training pairs from the plain cycle at the converged state: right-hand sides of the next load
    # increment (the residual at load 1.1 from the lifted predictor) and a seeded N(0, 1) vector
    t1 = time.perf_counter()
    mf = op.allocate_jacobian(x)
    ls = _batch_solver(U2, U1, args.batch_precision)
    from hfk import solvers as S

    dv = torch.as_tensor(g, device="cuda")
    mf.prepare(x, dv)
    ns = S.numerical_setup(ls, mf)
    r = torch.zeros_like(x)
    op.residual(r, x + 0.1 * torch.as_tensor(lift, device="cuda"), 1.1 * dv)
    rhs = [-r, torch.as_tensor(np.random.default_rng(11).standard_normal(U2.nfree), device="cuda")]
    feats, targets = [], []
    for b in rhs:
        f, t = learned.collect_samples(ns.prec, mf, b, cycles=2)
        feats.append(f)
        targets.append(t)
    del ns
    feats, targets = torch.cat(feats), torch.cat(targets)
    net = learned.MLP(seed=4)
    loss = net.train(feats, targets, steps=3000, batch=8192, lr=1e-3)
    t_train = time.perf_counter() - t1
    del feats, targets
    holder = {}

    def attach(ns):
        learned.attach(ns.prec, net)
        holder["prec"] = ns.prec

    if world > 1:
        torch.cuda.synchronize()
        dist.barrier()
    x2, st2 = B.newton_solve_batched(op, _batch_solver(U2, U1, args.batch_precision), g, BATCH_LOADS, lift=lift,
                                     on_setup=attach)
    st2.seconds = max_over_ranks(st2.seconds)
    acc = learned.stats(holder["prec"]) if "prec" in holder else {}
    lrn = {"seconds": st2.seconds, "newton_sweeps": st2.newton_sweeps, "krylov_sweeps": int(sum(st2.krylov_sweeps)),
           "newton_iters_mean": float(st2.newton_iters.mean()), "krylov_iters_mean": float(st2.krylov_iters.mean()),
           "krylov_iters_max": int(st2.krylov_iters.max()), "converged": int(st2.converged.sum()),
           "corrections": acc, "train_seconds": t_train, "train_loss": loss,
           "solution_rel_diff_vs_plain": float(torch.linalg.norm(x2 - x) / torch.linalg.norm(x))}
    cpu = None if (args.no_cpu or rank != 0) else batch_cpu_sample(problems)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {"metric": f"seconds to 1e-8 for {args.batch_count} batched SVK Q2 Newton solves (plain p-MG)",
            "value": plain["seconds"], "unit": "s", "n_gpus": world, "steps": 1, "warmup": 1,
            "ms_per_step": plain["seconds"] * 1e3, "higher_is_better": False, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64" if args.batch_precision == "fp64" else "f64 outer / f32 cycle",
            "data": "synthetic",
            "config": {"workload": "batched Newton, SVK Q2 cubes n ~ U{8..24}, (lambda, mu) log-uniform, seed 4",
                       "problems": args.batch_count, "parallelism": f"problems sharded over {world} GPU(s)",
                       "free_dofs_rank0": U2.nfree, "coarse_free_dofs": U1.nfree,
                       "cells": U2.mesh.ncells, "loads": list(BATCH_LOADS), "setup_seconds": t_setup,
                       "levels": f"Q2 -> Q1 (Chebyshev 4; coarse: {BATCH_COARSE_STEPS} block-Jacobi CG steps per problem)",
                       "precision": args.batch_precision},
            "clocks": clocks.summary(), "plain": plain, "learned": lrn,
            "gain_learned_vs_plain": plain["seconds"] / lrn["seconds"]}
    if cpu is not None:
        all_free = sum(3 * (2 * q.n - 1) * (2 * q.n + 1) ** 2 for q in B.draw_batch(256, seed=4)[:args.batch_count])
        est = cpu["seconds_per_free_dof"] * all_free
        line["cpu_baseline"] = {"value": est, "unit": "s (extrapolated by free dofs)", "cores": cpu["cores"],
                                "kind": cpu["kind"], "sample": cpu["sample"]}
    print(json.dumps(line))


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        reference(a)
    elif a.batch:
        batch_main(a)
    elif a.oseen or a.assembly:
        oseen_main(a)
    elif a.vcycle:
        vcycle_main(a)
    else:
        engine(a)
