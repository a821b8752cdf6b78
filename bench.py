"""Benchmark of the hot path: the FP64 CSC Jacobian assembly of the SVK Q2 20x10x10 cube.

One step = one `jacobian!` (src/assembly.jl:918-927): zero-fill of the CSC values, the element
Jacobians of all 2 000 Q2 cells (27 Gauss points each) and their scatter into the reference's
CSC pattern (52 077 free dofs, 8 990 127 nonzeros), FP64. `value` = free dofs / step time with
the state resident in HBM (GDOF/s); `e2e` runs the same assembly through the public C ABI with
page-locked host buffers (state copied in, CSC values copied out every step). Prints one JSON line
(rank 0). `extra` carries the other configurations: the matrix-free J*v on Q2 64^3 (with its own
e2e, roofline and full-size CPU comparison), the other J*v sizes, the Oseen P2-P1 assembly and the
p-multigrid Newton solve.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

`--impl reference` times the CPU restatement of the reference algorithm (the oracle: the
reference's matrix-product element Jacobian with register-tiled products and the colour loop,
OpenMP over all host cores) on the same configuration.

With N > 1 GPUs (torchrun, one process per GPU) each rank assembles the owned rows of one slab of
a 20 x 10 x 10N mesh cut along z (owner computes: the rank also assembles the cells that touch its
dofs, so no data is exchanged); value = all ranks' free dofs / the slowest rank's step time.
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

METRIC = "Q2 SVK Jacobian GDOF/s"
UNIT = "GDOF/s"
C0_CELLS = (20, 10, 10)
WORKLOAD = ("CSC Jacobian assembly (jacobian!: zero-fill, element Jacobians, scatter), SVK lambda=2 mu=1, "
            "Q2 hexahedra 20x10x10 on the unit cube, Gauss degree 4 (27 points), x=0 clamped, x=1 displaced 0.05 "
            "(open faces), FP64")
# FP64 flops of one Q2 element Jacobian, the reference's own count (benchmark/roofline.jl:65-74):
# block products G*B, 3*3*2*27*27*27*3, plus G at the points, 3*3*3*27*27*3*2
C0_FLOPS_PER_CELL = 3 * 3 * 2 * 27 * 27 * 27 * 3 + 3 * 3 * 3 * 27 * 27 * 3 * 2
L2_FLUSH_BYTES = 256 << 20  # twice the B200's 126 MB L2
JV_CELLS = 64


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-extra", action="store_true", help="skip the secondary measurements")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--batch", action="store_true",
                    help="the batched workload instead: 256 SVK Q2 Newton solves (plain p-MG vs learned correction)")
    ap.add_argument("--batch-count", type=int, default=256)
    ap.add_argument("--batch-precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--oseen", type=int, default=0, metavar="N",
                    help="only the Oseen P2-P1 assembly on the N^3 tetrahedral cube (the secondary case; 0 = off)")
    ap.add_argument("--launch", default="auto", choices=["auto", "line2", "line4", "point", "tensor"],
                    help="launch shape of the J*v in --jv (auto: the autotuner's; a fixed one for profiling, "
                         "where the profiler's overhead would skew the autotuner's timings)")
    ap.add_argument("--jv", type=int, default=0, metavar="N",
                    help="only the matrix-free Q2 J*v on the N^3 cube (the case for profiling its kernel)")
    ap.add_argument("--assembly", action="store_true",
                    help="only the Q2 SVK 20x10x10 residual + CSC Jacobian, a few steps (the case for profiling)")
    ap.add_argument("--newton", type=int, default=0, metavar="N",
                    help="only the matrix-free Newton + p-MG solve on the Q4 N^3 cube (FP64 and mixed)")
    ap.add_argument("--vcycle", type=int, default=0, metavar="K",
                    help="only K V-cycles of the Q4 16^3 p-multigrid 4 -> 2 -> 1 (the Newton case's preconditioner)")
    return ap.parse_args()


def svk_dirichlet():
    return [lambda x: 0 * x, lambda x: np.tile([0.05, 0.0, 0.0], (len(x), 1))]


def svk_state(V, seed=0):
    """u = 0.05 x e_x + U(-1e-3, 1e-3) on the free dofs (seeded)."""
    rng = np.random.default_rng(seed)
    x, _ = V.interpolate(lambda p: np.stack([0.05 * p[:, 0], 0 * p[:, 0], 0 * p[:, 0]], axis=1))
    return x + rng.uniform(-1e-3, 1e-3, V.nfree)


def c0_space(nz=10):
    """The assembly configuration: Q2 vector Lagrange on a 20 x 10 x nz cube of the unit cube, Gridap's
    open face tags (face interiors fixed): 52 077 free dofs at nz = 10."""
    from hfk.fespace import CartesianMesh, VectorLagrangeSpace

    m = CartesianMesh((C0_CELLS[0], C0_CELLS[1], nz))
    return VectorLagrangeSpace(m, 2, ("x0", "x1"), g=svk_dirichlet(), open_faces=True)


def build_case(n, order=2, seed=0):
    """The matrix-free configuration: Q_order on the n^3 cube (closed faces), the SVK state and a
    seeded N(0, 1) increment."""
    from hfk.fespace import CartesianMesh, VectorLagrangeSpace

    V = VectorLagrangeSpace(CartesianMesh((n, n, n)), order, ("x0", "x1"), g=svk_dirichlet())
    x = svk_state(V, seed)
    dx = np.random.default_rng(seed + 1).standard_normal(V.nfree)
    return V, x, dx


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms; the summary keeps the samples
    taken inside the window marked by ``start()`` / ``stop()`` (the timed region)."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.t0 = self.t1 = None

    def start(self):
        self.t0 = time.time()

    def stop(self):
        self.t1 = time.time()

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
        import datetime

        rows = []
        for l in self.lines:
            f = [s.strip() for s in l.split(",")]
            if len(f) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                rows.append((ts, float(f[2]), float(f[3]), f[6:10]))
            except ValueError:
                continue
        inside = [r for r in rows if self.t0 is not None and self.t1 is not None and self.t0 <= r[0] <= self.t1]
        window = "timed region" if inside else "whole sampler run (no sample fell inside the timed region)"
        use = inside or rows
        if not use:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = {nm for r in use for nm, v in zip(names, r[3]) if v.lower() == "active"}
        return {"sm_mhz": statistics.median(r[1] for r in use), "sm_max_mhz": max(r[2] for r in use),
                "reasons": sorted(reasons), "samples": len(use), "window": window}


def jv_flops_per_cell(Q, P):
    """FP64 flops of one recompute J*v cell: 3 interpolations (the components of dx), 3
    contractions, the pointwise law (F is stored, not interpolated)."""
    interp = 2 * (2 * P * Q**3 + 3 * P**2 * Q**2 + 3 * P**3 * Q)  # x, y, z sweeps (FMA = 2)
    contract = 2 * (3 * P**3 * Q + 3 * P**2 * Q**2 + 2 * P * Q**3)
    pointwise = P**3 * (2 * (27 + 27 + 18 + 27 + 27 + 27 + 27) + 60)  # grads, F'F, F'Hd, Hd S, F W, pull-back
    return 3 * interp + 3 * contract + pointwise


def hbm_peak():
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Timer:
    """Device timing on one stream: `steps(fn, K, W)` runs W untimed calls, then K calls each between
    its own pair of CUDA events (an L2 flush, untimed, before every call when `flush` is set), with a
    synchronize (and a barrier across ranks) on both sides of the timed calls; returns the summed
    event time in ms, the max over ranks."""

    def __init__(self, torch, dev, stream, world=1, flush=True):
        self.torch, self.dev, self.stream, self.world = torch, dev, stream, world
        self.buf = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev) if flush else None

    def _sync(self):
        self.torch.cuda.synchronize()
        if self.world > 1:
            import torch.distributed as dist

            dist.barrier()
            self.torch.cuda.synchronize()

    def steps(self, fn, k, w, on_start=None, on_stop=None):
        torch = self.torch
        for _ in range(w):
            if self.buf is not None:
                self.buf.zero_()
            fn()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
        self._sync()
        if on_start:
            on_start()
        for e0, e1 in ev:
            if self.buf is not None:
                self.buf.zero_()
            e0.record(self.stream)
            fn()
            e1.record(self.stream)
        self._sync()
        if on_stop:
            on_stop()
        ms = sum(e0.elapsed_time(e1) for e0, e1 in ev)
        return self.max_over_ranks(ms)

    def max_over_ranks(self, v):
        if self.world == 1:
            return v
        import torch.distributed as dist

        t = self.torch.tensor([v], dtype=torch_float64(self.torch), device=self.dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(self, v):
        if self.world == 1:
            return v
        import torch.distributed as dist

        t = self.torch.tensor([v], dtype=torch_float64(self.torch), device=self.dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())


def torch_float64(torch):
    return torch.float64


def c0_problem(world, rank):
    """(space the rank assembles, its state, free dofs of the whole job, cells it assembles): the
    C0 space at one rank; at N ranks, rank r's ghost subdomain of the 20 x 10 x 10N mesh."""
    if world == 1:
        V = c0_space()
        return V, svk_state(V), V.nfree, V.mesh.ncells
    from hfk import distributed as D

    G = c0_space(10 * world)
    xg = svk_state(G)
    sub = D.Subdomain(G, D.slab_partition(G.mesh, world), rank, ghost=True)
    return sub.space, sub.restrict(xg), G.nfree, len(sub.cells)


def engine(args):
    import torch
    import torch.distributed as dist

    from hfk import _lib, forms
    from hfk.operator import KernelOperator

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    T = Timer(torch, dev, stream, world)

    # ---- headline: device-resident FP64 CSC Jacobian assembly (C0) ----
    V, x, nfree_job, ncells = c0_problem(world, rank)
    op = KernelOperator(forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4), V)
    op.problem.set_stream(stream.cuda_stream)
    nnz = op.sparsity_pattern().nnz
    xd = torch.from_numpy(x).to(dev)
    dd = torch.from_numpy(np.ascontiguousarray(V.dirichlet_values)).to(dev)
    nz = torch.zeros(nnz, dtype=torch.float64, device=dev)
    h = op.problem.h

    def step():
        _lib.call("hfk_jacobian", h, _lib.ptr(xd), _lib.ptr(dd), _lib.ptr(nz))

    step()
    torch.cuda.synchronize()
    l0 = op.problem.launches()
    with ClockSampler(local) as clk:
        ms = T.steps(step, args.steps, args.warmup, on_start=clk.start, on_stop=clk.stop)
    launches = (op.problem.launches() - l0) // (args.steps + args.warmup) * args.steps
    # the assembly kernel's own time, in a separate loop (its launch bracketed by events on the
    # problem's stream, so that the timed steps above carry no extra event records)
    op.problem.set_timing(True)
    T.steps(step, min(args.steps, 500), 0)
    k_ms, k_n = op.problem.kernel_time()
    op.problem.set_timing(False)
    ms_step = ms / args.steps
    value = nfree_job / (ms_step * 1e-3) / 1e9
    clocks = clk.summary()
    kernel_ms = T.max_over_ranks(k_ms / max(k_n, 1))

    # ---- e2e: the same assembly through the C ABI with page-locked host buffers ----
    xh = torch.from_numpy(x).pin_memory()
    dh = torch.from_numpy(np.ascontiguousarray(V.dirichlet_values)).pin_memory()
    nzh = torch.zeros(nnz, dtype=torch.float64).pin_memory()

    def step_e2e():
        _lib.call("hfk_jacobian", h, _lib.ptr(xh), _lib.ptr(dh), _lib.ptr(nzh))

    k_e2e = max(3, args.steps // 4)
    ms_e2e = T.steps(step_e2e, k_e2e, 2) / k_e2e
    e2e_err = float(torch.linalg.norm(nzh.to(dev) - nz) / torch.linalg.norm(nz))
    e2e = {"value": nfree_job / (ms_e2e * 1e-3) / 1e9, "unit": UNIT,
           "h2d_bytes_per_step": 8 * (V.nfree + V.ndir), "d2h_bytes_per_step": 8 * nnz, "ms_per_step": ms_e2e,
           "mode": "one synchronous hfk_jacobian per step: state (free + Dirichlet values) H2D, CSC values D2H",
           "rel_diff_vs_device_resident": e2e_err}

    # ---- roofline of the dominant kernel (the element Jacobian + scatter kernel) ----
    dmma, dfma = ctypes.c_double(), ctypes.c_double()
    _lib.call("hfk_device_peak_fp64", ctypes.byref(dmma), ctypes.byref(dfma))
    flops = C0_FLOPS_PER_CELL * ncells
    peak = max(dmma.value, dfma.value)
    achieved = flops / (kernel_ms * 1e-3) / 1e12
    # DRAM bytes (read + write) of one launch of the assembly kernel on this configuration (ncu
    # dram__bytes_read.sum + dram__bytes_write.sum, one launch), scaled by the cells of this rank
    traffic = C0_TRAFFIC_BYTES * ncells / 2000 if C0_TRAFFIC_BYTES else None
    alg_bytes = 8 * nnz + 4 * 81 * 81 * ncells + 4 * 81 * ncells + 8 * (V.nfree + V.ndir)
    roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": traffic,
                "kernel": "jacobian_kernel_sym27<TP> (FP64 FMA: symmetric element blocks, sum-factorised "
                          "contraction, persistent CTAs)",
                "kernel_ms": kernel_ms, "flops_per_launch": flops,
                "flops_source": "benchmark/roofline.jl:65-74: 1 180 980 FP64 flops per Q2 cell (products + G), the "
                                "reference's dense formulation; the kernel executes about 0.37 MFLOP per cell "
                                "(symmetric blocks only, sum-factorised contraction)",
                "peak_source": "FP64 measured in-process on this GPU (hfk_device_peak_fp64: mma m8n8k4 f64 "
                               f"{dmma.value:.1f} TFLOP/s, DFMA {dfma.value:.1f} TFLOP/s); the measured-peaks file "
                               "has no FP64 figure",
                "algorithmic_bytes_per_launch": alg_bytes,
                "hbm_frac": alg_bytes / (kernel_ms * 1e-3) / 1e9 / hbm_peak()[0],
                "traffic_source": "ncu one launch, this configuration" if traffic else None}

    extra = {}
    if not args.no_extra and world == 1:
        extra.update(assembly_extra(torch, dev, stream, op, xd, dd, nz, T))
        del op
        torch.cuda.empty_cache()
        extra.update(jv_headline_case(torch, dev, stream, T, cpu=not args.no_cpu))
        extra.update(jv_sizes_case(torch, dev, stream, T.steps))
        extra.update(oseen_case(torch, dev, stream, T.steps))
        extra.update(newton_case())

    cpu = c0_cpu_baseline(budget_s=15.0) if world == 1 and not args.no_cpu else None
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": WORKLOAD, "cells_per_gpu": ncells, "free_dofs": nfree_job, "nnz_rank0": int(nnz),
                           "quadrature_points_per_cell": 27, "qps": 27 * ncells * world / (ms_step * 1e-3),
                           "parallelism": "1 GPU" if world == 1 else
                           f"owner-computes z-slabs of a 20x10x{10 * world} mesh over {world} GPUs, no exchange",
                           "l2": f"flushed before every timed step ({L2_FLUSH_BYTES >> 20} MB written; the step "
                                 "touches about 125 MB)",
                           "state": "u = 0.05 x e_x + U(-1e-3, 1e-3) on the free dofs, seed 0"},
                "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks, "roofline": roofline,
                "cpu_baseline": cpu, "extra": extra}
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# DRAM traffic of one jacobian_kernel_sym27<TP> launch on the 20x10x10 case (ncu, one launch:
# 125 709 312 B read + 18 921 472 B written); None = not captured
C0_TRAFFIC_BYTES = 144630784


def assembly_extra(torch, dev, stream, op, xd, dd, nz, T):
    """Secondary C0 figures: the residual, the bit-reproducible colour-by-colour scatter, and the
    relative difference of the CSC values from the CPU restatement."""
    from hfk import _lib

    V = op.U
    h = op.problem.h
    b = torch.zeros(V.nfree, dtype=torch.float64, device=dev)
    ms_r = T.steps(lambda: _lib.call("hfk_residual", h, _lib.ptr(xd), _lib.ptr(dd), _lib.ptr(b)), 20, 3) / 20
    op.problem.set_scatter("coloured")
    ms_jc = T.steps(lambda: _lib.call("hfk_jacobian", h, _lib.ptr(xd), _lib.ptr(dd), _lib.ptr(nz)), 20, 3) / 20
    nz_c = nz.cpu().numpy().copy()
    op.problem.set_scatter("auto")
    _lib.call("hfk_jacobian", h, _lib.ptr(xd), _lib.ptr(dd), _lib.ptr(nz))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from hfk.fespace import Quadrature

    orc = O.OracleProblem(V, Quadrature.gauss(4))
    orc.pattern()
    x = xd.cpu().numpy()
    d = np.ascontiguousarray(V.dirichlet_values)
    ref = orc.jacobian_values(x, d)
    rref = orc.residual(x, d)
    got = nz.cpu().numpy()
    return {"assembly_q2_20x10x10": {
        "residual_ms": ms_r, "jacobian_coloured_ms": ms_jc,
        "rel_diff_vs_cpu": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
        "rel_diff_coloured_vs_cpu": float(np.linalg.norm(nz_c - ref) / np.linalg.norm(ref)),
        "residual_rel_diff_vs_cpu": float(np.linalg.norm(b.cpu().numpy() - rref) / np.linalg.norm(rref))}}


def jv_headline_case(torch, dev, stream, T, n=JV_CELLS, cpu=True, launch="auto"):
    """The matrix-free configuration: FP64 recompute J*v on the Q2 n^3 cube (6.34 M free dofs at
    n = 64) with inputs resident in HBM, through the C ABI with host vectors (e2e), the roofline of
    its cell kernel, the FP32 and the stored-tangent products, and the CPU restatement's
    stored-tangent product on the same mesh."""
    from hfk import _lib, forms
    from hfk.operator import KernelOperator, MatrixFreeJacobian

    V, x, dx = build_case(n)
    op = KernelOperator(forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4), V, jacobian="matrixfree")
    op.problem.set_stream(stream.cuda_stream)
    nfree = V.nfree
    xd = torch.from_numpy(x).to(dev)
    dd = torch.from_numpy(np.ascontiguousarray(V.dirichlet_values)).to(dev)
    dxd = torch.from_numpy(dx).to(dev)
    yd = torch.zeros(nfree, dtype=torch.float64, device=dev)
    if launch != "auto":
        op.problem.set_scatter("atomic")
        if launch in ("point", "tensor"):
            op.problem.set_launch(launch, 0)
        else:
            op.problem.set_launch("line", int(launch[-1]))
    mf = MatrixFreeJacobian(op, "recompute")
    mf.prepare(xd, dd)
    h = op.problem.h

    def step():
        _lib.call("hfk_mf_apply", h, _lib.ptr(dxd), _lib.ptr(yd))

    step()
    op.problem.set_timing(True)
    steps = 100
    ms = T.steps(step, steps, 3) / steps
    k_ms, k_n = op.problem.kernel_time()
    op.problem.set_timing(False)
    kernel_ms = k_ms / max(k_n, 1)
    ncells = V.mesh.ncells
    alg_bytes = 4 * V.ndl * ncells + 8 * nfree * 3 + 72 * 27 * ncells + 81 * ncells
    hbm, src = hbm_peak()
    flops = jv_flops_per_cell(3, 3) * ncells
    out = {"free_dofs": nfree, "ms": ms, "gdofs": nfree / (ms * 1e-3) / 1e9, "kernel_ms": kernel_ms,
           "roofline": {"bound": "hbm", "achieved": alg_bytes / (kernel_ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                        "frac": alg_bytes / (kernel_ms * 1e-3) / 1e9 / hbm, "peak_source": src,
                        "bytes_per_launch": alg_bytes, "fp64_tflops": flops / (kernel_ms * 1e-3) / 1e12}}
    # e2e: a stream of host vectors in one hfk_mf_apply_many call (the copies of one vector overlap
    # the product of the next), and one synchronous hfk_mf_apply per vector
    ring = 4
    dxh = [torch.from_numpy(dx).pin_memory() for _ in range(ring)]
    yh = [torch.zeros(nfree, dtype=torch.float64).pin_memory() for _ in range(ring)]
    k_e2e = 60
    pin = (ctypes.c_void_p * k_e2e)(*[dxh[i % ring].data_ptr() for i in range(k_e2e)])
    pout = (ctypes.c_void_p * k_e2e)(*[yh[i % ring].data_ptr() for i in range(k_e2e)])
    ms_many = T.steps(lambda: _lib.call("hfk_mf_apply_many", h, k_e2e, ctypes.cast(pin, ctypes.c_void_p),
                                        ctypes.cast(pout, ctypes.c_void_p)), 1, 1) / k_e2e
    ms_single = T.steps(lambda: _lib.call("hfk_mf_apply", h, _lib.ptr(dxh[0]), _lib.ptr(yh[0])), 20, 2) / 20
    out["e2e"] = {"value": nfree / (ms_many * 1e-3) / 1e9, "unit": UNIT, "h2d_bytes_per_step": 8 * nfree,
                  "d2h_bytes_per_step": 8 * nfree, "ms_per_step": ms_many,
                  "mode": f"{k_e2e} host vectors per hfk_mf_apply_many call (pinned ring of {ring})",
                  "single_call_gdofs": nfree / (ms_single * 1e-3) / 1e9,
                  "rel_diff_vs_device_resident": float(torch.linalg.norm(yh[0].to(dev) - yd) / torch.linalg.norm(yd))}
    # FP32 and the stored (reference) formulation
    dx32 = dxd.float()
    y32 = torch.zeros(nfree, dtype=torch.float32, device=dev)
    ms32 = T.steps(lambda: _lib.call("hfk_mf_apply_f32", h, _lib.ptr(dx32, np.float32), _lib.ptr(y32, np.float32)),
                   50, 3) / 50
    step()
    torch.cuda.synchronize()
    out["fp32"] = {"ms": ms32, "gdofs": nfree / (ms32 * 1e-3) / 1e9,
                   "rel_err_vs_fp64": float(torch.linalg.norm(y32.double() - yd) / torch.linalg.norm(yd))}
    out["autotuned_launch_shape"] = {k: op.problem.tuning(*k.split("_")) for k in ("jv_fp64", "jv_fp32")}
    y64 = yd.cpu().numpy()
    mfs = MatrixFreeJacobian(op, "stored")
    mfs.prepare(xd, dd)
    ms_s = T.steps(step, 30, 3) / 30
    stored_bytes = 8 * 91 * 27 * ncells + 8 * nfree * 2 + 4 * V.ndl * ncells
    out["stored_fp64"] = {"ms": ms_s, "gdofs": nfree / (ms_s * 1e-3) / 1e9,
                          "hbm_frac": stored_bytes / (ms_s * 1e-3) / 1e9 / hbm}
    del mf, mfs, op, xd, dd, dxd, yd, dx32, y32
    torch.cuda.empty_cache()
    if cpu:
        # the CPU restatement of the reference's mul! (stored tangents, OpenMP, all host cores) on
        # the same mesh, state and increment
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        from hfk.fespace import Quadrature

        p = O.OracleProblem(V, Quadrature.gauss(4))
        t0 = time.perf_counter()
        p.mf_prepare(x, V.dirichlet_values)
        t_prep = time.perf_counter() - t0
        yr = p.mf_apply(dx)
        yw = np.zeros_like(yr)  # written in place, as mul!(y, J, dx) does
        p.mf_apply(dx, out=yw)
        ts = []
        for _ in range(5):
            t0 = time.perf_counter()
            p.mf_apply(dx, out=yw)
            ts.append(time.perf_counter() - t0)
        t = min(ts)
        out["cpu"] = {"gdofs": nfree / t / 1e9, "ms": 1e3 * t, "prepare_ms": 1e3 * t_prep, "cores": O.lib().o_max_threads(),
                      "kind": "port", "rel_diff_engine_vs_cpu": float(np.linalg.norm(y64 - yr) / np.linalg.norm(yr)),
                      "sample": f"full Q2 {n}^3 ({nfree} free dofs), stored-tangent mul! into one preallocated vector, best of 5"}
        del p
    return {f"jv_q2_{n}": out}


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
    nzw = orc.jacobian_values()  # then assembled in place, as jacobian!(A, ...) does
    t0 = time.perf_counter()
    orc.jacobian_values(out=nzw)
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


def profile_main(args):
    """One case alone, one JSON line, for profiling its kernel: ``--assembly`` (the Q2 SVK 20x10x10
    residual + CSC Jacobian, 20 steps each), ``--jv N`` (the Q2 N^3 matrix-free product, FP64 and
    FP32) or ``--oseen N`` (the Oseen P2-P1 assembly on the N^3 tetrahedral cube)."""
    import torch

    from hfk import _lib, forms
    from hfk.operator import KernelOperator

    dev = torch.device("cuda")
    stream = torch.cuda.current_stream()
    T = Timer(torch, dev, stream, 1, flush=False)
    if args.assembly:
        V = c0_space()
        x = svk_state(V)
        op = KernelOperator(forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4), V)
        op.problem.set_stream(stream.cuda_stream)
        nnz = op.sparsity_pattern().nnz
        xd = torch.from_numpy(x).to(dev)
        dd = torch.from_numpy(np.ascontiguousarray(V.dirichlet_values)).to(dev)
        nz = torch.zeros(nnz, dtype=torch.float64, device=dev)
        b = torch.zeros(V.nfree, dtype=torch.float64, device=dev)
        def jac():
            _lib.call("hfk_jacobian", op.problem.h, _lib.ptr(xd), _lib.ptr(dd), _lib.ptr(nz))

        # both element-block kernels: the FP64 FMA one (default) and the FP64 tensor-core one
        out = {"case": "assembly Q2 SVK 20x10x10", "nnz": int(nnz)}
        vals = {}
        for kern in ("fma", "tensor"):
            op.problem.set_assembly_kernel(kern)
            jac()
            op.problem.set_timing(True)
            ms_j = T.steps(jac, 20, 3) / 20
            k_ms, k_n = op.problem.kernel_time()
            op.problem.set_timing(False)
            vals[kern] = nz.cpu().numpy().copy()
            out[f"jacobian_ms_{kern}"] = ms_j
            out[f"kernel_ms_{kern}"] = k_ms / max(k_n, 1)
        op.problem.set_assembly_kernel("fma")
        out["rel_diff_fma_vs_tensor"] = float(np.linalg.norm(vals["fma"] - vals["tensor"]) /
                                              np.linalg.norm(vals["tensor"]))
        out["residual_ms"] = T.steps(lambda: _lib.call("hfk_residual", op.problem.h, _lib.ptr(xd), _lib.ptr(dd),
                                                       _lib.ptr(b)), 20, 3) / 20
    elif args.jv:
        out = jv_headline_case(torch, dev, stream, T, n=args.jv, cpu=False, launch=args.launch)
    else:
        out = oseen_case(torch, dev, stream, T.steps, n=args.oseen, cpu_n=min(args.oseen, 8))
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
                      "ms_per_cycle": e0.elapsed_time(e1) / args.vcycle, "update_stats_ms": st.stats()}))


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
    return {f"newton_pmg_svk_q4_{n}": {"free_dofs": Vs[0].nfree, "coarse_free_dofs": Vs[2].nfree,
                                      "levels": "Q4 -> Q2 -> Q1 (assembled, Cholesky over the band)",
                                     "loads": list(loads), **out}}


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def c0_oracle():
    """The CPU restatement on the C0 configuration: (oracle problem, state, Dirichlet values, free dofs)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from hfk.fespace import Quadrature

    V = c0_space()
    orc = O.OracleProblem(V, Quadrature.gauss(4))
    orc.pattern()
    return O, orc, svk_state(V), np.ascontiguousarray(V.dirichlet_values), V.nfree


def c0_cpu_baseline(budget_s=15.0):
    """The CPU restatement (jacobian!: zero-fill, matrix-product element Jacobians, colour loop,
    OpenMP on all host cores) on the full C0 configuration, repeated until ``budget_s``."""
    O, orc, x, d, nfree = c0_oracle()
    out = orc.jacobian_values(x, d)  # assembled in place from here on, as jacobian!(A, ...) does
    t0 = time.perf_counter()
    k = 0
    ts = []
    while True:
        t1 = time.perf_counter()
        orc.jacobian_values(x, d, out=out)
        ts.append(time.perf_counter() - t1)
        k += 1
        if time.perf_counter() - t0 > budget_s or k >= 200:
            break
    t = statistics.median(ts)
    return {"value": nfree / t / 1e9, "unit": UNIT, "cores": O.lib().o_max_threads(), "kind": "port",
            "ms_per_assembly": 1e3 * t,
            "sample": f"the full configuration (Q2 SVK 20x10x10, {nfree} free dofs), {k} CSC Jacobian assemblies, "
                      "median"}


def reference(args):
    """The reference arm: the CPU restatement of the reference's jacobian! (the oracle, all host
    cores) on the headline configuration, one assembly per step; rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    O, orc, x, d, nfree = c0_oracle()
    out = orc.jacobian_values(x, d)  # assembled in place from here on, as jacobian!(A, ...) does
    for _ in range(max(1, args.warmup)):
        orc.jacobian_values(x, d, out=out)
    steps = min(args.steps, 200)
    t0 = time.perf_counter()
    for _ in range(steps):
        orc.jacobian_values(x, d, out=out)
    t = (time.perf_counter() - t0) / steps
    value = nfree / t / 1e9
    cores = O.lib().o_max_threads()
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "cells": 2000, "free_dofs": nfree, "quadrature_points_per_cell": 27},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"the full configuration, {steps} CSC Jacobian assemblies into one "
                                       "preallocated array (zero-fill included), OpenMP on all host cores"},
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
        clocks.start()
        x, st = B.newton_solve_batched(op, _batch_solver(U2, U1, args.batch_precision), g, BATCH_LOADS, lift=lift)
        clocks.stop()
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
    elif a.oseen or a.assembly or a.jv:
        profile_main(a)
    elif a.vcycle:
        vcycle_main(a)
    elif a.newton:
        print(json.dumps(newton_case(n=a.newton)))
    else:
        engine(a)
