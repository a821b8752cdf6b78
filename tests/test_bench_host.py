"""Host logic of the benchmark script, no GPU: the clock record keeps only the nvidia-smi samples
taken inside the timed region (median SM clock, the highest maximum, the throttle reasons seen),
and says when none fell inside it."""
import datetime
import importlib.util
import os
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    return b


def _line(t, mhz, cap="Not Active", thermal="Not Active"):
    ts = datetime.datetime.fromtimestamp(t).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
    return f"{ts}, 0, {mhz}, 1965, 500.0, 0x0, Not Active, Not Active, {thermal}, {cap}"


def test_clock_samples_are_windowed_to_the_timed_region():
    c = _bench().ClockSampler(0)
    now = time.time()
    c.lines = [_line(now - 1.0, 345, thermal="Active"),  # idle, before: ignored with its reason
               _line(now + 0.1, 1965), _line(now + 0.3, 1950, cap="Active"), _line(now + 0.5, 1965),
               _line(now + 2.0, 300)]  # after: ignored
    c.t0, c.t1 = now, now + 1.0
    s = c.summary()
    assert s["samples"] == 3 and s["window"] == "timed region"
    assert s["sm_mhz"] == 1965 and s["sm_max_mhz"] == 1965
    assert s["reasons"] == ["sw_power_cap"]


def test_clock_summary_without_samples_in_the_window():
    c = _bench().ClockSampler(0)
    now = time.time()
    c.lines = [_line(now - 1.0, 1965), "garbage line", ""]
    c.t0, c.t1 = now, now + 0.01
    s = c.summary()
    assert s["samples"] == 1 and s["window"].startswith("whole sampler run")
    c.lines = []
    assert c.summary()["reasons"] == ["unsampled"]


def test_multi_rank_slabs_of_the_headline_configuration():
    # what each of N ranks assembles in `bench.py --gpus N` (owner computes on z-slabs of the
    # 20 x 10 x 10N mesh): about 2 000 cells and at most one ghost layer on each side; the owned free
    # dofs of the ranks partition the job's free dofs
    import numpy as np

    from hfk import distributed as D

    b = _bench()
    for world in (2, 4):
        G = b.c0_space(10 * world)
        owned = np.zeros(G.nfree, dtype=np.int32)
        for rank in range(world):
            V, x, nfree_job, ncells = b.c0_problem(world, rank)
            assert nfree_job == G.nfree
            assert 2000 <= ncells <= 2000 + 2 * 200
            assert len(x) == V.nfree and np.isfinite(x).all()
            sub = D.Subdomain(G, D.slab_partition(G.mesh, world), rank, ghost=True)
            assert V.nfree == len(sub.free_global) and len(sub.cells) == ncells
            owned[sub.free_global[sub.owned]] += 1
        assert (owned == 1).all()
