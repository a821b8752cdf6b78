"""Host-side unit test of the per-device caches (csrc/devcache.h): a kernel attribute raised on one
GPU is recorded for that GPU only, the limit only grows, and the setter runs under the lock (a
second thread never sees the new limit before the attribute is set). Compiled with g++ and run on
the CPU; no GPU involved."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "hyperfemkernels.jl_b200", "csrc")

PROGRAM = r"""
#include <atomic>
#include <cstdio>
#include <stdexcept>
#include <thread>
#include <vector>
#include "devcache.h"

#define CHECK(c) do { if (!(c)) { std::printf("FAILED: %s (line %d)\n", #c, __LINE__); return 1; } } while (0)

int main() {
  hfk::PerDeviceLimit lim;
  int sets = 0;
  auto set = [&] { ++sets; };
  // device 0 raised to 100 KB: device 1 still needs its own set
  CHECK(lim.raise(0, 100000, set) && sets == 1);
  CHECK(!lim.raise(0, 100000, set) && sets == 1);
  CHECK(!lim.raise(0, 50000, set) && sets == 1);     // never lowered
  CHECK(lim.get(0) == 100000);
  CHECK(lim.raise(1, 50000, set) && sets == 2);      // another GPU: set again
  CHECK(lim.get(1) == 50000 && lim.get(2) == 0);
  CHECK(lim.raise(1, 120000, set) && sets == 3 && lim.get(1) == 120000);
  CHECK(lim.raise(-1, 10, set) && lim.raise(64, 10, set) && sets == 5);  // uncached devices: always set
  // a failing setter leaves the record unchanged
  bool threw = false;
  try { lim.raise(3, 70000, [] { throw std::runtime_error("x"); }); } catch (const std::exception&) { threw = true; }
  CHECK(threw && lim.get(3) == 0);
  // threads: the attribute is set exactly once per (device, value), and a thread that returns
  // without setting never does so before the setting thread has finished set()
  hfk::PerDeviceLimit lim2;
  std::atomic<int> done{0}, calls{0}, early{0};
  std::vector<std::thread> th;
  for (int t = 0; t < 8; ++t)
    th.emplace_back([&] {
      bool ran = lim2.raise(5, 90000, [&] {
        ++calls;
        std::this_thread::sleep_for(std::chrono::milliseconds(20));
        done = 1;
      });
      if (!ran && !done) ++early;
    });
  for (auto& t : th) t.join();
  CHECK(calls == 1 && early == 0 && lim2.get(5) == 90000);
  hfk::PerDeviceValue sm;
  int reads = 0;
  CHECK(sm.get(0, [&] { ++reads; return 148; }) == 148);
  CHECK(sm.get(0, [&] { ++reads; return 7; }) == 148 && reads == 1);
  CHECK(sm.get(1, [&] { ++reads; return 132; }) == 132 && reads == 2);
  std::printf("ok\n");
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_per_device_limit_cache(tmp_path):
    src = tmp_path / "devcache_check.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "devcache_check"
    subprocess.run(["g++", "-std=c++17", "-O1", "-pthread", "-I", CSRC, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
