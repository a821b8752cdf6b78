// Per-device caches of the engine's one-time device settings (plain C++, no CUDA: unit-tested on the
// host).
#pragma once
#include <cstddef>
#include <mutex>

namespace hfk {

// A kernel's raised dynamic shared-memory limit, per device. cudaFuncSetAttribute acts on the
// current device only, so a limit raised on one GPU says nothing about another GPU the process
// drives. The limit only grows, and the attribute is set under the lock: a thread about to launch
// with a large limit must not see it lowered by a thread that needs less, nor launch before the
// attribute it relies on has been set.
class PerDeviceLimit {
 public:
  static constexpr int kMaxDevices = 64;

  // Make sure device `dev` has a limit of at least `want`: calls set() (which sets the attribute
  // on the current device and may throw) when the recorded limit is lower, then records `want`.
  // Returns whether set() ran. Devices outside [0, kMaxDevices) are not cached: set() always runs.
  template <typename Set>
  bool raise(int dev, size_t want, Set set) {
    if (dev < 0 || dev >= kMaxDevices) {
      set();
      return true;
    }
    std::lock_guard<std::mutex> lock(mu_);
    if (want <= v_[dev]) return false;
    set();
    v_[dev] = want;
    return true;
  }

  size_t get(int dev) const { return dev >= 0 && dev < kMaxDevices ? v_[dev] : 0; }

 private:
  size_t v_[kMaxDevices] = {};
  std::mutex mu_;
};

// A per-device integer property read once (the SM count): get(dev, read) calls read() the first
// time for each device.
class PerDeviceValue {
 public:
  template <typename Read>
  int get(int dev, Read read) {
    if (dev < 0 || dev >= PerDeviceLimit::kMaxDevices) return read();
    std::lock_guard<std::mutex> lock(mu_);
    if (!v_[dev]) v_[dev] = read();
    return v_[dev];
  }

 private:
  int v_[PerDeviceLimit::kMaxDevices] = {};
  std::mutex mu_;
};

}  // namespace hfk
