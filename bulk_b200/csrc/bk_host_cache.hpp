// bk_host_cache.hpp -- per-device, per-call-site one-time set-up on the host.
//
// Kernel attributes (the dynamic shared-memory opt-in, the carveout) are set
// on the kernel as seen by one device's context, and occupancy-derived
// numbers (resident CTAs) are properties of one device.  A cache of either
// must therefore be keyed by device, not by host thread: a thread that calls
// on GPU 0 and then on GPU 1 must set the opt-in again on GPU 1.
//
// PerDevice<T>::get(dev, make) runs make(&value) the first time a device is
// seen by this call site (each distinct `Site` type: in practice a lambda or
// a kernel-specific tag), caches the value only when make() returns 0, and
// hands back the cached value afterwards.  It is thread-safe: the fast path
// is one acquire load; set-up runs under a mutex, once per device.  Plain
// C++ (no CUDA headers), so it is unit-tested on the CPU.
#pragma once

#include <atomic>
#include <mutex>

namespace bk {
namespace host {

constexpr int kMaxCachedDevices = 64;

template <typename T, typename Site>
struct PerDevice {
  // Returns make()'s status on failure (nothing cached, the next call tries
  // again), 0 on success with *out set, and bad_device for a device index
  // outside [0, kMaxCachedDevices).
  template <typename Make>
  static int get(int dev, T *out, Make &&make, int bad_device) {
    if (dev < 0 || dev >= kMaxCachedDevices) return bad_device;
    Slot &s = slots()[dev];
    if (!s.ready.load(std::memory_order_acquire)) {
      std::lock_guard<std::mutex> g(mutex());
      if (!s.ready.load(std::memory_order_relaxed)) {
        T v{};
        const int st = make(&v);
        if (st != 0) return st;
        s.value = v;
        s.ready.store(true, std::memory_order_release);
      }
    }
    *out = s.value;
    return 0;
  }
  // Test hook: how many devices this call site has set up.
  static int ready_count() {
    int c = 0;
    for (int d = 0; d < kMaxCachedDevices; ++d) c += slots()[d].ready.load(std::memory_order_acquire) ? 1 : 0;
    return c;
  }

 private:
  struct Slot {
    std::atomic<bool> ready{false};
    T value{};
  };
  static Slot *slots() {
    static Slot s[kMaxCachedDevices];
    return s;
  }
  static std::mutex &mutex() {
    static std::mutex m;
    return m;
  }
};

}  // namespace host
}  // namespace bk
