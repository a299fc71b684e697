// Unit check of bk::host::PerDevice (bulk_b200/csrc/bk_host_cache.hpp), the
// per-device cache that guards kernel-attribute set-up: set-up runs once per
// (device, call site), failures are not cached, and concurrent first calls
// run it once.  Plain C++; prints "ok" and exits 0 on success.
#include <atomic>
#include <cstdio>
#include <thread>
#include <vector>

#include "bk_host_cache.hpp"

using bk::host::PerDevice;

struct SiteA {};
struct SiteB {};

#define CHECK(c)                                                   \
  do {                                                             \
    if (!(c)) {                                                    \
      std::printf("FAILED line %d: %s\n", __LINE__, #c);           \
      return 1;                                                    \
    }                                                              \
  } while (0)

int main() {
  std::atomic<int> calls{0};
  auto make = [&](int dev) {
    return [&, dev](long *v) -> int {
      calls.fetch_add(1);
      *v = 1000 + dev;
      return 0;
    };
  };
  long v = 0;
  // once per device
  CHECK((PerDevice<long, SiteA>::get(0, &v, make(0), -99)) == 0 && v == 1000);
  CHECK((PerDevice<long, SiteA>::get(0, &v, make(0), -99)) == 0 && v == 1000);
  CHECK(calls.load() == 1);
  // a second device sets up again (the per-thread cache this replaces did not)
  CHECK((PerDevice<long, SiteA>::get(1, &v, make(1), -99)) == 0 && v == 1001);
  CHECK(calls.load() == 2);
  // another call site is independent
  CHECK((PerDevice<long, SiteB>::get(0, &v, make(7), -99)) == 0 && v == 1007);
  CHECK(calls.load() == 3);
  CHECK((PerDevice<long, SiteA>::ready_count()) == 2);
  CHECK((PerDevice<long, SiteB>::ready_count()) == 1);
  // failures are returned and not cached; a later success is
  int tries = 0;
  auto flaky = [&](long *out) -> int {
    ++tries;
    if (tries == 1) return 42;
    *out = 5;
    return 0;
  };
  CHECK((PerDevice<long, SiteB>::get(3, &v, flaky, -99)) == 42);
  CHECK((PerDevice<long, SiteB>::get(3, &v, flaky, -99)) == 0 && v == 5);
  CHECK((PerDevice<long, SiteB>::get(3, &v, flaky, -99)) == 0 && tries == 2);
  // device index out of range
  CHECK((PerDevice<long, SiteA>::get(-1, &v, make(0), -99)) == -99);
  CHECK((PerDevice<long, SiteA>::get(bk::host::kMaxCachedDevices, &v, make(0), -99)) == -99);
  // concurrent first calls: set-up runs once per device
  struct SiteC {};
  std::atomic<int> ccalls{0};
  std::atomic<int> wrong{0};
  std::vector<std::thread> th;
  for (int t = 0; t < 16; ++t)
    th.emplace_back([&, t]() {
      for (int r = 0; r < 2000; ++r) {
        const int dev = (t + r) % 8;
        long x = -1;
        const int st = PerDevice<long, SiteC>::get(dev, &x, [&, dev](long *o) -> int {
          ccalls.fetch_add(1);
          *o = 10 * dev;
          return 0;
        }, -99);
        if (st != 0 || x != 10 * dev) wrong.fetch_add(1);
      }
    });
  for (auto &x : th) x.join();
  CHECK(wrong.load() == 0);
  CHECK(ccalls.load() == 8);
  std::printf("ok\n");
  return 0;
}
