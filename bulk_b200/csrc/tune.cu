// tune.cu -- the launch-shape table and its C-ABI (lookup, override).
#include <atomic>
#include <mutex>

#include "bk_common.cuh"
#include "bk_tune.hpp"

namespace bk {
namespace tune {
namespace {

const Entry kTable[] = {
#include "tuning_table.inc"
};

constexpr int kBytesSlots = 17;  // element bytes 0..16
struct Override {
  std::atomic<int32_t> ctas{0};
  std::atomic<int32_t> prefetch{0};
};
Override g_override[kOps][kBytesSlots][kSizeClasses];

}  // namespace

Knobs knobs_for(int op, int elem_bytes, uint64_t n) {
  const int sc = size_class(n);
  if (op >= 0 && op < kOps && elem_bytes >= 0 && elem_bytes < kBytesSlots) {
    const Override &o = g_override[op][elem_bytes][sc];
    const int32_t c = o.ctas.load(std::memory_order_acquire);
    if (c > 0) return Knobs{c, o.prefetch.load(std::memory_order_relaxed)};
  }
  for (const Entry &e : kTable)
    if (e.op == op && e.elem_bytes == elem_bytes && e.size_class == sc) return e.knobs;
  return default_knobs(op);
}

bool set_override(int op, int elem_bytes, int sc, int32_t ctas_per_sm, int32_t prefetch) {
  if (op < 0 || op >= kOps || elem_bytes < 0 || elem_bytes >= kBytesSlots || sc < 0 || sc >= kSizeClasses)
    return false;
  if (ctas_per_sm < 0 || ctas_per_sm > max_ctas_per_sm(op) || prefetch < 0 || prefetch > 4) return false;
  Override &o = g_override[op][elem_bytes][sc];
  o.prefetch.store(prefetch, std::memory_order_relaxed);
  o.ctas.store(ctas_per_sm, std::memory_order_release);
  return true;
}

}  // namespace tune
}  // namespace bk

extern "C" int bk_tune_lookup(int op, int elem_bytes, uint64_t n, int32_t *ctas_per_sm, int32_t *prefetch) {
  if (op < 0 || op >= bk::tune::kOps || ctas_per_sm == nullptr || prefetch == nullptr) return BK_ERR_INVALID_ARGUMENT;
  const bk::tune::Knobs k = bk::tune::knobs_for(op, elem_bytes, n);
  *ctas_per_sm = k.ctas_per_sm;
  *prefetch = k.prefetch;
  return BK_OK;
}

extern "C" int bk_tune_override(int op, int elem_bytes, int size_class, int32_t ctas_per_sm, int32_t prefetch) {
  return bk::tune::set_override(op, elem_bytes, size_class, ctas_per_sm, prefetch) ? BK_OK : BK_ERR_INVALID_ARGUMENT;
}
