// bk_tune.hpp -- launch shapes chosen per op, element size and size class
// from a measured table, in place of fixed per-kernel constants (the role
// the reference's choose_sizes / cuda_launch_config play for its launches,
// bulk/detail/choose_sizes.inl:32-117, cuda_launch_config.hpp:240-379, which
// derive them from a pre-Maxwell occupancy model).
//
// The table (tuning_table.inc, generated by bulk_b200/tune.py on a B200 and
// compiled in) maps (op, element bytes, size class) to knobs:
//   ctas_per_sm  persistent / grid-stride CTAs per SM (the grid is that many
//                times the SM count, or the tile count when smaller);
//   prefetch     L2 prefetch distance in residencies (0: none; read by the
//                radix sort, whose tiles are not persistent).
// Size classes: 0 below 2^16 elements, 1 below 2^20, 2 below 2^24, 3 from
// 2^24.  A missing entry takes the op's default.  A process-wide override
// per (op, element bytes, size class) lets the tuning procedure try knobs
// without rebuilding.  Plain C++, tested on the CPU through the C-ABI.
#pragma once

#include <stdint.h>

namespace bk {
namespace tune {

enum Op : int { kReduce = 0, kScan = 1, kReduceByKey = 2, kMerge = 3, kSort = 4, kOps = 5 };
constexpr int kSizeClasses = 4;

struct Knobs {
  int32_t ctas_per_sm;
  int32_t prefetch;
};

struct Entry {
  int op;
  int elem_bytes;  // key + value bytes for by-key ops
  int size_class;
  Knobs knobs;
};

inline int size_class(uint64_t n) {
  if (n < (1ull << 16)) return 0;
  if (n < (1ull << 20)) return 1;
  if (n < (1ull << 24)) return 2;
  return 3;
}

// The knobs bounds each op accepts (the kernels' residency limits).
inline int max_ctas_per_sm(int op) {
  switch (op) {
    case kReduce: return 8;
    case kScan: return 2;
    case kReduceByKey: return 3;  // the kernel caps it at 2 unless key and value are 4 bytes each
    case kMerge: return 3;
    default: return 1;
  }
}
inline Knobs default_knobs(int op) {
  switch (op) {
    case kReduce: return Knobs{4, 0};
    case kScan: return Knobs{2, 0};
    case kReduceByKey: return Knobs{3, 0};
    case kMerge: return Knobs{3, 0};
    default: return Knobs{1, 1};  // sort: L2 prefetch one residency ahead
  }
}

// The knobs for a call: override, else table, else default.
Knobs knobs_for(int op, int elem_bytes, uint64_t n);
// Sets (ctas_per_sm > 0) or clears (ctas_per_sm == 0) an override; returns
// false for arguments out of range.
bool set_override(int op, int elem_bytes, int size_class, int32_t ctas_per_sm, int32_t prefetch);

}  // namespace tune
}  // namespace bk
