// compat.h -- force-included when the reference's headers are compiled for
// the host with the CUDA 12.9 / Thrust 2.8 headers: re-creates the few names
// the reference uses that newer Thrust no longer provides.
#pragma once
#include <cuda_runtime_api.h>
#ifndef __thrust_forceinline__
#define __thrust_forceinline__ inline
#endif
#ifndef __forceinline__
#define __forceinline__ inline
#endif
#include <thrust/detail/config.h>
#include <type_traits>
THRUST_NAMESPACE_BEGIN
namespace detail {
template <bool B, class T = void>
struct enable_if : std::enable_if<B, T> {};
}  // namespace detail
THRUST_NAMESPACE_END
// the reference's device code calls an unqualified min()
template <class T>
inline T min(T a, T b) { return b < a ? b : a; }
