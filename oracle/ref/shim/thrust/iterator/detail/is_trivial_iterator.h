#pragma once
#include <thrust/type_traits/is_contiguous_iterator.h>
THRUST_NAMESPACE_BEGIN
namespace detail {
template <class T>
struct is_trivial_iterator : thrust::is_contiguous_iterator<T> {};
}  // namespace detail
THRUST_NAMESPACE_END
