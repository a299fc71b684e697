#pragma once
#include <thrust/detail/type_traits.h>
#include <thrust/detail/type_traits/has_nested_type.h>
#include <thrust/detail/type_traits/is_commutative.h>
THRUST_NAMESPACE_BEGIN
namespace detail {
__THRUST_DEFINE_HAS_NESTED_TYPE(has_result_type, result_type)
template <class F>
struct result_type { typedef typename F::result_type type; };
}  // namespace detail
THRUST_NAMESPACE_END
