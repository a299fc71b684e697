// bulk/uninitialized.hpp -- storage for a T (or an array of T) that is not
// constructed until construct() is called; lets types without a trivial
// constructor live in __shared__ memory.
//
// Interface of the reference's bulk/uninitialized.hpp (uninitialized<T>
// :30-185: get, conversions, assignment, construct(args...), destroy;
// uninitialized_array<T, N> :188-260: size, operator[], data, begin/end).
#pragma once

#include <cstddef>
#include <new>

namespace bulk {

template <typename T>
class uninitialized {
 public:
  __host__ __device__ T &get() { return *ptr(); }
  __host__ __device__ const T &get() const { return *ptr(); }
  __host__ __device__ operator T &() { return get(); }
  __host__ __device__ operator const T &() const { return get(); }
  __host__ __device__ uninitialized &operator=(const T &other) {
    get() = other;
    return *this;
  }

  template <typename... Args>
  __host__ __device__ void construct(Args &&...args) {
    ::new (static_cast<void *>(storage)) T(static_cast<Args &&>(args)...);
  }
  __host__ __device__ void destroy() { ptr()->~T(); }

 private:
  __host__ __device__ T *ptr() { return reinterpret_cast<T *>(storage); }
  __host__ __device__ const T *ptr() const { return reinterpret_cast<const T *>(storage); }
  alignas(T) unsigned char storage[sizeof(T)];
};

template <typename T, std::size_t N>
class uninitialized_array {
 public:
  typedef T value_type;
  typedef T &reference;
  typedef const T &const_reference;
  typedef T *pointer;
  typedef const T *const_pointer;
  typedef pointer iterator;
  typedef const_pointer const_iterator;
  typedef std::size_t size_type;

  __host__ __device__ size_type size() const { return N; }
  __host__ __device__ iterator begin() { return data(); }
  __host__ __device__ const_iterator begin() const { return data(); }
  __host__ __device__ iterator end() { return data() + N; }
  __host__ __device__ const_iterator end() const { return data() + N; }
  __host__ __device__ reference operator[](size_type n) { return data()[n]; }
  __host__ __device__ const_reference operator[](size_type n) const { return data()[n]; }
  __host__ __device__ pointer data() { return reinterpret_cast<pointer>(storage); }
  __host__ __device__ const_pointer data() const { return reinterpret_cast<const_pointer>(storage); }

 private:
  alignas(T) unsigned char storage[sizeof(T) * N];
};

}  // namespace bulk
