// bulk/iterator.hpp -- strided_iterator: a random-access view of every
// stride-th element of an underlying iterator.
//
// Interface of the reference's bulk/iterator/strided_iterator.hpp:28-108
// (constructor (base, stride), stride(), base(), make_strided_iterator, the
// distance rounding toward the far end), written as a plain random-access
// iterator so it needs no Thrust.
#pragma once

#include <cstddef>
#include <iterator>

namespace bulk {

template <typename Iterator, typename Size = typename std::iterator_traits<Iterator>::difference_type>
class strided_iterator {
 public:
  typedef std::random_access_iterator_tag iterator_category;
  typedef typename std::iterator_traits<Iterator>::value_type value_type;
  typedef typename std::iterator_traits<Iterator>::difference_type difference_type;
  typedef typename std::iterator_traits<Iterator>::reference reference;
  typedef typename std::iterator_traits<Iterator>::pointer pointer;
  typedef Size stride_type;

  __host__ __device__ strided_iterator() : m_base(), m_stride(1) {}
  __host__ __device__ strided_iterator(const Iterator &base, stride_type stride) : m_base(base), m_stride(stride) {}

  __host__ __device__ stride_type stride() const { return m_stride; }
  __host__ __device__ Iterator base() const { return m_base; }

  __host__ __device__ reference operator*() const { return *m_base; }
  __host__ __device__ reference operator[](difference_type n) const { return m_base[n * m_stride]; }
  __host__ __device__ strided_iterator &operator++() { m_base += m_stride; return *this; }
  __host__ __device__ strided_iterator operator++(int) { strided_iterator t = *this; ++*this; return t; }
  __host__ __device__ strided_iterator &operator--() { m_base -= m_stride; return *this; }
  __host__ __device__ strided_iterator operator--(int) { strided_iterator t = *this; --*this; return t; }
  __host__ __device__ strided_iterator &operator+=(difference_type n) { m_base += n * m_stride; return *this; }
  __host__ __device__ strided_iterator &operator-=(difference_type n) { m_base -= n * m_stride; return *this; }
  __host__ __device__ strided_iterator operator+(difference_type n) const { strided_iterator t = *this; return t += n; }
  __host__ __device__ strided_iterator operator-(difference_type n) const { strided_iterator t = *this; return t -= n; }

  // number of strides from this to other, rounded away from zero
  __host__ __device__ difference_type operator-(const strided_iterator &other) const {
    const difference_type d = m_base - other.m_base;
    return d >= 0 ? (d + (m_stride - 1)) / m_stride : (d - (m_stride - 1)) / m_stride;
  }
  __host__ __device__ bool operator==(const strided_iterator &o) const { return m_base == o.m_base; }
  __host__ __device__ bool operator!=(const strided_iterator &o) const { return m_base != o.m_base; }
  __host__ __device__ bool operator<(const strided_iterator &o) const { return m_base < o.m_base; }
  __host__ __device__ bool operator<=(const strided_iterator &o) const { return m_base <= o.m_base; }
  __host__ __device__ bool operator>(const strided_iterator &o) const { return m_base > o.m_base; }
  __host__ __device__ bool operator>=(const strided_iterator &o) const { return m_base >= o.m_base; }

 private:
  Iterator m_base;
  stride_type m_stride;
};

template <typename Iterator, typename Size>
__host__ __device__ strided_iterator<Iterator, Size> make_strided_iterator(Iterator iter, Size stride) {
  return strided_iterator<Iterator, Size>(iter, stride);
}

}  // namespace bulk
