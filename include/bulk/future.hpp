// bulk/future.hpp -- completion handle of bulk::async.
//
// Same interface as the reference's bulk::future<void> (bulk/future.hpp:44-153):
// wait() blocks until the launch finished, valid() says whether the future
// refers to a launch; a future may own the stream it was launched into (when
// the launch was ordered after another future, bulk/detail/async.inl:52-81).
// Errors raise thrust::system_error in thrust::cuda_category() carrying the
// cudaError_t, as the reference does (bulk/detail/throw_on_error.hpp:33-49);
// it derives from std::runtime_error.
#pragma once

#include <stdexcept>
#include <string>
#include <utility>

#include <cuda_runtime.h>
#include <thrust/system/cuda/error.h>
#include <thrust/system_error.h>

#include "execution_policy.hpp"

namespace bulk {
namespace detail {

inline void throw_on_error(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw thrust::system_error(e, thrust::cuda_category(), what);
}

struct future_core_access;

}  // namespace detail

template <>
class future<void> {
 public:
  future() : m_stream(0), m_event(0), m_owns_stream(false) {}
  future(future &&o) noexcept : m_stream(o.m_stream), m_event(o.m_event), m_owns_stream(o.m_owns_stream) {
    o.m_event = 0;
    o.m_owns_stream = false;
  }
  future &operator=(future &&o) noexcept {
    std::swap(m_stream, o.m_stream);
    std::swap(m_event, o.m_event);
    std::swap(m_owns_stream, o.m_owns_stream);
    return *this;
  }
  future(const future &) = delete;
  future &operator=(const future &) = delete;
  ~future() {
    // destructors never throw: errors surface through wait()
    if (m_event) cudaEventDestroy(m_event);
    if (m_owns_stream) cudaStreamDestroy(m_stream);  // pending work still completes
  }

  void wait() const {
    if (!valid()) throw thrust::system_error(cudaErrorInvalidResourceHandle, thrust::cuda_category(),
                                             "bulk::future::wait: no launch");
    detail::throw_on_error(cudaEventSynchronize(m_event), "bulk::future::wait");
  }
  bool valid() const { return m_event != 0; }

 private:
  friend struct detail::future_core_access;
  future(cudaStream_t s, cudaEvent_t e, bool owns) : m_stream(s), m_event(e), m_owns_stream(owns) {}
  cudaStream_t m_stream;
  cudaEvent_t m_event;
  bool m_owns_stream;
};

namespace detail {
struct future_core_access {
  // records an event on s after the work just enqueued
  static future<void> create(cudaStream_t s, bool owns_stream) {
    cudaEvent_t e;
    throw_on_error(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "bulk::async: event");
    throw_on_error(cudaEventRecord(e, s), "bulk::async: event record");
    return future<void>(s, e, owns_stream);
  }
  static cudaEvent_t event(const future<void> &f) { return f.m_event; }
};
}  // namespace detail

inline async_launch<parallel_group<>> par(future<void> &before, size_t num_threads) {
  return async_launch<parallel_group<>>(par(num_threads), detail::future_core_access::event(before));
}

}  // namespace bulk
