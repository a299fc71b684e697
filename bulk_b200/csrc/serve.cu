// serve.cu -- the serving loop: a stream of mixed requests answered one
// library call per request ("plain") or by continuous batching ("batched").
//
// No counterpart in the reference, whose drivers run one array at a time.
// The loop is host code over the C-ABI: admission against an HBM budget, a
// pooled allocator over one caller-owned device buffer, completion by event
// polling, and per-request start / done times on the host's steady clock.
// Plain mode issues everything on the caller's stream.  Batched mode issues
// each admission round as one batch per request kind, the kinds on three
// streams of their own (forked from the caller's stream and joined back to
// it, each with its own slice of the workspace) so that a round's sorts,
// reduce_by_keys and scans run side by side on the device; a kind with a
// single request in the round is issued as a plain single-array call, and a
// round of at most four requests as plain calls on the caller's stream, at
// once (not counted against max_inflight).  Batched mode's sorts run out of
// place, lone ones of 2^20 elements and more too: the sort reads each
// request's source window and writes the request's own buffers, where plain
// mode copies the window into the buffers and sorts them in place.
#include <algorithm>
#include <chrono>
#include <deque>
#include <map>
#include <unordered_map>
#include <vector>

#include "bk_common.cuh"
#include "bulk_b200.h"

namespace bk {
namespace serve {

// ---------------------------------------------------------------------------
// Pooled allocator: offsets into one buffer, first fit over an address-
// ordered free list, 256-byte granules, neighbours coalesced on free.  It
// never touches device memory, so it runs (and is tested) without a GPU.
class Pool {
 public:
  static constexpr uint64_t kGranule = 256;
  explicit Pool(uint64_t capacity) : cap_(capacity / kGranule * kGranule) {
    if (cap_ > 0) free_[0] = cap_;
  }
  bool alloc(uint64_t bytes, uint64_t *off) {
    const uint64_t need = std::max<uint64_t>(kGranule, (bytes + kGranule - 1) / kGranule * kGranule);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < need) continue;
      const uint64_t o = it->first, rest = it->second - need;
      free_.erase(it);
      if (rest) free_[o + need] = rest;
      used_[o] = need;
      in_use_ += need;
      high_ = std::max(high_, in_use_);
      *off = o;
      return true;
    }
    return false;
  }
  bool release(uint64_t off) {
    auto u = used_.find(off);
    if (u == used_.end()) return false;
    uint64_t o = off, size = u->second;
    used_.erase(u);
    in_use_ -= size;
    auto right = free_.lower_bound(o);
    if (right != free_.end() && o + size == right->first) {
      size += right->second;
      free_.erase(right);
    }
    auto it = free_.lower_bound(o);
    if (it != free_.begin()) {
      auto left = std::prev(it);
      if (left->first + left->second == o) {
        left->second += size;
        return true;
      }
    }
    free_[o] = size;
    return true;
  }
  uint64_t in_use() const { return in_use_; }
  uint64_t high_water() const { return high_; }
  uint64_t capacity() const { return cap_; }
  uint32_t free_blocks() const { return (uint32_t)free_.size(); }

 private:
  uint64_t cap_;
  std::map<uint64_t, uint64_t> free_;  // offset -> bytes
  std::unordered_map<uint64_t, uint64_t> used_;
  uint64_t in_use_ = 0, high_ = 0;
};

// ---------------------------------------------------------------------------
struct Req {
  const bk_serve_request *r;
  bk_serve_record *rec;
  uint64_t off[3];
  int nbuf;
};

uint64_t request_bytes(uint32_t kind, uint64_t n) {
  // the request's own buffers (sort: keys and payload; rbk: outputs and the
  // count word; scan: output) plus slack for granule rounding
  return (kind == BK_SERVE_SCAN ? 4 : 8) * n + 512;
}

// Batched mode: the workspace holds one slice per request kind (the kinds'
// batches run on separate streams at once), each a multiple of 256 bytes.
struct WsSlices {
  size_t off[3];
  size_t bytes[3];
  size_t total;
};
WsSlices batched_slices(const bk_serve_request *reqs, uint32_t count);

class Loop {
 public:
  Loop(const bk_serve_config &c, uint64_t count) : c_(c), pool_(c.pool_bytes) {
    (void)count;
    st_ = reinterpret_cast<cudaStream_t>(c.stream);
    base_ = reinterpret_cast<char *>(c.pool);
    for (int k = 0; k < 3; ++k) ks_[k] = nullptr;
  }
  ~Loop() {
    for (cudaEvent_t e : events_) cudaEventDestroy(e);
    for (int k = 0; k < 3; ++k)
      if (ks_[k]) cudaStreamDestroy(ks_[k]);
  }

  // Batched mode: the kinds' streams and workspace slices.
  int setup_batched(const WsSlices &sl) {
    for (int k = 0; k < 3; ++k) {
      const cudaError_t e = cudaStreamCreateWithFlags(&ks_[k], cudaStreamNonBlocking);
      if (e != cudaSuccess) return host::from_cuda(e);
      ws_[k] = static_cast<char *>(c_.ws) + sl.off[k];
      ws_bytes_[k] = sl.bytes[k];
    }
    return BK_OK;
  }

  int run(const bk_serve_request *reqs, uint32_t count, bk_serve_record *recs, bk_serve_stats *stats) {
    using clock = std::chrono::steady_clock;
    const auto t0 = clock::now();
    auto now = [&] { return std::chrono::duration<double>(clock::now() - t0).count(); };
    std::vector<Req> all(count);
    for (uint32_t i = 0; i < count; ++i) all[i] = Req{&reqs[i], &recs[i], {0, 0, 0}, 0};
    uint32_t next = 0, done = 0;
    std::vector<Req *> waiting;
    std::deque<std::pair<cudaEvent_t, std::vector<Req *>>> inflight;
    int st = BK_OK;
    while (done < count) {
      if (now() > c_.timeout_s) {
        st = BK_ERR_SPIN_TIMEOUT;
        break;
      }
      // completions, in stream order
      while (!inflight.empty()) {
        const cudaError_t q = cudaEventQuery(inflight.front().first);
        if (q == cudaErrorNotReady) break;
        if (q != cudaSuccess) return finish(host::from_cuda(q), stats, t0);
        const double td = now();
        for (Req *r : inflight.front().second) {
          r->rec->done_s = td;
          release(r);
          ++done;
        }
        free_events_.push_back(inflight.front().first);
        inflight.pop_front();
      }
      // arrivals and admission, in arrival order
      const double ta = now();
      while (next < count && all[next].r->arrival_s <= ta) {
        const int a = admit(&all[next]);
        if (a == 0) break;  // over budget: wait for completions
        if (a < 0) {
          // cannot fit even with nothing else admitted
          if (admitted_ == 0 && inflight.empty() && waiting.empty()) return finish(BK_ERR_TOO_LARGE, stats, t0);
          break;
        }
        Req *r = &all[next++];
        if (c_.mode == BK_SERVE_PLAIN) {
          r->rec->start_s = ta;
          if ((st = issue_one(r)) != BK_OK) return finish(st, stats, t0);
          cudaEvent_t ev;
          if ((st = record(&ev)) != BK_OK) return finish(st, stats, t0);
          inflight.emplace_back(ev, std::vector<Req *>{r});
        } else {
          waiting.push_back(r);
        }
      }
      // a round small enough to go out as plain calls is issued at once, as
      // plain mode would (queued behind the rounds in flight on the GPU,
      // not held on the host until one of them completes); larger rounds
      // wait for a free slot among the max_inflight
      if (c_.mode == BK_SERVE_BATCHED && !waiting.empty() &&
          ((int)inflight.size() < c_.max_inflight || waiting.size() <= (size_t)kPlainRound)) {
        const double ti = now();
        for (Req *r : waiting) r->rec->start_s = ti;
        if ((st = issue_batches(waiting)) != BK_OK) return finish(st, stats, t0);
        cudaEvent_t ev;
        if ((st = record(&ev)) != BK_OK) return finish(st, stats, t0);
        inflight.emplace_back(ev, std::move(waiting));
        waiting.clear();
      }
    }
    return finish(st, stats, t0);
  }

 private:
  int finish(int st, bk_serve_stats *stats, std::chrono::steady_clock::time_point t0) {
    // the kinds' streams first: after a failure mid-round they may hold work
    // that was never joined to the caller's stream
    for (int k = 0; k < 3; ++k) {
      if (ks_[k] == nullptr) continue;
      const cudaError_t ek = cudaStreamSynchronize(ks_[k]);
      if (st == BK_OK) st = host::from_cuda(ek);
    }
    const cudaError_t e = cudaStreamSynchronize(st_);
    if (st == BK_OK) st = host::from_cuda(e);
    if (stats) {
      stats->makespan_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      stats->pool_high_water = pool_.high_water();
      stats->calls = calls_;
      stats->batches = batches_;
    }
    return st;
  }

  int record(cudaEvent_t *ev) { return record_on(ev, st_); }

  int record_on(cudaEvent_t *ev, cudaStream_t s) {
    if (free_events_.empty()) {
      cudaEvent_t e;
      const cudaError_t r = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
      if (r != cudaSuccess) return host::from_cuda(r);
      events_.push_back(e);
      free_events_.push_back(e);
    }
    *ev = free_events_.back();
    free_events_.pop_back();
    return host::from_cuda(cudaEventRecord(*ev, s));
  }

  // Fork/join helper events are reusable once the stream that waits on them
  // has been told to: a later record only affects later waits.
  int helper_event(cudaEvent_t *ev, cudaStream_t s) {
    const int st = record_on(ev, s);
    free_events_.push_back(*ev);
    return st;
  }

  // 1 admitted, 0 over budget (wait), -1 the pool has no room (wait, or fail
  // if nothing is admitted)
  int admit(Req *q) {
    const uint64_t n = q->r->n, need = request_bytes(q->r->kind, n);
    if (admitted_ > 0 && admitted_ + need > c_.budget_bytes) return 0;
    uint64_t sizes[3];
    int nb = 0;
    switch (q->r->kind) {
      case BK_SERVE_SORT: sizes[nb++] = 4 * n; sizes[nb++] = 4 * n; break;
      case BK_SERVE_RBK: sizes[nb++] = 4 * n; sizes[nb++] = 4 * n; sizes[nb++] = 8; break;
      default: sizes[nb++] = 4 * n; break;
    }
    for (int i = 0; i < nb; ++i) {
      if (!pool_.alloc(sizes[i], &q->off[i])) {
        for (int j = 0; j < i; ++j) pool_.release(q->off[j]);
        return -1;
      }
    }
    q->nbuf = nb;
    for (int i = 0; i < 3; ++i) q->rec->out[i] = i < nb ? q->off[i] : 0;
    admitted_ += need;
    return 1;
  }

  void release(Req *q) {
    if (!c_.keep_buffers)
      for (int i = 0; i < q->nbuf; ++i) pool_.release(q->off[i]);
    q->nbuf = 0;
    admitted_ -= request_bytes(q->r->kind, q->r->n);
  }

  template <typename T>
  T *buf(const Req *q, int i) const {
    return reinterpret_cast<T *>(base_ + q->off[i]);
  }

  // One request as its own single-array call on stream s with workspace ws.
  int issue_one(Req *q) { return issue_one_on(q, st_, c_.ws, c_.ws_bytes); }

  int issue_one_on(Req *q, cudaStream_t s, void *ws, size_t ws_bytes) {
    const uint64_t n = q->r->n, o = q->r->src_offset;
    ++calls_;
    switch (q->r->kind) {
      case BK_SERVE_SORT: {
        uint32_t *k = buf<uint32_t>(q, 0), *v = buf<uint32_t>(q, 1);
        cudaError_t e = cudaMemcpyAsync(k, c_.sort_keys + o, 4 * n, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(v, c_.sort_vals + o, 4 * n, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return host::from_cuda(e);
        return bk_sort_by_key_u32_u32(k, v, n, ws, ws_bytes, (bk_stream_t)s);
      }
      case BK_SERVE_RBK:
        return bk_reduce_by_key_i32_f32(c_.rbk_keys + o, c_.rbk_vals + o, n, buf<int32_t>(q, 0), buf<float>(q, 1),
                                        buf<uint64_t>(q, 2), ws, ws_bytes, (bk_stream_t)s);
      default:
        return bk_inclusive_scan_sum_f32(c_.scan_vals + o, n, 0.0f, buf<float>(q, 0), ws, ws_bytes, (bk_stream_t)s);
    }
  }

  // Batched mode, a request issued alone: as its plain call, except that a
  // sort of at least kLoneDirect elements reads its source window directly (a
  // one-item out-of-place batch) instead of first copying the window into its
  // buffers.  Below that the batch call's larger launches cost more than the
  // copy saves (measured on a B200: open-loop p99 of the 2^10-2^16 mix 5 %
  // higher with every lone sort out of place, of the 2^10-2^24 mix 8 % lower).
  static constexpr uint64_t kLoneDirect = 1ull << 20;
  int issue_lone(Req *q, cudaStream_t s, void *ws, size_t ws_bytes) {
    if (q->r->kind != BK_SERVE_SORT || q->r->n < kLoneDirect) return issue_one_on(q, s, ws, ws_bytes);
    ++calls_;
    const uint64_t o = q->r->src_offset;
    const bk_sort_copy_item_u32_u32 it{c_.sort_keys + o, c_.sort_vals + o, buf<uint32_t>(q, 0), buf<uint32_t>(q, 1),
                                       q->r->n};
    return bk_sort_by_key_u32_u32_copy_batch(&it, 1u, ws, ws_bytes, (bk_stream_t)s);
  }

  static constexpr int kPlainRound = 4;

  // One admission round: per kind, one batched call (at most BK_BATCH_MAX
  // arrays each; sorts out of place, from the requests' source windows), or
  // a plain call for a kind with one request.  With more than
  // one kind present, each kind runs on its own stream, forked from the
  // caller's stream and joined back to it; otherwise the kind runs on the
  // caller's stream (its slice is free there: the caller's stream has
  // joined every earlier use of it).
  int issue_batches(const std::vector<Req *> &reqs) {
    // a round of up to four requests (light load) is issued as plain calls on
    // the caller's stream: batch descriptors and stream fork/join would only
    // add latency there
    if (reqs.size() <= (size_t)kPlainRound) {
      for (Req *r : reqs) {
        const int kind = (int)r->r->kind;
        const int st = issue_lone(r, st_, ws_[kind], ws_bytes_[kind]);
        if (st != BK_OK) return st;
      }
      return BK_OK;
    }
    std::vector<Req *> by[3];
    for (Req *r : reqs) by[r->r->kind].push_back(r);
    const int kinds = (by[0].empty() ? 0 : 1) + (by[1].empty() ? 0 : 1) + (by[2].empty() ? 0 : 1);
    int st;
    cudaEvent_t fork = nullptr;
    if (kinds > 1 && (st = helper_event(&fork, st_)) != BK_OK) return st;
    for (int kind = 0; kind < 3; ++kind) {
      if (by[kind].empty()) continue;
      cudaStream_t s = st_;
      if (kinds > 1) {
        s = ks_[kind];
        if ((st = host::from_cuda(cudaStreamWaitEvent(s, fork, 0))) != BK_OK) return st;
      }
      if (by[kind].size() == 1) st = issue_lone(by[kind][0], s, ws_[kind], ws_bytes_[kind]);
      else st = issue_kind(kind, by[kind], s);
      if (st != BK_OK) return st;
      if (kinds > 1) {
        cudaEvent_t join;
        if ((st = helper_event(&join, s)) != BK_OK) return st;
        if ((st = host::from_cuda(cudaStreamWaitEvent(st_, join, 0))) != BK_OK) return st;
      }
    }
    return BK_OK;
  }

  // One kind's batched calls on stream s with the kind's workspace slice.
  int issue_kind(int kind, const std::vector<Req *> &v, cudaStream_t s) {
    int st = BK_OK;
    void *ws = ws_[kind];
    const size_t wsb = ws_bytes_[kind];
    for (size_t lo = 0; lo < v.size(); lo += BK_BATCH_MAX) {
      const size_t hi = std::min(v.size(), lo + (size_t)BK_BATCH_MAX);
      ++calls_;
      ++batches_;
      if (kind == BK_SERVE_SORT) {
        // out of place: the first radix pass reads each request's source
        // window and the result lands in its own buffers (no separate copy)
        bk_sort_copy_item_u32_u32 it[BK_BATCH_MAX];
        for (size_t i = lo; i < hi; ++i) {
          const uint64_t o = v[i]->r->src_offset;
          it[i - lo] = bk_sort_copy_item_u32_u32{c_.sort_keys + o, c_.sort_vals + o, buf<uint32_t>(v[i], 0),
                                                 buf<uint32_t>(v[i], 1), v[i]->r->n};
        }
        st = bk_sort_by_key_u32_u32_copy_batch(it, (uint32_t)(hi - lo), ws, wsb, (bk_stream_t)s);
      } else if (kind == BK_SERVE_RBK) {
        bk_rbk_item_i32_f32 it[BK_BATCH_MAX];
        for (size_t i = lo; i < hi; ++i) {
          const uint64_t o = v[i]->r->src_offset;
          it[i - lo] = bk_rbk_item_i32_f32{c_.rbk_keys + o, c_.rbk_vals + o, v[i]->r->n, buf<int32_t>(v[i], 0),
                                          buf<float>(v[i], 1), buf<uint64_t>(v[i], 2)};
        }
        st = bk_reduce_by_key_i32_f32_batch(it, (uint32_t)(hi - lo), ws, wsb, (bk_stream_t)s);
      } else {
        bk_scan_item_f32 it[BK_BATCH_MAX];
        for (size_t i = lo; i < hi; ++i)
          it[i - lo] = bk_scan_item_f32{c_.scan_vals + v[i]->r->src_offset, buf<float>(v[i], 0), v[i]->r->n, 0.0f};
        st = bk_inclusive_scan_sum_f32_batch(it, (uint32_t)(hi - lo), ws, wsb, (bk_stream_t)s);
      }
      if (st != BK_OK) return st;
    }
    return BK_OK;
  }

  const bk_serve_config c_;
  Pool pool_;
  cudaStream_t st_;
  cudaStream_t ks_[3];   // batched mode: one stream per request kind
  void *ws_[3] = {nullptr, nullptr, nullptr};
  size_t ws_bytes_[3] = {0, 0, 0};
  char *base_;
  uint64_t admitted_ = 0;
  uint64_t calls_ = 0, batches_ = 0;
  std::vector<cudaEvent_t> events_, free_events_;
};

int check_requests(const bk_serve_config &c, const bk_serve_request *reqs, uint32_t count) {
  double prev = 0.0;
  for (uint32_t i = 0; i < count; ++i) {
    const bk_serve_request &r = reqs[i];
    if (r.kind > BK_SERVE_SCAN || r.n == 0 || r.src_offset + r.n > c.source_len) return BK_ERR_INVALID_ARGUMENT;
    if ((r.src_offset * 4) % 16 != 0) return BK_ERR_MISALIGNED;  // windows keep the sources' 16-byte alignment
    if (r.arrival_s < prev) return BK_ERR_INVALID_ARGUMENT;
    prev = r.arrival_s;
  }
  return BK_OK;
}

}  // namespace serve
}  // namespace bk

using bk::serve::Pool;

extern "C" uint64_t bk_serve_request_bytes(uint32_t kind, uint64_t n) { return bk::serve::request_bytes(kind, n); }

extern "C" size_t bk_serve_workspace_bytes(const bk_serve_request *reqs, uint32_t count, int mode) {
  if (count > 0 && reqs == nullptr) return 0;
  size_t need = bk::kHeaderBytes;
  static const int algo[3] = {BK_ALGO_SORT_BY_KEY, BK_ALGO_REDUCE_BY_KEY, BK_ALGO_INCLUSIVE_SCAN};
  static const int key[3] = {BK_DTYPE_U32, BK_DTYPE_I32, BK_DTYPE_F32};
  static const int val[3] = {BK_DTYPE_U32, BK_DTYPE_F32, BK_DTYPE_NONE};
  if (mode == BK_SERVE_PLAIN) {
    for (uint32_t i = 0; i < count; ++i) {
      const uint32_t k = reqs[i].kind;
      if (k > BK_SERVE_SCAN) return 0;
      need = std::max(need, bk_workspace_bytes(algo[k], key[k], val[k], reqs[i].n));
    }
    return need;
  }
  for (uint32_t i = 0; i < count; ++i)
    if (reqs[i].kind > BK_SERVE_SCAN) return 0;
  return std::max(need, bk::serve::batched_slices(reqs, count).total);
}

namespace bk {
namespace serve {
// Batched mode: one workspace slice per kind (the kinds run at once on their
// own streams).  A batch's workspace grows with its arrays, so the largest
// BK_BATCH_MAX requests of a kind bound every batch of that kind; a slice
// also covers the kind's largest request run alone.
WsSlices batched_slices(const bk_serve_request *reqs, uint32_t count) {
  static const int algo[3] = {BK_ALGO_SORT_BY_KEY, BK_ALGO_REDUCE_BY_KEY, BK_ALGO_INCLUSIVE_SCAN};
  static const int key[3] = {BK_DTYPE_U32, BK_DTYPE_I32, BK_DTYPE_F32};
  static const int val[3] = {BK_DTYPE_U32, BK_DTYPE_F32, BK_DTYPE_NONE};
  WsSlices sl{};
  size_t off = 0;
  for (uint32_t k = 0; k < 3; ++k) {
    std::vector<uint64_t> sizes;
    for (uint32_t i = 0; i < count; ++i)
      if (reqs[i].kind == k) sizes.push_back(reqs[i].n);
    if (sizes.size() > (size_t)BK_BATCH_MAX) {
      std::nth_element(sizes.begin(), sizes.begin() + BK_BATCH_MAX, sizes.end(), std::greater<uint64_t>());
      sizes.resize(BK_BATCH_MAX);
    }
    size_t need = std::max<size_t>(
        bk::kHeaderBytes, bk_batch_workspace_bytes(algo[k], key[k], val[k], sizes.data(), (uint32_t)sizes.size()));
    for (uint64_t n : sizes) need = std::max(need, bk_workspace_bytes(algo[k], key[k], val[k], n));
    need = bk::align_up(need, 256);
    sl.off[k] = off;
    sl.bytes[k] = need;
    off += need;
  }
  sl.total = off;
  return sl;
}
}  // namespace serve
}  // namespace bk

extern "C" int bk_serve_run(const bk_serve_config *cfg, const bk_serve_request *reqs, uint32_t count,
                            bk_serve_record *records, bk_serve_stats *stats) {
  if (cfg == nullptr || (count > 0 && (reqs == nullptr || records == nullptr))) return BK_ERR_INVALID_ARGUMENT;
  const bk_serve_config &c = *cfg;
  if (c.mode != BK_SERVE_PLAIN && c.mode != BK_SERVE_BATCHED) return BK_ERR_INVALID_ARGUMENT;
  if (c.mode == BK_SERVE_BATCHED && c.max_inflight < 1) return BK_ERR_INVALID_ARGUMENT;
  if (c.pool == nullptr || c.ws == nullptr || c.sort_keys == nullptr || c.sort_vals == nullptr ||
      c.rbk_keys == nullptr || c.rbk_vals == nullptr || c.scan_vals == nullptr)
    return BK_ERR_INVALID_ARGUMENT;
  if (reinterpret_cast<uintptr_t>(c.pool) % 256 != 0) return BK_ERR_MISALIGNED;
  int st = bk::serve::check_requests(c, reqs, count);
  if (st != BK_OK) return st;
  if (c.ws_bytes < bk_serve_workspace_bytes(reqs, count, c.mode)) return BK_ERR_WORKSPACE_TOO_SMALL;
  for (uint32_t i = 0; i < count; ++i) records[i] = bk_serve_record{-1.0, -1.0, {0, 0, 0}};
  bk::serve::Loop loop(c, count);
  if (c.mode == BK_SERVE_BATCHED) {
    // each slice is a workspace of its own: its header (the counters every
    // call leaves at zero) must start zeroed
    const bk::serve::WsSlices sl = bk::serve::batched_slices(reqs, count);
    for (int k = 0; k < 3; ++k)
      if ((st = bk::host::from_cuda(cudaMemsetAsync(static_cast<char *>(c.ws) + sl.off[k], 0, bk::kHeaderBytes,
                                                    (cudaStream_t)c.stream))) != BK_OK)
        return st;
    if ((st = loop.setup_batched(sl)) != BK_OK) return st;
  }
  return loop.run(reqs, count, records, stats);
}

// ---- host-side pool (offsets only) -----------------------------------------
extern "C" void *bk_pool_create(uint64_t capacity) { return new (std::nothrow) Pool(capacity); }

extern "C" void bk_pool_destroy(void *pool) { delete static_cast<Pool *>(pool); }

extern "C" int bk_pool_alloc(void *pool, uint64_t bytes, uint64_t *offset) {
  if (pool == nullptr || offset == nullptr) return BK_ERR_INVALID_ARGUMENT;
  return static_cast<Pool *>(pool)->alloc(bytes, offset) ? BK_OK : BK_ERR_TOO_LARGE;
}

extern "C" int bk_pool_free(void *pool, uint64_t offset) {
  if (pool == nullptr) return BK_ERR_INVALID_ARGUMENT;
  return static_cast<Pool *>(pool)->release(offset) ? BK_OK : BK_ERR_INVALID_ARGUMENT;
}

extern "C" uint64_t bk_pool_in_use(const void *pool) { return pool ? static_cast<const Pool *>(pool)->in_use() : 0; }

extern "C" uint64_t bk_pool_high_water(const void *pool) {
  return pool ? static_cast<const Pool *>(pool)->high_water() : 0;
}

extern "C" uint32_t bk_pool_free_blocks(const void *pool) {
  return pool ? static_cast<const Pool *>(pool)->free_blocks() : 0;
}
