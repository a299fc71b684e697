// api_check.cu -- programs written against the bulk:: C++ interface
// (include/bulk/bulk.hpp), each checked on the host against std::
// algorithms.  Prints one "ok <name>" or "FAIL <name> ..." line per check and
// exits non-zero when any check fails.
//
// Covers the usage patterns of the reference's drivers (hello_world.cu,
// saxpy.cu, sum.cu, for_each.cu, futures.cu: bulk::async over par / con /
// grid with root placeholders, stream and future policies) and every agent-
// and group-level algorithm of bulk/algorithm/*.hpp.  The cross-stream spin
// programs (ping_pong.cu, async_reduce.cu) are not reproduced: two kernels
// that wait on each other are not guaranteed to run at the same time.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <numeric>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include <unistd.h>

#include <bulk/bulk.hpp>

static int g_failures = 0;

// Host watchdog: a check that makes no progress for kStallSeconds ends the
// process (which ends its kernels) and names the check.
static constexpr int kStallSeconds = 30;
static std::atomic<long long> g_progress{0};
static char g_stage[128] = "start";
static void stage(const char *name) {
  std::snprintf(g_stage, sizeof g_stage, "%s", name);
  std::printf("run %s\n", name);
  ++g_progress;
}
static void start_watchdog() {
  std::thread([] {
    long long seen = -1;
    auto since = std::chrono::steady_clock::now();
    for (;;) {
      std::this_thread::sleep_for(std::chrono::milliseconds(200));
      const long long p = g_progress.load();
      if (p != seen) {
        seen = p;
        since = std::chrono::steady_clock::now();
      } else if (std::chrono::steady_clock::now() - since > std::chrono::seconds(kStallSeconds)) {
        std::printf("FAIL stalled in %s\n", g_stage);
        std::fflush(stdout);
        _exit(3);
      }
    }
  }).detach();
}

#define CUDA_OK(x)                                                              \
  do {                                                                          \
    cudaError_t e_ = (x);                                                       \
    if (e_ != cudaSuccess) {                                                    \
      std::printf("FAIL cuda %s: %s\n", #x, cudaGetErrorString(e_));           \
      std::exit(2);                                                             \
    }                                                                           \
  } while (0)

template <typename T>
struct dvec {
  T *p = nullptr;
  size_t n = 0;
  explicit dvec(size_t n_) : n(n_) { CUDA_OK(cudaMalloc(&p, sizeof(T) * (n ? n : 1))); }
  dvec(const std::vector<T> &h) : dvec(h.size()) { put(h); }
  ~dvec() { cudaFree(p); }
  dvec(const dvec &) = delete;
  void put(const std::vector<T> &h) { CUDA_OK(cudaMemcpy(p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice)); }
  std::vector<T> get() const {
    std::vector<T> h(n);
    CUDA_OK(cudaMemcpy(h.data(), p, sizeof(T) * n, cudaMemcpyDeviceToHost));
    return h;
  }
};

template <typename T>
static void check(const char *name, const std::vector<T> &got, const std::vector<T> &want) {
  if (got.size() != want.size()) {
    std::printf("FAIL %s size %zu != %zu\n", name, got.size(), want.size());
    ++g_failures;
    return;
  }
  ++g_progress;
  for (size_t i = 0; i < got.size(); ++i)
    if (!(got[i] == want[i])) {
      std::printf("FAIL %s at %zu of %zu\n", name, i, got.size());
      ++g_failures;
      return;
    }
  std::printf("ok %s\n", name);
}

static void check_true(const char *name, bool c) {
  ++g_progress;
  if (c) std::printf("ok %s\n", name);
  else {
    std::printf("FAIL %s\n", name);
    ++g_failures;
  }
}

static std::vector<int> random_ints(size_t n, uint32_t seed, int lo, int hi) {
  std::mt19937 r(seed);
  std::uniform_int_distribution<int> d(lo, hi);
  std::vector<int> v(n);
  for (auto &x : v) x = d(r);
  return v;
}

// ---- an associative, non-commutative operator: composition of affine maps
// x -> a*x + b over uint32 (wrap-around) -------------------------------------
struct affine {
  uint32_t a, b;
  __host__ __device__ bool operator==(const affine &o) const { return a == o.a && b == o.b; }
};
struct compose {  // apply l, then r
  __host__ __device__ affine operator()(const affine &l, const affine &r) const {
    return affine{l.a * r.a, l.b * r.a + r.b};
  }
};
static std::vector<affine> random_affine(size_t n, uint32_t seed) {
  std::mt19937 r(seed);
  std::vector<affine> v(n);
  for (auto &x : v) x = affine{uint32_t(r() | 1u), uint32_t(r())};
  return v;
}

struct plus_i {
  __host__ __device__ int operator()(int a, int b) const { return a + b; }
};
struct minus_i {
  __host__ __device__ int operator()(int a, int b) const { return a - b; }
};
struct less_i {
  __host__ __device__ bool operator()(int a, int b) const { return a < b; }
};
struct eq_i {
  __host__ __device__ bool operator()(int a, int b) const { return a == b; }
};

// ============================================================================
// driver-style programs
// ============================================================================
struct hello {
  __device__ void operator()(bulk::parallel_group<> &g, int *out) {
    out[g.this_exec.index()] = g.this_exec.index() * g.this_exec.index();
  }
};

struct saxpy {
  __device__ void operator()(bulk::agent<> &self, float a, const float *x, float *y) {
    const int i = self.index();
    y[i] = a * x[i] + y[i];
  }
};

struct sum {
  __device__ void operator()(bulk::concurrent_group<> &g, const int *data, int n, int *result) {
    const int s = bulk::reduce(g, data, data + n, 0, plus_i());
    if (g.this_exec.index() == 0) *result = s;
  }
};

struct for_each_kernel {
  struct square {
    __device__ void operator()(int &x) const { x = x * x; }
  };
  __device__ void operator()(bulk::agent<> &self, int *first) { square()(first[self.index()]); }
};

struct append_task {
  __device__ void operator()(int *log, int value) {
    const int slot = log[0]++;
    log[1 + slot] = value;
  }
};

struct segment_scan {  // one group per segment
  __device__ void operator()(bulk::concurrent_group<bulk::agent<4>, 128> &g, const int *in, int *out, int seg) {
    const int *first = in + (size_t)g.index() * seg;
    bulk::inclusive_scan(g, first, first + seg, out + (size_t)g.index() * seg, 7, plus_i());
  }
};

struct count_groups {  // one mark per group, written by its first agent
  __device__ void operator()(bulk::concurrent_group<> &g, int *marks, int cap) {
    if (g.this_exec.index() == 0 && g.index() < cap) atomicAdd(&marks[g.index()], 1);
    if (g.this_exec.index() == 0 && g.index() >= cap) atomicAdd(&marks[cap], 1);
  }
};

static void driver_programs() {
  {
    dvec<int> out(32);
    stage("hello");
    bulk::async(bulk::par(32), hello(), bulk::root, out.p).wait();
    std::vector<int> want(32);
    for (int i = 0; i < 32; ++i) want[i] = i * i;
    check("hello_world par(32) root", out.get(), want);
  }
  {
    const int n = 1 << 20;
    std::vector<float> x(n), y(n);
    for (int i = 0; i < n; ++i) {
      x[i] = float(i % 1000) * 0.5f;
      y[i] = float(i % 77);
    }
    dvec<float> dx(x), dy(y);
    stage("saxpy");
    bulk::async(bulk::par(n), saxpy(), bulk::root.this_exec, 2.0f, dx.p, dy.p).wait();
    std::vector<float> want(n);
    for (int i = 0; i < n; ++i) want[i] = 2.0f * x[i] + y[i];
    check("saxpy par(2^20) root.this_exec", dy.get(), want);
  }
  {
    const int n = 1 << 20;
    std::vector<int> h = random_ints(n, 1, -1000, 1000);
    dvec<int> d(h), r(1);
    stage("sum");
    bulk::async(bulk::con(512), sum(), bulk::root, d.p, n, r.p).wait();
    check("sum con(512) reduce", r.get(), std::vector<int>{std::accumulate(h.begin(), h.end(), 0)});
  }
  {
    const int n = 32;
    std::vector<int> h(n);
    std::iota(h.begin(), h.end(), 0);
    dvec<int> d(h);
    stage("for_each_kernel");
    bulk::async(bulk::par(n), for_each_kernel(), bulk::root.this_exec, d.p).wait();
    for (auto &x : h) x = x * x;
    check("for_each par(32)", d.get(), h);
  }
  {
    // stream policy, then a future policy ordered after it
    cudaStream_t s1;
    CUDA_OK(cudaStreamCreate(&s1));
    dvec<int> log(8);
    CUDA_OK(cudaMemset(log.p, 0, sizeof(int) * 8));
    stage("append_task");
    bulk::future<void> t1 = bulk::async(bulk::par(s1, 1), append_task(), log.p, 1);
    stage("append_task");
    bulk::future<void> t2 = bulk::async(bulk::par(t1, 1), append_task(), log.p, 2);
    stage("append_task");
    bulk::future<void> t3 = bulk::async(bulk::par(t2, 1), append_task(), log.p, 3);
    t3.wait();
    t1.wait();
    t2.wait();
    check_true("futures valid", t1.valid() && t2.valid() && t3.valid());
    std::vector<int> got = log.get();
    got.resize(4);
    check("futures par(stream) -> par(future) order", got, std::vector<int>{3, 1, 2, 3});
    CUDA_OK(cudaStreamDestroy(s1));
  }
  {
    // an unspecified grid: as many 256-thread groups as the occupancy model
    // says are resident at once (a whole number per SM), each launched once
    int sms = 0;
    CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0));
    const int cap = 1 << 16;
    dvec<int> marks(cap + 1);
    CUDA_OK(cudaMemset(marks.p, 0, sizeof(int) * (cap + 1)));
    stage("count_groups");
    const std::pair<int, int> sz = bulk::choose_sizes(bulk::grid(), count_groups(), bulk::root.this_exec, marks.p, cap);
    check_true("choose_sizes default grid: 256 threads, whole groups per SM",
               sz.second == 256 && sz.first >= sms && sz.first % sms == 0 && sz.first <= 8 * sms);
    bulk::async(bulk::grid(), count_groups(), bulk::root.this_exec, marks.p, cap).wait();
    std::vector<int> want(cap + 1, 0);
    for (int i = 0; i < sz.first && i < cap; ++i) want[i] = 1;
    check("default grid launches the chosen number of groups", marks.get(), want);
  }
  {
    const int groups = 300, seg = 1000;
    std::vector<int> h = random_ints((size_t)groups * seg, 2, -50, 50);
    dvec<int> d(h), o(h.size());
    stage("segment_scan");
    bulk::async(bulk::grid<128, 4>(groups, 16 * 1024), segment_scan(), bulk::root.this_exec, d.p, o.p, seg).wait();
    std::vector<int> want(h.size());
    for (int g = 0; g < groups; ++g) {
      int run = 7;
      for (int i = 0; i < seg; ++i) want[(size_t)g * seg + i] = (run += h[(size_t)g * seg + i]);
    }
    check("grid<128,4>(300) inclusive_scan per group", o.get(), want);
  }
}

// ============================================================================
// group algorithms: one CTA of 128 agents with grainsize 4
// ============================================================================
typedef bulk::concurrent_group<bulk::agent<4>, 128> group_t;

struct k_reduce {
  __device__ void operator()(group_t &g, const int *x, int n, int *out) {
    const int r = bulk::reduce(g, x, x + n, 5, plus_i());
    out[g.this_exec.index()] = r;  // every agent receives the result
  }
};
struct k_reduce_affine {
  __device__ void operator()(group_t &g, const affine *x, int n, affine *out) {
    const affine r = bulk::reduce(g, x, x + n, affine{1u, 0u}, compose());
    const affine r2 = bulk::accumulate(g, x, x + n, affine{3u, 1u}, compose());
    if (g.this_exec.index() == 0) {
      out[0] = r;
      out[1] = r2;
    }
  }
};
struct k_scans {
  __device__ void operator()(group_t &g, const int *x, int n, int *incl, int *incl_noinit, int *excl) {
    bulk::inclusive_scan(g, x, x + n, incl, 11, plus_i());
    bulk::inclusive_scan(g, x, x + n, incl_noinit, plus_i());
    bulk::exclusive_scan(g, x, x + n, excl, 11, plus_i());
  }
};
struct k_scan_affine {
  __device__ void operator()(group_t &g, const affine *x, int n, affine *incl, affine *excl) {
    bulk::inclusive_scan(g, x, x + n, incl, compose());
    bulk::exclusive_scan(g, x, x + n, excl, affine{1u, 0u}, compose());
  }
};
struct k_moves {
  struct nonneg {
    __device__ bool operator()(int) const { return true; }
  };
  struct twice {
    __device__ void operator()(int &v) const { v *= 2; }
  };
  __device__ void operator()(group_t &g, const int *x, int n, const int *map, const int *stencil, int *copied,
                             int *gathered, int *scattered, int *doubled, int *diff, int *diff_init, int *inplace) {
    bulk::copy_n(g, x, n, copied);
    bulk::gather(g, map, map + n, x, gathered);
    bulk::scatter_if(g, x, x + n, map, stencil, scattered);
    bulk::copy_n(g, x, n, doubled);
    bulk::for_each_n(g, doubled, n, twice());
    bulk::adjacent_difference(g, x, x + n, diff, minus_i());
    bulk::adjacent_difference(g, x, x + n, diff_init, 100, minus_i());
    bulk::copy_n(g, x, n, inplace);
    bulk::adjacent_difference(g, inplace, inplace + n, inplace, minus_i());
  }
};
struct k_merge {
  __device__ void operator()(group_t &g, const int *a, int na, const int *b, int nb, const int *av, const int *bv,
                             int *out, int *ok, int *ov, int *inplace) {
    bulk::merge(g, a, a + na, b, b + nb, out, less_i());
    bulk::merge_by_key(g, a, a + na, b, b + nb, av, bv, ok, ov, less_i());
    bulk::inplace_merge(g, inplace, inplace + na, inplace + na + nb, less_i());
  }
};
struct k_sort {
  __device__ void operator()(group_t &g, int *keys, int *vals, int n, int *keys_only) {
    bulk::stable_sort_by_key(bulk::bound<512>(g), keys, keys + n, vals, less_i());
    bulk::stable_sort(bulk::bound<512>(g), keys_only, keys_only + n, less_i());
  }
};
struct k_reduce_by_key {
  __device__ void operator()(group_t &g, const int *keys, const int *vals, int n, int *ok, int *ov, int *count) {
    auto r = bulk::reduce_by_key(g, keys, keys + n, vals, ok, ov, -1, 1000, eq_i(), plus_i());
    if (g.this_exec.index() == 0) {
      // the result is a thrust::tuple, read the way the reference's callers do
      int *k_end = thrust::get<0>(r);
      int *v_end = thrust::get<1>(r);
      *k_end = thrust::get<2>(r);  // the open run closes at the end
      *v_end = thrust::get<3>(r);
      *count = int(k_end - ok) + 1;
    }
  }
};
struct k_heap {
  __device__ void operator()(group_t &g, int *flags) {
    int *a = static_cast<int *>(bulk::malloc(g, 1024));
    int *b = static_cast<int *>(bulk::malloc(g, 1 << 20));  // larger than the heap: device heap
    if (g.this_exec.index() == 0) {
      flags[0] = bulk::is_on_chip(a);
      flags[1] = b != nullptr && !bulk::is_on_chip(b);
    }
    a[g.this_exec.index()] = g.this_exec.index();
    g.wait();
    int s = bulk::reduce(g, a, a + g.size(), 0, plus_i());
    if (g.this_exec.index() == 0) flags[2] = s;
    bulk::free(g, b);
    bulk::free(g, a);
    int *c = static_cast<int *>(bulk::malloc(g, 1024));
    if (g.this_exec.index() == 0) flags[3] = (c == a);  // the heap is a stack: a's block is reused
    bulk::free(g, c);
  }
};
struct k_strided {
  __device__ void operator()(group_t &g, const int *x, int n, int stride, int *out) {
    auto f = bulk::make_strided_iterator(x, stride);
    auto l = bulk::make_strided_iterator(x + n, stride);
    const int r = bulk::reduce(g, f, l, 0, plus_i());
    if (g.this_exec.index() == 0) *out = r;
  }
};
struct k_uninit {
  __device__ void operator()(group_t &g, int *out) {
    __shared__ bulk::uninitialized<affine> u;
    __shared__ bulk::uninitialized_array<int, 128> arr;
    if (g.this_exec.index() == 0) u.construct(affine{3u, 4u});
    arr[g.this_exec.index()] = g.this_exec.index() + 1;
    g.wait();
    if (g.this_exec.index() == 0) {
      out[0] = (int)u.get().a + (int)u.get().b;
      int s = 0;
      for (const int *it = arr.begin(); it != arr.end(); ++it) s += *it;
      out[1] = s;
      out[2] = (int)arr.size();
    }
  }
};

static std::vector<int> sorted_ints(size_t n, uint32_t seed, int hi) {
  std::vector<int> v = random_ints(n, seed, 0, hi);
  std::sort(v.begin(), v.end());
  return v;
}

static void group_algorithms() {
  const int heap = 64 * 1024;
  for (int n : {0, 1, 7, 127, 128, 513, 4096, 100003}) {
    char name[96];
    std::vector<int> h = random_ints(n, 10 + n, -1000, 1000);
    dvec<int> d(h);
    {
      dvec<int> out(128);
      stage("k_reduce");
      bulk::async(bulk::con<128, 4>(heap), k_reduce(), bulk::root, d.p, n, out.p).wait();
      std::snprintf(name, sizeof name, "group reduce n=%d (all agents)", n);
      check(name, out.get(), std::vector<int>(128, std::accumulate(h.begin(), h.end(), 5)));
    }
    {
      std::vector<affine> ha = random_affine(n, 20 + n);
      dvec<affine> da(ha), out(2);
      stage("k_reduce_affine");
      bulk::async(bulk::con<128, 4>(heap), k_reduce_affine(), bulk::root, da.p, n, out.p).wait();
      affine w1{1u, 0u}, w2{3u, 1u};
      for (auto &x : ha) {
        w1 = compose()(w1, x);
        w2 = compose()(w2, x);
      }
      std::snprintf(name, sizeof name, "group reduce/accumulate non-commutative n=%d", n);
      check(name, out.get(), std::vector<affine>{w1, w2});
      dvec<affine> incl(n), excl(n);
      stage("k_scan_affine");
      bulk::async(bulk::con<128, 4>(heap), k_scan_affine(), bulk::root, da.p, n, incl.p, excl.p).wait();
      std::vector<affine> wi(n), we(n);
      affine run{1u, 0u};
      for (int i = 0; i < n; ++i) {
        we[i] = run;
        run = compose()(run, ha[i]);
        wi[i] = i == 0 ? ha[0] : compose()(wi[i - 1], ha[i]);
      }
      std::snprintf(name, sizeof name, "group inclusive_scan non-commutative n=%d", n);
      check(name, incl.get(), wi);
      std::snprintf(name, sizeof name, "group exclusive_scan non-commutative n=%d", n);
      check(name, excl.get(), we);
    }
    {
      dvec<int> incl(n), incl0(n), excl(n);
      stage("k_scans");
      bulk::async(bulk::con<128, 4>(heap), k_scans(), bulk::root, d.p, n, incl.p, incl0.p, excl.p).wait();
      std::vector<int> wi(n), w0(n), we(n);
      int run = 11, run0 = 0, rune = 11;
      for (int i = 0; i < n; ++i) {
        wi[i] = (run += h[i]);
        w0[i] = (run0 += h[i]);
        we[i] = rune;
        rune += h[i];
      }
      std::snprintf(name, sizeof name, "group inclusive_scan init n=%d", n);
      check(name, incl.get(), wi);
      std::snprintf(name, sizeof name, "group inclusive_scan no init n=%d", n);
      check(name, incl0.get(), w0);
      std::snprintf(name, sizeof name, "group exclusive_scan n=%d", n);
      check(name, excl.get(), we);
    }
    {
      std::vector<int> map(n), stencil(n);
      std::iota(map.begin(), map.end(), 0);
      std::shuffle(map.begin(), map.end(), std::mt19937(30 + n));
      for (int i = 0; i < n; ++i) stencil[i] = (h[i] & 1);
      dvec<int> dm(map), ds(stencil), copied(n), gathered(n), scattered(n), doubled(n), diff(n), diff_init(n),
          inplace(n);
      CUDA_OK(cudaMemset(scattered.p, 0xff, sizeof(int) * (n ? n : 1)));
      stage("k_moves");
      bulk::async(bulk::con<128, 4>(heap), k_moves(), bulk::root, d.p, n, dm.p, ds.p, copied.p, gathered.p,
                  scattered.p, doubled.p, diff.p, diff_init.p, inplace.p)
          .wait();
      std::vector<int> wg(n), wsc(n, -1), wd(n), wdiff(n), wdi(n);
      for (int i = 0; i < n; ++i) {
        wg[i] = h[map[i]];
        if (stencil[i]) wsc[map[i]] = h[i];
        wd[i] = 2 * h[i];
        wdiff[i] = i == 0 ? h[0] : h[i] - h[i - 1];
        wdi[i] = h[i] - (i == 0 ? 100 : h[i - 1]);
      }
      std::snprintf(name, sizeof name, "group copy_n n=%d", n);
      check(name, copied.get(), h);
      std::snprintf(name, sizeof name, "group gather n=%d", n);
      check(name, gathered.get(), wg);
      std::snprintf(name, sizeof name, "group scatter_if n=%d", n);
      check(name, scattered.get(), wsc);
      std::snprintf(name, sizeof name, "group for_each_n n=%d", n);
      check(name, doubled.get(), wd);
      std::snprintf(name, sizeof name, "group adjacent_difference n=%d", n);
      check(name, diff.get(), wdiff);
      std::snprintf(name, sizeof name, "group adjacent_difference init n=%d", n);
      check(name, diff_init.get(), wdi);
      std::snprintf(name, sizeof name, "group adjacent_difference in place n=%d", n);
      check(name, inplace.get(), wdiff);
    }
    {
      dvec<int> out(1);
      stage("k_strided");
      bulk::async(bulk::con<128, 4>(heap), k_strided(), bulk::root, d.p, n, 3, out.p).wait();
      int w = 0;
      for (int i = 0; i < n; i += 3) w += h[i];
      std::snprintf(name, sizeof name, "group reduce strided_iterator n=%d", n);
      check(name, out.get(), std::vector<int>{w});
    }
  }
  // merge family: A and B with many equal keys across the two ranges
  for (auto nn : {std::pair<int, int>{0, 0}, {0, 5}, {9, 0}, {200, 311}, {3000, 2000}, {40000, 1}}) {
    const int na = nn.first, nb = nn.second;
    char name[96];
    std::vector<int> a = sorted_ints(na, 40 + na, 300), b = sorted_ints(nb, 50 + nb, 300);
    std::vector<int> av(na), bv(nb);
    for (int i = 0; i < na; ++i) av[i] = i;
    for (int i = 0; i < nb; ++i) bv[i] = 1000000 + i;
    std::vector<int> ab(a);
    ab.insert(ab.end(), b.begin(), b.end());
    dvec<int> da(a), db(b), dav(av), dbv(bv), out(na + nb), ok(na + nb), ov(na + nb), inplace(ab);
    stage("k_merge");
    bulk::async(bulk::con<128, 4>(heap), k_merge(), bulk::root, da.p, na, db.p, nb, dav.p, dbv.p, out.p, ok.p,
                ov.p, inplace.p)
        .wait();
    // stable merge, ties from A first
    std::vector<std::pair<int, int>> pa(na), pb(nb), pm;
    for (int i = 0; i < na; ++i) pa[i] = {a[i], av[i]};
    for (int i = 0; i < nb; ++i) pb[i] = {b[i], bv[i]};
    std::merge(pa.begin(), pa.end(), pb.begin(), pb.end(), std::back_inserter(pm),
               [](const std::pair<int, int> &x, const std::pair<int, int> &y) { return x.first < y.first; });
    std::vector<int> wk(na + nb), wv(na + nb);
    for (int i = 0; i < na + nb; ++i) {
      wk[i] = pm[i].first;
      wv[i] = pm[i].second;
    }
    std::snprintf(name, sizeof name, "group merge na=%d nb=%d", na, nb);
    check(name, out.get(), wk);
    std::snprintf(name, sizeof name, "group merge_by_key keys na=%d nb=%d", na, nb);
    check(name, ok.get(), wk);
    std::snprintf(name, sizeof name, "group merge_by_key values (ties take A) na=%d nb=%d", na, nb);
    check(name, ov.get(), wv);
    std::snprintf(name, sizeof name, "group inplace_merge na=%d nb=%d", na, nb);
    check(name, inplace.get(), wk);
  }
  // bounded group sort: n <= 128 x 4, few distinct keys to expose stability
  for (int n : {0, 1, 4, 5, 100, 333, 512}) {
    char name[96];
    std::vector<int> k = random_ints(n, 60 + n, 0, 9), v(n);
    std::iota(v.begin(), v.end(), 0);
    dvec<int> dk(k), dv(v), dko(k);
    stage("k_sort");
    bulk::async(bulk::con<128, 4>(heap), k_sort(), bulk::root, dk.p, dv.p, n, dko.p).wait();
    std::vector<int> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return k[x] < k[y]; });
    std::vector<int> wk(n), wv(n);
    for (int i = 0; i < n; ++i) {
      wk[i] = k[idx[i]];
      wv[i] = idx[i];
    }
    std::snprintf(name, sizeof name, "group stable_sort_by_key keys n=%d", n);
    check(name, dk.get(), wk);
    std::snprintf(name, sizeof name, "group stable_sort_by_key values (stable) n=%d", n);
    check(name, dv.get(), wv);
    std::snprintf(name, sizeof name, "group stable_sort n=%d", n);
    check(name, dko.get(), wk);
  }
  // reduce_by_key with a carried (key, value) = (-1, 1000)
  for (int n : {0, 1, 2, 513, 5000, 70001}) {
    char name[96];
    std::vector<int> k(n), v = random_ints(n, 70 + n, -5, 5);
    std::mt19937 r(80 + n);
    int key = (n % 2) ? -1 : 0;  // odd sizes continue the carried key's run
    for (int i = 0; i < n; ++i) {
      if (r() % 4 == 0) key += 1 + int(r() % 3);
      k[i] = key;
    }
    dvec<int> dk(k), dv(v), ok(n + 1), ov(n + 1), cnt(1);
    stage("k_reduce_by_key");
    bulk::async(bulk::con<128, 4>(heap), k_reduce_by_key(), bulk::root, dk.p, dv.p, n, ok.p, ov.p, cnt.p).wait();
    std::vector<int> wk{-1}, wv{1000};
    for (int i = 0; i < n; ++i) {
      if (k[i] == wk.back()) wv.back() += v[i];
      else {
        wk.push_back(k[i]);
        wv.push_back(v[i]);
      }
    }
    const int c = cnt.get()[0];
    std::vector<int> gk = ok.get(), gv = ov.get();
    gk.resize(std::max(c, 0));
    gv.resize(std::max(c, 0));
    std::snprintf(name, sizeof name, "group reduce_by_key keys n=%d", n);
    check(name, gk, wk);
    std::snprintf(name, sizeof name, "group reduce_by_key values n=%d", n);
    check(name, gv, wv);
  }
  {
    dvec<int> flags(4);
    stage("k_heap");
    bulk::async(bulk::con<128, 4>(4096), k_heap(), bulk::root, flags.p).wait();
    check("group malloc on chip / device heap fallback / stack reuse", flags.get(),
          std::vector<int>{1, 1, 127 * 128 / 2, 1});
  }
  {
    dvec<int> out(3);
    stage("k_uninit");
    bulk::async(bulk::con<128, 4>(heap), k_uninit(), bulk::root, out.p).wait();
    check("uninitialized / uninitialized_array in shared memory", out.get(), std::vector<int>{7, 128 * 129 / 2, 128});
  }
}

// ============================================================================
// agent-level bounded algorithms: every agent works on its own 8 elements
// ============================================================================
struct k_agent {
  __device__ void operator()(bulk::agent<8> &self, const int *x, int n, int *red, int *incl, int *excl, int *sorted,
                             int *sv, int *merged, int *mk, int *mv) {
    const int i = self.index();
    const int *xi = x + 8 * i;
    const int cnt = n - 8 * i < 8 ? n - 8 * i : 8;
    if (cnt <= 0) return;
    red[i] = bulk::reduce(bulk::bound<8>(self), xi, xi + cnt, 1, plus_i());
    bulk::inclusive_scan(bulk::bound<8>(self), xi, xi + cnt, incl + 8 * i, 1, plus_i());
    bulk::exclusive_scan(bulk::bound<8>(self), xi, xi + cnt, excl + 8 * i, 1, plus_i());
    int k[8], v[8];
    for (int j = 0; j < cnt; ++j) {
      k[j] = xi[j] & 3;
      v[j] = j;
    }
    bulk::stable_sort_by_key(bulk::bound<8>(self), k, k + cnt, v, less_i());
    for (int j = 0; j < cnt; ++j) {
      sorted[8 * i + j] = k[j];
      sv[8 * i + j] = v[j];
    }
    // merge the two sorted halves of k; the bound caps the output at 8
    const int h = cnt / 2;
    int out[8];
    bulk::merge(bulk::bound<8>(self), k, k + h, k + h, k + cnt, out, less_i());
    for (int j = 0; j < cnt; ++j) merged[8 * i + j] = out[j];
    int ok[8], ov[8];
    bulk::merge_by_key(bulk::bound<8>(self), k, k + h, k + h, k + cnt, v, v + h, ok, ov, less_i());
    for (int j = 0; j < cnt; ++j) {
      mk[8 * i + j] = ok[j];
      mv[8 * i + j] = ov[j];
    }
  }
};

static void agent_algorithms() {
  const int n = 8 * 1000 + 5, agents = (n + 7) / 8;
  std::vector<int> h = random_ints(n, 90, -100, 100);
  dvec<int> d(h), red(agents), incl(n), excl(n), sorted(n), sv(n), merged(n), mk(n), mv(n);
  stage("k_agent");
  bulk::async(bulk::par(bulk::agent<8>(), agents), k_agent(), bulk::root.this_exec, d.p, n, red.p, incl.p, excl.p,
              sorted.p, sv.p, merged.p, mk.p, mv.p)
      .wait();
  std::vector<int> wr(agents), wi(n), we(n), ws(n), wsv(n), wm(n), wmk(n), wmv(n);
  for (int a = 0; a < agents; ++a) {
    const int b = 8 * a, cnt = std::min(8, n - b);
    int run = 1;
    for (int j = 0; j < cnt; ++j) {
      we[b + j] = run;
      run += h[b + j];
      wi[b + j] = run;
    }
    wr[a] = run;
    std::vector<int> idx(cnt);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return (h[b + x] & 3) < (h[b + y] & 3); });
    std::vector<int> k(cnt), v(cnt);
    for (int j = 0; j < cnt; ++j) {
      k[j] = ws[b + j] = h[b + idx[j]] & 3;
      v[j] = wsv[b + j] = idx[j];
    }
    const int hh = cnt / 2;
    std::vector<std::pair<int, int>> pa, pb, pm;
    for (int j = 0; j < hh; ++j) pa.push_back({k[j], v[j]});
    for (int j = hh; j < cnt; ++j) pb.push_back({k[j], v[j]});
    std::merge(pa.begin(), pa.end(), pb.begin(), pb.end(), std::back_inserter(pm),
               [](const std::pair<int, int> &x, const std::pair<int, int> &y) { return x.first < y.first; });
    for (int j = 0; j < cnt; ++j) {
      wm[b + j] = wmk[b + j] = pm[j].first;
      wmv[b + j] = pm[j].second;
    }
  }
  check("agent bounded reduce", red.get(), wr);
  check("agent bounded inclusive_scan", incl.get(), wi);
  check("agent bounded exclusive_scan", excl.get(), we);
  check("agent bounded stable_sort_by_key keys", sorted.get(), ws);
  check("agent bounded stable_sort_by_key values", sv.get(), wsv);
  check("agent bounded merge", merged.get(), wm);
  check("agent bounded merge_by_key keys", mk.get(), wmk);
  check("agent bounded merge_by_key values", mv.get(), wmv);
}

// ============================================================================
// thread-block clusters: concurrent groups of CTAs, distributed shared memory
// ============================================================================
typedef bulk::concurrent_group<bulk::agent<1>, 128> cta128_t;
typedef bulk::concurrent_group<cta128_t, 4> cluster4_t;
typedef bulk::concurrent_group<bulk::agent<1>, 64> cta64_t;
typedef bulk::concurrent_group<cta64_t, 2> cluster2_t;

struct k_cluster_reduce {  // one cluster of 4 CTAs reduces the whole range
  __device__ void operator()(cluster4_t &g, const int *data, int n, int *out, int *ranks) {
    const int s = bulk::reduce(g, data, data + n, 7, plus_i());
    const int rank = g.this_exec.index(), t = g.this_exec.this_exec.index();
    if (t == 0) {
      out[rank] = s;  // every CTA holds the same result
      ranks[rank] = (int)bulk::detail::cluster_ctarank() + 100 * g.size();
    }
  }
};
struct k_cluster_reduce_affine {  // a non-commutative operator across the cluster
  __device__ void operator()(cluster4_t &g, const affine *data, int n, affine *out) {
    const affine r = bulk::reduce(g, data, data + n, affine{1u, 0u}, compose());
    if (g.this_exec.index() == 0 && g.this_exec.this_exec.index() == 0) *out = r;
  }
};
struct k_cluster_grid {  // a grid of clusters, one segment per cluster
  __device__ void operator()(bulk::parallel_group<cluster2_t> &grid, const int *data, int seg, int *out) {
    cluster2_t &g = grid.this_exec;
    const int *first = data + (size_t)g.index() * seg;
    const int s = bulk::reduce(g, first, first + seg, 0, plus_i());
    if (g.this_exec.index() == 1 && g.this_exec.this_exec.index() == 0) out[g.index()] = s;
  }
};
// CTA 0 fills its own heap, so its next block comes from CTA 1's shared
// memory; CTA 1 checks the pattern in its own heap, then CTA 0 frees it.
struct k_cluster_dsmem {
  __device__ void operator()(cluster2_t &g, int *res) {
    const int rank = g.this_exec.index(), t = g.this_exec.this_exec.index();
    __shared__ int *s_far;
    if (rank == 0 && t == 0) {
      void *a = bulk::shmalloc(600);   // this CTA's heap (1024 bytes)
      void *b = bulk::shmalloc(600);   // does not fit here: the peer's heap
      res[0] = __isShared(a) ? 1 : 0;
      res[1] = (!__isShared(b) && bulk::is_on_chip(b)) ? 1 : 0;
      int *bi = static_cast<int *>(b);
      for (int i = 0; i < 150; ++i) bi[i] = 1000 + i;
      s_far = bi;
      bulk::shfree(a);
    }
    g.wait();
    if (rank == 1 && t == 0) {  // the block lives in this CTA's heap
      const unsigned char *heap = bulk::detail::s_bulk_heap;
      const int *mine = reinterpret_cast<const int *>(heap + sizeof(bulk::detail::heap_block_header));
      int ok = 1;
      for (int i = 0; i < 150; ++i) ok &= mine[i] == 1000 + i;
      res[2] = ok;
      res[3] = (int)bulk::detail::s_heap_top;
    }
    g.wait();
    if (rank == 0 && t == 0) bulk::shfree(s_far);
    g.wait();
    if (rank == 1 && t == 0) res[4] = (int)bulk::detail::s_heap_top;  // popped: 0
    // a collective allocation of the whole cluster: one block every CTA reaches
    int *shared_block = static_cast<int *>(bulk::malloc(g, 64 * sizeof(int)));
    if (rank == 1 && t < 64) shared_block[t] = 3 * t + 1;
    g.wait();
    if (rank == 0 && t == 0) {
      int ok = 1;
      for (int i = 0; i < 64; ++i) ok &= shared_block[i] == 3 * i + 1;
      res[5] = ok;
      res[6] = bulk::is_on_chip(shared_block) ? 1 : 0;
    }
    bulk::free(g, shared_block);
  }
};

static void cluster_programs() {
  {
    stage("cluster reduce");
    const int n = 100003;
    std::vector<int> h = random_ints(n, 41, -1000, 1000);
    dvec<int> d(h), out(4), ranks(4);
    bulk::async(bulk::cluster<4>(bulk::con<128, 1>(4096)), k_cluster_reduce(), bulk::root, d.p, n, out.p, ranks.p)
        .wait();
    const int want = std::accumulate(h.begin(), h.end(), 7);
    check("cluster group reduce (4 CTAs, every CTA's result)", out.get(), std::vector<int>(4, want));
    check("cluster group ranks", ranks.get(), std::vector<int>{400, 401, 402, 403});
  }
  {
    stage("cluster reduce affine");
    const int n = 77777;
    std::vector<affine> h = random_affine(n, 43);
    dvec<affine> d(h), out(1);
    bulk::async(bulk::cluster<4>(bulk::con<128, 1>(4096)), k_cluster_reduce_affine(), bulk::root, d.p, n, out.p)
        .wait();
    affine want{1u, 0u};
    for (const affine &x : h) want = compose()(want, x);
    check("cluster group reduce non-commutative", out.get(), std::vector<affine>{want});
  }
  {
    stage("cluster grid");
    const int clusters = 37, seg = 5001;
    std::vector<int> h = random_ints((size_t)clusters * seg, 47, -100, 100);
    dvec<int> d(h), out(clusters);
    bulk::async(bulk::par(bulk::cluster<2>(bulk::con<64, 1>(2048)), clusters), k_cluster_grid(), bulk::root, d.p, seg,
                out.p)
        .wait();
    std::vector<int> want(clusters);
    for (int c = 0; c < clusters; ++c) want[c] = std::accumulate(h.begin() + (size_t)c * seg, h.begin() + (size_t)(c + 1) * seg, 0);
    check("grid of clusters reduce", out.get(), want);
  }
  {
    stage("cluster dsmem malloc");
    dvec<int> res(7);
    res.put(std::vector<int>(7, -1));
    bulk::async(bulk::cluster<2>(bulk::con<64, 1>(1024)), k_cluster_dsmem(), bulk::root, res.p).wait();
    check("cluster heap: local block, then a block in the peer CTA's shared memory (DSMEM)", res.get(),
          std::vector<int>{1, 1, 1, 624, 0, 1, 1});
  }
  {
    stage("errors raise thrust::system_error");
    bool caught = false;
    try {
      bulk::async(bulk::con(2048), sum(), bulk::root, (const int *)nullptr, 0, (int *)nullptr).wait();
    } catch (const thrust::system_error &e) {
      caught = e.code().value() != 0;
    }
    check_true("errors raise thrust::system_error", caught);
  }
}

int main(int argc, char **argv) {
  std::setvbuf(stdout, nullptr, _IONBF, 0);
  const std::string only = argc > 1 ? argv[1] : "";
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) {
    std::printf("FAIL no CUDA device\n");
    return 2;
  }
  start_watchdog();
  if (only.empty() || only == "drivers") driver_programs();
  if (only.empty() || only == "group") group_algorithms();
  if (only.empty() || only == "agent") agent_algorithms();
  if (only.empty() || only == "cluster") cluster_programs();
  CUDA_OK(cudaDeviceSynchronize());
  std::printf("%s: %d failure(s)\n", g_failures ? "FAILED" : "PASSED", g_failures);
  return g_failures ? 1 : 0;
}
