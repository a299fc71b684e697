/*
 * oracle.c -- TEST INFRASTRUCTURE ONLY.  CPU restatement of the reference's
 * device-wide algorithms (jaredhoberock/bulk), used by tests/, smoke() and the
 * CPU-baseline leg of bench.py to check the CUDA library.  Nothing in the
 * product links, loads or calls this file.
 *
 * Each function cites the reference file:line whose semantics it restates.
 * Integer results are exact; floating-point reductions and scans accumulate in
 * long double (x87 80-bit) so they are more accurate than any float/double
 * result they check, and also return the sum of magnitudes used in the error
 * bound |got - ref| <= 2*ceil(log2 n)*eps*sum|x|.
 *
 * Pinning: see tests/test_oracle.py (known-answer tests of the reference's
 * drivers and the fixtures in tests/golden/).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Data generators (counter-based, identical on CPU and GPU)                */
/* ------------------------------------------------------------------------ */

/* splitmix64 finaliser of (seed, index): a published counter-based mixer
 * (Steele, Lea, Flood 2014). */
uint64_t bko_mix64(uint64_t seed, uint64_t i) {
  uint64_t z = seed * 0x9E3779B97F4A7C15ull + (i + 1) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

void bko_gen_i32(int32_t *out, uint64_t n, uint64_t seed, int32_t lo, int32_t hi) {
  const uint64_t span = (uint64_t)((int64_t)hi - (int64_t)lo + 1);
  for (uint64_t i = 0; i < n; ++i) out[i] = (int32_t)((int64_t)lo + (int64_t)(bko_mix64(seed, i) % span));
}

void bko_gen_u32(uint32_t *out, uint64_t n, uint64_t seed) {
  for (uint64_t i = 0; i < n; ++i) out[i] = (uint32_t)(bko_mix64(seed, i) >> 32);
}

void bko_gen_u64(uint64_t *out, uint64_t n, uint64_t seed) {
  for (uint64_t i = 0; i < n; ++i) out[i] = bko_mix64(seed, i);
}

/* uniform in [lo, hi): 24 random mantissa bits, exact in float */
void bko_gen_f32(float *out, uint64_t n, uint64_t seed, float lo, float hi) {
  for (uint64_t i = 0; i < n; ++i) {
    float u = (float)(bko_mix64(seed, i) >> 40) * (1.0f / 16777216.0f);
    out[i] = lo + (hi - lo) * u;
  }
}

/* uniform in [lo, hi): 53 random mantissa bits */
void bko_gen_f64(double *out, uint64_t n, uint64_t seed, double lo, double hi) {
  for (uint64_t i = 0; i < n; ++i) {
    double u = (double)(bko_mix64(seed, i) >> 11) * (1.0 / 9007199254740992.0);
    out[i] = lo + (hi - lo) * u;
  }
}

/* The reference drivers' random_fill: thrust::tabulate of a Jenkins-style
 * 32-bit integer hash (merge.cu:203-218, merge_sort_by_key.cu:264-279,
 * reduce_by_key.cu:305-321).  thrust::tabulate passes the element index as the
 * iterator's difference type (64-bit ptrdiff_t), so the mixing runs on a
 * 64-bit signed value and the result is truncated to the element type. */
int64_t bko_ref_hash(int64_t x) {
  x = (x + 0x7ed55d16) + (x << 12);
  x = (x ^ 0xc761c23c) ^ (x >> 19);
  x = (x + 0x165667b1) + (x << 5);
  x = (x + 0xd3a2646c) ^ (x << 9);
  x = (x + 0xfd7046c5) + (x << 3);
  x = (x ^ 0xb55a4f09) ^ (x >> 16);
  return x;
}

void bko_ref_hash_fill_i32(int32_t *out, uint64_t n, int32_t modulus) {
  for (uint64_t i = 0; i < n; ++i) {
    int64_t h = bko_ref_hash((int64_t)i);
    out[i] = modulus > 0 ? (int32_t)(h % modulus) : (int32_t)(uint32_t)(uint64_t)h;
  }
}

/* ------------------------------------------------------------------------ */
/* reduce: reduce.cu:58-97 / bulk/algorithm/reduce.hpp:110-219               */
/* result = init (+) x[0] (+) ... (+) x[n-1]; n == 0 returns init            */
/* ------------------------------------------------------------------------ */
#define DEF_REDUCE_INT(NAME, T)                                            \
  T bko_reduce_sum_##NAME(const T *x, uint64_t n, T init) {                \
    typedef __typeof__((T)0 + (T)0) W;                                     \
    uint64_t acc = (uint64_t)(W)init; /* modular arithmetic */             \
    for (uint64_t i = 0; i < n; ++i) acc += (uint64_t)(int64_t)(W)x[i];    \
    return (T)acc;                                                         \
  }                                                                        \
  T bko_reduce_min_##NAME(const T *x, uint64_t n, T init) {                \
    T acc = init;                                                          \
    for (uint64_t i = 0; i < n; ++i) acc = acc < x[i] ? acc : x[i];        \
    return acc;                                                            \
  }                                                                        \
  T bko_reduce_max_##NAME(const T *x, uint64_t n, T init) {                \
    T acc = init;                                                          \
    for (uint64_t i = 0; i < n; ++i) acc = acc < x[i] ? x[i] : acc;        \
    return acc;                                                            \
  }
DEF_REDUCE_INT(i32, int32_t)
DEF_REDUCE_INT(u32, uint32_t)
DEF_REDUCE_INT(i64, int64_t)
DEF_REDUCE_INT(u64, uint64_t)

#define DEF_REDUCE_FLT(NAME, T)                                                         \
  double bko_reduce_sum_##NAME(const T *x, uint64_t n, T init, double *abs_sum) {      \
    long double acc = init, mag = init < 0 ? -(long double)init : (long double)init;   \
    for (uint64_t i = 0; i < n; ++i) {                                                  \
      acc += x[i];                                                                      \
      mag += x[i] < 0 ? -(long double)x[i] : (long double)x[i];                         \
    }                                                                                   \
    if (abs_sum) *abs_sum = (double)mag;                                                \
    return (double)acc;                                                                 \
  }                                                                                     \
  T bko_reduce_min_##NAME(const T *x, uint64_t n, T init) {                             \
    T acc = init;                                                                       \
    for (uint64_t i = 0; i < n; ++i) acc = acc < x[i] ? acc : x[i];                     \
    return acc;                                                                         \
  }                                                                                     \
  T bko_reduce_max_##NAME(const T *x, uint64_t n, T init) {                             \
    T acc = init;                                                                       \
    for (uint64_t i = 0; i < n; ++i) acc = acc < x[i] ? x[i] : acc;                     \
    return acc;                                                                         \
  }
DEF_REDUCE_FLT(f32, float)
DEF_REDUCE_FLT(f64, double)

/* ------------------------------------------------------------------------ */
/* inclusive scan: scan.cu:87-148, semantics scan.cu:158-184 (result[i] =    */
/* init + x[0] + ... + x[i]) and bulk/algorithm/scan.hpp:455-486            */
/* ------------------------------------------------------------------------ */
#define DEF_SCAN_INT(NAME, T)                                                            \
  void bko_inclusive_scan_sum_##NAME(const T *x, uint64_t n, T init, T *out) {          \
    uint64_t acc = (uint64_t)(int64_t)init;                                              \
    for (uint64_t i = 0; i < n; ++i) {                                                   \
      acc += (uint64_t)(int64_t)x[i];                                                    \
      out[i] = (T)acc;                                                                   \
    }                                                                                    \
  }                                                                                      \
  void bko_inclusive_scan_min_##NAME(const T *x, uint64_t n, T init, T *out) {          \
    T acc = init;                                                                        \
    for (uint64_t i = 0; i < n; ++i) out[i] = acc = acc < x[i] ? acc : x[i];             \
  }                                                                                      \
  void bko_inclusive_scan_max_##NAME(const T *x, uint64_t n, T init, T *out) {          \
    T acc = init;                                                                        \
    for (uint64_t i = 0; i < n; ++i) out[i] = acc = acc < x[i] ? x[i] : acc;             \
  }
DEF_SCAN_INT(i32, int32_t)
DEF_SCAN_INT(u32, uint32_t)
DEF_SCAN_INT(i64, int64_t)
DEF_SCAN_INT(u64, uint64_t)

#define DEF_SCAN_FLT(NAME, T)                                                                    \
  void bko_inclusive_scan_sum_##NAME(const T *x, uint64_t n, T init, double *out, double *abs_prefix) { \
    long double acc = init, mag = init < 0 ? -(long double)init : (long double)init;             \
    for (uint64_t i = 0; i < n; ++i) {                                                           \
      acc += x[i];                                                                               \
      mag += x[i] < 0 ? -(long double)x[i] : (long double)x[i];                                  \
      out[i] = (double)acc;                                                                      \
      if (abs_prefix) abs_prefix[i] = (double)mag;                                               \
    }                                                                                            \
  }                                                                                              \
  void bko_inclusive_scan_min_##NAME(const T *x, uint64_t n, T init, T *out) {                  \
    T acc = init;                                                                                \
    for (uint64_t i = 0; i < n; ++i) out[i] = acc = acc < x[i] ? acc : x[i];                     \
  }                                                                                              \
  void bko_inclusive_scan_max_##NAME(const T *x, uint64_t n, T init, T *out) {                  \
    T acc = init;                                                                                \
    for (uint64_t i = 0; i < n; ++i) out[i] = acc = acc < x[i] ? x[i] : acc;                     \
  }
DEF_SCAN_FLT(f32, float)
DEF_SCAN_FLT(f64, double)

/* ------------------------------------------------------------------------ */
/* merge_path: bulk/algorithm/merge.hpp:35-60.  Number of elements taken from */
/* A among the first `diag` outputs; on ties A goes first.                   */
/* ------------------------------------------------------------------------ */
#define DEF_MERGE(NAME, K)                                                                        \
  uint64_t bko_merge_path_##NAME(const K *a, uint64_t na, const K *b, uint64_t nb, uint64_t diag) { \
    uint64_t lo = diag > nb ? diag - nb : 0, hi = diag < na ? diag : na;                           \
    while (lo < hi) {                                                                              \
      uint64_t mid = (lo + hi) >> 1;                                                               \
      if (b[diag - 1 - mid] < a[mid]) hi = mid; else lo = mid + 1;                                 \
    }                                                                                              \
    return lo;                                                                                     \
  }                                                                                                \
  /* stable merge (merge.hpp:63-170 agent loop; ties take A: merge.hpp:111) with an opaque */     \
  /* payload of vbytes bytes per element (0 = keys only; merge.hpp:507-607 by-key)          */     \
  void bko_merge_##NAME(const K *a, const void *av, uint64_t na, const K *b, const void *bv,      \
                        uint64_t nb, K *out, void *outv, int vbytes) {                             \
    uint64_t i = 0, j = 0, o = 0;                                                                  \
    const char *pa = (const char *)av, *pb = (const char *)bv;                                     \
    char *po = (char *)outv;                                                                       \
    while (i < na || j < nb) {                                                                     \
      int take_a = (j >= nb) || (i < na && !(b[j] < a[i]));                                        \
      if (take_a) {                                                                                \
        out[o] = a[i];                                                                             \
        if (vbytes) memcpy(po + o * vbytes, pa + i * vbytes, (size_t)vbytes);                      \
        ++i;                                                                                       \
      } else {                                                                                     \
        out[o] = b[j];                                                                             \
        if (vbytes) memcpy(po + o * vbytes, pb + j * vbytes, (size_t)vbytes);                      \
        ++j;                                                                                       \
      }                                                                                            \
      ++o;                                                                                         \
    }                                                                                              \
  }                                                                                                \
  /* stable sort by key: the reference's stable_merge_sort_by_key (merge_sort_by_key.cu:150-209, */ \
  /* block sort bulk/algorithm/detail/stable_merge_sort.hpp:125-206) is a stable merge sort;      */ \
  /* a stable sort's output is unique, so a bottom-up merge sort restates it exactly.             */ \
  void bko_stable_sort_by_key_##NAME(K *keys, void *vals, uint64_t n, int vbytes) {               \
    if (n < 2) return;                                                                             \
    K *tk = (K *)malloc(n * sizeof(K));                                                            \
    char *tv = vbytes ? (char *)malloc(n * (size_t)vbytes) : NULL;                                 \
    K *sk = keys, *dk = tk;                                                                        \
    char *sv = (char *)vals, *dv = tv;                                                             \
    for (uint64_t w = 1; w < n; w *= 2) {                                                          \
      for (uint64_t lo = 0; lo < n; lo += 2 * w) {                                                 \
        uint64_t mid = lo + w < n ? lo + w : n, hi = lo + 2 * w < n ? lo + 2 * w : n;              \
        bko_merge_##NAME(sk + lo, vbytes ? sv + lo * vbytes : NULL, mid - lo, sk + mid,            \
                         vbytes ? sv + mid * vbytes : NULL, hi - mid, dk + lo,                     \
                         vbytes ? dv + lo * vbytes : NULL, vbytes);                                \
      }                                                                                            \
      K *t = sk; sk = dk; dk = t;                                                                  \
      char *u = sv; sv = dv; dv = u;                                                               \
    }                                                                                              \
    if (sk != keys) {                                                                              \
      memcpy(keys, sk, n * sizeof(K));                                                             \
      if (vbytes) memcpy(vals, sv, n * (size_t)vbytes);                                            \
    }                                                                                              \
    free(tk);                                                                                      \
    free(tv);                                                                                      \
  }
DEF_MERGE(i32, int32_t)
DEF_MERGE(u32, uint32_t)
DEF_MERGE(i64, int64_t)
DEF_MERGE(u64, uint64_t)
DEF_MERGE(f32, float)
DEF_MERGE(f64, double)

/* ------------------------------------------------------------------------ */
/* reduce_by_key: reduce_by_key.cu:176-272 with bulk/algorithm/             */
/* reduce_by_key.hpp:115-216.  One output pair per maximal run of equal      */
/* consecutive keys (pred = equal_to), in run order; value = left fold with  */
/* plus.  Returns the number of runs.                                        */
/* ------------------------------------------------------------------------ */
#define DEF_RBK_INT(KN, K, VN, V)                                                                   \
  uint64_t bko_reduce_by_key_##KN##_##VN(const K *keys, const V *vals, uint64_t n, K *out_keys,    \
                                         V *out_vals) {                                            \
    uint64_t r = 0;                                                                                 \
    for (uint64_t i = 0; i < n; ++i) {                                                              \
      if (i == 0 || !(keys[i] == keys[i - 1])) {                                                    \
        out_keys[r] = keys[i];                                                                      \
        out_vals[r] = vals[i];                                                                      \
        ++r;                                                                                        \
      } else {                                                                                      \
        out_vals[r - 1] = (V)((uint64_t)(int64_t)out_vals[r - 1] + (uint64_t)(int64_t)vals[i]);     \
      }                                                                                             \
    }                                                                                               \
    return r;                                                                                       \
  }
#define DEF_RBK_FLT(KN, K, VN, V)                                                                   \
  uint64_t bko_reduce_by_key_##KN##_##VN(const K *keys, const V *vals, uint64_t n, K *out_keys,    \
                                         double *out_vals, double *out_abs) {                      \
    uint64_t r = 0;                                                                                 \
    long double acc = 0, mag = 0;                                                                   \
    for (uint64_t i = 0; i < n; ++i) {                                                              \
      if (i == 0 || !(keys[i] == keys[i - 1])) {                                                    \
        if (r > 0) { out_vals[r - 1] = (double)acc; if (out_abs) out_abs[r - 1] = (double)mag; }    \
        out_keys[r] = keys[i];                                                                      \
        acc = 0; mag = 0;                                                                           \
        ++r;                                                                                        \
      }                                                                                             \
      acc += vals[i];                                                                               \
      mag += vals[i] < 0 ? -(long double)vals[i] : (long double)vals[i];                            \
    }                                                                                               \
    if (r > 0) { out_vals[r - 1] = (double)acc; if (out_abs) out_abs[r - 1] = (double)mag; }        \
    return r;                                                                                       \
  }
DEF_RBK_INT(i32, int32_t, i32, int32_t)
DEF_RBK_INT(i32, int32_t, i64, int64_t)
DEF_RBK_FLT(i32, int32_t, f32, float)
DEF_RBK_FLT(i32, int32_t, f64, double)
DEF_RBK_INT(i64, int64_t, i32, int32_t)
DEF_RBK_INT(i64, int64_t, i64, int64_t)
DEF_RBK_FLT(i64, int64_t, f32, float)
DEF_RBK_FLT(i64, int64_t, f64, double)
DEF_RBK_INT(u32, uint32_t, i32, int32_t)
DEF_RBK_FLT(u32, uint32_t, f32, float)
DEF_RBK_FLT(u32, uint32_t, f64, double)

/* Run-length generators for reduce_by_key inputs: keys are run indices
 * (sorted runs), lengths 1 + Geometric(p) or Zipf(s) capped at cap.  The
 * uniform draws come from bko_mix64(seed, run). */
uint64_t bko_gen_runs_geometric(int32_t *keys, uint64_t n, uint64_t seed, double mean) {
  /* 1 + Geom(p) with p = 1/mean (mean length ~ mean) by inversion */
  const double p = 1.0 / mean;
  uint64_t i = 0, run = 0;
  const long double lq = logl(1.0L - (long double)p);
  while (i < n) {
    double u = (double)(bko_mix64(seed, run) >> 11) * (1.0 / 9007199254740992.0);
    uint64_t len = 1 + (uint64_t)floorl(logl(1.0L - (long double)u) / lq);
    for (uint64_t k = 0; k < len && i < n; ++k) keys[i++] = (int32_t)run;
    ++run;
  }
  return run;
}

uint64_t bko_gen_runs_zipf(int32_t *keys, uint64_t n, uint64_t seed, double s, uint64_t cap) {
  /* Zipf(s) over {1..cap} by inversion of the continuous approximation
   * F(x) ~ (x^(1-s) - 1) / (cap^(1-s) - 1) (a bounded Pareto draw, rounded). */
  uint64_t i = 0, run = 0;
  const long double a = 1.0L - (long double)s;
  const long double top = powl((long double)cap + 1.0L, a) - 1.0L;
  while (i < n) {
    long double u = (long double)(bko_mix64(seed, run) >> 11) * (1.0L / 9007199254740992.0L);
    long double x = powl(1.0L + u * top, 1.0L / a);
    uint64_t len = (uint64_t)floorl(x);
    if (len < 1) len = 1;
    if (len > cap) len = cap;
    for (uint64_t k = 0; k < len && i < n; ++k) keys[i++] = (int32_t)run;
    ++run;
  }
  return run;
}

/* ------------------------------------------------------------------------ */
/* CPU baseline (timed by bench.py, not used for checking): the reference's  */
/* device-wide reduce and scan restated for host threads.  Like my_reduce    */
/* (reduce.cu:58-97) and the three-pass scan (scan.cu:87-148), the range is  */
/* split into `threads` aligned partitions; each partition is folded in T    */
/* (the element type), the partition sums are combined in order, and for the */
/* scan each partition is rescanned with its carry.                          */
/* ------------------------------------------------------------------------ */
#include <pthread.h>

typedef struct {
  const void *x;
  void *out;
  uint64_t lo, hi;
  int kind; /* 0 reduce, 1 scan-upsweep, 2 scan-downsweep */
  int type; /* 0 f32, 1 f64, 2 i32 */
  double carry_f;
  int64_t carry_i;
  double sum_f;
  int64_t sum_i;
} bko_part;

static void *bko_part_run(void *arg) {
  bko_part *p = (bko_part *)arg;
  if (p->type == 0) {
    const float *x = (const float *)p->x;
    float *o = (float *)p->out;
    float acc = p->kind == 2 ? (float)p->carry_f : 0.0f;
    if (p->kind == 2) {
      for (uint64_t i = p->lo; i < p->hi; ++i) { acc += x[i]; o[i] = acc; }
    } else {
      for (uint64_t i = p->lo; i < p->hi; ++i) acc += x[i];
    }
    p->sum_f = acc;
  } else if (p->type == 1) {
    const double *x = (const double *)p->x;
    double *o = (double *)p->out;
    double acc = p->kind == 2 ? p->carry_f : 0.0;
    if (p->kind == 2) {
      for (uint64_t i = p->lo; i < p->hi; ++i) { acc += x[i]; o[i] = acc; }
    } else {
      for (uint64_t i = p->lo; i < p->hi; ++i) acc += x[i];
    }
    p->sum_f = acc;
  } else {
    const int32_t *x = (const int32_t *)p->x;
    int32_t *o = (int32_t *)p->out;
    uint32_t acc = p->kind == 2 ? (uint32_t)p->carry_i : 0u;
    if (p->kind == 2) {
      for (uint64_t i = p->lo; i < p->hi; ++i) { acc += (uint32_t)x[i]; o[i] = (int32_t)acc; }
    } else {
      for (uint64_t i = p->lo; i < p->hi; ++i) acc += (uint32_t)x[i];
    }
    p->sum_i = (int32_t)acc;
  }
  return NULL;
}

static void bko_run_parts(bko_part *parts, int threads) {
  pthread_t tid[256];
  for (int t = 1; t < threads; ++t) pthread_create(&tid[t], NULL, bko_part_run, &parts[t]);
  bko_part_run(&parts[0]);
  for (int t = 1; t < threads; ++t) pthread_join(tid[t], NULL);
}

/* type: 0 f32, 1 f64, 2 i32.  Returns the reduction (as double / int64). */
double bko_baseline_reduce(const void *x, uint64_t n, int type, int threads) {
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  bko_part parts[256];
  for (int t = 0; t < threads; ++t) {
    parts[t] = (bko_part){x, NULL, n * t / threads, n * (t + 1) / threads, 0, type, 0, 0, 0, 0};
  }
  bko_run_parts(parts, threads);
  double f = 0; uint32_t s = 0;
  for (int t = 0; t < threads; ++t) {
    if (type == 2) s += (uint32_t)parts[t].sum_i;
    else f = type == 0 ? (double)((float)f + (float)parts[t].sum_f) : f + parts[t].sum_f;
  }
  return type == 2 ? (double)(int32_t)s : f;
}

void bko_baseline_inclusive_scan(const void *x, void *out, uint64_t n, int type, int threads) {
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  bko_part parts[256];
  for (int t = 0; t < threads; ++t) {
    parts[t] = (bko_part){x, out, n * t / threads, n * (t + 1) / threads, 1, type, 0, 0, 0, 0};
  }
  bko_run_parts(parts, threads); /* upsweep: partition sums */
  double cf = 0; uint32_t ci = 0;
  for (int t = 0; t < threads; ++t) { /* spine: exclusive scan of the sums */
    parts[t].kind = 2;
    parts[t].carry_f = cf;
    parts[t].carry_i = (int32_t)ci;
    if (type == 2) ci += (uint32_t)parts[t].sum_i;
    else cf = type == 0 ? (double)((float)cf + (float)parts[t].sum_f) : cf + parts[t].sum_f;
  }
  bko_run_parts(parts, threads); /* downsweep: rescan with carries */
}
