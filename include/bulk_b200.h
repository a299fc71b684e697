/*
 * bulk_b200.h -- C-ABI of the B200 (sm_100a) device-wide algorithm library.
 *
 * Every entry point takes plain device pointers, 64-bit element counts, a
 * caller-owned device workspace and a CUDA stream, and returns an int status
 * (BK_OK, a positive cudaError_t value, or a negative BK_ERR_* library code).
 * Calls are stream-ordered and asynchronous: results stay in device memory and
 * the caller synchronizes.  No entry point allocates memory.
 *
 * Each entry replaces one device-wide driver of the reference library
 * (jaredhoberock/bulk); the replaced interface is cited above each group as
 * file:line within that project.
 *
 * Workspace contract: query the size with bk_workspace_bytes(), allocate it on
 * the device, and zero-fill it once (bk_workspace_init or cudaMemset).  Every
 * call leaves its counters zeroed again.  One workspace serves one stream at a
 * time: calls that overlap on the device must use different workspaces.
 * Device-side failures (a look-back wait that ran out) are recorded in the
 * workspace and returned by bk_workspace_status().
 */
#ifndef BULK_B200_H
#define BULK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define BK_API __attribute__((visibility("default")))
#else
#define BK_API
#endif

/* Same underlying type as cudaStream_t; NULL is the legacy default stream. */
typedef struct CUstream_st *bk_stream_t;

/* ---- status codes ------------------------------------------------------ */
#define BK_OK 0
#define BK_ERR_INVALID_ARGUMENT (-1)    /* null pointer with n > 0, bad enum, ... */
#define BK_ERR_WORKSPACE_TOO_SMALL (-2) /* ws_bytes < bk_workspace_bytes(...)      */
#define BK_ERR_SPIN_TIMEOUT (-3)        /* a device-side wait hit its time limit   */
#define BK_ERR_MISALIGNED (-4)          /* pointer not aligned to its element size */
#define BK_ERR_TOO_LARGE (-5)           /* n beyond the supported maximum          */
#define BK_ERR_UNSUPPORTED (-6)         /* no sm_100 device / unsupported combo    */

/* ---- enums used by the workspace query ---------------------------------- */
#define BK_ALGO_REDUCE 1
#define BK_ALGO_INCLUSIVE_SCAN 2
#define BK_ALGO_MERGE 3
#define BK_ALGO_SORT_BY_KEY 4
#define BK_ALGO_REDUCE_BY_KEY 5

#define BK_DTYPE_NONE 0
#define BK_DTYPE_I32 1
#define BK_DTYPE_U32 2
#define BK_DTYPE_I64 3
#define BK_DTYPE_U64 4
#define BK_DTYPE_F32 5
#define BK_DTYPE_F64 6

/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
BK_API int bk_version(void);

/* Human-readable text for any status this library returns. */
BK_API const char *bk_status_string(int status);

/* Bytes of device workspace that one call of `algo` over n elements needs.
 * key_dtype is the element (reduce/scan) or key type; value_dtype is the
 * payload type (BK_DTYPE_NONE for keys-only / value-less algorithms).
 * Returns 0 for an unknown combination. */
BK_API size_t bk_workspace_bytes(int algo, int key_dtype, int value_dtype, uint64_t n);

/* Bytes of device workspace that one batched call (the *_batch entry points
 * below) of `algo` over `count` arrays needs; sizes[i] (host memory) is the
 * element count of array i.  Returns 0 for an unknown combination. */
BK_API size_t bk_batch_workspace_bytes(int algo, int key_dtype, int value_dtype, const uint64_t *sizes, uint32_t count);

/* Zero-fill a workspace on `stream` (the one-time initialisation). */
BK_API int bk_workspace_init(void *d_ws, size_t ws_bytes, bk_stream_t stream);

/* Synchronize `stream`, return the device-side status recorded in the
 * workspace by earlier calls (BK_OK or BK_ERR_SPIN_TIMEOUT) and clear it. */
BK_API int bk_workspace_status(void *d_ws, size_t ws_bytes, bk_stream_t stream);

/* Test hook (not thread-safe; process-wide).  Subsequent look-back kernels
 * make the tile with index skip_publish_tile (-1 = none) skip publishing its
 * status, and bound every look-back wait by spin_limit_ns (0 = default, 2 s).
 * Waiting tiles then give up, record BK_ERR_SPIN_TIMEOUT and return. */
BK_API int bk_debug_set_fault(int64_t skip_publish_tile, uint64_t spin_limit_ns);

/* ---- launch shapes ------------------------------------------------------
 * The device-wide algorithms size their grids (CTAs per SM) and L2 prefetch
 * distance from a table measured on a B200 by bulk_b200/tune.py and compiled
 * into the library, per op, element bytes (key + value bytes for the by-key
 * ops) and size class (n < 2^16, < 2^20, < 2^24, larger).  This replaces the
 * reference's choose_sizes / occupancy heuristics
 * (bulk/detail/choose_sizes.inl:32-117, cuda_launch_config.hpp:240-379).
 * bk_tune_lookup reports the shape a call of n elements would use;
 * bk_tune_override sets a process-wide shape for one table cell
 * (ctas_per_sm = 0 clears it), which is how the tuning procedure tries
 * shapes.  Ops: BK_TUNE_*; ctas_per_sm at most 8 (reduce), 2 (scan,
 * reduce_by_key), 3 (merge), 1 (sort); prefetch 0-4. */
#define BK_TUNE_REDUCE 0
#define BK_TUNE_SCAN 1
#define BK_TUNE_REDUCE_BY_KEY 2
#define BK_TUNE_MERGE 3
#define BK_TUNE_SORT 4
BK_API int bk_tune_lookup(int op, int elem_bytes, uint64_t n, int32_t *ctas_per_sm, int32_t *prefetch);
BK_API int bk_tune_override(int op, int elem_bytes, int size_class, int32_t ctas_per_sm, int32_t prefetch);

/* ---- reduce -------------------------------------------------------------
 * *d_out = init (+) in[0] (+) ... (+) in[n-1]; n == 0 writes init.
 * Replaces my_reduce(first, last, init, binary_op), reduce.cu:58-97, whose
 * partition kernel calls bulk::reduce(group, ...), bulk/algorithm/reduce.hpp:110-219.
 * Integer sums wrap modulo 2^32 / 2^64 like the reference's.  Floating-point
 * results are reproducible run to run for a given n and device. */
BK_API int bk_reduce_sum_i32(const int32_t *d_in, uint64_t n, int32_t init, int32_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_sum_u32(const uint32_t *d_in, uint64_t n, uint32_t init, uint32_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_sum_i64(const int64_t *d_in, uint64_t n, int64_t init, int64_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_sum_u64(const uint64_t *d_in, uint64_t n, uint64_t init, uint64_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_sum_f32(const float *d_in, uint64_t n, float init, float *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_sum_f64(const double *d_in, uint64_t n, double init, double *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_min_i32(const int32_t *d_in, uint64_t n, int32_t init, int32_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_min_u32(const uint32_t *d_in, uint64_t n, uint32_t init, uint32_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_min_i64(const int64_t *d_in, uint64_t n, int64_t init, int64_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_min_u64(const uint64_t *d_in, uint64_t n, uint64_t init, uint64_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_min_f32(const float *d_in, uint64_t n, float init, float *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_min_f64(const double *d_in, uint64_t n, double init, double *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_max_i32(const int32_t *d_in, uint64_t n, int32_t init, int32_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_max_u32(const uint32_t *d_in, uint64_t n, uint32_t init, uint32_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_max_i64(const int64_t *d_in, uint64_t n, int64_t init, int64_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_max_u64(const uint64_t *d_in, uint64_t n, uint64_t init, uint64_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_max_f32(const float *d_in, uint64_t n, float init, float *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_max_f64(const double *d_in, uint64_t n, double init, double *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);

/* ---- inclusive scan -----------------------------------------------------
 * d_out[i] = init (+) in[0] (+) ... (+) in[i]; in-place (d_out == d_in) is allowed.
 * Replaces ::inclusive_scan(first, last, result, init, binary_op), scan.cu:87-148
 * (upsweep accumulate_tiles :57-84, spine exclusive_scan_n :24-31, downsweep
 * inclusive_downsweep :34-54, which call bulk::inclusive_scan(group, ...),
 * bulk/algorithm/scan.hpp:455-486), as one single-pass look-back kernel. */
BK_API int bk_inclusive_scan_sum_i32(const int32_t *d_in, uint64_t n, int32_t init, int32_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_sum_u32(const uint32_t *d_in, uint64_t n, uint32_t init, uint32_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_sum_i64(const int64_t *d_in, uint64_t n, int64_t init, int64_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_sum_u64(const uint64_t *d_in, uint64_t n, uint64_t init, uint64_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_sum_f32(const float *d_in, uint64_t n, float init, float *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_sum_f64(const double *d_in, uint64_t n, double init, double *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_min_i32(const int32_t *d_in, uint64_t n, int32_t init, int32_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_min_u32(const uint32_t *d_in, uint64_t n, uint32_t init, uint32_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_min_i64(const int64_t *d_in, uint64_t n, int64_t init, int64_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_min_u64(const uint64_t *d_in, uint64_t n, uint64_t init, uint64_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_min_f32(const float *d_in, uint64_t n, float init, float *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_min_f64(const double *d_in, uint64_t n, double init, double *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_max_i32(const int32_t *d_in, uint64_t n, int32_t init, int32_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_max_u32(const uint32_t *d_in, uint64_t n, uint32_t init, uint32_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_max_i64(const int64_t *d_in, uint64_t n, int64_t init, int64_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_max_u64(const uint64_t *d_in, uint64_t n, uint64_t init, uint64_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_max_f32(const float *d_in, uint64_t n, float init, float *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_max_f64(const double *d_in, uint64_t n, double init, double *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);

/* The same with init read from device memory when the scan runs: *d_init
 * (non-null, aligned) replaces init, so a scan can continue from a value that
 * is still on the device -- e.g. the last output of the previous chunk of a
 * stream (d_init = d_out_prev + n_prev - 1), with no copy to the host between
 * the chunks.  The reference's scan takes init by value (scan.cu:87). */
BK_API int bk_inclusive_scan_sum_i32_dinit(const int32_t *d_in, uint64_t n, const int32_t *d_init, int32_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_sum_u32_dinit(const uint32_t *d_in, uint64_t n, const uint32_t *d_init, uint32_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_sum_i64_dinit(const int64_t *d_in, uint64_t n, const int64_t *d_init, int64_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_sum_u64_dinit(const uint64_t *d_in, uint64_t n, const uint64_t *d_init, uint64_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_sum_f32_dinit(const float *d_in, uint64_t n, const float *d_init, float *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_sum_f64_dinit(const double *d_in, uint64_t n, const double *d_init, double *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_min_i32_dinit(const int32_t *d_in, uint64_t n, const int32_t *d_init, int32_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_min_u32_dinit(const uint32_t *d_in, uint64_t n, const uint32_t *d_init, uint32_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_min_i64_dinit(const int64_t *d_in, uint64_t n, const int64_t *d_init, int64_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_min_u64_dinit(const uint64_t *d_in, uint64_t n, const uint64_t *d_init, uint64_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_min_f32_dinit(const float *d_in, uint64_t n, const float *d_init, float *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_min_f64_dinit(const double *d_in, uint64_t n, const double *d_init, double *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_max_i32_dinit(const int32_t *d_in, uint64_t n, const int32_t *d_init, int32_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_max_u32_dinit(const uint32_t *d_in, uint64_t n, const uint32_t *d_init, uint32_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_max_i64_dinit(const int64_t *d_in, uint64_t n, const int64_t *d_init, int64_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_max_u64_dinit(const uint64_t *d_in, uint64_t n, const uint64_t *d_init, uint64_t *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_max_f32_dinit(const float *d_in, uint64_t n, const float *d_init, float *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_max_f64_dinit(const double *d_in, uint64_t n, const double *d_init, double *d_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);


/* ---- merge ----------------------------------------------------------------
 * Stable merge of two sorted ranges under operator<: equal keys keep A before
 * B and each input's own order (merge_path, bulk/algorithm/merge.hpp:35-60,
 * and the serial merge, merge.hpp:63-170).  out has na + nb elements.
 * bk_merge_* replaces my_merge(first1, last1, first2, last2, result, comp),
 * merge.cu:127-162 (keys only); bk_merge_by_key_* adds a 4- or 8-byte payload
 * moved with each key, as the bounded group merge_by_key does,
 * bulk/algorithm/merge.hpp:507-607.  Keys must not be NaN. */
BK_API int bk_merge_i32(const int32_t *a, uint64_t na, const int32_t *b, uint64_t nb, int32_t *out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_merge_u32(const uint32_t *a, uint64_t na, const uint32_t *b, uint64_t nb, uint32_t *out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_merge_i64(const int64_t *a, uint64_t na, const int64_t *b, uint64_t nb, int64_t *out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_merge_u64(const uint64_t *a, uint64_t na, const uint64_t *b, uint64_t nb, uint64_t *out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_merge_f32(const float *a, uint64_t na, const float *b, uint64_t nb, float *out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_merge_f64(const double *a, uint64_t na, const double *b, uint64_t nb, double *out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_merge_by_key_i32_u32(const int32_t *a_keys, const uint32_t *a_vals, uint64_t na, const int32_t *b_keys, const uint32_t *b_vals, uint64_t nb, int32_t *out_keys, uint32_t *out_vals, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_merge_by_key_i32_u64(const int32_t *a_keys, const uint64_t *a_vals, uint64_t na, const int32_t *b_keys, const uint64_t *b_vals, uint64_t nb, int32_t *out_keys, uint64_t *out_vals, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_merge_by_key_u32_u32(const uint32_t *a_keys, const uint32_t *a_vals, uint64_t na, const uint32_t *b_keys, const uint32_t *b_vals, uint64_t nb, uint32_t *out_keys, uint32_t *out_vals, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_merge_by_key_u32_u64(const uint32_t *a_keys, const uint64_t *a_vals, uint64_t na, const uint32_t *b_keys, const uint64_t *b_vals, uint64_t nb, uint32_t *out_keys, uint64_t *out_vals, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_merge_by_key_i64_u32(const int64_t *a_keys, const uint32_t *a_vals, uint64_t na, const int64_t *b_keys, const uint32_t *b_vals, uint64_t nb, int64_t *out_keys, uint32_t *out_vals, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_merge_by_key_i64_u64(const int64_t *a_keys, const uint64_t *a_vals, uint64_t na, const int64_t *b_keys, const uint64_t *b_vals, uint64_t nb, int64_t *out_keys, uint64_t *out_vals, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_merge_by_key_u64_u32(const uint64_t *a_keys, const uint32_t *a_vals, uint64_t na, const uint64_t *b_keys, const uint32_t *b_vals, uint64_t nb, uint64_t *out_keys, uint32_t *out_vals, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_merge_by_key_u64_u64(const uint64_t *a_keys, const uint64_t *a_vals, uint64_t na, const uint64_t *b_keys, const uint64_t *b_vals, uint64_t nb, uint64_t *out_keys, uint64_t *out_vals, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_merge_by_key_f32_u32(const float *a_keys, const uint32_t *a_vals, uint64_t na, const float *b_keys, const uint32_t *b_vals, uint64_t nb, float *out_keys, uint32_t *out_vals, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_merge_by_key_f32_u64(const float *a_keys, const uint64_t *a_vals, uint64_t na, const float *b_keys, const uint64_t *b_vals, uint64_t nb, float *out_keys, uint64_t *out_vals, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_merge_by_key_f64_u32(const double *a_keys, const uint32_t *a_vals, uint64_t na, const double *b_keys, const uint32_t *b_vals, uint64_t nb, double *out_keys, uint32_t *out_vals, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_merge_by_key_f64_u64(const double *a_keys, const uint64_t *a_vals, uint64_t na, const double *b_keys, const uint64_t *b_vals, uint64_t nb, double *out_keys, uint64_t *out_vals, void *d_ws, size_t ws_bytes, bk_stream_t stream);

/* ---- stable sort by key -----------------------------------------------------
 * In-place stable sort of keys[0..n) under operator<, moving vals with their
 * keys; equal keys keep their input order (-0.0 and +0.0 are equal).
 * Replaces stable_merge_sort_by_key(keys_first, keys_last, values_first,
 * comp), merge_sort_by_key.cu:150-209 (block sort bulk/algorithm/sort.hpp:
 * 152-166, stable_merge_sort.hpp:125-206, then merge-path passes).  The
 * stable order is unique, so the result is the reference's whichever way it
 * is computed: one block sort for an array of one tile (8192 4-byte / 4096
 * 8-byte keys), a stable LSD radix sort below 2^30 elements (up to 131,072
 * keys as one launch of one thread-block cluster, above that as passes of
 * three launches each), block sort and merge-path passes from 2^30 on.  Keys
 * must not be NaN.  bk_sort_keys_* sorts keys alone. */
BK_API int bk_sort_keys_i32(int32_t *keys, uint64_t n, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_keys_u32(uint32_t *keys, uint64_t n, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_keys_i64(int64_t *keys, uint64_t n, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_keys_u64(uint64_t *keys, uint64_t n, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_keys_f32(float *keys, uint64_t n, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_keys_f64(double *keys, uint64_t n, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_i32_u32(int32_t *keys, uint32_t *vals, uint64_t n, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_i32_u64(int32_t *keys, uint64_t *vals, uint64_t n, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_u32_u32(uint32_t *keys, uint32_t *vals, uint64_t n, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_u32_u64(uint32_t *keys, uint64_t *vals, uint64_t n, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_i64_u32(int64_t *keys, uint32_t *vals, uint64_t n, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_i64_u64(int64_t *keys, uint64_t *vals, uint64_t n, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_u64_u32(uint64_t *keys, uint32_t *vals, uint64_t n, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_u64_u64(uint64_t *keys, uint64_t *vals, uint64_t n, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_f32_u32(float *keys, uint32_t *vals, uint64_t n, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_f32_u64(float *keys, uint64_t *vals, uint64_t n, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_f64_u32(double *keys, uint32_t *vals, uint64_t n, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_f64_u64(double *keys, uint64_t *vals, uint64_t n, void *d_ws, size_t ws_bytes, bk_stream_t stream);


/* ---- reduce_by_key (pred = equal_to, op = plus) -----------------------------
 * One output pair per maximal run of equal consecutive keys, in run order:
 * out_keys[r] = the run's key, out_vals[r] = the sum of its values, and
 * *d_num_out = the number of runs (written on the device; n == 0 writes 0).
 * out_keys / out_vals need room for n elements in the worst case.  Integer
 * sums wrap.  n < 2^32.  Replaces my_reduce_by_key(keys_first, keys_last,
 * values_first, keys_result, values_result, pred, binary_op),
 * reduce_by_key.cu:176-272 (bulk::reduce_by_key,
 * bulk/algorithm/reduce_by_key.hpp:115-216), whose result size the reference
 * returns through a synchronous device-to-host copy (:269). */
BK_API int bk_reduce_by_key_i32_i32(const int32_t *keys, const int32_t *vals, uint64_t n, int32_t *out_keys, int32_t *out_vals, uint64_t *d_num_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_by_key_i32_i64(const int32_t *keys, const int64_t *vals, uint64_t n, int32_t *out_keys, int64_t *out_vals, uint64_t *d_num_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_by_key_i32_f32(const int32_t *keys, const float *vals, uint64_t n, int32_t *out_keys, float *out_vals, uint64_t *d_num_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_by_key_i32_f64(const int32_t *keys, const double *vals, uint64_t n, int32_t *out_keys, double *out_vals, uint64_t *d_num_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_by_key_u32_f32(const uint32_t *keys, const float *vals, uint64_t n, uint32_t *out_keys, float *out_vals, uint64_t *d_num_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_by_key_u32_f64(const uint32_t *keys, const double *vals, uint64_t n, uint32_t *out_keys, double *out_vals, uint64_t *d_num_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_by_key_i64_i32(const int64_t *keys, const int32_t *vals, uint64_t n, int64_t *out_keys, int32_t *out_vals, uint64_t *d_num_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_by_key_i64_i64(const int64_t *keys, const int64_t *vals, uint64_t n, int64_t *out_keys, int64_t *out_vals, uint64_t *d_num_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_by_key_i64_f32(const int64_t *keys, const float *vals, uint64_t n, int64_t *out_keys, float *out_vals, uint64_t *d_num_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_by_key_i64_f64(const int64_t *keys, const double *vals, uint64_t n, int64_t *out_keys, double *out_vals, uint64_t *d_num_out, void *d_ws, size_t ws_bytes, bk_stream_t stream);

/* Allocation-free variant of bk_inclusive_scan_sum_f32 (no counterpart in the
 * reference).  For callers that cannot allocate device memory: the scan's
 * scratch lives in a fixed 1 MiB + 256-byte array inside the library's own
 * device memory, held by every GPU that loads the library until exit.
 * n is limited to 2^30 elements (BK_ERR_TOO_LARGE beyond).  The first call on
 * a device looks up the array's device address; make that call before any
 * stream capture.  All calls share the one array: calls that overlap on the
 * GPU (concurrent streams, other threads) race and corrupt each other, so
 * serialise them.  Device-side wait errors are not reported by this variant. */
BK_API int bk_inclusive_scan_sum_f32_noalloc(const float *d_in, uint64_t n, float init, float *d_out, bk_stream_t stream);

/* ---- batched entry points --------------------------------------------------
 * No counterpart in the reference, whose drivers launch once per array.  One
 * call processes up to BK_BATCH_MAX independent arrays with a single
 * persistent launch (plus one small initialisation kernel): every array's
 * result is exactly what the single-array entry point gives for it, and the
 * GPU stays full even when each array is small.  `items` is in host memory;
 * items with n == 0 are skipped.  Workspace: bk_batch_workspace_bytes over
 * the items' sizes, same contract as above. */
#define BK_BATCH_MAX 256

typedef struct bk_scan_item_i32 { const int32_t *d_in; int32_t *d_out; uint64_t n; int32_t init; } bk_scan_item_i32;
typedef struct bk_scan_item_u32 { const uint32_t *d_in; uint32_t *d_out; uint64_t n; uint32_t init; } bk_scan_item_u32;
typedef struct bk_scan_item_i64 { const int64_t *d_in; int64_t *d_out; uint64_t n; int64_t init; } bk_scan_item_i64;
typedef struct bk_scan_item_u64 { const uint64_t *d_in; uint64_t *d_out; uint64_t n; uint64_t init; } bk_scan_item_u64;
typedef struct bk_scan_item_f32 { const float *d_in; float *d_out; uint64_t n; float init; } bk_scan_item_f32;
typedef struct bk_scan_item_f64 { const double *d_in; double *d_out; uint64_t n; double init; } bk_scan_item_f64;

/* Inclusive sum scans of up to BK_BATCH_MAX arrays: for each item,
 * d_out[i] = init + d_in[0] + ... + d_in[i] (as bk_inclusive_scan_sum_*). */
BK_API int bk_inclusive_scan_sum_i32_batch(const bk_scan_item_i32 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_sum_u32_batch(const bk_scan_item_u32 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_sum_i64_batch(const bk_scan_item_i64 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_sum_u64_batch(const bk_scan_item_u64 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_sum_f32_batch(const bk_scan_item_f32 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_inclusive_scan_sum_f64_batch(const bk_scan_item_f64 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);

/* reduce_by_key of up to BK_BATCH_MAX arrays: for each item, the runs of
 * its keys go to its out_keys / out_vals and their count to its d_num_out
 * (as bk_reduce_by_key_*). */
typedef struct bk_rbk_item_i32_i32 { const int32_t *keys; const int32_t *vals; uint64_t n; int32_t *out_keys; int32_t *out_vals; uint64_t *d_num_out; } bk_rbk_item_i32_i32;
typedef struct bk_rbk_item_i32_i64 { const int32_t *keys; const int64_t *vals; uint64_t n; int32_t *out_keys; int64_t *out_vals; uint64_t *d_num_out; } bk_rbk_item_i32_i64;
typedef struct bk_rbk_item_i32_f32 { const int32_t *keys; const float *vals; uint64_t n; int32_t *out_keys; float *out_vals; uint64_t *d_num_out; } bk_rbk_item_i32_f32;
typedef struct bk_rbk_item_i32_f64 { const int32_t *keys; const double *vals; uint64_t n; int32_t *out_keys; double *out_vals; uint64_t *d_num_out; } bk_rbk_item_i32_f64;
typedef struct bk_rbk_item_u32_f32 { const uint32_t *keys; const float *vals; uint64_t n; uint32_t *out_keys; float *out_vals; uint64_t *d_num_out; } bk_rbk_item_u32_f32;
typedef struct bk_rbk_item_u32_f64 { const uint32_t *keys; const double *vals; uint64_t n; uint32_t *out_keys; double *out_vals; uint64_t *d_num_out; } bk_rbk_item_u32_f64;
typedef struct bk_rbk_item_i64_i32 { const int64_t *keys; const int32_t *vals; uint64_t n; int64_t *out_keys; int32_t *out_vals; uint64_t *d_num_out; } bk_rbk_item_i64_i32;
typedef struct bk_rbk_item_i64_i64 { const int64_t *keys; const int64_t *vals; uint64_t n; int64_t *out_keys; int64_t *out_vals; uint64_t *d_num_out; } bk_rbk_item_i64_i64;
typedef struct bk_rbk_item_i64_f32 { const int64_t *keys; const float *vals; uint64_t n; int64_t *out_keys; float *out_vals; uint64_t *d_num_out; } bk_rbk_item_i64_f32;
typedef struct bk_rbk_item_i64_f64 { const int64_t *keys; const double *vals; uint64_t n; int64_t *out_keys; double *out_vals; uint64_t *d_num_out; } bk_rbk_item_i64_f64;
BK_API int bk_reduce_by_key_i32_i32_batch(const bk_rbk_item_i32_i32 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_by_key_i32_i64_batch(const bk_rbk_item_i32_i64 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_by_key_i32_f32_batch(const bk_rbk_item_i32_f32 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_by_key_i32_f64_batch(const bk_rbk_item_i32_f64 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_by_key_u32_f32_batch(const bk_rbk_item_u32_f32 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_by_key_u32_f64_batch(const bk_rbk_item_u32_f64 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_by_key_i64_i32_batch(const bk_rbk_item_i64_i32 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_by_key_i64_i64_batch(const bk_rbk_item_i64_i64 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_by_key_i64_f32_batch(const bk_rbk_item_i64_f32 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_reduce_by_key_i64_f64_batch(const bk_rbk_item_i64_f64 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);

/* Stable sort_by_key of up to BK_BATCH_MAX arrays, each in place (as
 * bk_sort_by_key_*): one block-sort launch for all arrays, then per merge
 * pass one launch for all arrays that still need it. */
typedef struct bk_sort_item_i32_u32 { int32_t *keys; uint32_t *vals; uint64_t n; } bk_sort_item_i32_u32;
typedef struct bk_sort_item_i32_u64 { int32_t *keys; uint64_t *vals; uint64_t n; } bk_sort_item_i32_u64;
typedef struct bk_sort_item_u32_u32 { uint32_t *keys; uint32_t *vals; uint64_t n; } bk_sort_item_u32_u32;
typedef struct bk_sort_item_u32_u64 { uint32_t *keys; uint64_t *vals; uint64_t n; } bk_sort_item_u32_u64;
typedef struct bk_sort_item_i64_u32 { int64_t *keys; uint32_t *vals; uint64_t n; } bk_sort_item_i64_u32;
typedef struct bk_sort_item_i64_u64 { int64_t *keys; uint64_t *vals; uint64_t n; } bk_sort_item_i64_u64;
typedef struct bk_sort_item_u64_u32 { uint64_t *keys; uint32_t *vals; uint64_t n; } bk_sort_item_u64_u32;
typedef struct bk_sort_item_u64_u64 { uint64_t *keys; uint64_t *vals; uint64_t n; } bk_sort_item_u64_u64;
typedef struct bk_sort_item_f32_u32 { float *keys; uint32_t *vals; uint64_t n; } bk_sort_item_f32_u32;
typedef struct bk_sort_item_f32_u64 { float *keys; uint64_t *vals; uint64_t n; } bk_sort_item_f32_u64;
typedef struct bk_sort_item_f64_u32 { double *keys; uint32_t *vals; uint64_t n; } bk_sort_item_f64_u32;
typedef struct bk_sort_item_f64_u64 { double *keys; uint64_t *vals; uint64_t n; } bk_sort_item_f64_u64;
BK_API int bk_sort_by_key_i32_u32_batch(const bk_sort_item_i32_u32 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_i32_u64_batch(const bk_sort_item_i32_u64 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_u32_u32_batch(const bk_sort_item_u32_u32 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_u32_u64_batch(const bk_sort_item_u32_u64 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_i64_u32_batch(const bk_sort_item_i64_u32 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_i64_u64_batch(const bk_sort_item_i64_u64 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_u64_u32_batch(const bk_sort_item_u64_u32 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_u64_u64_batch(const bk_sort_item_u64_u64 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_f32_u32_batch(const bk_sort_item_f32_u32 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_f32_u64_batch(const bk_sort_item_f32_u64 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_f64_u32_batch(const bk_sort_item_f64_u32 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_f64_u64_batch(const bk_sort_item_f64_u64 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
/* Out-of-place form of the batched sort: for each item, in_keys / in_vals
 * (left unchanged) are stably sorted into keys / vals (n elements each; the
 * ranges must not overlap).  The first pass reads the sources directly, so a
 * caller that would copy each input window before an in-place sort saves
 * that copy.  Workspace as for the in-place batch.  No counterpart in the
 * reference (its sort is in place, merge_sort_by_key.cu:150-209). */
typedef struct bk_sort_copy_item_i32_u32 { const int32_t *in_keys; const uint32_t *in_vals; int32_t *keys; uint32_t *vals; uint64_t n; } bk_sort_copy_item_i32_u32;
typedef struct bk_sort_copy_item_i32_u64 { const int32_t *in_keys; const uint64_t *in_vals; int32_t *keys; uint64_t *vals; uint64_t n; } bk_sort_copy_item_i32_u64;
typedef struct bk_sort_copy_item_u32_u32 { const uint32_t *in_keys; const uint32_t *in_vals; uint32_t *keys; uint32_t *vals; uint64_t n; } bk_sort_copy_item_u32_u32;
typedef struct bk_sort_copy_item_u32_u64 { const uint32_t *in_keys; const uint64_t *in_vals; uint32_t *keys; uint64_t *vals; uint64_t n; } bk_sort_copy_item_u32_u64;
typedef struct bk_sort_copy_item_i64_u32 { const int64_t *in_keys; const uint32_t *in_vals; int64_t *keys; uint32_t *vals; uint64_t n; } bk_sort_copy_item_i64_u32;
typedef struct bk_sort_copy_item_i64_u64 { const int64_t *in_keys; const uint64_t *in_vals; int64_t *keys; uint64_t *vals; uint64_t n; } bk_sort_copy_item_i64_u64;
typedef struct bk_sort_copy_item_u64_u32 { const uint64_t *in_keys; const uint32_t *in_vals; uint64_t *keys; uint32_t *vals; uint64_t n; } bk_sort_copy_item_u64_u32;
typedef struct bk_sort_copy_item_u64_u64 { const uint64_t *in_keys; const uint64_t *in_vals; uint64_t *keys; uint64_t *vals; uint64_t n; } bk_sort_copy_item_u64_u64;
typedef struct bk_sort_copy_item_f32_u32 { const float *in_keys; const uint32_t *in_vals; float *keys; uint32_t *vals; uint64_t n; } bk_sort_copy_item_f32_u32;
typedef struct bk_sort_copy_item_f32_u64 { const float *in_keys; const uint64_t *in_vals; float *keys; uint64_t *vals; uint64_t n; } bk_sort_copy_item_f32_u64;
typedef struct bk_sort_copy_item_f64_u32 { const double *in_keys; const uint32_t *in_vals; double *keys; uint32_t *vals; uint64_t n; } bk_sort_copy_item_f64_u32;
typedef struct bk_sort_copy_item_f64_u64 { const double *in_keys; const uint64_t *in_vals; double *keys; uint64_t *vals; uint64_t n; } bk_sort_copy_item_f64_u64;
BK_API int bk_sort_by_key_i32_u32_copy_batch(const bk_sort_copy_item_i32_u32 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_i32_u64_copy_batch(const bk_sort_copy_item_i32_u64 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_u32_u32_copy_batch(const bk_sort_copy_item_u32_u32 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_u32_u64_copy_batch(const bk_sort_copy_item_u32_u64 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_i64_u32_copy_batch(const bk_sort_copy_item_i64_u32 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_i64_u64_copy_batch(const bk_sort_copy_item_i64_u64 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_u64_u32_copy_batch(const bk_sort_copy_item_u64_u32 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_u64_u64_copy_batch(const bk_sort_copy_item_u64_u64 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_f32_u32_copy_batch(const bk_sort_copy_item_f32_u32 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_f32_u64_copy_batch(const bk_sort_copy_item_f32_u64 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_f64_u32_copy_batch(const bk_sort_copy_item_f64_u32 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);
BK_API int bk_sort_by_key_f64_u64_copy_batch(const bk_sort_copy_item_f64_u64 *items, uint32_t count, void *d_ws, size_t ws_bytes, bk_stream_t stream);

/* ---- serving loop -----------------------------------------------------------
 * No counterpart in the reference, whose drivers run one array at a time.
 * bk_serve_run answers a stream of mixed requests on the caller's stream,
 * either one library call per request (BK_SERVE_PLAIN: the single-array entry
 * points above, sort inputs copied with cudaMemcpyAsync) or by continuous
 * batching (BK_SERVE_BATCHED: every admitted request that has arrived is
 * issued at once as one round -- per kind one *_batch call, sorts out of
 * place from the requests' source windows, the kinds on streams of their
 * own forked from the caller's stream and joined back to it; a kind with one
 * request, and a round of at most four requests, go out as plain calls (a
 * sort of 2^20 elements or more as a one-item out-of-place batch); at most
 * max_inflight rounds of more than four requests are queued at once).
 * A request reads
 * a window of the caller's source arrays; its own buffers (sort: keys and
 * payload, sorted in place; rbk: out_keys, out_vals, count; scan: output)
 * come from a first-fit pool over the caller's device buffer, and requests
 * are admitted in arrival order while the bytes of admitted, unfinished
 * requests (bk_serve_request_bytes each) stay within budget_bytes; a request
 * larger than the budget runs alone.  Start and done times are the host's
 * steady clock, in seconds from the start of the run; a request is done when
 * the host sees the event recorded after its call.  Blocks until every
 * request is done (or timeout_s passes: BK_ERR_SPIN_TIMEOUT).  The workspace
 * must hold bk_serve_workspace_bytes(requests, mode) and be zeroed once. */
#define BK_SERVE_SORT 0 /* stable sort_by_key: u32 keys, u32 payload */
#define BK_SERVE_RBK 1  /* reduce_by_key (equal_to, plus): i32 keys, f32 values */
#define BK_SERVE_SCAN 2 /* inclusive sum scan: f32, init 0 */
#define BK_SERVE_PLAIN 0
#define BK_SERVE_BATCHED 1

typedef struct bk_serve_request {
  uint32_t kind;       /* BK_SERVE_SORT / _RBK / _SCAN */
  uint32_t reserved;
  uint64_t n;          /* elements (> 0) */
  uint64_t src_offset; /* first element of the input window; a multiple of 4 */
  double arrival_s;    /* seconds after the start of the run; nondecreasing */
} bk_serve_request;

typedef struct bk_serve_record {
  double start_s;  /* issued */
  double done_s;   /* completion seen by the host */
  uint64_t out[3]; /* byte offsets in the pool of the request's buffers, in the order above */
} bk_serve_record;

typedef struct bk_serve_config {
  const uint32_t *sort_keys; /* sources, source_len elements each */
  const uint32_t *sort_vals;
  const int32_t *rbk_keys;
  const float *rbk_vals;
  const float *scan_vals;
  uint64_t source_len;
  void *pool;                /* device buffer for the requests' buffers (256-byte aligned) */
  uint64_t pool_bytes;
  void *ws;                  /* workspace */
  uint64_t ws_bytes;
  uint64_t budget_bytes;
  bk_stream_t stream;
  int32_t mode;              /* BK_SERVE_PLAIN / BK_SERVE_BATCHED */
  int32_t max_inflight;      /* batched: rounds of more than four requests queued at once (>= 1) */
  int32_t keep_buffers;      /* 1: buffers are not reused, so every result stays readable */
  int32_t reserved;
  double timeout_s;
} bk_serve_config;

typedef struct bk_serve_stats {
  double makespan_s;
  uint64_t pool_high_water; /* bytes */
  uint64_t calls;           /* library calls issued */
  uint64_t batches;         /* of which batched calls */
} bk_serve_stats;

BK_API uint64_t bk_serve_request_bytes(uint32_t kind, uint64_t n);
BK_API size_t bk_serve_workspace_bytes(const bk_serve_request *requests, uint32_t count, int mode);
BK_API int bk_serve_run(const bk_serve_config *cfg, const bk_serve_request *requests, uint32_t count, bk_serve_record *records, bk_serve_stats *stats);

/* The serving loop's pooled allocator on its own (host memory only: it hands
 * out byte offsets into a buffer of `capacity` bytes).  256-byte granules,
 * first fit over an address-ordered free list, neighbours coalesced on free.
 * bk_pool_alloc returns BK_ERR_TOO_LARGE when no free block fits. */
BK_API void *bk_pool_create(uint64_t capacity);
BK_API void bk_pool_destroy(void *pool);
BK_API int bk_pool_alloc(void *pool, uint64_t bytes, uint64_t *offset);
BK_API int bk_pool_free(void *pool, uint64_t offset);
BK_API uint64_t bk_pool_in_use(const void *pool);
BK_API uint64_t bk_pool_high_water(const void *pool);
BK_API uint32_t bk_pool_free_blocks(const void *pool);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* BULK_B200_H */
