/* oracle.h -- TEST INFRASTRUCTURE ONLY: CPU restatement of the reference's
 * device-wide algorithms.  Declarations are generated per type by the macros
 * in oracle.c; see oracle.c for the reference citations. */
#ifndef BK_ORACLE_H
#define BK_ORACLE_H
#include <stdint.h>

uint64_t bko_mix64(uint64_t seed, uint64_t i);
void bko_gen_i32(int32_t *out, uint64_t n, uint64_t seed, int32_t lo, int32_t hi);
void bko_gen_u32(uint32_t *out, uint64_t n, uint64_t seed);
void bko_gen_u64(uint64_t *out, uint64_t n, uint64_t seed);
void bko_gen_f32(float *out, uint64_t n, uint64_t seed, float lo, float hi);
void bko_gen_f64(double *out, uint64_t n, uint64_t seed, double lo, double hi);
int64_t bko_ref_hash(int64_t x);
void bko_ref_hash_fill_i32(int32_t *out, uint64_t n, int32_t modulus);
uint64_t bko_gen_runs_geometric(int32_t *keys, uint64_t n, uint64_t seed, double mean);
uint64_t bko_gen_runs_zipf(int32_t *keys, uint64_t n, uint64_t seed, double s, uint64_t cap);

#endif
