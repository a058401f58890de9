/* CPU oracle for the big-integer multiply path (test infrastructure only).
 * See bigint_oracle.c for the reference citations. */
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_ERR_INVALID -1
#define ORC_ERR_NOMEM -2
#define ORC_ERR_CAPACITY -3     /* transform length beyond 2^26 points */
#define ORC_ERR_CAPACITY_OUT -4 /* caller buffer too small; *out_len = need */

int orc_ntt_mul(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out,
                size_t cap, size_t* out_len);
int orc_brute_mul(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out,
                  size_t cap, size_t* out_len);
int orc_mul(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out, size_t cap,
            size_t* out_len);
int orc_mul_digits(const uint32_t* a, size_t na, const uint32_t* b, size_t nb, int same,
                   size_t output_precision, int64_t* point_pos, uint32_t* out, size_t cap,
                   size_t* out_len);
uint64_t orc_mod_m61(const uint64_t* x, size_t n);
int orc_product_tree(const uint64_t* leaves, size_t n, uint64_t* out, size_t cap,
                     size_t* out_len);

#ifdef __cplusplus
}
#endif
