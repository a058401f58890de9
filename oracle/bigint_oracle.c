/* CPU oracle: a plain-C restatement of the reference multiply path of
 * Looading99/BigInt.  TEST INFRASTRUCTURE ONLY: it is the checker that the
 * parity tests, __graft_entry__.smoke() and the bench's CPU-baseline leg call;
 * the product (bigint_b200) never links, loads or calls it.
 *
 * Pinned: tests/test_oracle.py checks every function here against the
 * committed golden vectors in tests/golden/ (generated by running the
 * unmodified reference through oracle/_ref) and, when oracle/_ref is built,
 * directly against the reference on seeded inputs.
 *
 * Citations are paths inside the reference project.
 *   orc_ntt_mul      src/mul/ntt_multithread.cpp:444-530  (three-prime NTT)
 *   orc_brute_mul    include/bigint/mul.h:82-102          (schoolbook)
 *   orc_mul          include/bigint/mul.h:208-220         (dispatcher; every
 *                    branch returns the same exact integer product, so the
 *                    oracle routes small sizes to brute and the rest to NTT)
 *   orc_mul_digits   include/bigint/mul.h:223-318         (Digits boundary)
 *   orc_mod_m61      residue mod 2^61-1 (property check for the largest sizes)
 *   orc_product_tree examples/pi.cpp:41-80 merge pattern, pairwise levels
 */
#include "bigint_oracle.h"

#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* ---- constants: include/bigint/ntt_base.h:14-27 ---------------------- */
static const uint32_t P[3] = {469762049u, 2013265921u, 2281701377u};
static const uint32_t G[3] = {3u, 31u, 3u};
#define DIGIT_BITS 28u
#define DIGIT_MASK ((1u << DIGIT_BITS) - 1u)
#define MAX_LEN_EXP 26u /* min over P of countr_zero(P-1) */

static uint32_t pow_mod(uint32_t b, uint64_t e, uint32_t p) {
    uint64_t r = 1, x = b % p;
    while (e) {
        if (e & 1) r = r * x % p;
        x = x * x % p;
        e >>= 1;
    }
    return (uint32_t)r;
}

/* Montgomery with R = 2^32, values in [0,p): ntt_base.h:40-71. */
typedef struct {
    uint32_t p, neg_inv, r_sq;
} mont_t;

static mont_t mont_make(uint32_t p) {
    mont_t m;
    uint32_t inv = 1; /* p^-1 mod 2^32 by Newton iteration */
    for (int i = 0; i < 5; ++i) inv *= 2u - p * inv;
    m.p = p;
    m.neg_inv = (uint32_t)(0u - inv);
    uint64_t r_mod = ((uint64_t)1 << 32) % p;
    m.r_sq = (uint32_t)(r_mod * r_mod % p);
    return m;
}

static inline uint32_t mont_mul(const mont_t* m, uint32_t a, uint32_t b) {
    uint64_t t = (uint64_t)a * b;
    uint32_t u = (uint32_t)t * m->neg_inv;
    uint64_t t2 = t + (uint64_t)u * m->p;
    uint32_t r = (uint32_t)(t2 >> 32);
    return r < m->p ? r : r - m->p;
}

static inline uint32_t add_mod(uint32_t a, uint32_t b, uint32_t p) {
    uint32_t d = p - b; /* bigint_base.h:93-99 */
    return a < d ? a + b : a - d;
}

static inline uint32_t sub_mod(uint32_t a, uint32_t b, uint32_t p) {
    uint32_t t = a - b; /* bigint_base.h:102-108 */
    return t + ((0u - (uint32_t)(t > a)) & p);
}

static uint32_t to_mont(const mont_t* m, uint32_t x) { return mont_mul(m, x, m->r_sq); }

/* Bit reversal (ntt_base.h:268-287, applied per prime plane here). */
static void bit_reverse(uint32_t* v, size_t n) {
    for (size_t i = 1, j = n >> 1; i + 1 < n; ++i) {
        if (i < j) {
            uint32_t t = v[i];
            v[i] = v[j];
            v[j] = t;
        }
        size_t k = n >> 1;
        while (j >= k) {
            j -= k;
            k >>= 1;
        }
        j += k;
    }
}

/* imm_ntt (ntt_multithread.cpp:333-379): bit reversal, then radix-2 DIT
 * stages len = 2..n with the level root steps[rev][log2(len)-1]
 * (ntt_base.h:195-208), running twiddle cur *= step; the inverse multiplies
 * by inv_pow_of_two (ntt_base.h:210-222).  All values in Montgomery form. */
static void ntt_plane(uint32_t* v, size_t n, int rev, const mont_t* m, uint32_t g) {
    if (n == 1) return;
    bit_reverse(v, n);
    uint32_t g_use = rev ? pow_mod(g, m->p - 2, m->p) : g;
    uint32_t one = to_mont(m, 1);
    for (size_t len = 2; len <= n; len <<= 1) {
        size_t half = len >> 1;
        uint32_t step = to_mont(m, pow_mod(g_use, (m->p - 1) / len, m->p));
        for (size_t i = 0; i < n; i += len) {
            uint32_t cur = one;
            for (size_t j = 0; j < half; ++j) {
                uint32_t a = v[i + j];
                uint32_t b = mont_mul(m, cur, v[i + j + half]);
                v[i + j] = add_mod(a, b, m->p);
                v[i + j + half] = sub_mod(a, b, m->p);
                cur = mont_mul(m, cur, step);
            }
        }
    }
    if (rev) {
        uint32_t inv_n = pow_mod((uint32_t)(n % m->p), m->p - 2, m->p);
        uint32_t c = to_mont(m, inv_n);
        for (size_t i = 0; i < n; ++i) v[i] = mont_mul(m, v[i], c);
    }
}

/* garner_merge (ntt_base.h:228-246). */
static u128 garner(uint32_t c0, uint32_t c1, uint32_t c2) {
    const uint32_t i01 = pow_mod(P[0] % P[1], P[1] - 2, P[1]);
    const uint32_t i02 = pow_mod(P[0] % P[2], P[2] - 2, P[2]);
    const uint32_t i12 = pow_mod(P[1] % P[2], P[2] - 2, P[2]);
    uint32_t v0 = c0;
    uint32_t v1 = (uint32_t)((uint64_t)sub_mod(c1, v0 % P[1], P[1]) * i01 % P[1]);
    uint32_t v2 = (uint32_t)((uint64_t)sub_mod(c2, v0, P[2]) * i02 % P[2]);
    v2 = (uint32_t)((uint64_t)sub_mod(v2, v1, P[2]) * i12 % P[2]);
    u128 x = (u128)((uint64_t)P[0] * P[1]) * v2;
    x += (uint64_t)P[0] * v1;
    x += v0;
    return x;
}

static size_t bit_ceil(size_t x) {
    size_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

static size_t strip64(const uint64_t* x, size_t n) {
    while (n > 0 && x[n - 1] == 0) --n;
    return n;
}

/* vec64_to_vec32_and_repeat with k=1 (ntt_multithread.cpp:447-475): 28-bit
 * digits of a limb array, zero-padded to `len`. */
static void limbs_to_digits28(const uint64_t* x, size_t n, uint32_t* d, size_t len) {
    memset(d, 0, len * sizeof(uint32_t));
    size_t total_bits = n * 64, k = 0;
    for (size_t bit = 0; bit < total_bits && k < len; bit += DIGIT_BITS, ++k) {
        size_t w = bit >> 6, s = bit & 63;
        uint64_t v = x[w] >> s;
        if (s > 64 - DIGIT_BITS && w + 1 < n) v |= x[w + 1] << (64 - s);
        d[k] = (uint32_t)v & DIGIT_MASK;
    }
}

int orc_ntt_mul(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out,
                size_t cap, size_t* out_len) {
    na = strip64(a, na);
    nb = strip64(b, nb);
    if (na == 0 || nb == 0) {
        *out_len = 0;
        return 0;
    }
    /* ntt_multithread.cpp:477-479 */
    size_t da = (na * 64 + DIGIT_BITS - 1) / DIGIT_BITS;
    size_t db = (nb * 64 + DIGIT_BITS - 1) / DIGIT_BITS;
    size_t n = bit_ceil(da + db - 1);
    if (n > ((size_t)1 << MAX_LEN_EXP)) return ORC_ERR_CAPACITY;
    int same = (a == b);
    uint32_t* dig_a = malloc(n * sizeof(uint32_t));
    uint32_t* dig_b = malloc(n * sizeof(uint32_t));
    uint32_t* planes = malloc(3 * n * sizeof(uint32_t));
    uint32_t* planes_b = same ? NULL : malloc(3 * n * sizeof(uint32_t));
    if (!dig_a || !dig_b || !planes || (!same && !planes_b)) {
        free(dig_a), free(dig_b), free(planes), free(planes_b);
        return ORC_ERR_NOMEM;
    }
    limbs_to_digits28(a, na, dig_a, n);
    if (!same) limbs_to_digits28(b, nb, dig_b, n);
    for (int q = 0; q < 3; ++q) {
        mont_t m = mont_make(P[q]);
        uint32_t* va = planes + (size_t)q * n;
        for (size_t i = 0; i < n; ++i) va[i] = to_mont(&m, dig_a[i]); /* :484 */
        ntt_plane(va, n, 0, &m, G[q]);                                 /* :485 */
        if (same) {
            for (size_t i = 0; i < n; ++i) va[i] = mont_mul(&m, va[i], va[i]); /* :488 */
        } else {
            uint32_t* vb = planes_b + (size_t)q * n;
            for (size_t i = 0; i < n; ++i) vb[i] = to_mont(&m, dig_b[i]);
            ntt_plane(vb, n, 0, &m, G[q]);
            for (size_t i = 0; i < n; ++i) va[i] = mont_mul(&m, va[i], vb[i]); /* :496 */
        }
        ntt_plane(va, n, 1, &m, G[q]);                                  /* :499 */
        for (size_t i = 0; i < n; ++i) va[i] = mont_mul(&m, va[i], 1); /* :500 */
    }
    /* crt_merge (:384-403) and trim (:418-442): point k carries
     * lo/mid/hi 28-bit pieces at digit positions k, k+1, k+2. */
    size_t nd = n + 3;
    uint32_t* digits = malloc(nd * sizeof(uint32_t));
    if (!digits) {
        free(dig_a), free(dig_b), free(planes), free(planes_b);
        return ORC_ERR_NOMEM;
    }
    uint32_t prev_mid = 0, prev_hi = 0, prev2_hi = 0, carry = 0;
    for (size_t k = 0; k < nd; ++k) {
        uint32_t lo = 0, mid = 0, hi = 0;
        if (k < n) {
            u128 x = garner(planes[k], planes[n + k], planes[2 * n + k]);
            lo = (uint32_t)x & DIGIT_MASK;
            mid = (uint32_t)(x >> DIGIT_BITS) & DIGIT_MASK;
            hi = (uint32_t)(x >> (2 * DIGIT_BITS)) & DIGIT_MASK;
        }
        uint32_t s = lo + prev_mid + prev2_hi + carry;
        digits[k] = s & DIGIT_MASK;
        carry = s >> DIGIT_BITS;
        prev2_hi = prev_hi;
        prev_hi = hi;
        prev_mid = mid;
    }
    /* repack 28 -> 64 (:504-527) and strip leading zeros */
    size_t nlimbs = (nd * DIGIT_BITS + 63) / 64;
    size_t need = 0;
    int rc = 0;
    uint64_t* tmp = calloc(nlimbs, sizeof(uint64_t));
    if (!tmp) {
        rc = ORC_ERR_NOMEM;
    } else {
        for (size_t k = 0; k < nd; ++k) {
            size_t bit = k * DIGIT_BITS, w = bit >> 6, s = bit & 63;
            tmp[w] |= (uint64_t)digits[k] << s;
            if (s > 64 - DIGIT_BITS && w + 1 < nlimbs) tmp[w + 1] |= (uint64_t)digits[k] >> (64 - s);
        }
        need = strip64(tmp, nlimbs);
        *out_len = need;
        if (need > cap) rc = ORC_ERR_CAPACITY_OUT;
        else memcpy(out, tmp, need * sizeof(uint64_t));
    }
    free(tmp), free(digits), free(dig_a), free(dig_b), free(planes), free(planes_b);
    return rc;
}

/* brute::mul (mul.h:82-102) */
int orc_brute_mul(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out,
                  size_t cap, size_t* out_len) {
    size_t n = na + nb;
    uint64_t* res = calloc(n ? n : 1, sizeof(uint64_t));
    if (!res) return ORC_ERR_NOMEM;
    for (size_t i = 0; i < na; ++i) {
        uint64_t carry = 0;
        size_t j = 0;
        for (; j < nb; ++j) {
            u128 t = (u128)a[i] * b[j] + res[i + j] + carry;
            res[i + j] = (uint64_t)t;
            carry = (uint64_t)(t >> 64);
        }
        for (; carry; ++j) {
            u128 t = (u128)res[i + j] + carry;
            res[i + j] = (uint64_t)t;
            carry = (uint64_t)(t >> 64);
        }
    }
    size_t need = strip64(res, n);
    *out_len = need;
    int rc = 0;
    if (need > cap) rc = ORC_ERR_CAPACITY_OUT;
    else if (need) memcpy(out, res, need * sizeof(uint64_t));
    free(res);
    return rc;
}

/* _mul (mul.h:208-220): brute up to 2*128*64 total bits, otherwise the exact
 * three-prime NTT (the reference's FFT branch returns the same product). */
int orc_mul(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out, size_t cap,
            size_t* out_len) {
    if ((na + nb) * 64 <= 2 * 128 * 64) return orc_brute_mul(a, na, b, nb, out, cap, out_len);
    return orc_ntt_mul(a, na, b, nb, out, cap, out_len);
}

/* mul_digits (mul.h:223-318).  Preconditions as in the reference: inputs are
 * non-empty, not all zero from their offset, digits < 2^28. */
int orc_mul_digits(const uint32_t* a, size_t na, const uint32_t* b, size_t nb, int same,
                   size_t prec, int64_t* point_pos, uint32_t* out, size_t cap, size_t* out_len) {
    if (same) {
        b = a;
        nb = na;
    }
    size_t off_a = (prec == 0 || na <= prec) ? 0 : na - prec;
    size_t off_b = (prec == 0 || nb <= prec) ? 0 : nb - prec;
    size_t tz_a = 0, tz_b = 0;
    while (off_a + tz_a < na && a[off_a + tz_a] == 0) ++tz_a;
    if (same) tz_b = tz_a;
    else
        while (off_b + tz_b < nb && b[off_b + tz_b] == 0) ++tz_b;
    if (off_a + tz_a == na || off_b + tz_b == nb) return ORC_ERR_INVALID; /* all zero: UB there */
    off_a += tz_a;
    off_b += tz_b;
    /* digits_to_vec64 (:245-268) */
    size_t la = ((na - off_a) * DIGIT_BITS + 63) / 64, lb = ((nb - off_b) * DIGIT_BITS + 63) / 64;
    uint64_t* A = calloc(la, sizeof(uint64_t));
    uint64_t* B = calloc(lb, sizeof(uint64_t));
    uint64_t* C = calloc(la + lb, sizeof(uint64_t));
    if (!A || !B || !C) {
        free(A), free(B), free(C);
        return ORC_ERR_NOMEM;
    }
    for (size_t i = off_a; i < na; ++i) {
        size_t bit = (i - off_a) * DIGIT_BITS, w = bit >> 6, s = bit & 63;
        A[w] |= (uint64_t)a[i] << s;
        if (s > 64 - DIGIT_BITS && w + 1 < la) A[w + 1] |= (uint64_t)a[i] >> (64 - s);
    }
    for (size_t i = off_b; i < nb; ++i) {
        size_t bit = (i - off_b) * DIGIT_BITS, w = bit >> 6, s = bit & 63;
        B[w] |= (uint64_t)b[i] << s;
        if (s > 64 - DIGIT_BITS && w + 1 < lb) B[w + 1] |= (uint64_t)b[i] >> (64 - s);
    }
    la = strip64(A, la);
    lb = strip64(B, lb);
    size_t lc = 0;
    int rc = orc_mul(A, la, same ? A : B, same ? la : lb, C, la + lb, &lc);
    if (rc) {
        free(A), free(B), free(C);
        return rc;
    }
    /* 64 -> 28 (:274-300) */
    size_t nres = (lc * 64 + DIGIT_BITS - 1) / DIGIT_BITS;
    uint32_t* res = calloc(nres ? nres : 1, sizeof(uint32_t));
    if (!res) {
        free(A), free(B), free(C);
        return ORC_ERR_NOMEM;
    }
    for (size_t k = 0; k < nres; ++k) {
        size_t bit = k * DIGIT_BITS, w = bit >> 6, s = bit & 63;
        uint64_t v = C[w] >> s;
        if (s > 64 - DIGIT_BITS && w + 1 < lc) v |= C[w + 1] << (64 - s);
        res[k] = (uint32_t)v & DIGIT_MASK;
    }
    while (nres > 0 && res[nres - 1] == 0) --nres;
    size_t lead = 0, need;
    if (prec) {
        size_t off_r = nres <= prec ? 0 : nres - prec;
        while (res[off_r] == 0) ++off_r;
        lead = off_r;
        need = nres - off_r;
        if (point_pos) *point_pos -= (int64_t)(off_a + off_b + off_r);
        *out_len = need;
        if (need > cap) rc = ORC_ERR_CAPACITY_OUT;
        else memcpy(out, res + lead, need * sizeof(uint32_t));
    } else {
        size_t z = tz_a + tz_b;
        need = z + nres;
        *out_len = need;
        if (need > cap) rc = ORC_ERR_CAPACITY_OUT;
        else {
            memset(out, 0, z * sizeof(uint32_t));
            memcpy(out + z, res, nres * sizeof(uint32_t));
        }
    }
    free(res), free(A), free(B), free(C);
    return rc;
}

/* x mod (2^61-1): 2^64 = 8 (mod 2^61-1), Horner from the top limb. */
uint64_t orc_mod_m61(const uint64_t* x, size_t n) {
    const uint64_t M = ((uint64_t)1 << 61) - 1;
    u128 r = 0;
    for (size_t i = n; i-- > 0;) {
        r = r * 8 + (x[i] % M);
        r = (r & M) + (r >> 61);
        r = (r & M) + (r >> 61);
    }
    uint64_t v = (uint64_t)r;
    while (v >= M) v -= M;
    return v;
}

/* Pairwise product tree over u64 leaves, odd tail carried up a level. */
int orc_product_tree(const uint64_t* leaves, size_t n, uint64_t* out, size_t cap,
                     size_t* out_len) {
    if (n == 0) {
        *out_len = 0;
        return 0;
    }
    uint64_t** vals = malloc(n * sizeof(uint64_t*));
    size_t* lens = malloc(n * sizeof(size_t));
    if (!vals || !lens) {
        free(vals), free(lens);
        return ORC_ERR_NOMEM;
    }
    for (size_t i = 0; i < n; ++i) {
        vals[i] = malloc(sizeof(uint64_t));
        vals[i][0] = leaves[i];
        lens[i] = strip64(vals[i], 1);
    }
    size_t m = n;
    int rc = 0;
    while (m > 1 && rc == 0) {
        size_t k = 0;
        for (size_t i = 0; i + 1 < m; i += 2) {
            size_t cl = lens[i] + lens[i + 1], got = 0;
            uint64_t* c = calloc(cl ? cl : 1, sizeof(uint64_t));
            if (lens[i] && lens[i + 1]) rc = orc_mul(vals[i], lens[i], vals[i + 1], lens[i + 1], c, cl, &got);
            free(vals[i]), free(vals[i + 1]);
            vals[k] = c;
            lens[k++] = got;
        }
        if (m % 2) {
            vals[k] = vals[m - 1];
            lens[k++] = lens[m - 1];
        }
        m = k;
    }
    if (rc == 0) {
        *out_len = lens[0];
        if (lens[0] > cap) rc = ORC_ERR_CAPACITY_OUT;
        else memcpy(out, vals[0], lens[0] * sizeof(uint64_t));
    }
    for (size_t i = 0; i < m; ++i) free(vals[i]);
    free(vals), free(lens);
    return rc;
}
