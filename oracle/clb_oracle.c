/*
 * clb_oracle.c -- CPU restatement of clBool's boolean sparse hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: only the test
 * suite, the smoke check and the CPU-baseline leg of the benchmark load it,
 * and only to check or to time against.  The product (libclbool_b200.so)
 * never links or calls it.
 *
 * Every function restates the reference's CPU semantics (cited by file:line
 * of the clBool sources) with 64-bit offsets and OpenMP, so that it stays a
 * valid oracle at sizes where the reference's uint32 offsets overflow.
 * Outputs are canonical (rows strictly increasing, columns strictly
 * increasing inside a row), so any correct restatement pins the same bytes.
 *
 * Layouts (all host memory):
 *   DCSR: rpt u64[nzr+1], rows u32[nzr], cols u32[nnz]
 *   CSR : rpt u64[nrows+1], cols u32[nnz]
 *   COO : rows u32[nnz], cols u32[nnz], lexicographically sorted
 * Arrays returned through out-pointers are malloc'ed here; release them with
 * orc_free().
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

typedef struct {
    uint64_t nrows, ncols, nnz, nzr;
    uint64_t *rpt;
    uint32_t *rows;
    uint32_t *cols;
} orc_dcsr;

void orc_free(void *p) { free(p); }

int orc_set_threads(int n) {
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
}

/* ------------------------------------------------------------------------ */
/* FastRandom: xorshift generator used by the reference's test generators.  */
/* Follows libs/utils/libutils/fast_random.h:8-40 (64-bit `unsigned long`   */
/* state on LP64).  Restated so the reference's randomised test inputs can  */
/* be regenerated bit-exactly.                                              */
/* ------------------------------------------------------------------------ */
typedef struct { uint64_t x, y, z; } orc_rng;

static void rng_reset(orc_rng *r, uint64_t seed) {
    r->x = seed;
    r->y = 362436069ull;
    r->z = 521288629ull;
}

/* Value in [lo, hi] inclusive; fast_random.h:23-33. */
static uint32_t rng_next(orc_rng *r, int32_t lo, int32_t hi) {
    r->x ^= r->x << 16;
    r->x ^= r->x >> 5;
    r->x ^= r->x << 1;
    uint64_t t = r->x;
    r->x = r->y;
    r->y = r->z;
    r->z = t ^ r->x ^ r->y;
    uint64_t span = (uint64_t)(int64_t)hi - (uint64_t)(int64_t)lo + 1ull;
    return (uint32_t)lo + (uint32_t)(r->z % span);
}

/* utils.cpp:208-217 fill_random_buffer: buf[i] = next(0, max), seed = n. */
void orc_fill_random_buffer(uint32_t *buf, uint32_t n, uint32_t max) {
    orc_rng r;
    rng_reset(&r, n);
    for (uint32_t i = 0; i < n; ++i) buf[i] = rng_next(&r, 0, (int32_t)max);
}

/* coo_utils.cpp:135-151 fill_random_matrix: rows/cols in [0, max_size-1],
 * seed = n, one row draw then one column draw per entry. */
void orc_fill_random_matrix(uint32_t *rows, uint32_t *cols, uint32_t n, uint32_t max_size) {
    if (max_size == 0) return;
    orc_rng r;
    rng_reset(&r, n);
    for (uint32_t i = 0; i < n; ++i) {
        rows[i] = rng_next(&r, 0, (int32_t)(max_size - 1));
        cols[i] = rng_next(&r, 0, (int32_t)(max_size - 1));
    }
}

/* coo_utils.cpp:153-160 fill_random_matrix_pairs: values in [0, max_size]. */
void orc_fill_random_pairs_inclusive(uint32_t *rows, uint32_t *cols, uint32_t n, uint32_t max_size) {
    orc_rng r;
    rng_reset(&r, n);
    for (uint32_t i = 0; i < n; ++i) {
        rows[i] = rng_next(&r, 0, (int32_t)max_size);
        cols[i] = rng_next(&r, 0, (int32_t)max_size);
    }
}

/* ------------------------------------------------------------------------ */
/* Sorting of (row, col) pairs: lexicographic, as std::sort on              */
/* std::pair<uint32_t,uint32_t> (coo_utils.cpp:214, test/src/procedures.cpp */
/* :74).  LSD radix sort on the 64-bit key row<<32|col.                     */
/* ------------------------------------------------------------------------ */
static void radix_sort_u64(uint64_t *keys, uint64_t n) {
    if (n < 2) return;
    uint64_t *tmp = (uint64_t *)malloc(n * sizeof(uint64_t));
    uint64_t *src = keys, *dst = tmp;
    for (int pass = 0; pass < 4; ++pass) {
        int shift = pass * 16;
        uint64_t *hist = (uint64_t *)calloc(65536, sizeof(uint64_t));
        for (uint64_t i = 0; i < n; ++i) hist[(src[i] >> shift) & 0xFFFF]++;
        if (hist[(src[0] >> shift) & 0xFFFF] == n) { free(hist); continue; }
        uint64_t s = 0;
        for (int b = 0; b < 65536; ++b) { uint64_t c = hist[b]; hist[b] = s; s += c; }
        for (uint64_t i = 0; i < n; ++i) dst[hist[(src[i] >> shift) & 0xFFFF]++] = src[i];
        free(hist);
        uint64_t *t = src; src = dst; dst = t;
    }
    if (src != keys) memcpy(keys, src, n * sizeof(uint64_t));
    free(tmp);
}

/* Sort pairs in place (coo::sort_arrays semantics, coo_initialization.cpp:6-32). */
void orc_sort_pairs(uint32_t *rows, uint32_t *cols, uint64_t n) {
    uint64_t *k = (uint64_t *)malloc((n ? n : 1) * sizeof(uint64_t));
    for (uint64_t i = 0; i < n; ++i) k[i] = ((uint64_t)rows[i] << 32) | cols[i];
    radix_sort_u64(k, n);
    for (uint64_t i = 0; i < n; ++i) { rows[i] = (uint32_t)(k[i] >> 32); cols[i] = (uint32_t)k[i]; }
    free(k);
}

/* Remove adjacent duplicate pairs of a sorted COO in place; returns the new
 * length.  Restates std::unique after std::sort (coo_utils.cpp:216,
 * matrix_coo::reduce_duplicates2 matrix_coo.cpp:117-170). */
uint64_t orc_unique_pairs(uint32_t *rows, uint32_t *cols, uint64_t n) {
    if (n == 0) return 0;
    uint64_t w = 1;
    for (uint64_t i = 1; i < n; ++i) {
        if (rows[i] != rows[w - 1] || cols[i] != cols[w - 1]) {
            rows[w] = rows[i];
            cols[w] = cols[i];
            ++w;
        }
    }
    return w;
}

/* coo_utils.cpp:204-218 generate_coo_pairs_cpu: draw `pseudo_nnz` pairs in
 * [0, max_size-1]^2 with FastRandom(pseudo_nnz), sort, unique. */
uint64_t orc_gen_coo_pairs(uint32_t pseudo_nnz, uint32_t max_size, uint32_t **rows_out, uint32_t **cols_out) {
    uint32_t *r = (uint32_t *)malloc(((uint64_t)pseudo_nnz + 1) * sizeof(uint32_t));
    uint32_t *c = (uint32_t *)malloc(((uint64_t)pseudo_nnz + 1) * sizeof(uint32_t));
    uint64_t n = pseudo_nnz;
    if (max_size == 0) n = 0;
    orc_fill_random_matrix(r, c, (uint32_t)n, max_size);
    orc_sort_pairs(r, c, n);
    n = orc_unique_pairs(r, c, n);
    *rows_out = r;
    *cols_out = c;
    return n;
}

/* coo_utils.cpp:220-239 generate_coo_cpu: pairs in [0, max_size]^2. */
uint64_t orc_gen_coo_inclusive(uint32_t pseudo_nnz, uint32_t max_size, uint32_t **rows_out, uint32_t **cols_out) {
    uint32_t *r = (uint32_t *)malloc(((uint64_t)pseudo_nnz + 1) * sizeof(uint32_t));
    uint32_t *c = (uint32_t *)malloc(((uint64_t)pseudo_nnz + 1) * sizeof(uint32_t));
    orc_fill_random_pairs_inclusive(r, c, pseudo_nnz, max_size);
    orc_sort_pairs(r, c, pseudo_nnz);
    uint64_t n = orc_unique_pairs(r, c, pseudo_nnz);
    *rows_out = r;
    *cols_out = c;
    return n;
}

/* ------------------------------------------------------------------------ */
/* Scans                                                                    */
/* ------------------------------------------------------------------------ */

/* prefix_sum semantics (cl_operations.cpp:4-88, checked by
 * test/src/procedures.cpp:7-49): exclusive scan in place, returns total. */
uint64_t orc_prefix_sum_u32(uint32_t *a, uint64_t n) {
    uint64_t s = 0;
    for (uint64_t i = 0; i < n; ++i) { uint32_t v = a[i]; a[i] = (uint32_t)s; s += v; }
    return s;
}

uint64_t orc_prefix_sum_u64(uint64_t *a, uint64_t n) {
    uint64_t s = 0;
    for (uint64_t i = 0; i < n; ++i) { uint64_t v = a[i]; a[i] = s; s += v; }
    return s;
}

/* ------------------------------------------------------------------------ */
/* Conversions                                                              */
/* ------------------------------------------------------------------------ */

/* coo_utils.cpp:268-294 coo_to_dcsr_cpu (and the device path
 * matrices_conversions.cpp:7-37,78-91): one DCSR row per distinct COO row.
 * Returns nzr; *rpt (nzr+1) and *rows (nzr) are allocated here; the column
 * array of the COO is the DCSR column array. */
uint64_t orc_coo_to_dcsr(const uint32_t *rows, uint64_t nnz, uint64_t **rpt_out, uint32_t **rows_out) {
    uint64_t nzr = 0;
    for (uint64_t i = 0; i < nnz; ++i)
        if (i == 0 || rows[i] != rows[i - 1]) ++nzr;
    uint64_t *rpt = (uint64_t *)malloc((nzr + 1) * sizeof(uint64_t));
    uint32_t *rr = (uint32_t *)malloc((nzr ? nzr : 1) * sizeof(uint32_t));
    uint64_t k = 0;
    for (uint64_t i = 0; i < nnz; ++i) {
        if (i == 0 || rows[i] != rows[i - 1]) { rpt[k] = i; rr[k] = rows[i]; ++k; }
    }
    rpt[nzr] = nnz;
    *rpt_out = rpt;
    *rows_out = rr;
    return nzr;
}

/* dcsr_to_coo (matrices_conversions.cpp:43-76 + dscr_to_coo.cl:8-23):
 * expand the row of every entry. rows_out has nnz entries. */
void orc_dcsr_to_coo_rows(const uint64_t *rpt, const uint32_t *rows, uint64_t nzr, uint32_t *rows_out) {
    for (uint64_t i = 0; i < nzr; ++i)
        for (uint64_t j = rpt[i]; j < rpt[i + 1]; ++j) rows_out[j] = rows[i];
}

/* dcsr_to_csr (matrices_conversions.cpp:247-271): dense rpt of nrows+1. */
void orc_dcsr_to_csr_rpt(const uint64_t *rpt, const uint32_t *rows, uint64_t nzr, uint64_t nrows, uint64_t *csr_rpt) {
    memset(csr_rpt, 0, (nrows + 1) * sizeof(uint64_t));
    for (uint64_t i = 0; i < nzr; ++i) csr_rpt[rows[i]] = rpt[i + 1] - rpt[i];
    orc_prefix_sum_u64(csr_rpt, nrows + 1);
}

/* csr_to_dcsr (matrices_conversions.cpp:211-244): keep the non-empty rows.
 * Returns nzr; allocates *rpt_out (nzr+1) and *rows_out (nzr). */
uint64_t orc_csr_to_dcsr(const uint64_t *csr_rpt, uint64_t nrows, uint64_t **rpt_out, uint32_t **rows_out) {
    uint64_t nzr = 0;
    for (uint64_t i = 0; i < nrows; ++i) nzr += csr_rpt[i + 1] > csr_rpt[i];
    uint64_t *rpt = (uint64_t *)malloc((nzr + 1) * sizeof(uint64_t));
    uint32_t *rr = (uint32_t *)malloc((nzr ? nzr : 1) * sizeof(uint32_t));
    uint64_t k = 0;
    for (uint64_t i = 0; i < nrows; ++i)
        if (csr_rpt[i + 1] > csr_rpt[i]) { rpt[k] = csr_rpt[i]; rr[k] = (uint32_t)i; ++k; }
    rpt[nzr] = nrows ? csr_rpt[nrows] : 0;
    *rpt_out = rpt;
    *rows_out = rr;
    return nzr;
}

/* csr_cpu_from_pairs (matrices_conversions.cpp:158-177): dense rpt from a
 * sorted COO.  csr_rpt has nrows+1 entries. */
void orc_csr_rpt_from_coo(const uint32_t *rows, uint64_t nnz, uint64_t nrows, uint64_t *csr_rpt) {
    memset(csr_rpt, 0, (nrows + 1) * sizeof(uint64_t));
    for (uint64_t i = 0; i < nnz; ++i) csr_rpt[rows[i]]++;
    orc_prefix_sum_u64(csr_rpt, nrows + 1);
}

/* ------------------------------------------------------------------------ */
/* SpGEMM over the boolean semiring                                          */
/* ------------------------------------------------------------------------ */

/* Position of B's row `k` in B.rows, or -1.  B.rows is strictly increasing. */
static int64_t find_row(const orc_dcsr *b, uint32_t k) {
    uint64_t lo = 0, hi = b->nzr;
    while (lo < hi) {
        uint64_t m = lo + (hi - lo) / 2;
        if (b->rows[m] < k) lo = m + 1; else hi = m;
    }
    return (lo < b->nzr && b->rows[lo] == k) ? (int64_t)lo : -1;
}

/* Products of every A row: P_i = sum over k in A_i of |B_k|.
 * Restates get_workload (coo_utils.cpp:439-456) and count_workload.cl:30-53. */
void orc_workload(const orc_dcsr *a, const orc_dcsr *b, uint64_t *out) {
    #pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < (int64_t)a->nzr; ++i) {
        uint64_t s = 0;
        for (uint64_t j = a->rpt[i]; j < a->rpt[i + 1]; ++j) {
            int64_t p = find_row(b, a->cols[j]);
            if (p >= 0) s += b->rpt[p + 1] - b->rpt[p];
        }
        out[i] = s;
    }
}

/* Per-thread accumulator: a bitmap over B's columns plus the list of touched
 * words, so that each row costs O(products + touched words log touched). */
typedef struct {
    uint64_t *bits;
    uint32_t *touched;
    uint64_t ntouched;
    uint64_t nwords;
} acc_t;

static int cmp_u32(const void *x, const void *y) {
    uint32_t a = *(const uint32_t *)x, b = *(const uint32_t *)y;
    return a < b ? -1 : a > b;
}

static inline void acc_insert(acc_t *acc, uint32_t c, uint64_t *count) {
    uint64_t w = c >> 6;
    uint64_t m = 1ull << (c & 63);
    uint64_t old = acc->bits[w];
    if (!(old & m)) {
        if (!old) acc->touched[acc->ntouched++] = (uint32_t)w;
        acc->bits[w] = old | m;
        ++*count;
    }
}

/* Emit the set columns in increasing order into out (may be NULL to only
 * clear), clearing the accumulator. */
static void acc_drain(acc_t *acc, uint32_t *out) {
    if (acc->ntouched > 1) qsort(acc->touched, acc->ntouched, sizeof(uint32_t), cmp_u32);
    uint64_t k = 0;
    for (uint64_t t = 0; t < acc->ntouched; ++t) {
        uint32_t w = acc->touched[t];
        uint64_t bitsw = acc->bits[w];
        if (out) {
            while (bitsw) {
                int b = __builtin_ctzll(bitsw);
                out[k++] = (uint32_t)(((uint64_t)w << 6) + (uint64_t)b);
                bitsw &= bitsw - 1;
            }
        }
        acc->bits[w] = 0;
    }
    acc->ntouched = 0;
}

/* Row-wise product of one A row into the accumulator; returns the number of
 * distinct columns (the exact nnz of C's row). */
static uint64_t row_product(const orc_dcsr *a, const orc_dcsr *b, const int64_t *bmap, uint64_t i, acc_t *acc) {
    uint64_t cnt = 0;
    for (uint64_t j = a->rpt[i]; j < a->rpt[i + 1]; ++j) {
        uint32_t k = a->cols[j];
        int64_t p = bmap ? (k < b->nrows ? bmap[k] : -1) : find_row(b, k);
        if (p < 0) continue;
        for (uint64_t q = b->rpt[p]; q < b->rpt[p + 1]; ++q) acc_insert(acc, b->cols[q], &cnt);
    }
    return cnt;
}

/* C = A * B over (or, and).  Semantics of matrix_multiplication_cpu
 * (coo_utils.cpp:470-514): C keeps A's row ids that have at least one
 * product, each row's columns sorted and unique; shape A.nrows x B.ncols.
 * Two phases (exact count, then fill), 64-bit offsets.  Returns 0 on
 * success, -1 if B.ncols is too wide for the bitmap accumulator. */
int orc_spgemm(const orc_dcsr *a, const orc_dcsr *b, orc_dcsr *c) {
    memset(c, 0, sizeof(*c));
    c->nrows = a->nrows;
    c->ncols = b->ncols;
    if (a->nnz == 0 || b->nnz == 0 || a->nzr == 0 || b->nzr == 0) return 0;
    if (b->ncols > (1ull << 31)) return -1;

    int64_t *bmap = NULL;
    if (b->nrows <= (1ull << 27)) {
        bmap = (int64_t *)malloc((b->nrows + 1) * sizeof(int64_t));
        for (uint64_t k = 0; k < b->nrows; ++k) bmap[k] = -1;
        for (uint64_t p = 0; p < b->nzr; ++p)
            if (b->rows[p] < b->nrows) bmap[b->rows[p]] = (int64_t)p;  /* rows past nrows never match */
    }
    uint64_t nwords = (b->ncols + 63) / 64;
    uint64_t *rownnz = (uint64_t *)malloc(a->nzr * sizeof(uint64_t));

    #pragma omp parallel
    {
        acc_t acc;
        acc.nwords = nwords;
        acc.bits = (uint64_t *)calloc(nwords, sizeof(uint64_t));
        acc.touched = (uint32_t *)malloc(nwords * sizeof(uint32_t));
        acc.ntouched = 0;
        #pragma omp for schedule(dynamic, 64)
        for (int64_t i = 0; i < (int64_t)a->nzr; ++i) {
            rownnz[i] = row_product(a, b, bmap, (uint64_t)i, &acc);
            acc_drain(&acc, NULL);
        }
        free(acc.bits);
        free(acc.touched);
    }

    uint64_t nzr = 0, nnz = 0;
    for (uint64_t i = 0; i < a->nzr; ++i) { nzr += rownnz[i] > 0; nnz += rownnz[i]; }
    c->nzr = nzr;
    c->nnz = nnz;
    c->rpt = (uint64_t *)malloc((nzr + 1) * sizeof(uint64_t));
    c->rows = (uint32_t *)malloc((nzr ? nzr : 1) * sizeof(uint32_t));
    c->cols = (uint32_t *)malloc((nnz ? nnz : 1) * sizeof(uint32_t));
    uint64_t *off = (uint64_t *)malloc(a->nzr * sizeof(uint64_t));
    {
        uint64_t k = 0, s = 0;
        for (uint64_t i = 0; i < a->nzr; ++i) {
            off[i] = s;
            if (rownnz[i]) { c->rpt[k] = s; c->rows[k] = a->rows[i]; ++k; }
            s += rownnz[i];
        }
        c->rpt[nzr] = s;
    }

    #pragma omp parallel
    {
        acc_t acc;
        acc.nwords = nwords;
        acc.bits = (uint64_t *)calloc(nwords, sizeof(uint64_t));
        acc.touched = (uint32_t *)malloc(nwords * sizeof(uint32_t));
        acc.ntouched = 0;
        #pragma omp for schedule(dynamic, 64)
        for (int64_t i = 0; i < (int64_t)a->nzr; ++i) {
            if (!rownnz[i]) continue;
            row_product(a, b, bmap, (uint64_t)i, &acc);
            acc_drain(&acc, c->cols + off[i]);
        }
        free(acc.bits);
        free(acc.touched);
    }
    free(off);
    free(rownnz);
    free(bmap);
    return 0;
}

/* Exact nnz of every C row (0 for rows without products), i.e. the output
 * of the symbolic pass (hash_symbolic_* kernels). */
int orc_spgemm_row_nnz(const orc_dcsr *a, const orc_dcsr *b, uint64_t *rownnz) {
    if (b->ncols > (1ull << 31)) return -1;
    memset(rownnz, 0, a->nzr * sizeof(uint64_t));
    if (a->nnz == 0 || b->nnz == 0 || b->nzr == 0) return 0;
    int64_t *bmap = NULL;
    if (b->nrows <= (1ull << 27)) {
        bmap = (int64_t *)malloc((b->nrows + 1) * sizeof(int64_t));
        for (uint64_t k = 0; k < b->nrows; ++k) bmap[k] = -1;
        for (uint64_t p = 0; p < b->nzr; ++p)
            if (b->rows[p] < b->nrows) bmap[b->rows[p]] = (int64_t)p;  /* rows past nrows never match */
    }
    uint64_t nwords = (b->ncols + 63) / 64;
    #pragma omp parallel
    {
        acc_t acc;
        acc.nwords = nwords;
        acc.bits = (uint64_t *)calloc(nwords, sizeof(uint64_t));
        acc.touched = (uint32_t *)malloc(nwords * sizeof(uint32_t));
        acc.ntouched = 0;
        #pragma omp for schedule(dynamic, 64)
        for (int64_t i = 0; i < (int64_t)a->nzr; ++i) {
            rownnz[i] = row_product(a, b, bmap, (uint64_t)i, &acc);
            acc_drain(&acc, NULL);
        }
        free(acc.bits);
        free(acc.touched);
    }
    free(bmap);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Additions                                                                */
/* ------------------------------------------------------------------------ */

/* COO addition: std::merge + std::unique (coo_utils.cpp:315-324).
 * Allocates *rows_out/*cols_out; returns nnz of the sum. */
uint64_t orc_coo_add(const uint32_t *ar, const uint32_t *ac, uint64_t na,
                     const uint32_t *br, const uint32_t *bc, uint64_t nb,
                     uint32_t **rows_out, uint32_t **cols_out) {
    uint64_t cap = na + nb;
    uint32_t *r = (uint32_t *)malloc((cap ? cap : 1) * sizeof(uint32_t));
    uint32_t *c = (uint32_t *)malloc((cap ? cap : 1) * sizeof(uint32_t));
    uint64_t i = 0, j = 0, k = 0;
    while (i < na || j < nb) {
        uint64_t ka = i < na ? (((uint64_t)ar[i] << 32) | ac[i]) : UINT64_MAX;
        uint64_t kb = j < nb ? (((uint64_t)br[j] << 32) | bc[j]) : UINT64_MAX;
        uint64_t key;
        if (i < na && (j >= nb || ka <= kb)) { key = ka; ++i; } else { key = kb; ++j; }
        uint32_t rr = (uint32_t)(key >> 32), cc = (uint32_t)key;
        if (k == 0 || r[k - 1] != rr || c[k - 1] != cc) { r[k] = rr; c[k] = cc; ++k; }
    }
    *rows_out = r;
    *cols_out = c;
    return k;
}

/* CSR addition (csr_addition.cpp:26-168; checked in the reference against
 * matrix_addition_cpu + csr_cpu_from_pairs, test/src/operations.cpp:420-452).
 * c_rpt has nrows+1 entries; *cols_out is allocated; returns nnz. */
uint64_t orc_csr_add(const uint64_t *arpt, const uint32_t *acols,
                     const uint64_t *brpt, const uint32_t *bcols,
                     uint64_t nrows, uint64_t *c_rpt, uint32_t **cols_out) {
    uint64_t *cnt = (uint64_t *)malloc((nrows + 1) * sizeof(uint64_t));
    #pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t r = 0; r < (int64_t)nrows; ++r) {
        uint64_t i = arpt[r], ie = arpt[r + 1], j = brpt[r], je = brpt[r + 1], k = 0;
        while (i < ie && j < je) {
            if (acols[i] < bcols[j]) ++i;
            else if (bcols[j] < acols[i]) ++j;
            else { ++i; ++j; }
            ++k;
        }
        cnt[r] = k + (ie - i) + (je - j);
    }
    uint64_t s = 0;
    for (uint64_t r = 0; r < nrows; ++r) { c_rpt[r] = s; s += cnt[r]; }
    c_rpt[nrows] = s;
    uint32_t *out = (uint32_t *)malloc((s ? s : 1) * sizeof(uint32_t));
    #pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t r = 0; r < (int64_t)nrows; ++r) {
        uint64_t i = arpt[r], ie = arpt[r + 1], j = brpt[r], je = brpt[r + 1], k = c_rpt[r];
        while (i < ie && j < je) {
            if (acols[i] < bcols[j]) out[k++] = acols[i++];
            else if (bcols[j] < acols[i]) out[k++] = bcols[j++];
            else { out[k++] = acols[i]; ++i; ++j; }
        }
        while (i < ie) out[k++] = acols[i++];
        while (j < je) out[k++] = bcols[j++];
    }
    free(cnt);
    *cols_out = out;
    return s;
}

/* ------------------------------------------------------------------------ */
/* Kronecker product and transpose                                          */
/* ------------------------------------------------------------------------ */

/* DCSR Kronecker (dcsr_kronecker_product.cpp:5-64, dcsr_kronecker.cl:38-97;
 * CPU check kronecker_product_cpu coo_utils.cpp:326-342): C row
 * (ia, ib) -> a.rows[ia]*b.nrows + b.rows[ib], row-major over (ia, ib);
 * entry (ja, jb) -> a.cols[ja]*b.ncols + b.cols[jb], ja-major. */
void orc_kronecker(const orc_dcsr *a, const orc_dcsr *b, orc_dcsr *c) {
    memset(c, 0, sizeof(*c));
    c->nrows = a->nrows * b->nrows;
    c->ncols = a->ncols * b->ncols;
    uint64_t nzr = a->nzr * b->nzr, nnz = a->nnz * b->nnz;
    if (nnz == 0) return;
    c->nzr = nzr;
    c->nnz = nnz;
    c->rpt = (uint64_t *)malloc((nzr + 1) * sizeof(uint64_t));
    c->rows = (uint32_t *)malloc(nzr * sizeof(uint32_t));
    c->cols = (uint32_t *)malloc(nnz * sizeof(uint32_t));
    uint64_t s = 0, r = 0;
    for (uint64_t ia = 0; ia < a->nzr; ++ia) {
        uint64_t la = a->rpt[ia + 1] - a->rpt[ia];
        for (uint64_t ib = 0; ib < b->nzr; ++ib) {
            uint64_t lb = b->rpt[ib + 1] - b->rpt[ib];
            c->rpt[r] = s;
            c->rows[r] = (uint32_t)((uint64_t)a->rows[ia] * b->nrows + b->rows[ib]);
            ++r;
            s += la * lb;
        }
    }
    c->rpt[nzr] = s;
    #pragma omp parallel for schedule(dynamic, 64)
    for (int64_t row = 0; row < (int64_t)nzr; ++row) {
        uint64_t ia = (uint64_t)row / b->nzr, ib = (uint64_t)row % b->nzr;
        uint64_t k = c->rpt[row];
        for (uint64_t ja = a->rpt[ia]; ja < a->rpt[ia + 1]; ++ja)
            for (uint64_t jb = b->rpt[ib]; jb < b->rpt[ib + 1]; ++jb)
                c->cols[k++] = (uint32_t)((uint64_t)a->cols[ja] * b->ncols + b->cols[jb]);
    }
}

/* Transpose (dcsr_transpose.cpp:5-16: DCSR -> COO -> swap -> sort -> DCSR). */
void orc_transpose(const orc_dcsr *a, orc_dcsr *c) {
    memset(c, 0, sizeof(*c));
    c->nrows = a->ncols;
    c->ncols = a->nrows;
    if (a->nnz == 0) return;
    uint32_t *r = (uint32_t *)malloc(a->nnz * sizeof(uint32_t));
    uint32_t *cc = (uint32_t *)malloc(a->nnz * sizeof(uint32_t));
    orc_dcsr_to_coo_rows(a->rpt, a->rows, a->nzr, cc);
    memcpy(r, a->cols, a->nnz * sizeof(uint32_t));
    orc_sort_pairs(r, cc, a->nnz);
    c->nnz = a->nnz;
    c->nzr = orc_coo_to_dcsr(r, a->nnz, &c->rpt, &c->rows);
    c->cols = cc;
    free(r);
}

/* ------------------------------------------------------------------------ */
/* Row-size predictor (learned sizing of the single-pass SpGEMM): FP64       */
/* reference of the network the CUDA kernels train, used to check their      */
/* gradients.  Architecture: 6 -> 64 -> 64 -> 1, ReLU; weights used as BF16  */
/* (round to nearest even of the FP32 masters); loss = mean squared error.   */
/* Parameter layout: W1[64][6], b1[64], W2[64][64], b2[64], w3[64], b3.      */
/* ------------------------------------------------------------------------ */
#define MLP_F 6
#define MLP_H 64
#define MLP_NP (MLP_H * MLP_F + MLP_H + MLP_H * MLP_H + MLP_H + MLP_H + 1)

static double bf16_round(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7F800000u) != 0x7F800000u) u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
    else u &= 0xFFFF0000u;
    float r;
    memcpy(&r, &u, 4);
    return (double)r;
}

int orc_mlp_num_params(void) { return MLP_NP; }

/* Loss and gradient over n rows; grads (MLP_NP doubles) w.r.t. the rounded
 * weights.  preds (n doubles) may be NULL. */
void orc_mlp_grad(const float *params, const float *feat, const float *target, uint64_t n, double *grads,
                  double *loss, double *preds) {
    double w[MLP_NP];
    for (int k = 0; k < MLP_NP; ++k) w[k] = bf16_round(params[k]);
    const double *W1 = w, *b1 = W1 + MLP_H * MLP_F, *W2 = b1 + MLP_H, *b2 = W2 + MLP_H * MLP_H, *w3 = b2 + MLP_H,
                 *b3 = w3 + MLP_H;
    memset(grads, 0, sizeof(double) * MLP_NP);
    double *gW1 = grads, *gb1 = gW1 + MLP_H * MLP_F, *gW2 = gb1 + MLP_H, *gb2 = gW2 + MLP_H * MLP_H,
           *gw3 = gb2 + MLP_H, *gb3 = gw3 + MLP_H;
    double L = 0;
    for (uint64_t r = 0; r < n; ++r) {
        const float *x = feat + r * MLP_F;
        double h1[MLP_H], h2[MLP_H], y = *b3;
        for (int j = 0; j < MLP_H; ++j) {
            double a = b1[j];
            for (int f = 0; f < MLP_F; ++f) a += W1[j * MLP_F + f] * x[f];
            h1[j] = a > 0 ? a : 0;
        }
        for (int j = 0; j < MLP_H; ++j) {
            double a = b2[j];
            for (int k = 0; k < MLP_H; ++k) a += W2[j * MLP_H + k] * h1[k];
            h2[j] = a > 0 ? a : 0;
            y += w3[j] * h2[j];
        }
        if (preds) preds[r] = y;
        const double e = y - target[r];
        L += e * e / (double)n;
        const double dy = 2.0 * e / (double)n;
        double g2[MLP_H], g1[MLP_H];
        *gb3 += dy;
        for (int j = 0; j < MLP_H; ++j) {
            gw3[j] += dy * h2[j];
            g2[j] = h2[j] > 0 ? dy * w3[j] : 0;
            gb2[j] += g2[j];
            for (int k = 0; k < MLP_H; ++k) gW2[j * MLP_H + k] += g2[j] * h1[k];
        }
        for (int k = 0; k < MLP_H; ++k) {
            double a = 0;
            for (int j = 0; j < MLP_H; ++j) a += W2[j * MLP_H + k] * g2[j];
            g1[k] = h1[k] > 0 ? a : 0;
            gb1[k] += g1[k];
            for (int f = 0; f < MLP_F; ++f) gW1[k * MLP_F + f] += g1[k] * x[f];
        }
    }
    *loss = L;
}


/* ------------------------------------------------------------------------ */
/* dcsr::submatrix (src/dcsr/dcsr_submatrix.cpp:98-155, CPU form            */
/* src/common/cpu_matrix_operations.cpp:6-52): rows [i, i+nrows) and columns */
/* [j, j+ncols) of A, re-indexed to start at 0; empty rows dropped.          */
/* ------------------------------------------------------------------------ */
static uint64_t lb_u32(const uint32_t *a, uint64_t n, uint64_t key) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        uint64_t m = lo + (hi - lo) / 2;
        if ((uint64_t)a[m] < key) lo = m + 1; else hi = m;
    }
    return lo;
}

void orc_submatrix(const orc_dcsr *a, uint64_t i, uint64_t j, uint64_t nrows, uint64_t ncols, orc_dcsr *out) {
    memset(out, 0, sizeof(*out));
    out->nrows = nrows;
    out->ncols = ncols;
    if (a->nnz == 0) return;
    uint64_t r0 = lb_u32(a->rows, a->nzr, i), r1 = lb_u32(a->rows, a->nzr, i + nrows);
    uint64_t n = r1 > r0 ? r1 - r0 : 0;
    uint64_t *beg = (uint64_t *)malloc((n ? n : 1) * 8), *len = (uint64_t *)malloc((n ? n : 1) * 8);
    uint64_t nnz = 0, nzr = 0;
    for (uint64_t k = 0; k < n; ++k) {
        const uint64_t s = a->rpt[r0 + k], e = a->rpt[r0 + k + 1];
        const uint64_t b = s + lb_u32(a->cols + s, e - s, j), f = s + lb_u32(a->cols + s, e - s, j + ncols);
        beg[k] = b;
        len[k] = f - b;
        nnz += len[k];
        nzr += len[k] > 0;
    }
    out->nnz = nnz;
    out->nzr = nzr;
    out->rpt = (uint64_t *)malloc((nzr + 1) * 8);
    out->rows = (uint32_t *)malloc((nzr ? nzr : 1) * 4);
    out->cols = (uint32_t *)malloc((nnz ? nnz : 1) * 4);
    uint64_t o = 0, q = 0;
    for (uint64_t k = 0; k < n; ++k) {
        if (!len[k]) continue;
        out->rpt[q] = o;
        out->rows[q] = (uint32_t)(a->rows[r0 + k] - i);
        for (uint64_t t = 0; t < len[k]; ++t) out->cols[o + t] = (uint32_t)(a->cols[beg[k] + t] - j);
        o += len[k];
        ++q;
    }
    out->rpt[nzr] = nnz;
    free(beg);
    free(len);
}

/* dcsr::reduce (src/dcsr/dcsr_reduce.cpp:5-31, cpu_matrix_operations.cpp:63-75):
 * the row-wise OR, a column vector with one entry (column 0) per stored row. */
void orc_reduce(const orc_dcsr *a, orc_dcsr *out) {
    memset(out, 0, sizeof(*out));
    out->nrows = a->nrows;
    out->ncols = 1;
    if (a->nnz == 0) return;
    out->nnz = out->nzr = a->nzr;
    out->rpt = (uint64_t *)malloc((a->nzr + 1) * 8);
    out->rows = (uint32_t *)malloc(a->nzr * 4);
    out->cols = (uint32_t *)calloc(a->nzr, 4);
    for (uint64_t k = 0; k <= a->nzr; ++k) out->rpt[k] = k;
    memcpy(out->rows, a->rows, a->nzr * 4);
}
