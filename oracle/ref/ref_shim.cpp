// ref_shim.cpp -- C entry points over the reference's own CPU functions.
//
// TEST INFRASTRUCTURE ONLY: built by oracle/Makefile together with the
// reference's sources (compiled where they lie) into oracle/_ref/, and used
// by the test suite to pin the oracle restatement, and by the benchmark's
// reference arm as the reference's CPU implementation of the path.
//
// Wrapped functions (clBool sources):
//   coo_utils::generate_coo_pairs_cpu      src/coo/coo_utils.cpp:204-218
//   coo_utils::generate_coo_cpu            src/coo/coo_utils.cpp:220-239
//   coo_utils::coo_pairs_to_dcsr_cpu       src/coo/coo_utils.cpp:241-266
//   coo_utils::matrix_multiplication_cpu   src/coo/coo_utils.cpp:470-514
//   coo_utils::get_workload                src/coo/coo_utils.cpp:439-456
//   coo_utils::matrix_addition_cpu         src/coo/coo_utils.cpp:315-324
//   coo_utils::kronecker_product_cpu       src/coo/coo_utils.cpp:326-342
//   csr_cpu_from_pairs                     src/common/matrices_conversions.cpp:158-177
//   utils::fill_random_buffer              src/common/utils.cpp:208-217
//   coo_utils::fill_random_matrix          src/coo/coo_utils.cpp:135-151
//   coo_utils::generate_random_matrices_large / _esc   src/coo/coo_utils.cpp:13-132
//   submatrix_cpu, reduce                  src/common/cpu_matrix_operations.cpp:6-75
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "coo/coo_utils.hpp"
#include "common/matrices_conversions.hpp"
#include "common/utils.hpp"

using namespace clbool;

template <class T>
static T *dup_vec(const std::vector<T> &v) {
    T *p = (T *)std::malloc((v.size() ? v.size() : 1) * sizeof(T));
    if (!v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(T));
    return p;
}

static matrix_dcsr_cpu to_dcsr(const uint32_t *rpt, const uint32_t *rows, const uint32_t *cols,
                               uint32_t nzr, uint32_t nnz) {
    cpu_buffer r(rpt, rpt + (nzr ? nzr + 1 : 0)), rr(rows, rows + nzr), c(cols, cols + nnz);
    return matrix_dcsr_cpu(r, rr, c);
}

static matrix_coo_cpu_pairs to_pairs(const uint32_t *rows, const uint32_t *cols, uint32_t n) {
    matrix_coo_cpu_pairs p(n);
    for (uint32_t i = 0; i < n; ++i) p[i] = {rows[i], cols[i]};
    return p;
}

static uint64_t from_pairs(const matrix_coo_cpu_pairs &p, uint32_t **rows, uint32_t **cols) {
    std::vector<uint32_t> r(p.size()), c(p.size());
    for (size_t i = 0; i < p.size(); ++i) { r[i] = p[i].first; c[i] = p[i].second; }
    *rows = dup_vec(r);
    *cols = dup_vec(c);
    return p.size();
}

extern "C" {

void ref_free(void *p) { std::free(p); }

uint64_t ref_gen_coo_pairs(uint32_t pseudo_nnz, uint32_t max_size, uint32_t **rows, uint32_t **cols) {
    return from_pairs(coo_utils::generate_coo_pairs_cpu(pseudo_nnz, max_size), rows, cols);
}

uint64_t ref_gen_coo_cpu(uint32_t pseudo_nnz, uint32_t max_size, uint32_t **rows, uint32_t **cols) {
    matrix_coo_cpu m = coo_utils::generate_coo_cpu(pseudo_nnz, max_size);
    *rows = dup_vec(m.rows());
    *cols = dup_vec(m.cols());
    return m.rows().size();
}

void ref_fill_random_buffer(uint32_t *buf, uint32_t n, uint32_t max) {
    cpu_buffer b(n);
    utils::fill_random_buffer(b, max);
    if (n) std::memcpy(buf, b.data(), n * sizeof(uint32_t));
}

void ref_fill_random_matrix(uint32_t *rows, uint32_t *cols, uint32_t n, uint32_t max_size) {
    cpu_buffer r(n), c(n);
    coo_utils::fill_random_matrix(r, c, max_size);
    if (n) {
        std::memcpy(rows, r.data(), n * sizeof(uint32_t));
        std::memcpy(cols, c.data(), n * sizeof(uint32_t));
    }
}

// DCSR from sorted unique pairs; outputs rpt[nzr+1] (0 entries when empty).
uint32_t ref_pairs_to_dcsr(const uint32_t *rows, const uint32_t *cols, uint32_t n,
                           uint32_t **rpt, uint32_t **rows_out, uint32_t **cols_out) {
    matrix_dcsr_cpu d = coo_utils::coo_pairs_to_dcsr_cpu(to_pairs(rows, cols, n));
    *rpt = dup_vec(d.rpt());
    *rows_out = dup_vec(d.rows());
    *cols_out = dup_vec(d.cols());
    return (uint32_t)d.rows().size();
}

// C = A * B with the reference's CPU product. Returns nnz; *nzr gets C's nzr.
uint32_t ref_spgemm(const uint32_t *a_rpt, const uint32_t *a_rows, const uint32_t *a_cols, uint32_t a_nzr, uint32_t a_nnz,
                    const uint32_t *b_rpt, const uint32_t *b_rows, const uint32_t *b_cols, uint32_t b_nzr, uint32_t b_nnz,
                    uint32_t **rpt, uint32_t **rows, uint32_t **cols, uint32_t *nzr) {
    matrix_dcsr_cpu a = to_dcsr(a_rpt, a_rows, a_cols, a_nzr, a_nnz);
    matrix_dcsr_cpu b = to_dcsr(b_rpt, b_rows, b_cols, b_nzr, b_nnz);
    matrix_dcsr_cpu c;
    coo_utils::matrix_multiplication_cpu(c, a, b);
    *rpt = dup_vec(c.rpt());
    *rows = dup_vec(c.rows());
    *cols = dup_vec(c.cols());
    *nzr = (uint32_t)c.rows().size();
    return (uint32_t)c.cols().size();
}

void ref_workload(const uint32_t *a_rpt, const uint32_t *a_rows, const uint32_t *a_cols, uint32_t a_nzr, uint32_t a_nnz,
                  const uint32_t *b_rpt, const uint32_t *b_rows, const uint32_t *b_cols, uint32_t b_nzr, uint32_t b_nnz,
                  uint32_t *out) {
    matrix_dcsr_cpu a = to_dcsr(a_rpt, a_rows, a_cols, a_nzr, a_nnz);
    matrix_dcsr_cpu b = to_dcsr(b_rpt, b_rows, b_cols, b_nzr, b_nnz);
    cpu_buffer w(a_nzr);
    coo_utils::get_workload(w, a, b);
    if (a_nzr) std::memcpy(out, w.data(), a_nzr * sizeof(uint32_t));
}

uint64_t ref_coo_add(const uint32_t *ar, const uint32_t *ac, uint32_t na,
                     const uint32_t *br, const uint32_t *bc, uint32_t nb,
                     uint32_t **rows, uint32_t **cols) {
    matrix_coo_cpu_pairs out;
    coo_utils::matrix_addition_cpu(out, to_pairs(ar, ac, na), to_pairs(br, bc, nb));
    return from_pairs(out, rows, cols);
}

// CSR of sorted unique pairs: rpt[m+1] (allocated) and cols[n] (allocated).
void ref_csr_from_pairs(const uint32_t *rows, const uint32_t *cols, uint32_t n, uint32_t m, uint32_t ncols,
                        uint32_t **rpt, uint32_t **cols_out) {
    matrix_csr_cpu c = csr_cpu_from_pairs(to_pairs(rows, cols, n), m, ncols);
    *rpt = dup_vec(c.rpt());
    *cols_out = dup_vec(c.cols());
}

uint64_t ref_kronecker_pairs(const uint32_t *ar, const uint32_t *ac, uint32_t na,
                             const uint32_t *br, const uint32_t *bc, uint32_t nb,
                             uint32_t b_nrows, uint32_t b_ncols, uint32_t **rows, uint32_t **cols) {
    matrix_coo_cpu_pairs out;
    coo_utils::kronecker_product_cpu(out, to_pairs(ar, ac, na), to_pairs(br, bc, nb), b_nrows, b_ncols);
    return from_pairs(out, rows, cols);
}

// Fixture generators of the reference's ESC / large-row kernel tests: a
// hand-written A and a FastRandom-seeded B.  which = 0: esc, 1: large.
// Arrays are returned as DCSR (rpt, rows, cols) for A then B.
void ref_random_matrices(int which, uint32_t max_size, uint32_t seed,
                         uint32_t **a_rpt, uint32_t **a_rows, uint32_t **a_cols, uint32_t *a_sizes,
                         uint32_t **b_rpt, uint32_t **b_rows, uint32_t **b_cols, uint32_t *b_sizes) {
    auto ab = which ? coo_utils::generate_random_matrices_large(max_size, seed)
                    : coo_utils::generate_random_matrices_esc(max_size, seed);
    *a_rpt = dup_vec(ab.first.rpt());
    *a_rows = dup_vec(ab.first.rows());
    *a_cols = dup_vec(ab.first.cols());
    a_sizes[0] = ab.first.rpt().size();
    a_sizes[1] = ab.first.rows().size();
    a_sizes[2] = ab.first.cols().size();
    *b_rpt = dup_vec(ab.second.rpt());
    *b_rows = dup_vec(ab.second.rows());
    *b_cols = dup_vec(ab.second.cols());
    b_sizes[0] = ab.second.rpt().size();
    b_sizes[1] = ab.second.rows().size();
    b_sizes[2] = ab.second.cols().size();
}

uint32_t ref_submatrix(const uint32_t *rpt, const uint32_t *rows, const uint32_t *cols, uint32_t nzr, uint32_t nnz,
                       uint32_t i, uint32_t j, uint32_t nrows, uint32_t ncols, uint32_t **orpt, uint32_t **orows,
                       uint32_t **ocols, uint32_t *onzr) {
    matrix_dcsr_cpu a = to_dcsr(rpt, rows, cols, nzr, nnz);
    matrix_dcsr_cpu c;
    utils::submatrix_cpu(c, a, i, j, nrows, ncols);
    *orpt = dup_vec(c.rpt());
    *orows = dup_vec(c.rows());
    *ocols = dup_vec(c.cols());
    *onzr = (uint32_t)c.rows().size();
    return (uint32_t)c.cols().size();
}

uint32_t ref_reduce(const uint32_t *rpt, const uint32_t *rows, const uint32_t *cols, uint32_t nzr, uint32_t nnz,
                    uint32_t **orpt, uint32_t **orows, uint32_t **ocols) {
    matrix_dcsr_cpu a = to_dcsr(rpt, rows, cols, nzr, nnz);
    matrix_dcsr_cpu c;
    utils::reduce(c, a);
    *orpt = dup_vec(c.rpt());
    *orows = dup_vec(c.rows());
    *ocols = dup_vec(c.cols());
    return (uint32_t)c.rows().size();
}

}  // extern "C"
