/*
 * clbool_b200.h -- C ABI of libclbool_b200.so, the sm_100a (B200) back end
 * of clBool's boolean sparse hot path.
 *
 * Plain pointers and sizes only.  All matrix arrays live in device memory of
 * the controls' device.  Index arrays (rows, cols) are uint32; offsets (rpt)
 * are uint64 so that products with more than 2^32 output entries stay
 * representable (the reference stores them as uint32).
 *
 * Every entry point returns a clb_status (0 = success).  Operations are
 * synchronous on return, like the reference's host functions, and run on the
 * controls' stream.  Output arrays are allocated through the controls'
 * allocator (stream-ordered cudaMallocAsync by default) and released with
 * clb_free() or clb_*_release().  An empty matrix carries NULL arrays, as
 * the reference's matrix_dcsr(nrows, ncols) carries no buffers
 * (src/core/matrix_dcsr.hpp:44-48).  Output structs may alias input structs:
 * inputs are read before the output struct is written.
 */
#ifndef CLBOOL_B200_H
#define CLBOOL_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define CLB_API __attribute__((visibility("default")))
#else
#define CLB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  1..14 are clbool::Status (src/core/error.hpp:130-151) in
 * the reference's order, shifted by one so that 0 means success. */
typedef enum clb_status {
    CLB_SUCCESS = 0,
    CLB_NO_SUCH_PROGRAM = 1,
    CLB_CREATE_KERNEL_ERROR = 2,
    CLB_BUILD_PROGRAM_ERROR = 3,
    CLB_INCOMPLETE_KERNEL = 4,
    CLB_RUN_KERNEL_FAILURE = 5,
    CLB_EVENT_WAITING_ERROR = 6,
    CLB_CREATE_BUFFER_ERROR = 7,
    CLB_COPY_BUFFER_ERROR = 8,
    CLB_READ_BUFFER_ERROR = 9,
    CLB_WRITE_BUFFER_ERROR = 10,
    CLB_CREATE_CONTROLS_ERROR = 11,
    CLB_INVALID_ARGUMENT = 12,
    CLB_INVALID_VALUE = 13,
    CLB_INITIALIZATION_ERROR = 14,
    /* Not in the reference: a kernel reported failure through the device
     * status word (bounded wait gave up, accumulator overflow that has no
     * fallback, bounds check). */
    CLB_DEVICE_STATUS_ERROR = 64,
    /* Not in the reference: a size limit of this implementation. */
    CLB_NOT_SUPPORTED = 65
} clb_status;

/* DCSR (src/core/matrix_dcsr.hpp:11-84): only non-empty rows are stored. */
typedef struct clb_dcsr {
    uint64_t nrows, ncols, nnz, nzr;
    uint64_t *rpt;  /* nzr + 1 */
    uint32_t *rows; /* nzr, strictly increasing */
    uint32_t *cols; /* nnz, strictly increasing inside a row */
} clb_dcsr;

/* COO (src/core/matrix_coo.hpp:12-83): lexicographically sorted pairs. */
typedef struct clb_coo {
    uint64_t nrows, ncols, nnz;
    uint32_t *rows; /* nnz */
    uint32_t *cols; /* nnz */
} clb_coo;

/* CSR (src/core/matrix_csr.hpp:7-42). */
typedef struct clb_csr {
    uint64_t nrows, ncols, nnz;
    uint64_t *rpt;  /* nrows + 1 */
    uint32_t *cols; /* nnz */
} clb_csr;

/* Per-call SpGEMM statistics (optional out-parameter). */
typedef struct clb_spgemm_stats {
    uint64_t products;        /* sum over A rows of the B-row lengths hit  */
    uint64_t nnz, nzr;        /* of C                                       */
    uint64_t rows_per_bin[16];/* A rows routed to each accumulator bin      */
    uint64_t fallback_rows;   /* single-pass forms: rows re-run by two passes */
    uint64_t capacity;        /* single-pass forms: slots allocated for C   */
    uint32_t kernel_launches; /* kernels this call launched                 */
    uint32_t reserved;
    uint64_t spilled_rows;    /* learned form: rows over their slot that went
                                 to the spill arena in the same pass        */
} clb_spgemm_stats;

typedef struct clb_controls clb_controls;

/* Caller-supplied device allocator: alloc returns NULL on failure. */
typedef void *(*clb_alloc_fn)(void *ctx, size_t bytes, void *stream);
typedef void (*clb_free_fn)(void *ctx, void *ptr, void *stream);

/* ------------------------------------------------------------- runtime -- */
/* Name of a status code; never NULL.  Replaces operator<<(ostream&, Status)
 * (src/core/error.hpp:154-180) over the same Status order (error.hpp:130-151). */
CLB_API const char *clb_status_string(int status);
/* Message of the last failing call on this host thread ("" if none): what
 * clbool::Exception carried across the C++ surface (src/core/error.hpp:183-213). */
CLB_API const char *clb_last_error(void);
/* Library version: major*10000 + minor*100 + patch (no counterpart). */
CLB_API int clb_version(void);

/* Replaces create_controls(platform_id, device_id)
 * (src/common/env.cpp:7-36): one controls object per CUDA device. */
CLB_API int clb_controls_create(int device, clb_controls **out);
/* End of a Controls' lifetime (src/core/controls.hpp:12-28). */
CLB_API int clb_controls_destroy(clb_controls *ctl);
/* Run subsequent operations on `stream` (a cudaStream_t; NULL = own stream):
 * the counterpart of Controls::queue / async_queue (src/core/controls.hpp:15-16);
 * clb_controls_sync waits for it like queue.finish(). */
CLB_API int clb_controls_set_stream(clb_controls *ctl, void *stream);
CLB_API void *clb_controls_get_stream(clb_controls *ctl);
/* Caller-supplied allocator for every device buffer (no counterpart: the
 * reference allocates cl::Buffer objects itself). */
CLB_API int clb_controls_set_allocator(clb_controls *ctl, clb_alloc_fn alloc, clb_free_fn release, void *ctx);
CLB_API int clb_controls_sync(clb_controls *ctl);
/* No counterpart in the reference.  Waits for the controls' stream, then
 * returns the device memory that the library's stream-ordered pool keeps
 * cached (freed buffers are kept for reuse and never handed back on their
 * own) to the driver, for a caller that needs that memory elsewhere (another
 * library, another process).  Buffers still in use are not touched; the next
 * large requests grow the pool again. */
CLB_API int clb_controls_trim(clb_controls *ctl);
/* CUDA graphs over the controls' stream (no counterpart in the reference,
 * which enqueues OpenCL commands one by one).  clb_graph_begin starts
 * capturing the stream (thread-local mode); operations that read nothing back
 * to the host -- clb_dcsr_spgemm_batched_capture -- can then be recorded;
 * clb_graph_end stops and instantiates (*graph = a cudaGraphExec_t);
 * clb_graph_launch replays it on the stream without synchronising.  The
 * stream must not be the legacy default stream. */
CLB_API int clb_graph_begin(clb_controls *ctl);
CLB_API int clb_graph_end(clb_controls *ctl, void **graph);
CLB_API int clb_graph_launch(clb_controls *ctl, void *graph);
CLB_API int clb_graph_destroy(void *graph);
/* Controls::device (src/core/controls.hpp:13) as a CUDA device ordinal. */
CLB_API int clb_controls_device(clb_controls *ctl);

/* Replaces show_devices() (src/common/env.cpp:38-54). */
CLB_API int clb_device_count(int *count);
CLB_API int clb_device_info(int device, char *name, size_t name_len, int *sm_count, uint64_t *total_mem);

/* Opt-in kernel timing: with profiling on, every kernel launch (or group of
 * launches of one name) is bracketed by CUDA events on the controls' stream.
 * clb_profile_read synchronises, aggregates the records by name and clears
 * them.  Not in the reference (its timing is wall-clock logging,
 * src/common/cl_includes.hpp:61-71). */
typedef struct clb_profile_entry {
    char name[48];
    uint32_t launches;
    uint32_t reserved;
    double ms;
} clb_profile_entry;
CLB_API int clb_profile_enable(clb_controls *ctl, int on);
CLB_API int clb_profile_read(clb_controls *ctl, clb_profile_entry *out, int capacity, int *count);

/* Device memory through the controls' allocator (the reference creates
 * cl::Buffer objects inside its matrix constructors, src/core/matrix_dcsr.hpp:28-43). */
CLB_API int clb_malloc(clb_controls *ctl, size_t bytes, void **out);
CLB_API int clb_free(clb_controls *ctl, void *ptr);
/* Stream-ordered copies; synchronous on return (the buffer transfers of
 * matrix_dcsr_from_cpu / matrix_dcsr_from_gpu, src/common/matrices_conversions.cpp:93-140). */
CLB_API int clb_memcpy_h2d(clb_controls *ctl, void *dst, const void *src, size_t bytes);
CLB_API int clb_memcpy_d2h(clb_controls *ctl, void *dst, const void *src, size_t bytes);
CLB_API int clb_memcpy_d2d(clb_controls *ctl, void *dst, const void *src, size_t bytes);
/* Pinned host memory for staging (no counterpart). */
CLB_API int clb_host_alloc(size_t bytes, void **out);
CLB_API int clb_host_free(void *ptr);

/* A matrix's buffers are freed: the end of the refcounted cl::Buffer members of
 * matrix_dcsr / matrix_coo / matrix_csr (src/core/matrix_dcsr.hpp:11-84,
 * matrix_coo.hpp:12-83, matrix_csr.hpp:7-42). */
CLB_API int clb_dcsr_release(clb_controls *ctl, clb_dcsr *m);
CLB_API int clb_coo_release(clb_controls *ctl, clb_coo *m);
CLB_API int clb_csr_release(clb_controls *ctl, clb_csr *m);

/* ----------------------------------------------------------- primitives -- */
/* prefix_sum (src/common/cl_operations.hpp:9-12, cl_operations.cpp:4-88):
 * exclusive scan of `n` entries in place; *total = sum of the inputs. */
CLB_API int clb_prefix_sum_u32(clb_controls *ctl, uint32_t *array, uint64_t n, uint64_t *total);
CLB_API int clb_prefix_sum_u64(clb_controls *ctl, uint64_t *array, uint64_t n, uint64_t *total);

/* No counterpart in the reference.  The same exclusive scan of `n` uint32
 * entries in place, for callers that cannot allocate device memory when they
 * need it (for instance a runtime that has reserved all of the GPU's memory
 * for its own pool, or a hot loop that must not pay for cudaMalloc's implicit
 * synchronisation).  It allocates nothing: its scratch is a fixed 256 KiB
 * array inside the library, so n is limited to 2^28 entries (larger n is
 * rejected with CLB_INVALID_ARGUMENT).  It takes no controls object, launches
 * on `stream` (a cudaStream_t; NULL = legacy default stream of the current
 * device) with the stream's own device made current for the call, does not
 * synchronise, and writes the sum of the inputs to the device pointer
 * `d_total` when it is not NULL.  The first call on a device looks up the
 * scratch array's device address for that device (loading the library's
 * device code there if nothing has yet); make that first call before any
 * stream capture.  Later calls look the address up again unless their stream
 * is being captured, so the address stays right after cudaDeviceReset.
 * Every call on one device shares the one array, so calls whose work
 * overlaps on the GPU (different streams, or different host threads or
 * controls on one device) race: serialise them. */
CLB_API int clb_prefix_sum_u32_noalloc(uint32_t *array, uint64_t n, uint64_t *d_total, void *stream);

/* fill_with (src/common/cl_operations.hpp:14, cl_operations.cpp:94-100). */
CLB_API int clb_fill_u32(clb_controls *ctl, uint32_t *array, uint64_t n, uint32_t value);

/* coo::sort_arrays (src/coo/coo_initialization.hpp:9): sort (row, col)
 * pairs lexicographically, in place. */
CLB_API int clb_coo_sort(clb_controls *ctl, uint32_t *rows, uint32_t *cols, uint64_t n);

/* matrix_coo(..., sorted, noDuplicates=false) dedupe
 * (src/core/matrix_coo.cpp:117-170): `in` must be sorted; `out` gets new
 * arrays without adjacent duplicates. */
CLB_API int clb_coo_reduce_duplicates(clb_controls *ctl, const clb_coo *in, clb_coo *out);

/* ---------------------------------------------------------- conversions -- */
/* coo_to_dcsr_shallow (src/common/matrices_conversions.hpp:11):
 * out->rpt/rows are new; out->cols aliases in->cols unless deep != 0. */
CLB_API int clb_coo_to_dcsr(clb_controls *ctl, const clb_coo *in, clb_dcsr *out, int deep);
/* dcsr_to_coo_shallow / dcsr_to_coo_deep (matrices_conversions.hpp:9-10). */
CLB_API int clb_dcsr_to_coo(clb_controls *ctl, const clb_dcsr *in, clb_coo *out, int deep);
/* dcsr_to_csr (matrices_conversions.hpp:26): out->cols aliases in->cols. */
CLB_API int clb_dcsr_to_csr(clb_controls *ctl, const clb_dcsr *in, clb_csr *out);
/* csr_to_dcsr (matrices_conversions.hpp:24): out->cols aliases in->cols. */
CLB_API int clb_csr_to_dcsr(clb_controls *ctl, const clb_csr *in, clb_dcsr *out);

/* ------------------------------------------------------------ operations -- */
/* dcsr::matrix_multiplication_hash (src/dcsr/dcsr.hpp:33-36,
 * dcsr_matrix_multiplication_hash.cpp:51-119): C = A*B over (or, and), the
 * exact two-pass form (symbolic count, scan, numeric fill). */
CLB_API int clb_dcsr_spgemm_hash(clb_controls *ctl, const clb_dcsr *a, const clb_dcsr *b, clb_dcsr *c,
                         clb_spgemm_stats *stats);

/* coo::matrix_addition (src/coo/coo.hpp:9-14, coo_matrix_addition.cpp:32-73):
 * C = A | B of sorted unique COOs; same shapes or CLB_INVALID_ARGUMENT. */
CLB_API int clb_coo_add(clb_controls *ctl, const clb_coo *a, const clb_coo *b, clb_coo *c);

/* csr::matrix_addition (src/csr/csr.hpp:12, csr_addition.cpp:26-168). */
CLB_API int clb_csr_add(clb_controls *ctl, const clb_csr *a, const clb_csr *b, clb_csr *c);
/* No counterpart in the reference, which adds one pair per call
 * (src/csr/csr.hpp:12): c[k] = a[k] + b[k] for k < count in one set of
 * launches.  The pairs' rows are stacked (row pointers shifted, columns
 * copied), one csr::matrix_addition runs over the stack (merge path, or the
 * insertion path when one side of the stack is much sparser) and its rows
 * are cut back into the pairs.  Each c[k] owns its buffers; a pair whose
 * shapes differ fails the call with CLB_INVALID_ARGUMENT before any device
 * work. */
CLB_API int clb_csr_add_batched(clb_controls *ctl, uint32_t count, const clb_csr *a, const clb_csr *b, clb_csr *c);

/* dcsr::kronecker_product (src/dcsr/dcsr.hpp:38-41,
 * dcsr_kronecker_product.cpp:5-64): C row (ia, ib) = A.rows[ia]*B.nrows +
 * B.rows[ib], columns A.cols[ja]*B.ncols + B.cols[jb]. */
CLB_API int clb_dcsr_kronecker(clb_controls *ctl, const clb_dcsr *a, const clb_dcsr *b, clb_dcsr *c);

/* dcsr::transpose (src/dcsr/dcsr.hpp:17-19, dcsr_transpose.cpp:5-16). */
CLB_API int clb_dcsr_transpose(clb_controls *ctl, const clb_dcsr *in, clb_dcsr *out);

/* dcsr::submatrix (src/dcsr/dcsr.hpp:12-16, dcsr_submatrix.cpp:98-155): rows
 * [i, i+nrows) and columns [j, j+ncols) of `in`, re-indexed to start at 0,
 * empty rows dropped; `out` is nrows x ncols (also when it has no entries). */
CLB_API int clb_dcsr_submatrix(clb_controls *ctl, const clb_dcsr *in, uint64_t i, uint64_t j, uint64_t nrows,
                               uint64_t ncols, clb_dcsr *out);
/* dcsr::reduce (src/dcsr/dcsr.hpp:22-24, dcsr_reduce.cpp:5-31): the row-wise
 * OR of `in` as an nrows x 1 matrix, one entry (column 0) per stored row. */
CLB_API int clb_dcsr_reduce(clb_controls *ctl, const clb_dcsr *in, clb_dcsr *out);

/* dcsr::matrix_multiplication (src/dcsr/dcsr.hpp:27-30,
 * dcsr_matrix_multiplication.cpp:26-97): the ESC/merge form -- every row gets
 * its upper bound of slots, one expand-sort-compress (or bitmap) pass fills
 * them, and the rows are compacted into C. Same result as the hash form. */
CLB_API int clb_dcsr_spgemm_esc(clb_controls *ctl, const clb_dcsr *a, const clb_dcsr *b, clb_dcsr *c,
                                clb_spgemm_stats *stats);

/* ------------------------------------------------------ learned sizing -- */
/* Not in the reference.  A row-size predictor (MLP 6 -> 64 -> 64 -> 1, ReLU,
 * BF16 weights, FP32 accumulation) estimates log2(1 + nnz) of every row of
 * C = A*B from six features of its A row; clb_dcsr_spgemm_learned gives each
 * row that many output slots (times 2^margin_log2, plus slack, never above
 * the exact bound min(products, ncols)), runs ONE numeric pass, and re-runs
 * the rows that overflow with the exact two-pass form, so C is always exact. */
typedef struct clb_sizer clb_sizer;
CLB_API int clb_sizer_num_params(void);
CLB_API int clb_sizer_create(clb_controls *ctl, uint64_t seed, clb_sizer **out);
CLB_API int clb_sizer_destroy(clb_sizer *sizer);
/* FP32 master weights (checkpoint): `count` must be clb_sizer_num_params(). */
CLB_API int clb_sizer_get_params(clb_sizer *sizer, float *host, size_t count);
CLB_API int clb_sizer_set_params(clb_sizer *sizer, const float *host, size_t count);
/* Device arrays: features[6 * a->nzr] (scaled log2 features) and, when not
 * NULL, workload[a->nzr] (products per A row). */
CLB_API int clb_dcsr_row_features(clb_controls *ctl, const clb_dcsr *a, const clb_dcsr *b, float *features,
                                  uint32_t *workload);
/* Exact nnz of every C row (the symbolic pass alone), device u32[a->nzr]. */
CLB_API int clb_dcsr_row_nnz(clb_controls *ctl, const clb_dcsr *a, const clb_dcsr *b, uint32_t *row_nnz);
/* Predictions (scaled log2(1 + nnz)) of n rows; device arrays. */
CLB_API int clb_sizer_predict(clb_sizer *sizer, const float *features, uint64_t n, float *out);
/* Mean-squared-error loss and its gradient w.r.t. the BF16-rounded weights
 * over n rows (device features/targets; host grads of num_params floats). */
CLB_API int clb_sizer_gradients(clb_sizer *sizer, const float *features, const float *targets, uint64_t n,
                                float *grads_host, float *loss_host);
/* Adam training over n rows (device arrays; targets = log2(1 + nnz) / 16). */
CLB_API int clb_sizer_train(clb_sizer *sizer, const float *features, const float *targets, uint64_t n,
                            uint32_t epochs, uint32_t batch, float lr, uint64_t seed, float *final_loss);
/* tuning: accumulator tuning (NULL = defaults; `form` is ignored). */
CLB_API int clb_dcsr_spgemm_learned(clb_controls *ctl, const clb_dcsr *a, const clb_dcsr *b, const clb_sizer *sizer,
                                    float margin_log2, float slack, const struct clb_spgemm_tuning *tuning,
                                    clb_dcsr *c, clb_spgemm_stats *stats);

/* ------------------------------------------------- tuning and batching -- */
/* Not in the reference.  Accumulator tuning; every setting gives the same C.
 *   form            0: exact two-pass (hash form), 1: one pass into
 *                   upper-bound slots (ESC form) + compaction, 2: exact
 *                   two-pass whose symbolic pass keeps the bitmap rows'
 *                   bitmaps (4 bytes per 32 columns per bitmap row: 128 KB
 *                   a row at 2^20 columns) and whose numeric pass expands
 *                   them instead of inserting their products again (falls
 *                   back to 0 without room for them and for products wider
 *                   than 2^20 columns)
 *   warp_max        rows with at most this many products use the warp ESC
 *                   kernels: 32, 64, 128 or 256 (threads per row: 32)
 *   bitmap_min      rows with more products use the bitmap kernel: 256..4096
 *                   (the rest use the CTA hash / CTA ESC kernels, whose table
 *                   size follows the row's bound: 1K, 2K, 4K or 8K slots)
 *   bitmap_threads  threads per bitmap row: 256, 512 or 1024
 *   small_lanes     lanes per row for rows of at most 8 / 16 products: 8
 *                   (four / two rows per warp), 16, or 32 (a warp per row)
 *   wide_rows       rows with 2^20 < ncols <= 2^22: 1 = one thread-block
 *                   cluster (2 or 4 CTAs) per row, 2 = one CTA per row that
 *                   walks the products once per 2^20-column chunk (default)
 * Zero fields take the defaults (clb_spgemm_tuning_default). */
typedef struct clb_spgemm_tuning {
    uint32_t form;
    uint32_t warp_max;
    uint32_t bitmap_min;
    uint32_t bitmap_threads;
    uint32_t small_lanes;
    uint32_t wide_rows;
    uint32_t reserved[2];
} clb_spgemm_tuning;
CLB_API void clb_spgemm_tuning_default(clb_spgemm_tuning *tuning);
/* C = A*B with a tuning (NULL = defaults, i.e. clb_dcsr_spgemm_hash). */
CLB_API int clb_dcsr_spgemm_tuned(clb_controls *ctl, const clb_dcsr *a, const clb_dcsr *b,
                                  const clb_spgemm_tuning *tuning, clb_dcsr *c, clb_spgemm_stats *stats);
/* c[k] = a[k] * b[k] for k < count, all pairs in one pass: the pairs are
 * stacked block-diagonally and multiplied by one set of launches (the launch
 * count does not grow with the batch), then C is split per pair.  Each c[k]
 * owns its buffers.  stats (optional) covers the whole batch. */
CLB_API int clb_dcsr_spgemm_batched(clb_controls *ctl, uint32_t count, const clb_dcsr *a, const clb_dcsr *b,
                                    clb_dcsr *c, const clb_spgemm_tuning *tuning, clb_spgemm_stats *stats);
/* The learned-sized batched product (no counterpart in the reference): the
 * pairs are stacked as in clb_dcsr_spgemm_batched, and the stack is
 * multiplied by the learned single pass of clb_dcsr_spgemm_learned: row
 * features relative to each row's own pair (row position in the pair's A,
 * density of the pair's B), predicted slots for the rows over
 * tuning->bitmap_min products (exact bounds below), the spill arena for rows
 * over their slot, and the exact two-pass form for the rows that outgrow
 * both.  The result never depends on the predictor. */
CLB_API int clb_dcsr_spgemm_batched_learned(clb_controls *ctl, uint32_t count, const clb_dcsr *a,
                                            const clb_dcsr *b, clb_dcsr *c, const clb_sizer *sizer,
                                            float margin_log2, float slack, const clb_spgemm_tuning *tuning,
                                            clb_spgemm_stats *stats);
/* No counterpart in the reference (whose additions take two operands,
 * src/coo/coo.hpp:9-14, src/csr/csr.hpp:12): out = mats[0] v mats[1] v ...
 * v mats[count - 1] (count <= 32 matrices of one shape, count * nrows <
 * 2^32) in one pass.  The union is the product A_u B_u with B_u the mats
 * stacked row-wise and A_u's row r holding column j * nrows + r for every
 * matrix j that stores row r, so the SpGEMM accumulators merge the (at most
 * count) sorted rows r and drop duplicates.  tuning: the accumulator tuning
 * of that product (NULL = the single pass into upper-bound slots); stats
 * (optional) are the product's, products = the entries of all mats. */
CLB_API int clb_dcsr_union(clb_controls *ctl, uint32_t count, const clb_dcsr *mats,
                           const clb_spgemm_tuning *tuning, clb_dcsr *out, clb_spgemm_stats *stats);
/* Times the batched product under every candidate tuning (32: form x
 * bitmap_min x bitmap_threads x warp_max x small_lanes; twice that with both
 * wide_rows settings when a pair has more than 2^20 columns) on the given
 * pairs and returns the
 * fastest in *best (each candidate: one warm-up call, then the best of three
 * timed calls); tried/ms (optional, max_tried entries) receive each
 * candidate and its device time in ms, *n_tried their number.  Pairs of at
 * most 2^20 columns also try form 2 (48 candidates); a single pair (count =
 * 1) is timed through clb_dcsr_spgemm_tuned. */
CLB_API int clb_spgemm_autotune(clb_controls *ctl, uint32_t count, const clb_dcsr *a, const clb_dcsr *b,
                                clb_spgemm_tuning *best, clb_spgemm_tuning *tried, double *ms, uint32_t max_tried,
                                uint32_t *n_tried);

/* C = A*B written into host memory (no counterpart in the reference, whose
 * product stays on the device until matrix_dcsr_from_gpu,
 * src/common/matrices_conversions.cpp:121-140).  A's stored rows are cut into
 * `blocks` (1..64) ranges of about equal products; each block is one call of
 * the learned form (sizer != NULL, with margin_log2 / slack / tuning as in
 * clb_dcsr_spgemm_learned) or of clb_dcsr_spgemm_tuned (sizer == NULL), and
 * its rows are copied to the host on a second stream while the next block
 * is multiplied.  h_rpt: rows_capacity + 1 entries, h_rows: rows_capacity,
 * h_cols: cols_capacity (page-locked memory, e.g. clb_host_alloc, lets the
 * copies overlap; pageable memory works without overlap).  On return
 * *nzr / *nnz give C's size and the arrays hold C; too small arrays give
 * CLB_INVALID_VALUE.  stats (optional) sums the blocks. */
CLB_API int clb_dcsr_spgemm_to_host(clb_controls *ctl, const clb_dcsr *a, const clb_dcsr *b, const clb_sizer *sizer,
                                    float margin_log2, float slack, const clb_spgemm_tuning *tuning,
                                    uint32_t blocks, uint64_t *h_rpt, uint32_t *h_rows, uint32_t *h_cols,
                                    uint64_t rows_capacity, uint64_t cols_capacity, uint64_t *nzr, uint64_t *nnz,
                                    clb_spgemm_stats *stats);

/* No counterpart in the reference (a single-device library,
 * src/core/controls.hpp:12-28): the stored rows [lo, hi) of A as a DCSR of
 * A's shape that owns copies of them (row ids kept, row pointers rebased to
 * 0) -- one rank's share of A when A's rows are split over GPUs.  An empty
 * range gives an empty matrix; a range past nzr(A) is rejected with
 * CLB_INVALID_ARGUMENT. */
CLB_API int clb_dcsr_row_block(clb_controls *ctl, const clb_dcsr *a, uint64_t lo, uint64_t hi, clb_dcsr *out);

/* Host-sync-free batched product (no counterpart in the reference): the
 * pairs are stacked as in clb_dcsr_spgemm_batched and multiplied by the
 * single-pass form into upper-bound slots, but every size comes from the
 * caller and nothing is read back to the host, so the call can be recorded
 * into a CUDA graph (clb_graph_begin / clb_graph_end) and replayed while the
 * pairs' device arrays keep their sizes and change their contents.
 * Temporaries come from the controls' stream-ordered pool (graph memory
 * nodes when captured); tuning->form is ignored.
 *   slot_capacity  slot entries; clb_spgemm_batched_plan gives the need of the
 *                  current contents (sum over stacked rows of
 *                  round_up(min(products, ncols), 4));
 *   c_rpt, c_rows  device, rows_need + 1 and rows_need entries (rows_need =
 *                  stored rows of the pairs with entries on both sides);
 *   c_cols         device, cols_capacity entries (slots_need always suffices);
 *   result         device u64[2 + 2 * (count + 1)]: [0] nzr, [1] nnz of the
 *                  stacked C, [2 + k] its first row of pair k, [3 + count + k]
 *                  its first column position of pair k (k = count: totals).
 *                  Pair k is rows [r_k, r_k+1) with rpt c_rpt[r_k..r_k+1]
 *                  minus c_rpt[r_k], row ids local to the pair, and columns
 *                  c_cols[j_k, j_k+1);
 *   flags          device u32, 0 when C is complete; bit 0: slot capacity
 *                  too small (rows left empty), bit 1: cols_capacity too
 *                  small (rows not written), bit 2: a device check failed,
 *                  bit 3 (learned form only): a row outgrew its slot and
 *                  the spill arena (left empty).
 * Returns once the work is enqueued (no synchronisation). */
CLB_API int clb_dcsr_spgemm_batched_capture(clb_controls *ctl, uint32_t count, const clb_dcsr *a, const clb_dcsr *b,
                                            const clb_spgemm_tuning *tuning, uint64_t slot_capacity,
                                            uint64_t *c_rpt, uint32_t *c_rows, uint32_t *c_cols,
                                            uint64_t cols_capacity, uint64_t *result, uint32_t *flags);
/* Sizes for clb_dcsr_spgemm_batched_capture on the pairs' current contents
 * (runs the workload pass and synchronises; call it outside a capture). */
CLB_API int clb_spgemm_batched_plan(clb_controls *ctl, uint32_t count, const clb_dcsr *a, const clb_dcsr *b,
                                    uint64_t *rows_need, uint64_t *slots_need);
/* The host-sync-free batched product with learned slots (no counterpart in
 * the reference): as clb_dcsr_spgemm_batched_capture, but the rows over
 * tuning->bitmap_min products get the slots the predictor gives them (as in
 * clb_dcsr_spgemm_batched_learned), and a row whose exact count outgrows its
 * slot reserves it in a spill arena of arena_capacity entries (a temporary
 * of the call) in the same pass.  A row that finds no room there is left
 * empty and raises bit 3 of *flags (the caller then recomputes the batch by
 * an exact form: clb_dcsr_spgemm_batched); cols_capacity must hold C, i.e.
 * the slots plus the spilled rows (slot_capacity + arena_capacity always
 * suffices).  The call can be recorded into a CUDA graph like the
 * upper-bound form. */
CLB_API int clb_dcsr_spgemm_batched_capture_learned(clb_controls *ctl, uint32_t count, const clb_dcsr *a,
                                                    const clb_dcsr *b, const clb_sizer *sizer, float margin_log2,
                                                    float slack, const clb_spgemm_tuning *tuning,
                                                    uint64_t slot_capacity, uint64_t arena_capacity,
                                                    uint64_t *c_rpt, uint32_t *c_rows, uint32_t *c_cols,
                                                    uint64_t cols_capacity, uint64_t *result, uint32_t *flags);
/* Sizes for clb_dcsr_spgemm_batched_capture_learned on the pairs' current
 * contents: stored rows and the learned slots (runs the feature and
 * prediction passes and synchronises; call it outside a capture). */
CLB_API int clb_spgemm_batched_plan_learned(clb_controls *ctl, uint32_t count, const clb_dcsr *a,
                                            const clb_dcsr *b, const clb_sizer *sizer, float margin_log2,
                                            float slack, const clb_spgemm_tuning *tuning, uint64_t *rows_need,
                                            uint64_t *slots_need);

/* Products per A row (count_workload, dcsr_matrix_multiplication.cpp:388-404):
 * workload has a->nzr entries in device memory; *total = their sum. */
CLB_API int clb_dcsr_workload(clb_controls *ctl, const clb_dcsr *a, const clb_dcsr *b, uint32_t *workload,
                      uint64_t *total);

#ifdef __cplusplus
}
#endif
#endif /* CLBOOL_B200_H */
