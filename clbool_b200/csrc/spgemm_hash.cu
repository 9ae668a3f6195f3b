// spgemm_hash.cu -- dcsr::matrix_multiplication_hash, exact two-pass form.
//
// Reference: src/dcsr/dcsr_matrix_multiplication_hash.cpp:51-119 (flow),
// count_workload (dcsr_matrix_multiplication.cpp:388-404, count_workload.cl),
// binning (..._hash.cpp:13-47, 301-345), count_nnz (:122-201), fill_nnz
// (:203-299).  Differences of mechanism, not of result:
//   * B's rows are found through a dense row map built once per call (two
//     loads) instead of a binary search per A entry;
//   * binning is a device histogram + scatter (no host loop, no host copy of
//     the workload);
//   * C's row list is known right after the workload pass (a row has output
//     iff it has products), so no empty-row compaction pass runs at the end;
//   * offsets are 64-bit.
#include <cstring>
#include <string>

#include "spgemm.cuh"

namespace clb {

namespace {

constexpr int WL_NT = 256;
constexpr int WL_GROUP = 8;        // lanes per A row in the workload kernel
constexpr uint32_t WL_LONG = 256;  // rows with more A entries: one CTA each

// Products of every A row: a group of 8 lanes per row; rows over WL_LONG
// entries are listed for workload_long_kernel (R-MAT hub rows hold tens of
// thousands of entries, which 8 lanes would walk long after the rest).
__global__ void __launch_bounds__(WL_NT) workload_kernel(AView a, BRows b, uint32_t *__restrict__ work,
                                                         unsigned long long *__restrict__ total,
                                                         uint32_t *__restrict__ long_rows,
                                                         uint32_t *__restrict__ n_long) {
    __shared__ unsigned long long ptot;
    if (threadIdx.x == 0) ptot = 0;
    __syncthreads();
    const uint32_t gl = threadIdx.x & (WL_GROUP - 1);
    const uint32_t gmask = 0xFFu << (lane_id() & 24u);
    unsigned long long mine = 0;
    for (uint64_t row = ((uint64_t)blockIdx.x * WL_NT + threadIdx.x) / WL_GROUP; row < a.nzr;
         row += (uint64_t)gridDim.x * (WL_NT / WL_GROUP)) {
        const uint64_t ja = a.rpt[row], je = a.rpt[row + 1];
        if (je - ja > WL_LONG) {  // the whole group takes this branch
            if (gl == 0) long_rows[atomicAdd(n_long, 1u)] = (uint32_t)row;
            continue;
        }
        uint32_t s = 0;
        for (uint64_t j = ja + gl; j < je; j += WL_GROUP) {
            uint64_t bb;
            s += b_row(b, __ldg(a.cols + j), bb);
        }
#pragma unroll
        for (int d = WL_GROUP / 2; d > 0; d >>= 1) s += __shfl_xor_sync(gmask, s, d);
        if (gl == 0) {
            work[row] = s;
            mine += s;
        }
    }
    if (mine) atomicAdd(&ptot, mine);
    __syncthreads();
    if (threadIdx.x == 0 && ptot) atomicAdd(total, ptot);
}

// The listed long rows, one CTA per row.
__global__ void __launch_bounds__(WL_NT) workload_long_kernel(AView a, BRows b, const uint32_t *__restrict__ long_rows,
                                                              const uint32_t *__restrict__ n_long,
                                                              uint32_t *__restrict__ work,
                                                              unsigned long long *__restrict__ total) {
    __shared__ uint32_t scratch[33];
    const uint32_t n = *n_long;
    for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
        const uint32_t row = long_rows[i];
        const uint64_t ja = a.rpt[row], je = a.rpt[row + 1];
        uint32_t s = 0;
#pragma unroll 4
        for (uint64_t j = ja + threadIdx.x; j < je; j += WL_NT) {
            uint64_t bb;
            s += b_row(b, __ldg(a.cols + j), bb);
        }
        s = block_sum<uint32_t, WL_NT>(s, scratch);
        if (threadIdx.x == 0) {
            work[row] = s;
            atomicAdd(total, (unsigned long long)s);
        }
    }
}

}  // namespace

int launch_workload(clb_controls *ctl, const AView &a, const BRows &b, uint32_t *work, uint64_t *d_total) {
    Temp<uint32_t> long_rows, n_long;
    CLB_RETURN_IF(n_long.alloc(ctl, 1));
    CLB_RETURN_IF(long_rows.alloc(ctl, a.nzr ? a.nzr : 1));
    CLB_TRY_CUDA(cudaMemsetAsync(n_long.ptr, 0, 4, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    unsigned grid = persistent_grid(ctl, 8, ceil_div_u(a.nzr, WL_NT / WL_GROUP));
    ProfScope ps(ctl, "workload");
    workload_kernel<<<grid, WL_NT, 0, ctl->stream>>>(a, b, work, (unsigned long long *)d_total, long_rows.ptr,
                                                     n_long.ptr);
    workload_long_kernel<<<ctl->sm_count * 4, WL_NT, 0, ctl->stream>>>(a, b, long_rows.ptr, n_long.ptr, work,
                                                                       (unsigned long long *)d_total);
    ctl->launches += 2;
    CLB_CHECK_LAUNCH();
    return CLB_SUCCESS;
}

namespace {

// flag[j] = 1 where entry j starts a word run: a new bitmap word (c >> 5)
// or, set by the next kernel, the first entry of a row.
__global__ void run_flags_kernel(const uint32_t *__restrict__ cols, uint64_t nnz, uint32_t *__restrict__ flag) {
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nnz; j += (uint64_t)gridDim.x * blockDim.x)
        flag[j] = (j == 0 || (__ldg(cols + j) >> 5) != (__ldg(cols + j - 1) >> 5)) ? 1u : 0u;
}

__global__ void row_start_flags_kernel(const uint64_t *__restrict__ rpt, uint64_t nzr, uint32_t *__restrict__ flag) {
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nzr; r += (uint64_t)gridDim.x * blockDim.x)
        if (rpt[r] < rpt[r + 1]) flag[rpt[r]] = 1u;
}

// pairs[p] = (word, OR of the run's bits) for run p.  pos = exclusive scan of
// the flags over nnz + 1 entries, so entry j is in run pos[j + 1] - 1.  The
// bits are OR-ed within each warp over the lanes of one run (consecutive, the
// rows being sorted), then one atomic per run and warp into zeroed pairs.
__global__ void run_pairs_kernel(const uint32_t *__restrict__ cols, uint64_t nnz, const uint32_t *__restrict__ pos,
                                 uint2 *__restrict__ pairs) {
    const uint32_t lane = lane_id();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t j0 = (uint64_t)blockIdx.x * blockDim.x; j0 < nnz; j0 += stride) {
        const uint64_t j = j0 + threadIdx.x;
        const bool valid = j < nnz;
        const uint32_t c = valid ? __ldg(cols + j) : 0u;
        const uint32_t run = valid ? pos[j + 1] - 1u : 0xFFFFFFFFu;
        const bool start = valid && pos[j + 1] != pos[j];
        uint32_t m = valid ? 1u << (c & 31) : 0u;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t om = __shfl_down_sync(0xFFFFFFFFu, m, d);
            const uint32_t orun = __shfl_down_sync(0xFFFFFFFFu, run, d);
            if (lane + d < 32 && orun == run) m |= om;
        }
        const uint32_t prev = __shfl_up_sync(0xFFFFFFFFu, run, 1);
        if (valid && (lane == 0 || prev != run)) {
            if (start) pairs[run].x = c >> 5;
            atomicOr(&pairs[run].y, m);
        }
    }
}

// wdense[k] = first run of B row k (B's dense row map `dense`, nrows + 1).
__global__ void run_rows_kernel(const uint64_t *__restrict__ dense, uint64_t nrows, uint64_t nnz,
                                const uint32_t *__restrict__ pos, uint64_t *__restrict__ wdense) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k <= nrows; k += (uint64_t)gridDim.x * blockDim.x)
        wdense[k] = pos[min(dense[k], nnz)];
}

}  // namespace

int prepare_b_words(clb_controls *ctl, const clb_dcsr &B, const uint32_t *hinfo, Temp<uint64_t> &wdense,
                    Temp<uint2> &wpairs, BRows &b, uint64_t products) {
    // the word form rides on the dense row map; it pays for its passes over B
    // only when bitmap rows multiply a large B whose entries are read several
    // times (a union's stacked operands are read once each: products = nnz(B))
    if (!b.dense || B.nzr == 0 || B.nnz < B_WORDS_MIN_NNZ) return CLB_SUCCESS;
    if (products && products < B_WORDS_MIN_REUSE * B.nnz) return CLB_SUCCESS;
    if (hinfo && hinfo[BIN_BMP_XL] + hinfo[BIN_BMP_L] + hinfo[BIN_BMP] == 0) return CLB_SUCCESS;
    const uint64_t nnz = B.nnz;
    // runs <= entries: the pairs are sized by the entries (no host read).
    // Without room for them the bitmap rows insert B's entries instead.
    Temp<uint32_t> pos;
    if (!pos.try_alloc(ctl, nnz + 1) || !wpairs.try_alloc(ctl, nnz) || !wdense.try_alloc(ctl, B.nrows + 1)) {
        wpairs.reset();
        wdense.reset();
        return CLB_SUCCESS;
    }
    ProfScope ps(ctl, "b_word_runs");
    const unsigned ge = persistent_grid(ctl, 8, ceil_div_u(nnz, 256));
    run_flags_kernel<<<ge, 256, 0, ctl->stream>>>(B.cols, nnz, pos.ptr);
    CLB_CHECK_LAUNCH();
    row_start_flags_kernel<<<persistent_grid(ctl, 8, ceil_div_u(B.nzr, 256)), 256, 0, ctl->stream>>>(B.rpt, B.nzr,
                                                                                                       pos.ptr);
    CLB_CHECK_LAUNCH();
    CLB_TRY_CUDA(cudaMemsetAsync(pos.ptr + nnz, 0, 4, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    CLB_RETURN_IF(scan_u32_inplace(ctl, pos.ptr, nnz + 1, nullptr));
    CLB_TRY_CUDA(cudaMemsetAsync(wpairs.ptr, 0, nnz * sizeof(uint2), ctl->stream), CLB_RUN_KERNEL_FAILURE);
    run_pairs_kernel<<<ge, 256, 0, ctl->stream>>>(B.cols, nnz, pos.ptr, wpairs.ptr);
    CLB_CHECK_LAUNCH();
    run_rows_kernel<<<persistent_grid(ctl, 8, ceil_div_u(B.nrows + 1, 256)), 256, 0, ctl->stream>>>(
        b.dense, B.nrows, nnz, pos.ptr, wdense.ptr);
    CLB_CHECK_LAUNCH();
    ctl->launches += 4;
    b.wdense = wdense.ptr;
    b.wpairs = wpairs.ptr;
    return CLB_SUCCESS;
}

int prepare_b(clb_controls *ctl, const clb_dcsr &B, Temp<uint64_t> &dense, BRows &b) {
    b.rpt = B.rpt;
    b.rows = B.rows;
    b.cols = B.cols;
    b.nzr = B.nzr;
    b.nrows = B.nrows;
    b.dense = nullptr;
    if (use_dense_map(B.nrows, B.nnz)) {
        CLB_RETURN_IF(dense.alloc(ctl, B.nrows + 1));
        CLB_RETURN_IF(dcsr_dense_rpt(ctl, &B, dense.ptr));
        b.dense = dense.ptr;
    }
    return CLB_SUCCESS;
}

int validate_spgemm(const clb_dcsr &A, const clb_dcsr &B) {
    if (A.ncols != B.nrows)
        return fail(CLB_INVALID_ARGUMENT, "Invalid input matrix size! a : " + std::to_string(A.nrows) + " x " +
                                              std::to_string(A.ncols) + ", b: " + std::to_string(B.nrows) + " x " +
                                              std::to_string(B.ncols));
    // 32-bit positions into B.cols, with room for one aligned 1024-entry window
    if (B.nnz > 0xFFFFF000ull || A.nzr >= (1ull << 32))
        return fail(CLB_NOT_SUPPORTED, "right operand with 2^32 - 4096 or more entries, or left with 2^32 stored rows");
    if (B.ncols > 0xFFFFFFFFull) return fail(CLB_NOT_SUPPORTED, "more than 2^32-1 columns");
    if ((A.nnz && (!A.rpt || !A.rows || !A.cols)) || (B.nnz && (!B.rpt || !B.rows || !B.cols)))
        return fail(CLB_INVALID_ARGUMENT, "matrix with entries but NULL arrays");
    return CLB_SUCCESS;
}

int spgemm_hash_two_pass(clb_controls *ctl, const clb_dcsr &A, const clb_dcsr &B, clb_dcsr *out,
                         clb_spgemm_stats *stats, const Tuning &t, bool keep) {
    clb_dcsr C{};
    C.nrows = A.nrows;
    C.ncols = B.ncols;
    clb_spgemm_stats st{};
    ctl->launches = 0;
    if (A.nnz == 0 || B.nnz == 0 || A.nzr == 0 || B.nzr == 0) {
        *out = C;
        if (stats) *stats = st;
        return CLB_SUCCESS;
    }
    CLB_RETURN_IF(clear_status(ctl));
    const AView a{A.rpt, A.rows, A.cols, A.nzr};
    BRows b;
    Temp<uint64_t> dense;
    CLB_RETURN_IF(prepare_b(ctl, B, dense, b));

    const uint64_t n = A.nzr;
    // scalars: [0] products, [1] nnz(C), [2] nzr(C)
    Temp<uint64_t> scal;
    CLB_RETURN_IF(scal.alloc(ctl, 4));
    CLB_TRY_CUDA(cudaMemsetAsync(scal.ptr, 0, 4 * sizeof(uint64_t), ctl->stream), CLB_RUN_KERNEL_FAILURE);
    Temp<uint32_t> work, row_nnz, flags, list, info;
    Temp<uint64_t> off;
    CLB_RETURN_IF(work.alloc(ctl, n));
    CLB_RETURN_IF(row_nnz.alloc(ctl, n));
    CLB_RETURN_IF(flags.alloc(ctl, n));
    CLB_RETURN_IF(list.alloc(ctl, n));
    CLB_RETURN_IF(info.alloc(ctl, 2 * NUM_BINS));
    CLB_RETURN_IF(off.alloc(ctl, n));

    CLB_RETURN_IF(launch_workload(ctl, a, b, work.ptr, scal.ptr + 0));
    CLB_RETURN_IF(launch_binning(ctl, work.ptr, nullptr, n, B.ncols, info.ptr, list.ptr, flags.ptr, t));
    CLB_TRY_CUDA(cudaMemsetAsync(row_nnz.ptr, 0, n * sizeof(uint32_t), ctl->stream), CLB_RUN_KERNEL_FAILURE);
    // rows per bin: only the bins with rows are launched, sized to them
    uint32_t hinfo[NUM_BINS];
    uint64_t products = 0;
    const SmallRead rd[2] = {{info.ptr, hinfo, sizeof(hinfo)}, {scal.ptr, &products, sizeof(products)}};
    CLB_RETURN_IF(read_small_multi(ctl, rd, 2));
    Temp<uint64_t> wdense;
    Temp<uint2> wpairs;
    CLB_RETURN_IF(prepare_b_words(ctl, B, hinfo, wdense, wpairs, b, products));

    BinLists bl{list.ptr, info.ptr};
    RowOut sym{row_nnz.ptr, nullptr, nullptr, nullptr, nullptr, ctl->d_status};
    sym.row_ncols = t.row_ncols;
    sym.row_products = work.ptr;
    // bitmaps kept from the symbolic pass for the numeric pass's expansion
    const uint64_t nbmp = (uint64_t)hinfo[BIN_BMP_XL] + hinfo[BIN_BMP_L] + hinfo[BIN_BMP];
    const uint32_t kw = bitmap_words(B.ncols);
    Temp<uint32_t> kbits, krec, klist, kcount;
    Temp<uint64_t> koff;
    // (batched rows of narrower pairs use the first words of their stride)
    keep = keep && nbmp && B.ncols <= (uint64_t)kw * 32 && kbits.try_alloc(ctl, nbmp * kw) &&
           krec.try_alloc(ctl, nbmp * BMP_STEP_REC) && klist.try_alloc(ctl, nbmp) && kcount.try_alloc(ctl, 1) &&
           koff.try_alloc(ctl, n);
    const uint32_t h_nbmp = (uint32_t)nbmp;  // (a pageable copy: staged before the call returns)
    if (keep) {
        CLB_TRY_CUDA(cudaMemcpyAsync(kcount.ptr, &h_nbmp, 4, cudaMemcpyHostToDevice, ctl->stream),
                     CLB_RUN_KERNEL_FAILURE);
        sym.keep = kbits.ptr;
        sym.keep_stride = kw;
        sym.keep_off = koff.ptr;
        sym.defer_steps = krec.ptr;
        sym.defer_list = klist.ptr;
    }
    CLB_RETURN_IF(launch_accumulators(ctl, false, bl, a, b, sym, B.ncols, n, t, hinfo));

    CLB_RETURN_IF(scan_u32_to_u64(ctl, row_nnz.ptr, off.ptr, n, scal.ptr + 1));
    CLB_RETURN_IF(scan_u32_inplace(ctl, flags.ptr, n, scal.ptr + 2));
    uint64_t h[3];
    CLB_RETURN_IF(read_scalars(ctl, scal.ptr, h, 3));
    st.products = h[0];
    const uint64_t nnz = h[1], nzr = h[2];
    st.nnz = nnz;
    st.nzr = nzr;
    for (int k = 0; k < NUM_BINS; ++k) st.rows_per_bin[k] = hinfo[k];
    if (nnz == 0) {
        CLB_RETURN_IF(check_status(ctl, "matrix_multiplication_hash"));
        st.kernel_launches = ctl->launches;
        *out = C;
        if (stats) *stats = st;
        return CLB_SUCCESS;
    }

    Temp<uint64_t> c_rpt;
    Temp<uint32_t> c_rows, c_cols;
    CLB_RETURN_IF(c_rpt.alloc(ctl, nzr + 1));
    CLB_RETURN_IF(c_rows.alloc(ctl, nzr));
    CLB_RETURN_IF(c_cols.alloc(ctl, nnz));
    CLB_RETURN_IF(launch_assemble(ctl, work.ptr, flags.ptr, off.ptr, A.rows, n, c_rpt.ptr, c_rows.ptr, nzr, nnz));

    RowOut num{nullptr, off.ptr, nullptr, nullptr, c_cols.ptr, ctl->d_status};
    num.row_ncols = t.row_ncols;
    num.row_products = work.ptr;
    if (keep) {
        CLB_RETURN_IF(launch_accumulators_subset(ctl, bl, a, b, num, B.ncols, n, true, t, hinfo, false));
        CLB_RETURN_IF(launch_bitmap_expand_steps(ctl, klist.ptr, kcount.ptr, krec.ptr, koff.ptr, kbits.ptr, off.ptr,
                                                 c_cols.ptr));
    } else {
        CLB_RETURN_IF(launch_accumulators(ctl, true, bl, a, b, num, B.ncols, n, t, hinfo));
    }
    CLB_RETURN_IF(check_status(ctl, "matrix_multiplication_hash"));

    C.nnz = nnz;
    C.nzr = nzr;
    C.rpt = c_rpt.release_ownership();
    C.rows = c_rows.release_ownership();
    C.cols = c_cols.release_ownership();
    *out = C;
    st.kernel_launches = ctl->launches;
    if (stats) *stats = st;
    return CLB_SUCCESS;
}

}  // namespace clb

using namespace clb;

extern "C" {

int clb_dcsr_spgemm_hash(clb_controls *ctl, const clb_dcsr *a, const clb_dcsr *b, clb_dcsr *c,
                         clb_spgemm_stats *stats) {
    if (!ctl || !a || !b || !c) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    const clb_dcsr A = *a, B = *b;
    CLB_RETURN_IF(validate_spgemm(A, B));
    DeviceGuard g(ctl);
    return spgemm_hash_two_pass(ctl, A, B, c, stats);
}

int clb_dcsr_workload(clb_controls *ctl, const clb_dcsr *a_, const clb_dcsr *b_, uint32_t *workload,
                      uint64_t *total) {
    if (!ctl || !a_ || !b_) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    const clb_dcsr A = *a_, B = *b_;
    CLB_RETURN_IF(validate_spgemm(A, B));
    DeviceGuard g(ctl);
    if (A.nzr == 0) {
        if (total) *total = 0;
        return CLB_SUCCESS;
    }
    if (!workload) return fail(CLB_INVALID_ARGUMENT, "workload is NULL");
    if (B.nnz == 0) {
        CLB_TRY_CUDA(cudaMemsetAsync(workload, 0, A.nzr * 4, ctl->stream), CLB_RUN_KERNEL_FAILURE);
        CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
        if (total) *total = 0;
        return CLB_SUCCESS;
    }
    const AView a{A.rpt, A.rows, A.cols, A.nzr};
    BRows b;
    Temp<uint64_t> dense, tot;
    CLB_RETURN_IF(prepare_b(ctl, B, dense, b));
    CLB_RETURN_IF(tot.alloc(ctl, 1));
    CLB_TRY_CUDA(cudaMemsetAsync(tot.ptr, 0, 8, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    CLB_RETURN_IF(launch_workload(ctl, a, b, workload, tot.ptr));
    uint64_t h = 0;
    CLB_RETURN_IF(read_scalars(ctl, tot.ptr, &h, 1));
    if (total) *total = h;
    return CLB_SUCCESS;
}

}  // extern "C"
