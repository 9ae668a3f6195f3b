// submatrix.cu -- dcsr::submatrix and dcsr::reduce.
//
// Reference: dcsr::submatrix (src/dcsr/dcsr_submatrix.cpp:98-155, kernels
// submatrix.cl: rows_range, submatrix_count_nnz, submatrix_fill_nnz; CPU form
// src/common/cpu_matrix_operations.cpp:6-52): rows [i, i+nrows) and columns
// [j, j+ncols) of A, re-indexed to start at 0, empty rows dropped.
// dcsr::reduce (src/dcsr/dcsr_reduce.cpp:5-31, reduce.cl:10-20): the row-wise
// OR, one entry at column 0 per stored row.
//
// Same steps as the reference (row range by binary search over the stored
// rows, per-row column range by two binary searches, scans, copy), with
// 64-bit offsets and without host syncs between the counting and the scans.
#include "common.cuh"

namespace clb {

namespace {

// [0] = first stored row >= lo, [1] = first stored row >= hi (keys may pass 2^32)
__global__ void row_range_kernel(const uint32_t *__restrict__ rows, uint64_t nzr, uint64_t lo, uint64_t hi,
                                 uint64_t *__restrict__ out) {
    if (threadIdx.x < 2) {
        const uint64_t key = threadIdx.x == 0 ? lo : hi;
        out[threadIdx.x] = key > 0xFFFFFFFFull ? nzr : lower_bound_dev<uint32_t, uint64_t>(rows, nzr, (uint32_t)key);
    }
}

__device__ __forceinline__ uint64_t col_bound(const uint32_t *cols, uint64_t n, uint64_t key) {
    return key > 0xFFFFFFFFull ? n : lower_bound_dev<uint32_t, uint64_t>(cols, n, (uint32_t)key);
}

// Column range of every row in the row range: beg[k], cnt[k], flags[k].
__global__ void sub_count_kernel(const uint64_t *__restrict__ rpt, const uint64_t *__restrict__ range,
                                 const uint32_t *__restrict__ cols, uint64_t n, uint64_t j0, uint64_t j1,
                                 uint64_t *__restrict__ beg, uint32_t *__restrict__ cnt, uint32_t *__restrict__ flags) {
    const uint64_t r0 = range[0];
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t s = rpt[r0 + k], e = rpt[r0 + k + 1];
        const uint64_t b = s + col_bound(cols + s, e - s, j0), f = s + col_bound(cols + s, e - s, j1);
        beg[k] = b;
        cnt[k] = (uint32_t)(f - b);
        flags[k] = f > b ? 1u : 0u;
    }
}

// One warp per row of the range: columns minus j, and the row's entry in
// rpt / rows (at its position among the non-empty rows).
__global__ void sub_fill_kernel(const uint64_t *__restrict__ range, const uint32_t *__restrict__ rows,
                                const uint32_t *__restrict__ cols, const uint64_t *__restrict__ beg,
                                const uint32_t *__restrict__ cnt, const uint64_t *__restrict__ off,
                                const uint32_t *__restrict__ pos, uint64_t n, uint32_t i, uint32_t j,
                                uint64_t nzr, uint64_t nnz, uint64_t *__restrict__ out_rpt,
                                uint32_t *__restrict__ out_rows, uint32_t *__restrict__ out_cols) {
    const uint64_t r0 = range[0];
    const uint32_t lane = lane_id();
    const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x / 32);
    for (uint64_t k = (uint64_t)blockIdx.x * (blockDim.x / 32) + warp_id(); k < n; k += nw) {
        const uint32_t c = cnt[k];
        if (!c) continue;
        const uint64_t b = beg[k], o = off[k];
        for (uint32_t t = lane; t < c; t += 32) out_cols[o + t] = cols[b + t] - j;
        if (lane == 0) {
            out_rpt[pos[k]] = o;
            out_rows[pos[k]] = rows[r0 + k] - i;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out_rpt[nzr] = nnz;
}

__global__ void reduce_kernel(uint64_t nzr, uint64_t *__restrict__ rpt, uint32_t *__restrict__ cols) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k <= nzr; k += (uint64_t)gridDim.x * blockDim.x) {
        rpt[k] = k;
        if (k < nzr) cols[k] = 0;
    }
}

unsigned grid_for(const clb_controls *ctl, uint64_t n, int nt = 256) {
    uint64_t g = (n + nt - 1) / nt, cap = (uint64_t)ctl->sm_count * 16;
    return (unsigned)(g > cap ? cap : (g ? g : 1));
}

}  // namespace

}  // namespace clb

using namespace clb;

extern "C" {

int clb_dcsr_submatrix(clb_controls *ctl, const clb_dcsr *in_, uint64_t i, uint64_t j, uint64_t nrows, uint64_t ncols,
                       clb_dcsr *out) {
    if (!ctl || !in_ || !out) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    const clb_dcsr A = *in_;
    if (i > 0xFFFFFFFFull || j > 0xFFFFFFFFull) return fail(CLB_INVALID_VALUE, "i and j are 32-bit indices");
    if (A.nnz && (!A.rpt || !A.rows || !A.cols)) return fail(CLB_INVALID_ARGUMENT, "matrix with entries but NULL arrays");
    DeviceGuard g(ctl);
    clb_dcsr C{};
    C.nrows = nrows;
    C.ncols = ncols;
    *out = C;
    if (A.nnz == 0 || A.nzr == 0 || nrows == 0 || ncols == 0) return CLB_SUCCESS;
    ProfScope ps(ctl, "submatrix");
    // scalars: [0..1] stored-row range, [2] nnz, [3] nzr
    Temp<uint64_t> sc;
    CLB_RETURN_IF(sc.alloc(ctl, 4));
    row_range_kernel<<<1, 32, 0, ctl->stream>>>(A.rows, A.nzr, i, i + nrows, sc.ptr);
    CLB_CHECK_LAUNCH();
    uint64_t h[2];
    CLB_RETURN_IF(read_scalars(ctl, sc.ptr, h, 2));
    const uint64_t n = h[1] > h[0] ? h[1] - h[0] : 0;
    if (n == 0) return CLB_SUCCESS;
    Temp<uint64_t> beg, off;
    Temp<uint32_t> cnt, pos;
    CLB_RETURN_IF(beg.alloc(ctl, n));
    CLB_RETURN_IF(off.alloc(ctl, n));
    CLB_RETURN_IF(cnt.alloc(ctl, n));
    CLB_RETURN_IF(pos.alloc(ctl, n));
    sub_count_kernel<<<grid_for(ctl, n), 256, 0, ctl->stream>>>(A.rpt, sc.ptr, A.cols, n, j, j + ncols, beg.ptr,
                                                                cnt.ptr, pos.ptr);
    CLB_CHECK_LAUNCH();
    CLB_RETURN_IF(scan_u32_to_u64(ctl, cnt.ptr, off.ptr, n, sc.ptr + 2));
    CLB_RETURN_IF(scan_u32_inplace(ctl, pos.ptr, n, sc.ptr + 3));
    CLB_RETURN_IF(read_scalars(ctl, sc.ptr + 2, h, 2));
    const uint64_t nnz = h[0], nzr = h[1];
    if (nnz == 0) return CLB_SUCCESS;
    Temp<uint64_t> rpt;
    Temp<uint32_t> rows, cols;
    CLB_RETURN_IF(rpt.alloc(ctl, nzr + 1));
    CLB_RETURN_IF(rows.alloc(ctl, nzr));
    CLB_RETURN_IF(cols.alloc(ctl, nnz));
    sub_fill_kernel<<<grid_for(ctl, n * 32), 256, 0, ctl->stream>>>(sc.ptr, A.rows, A.cols, beg.ptr, cnt.ptr, off.ptr,
                                                                     pos.ptr, n, (uint32_t)i, (uint32_t)j, nzr, nnz,
                                                                     rpt.ptr, rows.ptr, cols.ptr);
    CLB_CHECK_LAUNCH();
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    C.nnz = nnz;
    C.nzr = nzr;
    C.rpt = rpt.release_ownership();
    C.rows = rows.release_ownership();
    C.cols = cols.release_ownership();
    *out = C;
    return CLB_SUCCESS;
}

int clb_dcsr_reduce(clb_controls *ctl, const clb_dcsr *in_, clb_dcsr *out) {
    if (!ctl || !in_ || !out) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    const clb_dcsr A = *in_;
    if (A.nnz && (!A.rpt || !A.rows || !A.cols)) return fail(CLB_INVALID_ARGUMENT, "matrix with entries but NULL arrays");
    DeviceGuard g(ctl);
    clb_dcsr C{};
    C.nrows = A.nrows;
    C.ncols = 1;
    if (A.nnz == 0 || A.nzr == 0) {
        *out = C;
        return CLB_SUCCESS;
    }
    ProfScope ps(ctl, "reduce");
    Temp<uint64_t> rpt;
    Temp<uint32_t> rows, cols;
    CLB_RETURN_IF(rpt.alloc(ctl, A.nzr + 1));
    CLB_RETURN_IF(rows.alloc(ctl, A.nzr));
    CLB_RETURN_IF(cols.alloc(ctl, A.nzr));
    CLB_TRY_CUDA(cudaMemcpyAsync(rows.ptr, A.rows, A.nzr * 4, cudaMemcpyDeviceToDevice, ctl->stream),
                 CLB_COPY_BUFFER_ERROR);
    reduce_kernel<<<grid_for(ctl, A.nzr + 1), 256, 0, ctl->stream>>>(A.nzr, rpt.ptr, cols.ptr);
    CLB_CHECK_LAUNCH();
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    C.nnz = C.nzr = A.nzr;
    C.rpt = rpt.release_ownership();
    C.rows = rows.release_ownership();
    C.cols = cols.release_ownership();
    *out = C;
    return CLB_SUCCESS;
}

}  // extern "C"
