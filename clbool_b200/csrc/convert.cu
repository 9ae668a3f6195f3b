// convert.cu -- COO <-> DCSR <-> CSR conversions and fill_with.
//
// Reference: src/common/matrices_conversions.cpp:7-91 (COO<->DCSR),
// :211-271 (CSR<->DCSR), kernels prepare_positions.cl:29-84,
// set_positions.cl:46-113, conversions.cl:8-18, dscr_to_coo.cl:8-23.
// Same outputs; different mechanics: the dense CSR row pointer is built by
// one binary search per dense row (no scatter + scan), and DCSR->COO row
// expansion is one upper-bound search per entry (balanced for any row
// length distribution).
#include "common.cuh"

namespace clb {

namespace {

constexpr int NT = 256;

// out[r] = offset of the first stored row >= r, for r in [0, nrows].  Stored
// rows with an index >= nrows (out of the matrix) fall outside every dense
// row, so they are never looked up -- as the reference's exact row search
// (count_workload.cl:8-27) never matches them.
__global__ void dense_rpt_kernel(const uint64_t *__restrict__ rpt, const uint32_t *__restrict__ rows, uint64_t nzr,
                                 uint64_t nrows, uint64_t *__restrict__ out) {
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= nrows;
         r += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t p = r <= 0xFFFFFFFFull ? lower_bound_dev<uint32_t, uint64_t>(rows, nzr, (uint32_t)r) : nzr;
        out[r] = rpt[p];
    }
}

// flags[i] = 1 where a COO row starts (prepare_array_for_rows_positions).
__global__ void row_start_flags_kernel(const uint32_t *__restrict__ rows, uint64_t n, uint32_t *__restrict__ flags) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        flags[i] = (i == 0 || rows[i] != rows[i - 1]) ? 1u : 0u;
}

// Scatter DCSR rpt/rows at the row starts (set_positions_rows).
__global__ void coo_rows_scatter_kernel(const uint32_t *__restrict__ rows, const uint32_t *__restrict__ pos,
                                        uint64_t n, uint64_t *__restrict__ rpt, uint32_t *__restrict__ out_rows) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        bool start = (i == 0 || rows[i] != rows[i - 1]);
        if (start) {
            uint32_t p = pos[i];
            rpt[p] = i;
            out_rows[p] = rows[i];
        }
        // pos is the exclusive scan of the start flags: nzr = pos[n-1] + flag[n-1].
        if (i == n - 1) rpt[(uint64_t)pos[i] + (start ? 1 : 0)] = n;
    }
}

// rows_out[j] = row of entry j (dscr_to_coo).
__global__ void expand_rows_kernel(const uint64_t *__restrict__ rpt, const uint32_t *__restrict__ rows, uint64_t nzr,
                                   uint64_t nnz, uint32_t *__restrict__ out) {
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nnz; j += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t p = upper_bound_dev<uint64_t, uint64_t>(rpt, nzr + 1, j) - 1;
        out[j] = rows[p];
    }
}

// flags[i] = 1 for non-empty CSR rows (prepare_for_shift_empty_rows).
__global__ void nonempty_flags_kernel(const uint64_t *__restrict__ rpt, uint64_t nrows, uint32_t *__restrict__ flags) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nrows; i += (uint64_t)gridDim.x * blockDim.x)
        flags[i] = rpt[i + 1] > rpt[i] ? 1u : 0u;
}

// set_positions_pointers_and_rows_csr.
__global__ void csr_rows_scatter_kernel(const uint64_t *__restrict__ csr_rpt, const uint32_t *__restrict__ pos,
                                        uint64_t nrows, uint64_t *__restrict__ rpt, uint32_t *__restrict__ rows) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nrows; i += (uint64_t)gridDim.x * blockDim.x) {
        if (csr_rpt[i + 1] > csr_rpt[i]) {
            rpt[pos[i]] = csr_rpt[i];
            rows[pos[i]] = (uint32_t)i;
        }
    }
}

__global__ void set_last_kernel(uint64_t *__restrict__ rpt, const uint64_t *__restrict__ d_nzr, uint64_t value) {
    rpt[*d_nzr] = value;
}

__global__ void fill_u32_kernel(uint32_t *__restrict__ a, uint64_t n, uint32_t v) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        a[i] = v;
}

unsigned grid_for(const clb_controls *ctl, uint64_t n) {
    uint64_t g = (n + NT - 1) / NT;
    uint64_t cap = (uint64_t)ctl->sm_count * 16;
    if (g > cap) g = cap;
    return (unsigned)(g ? g : 1);
}

}  // namespace

int dcsr_dense_rpt(clb_controls *ctl, const clb_dcsr *m, uint64_t *out) {
    ProfScope ps(ctl, "dense_row_map");
    dense_rpt_kernel<<<grid_for(ctl, m->nrows + 1), NT, 0, ctl->stream>>>(m->rpt, m->rows, m->nzr, m->nrows, out);
    ctl->launches += 1;
    CLB_CHECK_LAUNCH();
    return CLB_SUCCESS;
}

}  // namespace clb

using namespace clb;

extern "C" {

int clb_fill_u32(clb_controls *ctl, uint32_t *array, uint64_t n, uint32_t value) {
    if (!ctl || (n && !array)) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    if (n == 0) return CLB_SUCCESS;
    DeviceGuard g(ctl);
    fill_u32_kernel<<<grid_for(ctl, n), NT, 0, ctl->stream>>>(array, n, value);
    CLB_CHECK_LAUNCH();
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    return CLB_SUCCESS;
}

int clb_coo_to_dcsr(clb_controls *ctl, const clb_coo *in_, clb_dcsr *out, int deep) {
    if (!ctl || !in_ || !out) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    clb_coo in = *in_;
    DeviceGuard g(ctl);
    clb_dcsr r{};
    r.nrows = in.nrows;
    r.ncols = in.ncols;
    if (in.nnz == 0) {
        *out = r;
        return CLB_SUCCESS;
    }
    if (in.nnz >= (1ull << 32)) return fail(CLB_NOT_SUPPORTED, "COO with 2^32 or more entries");
    Temp<uint32_t> pos;
    CLB_RETURN_IF(pos.alloc(ctl, in.nnz));
    row_start_flags_kernel<<<grid_for(ctl, in.nnz), NT, 0, ctl->stream>>>(in.rows, in.nnz, pos.ptr);
    CLB_CHECK_LAUNCH();
    Temp<uint64_t> tot;
    CLB_RETURN_IF(tot.alloc(ctl, 1));
    CLB_RETURN_IF(scan_u32_inplace(ctl, pos.ptr, in.nnz, tot.ptr));
    uint64_t nzr = 0;
    CLB_RETURN_IF(read_scalars(ctl, tot.ptr, &nzr, 1));
    Temp<uint64_t> rpt;
    Temp<uint32_t> rows, cols;
    CLB_RETURN_IF(rpt.alloc(ctl, nzr + 1));
    CLB_RETURN_IF(rows.alloc(ctl, nzr));
    coo_rows_scatter_kernel<<<grid_for(ctl, in.nnz), NT, 0, ctl->stream>>>(in.rows, pos.ptr, in.nnz, rpt.ptr, rows.ptr);
    CLB_CHECK_LAUNCH();
    if (deep) {
        CLB_RETURN_IF(cols.alloc(ctl, in.nnz));
        CLB_TRY_CUDA(cudaMemcpyAsync(cols.ptr, in.cols, in.nnz * 4, cudaMemcpyDeviceToDevice, ctl->stream),
                     CLB_COPY_BUFFER_ERROR);
    }
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    r.nnz = in.nnz;
    r.nzr = nzr;
    r.rpt = rpt.release_ownership();
    r.rows = rows.release_ownership();
    r.cols = deep ? cols.release_ownership() : in.cols;
    *out = r;
    return CLB_SUCCESS;
}

int clb_dcsr_to_coo(clb_controls *ctl, const clb_dcsr *in_, clb_coo *out, int deep) {
    if (!ctl || !in_ || !out) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    clb_dcsr in = *in_;
    DeviceGuard g(ctl);
    clb_coo r{};
    r.nrows = in.nrows;
    r.ncols = in.ncols;
    if (in.nnz == 0) {
        *out = r;
        return CLB_SUCCESS;
    }
    Temp<uint32_t> rows, cols;
    CLB_RETURN_IF(rows.alloc(ctl, in.nnz));
    expand_rows_kernel<<<grid_for(ctl, in.nnz), NT, 0, ctl->stream>>>(in.rpt, in.rows, in.nzr, in.nnz, rows.ptr);
    CLB_CHECK_LAUNCH();
    if (deep) {
        CLB_RETURN_IF(cols.alloc(ctl, in.nnz));
        CLB_TRY_CUDA(cudaMemcpyAsync(cols.ptr, in.cols, in.nnz * 4, cudaMemcpyDeviceToDevice, ctl->stream),
                     CLB_COPY_BUFFER_ERROR);
    }
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    r.nnz = in.nnz;
    r.rows = rows.release_ownership();
    r.cols = deep ? cols.release_ownership() : in.cols;
    *out = r;
    return CLB_SUCCESS;
}

int clb_dcsr_to_csr(clb_controls *ctl, const clb_dcsr *in_, clb_csr *out) {
    if (!ctl || !in_ || !out) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    clb_dcsr in = *in_;
    DeviceGuard g(ctl);
    clb_csr r{};
    r.nrows = in.nrows;
    r.ncols = in.ncols;
    if (in.nnz == 0) {
        *out = r;
        return CLB_SUCCESS;
    }
    Temp<uint64_t> rpt;
    CLB_RETURN_IF(rpt.alloc(ctl, in.nrows + 1));
    CLB_RETURN_IF(dcsr_dense_rpt(ctl, &in, rpt.ptr));
    // The reference checks that the CSR keeps every entry
    // (matrices_conversions.cpp:268): rows stored past nrows do not fit.
    uint64_t last = 0;
    CLB_RETURN_IF(read_scalars(ctl, rpt.ptr + in.nrows, &last, 1));
    if (last != in.nnz) return fail(CLB_INVALID_VALUE, "nnz in dcsr and csr matrices should be equal!");
    r.nnz = in.nnz;
    r.rpt = rpt.release_ownership();
    r.cols = in.cols;
    *out = r;
    return CLB_SUCCESS;
}

int clb_csr_to_dcsr(clb_controls *ctl, const clb_csr *in_, clb_dcsr *out) {
    if (!ctl || !in_ || !out) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    clb_csr in = *in_;
    DeviceGuard g(ctl);
    clb_dcsr r{};
    r.nrows = in.nrows;
    r.ncols = in.ncols;
    if (in.nnz == 0 || in.nrows == 0) {
        *out = r;
        return CLB_SUCCESS;
    }
    Temp<uint32_t> pos;
    CLB_RETURN_IF(pos.alloc(ctl, in.nrows));
    nonempty_flags_kernel<<<grid_for(ctl, in.nrows), NT, 0, ctl->stream>>>(in.rpt, in.nrows, pos.ptr);
    CLB_CHECK_LAUNCH();
    Temp<uint64_t> tot;
    CLB_RETURN_IF(tot.alloc(ctl, 1));
    CLB_RETURN_IF(scan_u32_inplace(ctl, pos.ptr, in.nrows, tot.ptr));
    uint64_t nzr = 0;
    CLB_RETURN_IF(read_scalars(ctl, tot.ptr, &nzr, 1));
    Temp<uint64_t> rpt;
    Temp<uint32_t> rows;
    CLB_RETURN_IF(rpt.alloc(ctl, nzr + 1));
    CLB_RETURN_IF(rows.alloc(ctl, nzr ? nzr : 1));
    csr_rows_scatter_kernel<<<grid_for(ctl, in.nrows), NT, 0, ctl->stream>>>(in.rpt, pos.ptr, in.nrows, rpt.ptr,
                                                                            rows.ptr);
    CLB_CHECK_LAUNCH();
    set_last_kernel<<<1, 1, 0, ctl->stream>>>(rpt.ptr, tot.ptr, in.nnz);
    CLB_CHECK_LAUNCH();
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    r.nnz = in.nnz;
    r.nzr = nzr;
    r.rpt = rpt.release_ownership();
    r.rows = rows.release_ownership();
    r.cols = in.cols;
    *out = r;
    return CLB_SUCCESS;
}

}  // extern "C"
