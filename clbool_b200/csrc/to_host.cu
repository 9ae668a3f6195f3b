// to_host.cu -- C = A*B delivered into host memory, the device-to-host copy
// of each row block of C overlapped with the product of the next block.
//
// No counterpart in the reference, where the product stays in device
// buffers until matrix_dcsr_from_gpu copies it out after the call
// (src/common/matrices_conversions.cpp:121-140).  For a large C the copy over
// PCIe outlasts the product (scale-20 R-MAT A*A: 38.9 GB of columns against
// ~90 ms of kernels), so the product runs in row blocks of A balanced by
// products: block j+1 is multiplied while block j travels on a second
// stream.  Each block is an ordinary call of the chosen form, so the result
// is the same C.
#include <algorithm>
#include <string>
#include <vector>

#include "spgemm.cuh"

namespace clb {

namespace {

// rpt of stored rows [r0, r0 + n] of A, rebased to start at 0.
__global__ void rebase_rpt_kernel(const uint64_t *__restrict__ rpt, uint64_t r0, uint64_t n,
                                  uint64_t *__restrict__ out) {
    const uint64_t base = rpt[r0];
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = rpt[r0 + i] - base;
}

// rpt[i] += add for i < n: a block's row starts inside the whole C.
__global__ void shift_rpt_kernel(uint64_t *__restrict__ rpt, uint64_t n, uint64_t add) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        rpt[i] += add;
}

unsigned grid_of(const clb_controls *ctl, uint64_t n) {
    const uint64_t g = (n + 255) / 256, cap = (uint64_t)ctl->sm_count * 8;
    return (unsigned)std::max<uint64_t>(1, std::min(g, cap));
}

// Owns the copy stream, its events and the blocks' C until the copies end.
struct Pipeline {
    clb_controls *ctl;
    cudaStream_t copy = nullptr;
    std::vector<cudaEvent_t> events;
    std::vector<clb_dcsr> parts;
    explicit Pipeline(clb_controls *c) : ctl(c) {}
    ~Pipeline() {
        if (copy) cudaStreamSynchronize(copy);
        for (auto &p : parts) clb_dcsr_release(ctl, &p);
        for (auto e : events) cudaEventDestroy(e);
        if (copy) cudaStreamDestroy(copy);
    }
};

void add_stats(clb_spgemm_stats &t, const clb_spgemm_stats &s) {
    t.products += s.products;
    t.nnz += s.nnz;
    t.nzr += s.nzr;
    t.capacity += s.capacity;
    t.fallback_rows += s.fallback_rows;
    t.spilled_rows += s.spilled_rows;
    t.kernel_launches += s.kernel_launches;
    for (int k = 0; k < NUM_BINS; ++k) t.rows_per_bin[k] += s.rows_per_bin[k];
}

}  // namespace

}  // namespace clb

using namespace clb;

extern "C" {

int clb_dcsr_row_block(clb_controls *ctl, const clb_dcsr *a_, uint64_t lo, uint64_t hi, clb_dcsr *out) {
    if (!ctl || !a_ || !out) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    const clb_dcsr A = *a_;
    if (lo > hi || hi > A.nzr) return fail(CLB_INVALID_ARGUMENT, "row range [" + std::to_string(lo) + ", " +
                                                                   std::to_string(hi) + ") outside the stored rows");
    clb_dcsr C{};
    C.nrows = A.nrows;
    C.ncols = A.ncols;
    if (hi == lo || A.nnz == 0) {
        *out = C;
        return CLB_SUCCESS;
    }
    DeviceGuard g(ctl);
    uint64_t j[2];
    CLB_TRY_CUDA(cudaMemcpyAsync(&j[0], A.rpt + lo, 8, cudaMemcpyDeviceToHost, ctl->stream), CLB_READ_BUFFER_ERROR);
    CLB_TRY_CUDA(cudaMemcpyAsync(&j[1], A.rpt + hi, 8, cudaMemcpyDeviceToHost, ctl->stream), CLB_READ_BUFFER_ERROR);
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    if (j[1] == j[0]) {
        *out = C;
        return CLB_SUCCESS;
    }
    const uint64_t n = hi - lo, nnz = j[1] - j[0];
    Temp<uint64_t> rpt;
    Temp<uint32_t> rows, cols;
    CLB_RETURN_IF(rpt.alloc(ctl, n + 1));
    CLB_RETURN_IF(rows.alloc(ctl, n));
    CLB_RETURN_IF(cols.alloc(ctl, nnz));
    rebase_rpt_kernel<<<grid_of(ctl, n + 1), 256, 0, ctl->stream>>>(A.rpt, lo, n, rpt.ptr);
    CLB_CHECK_LAUNCH();
    CLB_TRY_CUDA(cudaMemcpyAsync(rows.ptr, A.rows + lo, n * 4, cudaMemcpyDeviceToDevice, ctl->stream),
                 CLB_COPY_BUFFER_ERROR);
    CLB_TRY_CUDA(cudaMemcpyAsync(cols.ptr, A.cols + j[0], nnz * 4, cudaMemcpyDeviceToDevice, ctl->stream),
                 CLB_COPY_BUFFER_ERROR);
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    C.nnz = nnz;
    C.nzr = n;
    C.rpt = rpt.release_ownership();
    C.rows = rows.release_ownership();
    C.cols = cols.release_ownership();
    *out = C;
    return CLB_SUCCESS;
}

int clb_dcsr_spgemm_to_host(clb_controls *ctl, const clb_dcsr *a_, const clb_dcsr *b_, const clb_sizer *sizer,
                            float margin_log2, float slack, const clb_spgemm_tuning *tuning, uint32_t blocks,
                            uint64_t *h_rpt, uint32_t *h_rows, uint32_t *h_cols, uint64_t rows_capacity,
                            uint64_t cols_capacity, uint64_t *nzr_out, uint64_t *nnz_out, clb_spgemm_stats *stats) {
    if (!ctl || !a_ || !b_ || !h_rpt || !nzr_out || !nnz_out) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    if ((rows_capacity && !h_rows) || (cols_capacity && !h_cols)) return fail(CLB_INVALID_ARGUMENT, "NULL host array");
    CLB_RETURN_IF(check_tuning(tuning));
    const clb_dcsr A = *a_, B = *b_;
    CLB_RETURN_IF(validate_spgemm(A, B));
    DeviceGuard g(ctl);
    clb_spgemm_stats total{};
    *nzr_out = *nnz_out = 0;
    h_rpt[0] = 0;
    if (stats) *stats = total;
    if (A.nnz == 0 || B.nnz == 0 || A.nzr == 0 || B.nzr == 0) return CLB_SUCCESS;
    blocks = std::max<uint32_t>(1, std::min<uint32_t>(blocks, 64));
    const uint64_t n = A.nzr;

    // row blocks with about equal products (workload pass, read back once)
    std::vector<uint64_t> cut(1, 0);
    {
        const AView av{A.rpt, A.rows, A.cols, A.nzr};
        BRows bv;
        Temp<uint64_t> dense, tot;
        Temp<uint32_t> work;
        CLB_RETURN_IF(prepare_b(ctl, B, dense, bv));
        CLB_RETURN_IF(work.alloc(ctl, n));
        CLB_RETURN_IF(tot.alloc(ctl, 1));
        CLB_TRY_CUDA(cudaMemsetAsync(tot.ptr, 0, 8, ctl->stream), CLB_RUN_KERNEL_FAILURE);
        CLB_RETURN_IF(launch_workload(ctl, av, bv, work.ptr, tot.ptr));
        std::vector<uint32_t> hw(n);
        CLB_TRY_CUDA(cudaMemcpyAsync(hw.data(), work.ptr, n * 4, cudaMemcpyDeviceToHost, ctl->stream),
                     CLB_READ_BUFFER_ERROR);
        CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
        uint64_t sum = 0;
        for (uint32_t w : hw) sum += w;
        uint64_t run = 0;
        for (uint64_t i = 0; i < n && cut.size() < blocks; ++i) {
            run += hw[i];
            if (run * blocks >= sum * cut.size() && i + 1 < n) cut.push_back(i + 1);
        }
        cut.push_back(n);
    }
    std::vector<uint64_t> rpt_at(cut.size());
    for (size_t k = 0; k < cut.size(); ++k)
        CLB_TRY_CUDA(cudaMemcpyAsync(&rpt_at[k], A.rpt + cut[k], 8, cudaMemcpyDeviceToHost, ctl->stream),
                     CLB_READ_BUFFER_ERROR);
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);

    Pipeline pl(ctl);
    CLB_TRY_CUDA(cudaStreamCreateWithFlags(&pl.copy, cudaStreamNonBlocking), CLB_RUN_KERNEL_FAILURE);
    uint64_t nzr = 0, nnz = 0;
    for (size_t k = 0; k + 1 < cut.size(); ++k) {
        const uint64_t r0 = cut[k], r1 = cut[k + 1];
        if (r1 <= r0) continue;
        Temp<uint64_t> brpt;
        CLB_RETURN_IF(brpt.alloc(ctl, r1 - r0 + 1));
        rebase_rpt_kernel<<<grid_of(ctl, r1 - r0 + 1), 256, 0, ctl->stream>>>(A.rpt, r0, r1 - r0, brpt.ptr);
        CLB_CHECK_LAUNCH();
        const clb_dcsr Ab{A.nrows, A.ncols, rpt_at[k + 1] - rpt_at[k], r1 - r0, brpt.ptr, A.rows + r0,
                          A.cols + rpt_at[k]};
        clb_dcsr Cb{};
        clb_spgemm_stats s{};
        const int rc = sizer ? clb_dcsr_spgemm_learned(ctl, &Ab, &B, sizer, margin_log2, slack, tuning, &Cb, &s)
                             : clb_dcsr_spgemm_tuned(ctl, &Ab, &B, tuning, &Cb, &s);
        if (rc != CLB_SUCCESS) return rc;
        pl.parts.push_back(Cb);
        add_stats(total, s);
        if (Cb.nnz == 0) continue;
        if (nzr + Cb.nzr > rows_capacity || nnz + Cb.nnz > cols_capacity)
            return fail(CLB_INVALID_VALUE, "host arrays too small: C has more than " + std::to_string(rows_capacity) +
                                               " rows or " + std::to_string(cols_capacity) + " columns");
        // the block's rows start at nnz inside C; then hand it to the copy stream
        shift_rpt_kernel<<<grid_of(ctl, Cb.nzr), 256, 0, ctl->stream>>>(Cb.rpt, Cb.nzr, nnz);
        CLB_CHECK_LAUNCH();
        cudaEvent_t ev;
        CLB_TRY_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), CLB_RUN_KERNEL_FAILURE);
        pl.events.push_back(ev);
        CLB_TRY_CUDA(cudaEventRecord(ev, ctl->stream), CLB_RUN_KERNEL_FAILURE);
        CLB_TRY_CUDA(cudaStreamWaitEvent(pl.copy, ev, 0), CLB_RUN_KERNEL_FAILURE);
        CLB_TRY_CUDA(cudaMemcpyAsync(h_rpt + nzr, Cb.rpt, Cb.nzr * 8, cudaMemcpyDeviceToHost, pl.copy),
                     CLB_READ_BUFFER_ERROR);
        CLB_TRY_CUDA(cudaMemcpyAsync(h_rows + nzr, Cb.rows, Cb.nzr * 4, cudaMemcpyDeviceToHost, pl.copy),
                     CLB_READ_BUFFER_ERROR);
        CLB_TRY_CUDA(cudaMemcpyAsync(h_cols + nnz, Cb.cols, Cb.nnz * 4, cudaMemcpyDeviceToHost, pl.copy),
                     CLB_READ_BUFFER_ERROR);
        nzr += Cb.nzr;
        nnz += Cb.nnz;
    }
    CLB_TRY_CUDA(cudaStreamSynchronize(pl.copy), CLB_EVENT_WAITING_ERROR);
    h_rpt[nzr] = nnz;
    *nzr_out = nzr;
    *nnz_out = nnz;
    total.nzr = nzr;
    total.nnz = nnz;
    if (stats) *stats = total;
    return CLB_SUCCESS;
}

}  // extern "C"
