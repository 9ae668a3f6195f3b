// kron.cu -- dcsr::kronecker_product and dcsr::transpose.
//
// Reference: dcsr::kronecker_product (src/dcsr/dcsr_kronecker_product.cpp:5-64,
// kernels dcsr_kronecker.cl:38-97: per-row nnz, prefix sum, then one upper-bound
// search per output entry) and dcsr::transpose
// (src/dcsr/dcsr_transpose.cpp:5-16: DCSR -> COO -> swap -> sort -> DCSR).
//
// Kronecker here needs no scan and no per-entry search: C's row k = (ia, ib)
// starts at A.rpt[ia] * nnz(B) + len(A_ia) * B.rpt[ib] (all earlier rows of A
// contribute whole copies of B), and one warp writes row k, looping over
// (ja, jb) so that consecutive lanes write consecutive columns.
#include "common.cuh"

namespace clb {

int sort_pairs(clb_controls *ctl, uint32_t *rows, uint32_t *cols, uint64_t n);

namespace {

__global__ void kron_rows_kernel(const uint64_t *__restrict__ arpt, const uint32_t *__restrict__ arows, uint64_t anzr,
                                 const uint64_t *__restrict__ brpt, const uint32_t *__restrict__ brows, uint64_t bnzr,
                                 uint64_t bnnz, uint64_t bnrows, uint64_t *__restrict__ crpt,
                                 uint32_t *__restrict__ crows) {
    const uint64_t nzr = anzr * bnzr;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nzr; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t ia = k / bnzr, ib = k - ia * bnzr;
        const uint64_t la = arpt[ia + 1] - arpt[ia];
        crpt[k] = arpt[ia] * bnnz + la * brpt[ib];
        crows[k] = (uint32_t)((uint64_t)arows[ia] * bnrows + brows[ib]);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) crpt[nzr] = arpt[anzr] * bnnz;
}

constexpr int KR_NT = 256;

// One warp per C row, rows taken with a grid stride: (ia, ib) advance by the
// stride without dividing (dq, dr = stride / bnzr, stride % bnzr), and the
// next row's pointers are loaded before the current row is written, so the
// row-pointer latency overlaps the stores.  Rows whose B row has at most 128
// entries keep it in registers (four per lane) and write one A entry's copy
// per step; longer B rows loop over it; B rows shorter than 32 entries are
// flattened over (ja, jb) so all lanes write.
__global__ void __launch_bounds__(KR_NT) kron_cols_kernel(const uint64_t *__restrict__ arpt,
                                                          const uint32_t *__restrict__ acols, uint64_t anzr,
                                                          const uint64_t *__restrict__ brpt,
                                                          const uint32_t *__restrict__ bcols, uint64_t bnzr,
                                                          uint64_t bnnz, uint64_t bncols, uint64_t dq, uint64_t dr,
                                                          uint32_t *__restrict__ ccols) {
    const uint64_t nzr = anzr * bnzr;
    const uint32_t lane = lane_id();
    const uint64_t nwarps = (uint64_t)gridDim.x * (KR_NT / 32);
    uint64_t k = (uint64_t)blockIdx.x * (KR_NT / 32) + warp_id();
    if (k >= nzr) return;
    uint64_t ia = k / bnzr, ib = k - ia * bnzr;
    uint64_t a0 = arpt[ia], a1 = arpt[ia + 1], b0 = brpt[ib], b1 = brpt[ib + 1];
    while (k < nzr) {
        // the next row's pointers, in flight while this row is written
        const uint64_t kn = k + nwarps;
        uint64_t ian = ia + dq, ibn = ib + dr;
        if (ibn >= bnzr) {
            ibn -= bnzr;
            ++ian;
        }
        uint64_t na0 = 0, na1 = 0, nb0 = 0, nb1 = 0;
        if (kn < nzr) {
            na0 = __ldg(arpt + ian);
            na1 = __ldg(arpt + ian + 1);
            nb0 = __ldg(brpt + ibn);
            nb1 = __ldg(brpt + ibn + 1);
        }
        const uint64_t la = a1 - a0, lb = b1 - b0;
        uint32_t *dst = ccols + a0 * bnnz + la * b0;  // C's row pointer, closed form
        if (lb > 128) {
            for (uint64_t ja = 0; ja < la; ++ja) {
                const uint64_t base = (uint64_t)__ldg(acols + a0 + ja) * bncols;
                for (uint64_t jb = lane; jb < lb; jb += 32)
                    dst[ja * lb + jb] = (uint32_t)(base + __ldg(bcols + b0 + jb));
            }
        } else if (lb >= 32) {
            uint32_t bv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) bv[u] = lane + 32u * u < lb ? __ldg(bcols + b0 + lane + 32u * u) : 0u;
            for (uint64_t ja = 0; ja < la; ++ja) {
                const uint64_t base = (uint64_t)__ldg(acols + a0 + ja) * bncols;
                uint32_t *d = dst + ja * lb;
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (lane + 32u * u < lb) d[lane + 32u * u] = (uint32_t)(base + bv[u]);
            }
        } else if (lb) {
            const uint64_t n = la * lb;
            const uint32_t l = (uint32_t)lb, da = 32u / l, db = 32u % l;
            uint32_t ja = lane / l, jb = lane % l;
            for (uint64_t q = lane; q < n; q += 32) {
                dst[q] = (uint32_t)((uint64_t)__ldg(acols + a0 + ja) * bncols + __ldg(bcols + b0 + jb));
                ja += da;
                jb += db;
                if (jb >= l) {
                    jb -= l;
                    ++ja;
                }
            }
        }
        k = kn;
        ia = ian;
        ib = ibn;
        a0 = na0;
        a1 = na1;
        b0 = nb0;
        b1 = nb1;
    }
}

__global__ void expand_rows_kernel2(const uint64_t *__restrict__ rpt, const uint32_t *__restrict__ rows, uint64_t nzr,
                                    uint64_t nnz, uint32_t *__restrict__ out) {
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nnz; j += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t p = upper_bound_dev<uint64_t, uint64_t>(rpt, nzr + 1, j) - 1;
        out[j] = rows[p];
    }
}

unsigned grid_for(const clb_controls *ctl, uint64_t n, int nt = 256) {
    uint64_t g = (n + nt - 1) / nt, cap = (uint64_t)ctl->sm_count * 16;
    return (unsigned)(g > cap ? cap : (g ? g : 1));
}

}  // namespace

}  // namespace clb

using namespace clb;

extern "C" CLB_API int clb_coo_to_dcsr(clb_controls *ctl, const clb_coo *in, clb_dcsr *out, int deep);

extern "C" {

int clb_dcsr_kronecker(clb_controls *ctl, const clb_dcsr *a_, const clb_dcsr *b_, clb_dcsr *out) {
    if (!ctl || !a_ || !b_ || !out) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    const clb_dcsr a = *a_, b = *b_;
    DeviceGuard g(ctl);
    clb_dcsr c{};
    c.nrows = a.nrows * b.nrows;
    c.ncols = a.ncols * b.ncols;
    const uint64_t nnz = a.nnz * b.nnz, nzr = a.nzr * b.nzr;
    if (nnz == 0) {
        *out = c;
        return CLB_SUCCESS;
    }
    if (c.nrows > (1ull << 32) || c.ncols > 0xFFFFFFFFull)
        return fail(CLB_NOT_SUPPORTED, "Kronecker product with row or column indices past 2^32");
    ProfScope ps(ctl, "kronecker");
    Temp<uint64_t> rpt;
    Temp<uint32_t> rows, cols;
    CLB_RETURN_IF(rpt.alloc(ctl, nzr + 1));
    CLB_RETURN_IF(rows.alloc(ctl, nzr));
    CLB_RETURN_IF(cols.alloc(ctl, nnz));
    kron_rows_kernel<<<grid_for(ctl, nzr), 256, 0, ctl->stream>>>(a.rpt, a.rows, a.nzr, b.rpt, b.rows, b.nzr, b.nnz,
                                                                  b.nrows, rpt.ptr, rows.ptr);
    CLB_CHECK_LAUNCH();
    uint64_t warps = nzr, g2 = (warps + KR_NT / 32 - 1) / (KR_NT / 32), cap = (uint64_t)ctl->sm_count * 8;
    const unsigned grid2 = (unsigned)(g2 > cap ? cap : g2);
    const uint64_t stride = (uint64_t)grid2 * (KR_NT / 32);
    kron_cols_kernel<<<grid2, KR_NT, 0, ctl->stream>>>(a.rpt, a.cols, a.nzr, b.rpt, b.cols, b.nzr, b.nnz, b.ncols,
                                                        stride / b.nzr, stride % b.nzr, cols.ptr);
    CLB_CHECK_LAUNCH();
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    c.nnz = nnz;
    c.nzr = nzr;
    c.rpt = rpt.release_ownership();
    c.rows = rows.release_ownership();
    c.cols = cols.release_ownership();
    *out = c;
    return CLB_SUCCESS;
}

int clb_dcsr_transpose(clb_controls *ctl, const clb_dcsr *in_, clb_dcsr *out) {
    if (!ctl || !in_ || !out) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    const clb_dcsr in = *in_;
    DeviceGuard g(ctl);
    clb_dcsr c{};
    c.nrows = in.ncols;
    c.ncols = in.nrows;
    if (in.nnz == 0) {
        *out = c;
        return CLB_SUCCESS;
    }
    ProfScope ps(ctl, "transpose");
    // new rows = old cols, new cols = old rows (expanded)
    Temp<uint32_t> r, cc;
    CLB_RETURN_IF(r.alloc(ctl, in.nnz));
    CLB_RETURN_IF(cc.alloc(ctl, in.nnz));
    CLB_TRY_CUDA(cudaMemcpyAsync(r.ptr, in.cols, in.nnz * 4, cudaMemcpyDeviceToDevice, ctl->stream),
                 CLB_COPY_BUFFER_ERROR);
    expand_rows_kernel2<<<grid_for(ctl, in.nnz), 256, 0, ctl->stream>>>(in.rpt, in.rows, in.nzr, in.nnz, cc.ptr);
    CLB_CHECK_LAUNCH();
    CLB_RETURN_IF(sort_pairs(ctl, r.ptr, cc.ptr, in.nnz));
    clb_coo coo{c.nrows, c.ncols, in.nnz, r.ptr, cc.ptr};
    clb_dcsr d{};
    CLB_RETURN_IF(clb_coo_to_dcsr(ctl, &coo, &d, 0));
    // d.cols aliases cc: keep it, drop the row array of the COO.
    cc.release_ownership();
    *out = d;
    return CLB_SUCCESS;
}

}  // extern "C"
