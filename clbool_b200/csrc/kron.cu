// kron.cu -- dcsr::kronecker_product and dcsr::transpose.
//
// Reference: dcsr::kronecker_product (src/dcsr/dcsr_kronecker_product.cpp:5-64,
// kernels dcsr_kronecker.cl:38-97: per-row nnz, prefix sum, then one upper-bound
// search per output entry) and dcsr::transpose
// (src/dcsr/dcsr_transpose.cpp:5-16: DCSR -> COO -> swap -> sort -> DCSR).
//
// Kronecker here needs no scan and no per-entry search: C's row k = (ia, ib)
// starts at A.rpt[ia] * nnz(B) + len(A_ia) * B.rpt[ib] (all earlier rows of A
// contribute whole copies of B).  A warp takes 32 consecutive rows, writes
// their row pointers and indices and the columns of the short ones (a lane
// per row); the longer rows are listed and written a warp per row, so that
// consecutive lanes write consecutive columns.
#include "common.cuh"

namespace clb {

int sort_pairs(clb_controls *ctl, uint32_t *rows, uint32_t *cols, uint64_t n);

namespace {

constexpr int KR_NT = 256;
constexpr uint32_t KR_SMALL = 32;  // rows of at most this many entries are written by one lane
constexpr uint32_t KR_MED = 1024;  // rows of at most this many entries are written in their batch
constexpr uint32_t KR_CHUNK = 4096;  // longer rows are listed in chunks of at most this many entries

// (q / l, q % l) for q < 2^8 and 1 <= l < 2^8 without an integer divide:
// (q + 1/2) / l lies at least 1/(2l) >= 1/510 from every integer, far above
// the error of __fdividef (2 ulp of a quotient below 2^9: under 1.3e-4), so
// its floor is q / l.
__device__ __forceinline__ void kron_small_divmod(uint32_t q, uint32_t l, uint32_t &d, uint32_t &r) {
    d = (uint32_t)__fdividef((float)q + 0.5f, (float)l);
    r = q - d * l;
}

// A's entries ar[0, la) times B's row br[0, lb) (la, lb >= 1: a C row, or a
// chunk of one, which is a contiguous block of it) written by the whole warp.  B rows of at most 128 entries are
// held in registers (four per lane) and each A entry's copy is written by
// one step; longer B rows are looped over per A entry; B rows shorter than
// 32 entries are flattened: lane l writes entries l, l + 32, ... and moves
// (ja, jb) on by (32 / lb, 32 % lb) and one carry per pass.  Every A and B
// load is of an entry the row uses.
__device__ __forceinline__ void kron_row_warp(const uint32_t *__restrict__ ar, const uint32_t *__restrict__ br,
                                              uint32_t la, uint32_t lb, uint32_t *__restrict__ dst, uint32_t bncols,
                                              uint32_t lane) {
    if (lb > 128) {
        uint32_t *d = dst;
        for (uint32_t ja = 0; ja < la; ++ja, d += lb) {
            const uint32_t av = __ldg(ar + ja) * bncols;
            for (uint32_t jb = lane; jb < lb; jb += 32) d[jb] = av + __ldg(br + jb);
        }
    } else if (lb >= 32) {
        uint32_t bv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) bv[u] = lane + 32u * u < lb ? __ldg(br + lane + 32u * u) : 0u;
        uint32_t *d = dst;
        for (uint32_t ja = 0; ja < la; ++ja, d += lb) {
            const uint32_t av = __ldg(ar + ja) * bncols;
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (lane + 32u * u < lb) d[lane + 32u * u] = av + bv[u];
        }
    } else {
        const uint64_t n = (uint64_t)la * lb;
        uint32_t D, R, ja, jb;
        kron_small_divmod(32u, lb, D, R);
        kron_small_divmod(lane, lb, ja, jb);
        uint32_t *d = dst + lane;
        for (uint64_t q = lane; q < n; q += 32, d += 32) {
            *d = __ldg(ar + ja) * bncols + __ldg(br + jb);
            jb += R;
            ja += D;
            if (jb >= lb) {
                jb -= lb;
                ++ja;
            }
        }
    }
}

// C's rows by batches of 32 consecutive rows k = ia * bnzr + ib, a warp per
// batch with a grid stride ((ia, ib) of the batch's first row move on by
// dq, dr = stride / bnzr, stride % bnzr without dividing).  Lane l takes row
// k0 + l: it loads its row pointers (consecutive rows: coalesced), writes
// C's row pointer (closed form: A.rpt[ia] * nnz(B) + len(A_ia) * B.rpt[ib],
// all earlier rows of A contribute whole copies of B) and row index, and
// writes the row's columns itself when it has at most KR_SMALL of them
// (entry q = ja * lb + jb is acol(ja) * bncols + bcol(jb), 32 bits since C
// has fewer than 2^32 columns).  Rows of at most KR_MED entries are then
// written by the whole warp one after another (kron_row_warp, pointers
// shuffled from their lanes); longer rows are appended as (ia, ib) to `big`
// (one atomic per warp) for kron_big_rows_kernel, so no warp is held by a
// batch of heavy rows.
__global__ void __launch_bounds__(KR_NT) kron_batch_kernel(
    const uint64_t *__restrict__ arpt, const uint32_t *__restrict__ arows, const uint32_t *__restrict__ acols,
    uint64_t anzr, const uint64_t *__restrict__ brpt, const uint32_t *__restrict__ brows,
    const uint32_t *__restrict__ bcols, uint64_t bnzr, uint64_t bnnz, uint64_t bnrows, uint32_t bncols, uint64_t dq,
    uint64_t dr, uint64_t *__restrict__ crpt, uint32_t *__restrict__ crows, uint32_t *__restrict__ ccols,
    uint4 *__restrict__ big, uint32_t *__restrict__ nbig) {
    const uint64_t nzr = anzr * bnzr, nb = (nzr + 31) >> 5;
    const uint32_t lane = lane_id();
    const uint64_t nwarps = (uint64_t)gridDim.x * (KR_NT / 32);
    if (blockIdx.x == 0 && threadIdx.x == 0) crpt[nzr] = arpt[anzr] * bnnz;
    uint64_t w = (uint64_t)blockIdx.x * (KR_NT / 32) + warp_id();
    if (w >= nb) return;
    uint64_t ia0 = (w << 5) / bnzr, ib0 = (w << 5) - ia0 * bnzr;
    for (; w < nb; w += nwarps) {
        const uint64_t k = (w << 5) + lane;
        uint64_t ia = ia0, ib = ib0 + lane;
        while (ib >= bnzr) {  // at most 32 / bnzr steps
            ib -= bnzr;
            ++ia;
        }
        uint64_t a0 = 0, b0 = 0;
        uint32_t la = 0, lb = 0;
        if (k < nzr) {
            a0 = __ldg(arpt + ia);
            la = (uint32_t)(__ldg(arpt + ia + 1) - a0);
            b0 = __ldg(brpt + ib);
            lb = (uint32_t)(__ldg(brpt + ib + 1) - b0);
            crpt[k] = a0 * bnnz + (uint64_t)la * b0;
            crows[k] = (uint32_t)((uint64_t)__ldg(arows + ia) * bnrows + __ldg(brows + ib));
        }
        const uint64_t n = (uint64_t)la * lb;  // 0 past the last row
        if (n && n <= KR_SMALL) {
            const uint32_t *const ar = acols + a0, *const br = bcols + b0;
            uint32_t *const d = ccols + a0 * bnnz + (uint64_t)la * b0;
            uint32_t ja = 0, jb = 0, av = __ldg(ar) * bncols;
            for (uint32_t t = 0; t < (uint32_t)n; ++t) {
                d[t] = av + __ldg(br + jb);
                if (++jb == lb) {
                    jb = 0;
                    if (++ja < la) av = __ldg(ar + ja) * bncols;
                }
            }
        }
        // medium rows: the whole warp, one after another, pointers from their lanes
        for (uint32_t med = __ballot_sync(0xFFFFFFFFu, n > KR_SMALL && n <= KR_MED); med; med &= med - 1) {
            const int r = __ffs(med) - 1;
            const uint32_t rla = __shfl_sync(0xFFFFFFFFu, la, r), rlb = __shfl_sync(0xFFFFFFFFu, lb, r);
            const uint64_t ra0 = __shfl_sync(0xFFFFFFFFu, (unsigned long long)a0, r);
            const uint64_t rb0 = __shfl_sync(0xFFFFFFFFu, (unsigned long long)b0, r);
            kron_row_warp(acols + ra0, bcols + rb0, rla, rlb, ccols + ra0 * bnnz + (uint64_t)rla * rb0, bncols, lane);
        }
        // long rows: listed in chunks of JA consecutive A entries (JA * lb
        // <= KR_CHUNK entries, or one A entry's copy of a longer B row)
        if (__any_sync(0xFFFFFFFFu, n > KR_MED)) {
            uint32_t JA = 0, nch = 0;
            if (n > KR_MED) {
                JA = lb < KR_CHUNK ? KR_CHUNK / lb : 1u;
                nch = (la + JA - 1) / JA;
            }
            const uint32_t inc = warp_inclusive_scan(nch), tot = __shfl_sync(0xFFFFFFFFu, inc, 31);
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(nbig, tot);
            base = __shfl_sync(0xFFFFFFFFu, base, 0) + inc - nch;
            for (uint32_t c = 0; c < nch; ++c)
                big[base + c] = make_uint4((uint32_t)ia, (uint32_t)ib, c * JA, min(la, (c + 1) * JA));
        }
        ia0 += dq;
        ib0 += dr;
        if (ib0 >= bnzr) {
            ib0 -= bnzr;
            ++ia0;
        }
    }
}

// The chunks of the rows of more than KR_MED entries listed by
// kron_batch_kernel ({ia, ib, first and end A entry}), a warp per chunk
// (kron_row_warp: a chunk is a contiguous block of its C row) with a grid
// stride; the next chunk's pointers are loaded before the current one is
// written.
__global__ void __launch_bounds__(KR_NT) kron_big_rows_kernel(const uint64_t *__restrict__ arpt,
                                                              const uint32_t *__restrict__ acols,
                                                              const uint64_t *__restrict__ brpt,
                                                              const uint32_t *__restrict__ bcols, uint64_t bnnz,
                                                              uint32_t bncols, const uint4 *__restrict__ big,
                                                              const uint32_t *__restrict__ nbig,
                                                              uint32_t *__restrict__ ccols) {
    const uint32_t cnt = *nbig;
    const uint32_t lane = lane_id();
    const uint32_t nwarps = gridDim.x * (KR_NT / 32);
    uint32_t j = blockIdx.x * (KR_NT / 32) + warp_id();
    if (j >= cnt) return;
    uint4 e = big[j];
    uint64_t a0 = __ldg(arpt + e.x), a1 = __ldg(arpt + e.x + 1), b0 = __ldg(brpt + e.y), b1 = __ldg(brpt + e.y + 1);
    while (j < cnt) {
        const uint32_t jn = j + nwarps;
        uint4 en = make_uint4(0, 0, 0, 0);
        uint64_t na0 = 0, na1 = 0, nb0 = 0, nb1 = 0;
        if (jn < cnt) {
            en = big[jn];
            na0 = __ldg(arpt + en.x);
            na1 = __ldg(arpt + en.x + 1);
            nb0 = __ldg(brpt + en.y);
            nb1 = __ldg(brpt + en.y + 1);
        }
        const uint32_t la = (uint32_t)(a1 - a0), lb = (uint32_t)(b1 - b0);
        kron_row_warp(acols + a0 + e.z, bcols + b0, e.w - e.z, lb,
                      ccols + a0 * bnnz + (uint64_t)la * b0 + (uint64_t)e.z * lb, bncols, lane);
        j = jn;
        e = en;
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
    // rows of more than KR_MED entries: at most nnz / (KR_MED + 1) of them,
    // each in at most 2 n / KR_CHUNK + 1 chunks
    const uint64_t nbig_cap = std::min<uint64_t>(nzr, nnz / (KR_MED + 1)) + 2 * nnz / KR_CHUNK;
    if (nbig_cap >= (1ull << 32)) return fail(CLB_NOT_SUPPORTED, "Kronecker product with 2^32 or more long-row chunks");
    Temp<uint4> big;
    Temp<uint32_t> nbig;
    CLB_RETURN_IF(big.alloc(ctl, nbig_cap ? nbig_cap : 1));
    CLB_RETURN_IF(nbig.alloc(ctl, 1));
    CLB_TRY_CUDA(cudaMemsetAsync(nbig.ptr, 0, sizeof(uint32_t), ctl->stream), CLB_RUN_KERNEL_FAILURE);
    // 8 blocks per SM, more than it holds at once (6 and 5): the blocks of
    // the second wave take up uneven warps' slack (0.75 ms against 0.78 ms
    // with the resident count at s11 x s11)
    const uint64_t nbatch = (nzr + 31) / 32, cap = (uint64_t)ctl->sm_count * 8;
    const uint64_t g1 = (nbatch + KR_NT / 32 - 1) / (KR_NT / 32);
    const unsigned grid1 = (unsigned)(g1 > cap ? cap : g1);
    const uint64_t stride = (uint64_t)grid1 * (KR_NT / 32) * 32;  // rows per grid pass
    kron_batch_kernel<<<grid1, KR_NT, 0, ctl->stream>>>(a.rpt, a.rows, a.cols, a.nzr, b.rpt, b.rows, b.cols, b.nzr,
                                                         b.nnz, b.nrows, (uint32_t)b.ncols, stride / b.nzr,
                                                         stride % b.nzr, rpt.ptr, rows.ptr, cols.ptr, big.ptr,
                                                         nbig.ptr);
    CLB_CHECK_LAUNCH();
    if (nbig_cap) {
        const uint64_t g2 = (nbig_cap + KR_NT / 32 - 1) / (KR_NT / 32);
        const unsigned grid2 = (unsigned)(g2 > cap ? cap : g2);
        kron_big_rows_kernel<<<grid2, KR_NT, 0, ctl->stream>>>(a.rpt, a.cols, b.rpt, b.cols, b.nnz,
                                                                (uint32_t)b.ncols, big.ptr, nbig.ptr, cols.ptr);
        CLB_CHECK_LAUNCH();
    }
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
