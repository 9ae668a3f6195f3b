// add.cu -- coo::matrix_addition and csr::matrix_addition (boolean: union).
//
// Reference: coo::matrix_addition (src/coo/coo_matrix_addition.cpp:32-73:
// merge-path merge of (row, col) pairs, merge_path.cl:182-261, then
// reduce_duplicates2), csr::matrix_addition (src/csr/csr_addition.cpp:26-168:
// row bins, per-row symbolic merge, scan, per-row numeric merge,
// csr_addition.cl).
//
// Both are one balanced merge path over (row, col) keys here:
//   split   : one thread per 2048-output tile boundary finds how many A
//             entries precede the boundary (A first on ties);
//   count   : every tile stages its A and B keys in shared memory, merges
//             eight outputs per thread, drops an output equal to its
//             predecessor (the B copy of a shared entry), and reduces;
//   write   : same merge, written at the scanned tile offset.
// COO keys use the explicit row arrays.  CSR rows are implicit: a tile split
// first binary-searches the combined row pointer A.rpt[r] + B.rpt[r] (the
// merged start of row r), then splits inside the row; in the tile each
// entry's row comes from a search of the row pointer over the tile's row
// range.  C's CSR row pointer is lenA + lenB - (duplicates of the row),
// counted with one atomic per duplicate, then scanned.
#include "common.cuh"

namespace clb {

namespace {

constexpr int MP_NT = 256;
constexpr int MP_ITEMS = 8;
constexpr uint64_t MP_TILE = (uint64_t)MP_NT * MP_ITEMS;

struct CooSide {
    const uint32_t *rows;
    const uint32_t *cols;
    uint64_t n;
};

struct CsrSide {
    const uint64_t *rpt;
    const uint32_t *cols;
    uint64_t n;
};

__device__ __forceinline__ uint64_t coo_key(const CooSide &s, uint64_t i) {
    return ((uint64_t)__ldg(s.rows + i) << 32) | (uint64_t)__ldg(s.cols + i);
}

// Row of entry i of a CSR side, searching rows [lo, hi] (i is in one of them).
__device__ __forceinline__ uint64_t csr_row_of(const CsrSide &s, uint64_t i, uint64_t lo, uint64_t hi) {
    // largest r in [lo, hi] with rpt[r] <= i
    while (lo < hi) {
        uint64_t m = lo + (hi - lo + 1) / 2;
        if (__ldg(s.rpt + m) <= i) lo = m; else hi = m - 1;
    }
    return lo;
}

__device__ __forceinline__ uint64_t csr_key(const CsrSide &s, uint64_t i, uint64_t lo, uint64_t hi) {
    return (csr_row_of(s, i, lo, hi) << 32) | (uint64_t)__ldg(s.cols + i);
}

// ------------------------------------------------------------------ splits --
__global__ void coo_split_kernel(CooSide A, CooSide B, uint64_t ntiles, uint64_t *__restrict__ split_a) {
    const uint64_t total = A.n + B.n;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t <= ntiles; t += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t d = t * MP_TILE;
        if (d > total) d = total;
        uint64_t lo = d > B.n ? d - B.n : 0, hi = d < A.n ? d : A.n;
        while (lo < hi) {
            uint64_t m = lo + (hi - lo) / 2;
            if (coo_key(A, m) <= coo_key(B, d - 1 - m)) lo = m + 1; else hi = m;
        }
        split_a[t] = lo;
    }
}

__global__ void csr_split_kernel(CsrSide A, CsrSide B, uint64_t nrows, uint64_t ntiles, uint64_t *__restrict__ split_a,
                                 uint64_t *__restrict__ split_row) {
    const uint64_t total = A.n + B.n;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t <= ntiles; t += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t d = t * MP_TILE;
        if (d >= total) {
            split_a[t] = A.n;
            split_row[t] = nrows ? nrows - 1 : 0;
            continue;
        }
        // largest r in [0, nrows-1] with A.rpt[r] + B.rpt[r] <= d
        uint64_t lo = 0, hi = nrows - 1;
        while (lo < hi) {
            uint64_t m = lo + (hi - lo + 1) / 2;
            if (__ldg(A.rpt + m) + __ldg(B.rpt + m) <= d) lo = m; else hi = m - 1;
        }
        const uint64_t r = lo;
        const uint64_t ar = __ldg(A.rpt + r), br = __ldg(B.rpt + r);
        const uint64_t la = __ldg(A.rpt + r + 1) - ar, lb = __ldg(B.rpt + r + 1) - br;
        const uint64_t dl = d - ar - br;
        uint64_t i0 = dl > lb ? dl - lb : 0, i1 = dl < la ? dl : la;
        while (i0 < i1) {
            uint64_t m = i0 + (i1 - i0) / 2;
            if (__ldg(A.cols + ar + m) <= __ldg(B.cols + br + dl - 1 - m)) i0 = m + 1; else i1 = m;
        }
        split_a[t] = ar + i0;
        split_row[t] = r;
    }
}

// -------------------------------------------------------------- tile merge --
// MODE 0: count (tile totals; CSR: per-row duplicate counts); MODE 1: write.
template <bool CSR, int MODE>
__global__ void __launch_bounds__(MP_NT) merge_tile_kernel(CooSide Ac, CooSide Bc, CsrSide As, CsrSide Bs,
                                                           uint64_t nrows, const uint64_t *__restrict__ split_a,
                                                           const uint64_t *__restrict__ split_row,
                                                           uint32_t *__restrict__ tile_cnt,
                                                           const uint64_t *__restrict__ tile_off,
                                                           uint32_t *__restrict__ row_dup, uint32_t *__restrict__ out_rows,
                                                           uint32_t *__restrict__ out_cols) {
    __shared__ uint64_t s[MP_TILE];
    __shared__ uint32_t scratch[33];
    const uint64_t na = CSR ? As.n : Ac.n, nb = CSR ? Bs.n : Bc.n;
    const uint64_t total = na + nb;
    const uint64_t t = blockIdx.x;
    const uint64_t d0 = t * MP_TILE;
    const uint64_t d1 = min(d0 + MP_TILE, total);
    const uint64_t a0 = split_a[t], a1 = split_a[t + 1];
    const uint64_t b0 = d0 - a0, b1 = d1 - a1;
    const uint32_t nta = (uint32_t)(a1 - a0), ntb = (uint32_t)(b1 - b0);
    uint64_t rlo = 0, rhi = 0;
    if (CSR) {
        rlo = split_row[t];
        rhi = split_row[t + 1];
    }
    for (uint32_t k = threadIdx.x; k < nta; k += MP_NT)
        s[k] = CSR ? csr_key(As, a0 + k, rlo, rhi) : coo_key(Ac, a0 + k);
    for (uint32_t k = threadIdx.x; k < ntb; k += MP_NT)
        s[nta + k] = CSR ? csr_key(Bs, b0 + k, rlo, rhi) : coo_key(Bc, b0 + k);
    __syncthreads();

    const uint32_t nt = nta + ntb;
    const uint32_t dl = threadIdx.x * MP_ITEMS;
    uint32_t ia = 0, ib = 0;
    bool has_prev = false;
    uint64_t prev = 0;
    if (dl < nt) {
        uint32_t lo = dl > ntb ? dl - ntb : 0, hi = dl < nta ? dl : nta;
        while (lo < hi) {
            uint32_t m = (lo + hi) >> 1;
            if (s[m] <= s[nta + dl - 1 - m]) lo = m + 1; else hi = m;
        }
        ia = lo;
        ib = dl - lo;
        if (dl > 0) {
            has_prev = true;
            uint64_t pa = ia > 0 ? s[ia - 1] : 0, pb = ib > 0 ? s[nta + ib - 1] : 0;
            prev = pa > pb ? pa : pb;
        } else if (d0 > 0) {
            // predecessor of the tile: the larger of the last A and B entries consumed
            has_prev = true;
            uint64_t pa = 0, pb = 0;
            if (a0 > 0) pa = CSR ? csr_key(As, a0 - 1, 0, rlo) : coo_key(Ac, a0 - 1);
            if (b0 > 0) pb = CSR ? csr_key(Bs, b0 - 1, 0, rlo) : coo_key(Bc, b0 - 1);
            prev = pa > pb ? pa : pb;
        }
    }
    uint64_t keys[MP_ITEMS];
    uint32_t flags = 0, cnt = 0;
#pragma unroll
    for (int k = 0; k < MP_ITEMS; ++k) {
        keys[k] = 0;
        if (dl + k < nt) {
            bool takeA = ib >= ntb || (ia < nta && s[ia] <= s[nta + ib]);
            uint64_t key = takeA ? s[ia++] : s[nta + ib++];
            bool uniq = !has_prev || key != prev;
            if (MODE == 0 && CSR && !uniq) atomicAdd(row_dup + (key >> 32), 1u);
            prev = key;
            has_prev = true;
            keys[k] = key;
            flags |= (uniq ? 1u : 0u) << k;
            cnt += uniq ? 1u : 0u;
        }
    }
    if (MODE == 0) {
        uint32_t tot = block_sum<uint32_t, MP_NT>(cnt, scratch);
        if (threadIdx.x == 0) tile_cnt[t] = tot;
        return;
    }
    uint32_t tot;
    uint32_t off = block_exclusive_scan<uint32_t, MP_NT>(cnt, scratch, &tot);
    uint64_t p = tile_off[t] + off;
#pragma unroll
    for (int k = 0; k < MP_ITEMS; ++k) {
        if (flags & (1u << k)) {
            if (!CSR) out_rows[p] = (uint32_t)(keys[k] >> 32);
            out_cols[p] = (uint32_t)keys[k];
            ++p;
        }
    }
}

// c_cnt[r] = lenA + lenB - dup[r]  (scanned afterwards into C's rpt).
__global__ void csr_row_counts_kernel(const uint64_t *__restrict__ arpt, const uint64_t *__restrict__ brpt,
                                      const uint32_t *__restrict__ dup, uint64_t nrows, uint64_t *__restrict__ out) {
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += (uint64_t)gridDim.x * blockDim.x)
        out[r] = (arpt[r + 1] - arpt[r]) + (brpt[r + 1] - brpt[r]) - dup[r];
}

unsigned grid_for(const clb_controls *ctl, uint64_t n) {
    uint64_t g = (n + 255) / 256, cap = (uint64_t)ctl->sm_count * 16;
    return (unsigned)(g > cap ? cap : (g ? g : 1));
}

int shape_check(uint64_t ar, uint64_t ac, uint64_t br, uint64_t bc) {
    if (ar != br || ac != bc)
        return fail(CLB_INVALID_ARGUMENT, "Invalid matrixes size! a: " + std::to_string(ar) + " x " + std::to_string(ac) +
                                              ", b: " + std::to_string(br) + " x " + std::to_string(bc));
    return CLB_SUCCESS;
}

int copy_u32(clb_controls *ctl, const uint32_t *src, uint64_t n, uint32_t **dst) {
    Temp<uint32_t> t;
    CLB_RETURN_IF(t.alloc(ctl, n));
    if (n) CLB_TRY_CUDA(cudaMemcpyAsync(t.ptr, src, n * 4, cudaMemcpyDeviceToDevice, ctl->stream), CLB_COPY_BUFFER_ERROR);
    *dst = t.release_ownership();
    return CLB_SUCCESS;
}

}  // namespace

}  // namespace clb

using namespace clb;

extern "C" {

int clb_coo_add(clb_controls *ctl, const clb_coo *a_, const clb_coo *b_, clb_coo *out) {
    if (!ctl || !a_ || !b_ || !out) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    const clb_coo a = *a_, b = *b_;
    CLB_RETURN_IF(shape_check(a.nrows, a.ncols, b.nrows, b.ncols));
    DeviceGuard g(ctl);
    clb_coo c{};
    c.nrows = a.nrows;
    c.ncols = a.ncols;
    if (a.nnz == 0 && b.nnz == 0) {
        *out = c;
        return CLB_SUCCESS;
    }
    if (a.nnz == 0 || b.nnz == 0) {  // copy of the filled operand (coo_matrix_addition.cpp:48-64)
        const clb_coo &f = a.nnz ? a : b;
        CLB_RETURN_IF(copy_u32(ctl, f.rows, f.nnz, &c.rows));
        CLB_RETURN_IF(copy_u32(ctl, f.cols, f.nnz, &c.cols));
        c.nnz = f.nnz;
        CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
        *out = c;
        return CLB_SUCCESS;
    }
    ProfScope ps(ctl, "coo_add");
    const CooSide A{a.rows, a.cols, a.nnz}, B{b.rows, b.cols, b.nnz};
    const CsrSide none{nullptr, nullptr, 0};
    const uint64_t total = a.nnz + b.nnz, ntiles = (total + MP_TILE - 1) / MP_TILE;
    if (ntiles >= (1ull << 31)) return fail(CLB_NOT_SUPPORTED, "addition too large");
    Temp<uint64_t> split, toff, tot;
    Temp<uint32_t> tcnt;
    CLB_RETURN_IF(split.alloc(ctl, ntiles + 1));
    CLB_RETURN_IF(tcnt.alloc(ctl, ntiles));
    CLB_RETURN_IF(toff.alloc(ctl, ntiles));
    CLB_RETURN_IF(tot.alloc(ctl, 1));
    coo_split_kernel<<<grid_for(ctl, ntiles + 1), 256, 0, ctl->stream>>>(A, B, ntiles, split.ptr);
    merge_tile_kernel<false, 0><<<(unsigned)ntiles, MP_NT, 0, ctl->stream>>>(A, B, none, none, 0, split.ptr, nullptr,
                                                                             tcnt.ptr, nullptr, nullptr, nullptr, nullptr);
    CLB_CHECK_LAUNCH();
    CLB_RETURN_IF(scan_u32_to_u64(ctl, tcnt.ptr, toff.ptr, ntiles, tot.ptr));
    uint64_t nnz = 0;
    CLB_RETURN_IF(read_scalars(ctl, tot.ptr, &nnz, 1));
    Temp<uint32_t> rows, cols;
    CLB_RETURN_IF(rows.alloc(ctl, nnz));
    CLB_RETURN_IF(cols.alloc(ctl, nnz));
    merge_tile_kernel<false, 1><<<(unsigned)ntiles, MP_NT, 0, ctl->stream>>>(A, B, none, none, 0, split.ptr, nullptr,
                                                                             nullptr, toff.ptr, nullptr, rows.ptr, cols.ptr);
    CLB_CHECK_LAUNCH();
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    c.nnz = nnz;
    c.rows = rows.release_ownership();
    c.cols = cols.release_ownership();
    *out = c;
    return CLB_SUCCESS;
}

int clb_csr_add(clb_controls *ctl, const clb_csr *a_, const clb_csr *b_, clb_csr *out) {
    if (!ctl || !a_ || !b_ || !out) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    const clb_csr a = *a_, b = *b_;
    CLB_RETURN_IF(shape_check(a.nrows, a.ncols, b.nrows, b.ncols));
    DeviceGuard g(ctl);
    clb_csr c{};
    c.nrows = a.nrows;
    c.ncols = a.ncols;
    if (a.nnz == 0 && b.nnz == 0) {
        *out = c;
        return CLB_SUCCESS;
    }
    if (a.nnz == 0 || b.nnz == 0) {  // copy of the filled operand (csr_addition.cpp:38-55)
        const clb_csr &f = a.nnz ? a : b;
        Temp<uint64_t> rpt;
        CLB_RETURN_IF(rpt.alloc(ctl, f.nrows + 1));
        CLB_TRY_CUDA(cudaMemcpyAsync(rpt.ptr, f.rpt, (f.nrows + 1) * 8, cudaMemcpyDeviceToDevice, ctl->stream),
                     CLB_COPY_BUFFER_ERROR);
        CLB_RETURN_IF(copy_u32(ctl, f.cols, f.nnz, &c.cols));
        CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
        c.rpt = rpt.release_ownership();
        c.nnz = f.nnz;
        *out = c;
        return CLB_SUCCESS;
    }
    if (a.nrows >= (1ull << 32)) return fail(CLB_NOT_SUPPORTED, "2^32 or more rows");
    ProfScope ps(ctl, "csr_add");
    const CsrSide A{a.rpt, a.cols, a.nnz}, B{b.rpt, b.cols, b.nnz};
    const CooSide none{nullptr, nullptr, 0};
    const uint64_t total = a.nnz + b.nnz, ntiles = (total + MP_TILE - 1) / MP_TILE;
    if (ntiles >= (1ull << 31)) return fail(CLB_NOT_SUPPORTED, "addition too large");
    Temp<uint64_t> split, srow, toff, tot, rpt;
    Temp<uint32_t> tcnt, dup;
    CLB_RETURN_IF(split.alloc(ctl, ntiles + 1));
    CLB_RETURN_IF(srow.alloc(ctl, ntiles + 1));
    CLB_RETURN_IF(tcnt.alloc(ctl, ntiles));
    CLB_RETURN_IF(toff.alloc(ctl, ntiles));
    CLB_RETURN_IF(tot.alloc(ctl, 2));
    CLB_RETURN_IF(dup.alloc(ctl, a.nrows));
    CLB_RETURN_IF(rpt.alloc(ctl, a.nrows + 1));
    CLB_TRY_CUDA(cudaMemsetAsync(dup.ptr, 0, a.nrows * 4, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    csr_split_kernel<<<grid_for(ctl, ntiles + 1), 256, 0, ctl->stream>>>(A, B, a.nrows, ntiles, split.ptr, srow.ptr);
    merge_tile_kernel<true, 0><<<(unsigned)ntiles, MP_NT, 0, ctl->stream>>>(none, none, A, B, a.nrows, split.ptr,
                                                                            srow.ptr, tcnt.ptr, nullptr, dup.ptr,
                                                                            nullptr, nullptr);
    csr_row_counts_kernel<<<grid_for(ctl, a.nrows), 256, 0, ctl->stream>>>(a.rpt, b.rpt, dup.ptr, a.nrows, rpt.ptr);
    CLB_CHECK_LAUNCH();
    CLB_RETURN_IF(scan_u64_inplace(ctl, rpt.ptr, a.nrows, tot.ptr));
    CLB_RETURN_IF(scan_u32_to_u64(ctl, tcnt.ptr, toff.ptr, ntiles, tot.ptr + 1));
    uint64_t h[2];
    CLB_RETURN_IF(read_scalars(ctl, tot.ptr, h, 2));
    if (h[0] != h[1]) return fail(CLB_RUN_KERNEL_FAILURE, "row counts and tile counts disagree");
    const uint64_t nnz = h[0];
    CLB_TRY_CUDA(cudaMemcpyAsync(rpt.ptr + a.nrows, tot.ptr, 8, cudaMemcpyDeviceToDevice, ctl->stream),
                 CLB_COPY_BUFFER_ERROR);
    Temp<uint32_t> cols;
    CLB_RETURN_IF(cols.alloc(ctl, nnz));
    merge_tile_kernel<true, 1><<<(unsigned)ntiles, MP_NT, 0, ctl->stream>>>(none, none, A, B, a.nrows, split.ptr,
                                                                            srow.ptr, nullptr, toff.ptr, nullptr,
                                                                            nullptr, cols.ptr);
    CLB_CHECK_LAUNCH();
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    c.nnz = nnz;
    c.rpt = rpt.release_ownership();
    c.cols = cols.release_ownership();
    *out = c;
    return CLB_SUCCESS;
}

}  // extern "C"
