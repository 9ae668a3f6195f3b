// spgemm_batched.cu -- many independent boolean products C_k = A_k * B_k in
// one pass, plus the accumulator autotuner.  Not in the reference, which
// multiplies one pair per call (src/dcsr/dcsr.hpp:27-36).
//
// The pairs are stacked block-diagonally:
//   A' = [A_1; A_2; ...]  rows shifted by the rows of A_1..A_{k-1}, columns
//                         shifted by the rows of B_1..B_{k-1};
//   B' = [B_1; B_2; ...]  rows shifted likewise, columns NOT shifted
//                         (B'.ncols = max_k B_k.ncols).
// Row i of A' (pair k) only meets rows of B_k, so C' = A' B' holds C_k in the
// rows of pair k with C_k's own column indices.  One SpGEMM over (A', B')
// runs every pair in the same launches -- one workload pass, one binning,
// one persistent launch per accumulator kind -- balanced across the whole
// batch, so the launch count does not grow with the number of pairs.  A
// split kernel then cuts C' into the C_k.
#include <algorithm>
#include <string>
#include <vector>

#include "spgemm.cuh"

namespace clb {

namespace {

struct PairDesc {
    const uint64_t *rpt;
    const uint32_t *rows;
    const uint32_t *cols;
    uint64_t nzr, nnz;
    uint64_t nzr_off, nnz_off;  // position in the stacked matrix
    uint32_t row_add, col_add;  // added to row ids / column ids
    uint32_t ncols;             // columns of the pair's product
};

constexpr int CAT_NT = 256;

// Stacks the pairs' matrices: blockIdx.y = pair.
// row_ncols (may be null): per stacked row, the columns of its pair's product;
// row_pair (may be null): per stacked row, its pair.
__global__ void __launch_bounds__(CAT_NT) stack_kernel(const PairDesc *__restrict__ d, uint64_t *__restrict__ rpt,
                                                       uint32_t *__restrict__ rows, uint32_t *__restrict__ cols,
                                                       uint32_t *__restrict__ row_ncols,
                                                       uint32_t *__restrict__ row_pair, uint64_t total_nzr,
                                                       uint64_t total_nnz) {
    const PairDesc p = d[blockIdx.y];
    const uint64_t stride = (uint64_t)gridDim.x * CAT_NT;
    const uint64_t t0 = (uint64_t)blockIdx.x * CAT_NT + threadIdx.x;
    const uint64_t base = p.nzr ? p.rpt[0] : 0;
    for (uint64_t r = t0; r < p.nzr; r += stride) {
        rows[p.nzr_off + r] = p.rows[r] + p.row_add;
        rpt[p.nzr_off + r] = p.rpt[r] - base + p.nnz_off;
        if (row_ncols) row_ncols[p.nzr_off + r] = p.ncols;
        if (row_pair) row_pair[p.nzr_off + r] = blockIdx.y;
    }
    for (uint64_t j = t0; j < p.nnz; j += stride) cols[p.nnz_off + j] = p.cols[j] + p.col_add;
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) rpt[total_nzr] = total_nnz;
}

// bounds[k] = first row of C' at or after row_start[k] (k <= count), and
// nnz_bounds[k] = C'.rpt[bounds[k]].
__global__ void split_bounds_kernel(const uint32_t *__restrict__ crows, const uint64_t *__restrict__ crpt, uint64_t nzr,
                                    const uint64_t *__restrict__ row_start, uint32_t count,
                                    uint64_t *__restrict__ bounds) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k <= count; k += gridDim.x * blockDim.x) {
        const uint64_t key = row_start[k];
        uint64_t lo = 0, hi = nzr;
        while (lo < hi) {
            const uint64_t m = lo + (hi - lo) / 2;
            if ((uint64_t)crows[m] < key) lo = m + 1; else hi = m;
        }
        bounds[k] = lo;
        bounds[count + 1 + k] = crpt[lo];
    }
}

struct OutDesc {
    uint64_t *rpt;
    uint32_t *rows;
    uint32_t *cols;
    uint64_t r0, nzr;    // rows [r0, r0 + nzr) of C'
    uint64_t j0, nnz;    // columns [j0, j0 + nnz) of C'
    uint32_t row_sub;
};

__global__ void __launch_bounds__(CAT_NT) split_kernel(const OutDesc *__restrict__ d, const uint64_t *__restrict__ crpt,
                                                       const uint32_t *__restrict__ crows,
                                                       const uint32_t *__restrict__ ccols) {
    const OutDesc o = d[blockIdx.y];
    if (!o.nnz) return;
    const uint64_t stride = (uint64_t)gridDim.x * CAT_NT;
    const uint64_t t0 = (uint64_t)blockIdx.x * CAT_NT + threadIdx.x;
    for (uint64_t r = t0; r <= o.nzr; r += stride) {
        o.rpt[r] = crpt[o.r0 + r] - o.j0;
        if (r < o.nzr) o.rows[r] = crows[o.r0 + r] - o.row_sub;
    }
    for (uint64_t j = t0; j < o.nnz; j += stride) o.cols[j] = ccols[o.j0 + j];
}

// Blocks per pair: enough for the largest pair to be copied with ~4 items
// per thread; blocks of smaller pairs find nothing to do and exit.
unsigned stack_grid_x(const clb_controls *ctl, uint64_t largest, uint32_t count) {
    (void)ctl;
    (void)count;
    const uint64_t gx = (largest + 4 * CAT_NT - 1) / (4 * CAT_NT);
    return (unsigned)std::min<uint64_t>(std::max<uint64_t>(gx, 1), 65535);
}

// One product with a tuning: the exact two-pass form or the single pass into
// upper-bound slots (ESC accumulators for the rows below bitmap_min).
int spgemm_tuned(clb_controls *ctl, const clb_dcsr &A, const clb_dcsr &B, uint32_t form, const Tuning &t,
                 clb_dcsr *c, clb_spgemm_stats *st) {
    if (form == 0 || form == 2) return spgemm_hash_two_pass(ctl, A, B, c, st, t, form == 2);
    clb_spgemm_stats s{};
    ctl->launches = 0;
    if (A.nnz == 0 || B.nnz == 0 || A.nzr == 0 || B.nzr == 0) {
        clb_dcsr C{};
        C.nrows = A.nrows;
        C.ncols = B.ncols;
        *c = C;
        if (st) *st = s;
        return CLB_SUCCESS;
    }
    CLB_RETURN_IF(clear_status(ctl));
    const AView a{A.rpt, A.rows, A.cols, A.nzr};
    BRows b;
    Temp<uint64_t> dense, tot;
    CLB_RETURN_IF(prepare_b(ctl, B, dense, b));
    Temp<uint32_t> work, cap;
    CLB_RETURN_IF(work.alloc(ctl, A.nzr));
    CLB_RETURN_IF(cap.alloc(ctl, A.nzr));
    CLB_RETURN_IF(tot.alloc(ctl, 1));
    CLB_TRY_CUDA(cudaMemsetAsync(tot.ptr, 0, 8, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    CLB_RETURN_IF(launch_workload(ctl, a, b, work.ptr, tot.ptr));
    CLB_RETURN_IF(launch_upper_bound_caps(ctl, work.ptr, A.nzr, B.ncols, cap.ptr));
    uint64_t products = 0;
    CLB_RETURN_IF(read_scalars(ctl, tot.ptr, &products, 1));
    int rc = spgemm_single_pass(ctl, A, B, a, b, work.ptr, cap.ptr, true, products, c, &s, 0, t);
    s.kernel_launches = ctl->launches;
    if (st) *st = s;
    return rc;
}

// Pair descriptors reach the device as kernel parameters (by value), so no
// host memory is read when the launch is replayed from a CUDA graph.
constexpr uint32_t DESC_CHUNK = 24;
struct DescChunk {
    PairDesc a[DESC_CHUNK], b[DESC_CHUNK];
    PairFeat f[DESC_CHUNK];
};

__global__ void store_descs_kernel(DescChunk c, uint32_t k0, uint32_t n, PairDesc *__restrict__ da,
                                   PairDesc *__restrict__ db, uint64_t *__restrict__ first,
                                   uint32_t *__restrict__ row_base, PairFeat *__restrict__ pf) {
    const uint32_t j = threadIdx.x;
    if (j < n) {
        da[k0 + j] = c.a[j];
        db[k0 + j] = c.b[j];
        first[k0 + j] = c.a[j].nzr_off;
        row_base[k0 + j] = c.a[j].row_add;
        if (pf) pf[k0 + j] = c.f[j];
    }
}

// *need += sum over rows of round4(min(work, ncols)): the slots of the
// host-sync-free form (16-byte aligned upper-bound slots).
__global__ void slot_need_kernel(const uint32_t *__restrict__ work, uint64_t n, uint64_t ncols,
                                 unsigned long long *__restrict__ need) {
    unsigned long long mine = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = min((uint64_t)work[i], ncols);
        mine += (c + 3) & ~3ull;
    }
    mine = warp_sum(mine);
    if (lane_id() == 0 && mine) atomicAdd(need, mine);
}

// Host-side checks and stacking offsets shared by the batched entry points.
int pair_descs(uint32_t count, const clb_dcsr *a, const clb_dcsr *b, std::vector<PairDesc> &da,
               std::vector<PairDesc> &db, uint64_t &arows, uint64_t &brows, uint64_t &anzr, uint64_t &annz,
               uint64_t &bnzr, uint64_t &bnnz, uint64_t &bcols, uint64_t &amax, uint64_t &bmax) {
    da.resize(count);
    db.resize(count);
    arows = brows = anzr = annz = bnzr = bnnz = bcols = amax = bmax = 0;
    for (uint32_t k = 0; k < count; ++k) {
        const int rc = validate_spgemm(a[k], b[k]);
        if (rc != CLB_SUCCESS) return fail(rc, "pair " + std::to_string(k) + ": " + clb_last_error());
        const bool live = a[k].nnz && b[k].nnz;
        da[k] = PairDesc{a[k].rpt, a[k].rows, a[k].cols, live ? a[k].nzr : 0, live ? a[k].nnz : 0, anzr, annz,
                         (uint32_t)arows, (uint32_t)brows, (uint32_t)b[k].ncols};
        db[k] = PairDesc{b[k].rpt, b[k].rows, b[k].cols, live ? b[k].nzr : 0, live ? b[k].nnz : 0, bnzr, bnnz,
                         (uint32_t)brows, 0u, (uint32_t)b[k].ncols};
        if (live) {
            anzr += a[k].nzr;
            annz += a[k].nnz;
            bnzr += b[k].nzr;
            bnnz += b[k].nnz;
            amax = std::max(amax, std::max(a[k].nnz, a[k].nzr + 1));
            bmax = std::max(bmax, std::max(b[k].nnz, b[k].nzr + 1));
        }
        arows += a[k].nrows;
        brows += b[k].nrows;
        bcols = std::max(bcols, b[k].ncols);
        if (arows > 0xFFFFFFFFull || brows > 0xFFFFFFFFull)
            return fail(CLB_NOT_SUPPORTED, "the stacked batch exceeds 2^32 - 1 rows");
    }
    return CLB_SUCCESS;
}

// ------------------------------------------------------------- union ----
// The union of k matrices of one shape is the product A_u B_u with
// B_u = [M_0; M_1; ...; M_{k-1}] (k*nrows x ncols) and A_u (nrows x k*nrows)
// holding, in row r, the columns j*nrows + r of the M_j that store row r:
// row r of A_u B_u merges the k sorted rows r of the M_j and drops the
// duplicates, i.e. the accumulators do a k-way merge in one pass.

// flags[r] |= 1 << j for every stored row r of M_j (blockIdx.y = j).
__global__ void union_mark_kernel(const PairDesc *__restrict__ d, uint32_t *__restrict__ flags) {
    const PairDesc p = d[blockIdx.y];
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < p.nzr; k += (uint64_t)gridDim.x * blockDim.x)
        atomicOr(flags + p.rows[k], 1u << blockIdx.y);
}

// cnt[r] = number of M_j storing row r; nonempty[r] = cnt[r] > 0.
__global__ void union_counts_kernel(const uint32_t *__restrict__ flags, uint64_t n, uint32_t *__restrict__ cnt,
                                    uint32_t *__restrict__ nonempty) {
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t c = __popc(flags[r]);
        cnt[r] = c;
        nonempty[r] = c ? 1u : 0u;
    }
}

// A_u in DCSR: stored row pos[r] = r with columns j*nrows + r (j ascending).
__global__ void union_left_kernel(const uint32_t *__restrict__ flags, const uint64_t *__restrict__ off,
                                  const uint32_t *__restrict__ pos, uint64_t n, uint64_t nzr, uint64_t nnz,
                                  uint64_t *__restrict__ rpt, uint32_t *__restrict__ rows,
                                  uint32_t *__restrict__ cols) {
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t f = flags[r];
        if (!f) continue;
        const uint32_t p = pos[r];
        uint64_t o = off[r];
        rpt[p] = o;
        rows[p] = (uint32_t)r;
        while (f) {
            const uint32_t j = (uint32_t)(__ffs(f) - 1);
            cols[o++] = (uint32_t)(j * n + r);
            f &= f - 1;
        }
        if (p + 1 == nzr) rpt[nzr] = nnz;
    }
}

// The batched product: stack, one product over the stack (exact / tuned
// form, or the learned single pass when `sizer` is given), split.
int batched_impl(clb_controls *ctl, uint32_t count, const clb_dcsr *a, const clb_dcsr *b, clb_dcsr *c,
                 const clb_spgemm_tuning *tuning, const clb_sizer *sizer, float margin_log2, float slack,
                 clb_spgemm_stats *stats) {
    if (!ctl || (count && (!a || !b || !c))) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    if (count > 65535) return fail(CLB_NOT_SUPPORTED, "at most 65535 pairs per batch");
    CLB_RETURN_IF(check_tuning(tuning));
    clb_spgemm_stats st{};
    if (stats) *stats = st;
    if (count == 0) return CLB_SUCCESS;
    // pair checks and offsets
    std::vector<PairDesc> da(count), db(count);
    std::vector<uint64_t> row_start(count + 1);
    uint64_t arows = 0, brows = 0, anzr = 0, annz = 0, bnzr = 0, bnnz = 0, bcols = 0, amax = 0, bmax = 0;
    for (uint32_t k = 0; k < count; ++k) {
        const int rc = validate_spgemm(a[k], b[k]);
        if (rc != CLB_SUCCESS) return fail(rc, "pair " + std::to_string(k) + ": " + clb_last_error());
        row_start[k] = arows;
        const bool live = a[k].nnz && b[k].nnz;  // a pair without products contributes nothing
        da[k] = PairDesc{a[k].rpt, a[k].rows, a[k].cols, live ? a[k].nzr : 0, live ? a[k].nnz : 0, anzr, annz,
                         (uint32_t)arows, (uint32_t)brows, (uint32_t)b[k].ncols};
        db[k] = PairDesc{b[k].rpt, b[k].rows, b[k].cols, live ? b[k].nzr : 0, live ? b[k].nnz : 0, bnzr, bnnz,
                         (uint32_t)brows, 0u, (uint32_t)b[k].ncols};
        if (live) {
            anzr += a[k].nzr;
            annz += a[k].nnz;
            bnzr += b[k].nzr;
            bnnz += b[k].nnz;
            amax = std::max(amax, std::max(a[k].nnz, a[k].nzr + 1));
            bmax = std::max(bmax, std::max(b[k].nnz, b[k].nzr + 1));
        }
        arows += a[k].nrows;
        brows += b[k].nrows;
        bcols = std::max(bcols, b[k].ncols);
        if (arows > 0xFFFFFFFFull || brows > 0xFFFFFFFFull)
            return fail(CLB_NOT_SUPPORTED, "the stacked batch exceeds 2^32 - 1 rows");
    }
    row_start[count] = arows;
    for (uint32_t k = 0; k < count; ++k) {
        clb_dcsr C{};
        C.nrows = a[k].nrows;
        C.ncols = b[k].ncols;
        c[k] = C;
    }
    if (annz == 0) return CLB_SUCCESS;
    DeviceGuard g(ctl);
    const uint32_t form = tuning ? tuning->form : 0;
    Tuning t = to_tuning(tuning);

    // stacked operands
    Temp<PairDesc> dda, ddb;
    Temp<uint64_t> arpt, brpt, rs;
    Temp<uint32_t> arws, acls, brws, bcls, rnc, rpair;
    Temp<PairFeat> pf;
    CLB_RETURN_IF(dda.alloc(ctl, count));
    CLB_RETURN_IF(ddb.alloc(ctl, count));
    CLB_RETURN_IF(rs.alloc(ctl, count + 1));
    CLB_RETURN_IF(arpt.alloc(ctl, anzr + 1));
    CLB_RETURN_IF(arws.alloc(ctl, anzr));
    CLB_RETURN_IF(rnc.alloc(ctl, anzr));
    if (sizer) {
        // per-row pair context of the row features
        std::vector<PairFeat> hf(count);
        for (uint32_t k = 0; k < count; ++k)
            hf[k] = PairFeat{(uint32_t)row_start[k], (uint32_t)a[k].nrows, learned_density_feature(b[k]), 0u};
        CLB_RETURN_IF(rpair.alloc(ctl, anzr));
        CLB_RETURN_IF(pf.alloc(ctl, count));
        CLB_TRY_CUDA(cudaMemcpyAsync(pf.ptr, hf.data(), count * sizeof(PairFeat), cudaMemcpyHostToDevice, ctl->stream),
                     CLB_WRITE_BUFFER_ERROR);
    }
    CLB_RETURN_IF(acls.alloc(ctl, annz));
    CLB_RETURN_IF(brpt.alloc(ctl, bnzr + 1));
    CLB_RETURN_IF(brws.alloc(ctl, bnzr));
    CLB_RETURN_IF(bcls.alloc(ctl, bnnz));
    CLB_TRY_CUDA(cudaMemcpyAsync(dda.ptr, da.data(), count * sizeof(PairDesc), cudaMemcpyHostToDevice, ctl->stream),
                 CLB_WRITE_BUFFER_ERROR);
    CLB_TRY_CUDA(cudaMemcpyAsync(ddb.ptr, db.data(), count * sizeof(PairDesc), cudaMemcpyHostToDevice, ctl->stream),
                 CLB_WRITE_BUFFER_ERROR);
    CLB_TRY_CUDA(cudaMemcpyAsync(rs.ptr, row_start.data(), (count + 1) * 8, cudaMemcpyHostToDevice, ctl->stream),
                 CLB_WRITE_BUFFER_ERROR);
    {
        ProfScope ps(ctl, "batch_stack");
        stack_kernel<<<dim3(stack_grid_x(ctl, amax, count), count), CAT_NT, 0, ctl->stream>>>(
            dda.ptr, arpt.ptr, arws.ptr, acls.ptr, rnc.ptr, rpair.ptr, anzr, annz);
        stack_kernel<<<dim3(stack_grid_x(ctl, bmax, count), count), CAT_NT, 0, ctl->stream>>>(
            ddb.ptr, brpt.ptr, brws.ptr, bcls.ptr, nullptr, nullptr, bnzr, bnnz);
        CLB_CHECK_LAUNCH();
    }
    const clb_dcsr As{arows, brows, annz, anzr, arpt.ptr, arws.ptr, acls.ptr};
    const clb_dcsr Bs{brows, bcols, bnnz, bnzr, brpt.ptr, brws.ptr, bcls.ptr};
    CLB_RETURN_IF(validate_spgemm(As, Bs));
    clb_dcsr Cs{};
    t.row_ncols = rnc.ptr;  // each pair's rows use a bitmap as wide as its own product
    if (sizer) {
        const BatchRows br{rpair.ptr, pf.ptr};
        CLB_RETURN_IF(spgemm_learned(ctl, As, Bs, sizer, margin_log2, slack, t, &br, &Cs, &st));
    } else {
        CLB_RETURN_IF(spgemm_tuned(ctl, As, Bs, form, t, &Cs, &st));
    }
    const uint32_t inner_launches = st.kernel_launches;
    if (Cs.nnz == 0) {
        st.kernel_launches = inner_launches + 2;
        if (stats) *stats = st;
        return CLB_SUCCESS;
    }
    // split C' into the pairs' products
    Temp<uint64_t> bounds;
    int rc = bounds.alloc(ctl, 2 * (count + 1));
    std::vector<uint64_t> hb(2 * (count + 1));
    if (rc == CLB_SUCCESS) {
        split_bounds_kernel<<<(count + 256) / 256, 256, 0, ctl->stream>>>(Cs.rows, Cs.rpt, Cs.nzr, rs.ptr, count,
                                                                          bounds.ptr);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(hb.data(), bounds.ptr, hb.size() * 8, cudaMemcpyDeviceToHost, ctl->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctl->stream);
        if (e != cudaSuccess) rc = fail(CLB_RUN_KERNEL_FAILURE, cudaGetErrorString(e));
    }
    std::vector<OutDesc> od(count);
    std::vector<clb_dcsr> outs(count);
    uint64_t omax = 1;
    for (uint32_t k = 0; k < count && rc == CLB_SUCCESS; ++k) {
        const uint64_t r0 = hb[k], r1 = hb[k + 1], j0 = hb[count + 1 + k], j1 = hb[count + 1 + k + 1];
        clb_dcsr C{};
        C.nrows = a[k].nrows;
        C.ncols = b[k].ncols;
        OutDesc o{nullptr, nullptr, nullptr, r0, r1 - r0, j0, j1 - j0, (uint32_t)row_start[k]};
        if (j1 > j0) {
            Temp<uint64_t> p;
            Temp<uint32_t> r, cc;
            rc = p.alloc(ctl, r1 - r0 + 1);
            if (rc == CLB_SUCCESS) rc = r.alloc(ctl, r1 - r0);
            if (rc == CLB_SUCCESS) rc = cc.alloc(ctl, j1 - j0);
            if (rc != CLB_SUCCESS) break;
            o.rpt = p.ptr;
            o.rows = r.ptr;
            o.cols = cc.ptr;
            C.nnz = j1 - j0;
            C.nzr = r1 - r0;
            C.rpt = p.release_ownership();
            C.rows = r.release_ownership();
            C.cols = cc.release_ownership();
            omax = std::max(omax, std::max(C.nnz, C.nzr + 1));
        }
        od[k] = o;
        outs[k] = C;
    }
    Temp<OutDesc> dod;
    if (rc == CLB_SUCCESS) rc = dod.alloc(ctl, count);
    if (rc == CLB_SUCCESS) {
        cudaError_t e = cudaMemcpyAsync(dod.ptr, od.data(), count * sizeof(OutDesc), cudaMemcpyHostToDevice, ctl->stream);
        if (e == cudaSuccess) {
            ProfScope ps(ctl, "batch_split");
            split_kernel<<<dim3(stack_grid_x(ctl, omax, count), count), CAT_NT, 0, ctl->stream>>>(dod.ptr, Cs.rpt,
                                                                                                 Cs.rows, Cs.cols);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctl->stream);
        if (e != cudaSuccess) rc = fail(CLB_RUN_KERNEL_FAILURE, cudaGetErrorString(e));
    }
    clb_dcsr_release(ctl, &Cs);
    if (rc != CLB_SUCCESS) {
        for (auto &o : outs) clb_dcsr_release(ctl, &o);
        return rc;
    }
    for (uint32_t k = 0; k < count; ++k) c[k] = outs[k];
    st.kernel_launches = inner_launches + 4;
    if (stats) *stats = st;
    return CLB_SUCCESS;
}

// The pairs stacked block-diagonally on the device, with the pair
// descriptors passed as kernel parameters (no host memory is read when the
// launches are replayed from a CUDA graph).  pair_ctx: also the per-row pair
// context of the learned row features.
struct Stack {
    Temp<PairDesc> dda, ddb;
    Temp<uint64_t> first, arpt, brpt;
    Temp<uint32_t> rbase, arws, acls, brws, bcls, rnc, rpair;
    Temp<PairFeat> pf;
    clb_dcsr As{}, Bs{};
};

int build_stack(clb_controls *ctl, uint32_t count, const clb_dcsr *a, const clb_dcsr *b,
                const std::vector<PairDesc> &da, const std::vector<PairDesc> &db, uint64_t arows, uint64_t brows,
                uint64_t anzr, uint64_t annz, uint64_t bnzr, uint64_t bnnz, uint64_t bcols, uint64_t amax,
                uint64_t bmax, bool pair_ctx, Stack &st) {
    CLB_RETURN_IF(st.dda.alloc(ctl, count));
    CLB_RETURN_IF(st.ddb.alloc(ctl, count));
    CLB_RETURN_IF(st.first.alloc(ctl, count));
    CLB_RETURN_IF(st.rbase.alloc(ctl, count));
    CLB_RETURN_IF(st.arpt.alloc(ctl, anzr + 1));
    CLB_RETURN_IF(st.arws.alloc(ctl, anzr));
    CLB_RETURN_IF(st.rnc.alloc(ctl, anzr));
    CLB_RETURN_IF(st.acls.alloc(ctl, annz));
    CLB_RETURN_IF(st.brpt.alloc(ctl, bnzr + 1));
    CLB_RETURN_IF(st.brws.alloc(ctl, bnzr));
    CLB_RETURN_IF(st.bcls.alloc(ctl, bnnz));
    if (pair_ctx) {
        CLB_RETURN_IF(st.rpair.alloc(ctl, anzr));
        CLB_RETURN_IF(st.pf.alloc(ctl, count));
    }
    for (uint32_t k0 = 0; k0 < count; k0 += DESC_CHUNK) {
        DescChunk ch{};
        const uint32_t nk = std::min<uint32_t>(DESC_CHUNK, count - k0);
        for (uint32_t j = 0; j < nk; ++j) {
            ch.a[j] = da[k0 + j];
            ch.b[j] = db[k0 + j];
            ch.f[j] = PairFeat{da[k0 + j].row_add, (uint32_t)a[k0 + j].nrows, learned_density_feature(b[k0 + j]), 0u};
        }
        store_descs_kernel<<<1, DESC_CHUNK, 0, ctl->stream>>>(ch, k0, nk, st.dda.ptr, st.ddb.ptr, st.first.ptr,
                                                              st.rbase.ptr, st.pf.ptr);
        ctl->launches += 1;
    }
    CLB_CHECK_LAUNCH();
    {
        ProfScope ps(ctl, "batch_stack");
        stack_kernel<<<dim3(stack_grid_x(ctl, amax, count), count), CAT_NT, 0, ctl->stream>>>(
            st.dda.ptr, st.arpt.ptr, st.arws.ptr, st.acls.ptr, st.rnc.ptr, st.rpair.ptr, anzr, annz);
        stack_kernel<<<dim3(stack_grid_x(ctl, bmax, count), count), CAT_NT, 0, ctl->stream>>>(
            st.ddb.ptr, st.brpt.ptr, st.brws.ptr, st.bcls.ptr, nullptr, nullptr, bnzr, bnnz);
        ctl->launches += 2;
        CLB_CHECK_LAUNCH();
    }
    st.As = clb_dcsr{arows, brows, annz, anzr, st.arpt.ptr, st.arws.ptr, st.acls.ptr};
    st.Bs = clb_dcsr{brows, bcols, bnnz, bnzr, st.brpt.ptr, st.brws.ptr, st.bcls.ptr};
    return validate_spgemm(st.As, st.Bs);
}

// The host-sync-free batched product (upper-bound slots, or learned slots
// and a spill arena when `sizer` is given).
int capture_impl(clb_controls *ctl, uint32_t count, const clb_dcsr *a, const clb_dcsr *b,
                 const clb_spgemm_tuning *tuning, const clb_sizer *sizer, float margin_log2, float slack,
                 uint64_t slot_capacity, uint64_t arena_capacity, uint64_t *c_rpt, uint32_t *c_rows,
                 uint32_t *c_cols, uint64_t cols_capacity, uint64_t *result, uint32_t *flags) {
    if (!ctl || (count && (!a || !b)) || !result || !flags) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    if (count == 0) return fail(CLB_INVALID_ARGUMENT, "empty batch");
    if (count > 65535) return fail(CLB_NOT_SUPPORTED, "at most 65535 pairs per batch");
    CLB_RETURN_IF(check_tuning(tuning));
    std::vector<PairDesc> da, db;
    uint64_t arows, brows, anzr, annz, bnzr, bnnz, bcols, amax, bmax;
    CLB_RETURN_IF(pair_descs(count, a, b, da, db, arows, brows, anzr, annz, bnzr, bnnz, bcols, amax, bmax));
    if (!c_rpt || (anzr && !c_rows) || (cols_capacity && !c_cols))
        return fail(CLB_INVALID_ARGUMENT, "NULL output array");
    DeviceGuard g(ctl);
    CLB_TRY_CUDA(cudaMemsetAsync(flags, 0, 4, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    CLB_TRY_CUDA(cudaMemsetAsync(result, 0, (2 + 2 * ((uint64_t)count + 1)) * 8, ctl->stream),
                 CLB_RUN_KERNEL_FAILURE);
    CLB_TRY_CUDA(cudaMemsetAsync(c_rpt, 0, 8, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    if (annz == 0) return CLB_SUCCESS;
    CLB_RETURN_IF(clear_status(ctl));
    ctl->launches = 0;
    Tuning t = to_tuning(tuning);
    Stack stk;
    CLB_RETURN_IF(build_stack(ctl, count, a, b, da, db, arows, brows, anzr, annz, bnzr, bnnz, bcols, amax, bmax,
                              sizer != nullptr, stk));
    t.row_ncols = stk.rnc.ptr;
    if (!sizer)
        return spgemm_esc_capture(ctl, stk.As, stk.Bs, t, slot_capacity, stk.first.ptr, stk.rbase.ptr, count, c_rpt,
                                  c_rows, c_cols, cols_capacity, result, flags);
    const CaptureLearned lc{sizer, margin_log2, slack, BatchRows{stk.rpair.ptr, stk.pf.ptr}, arena_capacity};
    return spgemm_esc_capture(ctl, stk.As, stk.Bs, t, slot_capacity, stk.first.ptr, stk.rbase.ptr, count, c_rpt,
                              c_rows, c_cols, cols_capacity, result, flags, &lc);
}

}  // namespace

Tuning to_tuning(const clb_spgemm_tuning *t) {
    Tuning r;
    if (!t) return r;
    if (t->warp_max) r.warp_max = t->warp_max;
    if (t->bitmap_min) r.bitmap_min = t->bitmap_min;
    if (t->bitmap_threads) r.bitmap_threads = t->bitmap_threads;
    if (t->small_lanes) r.small_lanes = t->small_lanes;
    if (t->wide_rows) r.wide_cluster = t->wide_rows == 1;
    return r;
}

int check_tuning(const clb_spgemm_tuning *t) {
    if (!t) return CLB_SUCCESS;
    if (t->form > 2)
        return fail(CLB_INVALID_VALUE,
                    "tuning.form must be 0 (two-pass), 1 (single pass) or 2 (two-pass keeping its bitmaps)");
    if (t->warp_max && t->warp_max != 32 && t->warp_max != 64 && t->warp_max != 128 && t->warp_max != 256)
        return fail(CLB_INVALID_VALUE, "tuning.warp_max must be 32, 64, 128 or 256");
    if (t->bitmap_min && (t->bitmap_min < 256 || t->bitmap_min > ESC_MAX_PRODUCTS))
        return fail(CLB_INVALID_VALUE, "tuning.bitmap_min must be in [256, 4096]");
    if (t->bitmap_threads && t->bitmap_threads != 256 && t->bitmap_threads != 512 && t->bitmap_threads != 1024)
        return fail(CLB_INVALID_VALUE, "tuning.bitmap_threads must be 256, 512 or 1024");
    if (t->small_lanes && t->small_lanes != 8 && t->small_lanes != 16 && t->small_lanes != 32)
        return fail(CLB_INVALID_VALUE, "tuning.small_lanes must be 8, 16 or 32");
    if (t->wide_rows > 2) return fail(CLB_INVALID_VALUE, "tuning.wide_rows must be 1 (cluster) or 2 (chunks)");
    return CLB_SUCCESS;
}

}  // namespace clb

using namespace clb;

extern "C" {

void clb_spgemm_tuning_default(clb_spgemm_tuning *t) {
    if (!t) return;
    *t = clb_spgemm_tuning{};
    const Tuning d;
    t->form = 0;
    t->warp_max = d.warp_max;
    t->bitmap_min = d.bitmap_min;
    t->bitmap_threads = d.bitmap_threads;
    t->small_lanes = d.small_lanes;
    t->wide_rows = d.wide_cluster ? 1 : 2;
}

int clb_dcsr_spgemm_tuned(clb_controls *ctl, const clb_dcsr *a, const clb_dcsr *b, const clb_spgemm_tuning *tuning,
                          clb_dcsr *c, clb_spgemm_stats *stats) {
    if (!ctl || !a || !b || !c) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    CLB_RETURN_IF(check_tuning(tuning));
    CLB_RETURN_IF(validate_spgemm(*a, *b));
    DeviceGuard g(ctl);
    return spgemm_tuned(ctl, *a, *b, tuning ? tuning->form : 0, to_tuning(tuning), c, stats);
}

int clb_dcsr_spgemm_batched(clb_controls *ctl, uint32_t count, const clb_dcsr *a, const clb_dcsr *b, clb_dcsr *c,
                            const clb_spgemm_tuning *tuning, clb_spgemm_stats *stats) {
    return batched_impl(ctl, count, a, b, c, tuning, nullptr, 0.f, 0.f, stats);
}

int clb_dcsr_spgemm_batched_learned(clb_controls *ctl, uint32_t count, const clb_dcsr *a, const clb_dcsr *b,
                                    clb_dcsr *c, const clb_sizer *sizer, float margin_log2, float slack,
                                    const clb_spgemm_tuning *tuning, clb_spgemm_stats *stats) {
    if (!sizer) return fail(CLB_INVALID_ARGUMENT, "NULL sizer");
    return batched_impl(ctl, count, a, b, c, tuning, sizer, margin_log2, slack, stats);
}

int clb_spgemm_batched_plan(clb_controls *ctl, uint32_t count, const clb_dcsr *a, const clb_dcsr *b,
                            uint64_t *rows_need, uint64_t *slots_need) {
    if (!ctl || (count && (!a || !b)) || !rows_need || !slots_need) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    if (count > 65535) return fail(CLB_NOT_SUPPORTED, "at most 65535 pairs per batch");
    std::vector<PairDesc> da, db;
    uint64_t arows, brows, anzr, annz, bnzr, bnnz, bcols, amax, bmax;
    CLB_RETURN_IF(pair_descs(count, a, b, da, db, arows, brows, anzr, annz, bnzr, bnnz, bcols, amax, bmax));
    *rows_need = anzr;
    *slots_need = 0;
    if (annz == 0) return CLB_SUCCESS;
    DeviceGuard g(ctl);
    Temp<uint64_t> need;
    CLB_RETURN_IF(need.alloc(ctl, 2));
    CLB_TRY_CUDA(cudaMemsetAsync(need.ptr, 0, 16, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    for (uint32_t k = 0; k < count; ++k) {
        if (!da[k].nnz) continue;
        const AView av{a[k].rpt, a[k].rows, a[k].cols, a[k].nzr};
        BRows bv;
        Temp<uint64_t> dense;
        Temp<uint32_t> work;
        CLB_RETURN_IF(prepare_b(ctl, b[k], dense, bv));
        CLB_RETURN_IF(work.alloc(ctl, a[k].nzr));
        CLB_RETURN_IF(launch_workload(ctl, av, bv, work.ptr, need.ptr + 1));
        slot_need_kernel<<<std::max<unsigned>(1, std::min<uint64_t>((a[k].nzr + 255) / 256, ctl->sm_count * 8)), 256,
                           0, ctl->stream>>>(work.ptr, a[k].nzr, b[k].ncols, (unsigned long long *)need.ptr);
        CLB_CHECK_LAUNCH();
    }
    CLB_RETURN_IF(read_scalars(ctl, need.ptr, slots_need, 1));
    return CLB_SUCCESS;
}

int clb_dcsr_spgemm_batched_capture(clb_controls *ctl, uint32_t count, const clb_dcsr *a, const clb_dcsr *b,
                                    const clb_spgemm_tuning *tuning, uint64_t slot_capacity, uint64_t *c_rpt,
                                    uint32_t *c_rows, uint32_t *c_cols, uint64_t cols_capacity, uint64_t *result,
                                    uint32_t *flags) {
    return capture_impl(ctl, count, a, b, tuning, nullptr, 0.f, 0.f, slot_capacity, 0, c_rpt, c_rows, c_cols,
                        cols_capacity, result, flags);
}

int clb_dcsr_spgemm_batched_capture_learned(clb_controls *ctl, uint32_t count, const clb_dcsr *a, const clb_dcsr *b,
                                            const clb_sizer *sizer, float margin_log2, float slack,
                                            const clb_spgemm_tuning *tuning, uint64_t slot_capacity,
                                            uint64_t arena_capacity, uint64_t *c_rpt, uint32_t *c_rows,
                                            uint32_t *c_cols, uint64_t cols_capacity, uint64_t *result,
                                            uint32_t *flags) {
    if (!sizer) return fail(CLB_INVALID_ARGUMENT, "NULL sizer");
    return capture_impl(ctl, count, a, b, tuning, sizer, margin_log2, slack, slot_capacity, arena_capacity, c_rpt,
                        c_rows, c_cols, cols_capacity, result, flags);
}

int clb_spgemm_batched_plan_learned(clb_controls *ctl, uint32_t count, const clb_dcsr *a, const clb_dcsr *b,
                                    const clb_sizer *sizer, float margin_log2, float slack,
                                    const clb_spgemm_tuning *tuning, uint64_t *rows_need, uint64_t *slots_need) {
    if (!ctl || (count && (!a || !b)) || !sizer || !rows_need || !slots_need)
        return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    if (count > 65535) return fail(CLB_NOT_SUPPORTED, "at most 65535 pairs per batch");
    CLB_RETURN_IF(check_tuning(tuning));
    std::vector<PairDesc> da, db;
    uint64_t arows, brows, anzr, annz, bnzr, bnnz, bcols, amax, bmax;
    CLB_RETURN_IF(pair_descs(count, a, b, da, db, arows, brows, anzr, annz, bnzr, bnnz, bcols, amax, bmax));
    *rows_need = anzr;
    *slots_need = 0;
    if (annz == 0) return CLB_SUCCESS;
    DeviceGuard g(ctl);
    Stack stk;
    CLB_RETURN_IF(build_stack(ctl, count, a, b, da, db, arows, brows, anzr, annz, bnzr, bnnz, bcols, amax, bmax,
                              true, stk));
    Tuning t = to_tuning(tuning);
    t.row_ncols = stk.rnc.ptr;
    const AView av{stk.As.rpt, stk.As.rows, stk.As.cols, stk.As.nzr};
    BRows bv;
    Temp<uint64_t> dense, need;
    Temp<uint32_t> work, cap;
    CLB_RETURN_IF(prepare_b(ctl, stk.Bs, dense, bv));
    CLB_RETURN_IF(work.alloc(ctl, anzr));
    CLB_RETURN_IF(cap.alloc(ctl, anzr));
    CLB_RETURN_IF(need.alloc(ctl, 1));
    CLB_TRY_CUDA(cudaMemsetAsync(need.ptr, 0, 8, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    const BatchRows br{stk.rpair.ptr, stk.pf.ptr};
    CLB_RETURN_IF(learned_caps(ctl, stk.As, stk.Bs, av, bv, sizer, margin_log2, slack, t, &br, work.ptr, cap.ptr));
    // the slots the capture form gives these capacities (16-byte groups)
    slot_need_kernel<<<std::max<unsigned>(1, std::min<uint64_t>((anzr + 255) / 256, ctl->sm_count * 8)), 256, 0,
                       ctl->stream>>>(cap.ptr, anzr, ~0ull, (unsigned long long *)need.ptr);
    CLB_CHECK_LAUNCH();
    CLB_RETURN_IF(read_scalars(ctl, need.ptr, slots_need, 1));
    return CLB_SUCCESS;
}

int clb_dcsr_union(clb_controls *ctl, uint32_t count, const clb_dcsr *mats, const clb_spgemm_tuning *tuning,
                   clb_dcsr *out, clb_spgemm_stats *stats) {
    if (!ctl || !out || (count && !mats)) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    if (count == 0) return fail(CLB_INVALID_ARGUMENT, "union of no matrices");
    if (count > 32) return fail(CLB_NOT_SUPPORTED, "union of more than 32 matrices in one call");
    CLB_RETURN_IF(check_tuning(tuning));
    const uint64_t n = mats[0].nrows, ncols = mats[0].ncols;
    for (uint32_t k = 1; k < count; ++k)
        if (mats[k].nrows != n || mats[k].ncols != ncols)
            return fail(CLB_INVALID_ARGUMENT, "union: matrix " + std::to_string(k) + " is " +
                                                  std::to_string(mats[k].nrows) + " x " +
                                                  std::to_string(mats[k].ncols) + ", matrix 0 is " +
                                                  std::to_string(n) + " x " + std::to_string(ncols));
    if ((uint64_t)count * n > 0xFFFFFFFFull) return fail(CLB_NOT_SUPPORTED, "union: count x nrows >= 2^32");
    clb_spgemm_stats st{};
    if (stats) *stats = st;
    std::vector<PairDesc> db(count);
    uint64_t bnzr = 0, bnnz = 0, bmax = 1;
    for (uint32_t k = 0; k < count; ++k) {
        const bool live = mats[k].nnz && mats[k].nzr;
        db[k] = PairDesc{mats[k].rpt, mats[k].rows, mats[k].cols, live ? mats[k].nzr : 0, live ? mats[k].nnz : 0,
                         bnzr, bnnz, (uint32_t)(k * n), 0u, (uint32_t)ncols};
        if (live) {
            bnzr += mats[k].nzr;
            bnnz += mats[k].nnz;
            bmax = std::max(bmax, std::max(mats[k].nnz, mats[k].nzr + 1));
        }
    }
    clb_dcsr C{};
    C.nrows = n;
    C.ncols = ncols;
    if (bnnz == 0) {
        *out = C;
        return CLB_SUCCESS;
    }
    DeviceGuard g(ctl);
    Temp<PairDesc> ddb;
    Temp<uint64_t> brpt, off, tot;
    Temp<uint32_t> brws, bcls, flags, cnt, pos;
    CLB_RETURN_IF(ddb.alloc(ctl, count));
    CLB_RETURN_IF(brpt.alloc(ctl, bnzr + 1));
    CLB_RETURN_IF(brws.alloc(ctl, bnzr));
    CLB_RETURN_IF(bcls.alloc(ctl, bnnz));
    CLB_RETURN_IF(flags.alloc(ctl, n));
    CLB_RETURN_IF(cnt.alloc(ctl, n));
    CLB_RETURN_IF(pos.alloc(ctl, n));
    CLB_RETURN_IF(off.alloc(ctl, n));
    CLB_RETURN_IF(tot.alloc(ctl, 2));
    CLB_TRY_CUDA(cudaMemcpyAsync(ddb.ptr, db.data(), count * sizeof(PairDesc), cudaMemcpyHostToDevice, ctl->stream),
                 CLB_WRITE_BUFFER_ERROR);
    CLB_TRY_CUDA(cudaMemsetAsync(flags.ptr, 0, n * 4, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    {
        ProfScope ps(ctl, "union_stack");
        stack_kernel<<<dim3(stack_grid_x(ctl, bmax, count), count), CAT_NT, 0, ctl->stream>>>(
            ddb.ptr, brpt.ptr, brws.ptr, bcls.ptr, nullptr, nullptr, bnzr, bnnz);
        const uint64_t rmax = std::max<uint64_t>(1, bmax);
        union_mark_kernel<<<dim3((unsigned)std::min<uint64_t>((rmax + 255) / 256, 4096), count), 256, 0,
                            ctl->stream>>>(ddb.ptr, flags.ptr);
        const unsigned g1 = (unsigned)std::min<uint64_t>((n + 255) / 256, (uint64_t)ctl->sm_count * 16);
        union_counts_kernel<<<g1, 256, 0, ctl->stream>>>(flags.ptr, n, cnt.ptr, pos.ptr);
        CLB_CHECK_LAUNCH();
    }
    CLB_RETURN_IF(scan_u32_to_u64(ctl, cnt.ptr, off.ptr, n, tot.ptr + 0));  // A_u column offsets, nnz(A_u)
    CLB_RETURN_IF(scan_u32_inplace(ctl, pos.ptr, n, tot.ptr + 1));          // A_u row positions, nzr(A_u)
    uint64_t h[2];
    CLB_RETURN_IF(read_scalars(ctl, tot.ptr, h, 2));
    const uint64_t annz = h[0], anzr = h[1];
    Temp<uint64_t> arpt;
    Temp<uint32_t> arws, acls;
    CLB_RETURN_IF(arpt.alloc(ctl, anzr + 1));
    CLB_RETURN_IF(arws.alloc(ctl, anzr));
    CLB_RETURN_IF(acls.alloc(ctl, annz));
    {
        const unsigned g1 = (unsigned)std::min<uint64_t>((n + 255) / 256, (uint64_t)ctl->sm_count * 16);
        union_left_kernel<<<g1, 256, 0, ctl->stream>>>(flags.ptr, off.ptr, pos.ptr, n, anzr, annz, arpt.ptr,
                                                      arws.ptr, acls.ptr);
        CLB_CHECK_LAUNCH();
    }
    flags.reset();
    cnt.reset();
    pos.reset();
    off.reset();
    const clb_dcsr Au{n, (uint64_t)count * n, annz, anzr, arpt.ptr, arws.ptr, acls.ptr};
    const clb_dcsr Bu{(uint64_t)count * n, ncols, bnnz, bnzr, brpt.ptr, brws.ptr, bcls.ptr};
    CLB_RETURN_IF(validate_spgemm(Au, Bu));
    const uint32_t launches = 5;
    CLB_RETURN_IF(spgemm_tuned(ctl, Au, Bu, tuning ? tuning->form : 1, to_tuning(tuning), &C, &st));
    st.kernel_launches += launches;
    if (stats) *stats = st;
    *out = C;
    return CLB_SUCCESS;
}

int clb_spgemm_autotune(clb_controls *ctl, uint32_t count, const clb_dcsr *a, const clb_dcsr *b,
                        clb_spgemm_tuning *best, clb_spgemm_tuning *tried, double *ms, uint32_t max_tried,
                        uint32_t *n_tried) {
    if (!ctl || !best) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    DeviceGuard g(ctl);
    std::vector<clb_spgemm_tuning> cand;
    uint64_t widest = 0;
    for (uint32_t k = 0; k < count; ++k) widest = std::max(widest, b[k].ncols);
    const std::vector<uint32_t> wides = widest > (1ull << CLB_CHUNK_SHIFT) ? std::vector<uint32_t>{2u, 1u}
                                                                            : std::vector<uint32_t>{2u};
    // pairs within one bitmap chunk also try the two-pass form keeping its
    // bitmaps (form 2); a single pair is timed through the plain tuned call
    const bool single = count == 1;
    const std::vector<uint32_t> forms =
        widest <= (1ull << CLB_CHUNK_SHIFT) ? std::vector<uint32_t>{0u, 1u, 2u} : std::vector<uint32_t>{0u, 1u};
    for (uint32_t wide : wides)
    for (uint32_t form : forms)
        for (uint32_t bmin : {4096u, 1024u})
            for (uint32_t bthr : {1024u, 256u})
                for (uint32_t wmax : {256u, 64u})
                    for (uint32_t small : {8u, 32u}) {
                        clb_spgemm_tuning t;
                        clb_spgemm_tuning_default(&t);
                        t.form = form;
                        t.bitmap_min = bmin;
                        t.bitmap_threads = bthr;
                        t.warp_max = wmax;
                        t.small_lanes = small;
                        t.wide_rows = wide;
                        cand.push_back(t);
                    }
    cudaEvent_t e0, e1;
    CLB_TRY_CUDA(cudaEventCreate(&e0), CLB_RUN_KERNEL_FAILURE);
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(CLB_RUN_KERNEL_FAILURE, "event");
    }
    std::vector<clb_dcsr> out(std::max<uint32_t>(count, 1));
    double best_ms = 1e300;
    int rc = CLB_SUCCESS;
    uint32_t n = 0;
    for (const auto &t : cand) {
        double tms = 1e300;
        // first run warms up; the best of three timed runs (one run alone let
        // candidates within 1% of each other swap places from call to call)
        for (int rep = 0; rep < 4 && rc == CLB_SUCCESS; ++rep) {
            cudaEventRecord(e0, ctl->stream);
            rc = single ? clb_dcsr_spgemm_tuned(ctl, a, b, &t, out.data(), nullptr)
                        : clb_dcsr_spgemm_batched(ctl, count, a, b, out.data(), &t, nullptr);
            cudaEventRecord(e1, ctl->stream);
            cudaEventSynchronize(e1);
            float f = 0.f;
            cudaEventElapsedTime(&f, e0, e1);
            for (uint32_t k = 0; k < count; ++k) clb_dcsr_release(ctl, &out[k]);
            if (rep > 0 && f < tms) tms = f;
        }
        if (rc != CLB_SUCCESS) break;
        if (n < max_tried) {
            if (tried) tried[n] = t;
            if (ms) ms[n] = tms;
        }
        ++n;
        if (tms < best_ms) {
            best_ms = tms;
            *best = t;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (n_tried) *n_tried = n;
    return rc;
}

}  // extern "C"
