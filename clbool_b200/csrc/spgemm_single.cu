// spgemm_single.cu -- single-pass SpGEMM forms: ESC/merge (dcsr::matrix_multiplication)
// and the learned-capacity form.
//
// Reference ESC form: src/dcsr/dcsr_matrix_multiplication.cpp:26-97 -- count the
// workload, bin rows by it, give every row its upper bound of slots in a
// "pre" matrix (build_groups_and_allocate_new_matrix, :319-375), run one
// numeric kernel per group (copy_one_value / heap_merge / bitonic_esc /
// merge_large_rows, :193-317), then compact into C (create_final_matrix,
// :100-168).
//
// Here both single-pass forms share one driver:
//   capacity[i] -> slots (scan) -> one numeric pass into the slots, every row
//   recording its exact count and flagging overflow -> overflowed rows
//   re-run by the exact two-pass form -> compaction into contiguous C.
// ESC form: capacity = min(products, ncols) (an exact upper bound, never
//   overflows); accumulators: warp ESC (<= 256 products), CTA ESC -- expand
//   into shared memory, bitonic sort, keep first of every run -- (<= 4096
//   products), bitmap (the rest).
// Learned form: capacity from the row-size predictor (mlp.cu); accumulators
//   binned by the capacity; rows whose count exceeds it are re-run exactly.
#include <string>

#include "spgemm.cuh"

namespace clb {

namespace {

// ------------------------------------------------------------ CTA ESC ----
// Rows with at most MERGE_SEGS A entries merge their sorted B rows pairwise
// instead of sorting all products: on R-MAT scale 20 the rows of 512..4096
// products have a median of 1 to 3 such entries (a single B row is already
// sorted and duplicate-free).
template <int NP, int NT>
__global__ void __launch_bounds__(NT) cta_esc_kernel(BinLists bl, int bin, AView a, BRows b, RowOut o,
                                                     const uint32_t *__restrict__ work, uint32_t *counter) {
    constexpr int SPT = NP / NT;
    __shared__ uint32_t keys[NP];
    __shared__ uint32_t keys2[NP];                   // merge ping-pong buffer
    __shared__ uint32_t s_sb[MERGE_SEGS + 1];        // segment bounds of the merges
    __shared__ uint32_t s_pre[HASH_ECH + 1];
    __shared__ uint32_t s_beg[HASH_ECH];
    __shared__ uint32_t scratch[33];
    __shared__ uint32_t s_slot, s_row;
    uint32_t beg, cnt;
    bin_range(bl, bin, beg, cnt);
    // Rows are claimed one ahead: the next claim (a global atomic) and its
    // row index are in flight while this row runs; thread 0 publishes them
    // at the row's end.
    if (threadIdx.x == 0) {
        const uint32_t it = atomicAdd(counter, 1u);
        s_slot = it;
        s_row = it < cnt ? bl.list[beg + it] : 0;
    }
    __syncthreads();
    for (;;) {
        const uint32_t item = s_slot;
        if (item >= cnt) break;
        const uint32_t i = s_row;
        uint32_t nxt = 0;  // thread 0: the next row's claim, read after the expansion
        if (threadIdx.x == 0) nxt = atomicAdd(counter, 1u);
        uint32_t P = work[i];
        if (P > (uint32_t)NP) {  // binning guarantees P <= NP
            if (threadIdx.x == 0) raise_status(o.status, DEV_BOUNDS);
            P = NP;
        }
        // expand: product idx of the row goes to keys[idx]
        balanced_products<NT, HASH_ECH, 4>(a, b, i, s_pre, s_beg, scratch, [&](uint32_t c, bool valid, uint32_t idx) {
            if (valid && idx < (uint32_t)NP) keys[idx] = c;
        });
        if (threadIdx.x == 0 && nxt < cnt) asm volatile("prefetch.global.L1 [%0];" ::"l"(bl.list + beg + nxt));
        const uint32_t *sorted = keys;
        if (a.rpt[i + 1] - a.rpt[i] <= MERGE_SEGS) {
            // few sorted B rows: pairwise merges
            sorted = merge_row_segments<NT, NP / NT>(a, b, i, P, keys, keys2, s_sb);
        } else {
            for (uint32_t s = P + threadIdx.x; s < (uint32_t)NP; s += NT) keys[s] = EMPTY;
            __syncthreads();
            // sort (register-resident bitonic stages, few block barriers)
            block_sort_hybrid<NT, NP / NT>(keys);
        }
        // compress: keep the first of every run (thread-contiguous segments)
        uint32_t v[SPT], flags = 0, mine = 0;
#pragma unroll
        for (int k = 0; k < SPT; ++k) {
            const uint32_t s = threadIdx.x * SPT + k;
            v[k] = s < P ? sorted[s] : EMPTY;
            const bool f = s < P && (s == 0 || v[k] != sorted[s - 1]);
            flags |= (f ? 1u : 0u) << k;
            mine += f ? 1u : 0u;
        }
        uint32_t nnz;
        uint32_t pos = block_exclusive_scan<uint32_t, NT>(mine, scratch, &nnz);
        if (o.row_cap && nnz > o.row_cap[i]) {
            if (threadIdx.x == 0) o.overflow[i] = 1;
        } else {
            uint32_t *dst = o.cols + o.row_off[i] + pos;
#pragma unroll
            for (int k = 0; k < SPT; ++k)
                if (flags & (1u << k)) *dst++ = v[k];
            if (threadIdx.x == 0) o.row_nnz[i] = nnz;
        }
        if (threadIdx.x == 0) {
            s_slot = nxt;
            s_row = nxt < cnt ? bl.list[beg + nxt] : 0;
        }
        __syncthreads();
    }
}

// capacity = min(products, ncols): the exact upper bound of a row's count.
__global__ void upper_bound_cap_kernel(const uint32_t *__restrict__ work, uint64_t n, uint64_t ncols,
                                       uint32_t *__restrict__ cap) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t p = work[i];
        cap[i] = (uint32_t)(p < ncols ? p : ncols);
    }
}

// The overflowed rows of A as their own DCSR (A'), plus pos[i] = index of
// row i in A' for overflowed rows.
__global__ void gather_rows_lengths_kernel(const uint32_t *__restrict__ ovf, const uint64_t *__restrict__ arpt, uint64_t n,
                                           uint32_t *__restrict__ len) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        len[i] = ovf[i] ? (uint32_t)(arpt[i + 1] - arpt[i]) : 0u;
}

__global__ void gather_rows_kernel(const uint32_t *__restrict__ ovf, const uint32_t *__restrict__ pos,
                                   const uint64_t *__restrict__ dst_off, const uint64_t *__restrict__ arpt,
                                   const uint32_t *__restrict__ arows, const uint32_t *__restrict__ acols, uint64_t n,
                                   uint64_t *__restrict__ sub_rpt, uint32_t *__restrict__ sub_rows,
                                   uint32_t *__restrict__ sub_cols, uint64_t sub_nzr, uint64_t sub_nnz) {
    const uint32_t lane = lane_id();
    const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x / 32);
    for (uint64_t i = (uint64_t)blockIdx.x * (blockDim.x / 32) + warp_id(); i < n; i += nw) {
        if (!ovf[i]) continue;
        const uint32_t k = pos[i];
        const uint64_t s = arpt[i], e = arpt[i + 1], d = dst_off[i];
        if (lane == 0) {
            sub_rpt[k] = d;
            sub_rows[k] = arows[i];
        }
        for (uint64_t j = s + lane; j < e; j += 32) sub_cols[d + (j - s)] = acols[j];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) sub_rpt[sub_nzr] = sub_nnz;
}

// Exact counts of the overflowed rows from the re-run product C'.
__global__ void fallback_counts_kernel(const uint32_t *__restrict__ ovf, const uint32_t *__restrict__ pos,
                                       const uint64_t *__restrict__ sub_crpt, uint64_t n, uint32_t *__restrict__ row_nnz) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (ovf[i]) row_nnz[i] = (uint32_t)(sub_crpt[pos[i] + 1] - sub_crpt[pos[i]]);
}

// Slot sizes: capacities rounded up to whole 16-byte groups, so every slot
// (and every spill reservation) starts 16-byte aligned; *sum = sum of the
// unrounded capacities.
__global__ void slot_sizes_kernel(const uint32_t *__restrict__ cap, uint64_t n, uint32_t *__restrict__ capp,
                                  unsigned long long *__restrict__ sum) {
    unsigned long long mine = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t c = cap[i];
        capp[i] = (c + 3u) & ~3u;
        mine += c;
    }
    mine = warp_sum(mine);
    if (lane_id() == 0 && mine) atomicAdd(sum, mine);
}

// Copies len words from a 16-byte aligned src to dst (any alignment), one
// warp: scalar head up to dst's 16-byte boundary, then 16-byte stores whose
// four words come from two aligned 16-byte loads joined at the head's offset,
// then a scalar tail.  Reads may run up to 3 words past src[len - 1] (inside
// the slot padding / the buffers' slack).
template <int SH>
__device__ __forceinline__ uint32_t join4(const uint4 &a, const uint4 &b, uint32_t k) {
    // words SH+k of the 8-word sequence a.x..a.w, b.x..b.w (k = 0..3)
    const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    return w[SH + k];
}

template <int SH>
__device__ __forceinline__ void copy_body(const uint4 *__restrict__ s4, uint4 *__restrict__ d4, uint64_t nq) {
    // d4[q] = words 4q+SH .. 4q+SH+3 of the aligned source
    const uint32_t lane = lane_id();
    for (uint64_t q = lane; q < nq; q += 32) {
        const uint4 a = __ldg(s4 + q);
        const uint4 b = SH ? __ldg(s4 + q + 1) : a;
        d4[q] = make_uint4(join4<SH>(a, b, 0), join4<SH>(a, b, 1), join4<SH>(a, b, 2), join4<SH>(a, b, 3));
    }
}

__device__ __forceinline__ void warp_copy_aligned_src(const uint32_t *__restrict__ src, uint32_t *__restrict__ dst,
                                                      uint64_t len) {
    const uint32_t lane = lane_id();
    const uint32_t head = (uint32_t)(((16u - (reinterpret_cast<uintptr_t>(dst) & 15u)) & 15u) >> 2);
    const uint64_t h = head < len ? head : len;
    if (lane < h) dst[lane] = src[lane];
    const uint64_t rest = len - h, nq = rest >> 2;
    uint4 *d4 = reinterpret_cast<uint4 *>(dst + h);
    const uint4 *s4 = reinterpret_cast<const uint4 *>(src);  // words from h on are s4 words h, h+1, ...
    switch (h & 3) {  // warp-uniform
        case 0: copy_body<0>(s4 + (h >> 2), d4, nq); break;
        case 1: copy_body<1>(s4, d4, nq); break;
        case 2: copy_body<2>(s4, d4, nq); break;
        default: copy_body<3>(s4, d4, nq); break;
    }
    for (uint64_t t = h + (nq << 2) + lane; t < len; t += 32) dst[t] = src[t];
}

// C.cols <- every row from its slot (or the spill arena, both 16-byte
// aligned: vector copy), or from C' for recomputed rows (scalar copy),
// except the deferred bitmap rows.  One warp per row.
__global__ void compact_rows_kernel(const uint32_t *__restrict__ row_nnz, const uint64_t *__restrict__ slot_off,
                                    const uint64_t *__restrict__ off, const uint32_t *__restrict__ pre,
                                    const uint32_t *__restrict__ ovf, const uint32_t *__restrict__ pos,
                                    const uint64_t *__restrict__ sub_crpt, const uint32_t *__restrict__ sub_ccols,
                                    const uint64_t *__restrict__ spill, const uint32_t *__restrict__ arena,
                                    const uint32_t *__restrict__ defer, uint64_t n, uint32_t *__restrict__ ccols) {
    const uint32_t lane = lane_id();
    const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x / 32);
    for (uint64_t i = (uint64_t)blockIdx.x * (blockDim.x / 32) + warp_id(); i < n; i += nw) {
        const uint32_t len = row_nnz[i];
        if (!len || (defer && defer[i])) continue;  // deferred rows: the expansion kernels
        uint32_t *dst = ccols + off[i];
        if (ovf && ovf[i]) {
            const uint32_t *src = sub_ccols + sub_crpt[pos[i]];
            for (uint32_t t = lane; t < len; t += 32) dst[t] = __ldg(src + t);
            continue;
        }
        const uint64_t sp = spill ? spill[i] : ~0ull;
        warp_copy_aligned_src(sp != ~0ull ? arena + sp : pre + slot_off[i], dst, len);
    }
}

// Number of overflowed rows (nonzero ovf) and of spilled rows (spill != ~0).
__global__ void count_rows_kernel(const uint32_t *__restrict__ ovf, const uint64_t *__restrict__ spill, uint64_t n,
                                  unsigned long long *__restrict__ out) {
    unsigned long long mine = 0, sp = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        mine += ovf[i] != 0;
        if (spill) sp += spill[i] != ~0ull;
    }
    mine = warp_sum(mine);
    sp = warp_sum(sp);
    if (lane_id() == 0 && mine) atomicAdd(out, mine);
    if (lane_id() == 0 && sp) atomicAdd(out + 1, sp);
}

template <class K>
int occupancy_of(K kernel, int nt) {
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, nt, 0) != cudaSuccess) {
        cudaGetLastError();
        blocks = 1;
    }
    return blocks > 0 ? blocks : 1;
}

template <int NP, int NT>
int launch_cta_esc(clb_controls *ctl, const BinLists &bl, int bin, const AView &a, const BRows &b, const RowOut &o,
                   const uint32_t *work, uint64_t nmax, uint32_t *counter, const char *name) {
    static int occ = occupancy_of(cta_esc_kernel<NP, NT>, NT);
    unsigned grid = persistent_grid(ctl, occ, nmax);
    ProfScope ps(ctl, name);
    cta_esc_kernel<NP, NT><<<grid, NT, 0, ctl->stream>>>(bl, bin, a, b, o, work, counter);
    ctl->launches += 1;
    CLB_CHECK_LAUNCH();
    return CLB_SUCCESS;
}

unsigned grid_for(const clb_controls *ctl, uint64_t n, int per_sm = 16) {
    uint64_t g = (n + 255) / 256, cap = (uint64_t)ctl->sm_count * per_sm;
    return (unsigned)(g > cap ? cap : (g ? g : 1));
}

}  // namespace

int launch_upper_bound_caps(clb_controls *ctl, const uint32_t *work, uint64_t n, uint64_t ncols, uint32_t *cap) {
    upper_bound_cap_kernel<<<grid_for(ctl, n), 256, 0, ctl->stream>>>(work, n, ncols, cap);
    ctl->launches += 1;
    CLB_CHECK_LAUNCH();
    return CLB_SUCCESS;
}

// The accumulators of the ESC form for rows of up to 4096 products.
int launch_esc_accumulators(clb_controls *ctl, const BinLists &bl, const AView &a, const BRows &b, const RowOut &o,
                            const uint32_t *work, uint64_t nmax, const uint32_t *hc) {
    Temp<uint32_t> ctr;
    CLB_RETURN_IF(ctr.alloc(ctl, 4));
    CLB_TRY_CUDA(cudaMemsetAsync(ctr.ptr, 0, 4 * sizeof(uint32_t), ctl->stream), CLB_RUN_KERNEL_FAILURE);
    auto rows = [&](int bin) -> uint64_t { return hc ? hc[bin] : nmax; };
    if (rows(BIN_H8K))
        CLB_RETURN_IF((launch_cta_esc<4096, 512>(ctl, bl, BIN_H8K, a, b, o, work, rows(BIN_H8K), ctr.ptr + 0,
                                                 "cta_esc4096")));
    if (rows(BIN_H4K))
        CLB_RETURN_IF((launch_cta_esc<2048, 128>(ctl, bl, BIN_H4K, a, b, o, work, rows(BIN_H4K), ctr.ptr + 1,
                                                 "cta_esc2048")));
    if (rows(BIN_H2K))
        CLB_RETURN_IF((launch_cta_esc<1024, 128>(ctl, bl, BIN_H2K, a, b, o, work, rows(BIN_H2K), ctr.ptr + 2,
                                                 "cta_esc1024")));
    if (rows(BIN_H1K))
        CLB_RETURN_IF((launch_cta_esc<512, 128>(ctl, bl, BIN_H1K, a, b, o, work, rows(BIN_H1K), ctr.ptr + 3,
                                                "cta_esc512")));
    return CLB_SUCCESS;
}

// Single-pass driver.  `cap` (device, nzr_A entries) = capacity per A row; the
// ESC form passes the upper bound, the learned form the predicted capacity.
// `esc` selects the ESC accumulators for rows of <= 4096 products and bins
// those rows by products; otherwise rows are binned by capacity and use the
// hash accumulators.
int spgemm_single_pass(clb_controls *ctl, const clb_dcsr &A, const clb_dcsr &B, const AView &a, const BRows &b_in,
                       const uint32_t *work, uint32_t *cap, bool esc, uint64_t products, clb_dcsr *out,
                       clb_spgemm_stats *st, uint64_t arena_div, const Tuning &t) {
    const uint64_t n = A.nzr;
    clb_dcsr C{};
    C.nrows = A.nrows;
    C.ncols = B.ncols;
    Temp<uint32_t> list, info, flags, row_nnz, ovf, opos;
    Temp<uint64_t> slot_off, off, scal;
    CLB_RETURN_IF(list.alloc(ctl, n));
    CLB_RETURN_IF(info.alloc(ctl, 2 * NUM_BINS));
    CLB_RETURN_IF(flags.alloc(ctl, n));
    CLB_RETURN_IF(row_nnz.alloc(ctl, n));
    CLB_RETURN_IF(ovf.alloc(ctl, n));
    CLB_RETURN_IF(slot_off.alloc(ctl, n));
    CLB_RETURN_IF(off.alloc(ctl, n));
    CLB_RETURN_IF(scal.alloc(ctl, 8));
    CLB_TRY_CUDA(cudaMemsetAsync(scal.ptr, 0, 8 * sizeof(uint64_t), ctl->stream), CLB_RUN_KERNEL_FAILURE);
    CLB_TRY_CUDA(cudaMemsetAsync(row_nnz.ptr, 0, n * 4, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    CLB_TRY_CUDA(cudaMemsetAsync(ovf.ptr, 0, n * 4, ctl->stream), CLB_RUN_KERNEL_FAILURE);

    // bins: ESC by products (CTA ESC up to 4096), learned by capacity
    CLB_RETURN_IF(launch_binning(ctl, work, esc ? work : cap, n, B.ncols, info.ptr, list.ptr, flags.ptr, t));
    CLB_RETURN_IF(scan_u32_inplace(ctl, flags.ptr, n, scal.ptr + 0));        // C row positions, nzr
    // slots: capacities rounded up to 16-byte groups (aligned slot starts)
    Temp<uint32_t> capp;
    CLB_RETURN_IF(capp.alloc(ctl, n));
    slot_sizes_kernel<<<grid_for(ctl, n), 256, 0, ctl->stream>>>(cap, n, capp.ptr,
                                                                 (unsigned long long *)(scal.ptr + 7));
    ctl->launches += 1;
    CLB_CHECK_LAUNCH();
    CLB_RETURN_IF(scan_u32_to_u64(ctl, capp.ptr, slot_off.ptr, n, scal.ptr + 1));  // slot offsets, slots
    uint64_t h[2], capacity = 0;
    uint32_t hinfo[NUM_BINS];  // rows per bin: only bins with rows are launched
    const SmallRead rd[3] = {{scal.ptr, h, sizeof(h)}, {scal.ptr + 7, &capacity, sizeof(capacity)},
                             {info.ptr, hinfo, sizeof(hinfo)}};
    CLB_RETURN_IF(read_small_multi(ctl, rd, 3));
    const uint64_t nzr = h[0], slots = h[1];
    BRows b = b_in;
    Temp<uint64_t> wdense;
    Temp<uint2> wpairs;
    CLB_RETURN_IF(prepare_b_words(ctl, B, hinfo, wdense, wpairs, b, products));
    if (st) {
        for (int k = 0; k < NUM_BINS; ++k) st->rows_per_bin[k] = hinfo[k];
        st->capacity = capacity;
    }
    Temp<uint32_t> pre;  // + 4 words: the vector copy may read up to 3 words past a slot
    CLB_RETURN_IF(pre.alloc(ctl, slots + 4));

    BinLists bl{list.ptr, info.ptr};
    RowOut num{row_nnz.ptr, slot_off.ptr, cap, ovf.ptr, pre.ptr, ctl->d_status};
    num.row_ncols = t.row_ncols;
    num.row_products = work;
    // bitmap rows denser than their bitmap keep the bitmap in their slot
    // (without room for the row flags every row is emitted in place)
    const uint64_t nbmp = (uint64_t)hinfo[BIN_BMP_XL] + hinfo[BIN_BMP_L] + hinfo[BIN_BMP];
    Temp<uint32_t> defer, dlist, dcount, dsteps;
    const bool deferring =
        nbmp && defer.try_alloc(ctl, n) && dlist.try_alloc(ctl, nbmp) && dcount.try_alloc(ctl, 1);
    if (deferring) {
        CLB_TRY_CUDA(cudaMemsetAsync(defer.ptr, 0, n * 4, ctl->stream), CLB_RUN_KERNEL_FAILURE);
        CLB_TRY_CUDA(cudaMemsetAsync(dcount.ptr, 0, 4, ctl->stream), CLB_RUN_KERNEL_FAILURE);
        num.defer = defer.ptr;
        num.defer_list = dlist.ptr;
        num.defer_count = dcount.ptr;
        // step records for the by-step expansion (without room for them the
        // rows are expanded a row per CTA)
        if (dsteps.try_alloc(ctl, nbmp * BMP_STEP_REC)) num.defer_steps = dsteps.ptr;
    } else {
        defer.reset();
    }
    // spill arena for single-chunk bitmap rows over their capacity
    Temp<uint64_t> spill;
    Temp<uint32_t> arena;
    if (arena_div) {
        uint64_t acap = capacity / arena_div;
        if (acap < (1ull << 24)) acap = 1ull << 24;
        CLB_RETURN_IF(spill.alloc(ctl, n));
        CLB_RETURN_IF(arena.alloc(ctl, acap + 4));
        CLB_TRY_CUDA(cudaMemsetAsync(spill.ptr, 0xFF, n * 8, ctl->stream), CLB_RUN_KERNEL_FAILURE);
        num.spill = spill.ptr;
        num.arena = arena.ptr;
        num.arena_cursor = (unsigned long long *)(scal.ptr + 6);
        num.arena_cap = acap;
    }
    if (esc) {
        // warp ESC and bitmap rows through the shared launcher's bins; rows of
        // the hash bins go to the CTA ESC kernels instead.
        CLB_RETURN_IF(launch_esc_accumulators(ctl, bl, a, b, num, work, n, hinfo));
        CLB_RETURN_IF(launch_accumulators_subset(ctl, bl, a, b, num, B.ncols, n, /*hash_bins=*/false, t, hinfo));
    } else {
        CLB_RETURN_IF(launch_accumulators(ctl, true, bl, a, b, num, B.ncols, n, t, hinfo));
    }

    // the fallback below resets the device status word: check it first
    CLB_RETURN_IF(check_status(ctl, esc ? "matrix_multiplication" : "matrix_multiplication_learned"));
    // rows that outgrew their capacity: re-run them with the exact two-pass form
    unsigned long long *d_novf = (unsigned long long *)(scal.ptr + 2);  // [2] overflowed, [3] spilled
    count_rows_kernel<<<grid_for(ctl, n), 256, 0, ctl->stream>>>(ovf.ptr, spill.ptr, n, d_novf);
    ctl->launches += 1;
    CLB_CHECK_LAUNCH();
    uint64_t cnts[2] = {0, 0};
    CLB_RETURN_IF(read_scalars(ctl, scal.ptr + 2, cnts, 2));
    const uint64_t novf = cnts[0];
    if (st) {
        st->fallback_rows = novf;
        st->spilled_rows = cnts[1];
    }
    clb_dcsr sub_c{};
    Temp<uint64_t> sub_rpt, sub_off;
    Temp<uint32_t> sub_rows, sub_cols, sub_len;
    if (novf) {
        CLB_RETURN_IF(opos.alloc(ctl, n));
        CLB_RETURN_IF(sub_len.alloc(ctl, n));
        CLB_RETURN_IF(sub_off.alloc(ctl, n));
        CLB_TRY_CUDA(cudaMemcpyAsync(opos.ptr, ovf.ptr, n * 4, cudaMemcpyDeviceToDevice, ctl->stream),
                     CLB_COPY_BUFFER_ERROR);
        CLB_RETURN_IF(scan_u32_inplace(ctl, opos.ptr, n, scal.ptr + 3));
        gather_rows_lengths_kernel<<<grid_for(ctl, n), 256, 0, ctl->stream>>>(ovf.ptr, A.rpt, n, sub_len.ptr);
        ctl->launches += 1;
        CLB_CHECK_LAUNCH();
        CLB_RETURN_IF(scan_u32_to_u64(ctl, sub_len.ptr, sub_off.ptr, n, scal.ptr + 4));
        uint64_t sub_nnz = 0;
        CLB_RETURN_IF(read_scalars(ctl, scal.ptr + 4, &sub_nnz, 1));
        CLB_RETURN_IF(sub_rpt.alloc(ctl, novf + 1));
        CLB_RETURN_IF(sub_rows.alloc(ctl, novf));
        CLB_RETURN_IF(sub_cols.alloc(ctl, sub_nnz ? sub_nnz : 1));
        gather_rows_kernel<<<grid_for(ctl, n * 32), 256, 0, ctl->stream>>>(ovf.ptr, opos.ptr, sub_off.ptr, A.rpt,
                                                                           A.rows, A.cols, n, sub_rpt.ptr,
                                                                           sub_rows.ptr, sub_cols.ptr, novf, sub_nnz);
        ctl->launches += 1;
        CLB_CHECK_LAUNCH();
        clb_dcsr subA{A.nrows, A.ncols, sub_nnz, novf, sub_rpt.ptr, sub_rows.ptr, sub_cols.ptr};
        const uint32_t launches = ctl->launches;
        Tuning tf = t;
        tf.row_ncols = nullptr;  // indexed by the rows of A, not of the gathered A'
        CLB_RETURN_IF(spgemm_hash_two_pass(ctl, subA, B, &sub_c, nullptr, tf));
        ctl->launches += launches;
        if (sub_c.nzr != novf) {
            clb_dcsr_release(ctl, &sub_c);
            return fail(CLB_RUN_KERNEL_FAILURE, "fallback rows lost their products");
        }
        fallback_counts_kernel<<<grid_for(ctl, n), 256, 0, ctl->stream>>>(ovf.ptr, opos.ptr, sub_c.rpt, n,
                                                                           row_nnz.ptr);
        ctl->launches += 1;
        CLB_CHECK_LAUNCH();
    }

    // final layout
    CLB_RETURN_IF(scan_u32_to_u64(ctl, row_nnz.ptr, off.ptr, n, scal.ptr + 5));
    uint64_t nnz = 0;
    CLB_RETURN_IF(read_scalars(ctl, scal.ptr + 5, &nnz, 1));
    int rc = CLB_SUCCESS;
    Temp<uint64_t> c_rpt;
    Temp<uint32_t> c_rows, c_cols;
    if (nnz) {
        rc = c_rpt.alloc(ctl, nzr + 1);
        if (rc == CLB_SUCCESS) rc = c_rows.alloc(ctl, nzr);
        if (rc == CLB_SUCCESS) rc = c_cols.alloc(ctl, nnz);
        if (rc == CLB_SUCCESS)
            rc = launch_assemble(ctl, work, flags.ptr, off.ptr, A.rows, n, c_rpt.ptr, c_rows.ptr, nzr, nnz);
        if (rc == CLB_SUCCESS) {
            ProfScope ps(ctl, "compact");
            compact_rows_kernel<<<grid_for(ctl, n * 32, 32), 256, 0, ctl->stream>>>(
                row_nnz.ptr, slot_off.ptr, off.ptr, pre.ptr, novf ? ovf.ptr : nullptr, opos.ptr, sub_c.rpt,
                sub_c.cols, spill.ptr, arena.ptr, defer.ptr, n, c_cols.ptr);
            ctl->launches += 1;
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) rc = fail(CLB_RUN_KERNEL_FAILURE, cudaGetErrorString(e));
        }
        if (rc == CLB_SUCCESS && deferring && dsteps.ptr)
            rc = launch_bitmap_expand_steps(ctl, dlist.ptr, dcount.ptr, dsteps.ptr, slot_off.ptr, pre.ptr, off.ptr,
                                            c_cols.ptr);
        else if (rc == CLB_SUCCESS && deferring)
            rc = launch_bitmap_expand(ctl, dlist.ptr, dcount.ptr, nbmp, slot_off.ptr, pre.ptr, off.ptr, t.row_ncols,
                                      B.ncols, c_cols.ptr);
    }
    if (rc == CLB_SUCCESS) rc = check_status(ctl, esc ? "matrix_multiplication" : "matrix_multiplication_learned");
    if (sub_c.rpt) clb_dcsr_release(ctl, &sub_c);
    if (rc != CLB_SUCCESS) return rc;
    if (nnz) {
        C.nnz = nnz;
        C.nzr = nzr;
        C.rpt = c_rpt.release_ownership();
        C.rows = c_rows.release_ownership();
        C.cols = c_cols.release_ownership();
    }
    if (st) {
        st->products = products;
        st->nnz = nnz;
        st->nzr = C.nzr;
    }
    *out = C;
    return CLB_SUCCESS;
}

namespace {

// cap[i] = min(work[i], columns of row i's product) (row_ncols: per stacked
// row, from its pair; null = ncols).
__global__ void upper_bound_cap_rows_kernel(const uint32_t *__restrict__ work, uint64_t n, uint64_t ncols,
                                            const uint32_t *__restrict__ row_ncols, uint32_t *__restrict__ cap) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = row_ncols ? (uint64_t)row_ncols[i] : ncols;
        cap[i] = (uint32_t)min((uint64_t)work[i], c);
    }
}

// Rows whose slot would end past the caller's slot capacity get capacity 0:
// every accumulator then flags them as overflowed instead of writing.
__global__ void fit_slots_kernel(const uint64_t *__restrict__ slot_off, const uint32_t *__restrict__ capp, uint64_t n,
                                 uint64_t limit, uint32_t *__restrict__ cap, uint32_t *__restrict__ flags) {
    bool cut = false;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (slot_off[i] + capp[i] > limit) {
            cap[i] = 0;
            cut = true;
        }
    }
    if (__any_sync(0xFFFFFFFFu, cut) && lane_id() == 0) atomicOr(flags, CAPTURE_SLOTS_FULL);
}

// Overflowed rows keep no columns and raise `bit` in the flag word.  With
// upper-bound slots only rows cut by fit_slots_kernel can overflow; with
// learned slots also a row that outgrew its slot when the arena was full.
__global__ void drop_overflow_kernel(const uint32_t *__restrict__ ovf, uint64_t n, uint32_t *__restrict__ row_nnz,
                                     uint32_t *__restrict__ flags, uint32_t bit) {
    bool any = false;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (ovf[i]) {
            row_nnz[i] = 0;
            any = true;
        }
    }
    if (__any_sync(0xFFFFFFFFu, any) && lane_id() == 0) atomicOr(flags, bit);
}

// C.rpt / C.rows with sizes read on the device (nzr = *d_nzr, nnz = *d_nnz):
// row ids are made local to their pair (first[k] = first stacked row of
// pair k, row_base[k] = its row-id offset; count pairs).
__global__ void assemble_capture_kernel(const uint32_t *__restrict__ work, const uint32_t *__restrict__ pos,
                                        const uint64_t *__restrict__ off, const uint32_t *__restrict__ a_rows,
                                        uint64_t n, const uint64_t *__restrict__ first,
                                        const uint32_t *__restrict__ row_base, uint32_t count,
                                        const uint64_t *__restrict__ d_nzr, const uint64_t *__restrict__ d_nnz,
                                        uint64_t *__restrict__ c_rpt, uint32_t *__restrict__ c_rows) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (work[i] > 0) {
            uint32_t lo = 0, hi = count;  // last k with first[k] <= i
            while (hi - lo > 1) {
                const uint32_t m = (lo + hi) / 2;
                if (first[m] <= i) lo = m; else hi = m;
            }
            const uint32_t p = pos[i];
            c_rpt[p] = off[i];
            c_rows[p] = a_rows[i] - row_base[lo];
        }
        if (i == 0) c_rpt[*d_nzr] = *d_nnz;
    }
}

// Per-pair bounds: out[k] = first C row of pair k, out[count + 1 + k] = its
// first column position (k = count: the totals).
__global__ void capture_bounds_kernel(const uint32_t *__restrict__ pos, const uint64_t *__restrict__ off, uint64_t n,
                                      const uint64_t *__restrict__ first, uint32_t count,
                                      const uint64_t *__restrict__ d_nzr, const uint64_t *__restrict__ d_nnz,
                                      uint64_t *__restrict__ out) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k <= count; k += gridDim.x * blockDim.x) {
        const uint64_t f = k < count ? first[k] : n;
        out[k] = f < n ? (uint64_t)pos[f] : *d_nzr;
        out[count + 1 + k] = f < n ? off[f] : *d_nnz;
    }
}

// Compaction into the caller's column buffer (from the row's slot, or from
// the spill arena for spilled rows: spill[i] != ~0); rows past its capacity
// are not written and flag the call.
__global__ void compact_capture_kernel(const uint32_t *__restrict__ row_nnz, const uint64_t *__restrict__ slot_off,
                                       const uint64_t *__restrict__ off, const uint32_t *__restrict__ pre,
                                       const uint64_t *__restrict__ spill, const uint32_t *__restrict__ arena,
                                       uint64_t n, uint64_t cols_cap, uint32_t *__restrict__ ccols,
                                       uint32_t *__restrict__ flags) {
    const uint32_t lane = lane_id();
    const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x / 32);
    for (uint64_t i = (uint64_t)blockIdx.x * (blockDim.x / 32) + warp_id(); i < n; i += nw) {
        const uint32_t len = row_nnz[i];
        if (!len) continue;
        if (off[i] + len > cols_cap) {
            if (lane == 0) atomicOr(flags, CAPTURE_COLS_FULL);
            continue;
        }
        const uint64_t sp = spill ? spill[i] : ~0ull;
        warp_copy_aligned_src(sp != ~0ull ? arena + sp : pre + slot_off[i], ccols + off[i], len);
    }
}

// Device check failures of the accumulators (the controls' status word).
__global__ void capture_status_kernel(const uint32_t *__restrict__ status, uint32_t *__restrict__ flags) {
    if (threadIdx.x == 0 && *status) atomicOr(flags, CAPTURE_DEVICE_CHECK);
}

}  // namespace

int spgemm_esc_capture(clb_controls *ctl, const clb_dcsr &A, const clb_dcsr &B, const Tuning &t,
                       uint64_t slot_capacity, const uint64_t *first, const uint32_t *row_base, uint32_t count,
                       uint64_t *c_rpt, uint32_t *c_rows, uint32_t *c_cols, uint64_t cols_capacity,
                       uint64_t *d_result, uint32_t *d_flags, const CaptureLearned *learned) {
    const uint64_t n = A.nzr;
    const AView a{A.rpt, A.rows, A.cols, A.nzr};
    BRows b;
    Temp<uint64_t> dense;
    CLB_RETURN_IF(prepare_b(ctl, B, dense, b));
    Temp<uint32_t> work, cap, capp, list, info, flags, row_nnz, ovf, pre;
    Temp<uint64_t> slot_off, off, scal;
    CLB_RETURN_IF(work.alloc(ctl, n));
    CLB_RETURN_IF(cap.alloc(ctl, n));
    CLB_RETURN_IF(capp.alloc(ctl, n));
    CLB_RETURN_IF(list.alloc(ctl, n));
    CLB_RETURN_IF(info.alloc(ctl, 2 * NUM_BINS));
    CLB_RETURN_IF(flags.alloc(ctl, n));
    CLB_RETURN_IF(row_nnz.alloc(ctl, n));
    CLB_RETURN_IF(ovf.alloc(ctl, n));
    CLB_RETURN_IF(slot_off.alloc(ctl, n));
    CLB_RETURN_IF(off.alloc(ctl, n));
    CLB_RETURN_IF(scal.alloc(ctl, 8));
    CLB_RETURN_IF(pre.alloc(ctl, slot_capacity + 4));  // + 4: the vector copy reads up to 3 words past a slot
    CLB_TRY_CUDA(cudaMemsetAsync(scal.ptr, 0, 8 * sizeof(uint64_t), ctl->stream), CLB_RUN_KERNEL_FAILURE);
    CLB_TRY_CUDA(cudaMemsetAsync(row_nnz.ptr, 0, n * 4, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    CLB_TRY_CUDA(cudaMemsetAsync(ovf.ptr, 0, n * 4, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    if (learned) {
        // learned slots for the rows over t.bitmap_min products, exact below
        CLB_RETURN_IF(learned_caps(ctl, A, B, a, b, learned->sizer, learned->margin_log2, learned->slack, t,
                                   &learned->batch, work.ptr, cap.ptr));
    } else {
        CLB_RETURN_IF(launch_workload(ctl, a, b, work.ptr, scal.ptr + 6));
        upper_bound_cap_rows_kernel<<<grid_for(ctl, n), 256, 0, ctl->stream>>>(work.ptr, n, B.ncols, t.row_ncols,
                                                                               cap.ptr);
        ctl->launches += 1;
        CLB_CHECK_LAUNCH();
    }
    CLB_RETURN_IF(launch_binning(ctl, work.ptr, work.ptr, n, B.ncols, info.ptr, list.ptr, flags.ptr, t));
    CLB_RETURN_IF(scan_u32_inplace(ctl, flags.ptr, n, scal.ptr + 0));  // C row positions, nzr
    slot_sizes_kernel<<<grid_for(ctl, n), 256, 0, ctl->stream>>>(cap.ptr, n, capp.ptr,
                                                                 (unsigned long long *)(scal.ptr + 7));
    CLB_RETURN_IF(scan_u32_to_u64(ctl, capp.ptr, slot_off.ptr, n, scal.ptr + 1));
    fit_slots_kernel<<<grid_for(ctl, n), 256, 0, ctl->stream>>>(slot_off.ptr, capp.ptr, n, slot_capacity, cap.ptr,
                                                                d_flags);
    ctl->launches += 2;
    CLB_CHECK_LAUNCH();
    const BinLists bl{list.ptr, info.ptr};
    RowOut num{row_nnz.ptr, slot_off.ptr, cap.ptr, ovf.ptr, pre.ptr, ctl->d_status};
    num.row_ncols = t.row_ncols;
    num.row_products = work.ptr;
    // learned slots: a bitmap row over its slot reserves its exact count in
    // the caller-sized spill arena (the cursor is cleared with scal)
    Temp<uint64_t> spill;
    Temp<uint32_t> arena;
    if (learned) {
        CLB_RETURN_IF(spill.alloc(ctl, n));
        CLB_RETURN_IF(arena.alloc(ctl, learned->arena_capacity + 4));
        CLB_TRY_CUDA(cudaMemsetAsync(spill.ptr, 0xFF, n * 8, ctl->stream), CLB_RUN_KERNEL_FAILURE);
        num.spill = spill.ptr;
        num.arena = arena.ptr;
        num.arena_cursor = (unsigned long long *)(scal.ptr + 3);
        num.arena_cap = learned->arena_capacity;
    }
    // every bin is launched (no host read of the bin sizes); empty ones exit at once
    CLB_RETURN_IF(launch_esc_accumulators(ctl, bl, a, b, num, work.ptr, n, nullptr));
    CLB_RETURN_IF(launch_accumulators_subset(ctl, bl, a, b, num, B.ncols, n, /*hash_bins=*/false, t, nullptr));
    drop_overflow_kernel<<<grid_for(ctl, n), 256, 0, ctl->stream>>>(ovf.ptr, n, row_nnz.ptr, d_flags,
                                                                    learned ? CAPTURE_ROW_OVERFLOW : CAPTURE_SLOTS_FULL);
    ctl->launches += 1;
    CLB_CHECK_LAUNCH();
    CLB_RETURN_IF(scan_u32_to_u64(ctl, row_nnz.ptr, off.ptr, n, scal.ptr + 5));  // C row offsets, nnz
    const unsigned g = persistent_grid(ctl, 8, ceil_div_u(n, 256));
    assemble_capture_kernel<<<g, 256, 0, ctl->stream>>>(work.ptr, flags.ptr, off.ptr, A.rows, n, first, row_base,
                                                        count, scal.ptr + 0, scal.ptr + 5, c_rpt, c_rows);
    capture_bounds_kernel<<<(count + 256) / 256, 256, 0, ctl->stream>>>(flags.ptr, off.ptr, n, first, count,
                                                                        scal.ptr + 0, scal.ptr + 5, d_result + 2);
    compact_capture_kernel<<<grid_for(ctl, n * 32, 32), 256, 0, ctl->stream>>>(
        row_nnz.ptr, slot_off.ptr, off.ptr, pre.ptr, spill.ptr, arena.ptr, n, cols_capacity, c_cols, d_flags);
    capture_status_kernel<<<1, 32, 0, ctl->stream>>>(ctl->d_status, d_flags);
    ctl->launches += 4;
    CLB_CHECK_LAUNCH();
    CLB_TRY_CUDA(cudaMemcpyAsync(d_result, scal.ptr + 0, 8, cudaMemcpyDeviceToDevice, ctl->stream),
                 CLB_COPY_BUFFER_ERROR);
    CLB_TRY_CUDA(cudaMemcpyAsync(d_result + 1, scal.ptr + 5, 8, cudaMemcpyDeviceToDevice, ctl->stream),
                 CLB_COPY_BUFFER_ERROR);
    return CLB_SUCCESS;
}

}  // namespace clb

using namespace clb;

extern "C" {

int clb_dcsr_spgemm_esc(clb_controls *ctl, const clb_dcsr *a_, const clb_dcsr *b_, clb_dcsr *c,
                        clb_spgemm_stats *stats) {
    if (!ctl || !a_ || !b_ || !c) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    const clb_dcsr A = *a_, B = *b_;
    CLB_RETURN_IF(validate_spgemm(A, B));
    DeviceGuard g(ctl);
    clb_spgemm_stats st{};
    ctl->launches = 0;
    if (A.nnz == 0 || B.nnz == 0 || A.nzr == 0 || B.nzr == 0) {
        clb_dcsr C{};
        C.nrows = A.nrows;
        C.ncols = B.ncols;
        *c = C;
        if (stats) *stats = st;
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
    int rc = spgemm_single_pass(ctl, A, B, a, b, work.ptr, cap.ptr, true, products, c, &st, 0);
    st.kernel_launches = ctl->launches;
    if (stats) *stats = st;
    return rc;
}

}  // extern "C"
