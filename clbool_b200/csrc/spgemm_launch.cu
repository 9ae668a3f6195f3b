// spgemm_launch.cu -- binning, C assembly and accumulator launches.
#include <mutex>

#include "spgemm.cuh"

namespace clb {

namespace {

constexpr int BIN_NT = 256;

__global__ void __launch_bounds__(BIN_NT) bin_count_kernel(const uint32_t *__restrict__ work,
                                                           const uint32_t *__restrict__ cap, uint64_t n, uint64_t ncols,
                                                           uint32_t warp_max, uint32_t bitmap_min, uint32_t small,
                                                           uint32_t *__restrict__ info, uint32_t *__restrict__ flags) {
    __shared__ uint32_t hist[NUM_BINS];
    if (threadIdx.x < NUM_BINS) hist[threadIdx.x] = 0;
    __syncthreads();
    for (uint64_t i = (uint64_t)blockIdx.x * BIN_NT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * BIN_NT) {
        uint32_t p = work[i];
        uint64_t bound = cap ? (uint64_t)cap[i] : (p < ncols ? (uint64_t)p : ncols);
        int bin = bin_of(p, bound, warp_max, bitmap_min, small);
        atomicAdd(&hist[bin], 1u);
        flags[i] = p > 0 ? 1u : 0u;
    }
    __syncthreads();
    if (threadIdx.x < NUM_BINS && hist[threadIdx.x]) atomicAdd(&info[threadIdx.x], hist[threadIdx.x]);
}

__global__ void __launch_bounds__(BIN_NT) bin_scatter_kernel(const uint32_t *__restrict__ work,
                                                             const uint32_t *__restrict__ cap, uint64_t n,
                                                             uint64_t ncols, uint32_t warp_max, uint32_t bitmap_min,
                                                             uint32_t small, uint32_t *__restrict__ info,
                                                             uint32_t *__restrict__ list) {
    __shared__ uint32_t boff[NUM_BINS];
    if (threadIdx.x == 0) {
        uint32_t o = 0;
        boff[0] = 0;
        for (int b = 1; b < NUM_BINS; ++b) {
            boff[b] = o;
            o += info[b];
        }
    }
    __syncthreads();
    for (uint64_t i0 = (uint64_t)blockIdx.x * BIN_NT; i0 < n; i0 += (uint64_t)gridDim.x * BIN_NT) {
        uint64_t i = i0 + threadIdx.x;
        int bin = BIN_NONE;
        if (i < n) {
            uint32_t p = work[i];
            uint64_t bound = cap ? (uint64_t)cap[i] : (p < ncols ? (uint64_t)p : ncols);
            bin = bin_of(p, bound, warp_max, bitmap_min, small);
        }
        // warp-aggregated reservation per bin
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, bin);
        const int leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if ((int)lane_id() == leader && bin != BIN_NONE) base = atomicAdd(&info[NUM_BINS + bin], (uint32_t)__popc(peers));
        base = __shfl_sync(0xFFFFFFFFu, base, leader);
        if (bin != BIN_NONE) {
            uint32_t rank = __popc(peers & ((1u << lane_id()) - 1u));
            list[boff[bin] + base + rank] = (uint32_t)i;
        }
    }
}

__global__ void assemble_kernel(const uint32_t *__restrict__ work, const uint32_t *__restrict__ pos,
                                const uint64_t *__restrict__ off, const uint32_t *__restrict__ a_rows, uint64_t n,
                                uint64_t *__restrict__ c_rpt, uint32_t *__restrict__ c_rows, uint64_t nzr,
                                uint64_t nnz) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (work[i] > 0) {
            uint32_t p = pos[i];
            c_rpt[p] = off[i];
            c_rows[p] = a_rows[i];
        }
        if (i == 0) c_rpt[nzr] = nnz;
    }
}

// Occupancy of each accumulator kernel, measured once per process.
template <class K>
int occupancy(K kernel, int nt, size_t dyn_smem) {
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, nt, dyn_smem) != cudaSuccess) {
        cudaGetLastError();
        blocks = 1;
    }
    return blocks > 0 ? blocks : 1;
}

template <int E, bool NUM>
int launch_esc(clb_controls *ctl, const BinLists &bl, int bin, const AView &a, const BRows &b, const RowOut &o,
               uint64_t nmax, const char *name) {
    static int occ = occupancy(warp_esc_kernel<E, NUM>, ESC_WARPS * 32, 0);
    unsigned grid = persistent_grid(ctl, occ, ceil_div_u(nmax, ESC_WARPS));
    ProfScope ps(ctl, name);
    warp_esc_kernel<E, NUM><<<grid, ESC_WARPS * 32, 0, ctl->stream>>>(bl, bin, a, b, o);
    ctl->launches += 1;
    CLB_CHECK_LAUNCH();
    return CLB_SUCCESS;
}

template <int G, bool NUM>
int launch_group_esc(clb_controls *ctl, const BinLists &bl, int bin, const AView &a, const BRows &b, const RowOut &o,
                     uint64_t nmax, const char *name) {
    static int occ = occupancy(group_esc_kernel<G, NUM>, ESC_WARPS * 32, 0);
    unsigned grid = persistent_grid(ctl, occ, ceil_div_u(nmax, ESC_WARPS * (32 / G)));
    ProfScope ps(ctl, name);
    group_esc_kernel<G, NUM><<<grid, ESC_WARPS * 32, 0, ctl->stream>>>(bl, bin, a, b, o);
    ctl->launches += 1;
    CLB_CHECK_LAUNCH();
    return CLB_SUCCESS;
}

template <int T, int NT, bool NUM>
int launch_hash(clb_controls *ctl, const BinLists &bl, int bin, const AView &a, const BRows &b, const RowOut &o,
                uint64_t nmax, uint32_t *counter, const char *name) {
    static int occ = occupancy(hash_cta_kernel<T, NT, NUM>, NT, 0);
    unsigned grid = persistent_grid(ctl, occ, nmax);
    ProfScope ps(ctl, name);
    hash_cta_kernel<T, NT, NUM><<<grid, NT, 0, ctl->stream>>>(bl, bin, a, b, o, counter);
    ctl->launches += 1;
    CLB_CHECK_LAUNCH();
    return CLB_SUCCESS;
}

template <bool NUM, bool MULTI, int NT>
int launch_bitmap_t(clb_controls *ctl, const BinLists &bl, const AView &a, const BRows &b, const RowOut &o,
                    uint64_t ncols, uint64_t nmax, uint32_t *counter, const char *name) {
    const uint32_t W = bitmap_words(ncols);
    const size_t smem = bitmap_smem_bytes(W, NT);
    auto kern = bitmap_cta_kernel<NUM, MULTI, NT>;
    CLB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                 CLB_RUN_KERNEL_FAILURE);
    int occ = occupancy(kern, NT, smem);
    unsigned grid = persistent_grid(ctl, occ, nmax);
    ProfScope ps(ctl, name);
    kern<<<grid, NT, smem, ctl->stream>>>(bl, BIN_BMP_XL, BIN_BMP, a, b, o, ncols, W, counter);
    ctl->launches += 1;
    CLB_CHECK_LAUNCH();
    return CLB_SUCCESS;
}

template <bool NUM, int NT>
int launch_bitmap_nt(clb_controls *ctl, const BinLists &bl, const AView &a, const BRows &b, const RowOut &o,
                     uint64_t ncols, uint64_t nmax, uint32_t *counter, const char *name) {
    const bool multi = ncols > (uint64_t)bitmap_words(ncols) * 32;
    return multi ? launch_bitmap_t<NUM, true, NT>(ctl, bl, a, b, o, ncols, nmax, counter, name)
                 : launch_bitmap_t<NUM, false, NT>(ctl, bl, a, b, o, ncols, nmax, counter, name);
}

// Rows wider than one bitmap chunk (2^20 < ncols <= CL * 2^20): one row per
// thread-block cluster of CL CTAs, each holding a 2^20-column slice.
template <bool NUM, int CL>
int launch_bitmap_cluster(clb_controls *ctl, const BinLists &bl, const AView &a, const BRows &b, const RowOut &o,
                          uint64_t ncols, uint64_t nmax, uint32_t *counter, const char *name) {
    const size_t smem = bitmap_smem_bytes(1u << (CLB_CHUNK_SHIFT - 5), 1024);
    auto kern = bitmap_cluster_kernel<NUM, CL>;
    CLB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                 CLB_RUN_KERNEL_FAILURE);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(CL);
    cfg.blockDim = dim3(1024);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = ctl->stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) != cudaSuccess || clusters < 1) {
        cudaGetLastError();
        clusters = 1;
    }
    if ((uint64_t)clusters > nmax) clusters = (int)(nmax ? nmax : 1);
    cfg.gridDim = dim3((unsigned)(clusters * CL));
    ProfScope ps(ctl, name);
    CLB_TRY_CUDA(cudaLaunchKernelEx(&cfg, kern, bl, (int)BIN_BMP_XL, (int)BIN_BMP, a, b, o, ncols, counter),
                 CLB_RUN_KERNEL_FAILURE);
    ctl->launches += 1;
    return CLB_SUCCESS;
}

template <bool NUM>
int launch_bitmap(clb_controls *ctl, const BinLists &bl, const AView &a, const BRows &b, const RowOut &o,
                  uint64_t ncols, uint64_t nmax, uint32_t *counter, const char *name, uint32_t threads,
                  bool wide_cluster) {
    // wider than one chunk, uniform width: a cluster can hold the whole row
    if (wide_cluster && !o.row_ncols && ncols > (1ull << CLB_CHUNK_SHIFT)) {
        if (ncols <= (2ull << CLB_CHUNK_SHIFT))
            return launch_bitmap_cluster<NUM, 2>(ctl, bl, a, b, o, ncols, nmax, counter, name);
        if (ncols <= (4ull << CLB_CHUNK_SHIFT))
            return launch_bitmap_cluster<NUM, 4>(ctl, bl, a, b, o, ncols, nmax, counter, name);
    }
    if (threads <= 256) return launch_bitmap_nt<NUM, 256>(ctl, bl, a, b, o, ncols, nmax, counter, name);
    if (threads <= 512) return launch_bitmap_nt<NUM, 512>(ctl, bl, a, b, o, ncols, nmax, counter, name);
    return launch_bitmap_nt<NUM, 1024>(ctl, bl, a, b, o, ncols, nmax, counter, name);
}

// hc (host, may be null): rows per bin, read back after binning; bins
// without rows are not launched and the grids follow the bins' sizes.
template <bool NUM>
int launch_all(clb_controls *ctl, const BinLists &bl, const AView &a, const BRows &b, const RowOut &o, uint64_t ncols,
               uint64_t nmax, const Tuning &t, const uint32_t *hc, bool hash_bins = true, bool bitmap_bins = true) {
    auto rows = [&](int bin) -> uint64_t { return hc ? hc[bin] : nmax; };
    // work counters of the dynamically scheduled launches
    Temp<uint32_t> ctr;
    CLB_RETURN_IF(ctr.alloc(ctl, 8));
    CLB_TRY_CUDA(cudaMemsetAsync(ctr.ptr, 0, 8 * sizeof(uint32_t), ctl->stream), CLB_RUN_KERNEL_FAILURE);
    // Heavy bins first so the long rows start early.
    const uint64_t nbmp = hc ? (uint64_t)hc[BIN_BMP_XL] + hc[BIN_BMP_L] + hc[BIN_BMP] : nmax;
    if (nbmp && bitmap_bins)
        CLB_RETURN_IF(launch_bitmap<NUM>(ctl, bl, a, b, o, ncols, nbmp, ctr.ptr + 0,
                                         NUM ? "bitmap_numeric" : "bitmap_symbolic", t.bitmap_threads,
                                         t.wide_cluster));
    if (hash_bins) {
        if (rows(BIN_H8K))
            CLB_RETURN_IF((launch_hash<8192, 512, NUM>(ctl, bl, BIN_H8K, a, b, o, rows(BIN_H8K), ctr.ptr + 1,
                                                       NUM ? "hash8k_numeric" : "hash8k_symbolic")));
        if (rows(BIN_H4K))
            CLB_RETURN_IF((launch_hash<4096, 512, NUM>(ctl, bl, BIN_H4K, a, b, o, rows(BIN_H4K), ctr.ptr + 2,
                                                       NUM ? "hash4k_numeric" : "hash4k_symbolic")));
        if (rows(BIN_H2K))
            CLB_RETURN_IF((launch_hash<2048, 256, NUM>(ctl, bl, BIN_H2K, a, b, o, rows(BIN_H2K), ctr.ptr + 3,
                                                       NUM ? "hash2k_numeric" : "hash2k_symbolic")));
        if (rows(BIN_H1K))
            CLB_RETURN_IF((launch_hash<1024, 256, NUM>(ctl, bl, BIN_H1K, a, b, o, rows(BIN_H1K), ctr.ptr + 4,
                                                       NUM ? "hash1k_numeric" : "hash1k_symbolic")));
    }
    if (rows(BIN_W8))
        CLB_RETURN_IF((launch_esc<8, NUM>(ctl, bl, BIN_W8, a, b, o, rows(BIN_W8),
                                          NUM ? "esc256_numeric" : "esc256_symbolic")));
    if (rows(BIN_W4))
        CLB_RETURN_IF((launch_esc<4, NUM>(ctl, bl, BIN_W4, a, b, o, rows(BIN_W4),
                                          NUM ? "esc128_numeric" : "esc128_symbolic")));
    if (rows(BIN_W2))
        CLB_RETURN_IF((launch_esc<2, NUM>(ctl, bl, BIN_W2, a, b, o, rows(BIN_W2),
                                          NUM ? "esc64_numeric" : "esc64_symbolic")));
    if (rows(BIN_W1))
        CLB_RETURN_IF((launch_esc<1, NUM>(ctl, bl, BIN_W1, a, b, o, rows(BIN_W1),
                                          NUM ? "esc32_numeric" : "esc32_symbolic")));
    if (t.small_lanes <= 16 && rows(BIN_G16))
        CLB_RETURN_IF((launch_group_esc<16, NUM>(ctl, bl, BIN_G16, a, b, o, rows(BIN_G16),
                                                 NUM ? "esc16_numeric" : "esc16_symbolic")));
    if (t.small_lanes <= 8 && rows(BIN_G8))
        CLB_RETURN_IF((launch_group_esc<8, NUM>(ctl, bl, BIN_G8, a, b, o, rows(BIN_G8),
                                                NUM ? "esc8_numeric" : "esc8_symbolic")));
    return CLB_SUCCESS;
}

}  // namespace

int launch_binning(clb_controls *ctl, const uint32_t *work, const uint32_t *cap, uint64_t n, uint64_t ncols,
                   uint32_t *info, uint32_t *list, uint32_t *flags, const Tuning &t) {
    CLB_TRY_CUDA(cudaMemsetAsync(info, 0, 2 * NUM_BINS * sizeof(uint32_t), ctl->stream), CLB_RUN_KERNEL_FAILURE);
    unsigned grid = persistent_grid(ctl, 8, ceil_div_u(n, BIN_NT));
    ProfScope ps(ctl, "binning");
    bin_count_kernel<<<grid, BIN_NT, 0, ctl->stream>>>(work, cap, n, ncols, t.warp_max, t.bitmap_min, t.small_lanes,
                                                       info, flags);
    bin_scatter_kernel<<<grid, BIN_NT, 0, ctl->stream>>>(work, cap, n, ncols, t.warp_max, t.bitmap_min, t.small_lanes,
                                                         info, list);
    ctl->launches += 2;
    CLB_CHECK_LAUNCH();
    return CLB_SUCCESS;
}

int launch_accumulators(clb_controls *ctl, bool numeric, const BinLists &bl, const AView &a, const BRows &b,
                        const RowOut &o, uint64_t ncols, uint64_t nmax, const Tuning &t, const uint32_t *hc) {
    return numeric ? launch_all<true>(ctl, bl, a, b, o, ncols, nmax, t, hc)
                   : launch_all<false>(ctl, bl, a, b, o, ncols, nmax, t, hc);
}

int launch_accumulators_subset(clb_controls *ctl, const BinLists &bl, const AView &a, const BRows &b,
                               const RowOut &o, uint64_t ncols, uint64_t nmax, bool hash_bins, const Tuning &t,
                               const uint32_t *hc, bool bitmap_bins) {
    return launch_all<true>(ctl, bl, a, b, o, ncols, nmax, t, hc, hash_bins, bitmap_bins);
}

int launch_bitmap_expand(clb_controls *ctl, const uint32_t *list, const uint32_t *count, uint64_t nmax,
                         const uint64_t *slot_off, const uint32_t *slots, const uint64_t *off,
                         const uint32_t *row_ncols, uint64_t ncols, uint32_t *ccols) {
    constexpr int NT = 1024;
    const uint32_t W = bitmap_words(ncols);
    const size_t smem = bitmap_smem_bytes(W, NT);
    auto kern = bitmap_expand_kernel<NT>;
    CLB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                 CLB_RUN_KERNEL_FAILURE);
    Temp<uint32_t> ctr;
    CLB_RETURN_IF(ctr.alloc(ctl, 1));
    CLB_TRY_CUDA(cudaMemsetAsync(ctr.ptr, 0, sizeof(uint32_t), ctl->stream), CLB_RUN_KERNEL_FAILURE);
    const unsigned grid = persistent_grid(ctl, occupancy(kern, NT, smem), nmax);
    ProfScope ps(ctl, "bitmap_expand");
    kern<<<grid, NT, smem, ctl->stream>>>(list, count, slot_off, slots, off, row_ncols, ncols, W, ccols, ctr.ptr);
    ctl->launches += 1;
    CLB_CHECK_LAUNCH();
    return CLB_SUCCESS;
}

int launch_bitmap_expand_steps(clb_controls *ctl, const uint32_t *list, const uint32_t *count, const uint32_t *steps,
                               const uint64_t *slot_off, const uint32_t *slots, const uint64_t *off,
                               uint32_t *ccols) {
    constexpr int NT = 256;
    auto kern = bitmap_expand_steps_kernel<NT>;
    Temp<uint32_t> ctr;
    CLB_RETURN_IF(ctr.alloc(ctl, 1));
    CLB_TRY_CUDA(cudaMemsetAsync(ctr.ptr, 0, sizeof(uint32_t), ctl->stream), CLB_RUN_KERNEL_FAILURE);
    const unsigned grid = (unsigned)ctl->sm_count * (unsigned)occupancy(kern, NT, 0);
    ProfScope ps(ctl, "bitmap_expand");
    kern<<<grid, NT, 0, ctl->stream>>>(list, count, steps, slot_off, slots, off, ccols, ctr.ptr);
    ctl->launches += 1;
    CLB_CHECK_LAUNCH();
    return CLB_SUCCESS;
}

int launch_assemble(clb_controls *ctl, const uint32_t *work, const uint32_t *pos, const uint64_t *off,
                    const uint32_t *a_rows, uint64_t n, uint64_t *c_rpt, uint32_t *c_rows, uint64_t nzr, uint64_t nnz) {
    unsigned grid = persistent_grid(ctl, 8, ceil_div_u(n, 256));
    ProfScope ps(ctl, "assemble");
    assemble_kernel<<<grid, 256, 0, ctl->stream>>>(work, pos, off, a_rows, n, c_rpt, c_rows, nzr, nnz);
    ctl->launches += 1;
    CLB_CHECK_LAUNCH();
    return CLB_SUCCESS;
}

}  // namespace clb
