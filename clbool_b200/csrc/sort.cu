// sort.cu -- coo::sort_arrays and duplicate removal.
//
// Reference: coo::sort_arrays (src/coo/coo_initialization.cpp:6-32) sorts
// (row, col) pairs with a global bitonic network (coo_bitonic_sort.cl,
// O(n log^2 n) passes); matrix_coo::reduce_duplicates2
// (src/core/matrix_coo.cpp:117-170) removes adjacent duplicates.
//
// Here: a stable LSD radix sort of packed 64-bit keys row << bc | col, where
// bc/br are the bit widths actually used by the columns/rows, 8 bits per
// pass.  Each pass is upsweep (tile digit histograms) -> scan -> downsweep
// (stable scatter).  Stability inside a 2048-key tile comes from processing
// keys in index order per warp and ranking equal digits with __match_any_sync
// plus per-warp running digit counters in shared memory.
#include "common.cuh"

namespace clb {

namespace {

constexpr int RS_NT = 256;
constexpr int RS_WARPS = RS_NT / 32;
constexpr int RS_ROUNDS = 8;                       // 32-key rounds per warp
constexpr uint64_t RS_TILE = 32ull * RS_ROUNDS * RS_WARPS;  // 2048 keys
constexpr int RADIX = 256;
static_assert(RS_NT == RADIX, "the downsweep gives each thread one digit");

__global__ void max_pair_kernel(const uint32_t *__restrict__ rows, const uint32_t *__restrict__ cols, uint64_t n,
                                unsigned int *__restrict__ out) {
    uint32_t mr = 0, mc = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        mr = max(mr, rows[i]);
        mc = max(mc, cols[i]);
    }
    mr = warp_max(mr);
    mc = warp_max(mc);
    if (lane_id() == 0) {
        atomicMax(out + 0, mr);
        atomicMax(out + 1, mc);
    }
}

__global__ void pack_kernel(const uint32_t *__restrict__ rows, const uint32_t *__restrict__ cols, uint64_t n,
                            int bc, uint64_t *__restrict__ keys) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        keys[i] = ((uint64_t)rows[i] << bc) | (uint64_t)cols[i];
}

__global__ void unpack_kernel(const uint64_t *__restrict__ keys, uint64_t n, int bc, uint32_t *__restrict__ rows,
                              uint32_t *__restrict__ cols) {
    const uint64_t mask = bc >= 64 ? ~0ull : ((1ull << bc) - 1);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t k = keys[i];
        rows[i] = (uint32_t)(k >> bc);
        cols[i] = (uint32_t)(k & mask);
    }
}

// counts[d * ntiles + tile] = keys of `tile` with digit d.
__global__ void __launch_bounds__(RS_NT) radix_upsweep_kernel(const uint64_t *__restrict__ keys, uint64_t n, int shift,
                                                              uint32_t ntiles, uint32_t *__restrict__ counts) {
    __shared__ uint32_t hist[RADIX];
    hist[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * RS_TILE;
#pragma unroll
    for (int r = 0; r < (int)(RS_TILE / RS_NT); ++r) {
        uint64_t i = base + (uint64_t)r * RS_NT + threadIdx.x;
        if (i < n) atomicAdd(&hist[(keys[i] >> shift) & (RADIX - 1)], 1u);
    }
    __syncthreads();
    counts[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = hist[threadIdx.x];
}

// Stable scatter of one tile; offs = exclusive scan of counts (digit-major).
// The tile's keys are first placed in shared memory in their sorted order
// (digit buckets one after another), then written out by consecutive
// threads, so the keys of one digit leave as runs of consecutive addresses
// instead of one scattered 8-byte store per key.
__global__ void __launch_bounds__(RS_NT) radix_downsweep_kernel(const uint64_t *__restrict__ in, uint64_t *__restrict__ out,
                                                                uint64_t n, int shift, uint32_t ntiles,
                                                                const uint32_t *__restrict__ offs) {
    __shared__ uint32_t whist[RS_WARPS][RADIX];
    __shared__ uint32_t goff[RADIX];
    __shared__ uint32_t dstart[RADIX];     // first tile position of each digit
    __shared__ uint32_t scratch[33];
    __shared__ uint64_t skeys[RS_TILE];
    const uint32_t lane = lane_id(), w = warp_id();
    for (int d = threadIdx.x; d < RS_WARPS * RADIX; d += RS_NT) (&whist[0][0])[d] = 0;
    goff[threadIdx.x] = offs[(uint64_t)threadIdx.x * ntiles + blockIdx.x];
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * RS_TILE + (uint64_t)w * (32 * RS_ROUNDS);
    const unsigned lt = (1u << lane) - 1u;
    uint64_t key[RS_ROUNDS];
    uint32_t rank[RS_ROUNDS];
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; ++r) {
        uint64_t i = base + (uint64_t)r * 32 + lane;
        bool valid = i < n;
        key[r] = valid ? in[i] : 0;
        uint32_t digit = valid ? (uint32_t)((key[r] >> shift) & (RADIX - 1)) : RADIX;  // RADIX = padding group
        unsigned peers = __match_any_sync(0xFFFFFFFFu, digit);
        int leader = __ffs(peers) - 1;
        uint32_t old = 0;
        if ((int)lane == leader && valid) {
            old = whist[w][digit];
            whist[w][digit] = old + (uint32_t)__popc(peers);
        }
        old = __shfl_sync(0xFFFFFFFFu, old, leader);
        rank[r] = old + (uint32_t)__popc(peers & lt);
    }
    __syncthreads();
    uint32_t run = 0;
    {   // per digit: exclusive prefix over warps (warp order = key order)
#pragma unroll
        for (int q = 0; q < RS_WARPS; ++q) {
            uint32_t c = whist[q][threadIdx.x];
            whist[q][threadIdx.x] = run;
            run += c;
        }
    }
    // digit starts inside the tile (RS_NT == RADIX: thread d holds digit d)
    uint32_t tile_keys;
    dstart[threadIdx.x] = block_exclusive_scan<uint32_t, RS_NT>(run, scratch, &tile_keys);
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; ++r) {
        uint64_t i = base + (uint64_t)r * 32 + lane;
        if (i < n) {
            uint32_t digit = (uint32_t)((key[r] >> shift) & (RADIX - 1));
            skeys[dstart[digit] + whist[w][digit] + rank[r]] = key[r];
        }
    }
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < tile_keys; t += RS_NT) {
        const uint64_t k = skeys[t];
        const uint32_t digit = (uint32_t)((k >> shift) & (RADIX - 1));
        out[(uint64_t)goff[digit] + (t - dstart[digit])] = k;
    }
}

__global__ void run_start_flags_kernel(const uint32_t *__restrict__ rows, const uint32_t *__restrict__ cols, uint64_t n,
                                       uint32_t *__restrict__ flags) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        flags[i] = (i == 0 || rows[i] != rows[i - 1] || cols[i] != cols[i - 1]) ? 1u : 0u;
}

__global__ void compact_pairs_kernel(const uint32_t *__restrict__ rows, const uint32_t *__restrict__ cols, uint64_t n,
                                     const uint32_t *__restrict__ pos, uint32_t *__restrict__ out_rows,
                                     uint32_t *__restrict__ out_cols) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (i == 0 || rows[i] != rows[i - 1] || cols[i] != cols[i - 1]) {
            out_rows[pos[i]] = rows[i];
            out_cols[pos[i]] = cols[i];
        }
    }
}

int bits_for(uint32_t v) { return v ? 32 - __builtin_clz(v) : 0; }

unsigned grid_for(const clb_controls *ctl, uint64_t n) {
    uint64_t g = (n + 255) / 256, cap = (uint64_t)ctl->sm_count * 16;
    return (unsigned)(g > cap ? cap : (g ? g : 1));
}

}  // namespace

// Sorts the packed keys of (rows, cols) in place; shared by transpose.
int sort_pairs(clb_controls *ctl, uint32_t *rows, uint32_t *cols, uint64_t n) {
    if (n < 2) return CLB_SUCCESS;
    if (n >= (1ull << 32)) return fail(CLB_NOT_SUPPORTED, "sort of 2^32 or more pairs");
    ProfScope ps(ctl, "coo_sort");
    Temp<uint64_t> mx;
    CLB_RETURN_IF(mx.alloc(ctl, 1));
    CLB_TRY_CUDA(cudaMemsetAsync(mx.ptr, 0, 8, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    max_pair_kernel<<<grid_for(ctl, n), 256, 0, ctl->stream>>>(rows, cols, n, (unsigned int *)mx.ptr);
    CLB_CHECK_LAUNCH();
    uint64_t h = 0;
    CLB_RETURN_IF(read_scalars(ctl, mx.ptr, &h, 1));
    const int br = bits_for((uint32_t)(h & 0xFFFFFFFFu)), bc = bits_for((uint32_t)(h >> 32));
    const int total_bits = br + bc;
    Temp<uint64_t> k0, k1;
    CLB_RETURN_IF(k0.alloc(ctl, n));
    CLB_RETURN_IF(k1.alloc(ctl, n));
    pack_kernel<<<grid_for(ctl, n), 256, 0, ctl->stream>>>(rows, cols, n, bc, k0.ptr);
    CLB_CHECK_LAUNCH();
    const uint32_t ntiles = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
    Temp<uint32_t> counts;
    CLB_RETURN_IF(counts.alloc(ctl, (uint64_t)RADIX * ntiles));
    uint64_t *src = k0.ptr, *dst = k1.ptr;
    for (int shift = 0; shift < total_bits; shift += 8) {
        radix_upsweep_kernel<<<ntiles, RS_NT, 0, ctl->stream>>>(src, n, shift, ntiles, counts.ptr);
        CLB_CHECK_LAUNCH();
        CLB_RETURN_IF(scan_u32_inplace(ctl, counts.ptr, (uint64_t)RADIX * ntiles, nullptr));
        radix_downsweep_kernel<<<ntiles, RS_NT, 0, ctl->stream>>>(src, dst, n, shift, ntiles, counts.ptr);
        CLB_CHECK_LAUNCH();
        ctl->launches += 2;
        uint64_t *t = src;
        src = dst;
        dst = t;
    }
    unpack_kernel<<<grid_for(ctl, n), 256, 0, ctl->stream>>>(src, n, bc, rows, cols);
    CLB_CHECK_LAUNCH();
    ctl->launches += 3;
    return CLB_SUCCESS;
}

// Sorted pairs -> new arrays without adjacent duplicates.
int unique_pairs(clb_controls *ctl, const uint32_t *rows, const uint32_t *cols, uint64_t n, uint32_t **out_rows,
                 uint32_t **out_cols, uint64_t *out_n) {
    *out_rows = *out_cols = nullptr;
    *out_n = 0;
    if (n == 0) return CLB_SUCCESS;
    if (n >= (1ull << 32)) return fail(CLB_NOT_SUPPORTED, "2^32 or more pairs");
    Temp<uint32_t> pos;
    Temp<uint64_t> tot;
    CLB_RETURN_IF(pos.alloc(ctl, n));
    CLB_RETURN_IF(tot.alloc(ctl, 1));
    run_start_flags_kernel<<<grid_for(ctl, n), 256, 0, ctl->stream>>>(rows, cols, n, pos.ptr);
    CLB_CHECK_LAUNCH();
    CLB_RETURN_IF(scan_u32_inplace(ctl, pos.ptr, n, tot.ptr));
    uint64_t m = 0;
    CLB_RETURN_IF(read_scalars(ctl, tot.ptr, &m, 1));
    Temp<uint32_t> r, c;
    CLB_RETURN_IF(r.alloc(ctl, m));
    CLB_RETURN_IF(c.alloc(ctl, m));
    compact_pairs_kernel<<<grid_for(ctl, n), 256, 0, ctl->stream>>>(rows, cols, n, pos.ptr, r.ptr, c.ptr);
    CLB_CHECK_LAUNCH();
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    *out_rows = r.release_ownership();
    *out_cols = c.release_ownership();
    *out_n = m;
    return CLB_SUCCESS;
}

}  // namespace clb

using namespace clb;

extern "C" {

int clb_coo_sort(clb_controls *ctl, uint32_t *rows, uint32_t *cols, uint64_t n) {
    if (!ctl || (n && (!rows || !cols))) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    DeviceGuard g(ctl);
    CLB_RETURN_IF(sort_pairs(ctl, rows, cols, n));
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    return CLB_SUCCESS;
}

int clb_coo_reduce_duplicates(clb_controls *ctl, const clb_coo *in_, clb_coo *out) {
    if (!ctl || !in_ || !out) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    clb_coo in = *in_;
    DeviceGuard g(ctl);
    clb_coo r{};
    r.nrows = in.nrows;
    r.ncols = in.ncols;
    CLB_RETURN_IF(unique_pairs(ctl, in.rows, in.cols, in.nnz, &r.rows, &r.cols, &r.nnz));
    *out = r;
    return CLB_SUCCESS;
}

}  // extern "C"
