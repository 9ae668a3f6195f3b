// spgemm_kernels.cuh -- row accumulators of the boolean SpGEMM, shared by
// the exact two-pass form and the learned single-pass form.
//
// Reference algorithm (src/dcsr/dcsr_matrix_multiplication_hash.cpp:51-119):
// products per A row -> bins by size -> per-bin symbolic count -> scan ->
// per-bin numeric fill.  The accumulators here are designed for sm_100a:
//   * warp ESC (rows with <= 256 products): the warp copies the products into
//     a private shared buffer, sorts them in registers with a bitonic network
//     over shuffles, and drops duplicates with one neighbour shuffle;
//   * CTA hash (<= 4096 distinct columns possible): open-addressing table in
//     shared memory (Fibonacci hashing, linear probing, bounded), then a
//     shared-memory bitonic sort of the compacted keys;
//   * CTA bitmap (heavy rows): a 128 KB shared-memory bitmap over a column
//     chunk; the population count is the symbolic result and a warp scan of
//     per-word counts emits the columns already sorted (no sort pass).
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"

namespace clb {

struct AView {
    const uint64_t *rpt;
    const uint32_t *rows;
    const uint32_t *cols;
    uint64_t nzr;
};

// Accumulator bins (bin 0 = rows without products, not listed).
enum Bin : int {
    BIN_NONE = 0,
    BIN_W1 = 1,   // products <= 32
    BIN_W2 = 2,   // <= 64
    BIN_W4 = 3,   // <= 128
    BIN_W8 = 4,   // <= 256
    BIN_H1K = 5,  // distinct-column bound <= 512  -> table 1024
    BIN_H2K = 6,  // <= 1024 -> 2048
    BIN_H4K = 7,  // <= 2048 -> 4096
    BIN_H8K = 8,  // <= 4096 -> 8192
    // Bitmap rows, heaviest first: the three bins are contiguous in the row
    // list and one dynamically scheduled launch walks them in order.
    BIN_BMP_XL = 9,   // products > 2^20
    BIN_BMP_L = 10,   // products > 2^17
    BIN_BMP = 11,     // the rest
    BIN_G8 = 12,      // products <= 8, 8 lanes per row (tuning small_lanes <= 8)
    BIN_G16 = 13,     // products <= 16, 16 lanes per row (small_lanes <= 16)
    NUM_BINS = 14
};

// Rows with at most this many products never reach the bitmap accumulator
// under the default tuning (the CTA hash / CTA ESC kernels take them).
constexpr uint32_t ESC_MAX_PRODUCTS = 4096;

// Accumulator tuning (all settings give the same C):
//   warp_max       rows with at most this many products go to the warp ESC
//                  kernels (32, 64, 128 or 256);
//   bitmap_min     rows with more products go to the bitmap kernel (at most
//                  ESC_MAX_PRODUCTS; lower values pay off when the bitmap is
//                  narrow, i.e. few columns);
//   bitmap_threads threads per bitmap row (256, 512 or 1024).
//   small_lanes    lanes per row for the smallest rows: 8 (rows of <= 8
//                  products share a warp four ways, <= 16 two ways), 16, or
//                  32 (a warp per row);
//   wide_cluster   rows wider than one bitmap chunk (2^20 < ncols <= 2^22):
//                  false = one CTA walks the products once per chunk, true =
//                  a cluster of 2 or 4 CTAs holds the whole row (one pass,
//                  distributed shared memory; slower on R-MAT scale 21, but
//                  such rows can spill in the learned form).
struct Tuning {
    uint32_t warp_max = 256;
    uint32_t bitmap_min = ESC_MAX_PRODUCTS;
    uint32_t bitmap_threads = 1024;
    uint32_t small_lanes = 8;
    bool wide_cluster = false;
    // Per A row: columns of that row's product, when they differ by row (a
    // stacked batch of pairs); null = B.ncols for every row.
    const uint32_t *row_ncols = nullptr;
};

// Bin of a row from its product count and its distinct-column bound
// (min(products, ncols), or a capacity).
__host__ __device__ __forceinline__ int bin_of(uint64_t products, uint64_t distinct_bound, uint32_t warp_max,
                                               uint32_t bitmap_min, uint32_t small_lanes) {
    if (products == 0) return BIN_NONE;
    if (products <= 8 && small_lanes <= 8) return BIN_G8;
    if (products <= 16 && small_lanes <= 16) return BIN_G16;
    if (products <= warp_max) {
        if (products <= 32) return BIN_W1;
        if (products <= 64) return BIN_W2;
        if (products <= 128) return BIN_W4;
        return BIN_W8;
    }
    if (products > bitmap_min) {
        if (products > (1u << 20)) return BIN_BMP_XL;
        if (products > (1u << 17)) return BIN_BMP_L;
        return BIN_BMP;
    }
    if (distinct_bound <= 512) return BIN_H1K;
    if (distinct_bound <= 1024) return BIN_H2K;
    if (distinct_bound <= 2048) return BIN_H4K;
    return BIN_H8K;
}

// Row lists of all bins packed in one array; info[b] = count of bin b,
// info[NUM_BINS + b] = scatter cursor.  Offset of bin b = sum of counts below.
struct BinLists {
    const uint32_t *list;
    const uint32_t *info;
};

__device__ __forceinline__ void bin_range(const BinLists &bl, int bin, uint32_t &beg, uint32_t &cnt) {
    uint32_t o = 0;
    for (int b = 1; b < bin; ++b) o += bl.info[b];
    beg = o;
    cnt = bl.info[bin];
}

// Output side of an accumulator.  Symbolic: row_nnz[i] = distinct columns.
// Numeric: columns written at cols + row_off[i]; when row_cap is non-null
// (single-pass forms) a row whose count exceeds row_cap[i] is not written
// there.  A single-chunk bitmap row then reserves its exact count in the
// spill arena (when one is given and has room), writes there and records the
// arena offset in spill[i]; any other such row is flagged in overflow[i] and
// recomputed by the exact two-pass form.
struct RowOut {
    uint32_t *row_nnz;
    const uint64_t *row_off;
    const uint32_t *row_cap;
    uint32_t *overflow;
    uint32_t *cols;
    uint32_t *status;
    uint64_t *spill = nullptr;                     // arena offset per row, ~0 = not spilled
    uint32_t *arena = nullptr;
    unsigned long long *arena_cursor = nullptr;    // entries reserved so far
    uint64_t arena_cap = 0;                        // entries
    const uint32_t *row_ncols = nullptr;           // columns of row i's product (batched pairs), or all
    const uint32_t *row_products = nullptr;        // products of row i (picks the bitmap insertion path)
    // Single-pass forms: bitmap rows whose slot holds their bitmap (of at
    // least BMP_DEFER_MIN_WORDS words) and whose columns reach 1 /
    // BMP_DEFER_DIV of its words store the bitmap in their slot instead
    // (defer[i] = 1, listed in defer_list[0, *defer_count));
    // bitmap_expand_steps_kernel (or bitmap_expand_kernel) writes their
    // columns.
    uint32_t *defer = nullptr;
    uint32_t *defer_list = nullptr;
    uint32_t *defer_count = nullptr;
    // Optional: record d (BMP_STEP_REC words) of defer_list[d] gets its
    // non-empty steps and their output offsets (bitmap_expand_steps_kernel).
    uint32_t *defer_steps = nullptr;
    // Two-pass form keeping its bitmaps (symbolic pass, single-chunk rows):
    // the row claimed as item k of the bitmap bins stores its bitmap at
    // keep + k * keep_stride, its step record in defer_steps, its index in
    // defer_list[k] and the bitmap's offset in keep_off[row]; the numeric
    // pass expands it at C's row offset instead of inserting it again.
    uint32_t *keep = nullptr;
    uint64_t keep_stride = 0;
    uint64_t *keep_off = nullptr;
};

// ------------------------------------------------------------- warp ESC ----
template <int E>
__device__ __forceinline__ void warp_bitonic_sort(uint32_t (&v)[E]) {
    constexpr int N = 32 * E;
    const uint32_t lane = lane_id();
#pragma unroll
    for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j >= E) {
                const int lx = j / E;
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    uint32_t idx = lane * E + e;
                    uint32_t o = __shfl_xor_sync(0xFFFFFFFFu, v[e], lx);
                    bool up = (idx & k) == 0;
                    bool lower = (idx & j) == 0;
                    v[e] = (up == lower) ? min(v[e], o) : max(v[e], o);
                }
            } else {
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    if ((e & j) == 0) {
                        const int e2 = e | j;
                        uint32_t idx = lane * E + e;
                        bool up = (idx & k) == 0;
                        uint32_t x = v[e], y = v[e2];
                        if ((x > y) == up) {
                            v[e] = y;
                            v[e2] = x;
                        }
                    }
                }
            }
        }
    }
}

constexpr int ESC_WARPS = 8;

// One warp per row; the row's products (<= 32*E) are gathered into a
// warp-private shared buffer, sorted in registers, deduplicated.
template <int E, bool NUMERIC>
__global__ void __launch_bounds__(ESC_WARPS * 32) warp_esc_kernel(BinLists bl, int bin, AView a, BRows b, RowOut o) {
    constexpr int N = 32 * E;
    __shared__ uint32_t sbuf[ESC_WARPS][N];
    uint32_t *buf = sbuf[warp_id()];
    const uint32_t lane = lane_id();
    uint32_t beg, cnt;
    bin_range(bl, bin, beg, cnt);
    for (uint32_t w = blockIdx.x * ESC_WARPS + warp_id(); w < cnt; w += gridDim.x * ESC_WARPS) {
        const uint32_t i = bl.list[beg + w];
        const uint64_t ja = a.rpt[i], je = a.rpt[i + 1];
        uint32_t fill = 0;
        for (uint64_t j0 = ja; j0 < je; j0 += 32) {
            const uint64_t j = j0 + lane;
            uint64_t bb = 0;
            uint32_t len = 0;
            if (j < je) len = b_row(b, __ldg(a.cols + j), bb);
            uint32_t inc = warp_inclusive_scan(len);
            uint32_t off = fill + inc - len;
            uint32_t mask = __ballot_sync(0xFFFFFFFFu, len > 0);
            while (mask) {
                const int src = __ffs(mask) - 1;
                mask &= mask - 1;
                const uint64_t sb = __shfl_sync(0xFFFFFFFFu, bb, src);
                const uint32_t sl = __shfl_sync(0xFFFFFFFFu, len, src);
                const uint32_t so = __shfl_sync(0xFFFFFFFFu, off, src);
                for (uint32_t t = lane; t < sl; t += 32) {
                    if (so + t < (uint32_t)N) buf[so + t] = __ldg(b.cols + sb + t);
                }
            }
            fill += __shfl_sync(0xFFFFFFFFu, inc, 31);
        }
        __syncwarp();
        if (fill > (uint32_t)N) {  // binning guarantees fill <= N
            if (lane == 0) raise_status(o.status, DEV_BOUNDS);
            fill = N;
        }
        uint32_t v[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            uint32_t idx = lane * E + e;
            v[e] = idx < fill ? buf[idx] : EMPTY;
        }
        __syncwarp();
        warp_bitonic_sort<E>(v);
        const uint32_t prev_last = __shfl_up_sync(0xFFFFFFFFu, v[E - 1], 1);
        uint32_t flags = 0, mine = 0;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            bool first = (lane == 0 && e == 0);
            uint32_t pv = (e == 0) ? prev_last : v[e > 0 ? e - 1 : 0];
            bool f = v[e] != EMPTY && (first || v[e] != pv);
            flags |= (f ? 1u : 0u) << e;
            mine += f ? 1u : 0u;
        }
        if (!NUMERIC) {
            uint32_t total = warp_sum(mine);
            if (lane == 0) o.row_nnz[i] = total;
        } else {
            uint32_t inc = warp_inclusive_scan(mine);
            uint32_t total = __shfl_sync(0xFFFFFFFFu, inc, 31);
            if (o.row_cap) {
                if (total > o.row_cap[i]) {
                    if (lane == 0) o.overflow[i] = 1;
                    continue;
                }
                if (lane == 0) o.row_nnz[i] = total;
            }
            uint32_t *dst = o.cols + o.row_off[i] + (inc - mine);
#pragma unroll
            for (int e = 0; e < E; ++e) {
                if (flags & (1u << e)) *dst++ = v[e];
            }
        }
    }
}

// G lanes per row (G = 8 or 16), 32 / G rows per warp, for rows of at most
// G products: each lane gathers the B row of one A entry into the group's
// slice of a warp-private buffer, the group sorts its G values with a
// bitonic network over width-G shuffles and drops duplicates.  Loops and
// shuffles are warp-uniform; groups without a row carry EMPTY.
template <int G, bool NUMERIC>
__global__ void __launch_bounds__(ESC_WARPS * 32, 4) group_esc_kernel(BinLists bl, int bin, AView a, BRows b, RowOut o) {
    constexpr int RPW = 32 / G;  // rows per warp
    __shared__ uint32_t sbuf[ESC_WARPS][32];
    const uint32_t lane = lane_id(), lg = lane % G, grp = lane / G;
    uint32_t *buf = sbuf[warp_id()] + grp * G;
    const uint32_t gmask = (G == 32 ? 0xFFFFFFFFu : ((1u << G) - 1u)) << (grp * G);
    uint32_t beg, cnt;
    bin_range(bl, bin, beg, cnt);
    for (uint32_t w = blockIdx.x * ESC_WARPS + warp_id(); w * RPW < cnt; w += gridDim.x * ESC_WARPS) {
        const uint32_t item = w * RPW + grp;
        const bool has = item < cnt;
        const uint32_t i = has ? bl.list[beg + item] : 0;
        const uint64_t ja = has ? a.rpt[i] : 0, je = has ? a.rpt[i + 1] : 0;
        uint32_t fill = 0;
        for (uint64_t c = 0;; c += G) {
            const bool more = ja + c < je;
            if (!__any_sync(0xFFFFFFFFu, more)) break;
            const uint64_t j = ja + c + lg;
            uint64_t bb = 0;
            uint32_t len = 0;
            if (j < je) len = b_row(b, __ldg(a.cols + j), bb);
            uint32_t inc = len;
#pragma unroll
            for (int d = 1; d < G; d <<= 1) {
                const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, d, G);
                if ((int)lg >= d) inc += t;
            }
            const uint32_t off = fill + inc - len;
            for (uint32_t t = 0; t < len; ++t)
                if (off + t < (uint32_t)G) buf[off + t] = __ldg(b.cols + bb + t);
            fill += __shfl_sync(0xFFFFFFFFu, inc, G - 1, G);
        }
        __syncwarp();
        if (fill > (uint32_t)G) {  // binning guarantees fill <= G
            if (lg == 0) raise_status(o.status, DEV_BOUNDS);
            fill = G;
        }
        uint32_t v = lg < fill ? buf[lg] : EMPTY;
        __syncwarp();
#pragma unroll
        for (int k = 2; k <= G; k <<= 1) {
#pragma unroll
            for (int j = k >> 1; j > 0; j >>= 1) {
                const uint32_t x = __shfl_xor_sync(0xFFFFFFFFu, v, j, G);
                const bool up = (lg & k) == 0, lower = (lg & j) == 0;
                v = (up == lower) ? min(v, x) : max(v, x);
            }
        }
        const uint32_t pv = __shfl_up_sync(0xFFFFFFFFu, v, 1, G);
        const bool f = v != EMPTY && (lg == 0 || v != pv);
        const uint32_t fm = __ballot_sync(0xFFFFFFFFu, f) & gmask;
        const uint32_t total = __popc(fm);
        if (!has) continue;
        if (!NUMERIC) {
            if (lg == 0) o.row_nnz[i] = total;
            continue;
        }
        if (o.row_cap) {
            if (total > o.row_cap[i]) {
                if (lg == 0) o.overflow[i] = 1;
                continue;
            }
            if (lg == 0) o.row_nnz[i] = total;
        }
        if (f) o.cols[o.row_off[i] + __popc(fm & ((1u << lane) - 1u))] = v;
    }
}

// ------------------------------------------------------------- CTA hash ----
template <int T>
__device__ __forceinline__ uint32_t hash_insert(uint32_t *table, uint32_t c, uint32_t *status) {
    constexpr int LOG2T = (T == 1024) ? 10 : (T == 2048) ? 11 : (T == 4096) ? 12 : (T == 8192) ? 13 : 14;
    uint32_t h = (c * 0x9E3779B1u) >> (32 - LOG2T);
#pragma unroll 1
    for (int probe = 0; probe < T; ++probe) {
        uint32_t cur = *(volatile uint32_t *)(table + h);
        if (cur == c) return 0;
        if (cur == EMPTY) {
            uint32_t prev = atomicCAS(table + h, EMPTY, c);
            if (prev == EMPTY) return 1;
            if (prev == c) return 0;
        }
        h = (h + 1) & (T - 1);
    }
    raise_status(status, DEV_PROBE_LIMIT);
    return 0;
}

// Sort s[0, M) ascending, M a power of two; all NT threads participate.
template <int NT>
__device__ __forceinline__ void block_bitonic_sort(uint32_t *s, uint32_t M) {
    for (uint32_t k = 2; k <= M; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t t = threadIdx.x; t < (M >> 1); t += NT) {
                uint32_t lo = ((t & ~(j - 1)) << 1) | (t & (j - 1));
                uint32_t hi = lo | j;
                bool up = (lo & k) == 0;
                uint32_t x = s[lo], y = s[hi];
                if ((x > y) == up) {
                    s[lo] = y;
                    s[hi] = x;
                }
            }
            __syncthreads();
        }
    }
}

// One bitonic compare-exchange stage (k, j) over a warp's register chunk:
// lane l holds elements base + l*E + e; partners closer than E are in the
// same thread, farther ones (up to 32E) in lane l ^ (j / E).
template <int E>
__device__ __forceinline__ void warp_stage(uint32_t (&v)[E], uint32_t base, uint32_t k, uint32_t j) {
    const uint32_t lane = lane_id();
    if (j >= (uint32_t)E) {
        const int lx = (int)(j / E);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const uint32_t idx = base + lane * E + e;
            const uint32_t o = __shfl_xor_sync(0xFFFFFFFFu, v[e], lx);
            const bool up = (idx & k) == 0, lower = (idx & j) == 0;
            v[e] = (up == lower) ? min(v[e], o) : max(v[e], o);
        }
    } else {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            if ((e & j) == 0) {
                const int e2 = e | (int)j;
                const bool up = ((base + lane * E + e) & k) == 0;
                const uint32_t x = v[e], y = v[e2];
                if ((x > y) == up) {
                    v[e] = y;
                    v[e2] = x;
                }
            }
        }
    }
}

// Ascending sort of exactly NT*E keys in shared memory.  Bitonic network with
// every stage whose partners are less than 32E apart done in registers by
// the warp owning that 32E-element chunk (shuffles, no barrier); only the
// farther stages go through shared memory with a block barrier each: for
// 4096 keys on 512 threads, 10 barrier stages instead of 78.
template <int NT, int E>
__device__ __forceinline__ void block_sort_hybrid(uint32_t *s) {
    constexpr uint32_t M = NT * E, WCH = 32u * E;
    const uint32_t base = warp_id() * WCH, lane = lane_id();
    uint32_t v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = s[base + lane * E + e];
    // every chunk sorted, in the direction its position in the network asks
#pragma unroll
    for (uint32_t k = 2; k <= WCH; k <<= 1)
#pragma unroll
        for (uint32_t j = k >> 1; j > 0; j >>= 1) warp_stage<E>(v, base, k, j);
    for (uint32_t k = 2 * WCH; k <= M; k <<= 1) {
#pragma unroll
        for (int e = 0; e < E; ++e) s[base + lane * E + e] = v[e];
        __syncthreads();
        for (uint32_t j = k >> 1; j >= WCH; j >>= 1) {
            for (uint32_t t = threadIdx.x; t < (M >> 1); t += NT) {
                const uint32_t lo = ((t & ~(j - 1)) << 1) | (t & (j - 1));
                const uint32_t hi = lo | j;
                const bool up = (lo & k) == 0;
                const uint32_t x = s[lo], y = s[hi];
                if ((x > y) == up) {
                    s[lo] = y;
                    s[hi] = x;
                }
            }
            __syncthreads();
        }
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = s[base + lane * E + e];
#pragma unroll
        for (uint32_t j = WCH >> 1; j > 0; j >>= 1) warp_stage<E>(v, base, k, j);
    }
    __syncthreads();  // every thread done reading s before it is overwritten
#pragma unroll
    for (int e = 0; e < E; ++e) s[base + lane * E + e] = v[e];
    __syncthreads();
}

// Products of A row i, balanced over a whole CTA.  A entries are staged in
// chunks of ECH: B-row starts and the exclusive prefix of B-row lengths go to
// shared memory; then every warp takes 32*U consecutive products of the
// flattened chunk, each lane walking its own entry cursor forward (one
// binary search per warp chunk).  Consecutive lanes read consecutive columns
// of one B row (coalesced) and each lane has U loads in flight before f runs.
// f(col, valid, idx) is called warp-uniformly (all 32 lanes, valid or not);
// idx is the product's index in the row's flattened product list.
template <int NT, int ECH, int U, class F>
__device__ __forceinline__ void balanced_products(const AView &a, const BRows &b, uint32_t i, uint32_t *s_pre,
                                                  uint32_t *s_beg, uint32_t *scratch, F &&f, uint32_t part = 0,
                                                  uint32_t nparts = 1) {
    constexpr int EPT = ECH / NT;
    constexpr int NW = NT / 32;
    constexpr uint32_t WCH = 32u * U;
    const uint32_t lane = lane_id(), w = warp_id();
    const uint64_t ja = a.rpt[i], je = a.rpt[i + 1];
    uint32_t done = 0;  // products of the row in earlier entry chunks
    for (uint64_t c0 = ja; c0 < je; c0 += ECH) {
        const uint32_t n = (uint32_t)min((uint64_t)ECH, je - c0);
        for (uint32_t e = threadIdx.x; e < n; e += NT) {
            uint64_t bb;
            const uint32_t len = b_row(b, __ldg(a.cols + c0 + e), bb);
            s_beg[e] = (uint32_t)bb;
            s_pre[e] = len;
        }
        __syncthreads();
        uint32_t v[EPT];
        uint32_t sum = 0;
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
            const uint32_t e = threadIdx.x * EPT + k;
            v[k] = e < n ? s_pre[e] : 0u;
            sum += v[k];
        }
        uint32_t total;
        uint32_t run = block_exclusive_scan<uint32_t, NT>(sum, scratch, &total);
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
            const uint32_t e = threadIdx.x * EPT + k;
            if (e < n) s_pre[e] = run;
            run += v[k];
        }
        if (threadIdx.x == 0) s_pre[n] = total;
        __syncthreads();
        uint32_t e = 0;  // lane's entry cursor, carried from chunk to chunk
        // the CTAs of a cluster (part of nparts) interleave the warp chunks
        for (uint32_t base = (part * NW + w) * WCH; base < total; base += nparts * NW * WCH) {
            const uint32_t p = base + lane;
            {   // largest e in [e, n) with s_pre[e] <= p: short linear walk,
                // binary search when the cursor is more than 8 entries behind
                const uint32_t key = p < total ? p : total - 1;
                if (e + 8 < n && s_pre[e + 8] <= key) {
                    uint32_t lo = e + 8, hi = n - 1;
                    while (lo < hi) {
                        const uint32_t m = (lo + hi + 1) >> 1;
                        if (s_pre[m] <= key) lo = m; else hi = m - 1;
                    }
                    e = lo;
                } else {
                    while (s_pre[e + 1] <= key) ++e;
                }
            }
            // The current entry's end and the offset that maps a product
            // index to its position in B.cols (mod 2^32: positions < 2^32).
            uint32_t end = s_pre[e + 1];
            uint32_t off = s_beg[e] - s_pre[e];
            uint32_t col[U];
            bool val[U];
#pragma unroll
            for (int s = 0; s < U; ++s) {
                const uint32_t q = p + (uint32_t)s * 32u;
                val[s] = q < total;
                if (val[s] && q >= end) {
                    do {
                        ++e;
                        end = s_pre[e + 1];
                    } while (q >= end);
                    off = s_beg[e] - s_pre[e];
                }
                col[s] = val[s] ? __ldg(b.cols + (q + off)) : 0u;
            }
#pragma unroll
            for (int s = 0; s < U; ++s) f(col[s], val[s], done + p + (uint32_t)s * 32u);
        }
        done += total;
        __syncthreads();
    }
}

// Next work item of a dynamically scheduled persistent CTA.
__device__ __forceinline__ uint32_t next_item(uint32_t *counter, uint32_t *s_slot) {
    if (threadIdx.x == 0) *s_slot = atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t it = *s_slot;
    __syncthreads();
    return it;
}

constexpr int HASH_ECH = 1024;

template <int T, int NT, bool NUMERIC>
__global__ void __launch_bounds__(NT) hash_cta_kernel(BinLists bl, int bin, AView a, BRows b, RowOut o,
                                                      uint32_t *counter) {
    constexpr int SPT = T / NT;  // slots per thread
    __shared__ uint32_t table[T];
    __shared__ uint32_t s_pre[HASH_ECH + 1];
    __shared__ uint32_t s_beg[HASH_ECH];
    __shared__ uint32_t scratch[33];
    __shared__ uint32_t s_slot, s_full;
    uint32_t beg, cnt;
    bin_range(bl, bin, beg, cnt);
    for (;;) {
        const uint32_t item = next_item(counter, &s_slot);
        if (item >= cnt) break;
        const uint32_t i = bl.list[beg + item];
        for (int s = threadIdx.x; s < T; s += NT) table[s] = EMPTY;
        if (threadIdx.x == 0) s_full = 0;
        __syncthreads();
        uint32_t mine = 0;
        // With capacities (single-pass forms) a table that fills up means the
        // row outgrew its capacity: flag the row instead of the device status.
        uint32_t *probe_flag = o.row_cap ? &s_full : o.status;
        balanced_products<NT, HASH_ECH, 4>(a, b, i, s_pre, s_beg, scratch, [&](uint32_t c, bool valid, uint32_t) {
            if (valid) mine += hash_insert<T>(table, c, probe_flag);
        });
        if (o.row_cap && s_full) {  // block-uniform after the iterator's barrier
            if (threadIdx.x == 0) o.overflow[i] = 1;
            __syncthreads();
            continue;
        }
        if (!NUMERIC) {
            uint32_t total = block_sum<uint32_t, NT>(mine, scratch);
            if (threadIdx.x == 0) o.row_nnz[i] = total;
            continue;
        }
        uint32_t keys[SPT];
        uint32_t kc = 0;
#pragma unroll
        for (int s = 0; s < SPT; ++s) {
            keys[s] = table[threadIdx.x * SPT + s];
            kc += keys[s] != EMPTY ? 1u : 0u;
        }
        uint32_t nnz;
        uint32_t w = block_exclusive_scan<uint32_t, NT>(kc, scratch, &nnz);
        if (o.row_cap && nnz > o.row_cap[i]) {
            if (threadIdx.x == 0) o.overflow[i] = 1;
            continue;  // every thread takes this branch (nnz is block-uniform)
        }
#pragma unroll
        for (int s = 0; s < SPT; ++s)
            if (keys[s] != EMPTY) table[w++] = keys[s];
        __syncthreads();
        // the compacted keys (nnz <= T/2) padded to T/2 and sorted
        for (uint32_t s = nnz + threadIdx.x; s < (uint32_t)(T / 2); s += NT) table[s] = EMPTY;
        __syncthreads();
        block_sort_hybrid<NT, T / 2 / NT>(table);
        uint32_t *dst = o.cols + o.row_off[i];
        for (uint32_t s = threadIdx.x; s < nnz; s += NT) dst[s] = table[s];
        if (o.row_cap && threadIdx.x == 0) o.row_nnz[i] = nnz;
        __syncthreads();
    }
}

// ----------------------------------------------------------- CTA bitmap ----
constexpr int BMP_ECH = 1024;                 // A entries staged per chunk
constexpr uint32_t BMP_MAX_WORDS = 32768;     // 128 KB: 2^20 columns per chunk
constexpr int BMP_U = 8;                      // B-column loads in flight per lane
constexpr uint32_t BMP_STEP_WORDS = 128;      // emission step: 4 words per lane
constexpr uint32_t BMP_MAX_STEPS = BMP_MAX_WORDS / BMP_STEP_WORDS;
// A deferred row's step record: count of non-empty steps | the steps
// (BMP_MAX_STEPS) | their first outputs and the row's total (BMP_MAX_STEPS + 1).
constexpr uint32_t BMP_STEP_REC = 2 + 2 * BMP_MAX_STEPS;
constexpr uint32_t BMP_STAGE = 256;           // per-warp output staging (columns)
// Bitmaps at least this wide (2^18 columns) may be kept for the expansion
// kernels: narrower ones cost more per row to reload than their compaction.
constexpr uint32_t BMP_DEFER_MIN_WORDS = 8192;
// Rows with at least 1 / BMP_DEFER_DIV of their bitmap's words in outputs
// are deferred when their slot holds the bitmap.
constexpr uint32_t BMP_DEFER_DIV = 4;
constexpr uint32_t BMP_FEW = 16;  // steps with at most this many outputs skip the balanced windows
constexpr uint32_t BMP_DENSE = 1024;  // steps with at least this many outputs (1/4 of the bits) emit bit-parallel
constexpr uint32_t BMP_SHORT = 64;            // products per A entry below which a row uses the per-product mapping

// Words of the bitmap for `ncols` columns: a multiple of the emission step,
// at most BMP_MAX_WORDS.
__host__ __device__ inline uint32_t bitmap_words(uint64_t ncols) {
    uint64_t w = (ncols + 31) / 32;
    w = (w + BMP_STEP_WORDS - 1) / BMP_STEP_WORDS * BMP_STEP_WORDS;
    if (w > BMP_MAX_WORDS) w = BMP_MAX_WORDS;
    return (uint32_t)w;
}

// Dynamic shared memory of the bitmap kernel (32-bit words): bitmap W |
// entry stage (B row start, length, unit prefix) | non-empty step list and
// output offsets | per-warp output staging.
inline size_t bitmap_smem_bytes(uint32_t W, int nt) {
    return ((size_t)W + 3 * BMP_ECH + 1 + 2 * BMP_MAX_STEPS + 1 + (size_t)(nt / 32) * BMP_STAGE) * 4;
}

// Position of the n-th (0-based) set bit of w; w has more than n set bits.
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t w, uint32_t n) {
    uint32_t pos = 0, c;
    c = __popc(w & 0xFFFFu);
    if (n >= c) { n -= c; w >>= 16; pos += 16; }
    c = __popc(w & 0xFFu);
    if (n >= c) { n -= c; w >>= 8; pos += 8; }
    c = __popc(w & 0xFu);
    if (n >= c) { n -= c; w >>= 4; pos += 4; }
    c = __popc(w & 0x3u);
    if (n >= c) { n -= c; w >>= 2; pos += 2; }
    c = w & 1u;
    if (n >= c) pos += 1;
    return pos;
}

// Products of A row i in units of up to 2^shift products that read ONE B
// row: warp w takes units w, w + NW, ... of each staged chunk of ECH A
// entries, and its lanes read the unit's B columns with stride 32 (coalesced,
// BMP_U loads in flight per lane), calling f(col, valid) warp-uniformly for
// every 32 consecutive positions.  No per-product search: the entry of a
// unit is found once by a warp-wide ballot over the unit prefix (the warp's
// cursor only moves forward).  Chunk stage: s_beg = B row start, s_len = B
// row length, s_upre = exclusive prefix of units.  Requires B.nnz < 2^32.
template <int NT, int ECH, class F>
__device__ __forceinline__ void unit_products(const AView &a, const BRows &b, uint32_t i, uint32_t shift,
                                              uint32_t *s_beg, uint32_t *s_len, uint32_t *s_upre, uint32_t *scratch,
                                              F &&f) {
    static_assert(ECH % NT == 0, "entry chunk must be a multiple of the block");
    constexpr int EPT = ECH / NT;
    constexpr int NW = NT / 32;
    const uint32_t unit = 1u << shift;
    const uint32_t lane = lane_id(), w = warp_id();
    const uint64_t ja = a.rpt[i], je = a.rpt[i + 1];
    for (uint64_t c0 = ja; c0 < je; c0 += ECH) {
        const uint32_t n = (uint32_t)min((uint64_t)ECH, je - c0);
        uint32_t units[EPT], sum = 0;
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
            const uint32_t e = threadIdx.x * EPT + k;
            uint32_t len = 0;
            if (e < n) {
                uint64_t bb;
                len = b_row(b, __ldg(a.cols + c0 + e), bb);
                s_beg[e] = (uint32_t)bb;
                s_len[e] = len;
            }
            units[k] = (len + unit - 1) >> shift;
            sum += units[k];
        }
        uint32_t total;
        uint32_t run = block_exclusive_scan<uint32_t, NT>(sum, scratch, &total);
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
            const uint32_t e = threadIdx.x * EPT + k;
            if (e < n) s_upre[e] = run;
            run += units[k];
        }
        if (threadIdx.x == 0) s_upre[n] = total;
        __syncthreads();
        uint32_t e = 0;  // warp-uniform entry cursor
        for (uint32_t u = w; u < total; u += NW) {
            // largest e with s_upre[e] <= u: s_upre is non-decreasing and
            // s_upre[n] = total > u, so the lanes that pass form a prefix
            for (;;) {
                const uint32_t idx = e + 1 + lane;
                const bool le = idx <= n && s_upre[idx] <= u;
                const uint32_t m = __ballot_sync(0xFFFFFFFFu, le);
                e += __popc(m);
                if (m != 0xFFFFFFFFu) break;
            }
            const uint32_t first = (u - s_upre[e]) << shift;
            const uint32_t cnt = min(unit, s_len[e] - first);
            const uint32_t *src = b.cols + s_beg[e] + first;
            // whole sweeps of 32 * BMP_U positions: no per-position checks
            const uint32_t full = cnt / (32u * BMP_U) * (32u * BMP_U);
#pragma unroll 1
            for (uint32_t k0 = 0; k0 < full; k0 += 32u * BMP_U) {
                uint32_t col[BMP_U];
#pragma unroll
                for (int s = 0; s < BMP_U; ++s) col[s] = __ldg(src + k0 + (uint32_t)s * 32u + lane);
#pragma unroll
                for (int s = 0; s < BMP_U; ++s) f(col[s], true);
            }
#pragma unroll 1
            for (uint32_t k0 = full; k0 < cnt; k0 += 32u * BMP_U) {
                uint32_t col[BMP_U];
#pragma unroll
                for (int s = 0; s < BMP_U; ++s) {
                    const uint32_t q = k0 + (uint32_t)s * 32u + lane;
                    col[s] = q < cnt ? __ldg(src + q) : 0u;
                }
#pragma unroll
                for (int s = 0; s < BMP_U; ++s) {
                    if (k0 + (uint32_t)s * 32u < cnt)  // warp-uniform
                        f(col[s], k0 + (uint32_t)s * 32u + lane < cnt);
                }
            }
        }
        __syncthreads();
    }
}

// Single-chunk insertion (all columns fit the bitmap, or the cluster's
// bitmaps: `set_bit(c)` sets column c wherever it lives).  Units are the
// intersections of a B row with ALIGNED windows of 2^shift positions of
// B.cols, so all but a row's first and last unit are whole windows.  A warp
// sweeps 256 positions at a time; lane l takes the 8 consecutive positions
// 8l..8l+7 of the sweep (two 16-byte loads when B.cols is 16-byte aligned,
// coalesced over the warp) and issues one atomic per position, slot by slot:
// in each atomic instruction the lanes are 8 positions of a sorted B row
// apart, so they rarely share a word or a bank (neighbouring positions did,
// and those atomics serialised).  A 16-byte load is issued only when it
// covers a valid position, so it never leaves the 16-byte block of a valid
// column.  Columns are clamped to the bitmap (memory safety on malformed
// input).  Requires B.nnz <= 2^32 - 4096.
//
// With B's word runs (b.wpairs: (word, bits) per run of entries in one
// bitmap word, built once per call), the same sweeps run over the pairs and
// `set_word(w, m)` issues one atomic per run instead of one per entry: on
// R-MAT scale 20 the products fall in 1.69 times fewer words than entries.
// The runs of a unit lie in distinct words (one B row), so there the lanes
// of an instruction take 32 consecutive runs.
template <int NT, int ECH, class SetBit, class SetWord>
__device__ __forceinline__ void bitmap_insert_row(const AView &a, const BRows &b, uint32_t i, uint32_t shift,
                                                  uint32_t maxcol, SetBit &&set_bit, SetWord &&set_word,
                                                  uint32_t *s_beg, uint32_t *s_len, uint32_t *s_upre,
                                                  uint32_t *scratch, uint32_t part = 0, uint32_t nparts = 1) {
    const bool words = b.wpairs != nullptr;
    const uint32_t maxword = maxcol >> 5;
    static_assert(ECH % NT == 0, "entry chunk must be a multiple of the block");
    constexpr int EPT = ECH / NT;
    constexpr int NW = NT / 32;
    const uint32_t unit = 1u << shift;
    const uint32_t lane = lane_id(), w = warp_id();
    const bool vec = (reinterpret_cast<uintptr_t>(b.cols) & 15u) == 0;
    const uint64_t ja = a.rpt[i], je = a.rpt[i + 1];
    for (uint64_t c0 = ja; c0 < je; c0 += ECH) {
        const uint32_t n = (uint32_t)min((uint64_t)ECH, je - c0);
        uint32_t units[EPT], sum = 0;
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
            const uint32_t e = threadIdx.x * EPT + k;
            units[k] = 0;
            if (e < n) {
                uint64_t bb;
                const uint32_t k_col = __ldg(a.cols + c0 + e);
                const uint32_t len = words ? b_words(b, k_col, bb) : b_row(b, k_col, bb);
                s_beg[e] = (uint32_t)bb;
                s_len[e] = len;
                if (len) units[k] = (uint32_t)(((bb + len - 1) >> shift) - (bb >> shift) + 1);
            }
            sum += units[k];
        }
        uint32_t total;
        uint32_t run = block_exclusive_scan<uint32_t, NT>(sum, scratch, &total);
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
            const uint32_t e = threadIdx.x * EPT + k;
            if (e < n) s_upre[e] = run;
            run += units[k];
        }
        if (threadIdx.x == 0) s_upre[n] = total;
        __syncthreads();
        uint32_t e = 0;  // warp-uniform entry cursor
        for (uint32_t u = part * NW + w; u < total; u += nparts * NW) {
            for (;;) {
                const uint32_t idx = e + 1 + lane;
                const bool le = idx <= n && s_upre[idx] <= u;
                const uint32_t m = __ballot_sync(0xFFFFFFFFu, le);
                e += __popc(m);
                if (m != 0xFFFFFFFFu) break;
            }
            const uint32_t beg = s_beg[e];
            const uint32_t ws = ((beg >> shift) + (u - s_upre[e])) << shift;  // window start
            const uint32_t vlo = max(beg, ws), vhi = min(beg + s_len[e], ws + unit);
#pragma unroll 1
            for (uint32_t k0 = ws; k0 < vhi; k0 += 256u) {
                const uint32_t p0 = k0 + lane * 8u;
                if (words) {
                    // eight pairs per lane, lanes 32 pairs apart in each of
                    // them: a unit's runs come from one B row, so they lie in
                    // distinct, increasing words, and the 32 atomics of one
                    // instruction hit neighbouring words in distinct banks
                    // (lanes 8 pairs apart put several lanes on one bank).
                    // Each load instruction reads 32 consecutive pairs.
                    uint2 t[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const uint32_t q = k0 + 32u * (uint32_t)j + lane;
                        t[j] = (q >= vlo && q < vhi) ? __ldg(b.wpairs + q) : make_uint2(0, 0);
                    }
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const uint32_t q = k0 + 32u * (uint32_t)j + lane;
                        if (q >= vlo && q < vhi) set_word(min(t[j].x, maxword), t[j].y);
                    }
                    continue;
                }
                uint32_t v[8];
                if (vec) {
                    const uint4 *p4 = reinterpret_cast<const uint4 *>(b.cols + p0);
                    const uint4 x = (p0 + 4u > vlo && p0 < vhi) ? __ldg(p4) : make_uint4(0, 0, 0, 0);
                    const uint4 y = (p0 + 8u > vlo && p0 + 4u < vhi) ? __ldg(p4 + 1) : make_uint4(0, 0, 0, 0);
                    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
                    v[4] = y.x; v[5] = y.y; v[6] = y.z; v[7] = y.w;
                } else {
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const uint32_t q = p0 + (uint32_t)j;
                        v[j] = (q >= vlo && q < vhi) ? __ldg(b.cols + q) : 0u;
                    }
                }
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const uint32_t q = p0 + (uint32_t)j;
                    if (q >= vlo && q < vhi) {
                        set_bit(min(v[j], maxcol));
                    }
                }
            }
        }
        __syncthreads();
    }
}

// ---- chunk counting and emission, shared by the bitmap kernels ----------

// Pop-counts and clears `words` words of the bitmap; returns the block's sum.
template <int BMP_NT>
__device__ __forceinline__ uint32_t bitmap_count_clear(uint4 *bm4, uint32_t words, uint32_t *scratch) {
    uint32_t mine = 0;
    for (uint32_t w4 = threadIdx.x; w4 < words / 4; w4 += BMP_NT) {
        const uint4 x = bm4[w4];
        mine += __popc(x.x) + __popc(x.y) + __popc(x.z) + __popc(x.w);
        bm4[w4] = make_uint4(0, 0, 0, 0);
    }
    return block_sum<uint32_t, BMP_NT>(mine, scratch);
}

// Counts the set bits of the `nsteps` 128-word steps and lists the non-empty
// ones: s_list[g] = step, s_soff[g] = its first output, s_soff[nlist] =
// total.  TPS threads count one step (32 uint4); thread TPS*s ends up holding
// step s; one block scan of (count << 11 | nonempty) gives both offsets
// (counts <= 4096 per step, <= 2^20 per chunk; flags <= 256 < 2^11).
// Resets *s_next and ends with a block barrier.
template <int BMP_NT>
__device__ __forceinline__ uint32_t bitmap_list_steps(const uint4 *bm4, uint32_t nsteps, uint32_t *s_list,
                                                      uint32_t *s_soff, uint32_t *s_next, uint32_t *scratch,
                                                      uint32_t &nlist) {
    constexpr int TPS = BMP_NT / (int)BMP_MAX_STEPS;
    static_assert(TPS >= 1 && TPS <= 32 && (TPS & (TPS - 1)) == 0, "block size");
    uint32_t scnt = 0;
    if (threadIdx.x / TPS < nsteps) {
        const uint4 *p4 = bm4 + (threadIdx.x / TPS) * 32 + (threadIdx.x % TPS) * (32 / TPS);
#pragma unroll 8
        for (int k = 0; k < 32 / TPS; ++k) {
            const uint4 x = p4[k];
            scnt += __popc(x.x) + __popc(x.y) + __popc(x.z) + __popc(x.w);
        }
    }
#pragma unroll
    for (int d = 1; d < TPS; d <<= 1) scnt += __shfl_xor_sync(0xFFFFFFFFu, scnt, d);
    if ((threadIdx.x % TPS) != 0) scnt = 0;
    uint32_t ptot;
    const uint32_t ex = block_exclusive_scan<uint32_t, BMP_NT>((scnt << 11) | (scnt ? 1u : 0u), scratch, &ptot);
    const uint32_t ctot = ptot >> 11;
    nlist = ptot & 0x7FFu;
    if (scnt) {
        s_list[ex & 0x7FFu] = threadIdx.x / TPS;
        s_soff[ex & 0x7FFu] = ex >> 11;
    }
    if (threadIdx.x == 0) {
        s_soff[nlist] = ctot;
        *s_next = 0;
    }
    __syncthreads();
    return ctot;
}

// Emits one 128-word step holding T > 0 set bits, stored at sbm in shared
// memory, as the sorted columns cb + bit index to out[0, T); CLEAR zeroes
// the step's words after.  Lane l holds words 4l..4l+3 and a warp scan of
// their counts places them; the step's outputs are produced in windows of up
// to BMP_STAGE: the window's outputs are split evenly over the lanes, each
// lane finds the word and bit of its first output (shuffle search over the
// scan, then nth_set_bit) and walks the bitmap from there into the warp's
// staging buffer, which the warp copies out with coalesced stores.  A step
// with at most BMP_FEW outputs skips the windows: each lane writes its own
// bits at its scan offset.  A step with at least BMP_DENSE outputs is
// emitted bit-parallel instead.
template <bool CLEAR>
__device__ __forceinline__ void bitmap_emit_step(uint32_t *sbm, uint32_t T, uint32_t *out, uint32_t cb0,
                                                 uint32_t *stage) {
    const uint32_t lane = lane_id();
    uint4 *const sbm4 = reinterpret_cast<uint4 *>(sbm);
    if (T >= BMP_DENSE) {
        // dense step: bit-parallel.  Lane l tests bit l of every word (one
        // broadcast 16-byte load per four words); a word's outputs land at
        // consecutive addresses, one store instruction per word.
        const uint32_t lb = 1u << lane, lt = lb - 1u;
        const uint32_t cb = cb0 + lane;
        uint32_t off = 0;
#pragma unroll 4
        for (uint32_t q = 0; q < 32; ++q) {
            const uint4 y = sbm4[q];
            const uint32_t c = cb + q * 128u;
            if (y.x & lb) out[off + __popc(y.x & lt)] = c;
            off += __popc(y.x);
            if (y.y & lb) out[off + __popc(y.y & lt)] = c + 32u;
            off += __popc(y.y);
            if (y.z & lb) out[off + __popc(y.z & lt)] = c + 64u;
            off += __popc(y.z);
            if (y.w & lb) out[off + __popc(y.w & lt)] = c + 96u;
            off += __popc(y.w);
        }
        __syncwarp();  // every lane has read the step
        if (CLEAR) sbm4[lane] = make_uint4(0, 0, 0, 0);
        return;
    }
    const uint4 x = sbm4[lane];
    const uint32_t pc = __popc(x.x) + __popc(x.y) + __popc(x.z) + __popc(x.w);
    const uint32_t inc = warp_inclusive_scan(pc);
    if (T <= BMP_FEW) {
        // few outputs (a quarter of the steps of R-MAT rows hold <= 8):
        // every lane writes its own bits in place, no search, no staging
        uint32_t *o = out + inc - pc;
        const uint32_t wb = cb0 + lane * 128u;
        uint32_t cur = x.x, j = 0;
        for (uint32_t t = 0; t < pc; ++t) {
            while (!cur) {
                ++j;
                cur = j == 1 ? x.y : (j == 2 ? x.z : x.w);
            }
            o[t] = wb + j * 32u + (uint32_t)(__ffs(cur) - 1);
            cur &= cur - 1;
        }
        if (CLEAR && pc) sbm4[lane] = make_uint4(0, 0, 0, 0);
        return;
    }
    for (uint32_t w0 = 0; w0 < T; w0 += BMP_STAGE) {
        const uint32_t m = min(BMP_STAGE, T - w0);
        const uint32_t per = (m + 31) >> 5;  // outputs per lane
        const uint32_t k = w0 + lane * per;
        const uint32_t kend = min(k + per, w0 + m);
        const uint32_t key = min(k, T - 1);
        // L = first lane whose inclusive count exceeds key
        uint32_t L = 0;
#pragma unroll
        for (uint32_t sft = 16; sft >= 1; sft >>= 1) {
            const uint32_t v = __shfl_sync(0xFFFFFFFFu, inc, L + sft - 1);
            if (v <= key) L += sft;
        }
        const uint32_t exL = __shfl_sync(0xFFFFFFFFu, inc - pc, L);
        if (k < kend) {
            const uint4 y = sbm4[L];
            uint32_t r = key - exL, wv = y.x, widx = L * 4u, c;
            c = __popc(y.x);
            if (r >= c) {
                r -= c; wv = y.y; ++widx; c = __popc(y.y);
                if (r >= c) {
                    r -= c; wv = y.z; ++widx; c = __popc(y.z);
                    if (r >= c) { r -= c; wv = y.w; ++widx; }
                }
            }
            uint32_t cur = wv & (0xFFFFFFFFu << nth_set_bit(wv, r));
            for (uint32_t kk = k; kk < kend; ++kk) {
                while (!cur) cur = sbm[++widx];  // the step holds more outputs
                stage[kk - w0] = cb0 + widx * 32u + (uint32_t)(__ffs(cur) - 1);
                cur &= cur - 1;
            }
        }
        __syncwarp();
        uint32_t *const o2 = out + w0 + lane;
#pragma unroll
        for (uint32_t u = 0; u < BMP_STAGE / 32; ++u)
            if (lane + 32 * u < m) o2[32 * u] = stage[lane + 32 * u];
        __syncwarp();
    }
    if (CLEAR && pc) sbm4[lane] = make_uint4(0, 0, 0, 0);
}

// Emits the listed steps (bitmap_list_steps) as sorted columns colbase + bit
// index to out[], clearing the bitmap; warps take steps dynamically
// (bitmap_emit_step).  Cost follows the non-empty steps and the output, not
// the bitmap width.  The caller synchronises the block after.
__device__ __forceinline__ void bitmap_emit(uint32_t *bm, uint32_t nlist, const uint32_t *s_list,
                                            const uint32_t *s_soff, uint32_t *s_next, uint32_t *stage, uint32_t *out,
                                            uint32_t colbase) {
    const uint32_t lane = lane_id();
    for (;;) {
        uint32_t g = 0;
        if (lane == 0) g = atomicAdd(s_next, 1u);
        g = __shfl_sync(0xFFFFFFFFu, g, 0);
        if (g >= nlist) break;
        const uint32_t st = s_list[g];
        const uint32_t pos = s_soff[g];
        bitmap_emit_step<true>(bm + st * BMP_STEP_WORDS, s_soff[g + 1] - pos, out + pos,
                               colbase + st * (BMP_STEP_WORDS * 32u), stage);
    }
}

// One level of pairwise merges: segments [sb[2i], sb[2i+1]) and
// [sb[2i+1], sb[2i+2]) of src (nseg segments, sb[nseg] = P) merge into
// [sb[2i], sb[2i+2]) of dst, A side first on ties.  Each thread writes ITEMS
// consecutive outputs: it finds their pair, splits the pair by a merge-path
// search and merges sequentially.
template <int NT, int ITEMS>
__device__ __forceinline__ void merge_level(const uint32_t *src, uint32_t *dst, const uint32_t *sb, uint32_t nseg,
                                            uint32_t P) {
    const uint32_t npairs = (nseg + 1) / 2;
    for (uint32_t p0 = threadIdx.x * ITEMS; p0 < P; p0 += NT * ITEMS) {
        uint32_t p = p0;
        const uint32_t pend = min(p0 + (uint32_t)ITEMS, P);
        while (p < pend) {
            uint32_t lo = 0, hi = npairs - 1;  // last pair starting at or before p
            while (lo < hi) {
                const uint32_t m = (lo + hi + 1) >> 1;
                if (sb[2 * m] <= p) lo = m; else hi = m - 1;
            }
            const uint32_t a0 = sb[2 * lo], a1 = sb[min(2 * lo + 1, nseg)], b1 = sb[min(2 * lo + 2, nseg)];
            const uint32_t la = a1 - a0, lb = b1 - a1, d = p - a0;
            uint32_t x0 = d > lb ? d - lb : 0, x1 = min(d, la);
            while (x0 < x1) {
                const uint32_t m = (x0 + x1) >> 1;
                if (src[a0 + m] <= src[a1 + d - 1 - m]) x0 = m + 1; else x1 = m;
            }
            uint32_t ia = x0, ib = d - x0;
            const uint32_t stop = min(pend, b1);
            for (; p < stop; ++p) {
                const bool take_a = ib >= lb || (ia < la && src[a0 + ia] <= src[a1 + ib]);
                dst[p] = take_a ? src[a0 + ia++] : src[a1 + ib++];
            }
        }
    }
}

// Rows whose A entries are few merge their B rows (each sorted) instead of
// sorting or bitmapping all products.
constexpr uint32_t MERGE_SEGS = 64;

// Sorts the products of A row i (at most MERGE_SEGS A entries), expanded into
// buf0[0, P) in A-entry order, by pairwise merges of the B rows; returns the
// buffer holding the result (buf0 or buf1).  sb: MERGE_SEGS + 1 words of
// shared memory.  Ends with a block barrier.
template <int NT, int ITEMS>
__device__ __forceinline__ uint32_t *merge_row_segments(const AView &a, const BRows &b, uint32_t i, uint32_t P,
                                                         uint32_t *buf0, uint32_t *buf1, uint32_t *sb) {
    const uint64_t ja = a.rpt[i];
    const uint32_t nseg0 = (uint32_t)(a.rpt[i + 1] - ja);
    if (warp_id() == 0) {  // bounds = prefix of the B-row lengths (clamped to P)
        const uint32_t lane = lane_id();
        uint64_t bb;
        const uint32_t l0 = lane < nseg0 ? b_row(b, __ldg(a.cols + ja + lane), bb) : 0u;
        const uint32_t l1 = lane + 32 < nseg0 ? b_row(b, __ldg(a.cols + ja + lane + 32), bb) : 0u;
        const uint32_t i0 = warp_inclusive_scan(l0);
        const uint32_t t0 = __shfl_sync(0xFFFFFFFFu, i0, 31);
        const uint32_t i1 = warp_inclusive_scan(l1);
        if (lane < nseg0) sb[lane] = min(i0 - l0, P);
        if (lane + 32 < nseg0) sb[lane + 32] = min(t0 + i1 - l1, P);
        if (lane == 0) sb[nseg0] = P;
    }
    __syncthreads();
    uint32_t nseg = nseg0;
    uint32_t *src = buf0, *dst = buf1;
    while (nseg > 1) {
        merge_level<NT, ITEMS>(src, dst, sb, nseg, P);
        const uint32_t nn = (nseg + 1) / 2;
        const uint32_t nb = threadIdx.x < nn ? sb[2 * threadIdx.x] : 0u;
        __syncthreads();
        if (threadIdx.x < nn) sb[threadIdx.x] = nb;
        if (threadIdx.x == 0) sb[nn] = P;
        __syncthreads();
        nseg = nn;
        uint32_t *t = src;
        src = dst;
        dst = t;
    }
    return src;
}

// Shared-memory layout of the bitmap kernels (32-bit words, bitmap of W).
struct BitmapSmem {
    uint32_t *bm, *s_beg, *s_len, *s_upre, *s_list, *s_soff, *s_stage;
    __device__ __forceinline__ BitmapSmem(uint32_t *smem, uint32_t W) {
        bm = smem;
        s_beg = smem + W;
        s_len = s_beg + BMP_ECH;
        s_upre = s_len + BMP_ECH;             // BMP_ECH + 1
        s_list = s_upre + BMP_ECH + 1;        // BMP_MAX_STEPS
        s_soff = s_list + BMP_MAX_STEPS;      // BMP_MAX_STEPS + 1
        s_stage = s_soff + BMP_MAX_STEPS + 1; // (threads / 32) * BMP_STAGE
    }
};

// Rows of bins [bin_lo, bin_hi] (contiguous in the list, heaviest first),
// one row per CTA at a time, taken from `counter`.  MULTI: the columns do
// not fit one bitmap chunk, so every chunk re-walks the row's products.
// Insertion units: 512 products for rows over 2^17 products, 256 below (so
// the 32 warps of a lighter row still get several units each).  Plain
// shared atomics: B rows are mostly sparse over 2^20 columns, and warp-level
// aggregation of same-word bits cost more instructions than the conflicts
// it saved (measured on R-MAT scale 20).  Emission in 128-word steps
// (bitmap_list_steps, bitmap_emit).
template <bool NUMERIC, bool MULTI, int BMP_NT>
__global__ void __launch_bounds__(BMP_NT, 1024 / BMP_NT) bitmap_cta_kernel(BinLists bl, int bin_lo, int bin_hi, AView a, BRows b,
                                                               RowOut o, uint64_t ncols, uint32_t W,
                                                               uint32_t *counter) {
    extern __shared__ __align__(16) uint32_t smem[];
    const BitmapSmem S(smem, W);
    uint32_t *const bm = S.bm;
    __shared__ uint32_t scratch[33];
    __shared__ uint32_t s_slot, s_row, s_next, s_dslot;
    __shared__ unsigned long long s_spill;
    uint32_t beg, cnt = 0, tmp;
    bin_range(bl, bin_lo, beg, tmp);
    for (int q = bin_lo; q <= bin_hi; ++q) cnt += bl.info[q];
    // rows of the bins above BIN_BMP (over 2^17 products) come first
    const uint32_t nheavy = bin_hi > bin_lo ? cnt - bl.info[bin_hi] : 0;
    // Rows are claimed one ahead: the claim of the next row (a global atomic)
    // and its row index are in flight while this row runs, and thread 0
    // publishes both at the row's end (s_slot, s_row).
    if (threadIdx.x == 0) {
        const uint32_t it = atomicAdd(counter, 1u);
        s_slot = it;
        s_row = it < cnt ? bl.list[beg + it] : 0;
    }
    for (uint32_t w = threadIdx.x; w < W; w += BMP_NT) bm[w] = 0;
    __syncthreads();
    uint4 *bm4 = reinterpret_cast<uint4 *>(bm);
    uint32_t *const stage = S.s_stage + warp_id() * BMP_STAGE;
    for (;;) {
        const uint32_t item = s_slot;
        if (item >= cnt) break;
        const uint32_t i = s_row;
        uint32_t nxt = 0;  // thread 0: the next row's claim, read at the row's end
        if (threadIdx.x == 0) nxt = atomicAdd(counter, 1u);
        const uint32_t shift = item < nheavy ? 9u : 8u;
        // this row's columns (a batched pair can be narrower than the batch)
        const uint64_t rn = o.row_ncols ? (uint64_t)o.row_ncols[i] : ncols;
        const uint32_t Wr = bitmap_words(rn);
        const uint64_t chunk_cols = (uint64_t)Wr * 32;
        const uint32_t nsteps = Wr / BMP_STEP_WORDS;  // <= BMP_MAX_STEPS
        // Rows whose B rows average fewer than BMP_SHORT products would
        // leave most lanes of a unit idle: they take the per-product mapping.
        const bool short_b = o.row_products &&
                             (uint64_t)o.row_products[i] < (uint64_t)BMP_SHORT * (a.rpt[i + 1] - a.rpt[i]);
        uint64_t total = 0;
        const uint64_t out_base = NUMERIC ? o.row_off[i] : 0;
        bool overflowed = false;
        for (uint64_t c0 = 0; c0 < (MULTI ? rn : 1); c0 += chunk_cols) {
            if (MULTI) {
                unit_products<BMP_NT, BMP_ECH>(a, b, i, shift, S.s_beg, S.s_len, S.s_upre, scratch,
                                               [&](uint32_t c, bool valid) {
                    const uint64_t r = (uint64_t)c - c0;  // wraps for columns below c0
                    if (valid && r < chunk_cols) atomicOr(bm + (r >> 5), 1u << (r & 31));
                });
            } else if (short_b) {
                // many short B rows: per-product mapping over the whole row
                balanced_products<BMP_NT, BMP_ECH, 4>(a, b, i, S.s_upre, S.s_beg, scratch,
                                                      [&](uint32_t c, bool valid, uint32_t) {
                    if (valid && c < (uint32_t)chunk_cols) atomicOr(bm + (c >> 5), 1u << (c & 31));
                });
            } else {
                bitmap_insert_row<BMP_NT, BMP_ECH>(a, b, i, shift, (uint32_t)(chunk_cols - 1),
                                                   [&](uint32_t c) { atomicOr(bm + (c >> 5), 1u << (c & 31)); },
                                                   [&](uint32_t wd, uint32_t mk) { atomicOr(bm + wd, mk); },
                                                   S.s_beg, S.s_len, S.s_upre, scratch);
            }
            if (threadIdx.x == 0 && c0 == 0 && nxt < cnt)
                asm volatile("prefetch.global.L1 [%0];" ::"l"(bl.list + beg + nxt));
            if (!NUMERIC && !MULTI && o.keep && Wr <= o.keep_stride) {
                // two-pass form keeping its bitmaps: count by steps, store the
                // bitmap and its step record for the numeric pass's expansion
                uint32_t nlist;
                const uint32_t ctot =
                    bitmap_list_steps<BMP_NT>(bm4, nsteps, S.s_list, S.s_soff, &s_next, scratch, nlist);
                uint4 *dst = reinterpret_cast<uint4 *>(o.keep + (uint64_t)item * o.keep_stride);
                for (uint32_t w4 = threadIdx.x; w4 < Wr / 4; w4 += BMP_NT) {
                    __stcs(dst + w4, bm4[w4]);  // read once, by the expansion
                    bm4[w4] = make_uint4(0, 0, 0, 0);
                }
                uint32_t *rec = o.defer_steps + (uint64_t)item * BMP_STEP_REC;
                for (uint32_t g = threadIdx.x; g <= nlist; g += BMP_NT) {
                    if (g < nlist) rec[1 + g] = S.s_list[g];
                    rec[1 + BMP_MAX_STEPS + g] = S.s_soff[g];
                }
                if (threadIdx.x == 0) {
                    rec[0] = nlist;
                    o.defer_list[item] = i;
                    o.keep_off[i] = (uint64_t)item * o.keep_stride;
                }
                total += ctot;
                __syncthreads();
                continue;
            }
            if (!NUMERIC || overflowed) {
                total += bitmap_count_clear<BMP_NT>(bm4, Wr, scratch);
                continue;
            }
            uint32_t nlist;
            const uint32_t ctot = bitmap_list_steps<BMP_NT>(bm4, nsteps, S.s_list, S.s_soff, &s_next, scratch, nlist);
            uint32_t *out = o.cols + out_base + total;
            bool in_slot = true;
            if (o.row_cap && total + ctot > o.row_cap[i]) {
                // single-pass forms: the row does not fit its slot.  A
                // single-chunk row knows its exact count now: reserve it in
                // the spill arena and emit there.  Otherwise clear the bitmap
                // and flag the row for the exact recomputation.
                if (!MULTI && o.arena) {
                    if (threadIdx.x == 0) {
                        // reservations keep 16-byte alignment (vector compaction)
                        const unsigned long long at =
                            atomicAdd(o.arena_cursor, (unsigned long long)((ctot + 3u) & ~3u));
                        s_spill = at + ctot <= o.arena_cap ? at : ~0ull;
                    }
                    __syncthreads();
                }
                if (MULTI || !o.arena || s_spill == ~0ull) {
                    overflowed = true;
                    for (uint32_t w4 = threadIdx.x; w4 < Wr / 4; w4 += BMP_NT) bm4[w4] = make_uint4(0, 0, 0, 0);
                    total += ctot;
                    __syncthreads();
                    continue;
                }
                out = o.arena + s_spill;
                in_slot = false;
                if (threadIdx.x == 0) o.spill[i] = s_spill;
            }
            if (!MULTI && o.defer && in_slot && o.row_cap && o.row_cap[i] >= Wr &&
                (uint64_t)ctot * BMP_DEFER_DIV >= Wr && Wr >= BMP_DEFER_MIN_WORDS) {
                // the slot holds the bitmap (16-byte aligned, >= Wr words):
                // it is stored there and expanded straight into C once C's
                // offsets are known, so these columns skip the slot-to-C
                // compaction
                uint4 *dst = reinterpret_cast<uint4 *>(out);
                for (uint32_t w4 = threadIdx.x; w4 < Wr / 4; w4 += BMP_NT) {
                    __stcs(dst + w4, bm4[w4]);  // read once, by the expansion
                    bm4[w4] = make_uint4(0, 0, 0, 0);
                }
                if (threadIdx.x == 0) {
                    o.defer[i] = 1;
                    const uint32_t d = atomicAdd(o.defer_count, 1u);
                    o.defer_list[d] = i;
                    s_dslot = d;
                }
                __syncthreads();
                if (o.defer_steps) {
                    // the step list the expansion would otherwise recount
                    uint32_t *rec = o.defer_steps + (uint64_t)s_dslot * BMP_STEP_REC;
                    for (uint32_t g = threadIdx.x; g <= nlist; g += BMP_NT) {
                        if (g < nlist) rec[1 + g] = S.s_list[g];
                        rec[1 + BMP_MAX_STEPS + g] = S.s_soff[g];
                    }
                    if (threadIdx.x == 0) rec[0] = nlist;
                }
                total += ctot;
                __syncthreads();
                continue;
            }
            bitmap_emit(bm, nlist, S.s_list, S.s_soff, &s_next, stage, out, (uint32_t)c0);
            total += ctot;
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            if (!NUMERIC) {
                o.row_nnz[i] = (uint32_t)total;
            } else if (o.row_cap) {
                if (overflowed) o.overflow[i] = 1;
                else o.row_nnz[i] = (uint32_t)total;
            }
            s_slot = nxt;
            s_row = nxt < cnt ? bl.list[beg + nxt] : 0;
        }
        __syncthreads();
    }
}

// Deferred bitmap rows (RowOut::defer) when there was no room for their
// step records: each row's bitmap, stored in its slot by bitmap_cta_kernel,
// is loaded back into shared memory, its steps are counted again and it is
// emitted at the row's final offset in C, once the offsets are known.  One
// row per CTA at a time, rows taken from `counter`.  (Emitting straight
// from the bitmap in global memory, one warp per step and no block
// barriers, was measured slower: the emission's bitmap walk waits on every
// load.)  bitmap_expand_steps_kernel below is the usual form.
template <int BMP_NT>
__global__ void __launch_bounds__(BMP_NT, 1024 / BMP_NT) bitmap_expand_kernel(
    const uint32_t *__restrict__ list, const uint32_t *__restrict__ count, const uint64_t *__restrict__ slot_off,
    const uint32_t *__restrict__ slots, const uint64_t *__restrict__ off, const uint32_t *__restrict__ row_ncols,
    uint64_t ncols, uint32_t W, uint32_t *__restrict__ ccols, uint32_t *counter) {
    extern __shared__ __align__(16) uint32_t smem[];
    const BitmapSmem S(smem, W);
    uint32_t *const bm = S.bm;
    uint4 *const bm4 = reinterpret_cast<uint4 *>(bm);
    __shared__ uint32_t scratch[33];
    __shared__ uint32_t s_slot, s_next;
    uint32_t *const stage = S.s_stage + warp_id() * BMP_STAGE;
    const uint32_t cnt = *count;
    for (;;) {
        const uint32_t item = next_item(counter, &s_slot);
        if (item >= cnt) break;
        const uint32_t i = list[item];
        const uint32_t Wr = bitmap_words(row_ncols ? (uint64_t)row_ncols[i] : ncols);
        const uint4 *src = reinterpret_cast<const uint4 *>(slots + slot_off[i]);
        for (uint32_t w4 = threadIdx.x; w4 < Wr / 4; w4 += BMP_NT) bm4[w4] = src[w4];
        __syncthreads();
        uint32_t nlist;
        bitmap_list_steps<BMP_NT>(bm4, Wr / BMP_STEP_WORDS, S.s_list, S.s_soff, &s_next, scratch, nlist);
        bitmap_emit(bm, nlist, S.s_list, S.s_soff, &s_next, stage, ccols + off[i], 0u);
        __syncthreads();
    }
}

// Deferred rows by warp: the numeric kernel stored each deferred row's
// bitmap in its slot and, in record d of `steps` (row list[d]), the row's
// non-empty steps and their output offsets.  Each warp claims rows from
// `counter`; it holds 32 of the row's step entries at a time in registers,
// copies each step's 512 bytes into its own shared buffer (the next step's
// copy in flight while the current one is emitted) and emits it at its place
// in C (bitmap_emit_step).  No block barrier and no whole-row reload, so the
// warps of an SM work on different rows at their own pace.
template <int NT>
__global__ void __launch_bounds__(NT) bitmap_expand_steps_kernel(const uint32_t *__restrict__ list,
                                                                 const uint32_t *__restrict__ count,
                                                                 const uint32_t *__restrict__ steps,
                                                                 const uint64_t *__restrict__ slot_off,
                                                                 const uint32_t *__restrict__ slots,
                                                                 const uint64_t *__restrict__ off,
                                                                 uint32_t *__restrict__ ccols, uint32_t *counter) {
    constexpr int NW = NT / 32;
    __shared__ __align__(16) uint32_t s_bm[NW][BMP_STEP_WORDS];
    __shared__ uint32_t s_stage[NW][BMP_STAGE];
    const uint32_t lane = lane_id(), w = warp_id();
    uint4 *const sb4 = reinterpret_cast<uint4 *>(s_bm[w]);
    const uint32_t cnt = *count;
    for (;;) {
        uint32_t d = 0;
        if (lane == 0) d = atomicAdd(counter, 1u);
        d = __shfl_sync(0xFFFFFFFFu, d, 0);
        if (d >= cnt) break;
        const uint32_t *rec = steps + (uint64_t)d * BMP_STEP_REC;
        const uint32_t nlist = rec[0];
        const uint32_t i = list[d];
        const uint4 *src = reinterpret_cast<const uint4 *>(slots + slot_off[i]) + lane;
        uint32_t *const out = ccols + off[i];
        for (uint32_t g0 = 0; g0 < nlist; g0 += 32) {
            const uint32_t gl = g0 + lane, m = min(32u, nlist - g0);
            const uint32_t my_st = gl < nlist ? rec[1 + gl] : 0u;
            const uint32_t my_pos = gl < nlist ? rec[1 + BMP_MAX_STEPS + gl] : 0u;
            const uint32_t my_end = gl < nlist ? rec[2 + BMP_MAX_STEPS + gl] : 0u;
            uint4 nxt = __ldcs(src + __shfl_sync(0xFFFFFFFFu, my_st, 0) * 32u);  // bitmaps are read once
            for (uint32_t k = 0; k < m; ++k) {
                const uint32_t st = __shfl_sync(0xFFFFFFFFu, my_st, k);
                const uint32_t pos = __shfl_sync(0xFFFFFFFFu, my_pos, k);
                const uint32_t T = __shfl_sync(0xFFFFFFFFu, my_end, k) - pos;
                sb4[lane] = nxt;
                if (k + 1 < m) nxt = __ldcs(src + __shfl_sync(0xFFFFFFFFu, my_st, k + 1) * 32u);
                __syncwarp();
                bitmap_emit_step<false>(s_bm[w], T, out + pos, st * (BMP_STEP_WORDS * 32u), s_stage[w]);
                __syncwarp();  // the buffers serve the warp's next step
            }
        }
    }
}

// Columns per CTA of the cluster bitmap kernel.
constexpr uint32_t CLB_CHUNK_SHIFT = 20;

// Rows with 2^20 < ncols <= CL * 2^20: the CL CTAs of a thread-block cluster
// hold one 2^20-column slice of the row's bitmap each, in their own shared
// memory, and work on ONE row together.  Every CTA stages the row's A
// entries and takes its share of the insertion units; each product sets its
// bit in the owning CTA's slice through distributed shared memory (atomicOr
// on the mapped address).  After a cluster barrier every CTA counts its
// slice, the counts are exchanged through distributed shared memory, and
// each CTA emits its slice at its offset (the columns of lower slices come
// first).  One pass over the products instead of one per 2^20-column chunk.
// All control flow that reaches a cluster barrier is cluster-uniform: the
// row index is fetched by rank 0 and broadcast, and every decision after it
// depends only on values all CTAs share.
template <bool NUMERIC, int CL>
__global__ void __launch_bounds__(1024, 1) bitmap_cluster_kernel(BinLists bl, int bin_lo, int bin_hi, AView a, BRows b,
                                                                 RowOut o, uint64_t ncols, uint32_t *counter) {
    constexpr int NT = 1024;
    constexpr uint32_t W = 1u << (CLB_CHUNK_SHIFT - 5);  // words per CTA
    extern __shared__ __align__(16) uint32_t smem[];
    const BitmapSmem S(smem, W);
    uint32_t *const bm = S.bm;
    __shared__ uint32_t scratch[33];
    __shared__ uint32_t s_item, s_next;
    __shared__ uint32_t s_counts[CL];
    __shared__ unsigned long long s_spill;
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const uint32_t rank = cluster.block_rank();
    uint32_t *slices[CL];
#pragma unroll
    for (int q = 0; q < CL; ++q) slices[q] = cluster.map_shared_rank(bm, q);
    uint32_t beg, cnt = 0, tmp;
    bin_range(bl, bin_lo, beg, tmp);
    for (int q = bin_lo; q <= bin_hi; ++q) cnt += bl.info[q];
    const uint32_t nheavy = bin_hi > bin_lo ? cnt - bl.info[bin_hi] : 0;
    for (uint32_t w = threadIdx.x; w < W; w += NT) bm[w] = 0;
    uint4 *bm4 = reinterpret_cast<uint4 *>(bm);
    uint32_t *const stage = S.s_stage + warp_id() * BMP_STAGE;
    const uint32_t maxcol = (uint32_t)min(ncols, (uint64_t)CL << CLB_CHUNK_SHIFT) - 1;
    for (;;) {
        // every slice is clear and every CTA done with the previous row
        cluster.sync();
        if (rank == 0 && threadIdx.x == 0) {
            const uint32_t it = atomicAdd(counter, 1u);
#pragma unroll
            for (int q = 0; q < CL; ++q) *cluster.map_shared_rank(&s_item, q) = it;
        }
        cluster.sync();
        const uint32_t item = s_item;
        if (item >= cnt) break;  // cluster-uniform
        const uint32_t i = bl.list[beg + item];
        const uint32_t shift = item < nheavy ? 9u : 8u;
        const bool short_b = o.row_products &&
                             (uint64_t)o.row_products[i] < (uint64_t)BMP_SHORT * (a.rpt[i + 1] - a.rpt[i]);
        auto set_bit_word = [&](uint32_t wd, uint32_t mk) {  // wd: word of the cluster's bitmap
            const uint32_t q = wd >> (CLB_CHUNK_SHIFT - 5);
            uint32_t *sl = slices[0];  // select, not an indexed (local-memory) load
#pragma unroll
            for (int k = 1; k < CL; ++k)
                if (q == (uint32_t)k) sl = slices[k];
            atomicOr(sl + (wd & ((1u << (CLB_CHUNK_SHIFT - 5)) - 1)), mk);
        };
        auto set_bit = [&](uint32_t c) { set_bit_word(c >> 5, 1u << (c & 31)); };
        if (short_b) {
            balanced_products<NT, BMP_ECH, 4>(a, b, i, S.s_upre, S.s_beg, scratch,
                                              [&](uint32_t c, bool valid, uint32_t) {
                if (valid) set_bit(min(c, maxcol));
            }, rank, CL);
        } else {
            bitmap_insert_row<NT, BMP_ECH>(a, b, i, shift, maxcol, set_bit, set_bit_word, S.s_beg, S.s_len,
                                           S.s_upre, scratch, rank, CL);
        }
        cluster.sync();  // every product's bit is set, in every slice
        uint32_t nlist = 0, ctot;
        if (NUMERIC)
            ctot = bitmap_list_steps<NT>(bm4, W / BMP_STEP_WORDS, S.s_list, S.s_soff, &s_next, scratch, nlist);
        else
            ctot = bitmap_count_clear<NT>(bm4, W, scratch);
        if (threadIdx.x == 0) {
#pragma unroll
            for (int q = 0; q < CL; ++q) cluster.map_shared_rank(s_counts, q)[rank] = ctot;
        }
        cluster.sync();
        uint64_t before = 0, total = 0;
#pragma unroll
        for (int q = 0; q < CL; ++q) {
            before += (uint32_t)q < rank ? s_counts[q] : 0u;
            total += s_counts[q];
        }
        if (!NUMERIC) {
            if (rank == 0 && threadIdx.x == 0) o.row_nnz[i] = (uint32_t)total;
            continue;
        }
        uint32_t *out = o.cols + o.row_off[i];
        if (o.row_cap && total > o.row_cap[i]) {
            // over the slot: rank 0 reserves the whole row in the spill
            // arena and broadcasts the offset (~0: no room -> exact rerun)
            if (rank == 0 && threadIdx.x == 0) {
                unsigned long long at = ~0ull;
                if (o.arena) {
                    at = atomicAdd(o.arena_cursor, (unsigned long long)((total + 3u) & ~3ull));
                    if (at + total > o.arena_cap) at = ~0ull;
                }
#pragma unroll
                for (int q = 0; q < CL; ++q) *cluster.map_shared_rank(&s_spill, q) = at;
                if (o.spill) o.spill[i] = at;
                if (at == ~0ull) o.overflow[i] = 1;
            }
            cluster.sync();
            if (s_spill == ~0ull) {
                for (uint32_t w4 = threadIdx.x; w4 < W / 4; w4 += NT) bm4[w4] = make_uint4(0, 0, 0, 0);
                __syncthreads();
                continue;
            }
            out = o.arena + s_spill;
        }
        bitmap_emit(bm, nlist, S.s_list, S.s_soff, &s_next, stage, out + before, rank << CLB_CHUNK_SHIFT);
        if (o.row_cap && rank == 0 && threadIdx.x == 0) o.row_nnz[i] = (uint32_t)total;
        __syncthreads();
    }
}

}  // namespace clb
