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
#include <algorithm>
#include <string>
#include <vector>

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
    // the tile's A and B keys for the merge; then (MODE 1) its outputs,
    // compacted at position q + q / 8 (threads stage 8 outputs each, so the
    // skew keeps neighbouring lanes off the same banks)
    __shared__ uint64_t s[MP_TILE + MP_TILE / 8];
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
#pragma unroll 4
    for (uint32_t k = threadIdx.x; k < nta; k += MP_NT)
        s[k] = CSR ? csr_key(As, a0 + k, rlo, rhi) : coo_key(Ac, a0 + k);
#pragma unroll 4
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
    // (the block scan's barriers also end every thread's merge reads of s)
    uint32_t tot;
    uint32_t q = block_exclusive_scan<uint32_t, MP_NT>(cnt, scratch, &tot);
#pragma unroll
    for (int k = 0; k < MP_ITEMS; ++k) {
        if (flags & (1u << k)) {
            s[q + (q >> 3)] = keys[k];
            ++q;
        }
    }
    __syncthreads();
    // coalesced copy-out of the tile's outputs
    const uint64_t base = tile_off[t];
    for (uint32_t i = threadIdx.x; i < tot; i += MP_NT) {
        const uint64_t key = s[i + (i >> 3)];
        if (!CSR) out_rows[base + i] = (uint32_t)(key >> 32);
        out_cols[base + i] = (uint32_t)key;
    }
}

// ------------------------------------------------- CSR insertion path --
// When one operand is much sparser than the other (the closure step C + A,
// say), C's row r is the longer row X of the two with the shorter row Y
// inserted: every entry of Y finds its place in X by binary search (a warp
// takes 32 entries at a time, each search starting where the previous
// chunk ended), and X is copied in the segments between the insertions.
// X is read once, by coalesced copies; no keys are staged.

// Sum over rows of min(lenA, lenB): the entries that need a search.
__global__ void csr_min_sum_kernel(const uint64_t *__restrict__ arpt, const uint64_t *__restrict__ brpt, uint64_t nrows,
                                   unsigned long long *__restrict__ out) {
    unsigned long long mine = 0;
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += (uint64_t)gridDim.x * blockDim.x)
        mine += min(arpt[r + 1] - arpt[r], brpt[r + 1] - brpt[r]);
    mine = warp_sum(mine);
    if (lane_id() == 0 && mine) atomicAdd(out, mine);
}

// First position in x[lo, n) whose value is >= y.
__device__ __forceinline__ uint64_t lower_bound_from(const uint32_t *x, uint64_t lo, uint64_t n, uint32_t y) {
    uint64_t hi = n;
    while (lo < hi) {
        const uint64_t m = lo + (hi - lo) / 2;
        if (__ldg(x + m) < y) lo = m + 1; else hi = m;
    }
    return lo;
}

struct RowPair {
    const uint32_t *x, *y;  // longer and shorter row
    uint64_t nx, ny;
};

__device__ __forceinline__ RowPair row_pair(const CsrSide &A, const CsrSide &B, uint64_t r) {
    const uint64_t a0 = A.rpt[r], a1 = A.rpt[r + 1], b0 = B.rpt[r], b1 = B.rpt[r + 1];
    const uint64_t la = a1 - a0, lb = b1 - b0;
    return la >= lb ? RowPair{A.cols + a0, B.cols + b0, la, lb} : RowPair{B.cols + b0, A.cols + a0, lb, la};
}

// Warp copy of x[from, to) to dst[from .. to) (dst already shifted).
// Eight loads in flight per lane before the stores: a warp may copy a row
// of a million entries, which one load at a time would leave latency-bound.
__device__ __forceinline__ void warp_copy_seg(const uint32_t *__restrict__ x, uint64_t from, uint64_t to,
                                              uint32_t *__restrict__ dst) {
    uint64_t j = from + lane_id();
    for (; j + 7 * 32 < to; j += 8 * 32) {
        uint32_t v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = __ldg(x + j + u * 32);
#pragma unroll
        for (int u = 0; u < 8; ++u) dst[j + u * 32] = v[u];
    }
    for (; j < to; j += 32) dst[j] = __ldg(x + j);
}

// dst[j + base + (insertions at or before j)] = x[j] for j in [from, to):
// ins[0, n) are the sorted insertion positions (an insertion at p goes
// before x[p]).  Each lane keeps its own cursor into ins (its j only grow),
// so the copy keeps eight loads in flight per lane across the insertions and
// every store instruction writes 32 consecutive words.  (16-byte loads with
// word stores measured no faster on scale-20 C + A.)
__device__ __forceinline__ void warp_copy_shifted(const uint32_t *__restrict__ x, uint64_t from, uint64_t to,
                                                  uint32_t *__restrict__ dst, const uint32_t *ins, uint32_t n,
                                                  uint64_t base) {
    uint32_t q = 0;
    uint64_t nxt = n ? ins[0] : ~0ull;
    uint64_t j = from + lane_id();
    for (; j + 7 * 32 < to; j += 8 * 32) {
        uint32_t v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = __ldg(x + j + u * 32);
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const uint64_t jj = j + u * 32;
            while (nxt <= jj) {
                ++q;
                nxt = q < n ? ins[q] : ~0ull;
            }
            dst[jj + base + q] = v[u];
        }
    }
    for (; j < to; j += 32) {
        const uint32_t v = __ldg(x + j);
        while (nxt <= j) {
            ++q;
            nxt = q < n ? ins[q] : ~0ull;
        }
        dst[j + base + q] = v;
    }
}

// MODE 0: out_cnt[r] = |X| + |Y| - |X and Y|.  MODE 1: row r of the sum at
// cols + rpt[r].  One warp per row.
// Rows whose shorter side has more than INS_LONG entries (the hub rows of a
// power-law matrix) are listed by the count pass and left to
// csr_insert_long_kernel, which spreads their chunks over a CTA.
constexpr uint64_t INS_LONG = 256;
constexpr uint32_t INS_MAX_CHUNKS = 4096;  // the CTA kernel's chunk table (longer rows stay here)

__device__ __forceinline__ bool ins_long_row(uint64_t ny) {
    return ny > INS_LONG && ny <= (uint64_t)INS_MAX_CHUNKS * 32;
}
// Rows with a short Y but an X too long for one warp to copy in good time
// (power-law products: a short A row can reach a C row of ~10^6 entries) are
// filled by the CTA kernel too, X split into pieces over its warps.
constexpr uint64_t INS_WIDE = 32768;
constexpr uint64_t INS_PIECE = 8192;
__device__ __forceinline__ bool ins_wide_row(uint64_t nx, uint64_t ny) { return ny <= INS_LONG && nx > INS_WIDE; }

template <int MODE>
__global__ void __launch_bounds__(256) csr_insert_kernel(CsrSide A, CsrSide B, uint64_t nrows,
                                                         uint64_t *__restrict__ out_cnt,
                                                         const uint64_t *__restrict__ rpt,
                                                         uint32_t *__restrict__ cols,
                                                         uint32_t *__restrict__ long_rows,
                                                         uint32_t *__restrict__ n_long) {
    __shared__ uint32_t s_ins[8][INS_LONG];  // per warp: the row's insertion positions
    const uint32_t lane = lane_id();
    const uint32_t ltmask = (1u << lane) - 1u;
    uint32_t *const ins = s_ins[warp_id()];
    const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x / 32);
    for (uint64_t r = (uint64_t)blockIdx.x * (blockDim.x / 32) + warp_id(); r < nrows; r += nw) {
        const RowPair p = row_pair(A, B, r);
        if (ins_long_row(p.ny)) {
            if (MODE == 0 && lane == 0) long_rows[atomicAdd(n_long, 1u)] = (uint32_t)r;
            continue;
        }
        if (ins_wide_row(p.nx, p.ny)) {
            if (MODE == 1) continue;  // counted below, filled by the CTA kernel
            if (lane == 0) long_rows[atomicAdd(n_long, 1u)] = (uint32_t)r;
        }
        uint32_t *const dst = MODE ? cols + rpt[r] : nullptr;
        if (p.ny == 0) {
            if (MODE == 0) {
                if (lane == 0) out_cnt[r] = p.nx;
            } else {
                warp_copy_seg(p.x, 0, p.nx, dst);
            }
            continue;
        }
        // Y of at most INS_LONG entries: insertion positions listed, then one
        // shifted copy of X; longer Y (past the CTA kernel's table): X copied
        // segment by segment between the insertions
        const bool listed = p.ny <= INS_LONG;
        uint64_t lo = 0, dups = 0, copied = 0;
        uint32_t nins = 0;  // non-duplicate entries of Y so far
        for (uint64_t c0 = 0; c0 < p.ny; c0 += 32) {
            const uint64_t k = c0 + lane;
            const bool valid = k < p.ny;
            const uint32_t y = valid ? __ldg(p.y + k) : 0xFFFFFFFFu;
            const uint64_t pos = valid ? lower_bound_from(p.x, lo, p.nx, y) : p.nx;
            const bool dup = valid && pos < p.nx && __ldg(p.x + pos) == y;
            const uint32_t mdup = __ballot_sync(0xFFFFFFFFu, dup);
            const uint32_t mins = __ballot_sync(0xFFFFFFFFu, valid && !dup);
            dups += __popc(mdup);
            if (MODE == 1) {
                const uint32_t at = nins + __popc(mins & ltmask);
                if (valid && !dup) {
                    dst[pos + at] = y;
                    if (listed) ins[at] = (uint32_t)pos;
                }
                if (!listed) {
                    uint32_t m = mins, before = 0;
                    while (m) {
                        const uint32_t l = __ffs(m) - 1;
                        m &= m - 1;
                        const uint64_t pl = __shfl_sync(0xFFFFFFFFu, pos, l);
                        warp_copy_seg(p.x, copied, pl, dst + nins + before);
                        copied = pl;
                        ++before;
                    }
                }
            }
            nins += __popc(mins);
            // the next chunk's entries are larger: search from the last position
            const uint32_t last = p.ny - c0 >= 32 ? 31u : (uint32_t)(p.ny - 1 - c0);
            lo = __shfl_sync(0xFFFFFFFFu, pos, last);
        }
        if (MODE == 0) {
            if (lane == 0) out_cnt[r] = p.nx + p.ny - dups;
        } else if (listed) {
            __syncwarp();
            warp_copy_shifted(p.x, 0, p.nx, dst, ins, nins, 0);
            __syncwarp();
        } else {
            warp_copy_seg(p.x, copied, p.nx, dst + nins);
        }
    }
}

// The listed long rows, one CTA each.  Chunk c (Y entries 32c..32c+31)
// owns X[S_c, S_c+1) with S_0 = 0, S_c = position of its first entry (c > 0)
// and S_last = |X|; its entries' insertions shift that range by the
// non-duplicate entries of the chunks before it (a block scan over the
// chunks).  MODE 0: out_cnt[r]; MODE 1: the row at cols + rpt[r].
template <int MODE>
__global__ void __launch_bounds__(256) csr_insert_long_kernel(CsrSide A, CsrSide B, const uint32_t *__restrict__ long_rows,
                                                              const uint32_t *__restrict__ n_long,
                                                              uint64_t *__restrict__ out_cnt,
                                                              const uint64_t *__restrict__ rpt,
                                                              uint32_t *__restrict__ cols) {
    constexpr int NWARP = 8;
    __shared__ uint32_t s_start[INS_MAX_CHUNKS + 1];  // S_c
    __shared__ uint32_t s_nd[INS_MAX_CHUNKS];         // non-duplicate entries of chunk c, then their prefix
    __shared__ uint32_t scratch[33];
    __shared__ uint32_t s_ins[NWARP][32];  // per warp: its chunk's insertion positions
    __shared__ uint32_t s_all[INS_LONG];   // wide rows: all the row's insertion positions
    __shared__ uint32_t s_wpos[INS_LONG];  // wide rows: each Y entry's position (~0 = duplicate)
    const uint32_t lane = lane_id(), w = warp_id();
    const uint32_t ltmask = (1u << lane) - 1u;
    uint32_t *const ins = s_ins[w];
    const uint32_t nl = *n_long;
    for (uint32_t item = blockIdx.x; item < nl; item += gridDim.x) {
        const uint64_t r = long_rows[item];
        const RowPair p = row_pair(A, B, r);
        const bool wide = ins_wide_row(p.nx, p.ny);
        if (MODE == 0 && wide) continue;  // counted by the warp kernel (block-uniform)
        const uint32_t nch = (uint32_t)((p.ny + 31) / 32);
        // pass over the chunks: positions of the first entries and counts
        for (uint32_t c = w; c < nch; c += NWARP) {
            const uint64_t k = (uint64_t)c * 32 + lane;
            const bool valid = k < p.ny;
            const uint32_t y = valid ? __ldg(p.y + k) : 0xFFFFFFFFu;
            const uint64_t pos = valid ? lower_bound_from(p.x, 0, p.nx, y) : p.nx;
            const bool dup = valid && pos < p.nx && __ldg(p.x + pos) == y;
            const uint32_t mins = __ballot_sync(0xFFFFFFFFu, valid && !dup);
            if (lane == 0) {
                s_start[c] = c == 0 ? 0u : (uint32_t)pos;
                s_nd[c] = __popc(mins);
            }
            if (MODE == 1 && wide && valid) s_wpos[k] = dup ? 0xFFFFFFFFu : (uint32_t)pos;  // kept: no second search
        }
        if (threadIdx.x == 0) s_start[nch] = (uint32_t)p.nx;
        __syncthreads();
        // prefix of the non-duplicate counts over the chunks
        uint32_t run = 0;
        const uint32_t per = (nch + blockDim.x - 1) / blockDim.x;
        const uint32_t c0 = threadIdx.x * per, c1 = min(c0 + per, nch);
        for (uint32_t c = c0; c < c1; ++c) run += s_nd[c];
        uint32_t total;
        uint32_t base = block_exclusive_scan<uint32_t, 256>(run, scratch, &total);
        if (MODE == 0) {
            if (threadIdx.x == 0) out_cnt[r] = p.nx + total;
            __syncthreads();
        } else {
        for (uint32_t c = c0; c < c1; ++c) {
            const uint32_t v = s_nd[c];
            s_nd[c] = base;
            base += v;
        }
        __syncthreads();
        uint32_t *const dst = cols + rpt[r];
        for (uint32_t c = w; c < nch; c += NWARP) {
            const uint64_t k = (uint64_t)c * 32 + lane;
            const bool valid = k < p.ny;
            const uint32_t y = valid ? __ldg(p.y + k) : 0xFFFFFFFFu;
            const uint64_t lo = s_start[c];
            uint64_t pos;
            bool dup;
            if (wide) {
                const uint32_t wp = valid ? s_wpos[k] : 0xFFFFFFFFu;
                dup = valid && wp == 0xFFFFFFFFu;
                pos = valid && !dup ? (uint64_t)wp : p.nx;
            } else {
                pos = valid ? lower_bound_from(p.x, lo, p.nx, y) : p.nx;
                dup = valid && pos < p.nx && __ldg(p.x + pos) == y;
            }
            const uint32_t mins = __ballot_sync(0xFFFFFFFFu, valid && !dup);
            const uint64_t shift = s_nd[c];
            const uint32_t at = __popc(mins & ltmask);
            if (valid && !dup) {
                dst[pos + shift + at] = y;
                if (wide) s_all[shift + at] = (uint32_t)pos;
                else ins[at] = (uint32_t)pos;
            }
            if (!wide) {
                __syncwarp();
                warp_copy_shifted(p.x, lo, s_start[c + 1], dst, ins, __popc(mins), shift);
                __syncwarp();
            }
        }
        if (wide) {
            // X in pieces over the warps, each starting its cursor at the
            // first insertion at or after the piece
            __syncthreads();
            const uint32_t nins = total;
            for (uint64_t j0 = (uint64_t)w * INS_PIECE; j0 < p.nx; j0 += NWARP * INS_PIECE) {
                uint32_t q0 = 0, hi = nins;  // first insertion with position >= j0
                while (q0 < hi) {
                    const uint32_t m = (q0 + hi) / 2;
                    if (s_all[m] < j0) q0 = m + 1; else hi = m;
                }
                warp_copy_shifted(p.x, j0, min(j0 + INS_PIECE, p.nx), dst, s_all + q0, nins - q0, q0);
            }
        }
        __syncthreads();
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


// C = A v B (CSR, same shape checked by the caller, ctl's device current).
int csr_add_impl(clb_controls *ctl, const clb_csr &a, const clb_csr &b, clb_csr *out) {
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
    {
        // one operand much sparser (at most 1/16 of the entries need a
        // search): insertion path
        Temp<uint64_t> ms;
        CLB_RETURN_IF(ms.alloc(ctl, 1));
        CLB_TRY_CUDA(cudaMemsetAsync(ms.ptr, 0, 8, ctl->stream), CLB_RUN_KERNEL_FAILURE);
        csr_min_sum_kernel<<<grid_for(ctl, a.nrows), 256, 0, ctl->stream>>>(a.rpt, b.rpt, a.nrows,
                                                                             (unsigned long long *)ms.ptr);
        CLB_CHECK_LAUNCH();
        uint64_t searched = 0;
        CLB_RETURN_IF(read_scalars(ctl, ms.ptr, &searched, 1));
        if (searched * 16 <= a.nnz + b.nnz) {
            Temp<uint64_t> rpt, tot;
            CLB_RETURN_IF(rpt.alloc(ctl, a.nrows + 1));
            CLB_RETURN_IF(tot.alloc(ctl, 1));
            // grid-stride kernels: no more blocks than the SMs hold at once
            static const int w0_per_sm = blocks_per_sm(csr_insert_kernel<0>, 256);
            static const int w1_per_sm = blocks_per_sm(csr_insert_kernel<1>, 256);
            static const int l0_per_sm = blocks_per_sm(csr_insert_long_kernel<0>, 256);
            static const int l1_per_sm = blocks_per_sm(csr_insert_long_kernel<1>, 256);
            const uint64_t warps_rows = (a.nrows + 7) / 8;
            const unsigned gw0 = persistent_grid(ctl, w0_per_sm, warps_rows);
            const unsigned gw1 = persistent_grid(ctl, w1_per_sm, warps_rows);
            Temp<uint32_t> lrows, nlong;
            CLB_RETURN_IF(lrows.alloc(ctl, a.nrows));
            CLB_RETURN_IF(nlong.alloc(ctl, 1));
            CLB_TRY_CUDA(cudaMemsetAsync(nlong.ptr, 0, 4, ctl->stream), CLB_RUN_KERNEL_FAILURE);
            csr_insert_kernel<0><<<gw0, 256, 0, ctl->stream>>>(A, B, a.nrows, rpt.ptr, nullptr, nullptr, lrows.ptr,
                                                               nlong.ptr);
            csr_insert_long_kernel<0><<<ctl->sm_count * l0_per_sm, 256, 0, ctl->stream>>>(
                A, B, lrows.ptr, nlong.ptr, rpt.ptr, nullptr, nullptr);
            CLB_CHECK_LAUNCH();
            CLB_RETURN_IF(scan_u64_inplace(ctl, rpt.ptr, a.nrows, tot.ptr));
            uint64_t nnz = 0;
            CLB_RETURN_IF(read_scalars(ctl, tot.ptr, &nnz, 1));
            CLB_TRY_CUDA(cudaMemcpyAsync(rpt.ptr + a.nrows, tot.ptr, 8, cudaMemcpyDeviceToDevice, ctl->stream),
                         CLB_COPY_BUFFER_ERROR);
            Temp<uint32_t> cols;
            CLB_RETURN_IF(cols.alloc(ctl, nnz));
            csr_insert_kernel<1><<<gw1, 256, 0, ctl->stream>>>(A, B, a.nrows, nullptr, rpt.ptr, cols.ptr, nullptr,
                                                               nullptr);
            csr_insert_long_kernel<1><<<ctl->sm_count * l1_per_sm, 256, 0, ctl->stream>>>(
                A, B, lrows.ptr, nlong.ptr, nullptr, rpt.ptr, cols.ptr);
            CLB_CHECK_LAUNCH();
            CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
            c.nnz = nnz;
            c.rpt = rpt.release_ownership();
            c.cols = cols.release_ownership();
            *out = c;
            return CLB_SUCCESS;
        }
    }
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

// ------------------------------------------------------ batched addition --
// Many independent additions C_k = A_k v B_k in one set of launches: the
// pairs' rows are stacked (row pointers shifted by the entries before the
// pair, columns copied unshifted: a row of the stack only ever meets the
// other operand's row of the same pair), one addition runs over the stack,
// and its rows are cut back into the pairs' results.
struct AddDesc {
    const uint64_t *arpt, *brpt;
    const uint32_t *acols, *bcols;
    uint64_t nrows, anz, bnz;
    uint64_t row_off, aoff, boff;  // position in the stack
};

constexpr int ST_NT = 256;

__global__ void __launch_bounds__(ST_NT) add_stack_kernel(const AddDesc *__restrict__ d, uint64_t *__restrict__ arpt,
                                                          uint32_t *__restrict__ acols, uint64_t *__restrict__ brpt,
                                                          uint32_t *__restrict__ bcols, uint64_t rows, uint64_t anz,
                                                          uint64_t bnz) {
    const AddDesc p = d[blockIdx.y];
    const uint64_t stride = (uint64_t)gridDim.x * ST_NT;
    const uint64_t t0 = (uint64_t)blockIdx.x * ST_NT + threadIdx.x;
    const uint64_t a0 = p.arpt[0], b0 = p.brpt[0];
    for (uint64_t r = t0; r < p.nrows; r += stride) {
        arpt[p.row_off + r] = p.arpt[r] - a0 + p.aoff;
        brpt[p.row_off + r] = p.brpt[r] - b0 + p.boff;
    }
    for (uint64_t j = t0; j < p.anz; j += stride) acols[p.aoff + j] = p.acols[a0 + j];
    for (uint64_t j = t0; j < p.bnz; j += stride) bcols[p.boff + j] = p.bcols[b0 + j];
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
        arpt[rows] = anz;
        brpt[rows] = bnz;
    }
}

struct AddOut {
    uint64_t *rpt;
    uint32_t *cols;
    uint64_t nrows, row_off, c0, nnz;
};

// bounds[k] = C'.rpt[row_off of pair k] (k = count: the total).
__global__ void add_bounds_kernel(const uint64_t *__restrict__ crpt, const uint64_t *__restrict__ row_off,
                                  uint32_t count, uint64_t *__restrict__ bounds) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k <= count; k += gridDim.x * blockDim.x)
        bounds[k] = crpt[row_off[k]];
}

__global__ void __launch_bounds__(ST_NT) add_split_kernel(const AddOut *__restrict__ d, const uint64_t *__restrict__ crpt,
                                                          const uint32_t *__restrict__ ccols) {
    const AddOut o = d[blockIdx.y];
    if (!o.nnz) return;  // an empty sum has no arrays (its descriptor holds null pointers)
    const uint64_t stride = (uint64_t)gridDim.x * ST_NT;
    const uint64_t t0 = (uint64_t)blockIdx.x * ST_NT + threadIdx.x;
    for (uint64_t r = t0; r <= o.nrows; r += stride) o.rpt[r] = crpt[o.row_off + r] - o.c0;
    for (uint64_t j = t0; j < o.nnz; j += stride) o.cols[j] = ccols[o.c0 + j];
}

unsigned stack_blocks(uint64_t largest) {
    const uint64_t gx = (largest + 4 * ST_NT - 1) / (4 * ST_NT);
    return (unsigned)std::min<uint64_t>(std::max<uint64_t>(gx, 1), 65535);
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
    CLB_RETURN_IF(shape_check(a_->nrows, a_->ncols, b_->nrows, b_->ncols));
    DeviceGuard g(ctl);
    return csr_add_impl(ctl, *a_, *b_, out);
}

int clb_csr_add_batched(clb_controls *ctl, uint32_t count, const clb_csr *a, const clb_csr *b, clb_csr *c) {
    if (!ctl || (count && (!a || !b || !c))) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    if (count > 65535) return fail(CLB_NOT_SUPPORTED, "at most 65535 pairs per batch");
    std::vector<AddDesc> hd(count);
    std::vector<uint64_t> row_off(count + 1);
    uint64_t rows = 0, anz = 0, bnz = 0, ncols = 0, largest = 1;
    for (uint32_t k = 0; k < count; ++k) {
        const int rc = shape_check(a[k].nrows, a[k].ncols, b[k].nrows, b[k].ncols);
        if (rc != CLB_SUCCESS) return fail(rc, "pair " + std::to_string(k) + ": " + clb_last_error());
        if ((a[k].nnz && !a[k].rpt) || (b[k].nnz && !b[k].rpt)) return fail(CLB_INVALID_ARGUMENT, "NULL rpt");
        hd[k] = AddDesc{a[k].rpt, b[k].rpt, a[k].cols, b[k].cols, 0, a[k].nnz, b[k].nnz, rows, anz, bnz};
        row_off[k] = rows;
        rows += a[k].nrows;
        anz += a[k].nnz;
        bnz += b[k].nnz;
        ncols = std::max(ncols, a[k].ncols);
        largest = std::max(largest, std::max(a[k].nrows + 1, std::max(a[k].nnz, b[k].nnz)));
    }
    row_off[count] = rows;
    for (uint32_t k = 0; k < count; ++k) {
        clb_csr e{};
        e.nrows = a[k].nrows;
        e.ncols = a[k].ncols;
        c[k] = e;
    }
    if (anz + bnz == 0) return CLB_SUCCESS;
    if (rows >= (1ull << 32)) return fail(CLB_NOT_SUPPORTED, "the stacked batch has 2^32 or more rows");
    DeviceGuard g(ctl);
    // an operand without entries may come without row pointers: it stacks as
    // empty rows (its descriptor points at a zero row pointer array)
    Temp<uint64_t> zeros;
    uint64_t max_rows = 0;
    for (uint32_t k = 0; k < count; ++k) max_rows = std::max(max_rows, a[k].nrows);
    CLB_RETURN_IF(zeros.alloc(ctl, max_rows + 1));
    CLB_TRY_CUDA(cudaMemsetAsync(zeros.ptr, 0, (max_rows + 1) * 8, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    for (uint32_t k = 0; k < count; ++k) {
        hd[k].nrows = a[k].nrows;
        if (!a[k].nnz || !a[k].rpt) hd[k].arpt = zeros.ptr;
        if (!b[k].nnz || !b[k].rpt) hd[k].brpt = zeros.ptr;
    }
    Temp<AddDesc> dd;
    Temp<uint64_t> arpt, brpt, roff, bounds;
    Temp<uint32_t> acols, bcols;
    CLB_RETURN_IF(dd.alloc(ctl, count));
    CLB_RETURN_IF(arpt.alloc(ctl, rows + 1));
    CLB_RETURN_IF(brpt.alloc(ctl, rows + 1));
    CLB_RETURN_IF(acols.alloc(ctl, std::max<uint64_t>(anz, 1)));
    CLB_RETURN_IF(bcols.alloc(ctl, std::max<uint64_t>(bnz, 1)));
    CLB_RETURN_IF(roff.alloc(ctl, count + 1));
    CLB_RETURN_IF(bounds.alloc(ctl, count + 1));
    CLB_TRY_CUDA(cudaMemcpyAsync(dd.ptr, hd.data(), count * sizeof(AddDesc), cudaMemcpyHostToDevice, ctl->stream),
                 CLB_WRITE_BUFFER_ERROR);
    CLB_TRY_CUDA(cudaMemcpyAsync(roff.ptr, row_off.data(), (count + 1) * 8, cudaMemcpyHostToDevice, ctl->stream),
                 CLB_WRITE_BUFFER_ERROR);
    {
        ProfScope ps(ctl, "add_stack");
        add_stack_kernel<<<dim3(stack_blocks(largest), count), ST_NT, 0, ctl->stream>>>(
            dd.ptr, arpt.ptr, acols.ptr, brpt.ptr, bcols.ptr, rows, anz, bnz);
        CLB_CHECK_LAUNCH();
    }
    const clb_csr As{rows, ncols, anz, arpt.ptr, anz ? acols.ptr : nullptr};
    const clb_csr Bs{rows, ncols, bnz, brpt.ptr, bnz ? bcols.ptr : nullptr};
    clb_csr Cs{};
    CLB_RETURN_IF(csr_add_impl(ctl, As, Bs, &Cs));
    // cut the stacked sum into the pairs
    std::vector<uint64_t> hb(count + 1);
    int rc = CLB_SUCCESS;
    {
        add_bounds_kernel<<<(count + 256) / 256, 256, 0, ctl->stream>>>(Cs.rpt, roff.ptr, count, bounds.ptr);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(hb.data(), bounds.ptr, (count + 1) * 8, cudaMemcpyDeviceToHost,
                                                  ctl->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctl->stream);
        if (e != cudaSuccess) rc = fail(CLB_RUN_KERNEL_FAILURE, cudaGetErrorString(e));
    }
    std::vector<AddOut> ho(count);
    std::vector<clb_csr> outs(count);
    uint64_t omax = 1;
    for (uint32_t k = 0; k < count && rc == CLB_SUCCESS; ++k) {
        clb_csr o{};
        o.nrows = a[k].nrows;
        o.ncols = a[k].ncols;
        const uint64_t nnz = hb[k + 1] - hb[k];
        AddOut d{nullptr, nullptr, 0, row_off[k], hb[k], 0};
        if (nnz) {
            Temp<uint64_t> p;
            Temp<uint32_t> cc;
            rc = p.alloc(ctl, o.nrows + 1);
            if (rc == CLB_SUCCESS) rc = cc.alloc(ctl, nnz);
            if (rc != CLB_SUCCESS) break;
            d.rpt = p.ptr;
            d.cols = cc.ptr;
            d.nrows = o.nrows;
            d.nnz = nnz;
            o.nnz = nnz;
            o.rpt = p.release_ownership();
            o.cols = cc.release_ownership();
            omax = std::max(omax, std::max(o.nrows + 1, nnz));
        }
        ho[k] = d;
        outs[k] = o;
    }
    Temp<AddOut> dout;
    if (rc == CLB_SUCCESS) rc = dout.alloc(ctl, count);
    if (rc == CLB_SUCCESS) {
        cudaError_t e = cudaMemcpyAsync(dout.ptr, ho.data(), count * sizeof(AddOut), cudaMemcpyHostToDevice,
                                        ctl->stream);
        if (e == cudaSuccess) {
            ProfScope ps(ctl, "add_split");
            add_split_kernel<<<dim3(stack_blocks(omax), count), ST_NT, 0, ctl->stream>>>(dout.ptr, Cs.rpt, Cs.cols);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctl->stream);
        if (e != cudaSuccess) rc = fail(CLB_RUN_KERNEL_FAILURE, cudaGetErrorString(e));
    }
    clb_csr_release(ctl, &Cs);
    if (rc != CLB_SUCCESS) {
        for (auto &o : outs) clb_csr_release(ctl, &o);
        return rc;
    }
    for (uint32_t k = 0; k < count; ++k) c[k] = outs[k];
    return CLB_SUCCESS;
}

}  // extern "C"
