// common.cuh -- internal runtime and device primitives of libclbool_b200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "clbool_b200.h"

namespace clb {

constexpr uint32_t EMPTY = 0xFFFFFFFFu;  // empty slot / padding key
constexpr int WARP = 32;

// --------------------------------------------------------------- status ---
// Device status word bits (set by kernels; read by the host after a call).
enum DeviceStatus : uint32_t {
    DEV_OK = 0,
    DEV_PROBE_LIMIT = 1u << 0,   // a hash probe sequence exceeded its bound
    DEV_WAIT_LIMIT = 1u << 1,    // a bounded spin gave up
    DEV_BOUNDS = 1u << 2,        // an index check failed
    DEV_CAPACITY = 1u << 3,      // an accumulator overflowed with no fallback
};

void set_error(const std::string &msg);
int fail(int status, const std::string &msg);

#define CLB_TRY_CUDA(expr, status)                                                          \
    do {                                                                                    \
        cudaError_t e_ = (expr);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return ::clb::fail((status), std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define CLB_CHECK_LAUNCH() CLB_TRY_CUDA(cudaGetLastError(), CLB_RUN_KERNEL_FAILURE)

#define CLB_RETURN_IF(expr)         \
    do {                            \
        int s_ = (expr);            \
        if (s_ != CLB_SUCCESS) return s_; \
    } while (0)

}  // namespace clb

struct clb_controls {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int sm_count = 148;
    size_t smem_optin = 0;
    uint64_t *h_scalars = nullptr;  // pinned scalar staging (64 entries)
    uint64_t *d_h_scalars = nullptr;  // the same staging as the device addresses it
    uint32_t *d_status = nullptr;   // device status word
    clb_alloc_fn alloc = nullptr;
    clb_free_fn release = nullptr;
    void *alloc_ctx = nullptr;
    uint32_t launches = 0;          // kernels launched by the current call
    // Opt-in kernel timing: one event pair per launch on `stream`.
    struct ProfRec {
        const char *name;
        cudaEvent_t start, stop;
    };
    bool profiling = false;
    std::vector<ProfRec> prof;
    std::vector<cudaEvent_t> event_pool;
};

namespace clb {

// Makes ctl's device current for the scope of a call.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(const clb_controls *ctl) {
        cudaGetDevice(&prev);
        if (prev != ctl->device) cudaSetDevice(ctl->device);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

void *dev_alloc(clb_controls *ctl, size_t bytes);
void dev_free(clb_controls *ctl, void *p);

// Temporary device buffer released (stream-ordered) at scope exit.
template <class T>
struct Temp {
    clb_controls *ctl = nullptr;
    T *ptr = nullptr;
    size_t n = 0;
    Temp() = default;
    Temp(const Temp &) = delete;
    Temp &operator=(const Temp &) = delete;
    ~Temp() { reset(); }
    int alloc(clb_controls *c, size_t count) {
        reset();
        ctl = c;
        n = count;
        if (count == 0) return CLB_SUCCESS;
        ptr = static_cast<T *>(dev_alloc(c, count * sizeof(T)));
        if (!ptr) return fail(CLB_CREATE_BUFFER_ERROR, "device allocation of " + std::to_string(count * sizeof(T)) + " bytes failed");
        return CLB_SUCCESS;
    }
    // Like alloc, but a failure is not an error of the call (the caller has
    // another way); returns whether the buffer exists.
    bool try_alloc(clb_controls *c, size_t count) {
        reset();
        ctl = c;
        n = count;
        if (count == 0) return true;
        ptr = static_cast<T *>(dev_alloc(c, count * sizeof(T)));
        return ptr != nullptr;
    }
    T *release_ownership() {
        T *p = ptr;
        ptr = nullptr;
        return p;
    }
    void reset() {
        if (ptr && ctl) dev_free(ctl, ptr);
        ptr = nullptr;
    }
};

// Records a CUDA event pair around the launches issued in its scope when the
// controls have profiling enabled (clb_profile_enable).
struct ProfScope {
    clb_controls *ctl;
    const char *name;
    cudaEvent_t start = nullptr;
    ProfScope(clb_controls *c, const char *n);
    ~ProfScope();
};

// Reads `count` 64-bit scalars from device memory (one sync).
int read_scalars(clb_controls *ctl, const uint64_t *d_src, uint64_t *h_dst, int count);
// Reads `bytes` (a multiple of 4, at most 512) of device memory into h_dst
// through the page-locked staging: a one-warp kernel stores the words there
// over PCIe, so the read does not queue behind large copies on the copy
// engine (clb_dcsr_spgemm_to_host copies row blocks while the next block's
// call reads its sizes back).  Synchronises the stream.
int read_small(clb_controls *ctl, const void *d_src, void *h_dst, size_t bytes);
// Several such reads (each a multiple of 4 bytes, at most 512 bytes in all)
// with one synchronisation.
struct SmallRead {
    const void *src;
    void *dst;
    size_t bytes;
};
int read_small_multi(clb_controls *ctl, const SmallRead *r, int n);
// Clears, then after the call checks, the device status word.
int clear_status(clb_controls *ctl);
int check_status(clb_controls *ctl, const char *op);

// Grid size for a persistent kernel: `per_sm` resident CTAs on every SM,
// capped by the number of work items.
inline unsigned persistent_grid(const clb_controls *ctl, int per_sm, uint64_t items) {
    uint64_t g = (uint64_t)ctl->sm_count * (uint64_t)(per_sm > 0 ? per_sm : 1);
    if (items < g) g = items;
    return (unsigned)(g ? g : 1);
}

inline unsigned ceil_div_u(uint64_t a, uint64_t b) { return (unsigned)((a + b - 1) / b); }

// Blocks of `kernel` (`threads` per block, `smem` dynamic bytes) that one SM
// holds at once, 1 if the query fails.  A kernel whose blocks loop over
// their work with a grid stride gets at most this many blocks per SM: a
// block past it would start only after an earlier block had finished all
// of its work, and would then run its whole share at lower occupancy.
template <class K>
inline int blocks_per_sm(K kernel, int threads, size_t smem = 0) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem) != cudaSuccess) {
        (void)cudaGetLastError();
        n = 1;
    }
    return n > 0 ? n : 1;
}

// ------------------------------------------------------ device primitives --
__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned warp_id() { return threadIdx.x >> 5; }

template <class T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        T o = __shfl_up_sync(0xFFFFFFFFu, v, d);
        if ((int)lane_id() >= d) v += o;
    }
    return v;
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, d);
    return v;
}

template <class T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        T o = __shfl_xor_sync(0xFFFFFFFFu, v, d);
        v = o > v ? o : v;
    }
    return v;
}

// Block-wide exclusive scan; `scratch` holds >= 33 T.  Returns the exclusive
// prefix of v; *total gets the block sum.  All threads must call.
template <class T, int NT>
__device__ __forceinline__ T block_exclusive_scan(T v, T *scratch, T *total) {
    constexpr int NW = NT / 32;
    T inc = warp_inclusive_scan(v);
    if (lane_id() == 31) scratch[warp_id()] = inc;
    __syncthreads();
    if (warp_id() == 0) {
        T w = lane_id() < (unsigned)NW ? scratch[lane_id()] : T(0);
        T wi = warp_inclusive_scan(w);
        if (lane_id() < (unsigned)NW) scratch[lane_id()] = wi - w;
        if (lane_id() == 31) scratch[32] = wi;
    }
    __syncthreads();
    T r = inc - v + scratch[warp_id()];
    *total = scratch[32];
    __syncthreads();
    return r;
}

template <class T, int NT>
__device__ __forceinline__ T block_sum(T v, T *scratch) {
    T total;
    block_exclusive_scan<T, NT>(v, scratch, &total);
    return total;
}

__device__ __forceinline__ void raise_status(uint32_t *status, uint32_t bit) {
    if (status) atomicOr(status, bit);
}

// Lower bound of `key` in sorted a[0, n).
template <class T, class I>
__device__ __forceinline__ I lower_bound_dev(const T *a, I n, T key) {
    I lo = 0, hi = n;
    while (lo < hi) {
        I m = lo + (hi - lo) / 2;
        if (a[m] < key) lo = m + 1; else hi = m;
    }
    return lo;
}

// Upper bound of `key` in sorted a[0, n).
template <class T, class I>
__device__ __forceinline__ I upper_bound_dev(const T *a, I n, T key) {
    I lo = 0, hi = n;
    while (lo < hi) {
        I m = lo + (hi - lo) / 2;
        if (a[m] <= key) lo = m + 1; else hi = m;
    }
    return lo;
}

// ------------------------------------------------------------- B-row view --
// Row lookup of a DCSR right operand.  With a dense row map (CSR-style rpt
// over all B.nrows, built once per call) the lookup is two loads; otherwise
// it binary-searches B.rows (hypersparse B with huge nrows).
struct BRows {
    const uint64_t *dense;  // nrows + 1, or nullptr
    const uint64_t *rpt;
    const uint32_t *rows;
    const uint32_t *cols;
    uint64_t nzr;
    uint64_t nrows;
    // B's rows as runs of one 32-bit bitmap word: (word, OR of the run's
    // bits) pairs; wdense maps a row to its pairs like `dense` (null = absent)
    const uint64_t *wdense = nullptr;
    const uint2 *wpairs = nullptr;
};

// Pairs [beg, beg + n) of B row k (wdense present).
__device__ __forceinline__ uint32_t b_words(const BRows &b, uint32_t k, uint64_t &beg) {
    if (k >= b.nrows) { beg = 0; return 0; }
    beg = __ldg(b.wdense + k);
    return (uint32_t)(__ldg(b.wdense + k + 1) - beg);
}

__device__ __forceinline__ uint32_t b_row(const BRows &b, uint32_t k, uint64_t &beg) {
    if (b.dense) {
        if (k >= b.nrows) { beg = 0; return 0; }
        beg = __ldg(b.dense + k);
        return (uint32_t)(__ldg(b.dense + k + 1) - beg);
    }
    uint64_t p = lower_bound_dev<uint32_t, uint64_t>(b.rows, b.nzr, k);
    if (p >= b.nzr || __ldg(b.rows + p) != k) { beg = 0; return 0; }
    beg = __ldg(b.rpt + p);
    return (uint32_t)(__ldg(b.rpt + p + 1) - beg);
}

// Exclusive scan primitives implemented in scan.cu (stream-ordered, no host
// sync).  `out` may alias `in` when the types match.  `d_total` (may be
// null) receives the sum.
int scan_u32_to_u64(clb_controls *ctl, const uint32_t *in, uint64_t *out, uint64_t n, uint64_t *d_total);
int scan_u32_inplace(clb_controls *ctl, uint32_t *data, uint64_t n, uint64_t *d_total);
int scan_u64_inplace(clb_controls *ctl, uint64_t *data, uint64_t n, uint64_t *d_total);

// Dense row map of a DCSR matrix: out[r] = offset of row r, out[nrows] = nnz
// (the CSR rpt).  Implemented in convert.cu.
int dcsr_dense_rpt(clb_controls *ctl, const clb_dcsr *m, uint64_t *out);

// Whether a dense map of `nrows` rows is worth building for a matrix with
// `nnz` entries.
inline bool use_dense_map(uint64_t nrows, uint64_t nnz) {
    return nrows <= (1ull << 26) || nrows <= 4 * nnz;
}

}  // namespace clb
