// scan.cu -- exclusive prefix sums (prefix_sum, src/common/cl_operations.cpp:4-88).
//
// The reference runs a recursive Blelloch scan with a host wait after every
// level and a blocking read of the total.  Here a scan is three
// stream-ordered kernels with no host synchronisation:
//   1. tile_reduce: every tile sums its inputs (64-bit);
//   2. tiles_scan : one CTA scans the tile sums and writes the grand total;
//   3. downsweep  : every tile rescans its inputs from its tile offset.
// A tile is 256 threads x 8 16-byte vectors (8192 u32 or 4096 u64 entries).
// Each warp owns a contiguous segment and walks it in 8 steps of 32 lanes x
// one vector: loads and stores are 16 bytes per lane, coalesced over the
// warp, and one shuffle scan covers 128 (u32) entries, so no shared-memory
// transpose is needed.  On B200 a 2^28-entry u32 scan takes 0.51 ms (the
// reduce pass reads at the copy peak); a single-pass form with decoupled
// look-back between tiles moves a third less data but measured 0.52-0.85 ms
// here, its tiles waiting on their predecessors' published sums.
#include <mutex>
#include <string>

#include "common.cuh"

namespace clb {

namespace {

constexpr int SCAN_NT = 256;
constexpr int SCAN_WARPS = SCAN_NT / 32;
constexpr int SCAN_VECS = 8;  // 16-byte vectors per thread

template <class TIn>
struct ScanShape {
    static constexpr int V = 16 / (int)sizeof(TIn);         // entries per vector
    static constexpr uint64_t SEG = 32ull * SCAN_VECS * V;  // entries per warp
    static constexpr uint64_t TILE = SEG * SCAN_WARPS;      // entries per CTA
};

// The warp's segment [seg, seg + SEG): step k, lane l holds entries
// seg + (32k + l)V .. + V - 1.  16-byte loads when `vec` (16-byte aligned
// arrays) and the segment is whole; guarded loads (zeros past n) otherwise.
template <class TIn>
__device__ __forceinline__ void load_segment(const TIn *in, uint64_t seg, uint64_t n, bool vec,
                                             TIn (&v)[SCAN_VECS][ScanShape<TIn>::V]) {
    constexpr int V = ScanShape<TIn>::V;
    const uint32_t lane = lane_id();
    if (vec && seg + ScanShape<TIn>::SEG <= n) {
#pragma unroll
        for (int k = 0; k < SCAN_VECS; ++k) {
            const uint4 x = *reinterpret_cast<const uint4 *>(in + seg + (uint64_t)(32 * k + lane) * V);
            if constexpr (V == 4) {
                v[k][0] = x.x; v[k][1] = x.y; v[k][2] = x.z; v[k][3] = x.w;
            } else {
                v[k][0] = ((uint64_t)x.y << 32) | x.x;
                v[k][1] = ((uint64_t)x.w << 32) | x.z;
            }
        }
    } else {
#pragma unroll
        for (int k = 0; k < SCAN_VECS; ++k)
#pragma unroll
            for (int j = 0; j < V; ++j) {
                const uint64_t e = seg + (uint64_t)(32 * k + lane) * V + j;
                v[k][j] = e < n ? in[e] : TIn(0);
            }
    }
}

template <class TIn>
__global__ void __launch_bounds__(SCAN_NT) tile_reduce_kernel(const TIn *__restrict__ in, uint64_t n, bool vec,
                                                              uint64_t *__restrict__ tile_sums) {
    using S = ScanShape<TIn>;
    __shared__ uint64_t wsum[SCAN_WARPS];
    TIn v[SCAN_VECS][S::V];
    load_segment<TIn>(in, (uint64_t)blockIdx.x * S::TILE + warp_id() * S::SEG, n, vec, v);
    uint64_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_VECS; ++k)
#pragma unroll
        for (int j = 0; j < S::V; ++j) s += (uint64_t)v[k][j];
    s = warp_sum(s);
    if (lane_id() == 0) wsum[warp_id()] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t t = 0;
#pragma unroll
        for (int w = 0; w < SCAN_WARPS; ++w) t += wsum[w];
        tile_sums[blockIdx.x] = t;
    }
}

constexpr int TS_NT = 1024;

__global__ void __launch_bounds__(TS_NT) tiles_scan_kernel(uint64_t *__restrict__ sums, uint64_t ntiles,
                                                           uint64_t *__restrict__ d_total) {
    __shared__ uint64_t scratch[33];
    uint64_t carry = 0;
    for (uint64_t base = 0; base < ntiles; base += TS_NT) {
        uint64_t i = base + threadIdx.x;
        uint64_t v = i < ntiles ? sums[i] : 0;
        uint64_t tot;
        uint64_t ex = block_exclusive_scan<uint64_t, TS_NT>(v, scratch, &tot);
        if (i < ntiles) sums[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0 && d_total) *d_total = carry;
}

// tile_offsets == nullptr: the whole input is one tile (n <= TILE); the scan
// then takes this one launch, which also writes the total.  `vec`: both
// arrays 16-byte aligned.
template <class TIn, class TOut>
__global__ void __launch_bounds__(SCAN_NT) downsweep_kernel(const TIn *in, TOut *out, uint64_t n, bool vec,
                                                            const uint64_t *__restrict__ tile_offsets,
                                                            uint64_t *__restrict__ d_total = nullptr) {
    using S = ScanShape<TIn>;
    constexpr int V = S::V;
    __shared__ uint64_t wsum[SCAN_WARPS];
    const uint32_t lane = lane_id();
    const uint64_t seg = (uint64_t)blockIdx.x * S::TILE + warp_id() * S::SEG;
    // The segment is loaded in full before any write below, and no other
    // warp touches it, so `out` may alias `in`.
    TIn v[SCAN_VECS][V];
    load_segment<TIn>(in, seg, n, vec, v);
    uint64_t ex[SCAN_VECS], s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_VECS; ++k) {
        uint64_t t = 0;
#pragma unroll
        for (int j = 0; j < V; ++j) t += (uint64_t)v[k][j];
        const uint64_t inc = warp_inclusive_scan(t);
        ex[k] = s + inc - t;
        s += __shfl_sync(0xFFFFFFFFu, inc, 31);
    }
    if (lane == 0) wsum[warp_id()] = s;
    __syncthreads();
    if (!tile_offsets && d_total && threadIdx.x == 0) {
        uint64_t t = 0;
#pragma unroll
        for (int w = 0; w < SCAN_WARPS; ++w) t += wsum[w];
        *d_total = t;
    }
    uint64_t carry = tile_offsets ? tile_offsets[blockIdx.x] : 0;
    for (unsigned w = 0; w < warp_id(); ++w) carry += wsum[w];
    const bool whole = vec && seg + S::SEG <= n;
#pragma unroll
    for (int k = 0; k < SCAN_VECS; ++k) {
        uint64_t run = carry + ex[k];
        TOut o[V];
#pragma unroll
        for (int j = 0; j < V; ++j) {
            o[j] = (TOut)run;
            run += (uint64_t)v[k][j];
        }
        const uint64_t e0 = seg + (uint64_t)(32 * k + lane) * V;
        if (whole) {
            if constexpr (sizeof(TOut) == 4) {
                *reinterpret_cast<uint4 *>(out + e0) =
                    make_uint4((uint32_t)o[0], (uint32_t)o[1], (uint32_t)o[2], (uint32_t)o[3]);
            } else {
                uint4 *p = reinterpret_cast<uint4 *>(out + e0);
#pragma unroll
                for (int h = 0; h < V / 2; ++h)
                    p[h] = make_uint4((uint32_t)o[2 * h], (uint32_t)((uint64_t)o[2 * h] >> 32), (uint32_t)o[2 * h + 1],
                                      (uint32_t)((uint64_t)o[2 * h + 1] >> 32));
            }
        } else {
#pragma unroll
            for (int j = 0; j < V; ++j)
                if (e0 + j < n) out[e0 + j] = o[j];
        }
    }
}

inline bool aligned16(const void *a, const void *b) {
    return ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 15u) == 0;
}

template <class TIn, class TOut>
int scan_impl(clb_controls *ctl, const TIn *in, TOut *out, uint64_t n, uint64_t *d_total) {
    if (n == 0) {
        if (d_total) CLB_TRY_CUDA(cudaMemsetAsync(d_total, 0, sizeof(uint64_t), ctl->stream), CLB_RUN_KERNEL_FAILURE);
        return CLB_SUCCESS;
    }
    constexpr uint64_t TILE = ScanShape<TIn>::TILE;
    const bool vec = aligned16(in, out);
    uint64_t ntiles = (n + TILE - 1) / TILE;
    if (ntiles > 0x7FFFFFFFull) return fail(CLB_NOT_SUPPORTED, "scan too long");
    if (ntiles == 1) {  // one tile: one launch
        ProfScope ps(ctl, "scan");
        downsweep_kernel<TIn, TOut><<<1, SCAN_NT, 0, ctl->stream>>>(in, out, n, vec, nullptr, d_total);
        ctl->launches += 1;
        CLB_CHECK_LAUNCH();
        return CLB_SUCCESS;
    }
    Temp<uint64_t> sums;
    CLB_RETURN_IF(sums.alloc(ctl, ntiles));
    ProfScope ps(ctl, "scan");
    tile_reduce_kernel<TIn><<<(unsigned)ntiles, SCAN_NT, 0, ctl->stream>>>(in, n, vec, sums.ptr);
    tiles_scan_kernel<<<1, TS_NT, 0, ctl->stream>>>(sums.ptr, ntiles, d_total);
    downsweep_kernel<TIn, TOut><<<(unsigned)ntiles, SCAN_NT, 0, ctl->stream>>>(in, out, n, vec, sums.ptr);
    ctl->launches += 3;
    CLB_CHECK_LAUNCH();
    return CLB_SUCCESS;
}

}  // namespace

int scan_u32_to_u64(clb_controls *ctl, const uint32_t *in, uint64_t *out, uint64_t n, uint64_t *d_total) {
    return scan_impl<uint32_t, uint64_t>(ctl, in, out, n, d_total);
}

int scan_u32_inplace(clb_controls *ctl, uint32_t *data, uint64_t n, uint64_t *d_total) {
    return scan_impl<uint32_t, uint32_t>(ctl, data, data, n, d_total);
}

int scan_u64_inplace(clb_controls *ctl, uint64_t *data, uint64_t n, uint64_t *d_total) {
    return scan_impl<uint64_t, uint64_t>(ctl, data, data, n, d_total);
}

// ------------------------------------------------ allocation-free variant --
// Some callers cannot allocate device memory at the point where they need a
// scan: a runtime that has reserved all of the GPU's memory for its own pool,
// or a latency-critical loop that must not pay for cudaMalloc's implicit
// synchronisation.  For them, the scan's only scratch (one 64-bit partial
// sum per 8192-entry tile) lives in this fixed array that the library image
// brings with it.  Every GPU that loads the library holds the array
// (256 KiB) until the process exits.
constexpr uint64_t NOALLOC_MAX_ENTRIES = 1ull << 28;
constexpr uint64_t NOALLOC_MAX_TILES = 32768;  // 2^28 / ScanShape<uint32_t>::TILE
static __device__ __align__(256) uint64_t g_scan_scratch[NOALLOC_MAX_TILES];

namespace {

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_scratch_mutex;
uint64_t *g_scratch_addr[NOALLOC_MAX_DEVICES] = {};

// Device address of g_scan_scratch on `device`, which must be current.  In
// host code the array's name is only a host stand-in, never a device
// address, so kernels must get this pointer.  The first call on a device
// looks it up (and loads the library's device code there if nothing has
// yet); later calls look it up again whenever `s` is not being captured, so
// a primary context that was torn down and re-created (cudaDeviceReset)
// never leaves a stale address behind.  A call on a capturing stream takes
// the address of the device's previous call.
int scratch_address(int device, cudaStream_t s, uint64_t **out) {
    if (device < 0 || device >= NOALLOC_MAX_DEVICES)
        return fail(CLB_NOT_SUPPORTED, "device ordinal beyond the static scratch table");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
        (void)cudaGetLastError();
        cap = cudaStreamCaptureStatusActive;  // treat as captured: keep the known address
    }
    if (!g_scratch_addr[device] || cap == cudaStreamCaptureStatusNone) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scan_scratch);
        if (e != cudaSuccess || !p)
            return fail(CLB_INITIALIZATION_ERROR,
                        std::string("cudaGetSymbolAddress of the scan scratch: ") + cudaGetErrorString(e));
        g_scratch_addr[device] = static_cast<uint64_t *>(p);
    }
    *out = g_scratch_addr[device];
    return CLB_SUCCESS;
}

// Makes the device that owns stream `s` current for the scope (the current
// device for the legacy and per-thread default streams).
struct StreamDevice {
    int prev = -1, device = -1;
    int enter(cudaStream_t s) {
        CLB_TRY_CUDA(cudaGetDevice(&prev), CLB_RUN_KERNEL_FAILURE);
        device = prev;
        if (s != nullptr && s != cudaStreamLegacy && s != cudaStreamPerThread)
            CLB_TRY_CUDA(cudaStreamGetDevice(s, &device), CLB_INVALID_ARGUMENT);
        if (device != prev) CLB_TRY_CUDA(cudaSetDevice(device), CLB_RUN_KERNEL_FAILURE);
        return CLB_SUCCESS;
    }
    ~StreamDevice() {
        if (prev >= 0 && device != prev) cudaSetDevice(prev);
    }
};

}  // namespace

}  // namespace clb

using namespace clb;

extern "C" {

int clb_prefix_sum_u32_noalloc(uint32_t *array, uint64_t n, uint64_t *d_total, void *stream) {
    if (n && !array) return fail(CLB_INVALID_ARGUMENT, "array is NULL");
    static_assert(NOALLOC_MAX_ENTRIES / ScanShape<uint32_t>::TILE <= NOALLOC_MAX_TILES, "scratch too small");
    if (n > NOALLOC_MAX_ENTRIES)
        return fail(CLB_INVALID_ARGUMENT, "prefix sum of " + std::to_string(n) +
                                              " entries exceeds the static scratch limit of 2^28 entries");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // The scratch array is per device: take the one of the device that owns
    // the stream, with that device current.
    StreamDevice sd;
    CLB_RETURN_IF(sd.enter(s));
    if (n == 0) {
        if (d_total) CLB_TRY_CUDA(cudaMemsetAsync(d_total, 0, sizeof(uint64_t), s), CLB_RUN_KERNEL_FAILURE);
        return CLB_SUCCESS;
    }
    uint64_t *sums = nullptr;
    CLB_RETURN_IF(scratch_address(sd.device, s, &sums));
    // The tile sums are written in full by the first kernel before anything
    // reads them, so the array's leftovers from an earlier call need no
    // clearing.
    const uint64_t ntiles = (n + ScanShape<uint32_t>::TILE - 1) / ScanShape<uint32_t>::TILE;
    const bool vec = aligned16(array, array);
    tile_reduce_kernel<uint32_t><<<(unsigned)ntiles, SCAN_NT, 0, s>>>(array, n, vec, sums);
    tiles_scan_kernel<<<1, TS_NT, 0, s>>>(sums, ntiles, d_total);
    downsweep_kernel<uint32_t, uint32_t><<<(unsigned)ntiles, SCAN_NT, 0, s>>>(array, array, n, vec, sums);
    CLB_CHECK_LAUNCH();
    return CLB_SUCCESS;
}

int clb_prefix_sum_u32(clb_controls *ctl, uint32_t *array, uint64_t n, uint64_t *total) {
    if (!ctl || (n && !array)) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    DeviceGuard g(ctl);
    Temp<uint64_t> t;
    CLB_RETURN_IF(t.alloc(ctl, 1));
    CLB_RETURN_IF(scan_u32_inplace(ctl, array, n, t.ptr));
    uint64_t h = 0;
    CLB_RETURN_IF(read_scalars(ctl, t.ptr, &h, 1));
    if (total) *total = h;
    return CLB_SUCCESS;
}

int clb_prefix_sum_u64(clb_controls *ctl, uint64_t *array, uint64_t n, uint64_t *total) {
    if (!ctl || (n && !array)) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    DeviceGuard g(ctl);
    Temp<uint64_t> t;
    CLB_RETURN_IF(t.alloc(ctl, 1));
    CLB_RETURN_IF(scan_u64_inplace(ctl, array, n, t.ptr));
    uint64_t h = 0;
    CLB_RETURN_IF(read_scalars(ctl, t.ptr, &h, 1));
    if (total) *total = h;
    return CLB_SUCCESS;
}

}  // extern "C"
